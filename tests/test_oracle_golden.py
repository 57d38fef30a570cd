"""The oracle reproduces the committed golden fixtures (regression pin) and
its results do not depend on the thread count."""
import os

import numpy as np
import pytest

from conftest import oracle_params, seed_elements, small_network

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("name", ["golden_uniform_300.npz", "golden_mixture_400.npz"])
def test_oracle_reproduces_golden(oracle_mod, name):
    from relearn_b200 import default_params

    z = np.load(os.path.join(GOLDEN, name))
    n = len(z["signal"])
    params = default_params(n, float(z["side"]))
    params["seed"] = int(z["seed"])
    sim = oracle_mod.OracleSim(oracle_params(params), z["positions"], z["signal"])
    seed_elements(sim, n, int(z["seed"]) - 1000, float(z["lower"]), float(z["upper"]))
    sim.update_tree(sim.get_elements(1)["vacant"], sim.get_elements(2)["vacant"])
    t = sim.tree()
    for k in ("level", "neuron", "child_mask", "first_child", "cnt_exc", "cnt_inh"):
        assert np.array_equal(t[k], z["tree_" + k])
    req = sim.find_targets(100)
    assert np.array_equal(req, z["requests"])
    sim2 = oracle_mod.OracleSim(oracle_params(params), z["positions"], z["signal"])
    seed_elements(sim2, n, int(z["seed"]) - 1000, float(z["lower"]), float(z["upper"]))
    sim2.simulate(1, int(z["steps"]))
    nr = sim2.neurons()
    assert np.array_equal(nr["x"].view(np.uint64), z["final_x"].view(np.uint64))
    assert np.array_equal(nr["calcium"].view(np.uint64), z["final_calcium"].view(np.uint64))


def test_tree_invariants(oracle_mod):
    params, pos, sig = small_network(3000, 1200.0, 9, mixture=True)
    sim = oracle_mod.OracleSim(oracle_params(params), pos, sig)
    t = sim.tree()
    leaves = t["neuron"] >= 0
    assert np.array_equal(np.sort(t["neuron"][leaves]), np.arange(3000))
    # every leaf's neuron lies in its cell; children lie in their parent's cell
    p = pos[t["neuron"][leaves]]
    assert np.all(t["bmin"][leaves] <= p) and np.all(p <= t["bmax"][leaves])
    inner = np.nonzero(~leaves)[0]
    for i in inner[:500]:
        k = bin(int(t["child_mask"][i])).count("1")
        ch = np.arange(t["first_child"][i], t["first_child"][i] + k)
        assert np.all(t["level"][ch] == t["level"][i] + 1)
        assert np.all(t["bmin"][ch] >= t["bmin"][i]) and np.all(t["bmax"][ch] <= t["bmax"][i])


def test_thread_count_invariance(oracle_mod):
    params, pos, sig = small_network(4000, 1300.0, 12)
    out = []
    for threads in (1, 4):
        sim = oracle_mod.OracleSim(oracle_params(params), pos, sig, threads=threads)
        seed_elements(sim, 4000, 3, 0.0, 3.0)
        sim.simulate(1, 301)
        out.append((sim.neurons()["x"], sim.edges()))
    assert np.array_equal(out[0][0], out[1][0])
    for a, b in zip(out[0][1], out[1][1]):
        assert np.array_equal(a, b)
