"""Batched form: many networks of uneven size in one context.  Each network
must evolve exactly as it does in a context of its own (bit for bit in both
precision forms: every per-neuron computation and every per-lane search sum is
the same, only the grouping of the work differs)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def ensemble_spec(seed, k, lo, hi):
    rng = np.random.default_rng(seed)
    sizes = np.exp(rng.uniform(np.log(lo), np.log(hi), k)).astype(int)
    nets = []
    for i, n in enumerate(sizes):
        side = (1000.0 * n) ** (1 / 3)
        nets.append(dict(num_neurons=int(n), seed=10_000 + 17 * i, side=side, theta=float(rng.choice([0.2, 0.3, 0.5])),
                         sigma=float(rng.choice([500.0, 750.0, 1000.0])), growth_rate=float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-3))))))
    return nets


def net_inputs(d, k):
    from relearn_b200 import workloads

    n = d["num_neurons"]
    pos = workloads.uniform_cube(n, d["side"], 500 + k)
    sig = workloads.signal_types(n, 500 + k)
    grown = workloads.initial_elements(n, 600 + k, 0.0, 3.0)
    return pos, sig, grown


def single_params(base, d):
    p = dict(base)
    p.update(num_neurons=d["num_neurons"], seed=d["seed"], box_min=(0.0, 0.0, 0.0), box_max=(d["side"],) * 3, theta=d["theta"], sigma=d["sigma"],
             growth_rate=(d["growth_rate"],) * 3)
    return p


@pytest.mark.parametrize("precision", [0, 1])
def test_ensemble_equals_standalone(precision):
    from relearn_b200 import Network, default_params

    nets = ensemble_spec(precision, 5, 300, 3000)
    base = default_params(1, 1.0)
    base["precision"] = precision
    ens = Network(base, networks=nets)
    inputs = [net_inputs(d, k) for k, d in enumerate(nets)]
    ens.set_positions(np.concatenate([p for p, _, _ in inputs]), np.concatenate([s for _, s, _ in inputs]))
    for t in range(3):
        g = np.concatenate([gr[t][0] for _, _, gr in inputs])
        v = np.concatenate([gr[t][1] for _, _, gr in inputs])
        ens.set_elements(t, g, np.zeros(len(g)), np.zeros(len(g), np.uint32), v)
    ens.simulate(1, 601)
    ea = ens.neurons()
    eel = [ens.get_elements(t) for t in range(3)]
    et, es, ew = ens.edges()
    off = 0
    for k, d in enumerate(nets):
        n = d["num_neurons"]
        pos, sig, gr = inputs[k]
        one = Network(single_params(base, d))
        one.set_positions(pos, sig)
        for t in range(3):
            one.set_elements(t, gr[t][0], np.zeros(n), np.zeros(n, np.uint32), gr[t][1])
        one.simulate(1, 601)
        a = one.neurons()
        for key in ("x", "u", "calcium"):
            assert np.array_equal(a[key].view(np.uint64), ea[key][off:off + n].view(np.uint64)), (k, key)
        assert np.array_equal(a["fired"], ea["fired"][off:off + n])
        for t in range(3):
            el = one.get_elements(t)
            for key in ("connected", "vacant"):
                assert np.array_equal(el[key], eel[t][key][off:off + n]), (k, t, key)
            assert np.array_equal(el["grown"].view(np.uint64), eel[t]["grown"][off:off + n].view(np.uint64)), (k, t)
        t1, s1, w1 = one.edges()
        sel = (et >= off) & (et < off + n)
        assert np.array_equal(t1 + off, et[sel]) and np.array_equal(s1 + off, es[sel]) and np.array_equal(w1, ew[sel]), k
        assert np.all((es[sel] >= off) & (es[sel] < off + n))
        off += n
    assert ens.stats()["synapses_created"] > 0


def test_ensemble_tree_roots():
    from relearn_b200 import Network, default_params

    nets = ensemble_spec(7, 4, 1, 50)
    nets[0]["num_neurons"] = 1  # a network of one neuron: its root is a leaf
    ens = Network(default_params(1, 1.0), networks=nets)
    inputs = [net_inputs(d, k) for k, d in enumerate(nets)]
    ens.set_positions(np.concatenate([p for p, _, _ in inputs]), np.concatenate([s for _, s, _ in inputs]))
    t = ens.tree()
    assert np.all(t["level"][:4] == 0)
    assert t["neuron"][0] == 0  # the single neuron's root is its leaf
    one = np.ones(ens.n, np.uint32)
    ens.prepare_update_connectivity(one, one, one)
    req = ens.find_targets(100)
    # the single neuron finds nobody; every other request stays inside its network
    offs = np.cumsum([0] + [d["num_neurons"] for d in nets])
    net_of = np.searchsorted(offs, np.arange(ens.n), side="right") - 1
    assert not np.any(req["source"] == 0)
    assert np.array_equal(net_of[req["source"]], net_of[req["target"]])
