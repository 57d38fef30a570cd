"""Blocks of activity steps in one launch: while a network has no synapses, each
neuron's steps depend on nothing but its own state and draws, so a block of
steps runs as one launch with the state in registers.  It must give the same
bits as one launch per step, in both precision forms and for every neuron
model, with disabled neurons and per-neuron targets, and hand over to the
per-step kernels once synapses exist."""
import numpy as np
import pytest

from conftest import seed_elements, small_network

pytestmark = pytest.mark.gpu


def make(n, seed, precision, model=0):
    from relearn_b200 import Network

    params, pos, sig = small_network(n, 2500.0, seed)
    params["precision"] = precision
    params["neuron_model"] = model
    if model == 3:
        params["noise_mean"] = 600.0  # pA: enough drive for the AEIF neuron to spike
        params["noise_stddev"] = 200.0
    net = Network(params)
    net.set_positions(pos, sig)
    return net


def state(net):
    a = net.neurons()
    out = {k: a[k].view(np.uint64) if a[k].dtype == np.float64 else a[k] for k in ("x", "u", "calcium", "fired", "input")}
    for t in range(3):
        e = net.get_elements(t)
        out[f"delta{t}"] = e["delta"].view(np.uint64)
        out[f"grown{t}"] = e["grown"].view(np.uint64)
        out[f"connected{t}"] = e["connected"]
    return out


def assert_same(a, b, what):
    for k in a:
        assert np.array_equal(a[k], b[k]), (what, k)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("model", [0, 1, 2, 3])
@pytest.mark.parametrize("mode", ["all", "disabled", "targets"])
def test_fused_block_equals_steps(precision, model, mode):
    n = 20011  # odd: the last block of threads is partial
    runs = []
    for fused in (True, False):
        net = make(n, 31 + model, precision, model)
        net.set_step_fusion(fused)
        if mode == "disabled":
            net.set_enabled((np.random.default_rng(3).random(n) > 0.25).astype(np.uint8))
        elif mode == "targets":
            net.set_target_calcium(np.random.default_rng(4).uniform(0.3, 0.9, n))
        l0 = net.stats()["gpu_launches"]
        got = []
        for first, count in ((1, 37), (38, 64), (102, 1), (103, 2)):  # odd, even, one and two steps
            net.activity_block(first, count)
            got.append(state(net))
        runs.append((got, net.stats()["gpu_launches"] - l0))
        net.close()
    (fused_states, fused_launches), (step_states, step_launches) = runs
    for i, (a, b) in enumerate(zip(fused_states, step_states)):
        assert_same(a, b, (precision, model, mode, i))
    assert fused_launches < step_launches  # the fused blocks really ran as single launches
    if model in (0, 3):  # Izhikevich and AEIF neurons spike within these blocks at the default drive
        assert sum(int(st["fired"].sum()) for st in fused_states) > 0


@pytest.mark.parametrize("precision", [0, 1])
def test_simulation_hands_over_to_per_step_kernels(precision):
    """Through plasticity updates: the first intervals run fused, the ones after
    the first synapses per step; the whole run equals the unfused one."""
    n = 6000
    runs = []
    for fused in (True, False):
        net = make(n, 77, precision)
        net.set_step_fusion(fused)
        seed_elements(net, n, 5, 0.0, 3.0)
        net.simulate(1, 601)
        runs.append((state(net), net.edges()))
        net.close()
    (s1, e1), (s2, e2) = runs
    assert_same(s1, s2, precision)
    assert len(e1[0]) > 0
    for a, b in zip(e1, e2):
        assert np.array_equal(a, b)


def test_ensemble_fused_equals_steps():
    """Batched contexts (many networks per launch) too."""
    from relearn_b200 import Network, default_params

    nets = [dict(num_neurons=int(k), seed=500 + i, side=(1000.0 * k) ** (1 / 3), theta=0.3, sigma=750.0, growth_rate=1e-4)
            for i, k in enumerate((1201, 3000, 777, 4096))]
    total = sum(d["num_neurons"] for d in nets)
    from relearn_b200 import workloads

    pos = np.concatenate([workloads.uniform_cube(d["num_neurons"], d["side"], 900 + i) for i, d in enumerate(nets)])
    sig = np.concatenate([workloads.signal_types(d["num_neurons"], 900 + i) for i, d in enumerate(nets)])
    runs = []
    for precision in (0, 1):
        for fused in (True, False):
            base = default_params(1, 1.0)
            base["precision"] = precision
            ens = Network(base, networks=nets)
            ens.set_positions(pos, sig)
            ens.set_step_fusion(fused)
            ens.activity_block(1, 53)
            runs.append(state(ens))
            ens.close()
    assert_same(runs[0], runs[1], "fp64")
    assert_same(runs[2], runs[3], "fp32")
    assert len(runs[0]["x"]) == total
