"""Autotuned launch shapes: every candidate shape of the search and activity
kernels computes the same results (bit for bit), so tuning never changes what
a run produces."""
import numpy as np
import pytest

from conftest import seed_elements, small_network

pytestmark = pytest.mark.gpu


def make(n, side, seed, precision):
    from relearn_b200 import Network

    params, pos, sig = small_network(n, side, seed)
    params["precision"] = precision
    net = Network(params)
    net.set_positions(pos, sig)
    return net


@pytest.mark.parametrize("precision", [0, 1])
def test_every_search_shape_finds_the_same_targets(precision):
    from relearn_b200 import SEARCH_SHAPES

    n = 30000
    net = make(n, 3100.0, 21, precision)
    one = np.full(n, 2, np.uint32)
    net.prepare_update_connectivity(one, one, one)
    ref = None
    for w, p, cp, hot in SEARCH_SHAPES:
        net.set_tuning(search_warps=w, search_packet=p, search_cap=cp, search_hot=hot)
        req = net.find_targets(100)
        if ref is None:
            ref = req
        else:
            assert np.array_equal(req, ref), (w, p, cp, hot)
    assert len(ref) > 0


def _activity_state(net):
    a = net.neurons()
    got = [a["x"].view(np.uint64), a["u"].view(np.uint64), a["calcium"].view(np.uint64), a["fired"], a["input"].view(np.uint64)]
    for t in range(3):
        got.append(net.get_elements(t)["delta"].view(np.uint64))
    return got


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("mode", ["all", "disabled", "targets"])
def test_every_activity_shape_gives_the_same_state(precision, mode):
    """Every block size, grid form and neurons-per-thread count gives the same
    bits (state, input and deltas): with all neurons enabled, with neurons
    disabled and with per-neuron target calcium."""
    from relearn_b200 import ACT_SHAPES

    n = 50000
    ref = None
    for b, p, v in ACT_SHAPES:
        if precision == 0 and v != 1:
            continue
        net = make(n + 3, 3700.0, 8, precision)  # n % 4 == 3: the vector shapes have a tail
        if mode == "disabled":
            net.set_enabled((np.random.default_rng(5).random(n + 3) > 0.3).astype(np.uint8))
        elif mode == "targets":
            net.set_target_calcium(np.random.default_rng(6).uniform(0.3, 0.9, n + 3))
        net.set_tuning(act_block=b, act_persistent=p, act_vec=v)
        net.activity_block(1, 37)
        got = _activity_state(net)
        if ref is None:
            ref = got
        else:
            for j, (g, r) in enumerate(zip(got, ref)):
                assert np.array_equal(g, r), (b, p, v, j)
        net.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_tuned_run_equals_untuned(precision):
    n = 6000
    runs = []
    for tune in (False, True):
        net = make(n, 1820.0, 13, precision)
        seed_elements(net, n, 5, 0.0, 3.0)
        if tune:
            net.autotune(2)
        net.simulate(1, 401)
        a = net.neurons()
        runs.append((a["x"].view(np.uint64), a["calcium"].view(np.uint64), net.edges()))
        if tune:
            t = net.tuning()
            assert t["tuned"] == 3
            assert len(t["act_ms"]) == (18 if precision else 12) and len(t["search_ms"]) >= 6
        net.close()
    (x0, c0, e0), (x1, c1, e1) = runs
    assert np.array_equal(x0, x1) and np.array_equal(c0, c1)
    for a, b in zip(e0, e1):
        assert np.array_equal(a, b)
    assert len(e0[0]) > 0


@pytest.mark.parametrize("precision", [0, 1])
def test_every_search_shape_on_a_forest(precision):
    """Many networks in one context: the persistent form's shared-memory copy
    then holds the top levels of every network's octree."""
    from relearn_b200 import SEARCH_SHAPES, Network, default_params
    from test_gpu_ensemble import ensemble_spec, net_inputs

    nets = ensemble_spec(11 + precision, 9, 200, 6000)
    base = default_params(1, 1.0)
    base["precision"] = precision
    ens = Network(base, networks=nets)
    inputs = [net_inputs(d, k) for k, d in enumerate(nets)]
    ens.set_positions(np.concatenate([p for p, _, _ in inputs]), np.concatenate([s for _, s, _ in inputs]))
    n = sum(d["num_neurons"] for d in nets)
    one = np.full(n, 2, np.uint32)
    ens.prepare_update_connectivity(one, one, one)
    ref = None
    for w, p, cp, hot in SEARCH_SHAPES:
        ens.set_tuning(search_warps=w, search_packet=p, search_cap=cp, search_hot=hot)
        req = ens.find_targets(100)
        if ref is None:
            ref = req
        else:
            assert np.array_equal(req, ref), (w, p, cp, hot)
    assert len(ref) > 0


@pytest.mark.parametrize("precision", [0, 1])
def test_one_search_per_warp_on_a_sparse_list(precision):
    """The one-search-per-warp kernel gives the packet kernel's targets on the
    lists it is for: a few hundred sources spread over a large network, with
    1-3 vacant axons each."""
    n = 100000
    net = make(n, 4600.0, 33, precision)
    rng = np.random.default_rng(5)
    va = np.zeros(n, np.uint32)
    va[rng.choice(n, 900, replace=False)] = rng.integers(1, 4, 900).astype(np.uint32)
    ve = rng.integers(0, 3, n).astype(np.uint32)
    vi = rng.integers(0, 3, n).astype(np.uint32)
    net.prepare_update_connectivity(va, ve, vi)
    got = []
    for shape in ((2, 32, 1, 0), (4, 0, 0, 0)):
        net.set_tuning(search_warps=shape[0], search_packet=shape[1], search_cap=shape[2], search_hot=shape[3])
        got.append(net.find_targets(300))
    assert len(got[0]) > 1000
    assert np.array_equal(got[0], got[1])
