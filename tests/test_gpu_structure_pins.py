"""The product's octree, acceptance walk, target search and connector against
the reference's own tests of them, re-expressed, through the C ABI:

* cell octants and octant boxes (test/cell/test_cell.cpp:1314-1400) on every
  node of the device octree, in random boxes that reach negative coordinates;
* theta outside (0, 0.5] is refused (test_barnes_hut_base.cpp:57-92, 793-828);
* the candidates of the production FP64 evaluation (rl_candidate_weights)
  equal the golden stack walk of test_barnes_hut_base.cpp:457-517 applied to
  the device's own octree; no elements give no candidates (:420-455); the
  FP32 form's candidates are accepted cells that partition the vacant
  dendrites;
* searches through rl_find_targets: no dendrites, no / one / full choice
  (test_barnes_hut_base.cpp:830-1000), no autapse
  (test_barnes_hut_cuda.cpp:485-563);
* bottom-up sums (test_barnes_hut_cuda.cpp:250-357);
* the connector through rl_connect: matching and self requests
  (test_connector.cpp:140-330), more requests than vacancies, and the same
  accepted requests as the oracle;
* the reference's positions fixture (relearn/input/positions.txt, 51,842
  neurons): the octree, the requests of a seeded-vacancy snapshot and, through
  the C++ driver and its positions reader, 1,001 seeded steps, all bit for bit
  against the oracle."""
import lzma
import os
import subprocess

import numpy as np
import pytest

from conftest import oracle_params, splitmix64_uniform
from structure_pins import (check_bottom_up_sums, check_cell_structure, children, golden_walk, matching_requests, positions_in_box, random_box,
                            random_theta, self_requests)

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def O(oracle_mod):
    return oracle_mod


def params_for(n, lo, hi, theta=0.3, precision=0, seed=1):
    from relearn_b200 import default_params

    p = default_params(n, 1.0)
    p["box_min"], p["box_max"], p["theta"], p["precision"], p["seed"] = tuple(lo), tuple(hi), theta, precision, seed
    return p


def network(n, lo, hi, pos, sig=None, **kw):
    from relearn_b200 import Network

    net = Network(params_for(n, lo, hi, **kw))
    net.set_positions(pos, np.zeros(n, np.uint8) if sig is None else sig)
    return net


def same_f64(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


def assert_same_tree(got, expect):
    for k in ("level", "neuron", "child_mask", "first_child", "cnt_exc", "cnt_inh"):
        assert np.array_equal(got[k], expect[k]), k
    for k in ("bmin", "bmax", "pos_exc", "pos_inh"):
        assert same_f64(got[k], expect[k]), k


def test_octree_cells_in_random_boxes(O):
    rng = np.random.default_rng(230)
    for n in (1, 2, 3, 57, 1000, 5000):
        lo, hi = random_box(rng)
        pos = positions_in_box(rng, lo, hi, n)
        net = network(n, lo, hi, pos)
        tree = net.tree()
        check_cell_structure(O, tree, pos)
        sim = O.OracleSim(oracle_params(params_for(n, lo, hi)), pos, np.zeros(n, np.uint8))
        ref = sim.tree()
        for k in ("level", "neuron", "child_mask", "first_child"):
            assert np.array_equal(tree[k], ref[k]), (n, k)
        assert same_f64(tree["bmin"], ref["bmin"]) and same_f64(tree["bmax"], ref["bmax"])
        net.close()


def test_theta_outside_bounds_is_refused():
    from relearn_b200 import STATUS_NAMES, Network, RelearnError

    lo, hi = np.zeros(3), np.full(3, 100.0)
    for theta in (0.0, -0.1, -1000.0, 0.5 + 1e-9, 1000.0):
        with pytest.raises(RelearnError) as e:
            Network(params_for(10, lo, hi, theta=theta))
        assert STATUS_NAMES[e.value.status] == "RL_ERR_INVALID"
    Network(params_for(10, lo, hi, theta=0.5)).close()


def standard_network(rng, n=None, counts=(1, 2), precision=0):
    """OctreeFactory::get_standard_tree on the device: n neurons uniform in a
    random box, vacant dendrites of each type uniform in `counts`, random
    theta, random signal types."""
    n = int(rng.integers(1, 1001)) + 1 if n is None else n
    lo, hi = random_box(rng)
    pos = positions_in_box(rng, lo, hi, n)
    sig = (rng.random(n) < 0.2).astype(np.uint8)
    theta = random_theta(rng)
    net = network(n, lo, hi, pos, sig, theta=theta, precision=precision)
    ve = rng.integers(counts[0], counts[1] + 1, n).astype(np.uint32)
    vi = rng.integers(counts[0], counts[1] + 1, n).astype(np.uint32)
    net.prepare_update_connectivity(np.zeros(n, np.uint32), ve, vi)
    return net, pos, sig, theta, ve, vi


@pytest.mark.parametrize("seed", [457, 458, 459, 460])
def test_candidates_equal_golden_walk(O, seed):
    rng = np.random.default_rng(seed)
    net, pos, sig, theta, ve, vi = standard_network(rng)
    tree = net.tree()
    for src in rng.choice(len(pos), min(len(pos), 40), replace=False):
        nodes, w = net.candidate_weights(int(src), 0)
        assert nodes.tolist() == golden_walk(O, tree, pos[src], int(sig[src]), theta)
        # the searching neuron's own leaf is never a candidate (distance 0)
        own = np.flatnonzero(tree["neuron"] == src)
        assert own[0] not in set(nodes.tolist())
    net.close()


def test_no_elements_no_candidates():
    rng = np.random.default_rng(420)
    net, pos, *_ = standard_network(rng, counts=(0, 0))
    for src in range(min(len(pos), 50)):
        nodes, _ = net.candidate_weights(src, 0)
        assert len(nodes) == 0
    net.close()


def test_fp32_candidates_partition_vacant_dendrites(O):
    """FP32 form: every candidate is a leaf with vacant dendrites or a cell
    that passes the acceptance test in FP32 arithmetic, and the candidates'
    subtrees cover every vacant dendrite of the type except the source's own."""
    rng = np.random.default_rng(990)
    net, pos, sig, theta, ve, vi = standard_network(rng, n=3000, precision=1)
    tree = net.tree()
    m = len(tree["level"])
    for src in rng.choice(len(pos), 30, replace=False):
        t = int(sig[src])
        cnt = tree["cnt_exc" if t == 0 else "cnt_inh"]
        cpos = tree["pos_exc" if t == 0 else "pos_inh"]
        nodes, _ = net.candidate_weights(int(src), 1)
        covered = 0
        for i in nodes:
            assert cnt[i] > 0
            if tree["first_child"][i] >= 0:
                d = float(np.linalg.norm(cpos[i] - pos[src]))
                longest = float(np.max(tree["bmax"][i] - tree["bmin"][i]))
                assert longest < theta * d * (1 + 1e-5)
            covered += int(cnt[i])
        own = (ve if t == 0 else vi)[src]
        assert covered + int(own) == int(cnt[0])
        assert len(set(nodes.tolist())) == len(nodes) and max(nodes, default=0) < m
    net.close()


def find(net, n, axons, step):
    for k in range(3):
        net.set_elements(k, np.full(n, 1.5), np.zeros(n), np.zeros(n, np.uint32), axons if k == 0 else np.zeros(n, np.uint32))
    return net.find_targets(step)


def test_search_no_dendrites():
    rng = np.random.default_rng(830)
    net, pos, *_ = standard_network(rng, counts=(0, 0))
    n = len(pos)
    net.prepare_update_connectivity(np.ones(n, np.uint32), np.zeros(n, np.uint32), np.zeros(n, np.uint32))
    assert len(net.find_targets(100)) == 0
    net.close()


def test_search_no_choice():
    """A single neuron finds no target: the only candidate is itself."""
    rng = np.random.default_rng(866)
    lo, hi = random_box(rng)
    pos = positions_in_box(rng, lo, hi, 1)
    net = network(1, lo, hi, pos, theta=random_theta(rng))
    net.prepare_update_connectivity(np.array([3], np.uint32), np.array([2], np.uint32), np.array([2], np.uint32))
    for step in (100, 200, 300):
        assert len(net.find_targets(step)) == 0
    net.close()


def test_search_one_choice():
    rng = np.random.default_rng(905)
    for _ in range(10):
        lo, hi = random_box(rng)
        pos = positions_in_box(rng, lo, hi, 2)
        sig = np.full(2, int(rng.integers(0, 2)), np.uint8)
        net = network(2, lo, hi, pos, sig, theta=random_theta(rng))
        net.prepare_update_connectivity(np.array([2, 2], np.uint32), np.array([1, 2], np.uint32), np.array([1, 2], np.uint32))
        req = net.find_targets(100)
        assert len(req) == 4
        assert np.array_equal(req["target"], 1 - req["source"])
        net.close()


def test_search_full_choice():
    rng = np.random.default_rng(959)
    for _ in range(3):
        net, pos, sig, theta, ve, vi = standard_network(rng)
        n = len(pos)
        net.prepare_update_connectivity(np.ones(n, np.uint32), ve, vi)
        req = net.find_targets(100)
        assert len(req) == n
        assert np.array_equal(np.sort(req["source"]), np.arange(n))
        assert np.all(req["target"] != req["source"])
        need = np.where(sig[req["source"]] == 0, ve[req["target"]], vi[req["target"]])
        assert np.all(need > 0)
        net.close()


def test_bottom_up_sums():
    rng = np.random.default_rng(283)
    n = 100
    lo, hi = np.zeros(3), np.ones(3)
    net = network(n, lo, hi, positions_in_box(rng, lo, hi, n))
    net.prepare_update_connectivity(np.zeros(n, np.uint32), np.ones(n, np.uint32), np.zeros(n, np.uint32))
    tree = net.tree()
    check_bottom_up_sums(tree)
    assert tree["cnt_exc"][0] == n and not tree["cnt_inh"].any()
    assert np.all(tree["cnt_exc"][tree["neuron"] >= 0] == 1)
    zeros = np.zeros(n, np.uint32)
    net.prepare_update_connectivity(zeros, zeros, zeros)
    tree = net.tree()
    assert not tree["cnt_exc"].any() and not tree["cnt_inh"].any()
    net.close()


def test_no_autapse():
    rng = np.random.default_rng(485)
    n = 24
    lo, hi = np.zeros(3), np.ones(3)
    net = network(n, lo, hi, positions_in_box(rng, lo, hi, n))
    one = np.ones(n, np.uint32)
    found = 0
    for step in range(100, 1100, 100):
        net.prepare_update_connectivity(one, one, one)
        req = net.find_targets(step)
        found += len(req)
        assert np.all(req["source"] != req["target"])
    assert found > 0
    net.close()


def connector_pair(O, rng, n, upper=3):
    lo, hi = np.zeros(3), np.full(3, 100.0)
    pos = positions_in_box(rng, lo, hi, n)
    net = network(n, lo, hi, pos, seed=77)
    sim = O.OracleSim(oracle_params(params_for(n, lo, hi, seed=77)), pos, np.zeros(n, np.uint8))
    ve = rng.integers(0, upper + 1, n).astype(np.uint32)
    vi = rng.integers(0, upper + 1, n).astype(np.uint32)
    for x in (net, sim):
        x.set_elements(0, np.full(n, 100.0), np.zeros(n), np.zeros(n, np.uint32), np.full(n, 100, np.uint32))
        x.set_elements(1, ve + 0.5, np.zeros(n), np.zeros(n, np.uint32), ve)
        x.set_elements(2, vi + 0.5, np.zeros(n), np.zeros(n, np.uint32), vi)
    return net, sim, ve, vi


def assert_same_elements(net, sim):
    for t in range(3):
        a, b = net.get_elements(t), sim.get_elements(t)
        for k in ("connected", "vacant"):
            assert np.array_equal(a[k], b[k]), (t, k)


def assert_same_edges(net, sim):
    got, ref = net.edges(), sim.edges()
    for a, b in zip(got, ref):
        assert np.array_equal(np.asarray(a, np.int64), np.asarray(b, np.int64))


def test_connector_matching_requests(O):
    rng = np.random.default_rng(140)
    n = 700
    net, sim, ve, vi = connector_pair(O, rng, n)
    req = matching_requests(rng, n, ve, vi)
    created, acc = net.connect(100, req)
    assert created == len(req) == int(ve.sum() + vi.sum()) and acc.all()
    assert not net.get_elements(1)["vacant"].any() and not net.get_elements(2)["vacant"].any()
    assert np.array_equal(net.get_elements(1)["connected"], ve) and np.array_equal(net.get_elements(2)["connected"], vi)
    sim.connect_requests(100, req)
    assert_same_elements(net, sim)
    assert_same_edges(net, sim)
    net.close()


def test_connector_self_requests(O):
    rng = np.random.default_rng(232)
    n = 500
    net, sim, ve, vi = connector_pair(O, rng, n)
    before = [net.get_elements(t) for t in range(3)]
    created, acc = net.connect(100, self_requests(n, ve, vi))
    assert created == 0 and not acc.any()
    for t in range(3):
        after = net.get_elements(t)
        for k in ("grown", "delta", "connected", "vacant"):
            assert np.array_equal(after[k], before[t][k])
    assert len(net.edges()[0]) == 0
    net.close()


def test_connector_more_requests_than_vacancies(O):
    """Each (target, type) accepts exactly min(requests, vacant), and the
    accepted requests are the oracle's (the same keyed processing order)."""
    rng = np.random.default_rng(331)
    n = 300
    net, sim, ve, vi = connector_pair(O, rng, n)
    req = np.concatenate([matching_requests(rng, n, ve, vi), matching_requests(rng, n, ve + 1, vi + 2)])
    req["j"] = np.arange(len(req), dtype=np.uint32)
    created, acc = net.connect(100, req)
    assert created == int(ve.sum() + vi.sum())
    for sig, vac in ((0, ve), (1, vi)):
        got = np.bincount(req["target"][(req["signal"] == sig) & (acc == 1)], minlength=n)
        assert np.array_equal(got, vac)
    created_ref, acc_ref = sim.connect_requests(100, req)
    assert created_ref == created and np.array_equal(acc, acc_ref)
    assert_same_elements(net, sim)
    assert_same_edges(net, sim)
    net.close()


@pytest.fixture(scope="module")
def fixture_path(tmp_path_factory):
    import hashlib

    with lzma.open(os.path.join(GOLDEN, "reference_positions.txt.xz"), "rb") as f:
        data = f.read()
    assert hashlib.sha256(data).hexdigest() == open(os.path.join(GOLDEN, "reference_positions.txt.sha256")).read().split()[0]
    path = tmp_path_factory.mktemp("fixture") / "positions.txt"
    path.write_bytes(data)
    return str(path)


def test_reference_fixture_tree_and_requests(O, fixture_path):
    """The reference's 51,842 positions in its header box: the device octree
    and the requests of a seeded-vacancy snapshot (elements U[0, 4]) equal the
    oracle's bit for bit."""
    from relearn_b200 import Network, default_params, workloads

    pos, sig = workloads.read_positions_file(fixture_path)
    lo, hi = workloads.read_positions_box(fixture_path)
    n = len(pos)
    params = params_for(n, lo, hi, seed=31)
    net = Network(params)
    net.set_positions(pos, sig)
    sim = O.OracleSim(oracle_params(params), pos, sig, threads=os.cpu_count() or 1)
    check_cell_structure(O, net.tree(), pos)
    rng = np.random.default_rng(31)
    for x in (net, sim):
        x.set_elements(0, np.zeros(n), np.zeros(n), np.zeros(n, np.uint32), np.zeros(n, np.uint32))
    va = rng.integers(0, 5, n).astype(np.uint32)
    ve = rng.integers(0, 5, n).astype(np.uint32)
    vi = rng.integers(0, 5, n).astype(np.uint32)
    for t, v in enumerate((va, ve, vi)):
        for x in (net, sim):
            x.set_elements(t, v + 0.25, np.zeros(n), np.zeros(n, np.uint32), v)
    net.prepare_update_connectivity(va, ve, vi)
    sim.update_tree(ve, vi)
    assert_same_tree(net.tree(), sim.tree())
    got = net.find_targets(100)
    ref = sim.find_targets(100)
    assert len(got) == len(ref) > 0
    for k in ("target", "source", "j", "signal"):
        assert np.array_equal(got[k], ref[k]), k
    net.close()


def test_reference_fixture_driver_1001_steps(O, fixture_path, tmp_path):
    """The C++ driver reads the fixture with read_neuron_positions_and_signals
    (box from the header), seeds elements U[0, 3], runs 1,001 steps; final
    calcium and the synapse list equal the oracle's bit for bit."""
    from relearn_b200 import workloads

    pos, sig = workloads.read_positions_file(fixture_path)
    lo, hi = workloads.read_positions_box(fixture_path)
    n, seed = len(pos), 5
    prefix = str(tmp_path / "run")
    args = [os.path.join(ROOT, "relearn_b200", "bin", "relearn_b200_run"), "--file", fixture_path, "-s", "1000", "-r", str(seed),
            "--izhikevich-a", "0.02", "--izhikevich-d", "8", "--synapse-conductance", "3", "--growth-rate-axon", "1e-4",
            "--growth-rate-dendrite-exc", "1e-4", "--growth-rate-dendrite-inh", "1e-4", "--synaptic-elements-lower-bound", "0",
            "--synaptic-elements-upper-bound", "3", "--output-prefix", prefix]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ca = np.loadtxt(prefix + "_calcium.txt", dtype=np.float64)
    syn = np.loadtxt(prefix + "_synapses.txt", dtype=np.int64, ndmin=2)
    params = params_for(n, lo, hi, seed=seed)
    sim = O.OracleSim(oracle_params(params), pos, sig, threads=os.cpu_count() or 1)
    u = splitmix64_uniform(seed + 17, 3 * n).reshape(3, n)
    for t in range(3):
        g = 3.0 * u[t]
        sim.set_elements(t, g, np.zeros(n), np.zeros(n, np.uint32), np.floor(g).astype(np.uint32))
    sim.simulate(1, 1001)
    assert np.array_equal(ca.view(np.uint64), sim.neurons()["calcium"].view(np.uint64))
    t, s, w = sim.edges()
    assert len(t) > 0 and syn.shape[0] == len(t)
    assert np.array_equal(syn[:, 0], t) and np.array_equal(syn[:, 1], s) and np.array_equal(syn[:, 2], w)
