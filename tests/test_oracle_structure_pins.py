"""The oracle's octree, acceptance walk, target search and connector pinned
to the reference's own tests of them, re-expressed (no GPU needed):

* cell octants and octant boxes: test/cell/test_cell.cpp:1314-1400
  (testBarnesHutCellOctants, ...OctantsException, ...OctantsSize);
* acceptance criterion: test/barnes_hut/test_barnes_hut_base.cpp:57-239
  (testACException, testACLeafDendrites, testACLeafSamePositionDendrites,
  testACParentDendrite);
* nodes to consider: test_barnes_hut_base.cpp:420-517 (no synaptic elements;
  the walk equals the golden stack walk);
* target search: test_barnes_hut_base.cpp:830-1000 (no dendrites, no / one /
  full choice);
* bottom-up sums and no autapse: test/barnes_hut_cuda/test_barnes_hut_cuda.cpp:
  250-357, 485-563;
* connector: test/connector/test_connector.cpp:140-330 (matching requests,
  self requests), plus more requests than vacancies;
* the reference's own positions fixture (relearn/input/positions.txt) loads
  through the positions reader with its header box and builds an octree
  with the cell properties above."""
import lzma
import os

import numpy as np
import pytest

from conftest import oracle_params
from structure_pins import (check_bottom_up_sums, check_cell_structure, golden_walk, matching_requests, positions_in_box, random_box,
                            random_theta, self_requests)

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.fixture(scope="module")
def O(oracle_mod):
    return oracle_mod


def make_sim(O, n, lo, hi, pos, theta=0.3, sig=None, seed=1):
    from relearn_b200 import default_params

    p = default_params(n, 1.0)
    p["box_min"], p["box_max"], p["theta"], p["seed"] = tuple(lo), tuple(hi), theta, seed
    sig = np.zeros(n, np.uint8) if sig is None else sig
    return O.OracleSim(oracle_params(p), pos, sig)


def test_cell_octants(O):
    rng = np.random.default_rng(1314)
    for _ in range(20):
        lo, hi = random_box(rng)
        mid = (lo + hi) / 2
        for p in positions_in_box(rng, lo, hi, 200):
            expect = (1 if p[0] >= mid[0] else 0) + (2 if p[1] >= mid[1] else 0) + (4 if p[2] >= mid[2] else 0)
            assert O.octant_of(lo, hi, p) == expect


def test_cell_octants_outside_box(O):
    rng = np.random.default_rng(1337)
    lo, hi = random_box(rng)
    for a in range(3):
        e = np.zeros(3)
        e[a] = 1.0
        assert O.octant_of(lo, hi, hi + e) == -1
        assert O.octant_of(lo, hi, lo - e) == -1


def test_cell_octant_sizes(O):
    rng = np.random.default_rng(1361)
    for _ in range(50):
        lo, hi = random_box(rng)
        mid = (lo + hi) / 2
        for o in range(8):
            k = np.array([o & 1, o >> 1 & 1, o >> 2 & 1], dtype=np.float64)
            sub_lo, sub_hi = O.box_for_octant(lo, hi, o)
            exp_lo, exp_hi = lo + k * (mid - lo), mid + k * (mid - lo)
            assert np.linalg.norm(sub_lo - exp_lo) <= 8 * np.finfo(float).eps * max(np.linalg.norm(exp_lo), 1.0)
            assert np.linalg.norm(sub_hi - exp_hi) <= 8 * np.finfo(float).eps * max(np.linalg.norm(exp_hi), 1.0)
            # the reference's own rule: every bound is a corner or the midpoint
            assert np.array_equal(sub_lo, np.where(k == 1, mid, lo)) and np.array_equal(sub_hi, np.where(k == 1, hi, mid))


def test_acceptance_theta_bounds(O):
    lo, hi = np.zeros(3), np.full(3, 10.0)
    for theta in (0.0, -0.1, -1000.0, 0.5 + 1e-9, 1000.0):
        assert O.acceptance(False, lo, hi, 1, np.full(3, 5.0), np.full(3, 15.0), theta) == -1
    assert O.acceptance(False, lo, hi, 1, np.full(3, 5.0), np.full(3, 15.0), 0.5) == O.ACCEPT


def test_acceptance_leaf(O):
    """A leaf with vacant dendrites of the searched type is accepted from any
    other position; one without is discarded; from its own position it is
    discarded whatever it holds."""
    rng = np.random.default_rng(94)
    lo, hi = np.zeros(3), np.full(3, 10.0)
    node_pos = positions_in_box(rng, lo, hi, 1)[0]
    theta = random_theta(rng)
    for _ in range(1000):
        src = rng.uniform(-1e4, 1e4, 3)
        count = int(rng.integers(1, 1001))
        assert O.acceptance(False, lo, hi, count, node_pos, src, theta) == O.ACCEPT
        assert O.acceptance(False, lo, hi, 0, node_pos, src, theta) == O.DISCARD
        assert O.acceptance(False, lo, hi, int(rng.integers(0, 1001)), node_pos, node_pos, theta) == O.DISCARD


def test_acceptance_parent(O):
    """An inner node is accepted when theta > (largest cell edge) / distance
    and expanded otherwise; without vacant dendrites it is discarded."""
    rng = np.random.default_rng(182)
    lo, hi = random_box(rng)
    lo, hi = lo / 10.0, hi / 10.0
    node_pos = positions_in_box(rng, lo, hi, 1)[0]
    longest = float(np.max(hi - lo))
    seen = set()
    for _ in range(1000):
        theta = random_theta(rng)
        src = rng.uniform(-1e4, 1e4, 3)
        dist = float(np.linalg.norm(node_pos - src))
        count = int(rng.integers(1, 1001))
        st = O.acceptance(True, lo, hi, count, node_pos, src, theta)
        expect = O.ACCEPT if theta > longest / dist else O.EXPAND
        assert st == expect
        seen.add(st)
        assert O.acceptance(True, lo, hi, 0, node_pos, src, theta) == O.DISCARD
    assert seen == {O.ACCEPT, O.EXPAND}


def standard_tree(O, rng, n=None, counts=(1, 2), theta=None):
    """OctreeFactory::get_standard_tree: n neurons uniform in a random box,
    vacant dendrites of each type uniform in `counts`."""
    n = int(rng.integers(1, 1001)) + 1 if n is None else n
    lo, hi = random_box(rng)
    pos = positions_in_box(rng, lo, hi, n)
    sim = make_sim(O, n, lo, hi, pos, theta=random_theta(rng) if theta is None else theta)
    ve = rng.integers(counts[0], counts[1] + 1, n).astype(np.uint32)
    vi = rng.integers(counts[0], counts[1] + 1, n).astype(np.uint32)
    sim.update_tree(ve, vi)
    return sim, pos, lo, hi, ve, vi


def test_octree_cells(O):
    rng = np.random.default_rng(230)
    for n in (1, 2, 3, 57, 1000):
        sim, pos, *_ = standard_tree(O, rng, n)
        check_cell_structure(O, sim.tree(), pos)


def test_nodes_to_consider_without_elements(O):
    rng = np.random.default_rng(420)
    sim, pos, lo, hi, *_ = standard_tree(O, rng, counts=(0, 0))
    for _ in range(100):
        src = rng.uniform(-1e4, 1e4, 3)
        for t in (0, 1):
            assert len(sim.nodes_to_consider(src, t)) == 0


@pytest.mark.parametrize("seed", [457, 458, 459])
def test_nodes_to_consider_equals_golden_walk(O, seed):
    rng = np.random.default_rng(seed)
    sim, pos, lo, hi, *_ = standard_tree(O, rng)
    tree = sim.tree()
    theta = sim.params["theta"]
    for _ in range(60):
        src = rng.uniform(-1e4, 1e4, 3) if rng.random() < 0.5 else pos[int(rng.integers(0, len(pos)))]
        t = int(rng.integers(0, 2))
        assert sim.nodes_to_consider(src, t).tolist() == golden_walk(O, tree, src, t, theta)


def test_find_target_no_dendrites(O):
    rng = np.random.default_rng(830)
    sim, pos, *_ = standard_tree(O, rng, counts=(0, 0))
    for i in range(len(pos)):
        src = rng.uniform(-1e4, 1e4, 3)
        assert sim.find_target(i, src, int(rng.integers(0, 2)), 100, 0) == -1


def test_find_target_no_choice(O):
    """A single neuron: it finds no target itself; another source gets it."""
    rng = np.random.default_rng(866)
    lo, hi = random_box(rng)
    pos = positions_in_box(rng, lo, hi, 1)
    sim = make_sim(O, 1, lo, hi, pos, theta=random_theta(rng))
    sim.update_tree(np.array([2], np.uint32), np.array([2], np.uint32))
    for step in range(50):
        t = int(rng.integers(0, 2))
        src = rng.uniform(-1e4, 1e4, 3)
        assert sim.find_target(0, src, t, step, 0) == -1
        assert sim.find_target(1, src, t, step, 0) == 0


def test_find_target_one_choice(O):
    rng = np.random.default_rng(905)
    for _ in range(20):
        lo, hi = random_box(rng)
        pos = positions_in_box(rng, lo, hi, 2)
        sim = make_sim(O, 2, lo, hi, pos, theta=random_theta(rng))
        sim.update_tree(np.array([1, 2], np.uint32), np.array([1, 2], np.uint32))
        t = int(rng.integers(0, 2))
        assert sim.find_target(0, pos[0], t, 7, 0) == 1
        assert sim.find_target(1, pos[1], t, 7, 0) == 0


def test_find_target_full_choice(O):
    rng = np.random.default_rng(959)
    sim, pos, lo, hi, ve, vi = standard_tree(O, rng)
    for i in range(len(pos)):
        t = int(rng.integers(0, 2))
        tgt = sim.find_target(i, pos[i], t, 11, 0)
        assert tgt >= 0 and tgt != i
        assert (ve if t == 0 else vi)[tgt] > 0


def test_bottom_up_sums(O):
    rng = np.random.default_rng(283)
    n = 100
    lo, hi = np.zeros(3), np.ones(3)
    pos = positions_in_box(rng, lo, hi, n)
    sim = make_sim(O, n, lo, hi, pos)
    sim.update_tree(np.ones(n, np.uint32), np.zeros(n, np.uint32))
    tree = sim.tree()
    check_bottom_up_sums(tree)
    assert tree["cnt_exc"][0] == n and not tree["cnt_inh"].any()
    leaves = tree["neuron"] >= 0
    assert np.all(tree["cnt_exc"][leaves] == 1)
    # without dendrites anywhere the roll-up leaves every count at zero
    sim.update_tree(np.zeros(n, np.uint32), np.zeros(n, np.uint32))
    tree = sim.tree()
    assert not tree["cnt_exc"].any() and not tree["cnt_inh"].any()


def test_no_autapse(O):
    rng = np.random.default_rng(485)
    n = 24
    lo, hi = np.zeros(3), np.ones(3)
    pos = positions_in_box(rng, lo, hi, n)
    sim = make_sim(O, n, lo, hi, pos)
    one = np.ones(n, np.uint32)
    for t in range(3):
        sim.set_elements(t, np.full(n, 1.5), np.zeros(n), np.zeros(n, np.uint32), one)
    sim.update_tree(one, one)
    found = 0
    for step in range(100, 600, 100):
        req = sim.find_targets(step)
        found += len(req)
        assert np.all(req["source"] != req["target"])
    assert found > 0


def connector_sim(O, rng, n, upper=3):
    lo, hi = np.zeros(3), np.full(3, 100.0)
    pos = positions_in_box(rng, lo, hi, n)
    sim = make_sim(O, n, lo, hi, pos)
    ve = rng.integers(0, upper + 1, n).astype(np.uint32)
    vi = rng.integers(0, upper + 1, n).astype(np.uint32)
    sim.set_elements(0, np.full(n, 100.0), np.zeros(n), np.zeros(n, np.uint32), np.full(n, 100, np.uint32))
    sim.set_elements(1, ve + 0.5, np.zeros(n), np.zeros(n, np.uint32), ve)
    sim.set_elements(2, vi + 0.5, np.zeros(n), np.zeros(n, np.uint32), vi)
    return sim, ve, vi


def test_connector_matching_requests(O):
    rng = np.random.default_rng(140)
    n = int(rng.integers(2, 1001))
    sim, ve, vi = connector_sim(O, rng, n)
    req = matching_requests(rng, n, ve, vi)
    created, acc = sim.connect_requests(100, req)
    assert created == len(req) == int(ve.sum() + vi.sum()) and acc.all()
    assert not sim.get_elements(1)["vacant"].any() and not sim.get_elements(2)["vacant"].any()
    assert np.array_equal(sim.get_elements(1)["connected"], ve) and np.array_equal(sim.get_elements(2)["connected"], vi)
    assert_edges_from_requests(sim.edges(), req[acc == 1], n)


def assert_edges_from_requests(edges, accepted, n):
    """Each accepted request adds weight +1 (excitatory) or -1 (inhibitory)
    to its (target, source) pair; the edge list holds the nonzero sums."""
    t, s, w = edges
    sign = np.where(accepted["signal"] == 1, -1, 1)
    key = accepted["target"].astype(np.int64) * n + accepted["source"]
    uk, inv = np.unique(key, return_inverse=True)
    net = np.bincount(inv, weights=sign).astype(np.int64)
    keep = net != 0
    got = dict(zip((np.asarray(t, np.int64) * n + s).tolist(), np.asarray(w).tolist()))
    assert got == dict(zip(uk[keep].tolist(), net[keep].tolist()))


def test_connector_self_requests(O):
    rng = np.random.default_rng(232)
    n = int(rng.integers(2, 1001))
    sim, ve, vi = connector_sim(O, rng, n)
    before = [sim.get_elements(t) for t in range(3)]
    req = self_requests(n, ve, vi)
    created, acc = sim.connect_requests(100, req)
    assert created == 0 and not acc.any()
    for t in range(3):
        after = sim.get_elements(t)
        for k in ("grown", "delta", "connected", "vacant"):
            assert np.array_equal(after[k], before[t][k])
    assert len(sim.edges()[0]) == 0


def test_connector_more_requests_than_vacancies(O):
    """Requests past a target's vacant dendrites of a type fail ("other axons
    were faster"), so each (target, type) accepts exactly min(requests, vacant)."""
    rng = np.random.default_rng(331)
    n = 300
    sim, ve, vi = connector_sim(O, rng, n)
    req = np.concatenate([matching_requests(rng, n, ve, vi), matching_requests(rng, n, ve + 1, vi + 2)])
    req["j"] = np.arange(len(req), dtype=np.uint32)  # distinct keys
    created, acc = sim.connect_requests(100, req)
    assert created == int(ve.sum() + vi.sum())
    for sig, vac in ((0, ve), (1, vi)):
        got = np.bincount(req["target"][(req["signal"] == sig) & (acc == 1)], minlength=n)
        assert np.array_equal(got, vac)


def decompress_fixture(tmp_path):
    import hashlib

    with lzma.open(os.path.join(GOLDEN, "reference_positions.txt.xz"), "rb") as f:
        data = f.read()
    want = open(os.path.join(GOLDEN, "reference_positions.txt.sha256")).read().split()[0]
    assert hashlib.sha256(data).hexdigest() == want
    path = tmp_path / "positions.txt"
    path.write_bytes(data)
    return str(path)


def test_reference_positions_fixture(O, tmp_path):
    """relearn/input/positions.txt: 51,842 neurons, all excitatory as
    NeuronIO::read_neuron_positions_and_signals reads them (its fifth token is
    the area label, and only "in" means inhibitory), the box from the header,
    every neuron inside it; the oracle's octree over it has the reference's
    cell properties."""
    from relearn_b200 import workloads

    path = decompress_fixture(tmp_path)
    pos, sig = workloads.read_positions_file(path)
    box = workloads.read_positions_box(path)
    assert pos.shape == (51842, 3) and not sig.any()
    assert box is not None
    lo, hi = box
    assert np.array_equal(lo, np.zeros(3)) and np.array_equal(hi, [141.0981, 176.00237, 130.5685])
    assert np.all(pos >= lo) and np.all(pos <= hi)
    sim = make_sim(O, len(pos), lo, hi, pos)
    tree = sim.tree()
    check_cell_structure(O, tree, pos)
