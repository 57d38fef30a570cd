"""Helpers of the structural pins: the reference's octree, Barnes-Hut and
connector tests restated as properties, for the oracle (tests/test_oracle_structure_pins.py)
and the product (tests/test_gpu_structure_pins.py).

The reference's tests draw boxes, positions and counts from its test
factories (harness/factory): boxes with corners uniform in [-10,000, 10,000]
per axis (simulation_factory.cpp:23-37), at most 1,000 neurons
(neuron_id_factory.h:22), 1-2 vacant dendrites of each type per leaf in the
standard tree (octree_factory.h:33-60), theta uniform in (eps, 0.5]."""
import numpy as np

POSITION_BOUNDARY = 10_000.0
MAX_THETA = 0.5
EPS = 1e-6


def random_box(rng):
    """SimulationFactory::get_random_simulation_box_size."""
    a = rng.uniform(-POSITION_BOUNDARY, POSITION_BOUNDARY, 3)
    b = rng.uniform(-POSITION_BOUNDARY, POSITION_BOUNDARY, 3)
    return np.minimum(a, b), np.maximum(a, b)


def random_theta(rng):
    return float(rng.uniform(EPS, MAX_THETA))


def positions_in_box(rng, lo, hi, n):
    return lo + (hi - lo) * rng.random((n, 3))


def children(tree, i):
    """Children of node i in octant order, with their octants."""
    first = int(tree["first_child"][i])
    if first < 0:
        return []
    mask = int(tree["child_mask"][i])
    octs = [o for o in range(8) if mask >> o & 1]
    return [(first + k, o) for k, o in enumerate(octs)]


def parents(tree):
    m = len(tree["level"])
    par = np.full(m, -1, np.int64)
    octant = np.full(m, -1, np.int64)
    for i in np.flatnonzero(tree["first_child"] >= 0):
        for c, o in children(tree, int(i)):
            par[c] = i
            octant[c] = o
    return par, octant


def node_status(O, tree, i, src, dendrite_type, theta):
    """BarnesHutBase::test_acceptance_criterion of node i of a dumped tree
    (the oracle's single-node restatement)."""
    cnt = tree["cnt_exc" if dendrite_type == 0 else "cnt_inh"][i]
    pos = tree["pos_exc" if dendrite_type == 0 else "pos_inh"][i]
    parent = tree["first_child"][i] >= 0
    return O.acceptance(bool(parent), tree["bmin"][i], tree["bmax"][i], int(cnt), pos, src, theta)


def golden_walk(O, tree, src, dendrite_type, theta):
    """The golden list of test_barnes_hut_base.cpp:477-517: push the root's
    children, pop the top node, keep it on Accept, push its children on
    Expand, drop it on Discard; nodes in the order they are kept.  A root
    that is a leaf is itself the only candidate unless discarded
    (BarnesHutBase.h:141-156); a root without elements of the type gives none."""
    cnt = tree["cnt_exc" if dendrite_type == 0 else "cnt_inh"]
    if cnt[0] == 0:
        return []
    if tree["first_child"][0] < 0:
        return [0] if node_status(O, tree, 0, src, dendrite_type, theta) != O.DISCARD else []
    stack = [c for c, _ in children(tree, 0)]
    out = []
    while stack:
        i = stack.pop()
        st = node_status(O, tree, i, src, dendrite_type, theta)
        if st == O.ACCEPT:
            out.append(i)
        elif st == O.EXPAND:
            stack.extend(c for c, _ in children(tree, i))
    return out


def check_cell_structure(O, tree, positions):
    """Cell::get_octant_for_position and Cell::get_size_for_octant on every
    node of a dumped tree (test_cell.cpp:1314-1400): each child's box is the
    octant box of its parent (exactly the reference's midpoint rule, and
    within the reference test's tolerance of its own expectation), and each
    neuron's position lies in its leaf's box and in the octant of every
    ancestor that leads to it."""
    par, octant = parents(tree)
    m = len(par)
    for c in range(1, m):
        p = par[c]
        assert p >= 0, c
        lo, hi = O.box_for_octant(tree["bmin"][p], tree["bmax"][p], int(octant[c]))
        assert np.array_equal(lo.view(np.uint64), tree["bmin"][c].view(np.uint64)), c
        assert np.array_equal(hi.view(np.uint64), tree["bmax"][c].view(np.uint64)), c
        # the reference test's own expectation: min + k * (mid - min) per axis
        pmin, pmax = tree["bmin"][p], tree["bmax"][p]
        mid = (pmin + pmax) / 2
        k = np.array([octant[c] & 1, octant[c] >> 1 & 1, octant[c] >> 2 & 1], dtype=np.float64)
        exp_lo, exp_hi = pmin + k * (mid - pmin), mid + k * (mid - pmin)
        scale = max(np.linalg.norm(exp_hi), 1.0)
        assert np.linalg.norm(exp_lo - lo) <= 8 * np.finfo(float).eps * scale
        assert np.linalg.norm(exp_hi - hi) <= 8 * np.finfo(float).eps * scale
        assert tree["level"][c] == tree["level"][p] + 1
    leaves = np.flatnonzero(tree["neuron"] >= 0)
    assert len(leaves) == len(positions)
    assert np.array_equal(np.sort(tree["neuron"][leaves]), np.arange(len(positions)))
    for leaf in leaves:
        pos = positions[tree["neuron"][leaf]]
        assert np.all(tree["bmin"][leaf] <= pos) and np.all(pos <= tree["bmax"][leaf])
        c = leaf
        while par[c] >= 0:
            p = par[c]
            assert O.octant_of(tree["bmin"][p], tree["bmax"][p], pos) == octant[c], (leaf, p)
            c = p


def check_bottom_up_sums(tree):
    """test_barnes_hut_cuda.cpp:283-357: every inner node's vacant count is
    the sum of its children's, for both dendrite types."""
    for i in np.flatnonzero(tree["first_child"] >= 0):
        ch = [c for c, _ in children(tree, int(i))]
        for key in ("cnt_exc", "cnt_inh"):
            assert int(tree[key][i]) == int(sum(int(tree[key][c]) for c in ch)), (i, key)


def matching_requests(rng, n, vac_exc, vac_inh):
    """test_connector.cpp:140-230 re-expressed for one rank: every vacant
    dendrite of every neuron receives one request of its type from another
    neuron (the sources need a vacant axon per request)."""
    reqs = []
    for t in range(n):
        for sig, count in ((0, vac_exc[t]), (1, vac_inh[t])):
            for _ in range(int(count)):
                s = int(rng.integers(0, n - 1))
                s = s if s < t else s + 1
                reqs.append((t, s, 0, sig))
    req = np.zeros(len(reqs), dtype=[("target", "<u4"), ("source", "<u4"), ("j", "<u4"), ("signal", "<u4")])
    if reqs:
        a = np.array(reqs, np.uint32)
        req["target"], req["source"], req["signal"] = a[:, 0], a[:, 1], a[:, 3]
    # j numbers the requests of a source
    order = np.argsort(req["source"], kind="stable")
    src_sorted = req["source"][order]
    starts = np.r_[0, np.flatnonzero(np.diff(src_sorted)) + 1]
    j = np.arange(len(req)) - np.repeat(starts, np.diff(np.r_[starts, len(req)]))
    req["j"][order] = j.astype(np.uint32)
    return req


def self_requests(n, vac_exc, vac_inh):
    """test_connector.cpp:232-330: each vacant dendrite requested by its own
    neuron."""
    reqs = []
    for t in range(n):
        k = 0
        for sig, count in ((0, vac_exc[t]), (1, vac_inh[t])):
            for _ in range(int(count)):
                reqs.append((t, t, k, sig))
                k += 1
    req = np.zeros(len(reqs), dtype=[("target", "<u4"), ("source", "<u4"), ("j", "<u4"), ("signal", "<u4")])
    if reqs:
        a = np.array(reqs, np.uint32)
        req["target"], req["source"], req["j"], req["signal"] = a[:, 0], a[:, 1], a[:, 2], a[:, 3]
    return req
