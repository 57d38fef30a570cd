"""FP32 precision form against the FP64 drop-in on the same seed.

Tolerances (stated here, measured at scale by bench.py --precision-report):
* one activity step from the same state: x and u within 1e-4 relative for
  neurons that spike in neither form; calcium within 1e-12 relative;
* selection probabilities of the first descent: within 1e-5 relative for every
  candidate with probability >= 1e-6 in the FP64 form (weights from eval32, the
  production search's own evaluation), and the production search's picks
  distributed as the FP64 probabilities (chi-square, 100,000 searches);
* a seeded FP32 run keeps the element and synapse bookkeeping consistent;
* the other neuron models (Poisson, FitzHugh-Nagumo, AEIF) in FP32: one step
  from the same state within 2e-3 relative for neurons that spike in neither
  form (the background draw's 24-bit uniform dominates), the same spikes for
  99 % of the neurons, and after 1,001 steps the mean calcium within 1e-3
  relative and the synapse counts within 1 %."""
import numpy as np
import pytest

from conftest import seed_elements, small_network

pytestmark = pytest.mark.gpu


def make(n, side, seed, precision, mixture=False):
    from relearn_b200 import Network

    params, pos, sig = small_network(n, side, seed, mixture)
    params["precision"] = precision
    net = Network(params)
    net.set_positions(pos, sig)
    return net, params, pos, sig


def test_one_step_close_to_fp64():
    n = 20000
    a, *_ = make(n, 2000.0, 5, 0)
    b, *_ = make(n, 2000.0, 5, 1)
    rng = np.random.default_rng(1)
    x0 = rng.uniform(-70.0, -50.0, n)
    u0 = rng.uniform(-14.0, -10.0, n)
    ca0 = rng.uniform(0.0, 1.0, n)
    for net in (a, b):
        net.set_neurons(x=x0, u=u0, calcium=ca0)
        net.activity_block(7, 1)
    ga, gb = a.neurons(), b.neurons()
    quiet = (ga["fired"] == 0) & (gb["fired"] == 0)
    assert quiet.mean() > 0.5
    for k in ("x", "u"):
        rel = np.abs(ga[k][quiet] - gb[k][quiet]) / np.maximum(np.abs(ga[k][quiet]), 1.0)
        assert rel.max() < 1e-4, (k, rel.max())
    both = ga["fired"] == gb["fired"]
    assert both.mean() > 0.999
    rel_ca = np.abs(ga["calcium"][both] - gb["calcium"][both]) / np.abs(ga["calcium"][both])
    assert rel_ca.max() < 1e-12


@pytest.mark.parametrize("mixture", [False, True])
def test_selection_probabilities(mixture):
    n = 50000
    net, *_ = make(n, 3700.0, 9, 1, mixture)
    one = np.ones(n, np.uint32)
    net.prepare_update_connectivity(one, one, one)
    rng = np.random.default_rng(3)
    worst = 0.0
    for s in rng.choice(n, 40, replace=False):
        n64, w64 = net.candidate_weights(int(s), 0)
        n32, w32 = net.candidate_weights(int(s), 1)
        p64 = dict(zip(n64.tolist(), (w64 / w64.sum()).tolist()))
        p32 = dict(zip(n32.tolist(), (w32 / w32.sum()).tolist()))
        for node, p in p64.items():
            if p >= 1e-6:
                worst = max(worst, abs(p32.get(node, 0.0) - p) / p)
    assert worst <= 1e-5, worst


def first_descent_candidate_of(tree: dict, candidates: np.ndarray) -> np.ndarray:
    """For every octree node, the first-descent candidate whose subtree holds
    it (-1 for nodes above or outside the candidates).  The candidates of the
    walk from the root partition the neurons, and nodes are stored breadth
    first, so a parent comes before its children."""
    m = len(tree["level"])
    parent = np.full(m, -1, np.int64)
    for i in np.flatnonzero(tree["first_child"] >= 0):
        k = bin(int(tree["child_mask"][i])).count("1")
        parent[tree["first_child"][i]: tree["first_child"][i] + k] = i
    owner = np.full(m, -1, np.int64)
    is_cand = np.zeros(m, bool)
    is_cand[candidates] = True
    for i in range(m):
        owner[i] = i if is_cand[i] else (owner[parent[i]] if parent[i] >= 0 else -1)
    return owner


@pytest.mark.parametrize("precision", [0, 1])
def test_pick_frequencies_match_fp64_probabilities(precision):
    """The production search (k_search / k_search_f32: weights by eval32,
    Kahan-compensated running sums, the 24-bit threshold; Kernel.h:90-173 and
    ProbabilityPicker.h:97-112 in the reference) picks each first-descent
    candidate with its FP64 probability: 100,000 searches of one source,
    repeated over steps and vacant-axon indices, whose final targets are mapped
    to the first-descent candidate that contains them, against the FP64
    weights by a chi-square test."""
    from scipy.stats import chi2

    n, per_step, steps = 3000, 2000, 50
    net, *_ = make(n, 1000.0, 13, precision)
    source = 1234
    va = np.zeros(n, np.uint32)
    va[source] = per_step
    one = np.ones(n, np.uint32)
    net.prepare_update_connectivity(va, one, one)
    nodes, w64 = net.candidate_weights(source, 0)
    p = w64 / w64.sum()
    owner = first_descent_candidate_of(net.tree(), nodes)
    leaf_of = np.full(n, -1, np.int64)
    tree = net.tree()
    leaves = np.flatnonzero(tree["neuron"] >= 0)
    leaf_of[tree["neuron"][leaves]] = leaves
    index = {int(v): k for k, v in enumerate(nodes)}
    counts = np.zeros(len(nodes))
    for step in range(100, 100 + steps):
        req = net.find_targets(step)
        assert len(req) == per_step and np.all(req["source"] == source)
        cand = owner[leaf_of[req["target"]]]
        assert np.all(cand >= 0)
        np.add.at(counts, [index[int(c)] for c in cand], 1)
    total = counts.sum()
    expect = p * total
    big = expect >= 5
    obs = np.append(counts[big], counts[~big].sum())
    exp = np.append(expect[big], expect[~big].sum())
    keep = exp > 0
    stat = float(np.sum((obs[keep] - exp[keep]) ** 2 / exp[keep]))
    dof = int(keep.sum()) - 1
    pval = float(chi2.sf(stat, dof))
    assert counts[p == 0].sum() == 0
    assert pval > 1e-4, (stat, dof, pval)


def test_seeded_fp32_run_bookkeeping():
    n = 4000
    net, *_ = make(n, 1260.0, 11, 1)
    seed_elements(net, n, 4, 0.0, 3.0)
    net.simulate(1, 1001)
    st = net.stats()
    assert st["synapses_created"] > 0
    t, s, w = net.edges()
    ax = net.get_elements(0)["connected"]
    ex = net.get_elements(1)["connected"]
    ih = net.get_elements(2)["connected"]
    # every synapse is counted once on each side
    assert ax.sum() == np.abs(w).sum() == ex.sum() + ih.sum()
    out_deg = np.bincount(s, weights=np.abs(w), minlength=n)
    assert np.array_equal(out_deg.astype(np.uint32), ax)


@pytest.mark.parametrize("kernel", [dict(kernel_type=1, kernel_k=2.0, kernel_scale=400.0), dict(kernel_type=2, linear_cutoff=1500.0),
                                    dict(kernel_type=3, kernel_k=1.5, kernel_scale=0.002)])
def test_selection_probabilities_other_kernels(kernel):
    """Gamma, linear and Weibull kernels in FP32 (powers through log2 / exp2):
    the distribution over the first descent's candidates within 1e-5 total
    variation of the FP64 form; for gamma and Weibull also every candidate
    with probability >= 1e-6 within 1e-4 relative (the linear kernel's weight
    1 - d / cutoff loses relative precision as d approaches the cut-off)."""
    from relearn_b200 import Network

    n = 20000
    params, pos, sig = small_network(n, 2700.0, 12)
    params.update(kernel)
    params["precision"] = 1
    net = Network(params)
    net.set_positions(pos, sig)
    one = np.ones(n, np.uint32)
    net.prepare_update_connectivity(one, one, one)
    worst, tv = 0.0, 0.0
    for s in np.random.default_rng(4).choice(n, 20, replace=False):
        n64, w64 = net.candidate_weights(int(s), 0)
        n32, w32 = net.candidate_weights(int(s), 1)
        p64 = dict(zip(n64.tolist(), (w64 / w64.sum()).tolist()))
        p32 = dict(zip(n32.tolist(), (w32 / w32.sum()).tolist()))
        tv = max(tv, 0.5 * sum(abs(p64.get(k, 0.0) - p32.get(k, 0.0)) for k in set(p64) | set(p32)))
        for node, p in p64.items():
            if p >= 1e-6:
                worst = max(worst, abs(p32.get(node, 0.0) - p) / p)
    assert tv <= 1e-5, tv
    if kernel["kernel_type"] != 2:
        assert worst <= 1e-4, worst


def make_model(n, model, precision, seed):
    from relearn_b200 import Network

    params, pos, sig = small_network(n, 2000.0, seed)
    params["precision"] = precision
    params["neuron_model"] = model
    if model == 3:
        params["noise_mean"] = 600.0  # pA: enough drive for the AEIF neuron to spike
        params["noise_stddev"] = 200.0
    net = Network(params)
    net.set_positions(pos, sig)
    return net


@pytest.mark.parametrize("model", [1, 2, 3])
def test_other_models_track_fp64(model):
    n = 20000
    rng = np.random.default_rng(model)
    if model == 1:
        x0 = rng.uniform(0.0, 1.0, n)
        u0 = np.where(rng.random(n) < 0.2, 2.0, 0.0)  # refractory steps left
    elif model == 2:
        x0 = rng.uniform(-2.0, 2.0, n)
        u0 = rng.uniform(-1.0, 1.0, n)
    else:
        x0 = rng.uniform(-70.0, -50.0, n)
        u0 = rng.uniform(0.0, 50.0, n)
    ca0 = rng.uniform(0.0, 1.0, n)
    a, b = make_model(n, model, 0, 5), make_model(n, model, 1, 5)
    for net in (a, b):
        net.set_neurons(x=x0, u=u0, calcium=ca0)
        net.activity_block(7, 1)
    ga, gb = a.neurons(), b.neurons()
    assert (ga["fired"] == gb["fired"]).mean() > 0.99
    quiet = (ga["fired"] == 0) & (gb["fired"] == 0)
    assert quiet.sum() > 100
    for k in ("x", "u"):
        rel = np.abs(ga[k][quiet] - gb[k][quiet]) / np.maximum(np.abs(ga[k][quiet]), 1.0)
        assert rel.max() < 2e-3, (k, rel.max())

    a, b = make_model(n, model, 0, 9), make_model(n, model, 1, 9)
    for net in (a, b):
        seed_elements(net, n, 9, 0.0, 3.0)
        net.simulate(1, 1001)
    ga, gb = a.neurons(), b.neurons()
    assert abs(ga["calcium"].mean() - gb["calcium"].mean()) < 1e-3 * abs(ga["calcium"].mean())
    ea, eb = len(a.edges()[0]), len(b.edges()[0])
    assert ea > 0 and abs(ea - eb) <= 0.01 * ea
