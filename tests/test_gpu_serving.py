"""Serving form: continuous admission, overlap on the device and packing of
small requests must not change any result.  Every request's final state
(x, u, calcium, connected elements, synapses) is compared bit for bit between
a run alone (one slot, no packing) and a run in the mix (several slots,
packing), in both precision forms; the tolerance is zero."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def make_requests(seed, k, lo, hi, steps):
    from relearn_b200 import workloads

    rng = np.random.default_rng(seed)
    out = []
    for i in range(k):
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        net = dict(num_neurons=n, seed=1000 + 31 * i, side=(1000.0 * n) ** (1 / 3), theta=float(rng.uniform(0.2, 0.5)), sigma=750.0,
                   growth_rate=float(np.exp(rng.uniform(np.log(1e-4), np.log(1e-3)))))
        pos, sig = workloads.request_inputs(net)
        grown = [g for g, _ in workloads.initial_elements(n, 70 + i, 0.0, 3.0)]
        out.append((net, pos, sig, grown, steps))
    return out


def serve(params, reqs, **kw):
    from relearn_b200.serving import Server

    with Server(params, **kw) as srv:
        ids = [srv.submit(net, pos, sig, steps, grown=grown, keep_state=True) for net, pos, sig, grown, steps in reqs]
        done = {}
        while len(done) < len(ids):
            for d in srv.poll(wait_ms=1000):
                done[d["id"]] = d
        states = {i: srv.fetch(done[i]) for i in ids}
    return ids, done, states


@pytest.mark.parametrize("precision", [0, 1])
def test_same_alone_and_in_mix(precision):
    from relearn_b200 import default_params

    params = default_params(1, 1.0)
    params["precision"] = precision
    reqs = make_requests(precision, 10, 400, 12000, 301)
    ids_a, done_a, alone = serve(params, reqs, slots=1, pack_networks=1)
    ids_m, done_m, mix = serve(params, reqs, slots=4, pack_networks=4, pack_max_neurons=5000)
    assert all(d["status"] == 0 for d in list(done_a.values()) + list(done_m.values()))
    assert max(d["pack_size"] for d in done_m.values()) > 1
    # requests overlapped on the device in the mix
    iv = sorted((d["t_admit"], d["t_finish"]) for d in done_m.values())
    assert any(iv[k + 1][0] < iv[k][1] for k in range(len(iv) - 1))
    made = 0
    for a, m in zip(ids_a, ids_m):
        sa, sm = alone[a], mix[m]
        for key in ("x", "u", "calcium"):
            assert np.array_equal(sa[key].view(np.uint64), sm[key].view(np.uint64)), key
        for key in ("connected", "target", "source", "weight"):
            assert np.array_equal(sa[key], sm[key]), key
        made += len(sa["target"])
    assert made > 0


def test_request_equals_single_context():
    from relearn_b200 import Network, default_params

    params = default_params(1, 1.0)
    reqs = make_requests(5, 1, 3000, 3001, 401)
    _, done, states = serve(params, reqs, slots=2)
    net, pos, sig, grown, steps = reqs[0]
    p = dict(params)
    p.update(num_neurons=net["num_neurons"], seed=net["seed"], box_max=(net["side"],) * 3, theta=net["theta"], sigma=net["sigma"],
             growth_rate=(net["growth_rate"],) * 3)
    one = Network(p)
    one.set_positions(pos, sig)
    for t in range(3):
        one.set_elements(t, grown[t])
    one.simulate(1, steps)
    a = one.neurons()
    s = next(iter(states.values()))
    assert np.array_equal(a["calcium"].view(np.uint64), s["calcium"].view(np.uint64))
    t, src, w = one.edges()
    assert np.array_equal(t, s["target"]) and np.array_equal(src, s["source"]) and np.array_equal(w, s["weight"])


def test_admission_respects_budget():
    from relearn_b200 import default_params
    from relearn_b200.serving import Server

    params = default_params(1, 1.0)
    reqs = make_requests(9, 8, 3000, 30000, 201)
    with Server(params, slots=8, pack_networks=1) as probe:
        fps = [probe.footprint(net, steps, float(grown[0].sum())) for net, _, _, grown, steps in reqs]
    budget = 2.2 * max(fps)
    ids, done, _ = serve(params, reqs, slots=8, pack_networks=1, hbm_budget_bytes=budget)
    recs = list(done.values())
    assert all(d["status"] == 0 for d in recs)
    for d in recs:
        # the admitted footprint bounds the context's measured peak
        assert d["device_peak_bytes"] <= d["footprint_bytes"], d
        live = [e for e in recs if e["t_admit"] <= d["t_admit"] < e["t_finish"]]
        assert sum(e["footprint_bytes"] for e in live) <= budget
