"""Host side of the serving form (no GPU): the request stream of the serving
workload, the footprint model and the request loop's refusal and error paths."""
import numpy as np
import pytest


def test_serving_stream_shape():
    from relearn_b200 import workloads

    st = workloads.serving_stream(3, 20.0, 600.0)
    t = np.array([a for a, _ in st])
    n = np.array([d["num_neurons"] for _, d in st])
    assert np.all(np.diff(t) > 0) and t[-1] < 600.0
    # Poisson at 20/s over 600 s: 12,000 +- a few sigma
    assert abs(len(st) - 12000) < 5 * np.sqrt(12000)
    assert n.min() >= 2000 and n.max() <= 1_000_000
    # log-uniform sizes: the median sits near the geometric mean sqrt(2e3 * 1e6)
    assert 0.8 < np.median(n) / np.sqrt(2e3 * 1e6) < 1.25
    th = np.array([d["theta"] for _, d in st])
    gr = np.array([d["growth_rate"] for _, d in st])
    assert th.min() >= 0.2 and th.max() <= 0.5 and gr.min() >= 1e-5 and gr.max() <= 1e-3
    assert len({d["seed"] for _, d in st}) == len(st)
    pos, sig = workloads.request_inputs(st[0][1])
    assert pos.shape == (st[0][1]["num_neurons"], 3) and np.all(pos < st[0][1]["side"])


def test_footprint_model(built_lib):
    from relearn_b200 import default_params
    from relearn_b200.serving import Server

    with Server(default_params(1, 1.0), slots=1) as srv:
        net = dict(num_neurons=100_000, seed=1, side=4641.6, theta=0.3, sigma=750.0, growth_rate=1e-4)
        a = srv.footprint(net, 5000)
        b = srv.footprint(dict(net, num_neurons=200_000), 5000)
        c = srv.footprint(dict(net, growth_rate=1e-3), 5000)
        d = srv.footprint(net, 5000, initial_axons=300_000.0)
        assert a < b and a < c and a < d
        # linear in the neurons above the constant part
        e = srv.footprint(dict(net, num_neurons=300_000), 5000)
        assert abs((e - b) - (b - a)) <= 2


def test_refuses_request_above_budget(built_lib):
    from relearn_b200 import RelearnError, default_params, workloads
    from relearn_b200.serving import Server

    with Server(default_params(1, 1.0), hbm_budget_bytes=1e8, slots=1) as srv:
        net = dict(num_neurons=200_000, seed=1, side=5848.0, theta=0.3, sigma=750.0, growth_rate=1e-3)
        pos, sig = workloads.request_inputs(net)
        with pytest.raises(RelearnError) as e:
            srv.submit(net, pos, sig, 5000)
        assert e.value.status == 2


def test_failed_run_is_reported(built_lib):
    from conftest import has_gpu

    if has_gpu():
        pytest.skip("a device is present")
    from relearn_b200 import default_params, workloads
    from relearn_b200.serving import Server

    with Server(default_params(1, 1.0), slots=2) as srv:
        net = dict(num_neurons=500, seed=1, side=800.0, theta=0.3, sigma=750.0, growth_rate=1e-4)
        pos, sig = workloads.request_inputs(net)
        rid = srv.submit(net, pos, sig, 10)
        done = []
        for _ in range(100):
            done += srv.poll(wait_ms=100)
            if done:
                break
        assert len(done) == 1 and done[0]["id"] == rid
        assert done[0]["status"] == 3  # RL_ERR_DEVICE: no usable device
        assert srv.load() == (0, 0, 0)
