"""CPU checks of the C-ABI boundary and of the host-side code: the library
loads and exports every entry point declared in include/relearn_b200.h, the
ctypes mirror matches the C struct layout, and the product's shared arithmetic
header agrees bit for bit with the oracle's statement of it."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "relearn_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"RL_API\s+[\w\s\*]+?\b(rl_\w+)\s*\(", text)))


def test_header_and_mirror_agree():
    import relearn_b200

    assert declared_functions() == sorted(relearn_b200.ABI_FUNCTIONS)


def test_library_exports_every_declared_symbol(built_lib):
    out = subprocess.run(["nm", "-D", "--defined-only", built_lib], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(rl_\w+)", out))
    missing = [f for f in declared_functions() if f not in exported]
    assert not missing, missing
    lib = C.CDLL(built_lib)
    for f in declared_functions():
        assert hasattr(lib, f)


def test_struct_layout(tmp_path):
    import relearn_b200 as R

    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), os.path.join(ROOT, "tests", "helpers", "abi_layout.c")], check=True)
    lines = dict(l.rsplit(" ", 1) for l in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n") if l)
    assert int(lines["rl_config"]) == C.sizeof(R.RlConfig)
    assert int(lines["rl_stats"]) == C.sizeof(R.RlStats)
    assert int(lines["rl_request"]) == R.REQUEST_DTYPE.itemsize
    assert int(lines["rl_synapse"]) == R.SYNAPSE_DTYPE.itemsize
    for f in ("seed", "box_min", "theta", "growth_rate", "conductance", "device", "precision", "kernel_type", "kernel_k", "kernel_scale",
              "linear_cutoff"):
        assert int(lines[f"rl_config.{f}"]) == getattr(R.RlConfig, f).offset
    assert int(lines["rl_stats.max_level"]) == R.RlStats.max_level.offset
    assert int(lines["rl_stats.nodes_touched"]) == R.RlStats.nodes_touched.offset
    assert int(lines["RL_NUM_SEARCH_SHAPES"]) == R.NUM_SEARCH_SHAPES == len(R.SEARCH_SHAPES)
    assert int(lines["RL_NUM_ACT_SHAPES"]) == R.NUM_ACT_SHAPES == len(R.ACT_SHAPES)
    for name, cls in (("rl_tuning", R.RlTuning), ("rl_network", R.RlNetwork), ("rl_serve_config", R.RlServeConfig), ("rl_serve_request", R.RlServeRequest),
                      ("rl_serve_done", R.RlServeDone)):
        assert int(lines[name]) == C.sizeof(cls), name
    assert int(lines["rl_network.growth_rate"]) == R.RlNetwork.growth_rate.offset
    for f in ("slots", "use_graphs"):
        assert int(lines[f"rl_serve_config.{f}"]) == getattr(R.RlServeConfig, f).offset
    for f in ("xyz", "grown", "steps", "keep_state"):
        assert int(lines[f"rl_serve_request.{f}"]) == getattr(R.RlServeRequest, f).offset
    for f in ("t_submit", "num_synapses", "neuron_steps"):
        assert int(lines[f"rl_serve_done.{f}"]) == getattr(R.RlServeDone, f).offset


def test_host_only_entry_points(built_lib):
    import relearn_b200 as R

    L = R.load_library()
    assert L.rl_abi_version() == 4
    cfg = R.RlConfig()
    L.rl_config_default(C.byref(cfg), 2000, 1000.0)
    # reference defaults: Parameters.h:123-130, CalciumCalculatorBase.h:206-210, Gaussian.h:38-39
    assert (cfg.iz_a, cfg.iz_b, cfg.iz_c, cfg.iz_d) == (0.1, 0.2, -65.0, 2.0)
    assert (cfg.beta, cfg.tau_c, cfg.target_calcium, cfg.h_calcium) == (0.001, 10000.0, 0.7, 10)
    assert (cfg.sigma, cfg.mu, cfg.theta, cfg.plasticity_interval) == (750.0, 0.0, 0.3, 100)
    assert L.rl_status_string(1) == b"invalid argument or state"


def test_create_without_device_fails_cleanly(built_lib):
    from conftest import has_gpu

    if has_gpu():
        pytest.skip("a device is present")
    import relearn_b200 as R

    with pytest.raises(R.RelearnError) as e:
        R.Network(R.default_params(10, 100.0))
    assert e.value.status == 3  # RL_ERR_DEVICE


def test_invalid_config_is_rejected(built_lib):
    import relearn_b200 as R

    p = R.default_params(10, 100.0)
    p["theta"] = 0.7  # above Constants::bh_max_theta
    with pytest.raises(R.RelearnError) as e:
        R.Network(p)
    assert e.value.status in (1, 3)


@pytest.fixture(scope="module")
def probe(tmp_path_factory):
    so = tmp_path_factory.mktemp("probe") / "probe.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-ffp-contract=off", "-fPIC", "-shared", "-o", str(so),
                    os.path.join(ROOT, "tests", "helpers", "math_probe.cpp")], check=True)
    L = C.CDLL(str(so))
    for name in ("probe_exp", "probe_exp_flat", "probe_exp_flat_nonpos", "probe_log", "probe_quantile", "probe_next_up"):
        getattr(L, name).restype = C.c_double
        getattr(L, name).argtypes = [C.c_double]
    for name in ("probe_hypot3", "probe_std_hypot3"):
        getattr(L, name).restype = C.c_double
        getattr(L, name).argtypes = [C.c_double] * 3
    L.probe_kernel_prob.restype = C.c_double
    L.probe_kernel_prob.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_int]
    L.probe_normal.restype = C.c_double
    L.probe_normal.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_double, C.c_double]
    L.probe_philox.argtypes = [C.c_uint32] * 6 + [C.c_void_p]
    L.probe_hypot_sweep.restype = C.c_long
    L.probe_hypot_sweep.argtypes = [C.c_long, C.c_ulonglong]
    return L


def test_shared_math_bitwise_agreement(probe, oracle_mod):
    O = oracle_mod.lib()
    rng = np.random.default_rng(8)
    for x in np.concatenate([rng.uniform(-746, 710, 30000), rng.uniform(-2, 2, 10000), [-745.0, -740.0, 0.0, 709.7]]):
        assert probe.probe_exp(float(x)) == O.orc_exp(float(x)) or (np.isnan(probe.probe_exp(float(x))))
    for y in np.exp(rng.uniform(-37, 0, 20000)):
        assert probe.probe_log(float(y)) == O.orc_log(float(y))
    for p in rng.uniform(0, 1, 20000):
        assert probe.probe_quantile(float(p)) == O.orc_quantile(float(p))
    vs = rng.uniform(-1e4, 1e4, (5000, 3))
    ties = rng.choice([-3.5, 0.0, 2.0, 7.25, 1e-300], (600, 3))  # equal magnitudes, zeros, tiny values
    for v in np.concatenate([vs, ties]):
        h = probe.probe_hypot3(*map(float, v))
        # the restatement, the oracle's and libstdc++'s std::hypot(x, y, z) agree bit for bit
        assert h == O.orc_hypot3(*map(float, v)) == probe.probe_std_hypot3(*map(float, v)), v
    for s in range(1, 4):
        for i in range(2000):
            assert probe.probe_normal(42, s, i, 5.0, 2.0) == O.orc_normal(42, s, i, 5.0, 2.0)
    out = np.zeros(4, np.uint32)
    for c in rng.integers(0, 2**32, (500, 6), dtype=np.uint64):
        probe.probe_philox(*map(int, c), out.ctypes.data_as(C.c_void_p))
        assert list(out) == oracle_mod.philox(*map(int, c))
    for t in rng.uniform(1e-3, 1e6, 1000):
        assert probe.probe_next_up(float(t)) == np.nextafter(float(t), float(t) + 1e-5)


def test_hypot_from_one_reciprocal_equals_std_hypot(probe):
    """rl_hypot3 divides the two smaller components by the largest through one
    correctly rounded reciprocal (Markstein's correction); libstdc++'s
    std::hypot divides twice.  Four million vectors of many magnitudes give the
    same bits."""
    assert probe.probe_hypot_sweep(4_000_000, 17) == 0


def test_branch_free_exp_equals_exp(probe):
    """rl_exp_flat (the form the block activity kernel interleaves) gives
    rl_exp's bits for every argument: across the range, at the overflow and
    underflow edges, in the subnormal results, and for infinities and NaN."""
    rng = np.random.default_rng(12)
    xs = np.concatenate([rng.uniform(-750, 712, 30000), rng.uniform(-40, 0, 20000), rng.uniform(-745.2, -707.0, 10000),
                         rng.uniform(709.0, 709.8, 5000), [709.782712893384, 709.7827128933841, 709.78271289338397, -745.1332191019412,
                         -745.1332191019411, -708.3964185322641, -708.39641853226, 0.0, -0.0, 1e-300, -1e-300, 710.0, -746.0, 1e308,
                         -1e308, float("inf"), float("-inf")]])
    for x in xs:
        a, b = probe.probe_exp(float(x)), probe.probe_exp_flat(float(x))
        assert np.float64(a).view(np.uint64) == np.float64(b).view(np.uint64), (x, a, b)
    assert np.isnan(probe.probe_exp_flat(float("nan")))
    # the form for arguments <= 0 (the growth curves' exp(-q^2))
    for x in xs[xs <= 0]:
        a, b = probe.probe_exp(float(x)), probe.probe_exp_flat_nonpos(float(x))
        assert np.float64(a).view(np.uint64) == np.float64(b).view(np.uint64), (x, a, b)
    assert np.isnan(probe.probe_exp_flat_nonpos(float("nan")))


@pytest.mark.parametrize("kernel", [(1, 2.0, 400.0, 0.0), (1, 1.0, 300.0, 0.0), (2, 1.0, 1.0, 1500.0), (2, 1.0, 1.0, float("inf")),
                                    (3, 1.5, 0.002, 0.0), (3, 1.0, 0.001, 0.0), (0, 1.0, 1.0, 0.0)])
def test_kernel_probability_agrees_with_oracle(probe, oracle_mod, kernel):
    """The shared kernel formula (product) and the oracle's restatement of the
    reference's kernels give the same bits for every kernel type."""
    import math

    kt, k, sc, cut = kernel
    O = oracle_mod.lib()
    a = b = 0.0
    if kt == 1:
        a = 1.0 / (math.gamma(k) * sc**k)
        b = -1.0 / sc
    elif kt == 3:
        a = sc * k
        b = sc
    sigma = 750.0
    rng = np.random.default_rng(kt)
    for d in np.concatenate([rng.uniform(0.5, 4000.0, 3000), [1.0, 1499.99, 1500.0, 1500.01]]):
        mine = probe.probe_kernel_prob(kt, float(d), 0.0, -1.0 / (sigma * sigma), k - 1.0, a, b, cut, 1 if math.isinf(cut) else 0)
        ref = O.orc_kernel_prob(kt, float(d), 0.0, sigma, k, sc, cut)
        assert mine == ref, (kernel, d, mine, ref)
