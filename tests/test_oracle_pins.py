"""Pins of the CPU oracle against the reference's own known-answer and
property tests (read from relearn/test/**, re-expressed here), plus the
published known answers of Philox4x32-10 and AS241."""
import math
from statistics import NormalDist

import numpy as np
import pytest


# ---------------------------------------------------------------- picker
# test/probability_picker/test_probability_picker.cpp:122-143
def test_pick_target_manual(oracle_mod):
    pick = oracle_mod.pick_index
    assert pick([0.0, 2.0, 0.0, 1.421, 1.0], 1.0) == 1
    assert pick([0.0, 2.0, 0.0, 1.421, 1.0], 4.0) == 4
    assert pick([1.0, 0.0, 0.0, 1.0], 1.0) == 0
    assert pick([1.0, 0.0, 0.0, 1.0], math.nextafter(1.0, 2.0)) == 3


# test_probability_picker.cpp:144-199 (zeros in between) and :201-255 (zeros at end)
@pytest.mark.parametrize("zeros_at_end", [False, True])
def test_pick_target_properties(oracle_mod, zeros_at_end):
    rng = np.random.default_rng(11 + zeros_at_end)
    for _ in range(50):
        k = int(rng.integers(1, 100))
        p = rng.uniform(0.0, 3.0, k)
        p[0] += 1e-3
        if not zeros_at_end:
            p[1:][rng.random(k - 1) < 0.5] = 0.0
        else:
            p = np.concatenate([p, np.zeros(int(rng.integers(1, 100)))])
        prefix = np.concatenate([[0.0], np.cumsum(p)[:-1]])
        total = float(np.sum(p))
        for r in rng.uniform(np.nextafter(0.0, 1.0), total, 20):
            idx = oracle_mod.pick_index(p, r)
            expect = int(np.searchsorted(prefix, r, side="left")) - 1
            assert idx == expect and p[idx] > 0.0
        assert oracle_mod.pick_index(p, 0.0) == 0
        assert oracle_mod.pick_index(p, np.finfo(float).tiny) == 0
        last = int(np.nonzero(p > 0)[0][-1])
        for r in rng.uniform(0.0, total, 16) + total:
            assert oracle_mod.pick_index(p, r) == last


# ---------------------------------------------------------------- izhikevich
def _izh_reference(x, u, h, a, b, c, d, vs, k1, k2, k3, inp):
    """The host reference formula of test/neuron_models_gpu/test_neuron_models_gpu.cpp
    (per substep: x += (k1 x^2 + k2 x + k3 - u + I)/h, u += a(b x - u)/h)."""
    for _ in range(h):
        xi = (k1 * x * x) + (k2 * x) + k3 - u + inp
        ui = a * (b * x - u)
        x += xi * (1.0 / h)
        u += ui * (1.0 / h)
        if x >= vs:
            return c, u + d, True
    return x, u, False


# test_neuron_models_gpu.cpp:105-133: a=0.02, b=0.2, c=-65, d=8, h=5, no spike
def test_izhikevich_formula_without_spiking(oracle_mod):
    for x0, u0, inp in [(-65.0, -13.0, 0.0), (-60.0, -12.0, 1.0)]:
        x, u, f = oracle_mod.izhikevich(x0, u0, inp, 5, 0.02, 0.2, -65.0, 8.0)
        ex, eu, ef = _izh_reference(x0, u0, 5, 0.02, 0.2, -65.0, 8.0, 30.0, 0.04, 5.0, 140.0, inp)
        assert not f and not ef
        assert abs(x - ex) <= 1e-12 * max(1.0, abs(ex))
        assert abs(u - eu) <= 1e-12 * max(1.0, abs(eu))


# test_neuron_models_gpu.cpp:135-160: strong drive, h=20, spikes and resets to c
def test_izhikevich_spikes_and_resets(oracle_mod):
    x, u, f = oracle_mod.izhikevich(-65.0, -13.0, 50.0, 20, 0.02, 0.2, -65.0, 8.0)
    assert f and x == -65.0
    ex, eu, ef = _izh_reference(-65.0, -13.0, 20, 0.02, 0.2, -65.0, 8.0, 30.0, 0.04, 5.0, 140.0, 50.0)
    assert ef and abs(u - eu) <= 1e-12 * abs(eu)


# ---------------------------------------------------------------- calcium
# test/calcium_gpu/test_calcium_gpu.cpp:86-140: Euler formula, fired / not fired
@pytest.mark.parametrize("fired", [False, True])
def test_calcium_formula(oracle_mod, fired):
    rng = np.random.default_rng(3)
    for c0 in rng.uniform(0.0, 2.0, 20):
        c = c0
        for _ in range(10):
            c += (1.0 / 10) * (c * (-1.0 / 10000.0) + 0.001 * (1.0 if fired else 0.0))
        assert oracle_mod.calcium(c0, fired, 0.001, 10000.0, 10) == c


# ---------------------------------------------------------------- growth curve
# test/synaptic_elements/test_synaptic_elements.cpp:36-195
def test_growth_curve_intersections_and_peak(oracle_mod):
    rng = np.random.default_rng(5)
    for _ in range(40):
        eta, eps = sorted(rng.uniform(-100.0, 100.0, 2))
        mid = (eta + eps) / 2
        assert abs(oracle_mod.growth_curve(eta, eta, eps)) < 1e-6
        assert abs(oracle_mod.growth_curve(eps, eta, eps)) < 1e-6
        assert abs(oracle_mod.growth_curve(mid, eta, eps) - 1.0) < 1e-6
        xs = np.sort(rng.uniform(-1e5, eta, 20))
        vals = [oracle_mod.growth_curve(v, eta, eps) for v in xs]
        assert all(v <= 0.0 for v in vals) and all(a <= b + 1e-15 for a, b in zip(vals, vals[1:]))
        xs = np.sort(rng.uniform(eta, mid, 20))
        vals = [oracle_mod.growth_curve(v, eta, eps) for v in xs]
        assert all(-1e-12 <= v <= 1.0 + 1e-12 for v in vals) and all(a <= b + 1e-15 for a, b in zip(vals, vals[1:]))


def test_growth_curve_equal_intersections(oracle_mod):
    # GrowthCurves.h:36-42 corner case eta == epsilon
    assert oracle_mod.growth_curve(0.5, 0.5, 0.5) == 0.0
    assert oracle_mod.growth_curve(0.4, 0.5, 0.5) == -1.0
    assert oracle_mod.growth_curve(0.6, 0.5, 0.5) == -1.0


def test_growth_curve_shared_exp_matches_libm(oracle_mod):
    rng = np.random.default_rng(9)
    for c in rng.uniform(0.0, 1.0, 200):
        a = oracle_mod.growth_curve(c, 0.4, 0.7)
        b = oracle_mod.growth_curve(c, 0.4, 0.7, use_libm=True)
        assert abs(a - b) <= 4e-16 * max(1.0, abs(b))


# ---------------------------------------------------------------- commit
# test/element_base/test_element_base.cpp:1068-1350, cases of ElementBaseBase::update
def test_commit_growth_keeps_connected(oracle_mod):
    r = oracle_mod.commit_element(2.5, 0.75, 1, 1)
    assert r["to_delete"] == 0 and r["connected"] == 1
    assert r["grown"] == ((2.5 - 1.0) + 0.75) + 1.0 and r["vacant"] == 2 and r["delta"] == 0.0


def test_commit_shrink_within_vacant(oracle_mod):
    r = oracle_mod.commit_element(3.2, -1.0, 2, 1)
    assert r["to_delete"] == 0 and r["connected"] == 2 and r["vacant"] == 0


def test_commit_delete_bound(oracle_mod):
    r = oracle_mod.commit_element(3.2, -1.5, 3, 0)
    assert r["connected"] == 1 and r["to_delete"] == 2 and r["vacant"] == 0
    assert r["grown"] == (3.2 - 1.5 - math.floor(3.2 - 1.5)) + 1.0


def test_commit_delete_all(oracle_mod):
    r = oracle_mod.commit_element(1.5, -3.0, 1, 0)
    assert r == dict(grown=0.0, delta=0.0, connected=0, vacant=0, to_delete=1)


def test_commit_retract_ratio(oracle_mod):
    r = oracle_mod.commit_element(2.0, 1.0, 0, 2, retract=0.5)
    assert r["grown"] == 0.5 * 3.0 and r["vacant"] == 1


# ---------------------------------------------------------------- random stream
# Random123 known-answer vectors of philox4x32_10
@pytest.mark.parametrize("ctr,key,expect", [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0), (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
])
def test_philox_known_answers(oracle_mod, ctr, key, expect):
    assert tuple(oracle_mod.philox(*ctr, *key)) == expect


def test_normal_quantile_against_python(oracle_mod):
    L = oracle_mod.lib()
    nd = NormalDist()
    rng = np.random.default_rng(1)
    ps = np.concatenate([rng.uniform(1e-12, 1 - 1e-12, 5000), np.exp(rng.uniform(-36, -1, 2000))])
    for p in ps:
        ref = nd.inv_cdf(float(p))
        assert abs(L.orc_quantile(float(p)) - ref) <= 2e-15 * max(1.0, abs(ref))


def test_background_normal_moments(oracle_mod):
    L = oracle_mod.lib()
    z = np.array([L.orc_normal(77, s, i, 5.0, 2.0) for s in range(1, 6) for i in range(4000)])
    assert abs(z.mean() - 5.0) < 0.05 and abs(z.std() - 2.0) < 0.05


def test_own_exp_log_accuracy(oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(2)
    xs = np.concatenate([rng.uniform(-745.0, 709.0, 20000), rng.uniform(-1, 1, 20000)])
    for x in xs:
        a, b = L.orc_exp(float(x)), math.exp(float(x))
        assert a == b or abs(a - b) <= abs(b) * 2.3e-16 or (b < 2.3e-308 and abs(a - b) <= 5e-324)
    for y in np.exp(rng.uniform(-36, 0, 20000)):
        a, b = L.orc_log(float(y)), math.log(float(y))
        assert abs(a - b) <= abs(b) * 4.5e-16 + 1e-300


def test_hypot3_matches_libstdcxx_rule(oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(4)
    for v in rng.uniform(-1e4, 1e4, (2000, 3)):
        x, y, z = (abs(float(t)) for t in v)
        a = max(x, y, z)
        expect = a * math.sqrt((x / a) * (x / a) + (y / a) * (y / a) + (z / a) * (z / a))
        assert L.orc_hypot3(*map(float, v)) == expect
    assert L.orc_hypot3(0.0, 0.0, 0.0) == 0.0


def _model_params(model, **kw):
    from relearn_b200 import default_params

    p = default_params(1, 1.0)
    p["neuron_model"] = model
    p.update(kw)
    return p


def test_aeif_formula(oracle_mod):
    """AEIF update_activity against the formula of the reference's model test
    (test/neuron_models_gpu/test_neuron_models_gpu.cpp:186-254): parameters
    (C 281, g_L 30, E_L -70.6, V_T -50.4, d_T 2, tau_w 144, a 4, b 80.5,
    V_spike -40), h = 10, a resting and a driven neuron."""
    import math

    prm = dict(aeif_C=281.0, aeif_g_L=30.0, aeif_E_L=-70.6, aeif_V_T=-50.4, aeif_d_T=2.0, aeif_tau_w=144.0, aeif_a=4.0, aeif_b=80.5,
               aeif_V_spike=-40.0, h_model=10)
    p = _model_params(3, **prm)
    for x0, w0, inp in ((-70.6, 0.0, 0.0), (-60.0, 5.0, 200.0)):
        x, w, fired = oracle_mod.model_step(p, x0, w0, inp)
        # the test's reference formula, step by step
        ex, ew, ef = x0, w0, False
        for _ in range(10):
            lin = -prm["aeif_g_L"] * (ex - prm["aeif_E_L"])
            expp = prm["aeif_g_L"] * prm["aeif_d_T"] * math.exp((ex - prm["aeif_V_T"]) * (1.0 / prm["aeif_d_T"]))
            xi = (lin + expp - ew + inp) * (1.0 / prm["aeif_C"])
            wi = (prm["aeif_a"] * (ex - prm["aeif_E_L"]) - ew) * (1.0 / prm["aeif_tau_w"])
            ex += xi * 0.1
            ew += wi * 0.1
            if ex >= prm["aeif_V_spike"]:
                ex, ew, ef = prm["aeif_E_L"], ew + prm["aeif_b"], True
                break
        assert fired == ef
        assert abs(x - ex) <= 1e-12 * max(1.0, abs(ex)) and abs(w - ew) <= 1e-12 * max(1.0, abs(ew))


def test_fitzhugh_nagumo_formula(oracle_mod):
    """FitzHugh-Nagumo update_activity of the CPU model
    (models/fitzhughnagumo/FitzHughNagumoModelCPU.cpp: cubic term x^3 / 3, spike
    test after the h substeps) with the parameters and inputs of the reference's
    model test (test_neuron_models_gpu.cpp:256-310; that test's own formula
    writes the cubic coefficient as 1/2, the CPU model uses 1/3)."""
    p = _model_params(2, fhn_a=0.7, fhn_b=0.8, fhn_phi=0.08, h_model=10)
    for x0, w0, inp in ((-1.2, -0.6, 0.0), (0.5, 0.2, 1.5), (1.8, -1.0, 2.0)):
        x, w, fired = oracle_mod.model_step(p, x0, w0, inp)
        ex, ew = x0, w0
        for _ in range(10):
            xi = ex - (ex * ex * ex * (1.0 / 3.0)) - ew + inp
            wi = 0.08 * (ex + 0.7 - 0.8 * ew)
            ex += xi * 0.1
            ew += wi * 0.1
        assert (x, w) == (ex, ew)
        assert fired == (ew > ex - ex * ex * ex * (1.0 / 3.0) and ex > 1.0)


def test_poisson_refractory_and_firing(oracle_mod):
    """Poisson model contract of the reference's tests
    (test_neuron_models_gpu.cpp:316-365): a refractory neuron never fires and
    counts down; a potential far above any threshold in [0, 1) always fires and
    starts the refractory period."""
    p = _model_params(1, poisson_x0=0.0, poisson_tau_x=1000.0, poisson_refractory=5, h_model=1)
    x, r, fired = oracle_mod.model_step(p, 1e6, 3.0, 0.0)
    assert not fired and r == 2.0
    for step in range(1, 50):
        x, r, fired = oracle_mod.model_step(p, 1e6, 0.0, 0.0, step=step, neuron=step)
        assert fired and r == 5.0
    # below every threshold: never fires
    x, r, fired = oracle_mod.model_step(p, -1.0, 0.0, 0.0)
    assert not fired and r == 0.0
