"""ORACLE — test infrastructure only.

ctypes front end of the CPU restatement in ``rl_oracle.cpp``.  Only the
tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librl_oracle.so")
SOURCES = [os.path.join(HERE, "rl_oracle.cpp"), os.path.join(HERE, "shared_stream.h")]


def build(force: bool = False) -> str:
    """Compile the oracle with g++ (no FMA contraction, OpenMP)."""
    stale = not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in SOURCES)
    if force or stale:
        cmd = ["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-mfma", "-fopenmp", "-fPIC", "-shared", "-o", LIB_PATH, SOURCES[0]]
        subprocess.run(cmd, check=True)
    return LIB_PATH


class OrcConfig(C.Structure):
    _fields_ = [
        ("num_neurons", C.c_uint32),
        ("plasticity_interval", C.c_uint32),
        ("h_model", C.c_uint32),
        ("h_calcium", C.c_uint32),
        ("seed", C.c_uint64),
        ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3),
        ("theta", C.c_double),
        ("sigma", C.c_double),
        ("mu", C.c_double),
        ("iz_a", C.c_double),
        ("iz_b", C.c_double),
        ("iz_c", C.c_double),
        ("iz_d", C.c_double),
        ("iz_v_spike", C.c_double),
        ("iz_k1", C.c_double),
        ("iz_k2", C.c_double),
        ("iz_k3", C.c_double),
        ("beta", C.c_double),
        ("tau_c", C.c_double),
        ("target_calcium", C.c_double),
        ("initial_calcium", C.c_double),
        ("growth_rate", C.c_double * 3),
        ("min_calcium", C.c_double * 3),
        ("retract_ratio", C.c_double * 3),
        ("conductance", C.c_double),
        ("noise_mean", C.c_double),
        ("noise_stddev", C.c_double),
        ("use_libm", C.c_int32),
        ("kernel_type", C.c_int32),
        ("kernel_k", C.c_double),
        ("kernel_scale", C.c_double),
        ("linear_cutoff", C.c_double),
        ("neuron_model", C.c_int32),
        ("poisson_refractory", C.c_uint32),
        ("poisson_x0", C.c_double),
        ("poisson_tau_x", C.c_double),
        ("fhn_a", C.c_double),
        ("fhn_b", C.c_double),
        ("fhn_phi", C.c_double),
        ("fhn_init_x", C.c_double),
        ("fhn_init_w", C.c_double),
        ("aeif_C", C.c_double),
        ("aeif_g_L", C.c_double),
        ("aeif_E_L", C.c_double),
        ("aeif_V_T", C.c_double),
        ("aeif_d_T", C.c_double),
        ("aeif_tau_w", C.c_double),
        ("aeif_a", C.c_double),
        ("aeif_b", C.c_double),
        ("aeif_V_spike", C.c_double),
    ]


class OrcRequest(C.Structure):
    _fields_ = [("target", C.c_uint32), ("source", C.c_uint32), ("j", C.c_uint32), ("signal", C.c_uint32)]


REQ_DTYPE = np.dtype([("target", "<u4"), ("source", "<u4"), ("j", "<u4"), ("signal", "<u4")])

_lib = None


def lib():
    global _lib
    if _lib is None:
        _lib = C.CDLL(build())
        L = _lib
        vp, u32, u64, i32, dbl = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_double
        P = C.POINTER
        L.orc_create.restype = vp
        L.orc_create.argtypes = [P(OrcConfig), vp, vp, C.c_int]
        L.orc_error.argtypes = [vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [vp, C.c_int]
        L.orc_num_nodes.restype = u64
        L.orc_num_nodes.argtypes = [vp]
        L.orc_dump_tree.argtypes = [vp] + [vp] * 10
        L.orc_set_elements.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        L.orc_get_elements.argtypes = [vp, C.c_int, vp, vp, vp, vp]
        L.orc_set_enabled.argtypes = [vp, vp]
        L.orc_update_tree.argtypes = [vp, vp, vp]
        L.orc_find_targets.restype = u64
        L.orc_find_targets.argtypes = [vp, u32, vp, u64]
        L.orc_connect.restype = u64
        L.orc_connect.argtypes = [vp, u32, vp]
        L.orc_simulate.argtypes = [vp, u32, u32]
        L.orc_activity_step.argtypes = [vp, u32]
        L.orc_plasticity_step.argtypes = [vp, u32]
        L.orc_get_neurons.argtypes = [vp] * 6
        L.orc_set_neurons.argtypes = [vp] * 5
        L.orc_set_targets.argtypes = [vp, vp]
        L.orc_model_step.restype = C.c_int
        L.orc_model_step.argtypes = [P(OrcConfig), P(dbl), P(dbl), dbl, u32, u32]
        L.orc_kernel_prob.restype = C.c_double
        L.orc_kernel_prob.argtypes = [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double]
        L.orc_num_edges.restype = u64
        L.orc_num_edges.argtypes = [vp]
        L.orc_get_edges.argtypes = [vp, vp, vp, vp]
        L.orc_add_edges.argtypes = [vp, u64, vp, vp, vp]
        L.orc_stats.argtypes = [vp, vp]
        L.orc_pick_index.restype = C.c_long
        L.orc_pick_index.argtypes = [vp, C.c_long, dbl]
        L.orc_izhikevich.restype = C.c_int
        L.orc_izhikevich.argtypes = [P(dbl), P(dbl), dbl, u32] + [dbl] * 8
        L.orc_growth_curve.restype = dbl
        L.orc_growth_curve.argtypes = [dbl, dbl, dbl, C.c_int]
        L.orc_calcium.restype = dbl
        L.orc_calcium.argtypes = [dbl, C.c_int, dbl, dbl, u32]
        L.orc_commit_element.restype = u32
        L.orc_commit_element.argtypes = [P(dbl), P(dbl), P(u32), P(u32), dbl]
        for name in ("orc_exp", "orc_log", "orc_quantile"):
            getattr(L, name).restype = dbl
            getattr(L, name).argtypes = [dbl]
        L.orc_hypot3.restype = dbl
        L.orc_hypot3.argtypes = [dbl, dbl, dbl]
        L.orc_normal.restype = dbl
        L.orc_normal.argtypes = [u64, u32, u32, dbl, dbl]
        L.orc_philox.argtypes = [u32] * 6 + [vp]
        L.orc_connect_requests.restype = u64
        L.orc_connect_requests.argtypes = [vp, u32, vp, u64, vp]
        L.orc_process_requests.restype = u64
        L.orc_process_requests.argtypes = [vp, u32, vp, u64, vp]
        L.orc_process_responses.restype = C.c_int
        L.orc_process_responses.argtypes = [vp, vp, vp, vp, u64]
        L.orc_octant_of.restype = C.c_int
        L.orc_octant_of.argtypes = [vp, vp, vp]
        L.orc_box_for_octant.argtypes = [vp, vp, C.c_int, vp, vp]
        L.orc_acceptance.restype = C.c_int
        L.orc_acceptance.argtypes = [C.c_int, vp, vp, u32, vp, vp, dbl]
        L.orc_nodes_to_consider.restype = u64
        L.orc_nodes_to_consider.argtypes = [vp, vp, C.c_int, vp, u64]
        L.orc_find_target.restype = C.c_int64
        L.orc_find_target.argtypes = [vp, u32, vp, C.c_int, u32, u32]
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def make_config(params: dict) -> OrcConfig:
    cfg = OrcConfig()
    for key, val in params.items():
        if key in ("box_min", "box_max", "growth_rate", "min_calcium", "retract_ratio"):
            getattr(cfg, key)[:] = list(val)
        elif hasattr(cfg, key):
            setattr(cfg, key, val)
    return cfg


class OracleSim:
    """One network on the CPU oracle."""

    def __init__(self, params: dict, positions: np.ndarray, signal: np.ndarray, threads: int = 1):
        self.params = dict(params)
        self.n = int(params["num_neurons"])
        self._pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(self.n, 3)
        self._sig = np.ascontiguousarray(signal, dtype=np.uint8)
        self.cfg = make_config(params)
        self.h = lib().orc_create(C.byref(self.cfg), _p(self._pos), _p(self._sig), threads)
        err = lib().orc_error(self.h)
        if err:
            raise RuntimeError(f"oracle octree construction failed (code {err})")

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_threads(self, t: int):
        lib().orc_set_threads(self.h, t)

    def tree(self) -> dict:
        m = int(lib().orc_num_nodes(self.h))
        out = dict(
            level=np.zeros(m, np.int32), neuron=np.zeros(m, np.int32), child_mask=np.zeros(m, np.uint8),
            first_child=np.zeros(m, np.int32), bmin=np.zeros((m, 3)), bmax=np.zeros((m, 3)),
            cnt_exc=np.zeros(m, np.uint32), cnt_inh=np.zeros(m, np.uint32), pos_exc=np.zeros((m, 3)), pos_inh=np.zeros((m, 3)),
        )
        keys = ["level", "neuron", "child_mask", "first_child", "bmin", "bmax", "cnt_exc", "cnt_inh", "pos_exc", "pos_inh"]
        lib().orc_dump_tree(self.h, *[_p(out[k]) for k in keys])
        return out

    def set_elements(self, etype: int, grown, delta, connected, vacant):
        a = [np.ascontiguousarray(v, dt) for v, dt in zip((grown, delta, connected, vacant), (np.float64, np.float64, np.uint32, np.uint32))]
        lib().orc_set_elements(self.h, etype, *[_p(x) for x in a])

    def get_elements(self, etype: int):
        g = np.zeros(self.n); d = np.zeros(self.n)
        c = np.zeros(self.n, np.uint32); v = np.zeros(self.n, np.uint32)
        lib().orc_get_elements(self.h, etype, _p(g), _p(d), _p(c), _p(v))
        return dict(grown=g, delta=d, connected=c, vacant=v)

    def update_tree(self, vac_exc, vac_inh):
        e = np.ascontiguousarray(vac_exc, np.uint32); i = np.ascontiguousarray(vac_inh, np.uint32)
        lib().orc_update_tree(self.h, _p(e), _p(i))

    def find_targets(self, step: int) -> np.ndarray:
        cap = int(self.get_elements(0)["vacant"].astype(np.uint64).sum())
        out = np.zeros(max(cap, 1), REQ_DTYPE)
        m = int(lib().orc_find_targets(self.h, step, _p(out), cap))
        return out[:m].copy()

    def connect(self, step: int, m: int):
        acc = np.zeros(max(m, 1), np.uint8)
        created = int(lib().orc_connect(self.h, step, _p(acc)))
        return created, acc[:m].copy()

    def connect_requests(self, step: int, requests: np.ndarray):
        """Connector over a given request list (REQ_DTYPE): returns the
        number created and one accepted flag per request."""
        req = np.ascontiguousarray(requests, REQ_DTYPE)
        acc = np.zeros(max(len(req), 1), np.uint8)
        created = int(lib().orc_connect_requests(self.h, step, _p(req), len(req), _p(acc)))
        return created, acc[: len(req)].copy()

    def process_requests(self, step: int, requests: np.ndarray):
        """The target half of the connector (ForwardConnector::process_requests):
        returns the number created and one accepted flag per request."""
        req = np.ascontiguousarray(requests, REQ_DTYPE)
        acc = np.zeros(max(len(req), 1), np.uint8)
        created = int(lib().orc_process_requests(self.h, step, _p(req), len(req), _p(acc)))
        return created, acc[: len(req)].copy()

    def process_responses(self, requests: np.ndarray, accepted: np.ndarray, append=None) -> int:
        """The axon half (ForwardConnector::process_responses); synapses flagged
        in `append` join the synapse list.  Returns the number of axons bound."""
        req = np.ascontiguousarray(requests, REQ_DTYPE)
        acc = np.ascontiguousarray(accepted, np.uint8)
        app = None if append is None else np.ascontiguousarray(append, np.uint8)
        if lib().orc_process_responses(self.h, _p(req), _p(acc), None if app is None else _p(app), len(req)) != 0:
            raise RuntimeError("process_responses: a source has no vacant axon")
        return int(acc.astype(np.int64).sum())

    def nodes_to_consider(self, position, dendrite_type: int) -> np.ndarray:
        """Candidates of a walk from the root for a source at `position`, as
        breadth-first node indices (those of tree()), in visiting order."""
        p = np.ascontiguousarray(position, np.float64)
        cap = int(lib().orc_num_nodes(self.h))
        out = np.zeros(max(cap, 1), np.int32)
        k = int(lib().orc_nodes_to_consider(self.h, _p(p), dendrite_type, _p(out), cap))
        return out[:k].copy()

    def find_target(self, source: int, position, dendrite_type: int, step: int, j: int = 0) -> int:
        p = np.ascontiguousarray(position, np.float64)
        return int(lib().orc_find_target(self.h, source, _p(p), dendrite_type, step, j))

    def simulate(self, first_step: int, count: int):
        lib().orc_simulate(self.h, first_step, count)

    def activity_step(self, step: int):
        lib().orc_activity_step(self.h, step)

    def plasticity_step(self, step: int):
        lib().orc_plasticity_step(self.h, step)

    def neurons(self) -> dict:
        n = self.n
        x = np.zeros(n); u = np.zeros(n); ca = np.zeros(n); f = np.zeros(n, np.uint8); inp = np.zeros(n)
        lib().orc_get_neurons(self.h, _p(x), _p(u), _p(ca), _p(f), _p(inp))
        return dict(x=x, u=u, calcium=ca, fired=f, input=inp)

    def set_neurons(self, x=None, u=None, calcium=None, fired=None):
        arrs = []
        for v, dt in ((x, np.float64), (u, np.float64), (calcium, np.float64), (fired, np.uint8)):
            arrs.append(None if v is None else np.ascontiguousarray(v, dt))
        lib().orc_set_neurons(self.h, *[None if a is None else _p(a) for a in arrs])

    def set_targets(self, target):
        t = np.ascontiguousarray(target, np.float64)
        lib().orc_set_targets(self.h, _p(t))

    def edges(self):
        m = int(lib().orc_num_edges(self.h))
        t = np.zeros(m, np.uint32); s = np.zeros(m, np.uint32); w = np.zeros(m, np.int32)
        if m:
            lib().orc_get_edges(self.h, _p(t), _p(s), _p(w))
        return t, s, w

    def add_edges(self, target, source, weight):
        t = np.ascontiguousarray(target, np.uint32); s = np.ascontiguousarray(source, np.uint32)
        w = np.ascontiguousarray(weight, np.int32)
        lib().orc_add_edges(self.h, len(t), _p(t), _p(s), _p(w))

    def stats(self) -> dict:
        out = np.zeros(6, np.uint64)
        lib().orc_stats(self.h, _p(out))
        return dict(created=int(out[0]), to_delete=int(out[1]), searches=int(out[2]), nodes_touched=int(out[3]), descents=int(out[4]),
                    deleted=int(out[5]))


# ---- element-level helpers for the known-answer tests -------------------

def pick_index(values, r: float) -> int:
    v = np.ascontiguousarray(values, np.float64)
    return int(lib().orc_pick_index(_p(v), len(v), float(r)))


def izhikevich(x: float, u: float, inp: float, h: int, a, b, c, d, v_spike=30.0, k1=0.04, k2=5.0, k3=140.0):
    xc = C.c_double(x); uc = C.c_double(u)
    f = lib().orc_izhikevich(C.byref(xc), C.byref(uc), inp, h, a, b, c, d, v_spike, k1, k2, k3)
    return xc.value, uc.value, bool(f)


def growth_curve(current: float, eta: float, epsilon: float, use_libm: bool = False) -> float:
    return float(lib().orc_growth_curve(current, eta, epsilon, int(use_libm)))


def model_step(params: dict, x: float, u: float, inp: float, step: int = 1, neuron: int = 0):
    """One update_activity of the configured neuron model for one neuron:
    returns (x, u, fired)."""
    cfg = make_config(params)
    xc, uc = C.c_double(x), C.c_double(u)
    f = lib().orc_model_step(C.byref(cfg), C.byref(xc), C.byref(uc), inp, step, neuron)
    return xc.value, uc.value, bool(f)


def calcium(c: float, fired: bool, beta: float, tau: float, h: int) -> float:
    return float(lib().orc_calcium(c, int(fired), beta, tau, h))


def commit_element(grown, delta, connected, vacant, retract=0.0):
    g = C.c_double(grown); d = C.c_double(delta); c = C.c_uint32(connected); v = C.c_uint32(vacant)
    dele = lib().orc_commit_element(C.byref(g), C.byref(d), C.byref(c), C.byref(v), retract)
    return dict(grown=g.value, delta=d.value, connected=c.value, vacant=v.value, to_delete=int(dele))


def philox(c0, c1, c2, c3, k0, k1):
    out = np.zeros(4, np.uint32)
    lib().orc_philox(c0, c1, c2, c3, k0, k1, _p(out))
    return [int(v) for v in out]


def octant_of(bmin, bmax, position) -> int:
    """Cell::get_octant_for_position of one box; -1 outside the box."""
    a, b, p = (np.ascontiguousarray(v, np.float64) for v in (bmin, bmax, position))
    return int(lib().orc_octant_of(_p(a), _p(b), _p(p)))


def box_for_octant(bmin, bmax, octant: int):
    """Cell::get_size_for_octant of one box: (lo, hi)."""
    a, b = (np.ascontiguousarray(v, np.float64) for v in (bmin, bmax))
    lo = np.zeros(3)
    hi = np.zeros(3)
    lib().orc_box_for_octant(_p(a), _p(b), int(octant), _p(lo), _p(hi))
    return lo, hi


DISCARD, EXPAND, ACCEPT = 0, 1, 2


def acceptance(parent: bool, bmin, bmax, count: int, dendrite_position, source_position, theta: float) -> int:
    """BarnesHutBase::test_acceptance_criterion of one node: DISCARD, EXPAND,
    ACCEPT, or -1 for a theta outside (0, 0.5]."""
    a, b, d, s = (np.ascontiguousarray(v, np.float64) for v in (bmin, bmax, dendrite_position, source_position))
    return int(lib().orc_acceptance(int(parent), _p(a), _p(b), int(count), _p(d), _p(s), float(theta)))
