"""relearn_b200 — B200-native structural-plasticity hot path.

Host-side mirror of RELeARN's plugin surface for the path this package
accelerates (paths relative to ``relearn/source`` of tuda-hpclab/relearn):

* :class:`BarnesHut` — the ``Algorithm`` plugin selected by
  ``--algorithm barnes-hut`` (``algorithm/Algorithm.h:48-197``):
  ``init``, ``prepare_update_connectivity``, ``update_connectivity``.
* :class:`IzhikevichModel` — the ``NeuronModel`` plugin selected by
  ``--neuron-model izhikevich`` together with the calcium and synaptic-element
  updates that ``Neurons`` drives every step (``neurons/Neurons.cpp:351-384``).
* :class:`Simulation` — ``Simulation::simulate`` (``sim/Simulation.cpp:388-480``).

Everything runs in ``librelearn_b200.so`` (hand-written sm_100a kernels behind
a C ABI, ``include/relearn_b200.h``).  There is no CPU fallback: importing
the package fails when the library is missing.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "librelearn_b200.so")

ALGORITHMS = {"barnes-hut": "BarnesHut"}
NEURON_MODELS = {"izhikevich": 0, "poisson": 1, "fitzhughnagumo": 2, "aeif": 3}

RL_OK = 0
STATUS_NAMES = {0: "RL_OK", 1: "RL_ERR_INVALID", 2: "RL_ERR_OOM", 3: "RL_ERR_DEVICE", 4: "RL_ERR_TIMEOUT", 5: "RL_ERR_OVERFLOW",
                6: "RL_ERR_UNSUPPORTED"}
AXON, DENDRITE_EXC, DENDRITE_INH = 0, 1, 2
EXCITATORY, INHIBITORY = 0, 1


class RelearnError(RuntimeError):
    """Raised for every non-OK status (the reference throws RelearnException)."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class RlConfig(C.Structure):
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
        ("device", C.c_int32),
        ("precision", C.c_int32),
        ("kernel_type", C.c_int32),
        ("reserved", C.c_int32),
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


PRECISION_FP64, PRECISION_FP32 = 0, 1
KERNEL_GAUSSIAN, KERNEL_GAMMA, KERNEL_LINEAR, KERNEL_WEIBULL = 0, 1, 2, 3
MODEL_IZHIKEVICH, MODEL_POISSON, MODEL_FITZHUGH_NAGUMO, MODEL_AEIF = 0, 1, 2, 3
KERNELS = {"gaussian": KERNEL_GAUSSIAN, "gamma": KERNEL_GAMMA, "linear": KERNEL_LINEAR, "weibull": KERNEL_WEIBULL}


class RlNetwork(C.Structure):
    _fields_ = [
        ("num_neurons", C.c_uint32),
        ("reserved", C.c_uint32),
        ("seed", C.c_uint64),
        ("box_min", C.c_double * 3),
        ("box_max", C.c_double * 3),
        ("theta", C.c_double),
        ("sigma", C.c_double),
        ("growth_rate", C.c_double * 3),
    ]


class RlStats(C.Structure):
    _fields_ = [(k, C.c_uint64) for k in ("searches", "requests", "synapses_created", "bound_to_delete", "synapses_deleted", "activity_steps",
                                           "plasticity_updates", "gpu_launches", "num_nodes")] + [("max_level", C.c_uint32),
                                                                                                  ("reserved", C.c_uint32),
                                                                                                  ("nodes_touched", C.c_uint64)]


class RlTuning(C.Structure):
    _fields_ = [(k, C.c_int32) for k in ("search_warps", "search_hot", "search_packet", "search_cap", "act_block", "act_persistent", "act_vec",
                                         "tuned")]


NUM_SEARCH_SHAPES, NUM_ACT_SHAPES = 29, 18
# (warps, packet, cap, hot), timing order: plain shapes, then the persistent form
# with the top octree nodes in shared memory
SEARCH_SHAPES = ([(w, p, c, 0) for c in (0, 1) for p in (32, 16, 4, 1) for w in (2, 4, 8)] + [(32, p, 1, h) for h in (1024, 4096) for p in (32, 16)]
                 + [(4, 0, 0, 0)])  # packet 0: one search per warp
ACT_SHAPES = [(b, p, v) for p in (0, 1) for b in (128, 256, 512) for v in (1, 2, 4)]  # (block, persistent, neurons per thread)


class RlServeConfig(C.Structure):
    _fields_ = [("hbm_budget_bytes", C.c_uint64), ("pack_max_neurons", C.c_uint64), ("slots", C.c_int32), ("pack_networks", C.c_int32),
                ("use_graphs", C.c_int32), ("autotune", C.c_int32)]


class RlServeRequest(C.Structure):
    _fields_ = [("net", RlNetwork), ("xyz", C.c_void_p), ("signal", C.c_void_p), ("grown", C.c_void_p * 3), ("steps", C.c_uint32),
                ("keep_state", C.c_uint32)]


class RlServeDone(C.Structure):
    _fields_ = [("id", C.c_uint64), ("status", C.c_int32), ("pack_size", C.c_uint32), ("t_submit", C.c_double), ("t_admit", C.c_double),
                ("t_finish", C.c_double), ("num_neurons", C.c_uint64), ("num_synapses", C.c_uint64), ("footprint_bytes", C.c_uint64),
                ("device_peak_bytes", C.c_uint64), ("neuron_steps", C.c_uint64)]


REQUEST_DTYPE = np.dtype([("target", "<u4"), ("source", "<u4"), ("j", "<u4"), ("signal", "<u4")])
SYNAPSE_DTYPE = np.dtype([("target", "<u4"), ("source", "<u4"), ("weight", "<i4"), ("reserved", "<u4")])

# Every entry point declared in include/relearn_b200.h.
ABI_FUNCTIONS = [
    "rl_config_default", "rl_ctx_create", "rl_ensemble_create", "rl_ctx_destroy", "rl_last_error", "rl_status_string", "rl_abi_version",
    "rl_set_positions", "rl_tree_info", "rl_dump_tree", "rl_prepare_update_connectivity", "rl_find_targets",
    "rl_update_connectivity", "rl_connect", "rl_process_requests", "rl_process_responses", "rl_set_elements", "rl_get_elements", "rl_set_neurons", "rl_get_neurons", "rl_set_enabled",
    "rl_add_edges", "rl_get_edges", "rl_activity_block", "rl_plasticity_update", "rl_simulate", "rl_synchronize",
    "rl_get_stats", "rl_set_stream", "rl_set_profiling", "rl_get_phase_times", "rl_prepare_update_connectivity_noalloc",
    "rl_candidate_weights", "rl_set_graphs", "rl_set_step_fusion", "rl_ctx_memory", "rl_serve_footprint", "rl_serve_create", "rl_serve_submit", "rl_serve_poll",
    "rl_serve_fetch", "rl_serve_load", "rl_serve_destroy", "rl_autotune", "rl_get_tuning", "rl_set_tuning",
    "rl_set_target_calcium", "rl_get_target_calcium", "rl_snapshot_neurons", "rl_snapshot_wait",
]
PHASES = ["activity_kernel", "commit", "tree_update", "search_kernel", "search", "connector", "graph"]

_lib = None


def load_library(path: str = LIB_PATH):
    """Load librelearn_b200.so and declare its signatures; raises if missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(f"librelearn_b200.so not built ({path}); run relearn_b200/build.py")
    L = C.CDLL(path)
    vp, u32, u64, i32, dbl = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32, C.c_double
    P = C.POINTER
    st = C.c_int
    L.rl_config_default.restype = None
    L.rl_config_default.argtypes = [P(RlConfig), u32, dbl]
    L.rl_ctx_create.restype = st
    L.rl_ctx_create.argtypes = [P(RlConfig), P(vp)]
    L.rl_ensemble_create.restype = st
    L.rl_ensemble_create.argtypes = [P(RlConfig), P(RlNetwork), u32, P(vp)]
    L.rl_ctx_destroy.restype = st
    L.rl_ctx_destroy.argtypes = [vp]
    L.rl_last_error.restype = C.c_char_p
    L.rl_last_error.argtypes = [vp]
    L.rl_status_string.restype = C.c_char_p
    L.rl_status_string.argtypes = [st]
    L.rl_abi_version.restype = i32
    L.rl_abi_version.argtypes = []
    L.rl_set_positions.restype = st
    L.rl_set_positions.argtypes = [vp, vp, vp]
    L.rl_tree_info.restype = st
    L.rl_tree_info.argtypes = [vp, P(u64), P(u32)]
    L.rl_dump_tree.restype = st
    L.rl_dump_tree.argtypes = [vp] * 11
    L.rl_prepare_update_connectivity.restype = st
    L.rl_prepare_update_connectivity.argtypes = [vp] * 6
    L.rl_find_targets.restype = st
    L.rl_find_targets.argtypes = [vp, u32, vp, u64, P(u64)]
    L.rl_update_connectivity.restype = st
    L.rl_update_connectivity.argtypes = [vp, u32, vp, u64, P(u64)]
    L.rl_set_elements.restype = st
    L.rl_set_elements.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.rl_get_elements.restype = st
    L.rl_get_elements.argtypes = [vp, C.c_int, vp, vp, vp, vp]
    L.rl_set_neurons.restype = st
    L.rl_set_neurons.argtypes = [vp] * 5
    L.rl_get_neurons.restype = st
    L.rl_get_neurons.argtypes = [vp] * 6
    L.rl_set_enabled.restype = st
    L.rl_set_enabled.argtypes = [vp, vp]
    L.rl_snapshot_neurons.restype = st
    L.rl_snapshot_neurons.argtypes = [vp, vp, vp]
    L.rl_snapshot_wait.restype = st
    L.rl_snapshot_wait.argtypes = [vp]
    L.rl_add_edges.restype = st
    L.rl_add_edges.argtypes = [vp, u64, vp, vp, vp]
    L.rl_get_edges.restype = st
    L.rl_get_edges.argtypes = [vp, vp, vp, vp, u64, P(u64)]
    L.rl_activity_block.restype = st
    L.rl_activity_block.argtypes = [vp, u32, u32]
    L.rl_plasticity_update.restype = st
    L.rl_plasticity_update.argtypes = [vp, u32]
    L.rl_simulate.restype = st
    L.rl_simulate.argtypes = [vp, u32, u32]
    L.rl_synchronize.restype = st
    L.rl_synchronize.argtypes = [vp]
    L.rl_get_stats.restype = st
    L.rl_get_stats.argtypes = [vp, P(RlStats)]
    L.rl_set_stream.restype = st
    L.rl_set_stream.argtypes = [vp, vp]
    L.rl_set_profiling.restype = st
    L.rl_set_profiling.argtypes = [vp, C.c_int]
    L.rl_get_phase_times.restype = st
    L.rl_get_phase_times.argtypes = [vp, vp, vp]
    L.rl_set_graphs.restype = st
    L.rl_set_graphs.argtypes = [vp, C.c_int]
    L.rl_set_step_fusion.restype = st
    L.rl_set_step_fusion.argtypes = [vp, C.c_int]
    L.rl_connect.restype = st
    L.rl_connect.argtypes = [vp, u32, vp, u64, vp, P(u64)]
    L.rl_process_requests.restype = st
    L.rl_process_requests.argtypes = [vp, u32, vp, u64, vp, P(u64)]
    L.rl_process_responses.restype = st
    L.rl_process_responses.argtypes = [vp, vp, vp, vp, u64, P(u64)]
    L.rl_candidate_weights.restype = st
    L.rl_candidate_weights.argtypes = [vp, u32, C.c_int, vp, vp, u64, P(u64)]
    L.rl_prepare_update_connectivity_noalloc.restype = st
    L.rl_prepare_update_connectivity_noalloc.argtypes = [vp, vp, vp, vp, vp]
    L.rl_set_target_calcium.restype = st
    L.rl_set_target_calcium.argtypes = [vp, vp]
    L.rl_get_target_calcium.restype = st
    L.rl_get_target_calcium.argtypes = [vp, vp]
    L.rl_autotune.restype = st
    L.rl_autotune.argtypes = [vp, C.c_int]
    L.rl_get_tuning.restype = st
    L.rl_get_tuning.argtypes = [vp, P(RlTuning), vp, vp]
    L.rl_set_tuning.restype = st
    L.rl_set_tuning.argtypes = [vp, P(RlTuning)]
    L.rl_ctx_memory.restype = st
    L.rl_ctx_memory.argtypes = [vp, P(u64), P(u64)]
    L.rl_serve_footprint.restype = st
    L.rl_serve_footprint.argtypes = [P(RlConfig), P(RlNetwork), dbl, u32, P(u64)]
    L.rl_serve_create.restype = st
    L.rl_serve_create.argtypes = [P(RlConfig), P(RlServeConfig), P(vp)]
    L.rl_serve_submit.restype = st
    L.rl_serve_submit.argtypes = [vp, P(RlServeRequest), P(u64)]
    L.rl_serve_poll.restype = st
    L.rl_serve_poll.argtypes = [vp, P(RlServeDone), u64, P(u64), i32]
    L.rl_serve_fetch.restype = st
    L.rl_serve_fetch.argtypes = [vp, u64, vp, vp, vp, vp, vp, u64]
    L.rl_serve_load.restype = st
    L.rl_serve_load.argtypes = [vp, P(u64), P(u64), P(u64)]
    L.rl_serve_destroy.restype = st
    L.rl_serve_destroy.argtypes = [vp]
    _lib = L
    return L


def _p(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def default_params(num_neurons: int, side: float) -> dict:
    """Parameters of the structural-plasticity workloads: Izhikevich a=0.02,
    b=0.2, c=-65, d=8 (regular spiking), input combined(synaptic_equally_weighted
    with conductance 3, normal(5, 2)), Gaussian sigma 750 um, theta 0.3, growth
    rate 1e-4 for all element types, target calcium 0.7, plasticity every 100
    steps.  Reference defaults: IzhikevichParameters (Parameters.h:123-130),
    CalciumCalculatorBase.h:206-210, GaussianDistributionKernel (Gaussian.h:38-39)."""
    return dict(num_neurons=int(num_neurons), plasticity_interval=100, h_model=10, h_calcium=10, seed=1,
                box_min=(0.0, 0.0, 0.0), box_max=(float(side),) * 3, theta=0.3, sigma=750.0, mu=0.0,
                iz_a=0.02, iz_b=0.2, iz_c=-65.0, iz_d=8.0, iz_v_spike=30.0, iz_k1=0.04, iz_k2=5.0, iz_k3=140.0,
                beta=0.001, tau_c=10000.0, target_calcium=0.7, initial_calcium=0.0,
                growth_rate=(1e-4, 1e-4, 1e-4), min_calcium=(0.4, 0.1, 0.0), retract_ratio=(0.0, 0.0, 0.0),
                conductance=3.0, noise_mean=5.0, noise_stddev=2.0, device=0, precision=PRECISION_FP64,
                kernel_type=KERNEL_GAUSSIAN, kernel_k=1.0, kernel_scale=1.0, linear_cutoff=float("inf"),
                neuron_model=MODEL_IZHIKEVICH, poisson_refractory=4, poisson_x0=0.05, poisson_tau_x=5.0,
                fhn_a=0.7, fhn_b=0.8, fhn_phi=0.08, fhn_init_x=-1.2, fhn_init_w=-0.6,
                aeif_C=281.0, aeif_g_L=30.0, aeif_E_L=-70.6, aeif_V_T=-50.4, aeif_d_T=2.0, aeif_tau_w=144.0, aeif_a=4.0, aeif_b=0.0805,
                aeif_V_spike=20.0)


def make_config(params: dict) -> RlConfig:
    cfg = RlConfig()
    for key, val in params.items():
        if key in ("box_min", "box_max", "growth_rate", "min_calcium", "retract_ratio"):
            getattr(cfg, key)[:] = [float(v) for v in val]
        elif hasattr(cfg, key):
            setattr(cfg, key, val)
    return cfg


def fill_network(r: RlNetwork, d: dict) -> RlNetwork:
    """rl_network from a dict with num_neurons, seed, side (or box_min /
    box_max), theta, sigma and growth_rate (one rate or three)."""
    r.num_neurons = int(d["num_neurons"])
    r.seed = int(d["seed"])
    side = d.get("side")
    r.box_min[:] = list(d.get("box_min", (0.0, 0.0, 0.0)))
    r.box_max[:] = list(d.get("box_max", (side, side, side)))
    r.theta = float(d["theta"])
    r.sigma = float(d["sigma"])
    gr = d["growth_rate"]
    r.growth_rate[:] = list(gr) if hasattr(gr, "__len__") else [float(gr)] * 3
    return r


class Network:
    """One network in one device context (rl_ctx)."""

    def __init__(self, params: dict, networks: Optional[list] = None):
        """One network from `params`, or — with `networks`, a list of dicts
        with num_neurons, seed, side (or box_min/box_max), theta, sigma,
        growth_rate — an ensemble whose shared parameters come from `params`."""
        self.lib = load_library()
        self.params = dict(params)
        self.cfg = make_config(params)
        h = C.c_void_p()
        if networks is None:
            self.n = int(params["num_neurons"])
            s = self.lib.rl_ctx_create(C.byref(self.cfg), C.byref(h))
        else:
            arr = (RlNetwork * len(networks))()
            for k, d in enumerate(networks):
                fill_network(arr[k], d)
            self.networks = [dict(d) for d in networks]
            self.n = int(sum(int(d["num_neurons"]) for d in networks))
            s = self.lib.rl_ensemble_create(C.byref(self.cfg), arr, len(networks), C.byref(h))
        if s != RL_OK:
            raise RelearnError(s, "context creation failed")
        self.h = h

    # ---- plumbing
    def _check(self, status: int):
        if status != RL_OK:
            msg = self.lib.rl_last_error(self.h)
            raise RelearnError(status, msg.decode() if msg else "")

    def close(self):
        if getattr(self, "h", None):
            self.lib.rl_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---- octree
    def set_positions(self, positions: np.ndarray, signal: np.ndarray):
        self._pos = np.ascontiguousarray(positions, np.float64).reshape(self.n, 3)
        self._sig = np.ascontiguousarray(signal, np.uint8)
        self._check(self.lib.rl_set_positions(self.h, _p(self._pos), _p(self._sig)))

    def tree_info(self):
        m = C.c_uint64()
        lv = C.c_uint32()
        self._check(self.lib.rl_tree_info(self.h, C.byref(m), C.byref(lv)))
        return int(m.value), int(lv.value)

    def tree(self) -> dict:
        m, _ = self.tree_info()
        out = dict(level=np.zeros(m, np.int32), neuron=np.zeros(m, np.int32), child_mask=np.zeros(m, np.uint8),
                   first_child=np.zeros(m, np.int32), bmin=np.zeros((m, 3)), bmax=np.zeros((m, 3)),
                   cnt_exc=np.zeros(m, np.uint32), cnt_inh=np.zeros(m, np.uint32), pos_exc=np.zeros((m, 3)),
                   pos_inh=np.zeros((m, 3)))
        keys = ["level", "neuron", "child_mask", "first_child", "bmin", "bmax", "cnt_exc", "cnt_inh", "pos_exc", "pos_inh"]
        self._check(self.lib.rl_dump_tree(self.h, *[_p(out[k]) for k in keys]))
        return out

    # ---- algorithm surface
    def prepare_update_connectivity(self, vacant_axons, vacant_exc, vacant_inh, signal=None, update=None):
        va = np.ascontiguousarray(vacant_axons, np.uint32)
        self._search_capacity = int(va.astype(np.uint64).sum())
        ve = np.ascontiguousarray(vacant_exc, np.uint32)
        vi = np.ascontiguousarray(vacant_inh, np.uint32)
        sg = None if signal is None else np.ascontiguousarray(signal, np.uint8)
        up = None if update is None else np.ascontiguousarray(update, np.uint8)
        self._check(self.lib.rl_prepare_update_connectivity(self.h, _p(sg), _p(va), _p(ve), _p(vi), _p(up)))

    def find_targets(self, step: int) -> np.ndarray:
        cap = getattr(self, "_search_capacity", None)
        if cap is None:
            cap = int(self.get_elements(AXON)["vacant"].astype(np.uint64).sum())
        out = np.zeros(max(int(cap), 1), REQUEST_DTYPE)
        cnt = C.c_uint64()
        self._check(self.lib.rl_find_targets(self.h, step, _p(out), len(out), C.byref(cnt)))
        if int(cnt.value) > len(out):  # the vacancy changed since the last prepare: run again with room
            out = np.zeros(int(cnt.value), REQUEST_DTYPE)
            self._check(self.lib.rl_find_targets(self.h, step, _p(out), len(out), C.byref(cnt)))
        return out[: int(cnt.value)]

    def update_connectivity(self, step: int, capacity: Optional[int] = None) -> np.ndarray:
        if capacity is None:
            capacity = int(self.get_elements(AXON)["vacant"].astype(np.uint64).sum())
        out = np.zeros(max(capacity, 1), SYNAPSE_DTYPE)
        cnt = C.c_uint64()
        self._check(self.lib.rl_update_connectivity(self.h, step, _p(out), len(out), C.byref(cnt)))
        return out[: min(int(cnt.value), len(out))]

    def connect(self, step: int, requests: np.ndarray):
        """ForwardConnector::process_requests over a given request list
        (REQUEST_DTYPE): returns the number of synapses created and one
        accepted flag per request, in the given order."""
        req = np.ascontiguousarray(requests, REQUEST_DTYPE)
        acc = np.zeros(max(len(req), 1), np.uint8)
        cnt = C.c_uint64()
        self._check(self.lib.rl_connect(self.h, step, _p(req), len(req), _p(acc), C.byref(cnt)))
        return int(cnt.value), acc[: len(req)].copy()

    def process_requests(self, step: int, requests: np.ndarray):
        """ForwardConnector::process_requests on the rank owning the
        requests' targets: binds dendrites and adds synapses, leaves the
        sources' axons alone; returns (synapses created, accepted flag per
        request in the given order)."""
        req = np.ascontiguousarray(requests, REQUEST_DTYPE)
        acc = np.zeros(max(len(req), 1), np.uint8)
        cnt = C.c_uint64()
        self._check(self.lib.rl_process_requests(self.h, step, _p(req), len(req), _p(acc), C.byref(cnt)))
        return int(cnt.value), acc[: len(req)].copy()

    def process_responses(self, requests: np.ndarray, accepted: np.ndarray, append: Optional[np.ndarray] = None) -> int:
        """ForwardConnector::process_responses on the rank owning the
        requests' sources: binds one vacant axon per accepted request and adds
        the synapses flagged in `append`; returns the number of axons bound."""
        req = np.ascontiguousarray(requests, REQUEST_DTYPE)
        acc = np.ascontiguousarray(accepted, np.uint8)
        app = None if append is None else np.ascontiguousarray(append, np.uint8)
        if len(acc) != len(req) or (app is not None and len(app) != len(req)):
            raise ValueError("one accepted (and append) flag per request")
        cnt = C.c_uint64()
        self._check(self.lib.rl_process_responses(self.h, _p(req), _p(acc), _p(app), len(req), C.byref(cnt)))
        return int(cnt.value)

    # ---- state
    def set_elements(self, etype: int, grown=None, delta=None, connected=None, vacant=None):
        g = None if grown is None else np.ascontiguousarray(grown, np.float64)
        d = None if delta is None else np.ascontiguousarray(delta, np.float64)
        c = None if connected is None else np.ascontiguousarray(connected, np.uint32)
        v = None if vacant is None else np.ascontiguousarray(vacant, np.uint32)
        self._check(self.lib.rl_set_elements(self.h, etype, _p(g), _p(d), _p(c), _p(v)))

    def get_elements(self, etype: int) -> dict:
        g = np.zeros(self.n); d = np.zeros(self.n)
        c = np.zeros(self.n, np.uint32); v = np.zeros(self.n, np.uint32)
        self._check(self.lib.rl_get_elements(self.h, etype, _p(g), _p(d), _p(c), _p(v)))
        return dict(grown=g, delta=d, connected=c, vacant=v)

    def set_neurons(self, x=None, u=None, calcium=None, fired=None):
        arrs = [None if v is None else np.ascontiguousarray(v, dt)
                for v, dt in ((x, np.float64), (u, np.float64), (calcium, np.float64), (fired, np.uint8))]
        self._check(self.lib.rl_set_neurons(self.h, *[_p(a) for a in arrs]))

    def neurons(self) -> dict:
        n = self.n
        x = np.zeros(n); u = np.zeros(n); ca = np.zeros(n); f = np.zeros(n, np.uint8); inp = np.zeros(n)
        self._check(self.lib.rl_get_neurons(self.h, _p(x), _p(u), _p(ca), _p(f), _p(inp)))
        return dict(x=x, u=u, calcium=ca, fired=f, input=inp)

    def set_enabled(self, enabled):
        e = np.ascontiguousarray(enabled, np.uint8)
        self._check(self.lib.rl_set_enabled(self.h, _p(e)))

    def snapshot_neurons(self, calcium=None, fired=None):
        """Start an asynchronous copy of calcium (float64) and fired flags
        (uint8) into the given arrays (pinned memory keeps it asynchronous);
        they hold the values once snapshot_wait returns."""
        for a, dt in ((calcium, np.float64), (fired, np.uint8)):
            if a is not None and (a.dtype != dt or not a.flags["C_CONTIGUOUS"] or a.size < self.n):
                raise ValueError(f"snapshot buffers must be contiguous {np.dtype(dt).name} arrays of at least {self.n} entries")
        self._check(self.lib.rl_snapshot_neurons(self.h, _p(calcium) if calcium is not None else None, _p(fired) if fired is not None else None))

    def snapshot_wait(self):
        self._check(self.lib.rl_snapshot_wait(self.h))

    def add_edges(self, target, source, weight):
        t = np.ascontiguousarray(target, np.uint32); s = np.ascontiguousarray(source, np.uint32)
        w = np.ascontiguousarray(weight, np.int32)
        self._check(self.lib.rl_add_edges(self.h, len(t), _p(t), _p(s), _p(w)))

    def set_target_calcium(self, target):
        """Target calcium per neuron (the reference's --file-calcium targets)."""
        t = np.ascontiguousarray(np.broadcast_to(np.asarray(target, np.float64), (self.n,)))
        self._check(self.lib.rl_set_target_calcium(self.h, _p(t)))

    def target_calcium(self) -> np.ndarray:
        t = np.zeros(self.n)
        self._check(self.lib.rl_get_target_calcium(self.h, _p(t)))
        return t

    def load_network(self, target, source, weight):
        """Add synapses as the reference loads a network file
        (Neurons::init_synaptic_elements, neurons/Neurons.cpp:105-127): each
        adds |weight| connected and grown elements to its source's axons and to
        its target's excitatory (weight > 0) or inhibitory dendrites."""
        t = np.ascontiguousarray(target, np.uint32)
        s = np.ascontiguousarray(source, np.uint32)
        w = np.ascontiguousarray(weight, np.int32)
        self.add_edges(t, s, w)
        a = np.abs(w).astype(np.uint32)
        adds = [np.bincount(s, weights=a, minlength=self.n), np.bincount(t[w > 0], weights=a[w > 0], minlength=self.n),
                np.bincount(t[w < 0], weights=a[w < 0], minlength=self.n)]
        for typ in range(3):
            el = self.get_elements(typ)
            add = adds[typ].astype(np.uint32)
            self.set_elements(typ, el["grown"] + add, el["delta"], el["connected"] + add, el["vacant"])

    def edges(self):
        cnt = C.c_uint64()
        self._check(self.lib.rl_get_edges(self.h, None, None, None, 0, C.byref(cnt)))
        m = int(cnt.value)
        t = np.zeros(max(m, 1), np.uint32); s = np.zeros(max(m, 1), np.uint32); w = np.zeros(max(m, 1), np.int32)
        self._check(self.lib.rl_get_edges(self.h, _p(t), _p(s), _p(w), m, C.byref(cnt)))
        return t[:m], s[:m], w[:m]

    # ---- stepping
    def activity_block(self, first_step: int, nsteps: int):
        self._check(self.lib.rl_activity_block(self.h, first_step, nsteps))

    def plasticity_update(self, step: int):
        self._check(self.lib.rl_plasticity_update(self.h, step))

    def simulate(self, first_step: int, nsteps: int):
        self._check(self.lib.rl_simulate(self.h, first_step, nsteps))

    def synchronize(self):
        self._check(self.lib.rl_synchronize(self.h))

    def set_stream(self, cuda_stream: int):
        """Issue the context's work on an external cudaStream_t (e.g. torch's)."""
        self._check(self.lib.rl_set_stream(self.h, C.c_void_p(cuda_stream)))

    def prepare_update_connectivity_noalloc(self, d_vacant_exc: int, d_vacant_inh: int, d_update: int = 0, cuda_stream: int = 0):
        """Tree update from DEVICE arrays (addresses), allocating nothing; see
        rl_prepare_update_connectivity_noalloc in include/relearn_b200.h."""
        self._check(self.lib.rl_prepare_update_connectivity_noalloc(self.h, C.c_void_p(d_vacant_exc), C.c_void_p(d_vacant_inh),
                                                                    C.c_void_p(d_update or None), C.c_void_p(cuda_stream or None)))

    def candidate_weights(self, source: int, precision: int = PRECISION_FP64):
        """Descent-0 candidates (visiting order) and raw weights of a search by `source`."""
        cnt = C.c_uint64()
        self._check(self.lib.rl_candidate_weights(self.h, source, precision, None, None, 0, C.byref(cnt)))
        m = int(cnt.value)
        nodes = np.zeros(max(m, 1), np.uint32); w = np.zeros(max(m, 1))
        self._check(self.lib.rl_candidate_weights(self.h, source, precision, _p(nodes), _p(w), m, C.byref(cnt)))
        return nodes[:m], w[:m]

    def set_graphs(self, on: bool = True):
        self._check(self.lib.rl_set_graphs(self.h, int(on)))

    def set_step_fusion(self, on: bool = True):
        """Blocks of activity steps of a network without synapses in one
        launch (the default), or one launch per step; the same bits."""
        self._check(self.lib.rl_set_step_fusion(self.h, int(on)))

    def set_profiling(self, on: bool = True):
        self._check(self.lib.rl_set_profiling(self.h, int(on)))

    def phase_times(self) -> dict:
        ms = np.zeros(len(PHASES)); cnt = np.zeros(len(PHASES), np.uint64)
        self._check(self.lib.rl_get_phase_times(self.h, _p(ms), _p(cnt)))
        return {k: (float(ms[i]), int(cnt[i])) for i, k in enumerate(PHASES)}

    def autotune(self, mode: int = 1):
        """Time the launch shapes of the search and activity kernels on this
        context's data at the next search and activity block (mode 1 reuses the
        process's result for the same size class, mode 2 always times)."""
        self._check(self.lib.rl_autotune(self.h, int(mode)))

    def tuning(self) -> dict:
        t = RlTuning()
        sm = (C.c_float * NUM_SEARCH_SHAPES)()
        am = (C.c_float * NUM_ACT_SHAPES)()
        self._check(self.lib.rl_get_tuning(self.h, C.byref(t), sm, am))
        d = {f: getattr(t, f) for f, _ in RlTuning._fields_}
        d["search_ms"] = {f"w{w}_p{p}_c{cp}" + (f"_hot{h}" if h else ""): float(sm[k]) for k, (w, p, cp, h) in enumerate(SEARCH_SHAPES) if sm[k] > 0}
        d["act_ms"] = {f"b{b}_v{v}_{'persistent' if p else 'grid'}": float(am[k]) for k, (b, p, v) in enumerate(ACT_SHAPES) if am[k] > 0}
        return d

    def set_tuning(self, search_warps=2, search_packet=32, search_cap=1, search_hot=0, act_block=256, act_persistent=0, act_vec=1):
        t = RlTuning(search_warps, search_hot, search_packet, search_cap, act_block, act_persistent, act_vec, 0)
        self._check(self.lib.rl_set_tuning(self.h, C.byref(t)))

    def memory(self) -> tuple:
        """Device bytes the context holds now and at its peak."""
        cur, peak = C.c_uint64(), C.c_uint64()
        self._check(self.lib.rl_ctx_memory(self.h, C.byref(cur), C.byref(peak)))
        return int(cur.value), int(peak.value)

    def stats(self) -> dict:
        s = RlStats()
        self._check(self.lib.rl_get_stats(self.h, C.byref(s)))
        return {k: int(getattr(s, k)) for k, _ in RlStats._fields_ if k != "reserved"}


# ------------------------------------------------------------ plugin mirror
@dataclass
class ConnectivityUpdateResult:
    """Algorithm::update_connectivity's result (algorithm/Algorithm.h:37-42) on
    one rank: all synapses are local."""

    number_created_synapses: int
    local_synapses: np.ndarray = field(default_factory=lambda: np.zeros(0, SYNAPSE_DTYPE))


class BarnesHut:
    """The ``barnes-hut`` Algorithm plugin on one rank (algorithm/BarnesHutInternal/BarnesHut.h).

    The caller owns the synaptic elements, as in the reference: it passes the
    vacant counts to :meth:`prepare_update_connectivity`, and applies
    ``connect_elements`` for every synapse returned by
    :meth:`update_connectivity` (one dendrite of the target, one axon of the
    source)."""

    algorithm_type = "barnes-hut"

    def __init__(self, params: dict, network: Optional[Network] = None):
        self.net = network if network is not None else Network(params)
        self.n = self.net.n

    def init(self, positions: np.ndarray, signal: np.ndarray):
        """Algorithm::init(n): insert all neurons into the octree."""
        self.net.set_positions(positions, signal)

    def prepare_update_connectivity(self, signal_types, vacant_axons, vacant_excitatory_dendrites, vacant_inhibitory_dendrites):
        self.net.prepare_update_connectivity(vacant_axons, vacant_excitatory_dendrites, vacant_inhibitory_dendrites, signal=signal_types)

    def update_connectivity(self, step: int) -> ConnectivityUpdateResult:
        syn = self.net.update_connectivity(step)
        return ConnectivityUpdateResult(len(syn), syn)

    def get_algorithm_type(self) -> str:
        return self.algorithm_type


class NeuronModel:
    """A NeuronModel plugin (neurons/models/NeuronModelBase.h) with the calcium
    and growth updates that Neurons runs after it every step; the model is the
    network's ``neuron_model`` parameter."""

    name = "izhikevich"

    def __init__(self, network: Network):
        self.net = network
        self.name = {v: k for k, v in NEURON_MODELS.items()}[int(network.params.get("neuron_model", 0))]

    def update_electrical_activity(self, step: int):
        self.net.activity_block(step, 1)

    def get_x(self):
        return self.net.neurons()["x"]

    def get_fired(self):
        return self.net.neurons()["fired"]

    def get_model_type(self) -> str:
        return self.name


class IzhikevichModel(NeuronModel):
    """--neuron-model izhikevich (models/izhikevich)."""


class PoissonModel(NeuronModel):
    """--neuron-model poisson (models/poisson); u holds the refractory steps left."""


class FitzHughNagumoModel(NeuronModel):
    """--neuron-model fitzhughnagumo (models/fitzhughnagumo); u holds w."""


class AEIFModel(NeuronModel):
    """--neuron-model aeif (models/aeif); u holds the adaptation w."""


class Simulation:
    """Simulation::simulate on one rank.  The reference starts at step 1 and
    runs ``number_steps + 1`` steps (sim/Simulation.cpp:399-400)."""

    def __init__(self, params: dict, positions: np.ndarray, signal: np.ndarray, algorithm: str = "barnes-hut",
                 neuron_model: str = "izhikevich"):
        if algorithm not in ALGORITHMS:
            raise RelearnError(6, f"algorithm {algorithm!r} is not built here (have {sorted(ALGORITHMS)})")
        if neuron_model not in NEURON_MODELS:
            raise RelearnError(6, f"neuron model {neuron_model!r} is not built here (have {sorted(NEURON_MODELS)})")
        params = dict(params)
        params["neuron_model"] = NEURON_MODELS[neuron_model]
        self.net = Network(params)
        self.net.set_positions(positions, signal)
        self.algorithm = BarnesHut(params, self.net)
        self.model = {"izhikevich": IzhikevichModel, "poisson": PoissonModel, "fitzhughnagumo": FitzHughNagumoModel, "aeif": AEIFModel}[neuron_model](self.net)
        self.step = 1

    def simulate(self, number_steps: int):
        count = int(number_steps) + 1
        self.net.simulate(self.step, count)
        self.step += count


from . import workloads  # noqa: E402  (re-export)

__all__ = ["Network", "BarnesHut", "NeuronModel", "IzhikevichModel", "PoissonModel", "FitzHughNagumoModel", "AEIFModel", "Simulation", "ConnectivityUpdateResult", "RelearnError", "default_params",
           "make_config", "load_library", "workloads", "REQUEST_DTYPE", "SYNAPSE_DTYPE", "ABI_FUNCTIONS"]
