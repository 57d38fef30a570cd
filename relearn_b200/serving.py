"""Serving form: a request loop for sweep runs on one GPU (rl_serve_* in
``include/relearn_b200.h``).

Each request is one network (size, seed, cube, theta, sigma, growth rates)
simulated for steps 1..steps with the server's model parameters.  The native
server admits requests continuously as worker slots and HBM budget free up,
runs admitted requests side by side on their own streams, and packs small
pending requests into one batched context.  A request's result does not depend
on that grouping: every network evolves bit for bit as in a context of its own.

The reference has no counterpart (its Simulation runs one network per
process); the per-request work is the reference's Simulation::simulate
(sim/Simulation.cpp:388-480).
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import (RL_OK, SYNAPSE_DTYPE, RelearnError, RlNetwork, RlServeConfig, RlServeDone, RlServeRequest, fill_network, load_library,
               make_config)

DONE_FIELDS = [f for f, _ in RlServeDone._fields_]


class Server:
    """A running request loop.  `params` are the model parameters shared by
    every request (default_params); `precision` selects the form."""

    def __init__(self, params: dict, hbm_budget_bytes: float = 150e9, slots: int = 8, pack_networks: int = 16,
                 pack_max_neurons: int = 65536, use_graphs: bool = True, autotune: int = 1):
        self.lib = load_library()
        self.cfg = make_config(params)
        sc = RlServeConfig()
        sc.hbm_budget_bytes = int(hbm_budget_bytes)
        sc.slots = int(slots)
        sc.pack_networks = int(pack_networks)
        sc.pack_max_neurons = int(pack_max_neurons)
        sc.use_graphs = 1 if use_graphs else 0
        sc.autotune = int(autotune)
        self.sc = sc
        h = C.c_void_p()
        s = self.lib.rl_serve_create(C.byref(self.cfg), C.byref(sc), C.byref(h))
        if s != RL_OK:
            raise RelearnError(s, "rl_serve_create failed")
        self.h = h
        self.sizes = {}

    def footprint(self, net: dict, steps: int, initial_axons: float = 0.0) -> int:
        r = fill_network(RlNetwork(), net)
        out = C.c_uint64()
        s = self.lib.rl_serve_footprint(C.byref(self.cfg), C.byref(r), float(initial_axons), int(steps), C.byref(out))
        if s != RL_OK:
            raise RelearnError(s, "rl_serve_footprint failed")
        return int(out.value)

    def submit(self, net: dict, positions: np.ndarray, signal: np.ndarray, steps: int, grown: Optional[list] = None,
               keep_state: bool = False) -> int:
        n = int(net["num_neurons"])
        pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(n, 3)
        sig = np.ascontiguousarray(signal, dtype=np.uint8).reshape(n)
        req = RlServeRequest()
        fill_network(req.net, net)
        req.xyz = pos.ctypes.data
        req.signal = sig.ctypes.data
        keep = [pos, sig]
        for t in range(3):
            g = None if grown is None or grown[t] is None else np.ascontiguousarray(grown[t], dtype=np.float64).reshape(n)
            keep.append(g)
            req.grown[t] = None if g is None else g.ctypes.data
        req.steps = int(steps)
        req.keep_state = 1 if keep_state else 0
        rid = C.c_uint64()
        s = self.lib.rl_serve_submit(self.h, C.byref(req), C.byref(rid))
        if s != RL_OK:
            raise RelearnError(s, "rl_serve_submit refused the request")
        self.sizes[int(rid.value)] = n
        return int(rid.value)

    def poll(self, wait_ms: int = 0, capacity: int = 256) -> list:
        """Records of finished requests (dicts with the rl_serve_done fields)."""
        buf = (RlServeDone * capacity)()
        cnt = C.c_uint64()
        s = self.lib.rl_serve_poll(self.h, buf, capacity, C.byref(cnt), int(wait_ms))
        if s != RL_OK:
            raise RelearnError(s, "rl_serve_poll failed")
        return [{f: getattr(buf[k], f) for f in DONE_FIELDS} for k in range(cnt.value)]

    def fetch(self, done: dict) -> dict:
        """Final state of a finished request submitted with keep_state."""
        n = int(done["num_neurons"])
        x, u, ca = np.empty(n), np.empty(n), np.empty(n)
        con = np.empty(3 * n, np.uint32)
        syn = np.empty(max(int(done["num_synapses"]), 1), SYNAPSE_DTYPE)
        s = self.lib.rl_serve_fetch(self.h, int(done["id"]), x.ctypes.data, u.ctypes.data, ca.ctypes.data, con.ctypes.data, syn.ctypes.data,
                                    int(done["num_synapses"]))
        if s != RL_OK:
            raise RelearnError(s, f"no kept state for request {done['id']}")
        syn = syn[:int(done["num_synapses"])]
        return dict(x=x, u=u, calcium=ca, connected=con.reshape(3, n), target=syn["target"].copy(), source=syn["source"].copy(),
                    weight=syn["weight"].copy())

    def load(self) -> tuple:
        """(queued, running, reserved bytes)."""
        p, r, b = C.c_uint64(), C.c_uint64(), C.c_uint64()
        self.lib.rl_serve_load(self.h, C.byref(p), C.byref(r), C.byref(b))
        return int(p.value), int(r.value), int(b.value)

    def close(self):
        """Let every request finish, then stop the workers."""
        if getattr(self, "h", None):
            self.lib.rl_serve_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def latency_summary(done: list) -> dict:
    """p50 / p99 completion latency (submission to result) and the aggregate
    neuron-steps/s over the span from the first submission to the last result."""
    lat = np.array([d["t_finish"] - d["t_submit"] for d in done])
    wait = np.array([d["t_admit"] - d["t_submit"] for d in done])
    t0 = min(d["t_submit"] for d in done)
    t1 = max(d["t_finish"] for d in done)
    work = float(sum(d["neuron_steps"] for d in done))
    return dict(requests=len(done), p50_s=float(np.percentile(lat, 50)), p99_s=float(np.percentile(lat, 99)), max_s=float(lat.max()),
                mean_queue_s=float(wait.mean()), p99_queue_s=float(np.percentile(wait, 99)), span_s=t1 - t0, neuron_steps=work,
                neuron_steps_per_s=work / (t1 - t0))
