#!/usr/bin/env python
"""Benchmark of the structural-plasticity hot path on B200.

Workload (one bench step): one plasticity period of a 1,000,000-neuron
network — 100 activity steps (input + Izhikevich + calcium + growth, one fused
kernel each) followed by one plasticity update (commit, octree update,
Barnes-Hut search, connector, graph rebuild) — with the reference parameters
(Izhikevich a=0.02 b=0.2 c=-65 d=8, normal(5,2) input, conductance 3,
sigma 750 um, theta 0.3, growth 1e-4, target calcium 0.7), neurons uniform in
a 10,000 um cube, FP64.  Metric: neuron-steps/s = N * 100 * K / device time.

A second figure, Barnes-Hut searches/s, is measured on the reference
benchmark's search snapshot: one vacant axon and one vacant excitatory and
inhibitory dendrite per neuron (benchmark/benchmark_barnes_hut_cuda.cpp:53-77),
i.e. 1,000,000 searches per plasticity update.

`--impl reference` times the CPU restatement of the reference's barnes-hut +
izhikevich path (the oracle) on all host cores for the same metric.
Multi-GPU: independent replicas (one network per GPU, no exchange).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_DEFAULT = 1_000_000
SIDE_DEFAULT = 10_000.0
PERIOD = 100
# Algorithmic bytes per neuron-step of one launch per step (a network with
# synapses, or step fusion off), FP64 SoA, one target calcium for all neurons:
# the step kernel reads enabled 1 + x 8 + u 8 and writes x 8 + u 8 + spike
# flag 1 + spike-history byte 1 = 35; calcium and growth (one launch per chunk
# of up to 64 steps: two per 100-step block) read each history byte (1) and
# read and write calcium 8 and three deltas 24 once per chunk (2 x 64 / 100);
# the input (8) on the last step of each block only.
ACT_BYTES_PER_NEURON = 35 + 1 + (2 * 64 + 8) / 100
# With synapses: a block's first step pulls over the in-CSR (two row offsets 8
# per neuron, source id 4 + weight 4 + spike flag 1 per in-edge); the other
# steps read the pushed sum (8 B FP64, 4 B FP32) of every neuron (the pushes
# of the about 1 % of neurons that fire, along their out-edges, not counted).
ACT_BYTES_PER_EDGE = 9
ACT_BYTES_CSR_ROW = 8
ACT_BYTES_PUSHED = {0: 8, 1: 4}


def step_bytes(precision: int, n: int, edges: float) -> float:
    """Algorithmic bytes of one activity step of n neurons, one launch per step."""
    b = (ACT_BYTES_PER_NEURON if precision == 0 else ACT_BYTES_FP32) * n
    if edges:
        b += ACT_BYTES_PUSHED[precision] * n * (PERIOD - 1) / PERIOD + (ACT_BYTES_CSR_ROW * n + ACT_BYTES_PER_EDGE * edges) / PERIOD
    return b


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled during the timed region: NVML
    every 10 ms from a thread (the timed region of a short run lasts well under
    a second), nvidia-smi every 200 ms where NVML is missing.  The NVML device is
    the CUDA device's own, matched by UUID (NVML numbers every GPU of the host)."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    REASONS = {0x4: "sw_power_cap", 0x8: "hw_slowdown", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown"}

    def __init__(self, device: int, period_s: float = 0.01):
        self.device = device
        self.period = period_s
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []  # (sm_mhz, sm_max_mhz, reason bits)

    def _nvml_handle(self):
        import pynvml

        pynvml.nvmlInit()
        try:
            import torch

            uuid = str(torch.cuda.get_device_properties(self.device).uuid)
            for k in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(k)
                u = pynvml.nvmlDeviceGetUUID(h)
                u = u.decode() if isinstance(u, bytes) else u
                if u.replace("GPU-", "") == uuid.replace("GPU-", ""):
                    return pynvml, h
        except Exception:
            pass
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(self.device)

    def _loop(self, nv, h):
        get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
        while True:
            try:
                self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), float(smax), int(get_reasons(h))))
            except Exception:
                return
            if self.stop.wait(self.period):
                return

    def __enter__(self):
        import threading

        self.stop = threading.Event()
        try:
            nv, h = self._nvml_handle()
            self.thread = threading.Thread(target=self._loop, args=(nv, h), daemon=True)
            self.thread.start()
            return self
        except Exception:
            self.thread = None
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self) -> dict:
        if self.rows:
            sm = [r[0] for r in self.rows]
            reasons = sorted({name for r in self.rows for bit, name in self.REASONS.items() if r[2] & bit})
            return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(r[1] for r in self.rows), "reasons": reasons, "samples": len(self.rows),
                    "source": "nvml, 10 ms"}
        rows = []
        try:
            for line in open(self.path):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi, 200 ms"}


def max_over_ranks(x: float, world: int, device) -> float:
    """The largest of the ranks' values (device time of the timed region): the
    job is as slow as its slowest replica.  NCCL on the GPU, gloo on the CPU."""
    if world <= 1:
        return x
    import torch

    t = torch.tensor([x], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(world: int, units_per_rank: float, max_ms: float) -> float:
    """Whole-job throughput of independent replicas: the units all ranks
    processed over the slowest rank's time."""
    return world * units_per_rank / (max_ms / 1e3)


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def build_network(n, side, seed, placement):
    from relearn_b200 import Network, default_params, workloads

    params = default_params(n, side)
    params["seed"] = seed
    pos = workloads.uniform_cube(n, side, seed) if placement == "uniform" else workloads.gaussian_mixture(n, side, seed)
    sig = workloads.signal_types(n, seed)
    return params, pos, sig


# Figures taken from ncu captures of the kernels (instruction mix, DRAM bytes,
# warp-lane activity, hit rates).  Each group names the kernel sources it was
# captured at by a digest of them (kernel_digest below); a figure whose
# sources have changed since is reported with "stale": true until it is
# captured again.
CAPTURED = {
    # one launch per step at 1M neurons with synapses (bench.py --case
    # plasticity --step-fusion 0, launches of the second block): the step
    # kernel's DRAM read + write per launch plus that of a 64-step chunk's
    # calcium and growth launch per step (FP64 34.95 + 0.11 MB + (97.04 +
    # 7.33) / 64 MB; FP32 23.75 + 0.00 MB + (85.01 + 3.90) / 64 MB); FP64 warp
    # instructions per neuron-step of both (DMUL, DADD, DFMA, DSETP: 6.26 +
    # 3.72), and for the FP32 form warp instructions of every kind (7.98 +
    # 1.36).  The FP64 pipe of an SM takes 2 warp instructions per cycle (64
    # lanes).
    "activity64": {"sources": ("activity.cu", "rl_math.cuh"), "digest": "e6ef1fe863ecbbd9",
                   "traffic": 34.95e6 + 0.11e6 + (97.04e6 + 7.33e6) / 64, "fp64_warp_instr_per_neuron": 9.97},
    "activity32": {"sources": ("fp32.cu", "rl_math.cuh"), "digest": "ae16ba4013f08c25",
                   "traffic": 23.75e6 + (85.01e6 + 3.90e6) / 64, "warp_instr_per_neuron": 9.34},
    # the fused block kernels (a network without synapses: a block of steps per
    # launch, state in registers), from the instruction mix of one 100-step
    # launch at 1M neurons (bench.py --case activity --case-steps 100), per
    # neuron-step: k_activity_steps 10.08 FP64 warp instructions (DMUL 3.80,
    # DADD 3.55, DFMA 1.82, DSETP 0.92); k_activity_f32_steps 5.85 warp
    # instructions of every kind, issued at one per SM sub-partition (4 per
    # SM) per cycle; DRAM read + write of that launch
    "fused64": {"sources": ("activity.cu", "rl_math.cuh"), "digest": "e6ef1fe863ecbbd9", "fp64_warp_instr_per_neuron": 10.08,
                "traffic": 50.06e6 + 4.06e6},
    "fused32": {"sources": ("fp32.cu", "rl_math.cuh"), "digest": "ae16ba4013f08c25", "warp_instr_per_neuron": 5.85, "traffic": 30.02e6 + 0.14e6},
    # the batched block kernel over the 128-network configuration (7.15M
    # neurons, bench.py --case ensemble --case-steps 100 --precision fp32):
    # warp instructions per neuron-step, DRAM read + write of the launch
    "ensemble32": {"sources": ("fp32.cu", "rl_math.cuh"), "digest": "ae16ba4013f08c25", "warp_instr_per_neuron": 5.95,
                   "traffic": 215.10e6 + 187.94e6},
    # the search snapshot at 1M (bench.py --case search; the excitatory pass,
    # 0.8M searches): lanes active per warp instruction, L1 / L2 hit rates of
    # the walk, DRAM bytes per search
    "search64": {"sources": ("bh_search.cu", "bh_eval.cuh", "bh_wide.cuh", "rl_math.cuh"), "digest": "290d6ed0479e64d4", "lanes_active": 19.85,
                 "l1_hit": 0.924, "l2_hit": 0.774, "dram_bytes_per_search": 681.0},
    "search32": {"sources": ("fp32.cu", "rl_math.cuh"), "digest": "ae16ba4013f08c25", "lanes_active": 21.88, "l1_hit": 0.812, "l2_hit": 0.936},
}
B200_SMS = 148
# algorithmic memory of a fused block launch per neuron: reads enabled, spike
# flag, x, u, calcium, three deltas; writes x, u, calcium, deltas, both
# spike-flag buffers, the input
FUSED_BYTES = {0: 50 + 58, 1: 30 + 34}
# Bytes the reference's octree node carries for one acceptance test
# (both types' centroid and count 2 x (3 x 8 + 4) = 56 B,
# plus 8 B of child links); the search reads one type's record, so this
# over-counts what one walk step needs (48 B FP64: 32 B record + 8 B
# topology + 8 B cell length; 28 B FP32).
SEARCH_BYTES_PER_NODE = 64


def kernel_digest(files) -> str:
    import hashlib

    h = hashlib.sha256()
    for f in files:
        with open(os.path.join(ROOT, "relearn_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def captured(name: str) -> dict:
    """A captured figure group with its staleness against the current sources."""
    g = dict(CAPTURED[name])
    cur = kernel_digest(g["sources"])
    g["stale"] = g["digest"] != cur
    g["digest_now"] = cur
    return g


def fp64_pipe_roofline(roof: dict, n: int, sm_mhz) -> dict:
    """The per-step FP64 activity kernel is bound by its FP64 pipe, not by
    HBM: its floor time against its measured launch time."""
    mhz = sm_mhz or 1965.0
    cap = captured("activity64")
    instr = cap["fp64_warp_instr_per_neuron"]
    floor_us = instr * n / (2 * B200_SMS * mhz * 1e6) * 1e6
    avg = roof.get("avg_launch_us")
    return {"bound": "fp64 pipe", "warp_instr_per_neuron_step": instr, "sm_mhz": mhz, "floor_us": floor_us,
            "avg_launch_us": avg, "frac": floor_us / avg if avg else None, "stale": cap["stale"],
            "how": "FP64 warp instructions per launch (ncu instruction mix) / (2 per SM per cycle x 148 SMs x median SM clock)"}


def fused_roofline(precision: int, n: int, step_us: float, act_cnt: int, sm_mhz, hbm: float, peak_kind: str, profiled: bool) -> dict:
    """Roofline of the fused block kernel: compute-bound (the FP64 pipe for
    the FP64 drop-in, instruction issue for the FP32 form), with the memory
    side (state once per launch) beside it."""
    mhz = sm_mhz or 1965.0
    launch_us = step_us * PERIOD
    cap = captured("fused64" if precision == 0 else "fused32")
    if precision == 0:
        lane_ops = cap["fp64_warp_instr_per_neuron"] * 32  # FP64 lane operations per neuron-step
        achieved = lane_ops * n / (step_us * 1e-6) / 1e12
        peak = 64 * B200_SMS * mhz * 1e6 / 1e12
        roof = {"bound": "fp64", "kernel": "k_activity_steps", "achieved": achieved, "peak": peak, "unit": "T FP64 lane-op/s",
                "frac": achieved / peak, "ops_per_neuron_step": lane_ops,
                "peak_kind": "nominal issue rate at the median SM clock: 64 FP64 lanes per SM x 148 SMs (no measured FP64 peak)"}
    else:
        achieved = cap["warp_instr_per_neuron"] * n / (step_us * 1e-6) / 1e12
        peak = 4 * B200_SMS * mhz * 1e6 / 1e12
        roof = {"bound": "issue", "kernel": "k_activity_f32_steps", "achieved": achieved, "peak": peak, "unit": "T warp-inst/s",
                "frac": achieved / peak, "warp_instr_per_neuron_step": cap["warp_instr_per_neuron"],
                "peak_kind": "nominal issue rate at the median SM clock: 1 warp instruction per SM sub-partition per cycle x 592"}
    bytes_per_launch = FUSED_BYTES[precision] * n
    roof.update({"sm_mhz": mhz, "steps_per_launch": PERIOD, "avg_step_us": step_us, "avg_launch_us": launch_us, "launches": act_cnt // PERIOD,
                 "traffic": cap["traffic"] if profiled else None, "traffic_unit": "bytes per launch (ncu dram read + write)",
                 "stale": cap["stale"],
                 "hbm": {"bytes_per_launch": bytes_per_launch, "achieved": bytes_per_launch / (launch_us * 1e-6) / 1e9, "peak": hbm, "unit": "GB/s",
                         "frac": bytes_per_launch / (launch_us * 1e-6) / 1e9 / hbm if hbm else None, "peak_kind": peak_kind}})
    return roof


def step_compute(precision: int, n: int, step_us: float, sm_mhz=None) -> dict:
    """The compute side of one launch per step (step kernel + the chunk's
    calcium and growth) from the captured instruction counts: FP64 lane
    operations against the FP64 pipe (FP64 form), warp instructions against
    the issue rate (FP32 form)."""
    mhz = sm_mhz or 1965.0
    cap = captured("activity64" if precision == 0 else "activity32")
    if precision == 0:
        lane_ops = cap["fp64_warp_instr_per_neuron"] * 32
        achieved = lane_ops * n / (step_us * 1e-6) / 1e12
        peak = 64 * B200_SMS * mhz * 1e6 / 1e12
        return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "T FP64 lane-op/s", "frac": achieved / peak,
                "ops_per_neuron_step": lane_ops, "stale": cap["stale"], "peak_kind": "nominal: 64 FP64 lanes per SM x 148 SMs at %g MHz" % mhz}
    achieved = cap["warp_instr_per_neuron"] * n / (step_us * 1e-6) / 1e12
    peak = 4 * B200_SMS * mhz * 1e6 / 1e12
    return {"bound": "issue", "achieved": achieved, "peak": peak, "unit": "T warp-inst/s", "frac": achieved / peak,
            "warp_instr_per_neuron_step": cap["warp_instr_per_neuron"], "stale": cap["stale"],
            "peak_kind": "nominal: 1 warp instruction per SM sub-partition per cycle x 592 at %g MHz" % mhz}


# FP32: the step kernel reads enabled 1 + spike flag 1 + x 4 + u 4 and writes
# x 4 + u 4 + spike flag 1 + history byte 1 = 20; the chunks' calcium and
# growth read each history byte (1) and calcium 8 + three deltas 12, read and
# written once per chunk (2 x 40 / 100); the input (4) on a block's last step
ACT_BYTES_FP32 = 20 + 1 + (2 * 40 + 4) / 100


def measure_form(args, precision, dev, stream, world, pos, sig, params, clk=None):
    """Warm up and time args.steps plasticity periods of one network in the
    given precision form; returns the figures of that form."""
    import torch

    import relearn_b200 as R

    n = args.neurons
    p = dict(params)
    p["precision"] = precision
    net = R.Network(p)
    net.set_stream(stream.cuda_stream)
    net.set_positions(pos, sig)
    net.set_step_fusion(bool(args.step_fusion))
    apply_shapes(args, net, precision)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2
    step = 1
    for _ in range(args.warmup):
        net.simulate(step, PERIOD)
        step += PERIOD
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    launches0 = net.stats()["gpu_launches"]
    net.phase_times()
    net.set_profiling(True)
    times = []
    ctx = clk if clk is not None else _Null()
    with ctx:
        for _ in range(args.steps):
            flush.fill_(1.0)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            net.simulate(step, PERIOD)
            e1.record(stream)
            step += PERIOD
            e1.synchronize()
            times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    phases = net.phase_times()
    net.set_profiling(False)
    launches = net.stats()["gpu_launches"] - launches0
    total_ms = max_over_ranks(float(sum(times)), world, dev)
    value = replica_value(world, n * PERIOD * args.steps, total_ms)
    act_ms, act_cnt = phases["activity_kernel"]
    edges = int(net.stats().get("synapses_created", 0))
    bytes_per_launch = int(round(step_bytes(precision, n, edges)))
    hbm, peak_kind = peaks()
    achieved = bytes_per_launch / (act_ms / act_cnt / 1e3) / 1e9 if act_cnt else 0.0
    # DRAM bytes per launch from one ncu capture of the same kernel on this
    # workload: reads equal the algorithmic read bytes, writes stay in L2
    # during the launch
    cap = captured("activity64" if precision == 0 else "activity32")
    traffic = cap["traffic"] if (n == 1_000_000 and args.placement == "uniform") else None  # captured at 1M with synapses
    if args.step_fusion and not edges and act_cnt:
        # no synapses: each 100-step block ran as one launch of the fused kernel
        sm_mhz = clk.summary().get("sm_mhz") if clk is not None else None
        roof = fused_roofline(precision, n, 1e3 * act_ms / act_cnt, act_cnt, sm_mhz, hbm, peak_kind,
                              n == 1_000_000 and args.placement == "uniform")
        return dict(net=net, step=step, value=value, total_ms=total_ms, phases={k: v[0] for k, v in phases.items()}, launches=launches, roofline=roof,
                    tuning=net.tuning())
    roof = {"bound": "hbm", "kernel": "k_activity" if precision == 0 else "k_activity_f32", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm if hbm else None, "traffic": traffic, "traffic_unit": "bytes per launch (ncu dram read + write)",
            "stale": cap["stale"], "peak_kind": peak_kind, "bytes_per_launch": bytes_per_launch, "launches": act_cnt,
            "avg_launch_us": 1e3 * act_ms / act_cnt if act_cnt else None}
    return dict(net=net, step=step, value=value, total_ms=total_ms, phases={k: v[0] for k, v in phases.items()}, launches=launches, roofline=roof,
                tuning=net.tuning())


class _Null:
    def __enter__(self):
        return self

    def __exit__(self, *exc):
        return False


def apply_shapes(args, net, precision):
    """Launch shapes: timed during the warm-up (default), or set by hand with
    --act-shape / --search-shape (profiling runs, where timing under the
    profiler would pick shapes at random)."""
    if args.act_shape or args.search_shape:
        b, p, v = (int(x) for x in (args.act_shape or "256,0,1").split(","))
        w, pk, cp, hot = (int(x) for x in ((args.search_shape or "2,32") + ",1,0").split(",")[:4])
        net.set_tuning(search_warps=w, search_packet=pk, search_cap=cp, search_hot=hot, act_block=b, act_persistent=p, act_vec=v if precision else min(v, 2))
    else:
        net.autotune(1)


def bench_config(args, world, precision):
    """The workload of one bench step, the same for both arms."""
    return {"workload": f"{args.neurons} Izhikevich neurons {args.placement} in a {args.side:g} um cube, "
                        f"{'FP64 drop-in' if precision == 0 else 'FP32 form'}; one bench step = {PERIOD} activity steps + 1 plasticity update",
            "neurons": args.neurons, "placement": args.placement, "period": PERIOD, "l2": "256 MB buffer written between timed steps (GPU arm)",
            "parallelism": f"replicas{world}"}


def run_b200(args, world, rank, local):
    import torch

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120), device_id=dev)
    n, side = args.neurons, args.side
    params, pos, sig = build_network(n, side, args.seed + rank, args.placement)
    params["device"] = local
    # a stream of its own: the library captures the 100-step activity blocks as
    # CUDA graphs, which the legacy default stream does not allow
    stream = torch.cuda.Stream(dev)
    torch.cuda.set_stream(stream)
    main_prec = 1 if args.precision == "fp32" else 0
    clk = ClockSampler(local)
    m = measure_form(args, main_prec, dev, stream, world, pos, sig, params, clk)
    net, step = m["net"], m["step"]

    # e2e through the public C ABI with host buffers: every bench step uploads
    # the enable flags (a per-step host input of Simulation::simulate's
    # interrupts) and reads back calcium and fired flags, the reads as
    # snapshots that overlap the next step; the last one has landed before the
    # clock stops
    enabled = torch.ones(n, dtype=torch.uint8).pin_memory().numpy()
    ca = torch.empty(n, dtype=torch.float64).pin_memory().numpy()
    fired = torch.empty(n, dtype=torch.uint8).pin_memory().numpy()
    e2e_steps = max(2, min(args.steps, 5))
    # one untimed round sets up the staging buffers and the copy stream
    net.set_enabled(enabled)
    net.simulate(step, PERIOD)
    step += PERIOD
    net.snapshot_neurons(ca, fired)
    net.snapshot_wait()
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        net.set_enabled(enabled)
        net.simulate(step, PERIOD)
        step += PERIOD
        net.snapshot_neurons(ca, fired)
    net.snapshot_wait()
    torch.cuda.synchronize(dev)
    e2e_s = time.perf_counter() - t0
    e2e_val = world * n * PERIOD * e2e_steps / e2e_s

    bh = bh_snapshot(net, n, stream, step) if not args.skip_bh else None
    net.close()
    other = None
    if not args.skip_fp32 and main_prec == 0:
        o = measure_form(args, 1, dev, stream, world, pos, sig, params)
        bh32 = bh_snapshot(o["net"], n, stream, o["step"], 1, bh["roofline"]["touched_per_search"] if bh else None) if not args.skip_bh else None
        other = {"precision": "fp32", "value": o["value"], "unit": "neuron-steps/s", "ms_per_step": o["total_ms"] / args.steps,
                 "vs_fp64_drop_in": o["value"] / m["value"], "roofline": o["roofline"], "phases_ms": o["phases"], "tuning": o["tuning"]}
        if bh32:
            other["bh_search"] = bh32
            if bh:
                other["bh_search"]["vs_fp64_drop_in"] = bh32["value"] / bh["value"]
        o["net"].close()

    # the second placement of the same workload: a 64-component Gaussian
    # mixture (component std 200 um) that unbalances the octree
    mixture = None
    if not args.skip_mixture and args.placement == "uniform":
        mparams, mpos, msig = build_network(n, side, args.seed + rank, "mixture")
        mparams["device"] = local
        mm = measure_form(args, 0, dev, stream, world, mpos, msig, mparams)
        mixture = {"placement": "64-component Gaussian mixture, component std 200 um, centres uniform in the cube", "precision": "fp64",
                   "value": mm["value"], "unit": "neuron-steps/s", "ms_per_step": mm["total_ms"] / args.steps, "roofline": mm["roofline"],
                   "phases_ms": mm["phases"], "octree": {"nodes": mm["net"].tree_info()[0], "max_level": mm["net"].tree_info()[1]}}
        if not args.skip_bh:
            mixture["bh_search"] = bh_snapshot(mm["net"], n, stream, mm["step"])
        mm["net"].close()

    syn = None
    if not args.skip_synapses:
        syn = {"fp64": synapse_regime(args, dev, stream, world, 0)}
        if not args.skip_fp32:
            syn["fp32"] = synapse_regime(args, dev, stream, world, 1)
            syn["fp32"]["vs_fp64"] = syn["fp32"]["value"] / syn["fp64"]["value"]
    ens = None
    if not args.skip_ensemble:
        ens = ensemble_figure(args, dev, stream, world, rank)
    prec = None
    if rank == 0 and world == 1 and not args.skip_precision_report:
        prec = precision_report(args, dev, stream)
    serve = None
    if rank == 0 and world == 1 and not args.skip_serve:
        serve = serve_figure(args, dev)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, params, pos, sig)
    clocks = clk.summary()
    if main_prec == 0 and args.placement == "uniform" and m["roofline"]["kernel"] == "k_activity":
        m["roofline"]["fp64_pipe"] = fp64_pipe_roofline(m["roofline"], n, clocks.get("sm_mhz"))
    if main_prec == 1 and args.placement == "uniform" and m["roofline"]["kernel"] == "k_activity_f32" and m["roofline"].get("avg_launch_us"):
        # the FP32 step kernel (with its chunks' calcium and growth) against instruction issue
        m["roofline"]["issue"] = step_compute(1, n, m["roofline"]["avg_launch_us"], clocks.get("sm_mhz"))
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return None
    line = {
        "metric": "neuron-steps/s",
        "value": m["value"],
        "unit": "neuron-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": m["total_ms"] / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64" if main_prec == 0 else "f32",
        "data": "synthetic (seeded positions, reference parameters)",
        "config": bench_config(args, world, main_prec),
        "roofline": m["roofline"],
        "phases_ms": m["phases"],
        "e2e": {"value": e2e_val, "unit": "neuron-steps/s", "h2d_bytes_per_step": n, "d2h_bytes_per_step": 9 * n,
                "api": "rl_set_enabled + rl_simulate + rl_snapshot_neurons, rl_snapshot_wait after the last step (pinned host buffers)"},
        "gpu_launches": m["launches"],
        "tuning": m["tuning"],
        "clocks": clocks,
    }
    if bh:
        line["bh_search"] = bh
    if other:
        line["fp32_form"] = other
    if mixture:
        line["mixture"] = mixture
    if syn:
        line["synapse_regime"] = syn
    if ens:
        line["ensemble"] = ens
    if prec:
        line["precision_report"] = prec
    if serve:
        line["serving"] = serve
    if cpu:
        line["cpu_baseline"] = cpu
    return line


def synapse_regime(args, dev, stream, world, precision):
    """The regime with synapses: the bench network (1M neurons uniform in the
    10,000 um cube) with synaptic elements seeded U[0, 4] per type
    (--synaptic-elements-lower-bound / -upper-bound, relearn.cpp:620-624), so
    that every plasticity update searches for the vacant axons and the
    connector forms synapses, and activity runs one launch per step (the
    in-edges couple the neurons).  One bench step = 100 activity steps + 1
    plasticity update, as for the headline."""
    import torch

    import relearn_b200 as R
    from relearn_b200 import workloads

    n = args.neurons
    params, pos, sig = build_network(n, args.side, args.seed + 1000, "uniform")
    p = dict(params)
    p["precision"] = precision
    p["device"] = dev.index
    net = R.Network(p)
    net.set_stream(stream.cuda_stream)
    net.set_positions(pos, sig)
    net.set_step_fusion(bool(args.step_fusion))
    for t, (g, v) in enumerate(workloads.initial_elements(n, 77, 0.0, 4.0)):
        net.set_elements(t, g, np.zeros(n), np.zeros(n, np.uint32), v)
    apply_shapes(args, net, precision)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)
    step = 1
    # the first updates search for most initial axons, later ones for the few
    # still vacant: search shapes are tuned per density class of the search
    # list, so the warm-up runs until the sparse classes have been met
    for _ in range(max(args.warmup, 6)):
        net.simulate(step, PERIOD)
        step += PERIOD
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    edges_before = len(net.edges()[0])
    s0 = net.stats()
    net.phase_times()
    net.set_profiling(True)
    times = []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        net.simulate(step, PERIOD)
        e1.record(stream)
        step += PERIOD
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    torch.cuda.synchronize(dev)
    phases = net.phase_times()
    net.set_profiling(False)
    s1 = net.stats()
    edges_after = len(net.edges()[0])
    total_ms = max_over_ranks(float(sum(times)), world, dev)
    hbm, peak_kind = peaks()
    act_ms, act_cnt = phases["activity_kernel"]
    edges = 0.5 * (edges_before + edges_after)
    per_neuron = ACT_BYTES_PER_NEURON if precision == 0 else ACT_BYTES_FP32
    bytes_per_launch = step_bytes(precision, n, edges)
    act_achieved = bytes_per_launch / (act_ms / act_cnt / 1e3) / 1e9 if act_cnt else 0.0
    act_roof = {"bound": "hbm", "kernel": "k_activity" if precision == 0 else "k_activity_f32", "achieved": act_achieved, "peak": hbm,
                "unit": "GB/s", "frac": act_achieved / hbm, "peak_kind": peak_kind, "bytes_per_launch": bytes_per_launch,
                "avg_launch_us": 1e3 * act_ms / act_cnt if act_cnt else None, "launches": act_cnt,
                "bytes": f"{per_neuron:.2f} B per neuron-step + {ACT_BYTES_PUSHED[precision]} B pushed sum per neuron-step + per 100-step block "
                         f"{ACT_BYTES_CSR_ROW} B row offsets per neuron and {ACT_BYTES_PER_EDGE} B per in-edge",
                "kernels": "the step kernel (k_activity / k_activity_f32, one launch per step) and the chunks' calcium and growth (k_calcium_growth / "
                           "k_calcium_growth_f32, one launch per chunk of up to 64 steps)"}
    if act_cnt:
        comp = step_compute(precision, n, 1e3 * act_ms / act_cnt)
        act_roof["compute"] = comp
        if comp["frac"] > act_roof["frac"]:
            # the arithmetic side is the nearer bound: report it first
            act_roof = dict(comp, kernel=act_roof["kernel"], kernels=act_roof["kernels"], avg_launch_us=act_roof["avg_launch_us"],
                            launches=act_cnt, hbm={k: act_roof[k] for k in ("achieved", "peak", "unit", "frac", "peak_kind", "bytes_per_launch", "bytes")})
    searches = s1["searches"] - s0["searches"]
    touched = s1["nodes_touched"] - s0["nodes_touched"]
    search_ms = phases["search_kernel"][0]
    out = {"metric": "neuron-steps/s", "value": world * n * PERIOD * args.steps / (total_ms / 1e3), "unit": "neuron-steps/s",
           "precision": "fp64" if precision == 0 else "fp32", "ms_per_step": total_ms / args.steps, "neurons": n,
           "elements": "grown U[0, 4] per type at step 1 (vacant = floor)", "first_timed_step": step - PERIOD * args.steps,
           "timed_periods": args.steps, "edges": [edges_before, edges_after], "searches_per_update": searches / args.steps,
           "synapses_created_per_update": (s1["synapses_created"] - s0["synapses_created"]) / args.steps,
           "synapses_deleted_per_update": (s1["synapses_deleted"] - s0["synapses_deleted"]) / args.steps,
           "phases_ms": {k: v[0] for k, v in phases.items()}, "activity_roofline": act_roof,
           "period_ms": {"min": min(times), "median": float(np.median(times)), "max": max(times)}}
    if searches and search_ms > 0:
        tps = touched / searches if precision == 0 else None
        out["bh_searches_per_s"] = searches / (search_ms / 1e3)
        if tps:
            out["search_roofline"] = search_roofline(searches, tps, search_ms, precision)
    dom = max(("activity_kernel", "search_kernel", "connector", "graph", "commit", "tree_update"), key=lambda k: phases[k][0])
    out["dominant_phase"] = dom
    out["roofline"] = out.get("search_roofline") if dom == "search_kernel" and "search_roofline" in out else act_roof
    t = net.tuning()
    out["tuning"] = {k: t[k] for k in ("act_block", "act_persistent", "act_vec", "search_warps", "search_packet", "search_cap", "search_hot")}
    net.close()
    return out


def ensemble_spec(count, seed):
    """The batched configuration: `count` networks with sizes log-uniform in
    5,000-250,000 neurons, growth rates log-uniform in 1e-5-1e-3, theta from
    {0.2, 0.3, 0.5}, sigma from {500, 750, 1000} um, uniform placement at one
    neuron per 1000 um^3."""
    rng = np.random.default_rng(seed)
    nets = []
    for k in range(count):
        n = int(np.exp(rng.uniform(np.log(5_000), np.log(250_000))))
        nets.append(dict(num_neurons=n, seed=seed * 100_003 + k, side=(1000.0 * n) ** (1.0 / 3.0), theta=float(rng.choice([0.2, 0.3, 0.5])),
                         sigma=float(rng.choice([500.0, 750.0, 1000.0])), growth_rate=float(np.exp(rng.uniform(np.log(1e-5), np.log(1e-3))))))
    return nets


def ensemble_figure(args, dev, stream, world, rank):
    """128 networks in one FP32 context, each run for steps 1..5,000 (its
    stated length) with 50 plasticity updates: one launch per activity step
    (or per 100-step block while no network has synapses) over all networks,
    100-step blocks replayed as CUDA graphs, plasticity updates over all
    networks at once.  A first context of the same networks times the launch
    shapes (the tuner caches them per size class); a second one is timed from
    step 1 to the last step."""
    import torch

    import relearn_b200 as R
    from relearn_b200 import workloads

    nets = ensemble_spec(args.ensemble_networks, 7 + rank)
    base = R.default_params(1, 1.0)
    base["precision"] = 1
    base["device"] = dev.index
    total = sum(d["num_neurons"] for d in nets)
    pos = np.concatenate([workloads.uniform_cube(d["num_neurons"], d["side"], 900 + k) for k, d in enumerate(nets)])
    sig = np.concatenate([workloads.signal_types(d["num_neurons"], 900 + k) for k, d in enumerate(nets)])

    def make():
        e = R.Network(base, networks=nets)
        e.set_stream(stream.cuda_stream)
        e.set_positions(pos, sig)
        e.set_step_fusion(bool(args.step_fusion))
        e.autotune(1)
        return e

    warm = make()
    step = 1
    for _ in range(max(args.warmup, 3)):
        warm.simulate(step, PERIOD)
        step += PERIOD
    warm.close()
    ens = make()
    steps = args.ensemble_steps
    torch.cuda.synchronize(dev)
    if world > 1:
        torch.distributed.barrier()
    ens.phase_times()
    ens.set_profiling(True)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ens.simulate(1, steps)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1)
    ph = ens.phase_times()
    ens.set_profiling(False)
    ms = max_over_ranks(ms, world, dev)
    act_ms, act_cnt = ph["activity_kernel"]
    tuning = ens.tuning()
    st = ens.stats()
    hbm, peak_kind = peaks()
    ens.close()
    step_us = 1e3 * act_ms / steps
    if st["synapses_created"] == 0 and args.step_fusion:
        # no network formed a synapse: every block ran as one launch of the
        # batched block kernel, bound by instruction issue
        cap = captured("ensemble32")
        mhz = 1965.0
        achieved = cap["warp_instr_per_neuron"] * total / (step_us * 1e-6) / 1e12
        peak = 4 * B200_SMS * mhz * 1e6 / 1e12
        roof = {"bound": "issue", "kernel": "k_activity_f32_steps (batched: thread blocks of one network)", "achieved": achieved, "peak": peak,
                "unit": "T warp-inst/s", "frac": achieved / peak, "warp_instr_per_neuron_step": cap["warp_instr_per_neuron"], "stale": cap["stale"],
                "peak_kind": "nominal: 1 warp instruction per SM sub-partition per cycle x 592 at 1965 MHz", "avg_step_us": step_us,
                "traffic": cap["traffic"], "traffic_unit": "bytes per 100-step launch (ncu dram read + write)",
                "hbm": {"bytes_per_launch": FUSED_BYTES[1] * total, "achieved": FUSED_BYTES[1] * total / (step_us * PERIOD * 1e-6) / 1e9, "peak": hbm,
                        "unit": "GB/s", "frac": FUSED_BYTES[1] * total / (step_us * PERIOD * 1e-6) / 1e9 / hbm, "peak_kind": peak_kind}}
    else:
        bytes_per_step = step_bytes(1, total, 0)
        roof = {"bound": "hbm", "kernel": "k_activity_f32 / k_activity_f32_steps", "achieved": bytes_per_step / (step_us * 1e-6) / 1e9, "peak": hbm,
                "unit": "GB/s", "frac": bytes_per_step / (step_us * 1e-6) / 1e9 / hbm, "peak_kind": peak_kind, "bytes_per_step": bytes_per_step,
                "avg_step_us": step_us, "activity_launches": act_cnt,
                "note": "per activity step over the whole run: fused 100-step blocks while no network has synapses, one launch per step after"}
    return {"metric": "neuron-steps/s", "value": world * total * steps / (ms / 1e3), "unit": "neuron-steps/s", "networks": len(nets),
            "neurons": total, "steps": steps, "steps_of_config": 5000, "precision": "fp32", "timed": "steps 1..%d of a fresh context" % steps,
            "synapses_created": st["synapses_created"], "searches": st["searches"], "roofline": roof,
            "phases_ms": {k: v[0] for k, v in ph.items()}, "tuning": tuning}


def precision_report(args, dev, stream, n=4_000_000, side=16_000.0, steps=1000, sources=64):
    """The precision form against the FP64 drop-in on the same seed: 4M neurons
    uniform in a 16,000 um cube, 1,000 steps.  Reports selection-probability
    error, calcium drift and the chi-square of the formed-synapse distance
    histograms of one search per neuron on the same snapshot."""
    import torch

    import relearn_b200 as R

    params, pos, sig = build_network(n, side, 11, "uniform")
    params["device"] = dev.index
    out = {"neurons": n, "side_um": side, "steps": steps}
    nets = []
    for prec in (0, 1):
        p = dict(params)
        p["precision"] = prec
        net = R.Network(p)
        net.set_stream(stream.cuda_stream)
        net.set_positions(pos, sig)
        net.simulate(1, steps)
        nets.append(net)
    ca64 = nets[0].neurons()["calcium"]
    ca32 = nets[1].neurons()["calcium"]
    rel = np.abs(ca32 - ca64) / np.maximum(np.abs(ca64), 1e-300)
    fired_rate = [float(x.neurons()["fired"].mean()) for x in nets]
    out["calcium_drift"] = {"max_rel": float(rel.max()), "mean_rel": float(rel.mean()), "mean_fp64": float(ca64.mean()), "mean_fp32": float(ca32.mean()),
                            "mean_rel_of_means": float(abs(ca32.mean() - ca64.mean()) / ca64.mean())}
    out["last_step_fired_fraction"] = fired_rate
    # same snapshot in both forms: one vacant axon and dendrite of each type
    one = np.ones(n, np.uint32)
    for net in nets:
        for t in range(3):
            net.set_elements(t, np.full(n, 1.5), np.zeros(n), np.zeros(n, np.uint32), one)
        net.prepare_update_connectivity(one, one, one)
    rng = np.random.default_rng(5)
    worst, tv = 0.0, 0.0
    for src in rng.choice(n, sources, replace=False):
        n64, w64 = nets[0].candidate_weights(int(src), 0)
        n32, w32 = nets[1].candidate_weights(int(src), 1)
        p64 = dict(zip(n64.tolist(), (w64 / w64.sum()).tolist()))
        p32 = dict(zip(n32.tolist(), (w32 / w32.sum()).tolist()))
        keys = set(p64) | set(p32)
        tv = max(tv, 0.5 * sum(abs(p64.get(k, 0.0) - p32.get(k, 0.0)) for k in keys))
        for k, v in p64.items():
            if v >= 1e-6:
                worst = max(worst, abs(p32.get(k, 0.0) - v) / v)
    out["selection_probability"] = {"max_rel_err_p_ge_1e-6": worst, "max_total_variation": tv, "sources": sources, "descent": "first (from the root)"}
    hist = []
    edges = np.linspace(0.0, 3 * 750.0, 46)
    for net in nets:
        req = net.find_targets(100)
        d = np.linalg.norm(pos[req["source"]] - pos[req["target"]], axis=1)
        h, _ = np.histogram(d, bins=edges)
        hist.append(h.astype(np.float64))
    a, b = hist
    m = (a + b) > 0
    chi2 = float(np.sum((a[m] - b[m]) ** 2 / (a[m] + b[m])))
    from scipy.stats import chi2 as chi2_dist

    out["distance_histogram"] = {"bins": int(m.sum()), "chi2": chi2, "dof": int(m.sum()) - 1, "p_value": float(chi2_dist.sf(chi2, int(m.sum()) - 1)),
                                 "synapses": [int(a.sum()), int(b.sum())], "bin_um": float(edges[1] - edges[0])}
    for net in nets:
        net.close()
    return out


def serve_figure(args, dev):
    """The serving form: a seeded Poisson stream of sweep requests (20 per
    second; each one network of log-uniform 2,000-1,000,000 neurons with its own
    seed, growth rate log-uniform 1e-5-1e-3 and theta uniform 0.2-0.5, run for
    5,000 steps) submitted in real time to the native request loop, which admits
    them against a 150 GB HBM budget as slots free up, overlaps them on the GPU
    and packs small pending ones into batched contexts.  Reports p50 / p99
    completion latency (submission to result) and aggregate neuron-steps/s."""
    import relearn_b200 as R
    from relearn_b200 import workloads
    from relearn_b200.serving import Server, latency_summary

    prec = 1 if args.serve_precision == "fp32" else 0
    params = R.default_params(1, 1.0)
    params["precision"] = prec
    params["device"] = dev.index
    reqs = workloads.serving_stream(args.seed + 17, args.serve_rate, args.serve_seconds, steps=args.serve_steps)
    budget = 150e9
    done, max_running, max_reserved, max_pending, lag = [], 0, 0, 0, 0.0
    with Server(params, hbm_budget_bytes=budget, slots=args.serve_slots, pack_networks=16, pack_max_neurons=65_536) as srv:
        t0 = time.perf_counter()
        for t_arr, net in reqs:
            pos, sig = workloads.request_inputs(net)
            while True:
                wait = t_arr - (time.perf_counter() - t0)
                if wait <= 0:
                    break
                done += srv.poll(wait_ms=max(1, int(min(wait, 0.05) * 1e3)))
            lag = max(lag, time.perf_counter() - t0 - t_arr)
            srv.submit(net, pos, sig, net["steps"])
            p, r, b = srv.load()
            max_pending, max_running, max_reserved = max(max_pending, p), max(max_running, r), max(max_reserved, b)
        while len(done) < len(reqs):
            done += srv.poll(wait_ms=200)
            p, r, b = srv.load()
            max_pending, max_running, max_reserved = max(max_pending, p), max(max_running, r), max(max_reserved, b)
    # capacity: the same requests submitted at once, so the GPU never waits for arrivals
    burst = []
    with Server(params, hbm_budget_bytes=budget, slots=args.serve_slots, pack_networks=16, pack_max_neurons=65_536) as srv:
        for _, net in reqs:
            pos, sig = workloads.request_inputs(net)
            srv.submit(net, pos, sig, net["steps"])
        while len(burst) < len(reqs):
            burst += srv.poll(wait_ms=200)
    cap = latency_summary(burst)
    bad = [d for d in done + burst if d["status"] != 0]
    summ = latency_summary(done)
    hbm, peak_kind = peaks()
    per_ns = ACT_BYTES_FP32 if prec else ACT_BYTES_PER_NEURON
    achieved = summ["neuron_steps_per_s"] * per_ns / 1e9
    offered = sum(d["num_neurons"] * d["steps"] for _, d in reqs) / args.serve_seconds
    packs = [d["pack_size"] for d in done]
    return {"metric": "p50/p99 completion latency; aggregate neuron-steps/s", "p50_s": summ["p50_s"], "p99_s": summ["p99_s"],
            "max_s": summ["max_s"], "value": summ["neuron_steps_per_s"], "unit": "neuron-steps/s", "requests": len(done), "failed": len(bad),
            "precision": "fp32" if prec else "fp64", "arrivals": f"Poisson {args.serve_rate:g}/s over {args.serve_seconds:g} s (seeded)",
            "sample": f"the first {args.serve_seconds:g} s of the 600 s stream", "fraction_of_stream": args.serve_seconds / 600.0,
            "steps_per_request": args.serve_steps,
            "offered_neuron_steps_per_s": offered, "span_s": summ["span_s"], "mean_queue_s": summ["mean_queue_s"], "p99_queue_s": summ["p99_queue_s"],
            "slots": args.serve_slots, "hbm_budget_bytes": budget, "max_running": max_running, "max_pending": max_pending,
            "max_reserved_bytes": max_reserved, "mean_pack_size": float(np.mean(packs)), "max_pack_size": int(max(packs)),
            "max_peak_over_footprint": max(d["device_peak_bytes"] / d["footprint_bytes"] for d in done if d["pack_size"] == 1)
            if any(d["pack_size"] == 1 for d in done) else None,
            "max_submit_lag_s": lag,
            "capacity": {"neuron_steps_per_s": cap["neuron_steps_per_s"], "span_s": cap["span_s"],
                         "how": "the same requests submitted at once; aggregate over first submission to last result"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind,
                         "bytes_per_neuron_step": per_ns}}


def search_roofline(searches: float, touched_per_search: float, kernel_ms: float, precision: int) -> dict:
    """The search against HBM by algorithmic bytes (acceptance tests the
    reference's walk runs x the node bytes of one test), with the bound that
    actually holds beside it: the walk is served from L1 / L2 (ncu DRAM bytes
    per search are far below the algorithmic ones), so instruction issue with
    idle lanes bounds it."""
    hbm, peak_kind = peaks()
    cap = captured("search64" if precision == 0 else "search32")
    bytes_per_search = touched_per_search * SEARCH_BYTES_PER_NODE
    achieved = searches * bytes_per_search / (kernel_ms * 1e-3) / 1e9
    return {"bound": "issue (walk served from L1/L2)", "kernel": "k_search" if precision == 0 else "k_search_f32", "achieved": achieved,
            "peak": hbm, "unit": "GB/s", "frac": achieved / hbm, "peak_kind": peak_kind, "touched_per_search": touched_per_search,
            "bytes_per_touched_node": SEARCH_BYTES_PER_NODE, "lanes_active_of_32": cap["lanes_active"], "l1_hit_rate": cap["l1_hit"],
            "l2_hit_rate": cap["l2_hit"], "stale": cap["stale"],
            "how": "touched nodes from the library's counter (the acceptance tests the reference's walk runs) x bytes per node / search-kernel "
                   "time; lanes active and hit rates from ncu on the 1M snapshot"}


def bh_snapshot(net, n, stream, step, precision=0, touched_per_search=None):
    import torch

    one = np.ones(n, np.uint32)
    grown = np.full(n, 1.5)
    reps = 3
    search_ms = []
    update_ms = []
    t0 = net.stats()["nodes_touched"]
    for r in range(reps + 1):
        for t in range(3):
            net.set_elements(t, grown, np.zeros(n), np.zeros(n, np.uint32), one)
        net.set_profiling(True)
        net.phase_times()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        net.prepare_update_connectivity(one, one, one)
        net.find_targets(step)
        e1.record(stream)
        e1.synchronize()
        ph = net.phase_times()
        net.set_profiling(False)
        if r > 0:
            search_ms.append(ph["search_kernel"][0])
            update_ms.append(e0.elapsed_time(e1))
    searches = n
    if precision == 0:
        touched_per_search = (net.stats()["nodes_touched"] - t0) / ((reps + 1) * searches)
    t = net.tuning()
    out = {"metric": "BH searches/s", "value": searches / (min(search_ms) / 1e3), "unit": "searches/s",
           "with_tree_update_and_copies": searches / (min(update_ms) / 1e3), "searches_per_update": searches,
           "search_kernel_ms": min(search_ms), "update_ms": min(update_ms), "snapshot": "1 vacant axon + 1 vacant exc + 1 vacant inh dendrite per neuron",
           "search_shape": {"warps_per_block": t["search_warps"], "packet": t["search_packet"], "register_cap": t["search_cap"], "hot_nodes": t["search_hot"],
                            "timed_ms": t["search_ms"]}}
    if touched_per_search:
        out["roofline"] = search_roofline(searches, touched_per_search, min(search_ms), precision)
        if precision == 1:
            out["roofline"]["touched_from"] = "the FP64 form's counter on the same snapshot (the same walk)"
    return out


def cpu_baseline(args, params, pos, sig, activity_steps=1000, searches=100000):
    """The oracle (C++ restatement of the reference's CPU path, OpenMP) on all
    host cores: a bounded sample of the same workload (1,000 activity steps with
    their 10 plasticity updates, about 10 s on 16 cores, and 100,000 searches
    of the search snapshot)."""
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    p = dict(params)
    p.pop("device", None)
    p["use_libm"] = 0
    sim = O.OracleSim(p, pos, sig, threads=threads)
    steps = activity_steps
    t0 = time.perf_counter()
    sim.simulate(1, steps)  # includes the plasticity updates at steps 100, 200, ...
    dt = time.perf_counter() - t0
    n = params["num_neurons"]
    out = {"value": n * steps / dt, "unit": "neuron-steps/s", "cores": threads, "kind": "port",
           "sample": f"{n} neurons, {steps} activity steps incl. {steps // PERIOD} plasticity updates ({dt:.1f} s)"}
    # search snapshot on a subset of sources
    one = np.ones(n, np.uint32)
    sel = np.zeros(n, np.uint32)
    rng = np.random.default_rng(0)
    sel[rng.choice(n, size=min(searches, n), replace=False)] = 1
    for t in range(3):
        sim.set_elements(t, np.full(n, 1.5), np.zeros(n), np.zeros(n, np.uint32), sel if t == 0 else one)
    sim.update_tree(one, one)
    t0 = time.perf_counter()
    req = sim.find_targets(step := 100)
    ds = time.perf_counter() - t0
    out["bh_searches_per_s"] = int(sel.sum()) / ds
    out["bh_sample"] = f"{int(sel.sum())} searches on the snapshot ({ds:.1f} s)"
    return out


def run_reference(args, world, rank):
    if rank != 0:
        return None
    params, pos, sig = build_network(args.neurons, args.side, args.seed, args.placement)
    from oracle import oracle as O

    threads = os.cpu_count() or 1
    p = dict(params)
    p.pop("device", None)
    p["use_libm"] = 0
    sim = O.OracleSim(p, pos, sig, threads=threads)
    # each step is the bench step itself: 100 activity steps and the
    # plasticity update at the end of them
    sample_steps = PERIOD
    step = 1
    for _ in range(args.warmup):
        sim.simulate(step, sample_steps)
        step += sample_steps
    t0 = time.perf_counter()
    for _ in range(args.steps):
        sim.simulate(step, sample_steps)
        step += sample_steps
    dt = time.perf_counter() - t0
    value = args.neurons * sample_steps * args.steps / dt
    return {
        "impl": "reference",
        "metric": "neuron-steps/s",
        "value": value,
        "unit": "neuron-steps/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic (seeded positions, reference parameters)",
        "config": bench_config(args, world, 1 if args.precision == "fp32" else 0),
        "cpu_baseline": {"value": value, "unit": "neuron-steps/s", "cores": threads, "kind": "port",
                         "sample": f"the bench step itself: {sample_steps} activity steps of {args.neurons} neurons and 1 plasticity update, "
                                   f"{args.steps} timed after {args.warmup} warm-up"},
        "e2e": {"value": value, "unit": "neuron-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_case(args):
    """Small cases for kernel profiles: `activity` runs --case-steps (4)
    activity steps of a network of --neurons neurons (no octree needed; a
    network without synapses runs them as one launch of the block kernel
    unless --step-fusion 0); `search` runs the search
    snapshot (one vacant axon and dendrite of each type per neuron, or a vacant
    axon on --search-sources random neurons only) once;
    `plasticity` seeds 0-3 elements per type and runs two plasticity periods
    (100 activity steps + 1 plasticity update each); `ensemble` runs
    --case-steps activity steps of the batched configuration (--ensemble-networks
    networks; the bench measures it in the FP32 form, --precision fp32)."""
    import relearn_b200 as R

    if args.case == "ensemble":
        from relearn_b200 import workloads

        nets = ensemble_spec(args.ensemble_networks, 7)
        base = R.default_params(1, 1.0)
        base["precision"] = 1 if args.precision == "fp32" else 0
        ens = R.Network(base, networks=nets)
        ens.set_positions(np.concatenate([workloads.uniform_cube(d["num_neurons"], d["side"], 900 + k) for k, d in enumerate(nets)]),
                          np.concatenate([workloads.signal_types(d["num_neurons"], 900 + k) for k, d in enumerate(nets)]))
        ens.set_step_fusion(bool(args.step_fusion))
        ens.activity_block(1, args.case_steps)
        ens.synchronize()
        print(json.dumps({"case": args.case, "networks": len(nets), "neurons": int(sum(d["num_neurons"] for d in nets)), "stats": ens.stats()}))
        return
    params, pos, sig = build_network(args.neurons, args.side, args.seed, args.placement)
    params["precision"] = 1 if args.precision == "fp32" else 0
    net = R.Network(params)
    if args.act_shape or args.search_shape:
        apply_shapes(args, net, params["precision"])
    net.set_step_fusion(bool(args.step_fusion))
    if args.case == "activity":
        net.activity_block(1, args.case_steps)
    elif args.case == "plasticity":
        from relearn_b200 import workloads

        net.set_positions(pos, sig)
        for t, (g, v) in enumerate(workloads.initial_elements(args.neurons, 3, 0.0, 3.0)):
            net.set_elements(t, g, np.zeros(args.neurons), np.zeros(args.neurons, np.uint32), v)
        net.simulate(1, 200)
    else:
        net.set_positions(pos, sig)
        one = np.ones(args.neurons, np.uint32)
        axons = one
        if args.search_sources:
            # a sparse search list: a vacant axon on that many neurons drawn at random
            axons = np.zeros(args.neurons, np.uint32)
            axons[np.random.default_rng(3).choice(args.neurons, args.search_sources, replace=False)] = 1
        for t in range(3):
            net.set_elements(t, np.full(args.neurons, 1.5), np.zeros(args.neurons), np.zeros(args.neurons, np.uint32), axons if t == 0 else one)
        net.prepare_update_connectivity(axons, one, one)
        req = net.find_targets(100)
        print(json.dumps({"case": "search", "searches": int(axons.sum()), "requests": int(len(req))}))
    net.synchronize()
    print(json.dumps({"case": args.case, "neurons": args.neurons, "stats": net.stats()}))


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--neurons", type=int, default=N_DEFAULT)
    ap.add_argument("--side", type=float, default=SIDE_DEFAULT)
    ap.add_argument("--placement", choices=["uniform", "mixture"], default="uniform")
    ap.add_argument("--seed", type=int, default=1)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--skip-bh", action="store_true")
    ap.add_argument("--skip-fp32", action="store_true", help="do not measure the FP32 form beside the FP64 drop-in")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64", help="form of the headline figure")
    ap.add_argument("--skip-ensemble", action="store_true", help="do not measure the batched form (128 networks)")
    ap.add_argument("--skip-mixture", action="store_true", help="do not measure the Gaussian-mixture placement beside the uniform one")
    ap.add_argument("--ensemble-networks", type=int, default=128)
    ap.add_argument("--skip-precision-report", action="store_true", help="do not run the FP32-vs-FP64 error report (4M neurons, 1,000 steps)")
    ap.add_argument("--skip-synapses", action="store_true", help="do not measure the regime with synapses (elements seeded U[0, 4])")
    ap.add_argument("--ensemble-steps", type=int, default=5000, help="steps of every network of the batched form (config: 5,000)")
    ap.add_argument("--skip-serve", action="store_true", help="do not measure the serving form")
    ap.add_argument("--act-shape", default=None, help="activity launch shape 'block,persistent,vec' instead of the tuner's")
    ap.add_argument("--search-shape", default=None, help="search launch shape 'warps,packet[,cap[,hot]]' instead of the tuner's")
    ap.add_argument("--serve-seconds", type=float, default=30.0, help="length of the Poisson request stream (the full one is 600 s)")
    ap.add_argument("--serve-rate", type=float, default=20.0)
    ap.add_argument("--serve-steps", type=int, default=5000)
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-precision", choices=["fp64", "fp32"], default="fp32")
    ap.add_argument("--step-fusion", type=int, choices=[0, 1], default=1,
                    help="1: blocks of activity steps of a network without synapses in one launch (default); 0: one launch per step")
    ap.add_argument("--case-steps", type=int, default=4, help="activity steps of --case activity")
    ap.add_argument("--search-sources", type=int, default=0, help="--case search: vacant axons on this many random neurons (0: on every neuron)")
    ap.add_argument("--case", choices=["activity", "search", "plasticity", "ensemble"], default=None,
                    help="run a small profiling case of one kernel instead of the benchmark")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    if args.case:
        run_case(args)
        return
    if args.impl == "reference":
        line = run_reference(args, world, rank)
    else:
        line = run_b200(args, world, rank, local)
    if line is not None and rank == 0:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
