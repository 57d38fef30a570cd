"""The split-network Barnes-Hut update on the device, through the C ABI
(rl_find_targets over a rank's own sources, rl_process_requests on the
targets' rank, rl_process_responses on the sources' rank): two ranks as two
processes exchanging over gloo, each with its own context on the one device
(their kernels never wait on each other: the exchange runs on the host), and
one NCCL rank through the device-side collectives.  Both form the synapses
and leave the element counts and in-edges of one context running the whole
network."""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import ROOT, small_network

pytestmark = pytest.mark.gpu

N = 6000
STEPS = (100, 200, 300)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def initial_vacancy(n, seed):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, 4, n).astype(np.uint32) for _ in range(3)]


def extra_vacancy(n, step):
    rng = np.random.default_rng(step)
    return [(rng.random(n) < 0.2).astype(np.uint32) for _ in range(3)]


def _rank(rank, world, port, backend, out):
    import sys

    import torch
    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from relearn_b200 import Network
    from relearn_b200.distributed import Communicator, DistributedBarnesHut, RankLayout

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    device = "cpu"
    if backend == "nccl":
        torch.cuda.set_device(0)
        device = "cuda:0"
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        params, pos, sig = small_network(N, 2000.0, 41, True)
        layout = RankLayout(N, world)
        lo, hi = layout.range(rank)
        net = Network(params)
        net.set_positions(pos, sig)
        alg = DistributedBarnesHut(net, layout, Communicator(device=device))
        vac = [v[lo:hi].copy() for v in initial_vacancy(N, 7)]
        formed = []
        for step in STEPS:
            alg.prepare_update_connectivity(sig[lo:hi], vac[0], vac[1], vac[2])
            res = alg.update_connectivity(step)
            for r in np.concatenate([res.local_synapses, res.distant_in_synapses]):
                vac[1 + int(r["signal"])][int(r["target"]) - lo] -= 1
                formed.append((step, int(r["target"]), int(r["source"]), -1 if r["signal"] else 1))
            for r in np.concatenate([res.local_synapses, res.distant_out_synapses]):
                vac[0][int(r["source"]) - lo] -= 1
            for t, x in enumerate(extra_vacancy(N, step)):
                vac[t] += x[lo:hi]
        # the context's own counts of this rank's neurons follow the same updates
        for t in range(3):
            assert np.array_equal(net.get_elements(t)["vacant"][lo:hi] + (extra_vacancy(N, STEPS[-1])[t][lo:hi]), vac[t]), t
        e = net.edges()
        own = (e[0] >= lo) & (e[0] < hi)
        out.put((rank, formed, [v.tolist() for v in vac], [a[own].tolist() for a in e]))
        net.close()
        dist.barrier()
    finally:
        dist.destroy_process_group()


def one_context():
    from relearn_b200 import Network

    params, pos, sig = small_network(N, 2000.0, 41, True)
    net = Network(params)
    net.set_positions(pos, sig)
    vac = initial_vacancy(N, 7)
    formed = []
    for step in STEPS:
        net.prepare_update_connectivity(vac[0], vac[1], vac[2], signal=sig)
        syn = net.update_connectivity(step)
        for r in syn:
            vac[1 + (1 if r["weight"] < 0 else 0)][int(r["target"])] -= 1
            vac[0][int(r["source"])] -= 1
            formed.append((step, int(r["target"]), int(r["source"]), int(r["weight"])))
        for t, x in enumerate(extra_vacancy(N, step)):
            vac[t] += x
    e = net.edges()
    net.close()
    return formed, vac, e


def run_ranks(world, backend):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, backend, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=600) for _ in range(world))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    return got


@pytest.mark.parametrize("world,backend", [(2, "gloo"), (1, "nccl")])
def test_split_network_on_device_matches_one_context(world, backend):
    got = run_ranks(world, backend)
    formed_ref, vac_ref, edges_ref = one_context()
    assert len(formed_ref) > 1000
    assert sorted(sum((g[1] for g in got), [])) == sorted(formed_ref)
    for t in range(3):
        assert np.array_equal(np.concatenate([np.asarray(g[2][t], np.uint32) for g in got]), vac_ref[t]), t
    for k in range(3):
        assert np.array_equal(np.concatenate([np.asarray(g[3][k]) for g in got]), edges_ref[k]), k
