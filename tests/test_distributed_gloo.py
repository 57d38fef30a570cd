"""The split-network Barnes-Hut update (relearn_b200.distributed) on gloo
ranks on the CPU, each rank's engine the oracle: two and three ranks form the
same synapses, leave the same element counts and hold the same in-edges as
one rank running the whole network, over three plasticity updates with
vacancies that change between them.

This checks the host side of the multi-rank path — the tree replication by
all-gathered leaf counts, the search restricted to a rank's own sources, the
routing of requests to the targets' ranks and of responses back, and the
local / distant-in / distant-out split of the result (the reference's
ForwardCPUAlgorithm::update_connectivity, algorithm/Internal/ExchangingAlgorithm.h:58-87)."""
import datetime
import os
import socket

import numpy as np
import pytest

from conftest import ROOT, oracle_params, small_network

N = 1500
STEPS = (100, 200, 300)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


class OracleEngine:
    """The oracle in the engine role of DistributedBarnesHut (a context over
    every neuron's position)."""

    def __init__(self, params, pos, sig):
        from oracle import oracle as O

        self.sim = O.OracleSim(oracle_params(params), pos, sig)
        self.n = len(sig)

    def prepare_update_connectivity(self, va, ve, vi, signal=None, update=None):
        e = self.sim.get_elements(0)
        self.sim.set_elements(0, e["grown"], e["delta"], e["connected"], va)
        for t, v in ((1, ve), (2, vi)):
            e = self.sim.get_elements(t)
            self.sim.set_elements(t, e["grown"], e["delta"], e["connected"], v)
        self.sim.update_tree(ve, vi)

    def find_targets(self, step):
        return self.sim.find_targets(step)

    def process_requests(self, step, requests):
        return self.sim.process_requests(step, requests)

    def process_responses(self, requests, accepted, append):
        return self.sim.process_responses(requests, accepted, append)

    def edges(self):
        return self.sim.edges()


def initial_vacancy(n, seed):
    rng = np.random.default_rng(seed)
    return [rng.integers(0, 4, n).astype(np.uint32) for _ in range(3)]


def extra_vacancy(n, step):
    """Elements that grow between updates (the same draw on every rank)."""
    rng = np.random.default_rng(step)
    return [(rng.random(n) < 0.2).astype(np.uint32) for _ in range(3)]


def apply(vac, lo, hi, synapses, target_side, source_side):
    for r in synapses:
        t, s, sig = int(r["target"]), int(r["source"]), int(r["signal"])
        if target_side:
            assert lo <= t < hi
            vac[1 + sig][t - lo] -= 1
        if source_side:
            assert lo <= s < hi
            vac[0][s - lo] -= 1


def _rank(rank, world, port, out):
    import sys

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from relearn_b200.distributed import Communicator, DistributedBarnesHut, RankLayout

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        params, pos, sig = small_network(N, 1400.0, 31, True)
        layout = RankLayout(N, world)
        lo, hi = layout.range(rank)
        alg = DistributedBarnesHut(OracleEngine(params, pos, sig), layout, Communicator())
        vac = [v[lo:hi].copy() for v in initial_vacancy(N, 5)]
        formed = []
        kinds = [0, 0, 0]
        for step in STEPS:
            alg.prepare_update_connectivity(sig[lo:hi], vac[0], vac[1], vac[2])
            res = alg.update_connectivity(step)
            assert res.number_created_synapses == len(res.local_synapses) + len(res.distant_in_synapses)
            apply(vac, lo, hi, res.local_synapses, True, True)
            apply(vac, lo, hi, res.distant_in_synapses, True, False)
            apply(vac, lo, hi, res.distant_out_synapses, False, True)
            formed += [(int(r["target"]), int(r["source"]), int(r["j"]), int(r["signal"]), step)
                       for r in np.concatenate([res.local_synapses, res.distant_in_synapses])]
            kinds = [kinds[0] + len(res.local_synapses), kinds[1] + len(res.distant_in_synapses), kinds[2] + len(res.distant_out_synapses)]
            for t, x in enumerate(extra_vacancy(N, step)):
                vac[t] += x[lo:hi]
        e = alg.engine.edges()
        own = (e[0] >= lo) & (e[0] < hi)
        out.put((rank, formed, [v.tolist() for v in vac], kinds, [a[own].tolist() for a in e]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


def single_rank():
    """The whole network in one oracle with the one-rank connector."""
    params, pos, sig = small_network(N, 1400.0, 31, True)
    eng = OracleEngine(params, pos, sig)
    vac = initial_vacancy(N, 5)
    formed = []
    for step in STEPS:
        eng.prepare_update_connectivity(vac[0], vac[1], vac[2])
        req = eng.find_targets(step)
        _, acc = eng.sim.connect_requests(step, req)
        ok = req[acc.astype(bool)]
        apply(vac, 0, N, ok, True, True)
        formed += [(int(r["target"]), int(r["source"]), int(r["j"]), int(r["signal"]), step) for r in ok]
        for t, x in enumerate(extra_vacancy(N, step)):
            vac[t] += x
    return formed, vac, eng.edges()


@pytest.mark.parametrize("world", [2, 3])
def test_split_network_matches_one_rank(world, oracle_mod):
    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=300) for _ in range(world)]
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    got.sort()
    formed_ref, vac_ref, edges_ref = single_rank()
    assert len(formed_ref) > 200
    formed = sorted(sum((g[1] for g in got), []))
    assert formed == sorted(formed_ref)
    for t in range(3):
        assert np.array_equal(np.concatenate([np.asarray(g[2][t], np.uint32) for g in got]), vac_ref[t]), t
    # every rank holds the in-edges of its own neurons
    for k in range(3):
        assert np.array_equal(np.concatenate([np.asarray(g[4][k]) for g in got]), edges_ref[k])
    local = sum(g[3][0] for g in got)
    distant_in = sum(g[3][1] for g in got)
    distant_out = sum(g[3][2] for g in got)
    assert distant_in == distant_out > 0 and local > 0
    assert local + distant_in == len(formed_ref)
