"""Barnes-Hut connectivity update of one network split over ranks.

The reference's multi-rank path: every MPI rank owns a share of the neurons,
searches targets for its own vacant axons over the distributed octree
(BarnesHut::find_target_neurons, algorithm/BarnesHutInternal/BarnesHut.cpp:36-94,
descending into other ranks' subtrees through BarnesHutBase.h:311-427), sends
each request to the rank owning its target, which runs the target half of the
connector (ForwardConnector::process_requests, algorithm/Connector.cpp:33-117)
and answers; the source rank then binds its axons
(ForwardConnector::process_responses, Connector.cpp:119-197).  The sequence is
ForwardCPUAlgorithm::update_connectivity
(algorithm/Internal/ExchangingAlgorithm.h:58-87) and its result the
reference's ConnectivityUpdateResult {count, local, distant_in, distant_out}
(algorithm/Algorithm.h:37-42).

Here, one process per GPU, over torch.distributed (NCCL between GPUs, gloo
on the CPU):

* Positions are static, so every rank builds the octree over all neurons
  once (the same tree everywhere: its construction is deterministic).
* At each plasticity update the ranks all-gather their neurons' vacant
  dendrite counts and plasticity flags (9 bytes per neuron) and every rank
  runs the leaf update and the bottom-up reduction of the whole tree itself:
  the replicated tree is bit for bit the single-rank tree, and no octree node
  ever crosses the interconnect.
* Each rank searches for its own sources only (the other ranks' axon counts
  are zero in its context).  Neuron ids are global, so every draw — the pick of
  each descent, the connector's processing key — is the one a single context
  makes.
* Requests go to the rank owning their target with one all-to-all; the
  owner's connector accepts in the keyed order, which for one target depends
  only on the requests for that target, so the accepted set is the
  single-rank one; the responses return with a second all-to-all.

Ownership is a partition of the global ids into contiguous blocks
(`RankLayout`); ids in spatial order make each block a subdomain, as the
reference's ranks own subdomains, but any order gives the same synapses.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from . import REQUEST_DTYPE

__all__ = ["RankLayout", "Communicator", "DistributedBarnesHut", "DistributedConnectivityResult"]


class RankLayout:
    """Neuron ownership: rank r owns the global ids [bounds[r], bounds[r + 1])."""

    def __init__(self, num_neurons: int, world: int, bounds: Optional[np.ndarray] = None):
        if world < 1:
            raise ValueError("world size must be at least 1")
        if bounds is None:
            bounds = np.array([num_neurons * r // world for r in range(world + 1)], np.int64)
        bounds = np.asarray(bounds, np.int64)
        if len(bounds) != world + 1 or bounds[0] != 0 or bounds[-1] != num_neurons or np.any(np.diff(bounds) < 0):
            raise ValueError("bounds must rise from 0 to the neuron count, one block per rank")
        self.n = int(num_neurons)
        self.world = int(world)
        self.bounds = bounds

    def range(self, rank: int) -> tuple:
        return int(self.bounds[rank]), int(self.bounds[rank + 1])

    def count(self, rank: int) -> int:
        lo, hi = self.range(rank)
        return hi - lo

    def owner(self, ids) -> np.ndarray:
        ids = np.asarray(ids, np.int64)
        return (np.searchsorted(self.bounds, ids, side="right") - 1).astype(np.int64)


class Communicator:
    """The two collectives of the update over a torch.distributed process
    group: an all-gather of per-neuron arrays and an all-to-all of variable
    length.  Tensors live on `device` (a CUDA device for NCCL, the CPU for
    gloo); arrays go in and come out as numpy."""

    def __init__(self, group=None, device: str = "cpu"):
        import torch.distributed as dist

        self.dist = dist
        self.group = group
        self.rank = dist.get_rank(group)
        self.world = dist.get_world_size(group)
        self.device = device

    def _tensor(self, a: np.ndarray):
        import torch

        return torch.from_numpy(np.ascontiguousarray(a)).to(self.device)

    def all_gather_blocks(self, local: np.ndarray, layout: RankLayout) -> np.ndarray:
        """Every rank's block (layout.count(r) entries of one dtype, as int32
        words) concatenated in rank order."""
        import torch

        local = np.ascontiguousarray(local)
        width = max(layout.count(r) for r in range(layout.world))
        words = np.zeros(width, np.int32)
        words[: len(local)] = local.astype(np.int64).astype(np.int32)
        out = torch.empty(width * self.world, dtype=torch.int32, device=self.device)
        self.dist.all_gather_into_tensor(out, self._tensor(words), group=self.group)
        allw = out.cpu().numpy().reshape(self.world, width)
        return np.concatenate([allw[r, : layout.count(r)] for r in range(self.world)])

    def all_to_all(self, send_words: np.ndarray, send_counts: np.ndarray, width: int):
        """Rows of `width` int32 words: send_counts[r] rows to rank r (rows
        grouped by destination, in rank order).  Returns the received rows,
        grouped by source rank, and the per-rank counts."""
        import torch

        send_counts = np.asarray(send_counts, np.int64)
        counts_out = torch.empty(self.world, dtype=torch.int64, device=self.device)
        self.dist.all_to_all_single(counts_out, self._tensor(send_counts), group=self.group)
        recv_counts = counts_out.cpu().numpy().astype(np.int64)
        total = int(recv_counts.sum())
        out = torch.empty(max(total * width, 1), dtype=torch.int32, device=self.device)
        send = np.ascontiguousarray(send_words, np.int32).reshape(-1)
        if len(send) == 0:
            send = np.zeros(1, np.int32)  # splits of zero still need a buffer
        self.dist.all_to_all_single(out[: total * width] if total else out[:0], self._tensor(send)[: int(send_counts.sum()) * width],
                                    output_split_sizes=[int(c) * width for c in recv_counts],
                                    input_split_sizes=[int(c) * width for c in send_counts], group=self.group)
        return out[: total * width].cpu().numpy().reshape(total, width), recv_counts


@dataclass
class DistributedConnectivityResult:
    """ConnectivityUpdateResult (algorithm/Algorithm.h:37-42) of one rank:
    the synapses created on this rank (local: both ends here; distant_in: the
    target here, the source elsewhere) and distant_out (the source here, the
    target elsewhere), as request records (target, source, j, signal) with
    global ids."""

    number_created_synapses: int
    local_synapses: np.ndarray = field(default_factory=lambda: np.zeros(0, REQUEST_DTYPE))
    distant_in_synapses: np.ndarray = field(default_factory=lambda: np.zeros(0, REQUEST_DTYPE))
    distant_out_synapses: np.ndarray = field(default_factory=lambda: np.zeros(0, REQUEST_DTYPE))


def _rows(req: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(req, REQUEST_DTYPE).view(np.uint32).reshape(-1, 4).view(np.int32)


def _requests(rows: np.ndarray) -> np.ndarray:
    return np.ascontiguousarray(rows, np.int32).view(np.uint32).reshape(-1).view(REQUEST_DTYPE).copy()


class DistributedBarnesHut:
    """The ``barnes-hut`` Algorithm of one rank of a split network.

    `engine` is this rank's context over all neurons' positions (a
    relearn_b200.Network on which set_positions has run); `layout` says which
    neurons the rank owns.  As in the reference, the caller owns its neurons'
    synaptic elements: it passes their vacant counts to
    prepare_update_connectivity and applies the result (a dendrite of the
    target for local and distant_in synapses, an axon of the source for local
    and distant_out ones).  The engine's own element counts of the owned
    neurons follow the same updates, and its synapse list holds the local,
    distant-in and distant-out synapses."""

    algorithm_type = "barnes-hut"

    def __init__(self, engine, layout: RankLayout, comm: Communicator):
        if comm.world != layout.world:
            raise ValueError("layout and communicator disagree on the world size")
        self.engine = engine
        self.layout = layout
        self.comm = comm
        self.rank = comm.rank
        self.lo, self.hi = layout.range(self.rank)

    def prepare_update_connectivity(self, signal_types, vacant_axons, vacant_excitatory_dendrites, vacant_inhibitory_dendrites, update=None):
        """Algorithm::prepare_update_connectivity with this rank's neurons'
        arrays (layout.count(rank) entries each)."""
        k = self.hi - self.lo
        arrays = [signal_types, vacant_axons, vacant_excitatory_dendrites, vacant_inhibitory_dendrites]
        if update is None:
            update = np.ones(k, np.uint8)
        for a in arrays + [update]:
            if len(a) != k:
                raise ValueError(f"rank {self.rank} owns {k} neurons; got an array of {len(a)}")
        ve = self.comm.all_gather_blocks(np.asarray(vacant_excitatory_dendrites, np.uint32), self.layout).astype(np.uint32)
        vi = self.comm.all_gather_blocks(np.asarray(vacant_inhibitory_dendrites, np.uint32), self.layout).astype(np.uint32)
        # signal type and plasticity flag in one word per neuron
        packed = np.asarray(signal_types, np.uint32) | (np.asarray(update, np.uint32) << 8)
        both = self.comm.all_gather_blocks(packed, self.layout).astype(np.uint32)
        sig = (both & 0xFF).astype(np.uint8)
        upd = ((both >> 8) & 0xFF).astype(np.uint8)
        va = np.zeros(self.layout.n, np.uint32)
        va[self.lo:self.hi] = np.asarray(vacant_axons, np.uint32)
        self.engine.prepare_update_connectivity(va, ve, vi, signal=sig, update=upd)

    def update_connectivity(self, step: int) -> DistributedConnectivityResult:
        """ForwardCPUAlgorithm::update_connectivity: search, exchange the
        requests, process them on the targets' ranks, exchange the responses,
        process them on the sources' ranks."""
        world = self.layout.world
        out = self.engine.find_targets(step)
        dest = self.layout.owner(out["target"])
        order = np.argsort(dest, kind="stable")
        send = out[order]
        send_dest = dest[order]
        send_counts = np.bincount(send_dest, minlength=world)
        recv_rows, recv_counts = self.comm.all_to_all(_rows(send), send_counts, 4)
        recv = _requests(recv_rows)
        created, accepted = self.engine.process_requests(step, recv)
        back_rows, _ = self.comm.all_to_all(accepted.astype(np.int32).reshape(-1, 1), recv_counts, 1)
        answered = back_rows.reshape(-1).astype(np.uint8)
        remote = (send_dest != self.rank).astype(np.uint8)
        self.engine.process_responses(send, answered, remote)
        acc = accepted.astype(bool)
        from_here = self.layout.owner(recv["source"]) == self.rank
        return DistributedConnectivityResult(
            int(created),
            recv[acc & from_here].copy(),
            recv[acc & ~from_here].copy(),
            send[answered.astype(bool) & remote.astype(bool)].copy(),
        )

    def get_algorithm_type(self) -> str:
        return self.algorithm_type
