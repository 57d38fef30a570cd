"""The incremental octree update against a full one.

An update recomputes only the inner nodes above leaves whose vacant dendrite
counts changed: the leaf pass marks their parents, each marked node goes once
onto its level's list, and each level launch recomputes the nodes on its list
and marks their parents.  Once a network deletes synapses at every update,
the update runs once, after the deletions, instead of also before them.  After
a history of such updates (synapses formed and deleted, captured update
graphs), one more incremental update must give, bit for bit, the octree that
a fresh context computes in full from the same vacancies
(OctreeAlgorithm::update_tree, algorithm/Internal/OctreeAlgorithm.h:100-238:
every node from its children)."""
import numpy as np
import pytest

from conftest import seed_elements, small_network

pytestmark = pytest.mark.gpu


def same_f64(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


@pytest.mark.parametrize("precision", [0, 1])
def test_incremental_octree_after_deleting_updates(precision):
    import torch

    from relearn_b200 import Network

    n = 30011
    params, pos, sig = small_network(n, 2500.0, 41)
    params["precision"] = precision
    net = Network(params)
    net.set_positions(pos, sig)
    stream = torch.cuda.Stream()
    net.set_stream(stream.cuda_stream)  # updates replay the captured octree graph
    seed_elements(net, n, 41, 0.0, 4.0)
    net.simulate(1, 800)
    st = net.stats()
    assert st["plasticity_updates"] >= 7
    assert st["synapses_created"] > 0 and st["synapses_deleted"] > 0

    vac = [net.get_elements(t)["vacant"] for t in range(3)]
    net.prepare_update_connectivity(vac[0], vac[1], vac[2])
    got = net.tree()

    fresh = Network(params)
    fresh.set_positions(pos, sig)
    fresh.prepare_update_connectivity(vac[0], vac[1], vac[2])
    expect = fresh.tree()

    assert int(np.asarray(expect["cnt_exc"])[0]) == int(vac[1].sum()), "root counts every vacant excitatory dendrite"
    for k in ("cnt_exc", "cnt_inh", "level", "neuron", "child_mask", "first_child"):
        assert np.array_equal(got[k], expect[k]), k
    for k in ("pos_exc", "pos_inh", "bmin", "bmax"):
        assert same_f64(got[k], expect[k]), k
    stream.synchronize()
    net.close()
    fresh.close()
