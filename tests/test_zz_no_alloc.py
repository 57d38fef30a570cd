"""The allocation-free tree update, for callers that cannot allocate device
memory when they update the octree, gives the same octree as the regular
rl_prepare_update_connectivity: called through the C ABI twice in a row with
different vacancies, each result is compared with the regular entry point's
(bitwise, the tolerance of the other parity tests)."""
import numpy as np
import pytest

from conftest import small_network

pytestmark = pytest.mark.gpu


def same_f64(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


@pytest.mark.parametrize("n,mixture", [(5000, False), (8000, True)])
def test_noalloc_tree_update_matches_regular(n, mixture):
    import torch

    from relearn_b200 import Network

    params, pos, sig = small_network(n, 1200.0, 77 + n, mixture)
    net = Network(params)
    net.set_positions(pos, sig)
    zeros = np.zeros(n, np.uint32)
    rng = np.random.default_rng(n)
    for call in range(2):
        ve = rng.integers(0, 4, n).astype(np.uint32)
        vi = rng.integers(0, 3, n).astype(np.uint32)
        ve[rng.random(n) < 0.3] = 0
        net.prepare_update_connectivity(zeros, ve, vi)
        expect = net.tree()
        net.prepare_update_connectivity(zeros, zeros, zeros)  # clear, so the variant must recompute
        d_ve = torch.from_numpy(ve.astype(np.int32)).cuda()
        d_vi = torch.from_numpy(vi.astype(np.int32)).cuda()
        torch.cuda.synchronize()
        net.prepare_update_connectivity_noalloc(d_ve.data_ptr(), d_vi.data_ptr())
        net.synchronize()
        got = net.tree()
        for k in ("cnt_exc", "cnt_inh", "level", "neuron", "child_mask", "first_child"):
            assert np.array_equal(got[k], expect[k]), (call, k)
        for k in ("pos_exc", "pos_inh", "bmin", "bmax"):
            assert same_f64(got[k], expect[k]), (call, k)
