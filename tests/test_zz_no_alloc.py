"""The allocation-free tree update, for callers that cannot allocate device
memory when they update the octree (a runtime that hands out all device memory
from its own pool or budget, or a host that must not call the CUDA allocator
once set-up is done).

Checked through the C ABI against the regular rl_prepare_update_connectivity:
* the same octree, bitwise (the tolerance of the other parity tests), on two
  calls in a row with different vacancies;
* nothing allocated after the first call: the context's device bytes and the
  device's free memory are unchanged;
* with plasticity flags on a caller stream, a following update_connectivity
  forms the same synapses and leaves the same element counts as the regular
  path (the connector accepts against the counts this call hands over);
* a tree above the fixed scratch size is rejected with RL_ERR_OVERFLOW.
This file is collected last, so a run that stops at the first failure has run
every other test before it."""
import numpy as np
import pytest

from conftest import seed_elements, small_network

pytestmark = pytest.mark.gpu


def same_f64(a, b):
    return np.array_equal(np.asarray(a, np.float64).view(np.uint64), np.asarray(b, np.float64).view(np.uint64))


def assert_same_tree(got, expect, tag):
    for k in ("cnt_exc", "cnt_inh", "level", "neuron", "child_mask", "first_child"):
        assert np.array_equal(got[k], expect[k]), (tag, k)
    for k in ("pos_exc", "pos_inh", "bmin", "bmax"):
        assert same_f64(got[k], expect[k]), (tag, k)


def random_vacancy(rng, n):
    ve = rng.integers(0, 4, n).astype(np.uint32)
    vi = rng.integers(0, 3, n).astype(np.uint32)
    ve[rng.random(n) < 0.3] = 0
    return ve, vi


def device_u32(a):
    import torch

    return torch.from_numpy(a.astype(np.int32)).cuda()


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
        ve, vi = random_vacancy(rng, n)
        net.prepare_update_connectivity(zeros, ve, vi)
        expect = net.tree()
        net.prepare_update_connectivity(zeros, zeros, zeros)  # clear, so the variant must recompute
        d_ve, d_vi = device_u32(ve), device_u32(vi)
        torch.cuda.synchronize()
        net.prepare_update_connectivity_noalloc(d_ve.data_ptr(), d_vi.data_ptr())
        net.synchronize()
        assert_same_tree(net.tree(), expect, call)
    net.close()


def test_noalloc_allocates_nothing():
    """After the first call (which looks up the scratch array's address and
    loads the kernels), further calls change neither the context's device
    bytes nor the device's free memory."""
    import torch

    from relearn_b200 import Network

    n = 20000
    params, pos, sig = small_network(n, 2000.0, 5, False)
    net = Network(params)
    net.set_positions(pos, sig)
    rng = np.random.default_rng(3)
    inputs = [tuple(device_u32(a) for a in random_vacancy(rng, n)) for _ in range(3)]
    d_up = torch.ones(n, dtype=torch.uint8, device="cuda")
    net.prepare_update_connectivity_noalloc(inputs[0][0].data_ptr(), inputs[0][1].data_ptr(), d_up.data_ptr())
    net.synchronize()
    torch.cuda.synchronize()
    ctx_before = net.memory()
    free_before, _ = torch.cuda.mem_get_info()
    for ve, vi in inputs[1:]:
        net.prepare_update_connectivity_noalloc(ve.data_ptr(), vi.data_ptr(), d_up.data_ptr())
    net.synchronize()
    torch.cuda.synchronize()
    free_after, _ = torch.cuda.mem_get_info()
    assert net.memory() == ctx_before
    assert free_after == free_before, (free_before, free_after)
    net.close()


def test_noalloc_on_caller_stream_then_connectivity():
    """Plasticity flags and a caller stream; the synapses that the next
    update_connectivity forms, and the element counts after it, equal the
    regular path's."""
    import torch

    from relearn_b200 import Network

    n = 6000
    params, pos, sig = small_network(n, 1500.0, 21, True)
    rng = np.random.default_rng(21)
    ve, vi = random_vacancy(rng, n)
    mask = (rng.random(n) < 0.8).astype(np.uint8)
    nets = []
    for _ in range(2):
        net = Network(params)
        net.set_positions(pos, sig)
        seed_elements(net, n, 4, 0.0, 3.0)
        nets.append(net)
    va = nets[0].get_elements(0)["vacant"]
    regular, noalloc = nets
    regular.prepare_update_connectivity(va, ve, vi, update=mask)
    syn_regular = regular.update_connectivity(100)

    noalloc.prepare_update_connectivity(va, np.zeros(n, np.uint32), np.zeros(n, np.uint32))
    d_ve, d_vi = device_u32(ve), device_u32(vi)
    d_mask = torch.from_numpy(mask).cuda()
    side = torch.cuda.Stream()
    torch.cuda.synchronize()
    noalloc.prepare_update_connectivity_noalloc(d_ve.data_ptr(), d_vi.data_ptr(), d_mask.data_ptr(), side.cuda_stream)
    syn_noalloc = noalloc.update_connectivity(100)
    noalloc.synchronize()
    side.synchronize()

    assert len(syn_regular) > 0
    assert np.array_equal(syn_regular, syn_noalloc)
    for t in range(3):
        a, b = regular.get_elements(t), noalloc.get_elements(t)
        assert np.array_equal(a["vacant"], b["vacant"]), t
        assert np.array_equal(a["connected"], b["connected"]), t
    assert_same_tree(noalloc.tree(), regular.tree(), "after connectivity")
    for net in nets:
        net.close()


def test_noalloc_rejects_tree_above_limit():
    from relearn_b200 import STATUS_NAMES, Network, RelearnError, default_params, workloads

    n, side = 2_000_000, 10_000.0
    params = default_params(n, side)
    net = Network(params)
    net.set_positions(workloads.uniform_cube(n, side, 9), workloads.signal_types(n, 9))
    nodes, _ = net.tree_info()
    assert nodes > 2_097_152
    zeros = device_u32(np.zeros(n, np.uint32))
    with pytest.raises(RelearnError) as e:
        net.prepare_update_connectivity_noalloc(zeros.data_ptr(), zeros.data_ptr())
    assert STATUS_NAMES[e.value.status] == "RL_ERR_OVERFLOW"
    net.close()
