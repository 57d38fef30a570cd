"""Synaptic input with synapses: the first step of an activity block pulls each
neuron's synaptic sum over its in-edges (the reference's
NetworkGraph-based sum); at the later steps of the block each neuron whose
spike flag is set has added its out-edges' weights to its targets' sums of the
next step, and the targets read those.  Integer sums, so a block of many steps
must give the same bits as blocks of one step (which pull at every step):
with excitatory and inhibitory weights of several sizes, repeated
(target, source) entries, disabled neurons that keep a set spike flag, CUDA
graphs, the tuner's trial steps, and blocks of 1, 2, odd and even lengths."""
import numpy as np
import pytest

from conftest import small_network

pytestmark = pytest.mark.gpu


def make(n, precision, seed):
    from relearn_b200 import Network

    params, pos, sig = small_network(n, 2500.0, seed)
    params["precision"] = precision
    net = Network(params)
    net.set_positions(pos, sig)
    rng = np.random.default_rng(seed)
    m = 12 * n
    tgt = rng.integers(0, n, m).astype(np.uint32)
    src = rng.integers(0, n, m).astype(np.uint32)
    w = rng.choice(np.array([-3, -1, 1, 2, 5], np.int32), m)
    net.add_edges(tgt, src, w)
    net.add_edges(tgt[: n // 2], src[: n // 2], w[: n // 2])  # repeated pairs: separate entries of the graph
    net.set_enabled((rng.random(n) > 0.2).astype(np.uint8))
    net.set_neurons(fired=(rng.random(n) < 0.3).astype(np.uint8))  # disabled neurons keep these flags
    return net


def state(net):
    a = net.neurons()
    out = {k: a[k].view(np.uint64) if a[k].dtype == np.float64 else a[k] for k in ("x", "u", "calcium", "fired", "input")}
    for t in range(3):
        d = net.get_elements(t)["delta"]
        out[f"delta{t}"] = d.view(np.uint64) if d.dtype == np.float64 else d
    return out


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("mode", ["plain", "graphs", "tuned"])
def test_pushed_sums_equal_pulled(precision, mode):
    import torch

    n = 20011
    # the last block is longer than the 128 steps whose calcium and growth
    # one launch replays: three chunks in one block
    blocks = ((1, 37), (38, 64), (102, 1), (103, 2), (105, 100), (205, 100), (305, 300))
    ref = make(n, precision, 17)
    net = make(n, precision, 17)
    stream = torch.cuda.Stream()
    if mode == "graphs":
        net.set_stream(stream.cuda_stream)  # 100-step blocks replay a captured graph
    elif mode == "tuned":
        net.autotune(1)  # trial steps at the first block, then the state is put back
    fired = 0
    for first, count in blocks:
        for s in range(first, first + count):
            ref.activity_block(s, 1)
        net.activity_block(first, count)
        net.synchronize()
        a, b = state(ref), state(net)
        for k in a:
            assert np.array_equal(a[k], b[k]), (precision, mode, first, k)
        fired += int(a["fired"].sum())
    assert fired > 0
    assert net.stats()["gpu_launches"] > 0
    ref.close()
    net.close()
