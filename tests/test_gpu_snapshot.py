"""Asynchronous host transfers: snapshots of calcium and fired flags hold the
state as of the call although the simulation runs on while they are copied,
and uploads of enabled flags take effect in order with the queued work."""
import numpy as np
import pytest

from conftest import seed_elements, small_network

pytestmark = pytest.mark.gpu


def make(n, seed, precision=0):
    from relearn_b200 import Network

    params, pos, sig = small_network(n, 1000.0 * (n / 2000) ** (1 / 3), seed)
    params["precision"] = precision
    net = Network(params)
    net.set_positions(pos, sig)
    seed_elements(net, n, seed, 0.0, 3.0)
    return net


@pytest.mark.parametrize("precision", [0, 1])
def test_snapshots_hold_the_state_of_their_call(precision):
    n = 20000
    net = make(n, 5, precision)
    twin = make(n, 5, precision)
    ca = [np.zeros(n), np.zeros(n)]
    fired = [np.zeros(n, np.uint8), np.zeros(n, np.uint8)]
    net.simulate(1, 150)
    net.snapshot_neurons(ca[0], fired[0])
    net.simulate(151, 100)  # runs while the first copy may be in flight
    net.snapshot_neurons(ca[1], fired[1])
    net.simulate(251, 60)
    net.snapshot_wait()
    twin.simulate(1, 150)
    a = twin.neurons()
    assert np.array_equal(ca[0].view(np.uint64), a["calcium"].view(np.uint64))
    assert np.array_equal(fired[0], a["fired"])
    twin.simulate(151, 100)
    a = twin.neurons()
    assert np.array_equal(ca[1].view(np.uint64), a["calcium"].view(np.uint64))
    assert np.array_equal(fired[1], a["fired"])
    assert a["fired"].any()


def test_enabled_upload_is_ordered_with_queued_work():
    n = 20000
    net = make(n, 9)
    twin = make(n, 9)
    off = np.ones(n, np.uint8)
    off[::3] = 0
    net.simulate(1, 100)  # queued work the upload must not overtake
    net.set_enabled(off)
    net.simulate(101, 100)
    twin.simulate(1, 100)
    twin.synchronize()
    twin.set_enabled(off)
    twin.simulate(101, 100)
    a, b = net.neurons(), twin.neurons()
    for k in ("x", "calcium"):
        assert np.array_equal(a[k].view(np.uint64), b[k].view(np.uint64)), k
    assert np.array_equal(a["fired"][::3], b["fired"][::3])
