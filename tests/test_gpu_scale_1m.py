"""Bit-exact parity at the benchmark's size: 1M neurons in a 10,000 um cube
(uniform, and the 64-component Gaussian mixture) with the bench workload's
parameters, synaptic elements seeded U[0, 4] per
type so that every plasticity update searches for about a million axons, 301
steps (three plasticity updates) through the C ABI against the oracle on all
host cores: potentials, calcium, elements, octree and the synapse list must be
identical."""
import os

import numpy as np
import pytest

from conftest import oracle_params, seed_elements
from test_gpu_parity import assert_tree_equal, compare_state

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("placement", ["uniform", "mixture"])
def test_one_million_neurons_301_steps(placement):
    from oracle import oracle as O
    from relearn_b200 import Network, default_params, workloads

    n, side, seed = 1_000_000, 10_000.0, 1
    params = default_params(n, side)
    params["seed"] = seed
    pos = workloads.uniform_cube(n, side, seed) if placement == "uniform" else workloads.gaussian_mixture(n, side, seed)
    sig = workloads.signal_types(n, seed)
    net = Network(params)
    net.set_positions(pos, sig)
    sim = O.OracleSim(oracle_params(params), pos, sig, threads=os.cpu_count() or 1)
    seed_elements(net, n, 77, 0.0, 4.0)
    seed_elements(sim, n, 77, 0.0, 4.0)
    net.simulate(1, 301)
    sim.simulate(1, 301)
    compare_state(net, sim, n)
    assert_tree_equal(net.tree(), sim.tree())
    st, so = net.stats(), sim.stats()
    assert st["searches"] == so["searches"] > 1_000_000
    assert st["synapses_created"] == so["created"] > 100_000
