"""The C++ driver (relearn_b200/host/relearn_b200_run.cpp, Simulation over the
C ABI) reproduces the oracle on config[0]'s network: positions written in the
reference's positions-file format, 20,001 steps, final calcium and synapses
bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from conftest import oracle_params, small_network

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def write_positions(path, pos, sig):
    with open(path, "w") as f:
        f.write("# positions of a seeded synthetic network\n")
        for i, (p, s) in enumerate(zip(pos, sig)):
            f.write(f"{i + 1} {p[0]!r} {p[1]!r} {p[2]!r} {'in' if s else 'ex'}\n")


def test_driver_matches_oracle(tmp_path):
    from oracle import oracle as O

    n, side, seed = 2000, 1000.0, 3
    params, pos, sig = small_network(n, side, seed)
    path = str(tmp_path / "positions.txt")
    write_positions(path, pos, sig)
    prefix = str(tmp_path / "run")
    args = [os.path.join(ROOT, "relearn_b200", "bin", "relearn_b200_run"), "--file", path, "-s", "20000", "-r", str(params["seed"]), "--side",
            repr(side), "--izhikevich-a", "0.02", "--izhikevich-d", "8", "--synapse-conductance", "3", "--growth-rate-axon", "1e-4",
            "--growth-rate-dendrite-exc", "1e-4", "--growth-rate-dendrite-inh", "1e-4", "--output-prefix", prefix]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ca = np.loadtxt(prefix + "_calcium.txt", dtype=np.float64)
    syn = np.loadtxt(prefix + "_synapses.txt", dtype=np.int64, ndmin=2)
    sim = O.OracleSim(oracle_params(params), pos, sig, threads=8)
    sim.simulate(1, 20001)
    o = sim.neurons()
    assert np.array_equal(ca.view(np.uint64), o["calcium"].view(np.uint64))
    t, s, w = sim.edges()
    assert len(t) > 0 and syn.shape[0] == len(t)
    assert np.array_equal(syn[:, 0], t) and np.array_equal(syn[:, 1], s) and np.array_equal(syn[:, 2], w)
