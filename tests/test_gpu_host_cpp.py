"""The C++ driver (relearn_b200/host/relearn_b200_run.cpp, Simulation over the
C ABI) reproduces the oracle on a 2,000-neuron network with config[0]'s
parameters: positions written in the reference's positions-file format,
initial elements from the driver's SplitMix64 stream (restated here), 3,001
steps, final calcium and synapses bit for bit."""
import os
import subprocess

import numpy as np
import pytest

from conftest import oracle_params, small_network, splitmix64_uniform

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_driver_matches_oracle(tmp_path):
    from oracle import oracle as O
    from relearn_b200.workloads import write_positions_file

    n, side, seed = 2000, 1000.0, 3
    params, pos, sig = small_network(n, side, seed)
    path = str(tmp_path / "positions.txt")
    write_positions_file(path, pos, sig)
    prefix = str(tmp_path / "run")
    args = [os.path.join(ROOT, "relearn_b200", "bin", "relearn_b200_run"), "--file", path, "-s", "3000", "-r", str(params["seed"]), "--side",
            repr(side), "--izhikevich-a", "0.02", "--izhikevich-d", "8", "--synapse-conductance", "3", "--growth-rate-axon", "1e-4",
            "--growth-rate-dendrite-exc", "1e-4", "--growth-rate-dendrite-inh", "1e-4", "--synaptic-elements-lower-bound", "0",
            "--synaptic-elements-upper-bound", "3", "--output-prefix", prefix]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ca = np.loadtxt(prefix + "_calcium.txt", dtype=np.float64)
    syn = np.loadtxt(prefix + "_synapses.txt", dtype=np.int64, ndmin=2)
    sim = O.OracleSim(oracle_params(params), pos, sig, threads=8)
    u = splitmix64_uniform(params["seed"] + 17, 3 * n).reshape(3, n)
    for t in range(3):
        g = 0.0 + (3.0 - 0.0) * u[t]
        sim.set_elements(t, g, np.zeros(n), np.zeros(n, np.uint32), np.floor(g).astype(np.uint32))
    sim.simulate(1, 3001)
    o = sim.neurons()
    assert np.array_equal(ca.view(np.uint64), o["calcium"].view(np.uint64))
    t, s, w = sim.edges()
    assert len(t) > 0 and syn.shape[0] == len(t)
    assert np.array_equal(syn[:, 0], t) and np.array_equal(syn[:, 1], s) and np.array_equal(syn[:, 2], w)


def test_driver_loads_network(tmp_path):
    """-g DIR and --file-calcium: the driver loads plastic synapses from the
    reference's network file format (connected and grown elements follow them,
    as Neurons::init_synaptic_elements does) and initial / target calcium from
    a calcium file, and the run matches the oracle started from the same
    state."""
    from oracle import oracle as O
    from relearn_b200.workloads import write_network_files, write_positions_file

    n, side, seed = 1500, 900.0, 5
    params, pos, sig = small_network(n, side, seed)
    write_positions_file(str(tmp_path / "positions.txt"), pos, sig)
    rng = np.random.default_rng(6)
    pairs = np.unique(rng.integers(0, n, (4000, 2)), axis=0)
    pairs = pairs[pairs[:, 0] != pairs[:, 1]]
    t, s = pairs[:, 0].astype(np.uint32), pairs[:, 1].astype(np.uint32)
    w = np.where(sig[s] == 1, -1, 1).astype(np.int32)
    write_network_files(str(tmp_path), n, t, s, w)
    (tmp_path / "calcium.txt").write_text("# initial and target\ndefault 0.05 0.7\n" + ";".join(f"0:{k}" for k in range(1, n, 7)) + " 0.2 0.3\n")
    prefix = str(tmp_path / "run")
    args = [os.path.join(ROOT, "relearn_b200", "bin", "relearn_b200_run"), "--file", str(tmp_path / "positions.txt"), "-g", str(tmp_path), "-s",
            "1000", "-r", str(params["seed"]), "--side", repr(side), "--izhikevich-a", "0.02", "--izhikevich-d", "8", "--synapse-conductance", "3",
            "--growth-rate-axon", "1e-4", "--growth-rate-dendrite-exc", "1e-4", "--growth-rate-dendrite-inh", "1e-4",
            "--synaptic-elements-lower-bound", "0", "--synaptic-elements-upper-bound", "2", "--file-calcium", str(tmp_path / "calcium.txt"),
            "--output-prefix", prefix]
    r = subprocess.run(args, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    ca = np.loadtxt(prefix + "_calcium.txt", dtype=np.float64)
    syn = np.loadtxt(prefix + "_synapses.txt", dtype=np.int64, ndmin=2)
    from relearn_b200.workloads import read_calcium_file

    ini, tgt = read_calcium_file(str(tmp_path / "calcium.txt"), n)
    sim = O.OracleSim(oracle_params(params), pos, sig, threads=8)
    sim.set_neurons(calcium=ini)
    sim.set_targets(tgt)
    u = splitmix64_uniform(params["seed"] + 17, 3 * n).reshape(3, n)
    grown = [2.0 * u[k] for k in range(3)]
    a = np.abs(w).astype(np.float64)
    adds = [np.bincount(s, weights=a, minlength=n), np.bincount(t[w > 0], weights=a[w > 0], minlength=n),
            np.bincount(t[w < 0], weights=a[w < 0], minlength=n)]
    for k in range(3):
        sim.set_elements(k, grown[k] + adds[k].astype(np.uint32), np.zeros(n), adds[k].astype(np.uint32), np.floor(grown[k]).astype(np.uint32))
    sim.add_edges(t, s, w)
    sim.simulate(1, 1001)
    assert np.array_equal(ca.view(np.uint64), sim.neurons()["calcium"].view(np.uint64))
    ot, os_, ow = sim.edges()
    assert syn.shape[0] == len(ot) > 0
    assert np.array_equal(syn[:, 0], ot) and np.array_equal(syn[:, 1], os_) and np.array_equal(syn[:, 2], ow)
