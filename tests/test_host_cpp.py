"""The C++ host layer (relearn_b200/host): its self-test (positions-file
reader in the reference's format, status codes as RelearnException) and the
driver's command line, without a GPU."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "relearn_b200", "bin")


def test_host_selftest(built_lib, tmp_path):
    from conftest import has_gpu

    args = [os.path.join(BIN, "host_selftest"), str(tmp_path)] + ([] if has_gpu() else ["--no-device"])
    r = subprocess.run(args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == "ok"


def test_driver_command_line(built_lib):
    exe = os.path.join(BIN, "relearn_b200_run")
    r = subprocess.run([exe, "--help"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    for opt in ("--theta", "--gaussian-sigma", "--random-seed", "--synaptic-elements-lower-bound", "--growth-rate-axon", "--file"):
        assert opt in r.stdout
    r = subprocess.run([exe, "--no-such-option"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "unknown option" in r.stderr
    r = subprocess.run([exe, "--algorithm", "naive", "--num-neurons", "10", "-s", "1"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2


def test_driver_without_device_fails_cleanly(built_lib):
    from conftest import has_gpu

    if has_gpu():
        pytest.skip("a device is present")
    r = subprocess.run([os.path.join(BIN, "relearn_b200_run"), "--num-neurons", "100", "-s", "10"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "rl_ctx_create" in r.stderr


def test_positions_file_round_trip(tmp_path):
    from relearn_b200 import workloads

    pos = workloads.uniform_cube(500, 1234.5, 7)
    sig = workloads.signal_types(500, 7)
    path = str(tmp_path / "p.txt")
    workloads.write_positions_file(path, pos, sig)
    p2, s2 = workloads.read_positions_file(path)
    assert np.array_equal(p2.view(np.uint64), pos.view(np.uint64)) and np.array_equal(s2, sig)
    with open(path, "a") as f:
        f.write("not a neuron line\n502 1 1 1 ex\n")
    with pytest.raises(ValueError):
        workloads.read_positions_file(path)
