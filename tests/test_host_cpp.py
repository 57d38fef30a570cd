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


def test_network_file_round_trip(tmp_path):
    from relearn_b200 import workloads

    rng = np.random.default_rng(4)
    t = rng.integers(0, 50, 200).astype(np.uint32)
    s = rng.integers(0, 50, 200).astype(np.uint32)
    w = rng.choice([-2, -1, 1, 3], 200).astype(np.int32)
    workloads.write_network_files(str(tmp_path), 50, t, s, w)
    t2, s2, w2 = workloads.read_in_network_file(str(tmp_path / "rank_0_in_network.txt"), 50)
    order = np.lexsort((s, t))
    assert np.array_equal(t2, t[order]) and np.array_equal(s2, s[order]) and np.array_equal(w2, w[order])
    t3, s3, _ = workloads.read_in_network_file(str(tmp_path / "rank_0_out_network.txt"), 50)
    assert np.all(np.diff(s3.astype(np.int64)) >= 0)
    bad = tmp_path / "bad.txt"
    for line in ("0 1 0 2 1 0\n", "1 1 0 2 1 1\n", "0 51 0 2 1 1\n", "0 1 0 2 0 1\n"):
        bad.write_text(line)
        with pytest.raises(ValueError):
            workloads.read_in_network_file(str(bad), 50)


def test_calcium_file(tmp_path):
    from relearn_b200 import workloads

    p = tmp_path / "calcium.txt"
    p.write_text("# initial and target calcium\ndefault 0.1 0.7\n0:2;-1:4 0.3 0.9\n0:1 0.0 0.5\n")
    ini, tgt = workloads.read_calcium_file(str(p), 5)
    assert list(ini) == [0.0, 0.3, 0.1, 0.3, 0.1] and list(tgt) == [0.5, 0.9, 0.7, 0.9, 0.7]
    for text in ("default 0 0.7\n0:1 0 1\n0:1 0 1\n", "0:1 0 1\n", "default 0 0.7\nexcitatory 0 1\n", "default 0 0.7\n0:6 0 1\n",
                 "default 0 0.7\n2:1 0 1\n", "default 0 1\ndefault 0 1\n"):
        p.write_text(text)
        with pytest.raises(ValueError):
            workloads.read_calcium_file(str(p), 5)
