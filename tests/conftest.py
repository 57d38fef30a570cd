import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def built_lib():
    from relearn_b200 import build

    return build.build()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    oracle.build()
    return oracle


def small_network(n: int, side: float, seed: int, mixture: bool = False):
    """Positions, signal types and parameters of a seeded synthetic network."""
    from relearn_b200 import default_params, workloads

    pos = workloads.gaussian_mixture(n, side, seed, components=8, std=side / 20) if mixture else workloads.uniform_cube(n, side, seed)
    sig = workloads.signal_types(n, seed)
    params = default_params(n, side)
    params["seed"] = 1000 + seed
    return params, pos, sig


def oracle_params(params: dict) -> dict:
    p = dict(params)
    p.pop("device", None)
    p["use_libm"] = 0
    return p


def seed_elements(sim_or_net, n: int, seed: int, lower: float, upper: float):
    """Initial grown elements U[lower, upper] per type, vacant = floor(grown)."""
    from relearn_b200 import workloads

    for t, (g, v) in enumerate(workloads.initial_elements(n, seed, lower, upper)):
        sim_or_net.set_elements(t, g, np.zeros(n), np.zeros(n, np.uint32), v)


M64 = (1 << 64) - 1


def splitmix64_uniform(seed, count):
    """The C++ driver's SplitMix64 draws (relearn_b200_run.cpp) as doubles in
    [0, 1)."""
    x = seed & M64
    out = np.empty(count)
    for k in range(count):
        x = (x + 0x9E3779B97F4A7C15) & M64
        z = x
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M64
        z ^= z >> 31
        out[k] = float(z >> 11) * 2.0**-53
    return out
