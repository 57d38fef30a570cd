"""Host-side workload generation (seeded, deterministic, valid)."""
import numpy as np

from relearn_b200 import workloads


def test_uniform_is_seeded_and_in_box():
    a = workloads.uniform_cube(5000, 1000.0, 3)
    b = workloads.uniform_cube(5000, 1000.0, 3)
    assert np.array_equal(a, b)
    assert a.min() >= 0.0 and a.max() < 1000.0
    workloads.ensure_distinct(a)


def test_mixture_is_seeded_and_in_box():
    a = workloads.gaussian_mixture(20000, 10000.0, 5)
    assert np.array_equal(a, workloads.gaussian_mixture(20000, 10000.0, 5))
    assert a.shape == (20000, 3) and a.min() >= 0.0 and a.max() < 10000.0


def test_signal_fraction():
    s = workloads.signal_types(2000, 1)
    assert s.sum() == 400 and set(np.unique(s)) == {0, 1}


def test_initial_elements():
    e = workloads.initial_elements(100, 2, 0.0, 4.0)
    for g, v in e:
        assert np.all(v == np.floor(g)) and g.min() >= 0.0 and g.max() <= 4.0
