"""Generate the golden fixtures of tests/golden from the CPU oracle.

The reference ships no golden trajectories for this path (its tests are
property tests with clock seeds), so the fixtures are produced by the oracle,
whose building blocks are pinned against the reference's known-answer tests
(tests/test_oracle_pins.py).  Run from the repository root:

    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

from conftest import oracle_params, seed_elements, small_network  # noqa: E402
from oracle import oracle as O  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def tree_fields(t):
    return {f"tree_{k}": v for k, v in t.items()}


def make(name, n, side, seed, mixture, steps, lower, upper):
    params, pos, sig = small_network(n, side, seed, mixture)
    sim = O.OracleSim(oracle_params(params), pos, sig)
    seed_elements(sim, n, seed, lower, upper)
    out = dict(positions=pos, signal=sig, seed=np.uint64(params["seed"]), side=np.float64(side), lower=np.float64(lower),
               upper=np.float64(upper), steps=np.uint32(steps))
    # one prepare + search + connector on the seeded state
    ex = sim.get_elements(1)["vacant"]
    ih = sim.get_elements(2)["vacant"]
    sim.update_tree(ex, ih)
    out.update(tree_fields(sim.tree()))
    req = sim.find_targets(100)
    out["requests"] = req
    created, acc = sim.connect(100, len(req))
    out["accepted"] = acc
    t, s, w = sim.edges()
    out.update(edges_target=t, edges_source=s, edges_weight=w)
    # trajectory from a fresh copy of the same network
    sim2 = O.OracleSim(oracle_params(params), pos, sig)
    seed_elements(sim2, n, seed, lower, upper)
    sim2.simulate(1, steps)
    nr = sim2.neurons()
    out.update({f"final_{k}": v for k, v in nr.items()})
    for tpe in range(3):
        e = sim2.get_elements(tpe)
        out.update({f"final_el{tpe}_{k}": v for k, v in e.items()})
    t, s, w = sim2.edges()
    out.update(final_edges_target=t, final_edges_source=s, final_edges_weight=w)
    out["final_stats"] = np.array(list(sim2.stats().values()), np.uint64)
    np.savez_compressed(os.path.join(OUT, name), **out)
    print(name, "nodes", len(out["tree_level"]), "requests", len(req), "created", created, "final edges", len(t), sim2.stats())


if __name__ == "__main__":
    make("golden_uniform_300.npz", 300, 600.0, 21, False, 700, 0.0, 3.0)
    make("golden_mixture_400.npz", 400, 3000.0, 22, True, 500, 0.5, 2.5)
