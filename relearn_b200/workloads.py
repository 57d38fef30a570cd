"""Seeded synthetic networks with the shapes of the benchmark configurations.

The reference places ``--num-neurons`` neurons on a jittered grid shuffled by
a fixed seed (sim/random/BoxBasedRandomSubdomainAssignment.cpp:26-131); the
workloads here instead draw positions from a seeded generator and hand them
over as a position list, which the reference also accepts (a positions file,
io/NeuronIO.cpp:229-270).  Signal types are 80 % excitatory / 20 % inhibitory
after a seeded shuffle.
"""
from __future__ import annotations

import numpy as np


def uniform_cube(n: int, side: float, seed: int) -> np.ndarray:
    """n positions uniform in [0, side)^3."""
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, side, size=(n, 3))


def gaussian_mixture(n: int, side: float, seed: int, components: int = 64, std: float = 200.0) -> np.ndarray:
    """n positions from an isotropic Gaussian mixture (centres uniform in the
    cube, component std `std`), samples outside the cube rejected."""
    rng = np.random.default_rng(seed)
    centres = rng.uniform(0.0, side, size=(components, 3))
    out = np.empty((0, 3))
    while len(out) < n:
        k = rng.integers(0, components, size=2 * n)
        p = centres[k] + rng.normal(0.0, std, size=(2 * n, 3))
        ok = np.all((p >= 0.0) & (p < side), axis=1)
        out = np.concatenate([out, p[ok]])
    return np.ascontiguousarray(out[:n])


def signal_types(n: int, seed: int, inhibitory_fraction: float = 0.2) -> np.ndarray:
    """0 = excitatory, 1 = inhibitory; round(n * fraction) inhibitory after a seeded shuffle."""
    rng = np.random.default_rng(seed + 7919)
    sig = np.zeros(n, np.uint8)
    k = int(round(n * inhibitory_fraction))
    sig[rng.permutation(n)[:k]] = 1
    return sig


def initial_elements(n: int, seed: int, lower: float, upper: float) -> list:
    """Initial grown elements per type uniform in [lower, upper] (the reference's
    --synaptic-elements-lower-bound / --synaptic-elements-upper-bound,
    relearn.cpp:620-624, 1179-1185).  Returns [(grown, vacant)] for axon,
    excitatory dendrite and inhibitory dendrite; vacant = floor(grown) as in
    ElementBaseBase::init_values (ElementBaseBase.h:390-420) with nothing
    connected."""
    rng = np.random.default_rng(seed + 104729)
    out = []
    for _ in range(3):
        g = rng.uniform(lower, upper, size=n) if upper > lower else np.full(n, float(lower))
        out.append((g, np.floor(g).astype(np.uint32)))
    return out


def ensure_distinct(pos: np.ndarray) -> np.ndarray:
    """The point-region octree needs pairwise distinct positions."""
    u = np.unique(pos, axis=0)
    if len(u) != len(pos):
        raise ValueError("positions are not pairwise distinct")
    return pos


def serving_stream(seed: int, rate: float, duration: float, lo: int = 2_000, hi: int = 1_000_000, steps: int = 5_000,
                   theta=(0.2, 0.5), growth=(1e-5, 1e-3), sigma: float = 750.0, density_um3: float = 1000.0) -> list:
    """The serving workload: Poisson arrivals at `rate` per second over
    `duration` seconds; each request one network of log-uniform lo..hi neurons
    with its own seed, growth rate (log-uniform, the same for all element
    types) and theta (uniform), placed uniformly at one neuron per
    `density_um3` cubic micrometres, run for `steps` steps.  Returns
    [(arrival time, network dict)] in arrival order; positions and signal
    types come from :func:`request_inputs`."""
    rng = np.random.default_rng(seed)
    out = []
    t = 0.0
    k = 0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        n = int(np.exp(rng.uniform(np.log(lo), np.log(hi))))
        net = dict(num_neurons=n, seed=int(seed) * 1_000_003 + k, side=(density_um3 * n) ** (1.0 / 3.0),
                   theta=float(rng.uniform(*theta)), sigma=float(sigma), growth_rate=float(np.exp(rng.uniform(np.log(growth[0]), np.log(growth[1])))),
                   steps=int(steps))
        out.append((t, net))
        k += 1
    return out


def request_inputs(net: dict) -> tuple:
    """Positions and signal types of a serving request, seeded by its seed."""
    n = int(net["num_neurons"])
    s = int(net["seed"]) % (2**31)
    return uniform_cube(n, float(net["side"]), s), signal_types(n, s)


def write_positions_file(path: str, positions: np.ndarray, signal: np.ndarray) -> None:
    """Positions in the reference's positions-file format (read by
    NeuronIO::read_neuron_positions_and_signals, io/NeuronIO.cpp:229-300): one
    line "id x y z signal" per neuron, ids from 1, signal "in" or "ex";
    coordinates with 17 significant digits, so they read back bit for bit."""
    with open(path, "w") as f:
        f.write("# id x y z signal_type\n")
        for i, (p, s) in enumerate(zip(np.asarray(positions, np.float64), np.asarray(signal))):
            f.write(f"{i + 1} {float(p[0]):.17g} {float(p[1]):.17g} {float(p[2]):.17g} {'in' if s else 'ex'}\n")


def read_positions_file(path: str) -> tuple:
    """Positions and signal types (0 excitatory, 1 inhibitory) from a file in
    the reference's positions-file format; comment lines start with '#', lines
    that do not parse are skipped, ids must run 1, 2, ... in order."""
    pos, sig = [], []
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            parts = line.split()
            try:
                nid, x, y, z, s = int(parts[0]), float(parts[1]), float(parts[2]), float(parts[3]), parts[4]
            except (ValueError, IndexError):
                continue
            if min(x, y, z) < 0:
                raise ValueError(f"negative position of neuron {nid}")
            if nid != len(pos) + 1:
                raise ValueError(f"loaded neuron {nid - 1} but expected {len(pos)}")
            pos.append((x, y, z))
            sig.append(1 if s == "in" else 0)
    return np.array(pos, np.float64).reshape(-1, 3), np.array(sig, np.uint8)


BOX_KEYS = ("# Minimum x:", "# Minimum y:", "# Minimum z:", "# Maximum x:", "# Maximum y:", "# Maximum z:")


def read_positions_box(path: str):
    """The simulation box of a positions file from its "# Minimum x:" ..
    "# Maximum z:" comment lines (NeuronIO::parse_additional_position_information,
    io/NeuronIO.cpp:107-148; MultipleSubdomainsFromFile sets the box from them):
    (box_min, box_max), or None unless all six are present."""
    found = {}
    with open(path) as f:
        for line in f:
            if not line.startswith("#"):
                continue
            for k, key in enumerate(BOX_KEYS):
                if k not in found and line.startswith(key):
                    found[k] = float(line[len(key):])
    if len(found) < 6:
        return None
    return np.array([found[0], found[1], found[2]]), np.array([found[3], found[4], found[5]])


NETWORK_HEADER = "# <target rank> <target neuron id>\t<source rank> <source neuron id>\t<weight>\t<plastic>\n"


def write_network_files(directory: str, num_neurons: int, target, source, weight) -> None:
    """rank_0_in_network.txt (sorted by target, source) and
    rank_0_out_network.txt (sorted by source, target) in the reference's
    network-file format (NeuronIO::write_in_synapses / write_out_synapses,
    io/NeuronIO.cpp:935-1030): "target_rank target_id source_rank source_id
    weight plastic", ids from 1, all synapses plastic on rank 0."""
    t, s, w = (np.asarray(a) for a in (target, source, weight))
    for name, order in (("rank_0_in_network.txt", np.lexsort((s, t))), ("rank_0_out_network.txt", np.lexsort((t, s)))):
        with open(f"{directory}/{name}", "w") as f:
            f.write(f"# {num_neurons}\n" + NETWORK_HEADER)
            for k in order:
                f.write(f"0 {int(t[k]) + 1}\t0 {int(s[k]) + 1}\t{int(w[k])}\t1\n")


def read_in_network_file(path: str, num_neurons: int) -> tuple:
    """(target, source, weight) of the plastic synapses in a network file of
    the reference's format; one rank, plastic synapses only."""
    t, s, w = [], [], []
    with open(path) as f:
        for line in f:
            if not line.strip() or line.startswith("#"):
                continue
            parts = line.split()
            try:
                tr, ti, sr, si, wt, pl = (int(x) for x in parts[:6])
            except (ValueError, IndexError):
                continue
            if tr != 0 or sr != 0:
                raise ValueError("synapses of other ranks are not supported on one GPU")
            if not (1 <= ti <= num_neurons and 1 <= si <= num_neurons):
                raise ValueError(f"neuron id out of range: {line.strip()}")
            if wt == 0:
                raise ValueError("weight was 0")
            if not pl:
                raise ValueError("static synapses are not supported by this path")
            t.append(ti - 1)
            s.append(si - 1)
            w.append(wt)
    return np.array(t, np.uint32), np.array(s, np.uint32), np.array(w, np.int32)


def read_calcium_file(path: str, num_neurons: int) -> tuple:
    """Initial and target calcium per neuron from a calcium file of the
    reference (CalciumIO::load_initial_and_target_function,
    io/CalciumIO.cpp:27-130): lines "<description> <initial> <target>", where
    the description is "default" (at most once) or ';'-separated
    "<rank>:<neuron id>" with 1-based ids (rank -1 meaning this rank; one rank
    here).  Every neuron gets at most one pair; neurons without one take the
    default.  Neuron groups are not supported."""
    initial = np.full(num_neurons, np.nan)
    target = np.full(num_neurons, np.nan)
    default = None
    with open(path) as f:
        for line in f:
            if line.startswith("#"):
                continue
            parts = line.split()
            if len(parts) < 3:
                continue
            try:
                ini, tgt = float(parts[1]), float(parts[2])
            except ValueError:
                continue
            if parts[0] == "default":
                if default is not None:
                    raise ValueError("more than one default")
                default = (ini, tgt)
                continue
            for item in parts[0].split(";"):
                if ":" not in item:
                    raise ValueError(f"neuron groups are not supported: {item!r}")
                rank, nid = item.split(":", 1)
                rank, nid = int(rank), int(nid)
                if rank not in (0, -1):
                    raise ValueError(f"rank {rank}: one rank only")
                if nid < 1 or nid > num_neurons:
                    raise ValueError(f"neuron id {nid} out of range (ids are 1-based)")
                if not np.isnan(initial[nid - 1]):
                    raise ValueError(f"neuron {nid} assigned twice")
                initial[nid - 1], target[nid - 1] = ini, tgt
    missing = np.isnan(initial)
    if missing.any():
        if default is None:
            raise ValueError("neurons without values and no default")
        initial[missing], target[missing] = default
    return initial, target
