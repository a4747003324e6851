"""Seeded synthetic systems with the shapes of the benchmark configurations.

No public dataset is involved: every structure is generated from a fixed
seed.  Hyper-parameters not stated by a configuration (Gaussian width,
smoothing width) default to width 0.3 A and ShiftedCosine width 0.5 A.

* ``sc_lattice``       216 atoms, 6x6x6 simple cubic (a = 2.0 A) in a periodic
                       12 A cube, Gaussian jitter 0.1 A, types 1 / 8 in a 2:1
                       ratio by seeded shuffle; rc 5.0, nmax 5, lmax 4.
* ``random_box``       periodic cube at density 0.1 A^-3, uniform positions
                       rejection-sampled to a minimum pair distance, types
                       drawn uniformly from {1, 6, 7, 8}.
* ``molecules``        non-periodic molecules with N ~ U{5..60} atoms, types
                       {1, 6, 7, 8} with p = {.5, .3, .1, .1}, positions in a
                       sphere of radius 1.2 N^(1/3) A, minimum distance 1.0 A.
"""
import numpy as np


def hypers(cutoff, max_radial, max_angular, width=0.3, smoothing=0.5, spline_accuracy=1e-8):
    basis = {"type": "TensorProduct", "max_angular": max_angular, "radial": {"type": "Gto", "max_radial": max_radial}}
    if spline_accuracy != 1e-8:
        basis["spline_accuracy"] = spline_accuracy
    return {
        "cutoff": {"radius": cutoff, "smoothing": {"type": "ShiftedCosine", "width": smoothing}},
        "density": {"type": "Gaussian", "width": width},
        "basis": basis,
    }


def system_dict(types, positions, cell):
    return {
        "types": np.ascontiguousarray(types, dtype=np.int32),
        "positions": np.ascontiguousarray(positions, dtype=np.float64),
        "cell": np.ascontiguousarray(cell, dtype=np.float64).reshape(3, 3),
    }


def sc_lattice(seed=1):
    """216 atoms on a jittered simple-cubic lattice in a 12 A periodic cube."""
    rng = np.random.default_rng(seed)
    grid = np.arange(6) * 2.0
    pos = np.stack(np.meshgrid(grid, grid, grid, indexing="ij"), axis=-1).reshape(-1, 3)
    pos = pos + rng.normal(0.0, 0.1, size=pos.shape)
    types = np.array([1] * 144 + [8] * 72, dtype=np.int32)
    rng.shuffle(types)
    return system_dict(types, pos, np.eye(3) * 12.0)


def _min_distance_fill(rng, n, sampler, min_distance, cell_length=None, max_tries=200):
    """Sequential random insertion with a minimum pair distance, using a grid
    of bins of size min_distance (periodic when ``cell_length`` is set)."""
    accepted = np.zeros((n, 3))
    bins = {}
    h = min_distance
    count = 0
    tries = 0
    batch = sampler(4096)
    bi = 0
    while count < n:
        if bi == len(batch):
            batch = sampler(4096)
            bi = 0
        p = batch[bi]
        bi += 1
        tries += 1
        if tries > max_tries * n:
            raise RuntimeError("could not place atoms with the requested minimum distance")
        key = np.floor(p / h).astype(np.int64)
        ok = True
        for dx in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dz in (-1, 0, 1):
                    k = (key[0] + dx, key[1] + dy, key[2] + dz)
                    if cell_length is not None:
                        nb = int(np.ceil(cell_length / h))
                        k = (k[0] % nb, k[1] % nb, k[2] % nb)
                    for j in bins.get(k, ()):
                        d = accepted[j] - p
                        if cell_length is not None:
                            d -= cell_length * np.round(d / cell_length)
                        if d @ d < min_distance * min_distance:
                            ok = False
                            break
                    if not ok:
                        break
                if not ok:
                    break
            if not ok:
                break
        if not ok:
            continue
        if cell_length is not None:
            nb = int(np.ceil(cell_length / h))
            key = (key[0] % nb, key[1] % nb, key[2] % nb)
        else:
            key = tuple(key)
        bins.setdefault(tuple(key), []).append(count)
        accepted[count] = p
        count += 1
    return accepted


def random_box(n_atoms, density=0.1, min_distance=0.9, species=(1, 6, 7, 8), seed=2, strain=0.0):
    """Periodic cube holding ``n_atoms`` at ``density``; with ``strain`` > 0 the
    cell and positions are deformed by a seeded random strain in [-strain, strain]."""
    rng = np.random.default_rng(seed)
    length = (n_atoms / density) ** (1.0 / 3.0)
    pos = _min_distance_fill(rng, n_atoms, lambda k: rng.uniform(0.0, length, size=(k, 3)), min_distance, length)
    types = rng.choice(np.array(species, dtype=np.int32), size=n_atoms)
    cell = np.eye(3) * length
    if strain > 0:
        eps = rng.uniform(-strain, strain, size=(3, 3))
        deform = np.eye(3) + eps
        cell = cell @ deform
        pos = pos @ deform
    return system_dict(types, pos, cell)


def molecules(n_molecules, seed=3, min_atoms=5, max_atoms=60, min_distance=1.0):
    """Non-periodic molecules of uneven size."""
    rng = np.random.default_rng(seed)
    out = []
    species = np.array([1, 6, 7, 8], dtype=np.int32)
    for _ in range(n_molecules):
        n = int(rng.integers(min_atoms, max_atoms + 1))
        radius = 1.2 * n ** (1.0 / 3.0)

        def sampler(k):
            v = rng.normal(size=(k, 3))
            v /= np.linalg.norm(v, axis=1)[:, None]
            r = radius * rng.uniform(0.0, 1.0, size=(k, 1)) ** (1.0 / 3.0)
            return v * r

        pos = _min_distance_fill(rng, n, sampler, min_distance)
        types = rng.choice(species, size=n, p=[0.5, 0.3, 0.1, 0.1])
        out.append(system_dict(types, pos, np.zeros((3, 3))))
    return out


# the benchmark configurations (sizes and hyper-parameters)
CONFIGS = {
    "c1": dict(system=lambda: [sc_lattice()], hypers=hypers(5.0, 5, 4), gradients=()),
    "c2": dict(system=lambda: [random_box(1000)], hypers=hypers(5.5, 7, 6), gradients=("positions", "strain")),
    "c5": dict(system=lambda: [random_box(20000, strain=0.02, seed=5)], hypers=hypers(5.0, 7, 6), gradients=("positions",)),
}
