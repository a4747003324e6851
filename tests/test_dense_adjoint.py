"""Dense power spectrum and its adjoint backward pass.

* FP64 dense values equal the drop-in TensorMap values (same arithmetic);
  tolerance |d| <= 1e-12 |ref| + 1e-14 max|ref|.
* The FP64 adjoint gives the gradient of a linear energy E = sum_k W_k . P_k
  equal to the contraction of the explicit (materialised) positions / strain /
  cell gradients of the drop-in, which reproduce featomic's explicit
  gradients: |d| <= 1e-10 |ref| + 1e-12 max|ref|.
* Central finite differences of E (h = 1e-5 A, FP64) against the adjoint
  forces, strain and cell derivatives: |d| <= 1e-6 max|ref| + 1e-6 |ref|, on
  a system with no pair direction near the z axis (see off_pole_box).
* FP32 arithmetic against FP64: values and forces within 1e-4 of the
  largest magnitude, the stated error bound of the FP32 form.
* The torch interface: autograd through the blocks gives the same forces and
  cell gradient, and torch.autograd.gradcheck passes on a small system.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from layout import load_input

import rascaline_b200 as rb
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def assert_close(actual, expected, rtol, atol_fraction, what):
    actual = np.asarray(actual, dtype=np.float64)
    expected = np.asarray(expected, dtype=np.float64)
    assert actual.shape == expected.shape, (what, actual.shape, expected.shape)
    if expected.size == 0:
        return
    scale = np.max(np.abs(expected))
    bound = rtol * np.abs(expected) + atol_fraction * scale
    diff = np.abs(actual - expected)
    bad = diff > bound
    if bad.any():
        i = np.unravel_index(np.argmax(diff - bound), diff.shape)
        raise AssertionError(f"{what}: {bad.sum()}/{bad.size} elements differ; worst at {i}: "
                             f"{actual[i]} vs {expected[i]} (scale {scale})")


def batch(systems):
    positions = np.concatenate([np.asarray(s["positions"], dtype=np.float64).reshape(-1, 3) for s in systems])
    types = np.concatenate([np.asarray(s["types"], dtype=np.int32) for s in systems])
    cells = np.stack([np.asarray(s["cell"], dtype=np.float64).reshape(9) for s in systems])
    sizes = np.array([len(s["types"]) for s in systems])
    return positions, types, cells, sizes


def key_of(S):
    out, k = {}, 0
    for a in range(S):
        for b in range(a, S):
            out[(a, b)] = k
            k += 1
    return out


def linear_weights(species, n_props, seed=13):
    """Seeded N(0, 1/sqrt(d)) weights per (center, neighbour 1, neighbour 2) key."""
    rng = np.random.default_rng(seed)
    S = len(species)
    d = n_props * S * (S + 1) // 2
    return {(c, a, b): rng.normal(0.0, 1.0 / np.sqrt(d), size=n_props)
            for c in species for a in species for b in species if a <= b}


def dense_grad_values(types, species, weights, n_props):
    S = len(species)
    keys = key_of(S)
    G = np.zeros((len(types), len(keys), n_props))
    for i, t in enumerate(types):
        for (a, b), k in keys.items():
            G[i, k] = weights[(int(t), int(species[a]), int(species[b]))]
    return G


def explicit_energy_gradients(tm, weights, sizes):
    """dE/dpositions, dE/dstrain and dE/dcell from the drop-in's explicit
    gradient blocks (featomic's layout)."""
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    n_sys = len(sizes)
    forces = np.zeros((offsets[-1], 3))
    strain = np.zeros((n_sys, 3, 3))
    cell = np.zeros((n_sys, 3, 3))
    energy = 0.0
    for key, block in zip(tm["keys"], tm["blocks"]):
        W = weights[tuple(int(k) for k in key)]
        energy += float(np.sum(block["values"] @ W))
        g = block["gradients"]
        if "positions" in g:
            s = g["positions"]["samples"]
            np.add.at(forces, offsets[s[:, 1]] + s[:, 2], g["positions"]["values"] @ W)
        systems = block["samples"][:, 0]
        if "strain" in g:
            np.add.at(strain, systems, g["strain"]["values"] @ W)
        if "cell" in g:
            np.add.at(cell, systems, g["cell"]["values"] @ W)
    return energy, forces, strain, cell


def run_dense(calc, systems, precision=64, species=None):
    from rascaline_b200.torch_api import dense_power_spectrum
    positions, types, cells, sizes = batch(systems)
    pos = torch.as_tensor(positions, device="cuda").contiguous()
    values, state = dense_power_spectrum(calc, pos, types, cells, sizes, precision, species)
    return values, state


def run_backward(state, G, n_systems, dtype):
    from rascaline_b200.torch_api import dense_backward
    grad = torch.as_tensor(G, dtype=dtype, device="cuda")
    gpos, gstrain, gcell = dense_backward(state, grad, n_systems, strain=True, cell=True)
    torch.cuda.synchronize()
    return gpos.double().cpu().numpy(), gstrain.double().cpu().numpy(), gcell.double().cpu().numpy()


def cases():
    box = workloads.random_box(300, density=0.1, min_distance=0.9, seed=21, strain=0.02)
    golden, hypers_g = load_input(os.path.join(GOLDEN, "soap-power-spectrum-gradients-input.json"))
    mols = workloads.molecules(6, seed=4, max_atoms=30)
    small = workloads.random_box(120, density=0.1, min_distance=0.9, seed=23, strain=0.01)
    return [
        # splined, lmax <= 8, nmax <= 8: the fused pair adjoint
        ("box_300_strained", [box], workloads.hypers(5.5, 7, 6)),
        # analytic radial integral: features + pair adjoint kernels
        ("golden_gradients_input", golden, hypers_g),
        ("molecules_6", mols, workloads.hypers(5.0, 7, 6)),
        # nmax 12: the fused pair adjoint with 16 radial registers
        ("box_120_nmax12", [small], workloads.hypers(4.5, 11, 3)),
        # lmax 10: features + pair adjoint kernels
        ("box_120_lmax10", [small], workloads.hypers(4.0, 3, 10)),
    ]


@pytest.mark.parametrize("name, systems, hypers", cases(), ids=lambda x: x if isinstance(x, str) else "")
def test_dense_fp64_matches_drop_in_values_and_explicit_gradients(name, systems, hypers):
    calc = rb.SoapPowerSpectrum(**hypers)
    periodic = any(np.any(np.asarray(s["cell"]) != 0) for s in systems)
    gradients = ["positions", "strain", "cell"] if periodic else ["positions"]
    tm = calc.compute([rb.System.from_dict(s) for s in systems], gradients=gradients).to_dict(gradients)
    values, state = run_dense(calc, systems)
    dense = values.cpu().numpy()
    positions, types, cells, sizes = batch(systems)
    species = state.species()
    keys = key_of(len(species))
    offsets = np.concatenate([[0], np.cumsum(sizes)])
    covered = np.zeros(dense.shape[:2], dtype=bool)
    for key, block in zip(tm["keys"], tm["blocks"]):
        a = int(np.searchsorted(species, key[1]))
        b = int(np.searchsorted(species, key[2]))
        atoms = offsets[block["samples"][:, 0]] + block["samples"][:, 1]
        assert_close(dense[atoms, keys[(a, b)]], block["values"], 1e-12, 1e-14, f"{name} values {tuple(key)}")
        covered[atoms, keys[(a, b)]] = True
    assert np.all(dense[~covered] == 0.0), name

    n_props = dense.shape[2]
    weights = linear_weights([int(s) for s in species], n_props)
    G = dense_grad_values(types, species, weights, n_props)
    energy, forces, strain, cell = explicit_energy_gradients(tm, weights, sizes)
    assert abs(float(np.sum(dense * G)) - energy) <= 1e-12 * float(np.sum(np.abs(dense * G))) + 1e-14
    gpos, gstrain, gcell = run_backward(state, G, len(sizes), torch.float64)
    assert_close(gpos, forces, 1e-10, 1e-12, f"{name} dE/dpositions")
    if periodic:
        assert_close(gstrain, strain, 1e-10, 1e-12, f"{name} dE/dstrain")
        assert_close(gcell, cell, 1e-10, 1e-12, f"{name} dE/dcell")


def rotation(seed):
    q = np.random.default_rng(seed).normal(size=4)
    w, x, y, z = q / np.linalg.norm(q)
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def off_pole_box(cutoff):
    """A small strained periodic box (with self images at this cutoff),
    rotated so that no pair direction is within sin(theta) <= 0.12 of the z
    axis: there featomic's Y_lm gradient switches to an approximate formula
    (spherical_harmonics.rs:285-297, reproduced by this library) that is not
    the exact derivative of Y_lm, so finite differences would not match it."""
    base = workloads.random_box(30, density=0.1, min_distance=0.9, seed=8, strain=0.02)
    for seed in range(1000):
        R = rotation(seed)
        pos, cell = base["positions"] @ R.T, base["cell"] @ R.T
        nl = rb.neighbor_list(pos, cell, cutoff)
        u = nl["vector"] / nl["distance"][:, None]
        if np.min(np.hypot(u[:, 0], u[:, 1])) > 0.12:
            return {"types": base["types"], "positions": pos, "cell": cell}
    raise RuntimeError("no rotation keeps every pair away from the z axis")


def test_adjoint_matches_finite_differences():
    cutoff = 3.5
    box = off_pole_box(cutoff)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(cutoff, 7, 6))
    systems = [box]
    values, state = run_dense(calc, systems)
    species = state.species()
    n_props = values.shape[2]
    positions, types, cells, sizes = batch(systems)
    weights = linear_weights([int(s) for s in species], n_props, seed=5)
    G = dense_grad_values(types, species, weights, n_props)
    gpos, gstrain, gcell = run_backward(state, G, 1, torch.float64)

    def energy(pos, cell):
        v, _ = run_dense(calc, [{"types": types, "positions": pos, "cell": cell}])
        return float(np.sum(v.cpu().numpy() * G))

    h = 1e-5
    cell0 = cells[0].reshape(3, 3)
    fd_pos = np.zeros_like(positions)
    for atom in range(len(positions)):
        for x in range(3):
            p1, p2 = positions.copy(), positions.copy()
            p1[atom, x] += h
            p2[atom, x] -= h
            fd_pos[atom, x] = (energy(p1, cell0) - energy(p2, cell0)) / (2 * h)
    assert_close(gpos, fd_pos, 1e-6, 1e-6, "finite differences, positions")

    fd_cell, fd_strain = [], []
    for a in range(3):
        for b in range(3):
            c1, c2 = cell0.copy(), cell0.copy()
            c1[a, b] += h
            c2[a, b] -= h
            fd_cell.append((energy(positions, c1) - energy(positions, c2)) / (2 * h))
            eps = np.zeros((3, 3))
            eps[a, b] = h
            up, down = np.eye(3) + eps, np.eye(3) - eps
            fd_strain.append((energy(positions @ up, cell0 @ up) - energy(positions @ down, cell0 @ down)) / (2 * h))
    assert_close(gcell[0].reshape(-1), fd_cell, 1e-6, 1e-6, "finite differences, cell")
    assert_close(gstrain[0].reshape(-1), fd_strain, 1e-6, 1e-6, "finite differences, strain")


def test_fp32_error_against_fp64():
    box = workloads.random_box(1000, density=0.1, min_distance=0.9, seed=2)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.5, 7, 6))
    v64, s64 = run_dense(calc, [box], 64)
    v32, s32 = run_dense(calc, [box], 32)
    a64 = v64.cpu().numpy()
    a32 = v32.double().cpu().numpy()
    err = np.max(np.abs(a32 - a64)) / np.max(np.abs(a64))
    assert err <= 1e-4, err
    positions, types, cells, sizes = batch([box])
    species = s64.species()
    weights = linear_weights([int(s) for s in species], a64.shape[2], seed=3)
    G = dense_grad_values(types, species, weights, a64.shape[2])
    f64, st64, _ = run_backward(s64, G, 1, torch.float64)
    f32, st32, _ = run_backward(s32, G, 1, torch.float32)
    ferr = np.max(np.abs(f32 - f64)) / np.max(np.abs(f64))
    serr = np.max(np.abs(st32 - st64)) / np.max(np.abs(st64))
    assert ferr <= 1e-4, ferr
    assert serr <= 1e-4, serr


def test_torch_autograd_through_blocks():
    from rascaline_b200 import torch_api

    box = workloads.random_box(200, density=0.1, min_distance=0.9, seed=6, strain=0.02)
    hypers = workloads.hypers(5.0, 7, 6)
    calc = rb.SoapPowerSpectrum(**hypers)
    tm = calc.compute(rb.System.from_dict(box), gradients=["positions", "cell"]).to_dict(["positions", "cell"])

    tcalc = torch_api.SoapPowerSpectrum(**hypers, precision=64)
    positions = torch.tensor(box["positions"], device="cuda", requires_grad=True)
    cell = torch.tensor(box["cell"], device="cuda", requires_grad=True)
    result = tcalc.compute([torch_api.System(box["types"], positions, cell)])
    species = sorted(set(int(t) for t in box["types"]))
    n_props = tm["blocks"][0]["values"].shape[1]
    weights = linear_weights(species, n_props, seed=9)
    np.testing.assert_array_equal(result.keys.values, tm["keys"])
    energy = 0.0
    for key, block, ref in zip(result.keys.values, result.blocks(), tm["blocks"]):
        np.testing.assert_array_equal(block.samples.values, ref["samples"])
        assert_close(block.values.detach().cpu().numpy(), ref["values"], 1e-12, 1e-14, "torch block values")
        W = torch.as_tensor(weights[tuple(int(k) for k in key)], device="cuda")
        energy = energy + (block.values @ W).sum()
    energy.backward()
    _, forces, _, cell_grad = explicit_energy_gradients(tm, weights, [len(box["types"])])
    assert_close(positions.grad.cpu().numpy(), forces, 1e-10, 1e-12, "torch dE/dpositions")
    assert_close(cell.grad.cpu().numpy(), cell_grad[0], 1e-10, 1e-12, "torch dE/dcell")


def test_torch_gradcheck_small_system():
    from rascaline_b200 import torch_api

    rng = np.random.default_rng(17)
    cell = torch.tensor(np.diag([5.0, 5.5, 6.0]) + rng.uniform(-0.2, 0.2, (3, 3)), device="cuda",
                        requires_grad=True)
    frac = rng.uniform(0.0, 1.0, (6, 3))
    positions = torch.tensor(frac @ cell.detach().cpu().numpy(), device="cuda", requires_grad=True)
    types = [1, 1, 8, 8, 6, 1]
    tcalc = torch_api.SoapPowerSpectrum(**workloads.hypers(3.0, 3, 2), precision=64)

    def f(pos, c):
        return tcalc.dense([torch_api.System(types, pos, c)])

    assert torch.autograd.gradcheck(f, (positions, cell), eps=1e-6, atol=1e-7, rtol=1e-5, fast_mode=True)
