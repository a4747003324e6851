"""The adjoint form on the 20 000-atom strained box (density 0.1 A^-3, 4
species, seeded cell strain of +-2 %, rc 5 A, max_radial 7, max_angular 6):
forces and virial of a linear energy model E = sum_i w[type_i] . P_i with
seeded N(0, 1/sqrt(d)) weights.

* Against the drop-in's explicit gradients (featomic's positions and strain
  gradient blocks, all of them, kept in GPU memory: about 50 GB in FP64)
  contracted with the weights: |d| <= 1e-10 |ref| + 1e-12 max|ref|.
* Against central finite differences of E (h = 1e-5 A, FP64) for three atoms
  whose pair directions all stay away from the z axis (featomic's Y_lm
  gradient switches to an approximate formula there,
  spherical_harmonics.rs:285-297): |d| <= 1e-6 max|ref| + 1e-6 |ref|; and
  for the strain, where every pair contributes (those in the pole cone
  included): |d| <= 1e-2 max|ref|.
"""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads

from test_dense_adjoint import assert_close, dense_grad_values, linear_weights

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

N_ATOMS = 20000


@pytest.fixture(scope="module")
def c5():
    box = workloads.random_box(N_ATOMS, density=0.1, min_distance=0.9, seed=5, strain=0.02)
    hypers = workloads.hypers(5.0, 7, 6)
    calc = rb.SoapPowerSpectrum(**hypers)
    species = np.unique(box["types"]).astype(np.int32)
    n_props = 7 * 8 * 8
    weights = linear_weights([int(s) for s in species], n_props, seed=19)
    G = dense_grad_values(box["types"], species, weights, n_props)
    return box, calc, species, weights, G


def adjoint(calc, box, G):
    from rascaline_b200.torch_api import dense_backward, dense_power_spectrum
    pos = torch.tensor(box["positions"], device="cuda")
    values, state = dense_power_spectrum(calc, pos, box["types"], np.asarray(box["cell"]).reshape(1, 9),
                                         [len(box["types"])], 64)
    g = torch.as_tensor(G, device="cuda")
    forces, strain, _ = dense_backward(state, g, 1, strain=True, cell=False)
    energy = float((values * g).sum())
    return energy, forces.cpu().numpy(), strain[0].cpu().numpy()


def test_adjoint_matches_explicit_gradients(c5):
    box, calc, species, weights, G = c5
    energy, forces, strain = adjoint(calc, box, G)
    pos = torch.tensor(box["positions"], device="cuda")
    tm = calc.compute_device(pos, box["types"], np.asarray(box["cell"]).reshape(1, 9), [N_ATOMS],
                             gradients=["positions", "strain"])
    torch.cuda.synchronize()
    f_ref = torch.zeros((N_ATOMS, 3), dtype=torch.float64, device="cuda")
    s_ref = torch.zeros((3, 3), dtype=torch.float64, device="cuda")
    e_ref = 0.0
    for key, block in zip(tm.keys.values, tm.blocks()):
        W = torch.as_tensor(weights[tuple(int(k) for k in key)], device="cuda")
        e_ref += float((block.values @ W).sum())
        grad = block.gradient("positions")
        atoms = torch.as_tensor(grad.samples.values[:, 2].astype(np.int64), device="cuda")
        f_ref.index_add_(0, atoms, grad.values @ W)
        s_ref += (block.gradient("strain").values @ W).sum(dim=0)
    del tm
    assert abs(energy - e_ref) <= 1e-10 * abs(e_ref)
    assert_close(forces, f_ref.cpu().numpy(), 1e-10, 1e-12, "c5 dE/dpositions vs explicit gradients")
    assert_close(strain, s_ref.cpu().numpy(), 1e-10, 1e-12, "c5 dE/dstrain vs explicit gradients")


def test_adjoint_matches_finite_differences(c5):
    box, calc, species, weights, G = c5
    _, forces, strain = adjoint(calc, box, G)
    nl = rb.neighbor_list(box["positions"], box["cell"], 5.0)
    u = nl["vector"] / nl["distance"][:, None]
    off_pole = np.hypot(u[:, 0], u[:, 1]) > 0.12
    near = np.zeros(N_ATOMS, dtype=bool)
    near[nl["first"][~off_pole]] = True
    near[nl["second"][~off_pole]] = True
    # three atoms whose pairs are all off the pole cone (the energy depends
    # on an atom's position through its own pairs only)
    atoms = [int(a) for a in np.nonzero(~near)[0][:3]]
    assert len(atoms) == 3
    h = 1e-5
    positions = np.asarray(box["positions"])
    cell = np.asarray(box["cell"])

    def energy(p, c):
        e, _, _ = adjoint(calc, {"types": box["types"], "positions": p, "cell": c}, G)
        return e

    fd = np.zeros((3, 3))
    for k, a in enumerate(atoms):
        for x in range(3):
            p1, p2 = positions.copy(), positions.copy()
            p1[a, x] += h
            p2[a, x] -= h
            fd[k, x] = (energy(p1, cell) - energy(p2, cell)) / (2 * h)
    assert_close(forces[atoms], fd, 1e-6, 1e-6, "c5 finite differences, positions")
    # strain: positions and cell deformed together.  Every pair contributes,
    # including the ~0.5 % within featomic's pole cone, where its gradient is
    # not the derivative of Y_lm: a looser bound
    fd_strain = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            eps = np.zeros((3, 3))
            eps[a, b] = h
            up, down = np.eye(3) + eps, np.eye(3) - eps
            fd_strain[a, b] = (energy(positions @ up, cell @ up) - energy(positions @ down, cell @ down)) / (2 * h)
    scale = np.max(np.abs(strain))
    assert np.max(np.abs(strain - fd_strain)) <= 1e-2 * scale, (strain, fd_strain)
