"""Double backward and the torch spherical expansion.

featomic-torch makes its backward pass differentiable with respect to dA/dX
(featomic-torch/src/autograd.cpp:318-426) and tests it with gradcheck of the
forces and virial with respect to the weights of a linear model
(python/featomic_torch/tests/autograd.py:154-225).  Here the double backward
is the forward-mode derivative (JVP) of the dense forms:

* the JVP and the adjoint are transposes of each other:
  <G, J u> = <J^T G, u> for random G and displacements u of positions and
  cell, to 1e-12 relative (FP64);
* the JVP matches central finite differences of the power spectrum
  (h = 1e-5 A, FP64) to 1e-6 of the largest magnitude, on a box with no pair
  direction near the z axis (featomic's approximate Y_lm gradient there);
* gradcheck of the forces and of the cell gradient with respect to the
  weights passes, and a backward pass through positions warns that second
  derivatives with respect to positions (or the cell) are not accumulated;
* the torch SphericalExpansion equals the drop-in spherical expansion
  (1e-12), passes gradcheck with respect to positions and cell, and its
  double backward passes gradcheck with respect to the weights.
"""
import warnings

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads

from test_dense_adjoint import assert_close, batch, off_pole_box, run_dense

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def small_periodic(n=12, seed=17):
    rng = np.random.default_rng(seed)
    cell = np.diag([5.0, 5.5, 6.0]) + rng.uniform(-0.2, 0.2, (3, 3))
    positions = rng.uniform(0.0, 1.0, (n, 3)) @ cell
    types = rng.choice([1, 6, 8], size=n)
    return {"types": types, "positions": positions, "cell": cell}


def test_jvp_is_the_transpose_of_the_adjoint():
    from rascaline_b200.torch_api import dense_backward, dense_jvp

    box = workloads.random_box(150, density=0.1, min_distance=0.9, seed=41, strain=0.02)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(4.5, 5, 4))
    values, state = run_dense(calc, [box])
    rng = np.random.default_rng(3)
    G = torch.as_tensor(rng.normal(size=values.shape), device="cuda")
    u = torch.as_tensor(rng.normal(size=(len(box["types"]), 3)), device="cuda")
    U = torch.as_tensor(rng.normal(size=(1, 3, 3)), device="cuda")
    gpos, _, gcell = dense_backward(state, G, 1, strain=False, cell=True)
    tv, _ = dense_jvp(state, u, U)
    lhs = float((G * tv).sum())
    rhs = float((gpos * u).sum() + (gcell * U).sum())
    scale = float((G.abs() * tv.abs()).sum())
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)


def test_jvp_matches_finite_differences():
    from rascaline_b200.torch_api import dense_jvp

    cutoff = 3.5
    box = off_pole_box(cutoff)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(cutoff, 5, 4))
    values, state = run_dense(calc, [box])
    positions, types, cells, sizes = batch([box])
    rng = np.random.default_rng(11)
    u = rng.normal(size=positions.shape)
    U = 0.1 * rng.normal(size=(3, 3))
    tv, _ = dense_jvp(state, torch.as_tensor(u, device="cuda"), torch.as_tensor(U[None], device="cuda"))
    h = 1e-5
    cell0 = cells[0].reshape(3, 3)

    def P(sign):
        v, _ = run_dense(calc, [{"types": types, "positions": positions + sign * h * u,
                                 "cell": cell0 + sign * h * U}])
        return v.cpu().numpy()

    fd = (P(1) - P(-1)) / (2 * h)
    assert_close(tv.cpu().numpy(), fd, 1e-6, 1e-6, "JVP against finite differences")


def _forces_model(tcalc, system_args, weights, wrt):
    from rascaline_b200 import torch_api

    types, positions, cell = system_args
    X = tcalc.dense([torch_api.System(types, positions, cell)])
    A = (X.reshape(X.shape[0], -1) @ weights).sum()
    target = positions if wrt == "positions" else cell
    return torch.autograd.grad(A, target, create_graph=True)[0]


@pytest.mark.parametrize("wrt", ["positions", "cell"])
def test_double_backward_gradcheck_with_respect_to_weights(wrt):
    from rascaline_b200 import torch_api

    s = small_periodic()
    tcalc = torch_api.SoapPowerSpectrum(**workloads.hypers(3.0, 3, 2), precision=64)
    positions = torch.tensor(s["positions"], device="cuda", requires_grad=(wrt == "positions"))
    cell = torch.tensor(s["cell"], device="cuda", requires_grad=(wrt == "cell"))
    X = tcalc.dense([torch_api.System(s["types"], positions, cell)])
    weights = torch.rand((X.shape[1] * X.shape[2], 1), dtype=torch.float64, device="cuda", requires_grad=True)

    def compute(w):
        return _forces_model(tcalc, (s["types"], positions, cell), w, wrt)

    what = "positions" if wrt == "positions" else "cell matrix"
    message = f"second derivatives with respect to {what} are not implemented"
    with pytest.warns(UserWarning, match=message):
        compute(weights).sum().backward(retain_graph=True)
    with warnings.catch_warnings():
        warnings.filterwarnings("ignore", message=message)
        assert torch.autograd.gradcheck(compute, (weights,), fast_mode=True)


def test_torch_spherical_expansion_matches_the_drop_in():
    from rascaline_b200 import torch_api

    box = workloads.random_box(120, density=0.1, min_distance=0.9, seed=43, strain=0.02)
    hypers = workloads.hypers(4.5, 5, 4)
    tm = rb.SphericalExpansion(**hypers).compute(rb.System.from_dict(box)).to_dict()
    tcalc = torch_api.SphericalExpansion(**hypers, precision=64)
    positions = torch.tensor(box["positions"], device="cuda")
    cell = torch.tensor(box["cell"], device="cuda")
    result = tcalc.compute([torch_api.System(box["types"], positions, cell)])
    np.testing.assert_array_equal(result.keys.values, tm["keys"])
    for block, ref in zip(result.blocks(), tm["blocks"]):
        np.testing.assert_array_equal(block.samples.values, ref["samples"])
        assert_close(block.values.cpu().numpy(), ref["values"], 1e-12, 1e-14, "torch spherical expansion")
        assert block.components[0].names == ["o3_mu"]


def test_torch_spherical_expansion_gradients():
    from rascaline_b200 import torch_api

    s = small_periodic(seed=23)
    tcalc = torch_api.SphericalExpansion(**workloads.hypers(3.0, 3, 2), precision=64)
    positions = torch.tensor(s["positions"], device="cuda", requires_grad=True)
    cell = torch.tensor(s["cell"], device="cuda", requires_grad=True)

    def f(pos, c):
        return tcalc.dense([torch_api.System(s["types"], pos, c)])

    assert torch.autograd.gradcheck(f, (positions, cell), eps=1e-6, atol=1e-7, rtol=1e-5, fast_mode=True)

    X = f(positions.detach(), cell.detach())
    weights = torch.rand((X.shape[1] * X.shape[2], 1), dtype=torch.float64, device="cuda", requires_grad=True)
    pos = positions.detach().requires_grad_(True)

    def forces(w):
        return _forces_model(tcalc, (s["types"], pos, cell.detach()), w, "positions")

    with warnings.catch_warnings():
        warnings.filterwarnings("ignore", message="second derivatives with respect to")
        assert torch.autograd.gradcheck(forces, (weights,), fast_mode=True)
