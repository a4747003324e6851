"""featomic-torch's ``register_autograd`` (featomic-torch/src/calculator.cpp:
314-383): a TensorMap computed with explicit positions and cell gradients,
connected to the systems' positions and cells.  The backward contracts dA/dX
with the explicit gradient blocks (PositionsGrad / CellGrad,
featomic-torch/src/autograd.cpp:237-317, :429-503).

* the gradients of a linear energy equal the adjoint path's (the
  torch_api calculator, which never builds gradient blocks) to 1e-10;
* the backward is differentiable with respect to dA/dX: gradcheck of the
  forces and of the cell gradient with respect to the model weights, with
  featomic-torch's warning about second derivatives;
* the precomputed TensorMap must hold the gradients the systems ask for, and
  ``forward_gradients`` selects the gradients kept in the result.
"""
import warnings

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _system(seed=29, n=14):
    rng = np.random.default_rng(seed)
    cell = np.diag([5.2, 5.6, 6.1]) + rng.uniform(-0.3, 0.3, (3, 3))
    positions = rng.uniform(0.0, 1.0, (n, 3)) @ cell
    types = rng.choice([1, 6, 8], size=n).astype(np.int32)
    return types, positions, cell


HYPERS = workloads.hypers(3.5, 3, 2)


def _precomputed(types, positions, cell, gradients):
    calc = rb.SoapPowerSpectrum(**HYPERS)
    pos = torch.tensor(positions, device="cuda")
    return calc.compute_device(pos, types, np.asarray(cell).reshape(1, 9), [len(types)], gradients=gradients)


def _energy(tm, weights):
    return sum((b.values.reshape(b.values.shape[0], -1) @ weights[tuple(int(x) for x in k)]).sum()
               for k, b in zip(tm.keys.values, tm.blocks()))


def test_register_autograd_matches_the_adjoint():
    from rascaline_b200 import torch_api
    types, positions, cell = _system()
    tm = _precomputed(types, positions, cell, ["positions", "cell"])
    rng = np.random.default_rng(3)
    weights = {tuple(int(x) for x in k): torch.tensor(rng.normal(size=(b.values.shape[1], 1)), device="cuda")
               for k, b in zip(tm.keys.values, tm.blocks())}
    pos = torch.tensor(positions, device="cuda", requires_grad=True)
    c = torch.tensor(cell, device="cuda", requires_grad=True)
    attached = torch_api.register_autograd([torch_api.System(types, pos, c)], tm)
    _energy(attached, weights).backward()

    pos2 = torch.tensor(positions, device="cuda", requires_grad=True)
    c2 = torch.tensor(cell, device="cuda", requires_grad=True)
    adjoint = torch_api.SoapPowerSpectrum(**HYPERS, precision=64).compute([torch_api.System(types, pos2, c2)])
    np.testing.assert_array_equal(adjoint.keys.values, attached.keys.values)
    _energy(adjoint, weights).backward()
    for a, b in ((pos.grad, pos2.grad), (c.grad, c2.grad)):
        a, b = a.cpu().numpy(), b.cpu().numpy()
        assert np.all(np.abs(a - b) <= 1e-10 * np.abs(b) + 1e-12 * np.max(np.abs(b))), np.max(np.abs(a - b))


@pytest.mark.parametrize("wrt", ["positions", "cell"])
def test_register_autograd_double_backward(wrt):
    from rascaline_b200 import torch_api
    types, positions, cell = _system(seed=31, n=10)
    tm = _precomputed(types, positions, cell, ["positions", "cell"])
    pos = torch.tensor(positions, device="cuda", requires_grad=(wrt == "positions"))
    c = torch.tensor(cell, device="cuda", requires_grad=(wrt == "cell"))
    n_props = tm.block_by_id(0).values.shape[1]
    keys = [tuple(int(x) for x in k) for k in tm.keys.values]
    w0 = torch.rand((len(keys) * n_props, 1), dtype=torch.float64, device="cuda", requires_grad=True)

    def forces(w):
        attached = torch_api.register_autograd([torch_api.System(types, pos, c)], tm)
        weights = {k: w[i * n_props:(i + 1) * n_props] for i, k in enumerate(keys)}
        energy = _energy(attached, weights)
        return torch.autograd.grad(energy, pos if wrt == "positions" else c, create_graph=True)[0]

    what = "positions" if wrt == "positions" else "cell matrix"
    message = f"second derivatives with respect to {what} are not implemented"
    with pytest.warns(UserWarning, match=message):
        forces(w0).sum().backward()
    with warnings.catch_warnings():
        warnings.filterwarnings("ignore", message=message)
        assert torch.autograd.gradcheck(forces, (w0,), fast_mode=True)


def test_register_autograd_checks():
    from rascaline_b200 import torch_api
    types, positions, cell = _system(seed=37, n=8)
    tm = _precomputed(types, positions, cell, ["positions"])
    pos = torch.tensor(positions, device="cuda")
    c = torch.tensor(cell, device="cuda", requires_grad=True)
    with pytest.raises(ValueError, match="gradients with respect to 'cell'"):
        torch_api.register_autograd([torch_api.System(types, pos, c)], tm)
    pos.requires_grad_(True)
    attached = torch_api.register_autograd([torch_api.System(types, pos, c.detach())], tm, forward_gradients=[])
    assert attached.block(0).gradients_list() == []
    attached = torch_api.register_autograd([torch_api.System(types, pos, c.detach())], tm)
    assert attached.block(0).gradients_list() == ["positions"]
