"""Learned radial surrogate: training set, training kernels, output-layer
fit, inference kernels.

* The training targets (the exact analytic GTO radial integral and its
  r-derivative, evaluated on the GPU) match the CPU oracle's analytic radial
  integral to 1e-6 of each output's largest magnitude (FP32 roundings of FP64
  values).
* The loss (values plus lambda times x-derivatives) and the gradient of the
  GPU training kernels (FP32) match the FP64 restatement in
  oracle/surrogate_reference.py (torch autograd on the CPU):
  |d| <= 1e-3 |ref| + 1e-4 max|ref|.
* The least-squares refit of the output layer on the GPU (fitted on the
  tensor-core kernel's own features) predicts the same outputs as the FP64
  restatement of the fit to 5e-4 of the largest output, and its residual is
  at most a fifth of the Adam weights' residual.
* The tensor-core inference kernel (tcgen05, weights and activations as three
  BF16 parts, FP32 accumulation) matches the CUDA-core evaluation of the same
  network with FP32 weights and the FP64 reference to 2e-4 of each output's
  largest magnitude.
* Errors against the exact integral on r in [0.9, 6] A, per output relative to
  its largest magnitude: values RMS <= 2e-5 and max <= 2e-4, derivatives max
  <= 2e-3; the single-BF16 control is at least ten times worse.
* What the trained network gains over the method without it (the FP64
  spline of the same radial integral): more evaluations per second.
* Attached to a calculator, it replaces the spline in the FP32 dense power
  spectrum and adjoint: power spectrum within 1e-4 of FP64, forces within
  1e-3.
"""
import os
import sys

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
from oracle import surrogate_reference as ref  # noqa: E402

HYPERS = workloads.hypers(6.0, 11, 8)  # max_angular 8, max_radial 11: 108 outputs
CUTOFF = 6.0


@pytest.fixture(scope="module")
def trained():
    from rascaline_b200.surrogate import RadialSurrogate
    calc = rb.SoapPowerSpectrum(**HYPERS)
    s = RadialSurrogate(calc, seed=3)
    s.make_dataset(1 << 20, seed=7)
    loss = s.train(20000, 8192, 3e-3, derivative_weight=0.1)
    s.fit_output_layer(0.01)
    return calc, s, loss


def test_training_set_matches_oracle(oracle):
    from rascaline_b200.surrogate import RadialSurrogate
    calc = rb.SoapPowerSpectrum(**HYPERS)
    s = RadialSurrogate(calc, seed=1)
    s.make_dataset(4096, seed=11)
    r = s.samples()
    values, derivs = s.evaluate(torch.as_tensor(r.astype(np.float64), device="cuda"), "analytic")
    analytic = dict(HYPERS)
    analytic["basis"] = dict(HYPERS["basis"])
    analytic["basis"]["spline_accuracy"] = None
    expected, expected_d = oracle.radial_integral(analytic, r[:512].astype(np.float64))
    got = values[:512].cpu().numpy().reshape(512, 9, 12)
    got_d = derivs[:512].cpu().numpy().reshape(512, 9, 12)
    for a, e in ((got, expected), (got_d, expected_d)):
        scale = np.abs(e).max(axis=0) + 1e-30
        assert np.max(np.abs(a - e) / scale) <= 1e-6
    assert np.all((r >= 0.0) & (r <= CUTOFF))


def test_training_gradient_matches_reference():
    from rascaline_b200.surrogate import RadialSurrogate
    calc = rb.SoapPowerSpectrum(**HYPERS)
    s = RadialSurrogate(calc, seed=5)
    s.make_dataset(2048, seed=13)
    s.train(50, 512, 3e-3, derivative_weight=0.1)  # away from the initial weights
    n = 300
    loss, grad = s.loss_and_gradient(n, derivative_weight=0.1)
    r = s.samples()[:n]
    values, derivs = s.evaluate(torch.as_tensor(r.astype(np.float64), device="cuda"), "analytic")
    targets = values.cpu().numpy().astype(np.float64) / s.scales.astype(np.float64)
    dtargets = derivs.cpu().numpy().astype(np.float64) / s.scales.astype(np.float64)
    ref_loss, ref_grad = ref.loss_and_gradient(s.parameters, 64, s.n_outputs, r, targets, CUTOFF, dtargets, 0.1)
    assert abs(loss - ref_loss) <= 1e-3 * ref_loss
    bound = 1e-3 * np.abs(ref_grad) + 1e-4 * np.max(np.abs(ref_grad))
    bad = np.abs(grad - ref_grad) > bound
    assert not bad.any(), (np.argmax(np.abs(grad - ref_grad) - bound), bad.sum())


def test_output_layer_fit_matches_reference():
    from rascaline_b200.surrogate import RadialSurrogate
    calc = rb.SoapPowerSpectrum(**HYPERS)
    s = RadialSurrogate(calc, seed=9)
    s.make_dataset(4096, seed=17)
    s.train(300, 1024, 3e-3, derivative_weight=0.1)
    before = s.parameters
    s.fit_output_layer(0.01)
    fitted = s.parameters
    r = s.samples()
    values, derivs = s.evaluate(torch.as_tensor(r.astype(np.float64), device="cuda"), "analytic")
    targets = values.cpu().numpy().astype(np.float64) / s.scales.astype(np.float64)
    dtargets = derivs.cpu().numpy().astype(np.float64) / s.scales.astype(np.float64)
    expected = ref.fit_output_layer(before, 64, s.n_outputs, r, targets, dtargets, CUTOFF, 0.01)
    # the hidden layers are untouched
    n_hidden = 3 * 64 + 64 * 64
    np.testing.assert_array_equal(fitted[:n_hidden], before[:n_hidden])
    # the same predictions (the GPU fits the tensor-core kernel's FP32
    # features, the reference FP64 features of the same network) and as
    # small a residual
    y, _ = ref.forward(fitted, 64, s.n_outputs, r, CUTOFF)
    y_ref, _ = ref.forward(expected, 64, s.n_outputs, r, CUTOFF)
    assert np.max(np.abs(y - y_ref)) <= 5e-4 * np.max(np.abs(y_ref))
    # the fit is what makes the network accurate: its residual is far below
    # the one of the Adam weights it replaces
    y_adam, _ = ref.forward(before, 64, s.n_outputs, r, CUTOFF)
    rms = np.sqrt(np.mean((y - targets) ** 2))
    rms_adam = np.sqrt(np.mean((y_adam - targets) ** 2))
    assert rms <= 0.2 * rms_adam, (rms, rms_adam)


def test_tensor_core_inference_matches_cuda_cores_and_reference(trained):
    calc, s, _ = trained
    r = torch.linspace(0.0, CUTOFF, 5003, dtype=torch.float64, device="cuda")
    tc, dtc = s.evaluate(r, "tensor_cores")
    cc, dcc = s.evaluate(r, "cuda_cores")
    y, dy = ref.forward(s.parameters, 64, s.n_outputs, r.cpu().numpy(), CUTOFF)
    scales = s.scales.astype(np.float64)
    y, dy = y * scales, dy * scales
    for got, expected in ((tc, y), (dtc, dy), (cc, y), (dcc, dy)):
        got = got.double().cpu().numpy()
        scale = np.abs(expected).max(axis=0) + 1e-30
        assert np.max(np.abs(got - expected) / scale) <= 2e-4


def test_surrogate_error_and_gain_over_the_spline(trained):
    calc, s, loss = trained
    r = torch.linspace(0.9, CUTOFF, 20001, dtype=torch.float64, device="cuda")
    exact, dexact = s.evaluate(r, "analytic")
    scale, dscale = exact.abs().amax(dim=0), dexact.abs().amax(dim=0)

    def errors(method):
        v, d = s.evaluate(r, method)
        e, de = (v - exact) / scale, (d - dexact) / dscale
        return float((e ** 2).mean().sqrt()), float(e.abs().max()), float(de.abs().max())

    rms, vmax, dmax = errors("tensor_cores")
    assert rms <= 2e-5, rms
    assert vmax <= 2e-4, vmax
    assert dmax <= 2e-3, dmax
    # the single-BF16 control: one BF16 per weight is far from enough
    _, control_max, _ = errors("bf16_single")
    assert control_max >= 10 * vmax, (control_max, vmax)
    # throughput against the method without the network: the FP64 spline
    n = 1 << 22
    rr = torch.rand(n, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(3)) * CUTOFF
    rates = {}
    for method in ("tensor_cores", "spline"):
        # warm up at the full size, so that the timed calls reuse the cached
        # output buffers instead of timing their allocation
        s.evaluate(rr, method)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(3):
            s.evaluate(rr, method)
        e1.record()
        torch.cuda.synchronize()
        rates[method] = 3 * n / e0.elapsed_time(e1)
    assert rates["tensor_cores"] > rates["spline"], rates


def test_dense_fp32_with_surrogate(trained):
    from rascaline_b200.torch_api import dense_backward, dense_power_spectrum
    calc, s, _ = trained
    box = workloads.random_box(300, density=0.1, min_distance=0.9, seed=4)
    pos = torch.as_tensor(box["positions"], device="cuda")
    types = box["types"]
    cells = np.asarray(box["cell"]).reshape(1, 9)
    v64, st64 = dense_power_spectrum(calc, pos, types, cells, [300], 64)
    v32, st32 = dense_power_spectrum(calc, pos, types, cells, [300], 32)
    s.attach()
    try:
        vm, stm = dense_power_spectrum(calc, pos, types, cells, [300], 32)
        G = torch.randn(v64.shape, dtype=torch.float64, device="cuda", generator=torch.Generator("cuda").manual_seed(5))
        f64, _, _ = dense_backward(st64, G, 1, cell=False)
        fm, _, _ = dense_backward(stm, G.float(), 1, cell=False)
    finally:
        s.attach(False)
    spline_err = float((v32.double() - v64).abs().max() / v64.abs().max())
    mlp_err = float((vm.double() - v64).abs().max() / v64.abs().max())
    force_err = float((fm.double() - f64).abs().max() / f64.abs().max())
    assert spline_err <= 1e-5
    assert mlp_err <= 1e-4, mlp_err
    assert force_err <= 1e-3, force_err
    # detached again: the spline is back
    v32b, _ = dense_power_spectrum(calc, pos, types, cells, [300], 32)
    assert torch.equal(v32b, v32)


def test_freed_surrogate_falls_back_to_the_spline():
    from rascaline_b200.surrogate import RadialSurrogate
    from rascaline_b200.torch_api import dense_power_spectrum
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 5, 4))
    box = workloads.random_box(64, density=0.1, min_distance=0.9, seed=8)
    pos = torch.as_tensor(box["positions"], device="cuda")
    cells = np.asarray(box["cell"]).reshape(1, 9)
    spline, _ = dense_power_spectrum(calc, pos, box["types"], cells, [64], 32)
    s = RadialSurrogate(calc, seed=2)
    s.make_dataset(1024, seed=1)
    s.attach()
    del s
    again, _ = dense_power_spectrum(calc, pos, box["types"], cells, [64], 32)
    assert torch.equal(spline, again)
    # and a surrogate can outlive its calculator
    calc2 = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 5, 4))
    s2 = RadialSurrogate(calc2, seed=2)
    s2.attach()
    del calc2
    s2._calculator = None
    del s2


def test_batched_pipeline_with_surrogate_keeps_the_pair_features(trained):
    # The batch's dense pipeline asks for forces, so its forward pass computes
    # the surrogate's pair features with their derivatives once and its
    # backward reuses them.  Values and forces must agree with the dense
    # forward + backward, whose backward evaluates the network again
    # (tolerance 1e-4 of the largest force: the two sum dL/dc in different
    # orders in FP32).
    from rascaline_b200.torch_api import Batch, dense_backward, dense_power_spectrum
    calc, s, _ = trained
    mols = workloads.molecules(24, seed=11)
    positions = np.concatenate([m["positions"] for m in mols])
    types = np.concatenate([m["types"] for m in mols]).astype(np.int32)
    sizes = np.array([len(m["types"]) for m in mols])
    species = [1, 6, 7, 8]
    batch = Batch(calc, sizes, types, species)
    rng = np.random.default_rng(3)
    W = rng.normal(0.0, 1.0 / np.sqrt(batch.n_keys * batch.n_properties),
                   size=(len(species), batch.n_keys, batch.n_properties))
    weights = torch.as_tensor(W, dtype=torch.float32, device="cuda").contiguous()
    pos = torch.as_tensor(positions, device="cuda")
    out = batch.outputs()
    batch.config = {"warps": 4, "chunk": 32, "layout": 1, "ctas_per_sm": 2, "pipeline": 1}
    s.attach()
    try:
        batch.run(pos, out, weights=weights)
        values, state = dense_power_spectrum(calc, pos, types, np.zeros((len(mols), 9)), sizes, 32, species)
        G = torch.as_tensor(W[np.searchsorted(species, types)], dtype=torch.float32, device="cuda")
        grad, _, _ = dense_backward(state, G, len(mols), strain=False, cell=False)
        torch.cuda.synchronize()
    finally:
        s.attach(False)

    def rel(a, b):
        return float((a.double() - b.double()).abs().max() / b.double().abs().max())

    assert rel(out["values"], values) <= 1e-6
    assert rel(out["gradients"], grad) <= 1e-4
