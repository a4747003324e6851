"""Explicit spherical-expansion basis (featomic/src/calculators/shared/basis/
mod.rs:60-116): one GTO radial basis per angular channel.

The GTO functions of channel l depend only on l and on that channel's number
of functions, and its spline is built from them alone, so every channel of an
Explicit basis equals the same channel of a TensorProduct basis of that size.
The GPU tests check exactly that (values and gradients) against the
TensorProduct path, which the other parity tests pin to the oracle; the CPU
tests check the parameter rules."""
import json

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads


def explicit(cutoff, sizes, spline_accuracy=1e-8):
    h = workloads.hypers(cutoff, 1, 1)
    h["basis"] = {"type": "Explicit",
                  "by_angular": {str(l): {"type": "Gto", "max_radial": n - 1} for l, n in sizes.items()}}
    if spline_accuracy != 1e-8:
        h["basis"]["spline_accuracy"] = spline_accuracy
    return h


def test_explicit_basis_parameters():
    calc = rb.SoapPowerSpectrum(**explicit(4.0, {0: 4, 2: 3}))
    assert json.loads(calc.parameters)["basis"]["type"] == "Explicit"
    with pytest.raises(rb.FeatomicError, match="invalid digit"):
        h = explicit(4.0, {0: 4})
        h["basis"]["by_angular"]["x"] = {"type": "Gto", "max_radial": 2}
        rb.SoapPowerSpectrum(**h)
    with pytest.raises(rb.FeatomicError, match="unknown field `max_angular`"):
        h = explicit(4.0, {0: 4})
        h["basis"]["max_angular"] = 3
        rb.SoapPowerSpectrum(**h)
    with pytest.raises(rb.FeatomicError, match="Tabulated"):
        h = explicit(4.0, {0: 4})
        h["basis"]["by_angular"]["1"] = {"type": "Tabulated", "file": "x"}
        rb.SoapPowerSpectrum(**h)
    with pytest.raises(rb.FeatomicError, match="spline_accuracy can not be null"):
        h = explicit(4.0, {0: 4})
        h["basis"]["spline_accuracy"] = None
        rb.SoapPowerSpectrum(**h)


def _blocks(tm):
    return {tuple(k): b for k, b in zip(tm.keys.values, tm.blocks())}


GRADS = ["positions", "strain"]


@pytest.mark.gpu
@pytest.mark.parametrize("sizes", [{0: 6, 1: 4, 2: 5}, {0: 4, 2: 5}])
def test_explicit_spherical_expansion_equals_tensor_product(sizes):
    system = rb.System.from_dict(workloads.random_box(80, density=0.1, seed=31, strain=0.01))
    out = _blocks(rb.SphericalExpansion(**explicit(4.5, sizes)).compute(system, gradients=GRADS))
    lmax = max(sizes)
    assert {k[0] for k in out} == set(sizes)
    for l, n in sizes.items():
        ref = _blocks(rb.SphericalExpansion(**workloads.hypers(4.5, n - 1, lmax)).compute(system, gradients=GRADS))
        for key, block in out.items():
            if key[0] != l:
                continue
            r = ref[key]
            np.testing.assert_array_equal(block.samples.values, r.samples.values)
            np.testing.assert_array_equal(block.properties.values, r.properties.values)
            np.testing.assert_array_equal(block.values, r.values)
            for g in GRADS:
                np.testing.assert_array_equal(block.gradient(g).samples.values, r.gradient(g).samples.values)
                np.testing.assert_array_equal(block.gradient(g).values, r.gradient(g).values)


@pytest.mark.gpu
@pytest.mark.parametrize("sizes", [{0: 4, 1: 6, 2: 3}, {0: 3, 2: 4}])
def test_explicit_power_spectrum_equals_tensor_product(sizes):
    system = rb.System.from_dict(workloads.random_box(80, density=0.1, seed=32, strain=0.01))
    out = _blocks(rb.SoapPowerSpectrum(**explicit(4.5, sizes)).compute(system, gradients=GRADS))
    lmax = max(sizes)
    expected_props = [(l, a, b) for l in sorted(sizes) for a in range(sizes[l]) for b in range(sizes[l])]
    for l, n in sizes.items():
        ref = _blocks(rb.SoapPowerSpectrum(**workloads.hypers(4.5, n - 1, lmax)).compute(system, gradients=GRADS))
        for key, block in out.items():
            props = [tuple(p) for p in block.properties.values]
            assert props == expected_props
            cols = [i for i, p in enumerate(props) if p[0] == l]
            r = ref[key]
            rcols = [i for i, p in enumerate(r.properties.values) if p[0] == l]
            np.testing.assert_array_equal(block.samples.values, r.samples.values)
            np.testing.assert_array_equal(block.values[:, cols], r.values[:, rcols])
            for g in GRADS:
                np.testing.assert_array_equal(block.gradient(g).values[..., cols], r.gradient(g).values[..., rcols])


@pytest.mark.gpu
def test_explicit_basis_rejected_by_the_dense_forms():
    from rascaline_b200.torch_api import dense_power_spectrum
    import torch
    calc = rb.SoapPowerSpectrum(**explicit(4.0, {0: 3, 1: 3}))
    s = workloads.random_box(20, density=0.1, seed=3)
    with pytest.raises(rb.FeatomicError, match="Explicit"):
        dense_power_spectrum(calc, torch.tensor(s["positions"], device="cuda"), s["types"],
                             np.asarray(s["cell"]).reshape(1, 9), [20], 32)
