"""C ABI checks that need no GPU: the library loads, exports every symbol
declared in include/*.h, and the host side (hyper-parameter parsing, status
codes, error messages, buffer sizes) behaves like featomic's C API
(featomic/src/c_api/calculator.rs, status.rs)."""
import ctypes
import glob
import json
import os
import re

import numpy as np
import pytest

from conftest import ROOT

import rascaline_b200 as rb
from rascaline_b200 import _c_api as C
from rascaline_b200.workloads import hypers


def declared_symbols():
    names = set()
    for header in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(header).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b((?:featomic|mts)_[a-z0-9_]+)\s*\(", text):
            if not m.group(1).endswith("_t"):  # types used as return types of callbacks
                names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(C.LIBRARY)
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # and the Python bindings declare every one of them
    assert names == set(C.SIGNATURES)


def test_calculator_metadata():
    calc = rb.SoapPowerSpectrum(**hypers(5.5, 7, 6))
    assert calc.name == "SOAP power spectrum"
    assert json.loads(calc.parameters) == hypers(5.5, 7, 6)
    assert calc.cutoffs == [5.5]
    se = rb.SphericalExpansion(**hypers(4.0, 3, 2))
    assert se.name == "spherical expansion"


def test_buffer_size_error():
    calc = rb.SoapPowerSpectrum(**hypers(5.5, 7, 6))
    buf = ctypes.create_string_buffer(4)
    status = C.lib().featomic_calculator_name(calc._handle, buf, 4)
    assert status == 254
    assert "not big enough" in C.lib().featomic_last_error().decode()


def test_null_pointers():
    status = C.lib().featomic_calculator_name(None, None, 0)
    assert status == 1
    assert "NULL pointer" in C.lib().featomic_last_error().decode()


def _create(name, params):
    handle = C.lib().featomic_calculator(name.encode(), params.encode())
    err = C.lib().featomic_last_error().decode()
    if handle:
        C.lib().featomic_calculator_free(handle)
    return handle, err


def test_unknown_calculator():
    handle, err = _create("not_a_calculator", "{}")
    assert not handle
    assert "unknown calculator with name 'not_a_calculator'" in err


@pytest.mark.parametrize("params, fragment", [
    ("{bad json", "key must be a string"),
    ('{"cutoff": {"radius": 5.0, "smoothing": {"type": "ShiftedCosine", "width": 0.5}, "extra": 1},'
     '"density": {"type": "Gaussian", "width": 0.3},'
     '"basis": {"type": "TensorProduct", "max_angular": 4, "radial": {"type": "Gto", "max_radial": 5}}}',
     "unknown field `extra`"),
    ('{"cutoff": {"radius": 5.0, "smoothing": {"type": "ShiftedCosine", "width": 0.5}},'
     '"density": {"type": "Gaussian", "width": 0.3},'
     '"basis": {"type": "TensorProduct", "max_angular": 4.5, "radial": {"type": "Gto", "max_radial": 5}}}',
     "expected usize"),
    ('{"cutoff": {"radius": 5.0, "smoothing": {"type": "Cosine", "width": 0.5}},'
     '"density": {"type": "Gaussian", "width": 0.3},'
     '"basis": {"type": "TensorProduct", "max_angular": 4, "radial": {"type": "Gto", "max_radial": 5}}}',
     "unknown variant `Cosine`"),
])
def test_json_errors(params, fragment):
    handle = C.lib().featomic_calculator(b"soap_power_spectrum", params.encode())
    assert not handle
    assert fragment in C.lib().featomic_last_error().decode()


def test_invalid_parameters():
    h = hypers(5.0, 5, 4)
    h["cutoff"]["smoothing"]["width"] = -1.0
    with pytest.raises(rb.FeatomicError, match="expected positive width"):
        rb.SoapPowerSpectrum(**h)
    h = hypers(5.0, 5, 4)
    h["density"] = {"type": "DiracDelta"}
    with pytest.raises(rb.FeatomicError, match="not supported in SOAP"):
        rb.SoapPowerSpectrum(**h)
    h = hypers(5.0, 5, 4)
    h["basis"]["spline_accuracy"] = -1e-3
    with pytest.raises(rb.FeatomicError, match="invalid accuracy"):
        rb.SoapPowerSpectrum(**h)


def test_power_spectrum_accepts_unknown_top_level_fields():
    # PowerSpectrumParameters has no deny_unknown_fields (power_spectrum.rs:33-43)
    h = hypers(5.0, 5, 4)
    h["comment"] = "ignored"
    rb.CalculatorBase("soap_power_spectrum", h)
    with pytest.raises(rb.FeatomicError, match="unknown field `comment`"):
        rb.CalculatorBase("spherical_expansion", h)


def test_unsupported_gradient_is_rejected_before_compute():
    calc = rb.SoapPowerSpectrum(**hypers(5.0, 5, 4))
    with pytest.raises(rb.FeatomicError, match="unexpected gradient"):
        calc.compute(rb.System([1, 1], [[0, 0, 0], [1, 0, 0]]), gradients=["velocities"])


def test_zero_systems_is_a_no_op():
    calc = rb.SoapPowerSpectrum(**hypers(5.0, 5, 4))
    assert calc.compute([]) is None


def test_profiling_get_formats():
    rb.profiling_enable(True)
    rb.profiling_clear()
    assert rb.profiling_get("json") == "{}"
    with pytest.raises(rb.FeatomicError, match="invalid data format"):
        rb.profiling_get("xml")
    rb.profiling_enable(False)


def test_spline_tables_build_on_the_host():
    # the adaptive spline knots are built at construction, with no GPU
    for acc in (1e-8, 1e-10):
        rb.SoapPowerSpectrum(**hypers(6.0, 11, 8, spline_accuracy=acc))


@pytest.mark.parametrize("cutoff, nmax, lmax, acc", [
    (5.5, 7, 6, 1e-8),      # power spectrum benchmark box
    (5.0, 5, 4, 1e-8),      # simple-cubic lattice
    (6.0, 11, 8, 1e-8),     # 12 radial functions: ill-conditioned overlap (cond ~4e7)
    (5.5, 7, 8, None),      # analytic integral (golden inputs)
])
def test_radial_integral_matches_oracle(oracle, cutoff, nmax, lmax, acc):
    """The set-up math (Lanczos Gamma, 1F1, EISPACK eigensolver, adaptive
    spline knots) agrees with the oracle on the host: same knot counts, and
    radial integrals within 1e-13 of the largest value."""
    h = hypers(cutoff, nmax, lmax)
    h["basis"]["spline_accuracy"] = acc
    calc = rb.SoapPowerSpectrum(**h)
    r = np.linspace(0.0, cutoff, 97)
    values, grads, knots = calc.radial_integral(r)
    expected, expected_grads = oracle.radial_integral(h, r)
    if acc is not None:
        np.testing.assert_array_equal(knots, oracle.spline_sizes(h))
    scale = np.abs(expected).max()
    assert np.abs(values - expected).max() <= 1e-13 * scale
    assert np.abs(grads - expected_grads).max() <= 1e-13 * np.abs(expected_grads).max()
