"""soap_radial_spectrum: featomic's SoapRadialSpectrum
(featomic/src/calculators/soap/radial_spectrum.rs), the l = 0 spherical
expansion with keys (center_type, neighbor_type), properties n and no
components.

CPU tests: registry name, parameters, serde's rules on RadialSpectrumBasis.
GPU tests (through the C ABI): every value and gradient against the oracle at
the 1e-10 relative bound of the other parity tests, the metadata layout, and
finite differences with the recipe of radial_spectrum.rs:365-410
(featomic/src/calculators/tests_utils.rs)."""
import json

import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads


def rs_hypers(cutoff, max_radial, width=0.3, smoothing=0.5, spline_accuracy=None, **extra):
    basis = {"radial": {"type": "Gto", "max_radial": max_radial}}
    if spline_accuracy is not None:
        basis["spline_accuracy"] = spline_accuracy
    basis.update(extra)
    return {
        "cutoff": {"radius": cutoff, "smoothing": {"type": "ShiftedCosine", "width": smoothing}},
        "density": {"type": "Gaussian", "width": width},
        "basis": basis,
    }


def test_radial_spectrum_metadata():
    calc = rb.SoapRadialSpectrum(**rs_hypers(3.5, 5))
    assert calc.name == "radial spectrum"
    assert calc.cutoffs == [3.5]
    assert json.loads(calc.parameters) == rs_hypers(3.5, 5)


def test_radial_spectrum_basis_rules():
    # RadialSpectrumBasis has deny_unknown_fields and no `type` tag
    with pytest.raises(rb.FeatomicError, match="unknown field `max_angular`"):
        rb.SoapRadialSpectrum(**rs_hypers(3.5, 5, max_angular=2))
    with pytest.raises(rb.FeatomicError, match="unknown field `type`"):
        rb.SoapRadialSpectrum(**rs_hypers(3.5, 5, type="TensorProduct"))
    # the top-level struct accepts unknown fields, like the power spectrum's
    h = rs_hypers(3.5, 5)
    h["comment"] = "ignored"
    rb.CalculatorBase("soap_radial_spectrum", h)
    h = rs_hypers(3.5, 5, spline_accuracy=-1.0)
    with pytest.raises(rb.FeatomicError, match="invalid accuracy"):
        rb.SoapRadialSpectrum(**h)


def test_oracle_radial_spectrum_is_the_l0_expansion(oracle):
    system = workloads.random_box(40, density=0.1, seed=4)
    rs = oracle.compute("soap_radial_spectrum", rs_hypers(4.0, 4), [system], ("positions",))
    se = oracle.compute("spherical_expansion", workloads.hypers(4.0, 4, 0), [system], ("positions",))
    np.testing.assert_array_equal(rs["keys"], se["keys"][:, 2:])
    for a, b in zip(rs["blocks"], se["blocks"]):
        np.testing.assert_array_equal(a["values"], b["values"][:, 0, :])
        np.testing.assert_array_equal(a["gradients"]["positions"]["values"],
                                      b["gradients"]["positions"]["values"][:, :, 0, :])


# ---------------------------------------------------------------------------
# GPU
# ---------------------------------------------------------------------------
def _cases():
    return {
        "random_box_300": ([workloads.random_box(300, density=0.1, seed=9)], rs_hypers(5.0, 7)),
        "strained_box": ([workloads.random_box(200, strain=0.02, seed=7)], rs_hypers(4.5, 5, spline_accuracy=1e-6)),
        "molecules": (workloads.molecules(4, seed=5), rs_hypers(5.0, 7)),
        "sc_lattice": ([workloads.sc_lattice()], rs_hypers(5.0, 5)),
    }


@pytest.mark.gpu
@pytest.mark.parametrize("case", sorted(_cases()))
def test_radial_spectrum_matches_oracle(oracle, case):
    from test_gpu_parity import check_against_oracle
    systems, hypers = _cases()[case]
    periodic = all(np.abs(s["cell"]).sum() > 0 for s in systems)
    grads = ("positions", "strain", "cell") if periodic else ("positions",)
    product, expected = check_against_oracle(oracle, "soap_radial_spectrum", hypers, systems, grads)
    n = hypers["basis"]["radial"]["max_radial"] + 1
    assert product["keys"].shape[1] == 2
    for block in product["blocks"]:
        assert block["values"].shape[1:] == (n,)
        assert block["gradients"]["positions"]["values"].shape[1:] == (3, n)
        if periodic:
            assert block["gradients"]["strain"]["values"].shape[1:] == (3, 3, n)


@pytest.mark.gpu
def test_radial_spectrum_analytic_radial_integral(oracle):
    from test_gpu_parity import check_against_oracle
    h = rs_hypers(4.0, 5)
    h["basis"]["spline_accuracy"] = None
    check_against_oracle(oracle, "soap_radial_spectrum", h, [workloads.random_box(120, seed=8)], ("positions",))


@pytest.mark.gpu
def test_radial_spectrum_block_labels():
    calc = rb.SoapRadialSpectrum(**rs_hypers(3.5, 5))
    system = workloads.random_box(60, density=0.1, species=(1, 8), seed=3)
    tm = calc.compute(rb.System.from_dict(system), gradients=["positions", "cell"])
    assert tm.keys.names == ["center_type", "neighbor_type"]
    assert sorted(map(tuple, tm.keys.values)) == [(1, 1), (1, 8), (8, 1), (8, 8)]
    block = tm.block_by_id(0)
    assert block.samples.names == ["system", "atom"]
    assert block.components == []
    assert block.properties.names == ["n"]
    assert block.gradient("positions").components[0].names == ["xyz"]
    assert [c.names for c in block.gradient("cell").components] == [["xyz"], ["abc"]]


@pytest.mark.gpu
def test_radial_spectrum_finite_differences_positions():
    # displacement 1e-5, max relative 1e-4 (radial_spectrum.rs:365-378)
    calc = rb.SoapRadialSpectrum(**rs_hypers(3.5, 5))
    system = workloads.random_box(24, density=0.08, species=(1, 8), seed=12)
    h = 1e-5

    def dense(positions):
        s = dict(system, positions=positions)
        tm = calc.compute(rb.System.from_dict(s))
        return {tuple(k): b.values.copy() for k, b in zip(tm.keys.values, tm.blocks())}

    tm = calc.compute(rb.System.from_dict(system), gradients=["positions"])
    checked = 0
    for k, block in zip(tm.keys.values, tm.blocks()):
        g = block.gradient("positions")
        samples = block.samples.values
        for row, (sample, _, atom) in enumerate(g.samples.values):
            for x in range(3):
                plus, minus = system["positions"].copy(), system["positions"].copy()
                plus[atom, x] += h
                minus[atom, x] -= h
                fd = (dense(plus)[tuple(k)][sample] - dense(minus)[tuple(k)][sample]) / (2 * h)
                an = g.values[row, x]
                assert np.allclose(an, fd, rtol=1e-4, atol=1e-9), (tuple(k), samples[sample], atom, x)
                checked += 1
            if checked > 60:
                return
