"""Tabulated radial basis (featomic/src/calculators/shared/basis/radial/
tabulated.rs, radial_integral/mod.rs:86-113): the radial integral is a
user-given Hermite spline, with a Dirac density.

A Tabulated basis built from this library's own GTO spline (every channel's
control points, values and derivatives, as an Explicit basis) must give the
GTO results again: Hermite interpolation of a piecewise cubic at its own knots
reproduces it.  The CPU tests check the parameter rules."""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import workloads


def tabulated_from(calc, cutoff, lmax):
    """Explicit basis of Tabulated channels holding `calc`'s GTO spline."""
    _, _, knots = calc.radial_integral(np.array([0.0]))
    by_angular = {}
    for l in range(lmax + 1):
        r = np.linspace(0.0, cutoff, int(knots[l]))
        values, grads, _ = calc.radial_integral(r)
        by_angular[str(l)] = {"type": "Tabulated", "points": [
            {"position": float(x), "values": values[k, l].tolist(), "derivatives": grads[k, l].tolist()}
            for k, x in enumerate(r)]}
    h = workloads.hypers(cutoff, 1, 1)
    h["density"] = {"type": "DiracDelta"}
    h["basis"] = {"type": "Explicit", "by_angular": by_angular}
    return h


def simple_tabulated(size=3):
    h = workloads.hypers(4.0, 1, 2)
    h["density"] = {"type": "DiracDelta"}
    h["basis"]["radial"] = {"type": "Tabulated", "points": [
        {"position": 0.0, "values": [1.0] * size, "derivatives": [0.0] * size},
        {"position": 4.0, "values": [0.0] * size, "derivatives": [0.0] * size}]}
    return h


def test_tabulated_parameters():
    rb.SoapPowerSpectrum(**simple_tabulated())
    h = simple_tabulated()
    h["density"] = {"type": "Gaussian", "width": 0.3}
    with pytest.raises(rb.FeatomicError, match="combination of basis and density"):
        rb.SoapPowerSpectrum(**h)
    h = simple_tabulated()
    h["basis"]["radial"]["points"] = h["basis"]["radial"]["points"][:1]
    with pytest.raises(rb.FeatomicError, match="at least two points"):
        rb.SoapPowerSpectrum(**h)
    h = simple_tabulated()
    h["basis"]["radial"]["points"][1]["values"] = [0.0]
    with pytest.raises(rb.FeatomicError, match="'values' in 'Tabulated' radial basis to have the same size"):
        rb.SoapPowerSpectrum(**h)
    h = simple_tabulated()
    h["basis"]["radial"]["points"][1]["derivatives"] = [0.0, 1.0]
    with pytest.raises(rb.FeatomicError, match="'derivatives' in 'Tabulated' radial basis to have the same size"):
        rb.SoapPowerSpectrum(**h)


@pytest.mark.gpu
@pytest.mark.parametrize("calculator", ["spherical_expansion", "soap_power_spectrum"])
def test_tabulated_reproduces_the_gto_spline(calculator):
    cls = {"spherical_expansion": rb.SphericalExpansion, "soap_power_spectrum": rb.SoapPowerSpectrum}[calculator]
    cutoff, nmax, lmax = 4.5, 5, 3
    gto = cls(**workloads.hypers(cutoff, nmax, lmax))
    tab = cls(**tabulated_from(gto, cutoff, lmax))
    system = rb.System.from_dict(workloads.random_box(80, density=0.1, seed=41, strain=0.01))
    grads = ["positions", "strain"]
    a = gto.compute(system, gradients=grads)
    b = tab.compute(system, gradients=grads)
    np.testing.assert_array_equal(a.keys.values, b.keys.values)
    for x, y in zip(a.blocks(), b.blocks()):
        np.testing.assert_array_equal(x.samples.values, y.samples.values)
        scale = np.abs(x.values).max()
        np.testing.assert_allclose(y.values, x.values, rtol=1e-10, atol=1e-13 * scale)
        for g in grads:
            gs = max(np.abs(x.gradient(g).values).max(), 1e-300)
            np.testing.assert_allclose(y.gradient(g).values, x.gradient(g).values, rtol=1e-10, atol=1e-13 * gs)
