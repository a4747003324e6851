"""LODE spherical expansion (featomic/src/calculators/lode/).

CPU (the oracle, oracle/lode.py, pinned to featomic's reference data):

* values and positions gradients of the 9-atom periodic reference system for
  potential exponents 1 to 6 (featomic/tests/data/lode-spherical-expansion.py;
  featomic/tests/lode-spherical-expansion.rs compares at max_relative 1e-6):
  |x - ref| <= 1e-6 |ref| + 1e-9 max|ref| (the arrays are stored with 10
  significant digits, and one element of exponent 4 that cancels down to
  1e-6 of the largest value differs at 2.7e-6 relative);
* the central-atom contributions against the pyLODE values of gto.rs:261-286
  (max_relative 3e-6, as there).

GPU (the library through the C ABI against the oracle): values and
gradients on the reference system for exponents 0 to 9 and on a triclinic
box with three species, analytic radial integral, within
|x - ref| <= 1e-10 |ref| + 1e-12 max|ref|; the default splined integral
within 1e-6 of the largest value; the reference arrays themselves; the
device entry point equal to the host one; featomic's error messages.
"""
import json
import os

import numpy as np
import pytest

from oracle import lode as oracle_lode
from layout import load_input, spherical_expansion_golden

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _golden(p, what):
    return np.load(f"{GOLDEN}/lode-exponent-{p}-{what}.npz")["values"]


def _close(actual, expected, rel, scale_rel, what):
    actual, expected = np.asarray(actual), np.asarray(expected)
    assert actual.shape == expected.shape, (what, actual.shape, expected.shape)
    bound = rel * np.abs(expected) + scale_rel * np.max(np.abs(expected))
    diff = np.abs(actual - expected)
    assert np.all(diff <= bound), (what, float(np.max(diff / np.maximum(bound, 1e-300))))


@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6])
def test_oracle_against_featomic_reference_data(p):
    systems, hypers = load_input(f"{GOLDEN}/lode-exponent-{p}-values-input.json")
    values, _, _, _ = spherical_expansion_golden(oracle_lode.compute(hypers, systems))
    _close(values, _golden(p, "values"), 1e-6, 1e-9, f"values, exponent {p}")
    systems, hypers = load_input(f"{GOLDEN}/lode-exponent-{p}-gradients-input.json")
    tm = oracle_lode.compute(hypers, systems, ["positions"])
    _, positions, _, _ = spherical_expansion_golden(tm, n_atoms=len(systems[0]["types"]))
    _close(positions, _golden(p, "positions-gradient"), 1e-6, 1e-9, f"positions gradients, exponent {p}")


def test_oracle_central_atom_contribution():
    with open(f"{GOLDEN}/known_answers.json") as fd:
        known = json.load(fd)["lode_center"]
    for p, expected in zip(known["exponents"], known["values"]):
        h = {"smearing": known["smearing"], "exponent": p, "nmax": known["max_radial"] + 1,
             "radius": known["radius"]}
        c = oracle_lode.center_contribution(h)
        assert np.allclose(c, expected, rtol=3e-6, atol=0), (p, c, expected)


# ---- the library on the GPU ---------------------------------------------------

def _hypers(p, max_angular=4, max_radial=3, splined=False, smearing=0.3, radius=2.5, **extra):
    basis = {"type": "TensorProduct", "max_angular": max_angular,
             "radial": {"type": "Gto", "max_radial": max_radial, "radius": radius}}
    if not splined:
        basis["spline_accuracy"] = None
    h = {"density": {"type": "SmearedPowerLaw", "smearing": smearing, "exponent": p}, "basis": basis}
    h.update(extra)
    return h


def _triclinic_box(seed=5):
    rng = np.random.default_rng(seed)
    cell = np.array([[7.0, 0.0, 0.0], [1.2, 6.5, 0.0], [-0.8, 0.9, 6.8]])
    positions = rng.uniform(0.0, 1.0, (14, 3)) @ cell
    types = rng.choice([1, 6, 8], size=14)
    return {"types": types.astype(np.int32), "positions": positions, "cell": cell}


def _ours(hypers, systems, gradients=()):
    import rascaline_b200 as rb
    calc = rb.LodeSphericalExpansion(**hypers)
    return calc.compute([rb.System.from_dict(s) for s in systems], gradients=list(gradients)).to_dict(gradients)


def _compare(ours, ref, gradients, rel=1e-10, scale=1e-12):
    np.testing.assert_array_equal(ours["keys"], ref["keys"])
    for b, r in zip(ours["blocks"], ref["blocks"]):
        np.testing.assert_array_equal(b["samples"], r["samples"])
        np.testing.assert_array_equal(b["properties"], r["properties"])
    values = np.concatenate([b["values"].reshape(-1) for b in ours["blocks"]])
    expected = np.concatenate([b["values"].reshape(-1) for b in ref["blocks"]])
    _close(values, expected, rel, scale, "values")
    for name in gradients:
        for b, r in zip(ours["blocks"], ref["blocks"]):
            np.testing.assert_array_equal(b["gradients"][name]["samples"], r["gradients"][name]["samples"])
        g = np.concatenate([b["gradients"][name]["values"].reshape(-1) for b in ours["blocks"]])
        e = np.concatenate([b["gradients"][name]["values"].reshape(-1) for b in ref["blocks"]])
        _close(g, e, rel, scale, f"{name} gradients")


@pytest.mark.gpu
@pytest.mark.parametrize("p", list(range(10)))
def test_lode_matches_the_oracle(p):
    systems, _ = load_input(f"{GOLDEN}/lode-exponent-1-gradients-input.json")
    hypers = _hypers(p, max_angular=3, max_radial=2)
    _compare(_ours(hypers, systems, ["positions"]), oracle_lode.compute(hypers, systems, ["positions"]),
             ["positions"])


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 4])
def test_lode_triclinic_box_three_species(p):
    systems = [_triclinic_box(), _triclinic_box(seed=6)]
    hypers = _hypers(p, max_angular=5, max_radial=4, smearing=0.8, radius=3.0, k_cutoff=5.0)
    hypers["density"]["center_atom_weight"] = 0.5
    _compare(_ours(hypers, systems, ["positions"]), oracle_lode.compute(hypers, systems, ["positions"]),
             ["positions"])


@pytest.mark.gpu
def test_lode_splined_radial_integral():
    systems, _ = load_input(f"{GOLDEN}/lode-exponent-1-values-input.json")
    _compare(_ours(_hypers(2, splined=True), systems), oracle_lode.compute(_hypers(2), systems), [],
             rel=0.0, scale=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("p", [1, 2, 3, 4, 5, 6])
def test_lode_against_featomic_reference_data(p):
    systems, hypers = load_input(f"{GOLDEN}/lode-exponent-{p}-values-input.json")
    values, _, _, _ = spherical_expansion_golden(_ours(hypers, systems))
    _close(values, _golden(p, "values"), 1e-6, 1e-9, f"values, exponent {p}")
    systems, hypers = load_input(f"{GOLDEN}/lode-exponent-{p}-gradients-input.json")
    tm = _ours(hypers, systems, ["positions"])
    _, positions, _, _ = spherical_expansion_golden(tm, n_atoms=len(systems[0]["types"]))
    _close(positions, _golden(p, "positions-gradient"), 1e-6, 1e-9, f"positions gradients, exponent {p}")


@pytest.mark.gpu
def test_lode_device_entry_point():
    import torch
    import rascaline_b200 as rb
    box = _triclinic_box()
    hypers = _hypers(3, max_angular=3, max_radial=3, smearing=0.8, radius=3.0)
    calc = rb.LodeSphericalExpansion(**hypers)
    host = calc.compute(rb.System.from_dict(box), gradients=["positions"]).to_dict(["positions"])
    pos = torch.tensor(box["positions"], device="cuda")
    dev = calc.compute_device(pos, box["types"], box["cell"].reshape(1, 9), [len(box["types"])],
                              gradients=["positions"]).to_dict(["positions"])
    for a, b in zip(host["blocks"], dev["blocks"]):
        np.testing.assert_array_equal(a["values"], b["values"])
        np.testing.assert_array_equal(a["gradients"]["positions"]["values"], b["gradients"]["positions"]["values"])


@pytest.mark.gpu
def test_lode_errors():
    import rascaline_b200 as rb
    box = _triclinic_box()
    calc = rb.LodeSphericalExpansion(**_hypers(1))
    with pytest.raises(rb.FeatomicError, match="does not support gradients with respect to strain"):
        calc.compute(rb.System.from_dict(box), gradients=["strain"])
    infinite = dict(box, cell=np.zeros((3, 3)))
    with pytest.raises(rb.FeatomicError, match="LODE can only be used with periodic systems"):
        calc.compute(rb.System.from_dict(infinite))
    with pytest.raises(rb.FeatomicError, match="LODE is only implemented for potential_exponent < 10"):
        rb.LodeSphericalExpansion(**_hypers(10))
    with pytest.raises(rb.FeatomicError, match="LODE does not support custom density scaling"):
        h = _hypers(1)
        h["density"]["scaling"] = {"type": "Willatt2018", "scale": 1.0, "rate": 1.0, "exponent": 2.0}
        rb.LodeSphericalExpansion(**h)
