"""Pin the CPU oracle to featomic's own reference data.

Golden arrays come from featomic/tests/data/generated (regenerated into
tests/golden by tests/golden/make_golden.py); tolerances are the ones of the
reference's tests (featomic/tests/soap-power-spectrum.rs:10-64,
featomic/tests/soap-spherical-expansion.rs, featomic/tests/spherical-harmonics.rs)
with approx::assert_relative_eq semantics."""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN
from layout import assert_relative_eq, load_input, power_spectrum_golden, spherical_expansion_golden


def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))["values"]


def known():
    with open(os.path.join(GOLDEN, "known_answers.json")) as fd:
        return json.load(fd)


def test_power_spectrum_values(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "soap-power-spectrum-values-input.json"))
    tm = oracle.compute("soap_power_spectrum", hypers, systems)
    values, _, _, _ = power_spectrum_golden(tm)
    assert_relative_eq(values, golden("soap-power-spectrum-values"), 1e-5)


def test_power_spectrum_gradients(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "soap-power-spectrum-gradients-input.json"))
    tm = oracle.compute("soap_power_spectrum", hypers, systems, gradients=("positions", "strain", "cell"))
    _, positions, strain, cell = power_spectrum_golden(tm, n_atoms=9)
    assert_relative_eq(positions, golden("soap-power-spectrum-positions-gradient"), 1e-6)
    assert_relative_eq(strain, golden("soap-power-spectrum-strain-gradient"), 1e-6)
    assert_relative_eq(cell, golden("soap-power-spectrum-cell-gradient"), 1e-6)


def test_spherical_expansion_values(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "spherical-expansion-values-input.json"))
    values, _, _, _ = spherical_expansion_golden(oracle.compute("spherical_expansion", hypers, systems))
    assert_relative_eq(values, golden("spherical-expansion-values"), 5e-5)


def test_spherical_expansion_pbc_values(oracle):
    # molecular crystal where several atom pairs are neighbours twice
    systems, hypers = load_input(os.path.join(GOLDEN, "spherical-expansion-pbc-values-input.json"))
    values, _, _, _ = spherical_expansion_golden(oracle.compute("spherical_expansion", hypers, systems))
    assert_relative_eq(values, golden("spherical-expansion-pbc-values"), 1e-6)


def test_spherical_expansion_gradients(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "spherical-expansion-gradients-input.json"))
    tm = oracle.compute("spherical_expansion", hypers, systems, gradients=("positions", "strain", "cell"))
    _, positions, strain, cell = spherical_expansion_golden(tm, n_atoms=9)
    assert_relative_eq(positions, golden("spherical-expansion-positions-gradient"), 1e-6)
    assert_relative_eq(strain, golden("spherical-expansion-strain-gradient"), 1e-6)
    assert_relative_eq(cell, golden("spherical-expansion-cell-gradient"), 1e-6)


def test_spherical_harmonics(oracle):
    with open(os.path.join(GOLDEN, "spherical-harmonics-input.json")) as fd:
        data = json.load(fd)
    expected = golden("spherical-harmonics-values")
    for i, direction in enumerate(data["directions"]):
        values = oracle.spherical_harmonics(data["max_angular"], np.array(direction))
        for l in range(data["max_angular"]):
            assert_relative_eq(values[l * l:(l + 1) ** 2], expected[i, l, :2 * l + 1], 1e-11, epsilon=1e-11)


def test_spherical_harmonics_gradient_pole_branch(oracle):
    """featomic's Y_lm gradient (spherical_harmonics.rs:285-297) replaces
    m P_l^m / sin(theta) by -delta P_l^m / (2 cos(theta)) when sin(theta) <= 0.1.
    Away from the pole the gradient is the exact derivative of Y_lm(r / |r|);
    inside the pole region it is this approximation, which the oracle and the
    CUDA kernels reproduce: finite differences of featomic's own Y_lm do not
    match its gradient there."""
    lmax = 6

    def fd_error(theta):
        d = np.array([np.sin(theta) * np.cos(0.7), np.sin(theta) * np.sin(0.7), np.cos(theta)])
        _, grad = oracle.spherical_harmonics(lmax, d, gradients=True)
        fd = np.zeros_like(grad)
        h = 1e-6
        for x in range(3):
            e = np.zeros(3)
            e[x] = h
            plus = oracle.spherical_harmonics(lmax, (d + e) / np.linalg.norm(d + e))
            minus = oracle.spherical_harmonics(lmax, (d - e) / np.linalg.norm(d - e))
            fd[x] = (plus - minus) / (2 * h)
        return np.max(np.abs(fd - grad)) / np.max(np.abs(grad))

    for theta in (1.2, 0.5, 0.2, 0.11):
        assert fd_error(theta) < 1e-8, theta
    for theta in (0.09, 0.05):
        assert fd_error(theta) > 1e-3, theta


def test_hyp1f1_table(oracle):
    table = known()["hyp1f1"]
    for entry in table["table"]:
        a = 0.5 * (entry["n"] + entry["l"] + 3)
        b = entry["l"] + 1.5
        for z, expected in zip(table["z"], entry["values"]):
            assert_relative_eq(oracle.hyp1f1(a, b, z), expected, 1e-13)


def test_gamma_values(oracle):
    data = known()["gamma"]
    for x, expected in data["gamma"]:
        assert_relative_eq(oracle.gamma(x), expected, 1e-13)
    for x, expected in data["ln_gamma"]:
        # ln_gamma(1.0) == 0.0 is checked with epsilon=1e-15 (gamma.rs:370)
        assert_relative_eq(oracle.ln_gamma(x), expected, 1e-13, epsilon=1e-15)


def test_cutoff_values(oracle):
    data = known()["cutoff"]
    hypers = {"cutoff": {"radius": data["radius"], "smoothing": {"type": "ShiftedCosine", "width": data["width"]}},
              "density": {"type": "Gaussian", "width": 0.3},
              "basis": {"type": "TensorProduct", "max_angular": 0, "radial": {"type": "Gto", "max_radial": 0}}}
    for (r, v), (_, g) in zip(data["smoothing"], data["gradient"]):
        value, gradient = oracle.cutoff_function(hypers, r)
        assert value == v
        assert gradient == g


def test_neighbors_ase(oracle):
    data = known()["neighbors_non_periodic"]
    nl = oracle.neighbors(np.array(data["positions"]), np.zeros(9), data["cutoff"])
    assert len(nl["first"]) == len(data["pairs"])
    for k, (i, j, d) in enumerate(data["pairs"]):
        assert nl["first"][k] == i and nl["second"][k] == j
        assert abs(nl["distance"][k] - d) <= 4 * np.spacing(d)


def test_neighbors_fcc(oracle):
    # featomic/src/systems/neighbors.rs:447-474
    cell = np.array([[0.0, 1.5, 1.5], [1.5, 0.0, 1.5], [1.5, 1.5, 0.0]])
    nl = oracle.neighbors(np.zeros((1, 3)), cell, 3.0)
    assert len(nl["first"]) == 6
    assert np.all(nl["first"] == 0) and np.all(nl["second"] == 0)
    expected = {(-1, 0, 1), (-1, 1, 0), (0, -1, 1), (0, 0, 1), (0, 1, 0), (1, 0, 0)}
    assert {tuple(s) for s in nl["shift"]} == expected
    np.testing.assert_allclose(nl["distance"], 2.1213203435596424, rtol=1e-15)


def test_neighbors_small_cell_large_cutoff(oracle):
    # featomic/src/systems/neighbors.rs:507-527
    nl = oracle.neighbors(np.zeros((1, 3)), np.eye(3) * 0.5, 0.6)
    assert {tuple(s) for s in nl["shift"]} == {(0, 0, 1), (0, 1, 0), (1, 0, 0)}
    np.testing.assert_allclose(nl["distance"], 0.5, rtol=1e-15)


def test_neighbors_non_cubic(oracle):
    # featomic/src/systems/neighbors.rs:529-560
    cell = np.array([[4.26, -2.45951215, 0.0], [2.13, 1.22975607, 0.0], [0.0, 0.0, 50.0]])
    positions = np.array([[1.42, 0.0, 0.0], [2.84, 0.0, 0.0], [3.55, -1.22975607, 0.0], [4.97, -1.22975607, 0.0]])
    nl = oracle.neighbors(positions, cell, 6.4)
    assert len(nl["first"]) == 90
    found = {(int(a), int(b), tuple(s)) for a, b, s in zip(nl["first"], nl["second"], nl["shift"])}
    for missing in [(0, 3, (-2, 0, 0)), (0, 3, (-2, 1, 0)), (0, 3, (-2, 2, 0))]:
        assert missing in found


def test_gto_overlap_orthonormal(oracle):
    # featomic/src/calculators/shared/basis/radial/gto.rs:84-105 (S^-1/2 S S^-1/2 = 1
    # up to the normalisation): the orthonormalised basis integrates to identity
    M = oracle.gto_orthonormalization(8, 6.3)
    assert np.all(np.isfinite(M))
