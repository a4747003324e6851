"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
featomic's golden data.

Tolerances:
* neighbour lists: bit-exact (indices, shifts, distances, vectors);
* FP64 values and gradients vs the oracle: |gpu - cpu| <= 1e-10 |cpu| +
  1e-12 max|cpu| (relative 1e-10, with an absolute floor at 1e-12 of the
  array's largest magnitude for entries that cancel to ~0);
* vs the golden arrays: the reference tests' own tolerances.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN
from layout import assert_relative_eq, load_input, power_spectrum_golden, spherical_expansion_golden

import rascaline_b200 as rb
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu

RTOL = 1e-10
ATOL_FRACTION = 1e-12


def assert_close(actual, expected, what):
    actual = np.asarray(actual)
    expected = np.asarray(expected)
    assert actual.shape == expected.shape, (what, actual.shape, expected.shape)
    if expected.size == 0:
        return
    scale = np.max(np.abs(expected))
    bound = RTOL * np.abs(expected) + ATOL_FRACTION * scale
    diff = np.abs(actual - expected)
    bad = diff > bound
    if bad.any():
        i = np.unravel_index(np.argmax(diff - bound), diff.shape)
        raise AssertionError(f"{what}: {bad.sum()}/{bad.size} elements differ; worst at {i}: "
                             f"{actual[i]!r} vs {expected[i]!r} (scale {scale:.3e})")


def compare_tensormaps(product, oracle_tm, gradients):
    np.testing.assert_array_equal(product["keys"], oracle_tm["keys"])
    assert len(product["blocks"]) == len(oracle_tm["blocks"])
    for k, (p, o) in enumerate(zip(product["blocks"], oracle_tm["blocks"])):
        key = tuple(oracle_tm["keys"][k])
        np.testing.assert_array_equal(p["samples"], o["samples"], err_msg=f"samples of {key}")
        np.testing.assert_array_equal(p["properties"], o["properties"], err_msg=f"properties of {key}")
        assert_close(p["values"], o["values"], f"values of {key}")
        for g in gradients:
            np.testing.assert_array_equal(p["gradients"][g]["samples"], o["gradients"][g]["samples"],
                                          err_msg=f"{g} gradient samples of {key}")
            assert_close(p["gradients"][g]["values"], o["gradients"][g]["values"], f"{g} gradients of {key}")


def run_product(calculator, hypers, systems, gradients=(), use_native_system=True):
    cls = {"spherical_expansion": rb.SphericalExpansion, "soap_power_spectrum": rb.SoapPowerSpectrum,
           "soap_radial_spectrum": rb.SoapRadialSpectrum,
           "spherical_expansion_by_pair": rb.SphericalExpansionByPair}[calculator]
    calc = cls(**hypers)
    tm = calc.compute([rb.System.from_dict(s) for s in systems], gradients=list(gradients),
                      use_native_system=use_native_system)
    return tm.to_dict(gradients)


def check_against_oracle(oracle, calculator, hypers, systems, gradients=(), threads=8, **kw):
    product = run_product(calculator, hypers, systems, gradients, **kw)
    expected = oracle.compute(calculator, hypers, systems, gradients=gradients, threads=threads)
    compare_tensormaps(product, expected, gradients)
    return product, expected


# ---------------------------------------------------------------------------
# kernel (a): neighbour list, bit-exact
# ---------------------------------------------------------------------------
def nl_cases():
    rng = np.random.default_rng(11)
    tri = np.array([[7.0, 0.0, 0.0], [2.1, 6.5, 0.0], [-1.3, 1.7, 8.2]])
    frac = rng.uniform(-0.2, 1.2, size=(60, 3))  # some atoms outside the cell
    box = workloads.random_box(1000)
    mols = workloads.molecules(3)
    return {
        "sc_lattice": (workloads.sc_lattice()["positions"], np.eye(3) * 12.0, 5.0),
        "random_box_1000": (box["positions"], box["cell"], 5.5),
        "strained_box": (workloads.random_box(800, strain=0.02, seed=7)["positions"],
                         workloads.random_box(800, strain=0.02, seed=7)["cell"], 5.0),
        "triclinic_outside": (frac @ tri, tri, 4.5),
        "small_cell_large_cutoff": (np.zeros((1, 3)), np.eye(3) * 0.5, 0.6),
        "fcc": (np.zeros((1, 3)), np.array([[0.0, 1.5, 1.5], [1.5, 0.0, 1.5], [1.5, 1.5, 0.0]]), 3.0),
        "multi_image": (rng.uniform(0, 3.0, size=(5, 3)), np.eye(3) * 3.0, 4.0),
        "molecule": (mols[0]["positions"], np.zeros((3, 3)), 5.0),
        "non_periodic_small_cutoff": (rng.uniform(-2, 2, size=(30, 3)), np.zeros((3, 3)), 0.7),
        "non_cubic": (np.array([[1.42, 0.0, 0.0], [2.84, 0.0, 0.0], [3.55, -1.22975607, 0.0], [4.97, -1.22975607, 0.0]]),
                      np.array([[4.26, -2.45951215, 0.0], [2.13, 1.22975607, 0.0], [0.0, 0.0, 50.0]]), 6.4),
    }


@pytest.mark.parametrize("case", sorted(nl_cases()))
def test_neighbor_list_bitexact(oracle, case):
    positions, cell, cutoff = nl_cases()[case]
    gpu = rb.neighbor_list(positions, cell, cutoff)
    cpu = oracle.neighbors(positions, cell, cutoff)
    assert len(gpu["first"]) == len(cpu["first"]) > 0 or case == "non_periodic_small_cutoff"
    for name in ("first", "second", "shift"):
        np.testing.assert_array_equal(gpu[name], cpu[name], err_msg=name)
    # bit-identical floating point values
    np.testing.assert_array_equal(gpu["distance"].view(np.int64), cpu["distance"].view(np.int64))
    np.testing.assert_array_equal(gpu["vector"].view(np.int64), cpu["vector"].view(np.int64))


def test_neighbor_list_known_answers(oracle):
    import json
    with open(os.path.join(GOLDEN, "known_answers.json")) as fd:
        data = json.load(fd)["neighbors_non_periodic"]
    nl = rb.neighbor_list(np.array(data["positions"]), np.zeros(9), data["cutoff"])
    assert len(nl["first"]) == len(data["pairs"])
    for k, (i, j, d) in enumerate(data["pairs"]):
        assert nl["first"][k] == i and nl["second"][k] == j
        assert abs(nl["distance"][k] - d) <= 4 * np.spacing(d)


# ---------------------------------------------------------------------------
# featomic's golden data (analytic GTO, spline_accuracy = null)
# ---------------------------------------------------------------------------
def golden(name):
    return np.load(os.path.join(GOLDEN, name + ".npz"))["values"]


def test_golden_power_spectrum_values(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "soap-power-spectrum-values-input.json"))
    product, _ = check_against_oracle(oracle, "soap_power_spectrum", hypers, systems)
    values, _, _, _ = power_spectrum_golden(product)
    assert_relative_eq(values, golden("soap-power-spectrum-values"), 1e-5)


def test_golden_power_spectrum_gradients(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "soap-power-spectrum-gradients-input.json"))
    grads = ("positions", "strain", "cell")
    product, _ = check_against_oracle(oracle, "soap_power_spectrum", hypers, systems, grads)
    _, positions, strain, cell = power_spectrum_golden(product, n_atoms=9)
    assert_relative_eq(positions, golden("soap-power-spectrum-positions-gradient"), 1e-6)
    assert_relative_eq(strain, golden("soap-power-spectrum-strain-gradient"), 1e-6)
    assert_relative_eq(cell, golden("soap-power-spectrum-cell-gradient"), 1e-6)


def test_golden_spherical_expansion_values(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "spherical-expansion-values-input.json"))
    product, _ = check_against_oracle(oracle, "spherical_expansion", hypers, systems)
    values, _, _, _ = spherical_expansion_golden(product)
    assert_relative_eq(values, golden("spherical-expansion-values"), 5e-5)


def test_golden_spherical_expansion_pbc(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "spherical-expansion-pbc-values-input.json"))
    product, _ = check_against_oracle(oracle, "spherical_expansion", hypers, systems)
    values, _, _, _ = spherical_expansion_golden(product)
    assert_relative_eq(values, golden("spherical-expansion-pbc-values"), 1e-6)


def test_golden_spherical_expansion_gradients(oracle):
    systems, hypers = load_input(os.path.join(GOLDEN, "spherical-expansion-gradients-input.json"))
    grads = ("positions", "strain", "cell")
    product, _ = check_against_oracle(oracle, "spherical_expansion", hypers, systems, grads)
    _, positions, strain, cell = spherical_expansion_golden(product, n_atoms=9)
    assert_relative_eq(positions, golden("spherical-expansion-positions-gradient"), 1e-6)
    assert_relative_eq(strain, golden("spherical-expansion-strain-gradient"), 1e-6)
    assert_relative_eq(cell, golden("spherical-expansion-cell-gradient"), 1e-6)


# ---------------------------------------------------------------------------
# benchmark configurations (splined radial integral, the default)
# ---------------------------------------------------------------------------
def test_sc_lattice_spherical_expansion(oracle):
    cfg = workloads.CONFIGS["c1"]
    check_against_oracle(oracle, "spherical_expansion", cfg["hypers"], cfg["system"]())


def test_random_box_power_spectrum_with_gradients(oracle):
    cfg = workloads.CONFIGS["c2"]
    check_against_oracle(oracle, "soap_power_spectrum", cfg["hypers"], cfg["system"](),
                         ("positions", "strain", "cell"))


def test_spherical_expansion_gradients_random_box(oracle):
    systems = [workloads.random_box(300, seed=4)]
    check_against_oracle(oracle, "spherical_expansion", workloads.hypers(5.0, 5, 5), systems,
                         ("positions", "strain", "cell"))


def test_molecules_batch(oracle):
    systems = workloads.molecules(24)
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(5.0, 7, 6), systems, ("positions",))


def test_mixed_systems(oracle):
    systems = [workloads.sc_lattice()] + workloads.molecules(3) + [workloads.random_box(200, seed=9)]
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(4.5, 4, 3), systems,
                         ("positions", "strain"))


def test_power_spectrum_many_radial_functions(oracle):
    # more than 8 radial functions: the positions rows take the per-warp kernel
    systems = [workloads.random_box(80, seed=21)]
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(4.0, 9, 2), systems, ("positions", "strain"))


def test_dense_neighbourhoods(oracle):
    # 314 to 329 neighbours per centre within 8.5 A of the 216-atom lattice: more
    # than the 256 directions the warp-per-centre neighbourhood tables hold,
    # so these centres take the serial merge
    systems = [workloads.sc_lattice(seed=1)]
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(8.5, 3, 2), systems, ("positions",))


def test_many_species(oracle):
    # more than 10 atomic types: the positions rows take the per-warp kernel,
    # the strain rows ps_strain_cell_kernel and the values ps_values_kernel
    species = (1, 3, 5, 6, 7, 8, 9, 11, 12, 14, 15)
    systems = [workloads.random_box(70, density=0.12, species=species, seed=23)]
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(4.0, 3, 2), systems, ("positions", "strain"))


def test_strain_and_cell_without_positions(oracle):
    systems = [workloads.random_box(90, seed=22)]
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(4.5, 7, 5), systems, ("strain", "cell"))
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(4.0, 5, 3), systems, ("cell",))


def test_user_neighbor_list(oracle):
    # use_native_system = False: pairs come from the caller (here, the oracle's list)
    systems = [workloads.random_box(250, seed=12)]
    hypers = workloads.hypers(5.0, 5, 4)
    for s in systems:
        s["pairs"] = oracle.neighbors(s["positions"], s["cell"], 5.0)
    product = run_product("soap_power_spectrum", hypers, systems, ("positions",), use_native_system=False)
    for s in systems:
        del s["pairs"]
    expected = oracle.compute("soap_power_spectrum", hypers, systems, gradients=("positions",), threads=8)
    compare_tensormaps(product, expected, ("positions",))


def test_analytic_radial_integral(oracle):
    systems = [workloads.random_box(120, seed=13)]
    hypers = workloads.hypers(4.0, 4, 3)
    hypers["basis"]["spline_accuracy"] = None
    check_against_oracle(oracle, "soap_power_spectrum", hypers, systems, ("positions", "strain"))


def test_step_smoothing_and_radial_scaling(oracle):
    systems = [workloads.random_box(150, seed=14)]
    hypers = workloads.hypers(4.5, 4, 4)
    hypers["cutoff"]["smoothing"] = {"type": "Step"}
    hypers["density"]["scaling"] = {"type": "Willatt2018", "scale": 2.0, "rate": 1.5, "exponent": 4}
    hypers["density"]["center_atom_weight"] = 0.5
    check_against_oracle(oracle, "soap_power_spectrum", hypers, systems, ("positions", "cell"))


def test_isolated_atoms_and_negative_types(oracle):
    # featomic's test systems use atom type -42 (featomic/src/systems/test_utils.rs)
    systems = [
        {"types": np.array([-42, 1, 1], dtype=np.int32),
         "positions": np.array([[0.0, 0.0, 0.0], [0.0, 0.0, 0.9], [8.0, 8.0, 8.0]]),
         "cell": np.zeros((3, 3))},
        {"types": np.array([6], dtype=np.int32), "positions": np.zeros((1, 3)), "cell": np.zeros((3, 3))},
    ]
    check_against_oracle(oracle, "soap_power_spectrum", workloads.hypers(3.0, 3, 3), systems, ("positions",))
    check_against_oracle(oracle, "spherical_expansion", workloads.hypers(3.0, 3, 3), systems, ("positions",))


def test_device_output_matches_host_output():
    import torch
    system = workloads.random_box(300, seed=15)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 5, 4))
    host = calc.compute(rb.System.from_dict(system), gradients=["positions"]).to_dict(("positions",))
    positions = torch.tensor(system["positions"], device="cuda")
    dev = calc.compute_device(positions, system["types"], system["cell"].reshape(1, 9), [len(system["types"])],
                              gradients=["positions"])
    torch.cuda.synchronize()
    dev = dev.to_dict(("positions",))
    for h, d in zip(host["blocks"], dev["blocks"]):
        np.testing.assert_array_equal(h["values"], d["values"])
        np.testing.assert_array_equal(h["gradients"]["positions"]["values"], d["gradients"]["positions"]["values"])


def test_repeated_calls_are_deterministic():
    system = workloads.random_box(400, seed=16)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.0, 5, 4))
    a = calc.compute(rb.System.from_dict(system), gradients=["positions", "strain"]).to_dict(("positions", "strain"))
    b = calc.compute(rb.System.from_dict(system), gradients=["positions", "strain"]).to_dict(("positions", "strain"))
    for x, y in zip(a["blocks"], b["blocks"]):
        np.testing.assert_array_equal(x["values"], y["values"])
        np.testing.assert_array_equal(x["gradients"]["strain"]["values"], y["gradients"]["strain"]["values"])
