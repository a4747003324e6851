"""The fused spherical-expansion kernel (cutoff, Y_lm and R_nl of every pair
built in shared memory inside the expansion kernel) against the two-kernel
path (per-pair records written to device memory, then read back).  Both
evaluate featomic's expressions in the same order, so every value and every
gradient must be bit-identical: spherical expansion and power spectrum, with
positions, strain and cell gradients, on periodic boxes with several species,
periodic self-images (a small cell) and max_angular up to 8; hypers the fused
kernel does not take (max_angular 9, analytic radial integrals) fall back to
the two kernels.
"""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import _c_api as C
from rascaline_b200 import workloads

pytestmark = pytest.mark.gpu


def set_fused(fused):
    C.check(C.lib().featomic_b200_set_expansion_engine(int(fused)))


@pytest.fixture(autouse=True)
def restore_engine():
    yield
    set_fused(1)


GRADIENTS = ["positions", "strain", "cell"]


def compute_both(calculator, system):
    out = []
    for fused in (1, 0):
        set_fused(fused)
        out.append(calculator.compute(rb.System.from_dict(system), gradients=GRADIENTS).to_dict(GRADIENTS))
    return out


def assert_identical(a, b):
    np.testing.assert_array_equal(a["keys"], b["keys"])
    assert len(a["blocks"]) == len(b["blocks"])
    for ba, bb in zip(a["blocks"], b["blocks"]):
        np.testing.assert_array_equal(ba["samples"], bb["samples"])
        np.testing.assert_array_equal(ba["values"], bb["values"])
        for name in GRADIENTS:
            np.testing.assert_array_equal(ba["gradients"][name]["samples"], bb["gradients"][name]["samples"])
            np.testing.assert_array_equal(ba["gradients"][name]["values"], bb["gradients"][name]["values"])


def small_cell_system():
    # a 4.2 A triclinic cell with a 4.5 A cutoff: every atom sees its own
    # periodic images
    rng = np.random.default_rng(7)
    cell = np.array([[4.2, 0.0, 0.0], [0.6, 4.4, 0.0], [0.3, -0.4, 4.6]])
    positions = rng.uniform(0.0, 1.0, (9, 3)) @ cell
    return workloads.system_dict(rng.choice([1, 6, 8], size=9), positions, cell)


CASES = {
    "random box, 4 species": (lambda: workloads.random_box(300, density=0.1, min_distance=0.9, seed=31, strain=0.02),
                              workloads.hypers(5.0, 7, 6)),
    "self images": (small_cell_system, workloads.hypers(4.5, 5, 4)),
    "max_angular 8": (lambda: workloads.random_box(120, density=0.1, min_distance=0.9, seed=32),
                      workloads.hypers(4.5, 4, 8)),
    "max_angular 0": (lambda: workloads.random_box(120, density=0.1, min_distance=0.9, seed=33),
                      workloads.hypers(4.5, 3, 0)),
    "max_angular 9 (two kernels)": (lambda: workloads.random_box(80, density=0.1, min_distance=0.9, seed=34),
                                    workloads.hypers(4.0, 3, 9)),
}


@pytest.mark.parametrize("case", list(CASES))
@pytest.mark.parametrize("calculator", ["spherical_expansion", "power_spectrum"])
def test_fused_expansion_is_bit_identical(case, calculator):
    make, hypers = CASES[case]
    system = make()
    calc = rb.SphericalExpansion(**hypers) if calculator == "spherical_expansion" else rb.SoapPowerSpectrum(**hypers)
    fused, two = compute_both(calc, system)
    assert_identical(fused, two)


def test_analytic_radial_integral_falls_back():
    hypers = workloads.hypers(4.5, 4, 3)
    hypers["basis"]["spline_accuracy"] = None
    system = workloads.random_box(60, density=0.1, min_distance=0.9, seed=35)
    fused, two = compute_both(rb.SphericalExpansion(**hypers), system)
    assert_identical(fused, two)
