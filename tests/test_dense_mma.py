"""The FP32 power-spectrum contraction and its adjoint dL/dc on the tcgen05
tensor cores (TF32 hi + lo operands, FP32 accumulation) against the same
contractions on the CUDA cores and against FP64.

* tensor cores vs CUDA cores (both FP32): values, forces and cell derivatives
  within 2e-6 of the largest magnitude (a few FP32 roundings: the summation
  orders differ);
* tensor cores vs FP64: within 1e-4 of the largest magnitude, the stated
  error bound of the FP32 forms.
Shapes cover four centres per 128-row tile (S nmax <= 32), two (<= 64), one
(<= 128), a partial last tile, nmax not a multiple of 4 (scalar stores),
lmax 10 (m padded to 32) and every number of angular channels per round.
"""
import numpy as np
import pytest

import rascaline_b200 as rb
from rascaline_b200 import _c_api as C
from rascaline_b200 import workloads

from test_dense_adjoint import batch, run_backward, run_dense

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def engine(tensor_cores, channels_per_round=0):
    C.check(C.lib().featomic_b200_set_contraction_engine(int(tensor_cores), int(channels_per_round)))


@pytest.fixture(autouse=True)
def restore_engine():
    yield
    engine(1, 1)


def relative(a, b):
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))


def forward_backward(calc, systems, precision, seed=5):
    values, state = run_dense(calc, systems, precision)
    v = values.double().cpu().numpy()
    rng = np.random.default_rng(seed)
    G = rng.normal(size=v.shape) / np.sqrt(v.shape[1] * v.shape[2])
    dtype = torch.float32 if precision == 32 else torch.float64
    gpos, _, gcell = run_backward(state, G, len(systems), dtype)
    return v, gpos, gcell


CASES = [
    # S nmax = 32: four centres per tile; 301 atoms leave a partial last tile
    ("box_301_n8_l6", lambda: [workloads.random_box(301, density=0.1, min_distance=0.9, seed=31, strain=0.02)],
     workloads.hypers(5.0, 7, 6)),
    # S nmax = 48: two centres per tile
    ("box_150_n12_l3", lambda: [workloads.random_box(150, density=0.1, min_distance=0.9, seed=32)],
     workloads.hypers(4.5, 11, 3)),
    # nmax 5: scalar epilogue stores; molecules with fewer species
    ("molecules_n5_l4", lambda: workloads.molecules(5, seed=8, max_atoms=25), workloads.hypers(4.0, 4, 4)),
    # lmax 10: m padded to 32 in the adjoint, K padding 24 in the forward
    ("box_120_n4_l10", lambda: [workloads.random_box(120, density=0.1, min_distance=0.9, seed=33)],
     workloads.hypers(4.0, 3, 10)),
]


@pytest.mark.parametrize("name,make,hypers", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("channels", [1, 2, 4])
def test_tensor_cores_match_cuda_cores_and_fp64(name, make, hypers, channels):
    systems = make()
    calc = rb.SoapPowerSpectrum(**hypers)
    engine(1, channels)
    v_tc, f_tc, c_tc = forward_backward(calc, systems, 32)
    engine(0)
    v_cc, f_cc, c_cc = forward_backward(calc, systems, 32)
    v64, f64, c64 = forward_backward(calc, systems, 64)
    assert relative(v_tc, v_cc) <= 2e-6, ("values", relative(v_tc, v_cc))
    assert relative(f_tc, f_cc) <= 2e-6, ("forces", relative(f_tc, f_cc))
    assert relative(c_tc, c_cc) <= 2e-6, ("cell", relative(c_tc, c_cc))
    assert relative(v_tc, v64) <= 1e-4
    assert relative(f_tc, f64) <= 1e-4
    assert relative(c_tc, c64) <= 1e-4


def test_engine_switch_rejects_bad_values():
    with pytest.raises(Exception):
        engine(2)
    with pytest.raises(Exception):
        engine(1, 5)


def test_tensor_cores_error_on_1000_atom_box():
    """The 1000-atom benchmark box (rc 5.5, nmax 7, lmax 6): FP32 with the
    tensor-core contractions is within 1e-6 of FP64 on values and 1e-5 on
    forces (relative to the largest magnitude)."""
    box = workloads.random_box(1000, density=0.1, min_distance=0.9, seed=2)
    calc = rb.SoapPowerSpectrum(**workloads.hypers(5.5, 7, 6))
    engine(1, 1)
    v32, f32, _ = forward_backward(calc, [box], 32)
    v64, f64, _ = forward_backward(calc, [box], 64)
    assert relative(v32, v64) <= 1e-6, relative(v32, v64)
    assert relative(f32, f64) <= 1e-5, relative(f32, f64)
    positions, types, cells, sizes = batch([box])
    assert f32.shape == (len(types), 3)
