"""Clebsch-Gordan products and the equivariant power spectrum
(python/featomic/featomic/clebsch_gordan/).

CPU tests: the real CG coefficients of the C ABI against the oracle's
numpy restatement of _coefficients.py:137-224 (complex coefficients from
sympy's exact CG), their orthogonality, the lambda = 0 coefficients against
SOAP's power-spectrum normalisation, the output keys of
_utils.py:_compute_output_keys and the redundant-key filter.
GPU tests: block products against the oracle (FP64 and FP32, several tasks
in one launch), the lambda = 0 blocks of the equivariant power spectrum
against the drop-in SOAP power spectrum (itself pinned to featomic's
goldens), the rotation of the lambda = 1 blocks of a molecule, and the
neighbor-types-to-properties form against the keyed form."""
import numpy as np
import pytest

import rascaline_b200 as rb
from oracle import clebsch_gordan as ocg
from rascaline_b200 import clebsch_gordan as cg
from rascaline_b200 import workloads


def test_cg_coefficients_match_oracle():
    for l1 in range(4):
        for l2 in range(4):
            for lam in range(abs(l1 - l2), l1 + l2 + 1):
                np.testing.assert_allclose(cg.cg_coefficients(l1, l2, lam), ocg.real_cg(l1, l2, lam),
                                           rtol=0, atol=1e-14, err_msg=f"{(l1, l2, lam)}")


def test_cg_coefficients_orthogonality():
    # the real transforms are unitary, so the real coefficients of one (l1, l2)
    # form an orthogonal matrix over (m1, m2) x (lambda, mu)
    for l1, l2 in ((2, 3), (6, 6), (4, 7)):
        cols = np.concatenate([cg.cg_coefficients(l1, l2, lam).reshape((2 * l1 + 1) * (2 * l2 + 1), -1)
                               for lam in range(abs(l1 - l2), l1 + l2 + 1)], axis=1)
        np.testing.assert_allclose(cols.T @ cols, np.eye(cols.shape[1]), atol=1e-12)


def test_cg_lambda0_is_power_spectrum_normalisation():
    # featomic's power spectrum divides sum_m c1 c2 by (-1)^l sqrt(2l + 1)
    # (featomic/src/calculators/soap/power_spectrum.rs:529-780)
    for l in range(9):
        np.testing.assert_allclose(cg.cg_coefficients(l, l, 0)[:, :, 0],
                                   np.eye(2 * l + 1) * (-1) ** l / np.sqrt(2 * l + 1), atol=1e-14)


def test_cg_coefficients_errors():
    with pytest.raises(rb.FeatomicError, match="can not couple"):
        cg.cg_coefficients(1, 3, 1)
    with pytest.raises(rb.FeatomicError, match="non-negative"):
        cg.cg_coefficients(-1, 1, 0)


def test_output_keys_and_filter():
    k1 = rb.Labels(["o3_lambda", "o3_sigma", "center_type", "neighbor_1_type"], [[0, 1, 1, 1], [1, 1, 1, 8]])
    k2 = rb.Labels(["o3_lambda", "o3_sigma", "center_type", "neighbor_2_type"], [[1, 1, 1, 1], [2, 1, 8, 1]])
    keys, combos = cg.ClebschGordanProduct._output_keys(k1, k2, "l_1", "l_2")
    assert keys.names == ["o3_lambda", "o3_sigma", "center_type", "neighbor_1_type", "l_1", "neighbor_2_type", "l_2"]
    # centre types must match; lambda in |l1 - l2| .. l1 + l2, sigma from the parity
    np.testing.assert_array_equal(keys.values, [
        [1, 1, 1, 1, 0, 1, 1],
        [0, 1, 1, 8, 1, 1, 1],
        [1, -1, 1, 8, 1, 1, 1],
        [2, 1, 1, 8, 1, 1, 1],
    ])
    assert combos == [(0, 0), (1, 0), (1, 0), (1, 0)]
    lk = rb.Labels(["o3_lambda", "l_1", "l_2"], [[1, 0, 1], [1, 1, 0], [2, 2, 2]])
    assert cg._filter_redundant_keys(lk) == [0, 2]


def test_only_spherical_expansions():
    ps = rb.SoapPowerSpectrum(**workloads.hypers(3.0, 2, 2))
    with pytest.raises(ValueError, match="are supported for `calculator_1`"):
        cg.EquivariantPowerSpectrum(ps)


@pytest.mark.gpu
def test_cg_product_matches_oracle():
    import torch

    rng = np.random.default_rng(7)
    cases = [(0, 0, 5, 3), (1, 2, 4, 6), (3, 3, 7, 2), (6, 6, 8, 8), (2, 5, 1, 9)]
    for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 2e-5)):
        tasks, expected = [], []
        for l1, l2, p, q in cases:
            s = int(rng.integers(1, 40))
            a = rng.standard_normal((s, 2 * l1 + 1, p))
            b = rng.standard_normal((s, 2 * l2 + 1, q))
            ta = torch.tensor(a, dtype=dtype, device="cuda")
            tb = torch.tensor(b, dtype=dtype, device="cuda")
            for lam in range(abs(l1 - l2), l1 + l2 + 1):
                out = torch.full((s, 2 * lam + 1, p * q), float("nan"), dtype=dtype, device="cuda")
                tasks.append((ta, tb, out, lam))
                expected.append(ocg.cg_tensor_product(a, b, lam))
        # an empty task is skipped
        empty = torch.zeros((0, 3, 2), dtype=dtype, device="cuda")
        tasks.append((empty, empty, torch.zeros((0, 1, 4), dtype=dtype, device="cuda"), 0))
        expected.append(np.zeros((0, 1, 4)))
        cg.cg_tensor_products(tasks)
        torch.cuda.synchronize()
        for (_, _, out, lam), ref in zip(tasks, expected):
            got = out.double().cpu().numpy()
            scale = max(1.0, np.abs(ref).max()) if ref.size else 1.0
            np.testing.assert_allclose(got, ref, rtol=0, atol=tol * scale)


def _ps_hypers():
    return workloads.hypers(4.0, 3, 3, spline_accuracy=None)


@pytest.mark.gpu
def test_lambda0_blocks_are_the_power_spectrum():
    system = workloads.random_box(48, density=0.1, species=(1, 8), seed=11)
    se = rb.SphericalExpansion(**_ps_hypers())
    eq = cg.EquivariantPowerSpectrum(se).compute([system])
    ps = rb.SoapPowerSpectrum(**_ps_hypers()).compute([system])
    names = eq.keys.names
    assert names == ["o3_lambda", "o3_sigma", "center_type", "neighbor_1_type", "neighbor_2_type"]
    blk = eq.block_by_id(0)
    assert blk.properties.names == ["l_1", "l_2", "n_1", "n_2"]
    assert blk.components[0].names == ["o3_mu"]
    checked = 0
    for key, pblk in zip(ps.keys.values, ps.blocks()):
        ct, n1, n2 = (int(v) for v in key)
        eblk = eq.block(o3_lambda=0, o3_sigma=1, center_type=ct, neighbor_1_type=n1, neighbor_2_type=n2)
        ev = eblk.values.cpu().numpy()[:, 0, :]
        props = {tuple(p): i for i, p in enumerate(eblk.properties.values)}
        rows = {tuple(s): i for i, s in enumerate(eblk.samples.values)}
        pv = np.asarray(pblk.values)
        factor = 1.0 if n1 == n2 else np.sqrt(2.0)
        for j, (l, a, b) in enumerate(pblk.properties.values):
            col = props[(l, l, a, b)]
            for i, s in enumerate(pblk.samples.values):
                np.testing.assert_allclose(factor * ev[rows[tuple(s)], col], pv[i, j], rtol=1e-10, atol=1e-14)
                checked += 1
    assert checked > 1000


def _rotation(rng):
    q, r = np.linalg.qr(rng.standard_normal((3, 3)))
    q = q * np.sign(np.diag(r))
    if np.linalg.det(q) < 0:
        q[:, 0] = -q[:, 0]
    return q


@pytest.mark.gpu
def test_lambda1_blocks_rotate_as_vectors():
    rng = np.random.default_rng(3)
    mol = workloads.molecules(1, seed=5, min_atoms=12, max_atoms=12)[0]
    R = _rotation(rng)
    rotated = dict(mol)
    rotated["positions"] = np.ascontiguousarray(mol["positions"] @ R.T)
    se = rb.SphericalExpansion(**_ps_hypers())
    calc = cg.EquivariantPowerSpectrum(se)
    a, b = calc.compute([mol]), calc.compute([rotated])
    # real l = 1 harmonics in (m = -1, 0, 1) order are proportional to (y, z, x)
    perm = np.array([1, 2, 0])
    Rm = R[np.ix_(perm, perm)]
    n = 0
    for i, key in enumerate(a.keys.values):
        if key[0] != 1:
            continue
        va = a.block_by_id(i).values.cpu().numpy()
        vb = b.block_by_id(i).values.cpu().numpy()
        np.testing.assert_allclose(np.einsum("xy,syp->sxp", Rm, va), vb, rtol=0,
                                   atol=1e-9 * max(1.0, np.abs(va).max()))
        n += 1
    assert n > 0
    # and the lambda = 0 blocks do not change
    for i, key in enumerate(a.keys.values):
        if key[0] == 0:
            va = a.block_by_id(i).values.cpu().numpy()
            np.testing.assert_allclose(b.block_by_id(i).values.cpu().numpy(), va, rtol=0,
                                       atol=1e-9 * max(1.0, np.abs(va).max()))


@pytest.mark.gpu
def test_neighbors_to_properties_matches_keyed_form():
    system = workloads.random_box(40, density=0.1, species=(1, 6, 8), seed=12)
    se = rb.SphericalExpansion(**workloads.hypers(3.5, 2, 2, spline_accuracy=None))
    calc = cg.EquivariantPowerSpectrum(se)
    keyed = calc.compute([system])
    dense = calc.compute([system], neighbors_to_properties=True)
    assert dense.keys.names == ["o3_lambda", "o3_sigma", "center_type"]
    blk = dense.block_by_id(0)
    assert blk.properties.names == ["l_1", "l_2", "neighbor_1_type", "n_1", "neighbor_2_type", "n_2"]
    checked = 0
    for i, key in enumerate(keyed.keys.values):
        lam, sigma, ct, n1, n2 = (int(v) for v in key)
        kb = keyed.block_by_id(i)
        db = dense.block(o3_lambda=lam, o3_sigma=sigma, center_type=ct)
        props = {tuple(p): j for j, p in enumerate(db.properties.values)}
        rows = {tuple(s): j for j, s in enumerate(db.samples.values)}
        kv, dv = kb.values.cpu().numpy(), db.values.cpu().numpy()
        sel = [rows[tuple(s)] for s in kb.samples.values]
        for j, (l1, l2, a, b) in enumerate(kb.properties.values):
            col = props[(l1, l2, n1, a, n2, b)]
            np.testing.assert_allclose(dv[sel, :, col], kv[:, :, j], rtol=1e-12, atol=1e-15)
            checked += 1
    assert checked > 100
    # explicit neighbour types add zero-filled properties for absent types
    calc = cg.EquivariantPowerSpectrum(se, neighbor_types=[1, 6, 7, 8])
    padded = calc.compute([system], neighbors_to_properties=True)
    pb = padded.block(o3_lambda=0, o3_sigma=1, center_type=1)
    col = [j for j, p in enumerate(pb.properties.values) if p[2] == 7 or p[4] == 7]
    assert col and float(pb.values[:, :, col].abs().max()) == 0.0
