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
goldens), the rotation of the lambda = 1 blocks of a molecule, the
neighbor-types-to-properties form against the keyed form, and
DensityCorrelations (_density_correlations.py): nu = 2 against the
equivariant power spectrum, nu = 3 rotations and one block against the
oracle.  The property-name rule and the input checks of
_cg_product.py:336-432 run on the CPU."""
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


def test_increment_numeric_suffix():
    # the examples of _density_correlations.py:_increment_numeric_suffix
    f = cg._increment_numeric_suffix
    assert f("n", 1) == "n_1"
    assert f("n", 0) == "n_0"
    assert f("n_1", 1) == "n_2"
    assert f("center_type", 3) == "center_3_type"
    assert f("first_atom_1_type") == "first_atom_2_type"
    assert f("center_type_1_type", 7) == "center_type_8_type"


def _host_tensor(lmax, prop_name):
    import torch

    keys = rb.Labels(["o3_lambda", "o3_sigma", "center_type"], [[l, 1, 1] for l in range(lmax + 1)])
    blocks = [cg.Block(torch.zeros(2, 2 * l + 1, 3, dtype=torch.float64),
                       rb.Labels(["system", "atom"], [[0, 0], [0, 1]]),
                       [rb.Labels(["o3_mu"], np.arange(-l, l + 1).reshape(-1, 1))],
                       rb.Labels([prop_name], [[0], [1], [2]])) for l in range(lmax + 1)]
    return cg.EquivariantTensorMap(keys, blocks)


def test_product_input_checks():
    # _cg_product.py:336-432, checked before anything runs on a device
    a, b = _host_tensor(2, "n_1"), _host_tensor(3, "n_2")
    with pytest.raises(ValueError, match="exceeds the value of `max_angular=4`"):
        cg.ClebschGordanProduct(max_angular=4).plan(a, b, "l_1", "l_2")
    with pytest.raises(ValueError, match="present in both input tensors"):
        cg.ClebschGordanProduct(max_angular=8).plan(a, _host_tensor(3, "n_1"), "l_1", "l_2")
    with pytest.raises(ValueError, match="must only contain values of -1 or 1"):
        cg.ClebschGordanProduct(max_angular=8).plan(a, b, "l_1", "l_2",
                                                     selected_keys=rb.Labels(["o3_sigma"], [[2]]))
    with pytest.raises(ValueError, match="in `selected_keys` exceeds `max_angular=5`"):
        cg.ClebschGordanProduct(max_angular=5).plan(a, b, "l_1", "l_2",
                                                     selected_keys=rb.Labels(["o3_lambda"], [[6]]))


def _moved_density(system, hypers):
    se = rb.SphericalExpansion(**hypers)
    density = cg.as_tensormap(se.compute([system]), None)
    return cg.keys_to_properties(density, ["neighbor_type"]), se


@pytest.mark.gpu
def test_density_correlations_nu2_is_the_equivariant_power_spectrum():
    system = workloads.random_box(40, density=0.1, species=(1, 6, 8), seed=12)
    hypers = workloads.hypers(3.5, 2, 2, spline_accuracy=None)
    density, se = _moved_density(system, hypers)
    nu2 = cg.DensityCorrelations(n_correlations=1, max_angular=4).compute(density)
    assert nu2.keys.names == ["o3_lambda", "o3_sigma", "center_type", "l_1", "l_2"]
    assert nu2.block_by_id(0).properties.names == ["neighbor_1_type", "n_1", "neighbor_2_type", "n_2"]
    eps = cg.EquivariantPowerSpectrum(se).compute([system], neighbors_to_properties=True)
    for key, blk in zip(nu2.keys.values, nu2.blocks()):
        lam, sigma, ct, l1, l2 = (int(v) for v in key)
        eb = eps.block(o3_lambda=lam, o3_sigma=sigma, center_type=ct)
        cols = [j for j, p in enumerate(eb.properties.values) if p[0] == l1 and p[1] == l2]
        np.testing.assert_array_equal(eb.properties.values[cols][:, 2:], blk.properties.values)
        np.testing.assert_array_equal(eb.values[:, :, cols].cpu().numpy(), blk.values.cpu().numpy())


@pytest.mark.gpu
def test_density_correlations_nu3():
    rng = np.random.default_rng(8)
    mol = workloads.molecules(1, seed=9, min_atoms=10, max_atoms=10)[0]
    rotated = dict(mol)
    R = _rotation(rng)
    rotated["positions"] = np.ascontiguousarray(mol["positions"] @ R.T)
    hypers = workloads.hypers(4.0, 1, 2, spline_accuracy=None)
    calc = cg.DensityCorrelations(n_correlations=2, max_angular=6)
    density, _ = _moved_density(mol, hypers)
    a = calc.compute(density, angular_cutoff=2)
    b = calc.compute(_moved_density(rotated, hypers)[0], angular_cutoff=2)
    assert a.keys.names == ["o3_lambda", "o3_sigma", "center_type", "l_1", "l_2", "k_2", "l_3"]
    assert a.block_by_id(0).properties.names == ["neighbor_1_type", "n_1", "neighbor_2_type", "n_2",
                                                 "neighbor_3_type", "n_3"]
    # intermediate lambda <= 2, the redundant filter keeps l_1 <= l_2 <= l_3
    assert a.keys.column("k_2").max() <= 2
    assert all(k[3] <= k[4] <= k[6] for k in a.keys.values)
    perm = np.array([1, 2, 0])
    Rm = R[np.ix_(perm, perm)]
    for i, key in enumerate(a.keys.values):
        va, vb = a.block_by_id(i).values.cpu().numpy(), b.block_by_id(i).values.cpu().numpy()
        tol = 1e-9 * max(1.0, np.abs(va).max())
        if key[0] == 0:
            np.testing.assert_allclose(vb, va, rtol=0, atol=tol)
        elif key[0] == 1:
            np.testing.assert_allclose(np.einsum("xy,syp->sxp", Rm, va), vb, rtol=0, atol=tol)
    # one block recomputed with the oracle from the nu = 2 intermediate
    nu2 = cg.DensityCorrelations(n_correlations=1, max_angular=6).compute(density, angular_cutoff=2)
    key = next(k for k in a.keys.values if k[0] == 1 and k[5] == 1 and k[6] == 2)
    lam, sigma, ct, l1, l2, k2, l3 = (int(v) for v in key)
    # sigma = (-1)^(l_1 + l_2 + k_2) is fixed by the others
    idx = [i for i, k in enumerate(nu2.keys.values) if k[0] == k2 and k[2] == ct and k[3] == l1 and k[4] == l2]
    assert len(idx) == 1
    left = nu2.block_by_id(idx[0])
    right = density.block(o3_lambda=l3, center_type=ct)
    ref = ocg.cg_tensor_product(left.values.cpu().numpy(), right.values.cpu().numpy(), lam)
    got = a.block(o3_lambda=lam, o3_sigma=sigma, center_type=ct, l_1=l1, l_2=l2, k_2=k2, l_3=l3)
    np.testing.assert_allclose(got.values.cpu().numpy(), ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_power_spectrum_gradient_parameters():
    se = rb.SphericalExpansion(**workloads.hypers(3.0, 2, 2))
    ps = cg.PowerSpectrum(se)
    with pytest.raises(NotImplementedError, match="only supports gradients w.r.t. to positions"):
        ps.compute([workloads.random_box(10, seed=1)], gradients=["strain"])


@pytest.mark.gpu
def test_cg_power_spectrum_is_the_soap_power_spectrum():
    # _power_spectrum.py: the same invariants as SoapPowerSpectrum without the
    # sqrt(2) of mixed neighbour types, every neighbour type pair in the properties
    system = workloads.random_box(48, density=0.1, species=(1, 6, 8), seed=13)
    se = rb.SphericalExpansion(**_ps_hypers())
    out = cg.PowerSpectrum(se).compute([system])
    assert out.keys.names == ["center_type"]
    blk = out.block_by_id(0)
    assert blk.properties.names == ["l", "neighbor_1_type", "n_1", "neighbor_2_type", "n_2"]
    assert blk.components == []
    ps = rb.SoapPowerSpectrum(**_ps_hypers()).compute([system])
    checked = 0
    for key, pblk in zip(ps.keys.values, ps.blocks()):
        ct, n1, n2 = (int(v) for v in key)
        cblk = out.block(center_type=ct)
        props = {tuple(p): i for i, p in enumerate(cblk.properties.values)}
        rows = [{tuple(s): i for i, s in enumerate(cblk.samples.values)}[tuple(s)] for s in pblk.samples.values]
        cv = cblk.values.cpu().numpy()[rows]
        cols = [props[(l, n1, a, n2, b)] for l, a, b in pblk.properties.values]
        factor = 1.0 if n1 == n2 else np.sqrt(2.0)
        np.testing.assert_allclose(factor * cv[:, cols], np.asarray(pblk.values), rtol=1e-10, atol=1e-14)
        # the (n2, n1) properties hold the transposed invariants
        cols_t = [props[(l, n2, b, n1, a)] for l, a, b in pblk.properties.values]
        np.testing.assert_allclose(factor * cv[:, cols_t], np.asarray(pblk.values), rtol=1e-10, atol=1e-14)
        checked += cv[:, cols].size
    assert checked > 1000


def test_cg_product_rejects_bad_tasks():
    # checked on the host before anything is queued: no device memory is touched
    import ctypes

    from rascaline_b200 import _c_api as C

    task = C.featomic_b200_cg_task_t(16, 32, 48, 2, 1, 1, 0, 4, 4, 8)
    arr = (C.featomic_b200_cg_task_t * 1)(task)
    assert C.lib().featomic_b200_cg_product(arr, 1, 64, None) == 1
    assert "smaller than n_first * n_second" in C.lib().featomic_last_error().decode()
    task.output_stride = 0
    task.lambda_ = 3
    arr = (C.featomic_b200_cg_task_t * 1)(task)
    assert C.lib().featomic_b200_cg_product(arr, 1, 64, None) == 1
    assert "can not couple" in C.lib().featomic_last_error().decode()
    assert C.lib().featomic_b200_cg_product(arr, 1, 16, None) == 1
    assert "precision must be 32 or 64" in C.lib().featomic_last_error().decode()
    assert C.lib().featomic_b200_cg_product(None, 0, 64, None) == 0


@pytest.mark.gpu
def test_cg_power_spectrum_positions_gradients():
    # _power_spectrum.py:373-435 against the drop-in power spectrum's gradient
    # rows (pinned to featomic's goldens), matched by (centre, atom)
    system = workloads.random_box(40, density=0.1, species=(1, 8), seed=14)
    se = rb.SphericalExpansion(**_ps_hypers())
    out = cg.PowerSpectrum(se).compute([system], gradients=["positions"])
    ps = rb.SoapPowerSpectrum(**_ps_hypers()).compute([system], gradients=["positions"])
    checked = 0
    for key, pblk in zip(ps.keys.values, ps.blocks()):
        ct, n1, n2 = (int(v) for v in key)
        cblk = out.block(center_type=ct)
        cgrad = cblk.gradient("positions")
        assert cgrad.components[0].names == ["xyz"]
        props = {tuple(p): i for i, p in enumerate(cblk.properties.values)}
        cols = [props[(l, n1, a, n2, b)] for l, a, b in pblk.properties.values]
        crow = {(tuple(cblk.samples.values[g[0]]), int(g[2])): i for i, g in enumerate(cgrad.samples.values)}
        pgrad = pblk.gradient("positions")
        pv = np.asarray(pgrad.values)
        cv = cgrad.values.cpu().numpy()
        factor = 1.0 if n1 == n2 else np.sqrt(2.0)
        for i, g in enumerate(pgrad.samples.values):
            row = crow[(tuple(pblk.samples.values[g[0]]), int(g[2]))]
            np.testing.assert_allclose(factor * cv[row][:, cols], pv[i], rtol=1e-9,
                                       atol=1e-12 * max(1.0, np.abs(pv).max()))
            checked += 1
    assert checked > 100
    # the values are those of the values-only call
    plain = cg.PowerSpectrum(se).compute([system])
    for i in range(len(out)):
        np.testing.assert_array_equal(out.block_by_id(i).values.cpu().numpy(),
                                      plain.block_by_id(i).values.cpu().numpy())


@pytest.mark.gpu
def test_compute_metadata_matches_compute():
    system = workloads.random_box(30, density=0.1, species=(1, 8), seed=15)
    hypers = workloads.hypers(3.5, 2, 2, spline_accuracy=None)
    se = rb.SphericalExpansion(**hypers)
    eps = cg.EquivariantPowerSpectrum(se)
    density, _ = _moved_density(system, hypers)
    dc = cg.DensityCorrelations(n_correlations=2, max_angular=6)
    for full, meta in ((eps.compute([system]), eps.compute_metadata([system])),
                       (eps.compute([system], neighbors_to_properties=True),
                        eps.compute_metadata([system], neighbors_to_properties=True)),
                       (dc.compute(density, angular_cutoff=2), dc.compute_metadata(density, angular_cutoff=2))):
        np.testing.assert_array_equal(full.keys.values, meta.keys.values)
        assert full.keys.names == meta.keys.names
        for a, b in zip(full.blocks(), meta.blocks()):
            assert tuple(a.values.shape) == tuple(b.values.shape)
            np.testing.assert_array_equal(a.samples.values, b.samples.values)
            np.testing.assert_array_equal(a.properties.values, b.properties.values)
            assert a.properties.names == b.properties.names



def _cartesian_tensor(values, rank):
    import torch

    S, P = values.shape[0], values.shape[-1]
    keys = rb.Labels(["key"], [[0]])
    comps = [rb.Labels([f"xyz_{i + 1}"], [[0], [1], [2]]) for i in range(rank)]
    block = cg.Block(torch.tensor(values, device="cuda"), rb.Labels(["sample"], np.arange(S).reshape(-1, 1)), comps,
                     rb.Labels(["p"], np.arange(P).reshape(-1, 1)))
    return cg.EquivariantTensorMap(keys, [block])


@pytest.mark.gpu
def test_cg_couple_matches_oracle():
    import torch

    rng = np.random.default_rng(21)
    for dtype, tol in ((torch.float64, 1e-13), (torch.float32, 2e-6)):
        tasks, expected = [], []
        for l1, l2 in ((1, 1), (2, 1), (3, 2)):
            x = rng.standard_normal((7, 2 * l1 + 1, 2 * l2 + 1, 5))
            tx = torch.tensor(x, dtype=dtype, device="cuda")
            for lam in range(abs(l1 - l2), l1 + l2 + 1):
                out = torch.full((7, 2 * lam + 1, 5), float("nan"), dtype=dtype, device="cuda")
                tasks.append((tx, out, l1, l2, lam))
                expected.append(ocg.cg_couple(tx.double().cpu().numpy(), lam))
        cg.cg_couple(tasks)
        for (_, out, _, _, _), ref in zip(tasks, expected):
            np.testing.assert_allclose(out.double().cpu().numpy(), ref, rtol=0, atol=tol * max(1.0, np.abs(ref).max()))


@pytest.mark.gpu
def test_cartesian_to_spherical():
    rng = np.random.default_rng(22)
    # rank 1: (x, y, z) -> (y, z, x) as the o3_mu = -1, 0, 1 components
    v = rng.standard_normal((4, 3, 2))
    out = cg.cartesian_to_spherical(_cartesian_tensor(v, 1), ["xyz_1"])
    assert out.keys.names == ["o3_lambda", "o3_sigma", "key"]
    np.testing.assert_array_equal(out.keys.values, [[1, 1, 0]])
    np.testing.assert_array_equal(out.block_by_id(0).values.cpu().numpy(), v[:, [1, 2, 0], :])
    # rank 2: a symmetric matrix has no o3_sigma = -1 block; values from the oracle
    m = rng.standard_normal((5, 3, 3, 2))
    sym = m + m.transpose(0, 2, 1, 3)
    out = cg.cartesian_to_spherical(_cartesian_tensor(sym, 2), ["xyz_1", "xyz_2"])
    assert out.keys.names == ["o3_lambda", "o3_sigma", "key"]
    np.testing.assert_array_equal(out.keys.values, [[0, 1, 0], [2, 1, 0]])
    rolled = sym[:, [1, 2, 0]][:, :, [1, 2, 0]]
    for key, blk in zip(out.keys.values, out.blocks()):
        np.testing.assert_allclose(blk.values.cpu().numpy(), ocg.cg_couple(rolled, int(key[0])), atol=1e-13)
        assert blk.components[0].names == ["o3_mu"]
    # lambda = 0 is -trace / sqrt(3); rotations leave it and the lambda = 2 norm unchanged
    np.testing.assert_allclose(out.block_by_id(0).values.cpu().numpy()[:, 0, :],
                               -np.trace(sym, axis1=1, axis2=2) / np.sqrt(3), atol=1e-13)
    R = _rotation(rng)
    rot = np.einsum("ij,sjkp,lk->silp", R, sym, R)
    out_r = cg.cartesian_to_spherical(_cartesian_tensor(rot, 2), ["xyz_1", "xyz_2"])
    for a, b in zip(out.blocks(), out_r.blocks()):
        np.testing.assert_allclose(np.linalg.norm(b.values.cpu().numpy(), axis=1),
                                   np.linalg.norm(a.values.cpu().numpy(), axis=1), atol=1e-12)
    # rank 3: l / k dimensions in the keys, invariant lambda = 0 block
    t = rng.standard_normal((3, 3, 3, 3, 1))
    out = cg.cartesian_to_spherical(_cartesian_tensor(t, 3), ["xyz_1", "xyz_2", "xyz_3"])
    assert out.keys.names == ["o3_lambda", "o3_sigma", "l_3", "k_1", "l_2", "l_1", "key"]
    assert sorted(int(k[0]) for k in out.keys.values) == [0, 1, 1, 1, 2, 2, 3]
    rot = np.einsum("ia,jb,kc,sabcp->sijkp", R, R, R, t)
    out_r = cg.cartesian_to_spherical(_cartesian_tensor(rot, 3), ["xyz_1", "xyz_2", "xyz_3"])
    for key, a, b in zip(out.keys.values, out.blocks(), out_r.blocks()):
        va, vb = a.values.cpu().numpy(), b.values.cpu().numpy()
        np.testing.assert_allclose(np.linalg.norm(vb, axis=1), np.linalg.norm(va, axis=1), atol=1e-12)
        if key[0] == 0:
            np.testing.assert_allclose(vb, va, atol=1e-12)
    with pytest.raises(ValueError, match="must be `True` for tensors of rank 3"):
        cg.cartesian_to_spherical(_cartesian_tensor(t, 3), ["xyz_1", "xyz_2", "xyz_3"], keep_l_in_keys=False)


def _host_cartesian(rank, values=(0, 1, 2), keys=("key",)):
    comps = [rb.Labels([f"xyz_{i + 1}"], np.array(values).reshape(-1, 1)) for i in range(rank)]
    block = cg.Block(np.zeros((2,) + (len(values),) * rank + (1,)), rb.Labels(["sample"], [[0], [1]]), comps,
                     rb.Labels(["p"], [[0]]))
    return cg.EquivariantTensorMap(rb.Labels(list(keys), [[0] * len(keys)]), [block])


def test_cartesian_to_spherical_input_checks():
    # _cartesian_spherical.py:86-130, all raised before anything runs on a device
    with pytest.raises(ValueError, match="'xyz_9' is not part of this tensor components"):
        cg.cartesian_to_spherical(_host_cartesian(2), ["xyz_9"])
    with pytest.raises(ValueError, match=r"should have \[0, 1, 2\] as values"):
        cg.cartesian_to_spherical(_host_cartesian(1, values=(0, 1, 3)), ["xyz_1"])
    with pytest.raises(ValueError, match="only supports consecutive components"):
        cg.cartesian_to_spherical(_host_cartesian(3), ["xyz_1", "xyz_3"])
    with pytest.raises(ValueError, match="already has an `o3_lambda` key"):
        cg.cartesian_to_spherical(_host_cartesian(1, keys=("o3_lambda",)), ["xyz_1"])
    with pytest.raises(TypeError, match="should be a list"):
        cg.cartesian_to_spherical(_host_cartesian(1), "xyz_1")
    empty = _host_cartesian(1)
    assert cg.cartesian_to_spherical(empty, []) is empty


def test_cg_couple_rejects_bad_tasks():
    # host-side checks before anything is queued: no device memory is touched
    from rascaline_b200 import _c_api as C

    task = C.featomic_b200_cg_couple_task_t(16, 32, 2, 3, 1, 1, 3)
    arr = (C.featomic_b200_cg_couple_task_t * 1)(task)
    assert C.lib().featomic_b200_cg_couple(arr, 1, 64, None) == 1
    assert "can not couple" in C.lib().featomic_last_error().decode()
    assert C.lib().featomic_b200_cg_couple(arr, 1, 8, None) == 1
    assert "precision must be 32 or 64" in C.lib().featomic_last_error().decode()
    assert C.lib().featomic_b200_cg_couple(None, 0, 64, None) == 0


@pytest.mark.gpu
def test_cartesian_to_spherical_backends():
    """featomic's coupling backends differ on the o3_sigma = -1 blocks: the
    "python-sparse" backend (default for numpy values) couples x[m1, m2]
    with C[m1, m2, mu], the "python-dense" backend (default for torch values)
    swaps the coupled axes first, which multiplies each block by
    (-1)^(l1 + l2 + lambda) (_coefficients.py:440-455).  A non-symmetric
    rank-2 tensor has a lambda = 1, o3_sigma = -1 block: sparse equals the
    oracle's coupling, dense equals minus it (1e-13)."""
    rng = np.random.default_rng(31)
    m = rng.standard_normal((5, 3, 3, 2))
    rolled = m[:, [1, 2, 0]][:, :, [1, 2, 0]]
    sparse = cg.cartesian_to_spherical(_cartesian_tensor(m, 2), ["xyz_1", "xyz_2"], cg_backend="python-sparse")
    dense = cg.cartesian_to_spherical(_cartesian_tensor(m, 2), ["xyz_1", "xyz_2"])
    np.testing.assert_array_equal(sparse.keys.values, [[0, 1, 0], [1, -1, 0], [2, 1, 0]])
    np.testing.assert_array_equal(dense.keys.values, sparse.keys.values)
    for key, bs, bd in zip(sparse.keys.values, sparse.blocks(), dense.blocks()):
        ref = ocg.cg_couple(rolled, int(key[0]))
        np.testing.assert_allclose(bs.values.cpu().numpy(), ref, rtol=0, atol=1e-13)
        np.testing.assert_allclose(bd.values.cpu().numpy(), int(key[1]) * ref, rtol=0, atol=1e-13)
    # numpy values: the sparse default, numpy values back
    host = cg.EquivariantTensorMap(rb.Labels(["key"], [[0]]), [cg.Block(
        m, rb.Labels(["sample"], np.arange(5).reshape(-1, 1)),
        [rb.Labels([f"xyz_{i + 1}"], [[0], [1], [2]]) for i in range(2)], rb.Labels(["p"], [[0], [1]]))])
    out = cg.cartesian_to_spherical(host, ["xyz_1", "xyz_2"])
    assert isinstance(out.block_by_id(1).values, np.ndarray)
    np.testing.assert_allclose(out.block_by_id(1).values, ocg.cg_couple(rolled, 1), rtol=0, atol=1e-13)
    with pytest.raises(ValueError, match="invalid `cg_backend`"):
        cg.cartesian_to_spherical(host, ["xyz_1", "xyz_2"], cg_backend="python-fast")


def test_calculate_cg_coefficients_layout():
    """featomic's coefficient cache (_coefficients.py:35-134, 225-335): keys
    (l1, l2, lambda) for l1, l2 <= lambda_max and |l1 - l2| <= lambda <=
    min(lambda_max, l1 + l2); dense blocks [1, 2 l1 + 1, 2 l2 + 1, 2 lambda +
    1, 1], sparse blocks of the non-zero coefficients with (m1, m2, mu)
    samples; values equal cg_coefficients."""
    dense = cg.calculate_cg_coefficients(2, "python-dense", "numpy", np.float64, "cpu")
    sparse = cg.calculate_cg_coefficients(2, "python-sparse", "numpy", np.float64, "cpu")
    expected = [[l1, l2, lam] for l1 in range(3) for l2 in range(3) for lam in range(abs(l1 - l2), min(2, l1 + l2) + 1)]
    assert dense.keys.names == ["l1", "l2", "lambda"]
    np.testing.assert_array_equal(dense.keys.values, expected)
    np.testing.assert_array_equal(sparse.keys.values, expected)
    for (l1, l2, lam), bd, bs in zip(expected, dense.blocks(), sparse.blocks()):
        ref = cg.cg_coefficients(l1, l2, lam)
        assert bd.values.shape == (1,) + ref.shape + (1,)
        np.testing.assert_array_equal(bd.values[0, ..., 0], ref)
        assert [c.names[0] for c in bd.components] == ["m1", "m2", "mu"]
        assert bs.samples.names == ["m1", "m2", "mu"]
        rebuilt = np.zeros_like(ref)
        rebuilt[tuple(bs.samples.values.T)] = bs.values[:, 0]
        np.testing.assert_array_equal(rebuilt, np.where(np.abs(ref) > 1e-15, ref, 0.0))
    with pytest.raises(ValueError, match="invalid `cg_backend`"):
        cg.calculate_cg_coefficients(1, "python-fast", "numpy", np.float64, "cpu")
