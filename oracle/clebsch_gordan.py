"""Test infrastructure, never imported by the product: a numpy restatement of
featomic's Clebsch-Gordan coefficients and block tensor product
(python/featomic/featomic/clebsch_gordan/_coefficients.py), the checker of
``featomic_b200_cg_coefficients`` / ``featomic_b200_cg_product``.

The complex CG coefficients come from sympy's exact ``CG`` (the reference
takes them from the ``wigners`` package, absent here; both use the
Condon-Shortley convention), so this side shares no arithmetic with the C++
Racah sum it checks.
"""
import functools

import numpy as np


@functools.lru_cache(maxsize=None)
def complex_cg(l1, l2, lam):
    """[2 l1 + 1, 2 l2 + 1, 2 lam + 1] complex CG <l1 m1 l2 m2 | lam mu>."""
    from sympy.physics.quantum.cg import CG

    out = np.zeros((2 * l1 + 1, 2 * l2 + 1, 2 * lam + 1))
    for m1 in range(-l1, l1 + 1):
        for m2 in range(-l2, l2 + 1):
            mu = m1 + m2
            if abs(mu) <= lam:
                out[l1 + m1, l2 + m2, lam + mu] = float(CG(l1, m1, l2, m2, lam, mu).doit())
    return out


def real_to_complex(l):
    """_coefficients.py:336-369 (_real2complex)."""
    u = np.zeros((2 * l + 1, 2 * l + 1), dtype=complex)
    r = 1 / np.sqrt(2)
    for m in range(-l, l + 1):
        if m < 0:
            u[l + m, l + m] = -1j * r
            u[l + m, l - m] = 1j * r * (-1) ** m
        elif m == 0:
            u[l, l] = 1
        else:
            u[l + m, l - m] = r
            u[l + m, l + m] = r * (-1) ** m
    return u


@functools.lru_cache(maxsize=None)
def real_cg(l1, l2, lam):
    """_coefficients.py:137-224 (_build_dense_cg_coeff_dict), one entry."""
    c = complex_cg(l1, l2, lam).astype(complex)
    r = np.einsum("ab,bcd->acd", real_to_complex(l1), c)
    r = np.einsum("ab,cbd->cad", real_to_complex(l2), r)
    r = r @ np.conj(real_to_complex(lam)).T
    return np.real(r) if (l1 + l2 + lam) % 2 == 0 else np.imag(r)


def cg_tensor_product(a, b, lam):
    """_coefficients.py:677-709 (_cg_tensor_product_dense):
    a [s, 2 l1 + 1, p], b [s, 2 l2 + 1, q] -> [s, 2 lam + 1, p * q]."""
    l1 = (a.shape[1] - 1) // 2
    l2 = (b.shape[1] - 1) // 2
    s, p, q = a.shape[0], a.shape[2], b.shape[2]
    # outer product [s, p, q, m1, m2], then one matrix product with the
    # coefficients [(m1 m2), mu], as the reference's dense backend does
    outer = np.einsum("sxp,syq->spqxy", a, b).reshape(s * p * q, -1)
    out = outer @ real_cg(l1, l2, lam).reshape(-1, 2 * lam + 1)
    return out.reshape(s, p * q, 2 * lam + 1).transpose(0, 2, 1)


def cg_couple(x, lam):
    """_coefficients.py:387-545 (cg_couple): x [b, 2 l1 + 1, 2 l2 + 1, a]
    -> [b, 2 lam + 1, a]."""
    l1 = (x.shape[1] - 1) // 2
    l2 = (x.shape[2] - 1) // 2
    return np.einsum("xyz,bxya->bza", real_cg(l1, l2, lam), x)
