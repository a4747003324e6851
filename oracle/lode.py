"""TEST INFRASTRUCTURE -- CPU restatement of featomic's LODE spherical
expansion (featomic/src/calculators/lode/), FP64 numpy.

Only tests/ import this module, as the checker of the library's
``lode_spherical_expansion`` calculator.

Follows, function by function:

* k-vectors: ``compute_k_vectors`` (featomic/src/math/k_vectors.rs:19-87),
  same enumeration order (n1 = n2 = 0 first, then n1 = 0, then the rest);
* radial integral of the GTO basis at |k| (lode/radial_integral/gto.rs:
  62-131): sqrt(pi / 2) sigma_n^{n+3} sqrt(2)^n (k sigma_n / sqrt2)^l
  Gamma(a) / Gamma(b) 1F1(a, b, -k^2 sigma_n^2 / 2), a = (n + l + 3) / 2,
  b = l + 3/2, then the orthonormalisation; 1F1 and Gamma of the SOAP
  oracle (restated from featomic's math/hyp1f1.rs and math/gamma.rs, pinned
  to their tables);
* Fourier transform of the smeared power-law density
  (lode/spherical_expansion.rs:276-335) with the closed forms for p = 0..9
  (erfc and Ei from scipy);
* k = 0 term (:337-376) and the central-atom contribution (gto.rs:133-181,
  2F1 from scipy);
* structure factors (:92-159), projection of the k-vectors on (n, l, m)
  (:226-274), values (:616-723) and positions gradients (:725-873);
* keys ``AllTypesPairsKeys`` (labels/keys.rs:36-57) times the angular
  channels, samples and gradient samples ``LongRangeSamplesPerAtom``
  (labels/samples/long_range.rs:21-74).

Pinned against featomic's own reference data: the LODE spherical expansion
values and positions gradients for potential exponents 1 to 6
(featomic/tests/data/lode-spherical-expansion.py, compared like
featomic/tests/lode-spherical-expansion.rs at max_relative 1e-6) and the
pyLODE central-atom contributions of gto.rs:261-286.
"""
import numpy as np
from scipy import special

from . import oracle


def hypers_from_json(h):
    density = h["density"]
    basis = h["basis"]
    if density.get("type") != "SmearedPowerLaw":
        raise ValueError("only SmearedPowerLaw density can be used with LODE")
    radial = basis["radial"]
    smearing = float(density["smearing"])
    exponent = int(density["exponent"])
    k_cutoff = h.get("k_cutoff")
    return {
        "smearing": smearing,
        "exponent": exponent,
        "center_atom_weight": float(density.get("center_atom_weight", 1.0)),
        "k_cutoff": float(k_cutoff) if k_cutoff is not None else 1.2 * np.pi / smearing,
        "max_angular": int(basis["max_angular"]),
        "nmax": int(radial["max_radial"]) + 1,
        "radius": float(radial["radius"]),
    }


def k_vectors(cell, k_cutoff):
    """(norms, directions) of the reciprocal lattice points inside the
    k_cutoff ball, one of each +-k pair (k_vectors.rs:19-87)."""
    cell = np.asarray(cell, dtype=np.float64).reshape(3, 3)
    reciprocal = 2.0 * np.pi * np.linalg.inv(cell.T)
    b1, b2, b3 = reciprocal
    m = reciprocal @ reciprocal.T
    volume = np.linalg.det(reciprocal)
    n1_max = int(np.sqrt(m[1, 1] * m[2, 2] - m[1, 2] * m[1, 2]) / volume * k_cutoff)
    n2_max = int(np.sqrt(m[2, 2] * m[0, 0] - m[2, 0] * m[2, 0]) / volume * k_cutoff)
    n3_max = int(np.sqrt(m[0, 0] * m[1, 1] - m[0, 1] * m[0, 1]) / volume * k_cutoff)
    out = []

    def add(k):
        n2 = k @ k
        if n2 < k_cutoff * k_cutoff:
            norm = np.sqrt(n2)
            out.append((norm, k / norm))

    for n3 in range(1, n3_max + 1):
        add(n3 * b3)
    for n2 in range(1, n2_max + 1):
        for n3 in range(-n3_max, n3_max + 1):
            add(n2 * b2 + n3 * b3)
    for n1 in range(1, n1_max + 1):
        for n2 in range(-n2_max, n2_max + 1):
            for n3 in range(-n3_max, n3_max + 1):
                add(n1 * b1 + n2 * b2 + n3 * b3)
    norms = np.array([o[0] for o in out])
    directions = np.array([o[1] for o in out]).reshape(-1, 3)
    return norms, directions


def gto_widths(nmax, radius):
    return np.array([radius * max(np.sqrt(n), 1.0) / nmax for n in range(nmax)])


def radial_integral(l, k, nmax, radius):
    """Orthonormalised LODE radial integral of channel l at |k| = k
    (radial_integral/gto.rs:62-131), values only."""
    sigma = gto_widths(nmax, radius)
    values = np.zeros(nmax)
    for n in range(nmax):
        factor = np.sqrt(np.pi) / np.sqrt(2.0) * sigma[n] ** (n + 3) * np.sqrt(2.0) ** n \
            * (k * sigma[n] / np.sqrt(2.0)) ** l
        z = 0.5 * k * (-k * sigma[n] * sigma[n])
        a, b = 0.5 * (n + l + 3), l + 1.5
        values[n] = factor * (oracle.gamma(a) / oracle.gamma(b) * oracle.hyp1f1(a, b, z))
    ortho = oracle.gto_orthonormalization(nmax, radius)
    return ortho @ values


def center_contribution(hypers):
    """<n 0 0> contribution of the central atom (gto.rs:133-181)."""
    nmax, radius = hypers["nmax"], hypers["radius"]
    smearing, p = hypers["smearing"], float(hypers["exponent"])
    sigma = gto_widths(nmax, radius)
    contrib = np.zeros(nmax)
    for n in range(nmax):
        n_eff = 0.5 * (3.0 + n)
        if p == 0.0:
            factor = np.pi ** -0.25 / (smearing * smearing) ** 0.75
            alpha = 0.5 * (1.0 / smearing ** 2 + 1.0 / sigma[n] ** 2)
            contrib[n] = factor * special.gamma(n_eff) / alpha ** n_eff
        else:
            factor = 2.0 * np.sqrt(4.0 * np.pi) / special.gamma(p / 2.0) / p
            s = smearing / sigma[n]
            hyparg = 1.0 / (1.0 + s * s)
            contrib[n] = factor * 2.0 ** ((1.0 + n - p) / 2.0) * smearing ** (3 + n - int(p)) \
                * special.gamma(n_eff) * special.hyp2f1(1.0, n_eff, (p + 2.0) / 2.0, hyparg) * hyparg ** n_eff
    return oracle.gto_orthonormalization(nmax, radius) @ contrib


def density_fourier(hypers, norms):
    """Fourier transform of the smeared power-law density
    (spherical_expansion.rs:276-335)."""
    p, s2 = hypers["exponent"], hypers["smearing"] ** 2
    k2 = norms * norms
    if p == 0:
        return (4.0 * np.pi * s2) ** 0.75 * np.exp(-0.5 * k2 * s2)
    if p == 1:
        return 4.0 * np.pi * np.exp(-0.5 * k2 * s2) / k2
    p_eff = 3.0 - p
    factor = np.pi ** 1.5 * (2.0 * s2) ** (0.5 * p_eff) / special.gamma(0.5 * p)
    x = 0.5 * k2 * s2
    ei = special.expi(-x)
    ec = special.erfc(np.sqrt(x))
    forms = {
        2: np.sqrt(np.pi / x) * ec,
        3: -ei,
        4: 2.0 * (np.exp(-x) - np.sqrt(np.pi * x) * ec),
        5: np.exp(-x) + x * ei,
        6: ((2.0 - 4.0 * x) * np.exp(-x) + 4.0 * np.sqrt(np.pi) * x ** 1.5 * ec) / 3.0,
        7: (1.0 - x) * np.exp(-x) / 2.0 - x ** 2 / 2.0 * ei,
        8: -2.0 / 15.0 * ((-3.0 + 2.0 * x - 4.0 * x ** 2) * np.exp(-x) + 4.0 * np.sqrt(np.pi) * x ** 2.5 * ec),
        9: (x ** 2 - x + 2.0) * np.exp(-x) / 6.0 + x ** 3 / 6.0 * ei,
    }
    return factor * forms[p]


def k0_factor(hypers):
    """Prefactor of the k = 0 term (spherical_expansion.rs:337-376)."""
    p, smearing = hypers["exponent"], hypers["smearing"]
    if p == 0:
        s2 = smearing * smearing
        return (2.0 * np.pi * s2) ** 1.5 / (np.pi * s2) ** 0.75 / np.sqrt(4.0 * np.pi)
    if p > 3:
        p_eff = 3.0 - p
        return 0.5 * np.pi * 2.0 ** p_eff / special.gamma(0.5 * p) * 2.0 ** ((p - 1.0) / 2.0) / -p_eff \
            * smearing ** -p_eff / smearing ** (2.0 * p - 6.0)
    return 0.0


def compute(hypers_json, systems, gradients=()):
    """featomic's lode_spherical_expansion on ``systems`` (dicts with
    ``types``, ``positions``, ``cell``).  Same dict layout as oracle.compute:
    keys (o3_lambda, o3_sigma, center_type, neighbor_type); values
    [samples, 2l + 1, n]; positions gradients [rows, xyz, 2l + 1, n]."""
    h = hypers_from_json(hypers_json)
    L, nmax = h["max_angular"], h["nmax"]
    pairs = set()
    for s in systems:
        types = set(int(t) for t in s["types"])
        pairs |= {(a, b) for a in types for b in types}
    keys = [(l, 1, a, b) for a, b in sorted(pairs) for l in range(L + 1)]
    blocks = {k: {"samples": [], "values": [], "grad_samples": [], "grad_values": []} for k in keys}
    center = center_contribution(h) if L >= 0 else None
    k0 = k0_factor(h) * radial_integral(0, 0.0, nmax, h["radius"])
    ylm_lmax = L
    for system_i, s in enumerate(systems):
        types = np.asarray(s["types"])
        pos = np.asarray(s["positions"], dtype=np.float64).reshape(-1, 3)
        cell = np.asarray(s["cell"], dtype=np.float64).reshape(3, 3)
        norms, directions = k_vectors(cell, h["k_cutoff"])
        if len(norms) == 0:
            raise ValueError("No k-vectors for current combination of hyper parameters.")
        # k -> (l, m, n) projection: R_nl(|k|) Y_lm(k^)
        ylm = np.array([oracle.spherical_harmonics(ylm_lmax, d) for d in directions])  # [K, (L+1)^2]
        radial = np.array([[radial_integral(l, k, nmax, h["radius"]) for l in range(L + 1)] for k in norms])
        proj = {l: np.einsum("km,kn->mnk", ylm[:, l * l:(l + 1) * (l + 1)], radial[:, l, :]) for l in range(L + 1)}
        # structure factors
        phase = (norms[:, None] * directions) @ pos.T  # [K, N]
        cos, sin = np.cos(phase).T, np.sin(phase).T  # [N, K]
        all_types = sorted(set(int(t) for t in types))
        sum_cos = {t: cos[types == t].sum(axis=0) for t in all_types}
        sum_sin = {t: sin[types == t].sum(axis=0) for t in all_types}
        real = {t: 2.0 * (cos * sum_cos[t] + sin * sum_sin[t]) for t in all_types}
        imag = {t: 2.0 * (sin * sum_cos[t] - cos * sum_sin[t]) for t in all_types}
        fourier = density_fourier(h, norms)
        global_factor = 4.0 * np.pi / abs(np.linalg.det(cell))
        kvec = norms[:, None] * directions
        for (l, _, ct, nt) in keys:
            if nt not in all_types:
                continue
            block = blocks[(l, 1, ct, nt)]
            phase_l = (-1.0) ** (l // 2) if l % 2 == 0 else (-1.0) ** ((l + 1) // 2)
            sf = real[nt] if l % 2 == 0 else imag[nt]
            for i in np.nonzero(types == ct)[0]:
                row = np.zeros((2 * l + 1, nmax))
                if l == 0 and ct == nt:
                    row[0] -= (1.0 - h["center_atom_weight"]) * center
                if l == 0 and (h["exponent"] == 0 or h["exponent"] > 3):
                    row[0] += global_factor * k0 * np.count_nonzero(types == nt)
                weights = global_factor * phase_l * fourier * sf[i]
                row += proj[l] @ weights
                sample = len(block["samples"])
                block["samples"].append((system_i, int(i)))
                block["values"].append(row)
                if "positions" not in gradients:
                    continue
                for j in range(len(types)):
                    if types[j] != nt and j != i:
                        continue
                    if l % 2 == 0:
                        pair = 2.0 * (sin[i] * cos[j] - cos[i] * sin[j])
                    else:
                        pair = -2.0 * (cos[i] * cos[j] + sin[i] * sin[j])
                    if j == i:
                        sf_phase, sf_grad = (1.0, imag[nt]) if l % 2 == 0 else (-1.0, real[nt])
                        if nt == ct:
                            pair = -(sf_phase * sf_grad[i] - pair)
                        else:
                            pair = -sf_phase * sf_grad[i]
                    kd = pair * global_factor * phase_l * fourier
                    grad = np.einsum("mnk,k,kx->xmn", proj[l], kd, kvec)
                    block["grad_samples"].append((sample, system_i, j))
                    block["grad_values"].append(grad)
    out_blocks = []
    for k in keys:
        b = blocks[k]
        l = k[0]
        entry = {
            "samples": np.array(b["samples"], dtype=np.int32).reshape(-1, 2),
            "properties": np.arange(nmax, dtype=np.int32).reshape(-1, 1),
            "values": np.array(b["values"]).reshape(-1, 2 * l + 1, nmax),
            "gradients": {},
        }
        if "positions" in gradients:
            entry["gradients"]["positions"] = {
                "samples": np.array(b["grad_samples"], dtype=np.int32).reshape(-1, 3),
                "values": np.array(b["grad_values"]).reshape(-1, 3, 2 * l + 1, nmax),
            }
        out_blocks.append(entry)
    return {"keys": np.array(keys, dtype=np.int32).reshape(-1, 4), "blocks": out_blocks}
