"""TEST INFRASTRUCTURE -- ctypes front-end of the CPU oracle (soap_oracle.cpp).

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU legs import this
module, as the checker or the timed CPU baseline.  The product
(``rascaline_b200``) never does.

The oracle restates featomic's SOAP path on the CPU in FP64; see the header of
``soap_oracle.cpp`` for what it follows and how it is pinned.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "liboracle_soap.so")
SOURCE = os.path.join(HERE, "soap_oracle.cpp")


def build(force=False):
    """Compile the oracle with g++ (no FMA contraction, like rustc)."""
    if not force and os.path.exists(LIBRARY) and os.path.getmtime(LIBRARY) >= os.path.getmtime(SOURCE):
        return LIBRARY
    cmd = [
        "g++", "-O3", "-std=c++17", "-fPIC", "-shared", "-fopenmp",
        "-ffp-contract=off", "-fno-fast-math", SOURCE, "-o", LIBRARY,
    ]
    subprocess.check_call(cmd)
    return LIBRARY


class Hypers(ctypes.Structure):
    _fields_ = [
        ("cutoff", ctypes.c_double),
        ("smoothing", ctypes.c_int32),
        ("smoothing_width", ctypes.c_double),
        ("density_width", ctypes.c_double),
        ("center_atom_weight", ctypes.c_double),
        ("scaling", ctypes.c_int32),
        ("scaling_scale", ctypes.c_double),
        ("scaling_rate", ctypes.c_double),
        ("scaling_exponent", ctypes.c_double),
        ("max_angular", ctypes.c_int32),
        ("max_radial", ctypes.c_int32),
        ("spline_accuracy", ctypes.c_double),
    ]


class System(ctypes.Structure):
    _fields_ = [
        ("n_atoms", ctypes.c_uint64),
        ("types", ctypes.POINTER(ctypes.c_int32)),
        ("positions", ctypes.POINTER(ctypes.c_double)),
        ("cell", ctypes.c_double * 9),
    ]


_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY):
            build()
        L = ctypes.CDLL(LIBRARY)
        c = ctypes
        P = c.POINTER
        L.oracle_last_error.restype = c.c_char_p
        L.oracle_gamma.restype = c.c_double
        L.oracle_gamma.argtypes = [c.c_double]
        L.oracle_ln_gamma.restype = c.c_double
        L.oracle_ln_gamma.argtypes = [c.c_double]
        L.oracle_hyp1f1.argtypes = [c.c_double, c.c_double, c.c_double, P(c.c_double)]
        L.oracle_cutoff.argtypes = [P(Hypers), c.c_double, P(c.c_double), P(c.c_double)]
        L.oracle_spherical_harmonics.argtypes = [c.c_int32, P(c.c_double)] + [P(c.c_double)] * 4
        L.oracle_radial_integral.argtypes = [P(Hypers), c.c_int32, P(c.c_double), P(c.c_double), P(c.c_double)]
        L.oracle_spline_sizes.argtypes = [P(Hypers), P(c.c_int32)]
        L.oracle_gto_orthonormalization.argtypes = [c.c_int32, c.c_double, P(c.c_double)]
        L.oracle_neighbors.argtypes = [P(c.c_double), c.c_uint64, P(c.c_double), c.c_double,
                                       P(c.c_void_p), P(c.c_uint64)]
        L.oracle_neighbors_get.argtypes = [c.c_void_p, P(c.c_int64), P(c.c_double), P(c.c_double), P(c.c_int32)]
        L.oracle_neighbors_free.argtypes = [c.c_void_p]
        L.oracle_compute.argtypes = [c.c_int32, P(Hypers), P(System), c.c_uint64, c.c_int32, c.c_int32,
                                     c.c_int32, c.c_int32, c.c_int32, P(c.c_void_p)]
        L.oracle_result_free.argtypes = [c.c_void_p]
        L.oracle_result_n_blocks.argtypes = [c.c_void_p]
        L.oracle_result_n_blocks.restype = c.c_uint64
        L.oracle_result_keys.argtypes = [c.c_void_p, P(P(c.c_int32)), P(c.c_uint64), P(c.c_uint64)]
        L.oracle_block_labels.argtypes = [c.c_void_p, c.c_uint64, c.c_char_p, c.c_int32,
                                          P(P(c.c_int32)), P(c.c_uint64), P(c.c_uint64)]
        L.oracle_block_values.argtypes = [c.c_void_p, c.c_uint64, c.c_char_p, P(P(c.c_double)),
                                          P(P(c.c_uint64)), P(c.c_uint64)]
        _LIB = L
    return _LIB


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(status):
    if status != 0:
        raise RuntimeError(lib().oracle_last_error().decode())


def hypers_from_json(h):
    """featomic SOAP hyper-parameters (dict) -> oracle struct."""
    out = Hypers()
    out.cutoff = float(h["cutoff"]["radius"])
    smoothing = h["cutoff"]["smoothing"]
    if smoothing["type"] == "ShiftedCosine":
        out.smoothing = 0
        out.smoothing_width = float(smoothing["width"])
    elif smoothing["type"] == "Step":
        out.smoothing = 1
        out.smoothing_width = 0.0
    else:
        raise ValueError(smoothing)
    density = h["density"]
    assert density["type"] == "Gaussian"
    out.density_width = float(density["width"])
    out.center_atom_weight = float(density.get("center_atom_weight", 1.0))
    scaling = density.get("scaling")
    if scaling:
        assert scaling["type"] == "Willatt2018"
        out.scaling = 1
        out.scaling_scale = float(scaling["scale"])
        out.scaling_rate = float(scaling["rate"])
        out.scaling_exponent = float(scaling["exponent"])
    basis = h["basis"]
    if "type" in basis:
        assert basis["type"] == "TensorProduct" and basis["radial"]["type"] == "Gto"
        out.max_angular = int(basis["max_angular"])
    else:
        # RadialSpectrumBasis (featomic/src/calculators/soap/radial_spectrum.rs:44-57)
        assert basis["radial"]["type"] == "Gto"
        out.max_angular = 0
    out.max_radial = int(basis["radial"]["max_radial"])
    acc = basis.get("spline_accuracy", 1e-8)
    out.spline_accuracy = -1.0 if acc is None else float(acc)
    return out


def gamma(x):
    return lib().oracle_gamma(x)


def ln_gamma(x):
    return lib().oracle_ln_gamma(x)


def hyp1f1(a, b, x):
    out = ctypes.c_double()
    _check(lib().oracle_hyp1f1(a, b, x, ctypes.byref(out)))
    return out.value


def cutoff_function(hypers, r):
    h = hypers_from_json(hypers)
    v, g = ctypes.c_double(), ctypes.c_double()
    lib().oracle_cutoff(ctypes.byref(h), r, ctypes.byref(v), ctypes.byref(g))
    return v.value, g.value


def spherical_harmonics(lmax, direction, gradients=False):
    d = np.ascontiguousarray(direction, dtype=np.float64)
    n = (lmax + 1) ** 2
    values = np.zeros(n)
    if gradients:
        g = np.zeros((3, n))
        _check(lib().oracle_spherical_harmonics(lmax, _dptr(d), _dptr(values), _dptr(g[0]), _dptr(g[1]), _dptr(g[2])))
        return values, g
    null = ctypes.POINTER(ctypes.c_double)()
    _check(lib().oracle_spherical_harmonics(lmax, _dptr(d), _dptr(values), null, null, null))
    return values


def radial_integral(hypers, r):
    """(values, gradients) of shape [len(r), max_angular+1, max_radial+1]."""
    h = hypers_from_json(hypers)
    r = np.ascontiguousarray(r, dtype=np.float64)
    shape = (len(r), h.max_angular + 1, h.max_radial + 1)
    v = np.zeros(shape)
    g = np.zeros(shape)
    _check(lib().oracle_radial_integral(ctypes.byref(h), len(r), _dptr(r), _dptr(v), _dptr(g)))
    return v, g


def spline_sizes(hypers):
    h = hypers_from_json(hypers)
    out = np.zeros(h.max_angular + 1, dtype=np.int32)
    _check(lib().oracle_spline_sizes(ctypes.byref(h), out.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
    return out


def gto_orthonormalization(size, radius):
    out = np.zeros((size, size))
    _check(lib().oracle_gto_orthonormalization(size, radius, _dptr(out)))
    return out


def neighbors(positions, cell, cutoff):
    """Half neighbour list: dict(first, second, distance, vector, shift)."""
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    cell = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    handle = ctypes.c_void_p()
    count = ctypes.c_uint64()
    _check(lib().oracle_neighbors(_dptr(pos), len(pos), _dptr(cell), cutoff, ctypes.byref(handle), ctypes.byref(count)))
    n = count.value
    pairs = np.zeros((n, 2), dtype=np.int64)
    dist = np.zeros(n)
    vec = np.zeros((n, 3))
    shift = np.zeros((n, 3), dtype=np.int32)
    lib().oracle_neighbors_get(handle, pairs.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), _dptr(dist),
                               _dptr(vec), shift.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
    lib().oracle_neighbors_free(handle)
    return {"first": pairs[:, 0], "second": pairs[:, 1], "distance": dist, "vector": vec, "shift": shift}


def _labels(res, b, gradient, axis):
    ptr = ctypes.POINTER(ctypes.c_int32)()
    count, width = ctypes.c_uint64(), ctypes.c_uint64()
    _check(lib().oracle_block_labels(res, b, gradient, axis, ctypes.byref(ptr), ctypes.byref(count), ctypes.byref(width)))
    if count.value == 0:
        return np.zeros((0, width.value), dtype=np.int32)
    return np.ctypeslib.as_array(ptr, shape=(count.value, width.value)).copy()


def _values(res, b, gradient):
    ptr = ctypes.POINTER(ctypes.c_double)()
    shape = ctypes.POINTER(ctypes.c_uint64)()
    ndim = ctypes.c_uint64()
    _check(lib().oracle_block_values(res, b, gradient, ctypes.byref(ptr), ctypes.byref(shape), ctypes.byref(ndim)))
    shp = tuple(shape[i] for i in range(ndim.value))
    size = int(np.prod(shp))
    if size == 0:
        return np.zeros(shp)
    return np.ctypeslib.as_array(ptr, shape=(size,)).reshape(shp).copy()


def compute(calculator, hypers, systems, gradients=(), threads=1, se_over_centres=False):
    """Run the oracle.  ``systems`` is a list of dicts with ``types``
    (int32[n]), ``positions`` (float64[n, 3]) and ``cell`` (float64[3, 3]).

    Returns ``{"keys": int32[k, w], "blocks": [{"samples", "properties",
    "values", "gradients": {name: {"samples", "values"}}}]}``."""
    if calculator == "soap_radial_spectrum":
        return _radial_spectrum(compute("spherical_expansion", hypers, systems, gradients, threads, se_over_centres))
    kind = {"spherical_expansion": 0, "soap_power_spectrum": 1, "spherical_expansion_by_pair": 2}[calculator]
    h = hypers_from_json(hypers)
    keep = []
    arr = (System * len(systems))()
    for k, s in enumerate(systems):
        t = np.ascontiguousarray(s["types"], dtype=np.int32)
        p = np.ascontiguousarray(s["positions"], dtype=np.float64).reshape(-1, 3)
        c = np.ascontiguousarray(s["cell"], dtype=np.float64).reshape(9)
        keep += [t, p]
        arr[k].n_atoms = len(t)
        arr[k].types = t.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        arr[k].positions = _dptr(p)
        for x in range(9):
            arr[k].cell[x] = c[x]
    res = ctypes.c_void_p()
    _check(lib().oracle_compute(kind, ctypes.byref(h), arr, len(systems), int("positions" in gradients),
                                int("strain" in gradients), int("cell" in gradients), int(threads),
                                int(se_over_centres), ctypes.byref(res)))
    try:
        kptr = ctypes.POINTER(ctypes.c_int32)()
        count, width = ctypes.c_uint64(), ctypes.c_uint64()
        lib().oracle_result_keys(res, ctypes.byref(kptr), ctypes.byref(count), ctypes.byref(width))
        keys = np.ctypeslib.as_array(kptr, shape=(count.value, width.value)).copy()
        blocks = []
        for b in range(lib().oracle_result_n_blocks(res)):
            block = {
                "samples": _labels(res, b, None, 0),
                "properties": _labels(res, b, None, 1),
                "values": _values(res, b, None),
                "gradients": {},
            }
            for g in gradients:
                name = g.encode()
                block["gradients"][g] = {
                    "samples": _labels(res, b, name, 0),
                    "values": _values(res, b, name),
                }
            blocks.append(block)
    finally:
        lib().oracle_result_free(res)
    return {"keys": keys, "blocks": blocks}


def _radial_spectrum(se):
    """featomic's SoapRadialSpectrum::compute (featomic/src/calculators/soap/
    radial_spectrum.rs:237-323): the spherical expansion restricted to the
    l = 0 radial basis, keys (center_type, neighbor_type) and the o3_mu axis
    (size 1) dropped from values and gradients."""
    assert (se["keys"][:, 0] == 0).all()
    out = {"keys": np.ascontiguousarray(se["keys"][:, 2:4]), "blocks": []}
    for block in se["blocks"]:
        values = block["values"]
        new = {"samples": block["samples"], "properties": block["properties"],
               "values": values.reshape(values.shape[0], values.shape[2]), "gradients": {}}
        for name, g in block["gradients"].items():
            v = g["values"]
            assert v.shape[-2] == 1
            new["gradients"][name] = {"samples": g["samples"], "values": v.reshape(v.shape[:-2] + v.shape[-1:])}
        out["blocks"].append(new)
    return out
