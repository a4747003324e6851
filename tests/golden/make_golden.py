"""Regenerate the golden fixtures in this directory from the featomic sources.

featomic (formerly rascaline) ships reference data for the SOAP path in
``featomic/tests/data/generated/`` (gzip'd ``.npy`` arrays plus the JSON inputs
that produced them, rounded to 10 significant digits by
``featomic/tests/data/save_data.py:53-89``) and a handful of known answers
written inline in its Rust unit tests. This script reads both, as data, and
stores them here so that the test-suite is self-contained on machines where the
featomic sources are absent.

Usage::

    python tests/golden/make_golden.py /path/to/featomic-checkout

Outputs (all committed):

* ``<name>-input.json``          the calculator inputs, copied verbatim
* ``<name>.npz``                 the expected arrays (key ``values``)
* ``lode-exponent-<p>-<name>``   the LODE spherical expansion fixtures of
  ``generated/lode-spherical-expansion/exponent-<p>/`` (p = 1..6)
* ``known_answers.json``         inline known answers, extracted by regex from
  ``math/hyp1f1.rs`` (mpmath table), ``calculators/soap/cutoff.rs`` (shifted
  cosine values), ``systems/neighbors.rs`` (ASE neighbour distances),
  ``math/gamma.rs`` (gamma / ln_gamma spot values), ``math/exp.rs`` (scipy
  exp1 / expi values) and ``calculators/lode/radial_integral/gto.rs``
  (pyLODE central-atom contributions).
"""
import gzip
import io
import json
import os
import re
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

GENERATED = [
    "soap-power-spectrum-values",
    "soap-power-spectrum-positions-gradient",
    "soap-power-spectrum-strain-gradient",
    "soap-power-spectrum-cell-gradient",
    "spherical-expansion-values",
    "spherical-expansion-pbc-values",
    "spherical-expansion-positions-gradient",
    "spherical-expansion-strain-gradient",
    "spherical-expansion-cell-gradient",
    "spherical-harmonics-values",
]

INPUTS = [
    "soap-power-spectrum-values-input.json",
    "soap-power-spectrum-gradients-input.json",
    "spherical-expansion-values-input.json",
    "spherical-expansion-pbc-values-input.json",
    "spherical-expansion-gradients-input.json",
    "spherical-harmonics-input.json",
]

_FLOAT = r"[-+]?(?:\d+\.\d*|\.\d+|\d+)(?:[eE][-+]?\d+)?"


def _read(root, rel):
    with open(os.path.join(root, rel)) as fd:
        return fd.read()


def extract_hyp1f1(src):
    """ALL_Z and the (n, l) -> values table of `math/hyp1f1.rs` tests."""
    z_block = re.search(r"static ALL_Z: \[f64; \d+\] = \[(.*?)\];", src, re.S).group(1)
    all_z = [float(v) for v in re.findall(_FLOAT, z_block)]
    table = []
    for n, l, body in re.findall(r"\(\((\d+), (\d+)\), \[(.*?)\]\)", src, re.S):
        table.append({"n": int(n), "l": int(l),
                      "values": [float(v) for v in re.findall(_FLOAT, body)]})
    return {"z": all_z, "table": table}


def extract_cutoff(src):
    """`shifted_cosine` test of `calculators/soap/cutoff.rs`."""
    body = src[src.index("fn shifted_cosine"):]
    radius = float(re.search(r"radius: (" + _FLOAT + ")", body).group(1))
    width = float(re.search(r"width: (" + _FLOAT + ")", body).group(1))
    values = [(float(a), float(b)) for a, b in
              re.findall(r"cutoff\.smoothing\((" + _FLOAT + r")\), (" + _FLOAT + r")\)", body)]
    grads = [(float(a), float(b)) for a, b in
             re.findall(r"cutoff\.smoothing_gradient\((" + _FLOAT + r")\), (" + _FLOAT + r")\)", body)]
    return {"radius": radius, "width": width, "smoothing": values, "gradient": grads}


def extract_neighbors(src):
    """`non_periodic` test of `systems/neighbors.rs` (ASE distances)."""
    body = src[src.index("fn non_periodic"):src.index("fn fcc_cell")]
    pos_block = body[body.index("let positions"):body.index("];")]
    positions = [[float(v) for v in re.findall(_FLOAT, row)]
                 for row in re.findall(r"Vector3D::new\((.*?)\)", pos_block)]
    cutoff = float(re.search(r"UnitCell::infinite\(\), (" + _FLOAT + r")\)", body).group(1))
    ref_block = body[body.index("let reference"):]
    ref_block = ref_block[:ref_block.index("];")]
    pairs = [[int(a), int(b), float(c)] for a, b, c in
             re.findall(r"\((\d+), (\d+), (" + _FLOAT + r")\)", ref_block)]
    return {"positions": positions, "cutoff": cutoff, "pairs": pairs}


def extract_gamma(src):
    """`assert_relative_eq!(gamma(...), value)` spot values of `math/gamma.rs`."""
    out = {"gamma": [], "ln_gamma": []}
    consts = {
        "std::f64::consts::PI / 2.0": np.pi / 2.0, "f64::consts::PI/2.0": np.pi / 2.0,
        "std::f64::consts::PI": np.pi, "f64::consts::PI": np.pi,
    }
    for fn in ("gamma", "ln_gamma"):
        pat = r"assert_relative_eq!\(" + fn + r"\(([^()]*?)\), (" + _FLOAT + r")"
        for arg, expected in re.findall(pat, src):
            arg = arg.strip()
            if arg in consts:
                x = consts[arg]
            else:
                try:
                    x = float(arg)
                except ValueError:
                    continue
            out[fn].append([x, float(expected)])
    return out


def extract_exp(src):
    """scipy reference values of `math/exp.rs` tests: [x, expected] pairs for
    exp1 and expi (finite expected values only)."""
    out = {}
    for fn in ("exp1", "expi"):
        pat = r"assert_relative_eq!\(" + fn + r"\((" + _FLOAT + r")\), (" + _FLOAT + r")"
        out[fn] = [[float(a), float(b)] for a, b in re.findall(pat, src)]
    return out


def extract_lode_center(src):
    """`central_atom_contribution` test of `lode/radial_integral/gto.rs`:
    exponents, GTO (max_radial, radius), smearing and the pyLODE values."""
    body = src[src.index("fn central_atom_contribution"):]
    exponents = [int(v) for v in re.search(r"potential_exponents = \[(.*?)\]", body).group(1).split(",")]
    start = body.index("let reference_vals")
    block = body[start:body.index("]];", start) + 1]
    rows = [[float(v) for v in re.findall(_FLOAT, row)] for row in re.findall(r"\[([^\[\]]+)\]", block)]
    m = re.search(r"max_radial: (\d+), radius: (" + _FLOAT + r")", body)
    smearing = float(re.search(r"smearing: (" + _FLOAT + r")", body).group(1))
    return {"exponents": exponents, "values": rows, "max_radial": int(m.group(1)), "radius": float(m.group(2)),
            "smearing": smearing}


LODE = ["values-input.json", "values.npy.gz", "gradients-input.json", "positions-gradient.npy.gz"]


def main(root):
    generated = os.path.join(root, "featomic", "tests", "data", "generated")
    for name in INPUTS:
        shutil.copyfile(os.path.join(generated, name), os.path.join(HERE, name))
    for name in GENERATED:
        with gzip.open(os.path.join(generated, name + ".npy.gz"), "rb") as fd:
            array = np.load(io.BytesIO(fd.read()))
        np.savez_compressed(os.path.join(HERE, name + ".npz"), values=array)

    for p in range(1, 7):
        folder = os.path.join(generated, "lode-spherical-expansion", f"exponent-{p}")
        for name in LODE:
            target = os.path.join(HERE, f"lode-exponent-{p}-{name}")
            if name.endswith(".json"):
                shutil.copyfile(os.path.join(folder, name), target)
            else:
                with gzip.open(os.path.join(folder, name), "rb") as fd:
                    array = np.load(io.BytesIO(fd.read()))
                np.savez_compressed(target.replace(".npy.gz", ".npz"), values=array)

    src = os.path.join(root, "featomic", "src")
    known = {
        "hyp1f1": extract_hyp1f1(_read(src, "math/hyp1f1.rs")),
        "cutoff": extract_cutoff(_read(src, "calculators/soap/cutoff.rs")),
        "neighbors_non_periodic": extract_neighbors(_read(src, "systems/neighbors.rs")),
        "gamma": extract_gamma(_read(src, "math/gamma.rs")),
        "exp": extract_exp(_read(src, "math/exp.rs")),
        "lode_center": extract_lode_center(_read(src, "calculators/lode/radial_integral/gto.rs")),
        "sources": {
            "hyp1f1": "featomic/src/math/hyp1f1.rs:263-288",
            "cutoff": "featomic/src/calculators/soap/cutoff.rs:97-112",
            "neighbors_non_periodic": "featomic/src/systems/neighbors.rs:413-444",
            "gamma": "featomic/src/math/gamma.rs:330-390",
            "exp": "featomic/src/math/exp.rs:69-95",
            "lode_center": "featomic/src/calculators/lode/radial_integral/gto.rs:261-286",
        },
    }
    with open(os.path.join(HERE, "known_answers.json"), "w") as fd:
        json.dump(known, fd, indent=1)
        fd.write("\n")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py /path/to/featomic-checkout")
    main(sys.argv[1])
