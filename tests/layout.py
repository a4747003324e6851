"""Golden-data post-processing shared by the tests.

featomic's regression tests reshape the calculator output with metatensor's
``keys_to_samples`` / ``keys_to_properties`` / ``components_to_properties``
before comparing with the stored arrays (``featomic/tests/soap-power-spectrum.rs``,
``featomic/tests/soap-spherical-expansion.rs``).  metatensor is not installed
here, so the same reshaping is restated for the two layouts involved, on the
plain-dict TensorMaps used by the tests:

``{"keys": int32[k, w], "blocks": [{"samples": int32[s, 2],
  "properties": int32[p, w'], "values": float64[...], "gradients": {...}}]}``
"""
import numpy as np


def load_input(path):
    import json
    with open(path) as fd:
        data = json.load(fd)
    systems = []
    for s in data["systems"]:
        systems.append({
            "types": np.array(s["types"], dtype=np.int32),
            "positions": np.array(s["positions"], dtype=np.float64).reshape(-1, 3),
            "cell": np.array(s["cell"], dtype=np.float64).reshape(3, 3),
        })
    return systems, data["hyperparameters"]


def _merged_samples(tm, ct_column):
    """Union of (system, atom, center_type) over all blocks, sorted."""
    rows = set()
    for key, block in zip(tm["keys"], tm["blocks"]):
        for s in block["samples"]:
            rows.add((int(s[0]), int(s[1]), int(key[ct_column])))
    rows = sorted(rows)
    return rows, {r: i for i, r in enumerate(rows)}


def power_spectrum_golden(tm, n_atoms=None):
    """keys_to_samples("center_type") then
    keys_to_properties(["neighbor_1_type", "neighbor_2_type"]).

    Returns ``(values, positions_sum, strain, cell)``; the gradients are None
    when absent.  ``positions_sum`` sums the positions gradient rows per atom
    like the reference's ``sum_gradients`` helper."""
    keys = tm["keys"]
    rows, index = _merged_samples(tm, 0)
    pairs = sorted({(int(k[1]), int(k[2])) for k in keys})
    n_props = tm["blocks"][0]["values"].shape[1]
    offset = {p: i * n_props for i, p in enumerate(pairs)}
    values = np.zeros((len(rows), len(pairs) * n_props))
    grads = tm["blocks"][0]["gradients"]
    positions = strain = cell = None
    if "positions" in grads:
        positions = np.zeros((n_atoms, 3, len(pairs) * n_props))
    if "strain" in grads:
        strain = np.zeros((len(rows), 3, 3, len(pairs) * n_props))
    if "cell" in grads:
        cell = np.zeros((len(rows), 3, 3, len(pairs) * n_props))
    for key, block in zip(keys, tm["blocks"]):
        o = offset[(int(key[1]), int(key[2]))]
        rmap = [index[(int(s[0]), int(s[1]), int(key[0]))] for s in block["samples"]]
        values[rmap, o:o + n_props] = block["values"]
        g = block["gradients"]
        if positions is not None:
            gs = g["positions"]["samples"]
            np.add.at(positions, (gs[:, 2], slice(None), slice(o, o + n_props)), g["positions"]["values"])
        if strain is not None:
            strain[rmap, :, :, o:o + n_props] = g["strain"]["values"]
        if cell is not None:
            cell[rmap, :, :, o:o + n_props] = g["cell"]["values"]
    return values, positions, strain, cell


def spherical_expansion_golden(tm, n_atoms=None):
    """keys_to_samples("center_type"), keys_to_properties("neighbor_type"),
    components_to_properties("o3_mu"), keys_to_properties("o3_lambda").

    Final property order: o3_lambda (slowest), then o3_mu, then
    neighbor_type, then n."""
    keys = tm["keys"]
    rows, index = _merged_samples(tm, 2)
    lambdas = sorted({int(k[0]) for k in keys})
    ntypes = sorted({int(k[3]) for k in keys})
    nmax = tm["blocks"][0]["values"].shape[2]
    # column of (l, m, nt, n) = lstart[l] + (m * n_types + nt_index) * nmax + n
    lstart = {}
    total = 0
    for l in lambdas:
        lstart[l] = total
        total += (2 * l + 1) * len(ntypes) * nmax
    ntindex = {nt: i for i, nt in enumerate(ntypes)}

    def columns(l, nt):
        m = np.arange(2 * l + 1)[:, None]
        n = np.arange(nmax)[None, :]
        return (lstart[l] + (m * len(ntypes) + ntindex[nt]) * nmax + n).reshape(-1)
    values = np.zeros((len(rows), total))
    grads = tm["blocks"][0]["gradients"]
    positions = strain = cell = None
    if "positions" in grads:
        positions = np.zeros((n_atoms, 3, total))
    if "strain" in grads:
        strain = np.zeros((len(rows), 3, 3, total))
    if "cell" in grads:
        cell = np.zeros((len(rows), 3, 3, total))
    for key, block in zip(keys, tm["blocks"]):
        l, nt = int(key[0]), int(key[3])
        cols = columns(l, nt)
        size = (2 * l + 1) * nmax
        rmap = [index[(int(s[0]), int(s[1]), int(key[2]))] for s in block["samples"]]
        v = block["values"].reshape(len(rmap), size)
        values[np.ix_(rmap, cols)] = v
        g = block["gradients"]
        if positions is not None:
            gs = g["positions"]["samples"]
            gv = g["positions"]["values"].reshape(len(gs), 3, size)
            for r, atom in enumerate(gs[:, 2]):
                positions[atom][:, cols] += gv[r]
        if strain is not None:
            sv = g["strain"]["values"].reshape(len(rmap), 3, 3, size)
            for r, row in enumerate(rmap):
                strain[row][:, :, cols] = sv[r]
        if cell is not None:
            cv = g["cell"]["values"].reshape(len(rmap), 3, 3, size)
            for r, row in enumerate(rmap):
                cell[row][:, :, cols] = cv[r]
    return values, positions, strain, cell


def assert_relative_eq(actual, expected, max_relative, epsilon=np.finfo(np.float64).eps):
    """approx::assert_relative_eq semantics: |a - b| <= max(epsilon,
    max_relative * max(|a|, |b|)) element-wise."""
    actual = np.asarray(actual)
    expected = np.asarray(expected)
    assert actual.shape == expected.shape, (actual.shape, expected.shape)
    diff = np.abs(actual - expected)
    bound = np.maximum(epsilon, max_relative * np.maximum(np.abs(actual), np.abs(expected)))
    bad = diff > bound
    if bad.any():
        idx = np.argwhere(bad)[:5]
        worst = np.max(diff / np.maximum(np.abs(expected), 1e-300))
        raise AssertionError(
            f"{bad.sum()} / {bad.size} elements differ beyond rel {max_relative}; first at {idx.tolist()}: "
            f"{actual[tuple(idx[0])]} vs {expected[tuple(idx[0])]} (worst rel {worst:.3e})"
        )
