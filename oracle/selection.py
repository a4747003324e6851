"""TEST INFRASTRUCTURE -- featomic's labels selections restated on the
oracle's full output.

Only tests/ import this module, as the checker of the library's selections.

What it restates:

* keys (featomic/src/calculator.rs:287-307): an empty selection is an error;
  the calculator's key names: exactly these keys, in this order; fewer
  names: the default keys matching any row of the selection;
* samples and properties, ``LabelsSelection::select``
  (calculator.rs:71-158): ``Subset`` keeps, per block, the default entries
  whose values on the selection's names equal a row of the selection, in
  default order (metatensor's ``Labels::select``); ``Predefined`` takes, per
  key, the labels of the predefined TensorMap's block with that key;
* positions gradient samples of the selected samples, built from the
  neighbour list (featomic/src/labels/samples/atom_centered.rs:103-147,
  ``AtomCenteredSamples::gradients_for`` with self pairs): per sample, the
  atoms of the key's neighbour types within the cutoff, plus the centre when
  one of them matched or its own type is a neighbour type, by atom index;
  strain / cell gradients: one row per sample (calculator.rs:339-382);
* values: featomic computes only the selected entries, and an entry's value
  does not depend on what else is computed, so a selected entry equals the
  full calculation's entry; a predefined sample the full calculation does
  not produce (a centre without neighbours of one of the key's neighbour
  types: its expansion coefficients for that type vanish) is zero, values
  and gradients;
* errors with featomic's messages: an unknown name in a selection
  (calculator.rs:47-67), predefined key names, a key missing from the
  predefined TensorMap, predefined label names (calculator.rs:110-152).

Selections are given as ``("subset", names, values)`` or
``("predefined", {key tuple: (names, values)}, key_names)``.
"""
import numpy as np

from . import oracle

SAMPLE_NAMES = ["system", "atom"]
KEY_NAMES = {
    "spherical_expansion": ["o3_lambda", "o3_sigma", "center_type", "neighbor_type"],
    "soap_power_spectrum": ["center_type", "neighbor_1_type", "neighbor_2_type"],
    "soap_radial_spectrum": ["center_type", "neighbor_type"],
}
PROPERTY_NAMES = {
    "spherical_expansion": ["n"],
    "soap_power_spectrum": ["l", "n_1", "n_2"],
    "soap_radial_spectrum": ["n"],
}


class SelectionError(ValueError):
    pass


def _labels_select(names, values, sel_names, sel_values, kind):
    """metatensor Labels::select: indices of the entries matching any row of
    the selection on the selection's names (calculator.rs:94-108)."""
    for name in sel_names:
        if name not in names:
            raise SelectionError(f"'{name}' in {kind} selection is not part of the {kind} of this calculator")
    cols = [names.index(n) for n in sel_names]
    wanted = {tuple(int(x) for x in row) for row in np.asarray(sel_values).reshape(-1, len(sel_names))}
    return [i for i, row in enumerate(values) if tuple(int(row[c]) for c in cols) in wanted]


def _predefined(selection, keys, key_names, names, kind):
    _, blocks, predefined_key_names = selection
    if list(predefined_key_names) != list(key_names):
        raise SelectionError(f"invalid key names in predefined {kind}: expected [{','.join(key_names)}], "
                             f"but got [{', '.join(predefined_key_names)}]")
    out = []
    for key in keys:
        key = tuple(int(x) for x in key)
        if key not in blocks:
            printed = ", ".join(f"{n}={v}" for n, v in zip(key_names, key))
            raise SelectionError(f"expected a block for ({printed}) in predefined {kind} selection")
        block_names, block_values = blocks[key]
        if list(block_names) != list(names):
            raise SelectionError(f"invalid predefined {kind} names: expected [{', '.join(names)}], "
                                 f"but got [{', '.join(block_names)}]")
        out.append(np.asarray(block_values, dtype=np.int32).reshape(-1, len(names)))
    return out


def _neighbours(systems, cutoff):
    around = []
    for s in systems:
        nl = oracle.neighbors(s["positions"], s["cell"], cutoff)
        lists = [[] for _ in range(len(s["types"]))]
        for i, j in zip(nl["first"], nl["second"]):
            lists[i].append(int(j))
            lists[j].append(int(i))
        around.append(lists)
    return around


def _gradient_atoms(types, around, atom, neighbour_types):
    atoms = set()
    if int(types[atom]) in neighbour_types:
        atoms.add(atom)
    for j in around[atom]:
        if int(types[j]) in neighbour_types:
            atoms.add(j)
            atoms.add(atom)
    return sorted(atoms)


def select(calculator, full, systems, cutoff, gradients=(), keys=None, samples=None, properties=None):
    """The output featomic gives for these selections, from the oracle's full
    output ``full`` (oracle.compute of ``calculator`` on ``systems`` with
    ``gradients``).  Same dict layout as oracle.compute, with the label names
    added (``key_names``, and per block ``sample_names``,
    ``property_names``)."""
    key_names = KEY_NAMES[calculator]
    property_names = PROPERTY_NAMES[calculator]
    default_keys = [tuple(int(x) for x in k) for k in full["keys"]]
    by_key = dict(zip(default_keys, full["blocks"]))

    # keys (calculator.rs:287-307)
    if keys is None:
        out_keys = default_keys
    else:
        names, values = keys
        values = np.asarray(values, dtype=np.int32).reshape(-1, len(names))
        if len(values) == 0:
            raise SelectionError("selected keys can not be empty")
        if list(names) == key_names:
            out_keys = [tuple(int(x) for x in row) for row in values]
        else:
            out_keys = [default_keys[i] for i in _labels_select(key_names, default_keys, names, values, "keys")]

    neighbour_columns = [key_names.index(n) for n in key_names if n.startswith("neighbor")]
    around = _neighbours(systems, cutoff) if "positions" in gradients else None
    result = {"keys": np.array(out_keys, dtype=np.int32).reshape(-1, len(key_names)), "key_names": key_names,
              "blocks": []}
    selected_samples = (_predefined(samples, out_keys, key_names, SAMPLE_NAMES, "samples")
                        if samples is not None and samples[0] == "predefined" else None)
    selected_properties = (_predefined(properties, out_keys, key_names, property_names, "properties")
                           if properties is not None and properties[0] == "predefined" else None)
    for k, key in enumerate(out_keys):
        block = by_key.get(key)
        default_samples = block["samples"] if block is not None else np.zeros((0, 2), dtype=np.int32)
        if block is not None:
            default_properties = block["properties"]
        else:
            default_properties = full["blocks"][0]["properties"]
        # samples (calculator.rs:71-158)
        if samples is None:
            sample_values = default_samples
        elif samples[0] == "subset":
            rows = _labels_select(SAMPLE_NAMES, default_samples, samples[1], samples[2], "samples")
            sample_values = default_samples[rows]
        else:
            sample_values = selected_samples[k]
        # properties
        if properties is None:
            prop_values = default_properties
        elif properties[0] == "subset":
            prop_values = default_properties[_labels_select(property_names, default_properties, properties[1],
                                                            properties[2], "properties")]
        else:
            prop_values = selected_properties[k]
        prop_index = {tuple(int(x) for x in p): i for i, p in enumerate(default_properties)}
        cols = []
        for p in prop_values:
            if tuple(int(x) for x in p) not in prop_index:
                raise SelectionError("predefined properties selection contains an entry outside of this "
                                     "calculator's properties")
            cols.append(prop_index[tuple(int(x) for x in p)])
        sample_index = {tuple(int(x) for x in s): i for i, s in enumerate(default_samples)}

        middle = (block["values"].shape[1:-1] if block is not None
                  else ((2 * key[0] + 1,) if calculator == "spherical_expansion" else ()))
        values = np.zeros((len(sample_values),) + middle + (len(cols),))
        for r, s in enumerate(sample_values):
            old = sample_index.get(tuple(int(x) for x in s))
            if old is not None:
                values[r] = block["values"][old][..., cols]
        out = {"samples": np.asarray(sample_values, dtype=np.int32).reshape(-1, 2), "sample_names": SAMPLE_NAMES,
               "properties": np.asarray(prop_values, dtype=np.int32).reshape(-1, len(property_names)),
               "property_names": property_names, "values": values, "gradients": {}}

        for name in gradients:
            if name == "positions":
                neighbour_types = {key[c] for c in neighbour_columns}
                g_samples, g_values = [], []
                full_rows = {}
                if block is not None:
                    fg = block["gradients"]["positions"]
                    for r, gs in enumerate(fg["samples"]):
                        full_rows[(int(gs[0]), int(gs[1]), int(gs[2]))] = fg["values"][r]
                for r, (system, atom) in enumerate(sample_values):
                    types = systems[system]["types"]
                    old = sample_index.get((int(system), int(atom)))
                    for a in _gradient_atoms(types, around[system], int(atom), neighbour_types):
                        g_samples.append((r, int(system), a))
                        row = full_rows.get((old, int(system), a)) if old is not None else None
                        g_values.append(row[..., cols] if row is not None else np.zeros((3,) + middle + (len(cols),)))
                shape = (len(g_samples), 3) + middle + (len(cols),)
                out["gradients"][name] = {
                    "samples": np.array(g_samples, dtype=np.int32).reshape(-1, 3),
                    "values": np.array(g_values).reshape(shape),
                }
            else:
                shape = (len(sample_values), 3, 3) + middle + (len(cols),)
                gvalues = np.zeros(shape)
                for r, s in enumerate(sample_values):
                    old = sample_index.get(tuple(int(x) for x in s))
                    if old is not None:
                        gvalues[r] = block["gradients"][name]["values"][old][..., cols]
                out["gradients"][name] = {"samples": np.arange(len(sample_values), dtype=np.int32).reshape(-1, 1),
                                          "values": gvalues}
        result["blocks"].append(out)
    return result
