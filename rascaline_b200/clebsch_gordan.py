"""Clebsch-Gordan tensor products and the equivariant power spectrum on the GPU.

Mirrors featomic's ``featomic.clebsch_gordan`` Python module
(python/featomic/featomic/clebsch_gordan/): ``ClebschGordanProduct``
(_cg_product.py:29-436) and ``EquivariantPowerSpectrum``
(_equivariant_power_spectrum.py:23-365, "lambda-SOAP").  The coefficients
come from ``featomic_b200_cg_coefficients`` and every block product runs in
one launch of the sm_100a kernel behind ``featomic_b200_cg_product``; the
key / sample / property bookkeeping (metatensor operations in featomic) is
done here, on the host.  Values live in torch CUDA tensors.
"""
import ctypes
import json

import numpy as np

from . import _c_api as C
from .calculators import Labels


def cg_coefficients(l1, l2, o3_lambda):
    """Real CG coefficients [2 l1 + 1, 2 l2 + 1, 2 o3_lambda + 1]
    (_coefficients.py:137-224)."""
    out = np.zeros(max(1, (2 * l1 + 1) * (2 * l2 + 1) * (2 * o3_lambda + 1)))
    C.check(C.lib().featomic_b200_cg_coefficients(l1, l2, o3_lambda,
                                                  out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), out.size))
    return out.reshape(2 * l1 + 1, 2 * l2 + 1, 2 * o3_lambda + 1)


CG_BACKENDS = ("python-dense", "python-sparse")


def _check_cg_backend(cg_backend):
    if cg_backend not in CG_BACKENDS:
        raise ValueError(f"invalid `cg_backend`, got '{cg_backend}', only 'python-dense', or 'python-sparse' are "
                         "supported")


def calculate_cg_coefficients(lambda_max, cg_backend, arrays_backend, dtype, device):
    """The real Clebsch-Gordan coefficients of every (l1, l2, lambda) with
    l1, l2 <= lambda_max and |l1 - l2| <= lambda <= min(lambda_max, l1 + l2),
    in featomic's cache layout (_coefficients.py:35-134, 225-335): keys
    (l1, l2, lambda); "python-dense" blocks [1, 2 l1 + 1, 2 l2 + 1, 2 lambda + 1,
    1] with components m1, m2, mu; "python-sparse" blocks [n, 1] of the
    non-zero coefficients with samples (m1, m2, mu).  ``arrays_backend`` is
    "numpy" or "torch".  This library's own products take their coefficients
    from the GPU directly, so the cache is only for callers that read it."""
    _check_cg_backend(cg_backend)
    if arrays_backend == "torch":
        import torch

        if dtype not in (torch.float32, torch.float64):
            raise ValueError(f"invalid dtype ({dtype}), only torch.float32 and torch.float64 are supported")
        convert = lambda a: torch.as_tensor(a, dtype=dtype, device=device)  # noqa: E731
    elif arrays_backend == "numpy":
        if np.dtype(dtype) not in (np.float32, np.float64):
            raise ValueError(f"invalid dtype ({dtype}), only np.float32 and np.float64 are supported")
        convert = lambda a: np.ascontiguousarray(a, dtype=dtype)  # noqa: E731
    else:
        raise ValueError(f"invalid arrays_backend '{arrays_backend}', only 'numpy' and 'torch' are supported")
    keys, blocks = [], []
    for l1 in range(lambda_max + 1):
        for l2 in range(lambda_max + 1):
            for lam in range(abs(l1 - l2), min(lambda_max, l1 + l2) + 1):
                dense = cg_coefficients(l1, l2, lam)
                keys.append([l1, l2, lam])
                if cg_backend == "python-dense":
                    comps = [Labels([name], np.arange(n, dtype=np.int32).reshape(-1, 1))
                             for name, n in zip(("m1", "m2", "mu"), dense.shape)]
                    blocks.append(Block(convert(dense.reshape((1,) + dense.shape + (1,))), Labels(["_"], [[0]]),
                                        comps, Labels(["cg_coefficient"], [[0]])))
                else:
                    nonzero = np.argwhere(np.abs(dense) > 1e-15)
                    values = dense[tuple(nonzero.T)].reshape(-1, 1)
                    blocks.append(Block(convert(values), Labels(["m1", "m2", "mu"], nonzero.astype(np.int32)), [],
                                        Labels(["cg_coefficient"], [[0]])))
    return EquivariantTensorMap(Labels(["l1", "l2", "lambda"], np.array(keys, dtype=np.int32)), blocks)


def cg_tensor_products(tasks, stream=None):
    """Run ``(first, second, output, o3_lambda)`` products (contiguous CUDA
    tensors of one dtype, shapes [s, 2 l1 + 1, p], [s, 2 l2 + 1, q],
    [s, 2 o3_lambda + 1, p * q]) in one launch.  A task
    ``(first, second, output, o3_lambda, column)`` writes into the columns
    ``column .. column + p * q`` of a wider output [s, 2 o3_lambda + 1, w]."""
    import torch

    if not tasks:
        return
    dtype = tasks[0][0].dtype
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("Clebsch-Gordan products take float32 or float64 tensors")
    arr = (C.featomic_b200_cg_task_t * len(tasks))()
    for k, task in enumerate(tasks):
        a, b, out, lam = task[:4]
        column = task[4] if len(task) > 4 else None
        for t in (a, b, out):
            if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
                raise ValueError("Clebsch-Gordan tensors must be contiguous CUDA tensors of one dtype")
        s, m1, p = a.shape
        _, m2, q = b.shape
        if column is None:
            if b.shape[0] != s or tuple(out.shape) != (s, 2 * lam + 1, p * q):
                raise ValueError("inconsistent shapes in a Clebsch-Gordan product")
            ptr, stride = out.data_ptr(), 0
        else:
            if b.shape[0] != s or tuple(out.shape[:2]) != (s, 2 * lam + 1) or column < 0 or \
                    column + p * q > out.shape[2]:
                raise ValueError("inconsistent shapes in a Clebsch-Gordan product")
            ptr, stride = out.data_ptr() + column * out.element_size(), out.shape[2]
        arr[k] = C.featomic_b200_cg_task_t(a.data_ptr(), b.data_ptr(), ptr, s, (m1 - 1) // 2,
                                           (m2 - 1) // 2, lam, p, q, stride)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    C.check(C.lib().featomic_b200_cg_product(arr, len(tasks), 64 if dtype == torch.float64 else 32,
                                             ctypes.c_void_p(stream)))


class Block:
    """values (torch CUDA tensor [samples, components..., properties]) with its labels."""

    def __init__(self, values, samples, components, properties, gradients=None):
        self.values = values
        self.samples = samples
        self.components = components
        self.properties = properties
        self._gradients = dict(gradients or {})

    def gradients_list(self):
        return list(self._gradients)

    def gradient(self, parameter):
        if parameter not in self._gradients:
            raise ValueError(f"this block has no gradient with respect to {parameter}")
        return self._gradients[parameter]


class EquivariantTensorMap:
    """Keys and blocks of a Clebsch-Gordan product, with the accessors of the
    calculators' TensorMap."""

    def __init__(self, keys, blocks):
        self.keys = keys
        self._blocks = blocks

    def __len__(self):
        return len(self.keys)

    def block_by_id(self, index):
        return self._blocks[index]

    def blocks(self):
        return list(self._blocks)

    def block(self, **selection):
        matches = np.ones(len(self.keys), dtype=bool)
        for name, value in selection.items():
            matches &= self.keys.column(name) == value
        idx = np.nonzero(matches)[0]
        if len(idx) != 1:
            raise ValueError(f"selection {selection} matches {len(idx)} blocks")
        return self._blocks[int(idx[0])]


def _rename(labels, old, new):
    return Labels([new if n == old else n for n in labels.names], labels.values)


def _to_device(tensor, suffix, dtype):
    """A spherical expansion with "neighbor_type" / "n" renamed
    (_equivariant_power_spectrum.py:312-320), values on the GPU."""
    import torch

    keys = _rename(tensor.keys, "neighbor_type", f"neighbor_{suffix}_type")
    blocks = []
    for b in tensor.blocks():
        values = torch.as_tensor(np.ascontiguousarray(b.values) if isinstance(b.values, np.ndarray) else b.values)
        blocks.append(Block(values.to(device="cuda", dtype=dtype).contiguous(), b.samples, b.components,
                            _rename(b.properties, "n", f"n_{suffix}")))
    return EquivariantTensorMap(keys, blocks)


def _union_rows(arrays):
    """Union of the rows of int32 arrays in order of first appearance, and for
    each array the union index of each of its rows."""
    if all(len(a) == len(arrays[0]) and np.array_equal(a, arrays[0]) for a in arrays[1:]):
        same = np.arange(len(arrays[0]))
        return arrays[0], [same] * len(arrays)
    stacked = np.concatenate(arrays, axis=0)
    _, first, inverse = np.unique(stacked, axis=0, return_index=True, return_inverse=True)
    inverse = inverse.reshape(-1)
    order = np.argsort(first, kind="stable")
    position = np.empty(len(first), dtype=np.int64)
    position[order] = np.arange(len(first))
    union = stacked[first[order]]
    out, start = [], 0
    for a in arrays:
        out.append(position[inverse[start:start + len(a)]])
        start += len(a)
    return union, out


def _merge_blocks(members, moved_names, moved_values):
    """Blocks of one merged key, properties (moved key values, block
    properties) in the order of ``moved_values``; samples are the union in
    order of first appearance and absent entries are zero (metatensor's
    keys_to_properties)."""
    import torch

    present = [b for b in members.values() if b is not None]
    union, index = _union_rows([b.samples.values for b in present])
    rows_of = {id(b): idx for b, idx in zip(present, index)}
    ref = present[0]
    comp_shape = tuple(ref.values.shape[1:-1])
    nprop = ref.values.shape[-1]
    prop_names = list(moved_names) + ref.properties.names
    parts, prop_values = [], []
    for mv in moved_values:
        b = members.get(mv)
        block_props = b.properties.values if b is not None else ref.properties.values
        prop_values.append(np.concatenate([np.tile(np.asarray(mv, dtype=np.int32), (len(block_props), 1)),
                                           block_props], axis=1))
        if b is None:
            parts.append(torch.zeros((len(union),) + comp_shape + (nprop,), dtype=ref.values.dtype, device="cuda"))
            continue
        idx = rows_of[id(b)]
        if len(idx) == len(union) and np.array_equal(idx, np.arange(len(union))):
            parts.append(b.values)
        else:
            full = torch.zeros((len(union),) + comp_shape + (b.values.shape[-1],), dtype=ref.values.dtype,
                               device="cuda")
            full[torch.as_tensor(idx, device="cuda", dtype=torch.long)] = b.values
            parts.append(full)
    sample_names = ref.samples.names
    return Block(torch.cat(parts, dim=-1).contiguous(), Labels(sample_names, union),
                 ref.components, Labels(prop_names, np.concatenate(prop_values, axis=0)))


def keys_to_properties(tensor, names, values=None):
    """Move the key dimensions ``names`` to the properties: blocks that differ
    only in them are merged.  ``values`` (rows of those dimensions) fixes the
    merged entries and their order, zero-filling absent blocks; without it
    each merged block holds the values its own blocks have, in increasing
    order."""
    keys = tensor.keys
    move = [keys.names.index(n) for n in names]
    keep = [i for i in range(len(keys.names)) if i not in move]
    if values is not None:
        values = [tuple(int(x) for x in np.atleast_1d(v)) for v in values]
    groups, order = {}, []
    for i, row in enumerate(keys.values):
        rest = tuple(int(v) for v in row[keep])
        if rest not in groups:
            groups[rest] = {}
            order.append(rest)
        groups[rest][tuple(int(v) for v in row[move])] = tensor.block_by_id(i)
    blocks = []
    for rest in order:
        group_values = values if values is not None else sorted(groups[rest])
        members = {mv: groups[rest].get(mv) for mv in group_values}
        blocks.append(_merge_blocks(members, names, group_values))
    new_keys = Labels([keys.names[i] for i in keep], np.array(order, dtype=np.int32).reshape(len(order), len(keep)))
    return EquivariantTensorMap(new_keys, blocks)


def _products_into_properties(tensor, tasks, names, launch=True):
    """``keys_to_properties(tensor, names)`` for a planned, unallocated
    product: each merged block is allocated once and every task writes its
    columns of it (no copy of the product)."""
    import torch

    keys = tensor.keys
    move = [keys.names.index(n) for n in names]
    keep = [i for i in range(len(keys.names)) if i not in move]
    groups, order = {}, []
    for i, row in enumerate(keys.values):
        rest = tuple(int(v) for v in row[keep])
        if rest not in groups:
            groups[rest] = []
            order.append(rest)
        groups[rest].append((tuple(int(v) for v in row[move]), i))
    blocks, run = [], []
    for rest in order:
        members = sorted(groups[rest])
        first = tensor.block_by_id(members[0][1])
        for _, i in members[1:]:
            b = tensor.block_by_id(i)
            if len(b.samples) != len(first.samples) or not np.array_equal(b.samples.values, first.samples.values):
                # different samples: allocate every product and merge with zero fill
                for k, (a, bb, out, lam) in enumerate(tasks):
                    tasks[k] = (a, bb, torch.empty(out, dtype=a.dtype, device="cuda"), lam)
                    tensor.block_by_id(k).values = tasks[k][2]
                if launch:
                    cg_tensor_products(tasks)
                return keys_to_properties(tensor, names)
        width = sum(tensor.block_by_id(i).properties.values.shape[0] for _, i in members)
        a0 = tasks[members[0][1]][0]
        shape = tasks[members[0][1]][2]
        merged = torch.empty((shape[0], shape[1], width), dtype=a0.dtype, device="cuda")
        column, props = 0, []
        for mv, i in members:
            a, b, _, lam = tasks[i]
            run.append((a, b, merged, lam, column))
            p = tensor.block_by_id(i).properties.values
            props.append(np.concatenate([np.tile(np.asarray(mv, dtype=np.int32), (len(p), 1)), p], axis=1))
            column += len(p)
        names_all = list(names) + first.properties.names
        blocks.append(Block(merged, first.samples, first.components,
                            Labels(names_all, np.concatenate(props, axis=0))))
    if launch:
        cg_tensor_products(run)
    new_keys = Labels([keys.names[i] for i in keep], np.array(order, dtype=np.int32).reshape(len(order), len(keep)))
    return EquivariantTensorMap(new_keys, blocks)


def _filter_redundant_keys(keys):
    """Keep keys with sorted angular orders l_1 <= l_2 <= ...
    (_density_correlations.py:233-272)."""
    nu = 1
    while f"l_{nu + 1}" in keys.names:
        nu += 1
    cols = [keys.names.index(f"l_{k}") for k in range(1, nu + 1)]
    return [i for i, row in enumerate(keys.values) if list(row[cols]) == sorted(row[cols])]


def _select(keys, selected):
    """Entries of ``keys`` matching any entry of ``selected`` on its dimensions
    (metatensor Labels.select)."""
    if not isinstance(selected, Labels):
        selected = Labels(*selected)
    cols = [keys.names.index(n) for n in selected.names]
    wanted = {tuple(int(v) for v in row) for row in selected.values}
    return [i for i, row in enumerate(keys.values) if tuple(int(v) for v in row[cols]) in wanted]


def _match_samples(b1, b2):
    """(samples, values_1, values_2) on common samples (_utils.py:272-350):
    with the same sample names, the union (block 1's samples, then the new
    ones of block 2, metatensor's union_and_mapping) with zeros where a block
    has no entry; otherwise the block with fewer sample dimensions is
    broadcast onto the other's samples."""
    import torch

    s1, s2 = b1.samples, b2.samples
    if s1.names == s2.names:
        if len(s1) == len(s2) and np.array_equal(s1.values, s2.values):
            return s1, b1.values, b2.values
        union, index = _union_rows([s1.values, s2.values])
        samples = Labels(s1.names, union)
        out = []
        for blk, idx in ((b1, index[0]), (b2, index[1])):
            full = torch.zeros((len(union),) + tuple(blk.values.shape[1:]), dtype=blk.values.dtype, device="cuda")
            if len(idx):
                full[torch.as_tensor(idx, dtype=torch.long, device="cuda")] = blk.values
            out.append(full)
        return samples, out[0], out[1]
    swapped = len(s1.names) > len(s2.names)
    small, big = (b2, b1) if swapped else (b1, b2)
    for name in small.samples.names:
        if name not in big.samples.names:
            raise ValueError("Samples dimensions of the two blocks are not compatible. The block with fewer "
                             "samples dimensions must be a subset of the other block's dimensions. Got: "
                             f"{small.samples.names} and {big.samples.names}. Offending dimension: {name}")
    dims = [big.samples.names.index(n) for n in small.samples.names]
    rows = {tuple(v): i for i, v in enumerate(small.samples.values)}
    idx = torch.as_tensor([rows[tuple(v)] for v in big.samples.values[:, dims]], dtype=torch.long, device="cuda")
    expanded = small.values[idx]
    if swapped:
        return big.samples, big.values, expanded
    return big.samples, expanded, big.values


class ClebschGordanProduct:
    """CG tensor product of two equivariant TensorMaps (_cg_product.py:29-436);
    no gradients, as in featomic."""

    def __init__(self, *, max_angular, keys_filter=None):
        self.max_angular = max_angular
        self._keys_filter = keys_filter or (lambda keys: list(range(len(keys))))

    def compute(self, tensor_1, tensor_2, o3_lambda_1_new_name, o3_lambda_2_new_name, selected_keys=None):
        """The product TensorMap (_cg_product.py:139-212 / :262-334)."""
        result, tasks = self.plan(tensor_1, tensor_2, o3_lambda_1_new_name, o3_lambda_2_new_name, selected_keys)
        cg_tensor_products(tasks)
        return result

    def compute_metadata(self, tensor_1, tensor_2, o3_lambda_1_new_name, o3_lambda_2_new_name,
                         selected_keys=None):
        """The product's keys, samples, components and properties, with
        uninitialised values of the right shapes and no product computed
        (_cg_product.py:238-260)."""
        result, _ = self.plan(tensor_1, tensor_2, o3_lambda_1_new_name, o3_lambda_2_new_name, selected_keys)
        return result

    def plan(self, tensor_1, tensor_2, o3_lambda_1_new_name, o3_lambda_2_new_name, selected_keys=None,
             allocate=True):
        """(TensorMap with unfilled values, its block-product tasks for
        ``cg_tensor_products``); with ``allocate=False`` the blocks and tasks
        carry the output shape instead of an output tensor."""
        import torch

        self._check_inputs(tensor_1, tensor_2, selected_keys)

        keys, combos = self._output_keys(tensor_1.keys, tensor_2.keys, o3_lambda_1_new_name, o3_lambda_2_new_name)
        if selected_keys is not None:
            idx = _select(keys, selected_keys)
            keys, combos = Labels(keys.names, keys.values[idx]), [combos[i] for i in idx]
        idx = self._keys_filter(keys)
        keys, combos = Labels(keys.names, keys.values[idx]), [combos[i] for i in idx]
        # all lambda of one block pair consecutive (_utils.py:160-216)
        groups, order = {}, []
        for i, c in enumerate(combos):
            if c not in groups:
                groups[c] = []
                order.append(c)
            groups[c].append(i)
        lam_col = keys.names.index("o3_lambda")
        new_values, blocks, tasks = [], [], []
        for c in order:
            b1, b2 = tensor_1.block_by_id(c[0]), tensor_2.block_by_id(c[1])
            if b1.values.ndim != 3 or b2.values.ndim != 3:
                raise ValueError("Clebsch-Gordan products take blocks with one o3_mu component")
            samples, a, b = _match_samples(b1, b2)
            a, b = a.contiguous(), b.to(a.dtype).contiguous()
            p1, p2 = b1.properties.values, b2.properties.values
            props = Labels(b1.properties.names + b2.properties.names,
                           np.concatenate([np.repeat(p1, len(p2), axis=0), np.tile(p2, (len(p1), 1))], axis=1))
            for i in groups[c]:
                lam = int(keys.values[i][lam_col])
                shape = (a.shape[0], 2 * lam + 1, a.shape[2] * b.shape[2])
                out = torch.empty(shape, dtype=a.dtype, device="cuda") if allocate else shape
                tasks.append((a, b, out, lam))
                mu = Labels(["o3_mu"], np.arange(-lam, lam + 1, dtype=np.int32).reshape(-1, 1))
                blocks.append(Block(out, samples, [mu], props))
                new_values.append(keys.values[i])
        return EquivariantTensorMap(
            Labels(keys.names, np.array(new_values, dtype=np.int32).reshape(-1, len(keys.names))), blocks), tasks

    def _check_inputs(self, tensor_1, tensor_2, selected_keys):
        """_cg_product.py:336-432."""
        for tensor in (tensor_1, tensor_2):
            if "o3_lambda" not in tensor.keys.names:
                raise ValueError("input tensors must have a named key dimension `'o3_lambda`")
            if "o3_sigma" not in tensor.keys.names:
                raise ValueError("input tensors must have a named key dimension `'o3_sigma`")
            for b in tensor.blocks():
                if len(b.components) != 1 or b.components[0].names != ["o3_mu"]:
                    raise ValueError("input tensors must have a single component axis with a single named "
                                     "dimensions `'o3_mu'`")
        max_angular = int(tensor_1.keys.column("o3_lambda").max(initial=0)
                          + tensor_2.keys.column("o3_lambda").max(initial=0))
        if selected_keys is not None:
            if not isinstance(selected_keys, Labels):
                selected_keys = Labels(*selected_keys)
            if "o3_lambda" in selected_keys.names:
                lams = selected_keys.column("o3_lambda")
                if len(lams) and int(lams.max()) > self.max_angular:
                    raise ValueError("the maximum angular momentum value found in key dimension `'o3_lambda'` in "
                                     f"`selected_keys` exceeds `max_angular={self.max_angular}` used to calculate "
                                     "the CG coefficients in the constructor.")
                if len(lams):
                    max_angular = min(max_angular, int(lams.max()))
            if "o3_sigma" in selected_keys.names:
                if any(int(v) not in (-1, 1) for v in selected_keys.column("o3_sigma")):
                    raise ValueError("key dimension `'o3_sigma'` in `selected_keys` must only contain values of "
                                     "-1 or 1.")
        if max_angular > self.max_angular:
            raise ValueError(f"the maximum angular momentum `{max_angular}` required by the input tensors (and "
                             "perhaps lowered by angular selection via `selected_keys`) exceeds the value of "
                             f"`max_angular={self.max_angular}` used to calculate the CG coefficients")
        if len(tensor_1) and len(tensor_2):
            shared = set(tensor_1.block_by_id(0).properties.names) & set(tensor_2.block_by_id(0).properties.names)
            if shared:
                raise ValueError(f"property names {sorted(shared)} are present in both input tensors; they must "
                                 "be unique")

    @staticmethod
    def _output_keys(keys_1, keys_2, name_1, name_2):
        """_utils.py:30-157 (_compute_output_keys)."""
        cg = ["o3_lambda", "o3_sigma"]
        for n in cg:
            if n not in keys_1.names or n not in keys_2.names:
                raise ValueError(f"both tensors need the key dimension {n}")
        match = [n for n in keys_1.names if n not in cg and n in keys_2.names]
        other_1 = [n for n in keys_1.names if n not in cg and n not in match]
        other_2 = [n for n in keys_2.names if n not in cg and n not in match]
        names = cg + match + other_1 + [name_1] + other_2 + [name_2]
        i1 = {n: keys_1.names.index(n) for n in keys_1.names}
        i2 = {n: keys_2.names.index(n) for n in keys_2.names}
        values, combos = [], []
        for a, k1 in enumerate(keys_1.values):
            for b, k2 in enumerate(keys_2.values):
                if any(k1[i1[n]] != k2[i2[n]] for n in match):
                    continue
                l1, s1 = int(k1[i1["o3_lambda"]]), int(k1[i1["o3_sigma"]])
                l2, s2 = int(k2[i2["o3_lambda"]]), int(k2[i2["o3_sigma"]])
                for lam in range(abs(l1 - l2), l1 + l2 + 1):
                    sigma = s1 * s2 * (-1) ** (l1 + l2 + lam)
                    values.append([lam, sigma] + [int(k1[i1[n]]) for n in match] + [int(k1[i1[n]]) for n in other_1]
                                  + [l1] + [int(k2[i2[n]]) for n in other_2] + [l2])
                    combos.append((a, b))
        return Labels(names, np.array(values, dtype=np.int32).reshape(-1, len(names))), combos


class EquivariantPowerSpectrum:
    """Equivariant power spectrum ("lambda-SOAP") of one or two spherical
    expansions (_equivariant_power_spectrum.py:23-365)."""

    def __init__(self, calculator_1, calculator_2=None, neighbor_types=None, *, dtype=None, device=None):
        import torch

        supported = ["spherical_expansion"]
        for k, calc in ((1, calculator_1), (2, calculator_2)):
            if calc is None:
                continue
            if calc._name not in supported:
                raise ValueError(f"Only [{', '.join(supported)}] are supported for `calculator_{k}`, "
                                 f"got '{calc._name}'")
        p1 = json.loads(calculator_1.parameters)
        p2 = p1 if calculator_2 is None else json.loads(calculator_2.parameters)
        if calculator_2 is not None:
            for k, p in ((1, p1), (2, p2)):
                if p["basis"]["type"] != "TensorProduct":
                    raise ValueError(f"only 'TensorProduct' basis is supported for calculator_{k}")
        if device is not None and torch.device(device).type != "cuda":
            raise ValueError("the equivariant power spectrum runs on CUDA devices only")
        self.calculator_1 = calculator_1
        self.calculator_2 = calculator_2
        self.neighbor_types = neighbor_types
        self.dtype = dtype if dtype is not None else torch.float64
        self._cg_product = ClebschGordanProduct(
            max_angular=p1["basis"]["max_angular"] + p2["basis"]["max_angular"],
            keys_filter=_filter_redundant_keys)

    @property
    def name(self):
        return "EquivariantPowerSpectrum"

    def compute_metadata(self, systems, selected_keys=None, neighbors_to_properties=False):
        """Metadata of ``compute`` with uninitialised values, without the
        Clebsch-Gordan products (_equivariant_power_spectrum.py:276-294)."""
        return self.compute(systems, selected_keys, neighbors_to_properties, _metadata=True)

    def compute(self, systems, selected_keys=None, neighbors_to_properties=False, _metadata=False):
        """_equivariant_power_spectrum.py:215-256 / :296-365."""
        density_1 = self.calculator_1.compute(systems)
        density_2 = density_1 if self.calculator_2 is None else self.calculator_2.compute(systems)
        d1 = _to_device(density_1, 1, self.dtype)
        d2 = _to_device(density_2, 2, self.dtype)
        if neighbors_to_properties:
            values = None if self.neighbor_types is None else [[t] for t in self.neighbor_types]
            d1 = keys_to_properties(d1, ["neighbor_1_type"], values)
            d2 = keys_to_properties(d2, ["neighbor_2_type"], values)
        ps, tasks = self._cg_product.plan(d1, d2, "l_1", "l_2", selected_keys, allocate=False)
        return _products_into_properties(ps, tasks, ["l_1", "l_2"], launch=not _metadata)

    forward = compute


def as_tensormap(tensor, dtype=None):
    """An ``EquivariantTensorMap`` on the GPU from a calculator's TensorMap
    (host or device), labels unchanged."""
    import torch

    blocks = []
    for b in tensor.blocks():
        values = b.values
        values = torch.as_tensor(np.ascontiguousarray(values) if isinstance(values, np.ndarray) else values)
        blocks.append(Block(values.to(device="cuda", dtype=dtype or values.dtype).contiguous(), b.samples,
                            b.components, b.properties))
    return EquivariantTensorMap(tensor.keys, blocks)


def _increment_numeric_suffix(name, increment_by=1):
    """_density_correlations.py:320-359: "n" -> "n_1", "n_1" -> "n_2",
    "center_type" -> "center_1_type"."""
    if not isinstance(increment_by, int):
        raise ValueError("`increment_by` must be an integer.")
    if name.endswith("type"):
        prefix, suffix = name[: name.rfind("_type")], "_type"
    else:
        prefix, suffix = name, ""
    number = "0"
    if prefix.rfind("_") != -1:
        tail = prefix[prefix.rfind("_") + 1:]
        if tail.isdigit():
            number = tail
            prefix = prefix[: prefix.rfind("_")]
    return prefix + "_" + str(int(number) + increment_by) + suffix


def _increment_property_names(tensor, increment_by=1):
    """_density_correlations.py:275-317."""
    if increment_by < 0:
        raise ValueError("`increment_by` must be a non-negative integer.")
    blocks = [Block(b.values, b.samples, b.components,
                    Labels([_increment_numeric_suffix(n, increment_by) for n in b.properties.names],
                           b.properties.values))
              for b in tensor.blocks()]
    return EquivariantTensorMap(tensor.keys, blocks)


class DensityCorrelations:
    """Iterated Clebsch-Gordan products of a density with itself, to body
    order n_correlations + 2 (_density_correlations.py:23-231)."""

    def __init__(self, *, n_correlations, max_angular, skip_redundant=True, dtype=None, device=None):
        import torch

        if device is not None and torch.device(device).type != "cuda":
            raise ValueError("density correlations run on CUDA devices only")
        self._n_correlations = n_correlations
        self._dtype = dtype
        self._cg_product = ClebschGordanProduct(max_angular=max_angular,
                                                keys_filter=_filter_redundant_keys if skip_redundant else None)

    def compute_metadata(self, density, angular_cutoff=None, selected_keys=None):
        """Metadata of ``compute`` with uninitialised values
        (_density_correlations.py:140-158)."""
        return self.compute(density, angular_cutoff, selected_keys, _metadata=True)

    def compute(self, density, angular_cutoff=None, selected_keys=None, _metadata=False):
        """_density_correlations.py:70-120 / :160-231; ``density`` is a
        calculator TensorMap or an ``EquivariantTensorMap``."""
        if not isinstance(density, EquivariantTensorMap):
            density = as_tensormap(density, self._dtype)
        correlations = _increment_property_names(density, 1)
        density = _increment_property_names(density, 1)
        for i in range(self._n_correlations):
            density = _increment_property_names(density, 1)
            name_1 = f"l_{i + 1}" if i == 0 else f"k_{i + 1}"
            name_2 = f"l_{i + 2}"
            last = i == self._n_correlations - 1
            if last and selected_keys is not None:
                selection = selected_keys
            elif angular_cutoff is None:
                selection = None
            else:
                selection = Labels(["o3_lambda"], np.arange(angular_cutoff + 1, dtype=np.int32).reshape(-1, 1))
            if _metadata:
                correlations = self._cg_product.compute_metadata(correlations, density, name_1, name_2, selection)
            else:
                correlations = self._cg_product.compute(correlations, density, name_1, name_2, selection)
        return correlations

    forward = compute



def _moved_with_gradients(tm, types, dtype):
    """keys_to_properties(neighbor_type) of a spherical expansion with its
    positions gradients: per (o3_lambda, o3_sigma, center_type), values
    [samples, 2l+1, types * n] and gradients [gradient samples, 3, 2l+1,
    types * n], absent types zero; gradient samples (sample, system, atom)
    are the union over the merged blocks, "sample" renumbered to the merged
    samples."""
    import torch

    keys = tm.keys
    nt = keys.names.index("neighbor_type")
    groups, order = {}, []
    for i, row in enumerate(keys.values):
        rest = (int(row[0]), int(row[1]), int(row[2]))
        if rest not in groups:
            groups[rest] = {}
            order.append(rest)
        groups[rest][int(row[nt])] = i
    out_keys, blocks = [], []
    for rest in order:
        present = [(k, tm.block_by_id(groups[rest][t])) for k, t in enumerate(types) if t in groups[rest]]
        union, index = _union_rows([b.samples.values for _, b in present])
        ref = present[0][1]
        M, N = ref.values.shape[1], ref.values.shape[2]
        values = torch.zeros((len(union), M, len(types) * N), dtype=dtype, device="cuda")
        grads = []
        for (k, b), ix in zip(present, index):
            ixt = torch.as_tensor(ix, device="cuda", dtype=torch.long)
            values[ixt, :, k * N:(k + 1) * N] = torch.as_tensor(np.ascontiguousarray(b.values)).to("cuda", dtype)
            g = b.gradient("positions")
            gs = np.array(g.samples.values, dtype=np.int32).reshape(-1, 3)
            gs[:, 0] = ix[gs[:, 0]]
            grads.append((k, gs, g.values))
        gunion, gindex = _union_rows([gs for _, gs, _ in grads])
        gvalues = torch.zeros((len(gunion), 3, M, len(types) * N), dtype=dtype, device="cuda")
        for (k, gs, gv), gi in zip(grads, gindex):
            if len(gi):
                gvalues[torch.as_tensor(gi, device="cuda", dtype=torch.long), :, :, k * N:(k + 1) * N] = \
                    torch.as_tensor(np.ascontiguousarray(gv)).to("cuda", dtype)
        props = np.array([[t, int(n)] for t in types for n in ref.properties.values[:, 0]], dtype=np.int32)
        grad = Block(gvalues, Labels(["sample", "system", "atom"], gunion.reshape(-1, 3)), [], None)
        blocks.append(Block(values, Labels(ref.samples.names, union), ref.components,
                            Labels(["neighbor_type", "n"], props), {"positions": grad}))
        out_keys.append(list(rest))
    return EquivariantTensorMap(Labels(["o3_lambda", "o3_sigma", "center_type"], np.array(out_keys, dtype=np.int32)),
                                blocks)


class PowerSpectrum:
    """The invariant power spectrum of featomic's Clebsch-Gordan module
    (python/featomic/featomic/clebsch_gordan/_power_spectrum.py:27-352):
    keys (center_type), properties (l, neighbor_1_type, n_1, neighbor_2_type,
    n_2), values (-1)^l / sqrt(2l + 1) sum_m c1[m, a] c2[m, b] -- the
    lambda = 0 product of the two l blocks, computed by the Clebsch-Gordan
    kernel (its lambda = 0 coefficients are that factor).  Positions
    gradients (_power_spectrum.py:373-435) are two more lambda = 0 products
    per block: dc1 x c2 and c1 x dc2 on the gradient samples."""

    def __init__(self, calculator_1, calculator_2=None, neighbor_types=None, *, dtype=None, device=None):
        import torch

        for k, calc in ((1, calculator_1), (2, calculator_2)):
            if calc is not None and calc._name != "spherical_expansion":
                raise ValueError(f"Only [spherical_expansion] are supported for `calculator_{k}`, "
                                 f"got '{calc._name}'")
        if device is not None and torch.device(device).type != "cuda":
            raise ValueError("the power spectrum runs on CUDA devices only")
        self.calculator_1 = calculator_1
        self.calculator_2 = calculator_2
        self.neighbor_types = neighbor_types
        self.dtype = dtype if dtype is not None else torch.float64

    @property
    def name(self):
        return "PowerSpectrum"

    def _density(self, calc, systems, suffix):
        tm = calc.compute(systems)
        if tm.keys.names != ["o3_lambda", "o3_sigma", "center_type", "neighbor_type"]:
            raise ValueError("expected a spherical expansion")
        if self.neighbor_types is None:
            values = [[int(t)] for t in np.unique(tm.keys.column("neighbor_type"))]
        else:
            values = [[t] for t in self.neighbor_types]
        d = keys_to_properties(as_tensormap(tm, self.dtype), ["neighbor_type"], values)
        return _increment_property_names(d, suffix)

    def _types(self, tm):
        if self.neighbor_types is None:
            return [int(t) for t in np.unique(tm.keys.column("neighbor_type"))]
        return list(self.neighbor_types)

    def compute(self, systems, gradients=None, use_native_system=True):
        """_power_spectrum.py:196-351."""
        import torch

        if gradients:
            for parameter in gradients:
                if parameter != "positions":
                    raise NotImplementedError("PowerSpectrum currently only supports gradients w.r.t. to positions")
            return self._compute_with_gradients(systems)
        d1 = self._density(self.calculator_1, systems, 1)
        d2 = d1 if self.calculator_2 is None else self._density(self.calculator_2, systems, 1)
        d2 = _increment_property_names(d2, 1)
        tasks, values, keys = [], [], []
        for i, key in enumerate(d1.keys.values):
            lam, ct = int(key[0]), int(key[2])
            b1 = d1.block_by_id(i)
            for j, key2 in enumerate(d2.keys.values):
                if int(key2[0]) != lam or int(key2[2]) != ct:
                    continue
                b2 = d2.block_by_id(j)
                if len(b1.samples) != len(b2.samples) or not np.array_equal(b1.samples.values, b2.samples.values):
                    raise ValueError("the two spherical expansions have different samples")
                out = torch.empty((len(b1.samples), 1, b1.values.shape[2] * b2.values.shape[2]),
                                  dtype=b1.values.dtype, device="cuda")
                tasks.append((b1.values.contiguous(), b2.values.contiguous(), out, 0))
                p1, p2 = b1.properties.values, b2.properties.values
                props = Labels(["neighbor_1_type", "n_1", "neighbor_2_type", "n_2"],
                               np.concatenate([np.repeat(p1, len(p2), axis=0), np.tile(p2, (len(p1), 1))], axis=1))
                values.append(Block(out, b1.samples, [], props))
                keys.append([lam, ct])
        cg_tensor_products(tasks)
        blocks = [Block(b.values.reshape(b.values.shape[0], -1), b.samples, [], b.properties) for b in values]
        tm = EquivariantTensorMap(Labels(["l", "center_type"], np.array(keys, dtype=np.int32).reshape(-1, 2)),
                                  blocks)
        return keys_to_properties(tm, ["l"])

    forward = compute

    def _compute_with_gradients(self, systems):
        import torch

        tm1 = self.calculator_1.compute(systems, gradients=["positions"])
        d1 = _moved_with_gradients(tm1, self._types(tm1), self.dtype)
        if self.calculator_2 is None:
            d2 = d1
        else:
            tm2 = self.calculator_2.compute(systems, gradients=["positions"])
            d2 = _moved_with_gradients(tm2, self._types(tm2), self.dtype)
        tasks, pending = [], []
        for i, key in enumerate(d1.keys.values):
            lam, ct = int(key[0]), int(key[2])
            b1 = d1.block_by_id(i)
            for j, key2 in enumerate(d2.keys.values):
                if int(key2[0]) != lam or int(key2[2]) != ct:
                    continue
                b2 = d2.block_by_id(j)
                if len(b1.samples) != len(b2.samples) or not np.array_equal(b1.samples.values, b2.samples.values):
                    raise ValueError("the two spherical expansions have different samples")
                c1, c2 = b1.values, b2.values
                S, M, P = c1.shape
                Q = c2.shape[2]
                out = torch.empty((S, 1, P * Q), dtype=c1.dtype, device="cuda")
                tasks.append((c1, c2, out, 0))
                g1, g2 = b1.gradient("positions"), b2.gradient("positions")
                gs1, gs2 = g1.samples.values, g2.samples.values
                grad = None
                if len(gs1) and len(gs2):
                    # dc1[g, x] x c2[sample(g)] and c1[sample(g)] x dc2[g, x], (g, x) as samples
                    r1 = torch.as_tensor(gs1[:, 0], device="cuda", dtype=torch.long).repeat_interleave(3)
                    r2 = torch.as_tensor(gs2[:, 0], device="cuda", dtype=torch.long).repeat_interleave(3)
                    o1 = torch.empty((len(gs1) * 3, 1, P * Q), dtype=c1.dtype, device="cuda")
                    o2 = torch.empty((len(gs2) * 3, 1, P * Q), dtype=c1.dtype, device="cuda")
                    tasks.append((g1.values.reshape(-1, M, P), c2[r1].contiguous(), o1, 0))
                    tasks.append((c1[r2].contiguous(), g2.values.reshape(-1, M, Q), o2, 0))
                    grad = (gs1, gs2, o1, o2)
                p1, p2 = b1.properties.values, b2.properties.values
                props = np.concatenate([np.repeat(p1, len(p2), axis=0), np.tile(p2, (len(p1), 1))], axis=1)
                pending.append((lam, ct, b1.samples, out, props, grad))
        cg_tensor_products(tasks)
        # keys_to_properties("l"): one block per centre type, l-major properties
        groups, order = {}, []
        for entry in pending:
            if entry[1] not in groups:
                groups[entry[1]] = []
                order.append(entry[1])
            groups[entry[1]].append(entry)
        xyz = Labels(["xyz"], np.arange(3, dtype=np.int32).reshape(-1, 1))
        blocks = []
        for ct in order:
            members = sorted(groups[ct], key=lambda e: e[0])
            samples = members[0][2]
            values = torch.cat([e[3].reshape(e[3].shape[0], -1) for e in members], dim=1)
            props = np.concatenate([np.concatenate([np.full((len(e[4]), 1), e[0], dtype=np.int32), e[4]], axis=1)
                                    for e in members], axis=0)
            parts = []
            for e in members:
                if e[5] is None:
                    parts.append((np.zeros((0, 3), dtype=np.int32), None, e[4].shape[0]))
                    continue
                gs1, gs2, o1, o2 = e[5]
                gunion, (i1, i2) = _union_rows([gs1, gs2])
                gv = torch.zeros((len(gunion), 3, o1.shape[2]), dtype=o1.dtype, device="cuda")
                gv[torch.as_tensor(i1, device="cuda", dtype=torch.long)] += o1.reshape(len(gs1), 3, -1)
                gv[torch.as_tensor(i2, device="cuda", dtype=torch.long)] += o2.reshape(len(gs2), 3, -1)
                parts.append((gunion, gv, e[4].shape[0]))
            gunion, gindex = _union_rows([p[0] for p in parts])
            width = sum(p[2] for p in parts)
            gvalues = torch.zeros((len(gunion), 3, width), dtype=values.dtype, device="cuda")
            column = 0
            for (rows, gv, w), gi in zip(parts, gindex):
                if gv is not None and len(gi):
                    gvalues[torch.as_tensor(gi, device="cuda", dtype=torch.long), :, column:column + w] = gv
                column += w
            names = ["l", "neighbor_1_type", "n_1", "neighbor_2_type", "n_2"]
            prop_labels = Labels(names, props)
            grad = Block(gvalues, Labels(["sample", "system", "atom"], gunion.reshape(-1, 3)), [xyz], prop_labels)
            blocks.append(Block(values, samples, [], prop_labels, {"positions": grad}))
        return EquivariantTensorMap(Labels(["center_type"], np.array(order, dtype=np.int32).reshape(-1, 1)), blocks)



def cg_couple(tasks, stream=None):
    """Run ``(input, output, l1, l2, o3_lambda)`` couplings (contiguous CUDA
    tensors of one dtype, input [outer, 2 l1 + 1, 2 l2 + 1, inner], output
    [outer, 2 o3_lambda + 1, inner]) in one launch
    (_coefficients.py:387-545, cg_couple)."""
    import torch

    if not tasks:
        return
    dtype = tasks[0][0].dtype
    if dtype not in (torch.float32, torch.float64):
        raise TypeError("Clebsch-Gordan couplings take float32 or float64 tensors")
    arr = (C.featomic_b200_cg_couple_task_t * len(tasks))()
    for k, (x, out, l1, l2, lam) in enumerate(tasks):
        for t in (x, out):
            if not t.is_cuda or t.dtype != dtype or not t.is_contiguous():
                raise ValueError("Clebsch-Gordan tensors must be contiguous CUDA tensors of one dtype")
        if x.ndim != 4 or x.shape[1] != 2 * l1 + 1 or x.shape[2] != 2 * l2 + 1 or \
                tuple(out.shape) != (x.shape[0], 2 * lam + 1, x.shape[3]):
            raise ValueError("inconsistent shapes in a Clebsch-Gordan coupling")
        arr[k] = C.featomic_b200_cg_couple_task_t(x.data_ptr(), out.data_ptr(), x.shape[0], x.shape[3], l1, l2, lam)
    if stream is None:
        stream = torch.cuda.current_stream().cuda_stream
    C.check(C.lib().featomic_b200_cg_couple(arr, len(tasks), 64 if dtype == torch.float64 else 32,
                                            ctypes.c_void_p(stream)))


def _insert(labels, name, value):
    return Labels([name] + labels.names,
                  np.concatenate([np.full((len(labels), 1), value, dtype=np.int32), labels.values], axis=1))


def cartesian_to_spherical(tensor, components, keep_l_in_keys=None, remove_blocks_threshold=1e-9, cg_backend=None,
                           cg_coefficients=None):
    """A tensor with Cartesian (xyz) components in spherical form
    (_cartesian_spherical.py:21-304): the xyz axes become (y, z, x) = real
    l = 1 components, then the last two converted axes are coupled with
    Clebsch-Gordan coefficients until one o3_mu axis is left; keys gain
    o3_lambda, o3_sigma (and l_i / k_i with ``keep_l_in_keys``); blocks whose
    squared norm is at most ``remove_blocks_threshold`` are dropped.

    ``cg_backend`` follows featomic: "python-sparse" (the default for numpy
    values) couples x[m1, m2] with C[m1, m2, mu]; "python-dense" (the default
    for torch values) swaps the two coupled axes before contracting, which
    multiplies every coupled block by (-1)^(l1 + l2 + lambda), i.e. flips the
    sign of the o3_sigma = -1 blocks (_coefficients.py:440-455).  The
    coupling always runs on the GPU; ``cg_coefficients`` is accepted for
    featomic's signature and not needed (the coefficients are computed here).
    Values come back with the input's array type and device."""
    import torch

    if len(tensor) == 0 or len(components) == 0:
        return tensor
    values0 = tensor.block_by_id(0).values
    if isinstance(values0, np.ndarray):
        out_numpy, out_device = True, None
    elif isinstance(values0, torch.Tensor):
        out_numpy, out_device = False, values0.device
    else:
        raise TypeError(f"unknown array type in tensor ({type(values0)}), only numpy and torch are supported")
    if cg_backend is None:
        cg_backend = "python-sparse" if out_numpy else "python-dense"
    _check_cg_backend(cg_backend)
    dense_backend = cg_backend == "python-dense"
    if not isinstance(components, list):
        raise TypeError(f"`components` should be a list, got {type(components)}")
    if keep_l_in_keys is None:
        keep_l_in_keys = len(components) >= 3
    first = tensor.block_by_id(0)
    names = [c.names[0] for c in first.components]
    axes = []
    for component in components:
        if component not in names:
            raise ValueError(f"'{component}' is not part of this tensor components")
        axes.append(names.index(component) + 1)
    for key, block in zip(tensor.keys.values, tensor.blocks()):
        for idx in axes:
            values = [int(v) for v in block.components[idx - 1].values[:, 0]]
            if values != [0, 1, 2]:
                raise ValueError(f"component '{block.components[idx - 1].names[0]}' in block for key {list(key)} "
                                 f"should have [0, 1, 2] as values, got {values} instead")
    if list(range(axes[0], axes[-1] + 1)) != axes:
        raise ValueError(f"this function only supports consecutive components, {components} are not")
    if "o3_lambda" in tensor.keys.names:
        raise ValueError("this tensor already has an `o3_lambda` key, is it already in spherical form?")
    for i in range(len(components)):
        if f"l_{i}" in tensor.keys.names:
            raise ValueError(f"this tensor already has an `l_{i}` key, is it already in spherical form?")
    if len(components) > 2 and not keep_l_in_keys:
        raise ValueError("`keep_l_in_keys` must be `True` for tensors of rank 3 and above")

    blocks = []
    for block in tensor.blocks():
        values = block.values
        if isinstance(values, np.ndarray):
            values = torch.as_tensor(np.ascontiguousarray(values))
        values = values.to("cuda")
        values = torch.roll(values, shifts=[-1] * len(axes), dims=axes).contiguous()
        comps = []
        for idx, comp in enumerate(block.components):
            if idx + 1 in axes:
                name = "o3_mu" if len(axes) == 1 else f"__internal_to_convert_{idx}"
                comps.append(Labels([name], np.array([[-1], [0], [1]], dtype=np.int32)))
            else:
                comps.append(comp)
        blocks.append(Block(values, block.samples, comps, block.properties))
    keys = tensor.keys
    if len(axes) == 1:
        if keep_l_in_keys:
            keys = _insert(keys, "l_1", 1)
        keys = _insert(_insert(keys, "o3_sigma", 1), "o3_lambda", 1)
        return _to_input_arrays(EquivariantTensorMap(keys, blocks), out_numpy, out_device)
    current = EquivariantTensorMap(keys, blocks)
    iteration = 0
    while len(axes) > 1:
        current = _do_coupling(current, axes[-2] - 1, axes[-1] - 1, keep_l_in_keys, iteration, dense_backend)
        axes.pop()
        iteration += 1
    if remove_blocks_threshold is not None:
        kept = [i for i, b in enumerate(current.blocks())
                if float((b.values * b.values).sum()) > remove_blocks_threshold]
        current = EquivariantTensorMap(Labels(current.keys.names, current.keys.values[kept]),
                                       [current.block_by_id(i) for i in kept])
    return _to_input_arrays(current, out_numpy, out_device)


def _to_input_arrays(tensor, numpy_values, device):
    """The blocks' values as numpy arrays, or torch tensors on ``device``."""
    blocks = []
    for b in tensor.blocks():
        values = b.values.cpu().numpy() if numpy_values else b.values.to(device)
        blocks.append(Block(values, b.samples, b.components, b.properties))
    return EquivariantTensorMap(tensor.keys, blocks)


def _do_coupling(tensor, component_1, component_2, keep_l_in_keys, iteration, dense_backend=False):
    """_cartesian_spherical.py:307-444: couple two consecutive spherical
    component axes of every block to every allowed lambda; with
    ``dense_backend`` the result of featomic's "python-dense" backend, the
    coupled block times (-1)^(l1 + l2 + lambda)."""
    import torch

    assert component_2 == component_1 + 1
    keys = tensor.keys
    if "o3_lambda" in keys.names:
        old_sigmas = keys.column("o3_sigma").copy()
        keep = [i for i, n in enumerate(keys.names) if n != "o3_sigma"]
        keys = Labels([keys.names[i] for i in keep], keys.values[:, keep])
    else:
        old_sigmas = np.ones(len(keys), dtype=np.int32)
    if keep_l_in_keys:
        if "o3_lambda" in keys.names:
            keys = Labels([f"k_{iteration}" if n == "o3_lambda" else n for n in keys.names], keys.values)
            keys = _insert(keys, f"l_{iteration + 2}", 1)
        else:
            keys = _insert(_insert(keys, "l_1", 1), "l_2", 1)
    new_values, new_blocks, tasks = [], [], []
    for k, block in enumerate(tensor.blocks()):
        shape = tuple(block.values.shape)
        l1 = (shape[component_1 + 1] - 1) // 2
        l2 = (shape[component_2 + 1] - 1) // 2
        before = int(np.prod(shape[:component_1 + 1]))
        after = int(np.prod(shape[component_2 + 2:]))
        x = block.values.reshape(before, shape[component_1 + 1], shape[component_2 + 1], after)
        for lam in range(abs(l1 - l2), l1 + l2 + 1):
            sigma = int(old_sigmas[k]) * (-1) ** (l1 + l2 + lam)
            new_values.append([lam, sigma] + [int(v) for v in keys.values[k]])
            out = torch.empty((before, 2 * lam + 1, after), dtype=x.dtype, device="cuda")
            tasks.append((x, out, l1, l2, lam))
            new_shape = list(shape)
            new_shape.pop(component_2 + 1)
            new_shape[component_1 + 1] = 2 * lam + 1
            comps = list(block.components)
            comps.pop(component_2)
            comps[component_1] = Labels(["o3_mu"], np.arange(-lam, lam + 1, dtype=np.int32).reshape(-1, 1))
            new_blocks.append(Block(out.view(new_shape), block.samples, comps, block.properties))
    cg_couple(tasks)
    if dense_backend:
        for x, out, l1, l2, lam in tasks:
            if (l1 + l2 + lam) % 2 == 1:
                out.neg_()
    return EquivariantTensorMap(Labels(["o3_lambda", "o3_sigma"] + keys.names,
                                       np.array(new_values, dtype=np.int32).reshape(len(new_values), -1)),
                                new_blocks)
