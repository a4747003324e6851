"""Python front-end mirroring featomic's calculator API.

``SphericalExpansion(cutoff=..., density=..., basis=...)`` and
``SoapPowerSpectrum(...)`` take featomic's hyper-parameters
(featomic/src/calculators/soap/spherical_expansion_pair.rs:37-45,
power_spectrum.rs:35-43), and ``compute(systems, gradients=...,
use_native_system=...)`` follows python/featomic/featomic/calculator_base.py:187+.
Everything below goes through the C ABI of ``libfeatomic_b200.so``.
"""
import ctypes
import json

import numpy as np

from . import _c_api as C


class Labels:
    """Names and int32 values of a metatensor Labels object."""

    def __init__(self, names, values):
        self.names = list(names)
        self.values = np.asarray(values, dtype=np.int32).reshape(-1, len(self.names)) if self.names else \
            np.zeros((len(values), 0), dtype=np.int32)

    def __len__(self):
        return self.values.shape[0]

    def __repr__(self):
        return f"Labels({self.names}, {len(self)} entries)"

    def column(self, name):
        return self.values[:, self.names.index(name)]

    @staticmethod
    def _from_c(labels):
        names = [labels.names[i].decode() for i in range(labels.size)]
        if labels.count == 0 or labels.size == 0:
            return Labels(names, np.zeros((0, len(names)), dtype=np.int32))
        values = np.ctypeslib.as_array(labels.values, shape=(labels.count, labels.size)).copy()
        return Labels(names, values)


class _DeviceArray:
    """__cuda_array_interface__ view of a device block, keeping its TensorMap alive."""

    def __init__(self, ptr, shape, owner):
        self._owner = owner
        self.__cuda_array_interface__ = {
            "shape": tuple(shape),
            "typestr": "<f8",
            "data": (ptr, False),
            "version": 3,
            "strides": None,
            "stream": None,
        }


class TensorBlock:
    def __init__(self, handle, owner):
        self._handle = handle
        self._owner = owner

    def _labels(self, axis):
        out = C.mts_labels_t()
        C.check(C.lib().mts_block_labels(self._handle, axis, ctypes.byref(out)))
        return Labels._from_c(out)

    @property
    def shape(self):
        data = ctypes.POINTER(ctypes.c_double)()
        shape = ctypes.POINTER(ctypes.c_size_t)()
        ndim = ctypes.c_size_t()
        on_device = ctypes.c_int32()
        C.check(C.lib().featomic_b200_block_values(self._handle, ctypes.byref(data), ctypes.byref(shape),
                                                    ctypes.byref(ndim), ctypes.byref(on_device)))
        return tuple(shape[i] for i in range(ndim.value))

    @property
    def samples(self):
        return self._labels(0)

    @property
    def components(self):
        n = len(self.shape) - 2
        return [self._labels(1 + k) for k in range(n)]

    @property
    def properties(self):
        return self._labels(len(self.shape) - 1)

    @property
    def values(self):
        """numpy view (host TensorMap) or torch CUDA tensor view (device TensorMap)."""
        data = ctypes.POINTER(ctypes.c_double)()
        shape = ctypes.POINTER(ctypes.c_size_t)()
        ndim = ctypes.c_size_t()
        on_device = ctypes.c_int32()
        C.check(C.lib().featomic_b200_block_values(self._handle, ctypes.byref(data), ctypes.byref(shape),
                                                    ctypes.byref(ndim), ctypes.byref(on_device)))
        shp = tuple(shape[i] for i in range(ndim.value))
        size = int(np.prod(shp)) if shp else 0
        if on_device.value:
            import torch
            ptr = ctypes.cast(data, ctypes.c_void_p).value or 0
            if size == 0:
                return torch.zeros(shp, dtype=torch.float64, device="cuda")
            return torch.as_tensor(_DeviceArray(ptr, shp, self._owner), device="cuda")
        if size == 0:
            return np.zeros(shp)
        array = np.ctypeslib.as_array(data, shape=(size,)).reshape(shp)
        array.flags.writeable = True
        return _OwnedArray(array, self._owner)

    def gradients_list(self):
        names = ctypes.POINTER(ctypes.c_char_p)()
        count = ctypes.c_size_t()
        C.check(C.lib().mts_block_gradients_list(self._handle, ctypes.byref(names), ctypes.byref(count)))
        return [names[i].decode() for i in range(count.value)]

    def gradient(self, parameter):
        out = ctypes.c_void_p()
        C.check(C.lib().mts_block_gradient(self._handle, parameter.encode(), ctypes.byref(out)))
        return TensorBlock(out, self._owner)


class _OwnedArray(np.ndarray):
    """numpy view that keeps the owning TensorMap alive."""

    def __new__(cls, array, owner):
        obj = np.asarray(array).view(cls)
        obj._owner = owner
        return obj

    def __array_finalize__(self, obj):
        self._owner = getattr(obj, "_owner", None)


class TensorMap:
    def __init__(self, handle):
        self._handle = handle

    def __del__(self):
        if getattr(self, "_handle", None):
            try:
                C.lib().mts_tensormap_free(self._handle)
            except (AttributeError, TypeError):  # interpreter shutdown
                pass
            self._handle = None

    @property
    def keys(self):
        out = C.mts_labels_t()
        C.check(C.lib().mts_tensormap_keys(self._handle, ctypes.byref(out)))
        return Labels._from_c(out)

    def __len__(self):
        return len(self.keys)

    def block_by_id(self, index):
        out = ctypes.c_void_p()
        C.check(C.lib().mts_tensormap_block_by_id(self._handle, ctypes.byref(out), index))
        return TensorBlock(out, self)

    def blocks(self):
        return [self.block_by_id(i) for i in range(len(self))]

    def block(self, **selection):
        keys = self.keys
        matches = np.ones(len(keys), dtype=bool)
        for name, value in selection.items():
            matches &= keys.column(name) == value
        idx = np.nonzero(matches)[0]
        if len(idx) != 1:
            raise ValueError(f"selection {selection} matches {len(idx)} blocks")
        return self.block_by_id(int(idx[0]))

    def to_dict(self, gradients=()):
        """Plain-dict copy ({"keys", "blocks": [{"samples", "properties", "values", "gradients"}]})."""
        blocks = []
        for b in self.blocks():
            values = b.values
            if not isinstance(values, np.ndarray):
                values = values.cpu().numpy()
            entry = {"samples": b.samples.values, "properties": b.properties.values,
                     "values": np.array(values), "gradients": {}}
            for g in gradients:
                gb = b.gradient(g)
                gv = gb.values
                if not isinstance(gv, np.ndarray):
                    gv = gv.cpu().numpy()
                entry["gradients"][g] = {"samples": gb.samples.values, "values": np.array(gv)}
            blocks.append(entry)
        return {"keys": self.keys.values, "blocks": blocks}


def labels_tensormap(keys, samples=None, properties=None):
    """TensorMap holding labels only, for predefined selections: one block
    per key with ``samples[k]`` / ``properties[k]`` (``Labels`` or
    ``(names, values)``; None gives a single placeholder entry), what
    featomic users build with metatensor's ``TensorMap(keys, blocks)``."""
    keep = []
    keys = keys if isinstance(keys, Labels) else Labels(*keys)
    n = len(keys.values)

    def array(per_key):
        if per_key is None:
            return None
        if len(per_key) != n:
            raise ValueError("one Labels per key expected")
        arr = (C.mts_labels_t * max(1, n))()
        for k, labels in enumerate(per_key):
            arr[k] = _c_labels(labels, keep).contents
        keep.append(arr)
        return arr

    s, p = array(samples), array(properties)
    out = ctypes.c_void_p()
    C.check(C.lib().featomic_b200_labels_tensormap(_c_labels(keys, keep), s, p, ctypes.byref(out)))
    return TensorMap(out)


class System:
    """Atoms of one structure: atomic types, positions [n, 3] and the cell
    (3 x 3, rows are the cell vectors, all zero for a non-periodic system).
    ``pairs`` optionally supplies the caller's own half neighbour list, used
    with ``use_native_system=False`` (dict with first, second, distance,
    vector, shift)."""

    def __init__(self, types, positions, cell=None, pairs=None):
        self.types = np.ascontiguousarray(types, dtype=np.int32)
        self.positions = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
        self.cell = np.zeros(9) if cell is None else np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
        self.pairs = pairs

    @staticmethod
    def from_dict(d):
        if isinstance(d, System):
            return d
        return System(d["types"], d["positions"], d.get("cell"), d.get("pairs"))


class _CSystem:
    """featomic_system_t callbacks over a System (featomic/src/c_api/system.rs)."""

    def __init__(self, system):
        self.system = system
        s = system
        self._types = s.types
        self._positions = s.positions
        self._pairs_array = None
        if s.pairs is not None:
            n = len(s.pairs["first"])
            arr = (C.featomic_pair_t * max(n, 1))()
            for k in range(n):
                arr[k].first = int(s.pairs["first"][k])
                arr[k].second = int(s.pairs["second"][k])
                arr[k].distance = float(s.pairs["distance"][k])
                for x in range(3):
                    arr[k].vector[x] = float(s.pairs["vector"][k][x])
                    arr[k].cell_shift_indices[x] = int(s.pairs["shift"][k][x])
            self._pairs_array = arr
            self._pairs_count = n

        def size(_, out):
            out[0] = len(s.types)
            return 0

        def types(_, out):
            out[0] = self._types.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
            return 0

        def positions(_, out):
            out[0] = self._positions.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
            return 0

        def cell(_, out):
            for k in range(9):
                out[k] = s.cell[k]
            return 0

        def compute_neighbors(_, cutoff):
            return 0 if self._pairs_array is not None else -1

        def pairs(_, out, count):
            out[0] = ctypes.cast(self._pairs_array, ctypes.POINTER(C.featomic_pair_t))
            count[0] = self._pairs_count
            return 0

        def pairs_containing(_, atom, out, count):
            return -1

        self._callbacks = [C._size_cb(size), C._types_cb(types), C._positions_cb(positions), C._cell_cb(cell),
                           C._neighbors_cb(compute_neighbors), C._pairs_cb(pairs),
                           C._pairs_containing_cb(pairs_containing)]
        self.struct = C.featomic_system_t(None, *self._callbacks)


def _c_labels(labels, keep):
    """mts_labels_t view of a Labels (or (names, values)); `keep` holds the buffers."""
    if not isinstance(labels, Labels):
        labels = Labels(*labels)
    names = (ctypes.c_char_p * max(1, len(labels.names)))(*[n.encode() for n in labels.names])
    values = np.ascontiguousarray(labels.values, dtype=np.int32)
    c = C.mts_labels_t()
    c.names = ctypes.cast(names, ctypes.POINTER(ctypes.c_char_p))
    c.values = values.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    c.size = len(labels.names)
    c.count = values.shape[0]
    keep += [names, values, c]
    return ctypes.pointer(c)


def _selection(selection, target, keep):
    """featomic_labels_selection_t from None, Labels / (names, values) (a
    subset) or a TensorMap (predefined labels per block)."""
    if selection is None:
        return
    if isinstance(selection, TensorMap):
        target.predefined = selection._handle.value
        keep.append(selection)
    else:
        target.subset = _c_labels(selection, keep)


def _options(gradients, use_native_system, selected_samples=None, selected_properties=None, selected_keys=None):
    gradients = list(gradients or [])
    arr = (ctypes.c_char_p * max(1, len(gradients)))(*[g.encode() for g in gradients])
    opts = C.featomic_calculation_options_t()
    opts.gradients = ctypes.cast(arr, ctypes.POINTER(ctypes.c_char_p))
    opts.gradients_count = len(gradients)
    opts.use_native_system = bool(use_native_system)
    keep = [arr]
    _selection(selected_samples, opts.selected_samples, keep)
    _selection(selected_properties, opts.selected_properties, keep)
    if selected_keys is not None:
        opts.selected_keys = _c_labels(selected_keys, keep)
    return opts, keep


class CalculatorBase:
    def __init__(self, name, parameters):
        self._name = name
        if not isinstance(parameters, str):
            parameters = json.dumps(parameters)
        self._parameters = parameters
        handle = C.lib().featomic_calculator(name.encode(), parameters.encode())
        if not handle:
            message = C.lib().featomic_last_error().decode()
            raise C.FeatomicError(message, -1)
        self._handle = handle

    def __del__(self):
        if getattr(self, "_handle", None):
            try:
                C.lib().featomic_calculator_free(self._handle)
            except (AttributeError, TypeError):  # interpreter shutdown
                pass
            self._handle = None

    @property
    def name(self):
        buf = ctypes.create_string_buffer(256)
        C.check(C.lib().featomic_calculator_name(self._handle, buf, 256))
        return buf.value.decode()

    @property
    def parameters(self):
        size = len(self._parameters) + 1
        buf = ctypes.create_string_buffer(size)
        C.check(C.lib().featomic_calculator_parameters(self._handle, buf, size))
        return buf.value.decode()

    @property
    def cutoffs(self):
        ptr = ctypes.POINTER(ctypes.c_double)()
        count = ctypes.c_size_t()
        C.check(C.lib().featomic_calculator_cutoffs(self._handle, ctypes.byref(ptr), ctypes.byref(count)))
        return [ptr[i] for i in range(count.value)]

    def compute(self, systems, gradients=None, use_native_system=True, selected_samples=None,
                selected_properties=None, selected_keys=None):
        """Run the calculation on host systems; the result lives in host memory.
        Selections follow featomic's ``CalculatorBase.compute``
        (python/featomic/featomic/calculator_base.py:187+): ``Labels`` (or
        ``(names, values)``) select a subset, a ``TensorMap`` gives the labels
        of every block."""
        if isinstance(systems, (System, dict)):
            systems = [systems]
        csys = [_CSystem(System.from_dict(s)) for s in systems]
        arr = (C.featomic_system_t * max(1, len(csys)))(*[c.struct for c in csys])
        opts, keep = _options(gradients, use_native_system, selected_samples, selected_properties, selected_keys)
        out = ctypes.c_void_p()
        C.check(C.lib().featomic_calculator_compute(self._handle, ctypes.byref(out), arr, len(csys), opts))
        if not out.value:
            return None
        return TensorMap(out)

    def compute_device(self, positions, types, cells, system_sizes, gradients=None, stream=None,
                       selected_samples=None, selected_properties=None, selected_keys=None):
        """Run on positions already on the GPU (torch CUDA float64 tensor of
        shape [atoms, 3], all systems concatenated); the result stays on the
        GPU.  Selections as in ``compute``, applied on the device."""
        import torch
        assert positions.is_cuda and positions.dtype == torch.float64 and positions.is_contiguous()
        types = np.ascontiguousarray(types, dtype=np.int32)
        cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, 9)
        sizes = np.ascontiguousarray(system_sizes, dtype=np.uintp)
        dev = C.featomic_b200_device_systems_t()
        dev.n_systems = len(sizes)
        dev.system_sizes = sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t))
        dev.types = types.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
        dev.cells = cells.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
        dev.positions = positions.data_ptr()
        opts, keep = _options(gradients, True, selected_samples, selected_properties, selected_keys)
        if stream is None:
            stream = torch.cuda.current_stream().cuda_stream
        out = ctypes.c_void_p()
        C.check(C.lib().featomic_b200_calculator_compute_device(self._handle, ctypes.byref(out), ctypes.byref(dev),
                                                                opts, ctypes.c_void_p(stream)))
        return TensorMap(out)

    def radial_integral(self, r):
        """(values, gradients, knots): the radial integral the kernels use,
        evaluated on the host, shapes [len(r), max_angular + 1, max_radial + 1]."""
        h = json.loads(self._parameters)
        L = h["basis"].get("max_angular", 0)
        N = h["basis"]["radial"]["max_radial"] + 1
        r = np.ascontiguousarray(r, dtype=np.float64)
        values = np.zeros((len(r), L + 1, N))
        grads = np.zeros((len(r), L + 1, N))
        knots = np.zeros(L + 1, dtype=np.int32)
        dp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
        C.check(C.lib().featomic_b200_radial_integral(self._handle, dp(r), len(r), dp(values), dp(grads),
                                                      knots.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))))
        return values, grads, knots

    def timings(self):
        """Per-phase time (ms) of the last call."""
        out = (ctypes.c_double * 12)()
        C.check(C.lib().featomic_b200_calculator_timings(self._handle, out, 12))
        names = ["neighbors", "metadata", "features", "expansion", "contraction", "transfer", "total",
                 "ps_values", "ps_positions", "ps_strain_cell", "metadata_before_launch", "labels"]
        return dict(zip(names, list(out)))


class SphericalExpansion(CalculatorBase):
    def __init__(self, cutoff, density, basis):
        super().__init__("spherical_expansion", {"cutoff": cutoff, "density": density, "basis": basis})


class LodeSphericalExpansion(CalculatorBase):
    """featomic's ``lode_spherical_expansion``: long-range expansion of a
    smeared power-law density in periodic systems, computed in reciprocal
    space (featomic/src/calculators/lode/spherical_expansion.rs).  Keys
    (o3_lambda, o3_sigma, center_type, neighbor_type), samples (system,
    atom), positions gradients only."""

    def __init__(self, density, basis, k_cutoff=None):
        parameters = {"density": density, "basis": basis}
        if k_cutoff is not None:
            parameters["k_cutoff"] = k_cutoff
        super().__init__("lode_spherical_expansion", parameters)


class SphericalExpansionByPair(CalculatorBase):
    """featomic's ``spherical_expansion_by_pair``: one row per pair and
    direction, keys (o3_lambda, o3_sigma, first_atom_type, second_atom_type),
    samples (system, first_atom, second_atom, cell_shift_a/b/c)
    (featomic/src/calculators/soap/spherical_expansion_pair.rs)."""

    def __init__(self, cutoff, density, basis):
        super().__init__("spherical_expansion_by_pair", {"cutoff": cutoff, "density": density, "basis": basis})


class SoapPowerSpectrum(CalculatorBase):
    def __init__(self, cutoff, density, basis):
        super().__init__("soap_power_spectrum", {"cutoff": cutoff, "density": density, "basis": basis})


class SoapRadialSpectrum(CalculatorBase):
    """featomic's ``soap_radial_spectrum``: the l = 0 spherical expansion, keys
    (center_type, neighbor_type), properties n, no components
    (featomic/src/calculators/soap/radial_spectrum.rs).  ``basis`` is
    ``{"radial": {"type": "Gto", "max_radial": n}, "spline_accuracy": ...}``."""

    def __init__(self, cutoff, density, basis):
        super().__init__("soap_radial_spectrum", {"cutoff": cutoff, "density": density, "basis": basis})


def neighbor_list(positions, cell, cutoff):
    """Half neighbour list of one system from the GPU cell list: dict of
    numpy arrays (first, second, distance, vector, shift), ordered by
    (first, second, shift)."""
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    cell = np.ascontiguousarray(cell, dtype=np.float64).reshape(9)
    count = ctypes.c_size_t()
    dptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))  # noqa: E731
    status = C.lib().featomic_b200_neighbor_list(dptr(pos), len(pos), dptr(cell), float(cutoff), None, 0,
                                                 ctypes.byref(count))
    if status not in (0, 254):
        C.check(status)
    n = count.value
    arr = (C.featomic_pair_t * max(n, 1))()
    C.check(C.lib().featomic_b200_neighbor_list(dptr(pos), len(pos), dptr(cell), float(cutoff), arr, n,
                                                ctypes.byref(count)))
    raw = np.ctypeslib.as_array(arr)[:n]
    return {
        "first": raw["first"].astype(np.int64), "second": raw["second"].astype(np.int64),
        "distance": raw["distance"].copy(), "vector": raw["vector"].copy(),
        "shift": raw["cell_shift_indices"].astype(np.int32),
    }


def profiling_enable(enabled=True):
    C.check(C.lib().featomic_profiling_enable(enabled))


def profiling_clear():
    C.check(C.lib().featomic_profiling_clear())


def profiling_get(format="table"):
    buf = ctypes.create_string_buffer(1 << 16)
    C.check(C.lib().featomic_profiling_get(format.encode(), buf, 1 << 16))
    return buf.value.decode()
