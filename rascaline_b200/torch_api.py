"""featomic-torch style interface with an adjoint backward pass.

Mirrors featomic-torch (``featomic-torch/include/featomic/torch/calculator.hpp``,
``featomic-torch/src/calculator.cpp:190-383``): a calculator built from
``(name, hypers)`` whose ``compute(systems)`` returns the SOAP power spectrum
as a TensorMap of torch blocks connected to the systems' positions and cells
in torch's autograd graph.

featomic-torch's backward (``featomic-torch/src/autograd.cpp:237-317`` for
positions, ``:429-503`` for the cell) contracts dL/dX with materialised
explicit gradient blocks.  Here the backward pass is
``featomic_b200_power_spectrum_dense_backward``: a CUDA adjoint that recomputes
the per-pair terms and never builds the gradient blocks.  The forward runs in
FP64 (``precision=64``, the drop-in values) or in FP32 (``precision=32``).

Double backward follows featomic-torch (``PositionsGrad`` / ``CellGrad`` are
themselves autograd functions, ``autograd.cpp:22-54``, ``:318-426``): the
backward pass is differentiable with respect to its input dL/dX, through the
forward-mode derivative of X (``featomic_b200_dense_jvp``), so that losses on
forces and virials train the model that produced dL/dX.  Second derivatives
with respect to positions and cell are not computed; a warning says so, as in
featomic-torch.
"""
import ctypes
import json
import warnings

import numpy as np
import torch

from . import _c_api as C
from .calculators import CalculatorBase, Labels

__all__ = ["System", "Calculator", "SoapPowerSpectrum", "SphericalExpansion", "TorchTensorMap", "TorchBlock", "Batch",
           "dense_power_spectrum", "dense_spherical_expansion", "dense_jvp", "register_autograd"]


class System:
    """Atomic types, positions [n, 3] and cell [3, 3] (rows are the cell
    vectors; all zero for a non-periodic system) as torch tensors."""

    def __init__(self, types, positions, cell=None):
        self.types = torch.as_tensor(types, dtype=torch.int32).reshape(-1)
        self.positions = positions
        if cell is None:
            cell = torch.zeros((3, 3), dtype=positions.dtype, device=positions.device)
        self.cell = cell

    def __len__(self):
        return len(self.types)


class DenseState:
    """A forward pass kept for its backward pass (featomic_b200_dense_t)."""

    def __init__(self, handle, calculator):
        self._handle = handle
        # the state refers to its calculator's device tables and must be
        # freed before it (featomic_b200_dense_free): keep the calculator alive
        self._calculator = calculator
        n = [ctypes.c_size_t() for _ in range(5)]
        C.check(C.lib().featomic_b200_dense_shape(handle, *[ctypes.byref(x) for x in n]))
        self.n_atoms, self.n_species, self.n_keys, self.n_properties, self.n_pairs = [x.value for x in n]

    def species(self, with_counts=False):
        species = np.zeros(max(1, self.n_species), dtype=np.int32)
        counts = np.zeros((max(1, self.n_atoms), max(1, self.n_species)), dtype=np.int32)
        ptr = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))  # noqa: E731
        C.check(C.lib().featomic_b200_dense_species(self._handle, ptr(species),
                                                     ptr(counts) if with_counts else None))
        species = species[:self.n_species]
        if with_counts:
            return species, counts[:self.n_atoms, :self.n_species]
        return species

    def __del__(self):
        if getattr(self, "_handle", None):
            try:
                C.lib().featomic_b200_dense_free(self._handle)
            except (AttributeError, TypeError):  # interpreter shutdown
                pass
            self._handle = None


def _device_systems(positions, types, cells, sizes):
    dev = C.featomic_b200_device_systems_t()
    dev.n_systems = len(sizes)
    dev.system_sizes = sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t))
    dev.types = types.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))
    dev.cells = cells.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    dev.positions = positions.data_ptr()
    return dev


def dense_power_spectrum(calculator, positions, types, cells, sizes, precision=64, species=None):
    """Forward pass without autograd: (values [n_atoms, n_keys, n_properties]
    torch tensor on the GPU, DenseState).  ``positions``: CUDA float64 tensor
    [atoms, 3] of all systems; ``types`` [atoms]; ``cells`` [systems, 9] and
    ``sizes`` [systems] on the host."""
    if not (positions.is_cuda and positions.dtype == torch.float64 and positions.is_contiguous()):
        raise ValueError("positions must be a contiguous CUDA float64 tensor")
    types = np.ascontiguousarray(types, dtype=np.int32)
    cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, 9)
    sizes = np.ascontiguousarray(sizes, dtype=np.uintp)
    if species is None:
        sp = np.unique(types).astype(np.int32)
    else:
        sp = np.unique(np.asarray(species, dtype=np.int32)).astype(np.int32)
    S = len(sp)
    params = json.loads(calculator._parameters)
    if params["basis"].get("type") == "Explicit":
        raise C.FeatomicError("the dense power spectrum does not support the Explicit basis", 1)
    L = params["basis"]["max_angular"]
    N = params["basis"]["radial"]["max_radial"] + 1
    n_keys, n_props = S * (S + 1) // 2, (L + 1) * N * N
    dtype = torch.float64 if precision == 64 else torch.float32
    values = torch.empty((len(types), n_keys, n_props), dtype=dtype, device=positions.device)
    dev = _device_systems(positions, types, cells, sizes)
    handle = ctypes.c_void_p()
    stream = torch.cuda.current_stream(positions.device).cuda_stream
    C.check(C.lib().featomic_b200_power_spectrum_dense(
        calculator._handle, ctypes.byref(dev), sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), S, precision,
        values.data_ptr(), values.numel(), ctypes.byref(handle), ctypes.c_void_p(stream)))
    return values, DenseState(handle, calculator)


def dense_backward(state, grad_values, n_systems, strain=False, cell=True):
    """(dL/dpositions [atoms, 3], dL/dstrain [systems, 3, 3] or None,
    dL/dcell [systems, 3, 3] or None) for dL/dvalues ``grad_values``."""
    grad_values = grad_values.contiguous()
    device, dtype = grad_values.device, grad_values.dtype
    gpos = torch.empty((state.n_atoms, 3), dtype=dtype, device=device)
    gstrain = torch.empty((n_systems, 3, 3), dtype=dtype, device=device) if strain else None
    gcell = torch.empty((n_systems, 3, 3), dtype=dtype, device=device) if cell else None
    ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else None)  # noqa: E731
    stream = torch.cuda.current_stream(device).cuda_stream
    C.check(C.lib().featomic_b200_power_spectrum_dense_backward(
        state._handle, ptr(grad_values), ptr(gpos), ptr(gstrain), ptr(gcell), ctypes.c_void_p(stream)))
    return gpos, gstrain, gcell


def dense_spherical_expansion(calculator, positions, types, cells, sizes, precision=64, species=None):
    """Forward pass of a spherical_expansion calculator without autograd:
    (coefficients [n_atoms, n_species, (lmax + 1)^2 nmax] torch tensor on the
    GPU, DenseState); arguments as dense_power_spectrum."""
    if not (positions.is_cuda and positions.dtype == torch.float64 and positions.is_contiguous()):
        raise ValueError("positions must be a contiguous CUDA float64 tensor")
    types = np.ascontiguousarray(types, dtype=np.int32)
    cells = np.ascontiguousarray(cells, dtype=np.float64).reshape(-1, 9)
    sizes = np.ascontiguousarray(sizes, dtype=np.uintp)
    if species is None:
        sp = np.unique(types).astype(np.int32)
    else:
        sp = np.unique(np.asarray(species, dtype=np.int32)).astype(np.int32)
    params = json.loads(calculator._parameters)
    if params["basis"].get("type") == "Explicit":
        raise C.FeatomicError("the dense spherical expansion does not support the Explicit basis", 1)
    L = params["basis"]["max_angular"]
    N = params["basis"]["radial"]["max_radial"] + 1
    dtype = torch.float64 if precision == 64 else torch.float32
    values = torch.empty((len(types), len(sp), (L + 1) ** 2 * N), dtype=dtype, device=positions.device)
    dev = _device_systems(positions, types, cells, sizes)
    handle = ctypes.c_void_p()
    stream = torch.cuda.current_stream(positions.device).cuda_stream
    C.check(C.lib().featomic_b200_spherical_expansion_dense(
        calculator._handle, ctypes.byref(dev), sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), len(sp), precision,
        values.data_ptr(), values.numel(), ctypes.byref(handle), ctypes.c_void_p(stream)))
    return values, DenseState(handle, calculator)


def expansion_backward(state, grad_coefficients, n_systems, strain=False, cell=True):
    """dense_backward for a spherical-expansion state: dL/dcoefficients to
    (dL/dpositions, dL/dstrain or None, dL/dcell or None)."""
    grad_coefficients = grad_coefficients.contiguous()
    device, dtype = grad_coefficients.device, grad_coefficients.dtype
    gpos = torch.empty((state.n_atoms, 3), dtype=dtype, device=device)
    gstrain = torch.empty((n_systems, 3, 3), dtype=dtype, device=device) if strain else None
    gcell = torch.empty((n_systems, 3, 3), dtype=dtype, device=device) if cell else None
    ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else None)  # noqa: E731
    stream = torch.cuda.current_stream(device).cuda_stream
    C.check(C.lib().featomic_b200_spherical_expansion_dense_backward(
        state._handle, ptr(grad_coefficients), ptr(gpos), ptr(gstrain), ptr(gcell), ctypes.c_void_p(stream)))
    return gpos, gstrain, gcell


def dense_jvp(state, tangent_positions, tangent_cell=None, values=True, coefficients=False, dtype=None):
    """Forward-mode derivative of a dense forward pass along a displacement
    of the positions [atoms, 3] (and cells [systems, 3, 3]): (tangent of the
    power spectrum or None, tangent of the expansion coefficients or None)."""
    dtype = dtype or tangent_positions.dtype
    device = tangent_positions.device
    tpos = tangent_positions.to(dtype).contiguous()
    tcell = tangent_cell.to(dtype).contiguous() if tangent_cell is not None else None
    n = state.n_atoms
    tv = torch.empty((n, state.n_keys, state.n_properties), dtype=dtype, device=device) if values else None
    tc = None
    if coefficients:
        tc = torch.empty((n, state.n_species, state.expansion_width), dtype=dtype, device=device)
    ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else None)  # noqa: E731
    stream = torch.cuda.current_stream(device).cuda_stream
    C.check(C.lib().featomic_b200_dense_jvp(state._handle, ptr(tpos), ptr(tcell), ptr(tc), ptr(tv),
                                            ctypes.c_void_p(stream)))
    return tv, tc


SECOND_DERIVATIVE_WARNING = ("second derivatives with respect to {} are not implemented and will not be accumulated "
                             "during backward() calls")


class _DenseAdjoint(torch.autograd.Function):
    """The adjoint backward pass as a function of dL/dX (the power spectrum
    or the expansion coefficients), differentiable with respect to dL/dX: its
    own backward pass is the forward-mode derivative of X along the incoming
    gradients of dL/dpositions and dL/dcell."""

    @staticmethod
    def forward(ctx, grad_out, positions, cells, state, n_systems, need_cell, expansion):
        if expansion:
            gpos, _, gcell = expansion_backward(state, grad_out, n_systems, strain=False, cell=need_cell)
        else:
            gpos, _, gcell = dense_backward(state, grad_out, n_systems, strain=False, cell=need_cell)
        if gcell is None:
            gcell = torch.zeros((n_systems, 3, 3), dtype=gpos.dtype, device=gpos.device)
        ctx.state = state
        ctx.expansion = expansion
        ctx.need_cell = need_cell
        ctx.precision_dtype = grad_out.dtype
        return gpos.to(positions.dtype), gcell.to(cells.dtype)

    @staticmethod
    def backward(ctx, d_gpos, d_gcell):
        if ctx.needs_input_grad[1]:
            warnings.warn(SECOND_DERIVATIVE_WARNING.format("positions"), stacklevel=2)
        if ctx.needs_input_grad[2]:
            warnings.warn(SECOND_DERIVATIVE_WARNING.format("cell matrix"), stacklevel=2)
        d_grad_out = None
        if ctx.needs_input_grad[0]:
            st = ctx.state
            dtype = ctx.precision_dtype
            if d_gpos is None:
                d_gpos = torch.zeros((st.n_atoms, 3), dtype=dtype, device="cuda")
            if not ctx.need_cell:
                d_gcell = None  # the cell output was zeros, not a function of dL/dX
            tv, tc = dense_jvp(st, d_gpos, d_gcell, values=not ctx.expansion, coefficients=ctx.expansion, dtype=dtype)
            d_grad_out = tc if ctx.expansion else tv
        return d_grad_out, None, None, None, None, None, None


class _DenseForward(torch.autograd.Function):
    """positions [atoms, 3], cells [systems, 3, 3] -> dense power spectrum or
    expansion coefficients; the backward pass is the CUDA adjoint."""

    @staticmethod
    def forward(ctx, positions, cells, calculator, types, sizes, precision, species, holder, expansion):
        pos = positions.detach().to(torch.float64).contiguous()
        cell_host = cells.detach().to(torch.float64).cpu().numpy().reshape(-1, 9)
        run = dense_spherical_expansion if expansion else dense_power_spectrum
        values, state = run(calculator, pos, types, cell_host, sizes, precision, species)
        if expansion:
            state.expansion_width = values.shape[2]
        holder.append(state)
        ctx.state = state
        ctx.n_systems = len(sizes)
        ctx.expansion = expansion
        ctx.save_for_backward(positions, cells)
        return values

    @staticmethod
    def backward(ctx, grad_values):
        need_pos, need_cell = ctx.needs_input_grad[0], ctx.needs_input_grad[1]
        positions, cells = ctx.saved_tensors
        gpos, gcell = _DenseAdjoint.apply(grad_values.contiguous(), positions, cells, ctx.state, ctx.n_systems,
                                          need_cell, ctx.expansion)
        return gpos if need_pos else None, gcell if need_cell else None, None, None, None, None, None, None, None


class TorchBlock:
    def __init__(self, values, samples, properties, components=None, gradients=None):
        self.values = values
        self.samples = samples
        self.properties = properties
        self.components = components or []
        self._gradients = dict(gradients or {})

    def gradient(self, parameter):
        return self._gradients[parameter]

    def gradients_list(self):
        return list(self._gradients)


class _ExplicitGradients(torch.autograd.Function):
    """featomic-torch's FeatomicAutograd (autograd.cpp:99-233) with the
    contractions of PositionsGrad (:237-317) and CellGrad (:429-503): the
    block's values, whose backward contracts dA/dX with the precomputed
    explicit gradient blocks, on the device.  The backward is written with
    differentiable torch operations, so it is itself differentiable with
    respect to dA/dX (double backward, :318-426); second derivatives with
    respect to positions and cells are zero here, with featomic-torch's
    warning."""

    @staticmethod
    def forward(ctx, positions, cells, values, grad_samples, grad_values, atom_start, cell_values, sample_systems):
        ctx.save_for_backward(grad_samples, grad_values, atom_start, cell_values, sample_systems)
        ctx.shapes = (positions.shape, cells.shape)
        return values.detach().clone()

    @staticmethod
    def backward(ctx, dA_dX):
        grad_samples, grad_values, atom_start, cell_values, sample_systems = ctx.saved_tensors
        pos_shape, cell_shape = ctx.shapes
        dA_dr = dA_dH = None
        flat = dA_dX.reshape(dA_dX.shape[0], -1)
        if ctx.needs_input_grad[0]:
            if torch.is_grad_enabled():
                warnings.warn("second derivatives with respect to positions are not implemented and will not be "
                              "accumulated during backward() calls", stacklevel=2)
            rows = grad_values.reshape(grad_values.shape[0], 3, -1)
            sample = grad_samples[:, 0].long()
            atom = atom_start[grad_samples[:, 1].long()] + grad_samples[:, 2].long()
            contrib = torch.einsum("rxf,rf->rx", rows.to(flat.dtype), flat[sample])
            dA_dr = torch.zeros(pos_shape, dtype=flat.dtype, device=flat.device).index_add(0, atom, contrib)
        if ctx.needs_input_grad[1]:
            if torch.is_grad_enabled():
                warnings.warn("second derivatives with respect to cell matrix are not implemented and will not be "
                              "accumulated during backward() calls", stacklevel=2)
            rows = cell_values.reshape(cell_values.shape[0], 3, 3, -1)
            contrib = torch.einsum("sabf,sf->sab", rows.to(flat.dtype), flat)
            dA_dH = torch.zeros(cell_shape, dtype=flat.dtype, device=flat.device).index_add(
                0, sample_systems.long(), contrib)
        return dA_dr, dA_dH, None, None, None, None, None, None


def register_autograd(systems, precomputed, forward_gradients=None):
    """featomic-torch's ``register_autograd(systems, precomputed,
    forward_gradients)`` (featomic-torch/src/calculator.cpp:314-383): connect
    the blocks of a TensorMap computed with explicit gradients (``compute`` /
    ``compute_device`` with ``gradients=["positions", "cell"]``) to the
    systems' positions and cells in torch's autograd graph.  Returns a
    TorchTensorMap whose block values carry autograd and which keeps the
    gradients listed in ``forward_gradients`` (all of the precomputed ones
    when None)."""
    if isinstance(systems, System):
        systems = [systems]
    blocks = precomputed.blocks()
    if len(blocks) == 0:
        return precomputed
    positions = torch.cat([s.positions.reshape(-1, 3) for s in systems])
    cells = torch.stack([s.cell.reshape(3, 3) for s in systems])
    available = blocks[0].gradients_list()
    if positions.requires_grad and "positions" not in available:
        raise ValueError("expected the precomputed TensorMap to contain gradients with respect to 'positions' "
                         "since one of the system `requires_grad` for its positions")
    if cells.requires_grad and "cell" not in available:
        raise ValueError("expected the precomputed TensorMap to contain gradients with respect to 'cell' since "
                         "one of the system `requires_grad` for its cell")
    keep = available if forward_gradients is None else list(forward_gradients)
    starts = torch.tensor(np.concatenate([[0], np.cumsum([len(s) for s in systems])[:-1]]), dtype=torch.long,
                          device=positions.device)
    empty = torch.zeros(0, device=positions.device)
    out = []
    for block in blocks:
        values = torch.as_tensor(block.values, device=positions.device)
        samples = torch.as_tensor(np.asarray(block.samples.values), device=positions.device)
        gs = gv = cv = empty
        if positions.requires_grad:
            g = block.gradient("positions")
            gs = torch.as_tensor(np.asarray(g.samples.values), device=positions.device)
            gv = torch.as_tensor(g.values, device=positions.device)
        if cells.requires_grad:
            cv = torch.as_tensor(block.gradient("cell").values, device=positions.device)
        attached = _ExplicitGradients.apply(positions, cells, values, gs, gv, starts, cv,
                                            samples[:, 0] if len(samples) else empty)
        grads = {name: block.gradient(name) for name in keep if name in available}
        out.append(TorchBlock(attached, block.samples, block.properties, list(block.components), grads))
    return TorchTensorMap(precomputed.keys, out)


class TorchTensorMap:
    def __init__(self, keys, blocks):
        self.keys = keys
        self._blocks = blocks

    def __len__(self):
        return len(self._blocks)

    def block(self, index):
        return self._blocks[index]

    def blocks(self):
        return list(self._blocks)


class Calculator:
    """featomic-torch's CalculatorHolder for the SOAP power spectrum and the
    spherical expansion."""

    def __init__(self, name, parameters, precision=64, species=None):
        if name not in ("soap_power_spectrum", "spherical_expansion"):
            raise ValueError("the torch interface of featomic-b200 supports soap_power_spectrum and "
                             f"spherical_expansion, not {name}")
        if precision not in (32, 64):
            raise ValueError("precision must be 32 or 64")
        self._calculator = CalculatorBase(name, parameters)
        self._registry_name = name
        self.hypers = parameters if isinstance(parameters, dict) else json.loads(parameters)
        self.precision = precision
        self.species = None if species is None else sorted(set(int(s) for s in species))

    @property
    def name(self):
        return self._calculator.name

    @property
    def parameters(self):
        return self._calculator.parameters

    def _gather(self, systems):
        if isinstance(systems, System):
            systems = [systems]
        positions = torch.cat([s.positions.reshape(-1, 3) for s in systems])
        cells = torch.stack([s.cell.reshape(3, 3) for s in systems])
        types = np.concatenate([s.types.cpu().numpy() for s in systems]).astype(np.int32)
        sizes = np.array([len(s) for s in systems], dtype=np.uintp)
        return systems, positions, cells, types, sizes

    @property
    def _expansion(self):
        return self._registry_name == "spherical_expansion"

    def dense(self, systems):
        """Dense power spectrum [atoms, n_keys, n_properties] (or expansion
        coefficients [atoms, n_species, (lmax + 1)^2 nmax]) of all systems
        (see featomic_b200_power_spectrum_dense for the layout), differentiable
        w.r.t. the positions and cells."""
        systems, positions, cells, types, sizes = self._gather(systems)
        return _DenseForward.apply(positions, cells, self._calculator, types, sizes, self.precision, self.species, [],
                                   self._expansion)

    def compute(self, systems):
        """featomic's TensorMap layout.  Power spectrum: keys (center_type,
        neighbor_1_type, neighbor_2_type), samples (system, atom) of the
        centres that have both neighbour types, properties (l, n_1, n_2).
        Spherical expansion: keys (o3_lambda, o3_sigma, center_type,
        neighbor_type), samples (system, atom) of the centres that have the
        neighbour type, components (o3_mu), properties (n)."""
        systems, positions, cells, types, sizes = self._gather(systems)
        holder = []
        values = _DenseForward.apply(positions, cells, self._calculator, types, sizes, self.precision, self.species,
                                     holder, self._expansion)
        # which neighbour species every atom has, from the forward pass
        species, counts = holder[0].species(with_counts=True)
        S = len(species)
        present = counts > 0
        own = np.searchsorted(species, types)
        present[np.arange(len(types)), own] = True
        system_of = np.repeat(np.arange(len(sizes)), sizes.astype(np.int64))
        atom_of = np.concatenate([np.arange(n) for n in sizes.astype(np.int64)]) if len(types) else np.zeros(0, int)
        L = self.hypers["basis"]["max_angular"]
        N = self.hypers["basis"]["radial"]["max_radial"] + 1
        if self._expansion:
            return self._expansion_blocks(values, species, present, own, system_of, atom_of, L, N)
        properties = Labels(["l", "n_1", "n_2"],
                            [[l, n1, n2] for l in range(L + 1) for n1 in range(N) for n2 in range(N)])
        keys, blocks = [], []
        key = 0
        key_of = {}
        for a in range(S):
            for b in range(a, S):
                key_of[(a, b)] = key
                key += 1
        for c in range(S):
            centres = own == c
            for a in range(S):
                for b in range(a, S):
                    rows = np.nonzero(centres & present[:, a] & present[:, b])[0]
                    if len(rows) == 0:
                        continue
                    index = torch.as_tensor(rows, device=values.device)
                    block_values = values[index, key_of[(a, b)], :]
                    samples = Labels(["system", "atom"], np.stack([system_of[rows], atom_of[rows]], axis=1))
                    keys.append([species[c], species[a], species[b]])
                    blocks.append(TorchBlock(block_values, samples, properties))
        return TorchTensorMap(Labels(["center_type", "neighbor_1_type", "neighbor_2_type"], keys), blocks)

    @staticmethod
    def _expansion_blocks(values, species, present, own, system_of, atom_of, L, N):
        # keys (l, 1, center, neighbour) with l varying fastest
        # (featomic/src/calculators/soap/spherical_expansion.rs:662-742)
        S = len(species)
        properties = Labels(["n"], [[n] for n in range(N)])
        keys, blocks = [], []
        for c in range(S):
            for t in range(S):
                rows = np.nonzero((own == c) & present[:, t])[0]
                if len(rows) == 0:
                    continue
                index = torch.as_tensor(rows, device=values.device)
                samples = Labels(["system", "atom"], np.stack([system_of[rows], atom_of[rows]], axis=1))
                for l in range(L + 1):
                    block_values = values[index, t, l * l * N:(l + 1) * (l + 1) * N].reshape(len(rows), 2 * l + 1, N)
                    components = [Labels(["o3_mu"], [[m] for m in range(-l, l + 1)])]
                    keys.append([l, 1, species[c], species[t]])
                    blocks.append(TorchBlock(block_values, samples, properties, components))
        return TorchTensorMap(Labels(["o3_lambda", "o3_sigma", "center_type", "neighbor_type"], keys), blocks)


class SoapPowerSpectrum(Calculator):
    def __init__(self, cutoff, density, basis, precision=64, species=None):
        super().__init__("soap_power_spectrum", {"cutoff": cutoff, "density": density, "basis": basis},
                         precision=precision, species=species)


class SphericalExpansion(Calculator):
    def __init__(self, cutoff, density, basis, precision=64, species=None):
        super().__init__("spherical_expansion", {"cutoff": cutoff, "density": density, "basis": basis},
                         precision=precision, species=species)


class Batch:
    """Many non-periodic systems (molecules) through one persistent launch
    replayed from a captured CUDA graph, FP32 arithmetic
    (``featomic_b200_batch_*``).  ``sizes`` and ``types`` describe the
    systems; the positions can change between runs."""

    def __init__(self, calculator, sizes, types, species=None):
        calc = calculator._calculator if isinstance(calculator, Calculator) else calculator
        self._calculator = calc
        sizes = np.ascontiguousarray(sizes, dtype=np.uintp)
        types = np.ascontiguousarray(types, dtype=np.int32)
        sp = None if species is None else np.ascontiguousarray(sorted(set(int(s) for s in species)), dtype=np.int32)
        handle = ctypes.c_void_p()
        C.check(C.lib().featomic_b200_batch_create(
            calc._handle, len(sizes), sizes.ctypes.data_as(ctypes.POINTER(ctypes.c_size_t)),
            types.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            sp.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)) if sp is not None else None,
            0 if sp is None else len(sp), ctypes.byref(handle)))
        self._handle = handle
        n = [ctypes.c_size_t() for _ in range(5)]
        C.check(C.lib().featomic_b200_batch_shape(handle, *[ctypes.byref(x) for x in n]))
        self.n_atoms, self.n_systems, self.n_species, self.n_keys, self.n_properties = [x.value for x in n]

    def __del__(self):
        if getattr(self, "_handle", None):
            try:
                C.lib().featomic_b200_batch_free(self._handle)
            except (AttributeError, TypeError):  # interpreter shutdown
                pass
            self._handle = None

    def outputs(self, device="cuda", values=True, gradients=True, energies=True, strain=False):
        """Output buffers for run(): a dict of float32 CUDA tensors."""
        out = {}
        if values:
            out["values"] = torch.empty((self.n_atoms, self.n_keys, self.n_properties), dtype=torch.float32,
                                        device=device)
        if gradients:
            out["gradients"] = torch.empty((self.n_atoms, 3), dtype=torch.float32, device=device)
        if energies:
            out["energies"] = torch.empty(self.n_systems, dtype=torch.float32, device=device)
        if strain:
            out["strain"] = torch.empty((self.n_systems, 3, 3), dtype=torch.float32, device=device)
        return out

    def _pointers(self, positions, weights, grad_values, out):
        if not (positions.is_cuda and positions.dtype == torch.float64 and positions.is_contiguous()):
            raise ValueError("positions must be a contiguous CUDA float64 tensor")
        for t in (weights, grad_values):
            if t is not None and not (t.is_cuda and t.dtype == torch.float32 and t.is_contiguous()):
                raise ValueError("weights / grad_values must be contiguous CUDA float32 tensors")
        ptr = lambda t: ctypes.c_void_p(t.data_ptr() if t is not None else None)  # noqa: E731
        return [ptr(positions), ptr(weights), ptr(grad_values), ptr(out.get("values")), ptr(out.get("gradients")),
                ptr(out.get("energies")), ptr(out.get("strain"))]

    def run(self, positions, out, weights=None, grad_values=None):
        """One graph replay on the current stream, filling the tensors of ``out``."""
        stream = ctypes.c_void_p(torch.cuda.current_stream(positions.device).cuda_stream)
        C.check(C.lib().featomic_b200_batch_run(self._handle, *self._pointers(positions, weights, grad_values, out),
                                                 stream))
        return out

    def tune(self, positions, out, weights=None, grad_values=None):
        """Time every launch configuration and keep the fastest; returns ms per run."""
        stream = ctypes.c_void_p(torch.cuda.current_stream(positions.device).cuda_stream)
        best = ctypes.c_double()
        C.check(C.lib().featomic_b200_batch_tune(self._handle, *self._pointers(positions, weights, grad_values, out),
                                                  stream, ctypes.byref(best)))
        return best.value

    @property
    def config(self):
        c = (ctypes.c_int32 * 5)()
        C.check(C.lib().featomic_b200_batch_config(self._handle, c))
        return {"warps": c[0], "chunk": c[1], "layout": c[2], "ctas_per_sm": c[3], "pipeline": c[4]}

    @config.setter
    def config(self, value):
        c = (ctypes.c_int32 * 5)(value["warps"], value["chunk"], value["layout"], value["ctas_per_sm"],
                                 value.get("pipeline", 0))
        C.check(C.lib().featomic_b200_batch_set_config(self._handle, c))

    def status(self):
        s = ctypes.c_int32()
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        C.check(C.lib().featomic_b200_batch_status(self._handle, stream, ctypes.byref(s)))
        return s.value
