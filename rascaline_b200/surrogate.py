"""Learned radial surrogate (``featomic_b200_surrogate_*``).

An MLP r -> R_nl(r) for every (l, n) of a calculator's radial basis,
1 -> 64 -> 64 -> (max_angular + 1)(max_radial + 1) with SiLU activations,
trained on the GPU by this library's own kernels on exact (analytic GTO)
radial integrals (Adam, then :meth:`RadialSurrogate.fit_output_layer`, a
least-squares refit of the linear output layer on values and derivatives),
evaluated on the tensor cores with BF16 operands, each weight and activation
a sum of three BF16 parts, and FP32 accumulation.  Attached to a calculator
with :meth:`RadialSurrogate.attach`, it replaces the spline in the FP32 dense
power spectrum and its adjoint.
"""
import ctypes

import numpy as np

from . import _c_api as C

# "bf16_single": the CUDA cores with W2 and W3 rounded to one BF16 each, the
# control that shows what three-part operands buy
METHODS = {"tensor_cores": 0, "cuda_cores": 1, "spline": 2, "analytic": 3, "bf16_single": 4}


def _stream():
    import torch
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


class RadialSurrogate:
    def __init__(self, calculator, hidden=64, seed=1):
        self._calculator = calculator
        handle = ctypes.c_void_p()
        C.check(C.lib().featomic_b200_surrogate_create(calculator._handle, hidden, seed, ctypes.byref(handle)))
        self._handle = handle

    def __del__(self):
        if getattr(self, "_handle", None):
            try:
                C.lib().featomic_b200_surrogate_free(self._handle)
            except (AttributeError, TypeError):  # interpreter shutdown
                pass
            self._handle = None

    def _shape(self):
        n = [ctypes.c_size_t() for _ in range(3)]
        C.check(C.lib().featomic_b200_surrogate_shape(self._handle, *[ctypes.byref(x) for x in n]))
        return [x.value for x in n]

    @property
    def n_outputs(self):
        return self._shape()[0]

    @property
    def n_parameters(self):
        return self._shape()[1]

    @property
    def n_samples(self):
        return self._shape()[2]

    def make_dataset(self, n_samples=1 << 20, seed=7):
        C.check(C.lib().featomic_b200_surrogate_dataset(self._handle, n_samples, seed, _stream()))

    def train(self, steps, batch=8192, learning_rate=3e-3, derivative_weight=0.1):
        """Adam steps; the loss is the mean squared error of the normalised
        outputs plus ``derivative_weight`` times that of their derivatives
        with respect to x = 2 r / cutoff - 1.  Returns the last loss."""
        C.check(C.lib().featomic_b200_surrogate_set_derivative_weight(self._handle, float(derivative_weight)))
        loss = ctypes.c_double()
        C.check(C.lib().featomic_b200_surrogate_train(self._handle, steps, batch, learning_rate, ctypes.byref(loss),
                                                       _stream()))
        return loss.value

    def fit_output_layer(self, derivative_weight=0.01):
        """Refit W3 and b3 by least squares over the whole training set:
        squared error of the normalised outputs plus ``derivative_weight``
        times that of their r-derivatives (FP64 normal equations on the GPU)."""
        C.check(C.lib().featomic_b200_surrogate_fit_output_layer(self._handle, float(derivative_weight), _stream()))

    def loss_and_gradient(self, n, derivative_weight=0.1):
        C.check(C.lib().featomic_b200_surrogate_set_derivative_weight(self._handle, float(derivative_weight)))
        grad = np.zeros(self.n_parameters, dtype=np.float32)
        loss = ctypes.c_double()
        C.check(C.lib().featomic_b200_surrogate_gradient(self._handle, n,
                                                          grad.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                          ctypes.byref(loss), _stream()))
        return loss.value, grad

    @property
    def parameters(self):
        p = np.zeros(self.n_parameters, dtype=np.float32)
        C.check(C.lib().featomic_b200_surrogate_parameters(self._handle, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                            len(p), 0, _stream()))
        return p

    @parameters.setter
    def parameters(self, value):
        p = np.ascontiguousarray(value, dtype=np.float32)
        C.check(C.lib().featomic_b200_surrogate_parameters(self._handle, p.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                            len(p), 1, _stream()))

    @property
    def scales(self):
        s = np.zeros(self.n_outputs, dtype=np.float32)
        C.check(C.lib().featomic_b200_surrogate_scales(self._handle, s.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                        len(s)))
        return s

    def samples(self):
        r = np.zeros(self.n_samples, dtype=np.float32)
        C.check(C.lib().featomic_b200_surrogate_samples(self._handle, r.ctypes.data_as(ctypes.POINTER(ctypes.c_float)),
                                                         len(r), _stream()))
        return r

    def evaluate(self, r, method="tensor_cores", derivatives=True):
        """(R [n, outputs], dR/dr [n, outputs] or None) as float32 CUDA tensors
        for the float64 CUDA tensor of distances ``r``."""
        import torch
        r = r.to(torch.float64).contiguous()
        n = r.numel()
        values = torch.empty((n, self.n_outputs), dtype=torch.float32, device=r.device)
        derivs = torch.empty((n, self.n_outputs), dtype=torch.float32, device=r.device) if derivatives else None
        C.check(C.lib().featomic_b200_surrogate_evaluate(
            self._handle, ctypes.c_void_p(r.data_ptr()), n, ctypes.c_void_p(values.data_ptr()),
            ctypes.c_void_p(derivs.data_ptr() if derivs is not None else None), self.n_outputs, METHODS[method],
            _stream()))
        return values, derivs

    def attach(self, enable=True):
        """Use this surrogate (or, with enable=False, the spline again) for the
        FP32 dense forms of its calculator."""
        C.check(C.lib().featomic_b200_calculator_set_surrogate(self._calculator._handle,
                                                                self._handle if enable else None))
