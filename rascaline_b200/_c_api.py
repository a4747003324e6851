"""ctypes declarations of ``include/featomic_b200.h``."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIBRARY = os.path.join(HERE, "libfeatomic_b200.so")

featomic_status_t = ctypes.c_int32


class mts_labels_t(ctypes.Structure):
    _fields_ = [
        ("internal_ptr_", ctypes.c_void_p),
        ("names", ctypes.POINTER(ctypes.c_char_p)),
        ("values", ctypes.POINTER(ctypes.c_int32)),
        ("size", ctypes.c_size_t),
        ("count", ctypes.c_size_t),
    ]


class featomic_pair_t(ctypes.Structure):
    _fields_ = [
        ("first", ctypes.c_size_t),
        ("second", ctypes.c_size_t),
        ("distance", ctypes.c_double),
        ("vector", ctypes.c_double * 3),
        ("cell_shift_indices", ctypes.c_int32 * 3),
    ]


_size_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.POINTER(ctypes.c_size_t))
_types_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_int32)))
_positions_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_double)))
_cell_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.POINTER(ctypes.c_double))
_neighbors_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.c_double)
_pairs_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(featomic_pair_t)),
                             ctypes.POINTER(ctypes.c_size_t))
_pairs_containing_cb = ctypes.CFUNCTYPE(featomic_status_t, ctypes.c_void_p, ctypes.c_size_t,
                                        ctypes.POINTER(ctypes.POINTER(featomic_pair_t)), ctypes.POINTER(ctypes.c_size_t))


class featomic_system_t(ctypes.Structure):
    _fields_ = [
        ("user_data", ctypes.c_void_p),
        ("size", _size_cb),
        ("types", _types_cb),
        ("positions", _positions_cb),
        ("cell", _cell_cb),
        ("compute_neighbors", _neighbors_cb),
        ("pairs", _pairs_cb),
        ("pairs_containing", _pairs_containing_cb),
    ]


class featomic_labels_selection_t(ctypes.Structure):
    _fields_ = [("subset", ctypes.POINTER(mts_labels_t)), ("predefined", ctypes.c_void_p)]


class featomic_calculation_options_t(ctypes.Structure):
    _fields_ = [
        ("gradients", ctypes.POINTER(ctypes.c_char_p)),
        ("gradients_count", ctypes.c_size_t),
        ("use_native_system", ctypes.c_bool),
        ("selected_samples", featomic_labels_selection_t),
        ("selected_properties", featomic_labels_selection_t),
        ("selected_keys", ctypes.POINTER(mts_labels_t)),
    ]


class featomic_b200_device_systems_t(ctypes.Structure):
    _fields_ = [
        ("n_systems", ctypes.c_size_t),
        ("system_sizes", ctypes.POINTER(ctypes.c_size_t)),
        ("types", ctypes.POINTER(ctypes.c_int32)),
        ("cells", ctypes.POINTER(ctypes.c_double)),
        ("positions", ctypes.c_void_p),
    ]


class featomic_b200_cg_task_t(ctypes.Structure):
    _fields_ = [
        ("first", ctypes.c_void_p),
        ("second", ctypes.c_void_p),
        ("output", ctypes.c_void_p),
        ("n_samples", ctypes.c_int64),
        ("l1", ctypes.c_int32),
        ("l2", ctypes.c_int32),
        ("lambda_", ctypes.c_int32),
        ("n_first", ctypes.c_int32),
        ("n_second", ctypes.c_int32),
        ("output_stride", ctypes.c_int64),
    ]



class featomic_b200_cg_couple_task_t(ctypes.Structure):
    _fields_ = [
        ("input", ctypes.c_void_p),
        ("output", ctypes.c_void_p),
        ("n_outer", ctypes.c_int64),
        ("n_inner", ctypes.c_int64),
        ("l1", ctypes.c_int32),
        ("l2", ctypes.c_int32),
        ("lambda_", ctypes.c_int32),
    ]


# every symbol declared in include/featomic_b200.h: name -> (restype, argtypes)
SIGNATURES = {
    "featomic_last_error": (ctypes.c_char_p, []),
    "featomic_set_logging_callback": (featomic_status_t, [ctypes.c_void_p]),
    "featomic_calculator": (ctypes.c_void_p, [ctypes.c_char_p, ctypes.c_char_p]),
    "featomic_calculator_free": (featomic_status_t, [ctypes.c_void_p]),
    "featomic_calculator_name": (featomic_status_t, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "featomic_calculator_parameters": (featomic_status_t, [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_size_t]),
    "featomic_calculator_cutoffs": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_double)),
                                                        ctypes.POINTER(ctypes.c_size_t)]),
    "featomic_calculator_compute": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                                        ctypes.POINTER(featomic_system_t), ctypes.c_size_t,
                                                        featomic_calculation_options_t]),
    "featomic_profiling_clear": (featomic_status_t, []),
    "featomic_profiling_enable": (featomic_status_t, [ctypes.c_bool]),
    "featomic_profiling_get": (featomic_status_t, [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_size_t]),
    "mts_tensormap_free": (featomic_status_t, [ctypes.c_void_p]),
    "mts_tensormap_keys": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(mts_labels_t)]),
    "mts_tensormap_block_by_id": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_size_t]),
    "mts_block_labels": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t, ctypes.POINTER(mts_labels_t)]),
    "mts_block_gradient": (featomic_status_t, [ctypes.c_void_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_void_p)]),
    "mts_block_gradients_list": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_char_p)),
                                                     ctypes.POINTER(ctypes.c_size_t)]),
    "mts_labels_free": (featomic_status_t, [ctypes.POINTER(mts_labels_t)]),
    "featomic_b200_block_values": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.POINTER(ctypes.c_double)),
                                                       ctypes.POINTER(ctypes.POINTER(ctypes.c_size_t)),
                                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int32)]),
    "featomic_b200_calculator_compute_device": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p),
                                                                    ctypes.POINTER(featomic_b200_device_systems_t),
                                                                    featomic_calculation_options_t, ctypes.c_void_p]),
    "featomic_b200_neighbor_list": (featomic_status_t, [ctypes.POINTER(ctypes.c_double), ctypes.c_size_t,
                                                        ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                                        ctypes.POINTER(featomic_pair_t), ctypes.c_size_t,
                                                        ctypes.POINTER(ctypes.c_size_t)]),
    "featomic_b200_neighbor_list_noalloc": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t,
                                                                ctypes.POINTER(ctypes.c_double), ctypes.c_double,
                                                                ctypes.c_void_p, ctypes.c_size_t,
                                                                ctypes.POINTER(ctypes.c_size_t), ctypes.c_void_p]),
    "featomic_b200_power_spectrum_dense": (featomic_status_t, [ctypes.c_void_p,
                                                               ctypes.POINTER(featomic_b200_device_systems_t),
                                                               ctypes.POINTER(ctypes.c_int32), ctypes.c_size_t,
                                                               ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t,
                                                               ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    "featomic_b200_dense_shape": (featomic_status_t, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_size_t)] * 5),
    "featomic_b200_dense_species": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32),
                                                        ctypes.POINTER(ctypes.c_int32)]),
    "featomic_b200_power_spectrum_dense_backward": (featomic_status_t, [ctypes.c_void_p] + [ctypes.c_void_p] * 5),
    "featomic_b200_dense_free": (featomic_status_t, [ctypes.c_void_p]),
    "featomic_b200_spherical_expansion_dense": (featomic_status_t, [ctypes.c_void_p,
                                                                    ctypes.POINTER(featomic_b200_device_systems_t),
                                                                    ctypes.POINTER(ctypes.c_int32), ctypes.c_size_t,
                                                                    ctypes.c_int32, ctypes.c_void_p, ctypes.c_size_t,
                                                                    ctypes.POINTER(ctypes.c_void_p), ctypes.c_void_p]),
    "featomic_b200_spherical_expansion_dense_backward": (featomic_status_t, [ctypes.c_void_p, ctypes.c_void_p,
                                                                             ctypes.c_void_p, ctypes.c_void_p,
                                                                             ctypes.c_void_p, ctypes.c_void_p]),
    "featomic_b200_dense_jvp": (featomic_status_t, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_void_p, ctypes.c_void_p]),
    "featomic_b200_set_contraction_engine": (featomic_status_t, [ctypes.c_int32, ctypes.c_int32]),
    "featomic_b200_set_expansion_engine": (featomic_status_t, [ctypes.c_int32]),
    "featomic_b200_labels_tensormap": (featomic_status_t, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                         ctypes.POINTER(ctypes.c_void_p)]),
    "featomic_b200_batch_create": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t,
                                                       ctypes.POINTER(ctypes.c_size_t), ctypes.POINTER(ctypes.c_int32),
                                                       ctypes.POINTER(ctypes.c_int32), ctypes.c_size_t,
                                                       ctypes.POINTER(ctypes.c_void_p)]),
    "featomic_b200_batch_shape": (featomic_status_t, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_size_t)] * 5),
    "featomic_b200_batch_run": (featomic_status_t, [ctypes.c_void_p] * 9),
    "featomic_b200_batch_tune": (featomic_status_t, [ctypes.c_void_p] * 9 + [ctypes.POINTER(ctypes.c_double)]),
    "featomic_b200_batch_config": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "featomic_b200_batch_set_config": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]),
    "featomic_b200_batch_status": (featomic_status_t, [ctypes.c_void_p, ctypes.c_void_p,
                                                       ctypes.POINTER(ctypes.c_int32)]),
    "featomic_b200_batch_free": (featomic_status_t, [ctypes.c_void_p]),
    "featomic_b200_surrogate_create": (featomic_status_t, [ctypes.c_void_p, ctypes.c_int32, ctypes.c_uint64,
                                                           ctypes.POINTER(ctypes.c_void_p)]),
    "featomic_b200_surrogate_shape": (featomic_status_t, [ctypes.c_void_p] + [ctypes.POINTER(ctypes.c_size_t)] * 3),
    "featomic_b200_surrogate_dataset": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint64,
                                                            ctypes.c_void_p]),
    "featomic_b200_surrogate_train": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_size_t,
                                                          ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                                          ctypes.c_void_p]),
    "featomic_b200_surrogate_set_derivative_weight": (featomic_status_t, [ctypes.c_void_p, ctypes.c_double]),
    "featomic_b200_surrogate_fit_output_layer": (featomic_status_t, [ctypes.c_void_p, ctypes.c_double, ctypes.c_void_p]),
    "featomic_b200_surrogate_gradient": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t,
                                                             ctypes.POINTER(ctypes.c_float),
                                                             ctypes.POINTER(ctypes.c_double), ctypes.c_void_p]),
    "featomic_b200_surrogate_parameters": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                                               ctypes.c_size_t, ctypes.c_int32, ctypes.c_void_p]),
    "featomic_b200_surrogate_scales": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                                           ctypes.c_size_t]),
    "featomic_b200_surrogate_samples": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_float),
                                                            ctypes.c_size_t, ctypes.c_void_p]),
    "featomic_b200_surrogate_evaluate": (featomic_status_t, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t,
                                                             ctypes.c_int32, ctypes.c_void_p]),
    "featomic_b200_calculator_set_surrogate": (featomic_status_t, [ctypes.c_void_p, ctypes.c_void_p]),
    "featomic_b200_surrogate_free": (featomic_status_t, [ctypes.c_void_p]),
    "featomic_b200_radial_integral": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                                          ctypes.c_size_t, ctypes.POINTER(ctypes.c_double),
                                                          ctypes.POINTER(ctypes.c_double),
                                                          ctypes.POINTER(ctypes.c_int32)]),
    "featomic_b200_cg_coefficients": (featomic_status_t, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                          ctypes.POINTER(ctypes.c_double), ctypes.c_size_t]),
    "featomic_b200_cg_product": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32,
                                                     ctypes.c_void_p]),
    "featomic_b200_cg_couple": (featomic_status_t, [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int32,
                                                    ctypes.c_void_p]),
    "featomic_b200_dense_timings": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                                        ctypes.c_size_t]),
    "featomic_b200_calculator_timings": (featomic_status_t, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_double),
                                                             ctypes.c_size_t]),
}

_LIB = None


class FeatomicError(RuntimeError):
    def __init__(self, message, status):
        super().__init__(message)
        self.status = status


def lib():
    """Load the in-tree library (built by ``rascaline_b200.build``).  There is
    no fallback: a missing library is an error."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIBRARY):
            raise ImportError(
                f"{LIBRARY} is missing: build it with `python -m rascaline_b200.build` (needs nvcc)")
        L = ctypes.CDLL(LIBRARY)
        for name, (restype, argtypes) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.restype = restype
            fn.argtypes = argtypes
        _LIB = L
    return _LIB


def check(status):
    if status != 0:
        message = lib().featomic_last_error().decode("utf8", errors="replace")
        raise FeatomicError(message, status)
