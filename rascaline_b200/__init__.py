"""featomic-b200: B200-native SOAP spherical expansion, power spectrum and radial spectrum.

The numerical work runs in hand-written sm_100a CUDA kernels inside
``libfeatomic_b200.so`` (built in-tree by ``python -m rascaline_b200.build``),
reached through featomic's C ABI (``include/featomic_b200.h``).  There is no
CPU fallback: without the library or a CUDA device the calls fail.
"""
from .calculators import (  # noqa: F401
    CalculatorBase,
    Labels,
    LodeSphericalExpansion,
    SoapPowerSpectrum,
    SoapRadialSpectrum,
    SphericalExpansion,
    SphericalExpansionByPair,
    System,
    TensorBlock,
    TensorMap,
    labels_tensormap,
    neighbor_list,
    profiling_clear,
    profiling_enable,
    profiling_get,
)
from ._c_api import FeatomicError, LIBRARY  # noqa: F401
from . import clebsch_gordan  # noqa: F401

__version__ = "0.1.0"
