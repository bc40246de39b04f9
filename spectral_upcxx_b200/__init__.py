"""spectral_upcxx_b200 -- B200-native pseudo-spectral Navier-Stokes step and 3D FFT.

The product is ``lib/libspectral_b200.so``: hand-written sm_100a kernels
behind the C-ABI of ``include/spectral_b200.h`` plus the reference's C++
field API (``api/``: Scalar, Vector, Operators, FFT1D).  This package builds
and binds it for Python callers; torch supplies device memory and streams.
"""
from . import _native
from ._native import SNS_C64, SNS_C128, SNSError, lib
from .ns import ENS_EAGER, ENS_GRAPH, ENS_SEQUENTIAL, NSEnsemble, NSStepper
from .particles import Tracers
from .ops import (average, axpby, cross, curl, divergence, fft1d_many, fft3d, fft3d_tune, forward,
                  gradient, inverse, laplacian, laplacian_inverse, mul, vector_laplacian,
                  zero_high_modes)

__all__ = [
    "SNS_C64", "SNS_C128", "SNSError", "lib", "NSStepper", "NSEnsemble", "Tracers", "ENS_GRAPH", "ENS_EAGER",
    "ENS_SEQUENTIAL", "average", "axpby", "cross", "curl",
    "divergence", "fft1d_many", "fft3d", "fft3d_tune", "forward", "gradient", "inverse", "laplacian",
    "laplacian_inverse", "mul", "vector_laplacian", "zero_high_modes",
]
