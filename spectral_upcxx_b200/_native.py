"""ctypes binding of the C-ABI in include/spectral_b200.h.

The shared library is built in-tree by ``spectral_upcxx_b200.build`` (nvcc,
sm_100a).  There is no fallback: if the library is missing or a call fails,
an exception is raised.
"""
from __future__ import annotations

import ctypes as C
import os
import re

from . import build as _build

HEADER = os.path.join(_build.INCLUDE, "spectral_b200.h")

SNS_C64 = 0
SNS_C128 = 1
SNS_OK = 0
SNS_ERR_ARG = -1
SNS_ERR_UNSUPPORTED = -2
SNS_ERR_CUDA = -3
SNS_ERR_ALLOC = -4
SNS_ERR_TIMEOUT = -5
SNS_FFT_NORMALISE = 1
SNS_FFT_ZERO_NYQUIST = 2
SNS_CLOSURE_NONE = 0
SNS_CLOSURE_SMAGORINSKY = 1
SNS_CLOSURE_MLP = 2

_vp = C.c_void_p
_i64 = C.c_int64
_int = C.c_int
_dbl = C.c_double
_vp3 = C.POINTER(C.c_void_p)

# argument types of every entry point
SIGNATURES = {
    "sns_last_error": ([], C.c_char_p),
    "sns_version": ([], _int),
    "sns_malloc": ([C.POINTER(C.c_void_p), C.c_size_t], _int),
    "sns_free": ([_vp], _int),
    "sns_pool_trim": ([], _int),
    "sns_memcpy_h2d": ([_vp, _vp, C.c_size_t, _vp], _int),
    "sns_memcpy_d2h": ([_vp, _vp, C.c_size_t, _vp], _int),
    "sns_memcpy_d2d": ([_vp, _vp, C.c_size_t, _vp], _int),
    "sns_memset": ([_vp, _int, C.c_size_t, _vp], _int),
    "sns_stream_synchronize": ([_vp], _int),
    "sns_convert": ([_vp, _int, _vp, _int, _i64, _vp], _int),
    "sns_fft3d": ([_vp, _i64, _i64, _i64, _int, _int, _int, _vp], _int),
    "sns_fft3d_many": ([_vp3, _int, _i64, _i64, _i64, _int, _int, _int, _vp], _int),
    "sns_forward": ([_vp, _i64, _i64, _i64, _int, _vp], _int),
    "sns_inverse": ([_vp, _i64, _i64, _i64, _int, _vp], _int),
    "sns_fft3d_tune": ([_i64, _i64, _i64, _int, _int, _vp], _int),
    "sns_fft3d_check": ([_vp], _int),
    "sns_fft3d_axes": ([_vp, _i64, _i64, _i64, _int, _int, _dbl, _int, _vp], _int),
    "sns_fft1d_many": ([_vp, _i64, _i64, _i64, _i64, _int, _int, _vp], _int),
    "sns_fft1d_many_scaled": ([_vp, _i64, _i64, _i64, _i64, _int, _dbl, _int, _vp], _int),
    "sns_zero_high_modes": ([_vp, _i64, _i64, _i64, _int, _vp], _int),
    "sns_gradient": ([_vp, _vp, _vp, _vp, _i64, _i64, _i64, _int, _vp], _int),
    "sns_laplacian": ([_vp, _vp, _i64, _i64, _i64, _int, _vp], _int),
    "sns_laplacian_inverse": ([_vp, _dbl, _dbl, _i64, _i64, _i64, _int, _vp], _int),
    "sns_curl": ([_vp3, _vp3, _i64, _i64, _i64, _int, _vp], _int),
    "sns_divergence": ([_vp3, _vp, _i64, _i64, _i64, _int, _vp], _int),
    "sns_vector_laplacian": ([_vp3, _vp3, _i64, _i64, _i64, _int, _vp], _int),
    "sns_cross": ([_vp3, _vp3, _vp3, _i64, _i64, _i64, _int, _vp], _int),
    "sns_cross_noalloc": ([_vp3, _vp3, _vp3, _i64, _i64, _i64, _int, _vp], _int),
    "sns_average_abs": ([_vp, _i64, _int, C.POINTER(_dbl), _vp], _int),
    "sns_axpby": ([_dbl, _vp, _dbl, _vp, _vp, _i64, _int, _vp], _int),
    "sns_mul": ([_vp, _vp, _vp, _i64, _int, _vp], _int),
    "sns_ns_create": ([C.POINTER(_vp), _i64, _i64, _i64, _dbl, _dbl, _int, _vp], _int),
    "sns_ns_create_real": ([C.POINTER(_vp), _i64, _i64, _i64, _dbl, _dbl, _int, _vp], _int),
    "sns_ns_destroy": ([_vp], _int),
    "sns_ns_bootstrap": ([_vp, _vp3, _vp3], _int),
    "sns_ns_set_state": ([_vp, _vp3, _vp3], _int),
    "sns_ns_step": ([_vp, _int], _int),
    "sns_ns_get_state": ([_vp, _vp3, _vp3, _vp3], _int),
    "sns_ns_stats": ([_vp, C.POINTER(_dbl), C.POINTER(_dbl), C.POINTER(_dbl), C.POINTER(_dbl)],
                     _int),
    "sns_ns_check": ([_vp], _int),
    "sns_ns_launches_per_step": ([_vp], _int),
    "sns_ns_describe": ([_vp, C.c_char_p, _int], _int),
    "sns_ns_tune": ([_vp], _int),
    "sns_ns_stats_async": ([_vp, _vp], _int),
    "sns_ns_profile": ([_vp, _int], _int),
    "sns_ns_pass_times": ([_vp, C.POINTER(_dbl), C.POINTER(_int), _int], _int),
    "sns_ns_set_closure": ([_vp, _int, _dbl, _vp, _dbl], _int),
    "sns_ns_set_sgs_band": ([_vp, _dbl, _dbl], _int),
    "sns_mlp_sizes": ([C.POINTER(_i64), C.POINTER(_i64)], _int),
    "sns_mlp_pack": ([_vp, _dbl, _dbl, _vp, _vp], _int),
    "sns_mlp_infer": ([_vp, _vp, _i64, _vp, _vp], _int),
    "sns_mlp_status": ([], _int),
    "sns_particles_move": ([_vp, _vp, _i64, _vp3, _i64, _i64, _i64, _int, _dbl, _vp], _int),
    "sns_mlp_grad": ([_vp, _vp, _vp, _vp, _vp, _i64, _vp, _vp], _int),
    "sns_mlp_adam": ([_vp, _vp, _vp, _vp, _int, _dbl, _dbl, _dbl, _dbl, _vp, _vp], _int),
    "sns_spectral_truncate": ([_vp3, _vp3, _int, _i64, _i64, _dbl, _int, _vp], _int),
    "sns_spectral_pad": ([_vp3, _vp3, _int, _i64, _i64, _int, _vp], _int),
    "sns_sgs_sample": ([_vp3, _i64, _i64, _dbl, _dbl, _int, _vp, _vp, _vp, _vp3, _vp], _int),
    "sns_energy_spectrum": ([_vp3, _i64, _i64, _i64, _int, _vp, _int, _vp], _int),
    "sns_ens_create": ([C.POINTER(_vp), _int, C.POINTER(_i64), C.POINTER(_dbl), _dbl, _int, _int,
                        _vp], _int),
    "sns_ens_destroy": ([_vp], _int),
    "sns_ens_boxes": ([_vp], _int),
    "sns_ens_bootstrap": ([_vp, _int, _vp3, _vp3], _int),
    "sns_ens_set_state": ([_vp, _int, _vp3, _vp3], _int),
    "sns_ens_get_state": ([_vp, _int, _vp3, _vp3, _vp3], _int),
    "sns_ens_step": ([_vp, _int, _int], _int),
    "sns_ens_stats": ([_vp, C.POINTER(_dbl)], _int),
    "sns_ens_tuning": ([_vp, C.POINTER(_int), _int], _int),
    "sns_ens_launches_per_step": ([_vp, _int], _int),
    "sns_ens_stage_times": ([_vp, _int, C.POINTER(_dbl)], _int),
}

_LIB = None


class SNSError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, fn: str, rc: int, msg: str):
        super().__init__(f"{fn} failed ({rc}): {msg}")
        self.rc = rc


def header_functions():
    """Names of the functions declared in include/spectral_b200.h."""
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^(?:const\s+char\*|int)\s+(sns_\w+)\s*\(", text, re.M)))


def lib(build: bool = True):
    """Load libspectral_b200.so.  It is built first only when it is missing
    (or when SNS_REBUILD=1); __graft_entry__.build() rebuilds explicitly."""
    global _LIB
    if _LIB is None:
        path = _build.LIBPATH
        if build and (not os.path.exists(path) or os.environ.get("SNS_REBUILD") == "1"):
            _build.build_library()
        if not os.path.exists(path):
            raise ImportError(f"{path} is missing: run spectral_upcxx_b200.build.build_library()")
        L = C.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(L, name)
            fn.argtypes = args
            fn.restype = res
        _LIB = L
    return _LIB


def last_error() -> str:
    return lib().sns_last_error().decode()


def check(fn: str, rc: int) -> int:
    if rc != SNS_OK:
        raise SNSError(fn, rc, last_error())
    return rc


def call(fn: str, *args) -> int:
    return check(fn, getattr(lib(), fn)(*args))


def ptr3(ptrs):
    return (C.c_void_p * 3)(*[C.c_void_p(int(p)) for p in ptrs])


def ptrs(ps):
    return (C.c_void_p * len(ps))(*[C.c_void_p(int(p)) for p in ps])
