"""The C-ABI library builds, loads and exports every declared entry point;
argument checks fail cleanly without touching a GPU (no compute calls)."""
import ctypes as C
import os

import pytest


def test_library_exports_every_header_function(sns):
    from spectral_upcxx_b200 import _native as N
    names = N.header_functions()
    assert len(names) >= 30
    L = N.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(N.SIGNATURES), set(names) ^ set(N.SIGNATURES)


def test_version_and_error_string(sns):
    from spectral_upcxx_b200 import _native as N
    assert N.lib().sns_version() >= 1
    assert isinstance(N.last_error(), str)


@pytest.mark.parametrize("call,args", [
    ("sns_fft3d", (None, 8, 8, 8, -1, 0, 0, None)),
    ("sns_fft3d", (C.c_void_p(16), 8, 8, 8, 2, 0, 0, None)),
    ("sns_fft3d", (C.c_void_p(16), 8, 8, 8, -1, 8, 0, None)),
    ("sns_fft3d", (C.c_void_p(16), 8, 8, 8, -1, 0, 7, None)),
    ("sns_fft3d", (C.c_void_p(16), 0, 8, 8, -1, 0, 0, None)),
    ("sns_gradient", (None, None, None, None, 8, 8, 8, 0, None)),
    ("sns_laplacian", (C.c_void_p(16), None, 8, 8, 8, 0, None)),
    ("sns_axpby", (1.0, None, 0.0, None, None, 8, 0, None)),
    ("sns_mul", (C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), -1, 0, None)),
    ("sns_fft1d_many", (C.c_void_p(16), 0, 1, 1, 1, -1, 0, None)),
    ("sns_ns_step", (None, 1)),
    ("sns_ns_stats", (None, None, None, None, None)),
])
def test_bad_arguments_are_rejected(sns, call, args):
    from spectral_upcxx_b200 import _native as N
    rc = getattr(N.lib(), call)(*args)
    assert rc == N.SNS_ERR_ARG
    assert N.last_error()


def test_unsupported_sizes_are_reported(sns):
    from spectral_upcxx_b200 import _native as N
    rc = N.lib().sns_fft3d(C.c_void_p(16), 12, 8, 8, -1, 0, 0, None)
    assert rc == N.SNS_ERR_UNSUPPORTED
    assert "power" in N.last_error()
    h = C.c_void_p()
    rc = N.lib().sns_ns_create(C.byref(h), 24, 16, 16, 0.01, 1e-3, 0, None)
    assert rc == N.SNS_ERR_UNSUPPORTED and not h.value


def test_ensemble_arguments_are_checked_before_any_device_work(sns):
    from spectral_upcxx_b200 import _native as N
    L = N.lib()
    h = C.c_void_p()

    def create(shapes, nus, prec=0):
        dims = (C.c_int64 * max(1, 3 * len(shapes)))(*[n for s in shapes for n in s])
        nu = (C.c_double * max(1, len(nus)))(*nus)
        return L.sns_ens_create(C.byref(h), len(shapes), dims, nu, 2e-3, prec, 0, None)

    assert create([], []) == N.SNS_ERR_ARG
    assert create([(32, 32, 32)], [0.01], prec=5) == N.SNS_ERR_ARG
    assert create([(32, 32, 24)], [0.01]) == N.SNS_ERR_UNSUPPORTED
    assert create([(512, 512, 512)], [0.01]) == N.SNS_ERR_UNSUPPORTED
    assert create([(8, 16, 16)], [0.01]) == N.SNS_ERR_UNSUPPORTED
    nine = [(16 << (i % 5), 16 << (i // 5), 16) for i in range(9)]
    assert create(nine, [0.01] * 9) == N.SNS_ERR_UNSUPPORTED
    assert "distinct" in N.last_error()
    assert not h.value
    assert L.sns_ens_step(None, 1, 0) == N.SNS_ERR_ARG
    assert L.sns_ens_stats(None, None) == N.SNS_ERR_ARG
    assert L.sns_ens_bootstrap(None, 0, None, None) == N.SNS_ERR_ARG
    assert L.sns_ens_boxes(None) == N.SNS_ERR_ARG
    assert L.sns_ens_destroy(None) == 0


def test_call_wrapper_raises(sns):
    from spectral_upcxx_b200 import _native as N
    with pytest.raises(N.SNSError):
        N.call("sns_fft3d", None, 8, 8, 8, -1, 0, 0, None)


def test_kernels_target_sm100a():
    """The build recipe compiles for sm_100a only (no multi-arch fallback)."""
    from spectral_upcxx_b200 import build as B
    assert B.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert os.path.exists(B.LIBPATH)


def test_product_never_imports_oracle():
    """The product package neither imports nor links the CPU oracle."""
    import glob
    pkg = os.path.join(os.path.dirname(os.path.dirname(__file__)), "spectral_upcxx_b200")
    bad = ("import oracle", "from oracle", "pyoracle", "liboracle", "libref", "orc_")
    for path in glob.glob(os.path.join(pkg, "**", "*.*"), recursive=True):
        if path.endswith((".py", ".cu", ".cuh", ".cpp", ".H", ".hpp", ".h")):
            text = open(path).read()
            assert not any(b in text for b in bad), path
