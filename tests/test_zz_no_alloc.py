"""sns_cross_noalloc: Vector::cross for callers that cannot allocate.

Some callers cannot let a library call cudaMalloc -- their GPU memory is
already fully reserved by another allocator, or they run a loop that must
never enter the driver's allocation path.  sns_cross_noalloc serves them from
a static work area inside the library.  These tests call it through the C-ABI
twice in a row on each box (different inputs, so a stale work area would
show) and check each result against sns_cross and against the oracle's
Vector::cross, within the tolerances of the other cross-product tests
(complex128 <= 1e-12, complex64 <= 5e-6 relative L2 per component).  The boxes
include the largest one the static area takes in each precision and one with
a length-1 axis.  The second call must allocate no device memory; an oversize
box is refused with an error, and bad arguments get sns_cross's return codes.
The file name sorts last so a run that stops at the first failure has run
every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {torch.complex128: 1e-12, torch.complex64: 5e-6}
# (nz, ny, nx): a small box, the largest box of the static area for the
# precision (6 fields of 262144 complex128 / 524288 complex64 points), and a
# box with a length-1 axis
BOXES = {torch.complex128: [(16, 32, 64), (64, 64, 64), (1, 64, 32)],
         torch.complex64: [(16, 32, 64), (128, 64, 64), (32, 1, 16)]}


def _fourier_vector(oracle, shape, seed):
    from spectral_upcxx_b200 import ic
    return [oracle.forward(ic.uniform_complex(shape, seed + d)) for d in range(3)]


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_cross_noalloc_matches_cross_on_two_calls(sns, oracle, cuda, dtype):
    N = sns._native
    L = N.lib()
    prec = N.SNS_C128 if dtype == torch.complex128 else N.SNS_C64
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    for shape in BOXES[dtype]:
        nz, ny, nx = shape
        calls = []
        for seed in (100, 200):
            a = _fourier_vector(oracle, shape, seed)
            b = _fourier_vector(oracle, shape, seed + 50)
            ta = [torch.from_numpy(x).to(cuda, dtype) for x in a]
            tb = [torch.from_numpy(x).to(cuda, dtype) for x in b]
            want = sns.cross(ta, tb)  # the pooled path, allocated before any measurement
            got = [torch.empty_like(ta[0]) for _ in range(3)]
            calls.append((ta, tb, want, got, oracle.cross(a, b)))
        torch.cuda.synchronize()
        free_before = None
        for i, (ta, tb, want, got, exp) in enumerate(calls):
            if i == 1:
                free_before = torch.cuda.mem_get_info(cuda)[0]
            rc = L.sns_cross_noalloc(N.ptr3([x.data_ptr() for x in ta]),
                                     N.ptr3([x.data_ptr() for x in tb]),
                                     N.ptr3([x.data_ptr() for x in got]), nx, ny, nz, prec,
                                     stream)
            assert rc == N.SNS_OK, N.last_error()
            torch.cuda.synchronize()
            for g, w, e in zip(got, want, exp):
                g = g.cpu().to(torch.complex128).numpy()
                assert rel_l2(g, w.cpu().to(torch.complex128).numpy()) < TOL[dtype], shape
                assert rel_l2(g, e) < TOL[dtype], shape
        assert torch.cuda.mem_get_info(cuda)[0] == free_before, shape


def test_cross_noalloc_rejects_oversize_box_and_bad_arguments(sns, cuda):
    N = sns._native
    L = N.lib()
    dummy = torch.zeros(8, dtype=torch.complex128, device=cuda)
    p = N.ptr3([dummy.data_ptr()] * 3)
    rc = L.sns_cross_noalloc(p, p, p, 128, 64, 64, N.SNS_C128, None)
    assert rc == N.SNS_ERR_ARG
    assert "static work area" in N.last_error()
    # one past the complex64 limit
    rc = L.sns_cross_noalloc(p, p, p, 128, 64, 128, N.SNS_C64, None)
    assert rc == N.SNS_ERR_ARG and "static work area" in N.last_error()
    # the codes of sns_cross for the other bad arguments
    for args in ((12, 8, 8, N.SNS_C64), (8, 8, 8, 7), (0, 8, 8, N.SNS_C64)):
        rc_na = L.sns_cross_noalloc(p, p, p, *args, None)
        rc_pool = L.sns_cross(p, p, p, *args, None)
        assert rc_na == rc_pool != N.SNS_OK, args
