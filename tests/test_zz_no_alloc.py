"""sns_cross_noalloc: Vector::cross for callers that cannot allocate.

Some callers cannot let a library call cudaMalloc -- their GPU memory is
already fully reserved by another allocator, or they run a loop that must
never enter the driver's allocation path.  sns_cross_noalloc serves them from
a static work area inside the library.  This test calls it through the C-ABI
twice in a row (different inputs, so a stale work area would show) and checks
each result against sns_cross within the tolerances the other cross-product
tests use, checks that the second call allocates no device memory, and that
an oversize box is refused with an error.  The file name sorts last so a run
that stops at the first failure has run every other test first.
"""
import ctypes as C

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {torch.complex128: 1e-12, torch.complex64: 5e-6}


def _fourier_vector(oracle, shape, seed, dtype, device):
    from spectral_upcxx_b200 import ic
    v = [oracle.forward(ic.uniform_complex(shape, seed + d)) for d in range(3)]
    return [torch.from_numpy(x).to(device, dtype) for x in v]


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_cross_noalloc_matches_cross_on_two_calls(sns, oracle, cuda, dtype):
    N = sns._native
    L = N.lib()
    prec = N.SNS_C128 if dtype == torch.complex128 else N.SNS_C64
    shape = (16, 32, 64)  # (nz, ny, nx)
    nz, ny, nx = shape
    stream = C.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    calls = []
    for seed in (100, 200):
        a = _fourier_vector(oracle, shape, seed, dtype, cuda)
        b = _fourier_vector(oracle, shape, seed + 50, dtype, cuda)
        want = sns.cross(a, b)  # the pooled path, allocated before any measurement
        got = [torch.empty_like(a[0]) for _ in range(3)]
        calls.append((a, b, want, got))
    torch.cuda.synchronize()
    free_before = None
    for i, (a, b, want, got) in enumerate(calls):
        if i == 1:
            free_before = torch.cuda.mem_get_info(cuda)[0]
        rc = L.sns_cross_noalloc(N.ptr3([x.data_ptr() for x in a]),
                                 N.ptr3([x.data_ptr() for x in b]),
                                 N.ptr3([x.data_ptr() for x in got]), nx, ny, nz, prec, stream)
        assert rc == N.SNS_OK, N.last_error()
        torch.cuda.synchronize()
        for g, w in zip(got, want):
            assert rel_l2(g.cpu().numpy(), w.cpu().numpy()) < TOL[dtype]
    assert torch.cuda.mem_get_info(cuda)[0] == free_before


def test_cross_noalloc_rejects_oversize_box(sns, cuda):
    N = sns._native
    L = N.lib()
    dummy = torch.zeros(8, dtype=torch.complex128, device=cuda)
    p = N.ptr3([dummy.data_ptr()] * 3)
    rc = L.sns_cross_noalloc(p, p, p, 128, 64, 64, N.SNS_C128, None)
    assert rc == N.SNS_ERR_ARG
    assert "static work area" in N.last_error()
