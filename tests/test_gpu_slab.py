"""The slab-distributed 3D transform (z slabs, the decomposition of the
reference's Scalar::transform, src/Scalar.cpp:400-646) with P ranks emulated
in one process on one GPU: the library's line passes for the local phases and
an in-process all-to-all for the transposes.  Against the oracle:
complex128 relative L2 <= 1e-12, complex64 <= 2e-6."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {torch.complex128: 1e-12, torch.complex64: 2e-6}


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape,P", [((32, 64, 16), 2), ((64, 64, 64), 4), ((16, 32, 128), 8)])
def test_slab_transform_matches_oracle(sns, oracle, cuda, dtype, shape, P):
    from spectral_upcxx_b200 import ic
    from spectral_upcxx_b200.slab import SlabFFT3D, in_process_exchange
    f = ic.uniform_complex(shape, 31)
    nzl = shape[0] // P
    fft = SlabFFT3D(shape, P, exchange=in_process_exchange)

    def slabs_of(a):
        return [torch.from_numpy(np.ascontiguousarray(a[r * nzl:(r + 1) * nzl])).to(cuda, dtype)
                for r in range(P)]

    def whole(slabs):
        return np.concatenate([s.cpu().to(torch.complex128).numpy() for s in slabs])

    for direction in (-1, +1):
        s = slabs_of(f)
        fft.transform(s, direction)
        assert rel_l2(whole(s), oracle.transform(f, direction)) < TOL[dtype]
    s = slabs_of(f)
    fft.forward(s, range(P))
    assert rel_l2(whole(s), oracle.forward(f)) < TOL[dtype]
    s = slabs_of(f)
    fft.inverse(s)
    assert rel_l2(whole(s), oracle.inverse(f)) < TOL[dtype]


def test_slab_rejects_uneven_split(sns, cuda):
    from spectral_upcxx_b200.slab import SlabFFT3D
    with pytest.raises(ValueError):
        SlabFFT3D((12, 16, 16), 8)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_slab_cross_matches_oracle(sns, oracle, cuda, dtype):
    """Vector::cross of z-slab vectors (P = 4 emulated ranks) against the
    oracle (complex128 <= 1e-12, complex64 <= 5e-6)."""
    from spectral_upcxx_b200 import ic
    from spectral_upcxx_b200.slab import SlabFFT3D, in_process_exchange, slab_cross
    shape, P = (32, 32, 16), 4
    nzl = shape[0] // P
    va = [oracle.forward(ic.uniform_complex(shape, 40 + d)) for d in range(3)]
    vb = [oracle.forward(ic.uniform_complex(shape, 50 + d)) for d in range(3)]
    fft = SlabFFT3D(shape, P, exchange=in_process_exchange)
    to = lambda v: [[torch.from_numpy(np.ascontiguousarray(c[r * nzl:(r + 1) * nzl]))
                     .to(cuda, dtype) for r in range(P)] for c in v]
    got = slab_cross(fft, to(va), to(vb), range(P))
    want = oracle.cross(va, vb)
    tol = 1e-12 if dtype == torch.complex128 else 5e-6
    for d in range(3):
        g = np.concatenate([s.cpu().to(torch.complex128).numpy() for s in got[d]])
        assert rel_l2(g, want[d]) < tol, d
