"""Device 3D/1D transforms against the CPU oracle (and the reference's golden
vectors), plus size-independent properties at the benchmark sizes.

Tolerances: complex128 relative L2 <= 1e-12 against the FP64 oracle;
complex64 relative L2 <= 2e-6 per transform (single FFT, FP32 arithmetic with
FP64-generated twiddles)."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
TOL = {torch.complex128: 1e-12, torch.complex64: 2e-6}
DT = [torch.complex128, torch.complex64]


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("shape", [(2, 2, 2), (4, 8, 16), (16, 16, 16), (8, 32, 64), (64, 64, 64),
                                   (32, 16, 128), (1, 1, 256), (4, 1, 512), (2, 2, 1024),
                                   (1, 2048, 2), (4096, 1, 1)])
def test_fft3d_matches_oracle(sns, oracle, cuda, dtype, shape):
    from spectral_upcxx_b200 import ic
    f = ic.uniform_complex(shape, 1)
    for direction in (-1, +1):
        t = dev(f, dtype, cuda)
        sns.fft3d(t, direction)
        torch.cuda.synchronize()
        assert rel_l2(host(t), oracle.transform(f, direction)) < TOL[dtype]


@pytest.mark.parametrize("dtype", DT)
def test_forward_inverse_golden(sns, cuda, dtype):
    """Scalar::forward (ZERO on) and Scalar::inverse against the reference's outputs."""
    g = np.load(os.path.join(GOLD, "fft.npz"))
    for tag in ("8x8x8", "16x8x4"):
        f = g[f"fft_{tag}_in"]
        t = dev(f, dtype, cuda)
        sns.forward(t)
        assert rel_l2(host(t), g[f"fft_{tag}_forward_zero"]) < TOL[dtype]
        t = dev(f, dtype, cuda)
        sns.fft3d(t, -1)
        assert rel_l2(host(t), g[f"fft_{tag}_forward_raw"]) < TOL[dtype]
        t = dev(f, dtype, cuda)
        sns.inverse(t)
        assert rel_l2(host(t), g[f"fft_{tag}_inverse"]) < TOL[dtype]


@pytest.mark.parametrize("dtype", DT)
def test_zero_nyquist_planes_exact(sns, cuda, dtype):
    from spectral_upcxx_b200 import ic
    n = 32
    t = dev(ic.uniform_complex((n, n, n), 5), dtype, cuda)
    sns.forward(t)
    h = host(t)
    assert np.all(h[n // 2] == 0) and np.all(h[:, n // 2] == 0) and np.all(h[:, :, n // 2] == 0)


@pytest.mark.parametrize("dtype", DT)
def test_batched_fields_equal_single(sns, cuda, dtype):
    from spectral_upcxx_b200 import ic
    fs = [dev(ic.uniform_complex((16, 32, 64), 40 + i), dtype, cuda) for i in range(6)]
    singles = [f.clone() for f in fs]
    sns.fft3d(fs, -1, zero_nyquist=True)
    for s in singles:
        sns.fft3d(s, -1, zero_nyquist=True)
    for a, b in zip(fs, singles):
        assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("n,stride,howmany,dist", [(256, 1, 64, 256), (64, 64, 64, 1),
                                                   (128, 3, 5, 1000), (16, 1, 7, 19),
                                                   (1024, 4, 3, 1), (2048, 8, 8, 1)])
def test_fft1d_many_matches_numpy(sns, cuda, dtype, n, stride, howmany, dist):
    rng = np.random.default_rng(n + howmany)
    size = (howmany - 1) * dist + (n - 1) * stride + 1
    flat = rng.uniform(-1, 1, size) + 1j * rng.uniform(-1, 1, size)
    t = torch.from_numpy(flat).to(cuda, dtype)
    sns.fft1d_many(t, n, stride, howmany, dist, -1)
    out = t.cpu().to(torch.complex128).numpy()
    exp = flat.copy()
    for b in range(howmany):
        idx = b * dist + stride * np.arange(n)
        exp[idx] = np.fft.fft(flat[idx])
    assert rel_l2(out, exp) < TOL[dtype] * 2


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("n", [128, 256, 512])
def test_roundtrip_full_size(sns, cuda, dtype, n):
    """Benchmark sizes: forward+inverse returns the input; Parseval holds."""
    if dtype == torch.complex128 and n == 512:
        pass  # 2.1 GB field, fits
    g = torch.Generator(device=cuda).manual_seed(n)
    re = torch.rand((n, n, n), device=cuda, generator=g, dtype=torch.float64) * 2 - 1
    im = torch.rand((n, n, n), device=cuda, generator=g, dtype=torch.float64) * 2 - 1
    x = torch.complex(re, im).to(dtype)
    del re, im
    y = x.clone()
    sns.fft3d(y, -1)
    e_x = torch.sum(torch.abs(x.to(torch.complex128)) ** 2).item()
    e_y = torch.sum(torch.abs(y.to(torch.complex128)) ** 2).item() / x.numel()
    assert abs(e_y - e_x) / e_x < (1e-12 if dtype == torch.complex128 else 1e-5)
    sns.fft3d(y, +1, normalise=True)
    err = (torch.linalg.vector_norm((y - x).to(torch.complex128)) /
           torch.linalg.vector_norm(x.to(torch.complex128))).item()
    assert err < (1e-13 if dtype == torch.complex128 else 2e-6)
    del x, y
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dtype", DT)
def test_linearity(sns, cuda, dtype):
    from spectral_upcxx_b200 import ic
    a = ic.uniform_complex((32, 64, 128), 8)
    b = ic.uniform_complex((32, 64, 128), 9)
    ta, tb, tab = dev(a, dtype, cuda), dev(b, dtype, cuda), dev(2.0 * a - 3.0 * b, dtype, cuda)
    for t in (ta, tb, tab):
        sns.fft3d(t, -1)
    comb = 2.0 * ta.to(torch.complex128) - 3.0 * tb.to(torch.complex128)
    assert rel_l2(host(tab), comb.cpu().numpy()) < TOL[dtype] * 5


def test_empty_and_bad_inputs(sns, cuda):
    with pytest.raises(ValueError):
        sns.fft3d(torch.zeros((4, 4, 4), dtype=torch.complex64), -1)  # host tensor
    with pytest.raises(TypeError):
        sns.fft3d(torch.zeros((4, 4, 4), dtype=torch.float32, device=cuda), -1)
    with pytest.raises(sns.SNSError):
        sns.fft3d(torch.zeros((4, 4, 6), dtype=torch.complex64, device=cuda), -1)
    t = torch.zeros(8, dtype=torch.complex64, device=cuda)
    sns.fft1d_many(t, 8, 1, 0, 8, -1)  # zero lines: no-op


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("shape", [(4, 128, 128), (1, 128, 128), (16, 128, 128)])
def test_xy_plane_pass_matches_oracle(sns, oracle, cuda, dtype, shape):
    """nx = ny = 128: x and y in one cluster pass per plane (distributed shared
    memory), z separately; raw transforms and Scalar::forward/inverse (Nyquist
    zeroing, 1/N) against the oracle."""
    from spectral_upcxx_b200 import ic
    f = ic.uniform_complex(shape, 4)
    for direction in (-1, +1):
        t = dev(f, dtype, cuda)
        sns.fft3d(t, direction)
        assert rel_l2(host(t), oracle.transform(f, direction)) < TOL[dtype]
    t = dev(f, dtype, cuda)
    sns.forward(t)
    assert rel_l2(host(t), oracle.forward(f)) < TOL[dtype]
    t = dev(f, dtype, cuda)
    sns.inverse(t)
    assert rel_l2(host(t), oracle.inverse(f)) < TOL[dtype]


@pytest.mark.parametrize("dtype", DT)
def test_xy_plane_pass_batched_fields(sns, oracle, cuda, dtype):
    """Three fields in one batch through the plane pass (field index from the
    grid) equal the fields transformed one at a time."""
    from spectral_upcxx_b200 import ic
    fs = [ic.uniform_complex((8, 128, 128), 10 + i) for i in range(3)]
    ts = [dev(f, dtype, cuda) for f in fs]
    sns.fft3d(ts, -1, zero_nyquist=True)
    for f, t in zip(fs, ts):
        assert rel_l2(host(t), oracle.forward(f)) < TOL[dtype]


@pytest.mark.parametrize("stages", ["1", "2"])
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("shape", [(64, 128, 64), (512, 16, 32), (32, 256, 16), (8, 64, 128)])
def test_tma_staged_passes_match_direct_bit_for_bit(sns, oracle, cuda, monkeypatch, dtype, shape,
                                                    stages):
    """The passes of the 3D transform over TMA-staged tiles (SNS_FFT_TMA = 1
    or 2 stages; a tuned plan may choose them; x lines where a row fits one
    box) give the direct-load passes' results bit for bit, forward (with Nyquist zeroing)
    and inverse (with 1/N), 1 and 3 fields; the record of the bounded waits
    stays clear (sns_fft3d_check)."""
    from spectral_upcxx_b200 import ic
    N = sns._native
    fs = [ic.uniform_complex(shape, 31 + i) for i in range(3)]
    out = {}
    for mode in ("0", stages):
        monkeypatch.setenv("SNS_FFT_TMA", mode)
        t1 = dev(fs[0], dtype, cuda)
        sns.forward(t1)
        t3 = [dev(f, dtype, cuda) for f in fs]
        sns.fft3d(t3, +1, normalise=True)
        torch.cuda.synchronize()
        assert N.lib().sns_fft3d_check(None) == N.SNS_OK, N.last_error()
        out[mode] = [t1] + t3
    for a, b in zip(out[stages], out["0"]):
        assert torch.equal(a, b)
    assert rel_l2(host(out[stages][0]), oracle.forward(fs[0])) < TOL[dtype]
