"""The CPU oracle, pinned before it is trusted (no GPU needed).

* its FFT against numpy's pocketfft (an independent implementation),
* the C restatement against the golden fixtures made by the reference's own
  code (tests/golden/make_golden.py), bit-for-bit where the arithmetic is the
  same, and
* the known answers of the reference's test/operators.cpp and the round trip
  of test/3d_fft.cpp.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("shape", [(8, 8, 8), (16, 12, 10), (6, 5, 7), (32, 32, 32), (3, 9, 25),
                                   (1, 1, 16), (2, 4, 1)])
def test_oracle_fft_matches_numpy(oracle, shape):
    rng = np.random.default_rng(7)
    f = rng.uniform(-1, 1, shape) + 1j * rng.uniform(-1, 1, shape)
    F = oracle.transform(f, -1)
    assert rel_l2(F, np.fft.fftn(f)) < 1e-14
    B = oracle.transform(f, +1)
    assert rel_l2(B, np.fft.ifftn(f) * f.size) < 1e-14


@pytest.mark.parametrize("n", [17, 97, 128, 243, 1000])
def test_oracle_fft_1d_lengths(oracle, n):
    rng = np.random.default_rng(n)
    f = rng.standard_normal((1, 1, n)) + 1j * rng.standard_normal((1, 1, n))
    assert rel_l2(oracle.transform(f, -1), np.fft.fft(f, axis=-1)) < 1e-13


def test_oracle_fft_golden(oracle):
    g = np.load(os.path.join(GOLD, "fft.npz"))
    for tag in ("8x8x8", "16x8x4"):
        f = g[f"fft_{tag}_in"]
        np.testing.assert_array_equal(oracle.forward(f, zero=True), g[f"fft_{tag}_forward_zero"])
        np.testing.assert_array_equal(oracle.transform(f, -1), g[f"fft_{tag}_forward_raw"])
        np.testing.assert_array_equal(oracle.inverse(f), g[f"fft_{tag}_inverse"])


def test_oracle_operators_golden(oracle):
    g = np.load(os.path.join(GOLD, "operators.npz"))
    v = [g[f"v{d}"] for d in range(3)]
    w = [g[f"w{d}"] for d in range(3)]
    for d, x in enumerate(oracle.gradient(v[0])):
        np.testing.assert_array_equal(x, g[f"grad{d}"])
    np.testing.assert_array_equal(oracle.laplacian(v[0]), g["lap"])
    np.testing.assert_array_equal(oracle.laplacian_inverse(v[0], 0.0, 1.0), g["ilap_0_1"])
    np.testing.assert_array_equal(oracle.laplacian_inverse(v[0], 1.0, -0.25), g["ilap_1_m0.25"])
    for d, x in enumerate(oracle.curl(v)):
        np.testing.assert_array_equal(x, g[f"curl{d}"])
    np.testing.assert_array_equal(oracle.divergence(v), g["div"])
    for d, x in enumerate(oracle.vlaplacian(v)):
        np.testing.assert_array_equal(x, g[f"vlap{d}"])
    for d, x in enumerate(oracle.cross(v, w)):
        np.testing.assert_array_equal(x, g[f"cross{d}"])
    assert abs(oracle.average(v[0]) - float(g["average_v0"])) <= 1e-15 * float(g["average_v0"])


@pytest.mark.parametrize("case,nu", [("tg", 0.01), ("vx", 1e-3)])
def test_oracle_ns_golden(oracle, case, nu):
    g = np.load(os.path.join(GOLD, "ns16.npz"))
    steps = int(g["steps"])
    V0 = [g[f"{case}_V0_{d}"] for d in range(3)]
    w0 = [g[f"{case}_omega0_{d}"] for d in range(3)]
    ns = oracle.NS(V0[0].shape, nu, 1e-3)
    ns.bootstrap(V0, w0)
    divs = [ns.step() for _ in range(steps)]
    st = ns.state()
    for d in range(3):
        np.testing.assert_array_equal(st["V1"][d], g[f"{case}_V1_{d}"])
        np.testing.assert_array_equal(st["cross0"][d], g[f"{case}_cross0_{d}"])
    np.testing.assert_allclose(divs, g[f"{case}_div_avgs"], rtol=1e-12, atol=1e-300)


def test_oracle_vortex_ic_matches_reference(oracle):
    """ns.cpp's own initial condition, built by the C restatement."""
    g = np.load(os.path.join(GOLD, "ns16.npz"))
    n = 16
    from spectral_upcxx_b200 import ic
    wz = oracle.forward(ic.ns_vortex_tubes(n))
    np.testing.assert_allclose(wz, g["vx_omega0_2"], rtol=0, atol=1e-10)
    V0 = oracle.velocity_from_vorticity_z(g["vx_omega0_2"])
    for d in range(3):
        np.testing.assert_array_equal(V0[d], g[f"vx_V0_{d}"])


def test_oracle_operators_known_answers(oracle):
    """The analytic checks of test/operators.cpp:14-198 at 1e-3 absolute."""
    n = 16
    x = 2 * np.pi * np.arange(n) / n
    s = np.broadcast_to(np.sin(x)[None, None, :], (n, n, n)).astype(np.complex128).copy()
    c = np.broadcast_to(np.cos(x)[None, None, :], (n, n, n))
    sf = oracle.forward(s)
    grad = [oracle.inverse(g) for g in oracle.gradient(sf)]
    assert np.abs(grad[0].real - c).max() < 1e-3
    assert np.abs(grad[1].real).max() < 1e-3 and np.abs(grad[2].real).max() < 1e-3
    lap = oracle.inverse(oracle.laplacian(sf))
    assert np.abs(lap.real + s.real).max() < 1e-3
    li = oracle.inverse(oracle.laplacian_inverse(oracle.forward(lap)))
    assert np.abs(li.real - s.real).max() < 1e-3
    z = np.zeros_like(s)
    div = oracle.inverse(oracle.divergence([sf, oracle.forward(z), oracle.forward(z)]))
    assert np.abs(div.real - c).max() < 1e-3
    one = np.ones_like(s)
    v1 = [oracle.forward(z), oracle.forward(z), oracle.forward(one)]
    v2 = [oracle.forward(z), oracle.forward(one), oracle.forward(z)]
    cr = [oracle.inverse(q) for q in oracle.cross(v1, v2)]
    assert np.abs(cr[0].real + 1).max() < 1e-3
    assert np.abs(cr[1].real).max() < 1e-3 and np.abs(cr[2].real).max() < 1e-3
    cu = [oracle.inverse(q) for q in oracle.curl(oracle.gradient(sf))]
    assert max(np.abs(q.real).max() for q in cu) < 1e-3


def test_oracle_roundtrip_3d_fft(oracle):
    """test/3d_fft.cpp:46-80: forward+inverse of uniform data at 1e-3 (no ZERO)."""
    rng = np.random.default_rng(3)
    f = rng.uniform(0, 1, (16, 16, 16)).astype(np.complex128)
    back = oracle.inverse(oracle.forward(f, zero=False))
    assert np.abs(back - f).max() < 1e-12


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(__file__), "..", "oracle",
                                                    "_ref", "libref.so")),
                    reason="in-place reference build absent")
def test_oracle_matches_reference_build(oracle):
    """C restatement vs the reference's own code on a fresh seeded input."""
    from spectral_upcxx_b200 import ic
    f = ic.uniform_complex((16, 8, 32), 99)
    np.testing.assert_array_equal(oracle.forward(f), oracle.ref_forward(f))
    np.testing.assert_array_equal(oracle.inverse(f), oracle.ref_inverse(f))
    V0 = [oracle.forward(c) for c in ic.taylor_green(8)]
    w0 = oracle.curl(V0)
    r = oracle.ref_ns_run(V0, w0, 0.01, 1e-3, 3)
    ns = oracle.NS((8, 8, 8), 0.01, 1e-3)
    ns.bootstrap(V0, w0)
    for _ in range(3):
        ns.step()
    st = ns.state()
    for d in range(3):
        np.testing.assert_array_equal(st["V1"][d], r["V1"][d])
