"""Seeded synthetic inputs (host, numpy) for the benchmarks and tests.

All randomness comes from numpy's counter-based Philox generator keyed by
the seed, so every run and every consumer (device path, CPU oracle) sees the
same fields.  Fields are complex128 arrays of shape (nz, ny, nx).
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.Philox(key=int(seed)))


def uniform_complex(shape, seed: int, dtype=np.complex128) -> np.ndarray:
    """Real and imaginary parts i.i.d. uniform[-1, 1) (standalone FFT input)."""
    g = rng(seed)
    re = g.uniform(-1.0, 1.0, size=shape)
    im = g.uniform(-1.0, 1.0, size=shape)
    return (re + 1j * im).astype(dtype)


def taylor_green(n: int):
    """u = sin x cos y cos z, v = -cos x sin y cos z, w = 0 on [0, 2 pi)^3."""
    x = 2 * np.pi * np.arange(n) / n
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    u = np.sin(X) * np.cos(Y) * np.cos(Z)
    v = -np.cos(X) * np.sin(Y) * np.cos(Z)
    w = np.zeros_like(u)
    return [a.astype(np.complex128) for a in (u, v, w)]


def wavenumbers(n: int) -> np.ndarray:
    """Scalar::freq (src/Scalar.cpp:198-206): k = i for i <= n/2, else i - n."""
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64)


def solenoidal_spectrum(n: int, seed: int, k0: float = 4.0, u_rms: float = 1.0):
    """Random divergence-free velocity with E(k) ~ k^4 exp(-2 (k/k0)^2).

    Complex Gaussian amplitudes (uniform phases) are shaped so each shell
    carries E(k), projected with P = I - k k / |k|^2, made real by taking the
    real part of the physical field, re-projected, Nyquist planes zeroed, and
    scaled to u_rms = sqrt(<|u|^2> / 3).  Returns the physical velocity
    (3 complex128 fields with zero imaginary part).
    """
    g = rng(seed)
    k = wavenumbers(n)
    KZ, KY, KX = np.meshgrid(k, k, k, indexing="ij")
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    Kmag = np.sqrt(K2)
    with np.errstate(divide="ignore", invalid="ignore"):
        E = Kmag ** 4 * np.exp(-2.0 * (Kmag / k0) ** 2)
        amp = np.where(K2 > 0, np.sqrt(E / (4 * np.pi * np.maximum(K2, 1.0))), 0.0)
    uh = [amp * (g.standard_normal((n, n, n)) + 1j * g.standard_normal((n, n, n))) for _ in range(3)]

    def project(vh):
        with np.errstate(divide="ignore", invalid="ignore"):
            kdotv = (KX * vh[0] + KY * vh[1] + KZ * vh[2]) / np.where(K2 > 0, K2, 1.0)
        return [vh[0] - KX * kdotv, vh[1] - KY * kdotv, vh[2] - KZ * kdotv]

    uh = project(uh)
    u = [np.real(np.fft.ifftn(c)) for c in uh]
    uh = project([np.fft.fftn(c) for c in u])
    h = n // 2
    for c in uh:
        c[h, :, :] = 0
        c[:, h, :] = 0
        c[:, :, h] = 0
    u = [np.real(np.fft.ifftn(c)) for c in uh]
    rms = np.sqrt(np.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 3.0)
    return [(c * (u_rms / rms)).astype(np.complex128) for c in u]


def ns_vortex_tubes(n: int) -> np.ndarray:
    """exec/ns.cpp:90-112: omega_z of three Gaussian vortex tubes (physical)."""
    width, mag, dist = np.pi / 8, 50.0, np.pi / 2
    h = 2.0 * np.pi / n
    x = h * np.arange(n)
    Y, X = np.meshgrid(x, x, indexing="ij")

    def gauss(xc, yc):
        return np.exp(-(X - xc) ** 2 / width) * np.exp(-(Y - yc) ** 2 / width)

    w2d = mag * gauss(np.pi - dist, np.pi - dist) + mag * gauss(np.pi + dist, np.pi - dist) + \
        mag * gauss(np.pi, np.pi + dist)
    return np.broadcast_to(w2d, (n, n, n)).astype(np.complex128).copy()


def solenoidal_spectrum_hat(n: int, seed: int, device, k0: float = 4.0, u_rms: float = 1.0):
    """Fourier transform of ``solenoidal_spectrum(n, seed)`` (Nyquist planes
    zeroed) built on a torch device: the same seeded amplitudes, with the
    transforms of the construction done by torch.fft so that large ensembles
    of initial fields are quick to make.  Returns 3 complex128 tensors."""
    import torch
    g = rng(seed)
    k = torch.as_tensor(wavenumbers(n), device=device)
    KZ, KY, KX = torch.meshgrid(k, k, k, indexing="ij")
    K2 = KX ** 2 + KY ** 2 + KZ ** 2
    Kmag = torch.sqrt(K2)
    E = Kmag ** 4 * torch.exp(-2.0 * (Kmag / k0) ** 2)
    amp = torch.where(K2 > 0, torch.sqrt(E / (4 * np.pi * torch.clamp(K2, min=1.0))),
                      torch.zeros_like(K2))
    uh = []
    for _ in range(3):
        re = torch.as_tensor(g.standard_normal((n, n, n)), device=device)
        im = torch.as_tensor(g.standard_normal((n, n, n)), device=device)
        uh.append(amp * torch.complex(re, im))
    K2s = torch.where(K2 > 0, K2, torch.ones_like(K2))

    def project(vh):
        kdotv = (KX * vh[0] + KY * vh[1] + KZ * vh[2]) / K2s
        return [vh[0] - KX * kdotv, vh[1] - KY * kdotv, vh[2] - KZ * kdotv]

    uh = project(uh)
    u = [torch.fft.ifftn(c).real.to(torch.complex128) for c in uh]
    uh = project([torch.fft.fftn(c) for c in u])
    h = n // 2
    for c in uh:
        c[h, :, :] = 0
        c[:, h, :] = 0
        c[:, :, h] = 0
    u = [torch.fft.ifftn(c).real for c in uh]
    rms = torch.sqrt(torch.mean(u[0] ** 2 + u[1] ** 2 + u[2] ** 2) / 3.0)
    out = [torch.fft.fftn((c * (u_rms / rms)).to(torch.complex128)) for c in u]
    for c in out:
        c[h, :, :] = 0
        c[:, h, :] = 0
        c[:, :, h] = 0
    return out
