"""TEST INFRASTRUCTURE ONLY -- CPU oracle (numpy, FP64) of the tracer
particles of src/Particle.cpp.  Only tests/ and bench.py's CPU leg may import
this module; the product's particle kernel is csrc/sns_particles.cu.

move() restates Particle::move (src/Particle.cpp:12-46) for a whole
population: the cell index trunc(x / h) clamped to n - 2 (INT is uint64_t,
src/FFT1D.H:14), the fractions, the trilinear interpolation of the real parts
with the eight corner terms summed in the reference's order
(src/Particle.cpp:27-34), x += v K and the periodic wrap
(src/Particle.cpp:37-45); energy() is Particle::energy (src/Particle.cpp:48-55).
numpy evaluates each expression with the same IEEE double operations in the
same order, so its positions equal the reference's to the last bit.
"""
from __future__ import annotations

import numpy as np


def move(loc, u, K):
    """One move of every particle.  loc: (n, 3) positions (x, y, z); u: three
    physical velocity fields (nz, ny, nx), real parts used.  Returns the new
    positions and the interpolated velocities (n, 3)."""
    loc = np.array(loc, dtype=np.float64)
    nz, ny, nx = u[0].shape
    dims = (nx, ny, nz)
    ind = np.zeros(loc.shape, dtype=np.int64)
    rd = np.zeros(loc.shape)
    for d in range(3):
        h = 2 * np.pi / dims[d]
        i = np.trunc(loc[:, d] / h).astype(np.int64)
        i = np.where(i + 1 >= dims[d], dims[d] - 2, i)
        ind[:, d] = i
        rd[:, d] = (loc[:, d] - i * h) / h
    i, j, k = ind[:, 0], ind[:, 1], ind[:, 2]
    r0, r1, r2 = rd[:, 0], rd[:, 1], rd[:, 2]
    o0, o1, o2 = 1 - r0, 1 - r1, 1 - r2
    v = np.zeros(loc.shape)
    for d in range(3):
        f = np.asarray(u[d]).real
        at = lambda a, b, c: f[c, b, a]
        v[:, d] = (at(i, j, k) * o0 * o1 * o2 + at(i + 1, j, k) * r0 * o1 * o2 +
                   at(i + 1, j + 1, k) * r0 * r1 * o2 + at(i, j + 1, k) * o0 * r1 * o2 +
                   at(i, j, k + 1) * o0 * o1 * r2 + at(i + 1, j, k + 1) * r0 * o1 * r2 +
                   at(i + 1, j + 1, k + 1) * r0 * r1 * r2 + at(i, j + 1, k + 1) * o0 * r1 * r2)
    new = loc + v * K
    two_pi = 2 * np.pi
    new = np.where(new >= two_pi, new - two_pi, np.where(new <= 0, two_pi + new, new))
    return new, v


def energy(v):
    """0.5 |v|^2 per particle, summed over the components in order."""
    e = np.zeros(v.shape[0])
    for d in range(3):
        e = e + v[:, d] * v[:, d]
    return 0.5 * e
