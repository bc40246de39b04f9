"""Tracer particles advected by the velocity of a run (src/Particle.cpp,
exec/ns.cpp:157-203) on the GPU: the whole population moves in one launch of
sns_particles_move instead of one Particle::move call per particle."""
from __future__ import annotations

import ctypes
import math

import torch

from . import _native as N
from .ops import _check_field, _stream, inverse


def _vptr(t: torch.Tensor):
    return ctypes.c_void_p(t.data_ptr())


class Tracers:
    """n particles with FP64 positions (n, 3) = (x, y, z) in [0, 2 pi] on the
    device and their last interpolated velocities."""

    def __init__(self, positions: torch.Tensor):
        if positions.dtype != torch.float64 or positions.dim() != 2 or positions.shape[1] != 3:
            raise ValueError("positions: (n, 3) float64")
        self.pos = positions.contiguous()
        self.vel = torch.zeros_like(self.pos)

    @staticmethod
    def uniform(n: int, seed: int = 0, device="cuda") -> "Tracers":
        """n particles uniformly placed in [0, 2 pi)^3 (the reference draws
        rand() / RAND_MAX * 2 pi, src/Particle.cpp:5-10)."""
        g = torch.Generator(device="cpu").manual_seed(seed)
        p = torch.rand((n, 3), generator=g, dtype=torch.float64) * (2 * math.pi)
        return Tracers(p.to(device))

    def __len__(self):
        return self.pos.shape[0]

    def move(self, u, K: float):
        """One move through the physical velocity u (three complex fields)."""
        u = list(u)
        prec = _check_field(u[0])
        nz, ny, nx = u[0].shape
        for f in u[1:]:
            if _check_field(f) != prec or f.shape != u[0].shape:
                raise ValueError("velocity components must match")
        N.call("sns_particles_move", _vptr(self.pos), _vptr(self.vel), len(self),
               N.ptr3([f.data_ptr() for f in u]), nx, ny, nz, prec, float(K), _stream(u[0]))

    def advect(self, stepper, K: float):
        """Move through the current velocity of an NSStepper (its Fourier
        velocity inverse-transformed into scratch fields, as exec/ns.cpp does
        with V.inverse(vtmp) before moving its particles)."""
        u = stepper.velocity()
        for f in u:
            inverse(f)
        self.move(u, K)

    def energy(self) -> torch.Tensor:
        """0.5 |v|^2 per particle (Particle::energy)."""
        v = self.vel
        return 0.5 * (v[:, 0] * v[:, 0] + v[:, 1] * v[:, 1] + v[:, 2] * v[:, 2])
