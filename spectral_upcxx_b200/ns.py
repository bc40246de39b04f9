"""The fused Navier-Stokes stepper (sns_ns_*), mirroring exec/ns.cpp.

``NSStepper(shape, nu, dt, dtype)`` holds the AB2 state (Fourier velocity V1
and the previous cross product cross0) on the GPU.  ``bootstrap(V0, omega0)``
runs ns.cpp:132-153, ``step(n)`` runs n iterations of ns.cpp:167-217.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N
from .ops import _check_field, _stream


class NSStepper:
    def __init__(self, shape, nu: float, dt: float, dtype=torch.complex128, device="cuda"):
        nz, ny, nx = shape
        self.shape = tuple(shape)
        self.nu, self.dt = float(nu), float(dt)
        self.dtype = dtype
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.prec = N.SNS_C64 if dtype == torch.complex64 else N.SNS_C128
        self._stream = torch.cuda.current_stream(self.device)
        h = C.c_void_p()
        N.call("sns_ns_create", C.byref(h), nx, ny, nz, self.nu, self.dt, self.prec,
               C.c_void_p(self._stream.cuda_stream))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            N.lib().sns_ns_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _vec(self, v):
        v = list(v)
        for f in v:
            if _check_field(f) != self.prec or tuple(f.shape) != self.shape:
                raise ValueError("vector components must match the stepper's shape and dtype")
        return N.ptr3([f.data_ptr() for f in v])

    def bootstrap(self, V0, omega0):
        N.call("sns_ns_bootstrap", self.h, self._vec(V0), self._vec(omega0))

    def set_state(self, V1, cross0):
        N.call("sns_ns_set_state", self.h, self._vec(V1), self._vec(cross0))

    def step(self, n: int = 1):
        N.call("sns_ns_step", self.h, int(n))

    def state(self):
        mk = lambda: [torch.empty(self.shape, dtype=self.dtype, device=self.device) for _ in range(3)]
        V1, w1, c0 = mk(), mk(), mk()
        N.call("sns_ns_get_state", self.h, self._vec(V1), self._vec(w1), self._vec(c0))
        return {"V1": V1, "omega1": w1, "cross0": c0}

    def stats(self):
        v = [C.c_double() for _ in range(4)]
        N.call("sns_ns_stats", self.h, *[C.byref(x) for x in v])
        return {"div_avg": v[0].value, "energy": v[1].value, "enstrophy": v[2].value,
                "max_div": v[3].value}

    def launches_per_step(self) -> int:
        return N.lib().sns_ns_launches_per_step(self.h)

    def profile(self, enable: bool = True):
        """Record CUDA events between the passes of every following step."""
        N.call("sns_ns_profile", self.h, int(bool(enable)))

    def pass_times(self):
        """[(summed ms, launches)] per pass since profiling was enabled."""
        tot = (C.c_double * 8)()
        cnt = (C.c_int * 8)()
        n = N.lib().sns_ns_pass_times(self.h, tot, cnt, 8)
        if n < 0:
            N.check("sns_ns_pass_times", n)
        return [(tot[i], cnt[i]) for i in range(n)]
