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
    """real=True keeps the half spectrum of a real velocity field
    (sns_ns_create_real); the interface is unchanged.  tune=True chooses the
    plan's tile shapes by measurement before the first use (sns_ns_tune; cached
    per device and shape)."""

    def __init__(self, shape, nu: float, dt: float, dtype=torch.complex128, device="cuda",
                 real: bool = False, tune: bool = False):
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
        N.call("sns_ns_create_real" if real else "sns_ns_create", C.byref(h), nx, ny, nz, self.nu,
               self.dt, self.prec, C.c_void_p(self._stream.cuda_stream))
        self.h = h
        if tune:
            N.call("sns_ns_tune", self.h)

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

    def set_closure(self, model: int, cs_delta2: float = 0.0, mlp=None, kc: float = 0.0):
        """Eddy-viscosity closure of every following step: N.SNS_CLOSURE_NONE,
        _SMAGORINSKY (nu_t = cs_delta2 sqrt(2 S:S)) or _MLP (`mlp`: the packed
        model tensor, kept alive by the caller); kc > 0 evolves only the modes
        |k| <= kc."""
        self._mlp = mlp
        N.call("sns_ns_set_closure", self.h, int(model), float(cs_delta2),
               C.c_void_p(mlp.data_ptr()) if mlp is not None else None, float(kc))

    def set_sgs_band(self, k_lo: float = 0.0, k_hi: float = 0.0):
        """Weight the closure's eddy-stress divergence by the ramp
        clamp((|k| - k_lo) / (k_hi - k_lo), 0, 1); k_hi <= k_lo: the modes
        |k| > k_lo at full weight (default: every mode)."""
        N.call("sns_ns_set_sgs_band", self.h, float(k_lo), float(k_hi))

    def velocity(self, out=None):
        """The Fourier velocity V1 (into `out`, three device fields, if given)."""
        if out is None:
            out = [torch.empty(self.shape, dtype=self.dtype, device=self.device) for _ in range(3)]
        N.call("sns_ns_get_state", self.h, self._vec(out), None, None)
        return out

    def stats(self):
        v = [C.c_double() for _ in range(4)]
        N.call("sns_ns_stats", self.h, *[C.byref(x) for x in v])
        return {"div_avg": v[0].value, "energy": v[1].value, "enstrophy": v[2].value,
                "max_div": v[3].value}

    def stats_async(self, out: torch.Tensor):
        """Queue the four diagnostics (div_avg, energy, enstrophy, max_div) into
        `out` (4 float64, pinned host or device) without synchronising."""
        assert out.dtype == torch.float64 and out.numel() >= 4 and out.is_contiguous()
        N.call("sns_ns_stats_async", self.h, C.c_void_p(out.data_ptr()))
        return out

    def launches_per_step(self) -> int:
        return N.lib().sns_ns_launches_per_step(self.h)

    def describe(self) -> str:
        """The plan chosen for this box: pass structure and tile shapes."""
        buf = C.create_string_buffer(256)
        N.lib().sns_ns_describe(self.h, buf, 256)
        return buf.value.decode()

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


ENS_GRAPH, ENS_EAGER, ENS_SEQUENTIAL = 0, 1, 2


class NSEnsemble:
    """Independent boxes of uneven size advanced together (sns_ens_*).

    ``shapes`` holds one (nz, ny, nx) per box and ``nus`` one viscosity per
    box; dt and dtype are shared.  Each box follows ns.cpp exactly as
    ``NSStepper`` does; one ensemble step is five launches over every box.
    """

    def __init__(self, shapes, nus, dt: float, dtype=torch.complex64, tune: bool = True,
                 device="cuda"):
        shapes = [tuple(int(n) for n in s) for s in shapes]
        if len(shapes) != len(nus):
            raise ValueError("one viscosity per box")
        self.shapes = shapes
        self.nus = [float(v) for v in nus]
        self.dt = float(dt)
        self.dtype = dtype
        self.device = torch.device(device)
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self.prec = N.SNS_C64 if dtype == torch.complex64 else N.SNS_C128
        self._stream = torch.cuda.current_stream(self.device)
        dims = (C.c_int64 * (3 * len(shapes)))()
        for i, (nz, ny, nx) in enumerate(shapes):
            dims[3 * i], dims[3 * i + 1], dims[3 * i + 2] = nx, ny, nz
        nu = (C.c_double * len(shapes))(*self.nus)
        h = C.c_void_p()
        N.call("sns_ens_create", C.byref(h), len(shapes), dims, nu, self.dt, self.prec,
               int(bool(tune)), C.c_void_p(self._stream.cuda_stream))
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            N.lib().sns_ens_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self):
        return len(self.shapes)

    def _vec(self, box, v):
        v = list(v)
        for f in v:
            if _check_field(f) != self.prec or tuple(f.shape) != self.shapes[box]:
                raise ValueError("vector components must match the box's shape and dtype")
        return N.ptr3([f.data_ptr() for f in v])

    def bootstrap(self, box: int, V0, omega0):
        N.call("sns_ens_bootstrap", self.h, int(box), self._vec(box, V0), self._vec(box, omega0))

    def set_state(self, box: int, V1, cross0):
        N.call("sns_ens_set_state", self.h, int(box), self._vec(box, V1), self._vec(box, cross0))

    def step(self, n: int = 1, mode: int = ENS_GRAPH):
        N.call("sns_ens_step", self.h, int(n), int(mode))

    def state(self, box: int):
        shape = self.shapes[box]
        mk = lambda: [torch.empty(shape, dtype=self.dtype, device=self.device) for _ in range(3)]
        V1, w1, c0 = mk(), mk(), mk()
        N.call("sns_ens_get_state", self.h, int(box), self._vec(box, V1), self._vec(box, w1),
               self._vec(box, c0))
        return {"V1": V1, "omega1": w1, "cross0": c0}

    def stats(self):
        """Per box: div_avg, energy, enstrophy, max_div (as sns_ns_stats)."""
        out = (C.c_double * (4 * len(self.shapes)))()
        N.call("sns_ens_stats", self.h, out)
        keys = ("div_avg", "energy", "enstrophy", "max_div")
        return [dict(zip(keys, out[4 * i:4 * i + 4])) for i in range(len(self.shapes))]

    def tuning(self):
        """Per stage: (threads per CTA, line-run cap, persistent grid)."""
        out = (C.c_int * 15)()
        n = N.lib().sns_ens_tuning(self.h, out, 15)
        if n < 0:
            N.check("sns_ens_tuning", n)
        return [tuple(out[3 * s:3 * s + 3]) for s in range(n)]

    def launches_per_step(self, mode: int = ENS_GRAPH) -> int:
        return N.lib().sns_ens_launches_per_step(self.h, int(mode))

    def stage_times(self, n: int = 5):
        """Run n steps with events between the stages; mean ms per stage."""
        ms = (C.c_double * 5)()
        k = N.lib().sns_ens_stage_times(self.h, int(n), ms)
        if k < 0:
            N.check("sns_ens_stage_times", k)
        return list(ms[:k])
