"""TEST INFRASTRUCTURE ONLY -- ctypes bindings to the CPU oracle (checker).

Two libraries sit behind this module:

* ``oracle/_build/liboracle.so`` -- the project's FP64 C restatement of the
  reference's Scalar/Vector/Operators arithmetic and exec/ns.cpp step
  (orc_spectral.c), built from this directory by ``make -C oracle``.
* ``oracle/_ref/libref.so`` (+ ``libref_nozero.so``) -- the reference's own
  src/*.cpp compiled in place against the project-written UPC++/FFTW shims,
  with the project-written entry layer ref_capi.cpp.  Built by
  ``make -C oracle ref`` where the reference tree is available; the built
  files travel with the repository snapshot.

Only tests/, bench.py's CPU-baseline leg and __graft_entry__.smoke() may
import this module; the product never does.  Fields are numpy complex128
arrays of shape (nz, ny, nx) (x fastest, the reference layout
n = i + nx*j + nx*ny*k, src/Scalar.cpp:683).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = {}

_dp = C.POINTER(C.c_double)
_i64 = C.c_int64


def build(ref: str | None = None) -> None:
    """Compile the oracle, and the in-place build of the reference when given
    the path of its source tree."""
    cmd = ["make", "-s", "-C", HERE, "all"]
    if ref:
        cmd += ["ref", f"REF={ref}"]
    subprocess.run(cmd, check=True)


def _ptr(a: np.ndarray):
    assert a.dtype == np.complex128 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_dp)


def _ptr3(vs):
    arr = (_dp * 3)(*[_ptr(v) for v in vs])
    return arr


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.orc_transform.argtypes = [_dp, _i64, _i64, _i64, C.c_int]
        L.orc_forward.argtypes = [_dp, _i64, _i64, _i64, C.c_int]
        L.orc_inverse.argtypes = [_dp, _i64, _i64, _i64]
        L.orc_zero_high_modes.argtypes = [_dp, _i64, _i64, _i64]
        L.orc_gradient.argtypes = [_dp, _dp, _dp, _dp, _i64, _i64, _i64]
        L.orc_laplacian.argtypes = [_dp, _dp, _i64, _i64, _i64]
        L.orc_laplacian_inverse.argtypes = [_dp, C.c_double, C.c_double, _i64, _i64, _i64]
        for f in ("orc_curl", "orc_vlaplacian"):
            getattr(L, f).argtypes = [C.POINTER(_dp), C.POINTER(_dp), _i64, _i64, _i64]
        L.orc_divergence.argtypes = [C.POINTER(_dp), _dp, _i64, _i64, _i64]
        L.orc_cross.argtypes = [C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), _i64, _i64,
                                _i64, C.c_int]
        L.orc_average.argtypes = [_dp, _i64]
        L.orc_average.restype = C.c_double
        L.orc_ns_create.argtypes = [_i64, _i64, _i64, C.c_double, C.c_double, C.c_int]
        L.orc_ns_create.restype = C.c_void_p
        L.orc_ns_destroy.argtypes = [C.c_void_p]
        L.orc_ns_bootstrap.argtypes = [C.c_void_p, C.POINTER(_dp), C.POINTER(_dp)]
        L.orc_ns_step.argtypes = [C.c_void_p]
        L.orc_ns_step.restype = C.c_double
        L.orc_ns_field.argtypes = [C.c_void_p, C.c_int, C.c_int]
        L.orc_ns_field.restype = C.c_void_p
        L.orc_velocity_from_vorticity_z.argtypes = [_dp, C.POINTER(_dp), _i64, _i64, _i64]
        L.orc_ic_ns_vortices.argtypes = [_dp, _i64, _i64, _i64]
        _LIB = L
    return _LIB


def have_ref() -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", "libref.so"))


def ref(zero: bool = True):
    """The reference's own code (built in place), with or without ZERO."""
    key = bool(zero)
    if key not in _REF:
        name = "libref.so" if zero else "libref_nozero.so"
        path = os.path.join(HERE, "_ref", name)
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` with the reference tree present")
        L = C.CDLL(path)
        L.ref_set_threads.argtypes = [C.c_int]
        L.ref_set_threads.restype = C.c_int
        for f in ("ref_forward", "ref_inverse"):
            getattr(L, f).argtypes = [_dp, _i64, _i64, _i64]
        L.ref_fft_roundtrip.argtypes = [_dp, _i64, _i64, _i64, C.c_int]
        L.ref_fft_roundtrip.restype = C.c_double
        L.ref_gradient.argtypes = [_dp, _dp, _dp, _dp, _i64, _i64, _i64]
        L.ref_laplacian.argtypes = [_dp, _dp, _i64, _i64, _i64]
        L.ref_laplacian_inverse.argtypes = [_dp, C.c_double, C.c_double, _i64, _i64, _i64]
        for f in ("ref_curl", "ref_vlaplacian"):
            getattr(L, f).argtypes = [C.POINTER(_dp), C.POINTER(_dp), _i64, _i64, _i64]
        L.ref_divergence.argtypes = [C.POINTER(_dp), _dp, _i64, _i64, _i64]
        L.ref_cross.argtypes = [C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), _i64, _i64, _i64]
        L.ref_average.argtypes = [_dp, _i64, _i64, _i64]
        L.ref_average.restype = C.c_double
        L.ref_ns_vortex_ic.argtypes = [C.POINTER(_dp), C.POINTER(_dp), _i64, _i64, _i64]
        L.ref_ns_run.argtypes = [C.POINTER(_dp), C.POINTER(_dp), _i64, _i64, _i64, C.c_double,
                                 C.c_double, C.c_int, C.POINTER(_dp), C.POINTER(_dp),
                                 C.POINTER(_dp), _dp]
        L.ref_ns_run.restype = C.c_double
        L.ref_ns_steps.argtypes = [C.POINTER(_dp), C.POINTER(_dp), C.POINTER(_dp), _i64, _i64,
                                   _i64, C.c_double, C.c_double, C.c_int]
        L.ref_ns_steps.restype = C.c_double
        L.ref_particles.argtypes = [C.c_uint, _i64, C.POINTER(_dp), _i64, _i64, _i64, C.c_double,
                                    C.c_int, _dp, _dp, _dp]
        L.ref_particles.restype = None
        _REF[key] = L
    return _REF[key]


def _dims(a):
    nz, ny, nx = a.shape
    return nx, ny, nz


# ---------------- C restatement ----------------

def transform(f: np.ndarray, direction: int) -> np.ndarray:
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    lib().orc_transform(_ptr(out), *_dims(out), int(direction))
    return out


def forward(f, zero=True):
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    lib().orc_forward(_ptr(out), *_dims(out), int(bool(zero)))
    return out


def inverse(f):
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    lib().orc_inverse(_ptr(out), *_dims(out))
    return out


def zero_high_modes(f):
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    lib().orc_zero_high_modes(_ptr(out), *_dims(out))
    return out


def gradient(f):
    f = np.ascontiguousarray(f, dtype=np.complex128)
    g = [np.empty_like(f) for _ in range(3)]
    lib().orc_gradient(_ptr(f), _ptr(g[0]), _ptr(g[1]), _ptr(g[2]), *_dims(f))
    return g


def laplacian(f):
    f = np.ascontiguousarray(f, dtype=np.complex128)
    out = np.empty_like(f)
    lib().orc_laplacian(_ptr(f), _ptr(out), *_dims(f))
    return out


def laplacian_inverse(f, a=0.0, b=1.0):
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    lib().orc_laplacian_inverse(_ptr(out), a, b, *_dims(out))
    return out


def _vin(v):
    return [np.ascontiguousarray(c, dtype=np.complex128) for c in v]


def curl(v):
    v = _vin(v)
    out = [np.empty_like(v[0]) for _ in range(3)]
    lib().orc_curl(_ptr3(v), _ptr3(out), *_dims(v[0]))
    return out


def vlaplacian(v):
    v = _vin(v)
    out = [np.empty_like(v[0]) for _ in range(3)]
    lib().orc_vlaplacian(_ptr3(v), _ptr3(out), *_dims(v[0]))
    return out


def divergence(v):
    v = _vin(v)
    out = np.empty_like(v[0])
    lib().orc_divergence(_ptr3(v), _ptr(out), *_dims(v[0]))
    return out


def cross(a, b, zero=True):
    a, b = _vin(a), _vin(b)
    out = [np.empty_like(a[0]) for _ in range(3)]
    lib().orc_cross(_ptr3(a), _ptr3(b), _ptr3(out), *_dims(a[0]), int(bool(zero)))
    return out


def average(f):
    f = np.ascontiguousarray(f, dtype=np.complex128)
    return lib().orc_average(_ptr(f), f.size)


def velocity_from_vorticity_z(wz_hat):
    wz_hat = np.ascontiguousarray(wz_hat, dtype=np.complex128)
    out = [np.empty_like(wz_hat) for _ in range(3)]
    lib().orc_velocity_from_vorticity_z(_ptr(wz_hat), _ptr3(out), *_dims(wz_hat))
    return out


def ic_ns_vortices(n):
    w = np.zeros((n, n, n), np.complex128)
    lib().orc_ic_ns_vortices(_ptr(w), n, n, n)
    return w


class NS:
    """exec/ns.cpp integrator on the C restatement."""

    def __init__(self, shape, nu, dt, zero=True):
        nz, ny, nx = shape
        self.shape = shape
        self.h = lib().orc_ns_create(nx, ny, nz, nu, dt, int(bool(zero)))
        self._n = nx * ny * nz

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_ns_destroy(self.h)
            self.h = None

    def bootstrap(self, V0, omega0):
        V0, omega0 = _vin(V0), _vin(omega0)
        lib().orc_ns_bootstrap(self.h, _ptr3(V0), _ptr3(omega0))

    def step(self) -> float:
        return lib().orc_ns_step(self.h)

    def _field(self, slot: int, d: int) -> np.ndarray:
        addr = lib().orc_ns_field(self.h, slot, d)
        buf = (C.c_double * (2 * self._n)).from_address(addr)
        return np.frombuffer(buf, dtype=np.complex128).reshape(self.shape).copy()

    def state(self):
        return {name: [self._field(slot, d) for d in range(3)]
                for slot, name in enumerate(["V0", "V1", "omega0", "omega1", "cross0"])}


# ---------------- the reference itself ----------------

def ref_forward(f, zero=True):
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    ref(zero).ref_forward(_ptr(out), *_dims(out))
    return out


def ref_inverse(f):
    out = np.ascontiguousarray(f, dtype=np.complex128).copy()
    ref(True).ref_inverse(_ptr(out), *_dims(out))
    return out


def ref_ns_vortex_ic(n):
    V0 = [np.zeros((n, n, n), np.complex128) for _ in range(3)]
    w0 = [np.zeros((n, n, n), np.complex128) for _ in range(3)]
    ref(True).ref_ns_vortex_ic(_ptr3(V0), _ptr3(w0), n, n, n)
    return V0, w0


def ref_ns_steps(V1, omega1, cross0, nu, dt, nsteps, threads=0):
    """Continue the reference's ns.cpp loop from a state (updated in place);
    returns the loop's wall seconds."""
    L = ref(True)
    if threads:
        L.ref_set_threads(int(threads))
    nx, ny, nz = _dims(V1[0])
    return L.ref_ns_steps(_ptr3(V1), _ptr3(omega1), _ptr3(cross0), nx, ny, nz, nu, dt, nsteps)


def port_ns_seconds(V1, omega1, cross0, nu, dt, nsteps):
    """The C restatement's step, timed the same way (used when the reference
    build is absent)."""
    import time
    ns = NS(V1[0].shape, nu, dt)
    for d in range(3):
        for slot, src in ((1, V1), (3, omega1), (4, cross0)):
            addr = lib().orc_ns_field(ns.h, slot, d)
            buf = (C.c_double * (2 * V1[0].size)).from_address(addr)
            np.frombuffer(buf, dtype=np.complex128)[:] = np.ascontiguousarray(src[d]).ravel()
    t0 = time.perf_counter()
    for _ in range(nsteps):
        ns.step()
    return time.perf_counter() - t0


def ref_ns_run(V0, omega0, nu, dt, nsteps):
    V0, omega0 = _vin(V0), _vin(omega0)
    nx, ny, nz = _dims(V0[0])
    V1 = [np.empty_like(V0[0]) for _ in range(3)]
    w1 = [np.empty_like(V0[0]) for _ in range(3)]
    c0 = [np.empty_like(V0[0]) for _ in range(3)]
    divs = np.zeros(max(nsteps, 1), np.float64)
    el = ref(True).ref_ns_run(_ptr3(V0), _ptr3(omega0), nx, ny, nz, nu, dt, nsteps,
                              _ptr3(V1), _ptr3(w1), _ptr3(c0),
                              divs.ctypes.data_as(_dp))
    return {"V1": V1, "omega1": w1, "cross0": c0, "div_avgs": divs[:nsteps], "seconds": el}


def ref_particles(seed, n, u, K, nsteps):
    """src/Particle.cpp through the reference build: srand(seed), n particles,
    nsteps moves through the physical velocity u (three complex arrays).
    Returns (initial positions, final positions, energies)."""
    u = [np.ascontiguousarray(x, dtype=np.complex128) for x in u]
    nz, ny, nx = u[0].shape
    loc0 = np.zeros((n, 3))
    loc = np.zeros((n, 3))
    e = np.zeros(n)
    d = lambda a: a.ctypes.data_as(_dp)
    ref(True).ref_particles(seed, n, _ptr3(u), nx, ny, nz, K, nsteps, d(loc0), d(loc), d(e))
    return loc0, loc, e
