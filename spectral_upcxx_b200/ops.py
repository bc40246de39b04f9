"""Python entry points over the C-ABI for torch device tensors.

Fields are contiguous CUDA tensors of dtype complex64 or complex128 and shape
(nz, ny, nx) -- x fastest, the reference layout n = i + nx*j + nx*ny*k
(src/Scalar.cpp:683).  Work is queued on torch's current stream.  Every call
goes to libspectral_b200.so; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import torch

from . import _native as N


def _prec(t: torch.Tensor) -> int:
    if t.dtype == torch.complex64:
        return N.SNS_C64
    if t.dtype == torch.complex128:
        return N.SNS_C128
    raise TypeError(f"fields must be complex64 or complex128, got {t.dtype}")


def _check_field(t: torch.Tensor):
    if not t.is_cuda:
        raise ValueError("fields must be CUDA tensors")
    if not t.is_contiguous():
        raise ValueError("fields must be contiguous")
    if t.dim() != 3:
        raise ValueError("fields have shape (nz, ny, nx)")
    return _prec(t)


def _dims(t):
    nz, ny, nx = t.shape
    return nx, ny, nz


def _stream(t=None):
    dev = t.device if t is not None else None
    return C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)


def _same(fields):
    p = _check_field(fields[0])
    for f in fields[1:]:
        if _check_field(f) != p or f.shape != fields[0].shape or f.device != fields[0].device:
            raise ValueError("fields must share dtype, shape and device")
    return p


def fft3d(fields, direction: int, normalise: bool = False, zero_nyquist: bool = False):
    """In-place unnormalised 3D DFT of one field or a list of up to 6 fields.

    direction -1 is exp(-i..) (Scalar::forward's transform(-1)), +1 the inverse.
    """
    fs = [fields] if isinstance(fields, torch.Tensor) else list(fields)
    p = _same(fs)
    flags = (N.SNS_FFT_NORMALISE if normalise else 0) | (N.SNS_FFT_ZERO_NYQUIST if zero_nyquist else 0)
    N.call("sns_fft3d_many", N.ptrs([f.data_ptr() for f in fs]), len(fs), *_dims(fs[0]),
           int(direction), flags, p, _stream(fs[0]))
    return fields


def fft3d_tune(shape, dtype=torch.complex64, nfields: int = 1, device=None):
    """Choose the 3D transform plan of `nfields` fields of `shape` (nz, ny, nx)
    by measurement on scratch fields (sns_fft3d_tune); cached per device and
    shape, used by every later fft3d of that shape."""
    nz, ny, nx = shape
    prec = N.SNS_C128 if dtype == torch.complex128 else N.SNS_C64
    dev = torch.device(device) if device is not None else torch.device(
        "cuda", torch.cuda.current_device())
    s = torch.cuda.current_stream(dev)
    N.call("sns_fft3d_tune", nx, ny, nz, int(nfields), prec, C.c_void_p(s.cuda_stream))


def forward(f: torch.Tensor, zero: bool = True):
    """Scalar::forward (src/Scalar.cpp:208-215): transform(-1) + Nyquist zeroing."""
    return fft3d(f, -1, normalise=False, zero_nyquist=zero)


def inverse(f: torch.Tensor):
    """Scalar::inverse (src/Scalar.cpp:217-229): transform(+1), divide by N."""
    return fft3d(f, +1, normalise=True)


def fft1d_many(data: torch.Tensor, n: int, stride: int, howmany: int, dist: int, direction: int):
    """Batched strided in-place 1D DFTs over a flat complex CUDA tensor."""
    p = _prec(data)
    if not data.is_cuda or not data.is_contiguous():
        raise ValueError("data must be a contiguous CUDA tensor")
    if howmany > 0 and (howmany - 1) * dist + (n - 1) * stride >= data.numel():
        raise ValueError("lines exceed the tensor")
    N.call("sns_fft1d_many", C.c_void_p(data.data_ptr()), n, stride, howmany, dist,
           int(direction), p, _stream(data))
    return data


def zero_high_modes(f):
    p = _check_field(f)
    N.call("sns_zero_high_modes", C.c_void_p(f.data_ptr()), *_dims(f), p, _stream(f))
    return f


def gradient(f):
    p = _check_field(f)
    g = [torch.empty_like(f) for _ in range(3)]
    N.call("sns_gradient", C.c_void_p(f.data_ptr()), *[C.c_void_p(x.data_ptr()) for x in g],
           *_dims(f), p, _stream(f))
    return g


def laplacian(f):
    p = _check_field(f)
    out = torch.empty_like(f)
    N.call("sns_laplacian", C.c_void_p(f.data_ptr()), C.c_void_p(out.data_ptr()), *_dims(f), p,
           _stream(f))
    return out


def laplacian_inverse(f, a: float = 0.0, b: float = 1.0):
    """In place, as Scalar::laplacian_inverse (src/Scalar.cpp:308-334)."""
    p = _check_field(f)
    N.call("sns_laplacian_inverse", C.c_void_p(f.data_ptr()), float(a), float(b), *_dims(f), p,
           _stream(f))
    return f


def curl(v):
    p = _same(list(v))
    out = [torch.empty_like(v[0]) for _ in range(3)]
    N.call("sns_curl", N.ptr3([x.data_ptr() for x in v]), N.ptr3([x.data_ptr() for x in out]),
           *_dims(v[0]), p, _stream(v[0]))
    return out


def divergence(v):
    p = _same(list(v))
    out = torch.empty_like(v[0])
    N.call("sns_divergence", N.ptr3([x.data_ptr() for x in v]), C.c_void_p(out.data_ptr()),
           *_dims(v[0]), p, _stream(v[0]))
    return out


def vector_laplacian(v):
    p = _same(list(v))
    out = [torch.empty_like(v[0]) for _ in range(3)]
    N.call("sns_vector_laplacian", N.ptr3([x.data_ptr() for x in v]),
           N.ptr3([x.data_ptr() for x in out]), *_dims(v[0]), p, _stream(v[0]))
    return out


def cross(a, b):
    """Vector::cross (src/Vector.cpp:66-90) of two Fourier vectors."""
    p = _same(list(a) + list(b))
    out = [torch.empty_like(a[0]) for _ in range(3)]
    N.call("sns_cross", N.ptr3([x.data_ptr() for x in a]), N.ptr3([x.data_ptr() for x in b]),
           N.ptr3([x.data_ptr() for x in out]), *_dims(a[0]), p, _stream(a[0]))
    return out


def average(f) -> float:
    """Scalar::average: mean |f_i| (synchronises)."""
    p = _prec(f)
    out = C.c_double(0.0)
    N.call("sns_average_abs", C.c_void_p(f.data_ptr()), f.numel(), p, C.byref(out), _stream(f))
    return out.value


def axpby(alpha: float, x, beta: float = 0.0, y=None, out=None):
    p = _prec(x)
    out = torch.empty_like(x) if out is None else out
    N.call("sns_axpby", float(alpha), C.c_void_p(x.data_ptr()), float(beta),
           C.c_void_p(y.data_ptr() if y is not None else 0), C.c_void_p(out.data_ptr()), x.numel(),
           p, _stream(x))
    return out


def mul(a, b, out=None):
    p = _prec(a)
    out = torch.empty_like(a) if out is None else out
    N.call("sns_mul", C.c_void_p(a.data_ptr()), C.c_void_p(b.data_ptr()),
           C.c_void_p(out.data_ptr()), a.numel(), p, _stream(a))
    return out
