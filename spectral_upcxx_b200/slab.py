"""Slab-distributed 3D FFT: the z-slab decomposition of the reference's
Scalar::transform (src/Scalar.cpp:400-646) on one GPU per rank.

Each of P ranks holds nz/P consecutive z planes of an nx * ny * nz field (the
reference's m_Nz planes per UPC++ rank, src/Scalar.cpp:83-102).  A transform
(either direction, unnormalised) runs:

  1. the x and y line passes of the rank's own planes (sns_fft3d_axes);
  2. the transpose: the rank's planes are cut into P blocks of ny/P rows and
     block j goes to rank j -- one all-to-all.  Rank j then holds rows
     [j ny/P, (j+1) ny/P) of every z plane, laid out [z][row][x], which is the
     reference's `tmp` (src/Scalar.cpp:467-497) and a plain nx * ny/P * nz box;
  3. the z line passes of that box;
  4. the transpose back (the reverse all-to-all, src/Scalar.cpp:570-613) and the
     scatter of the received blocks into the rank's planes.

forward() zeroes the global Nyquist planes afterwards (Scalar::forward,
src/Scalar.cpp:208-215, with ZERO); inverse() scales by 1/(nx ny nz) in the z
pass (Scalar::inverse, src/Scalar.cpp:217-229).  The local transforms are the
library's line passes; the all-to-all is torch.distributed's (NCCL between
GPUs).  One object can also drive several slabs held by one process -- the
`ranks` of an in-process exchange -- which is how the decomposition is checked
on a single GPU.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, List, Optional, Sequence

import torch

from . import _native as N


def _stream(t: torch.Tensor):
    return C.c_void_p(torch.cuda.current_stream(t.device).cuda_stream)


def library_axes(t: torch.Tensor, dims, axes: int, direction: int, scale: float) -> None:
    """Line passes of the axes in the bit mask `axes` of the box `dims`
    (nz, ny, nx) held contiguously by `t` (sns_fft3d_axes)."""
    nz, ny, nx = dims
    prec = N.SNS_C128 if t.dtype == torch.complex128 else N.SNS_C64
    N.call("sns_fft3d_axes", C.c_void_p(t.data_ptr()), nx, ny, nz, int(axes), int(direction),
           float(scale), prec, _stream(t))


class SlabFFT3D:
    """3D transform of a field distributed over P ranks in z slabs.

    shape: the global (nz, ny, nx); nz and ny must be multiples of P.
    exchange: all-to-all of equal blocks, called with the list of this
        process's send buffers and returning the receive buffers in the same
        order; by default torch.distributed.all_to_all_single over `group`
        (one slab per process).
    axes_fn: the local line passes (the library's by default); a test of the
        data movement may substitute another implementation.
    """

    def __init__(self, shape: Sequence[int], ranks: int, group=None,
                 exchange: Optional[Callable[[List[torch.Tensor]], List[torch.Tensor]]] = None,
                 axes_fn: Callable = library_axes):
        nz, ny, nx = shape
        if nz % ranks or ny % ranks:
            raise ValueError(f"nz = {nz} and ny = {ny} must be multiples of the {ranks} ranks")
        self.shape = (nz, ny, nx)
        self.P = ranks
        self.group = group
        self.exchange = exchange or self._all_to_all
        self.axes_fn = axes_fn

    # -- the collective -------------------------------------------------------
    def _all_to_all(self, sends: List[torch.Tensor]) -> List[torch.Tensor]:
        import torch.distributed as dist
        out = []
        for s in sends:
            r = torch.empty_like(s)
            dist.all_to_all_single(r, s, group=self.group)
            out.append(r)
        return out

    # -- one transform of the slabs this process holds ------------------------
    def transform(self, slabs: List[torch.Tensor], direction: int, scale: float = 1.0) -> None:
        nz, ny, nx = self.shape
        P = self.P
        nzl, nyl = nz // P, ny // P
        for s in slabs:
            if s.shape != (nzl, ny, nx) or not s.is_contiguous():
                raise ValueError(f"a slab is a contiguous ({nzl}, {ny}, {nx}) tensor")
        # 1. x and y lines of the own planes
        for s in slabs:
            self.axes_fn(s, (nzl, ny, nx), 0b011, direction, 1.0)
        # 2. rows [j nyl, (j+1) nyl) of every own plane -> rank j
        sends = [torch.cat([s[:, j * nyl:(j + 1) * nyl, :].reshape(-1) for j in range(P)])
                 for s in slabs]
        recvs = self.exchange(sends)
        # the received blocks, rank-major, are the planes of all z in order: an
        # nx * nyl * nz box
        # 3. z lines of that box (the scale rides on this pass)
        for r in recvs:
            self.axes_fn(r, (nz, nyl, nx), 0b100, direction, scale)
        # 4. back: block i of the box (planes [i nzl, (i+1) nzl)) -> rank i
        backs = self.exchange([r.contiguous() for r in recvs])
        for s, b in zip(slabs, backs):
            b = b.view(P, nzl, nyl, nx)
            for j in range(P):
                s[:, j * nyl:(j + 1) * nyl, :].copy_(b[j])

    def forward(self, slabs: List[torch.Tensor], ranks_of: Sequence[int], zero: bool = True):
        """Scalar::forward on the slabs of the ranks `ranks_of` (transform(-1),
        then the global Nyquist planes zeroed)."""
        self.transform(slabs, -1)
        if zero:
            nz, ny, nx = self.shape
            nzl = nz // self.P
            for s, rank in zip(slabs, ranks_of):
                s[:, ny // 2, :] = 0
                s[:, :, nx // 2] = 0
                z = nz // 2 - rank * nzl
                if 0 <= z < nzl:
                    s[z] = 0

    def inverse(self, slabs: List[torch.Tensor]):
        """Scalar::inverse on the slabs (transform(+1) divided by nx ny nz)."""
        nz, ny, nx = self.shape
        self.transform(slabs, +1, 1.0 / (nz * ny * nx))


def in_process_exchange(sends: List[torch.Tensor]) -> List[torch.Tensor]:
    """All-to-all among the P slabs held by one process: block j of sender i
    becomes block i of receiver j (device copies)."""
    P = len(sends)
    blocks = [s.view(P, -1) for s in sends]
    return [torch.cat([blocks[i][j] for i in range(P)]) for j in range(P)]


def slab_cross(fft: SlabFFT3D, a: List[List[torch.Tensor]], b: List[List[torch.Tensor]],
               ranks_of: Sequence[int]) -> List[List[torch.Tensor]]:
    """Vector::cross (src/Vector.cpp:66-90) of two Fourier vectors held as z
    slabs: inverse copies of both operands, the complex point-wise a x b of
    each rank's own planes, forward with Nyquist zeroing.  a[c][k] is component
    c of the k-th slab this process holds; returns the product in the same
    form."""
    ua = [[x.clone() for x in comp] for comp in a]
    ub = [[x.clone() for x in comp] for comp in b]
    for comp in ua + ub:
        fft.inverse(comp)
    out = [[ua[1][k] * ub[2][k] - ua[2][k] * ub[1][k] for k in range(len(ranks_of))],
           [ua[2][k] * ub[0][k] - ua[0][k] * ub[2][k] for k in range(len(ranks_of))],
           [ua[0][k] * ub[1][k] - ua[1][k] * ub[0][k] for k in range(len(ranks_of))]]
    for comp in out:
        fft.forward(comp, ranks_of)
    return out
