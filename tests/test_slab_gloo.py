"""The data movement of the slab-distributed 3D transform with two gloo ranks
on the CPU: the transposes through torch.distributed.all_to_all_single, with a
stand-in for the local line passes (torch.fft on the CPU tensors, supplied by
the test) -- the decomposition must give the full 3D DFT."""
import os

import numpy as np
import torch
import torch.multiprocessing as mp


def _torch_axes(t, dims, axes, direction, scale):
    v = t.view(dims)
    for bit, dim in ((0, 2), (1, 1), (2, 0)):
        if (axes >> bit) & 1:
            n = v.shape[dim]
            v.copy_(torch.fft.fft(v, dim=dim) if direction < 0 else torch.fft.ifft(v, dim=dim) * n)
    if scale != 1.0:
        v.mul_(scale)


def _rank(rank, world, port, shape, q):
    import torch.distributed as dist
    from spectral_upcxx_b200.slab import SlabFFT3D
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        r = np.random.default_rng(5)
        f = r.uniform(-1, 1, shape) + 1j * r.uniform(-1, 1, shape)
        nzl = shape[0] // world
        fft = SlabFFT3D(shape, world, axes_fn=_torch_axes)
        mine = torch.from_numpy(np.ascontiguousarray(f[rank * nzl:(rank + 1) * nzl]))
        fwd = mine.clone()
        fft.transform([fwd], -1)
        inv = fwd.clone()
        fft.inverse([inv])
        want = np.fft.fftn(f)[rank * nzl:(rank + 1) * nzl]
        e1 = np.linalg.norm(fwd.numpy() - want) / np.linalg.norm(want)
        e2 = np.linalg.norm(inv.numpy() - mine.numpy()) / np.linalg.norm(mine.numpy())
        q.put((rank, float(e1), float(e2)))
    finally:
        dist.destroy_process_group()


def test_slab_transposes_with_two_gloo_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29600 + (os.getpid() % 200)
    shape = (8, 16, 4)
    ps = [ctx.Process(target=_rank, args=(r, 2, port, shape, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    for rank, e_fwd, e_inv in res:
        assert e_fwd < 1e-13 and e_inv < 1e-13, (rank, e_fwd, e_inv)
