"""Batched ensemble of uneven NS boxes (sns_ens_*).

Every box of an ensemble must advance as the single-box stepper advances it.
The sequential mode runs the single-box kernels and matches bit for bit; the
stage kernels of the graph and eager modes run the same tile bodies and match
to rounding (relative L2 < 2e-6 complex64, < 1e-14 complex128).  One
complex128 box is also checked directly against the FP64 oracle of the ns.cpp
sequence (relative L2 <= 1e-12 per field)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


def random_velocity_hat(shape, seed):
    """Fourier velocity of a divergence-free random field on an nz*ny*nx box,
    Nyquist planes zeroed."""
    from spectral_upcxx_b200 import ic
    nz, ny, nx = shape
    r = ic.rng(seed)
    kz, ky, kx = np.meshgrid(ic.wavenumbers(nz), ic.wavenumbers(ny), ic.wavenumbers(nx),
                             indexing="ij")
    k2 = kx * kx + ky * ky + kz * kz
    amp = np.exp(-k2 / 16.0)
    V = [amp * (r.standard_normal(shape) + 1j * r.standard_normal(shape)) for _ in range(3)]
    # project out the divergence: V -= k (k . V) / |k|^2
    kd = kx * V[0] + ky * V[1] + kz * V[2]
    with np.errstate(invalid="ignore", divide="ignore"):
        q = np.where(k2 > 0, kd / np.where(k2 > 0, k2, 1), 0)
    V = [V[0] - kx * q, V[1] - ky * q, V[2] - kz * q]
    for c in V:
        c[nz // 2, :, :] = 0
        c[:, ny // 2, :] = 0
        c[:, :, nx // 2] = 0
    return [np.ascontiguousarray(c) for c in V]


SHAPES = [(32, 32, 32), (64, 64, 64), (32, 32, 32), (16, 32, 64), (128, 128, 128), (16, 16, 16)]


def _build(sns, cuda, dtype, shapes, nus, dt, tune):
    import os
    ens = sns.NSEnsemble(shapes, nus, dt, dtype, tune=tune)
    singles = []
    # the ensemble steps its boxes with the fused K1 tile: single steppers of
    # the same plan (not the opt-in K1 line-pass variant)
    os.environ["SNS_K1_LINES"] = "0"
    for b, shape in enumerate(shapes):
        Vd = [dev(x, dtype, cuda) for x in random_velocity_hat(shape, seed=100 + b)]
        wd = sns.curl(Vd)
        ens.bootstrap(b, Vd, wd)
        st = sns.NSStepper(shape, nus[b], dt, dtype)
        st.bootstrap(Vd, wd)
        singles.append(st)
    del os.environ["SNS_K1_LINES"]
    return ens, singles


@pytest.mark.parametrize("dtype", [torch.complex64, torch.complex128])
@pytest.mark.parametrize("mode", [0, 1, 2])
def test_ensemble_boxes_equal_single_stepper(sns, cuda, dtype, mode):
    shapes = SHAPES
    nus = [1 / 100, 1 / 200, 1 / 300, 1 / 400, 1 / 800, 1 / 150]
    dt = 2e-3
    ens, singles = _build(sns, cuda, dtype, shapes, nus, dt, tune=False)
    ens.step(3, mode=mode)
    for st in singles:
        st.step(3)
    torch.cuda.synchronize()
    # The sequential mode runs the single-box kernels themselves: bit for bit.
    # The stage kernels inline the same tile bodies into other kernels, where
    # the compiler may contract multiply-adds differently: rounding level.
    tol = 0.0 if mode == 2 else (2e-6 if dtype == torch.complex64 else 1e-14)
    for b, st in enumerate(singles):
        got, ref = ens.state(b), st.state()
        for key in ("V1", "cross0", "omega1"):
            for d in range(3):
                if tol == 0.0:
                    assert torch.equal(got[key][d], ref[key][d]), (b, key, d)
                else:
                    assert rel_l2(host(got[key][d]), host(ref[key][d])) < tol, (b, key, d)
    es = ens.stats()
    # the divergence monitors are rounding noise, comparable only bit for bit
    keys = ("div_avg", "energy", "enstrophy", "max_div") if tol == 0.0 else ("energy", "enstrophy")
    stol = 1e-12 if tol == 0.0 else 10 * tol
    for b, st in enumerate(singles):
        ss = st.stats()
        for key in keys:
            assert abs(es[b][key] - ss[key]) <= stol * max(abs(ss[key]), 1e-300), (b, key)
    assert ens.launches_per_step(0) == 5
    assert ens.launches_per_step(2) == 5 * len(shapes)
    ens.close()
    for st in singles:
        st.close()


def test_tuned_ensemble_equals_untuned(sns, cuda):
    """The tuner only changes tile shapes and grid modes, never the result."""
    shapes = [(32, 32, 32)] * 4 + [(64, 64, 64)] * 2 + [(128, 128, 128)]
    nus = list(np.geomspace(1 / 800, 1 / 100, len(shapes)))
    dt = 2e-3
    runs = []
    for tune in (False, True):
        ens = sns.NSEnsemble(shapes, nus, dt, torch.complex64, tune=tune)
        for b, shape in enumerate(shapes):
            Vd = [dev(x, torch.complex64, cuda) for x in random_velocity_hat(shape, seed=7 + b)]
            ens.bootstrap(b, Vd, sns.curl(Vd))
        ens.step(5)
        runs.append(ens)
    cfg = runs[1].tuning()
    assert len(cfg) == 5
    for threads, wcap, persistent in cfg:
        assert threads in (96, 128, 192, 256, 384, 512, 768)
        assert wcap in (1, 4, 8, 16) and persistent in (0, 1)
    for b in range(len(shapes)):
        a, c = runs[0].state(b), runs[1].state(b)
        for d in range(3):
            assert rel_l2(host(a["V1"][d]), host(c["V1"][d])) < 2e-6, b
    for r in runs:
        r.close()


def test_fp64_box_in_ensemble_matches_oracle(sns, oracle, cuda):
    """A 16^3 and a 32^3 complex128 box, 10 steps, against the FP64 oracle."""
    shapes = [(16, 16, 16), (32, 32, 32)]
    nus, dt = [0.01, 1 / 400], 2e-3
    ens = sns.NSEnsemble(shapes, nus, dt, torch.complex128, tune=False)
    refs = []
    for b, shape in enumerate(shapes):
        V0 = random_velocity_hat(shape, seed=11 + b)
        w0 = oracle.curl(V0)
        ens.bootstrap(b, [dev(x, torch.complex128, cuda) for x in V0],
                      [dev(x, torch.complex128, cuda) for x in w0])
        ns = oracle.NS(shape, nus[b], dt)
        ns.bootstrap(V0, w0)
        refs.append(ns)
    ens.step(10)
    for b, ns in enumerate(refs):
        for _ in range(10):
            ns.step()
        ref, got = ns.state(), ens.state(b)
        for key in ("V1", "omega1", "cross0"):
            for d in range(3):
                assert rel_l2(host(got[key][d]), ref[key][d]) < 1e-12, (b, key, d)
    ens.close()


def test_ensemble_config_shapes_fp32_tracks_fp64(sns, cuda):
    """Uneven boxes at the ensemble benchmark's sizes and viscosity range:
    the complex64 ensemble against the complex128 ensemble after 20 steps."""
    shapes = [(32, 32, 32)] * 3 + [(64, 64, 64)] * 2 + [(128, 128, 128)]
    nus = list(np.exp(np.linspace(np.log(1 / 800), np.log(1 / 100), len(shapes))))
    dt = 2e-3
    from spectral_upcxx_b200 import ic
    runs = {}
    for dtype in (torch.complex128, torch.complex64):
        ens = sns.NSEnsemble(shapes, nus, dt, dtype, tune=False)
        for b, shape in enumerate(shapes):
            u = ic.solenoidal_spectrum(shape[0], seed=20 + b)
            V0 = []
            for c in u:
                f = np.fft.fftn(c)
                h = shape[0] // 2
                f[h, :, :] = 0
                f[:, h, :] = 0
                f[:, :, h] = 0
                V0.append(f)
            Vd = [dev(x, dtype, cuda) for x in V0]
            ens.bootstrap(b, Vd, sns.curl(Vd))
        ens.step(20)
        runs[dtype] = ens
    for b in range(len(shapes)):
        a, c = runs[torch.complex64].state(b), runs[torch.complex128].state(b)
        for d in range(3):
            assert rel_l2(host(a["V1"][d]), host(c["V1"][d])) < 2e-5, b
    ea, eb = runs[torch.complex64].stats(), runs[torch.complex128].stats()
    for b in range(len(shapes)):
        assert abs(ea[b]["energy"] / eb[b]["energy"] - 1) < 1e-5
    for r in runs.values():
        r.close()
