"""The fused NS stepper against the oracle and the reference's golden run.

Tolerances (relative L2 per field): complex128 vs the FP64 oracle <= 1e-12;
complex64 vs the complex128 device path <= 2e-5 per field per step."""
import os

import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


@pytest.mark.parametrize("case,nu", [("tg", 0.01), ("vx", 1e-3)])
def test_stepper_matches_reference_golden(sns, cuda, case, nu):
    """16^3, ns.cpp bootstrap + 5 steps, against the reference's own run."""
    g = np.load(os.path.join(GOLD, "ns16.npz"))
    steps = int(g["steps"])
    V0 = [dev(g[f"{case}_V0_{d}"], torch.complex128, cuda) for d in range(3)]
    w0 = [dev(g[f"{case}_omega0_{d}"], torch.complex128, cuda) for d in range(3)]
    st = sns.NSStepper((16, 16, 16), nu, 1e-3, torch.complex128)
    st.bootstrap(V0, w0)
    st.step(steps)
    s = st.state()
    scale = max(np.abs(g[f"{case}_V1_{d}"]).max() for d in range(3))
    for d in range(3):
        assert rel_l2(host(s["V1"][d]), g[f"{case}_V1_{d}"]) < 1e-12
        assert rel_l2(host(s["cross0"][d]), g[f"{case}_cross0_{d}"]) < 1e-12
    stats = st.stats()
    assert abs(stats["div_avg"] - g[f"{case}_div_avgs"][-1]) < 1e-12 * scale
    st.close()


def test_taylor_green_64_every_field(sns, oracle, cuda):
    """64^3 Taylor-Green, nu = 0.01, dt = 1e-3, 100 steps: V1, omega1 and
    cross0 against the oracle run of the ns.cpp sequence at steps 1, 10, 100."""
    from spectral_upcxx_b200 import ic
    n, nu, dt = 64, 0.01, 1e-3
    V0 = [oracle.forward(c) for c in ic.taylor_green(n)]
    w0 = oracle.curl(V0)
    st = sns.NSStepper((n, n, n), nu, dt, torch.complex128)
    st.bootstrap([dev(x, torch.complex128, cuda) for x in V0],
                 [dev(x, torch.complex128, cuda) for x in w0])
    ns = oracle.NS((n, n, n), nu, dt)
    ns.bootstrap(V0, w0)
    done = 0
    for target in (1, 10, 100):
        for _ in range(target - done):
            ns.step()
        st.step(target - done)
        done = target
        ref = ns.state()
        got = st.state()
        for key in ("V1", "omega1", "cross0"):
            for d in range(3):
                if np.linalg.norm(ref[key][d]) == 0:
                    assert np.abs(host(got[key][d])).max() < 1e-12
                else:
                    assert rel_l2(host(got[key][d]), ref[key][d]) < 1e-12, (target, key, d)
    # kinetic energy decays as exp(-2 nu |k|^2 t) = exp(-6 nu t) at early times
    e = st.stats()["energy"]
    e0 = 0.125  # <|u|^2>/2 of the Taylor-Green field
    assert abs(e / (e0 * np.exp(-6 * nu * 0.101)) - 1) < 2e-3
    st.close()


@pytest.mark.parametrize("n", [32, 64])
def test_fp32_tracks_fp64(sns, oracle, cuda, n):
    """Spectrum-seeded solenoidal field: complex64 vs complex128 device paths."""
    from spectral_upcxx_b200 import ic
    nu, dt = 1 / 400, 2e-3
    u = ic.solenoidal_spectrum(n, seed=3)
    V0 = [oracle.forward(c) for c in u]
    w0 = oracle.curl(V0)
    runs = {}
    for dt_ in (torch.complex128, torch.complex64):
        s = sns.NSStepper((n, n, n), nu, dt, dt_)
        s.bootstrap([dev(x, dt_, cuda) for x in V0], [dev(x, dt_, cuda) for x in w0])
        runs[dt_] = s
    worst = 0.0
    for step in range(20):
        for s in runs.values():
            s.step(1)
        a, b = runs[torch.complex64].state(), runs[torch.complex128].state()
        for key in ("V1", "cross0"):
            for d in range(3):
                worst = max(worst, rel_l2(host(a[key][d]), host(b[key][d])))
    assert worst < 2e-5, worst
    sa, sb = runs[torch.complex64].stats(), runs[torch.complex128].stats()
    assert abs(sa["energy"] / sb["energy"] - 1) < 1e-5
    for s in runs.values():
        s.close()


def test_divergence_free_and_energy_monotone(sns, oracle, cuda):
    from spectral_upcxx_b200 import ic
    n = 64
    u = ic.solenoidal_spectrum(n, seed=5)
    V0 = [oracle.forward(c) for c in u]
    w0 = oracle.curl(V0)
    s = sns.NSStepper((n, n, n), 1 / 400, 2e-3, torch.complex128)
    s.bootstrap([dev(x, torch.complex128, cuda) for x in V0],
                [dev(x, torch.complex128, cuda) for x in w0])
    last = None
    for _ in range(10):
        s.step(1)
        st = s.stats()
        vmax = max(torch.abs(x).max().item() for x in s.state()["V1"])
        assert st["max_div"] < 1e-12 * vmax * n
        if last is not None:
            assert st["energy"] < last
        last = st["energy"]
    s.close()


def test_fp32_vs_fp64_256_spectrum_seeded(sns, oracle, cuda):
    """Benchmark configuration: 256^3, nu = 1/400, 500 steps at dt = 5e-4.
    Per-field relative L2 of the complex64 path against the complex128 path,
    checked every 50 steps; energy-decay error at the end."""
    from spectral_upcxx_b200 import ic
    n, nu, dt = 256, 1 / 400, 5e-4  # the stated dt = 2e-3 diverges at 256^3 in FP64 too
    u = ic.solenoidal_spectrum(n, seed=1)
    V0 = [np.fft.fftn(c) for c in u]
    h = n // 2
    for c in V0:
        c[h, :, :] = 0
        c[:, h, :] = 0
        c[:, :, h] = 0
    runs = {}
    for dt_ in (torch.complex128, torch.complex64):
        Vd = [dev(x, dt_, cuda) for x in V0]
        wd = sns.curl(Vd)
        s = sns.NSStepper((n, n, n), nu, dt, dt_)
        s.bootstrap(Vd, wd)
        del Vd, wd
        runs[dt_] = s
    worst = 0.0
    e = {}
    for block in range(10):
        for s in runs.values():
            s.step(50)
        a, b = runs[torch.complex64].state(), runs[torch.complex128].state()
        for d in range(3):
            va = a["V1"][d].to(torch.complex128)
            err = (torch.linalg.vector_norm(va - b["V1"][d]) /
                   torch.linalg.vector_norm(b["V1"][d])).item()
            worst = max(worst, err if np.isfinite(err) else float("inf"))
        del a, b
        e = {k: s.stats()["energy"] for k, s in runs.items()}
    assert worst < 2e-5, worst
    assert abs(e[torch.complex64] / e[torch.complex128] - 1) < 1e-5
    for s in runs.values():
        s.close()
    torch.cuda.empty_cache()


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_xy_dataflow_and_slabs_match_separate_passes(sns, cuda, dtype, monkeypatch):
    """The persistent dataflow xy launch and the slab-chunked passes give the
    same step as the three separate passes (to rounding)."""
    from spectral_upcxx_b200 import ic
    n = 64
    V0 = [np.fft.fftn(c) for c in ic.solenoidal_spectrum(n, seed=9)]
    out = {}
    for name, env in (("separate", {}), ("dataflow", {"SNS_XY_PASSES": "1"}),
                      ("slabs", {"SNS_XY_CHUNK": "16"})):
        for k in ("SNS_XY_PASSES", "SNS_XY_CHUNK"):
            monkeypatch.delenv(k, raising=False)
        for k, v in env.items():
            monkeypatch.setenv(k, v)
        Vd = [dev(x, dtype, cuda) for x in V0]
        st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, dtype)
        st.bootstrap(Vd, sns.curl(Vd))
        st.step(4)
        assert sns._native.lib().sns_ns_check(st.h) == 0
        out[name] = [host(x) for x in st.state()["V1"]]
        st.close()
    tol = 1e-14 if dtype == torch.complex128 else 1e-6
    for name in ("dataflow", "slabs"):
        for a, b in zip(out[name], out["separate"]):
            assert rel_l2(a, b) < tol, name


@pytest.mark.parametrize("dtype,n", [(torch.complex128, 128), (torch.complex64, 128),
                                     (torch.complex64, 256)])
def test_xy_cluster_pass_matches_separate_passes(sns, cuda, dtype, n, monkeypatch):
    """The xy phase as one thread-block-cluster pass per plane (SNS_XYC=1)
    against the three separate passes (the default): same line FFTs and cross
    product, so the same step to rounding, over 3 steps of a spectrum-seeded
    field."""
    from spectral_upcxx_b200 import ic
    Vh = ic.solenoidal_spectrum_hat(n, 11, cuda)
    out = {}
    for name, env in (("cluster", "1"), ("separate", "0")):
        monkeypatch.setenv("SNS_XYC", env)
        Vd = [x.to(dtype) for x in Vh]
        st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, dtype)
        assert st.launches_per_step() == (3 if name == "cluster" else 5)
        st.bootstrap(Vd, sns.curl(Vd))
        st.step(3)
        assert sns._native.lib().sns_ns_check(st.h) == 0
        out[name] = [x.to(torch.complex128) for x in st.state()["V1"]]
        del Vd
        st.close()
    tol = 1e-14 if dtype == torch.complex128 else 1e-6
    for a, b in zip(out["cluster"], out["separate"]):
        err = (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()
        assert err < tol, err
    torch.cuda.empty_cache()


def test_stats_async_equals_stats(sns, cuda):
    """sns_ns_stats_async queues the diagnostics to pinned host memory without a
    stall; after a synchronise they equal sns_ns_stats bit for bit."""
    from spectral_upcxx_b200 import ic
    n = 64
    V = [x.to(torch.complex128) for x in ic.solenoidal_spectrum_hat(n, 8, cuda)]
    st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex128)
    st.bootstrap(V, sns.curl(V))
    buf = torch.zeros((3, 4), dtype=torch.float64).pin_memory()
    for t in range(3):
        st.step(1)
        st.stats_async(buf[t])
    torch.cuda.synchronize()
    s = st.stats()
    assert buf[2].tolist() == [s["div_avg"], s["energy"], s["enstrophy"], s["max_div"]]
    assert buf[0, 1].item() != buf[2, 1].item()  # one reading per step
    st.close()


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("variant,tag", [("SNS_K1_LINES", "(lines)"),
                                         ("SNS_K1_RELOAD", "(reload)")])
def test_k1_variants_match(sns, cuda, dtype, variant, tag, monkeypatch):
    """The K1 variants -- SNS_K1_LINES=1: z line pass of V and i kz V, the curl
    formed in the y pass; SNS_K1_RELOAD=1: the fused tile forming omega from
    reloads of V -- give the step of the default fused K1 tile."""
    from spectral_upcxx_b200 import ic
    n = 64
    Vh = ic.solenoidal_spectrum_hat(n, 13, cuda)
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv(variant, mode)
        V = [x.to(dtype) for x in Vh]
        st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, dtype)
        assert (tag in st.describe()) == (mode == "1")
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        out[mode] = [x.to(torch.complex128) for x in st.state()["V1"]]
        st.close()
    tol = 1e-13 if dtype == torch.complex128 else 2e-6
    for a, b in zip(out["1"], out["0"]):
        assert (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item() < tol


def _random_fourier(shape, dtype, device, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return [torch.complex(torch.randn(shape, generator=g, dtype=torch.float64),
                          torch.randn(shape, generator=g, dtype=torch.float64)).to(device, dtype)
            for _ in range(3)]


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 64, 128), (512, 16, 32)])
def test_k1_tma_stages_match_reload_bit_for_bit(sns, cuda, dtype, shape, monkeypatch):
    """K1 as a persistent pass over TMA-staged tiles (SNS_K1_TMA=1: one stage,
    2: two) does the arithmetic of the reload tile with V read from shared
    memory instead of HBM, so three steps are identical bit for bit.  The
    non-cubic boxes give tiles of other widths, and nz = 512 loads each
    component of a tile as two boxes of 256 planes."""
    N = sns._native
    V = _random_fourier(shape, dtype, cuda, 5)
    out = {}
    monkeypatch.setenv("SNS_GRAPH", "0")
    for mode in ("reload", "1", "2"):
        monkeypatch.delenv("SNS_K1_TMA", raising=False)
        monkeypatch.delenv("SNS_K1_RELOAD", raising=False)
        if mode == "reload":
            monkeypatch.setenv("SNS_K1_RELOAD", "1")
        else:
            monkeypatch.setenv("SNS_K1_TMA", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        if mode != "reload":
            assert f"(tma{mode})" in st.describe(), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        rc = N.lib().sns_ns_check(st.h)
        assert rc == N.SNS_OK, (mode, rc, N.last_error(), st.describe())
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        st.close()
    for mode in ("1", "2"):
        for a, b in zip(out[mode], out["reload"]):
            assert torch.equal(a, b), mode


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 64, 128), (16, 32, 512)])
def test_x_tma_matches_direct_bit_for_bit(sns, cuda, dtype, shape, monkeypatch):
    """The x cross pass over TMA-staged rows (SNS_X_TMA=1; by default the rows
    load straight from HBM) does the same arithmetic on the same values:
    three steps are identical bit for bit, for row lengths 64, 128 and 512."""
    N = sns._native
    V = _random_fourier(shape, dtype, cuda, 7)
    out = {}
    monkeypatch.setenv("SNS_GRAPH", "0")
    for mode in ("0", "1"):
        monkeypatch.setenv("SNS_X_TMA", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        assert ("(tma) pf" in st.describe()) == (mode == "1"), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        rc = N.lib().sns_ns_check(st.h)
        assert rc == N.SNS_OK, (mode, rc, N.last_error())
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        st.close()
    for a, b in zip(out["1"], out["0"]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("graph", ["0", "1"])
@pytest.mark.parametrize("real", [False, True])
@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 64, 128), (512, 16, 32), (8, 16, 32)])
def test_carried_k1_matches_separate_bit_for_bit(sns, cuda, dtype, shape, real, graph,
                                                 monkeypatch):
    """The update pass with the next step's K1 carried in it (SNS_CARRY=1:
    after the update the tile z-inverse-transforms the new V and its curl
    into the work fields, so the next step skips K1; 2: the new V read back
    from HBM's caches instead of shared memory) does K1's arithmetic on
    the same values: five steps, a new state set, three more steps -- the
    states and diagnostics are identical bit for bit to the plan without
    carrying (the FP64 diagnostics to 1e-12: their per-tile partials may be
    summed in another order), with and without the CUDA graph (whose captured
    step is the one without K1; after the new state K1 runs once before the
    replay), on complex and half-spectrum (real-field) steppers."""
    N = sns._native
    V = _random_fourier(shape, dtype, cuda, 13)
    V2 = _random_fourier(shape, dtype, cuda, 14)
    monkeypatch.setenv("SNS_GRAPH", graph)
    out, stats = {}, {}
    for mode in ("0", "1", "2"):
        monkeypatch.setenv("SNS_CARRY", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype, real=real)
        assert ("(+K1" in st.describe()) == (mode != "0"), st.describe()
        assert ("(+K1r)" in st.describe()) == (mode == "2"), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(5)
        first = st.stats()
        mid = [x.clone() for x in st.state()["V1"]]
        st.set_state(V2, V)
        st.step(3)
        rc = N.lib().sns_ns_check(st.h)
        assert rc == N.SNS_OK, (mode, rc, N.last_error())
        out[mode] = mid + [x.clone() for x in st.state()["V1"]] + \
            [x.clone() for x in st.state()["cross0"]]
        stats[mode] = (first, st.stats())
        st.close()
    for mode in ("1", "2"):
        for a, b in zip(out[mode], out["0"]):
            assert torch.equal(a, b), mode
        # the carrying plan may tile the update pass at another width, which
        # sums the per-tile FP64 diagnostics in another order
        for s1, s0 in zip(stats[mode], stats["0"]):
            for k in s0:
                assert abs(s1[k] - s0[k]) <= 1e-12 * abs(s0[k]), (mode, k, s1[k], s0[k])


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_update_self_prefetch_bit_for_bit(sns, cuda, dtype, monkeypatch):
    """Asking L2 for a tile's V and C0 while the update pass's cross-product
    loads are in flight (SNS_Z_PFSELF=1) is a hint only: three steps are
    identical bit for bit."""
    shape = (64, 32, 128)
    V = _random_fourier(shape, dtype, cuda, 16)
    out = {}
    for mode in ("0", "1"):
        monkeypatch.setenv("SNS_Z_PFSELF", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        assert ("(pfs)" in st.describe()) == (mode == "1"), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        st.close()
    for a, b in zip(out["1"], out["0"]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("real", [False, True])
@pytest.mark.parametrize("stages", ["1", "2"])
@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 128, 64), (16, 512, 32), (8, 32, 64)])
def test_y_tma_matches_direct_bit_for_bit(sns, cuda, dtype, shape, stages, real, monkeypatch):
    """The y line passes (K2, K4) over TMA-staged tiles (SNS_Y_TMA = 1 or 2
    stages; by default each CTA loads its tile straight from HBM) do the same
    arithmetic on the same values: three steps are identical bit for bit, for
    line lengths 32 to 512 (ny = 512: boxes of 256 positions), on complex and
    half-spectrum (real-field) steppers."""
    N = sns._native
    V = _random_fourier(shape, dtype, cuda, 17)
    out = {}
    monkeypatch.setenv("SNS_GRAPH", "0")
    for mode in ("0", stages):
        monkeypatch.setenv("SNS_Y_TMA", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype, real=real)
        assert ("(tma%s) zW" % stages in st.describe()) == (mode != "0"), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        rc = N.lib().sns_ns_check(st.h)
        assert rc == N.SNS_OK, (mode, rc, N.last_error())
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        st.close()
    for a, b in zip(out[stages], out["0"]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(256, 16, 64), (64, 64, 64), (32, 16, 128)])
def test_update_wide_tile_halves_bit_for_bit(sns, cuda, dtype, shape, monkeypatch):
    """An update-pass tile wider than the thread limit (SNS_Z_W=32 at nz = 256
    in complex64, 16 in complex128) is z-transformed in two halves of
    adjacent lines by half the threads: the same values as narrower tiles,
    three steps identical bit for bit (diagnostics to 1e-12: the per-tile
    partials are summed in another order)."""
    N = sns._native
    V = _random_fourier(shape, dtype, cuda, 18)
    out, stats = {}, {}
    monkeypatch.setenv("SNS_GRAPH", "0")
    wide = "32" if dtype == torch.complex64 else "16"
    for mode in ("4", wide):
        monkeypatch.setenv("SNS_Z_W", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        rc = N.lib().sns_ns_check(st.h)
        assert rc == N.SNS_OK, (mode, rc, N.last_error())
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        stats[mode] = st.stats()
        desc = st.describe()
        st.close()
    assert "zW=%s" % min(int(wide), shape[2]) in desc, desc
    for a, b in zip(out[wide], out["4"]):
        assert torch.equal(a, b)
    for k in stats["4"]:
        assert abs(stats[wide][k] - stats["4"][k]) <= 1e-12 * abs(stats["4"][k])


@pytest.mark.parametrize("waves", ["1", "2"])
@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
def test_next_wave_prefetch_bit_for_bit(sns, cuda, dtype, waves, monkeypatch):
    """Asking L2 for the tiles one or two waves of resident CTAs ahead
    (SNS_PF, issued once each tile's own loads are in flight; the direct-load
    K1, y passes, x pass and update pass) is a hint only: three steps are
    identical bit for bit to the run without it."""
    shape = (64, 64, 128)
    V = _random_fourier(shape, dtype, cuda, 19)
    out = {}
    monkeypatch.setenv("SNS_K1_TMA", "0")
    monkeypatch.setenv("SNS_K1_RELOAD", "1")
    for mode in ("0", waves):
        monkeypatch.setenv("SNS_PF", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        assert ("pf=%s" % mode) in st.describe(), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        st.close()
    for a, b in zip(out[waves], out["0"]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (16, 32, 256), (32, 16, 128)])
def test_x_occ_matches_direct_bit_for_bit(sns, cuda, dtype, shape, monkeypatch):
    """The x cross pass compiled for five CTAs of at most 192 threads per SM
    (SNS_X_OCC=1; used where its tile has at most 192 threads) does the same
    arithmetic: three steps are identical bit for bit."""
    V = _random_fourier(shape, dtype, cuda, 20)
    out = {}
    monkeypatch.setenv("SNS_GRAPH", "0")
    for mode in ("0", "1"):
        monkeypatch.setenv("SNS_X_OCC", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        assert ("(occ)" in st.describe()) == (mode == "1"), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        st.close()
    for a, b in zip(out["1"], out["0"]):
        assert torch.equal(a, b)


def test_carried_k1_pass_times(sns, cuda, monkeypatch):
    """Per-pass timing of a carrying plan: K1 runs in the first step only
    (its later pass times are empty), the update pass carries it."""
    monkeypatch.setenv("SNS_CARRY", "2")
    shape = (128, 128, 128)
    V = _random_fourier(shape, torch.complex64, cuda, 15)
    st = sns.NSStepper(shape, 1 / 400, 5e-4, torch.complex64)
    st.bootstrap(V, sns.curl(V))
    st.profile(True)
    st.step(1)
    (k1_first, n1), *_ = st.pass_times()
    st.profile(True)
    st.step(4)
    (k1_later, n4), *_ = st.pass_times()
    st.close()
    assert (n1, n4) == (1, 4)
    assert k1_first > 0
    assert k1_later / 4 < 0.25 * k1_first, (k1_first, k1_later)


@pytest.mark.parametrize("dtype", [torch.complex128, torch.complex64])
@pytest.mark.parametrize("shape", [(64, 64, 64), (32, 64, 128), (512, 16, 32)])
def test_z_tma_update_matches_direct_bit_for_bit(sns, cuda, dtype, shape, monkeypatch):
    """The update pass over TMA-staged z lines of the cross product
    (SNS_Z_TMA=1; by default they load straight from HBM) does the same
    arithmetic on the same values: three steps and their diagnostics are
    identical bit for bit (nz = 512: two boxes of 256 planes per line)."""
    N = sns._native
    V = _random_fourier(shape, dtype, cuda, 11)
    out, stats = {}, {}
    monkeypatch.setenv("SNS_GRAPH", "0")
    for mode in ("0", "1"):
        monkeypatch.setenv("SNS_Z_TMA", mode)
        st = sns.NSStepper(shape, 1 / 400, 5e-4, dtype)
        assert ("(tma) xG" in st.describe()) == (mode == "1"), st.describe()
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        rc = N.lib().sns_ns_check(st.h)
        assert rc == N.SNS_OK, (mode, rc, N.last_error())
        out[mode] = [x.clone() for x in st.state()["V1"]] + [x.clone() for x in st.state()["cross0"]]
        stats[mode] = st.stats()
        st.close()
    for a, b in zip(out["1"], out["0"]):
        assert torch.equal(a, b)
    assert stats["1"] == stats["0"]
