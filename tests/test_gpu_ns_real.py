"""The real-field stepper (half spectrum, R2C/C2R along x) against the oracle
and the complex stepper.  Tolerances as for the complex stepper: complex128
<= 1e-12 relative L2 per field, complex64 vs complex128 <= 2e-5."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


def _zero_nyq(V):
    out = []
    for c in V:
        c = c.copy()
        n0, n1, n2 = c.shape
        c[n0 // 2, :, :] = 0
        c[:, n1 // 2, :] = 0
        c[:, :, n2 // 2] = 0
        out.append(c)
    return out


def test_real_stepper_taylor_green_matches_oracle(sns, oracle, cuda):
    from spectral_upcxx_b200 import ic
    n, nu, dt = 64, 0.01, 1e-3
    V0 = [oracle.forward(c) for c in ic.taylor_green(n)]
    w0 = oracle.curl(V0)
    st = sns.NSStepper((n, n, n), nu, dt, torch.complex128, real=True)
    st.bootstrap([dev(x, torch.complex128, cuda) for x in V0],
                 [dev(x, torch.complex128, cuda) for x in w0])
    ns = oracle.NS((n, n, n), nu, dt)
    ns.bootstrap(V0, w0)
    for _ in range(10):
        ns.step()
    st.step(10)
    ref, got = ns.state(), st.state()
    for key in ("V1", "omega1", "cross0"):
        for d in range(3):
            if np.linalg.norm(ref[key][d]) == 0:
                assert np.abs(host(got[key][d])).max() < 1e-12
            else:
                assert rel_l2(host(got[key][d]), ref[key][d]) < 1e-12, (key, d)
    st.close()


@pytest.mark.parametrize("shape", [(32, 32, 32), (16, 32, 64)])
def test_real_stepper_equals_complex_stepper(sns, cuda, shape):
    from spectral_upcxx_b200 import ic
    r = ic.rng(5)
    nz, ny, nx = shape
    u = [r.standard_normal(shape) for _ in range(3)]
    V0 = _zero_nyq([np.fft.fftn(c) for c in u])
    Vd = [dev(x, torch.complex128, cuda) for x in V0]
    wd = sns.curl(Vd)
    out = {}
    for real in (False, True):
        st = sns.NSStepper(shape, 1 / 400, 1e-3, torch.complex128, real=real)
        st.bootstrap(Vd, wd)
        st.step(20)
        out[real] = (st.state(), st.stats())
        st.close()
    for key in ("V1", "omega1", "cross0"):
        for d in range(3):
            assert rel_l2(host(out[True][0][key][d]), host(out[False][0][key][d])) < 1e-12
    for key in ("energy", "enstrophy"):
        assert abs(out[True][1][key] / out[False][1][key] - 1) < 1e-12
    assert out[True][1]["max_div"] < 1e-10


def test_real_fp32_tracks_fp64(sns, cuda):
    from spectral_upcxx_b200 import ic
    n = 64
    V0 = ic.solenoidal_spectrum_hat(n, 3, cuda)
    runs = {}
    for dtype in (torch.complex128, torch.complex64):
        Vd = [x.to(dtype) for x in V0]
        st = sns.NSStepper((n, n, n), 1 / 400, 2e-3, dtype, real=dtype == torch.complex64)
        st.bootstrap(Vd, sns.curl(Vd))
        st.step(20)
        runs[dtype] = st
    a, b = runs[torch.complex64].state(), runs[torch.complex128].state()
    for d in range(3):
        assert rel_l2(host(a["V1"][d]), host(b["V1"][d])) < 2e-5
    ea = runs[torch.complex64].stats()["energy"]
    eb = runs[torch.complex128].stats()["energy"]
    assert abs(ea / eb - 1) < 1e-5
    for s in runs.values():
        s.close()


def test_real_fp32_vs_fp64_256_spectrum_seeded(sns, cuda):
    """The benchmark configuration on the real-field stepper: 256^3, nu = 1/400,
    500 steps at dt = 5e-4, complex64 half spectrum against the complex128
    complex stepper."""
    from spectral_upcxx_b200 import ic
    n, nu, dt = 256, 1 / 400, 5e-4
    V0 = ic.solenoidal_spectrum_hat(n, 1, cuda)
    runs = {}
    for dtype, real in ((torch.complex128, False), (torch.complex64, True)):
        Vd = [x.to(dtype) for x in V0]
        st = sns.NSStepper((n, n, n), nu, dt, dtype, real=real)
        st.bootstrap(Vd, sns.curl(Vd))
        del Vd
        st.step(500)
        runs[dtype] = st
    del V0
    worst = 0.0
    a, b = runs[torch.complex64], runs[torch.complex128]
    va, vb = a.velocity(), b.velocity()
    for d in range(3):
        err = (torch.linalg.vector_norm(va[d].to(torch.complex128) - vb[d]) /
               torch.linalg.vector_norm(vb[d])).item()
        worst = max(worst, err if np.isfinite(err) else float("inf"))
    assert worst < 2e-5, worst
    assert abs(a.stats()["energy"] / b.stats()["energy"] - 1) < 1e-5
    for s in runs.values():
        s.close()
    torch.cuda.empty_cache()


def test_real_stepper_rejects_closures(sns, cuda):
    st = sns.NSStepper((32, 32, 32), 0.01, 1e-3, torch.complex64, real=True)
    with pytest.raises(sns.SNSError):
        st.set_closure(sns._native.SNS_CLOSURE_SMAGORINSKY, cs_delta2=1e-3)
    st.close()
