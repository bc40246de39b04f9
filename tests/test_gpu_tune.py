"""The autotuner (the counterpart of the reference's FFTW_MEASURE planning,
src/FFT1D.cpp:18-22): every radix order of the line FFT against the oracle,
tuned 3D transforms and tuned steppers against the default plans (to
rounding: complex128 relative L2 <= 1e-12, complex64 <= 2e-6 per transform
and per field after 5 steps), and the tuner's refusal once a stepper holds
state."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu

TOL = {torch.complex128: 1e-12, torch.complex64: 2e-6}
DT = [torch.complex128, torch.complex64]


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


@pytest.mark.parametrize("order", [0, 1, 2])
@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("shape", [(64, 128, 64), (4, 512, 256), (2, 1024, 8)])
def test_radix_orders_match_oracle(sns, oracle, cuda, monkeypatch, order, dtype, shape):
    """Radix-16 first, remainder first, radix-8: the same transform."""
    from spectral_upcxx_b200 import ic
    monkeypatch.setenv("SNS_RADIX_ORDER", str(order))
    f = ic.uniform_complex(shape, 21)
    for direction in (-1, +1):
        t = dev(f, dtype, cuda)
        sns.fft3d(t, direction)
        assert rel_l2(host(t), oracle.transform(f, direction)) < TOL[dtype]


@pytest.mark.parametrize("dtype", DT)
@pytest.mark.parametrize("shape", [(128, 128, 128), (32, 64, 256)])
def test_tuned_fft3d_equals_default(sns, oracle, cuda, dtype, shape):
    from spectral_upcxx_b200 import ic
    f = ic.uniform_complex(shape, 22)
    before = dev(f, dtype, cuda)
    sns.forward(before)
    sns.fft3d_tune(shape, dtype, nfields=1, device=cuda)
    after = dev(f, dtype, cuda)
    sns.forward(after)
    assert rel_l2(host(after), host(before)) < TOL[dtype]
    assert rel_l2(host(after), oracle.forward(f)) < TOL[dtype]
    t = after.clone()
    sns.inverse(t)
    assert rel_l2(host(t), oracle.inverse(oracle.forward(f))) < TOL[dtype]


@pytest.mark.parametrize("dtype,n", [(torch.complex128, 64), (torch.complex64, 128)])
def test_tuned_stepper_equals_default(sns, cuda, dtype, n):
    from spectral_upcxx_b200 import ic
    Vh = ic.solenoidal_spectrum_hat(n, 12, cuda)
    out = {}
    for tune in (False, True):
        V = [x.to(dtype) for x in Vh]
        st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, dtype, tune=tune)
        assert ("tuned" in st.describe()) == tune
        st.bootstrap(V, sns.curl(V))
        st.step(5)
        assert sns._native.lib().sns_ns_check(st.h) == 0
        out[tune] = ([x.to(torch.complex128) for x in st.state()["V1"]], st.stats())
        st.close()
    tol = 1e-12 if dtype == torch.complex128 else 2e-6
    for a, b in zip(out[True][0], out[False][0]):
        err = (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item()
        assert err < tol, err
    assert abs(out[True][1]["energy"] / out[False][1]["energy"] - 1) < 10 * tol


def test_tune_refused_after_state(sns, cuda):
    from spectral_upcxx_b200 import ic
    n = 32
    V = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(n, 3, cuda)]
    st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
    st.bootstrap(V, sns.curl(V))
    st.step(1)
    rc = sns._native.lib().sns_ns_tune(st.h)
    assert rc == sns._native.SNS_ERR_ARG
    st.close()
