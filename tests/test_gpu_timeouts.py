"""Bounded waits that run out, in the safe form: no GPU fault, no hang.

* The persistent dataflow xy pass (SNS_XY_PASSES=1) with a poll budget of one
  (SNS_XY_SPIN=1) and a one-plane lag between producers and consumers: some
  consumer finds its plane unfinished and gives up at once; the launch still
  ends (every access stays in bounds), sns_ns_check reports SNS_ERR_TIMEOUT
  and clears the record, and a stepper run afterwards with the normal budget
  succeeds and matches the separate passes.
* The TMA-staged z pass of the step (SNS_K1_TMA) with a stall test
  (SNS_TMA_STALL_TEST=<cycles>): the first tile waits on a barrier nothing
  arrives at; sns_ns_check reports SNS_ERR_TIMEOUT, and the next run is normal.
* The tcgen05 MLP inference with a stall test (SNS_TC_STALL_TEST=<cycles>):
  each CTA also waits on a barrier nothing arrives at; the wait runs out,
  sns_mlp_status reports SNS_ERR_TIMEOUT, the MMA already issued is still
  waited for before tensor memory is freed, and the next inference is normal.
"""
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_dataflow_wait_runs_out_and_recovers(sns, cuda, monkeypatch):
    from spectral_upcxx_b200 import ic
    N = sns._native
    n = 64
    Vh = ic.solenoidal_spectrum_hat(n, 4, cuda)
    V = [x.to(torch.complex64) for x in Vh]
    monkeypatch.setenv("SNS_XY_PASSES", "1")
    monkeypatch.setenv("SNS_GRAPH", "0")
    monkeypatch.setenv("SNS_XY_LAG", "1")
    monkeypatch.setenv("SNS_XY_SPIN", "1")
    st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
    assert "xy=dataflow" in st.describe()
    st.bootstrap(V, sns.curl(V))
    codes = []
    for _ in range(10):
        st.step(1)
        codes.append(N.lib().sns_ns_check(st.h))
        if codes[-1] == N.SNS_ERR_TIMEOUT:
            break
    assert N.SNS_ERR_TIMEOUT in codes, codes
    assert "gave up" in N.last_error()
    assert N.lib().sns_ns_check(st.h) == N.SNS_OK  # the record was cleared
    st.close()
    # the normal budget: a fresh run matches the separate passes
    monkeypatch.delenv("SNS_XY_SPIN")
    monkeypatch.delenv("SNS_XY_LAG")
    out = {}
    for mode in ("1", "0"):
        monkeypatch.setenv("SNS_XY_PASSES", mode)
        st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
        st.bootstrap(V, sns.curl(V))
        st.step(3)
        assert N.lib().sns_ns_check(st.h) == N.SNS_OK
        out[mode] = [x.clone() for x in st.state()["V1"]]
        st.close()
    for a, b in zip(out["1"], out["0"]):
        assert (torch.linalg.vector_norm(a - b) / torch.linalg.vector_norm(b)).item() < 1e-6


def test_tensor_core_wait_runs_out_and_recovers(sns, cuda, monkeypatch):
    from spectral_upcxx_b200 import closure as CL
    N = sns._native
    m = CL.MLPModel.init(0, s_in=1.0, s_out=1.0, device=cuda)
    X = torch.randn((1 << 16, 16), device=cuda)
    X[:, 9:] = 0
    X = X.to(torch.bfloat16)
    want = m.infer(X)
    assert N.lib().sns_mlp_status() == N.SNS_OK
    monkeypatch.setenv("SNS_TC_STALL_TEST", "20000")
    m.infer(X)
    assert N.lib().sns_mlp_status() == N.SNS_ERR_TIMEOUT
    assert "gave up" in N.last_error()
    assert N.lib().sns_mlp_status() == N.SNS_OK  # the record was cleared
    monkeypatch.delenv("SNS_TC_STALL_TEST")
    got = m.infer(X)
    assert N.lib().sns_mlp_status() == N.SNS_OK
    assert torch.equal(got, want)


def test_tma_stage_wait_runs_out_and_recovers(sns, cuda, monkeypatch):
    """The TMA-staged K1 with a stall test (SNS_TMA_STALL_TEST=<cycles>): the
    first tile's wait also waits on a barrier that nothing arrives at, runs
    out, and the CTA records the timeout, waits for its copies in flight and
    ends; sns_ns_check reports SNS_ERR_TIMEOUT and clears the record, and a
    stepper run afterwards without the stall matches the reload tile."""
    from spectral_upcxx_b200 import ic
    N = sns._native
    n = 64
    V = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(n, 4, cuda)]
    monkeypatch.setenv("SNS_GRAPH", "0")
    monkeypatch.setenv("SNS_K1_TMA", "2")
    monkeypatch.setenv("SNS_TMA_STALL_TEST", "20000")
    st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
    assert "(tma2)" in st.describe()
    st.bootstrap(V, sns.curl(V))
    st.step(1)
    assert N.lib().sns_ns_check(st.h) == N.SNS_ERR_TIMEOUT
    assert "gave up" in N.last_error()
    assert N.lib().sns_ns_check(st.h) == N.SNS_OK  # the record was cleared
    st.close()
    monkeypatch.delenv("SNS_TMA_STALL_TEST")
    out = {}
    for env in ("SNS_K1_TMA", "SNS_K1_RELOAD"):
        monkeypatch.delenv("SNS_K1_TMA", raising=False)
        monkeypatch.setenv(env, "2" if env == "SNS_K1_TMA" else "1")
        st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
        st.bootstrap(V, sns.curl(V))
        st.step(2)
        assert N.lib().sns_ns_check(st.h) == N.SNS_OK
        out[env] = [x.clone() for x in st.state()["V1"]]
        st.close()
    for a, b in zip(out["SNS_K1_TMA"], out["SNS_K1_RELOAD"]):
        assert torch.equal(a, b)


@pytest.mark.parametrize("env", ["SNS_X_TMA", "SNS_Z_TMA", "SNS_Y_TMA"])
def test_tma_x_and_update_waits_run_out_and_recover(sns, cuda, monkeypatch, env):
    """The same stall test on the TMA-staged x pass, update pass and y passes
    (the z pass on its direct-load form, so the timeout is theirs)."""
    from spectral_upcxx_b200 import ic
    N = sns._native
    n = 64
    V = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(n, 4, cuda)]
    monkeypatch.setenv("SNS_GRAPH", "0")
    monkeypatch.setenv("SNS_K1_TMA", "0")
    monkeypatch.setenv(env, "1")
    monkeypatch.setenv("SNS_TMA_STALL_TEST", "20000")
    st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
    if env == "SNS_Y_TMA":
        assert "(tma1) zW" in st.describe() and "k1=" in st.describe(), st.describe()
    else:
        assert "(tma)" in st.describe() and "(tma1)" not in st.describe()
    st.bootstrap(V, sns.curl(V))
    st.step(1)
    assert N.lib().sns_ns_check(st.h) == N.SNS_ERR_TIMEOUT
    assert "gave up" in N.last_error()
    assert N.lib().sns_ns_check(st.h) == N.SNS_OK
    st.close()
    monkeypatch.delenv("SNS_TMA_STALL_TEST")
    st = sns.NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64)
    st.bootstrap(V, sns.curl(V))
    st.step(2)
    assert N.lib().sns_ns_check(st.h) == N.SNS_OK
    st.close()


def test_fft_tma_wait_runs_out_and_recovers(sns, cuda, monkeypatch):
    """The 3D transform's TMA-staged passes (SNS_FFT_TMA=1) with the stall
    test: the first tile's wait runs out, the CTA records it and ends;
    sns_fft3d_check reports SNS_ERR_TIMEOUT and clears the record, and a
    transform afterwards without the stall is correct and checks clean."""
    from spectral_upcxx_b200 import ic
    N = sns._native
    shape = (64, 64, 64)
    f = ic.uniform_complex(shape, 41)
    monkeypatch.setenv("SNS_FFT_TMA", "1")
    monkeypatch.setenv("SNS_TMA_STALL_TEST", "20000")
    t = torch.from_numpy(f).to(cuda, torch.complex64)
    sns.forward(t)
    assert N.lib().sns_fft3d_check(None) == N.SNS_ERR_TIMEOUT
    assert "gave up" in N.last_error()
    assert N.lib().sns_fft3d_check(None) == N.SNS_OK  # the record was cleared
    monkeypatch.delenv("SNS_TMA_STALL_TEST")
    t = torch.from_numpy(f).to(cuda, torch.complex64)
    sns.forward(t)
    assert N.lib().sns_fft3d_check(None) == N.SNS_OK
    monkeypatch.setenv("SNS_FFT_TMA", "0")
    r = torch.from_numpy(f).to(cuda, torch.complex64)
    sns.forward(r)
    assert torch.equal(t, r)
