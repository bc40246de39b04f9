"""The learned-closure path on the GPU against the closure oracle
(oracle/closure.py, numpy FP64).

Tolerances: filter, spectrum and the complex128 Smagorinsky step <= 1e-12
relative (FP64 on both sides), SGS targets <= 1e-6 (a ratio with S:S); MLP outputs and gradients
<= 2e-3 relative L2 (BF16 operands, FP32 accumulation on the GPU against
FP64 accumulation in the oracle, identical BF16 rounding points); the
complex128 MLP closure step <= 1e-5 (nu_t carries the MLP's FP32 rounding)."""
import numpy as np
import pytest
import torch

from conftest import rel_l2

pytestmark = pytest.mark.gpu


def dev(a, dtype, device):
    return torch.from_numpy(np.ascontiguousarray(a)).to(device=device, dtype=dtype)


def host(t):
    return t.detach().cpu().to(torch.complex128).numpy()


@pytest.fixture(scope="module")
def CO():
    from oracle import closure
    return closure


@pytest.fixture(scope="module")
def CL():
    from spectral_upcxx_b200 import closure
    return closure


def _field(n, seed):
    from spectral_upcxx_b200 import ic
    return [np.fft.fftn(c) for c in ic.solenoidal_spectrum(n, seed=seed)]


def _random_net(CO, seed):
    r = np.random.default_rng(seed)
    net = CO.MLP.init(seed)
    net.b1 = np.asarray(r.standard_normal(64) * 0.1, np.float32).astype(np.float64)
    net.b2 = np.asarray(r.standard_normal(64) * 0.1, np.float32).astype(np.float64)
    net.b3 = float(np.float32(0.3))
    return net


def _gpu_model(CL, net, cuda, s_in=1.0, s_out=1.0):
    return CL.MLPModel(net.W1, net.b1, net.W2, net.b2, net.w3, net.b3, s_in, s_out, device=cuda)


def _features(CO, M, seed):
    r = np.random.default_rng(seed)
    X = np.zeros((M, CO.KPAD))
    X[:, :CO.NIN] = r.standard_normal((M, CO.NIN))
    return CO.bf16(X)


def test_mlp_inference_matches_oracle(CO, CL, cuda):
    net = _random_net(CO, 1)
    net.s_out = 0.5
    model = _gpu_model(CL, net, cuda, s_out=0.5)
    X = _features(CO, 1000, 2)
    got = model.infer(dev(X, torch.bfloat16, cuda)).cpu().double().numpy()
    ref = net.nut(X)
    assert rel_l2(got, ref) < 2e-3


def test_mlp_inference_tensor_memory_path_large(CO, CL, sns, cuda):
    """sns_mlp_infer on the tcgen05 path at 300,001 points (a ragged last
    tile, more tiles than CTAs) against the oracle; no MMA wait ran out."""
    net = _random_net(CO, 7)
    net.s_out = 0.25
    model = _gpu_model(CL, net, cuda, s_out=0.25)
    X = _features(CO, 300001, 8)
    got = model.infer(dev(X, torch.bfloat16, cuda)).cpu().double().numpy()
    ref = net.nut(X)
    assert rel_l2(got, ref) < 2e-3
    assert np.abs(got - ref).max() < 1e-2 * np.abs(ref).max()
    assert sns._native.lib().sns_mlp_status() == 0


def test_mlp_gradient_matches_oracle(CO, CL, cuda):
    net = _random_net(CO, 3)
    model = _gpu_model(CL, net, cuda)
    B = 1000  # not a multiple of the 128-sample CTA
    X = _features(CO, 4096, 4)
    r = np.random.default_rng(5)
    t = np.abs(r.standard_normal(4096)).astype(np.float32)
    idx = r.integers(0, 4096, B).astype(np.int32)
    wt = (0.5 + r.random(4096)).astype(np.float32)
    g = model.gradient(dev(X, torch.bfloat16, cuda), dev(t, torch.float32, cuda),
                       idx=dev(idx, torch.int32, cuda),
                       weight=dev(wt, torch.float32, cuda)).cpu().double().numpy()
    loss, ref = net.loss_and_grads(X[idx], t[idx].astype(np.float64), w=wt[idx])
    assert abs(g[-1] / loss - 1) < 1e-4
    o = {"W1": (0, 1024), "b1": (1024, 1088), "W2": (1088, 5184), "b2": (5184, 5248),
         "w3": (5248, 5312), "b3": (5312, 5313)}
    for name, (a, b) in o.items():
        assert rel_l2(g[a:b], np.ravel(ref[name])) < 2e-3, name


def test_mlp_gradient_many_tiles_per_cta(CO, CL, sns, cuda):
    """A batch of 100,000 samples: every CTA of the tcgen05 training kernel
    accumulates dW1, dW2 in tensor memory over two or three tiles; the last
    tile is ragged.  Against the oracle; no MMA wait ran out."""
    net = _random_net(CO, 9)
    model = _gpu_model(CL, net, cuda)
    M, B = 120000, 100000
    X = _features(CO, M, 10)
    r = np.random.default_rng(11)
    t = np.abs(r.standard_normal(M)).astype(np.float32)
    idx = r.integers(0, M, B).astype(np.int32)
    wt = (0.5 + r.random(M)).astype(np.float32)
    g = model.gradient(dev(X, torch.bfloat16, cuda), dev(t, torch.float32, cuda),
                       idx=dev(idx, torch.int32, cuda),
                       weight=dev(wt, torch.float32, cuda)).cpu().double().numpy()
    loss, ref = net.loss_and_grads(X[idx], t[idx].astype(np.float64), w=wt[idx])
    assert abs(g[-1] / loss - 1) < 1e-4
    o = {"W1": (0, 1024), "b1": (1024, 1088), "W2": (1088, 5184), "b2": (5184, 5248),
         "w3": (5248, 5312), "b3": (5312, 5313)}
    for name, (a, b) in o.items():
        assert rel_l2(g[a:b], np.ravel(ref[name])) < 2e-3, name
    # the padding columns of W1 carry no gradient
    assert np.all(g[:1024].reshape(64, 16)[:, CO.NIN:] == 0)
    assert sns._native.lib().sns_mlp_status() == 0


def test_adam_step_and_training_reduce_the_loss(CO, CL, cuda):
    """One Adam step equals the textbook update of the masters; a short run
    fits a smooth synthetic target."""
    net = _random_net(CO, 6)
    model = _gpu_model(CL, net, cuda)
    X = _features(CO, 8192, 7)
    t = np.log1p(np.exp(0.5 * X[:, 0] - 0.3 * X[:, 4] + 0.2)).astype(np.float32)
    Xd, td = dev(X, torch.bfloat16, cuda), dev(t, torch.float32, cuda)
    w0 = model.master.cpu().double().numpy()
    g = model.gradient(Xd, td).cpu().double().numpy()[:-1]
    model.adam(1e-3)
    m = 0.1 * g
    v = 0.001 * g * g
    want = w0 - 1e-3 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    want[:1024].reshape(64, 16)[:, 9:] = 0
    assert np.allclose(model.master.cpu().double().numpy(), want, rtol=1e-5, atol=1e-7)
    losses = CL.train(model, Xd, td, steps=300, batch=2048, lr=3e-3)
    assert losses[-1][1] < 0.1 * losses[0][1]


def test_truncate_pad_spectrum_match_oracle(CO, CL, cuda):
    n, nc, kc = 32, 16, 5.5
    V = _field(n, 8)
    Vd = [dev(v, torch.complex128, cuda) for v in V]
    Vc = CL.truncate(Vd, nc, kc)
    for a, b in zip(Vc, V):
        assert rel_l2(host(a), CO.truncate(b, nc, kc)) < 1e-14
    P = CL.pad(Vc, n)
    for a, b in zip(P, Vc):
        assert rel_l2(host(a), CO.pad(host(b), n)) < 1e-14
    E = CL.spectrum(Vd)
    Eo = CO.spectrum(V)
    assert np.allclose(E[:len(Eo)], Eo, rtol=1e-12, atol=1e-300)
    # complex64 fields give the same spectrum to FP32 rounding
    E32 = CL.spectrum([v.to(torch.complex64) for v in Vd])
    assert np.allclose(E32[:len(Eo)], Eo, rtol=1e-5, atol=1e-12)


def test_sgs_sample_matches_oracle(CO, CL, cuda):
    n, nc, kc = 32, 16, 5
    V = _field(n, 9)
    X, nut, w, Vc = CL.sgs_sample([dev(v, torch.complex128, cuda) for v in V], nc, kc, 0.7,
                                  Vc=[torch.empty((nc,) * 3, dtype=torch.complex128, device=cuda)
                                      for _ in range(3)])
    Xo, nuto, wo, Vco = CO.sgs_sample(V, nc, kc, 0.7)
    assert rel_l2(w.cpu().double().numpy(), wo) < 1e-6
    for a, b in zip(Vc, Vco):
        assert rel_l2(host(a), b) < 1e-14
    # nu_t divides by S:S, which amplifies the FFTs' FP64 rounding where the
    # filtered strain is small
    assert rel_l2(nut.cpu().double().numpy(), nuto) < 1e-6
    Xg = X.float().cpu().double().numpy()
    # bf16 of the same FP64 features: equal except at rounding ties of the
    # last FP64 bits, which do not occur here
    assert np.array_equal(Xg, CO.bf16(Xo))


def _les_pair(CO, S, cuda, n, nu, dt, seed):
    V0 = _field(n, seed)
    h = n // 2
    for c in V0:
        c[h, :, :] = 0
        c[:, h, :] = 0
        c[:, :, h] = 0
    Vd = [dev(v, torch.complex128, cuda) for v in V0]
    st = S.NSStepper((n, n, n), nu, dt, torch.complex128)
    st.bootstrap(Vd, S.curl(Vd))
    s0 = st.state()
    return st, [host(x) for x in s0["V1"]], [host(x) for x in s0["cross0"]]


@pytest.mark.parametrize("kc,band", [(0.0, (0, 0)), (10.0, (0, 0)), (10.0, (4, 8.5)),
                                     (0.0, (6, 0))])
def test_smagorinsky_step_matches_oracle(CO, CL, sns, cuda, kc, band):
    """complex128 closure step (with and without the spectral cutoff, and with
    the eddy force on a ramp or a sharp band of small scales)."""
    n, nu, dt = 32, 1 / 400, 1e-3
    csd2 = CL.smagorinsky_cs_delta2(0.17, 10.0)
    st, V1, c0 = _les_pair(CO, sns, cuda, n, nu, dt, 10)
    st.set_closure(sns._native.SNS_CLOSURE_SMAGORINSKY, cs_delta2=csd2, kc=kc)
    st.set_sgs_band(*band)
    assert st.launches_per_step() == 5
    les = CO.LES(nu, dt, "smagorinsky", {"cs": 0.17, "delta": np.pi / 10.0},
                 kc=kc if kc > 0 else None, band=band)
    les.set_state(V1, c0)
    st.step(3)
    les.step(3)
    got = st.state()
    for d in range(3):
        assert rel_l2(host(got["V1"][d]), les.V1[d]) < 1e-12
        assert rel_l2(host(got["cross0"][d]), les.c0[d]) < 1e-12
    st.close()


def test_zero_viscosity_closure_is_the_plain_step(sns, cuda):
    """Smagorinsky with Cs = 0 through the closure passes = the fused plain step."""
    n = 32
    V0 = [dev(v, torch.complex128, cuda) for v in _field(n, 11)]
    a = sns.NSStepper((n, n, n), 0.01, 1e-3, torch.complex128)
    b = sns.NSStepper((n, n, n), 0.01, 1e-3, torch.complex128)
    for s in (a, b):
        s.bootstrap(V0, sns.curl(V0))
    b.set_closure(sns._native.SNS_CLOSURE_SMAGORINSKY, cs_delta2=0.0)
    a.step(4)
    b.step(4)
    for x, y in zip(a.velocity(), b.velocity()):
        assert rel_l2(host(y), host(x)) < 1e-13
    a.close()
    b.close()


def test_mlp_closure_step_matches_oracle(CO, CL, sns, cuda):
    n, nu, dt = 16, 1 / 400, 1e-3
    net = _random_net(CO, 12)
    net.s_in, net.s_out = 0.3, 1e-3
    model = _gpu_model(CL, net, cuda, s_in=0.3, s_out=1e-3)
    st, V1, c0 = _les_pair(CO, sns, cuda, n, nu, dt, 13)
    st.set_closure(sns._native.SNS_CLOSURE_MLP, mlp=model.packed)
    les = CO.LES(nu, dt, "mlp", {"mlp": net})
    les.set_state(V1, c0)
    st.step(2)
    les.step(2)
    got = st.state()
    for d in range(3):
        assert rel_l2(host(got["V1"][d]), les.V1[d]) < 1e-5
    st.close()


def test_closure_fp32_runs_and_dissipates(CL, sns, cuda):
    """complex64 closure steps stay finite and drain more energy than the plain step."""
    n, nu, dt = 64, 1 / 400, 2e-3
    from spectral_upcxx_b200 import ic
    V0 = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(n, 14, cuda)]
    e = {}
    for name in ("plain", "smag"):
        st = sns.NSStepper((n, n, n), nu, dt, torch.complex64)
        if name == "smag":
            st.set_closure(sns._native.SNS_CLOSURE_SMAGORINSKY,
                           cs_delta2=CL.smagorinsky_cs_delta2(0.17, n / 3))
        st.bootstrap(V0, sns.curl(V0))
        st.step(50)
        e[name] = st.stats()["energy"]
        st.close()
    assert np.isfinite(e["smag"]) and e["smag"] < e["plain"]


def test_trained_mlp_beats_the_unclosed_coarse_run(CL, sns, cuda):
    """Scaled-down closure experiment: 128^3 DNS filtered at kc = 10 onto
    32^3, a short training run, then 32^3 runs (modes |k| <= kc) from a
    held-out seed judged by their energy spectrum against the filtered DNS
    (shells 1..9)."""
    nf, nc, kc, nu, dt = 128, 32, 10, 1 / 400, 1e-3
    calib = {}
    X, nut, w, s_in, snaps = CL.dns_dataset(sns, nf, nc, kc, seeds=[1, 2], nu=nu, dt=dt,
                                            steps=400, every=10, device=cuda, calib=calib)
    assert snaps == 80 and X.shape[0] == 80 * nc ** 3
    s_out = float((nut * w).mean() / w.mean())
    model = CL.MLPModel.init(0, s_in=s_in, s_out=s_out, device=cuda)
    losses = CL.train(model, X, nut, steps=600, batch=16384, lr=2e-3, weight=w)
    assert losses[-1][1] < losses[0][1]
    res = CL.evaluate(sns, model, nf, nc, kc, seeds=[7], nu=nu, dt=dt, steps=400, device=cuda)
    assert res["mlp"] < res["plain"], res
    # the band and output scale fitted on the training seed (6 runs), then the
    # held-out seed: still ahead of the unclosed run
    errs, band = CL.calibrate(sns, model, calib, nu, dt, 400, kc, scales=(1.0, 2.0, 4.0),
                              bands=((0.0, 0.0), (2 / 3, 1.0)))
    assert len(errs) == 6 and band in ((0.0, 0.0), (round(2 / 3 * kc, 6), float(kc)))
    assert abs(model.s_out / s_out - min(errs, key=errs.get)[1]) < 1e-12
    res = CL.evaluate(sns, model, nf, nc, kc, seeds=[7], nu=nu, dt=dt, steps=400, device=cuda,
                      band=band)
    assert res["mlp"] < res["plain"], res
