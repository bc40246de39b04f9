"""The closure oracle (oracle/closure.py) on the CPU: consistency with the
reference-pinned C oracle, exact gradients, filter and spectrum identities."""
import numpy as np
import pytest

from conftest import rel_l2


@pytest.fixture(scope="module")
def C():
    from oracle import closure
    return closure


def _field(n, seed):
    from spectral_upcxx_b200 import ic
    return [np.fft.fftn(c) for c in ic.solenoidal_spectrum(n, seed=seed)]


def test_plain_les_step_is_the_ns_step(C, oracle):
    """With nu_t = 0 the LES step is the ns.cpp step of the C oracle."""
    n, nu, dt = 16, 0.01, 1e-3
    V0 = _field(n, 3)
    w0 = oracle.curl(V0)
    ref = oracle.NS((n, n, n), nu, dt)
    ref.bootstrap(V0, w0)
    s = ref.state()
    les = C.LES(nu, dt, "plain")
    les.set_state(s["V1"], s["cross0"])
    for _ in range(3):
        ref.step()
    les.step(3)
    got = ref.state()
    for d in range(3):
        assert rel_l2(les.V1[d], got["V1"][d]) < 1e-12
        assert rel_l2(les.c0[d], got["cross0"][d]) < 1e-12


def test_mlp_gradients_match_finite_differences(C):
    r = np.random.default_rng(0)
    net = C.MLP.init(1)
    net.b1 = r.standard_normal(C.HIDDEN) * 0.1
    net.b2 = r.standard_normal(C.HIDDEN) * 0.1
    X = np.zeros((64, C.KPAD))
    X[:, :C.NIN] = r.standard_normal((64, C.NIN))
    t = np.abs(r.standard_normal(64))
    loss, g = net.loss_and_grads(X, t, rounding=False)
    h = 1e-6
    for name, idx in (("W1", (3, 2)), ("W2", (5, 7)), ("w3", (11,)), ("b1", (4,)),
                      ("b2", (9,))):
        P = getattr(net, name)
        old = P[idx]
        P[idx] = old + h
        lp, _ = net.loss_and_grads(X, t, rounding=False)
        P[idx] = old - h
        lm, _ = net.loss_and_grads(X, t, rounding=False)
        P[idx] = old
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[name][idx]) <= 1e-6 * max(1.0, abs(fd)), name
    old = net.b3
    net.b3 = old + h
    lp, _ = net.loss_and_grads(X, t, rounding=False)
    net.b3 = old - h
    lm, _ = net.loss_and_grads(X, t, rounding=False)
    net.b3 = old
    assert abs((lp - lm) / (2 * h) - g["b3"][0]) < 1e-6


def test_bf16_rounding(C):
    assert C.bf16(1.0) == 1.0
    assert C.bf16(1.0 + 2 ** -9) == 1.0  # tie -> even
    assert C.bf16(1.0 + 3 * 2 ** -9) == 1.0 + 2 ** -7
    assert C.bf16(-3.14159) == pytest.approx(-3.140625)


def test_truncate_pad_and_spectrum(C):
    n, nc, kc = 32, 16, 5
    V = _field(n, 4)
    Vc = [C.truncate(v, nc, kc) for v in V]
    back = [C.truncate(C.pad(v, n), nc, kc) for v in Vc]
    for a, b in zip(back, Vc):
        assert rel_l2(a, b) < 1e-14
    # the coarse field's physical values are the fine field's filtered values
    uf = np.fft.ifftn(C.pad(Vc[0], n))
    uc = np.fft.ifftn(Vc[0])
    assert rel_l2(uf[::2, ::2, ::2], uc) < 1e-12
    E = C.spectrum(V)
    u = [np.fft.ifftn(v) for v in V]
    assert abs(E.sum() / (0.5 * np.mean(sum(np.abs(x) ** 2 for x in u))) - 1) < 1e-12
    Ec = C.spectrum(Vc)
    # shells below the cutoff are whole; shell kc holds only |k| <= kc
    assert np.allclose(Ec[:kc], E[:kc], rtol=1e-12, atol=0)
    assert 0 < Ec[kc] < E[kc]
    assert np.all(Ec[kc + 1:] == 0)


def test_smagorinsky_simple_shear(C):
    z = np.zeros((2, 2, 2))
    g = 3.0
    A = [[z, z + g, z], [z, z, z], [z, z, z]]  # du/dy = g
    nut = C.smagorinsky(A, 0.17, 0.1)
    assert np.allclose(nut, (0.17 * 0.1) ** 2 * g)


def test_sgs_target_of_a_resolved_field_vanishes(C):
    """A field already inside the cutoff has no subgrid stress."""
    n, nc, kc = 32, 16, 5
    V = [C.pad(C.truncate(v, nc, kc), n) for v in _field(n, 6)]
    X, nut, w, Vc = C.sgs_sample(V, nc, kc, s_in=1.0)
    assert X.shape == (nc ** 3, C.KPAD)
    assert np.max(np.abs(nut)) < 1e-10


def test_band_weight_and_band_restricted_force(C):
    """The default band weighs every mode but k = 0 by 1; a ramp and a sharp
    split leave the eddy force only on the small scales."""
    n = 16
    KX, KY, KZ = C.kgrid((n, n, n))
    km = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    b0 = C.band_weight((n, n, n), (0, 0))
    assert b0[0, 0, 0] == 0 and np.all(b0[km > 0] == 1)
    br = C.band_weight((n, n, n), (2, 6))
    assert np.all(br[km <= 2] == 0) and np.all(br[km >= 6] == 1)
    mid = (km > 2) & (km < 6)
    assert np.allclose(br[mid], (km[mid] - 2) / 4)
    bs = C.band_weight((n, n, n), (3, 0))
    assert np.array_equal(bs, (km > 3).astype(float))
    # the Smagorinsky force of a smooth field with a sharp split at 3: below
    # the split the LES nonlinear term is the plain one
    V = _field(n, 4)
    p = {"cs": 0.2, "delta": np.pi / 5}
    plain = C.nonlinear(V, "plain")
    full = C.nonlinear(V, "smagorinsky", p)
    split = C.nonlinear(V, "smagorinsky", p, band=(3, 0))
    low = km <= 3
    for d in range(3):
        assert np.allclose(split[d][low], plain[d][low], rtol=0, atol=1e-9)
        assert np.allclose(split[d][~low], full[d][~low], rtol=0, atol=1e-9)
        assert not np.allclose(full[d][low], plain[d][low], rtol=0, atol=1e-9)
