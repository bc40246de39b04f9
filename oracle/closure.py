"""TEST INFRASTRUCTURE ONLY -- CPU oracle (numpy, FP64) of the learned-closure path.

The reference has no subgrid model: these functions state the closure
extension of the exec/ns.cpp step that the GPU path implements, so that
tests can check the GPU kernels against an independent CPU computation.
Only tests/ and bench.py's CPU leg may import this module.

Conventions follow the reference (src/Scalar.cpp): fields are complex arrays
of shape (nz, ny, nx), forward = unnormalised DFT with exp(-i) followed by
zeroing of the Nyquist planes, inverse = DFT with exp(+i) divided by N
(numpy's fftn / ifftn), wavenumber k = i for i <= n/2 else i - n.

LES step (ns.cpp:167-217 with an eddy-viscosity term):
  u = inverse(V1), A_ij = inverse(i k_j V1_i)          (A_ij = d_j u_i)
  omega = (A_zy - A_yz, A_xz - A_zx, A_yx - A_xy)
  nu_t = model(Re A) >= 0,  S_ij = (A_ij + A_ji) / 2,  tau_ij = 2 nu_t S_ij
  cross1_i = zeroNyquist(fftn(u x omega)_i + b(|k|) sum_j i k_j fftn(tau_ij))
  then the AB2 / projection / Crank-Nicolson update of ns.cpp:170-187.
The band weight b(|k|) = clip((|k| - k_lo) / (k_hi - k_lo), 0, 1) (k_hi <= k_lo:
1 for |k| > k_lo, else 0) confines the eddy force to the small resolved
scales; the default band (0, 0) is 1 on every mode but k = 0.
The bootstrap is the plain one of ns.cpp:132-153.

Models: 'plain' (nu_t = 0), 'smagorinsky' (nu_t = (Cs Delta)^2 sqrt(2 S:S)),
'mlp' (nu_t = s_out softplus(MLP(s_in Re A))).  MLP 9 -> 64 -> 64 -> 1 with
ReLU hidden layers: BF16 weights, inputs and hidden activations, FP32 (here
FP64) accumulation, FP32 biases; the rounding points mirror the GPU kernels.
"""
from __future__ import annotations

import numpy as np

HIDDEN = 64
NIN = 9
KPAD = 16


# --------------------------------------------------------------------- BF16
def bf16(x) -> np.ndarray:
    """Round to bfloat16 (nearest, ties to even), returned as float64."""
    f = np.ascontiguousarray(np.asarray(x, dtype=np.float32))
    b = f.view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) & 0xFFFF0000
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


# --------------------------------------------------------------------- spectral helpers
def k1d(n):
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64)


def kgrid(shape):
    nz, ny, nx = shape
    KZ, KY, KX = np.meshgrid(k1d(nz), k1d(ny), k1d(nx), indexing="ij")
    return KX, KY, KZ


def zero_nyquist(f):
    f = f.copy()
    nz, ny, nx = f.shape
    f[nz // 2, :, :] = 0
    f[:, ny // 2, :] = 0
    f[:, :, nx // 2] = 0
    return f


def forward(f):
    return zero_nyquist(np.fft.fftn(f))


def inverse(f):
    return np.fft.ifftn(f)


def velocity_gradient(V):
    """A[i][j] = inverse(i k_j V_i) (physical, complex)."""
    K = kgrid(V[0].shape)
    return [[inverse(1j * K[j] * V[i]) for j in range(3)] for i in range(3)]


# --------------------------------------------------------------------- models
def smagorinsky(Ar, cs, delta):
    """(Cs Delta)^2 sqrt(2 S:S) from the real velocity gradient Ar[i][j]."""
    s2 = 0.0
    for i in range(3):
        for j in range(3):
            s = 0.5 * (Ar[i][j] + Ar[j][i])
            s2 = s2 + s * s
    return (cs * delta) ** 2 * np.sqrt(2.0 * s2)


def features(Ar, s_in):
    """(points, 16) inputs: s_in * A_ij in row-major (i, j) order, zero padded."""
    cols = [np.ravel(Ar[i][j]) * s_in for i in range(3) for j in range(3)]
    X = np.zeros((cols[0].size, KPAD))
    X[:, :NIN] = np.stack(cols, axis=1)
    return X


def softplus(z):
    return np.where(z > 20.0, z, np.log1p(np.exp(np.minimum(z, 20.0))))


def sigmoid(z):
    return 1.0 / (1.0 + np.exp(-z))


class MLP:
    """Master parameters (float64 copies of the GPU's FP32 masters)."""

    def __init__(self, W1, b1, W2, b2, w3, b3, s_in=1.0, s_out=1.0):
        self.W1 = np.asarray(W1, dtype=np.float64).reshape(HIDDEN, KPAD)
        self.b1 = np.asarray(b1, dtype=np.float64).reshape(HIDDEN)
        self.W2 = np.asarray(W2, dtype=np.float64).reshape(HIDDEN, HIDDEN)
        self.b2 = np.asarray(b2, dtype=np.float64).reshape(HIDDEN)
        self.w3 = np.asarray(w3, dtype=np.float64).reshape(HIDDEN)
        self.b3 = float(np.asarray(b3).reshape(-1)[0])
        self.s_in, self.s_out = float(s_in), float(s_out)

    @staticmethod
    def init(seed):
        """He-style initialisation (the GPU trainer takes the same arrays)."""
        r = np.random.default_rng(seed)
        W1 = np.zeros((HIDDEN, KPAD))
        W1[:, :NIN] = r.standard_normal((HIDDEN, NIN)) * np.sqrt(2.0 / NIN)
        W2 = r.standard_normal((HIDDEN, HIDDEN)) * np.sqrt(2.0 / HIDDEN)
        w3 = r.standard_normal(HIDDEN) * np.sqrt(1.0 / HIDDEN)
        f32 = lambda a: np.asarray(a, dtype=np.float32).astype(np.float64)
        return MLP(f32(W1), np.zeros(HIDDEN), f32(W2), np.zeros(HIDDEN), f32(w3), 0.0)

    def forward(self, X, rounding=True):
        """z (pre-softplus) per row of X (points, 16), plus the cache.
        rounding=False drops the BF16 rounding (exact FP64 network)."""
        r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
        Xb = r(X)
        pre1 = Xb @ r(self.W1).T + self.b1
        h1 = r(np.maximum(pre1, 0.0))
        pre2 = h1 @ r(self.W2).T + self.b2
        h2 = np.maximum(pre2, 0.0)
        z = h2 @ r(self.w3) + self.b3
        return z, (Xb, pre1, h1, pre2, h2)

    def nut(self, X):
        z, _ = self.forward(X)
        return self.s_out * softplus(z)

    def loss_and_grads(self, X, t, rounding=True, w=None):
        """Mean weighted squared error w (softplus(z) - t)^2 (targets in model
        units, w = 1 when None) and its gradients, with the GPU's BF16 rounding
        of the backward operands (dPre2, dPre1)."""
        r = bf16 if rounding else (lambda a: np.asarray(a, dtype=np.float64))
        B = X.shape[0]
        w = np.ones(B) if w is None else np.asarray(w, dtype=np.float64)
        z, (Xb, pre1, h1, pre2, h2) = self.forward(X, rounding)
        y = softplus(z)
        loss = float(np.mean(w * (y - t) ** 2))
        dz = (2.0 / B) * w * (y - t) * sigmoid(z)
        w3b = r(self.w3)
        g = {"w3": h2.T @ dz, "b3": np.array([dz.sum()])}
        dpre2 = (dz[:, None] * w3b[None, :]) * (pre2 > 0)
        g["b2"] = dpre2.sum(axis=0)
        dpre2b = r(dpre2)
        g["W2"] = dpre2b.T @ h1
        dh1 = dpre2b @ r(self.W2)
        dpre1 = dh1 * (pre1 > 0)
        g["b1"] = dpre1.sum(axis=0)
        g["W1"] = r(dpre1).T @ Xb
        return loss, g


def model_nut(model, Ar, params=None):
    if model == "plain":
        return np.zeros_like(Ar[0][0])
    if model == "smagorinsky":
        return smagorinsky(Ar, params["cs"], params["delta"])
    if model == "mlp":
        net = params["mlp"]
        return net.nut(features(Ar, net.s_in)).reshape(Ar[0][0].shape)
    raise ValueError(model)


# --------------------------------------------------------------------- LES step
def band_weight(shape, band):
    """b(|k|) of the module docstring on the grid of `shape`."""
    KX, KY, KZ = kgrid(shape)
    km = np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)
    lo, hi = band
    if hi > lo:
        return np.clip((km - lo) / (hi - lo), 0.0, 1.0)
    return (km > lo).astype(np.float64)


def nonlinear(V, model="plain", params=None, band=(0.0, 0.0)):
    """cross1 of the LES step (module docstring)."""
    K = kgrid(V[0].shape)
    u = [inverse(v) for v in V]
    A = velocity_gradient(V)
    w = [A[2][1] - A[1][2], A[0][2] - A[2][0], A[1][0] - A[0][1]]
    c = [u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]]
    out = [np.fft.fftn(x) for x in c]
    if model != "plain":
        nut = model_nut(model, [[a.real for a in row] for row in A], params)
        b = band_weight(V[0].shape, band)
        for i in range(3):
            for j in range(3):
                tau = 2.0 * nut * 0.5 * (A[i][j] + A[j][i])
                out[i] = out[i] + b * (1j * K[j] * np.fft.fftn(tau))
    return [zero_nyquist(x) for x in out]


def update(V1, c0, c1, nu, dt, kc=None):
    """ns.cpp:170-187 on Fourier fields.  With a cutoff kc the modes |k| > kc
    are not evolved: their nonlinear term, velocity and history are zero."""
    KX, KY, KZ = kgrid(V1[0].shape)
    K = (KX, KY, KZ)
    k2 = KX ** 2 + KY ** 2 + KZ ** 2
    if kc is not None:
        c1 = [np.where(k2 > kc * kc, 0, c) for c in c1]
    hK = dt / 2
    F = [hK * (3 * c1[d] - c0[d]) for d in range(3)]
    lap = [nu * hK * (-k2 * V1[d]) for d in range(3)]
    s = [V1[d] + lap[d] + F[d] for d in range(3)]
    G = 1j * KX * s[0] + 1j * KY * s[1] + 1j * KZ * s[2]
    nz = k2 != 0
    G = np.where(nz, G / np.where(nz, -k2, 1.0), G)
    den = 1.0 + nu * hK * k2
    out = []
    for d in range(3):
        vh = V1[d] + F[d] - 1j * K[d] * G
        vv = vh + lap[d]
        vv = np.where(nz, vv / den, vv)
        if kc is not None:
            vv = np.where(k2 > kc * kc, 0, vv)
        out.append(vv)
    return (out, c1) if kc is not None else out


class LES:
    """FP64 LES stepper: state (V1, cross0) as in exec/ns.cpp."""

    def __init__(self, nu, dt, model="plain", params=None, kc=None, band=(0.0, 0.0)):
        self.nu, self.dt, self.model, self.params, self.kc = nu, dt, model, params, kc
        self.band = band
        self.V1 = self.c0 = None

    def set_state(self, V1, cross0):
        self.V1 = [np.array(v, dtype=np.complex128) for v in V1]
        self.c0 = [np.array(c, dtype=np.complex128) for c in cross0]

    def step(self, n=1):
        for _ in range(n):
            c1 = nonlinear(self.V1, self.model, self.params, self.band)
            if self.kc is None:
                self.V1 = update(self.V1, self.c0, c1, self.nu, self.dt)
            else:
                self.V1, c1 = update(self.V1, self.c0, c1, self.nu, self.dt, self.kc)
            self.c0 = c1


# --------------------------------------------------------------------- filtering, targets
def truncate(Vf, nc, kc):
    """Sharp spherical cutoff |k| <= kc of a fine Fourier field onto an nc^3
    grid, rescaled to the coarse grid's unnormalised DFT (x nc^3 / nf^3)."""
    nf = Vf.shape[0]
    kk = k1d(nc).astype(int)
    idx = np.where(kk >= 0, kk, kk + nf)
    KX, KY, KZ = kgrid((nc, nc, nc))
    keep = (KX ** 2 + KY ** 2 + KZ ** 2 <= kc * kc) & (np.abs(KX) < nc // 2) & \
        (np.abs(KY) < nc // 2) & (np.abs(KZ) < nc // 2)
    out = Vf[np.ix_(idx, idx, idx)] * (nc ** 3 / nf ** 3)
    return np.where(keep, out, 0)


def pad(Vc, nf):
    """Coarse Fourier field onto an nf^3 grid (zero outside, x nf^3 / nc^3)."""
    nc = Vc.shape[0]
    kk = k1d(nc).astype(int)
    idx = np.where(kk >= 0, kk, kk + nf)
    out = np.zeros((nf, nf, nf), dtype=np.complex128)
    out[np.ix_(idx, idx, idx)] = Vc * (nf ** 3 / nc ** 3)
    return out


def sgs_sample(Vf, nc, kc, s_in, eps=1e-30):
    """Training pairs from one fine Fourier velocity: features of the filtered
    gradient (points, 16) and the eddy viscosity nu_t of the least-squares
    projection of the filtered SGS stress onto -2 nu_t S (pointwise):
      tau_ij = filter(u_i u_j) - filter(ubar_i ubar_j) on the fine grid,
      nu_t = -(tau^d : Sbar) / (2 Sbar : Sbar),
    with the weight Sbar : Sbar of each pair.  Also returns the coarse
    filtered velocity."""
    nf = Vf[0].shape[0]
    Vc = [truncate(v, nc, kc) for v in Vf]
    u = [inverse(v) for v in Vf]
    ub = [inverse(pad(v, nf)) for v in Vc]
    tau = {}
    for i in range(3):
        for j in range(i, 3):
            T = u[i] * u[j] - ub[i] * ub[j]
            tau[i, j] = tau[j, i] = inverse(truncate(np.fft.fftn(T), nc, kc)).real
    A = velocity_gradient(Vc)
    Ar = [[a.real for a in row] for row in A]
    tr = (tau[0, 0] + tau[1, 1] + tau[2, 2]) / 3.0
    num = 0.0
    den = 0.0
    for i in range(3):
        for j in range(3):
            S = 0.5 * (Ar[i][j] + Ar[j][i])
            td = tau[i, j] - (tr if i == j else 0.0)
            num = num + td * S
            den = den + S * S
    nut = -num / (2.0 * den + eps)
    return features(Ar, s_in), np.ravel(nut), np.ravel(den), Vc


def spectrum(V):
    """E(k) for shells k = round(|k|): sum over the shell of |V_hat|^2 / (2 N^2),
    N the number of points, so that sum_k E(k) = <|u|^2> / 2."""
    KX, KY, KZ = kgrid(V[0].shape)
    shell = np.rint(np.sqrt(KX ** 2 + KY ** 2 + KZ ** 2)).astype(int)
    N = V[0].size
    e = sum(np.abs(v) ** 2 for v in V) / (2.0 * N * N)
    return np.bincount(shell.ravel(), weights=e.ravel())
