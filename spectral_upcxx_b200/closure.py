"""Learned eddy-viscosity closure for coarse-grid runs of the NS step.

No reference counterpart: exec/ns.cpp has no subgrid model.  The pieces:

* ``MLPModel`` -- the pointwise MLP 9 -> 64 -> 64 -> 1 (BF16 weights, FP32
  accumulation, softplus output) with FP32 masters and Adam, trained and
  evaluated by the library's tensor-core kernels (sns_mlp_*).
* ``truncate`` / ``pad`` / ``sgs_sample`` / ``spectrum`` -- the sharp
  spectral filter, the training pairs of filtered DNS and the shell energy
  spectrum (sns_spectral_*, sns_sgs_sample, sns_energy_spectrum).
* ``NSStepper.set_closure`` -- Smagorinsky or the MLP inside the step.
* ``dns_dataset`` / ``train`` / ``evaluate`` -- the experiment: fine DNS of
  spectrum-seeded fields, filtered snapshots as training data, and coarse
  runs (plain, Smagorinsky, MLP) judged by their energy spectrum against the
  filtered DNS.

Conventions (fixed here, recorded in the design notes): the filter is a
sharp spherical cutoff |k| <= kc; spectrum shells are round(|k|); the
training target is the pointwise least-squares eddy viscosity
-(tau^d : S) / (2 S : S) of the filtered SGS stress; model inputs are the
nine components of the filtered velocity gradient A_ij = d_j u_i scaled by
s_in; outputs are nu_t / s_out.  Everything runs on the GPU; there is no
CPU path.
"""
from __future__ import annotations

import ctypes as C
import math
import time

import numpy as np
import torch

from . import _native as N
from .ops import _check_field, _same, _stream

HIDDEN, NIN, KPAD = 64, 9, 16


def _sizes():
    p, b = C.c_int64(), C.c_int64()
    N.call("sns_mlp_sizes", C.byref(p), C.byref(b))
    return p.value, b.value


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


class MLPModel:
    """FP32 masters + Adam state + the packed bf16 inference copy, on a device."""

    def __init__(self, W1, b1, W2, b2, w3, b3, s_in=1.0, s_out=1.0, device="cuda"):
        self.nparams, self.packed_bytes = _sizes()
        self.device = torch.device(device)
        flat = np.concatenate([np.asarray(W1, np.float64).reshape(HIDDEN, KPAD).ravel(),
                               np.asarray(b1, np.float64).ravel(),
                               np.asarray(W2, np.float64).ravel(),
                               np.asarray(b2, np.float64).ravel(),
                               np.asarray(w3, np.float64).ravel(),
                               np.asarray(b3, np.float64).reshape(1)])
        assert flat.size == self.nparams
        self.master = torch.tensor(flat, dtype=torch.float32, device=self.device)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.packed = torch.zeros(self.packed_bytes, dtype=torch.uint8, device=self.device)
        self.grad = torch.zeros(self.nparams + 1, dtype=torch.float32, device=self.device)
        self.steps = 0
        self.set_scales(s_in, s_out)

    @staticmethod
    def init(seed, s_in=1.0, s_out=1.0, device="cuda"):
        """He-style initial weights from a numpy generator (W1 padding zero)."""
        r = np.random.default_rng(seed)
        W1 = np.zeros((HIDDEN, KPAD))
        W1[:, :NIN] = r.standard_normal((HIDDEN, NIN)) * math.sqrt(2.0 / NIN)
        W2 = r.standard_normal((HIDDEN, HIDDEN)) * math.sqrt(2.0 / HIDDEN)
        w3 = r.standard_normal(HIDDEN) * math.sqrt(1.0 / HIDDEN)
        return MLPModel(W1, np.zeros(HIDDEN), W2, np.zeros(HIDDEN), w3, 0.0, s_in, s_out,
                        device)

    def set_scales(self, s_in, s_out):
        self.s_in, self.s_out = float(s_in), float(s_out)
        N.call("sns_mlp_pack", _p(self.master), self.s_in, self.s_out, _p(self.packed),
               _stream(self.master))

    def arrays(self):
        """Masters as numpy float64 arrays (W1, b1, W2, b2, w3, b3)."""
        f = self.master.detach().cpu().double().numpy()
        o = [0, 1024, 1088, 5184, 5248, 5312, 5313]
        return (f[o[0]:o[1]].reshape(HIDDEN, KPAD), f[o[1]:o[2]], f[o[2]:o[3]].reshape(HIDDEN, HIDDEN),
                f[o[3]:o[4]], f[o[4]:o[5]], f[o[5]])

    def infer(self, X):
        """nu_t for rows of X (bf16 tensor (M, 16) on the device)."""
        assert X.dtype == torch.bfloat16 and X.is_contiguous() and X.shape[1] == KPAD
        out = torch.empty(X.shape[0], dtype=torch.float32, device=X.device)
        N.call("sns_mlp_infer", _p(self.packed), _p(X), X.shape[0], _p(out), _stream(X))
        return out

    def gradient(self, X, target, idx=None, batch=None, weight=None):
        """Gradient vector (its last entry: the mean loss) of the weighted
        squared error of softplus(z) against target (model units) over rows
        idx of X (or the first `batch` rows)."""
        B = int(idx.numel()) if idx is not None else int(batch or X.shape[0])
        N.call("sns_mlp_grad", _p(self.packed), _p(X), _p(target), _p(weight), _p(idx), B,
               _p(self.grad), _stream(X))
        return self.grad

    def adam(self, lr, beta1=0.9, beta2=0.999, eps=1e-8):
        self.steps += 1
        N.call("sns_mlp_adam", _p(self.master), _p(self.m), _p(self.v), _p(self.grad),
               self.steps, float(lr), float(beta1), float(beta2), float(eps), _p(self.packed),
               _stream(self.master))


# --------------------------------------------------------------------- data kernels
def truncate(fields, nc: int, kc: float):
    fs = list(fields)
    p = _same(fs)
    nf = fs[0].shape[0]
    out = [torch.empty((nc, nc, nc), dtype=fs[0].dtype, device=fs[0].device) for _ in fs]
    N.call("sns_spectral_truncate", N.ptrs([f.data_ptr() for f in fs]),
           N.ptrs([o.data_ptr() for o in out]), len(fs), nf, nc, float(kc), p, _stream(fs[0]))
    return out


def pad(fields, nf: int):
    fs = list(fields)
    p = _same(fs)
    nc = fs[0].shape[0]
    out = [torch.empty((nf, nf, nf), dtype=fs[0].dtype, device=fs[0].device) for _ in fs]
    N.call("sns_spectral_pad", N.ptrs([f.data_ptr() for f in fs]),
           N.ptrs([o.data_ptr() for o in out]), len(fs), nc, nf, p, _stream(fs[0]))
    return out


def sgs_sample(V, nc: int, kc: float, s_in: float, Vc=None):
    """Training pairs of one fine Fourier velocity (see sns_sgs_sample).
    Returns (X (nc^3, 16) bf16, nu_t (nc^3,) float32, weight S:S (nc^3,)
    float32, Vc or None)."""
    V = list(V)
    p = _same(V)
    nf = V[0].shape[0]
    dev = V[0].device
    n3 = nc ** 3
    X = torch.empty((n3, KPAD), dtype=torch.bfloat16, device=dev)
    nut = torch.empty(n3, dtype=torch.float32, device=dev)
    w = torch.empty(n3, dtype=torch.float32, device=dev)
    vc = N.ptrs([v.data_ptr() for v in Vc]) if Vc is not None else None
    N.call("sns_sgs_sample", N.ptrs([v.data_ptr() for v in V]), nf, nc, float(kc), float(s_in), p,
           _p(X), _p(nut), _p(w), vc, _stream(V[0]))
    return X, nut, w, Vc


def spectrum(V, nshell=None):
    """E[k] (float64 numpy) for shells k = round(|k|)."""
    V = list(V)
    p = _same(V)
    nz, ny, nx = V[0].shape
    if nshell is None:
        nshell = int(math.ceil(math.sqrt(3) * max(nx, ny, nz) / 2)) + 2
    E = torch.empty(nshell, dtype=torch.float64, device=V[0].device)
    N.call("sns_energy_spectrum", N.ptrs([v.data_ptr() for v in V]), nx, ny, nz, p, _p(E), nshell,
           _stream(V[0]))
    return E.cpu().numpy()


# --------------------------------------------------------------------- experiment
def spectrum_error(E, Eref, kmax):
    """Mean relative error of shells 1..kmax-1 (the whole shells under the cutoff)."""
    k = np.arange(1, kmax)
    return float(np.mean(np.abs(E[k] - Eref[k]) / Eref[k]))


# bands (k_lo, k_hi) of the eddy force tried by the calibrations, in units of
# the cutoff kc: none, ramps from 2/3 kc to just below and to the cutoff, a
# sharp split at 3/4 kc
BANDS = ((0.0, 0.0), (2 / 3, 20 / 21), (2 / 3, 1.0), (4 / 7, 1.0), (16 / 21, 20 / 21),
         (16 / 21, 0.0))


def _bands(kc, bands):
    return [(round(lo * kc, 6), round(hi * kc, 6)) for lo, hi in bands]


def calibrate(S, model, calib, nu, dt, steps, kc, scales=(1.0, 1.5, 2.0, 3.0, 4.0, 5.0, 6.0, 8.0),
              bands=BANDS, dtype=torch.complex64):
    """Choose the model's output scale (a factor of `scales`) and the band of
    the eddy force (`bands`, fractions of kc) whose coarse run from a training
    seed's filtered field (calib from dns_dataset) ends with the smallest
    spectrum error against that seed's filtered DNS.  `steps` steps of `dt`.
    Leaves the best scale applied; returns ({(band, scale): error}, band)."""
    s_out0 = model.s_out
    errs = {}
    for band in _bands(kc, bands):
        for c in scales:
            model.set_scales(model.s_in, s_out0 * c)
            V = coarse_run(S, calib["Vc0"], nu, dt, steps, model=model, kc=kc, dtype=dtype,
                           band=band)
            errs[(band, c)] = spectrum_error(spectrum(V), calib["Eref"], int(kc))
    band, best = min(errs, key=errs.get)
    model.set_scales(model.s_in, s_out0 * best)
    return errs, band


def calibrate_smagorinsky(S, calib, nu, dt, steps, kc, cs=(0.08, 0.1, 0.13, 0.17, 0.2, 0.25),
                          bands=BANDS, dtype=torch.complex64):
    """The same choice for the Smagorinsky constant Cs and the band; returns
    ({(band, cs): error}, (band, cs))."""
    errs = {}
    for band in _bands(kc, bands):
        for c in cs:
            V = coarse_run(S, calib["Vc0"], nu, dt, steps, csd2=smagorinsky_cs_delta2(c, kc),
                           kc=kc, dtype=dtype, band=band)
            errs[(band, c)] = spectrum_error(spectrum(V), calib["Eref"], int(kc))
    return errs, min(errs, key=errs.get)


def smagorinsky_cs_delta2(cs: float, kc: float) -> float:
    """(Cs Delta)^2 with Delta = pi / kc, the width of the sharp cutoff."""
    return (cs * math.pi / kc) ** 2


def _initial(n, seed, dtype, device):
    from .ic import solenoidal_spectrum_hat
    return [x.to(dtype) for x in solenoidal_spectrum_hat(n, seed, device)]


def dns_dataset(S, nf, nc, kc, seeds, nu, dt, steps, every, dtype=torch.complex64, device="cuda",
                s_in=None, log=None, calib=None):
    """Run fine DNS from each seed for `steps` steps and take a filtered
    training sample every `every` steps.  Returns X (M, 16) bf16, nu_t (M,)
    float32, the weights S:S / mean(S:S) (M,) float32, s_in (the feature
    scale: 1 / rms of the first snapshot's gradient when not given) and the
    number of snapshots.  With `calib` (a dict), the first seed's filtered
    initial field ('Vc0') and filtered final spectrum ('Eref') are stored in
    it for calibrate()."""
    Xs, ts, ws = [], [], []
    snaps = 0
    for seed in seeds:
        V0 = _initial(nf, seed, dtype, device)
        if calib is not None and seed == seeds[0]:
            calib["Vc0"] = truncate(V0, nc, kc)
        st = S.NSStepper((nf, nf, nf), nu, dt, dtype, device=device)
        st.bootstrap(V0, S.curl(V0))
        del V0
        for step in range(1, steps + 1):
            st.step(1)
            if step % every:
                continue
            V1 = st.velocity()
            if s_in is None:
                X0, _, _, _ = sgs_sample(V1, nc, kc, 1.0)
                s_in = 1.0 / float(X0[:, :NIN].float().pow(2).mean().sqrt())
            X, t, w, _ = sgs_sample(V1, nc, kc, s_in)
            Xs.append(X)
            ts.append(t)
            ws.append(w)
            snaps += 1
        if calib is not None and seed == seeds[0]:
            calib["Eref"] = spectrum(truncate(st.velocity(), nc, kc))
        st.close()
        if log:
            log(f"seed {seed}: {snaps} snapshots so far")
    w = torch.cat(ws)
    w /= w.mean()
    return torch.cat(Xs), torch.cat(ts), w, s_in, snaps


def train(model, X, nut, steps, batch, lr, weight=None, seed=0, log=None):
    """Adam on the (weighted) mean squared error of nu_t / s_out over random
    batches (with replacement)."""
    g = torch.Generator(device=X.device).manual_seed(seed)
    target = (nut / model.s_out).contiguous()
    M = X.shape[0]
    losses = []
    for it in range(steps):
        idx = torch.randint(0, M, (batch,), device=X.device, generator=g, dtype=torch.int32)
        grad = model.gradient(X, target, idx=idx, weight=weight)
        model.adam(lr if it < steps * 3 // 4 else lr / 10)
        if it % max(1, steps // 20) == 0 or it == steps - 1:
            losses.append((it, float(grad[-1])))
            if log:
                log(f"train step {it}: loss {losses[-1][1]:.4e}")
    return losses


def coarse_run(S, Vc0, nu, dt, steps, model=None, csd2=0.0, kc=0.0, dtype=torch.complex64,
               band=(0.0, 0.0)):
    """Coarse run from the filtered field Vc0 over the modes |k| <= kc (all
    modes when kc = 0) with no closure, Smagorinsky (csd2 > 0, model None) or
    the MLP (model), the eddy force weighted by `band` (NSStepper.set_sgs_band).
    Returns the final velocity."""
    n = Vc0[0].shape[0]
    st = S.NSStepper((n, n, n), nu, dt, dtype, device=Vc0[0].device)
    if model is not None:
        st.set_closure(N.SNS_CLOSURE_MLP, mlp=model.packed, kc=kc)
    elif csd2 > 0:
        st.set_closure(N.SNS_CLOSURE_SMAGORINSKY, cs_delta2=csd2, kc=kc)
    else:
        st.set_closure(N.SNS_CLOSURE_NONE, kc=kc)
    st.set_sgs_band(*band)
    st.bootstrap(Vc0, S.curl(Vc0))
    st.step(steps)
    V = st.velocity()
    st.close()
    return V


def evaluate(S, model, nf, nc, kc, seeds, nu, dt, steps, cs=0.17, dtype=torch.complex64,
             device="cuda", coarse_dt=None, band=(0.0, 0.0), smag_band=(0.0, 0.0), extra=None):
    """Spectrum errors (shells 1..kc-1) at the end of `steps` steps against the
    filtered fine DNS, for the plain, Smagorinsky (cs, smag_band) and MLP
    (band) coarse runs and any `extra` runs ({name: coarse_run keywords}),
    plus the steps/s of the coarse MLP run and of the fine DNS.  The coarse
    runs take time step coarse_dt (default dt) and end at the same time."""
    coarse_dt = dt if coarse_dt is None else coarse_dt
    coarse_steps = int(round(steps * dt / coarse_dt))
    runs = {"plain": {}, "smagorinsky": {"csd2": smagorinsky_cs_delta2(cs, kc), "band": smag_band},
            "mlp": {"model": model, "band": band}}
    runs.update(extra or {})
    res = {name: [] for name in runs}
    spectra = {}
    t_dns = t_les = 0.0
    for seed in seeds:
        V0 = _initial(nf, seed, dtype, device)
        Vc0 = truncate(V0, nc, kc)
        st = S.NSStepper((nf, nf, nf), nu, dt, dtype, device=device)
        st.bootstrap(V0, S.curl(V0))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st.step(steps)
        torch.cuda.synchronize()
        t_dns += time.perf_counter() - t0
        Eref = spectrum(truncate(st.velocity(), nc, kc))
        st.close()
        for name, kw in runs.items():
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            V = coarse_run(S, Vc0, nu, coarse_dt, coarse_steps, kc=kc, dtype=dtype, **kw)
            torch.cuda.synchronize()
            if name == "mlp":
                t_les += time.perf_counter() - t0
            E = spectrum(V)
            res[name].append(spectrum_error(E, Eref, int(kc)))
            if seed == seeds[0]:
                spectra[name] = E[:int(kc) + 1].tolist()
        if seed == seeds[0]:
            spectra["filtered_dns"] = Eref[:int(kc) + 1].tolist()
    out = {k: float(np.mean(v)) for k, v in res.items()}
    out["spectra_first_seed"] = spectra
    out["dns_steps_per_s"] = steps * len(seeds) / t_dns
    out["mlp_run_steps_per_s"] = coarse_steps * len(seeds) / t_les
    out["coarse_dt"] = coarse_dt
    out["all_finite"] = bool(np.all(np.isfinite([v for k in res for v in res[k]])))
    return out
