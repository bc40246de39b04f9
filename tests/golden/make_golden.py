"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs the reference's own src/Scalar.cpp / Vector.cpp / Operators.cpp (built
in place by ``make -C oracle ref`` against the project's UPC++ and FFTW shims)
on small seeded inputs and stores inputs and outputs as .npz files.  Needs the
reference tree (its path from $SNS_REFERENCE or BASELINE.json's
reference_path); the fixtures are committed so the tests do not.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from spectral_upcxx_b200 import ic  # noqa: E402


def main():
    import __graft_entry__
    tree = __graft_entry__.reference_tree()
    if tree is None:
        sys.exit("the reference source tree is needed: set SNS_REFERENCE")
    O.build(ref=tree)
    O.ref(True).ref_set_threads(1)
    O.ref(False).ref_set_threads(1)
    out = {}

    # 3D transforms: Scalar::forward with and without ZERO, Scalar::inverse
    for shape, seed in [((8, 8, 8), 11), ((4, 8, 16), 12)]:
        f = ic.uniform_complex(shape, seed)
        tag = "x".join(str(s) for s in shape[::-1])
        out[f"fft_{tag}_in"] = f
        out[f"fft_{tag}_forward_zero"] = O.ref_forward(f, zero=True)
        out[f"fft_{tag}_forward_raw"] = O.ref_forward(f, zero=False)
        out[f"fft_{tag}_inverse"] = O.ref_inverse(f)
    np.savez_compressed(os.path.join(HERE, "fft.npz"), **out)

    # operators on a seeded Fourier vector (8^3)
    out = {}
    n = 8
    v = [O.ref_forward(ic.uniform_complex((n, n, n), 20 + d)) for d in range(3)]
    w = [O.ref_forward(ic.uniform_complex((n, n, n), 30 + d)) for d in range(3)]
    L = O.ref(True)
    for d in range(3):
        out[f"v{d}"] = v[d]
        out[f"w{d}"] = w[d]
    g = [np.empty_like(v[0]) for _ in range(3)]
    L.ref_gradient(O._ptr(v[0]), O._ptr(g[0]), O._ptr(g[1]), O._ptr(g[2]), n, n, n)
    for d in range(3):
        out[f"grad{d}"] = g[d]
    lap = np.empty_like(v[0])
    L.ref_laplacian(O._ptr(v[0]), O._ptr(lap), n, n, n)
    out["lap"] = lap
    il = v[0].copy()
    L.ref_laplacian_inverse(O._ptr(il), 0.0, 1.0, n, n, n)
    out["ilap_0_1"] = il
    il = v[0].copy()
    L.ref_laplacian_inverse(O._ptr(il), 1.0, -0.25, n, n, n)
    out["ilap_1_m0.25"] = il
    c = [np.empty_like(v[0]) for _ in range(3)]
    L.ref_curl(O._ptr3(v), O._ptr3(c), n, n, n)
    for d in range(3):
        out[f"curl{d}"] = c[d]
    dv = np.empty_like(v[0])
    L.ref_divergence(O._ptr3(v), O._ptr(dv), n, n, n)
    out["div"] = dv
    vl = [np.empty_like(v[0]) for _ in range(3)]
    L.ref_vlaplacian(O._ptr3(v), O._ptr3(vl), n, n, n)
    for d in range(3):
        out[f"vlap{d}"] = vl[d]
    cr = [np.empty_like(v[0]) for _ in range(3)]
    L.ref_cross(O._ptr3(v), O._ptr3(w), O._ptr3(cr), n, n, n)
    for d in range(3):
        out[f"cross{d}"] = cr[d]
    out["average_v0"] = np.array(L.ref_average(O._ptr(v[0]), n, n, n))
    np.savez_compressed(os.path.join(HERE, "operators.npz"), **out)

    # the ns.cpp integrator: Taylor-Green (nu = 0.01) and ns.cpp's own vortex
    # tubes (nu = 1e-3), 16^3, dt = 1e-3, 5 steps
    n, steps = 16, 5
    out = {}
    tg = ic.taylor_green(n)
    V0 = [O.ref_forward(c) for c in tg]
    w0 = O.curl(V0)
    r = O.ref_ns_run(V0, w0, 0.01, 1e-3, steps)
    for d in range(3):
        out[f"tg_V0_{d}"] = V0[d]
        out[f"tg_omega0_{d}"] = w0[d]
        out[f"tg_V1_{d}"] = r["V1"][d]
        out[f"tg_cross0_{d}"] = r["cross0"][d]
    out["tg_div_avgs"] = r["div_avgs"]
    V0, w0 = O.ref_ns_vortex_ic(n)
    r = O.ref_ns_run(V0, w0, 1e-3, 1e-3, steps)
    for d in range(3):
        out[f"vx_V0_{d}"] = V0[d]
        out[f"vx_omega0_{d}"] = w0[d]
        out[f"vx_V1_{d}"] = r["V1"][d]
        out[f"vx_cross0_{d}"] = r["cross0"][d]
    out["vx_div_avgs"] = r["div_avgs"]
    out["steps"] = np.array(steps)
    np.savez_compressed(os.path.join(HERE, "ns16.npz"), **out)
    for fn in ("fft.npz", "operators.npz", "ns16.npz"):
        print(fn, os.path.getsize(os.path.join(HERE, fn)), "bytes")


if __name__ == "__main__":
    main()
