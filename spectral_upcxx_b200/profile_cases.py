"""Small, fixed workloads for profiling the kernels under ncu.

    python -m spectral_upcxx_b200.profile_cases ns128|ns256|ns256r|ns256d|ens|closure64|mlp|misc

Each case builds its inputs on the device, runs a few steps of one path and
exits; sizes keep every case to a few GB of device memory so that a full ncu
capture of one launch ends in seconds.  SNS_GRAPH=0 in the environment keeps
the stepper's launches direct (one kernel per launch in the profile).  The
stepper cases tune their plan first and run the profiled steps inside the NVTX
range "profiled" (ncu --nvtx --nvtx-include "profiled/").
"""
from __future__ import annotations

import sys

import numpy as np
import torch

from . import NSEnsemble, NSStepper, Tracers, curl, ENS_EAGER
from . import ops
from . import _native as N
from . import closure as CL
from . import ic


def run(case: str) -> None:
    dev = torch.device("cuda", 0)
    if case.startswith("ns"):
        # a trailing r: the real-field stepper (half spectrum); d: complex128.
        # The plan is tuned, as the benchmark's is.
        real = case.endswith("r")
        dtype = torch.complex128 if case.endswith("d") else torch.complex64
        n = int(case[2:].rstrip("rd"))
        V0 = [x.to(dtype) for x in ic.solenoidal_spectrum_hat(n, 1, dev)]
        st = NSStepper((n, n, n), 1 / 400, 5e-4, dtype, device=dev, real=real, tune=True)
        st.bootstrap(V0, curl(V0))
        st.step(1)
        # the steps to profile, inside an NVTX range ("profiled/" for ncu --nvtx-include)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("profiled")
        st.step(2)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
    elif case == "ens":
        # the ensemble benchmark's boxes, untuned tiles, eager stage launches
        shapes = [(32, 32, 32)] * 32 + [(64, 64, 64)] * 24 + [(128, 128, 128)] * 8
        nus = list(np.geomspace(1 / 800, 1 / 100, len(shapes)))
        ens = NSEnsemble(shapes, nus, 1e-3, torch.complex64, tune=False, device=dev)
        for b, s in enumerate(shapes):
            V = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(s[0], 50 + b, dev)]
            ens.set_state(b, V, [torch.zeros_like(v) for v in V])
        ens.step(2, ENS_EAGER)
    elif case == "closure64":
        n = 64
        V0 = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(n, 3, dev)]
        m = CL.MLPModel.init(0, s_in=0.4, s_out=1e-3, device=dev)
        st = NSStepper((n, n, n), 1 / 400, 5e-4, torch.complex64, device=dev)
        st.set_closure(N.SNS_CLOSURE_MLP, mlp=m.packed, kc=21)
        st.bootstrap(V0, curl(V0))
        st.step(2)
    elif case == "mlp":
        m = CL.MLPModel.init(0, s_in=1.0, s_out=1.0, device=dev)
        M = 1 << 20
        X = torch.randn((M, 16), device=dev)
        X[:, 9:] = 0
        X = X.to(torch.bfloat16)
        t = torch.rand(M, device=dev)
        m.infer(X)
        m.gradient(X, t, batch=M)
        m.adam(1e-3)
    elif case == "misc":
        # the kernels outside the steppers, each launched once in this order:
        # 3D FFT forward + inverse at 128^3 (cluster plane pass + z pass) and
        # 256^3 (three line passes each), tracer particles, the eager
        # operators at 128^3, the closure data kernels (256^3 -> 64^3), Adam
        g = torch.Generator(device=dev).manual_seed(5)
        for n in (128, 256):
            x = torch.randn((n, n, n), device=dev, generator=g, dtype=torch.complex64)
            ops.forward(x)
            ops.inverse(x)
            del x
        u = [torch.randn((256, 256, 256), device=dev, generator=g, dtype=torch.complex64)
             for _ in range(3)]
        tr = Tracers.uniform(1 << 20, seed=1, device=dev)
        tr.move(u, 1e-3)
        del u
        V = [torch.randn((128, 128, 128), device=dev, generator=g, dtype=torch.complex64)
             for _ in range(3)]
        gr = ops.gradient(V[0])
        w = ops.curl(V)
        cr = ops.cross(V, w)
        dv = ops.divergence(V)
        ops.laplacian_inverse(dv)
        ops.average(dv)
        del gr, w, cr, dv, V
        Vf = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(256, 2, dev)]
        Vc = CL.truncate(Vf, 64, 21)
        CL.pad(Vc, 256)
        CL.sgs_sample(Vf, 64, 21, 1.0)
        CL.spectrum(Vc)
        m = CL.MLPModel.init(0, s_in=1.0, s_out=1.0, device=dev)
        m.adam(1e-3)
    else:
        raise SystemExit(f"unknown case {case}")
    torch.cuda.synchronize()
    print("ok", case)


if __name__ == "__main__":
    run(sys.argv[1] if len(sys.argv) > 1 else "ns128")
