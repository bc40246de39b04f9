#!/usr/bin/env python
"""Benchmark: pseudo-spectral NS steps/s at 256^3 (FP32 bulk, FP64
reductions) on B200, with the 3D-FFT GB/s and the FP64 step as secondary
figures.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]
                    [--workload ns256_fp32|ns256_fp64|fft256_c64|fft256_c128|...]

A step is one fused NS step (exec/ns.cpp:167-217) of the stepper state that
stays in HBM; `value` counts steps of all ranks per second (independent
replicas, one per GPU, no collectives).  The 12 resident fields
(1.6 GB at 256^3 complex64) exceed the 126 MB L2, so every step streams from
HBM without a flush.  `e2e` runs the same job through the C-ABI from pinned
host buffers: upload of the initial fields, bootstrap, K steps each followed
by the divergence-monitor read (ns.cpp:210), download of the final velocity.

`--impl reference` times the reference's own CPU code (src/*.cpp built in
place against the project's FFTW/UPC++ shims, oracle/_ref) on the host cores.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "NS steps/s @256^3 FP32 (3D FFT GB/s secondary)"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes of each pass of the fused step, in units of one field
# (N^3 elements): the bytes it must read and write once.
PASSES = {
    5: (["K1 z-inverse+curl", "K2 y-inverse x6", "K3 x-inv+cross+x-fwd", "K4 y-forward x3",
         "K5 z-forward+update"], [3 + 6, 6 + 6, 6 + 3, 3 + 3, 9 + 6]),
    3: (["K1 z-inverse+curl", "K234 xy %s (y-inv x6, x cross, y-fwd x3)",
         "K5 z-forward+update"], [3 + 6, 6 + 3, 9 + 6]),
}


def pass_names(npasses, plan):
    """Names of the timed passes; the xy phase is named by the plan's mode.
    A plan whose update pass carries the next step's K1 ("(+K1") runs K1 in
    its first step only: the update pass then also writes the six z-inverted
    fields (9 + 6 + 6) and K1's steady-state share is empty."""
    names, fields = PASSES[npasses]
    mode = "cluster" if "xy=cluster" in plan else "dataflow" if "xy=dataflow" in plan else "slabs"
    names = [nm % mode if "%s" in nm else nm for nm in names]
    if "(+K1" in plan:
        names = names[:-1] + ["K5+K1 z-forward+update+z-inverse+curl"]
        fields = [0] + list(fields[1:-1]) + [fields[-1] + 6]
    return names, fields
STEP_FIELDS = 30  # 9 FFTs x 2 + 12 for the spectral update: 30 N^3 S per step

# DRAM bytes (read + write) per launch of each pass at 256^3 complex64 with the
# tuned plan, from the one-kernel ncu captures summarised in
# profiles/ns_step_256_c64_launches.md (K1 and K2: their TMA-staged forms).
NCU_TRAFFIC = {
    ("ns256_fp32", "K1 z-inverse+curl"): (404 + 773) * 1e6,
    ("ns256_fp32", "K2 y-inverse x6"): (810 + 749) * 1e6,
    ("ns256_fp32", "K3 x-inv+cross+x-fwd"): (805 + 359) * 1e6,
    ("ns256_fp32", "K4 y-forward x3"): (403 + 341) * 1e6,
    ("ns256_fp32", "K5 z-forward+update"): (1208 + 752) * 1e6,
}

WORKLOADS = {
    "ns256_fp32": dict(kind="ns", n=256, prec="c64"),
    # the same step on the real-field stepper (half spectrum, R2C/C2R along x)
    "ns256_fp32_real": dict(kind="ns", n=256, prec="c64", real=True),
    "ns256_fp64": dict(kind="ns", n=256, prec="c128"),
    "ns128_fp32": dict(kind="ns", n=128, prec="c64"),
    "ns64_fp64": dict(kind="ns", n=64, prec="c128"),
    "fft128_c64": dict(kind="fft", n=128, prec="c64"),
    "fft256_c64": dict(kind="fft", n=256, prec="c64"),
    "fft512_c64": dict(kind="fft", n=512, prec="c64"),
    "fft128_c128": dict(kind="fft", n=128, prec="c128"),
    "fft256_c128": dict(kind="fft", n=256, prec="c128"),
    "fft512_c128": dict(kind="fft", n=512, prec="c128"),
    "ens_64boxes_32_64_128": dict(kind="ens", n=128, prec="c64"),
    "les64_closure_dns256": dict(kind="closure", n=256, prec="c64"),
}
# learned closure: 256^3 DNS (nu = 1/400, dt = 5e-4 as the plain benchmark)
# filtered at kc = 21 onto 64^3; training snapshots every 5 steps of 2000 from
# 5 seeds (2000 snapshots), evaluation on 3 held-out seeds over 2000 steps
CLOSURE = dict(nf=256, nc=64, kc=21, train_seeds=[101, 102, 103, 104, 105],
               eval_seeds=[201, 202, 203], steps=2000, every=5, train_steps=3000,
               batch=65536, lr=2e-3, cs=0.17, coarse_dt_factor=4)
# batched ensemble: 32 boxes of 32^3, 24 of 64^3 and 8 of 128^3, each with its
# own spectrum-seeded field and nu log-uniform in [1/800, 1/100].  dt = 1e-3:
# at the stated 2e-3 the AB2/CN scheme blows up in the 128^3 boxes of smallest
# nu within about 200 steps (3 of 64 boxes non-finite after 205 steps), as it
# does in FP64 at 128^3 and 256^3
ENS_BOXES = [(32, 32), (64, 24), (128, 8)]
ENS_DT = 1e-3
ENS_NU_RANGE = (1.0 / 800, 1.0 / 100)
ENS_STAGES = ["S1 z-inverse+curl", "S2 y-inverse x6", "S3 x-inv+cross+x-fwd", "S4 y-forward x3",
              "S5 z-forward+update"]
# 256^3 spectrum-seeded run: nu = 1/400; dt = 5e-4 because dt = 2e-3 makes the reference's
# AB2/CN scheme diverge at 256^3 (FP64 energy -> NaN within 75 steps)
NU, DT = 1.0 / 400, 5e-4


def peaks():
    try:
        with open(PEAKS_FILE) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def bf16_peak():
    """Dense bf16 TFLOP/s: measured burst figure, else the fallback."""
    try:
        with open(PEAKS_FILE) as f:
            return float(json.load(f)["bf16_tflops"]), "measured"
    except Exception:
        return 1590.0, "fallback"


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """SM clock and throttle reasons sampled during a window: NVML every 2 ms
    from a thread (so even a window of a few milliseconds holds samples), or
    nvidia-smi every 100 ms where NVML cannot be loaded.  Reads only."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_index: int, device=None):
        self.gpu = gpu_index
        self.device = device
        self.samples = []  # (time, sm_mhz, max_mhz, set of reason names)
        self.proc = None
        self.nvml = None
        self.stop_flag = threading.Event()
        self.thread = None
        self.t0 = self.t1 = None

    def _nvml_handle(self):
        import pynvml as N
        N.nvmlInit()
        try:  # the device this process runs on, matched by PCI bus id
            import torch
            p = torch.cuda.get_device_properties(self.device or 0)
            bus = f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
            return N, N.nvmlDeviceGetHandleByPciBusId(bus.encode())
        except Exception:
            return N, N.nvmlDeviceGetHandleByIndex(self.gpu)

    def start(self):
        self.stop_flag.clear()
        try:
            N, h = self._nvml_handle()
            bits = {"hw_slowdown": N.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": N.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": N.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": N.nvmlClocksEventReasonSwPowerCap}
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
            self.nvml = (N, h, bits, mx)
            self.thread = threading.Thread(target=self._nvml_loop, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except FileNotFoundError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._smi_loop, daemon=True)
        self.thread.start()

    def _nvml_loop(self):
        N, h, bits, mx = self.nvml
        while not self.stop_flag.is_set():
            try:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.time(), float(sm), float(mx),
                                     {k for k, b in bits.items() if r & b}))
            except Exception:
                pass
            time.sleep(0.002)

    def _smi_loop(self):
        def num(x):
            try:
                return float(x)
            except ValueError:
                return None
        for line in self.proc.stdout:
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9 or num(p[1]) is None:
                continue
            reasons = {k for k, v in zip(self.NAMES, p[5:9])
                       if v.lower() in ("active", "1", "yes")}
            self.samples.append((time.time(), num(p[1]), num(p[2]), reasons))

    def window(self, t0, t1):
        self.t0, self.t1 = t0, t1

    def stop(self):
        self.stop_flag.set()
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=5)

    def summary(self):
        if self.nvml is None and self.proc is None:
            return None
        inwin = [s for s in self.samples
                 if self.t0 is not None and self.t0 <= s[0] <= self.t1]
        used = inwin if inwin else self.samples
        if not used:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        reasons = set()
        for s in used:
            reasons |= s[3]
        return {"sm_mhz": statistics.median(s[1] for s in used),
                "sm_max_mhz": max(s[2] for s in used), "reasons": sorted(reasons),
                "samples": len(used), "in_timed_window": bool(inwin),
                "source": "nvml 2 ms" if self.nvml is not None else "nvidia-smi 100 ms"}


# ---------------------------------------------------------------- helpers
def make_collectives(world, device):
    """barrier() and max_over_ranks(x) over the initialised process group
    (any backend; no-ops for one rank).  Timings are taken per rank on the
    device and the job's time is the slowest rank's."""
    import torch

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(x):
        if world == 1:
            return x
        import torch.distributed as dist
        t = torch.tensor([x], dtype=torch.float64, device=device)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return t.item()

    return barrier, max_over_ranks


def whole_job_rate(world, units_per_rank, ms):
    """Units of all replicas per second over the slowest rank's time."""
    return world * units_per_rank / (ms / 1e3)


def dist_setup(args):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def initial_velocity_hat(n, seed):
    """The 256^3 benchmark input: spectrum-seeded solenoidal field, Fourier, Nyquist zeroed."""
    from spectral_upcxx_b200 import ic
    u = ic.solenoidal_spectrum(n, seed=seed)
    h = n // 2
    out = []
    for c in u:
        f = np.fft.fftn(c)
        f[h, :, :] = 0
        f[:, h, :] = 0
        f[:, :, h] = 0
        out.append(f)
    return out


# ---------------------------------------------------------------- CPU side
def cpu_ns_sample(n, V1, w1, c0, budget_s=25.0, max_steps=1):
    """Time the reference's own ns.cpp loop body on the host cores."""
    from oracle import pyoracle as O
    cores = os.cpu_count() or 1
    V = [np.ascontiguousarray(x, dtype=np.complex128) for x in V1]
    W = [np.ascontiguousarray(x, dtype=np.complex128) for x in w1]
    Cc = [np.ascontiguousarray(x, dtype=np.complex128) for x in c0]
    if O.have_ref():
        kind = "reference"
        O.ref(True).ref_set_threads(cores)
        secs, steps = 0.0, 0
        while steps < max_steps and secs < budget_s:
            secs += O.ref_ns_steps(V, W, Cc, NU, DT, 1)
            steps += 1
    else:
        kind = "port"
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
        steps = 1
        secs = O.port_ns_seconds(V, W, Cc, NU, DT, 1)
    return {"value": steps / secs, "unit": "steps/s", "cores": cores, "kind": kind,
            "sample": f"{steps} NS step(s) of the {n}^3 complex128 exec/ns.cpp loop body "
                      f"({secs:.2f} s), OpenMP over {cores} host threads"}


def cpu_fft_sample(n, budget_s=20.0):
    from oracle import pyoracle as O
    from spectral_upcxx_b200 import ic
    cores = os.cpu_count() or 1
    f = ic.uniform_complex((n, n, n), 0)
    if O.have_ref():
        kind = "reference"
        L = O.ref(False)
        L.ref_set_threads(cores)
        secs = L.ref_fft_roundtrip(O._ptr(f), n, n, n, 1)
    else:
        kind = "port"
        t0 = time.perf_counter()
        O.inverse(O.forward(f, zero=False))
        secs = time.perf_counter() - t0
    gbs = 4 * n ** 3 * 16 / secs / 1e9
    return {"value": gbs, "unit": "GB/s", "cores": cores, "kind": kind,
            "sample": f"1 forward+inverse 3D FFT of {n}^3 complex128 (exec/fft.cpp), "
                      f"{secs:.2f} s"}


def _curl_np(Vh, n):
    k = _k1d(n)
    KZ, KY, KX = np.meshgrid(k, k, k, indexing="ij")
    return [1j * (KY * Vh[2] - KZ * Vh[1]), 1j * (KZ * Vh[0] - KX * Vh[2]),
            1j * (KX * Vh[1] - KY * Vh[0])]


def cpu_ens_sample():
    """The reference's ns.cpp loop body on the host cores, one warm-up and one
    timed step per box size, weighted by the ensemble's box counts."""
    from oracle import pyoracle as O
    cores = os.cpu_count() or 1
    have = O.have_ref()
    if have:
        O.ref(True).ref_set_threads(cores)
    else:
        os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    per = {}
    for n, _ in ENS_BOXES:
        Vh = initial_velocity_hat(n, 1)
        w = _curl_np(Vh, n)
        c0 = [np.zeros_like(Vh[0]) for _ in range(3)]
        run = (lambda: O.ref_ns_steps(Vh, w, c0, NU, ENS_DT, 1)) if have else \
            (lambda: O.port_ns_seconds(Vh, w, c0, NU, ENS_DT, 1))
        run()
        per[n] = run()
    boxes = sum(c for _, c in ENS_BOXES)
    secs = sum(c * per[n] for n, c in ENS_BOXES)
    return {"value": boxes / secs, "unit": "box-steps/s", "cores": cores,
            "kind": "reference" if have else "port",
            "sample": "1 timed complex128 exec/ns.cpp loop-body step per box size (" +
                      ", ".join(f"{n}^3: {per[n]:.3f} s" for n, _ in ENS_BOXES) +
                      f") after 1 warm-up, weighted by the box counts, {cores} host threads"}


# ---------------------------------------------------------------- reference arm
def run_reference(args, rank, world):
    if rank != 0:
        return 0
    from oracle import pyoracle as O
    wl = WORKLOADS[args.workload]
    n = wl["n"]
    cores = os.cpu_count() or 1
    if wl["kind"] == "ens":
        cb = cpu_ens_sample()
        line = {
            "impl": "reference", "metric": "NS ensemble box-steps/s (32x32^3 + 24x64^3 + 8x128^3)",
            "value": cb["value"], "unit": cb["unit"], "n_gpus": world, "steps": 1, "warmup": 1,
            "ms_per_step": 1000.0 * sum(c for _, c in ENS_BOXES) / cb["value"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded)",
            "config": {"workload": "ens_64boxes_32_64_128: boxes run one after another by the reference "
                                   "loop body", "dt": ENS_DT},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": cb["unit"], "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return 0
    if wl["kind"] == "ns":
        Vh = initial_velocity_hat(n, 1)
        k = _k1d(n)
        KZ, KY, KX = np.meshgrid(k, k, k, indexing="ij")
        w = [1j * (KY * Vh[2] - KZ * Vh[1]), 1j * (KZ * Vh[0] - KX * Vh[2]),
             1j * (KX * Vh[1] - KY * Vh[0])]
        c0 = [np.zeros_like(Vh[0]) for _ in range(3)]
        have = O.have_ref()
        if have:
            O.ref(True).ref_set_threads(cores)
        step = (lambda: O.ref_ns_steps(Vh, w, c0, NU, DT, 1)) if have else \
            (lambda: O.port_ns_seconds(Vh, w, c0, NU, DT, 1))
        first = step()  # warm-up (page-in, plan caches)
        budget = 150.0
        steps = max(1, min(args.steps, int(budget / max(first, 1e-9))))
        secs = sum(step() for _ in range(steps))
        value = steps / secs
        unit = "steps/s"
        sample = (f"{steps} timed NS step(s) of {n}^3 complex128 (exec/ns.cpp loop body) after "
                  f"1 warm-up step, {cores} host threads")
        dtype = "f64"
    else:
        f = __import__("spectral_upcxx_b200.ic", fromlist=["ic"]).uniform_complex((n, n, n), 0)
        if O.have_ref():
            L = O.ref(False)
            L.ref_set_threads(cores)
            L.ref_fft_roundtrip(O._ptr(f), n, n, n, 1)
            steps = max(1, min(args.steps, 10))
            secs = sum(L.ref_fft_roundtrip(O._ptr(f), n, n, n, 1) for _ in range(steps))
        else:
            steps = 1
            t0 = time.perf_counter()
            O.inverse(O.forward(f, zero=False))
            secs = time.perf_counter() - t0
        value = 4 * n ** 3 * 16 * steps / secs / 1e9
        unit = "GB/s"
        sample = f"{steps} forward+inverse 3D FFT(s) of {n}^3 complex128 (exec/fft.cpp)"
        dtype = "f64"
    kind = "reference" if O.have_ref() else "port"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit, "n_gpus": world,
        "steps": steps, "warmup": 1, "ms_per_step": 1000.0 / value if unit == "steps/s" else None,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
        "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "grid": f"{n}^3", "nu": NU, "dt": DT,
                   "backend": "reference src/*.cpp + project FP64 FFT behind the FFTW API"
                   if kind == "reference" else "CPU oracle port"},
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def _k1d(n):
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n).astype(np.float64)


# ---------------------------------------------------------------- B200 arm
def run_b200(args, rank, world, local):
    import torch
    import spectral_upcxx_b200 as S

    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
    S.lib()
    wl = WORKLOADS[args.workload]
    n = wl["n"]
    dtype = torch.complex64 if wl["prec"] == "c64" else torch.complex128
    esz = 8 if wl["prec"] == "c64" else 16
    real = wl.get("real", False)
    # stored field: the half spectrum of a real-field run
    field_bytes = n ** 3 * esz // (2 if real else 1)
    hbm, peak_src = peaks()
    stream = torch.cuda.Stream(dev)
    clocks = ClockSampler(local, dev)

    barrier, max_over_ranks = make_collectives(world, dev)

    result = {}
    if wl["kind"] == "ns":
        Vh = initial_velocity_hat(n, 1 + rank)
        with torch.cuda.stream(stream):
            Vd = [torch.from_numpy(x).to(dev, dtype) for x in Vh]
            wd = S.curl(Vd)
            st = S.NSStepper((n, n, n), NU, DT, dtype, device=dev, real=real, tune=True)
            st.bootstrap(Vd, wd)
            st.step(args.warmup)
        stream.synchronize()
        clocks.start()
        time.sleep(0.3)
        barrier()
        stream.synchronize()
        st.profile(True)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t_wall0 = time.time()
        with torch.cuda.stream(stream):
            e0.record(stream)
            st.step(args.steps)
            e1.record(stream)
        stream.synchronize()
        t_wall1 = time.time()
        barrier()
        clocks.window(t_wall0, t_wall1)
        ms = e0.elapsed_time(e1)
        ms = max_over_ranks(ms)
        passes = st.pass_times()
        st.profile(False)
        time.sleep(0.2)
        clocks.stop()
        stats = st.stats()
        value = whole_job_rate(world, args.steps, ms)
        # dominant kernel
        avg = [tot / max(cnt, 1) for tot, cnt in passes]
        plan = st.describe()
        PASS_NAMES, PASS_FIELDS = pass_names(len(avg), plan)
        top = int(np.argmax(avg))
        alg = PASS_FIELDS[top] * field_bytes
        achieved = alg / (avg[top] / 1e3) / 1e9
        share = [a / sum(avg) for a in avg]
        step_ms = ms / args.steps
        result.update(
            metric=METRIC, value=value, unit="steps/s", ms_per_step=step_ms,
            dtype="fp32 bulk + fp64 reductions" if esz == 8 else "fp64",
            roofline={"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                      "frac": achieved / hbm,
                      "traffic": NCU_TRAFFIC.get((args.workload, PASS_NAMES[top])),
                      "kernel": PASS_NAMES[top],
                      "algorithmic_bytes_per_launch": alg,
                      "peak_source": f"{peak_src} hbm_gbs",
                      "step": {"algorithmic_bytes": STEP_FIELDS * field_bytes,
                               "achieved_gbs": STEP_FIELDS * field_bytes / (step_ms / 1e3) / 1e9,
                               "frac": STEP_FIELDS * field_bytes / (step_ms / 1e3) / 1e9 / hbm,
                               "half_spectrum": real},
                      "passes": [{"name": nm, "ms": a, "share": sh,
                                  "gbs": PASS_FIELDS[i] * field_bytes / (a / 1e3) / 1e9}
                                 for i, (nm, a, sh) in enumerate(zip(PASS_NAMES, avg, share))
                                 if PASS_FIELDS[i] > 0]},
            gpu_launches=args.steps * st.launches_per_step(),
            diagnostics=stats)
        # ---- e2e through the C-ABI from pinned host buffers
        host_V = [torch.from_numpy(x).to(dtype).pin_memory() for x in Vh]
        w_np = [w.cpu() for w in wd]
        host_w = [w.pin_memory() for w in w_np]
        out_V = [torch.empty((n, n, n), dtype=dtype).pin_memory() for _ in range(3)]
        st.close()
        # the caller's device buffers exist before the timed region; Vd/wd are
        # overwritten from the pinned host copies inside it
        fin = [torch.empty((n, n, n), dtype=dtype, device=dev) for _ in range(3)]
        e2e_steps = args.steps
        monitor = torch.zeros((e2e_steps, 4), dtype=torch.float64).pin_memory()
        barrier()
        torch.cuda.synchronize()
        s0 = torch.cuda.Event(enable_timing=True)
        s1 = torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            s0.record(stream)
            for a, b in zip(Vd + wd, host_V + host_w):
                a.copy_(b, non_blocking=True)
            st2 = S.NSStepper((n, n, n), NU, DT, dtype, device=dev, real=real, tune=True)
            st2.bootstrap(Vd, wd)
            for t in range(e2e_steps):
                st2.step(1)
                # ns.cpp:206-210 monitor of every step, read back to pinned host
                # memory without stalling the stream
                st2.stats_async(monitor[t])
            st2.velocity(fin)
            for a, b in zip(out_V, fin):
                a.copy_(b, non_blocking=True)
            s1.record(stream)
        stream.synchronize()
        e2e_ms = max_over_ranks(s0.elapsed_time(s1))
        assert S._native.lib().sns_ns_check(st2.h) == 0
        divs = monitor[:, 0].tolist()  # noqa: F841 (the monitor values, read after the run)
        st2.close()
        result["e2e"] = {
            "value": world * e2e_steps / (e2e_ms / 1e3), "unit": "steps/s",
            "h2d_bytes_per_step": 6 * field_bytes / e2e_steps,
            "d2h_bytes_per_step": (3 * field_bytes + 32 * e2e_steps) / e2e_steps,
            "includes": "upload of V0/omega0 from pinned host, creation of the (tuned) stepper, "
                        "bootstrap (ns.cpp:132-153), K steps each with its diagnostics "
                        "(div.average() of ns.cpp:210, energy, enstrophy, max |div|) copied to "
                        "pinned host memory without a stall, download of V1"}
        del Vd, wd, fin
        torch.cuda.empty_cache()
        # ---- secondary figures (untimed for the headline)
        if not args.no_secondary and rank == 0:
            sec = secondary(S, torch, dev, stream, n, hbm)
            key = "closure64_mlp_steps_per_s"
            if key in sec and not real and n == CLOSURE["nf"]:
                # the coarse closure run against this DNS step (target 20x)
                sec["closure64_mlp_vs_dns256_step_ratio"] = sec[key] / (1e3 / step_ms)
                # per unit of simulated time: the coarse run is evaluated at
                # coarse_dt_factor x the DNS step (its spectrum errors at that
                # step are in the les64_closure_dns256 workload's line)
                sec["closure64_mlp_vs_dns256_simulated_time_ratio"] = (
                    sec["closure64_mlp_vs_dns256_step_ratio"] * CLOSURE["coarse_dt_factor"])
            result["secondary"] = sec
        # ---- CPU baseline (rank 0, N = 1 only)
        if rank == 0 and world == 1 and not args.no_cpu:
            c0 = [np.zeros_like(Vh[0]) for _ in range(3)]
            k = _k1d(n)
            KZ, KY, KX = np.meshgrid(k, k, k, indexing="ij")
            w = [1j * (KY * Vh[2] - KZ * Vh[1]), 1j * (KZ * Vh[0] - KX * Vh[2]),
                 1j * (KX * Vh[1] - KY * Vh[0])]
            result["cpu_baseline"] = cpu_ns_sample(n, Vh, w, c0)
            if "secondary" in result:
                # the standalone 3D FFT on the same host cores (exec/fft.cpp)
                result["secondary"]["fft_cpu_baseline"] = cpu_fft_sample(n)
        cfg = {"workload": f"{args.workload}: plain NS step {n}^3" +
                           (" on the real-field stepper (half spectrum)" if real else "") +
                           ", spectrum-seeded solenoidal field (seed 1+rank), nu=1/400, dt=5e-4 "
                           "(2e-3 diverges in FP64 as well)",
               "grid": f"{n}^3", "precision": wl["prec"], "parallelism": f"replicas x{world}",
               "plan": plan,
               "l2": "no flush: 12 resident fields (%.2f GB) exceed the 126 MB L2" % (
                   12 * field_bytes / 1e9)}
    elif wl["kind"] == "closure":
        result.update(closure_bench(S, torch, dev, args, world, rank, hbm, peak_src, clocks))
        cfg = {"workload": "les64_closure_dns256: %d^3 DNS (nu=1/400, dt=5e-4) sharp-spectral filtered "
                           "at kc=%d onto %d^3; MLP 9-64-64-1 trained on %d snapshots of %d "
                           "seeds; %d^3 runs (modes |k| <= kc) of %d held-out seeds over %d "
                           "steps" % (CLOSURE["nf"], CLOSURE["kc"], CLOSURE["nc"],
                                      result["snapshots"], len(CLOSURE["train_seeds"]),
                                      CLOSURE["nc"], len(CLOSURE["eval_seeds"]), CLOSURE["steps"]),
               "precision": "c64 fields, bf16 MLP with fp32 accumulation",
               "parallelism": f"replicas x{world}", "l2": "coarse fields L2-resident by size"}
    elif wl["kind"] == "ens":
        result.update(ens_bench(S, torch, dev, stream, args, world, rank, hbm, peak_src, clocks,
                                barrier, max_over_ranks))
        if rank == 0 and world == 1 and not args.no_cpu:
            result["cpu_baseline"] = cpu_ens_sample()
        cfg = {"workload": "ens_64boxes_32_64_128: 32 boxes of 32^3 + 24 of 64^3 + 8 of 128^3 "
                           "(24,117,248 points), spectrum-seeded solenoidal field per box "
                           "(distinct seeds), nu log-uniform in [1/800, 1/100], dt=1e-3 (2e-3 blows up "
                           "in the 128^3 boxes of smallest nu), complex64",
               "boxes": {f"{n}^3": c for n, c in ENS_BOXES}, "precision": "c64",
               "parallelism": f"replicas x{world}",
               "l2": "no flush: 12 resident fields per box (%.2f GB) exceed the 126 MB L2" % (
                   12 * result["points"] * 8 / 1e9)}
    else:
        result.update(fft_bench(S, torch, dev, stream, n, dtype, esz, args, world, hbm, peak_src,
                                clocks, barrier, max_over_ranks))
        if rank == 0 and world == 1 and not args.no_cpu:
            result["cpu_baseline"] = cpu_fft_sample(n)
        cfg = {"workload": f"{args.workload}: 3D C2C FFT forward+inverse {n}^3 {wl['prec']}, "
                           f"uniform[-1,1) re/im (seeded)",
               "grid": f"{n}^3", "precision": wl["prec"], "parallelism": f"replicas x{world}",
               "plan": "tuned by sns_fft3d_tune (per-axis tile, threads, radix order)",
               "l2": "inputs of %.2f GB per transform vs 126 MB L2" % (field_bytes / 1e9)}
    clk = clocks.summary()
    line = {"metric": result.pop("metric", METRIC), "value": result.pop("value"),
            "unit": result.pop("unit"), "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": result.pop("ms_per_step"),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": result.pop("dtype"), "data": "synthetic (seeded)", "config": cfg}
    if clk is not None:
        line["clocks"] = clk
    line.update(result)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def fft_bench(S, torch, dev, stream, n, dtype, esz, args, world, hbm, peak_src, clocks, barrier,
              max_over_ranks):
    g = torch.Generator(device=dev).manual_seed(1)
    with torch.cuda.stream(stream):
        S.fft3d_tune((n, n, n), dtype, device=dev)
        x = torch.complex(torch.rand((n, n, n), device=dev, generator=g) * 2 - 1,
                          torch.rand((n, n, n), device=dev, generator=g) * 2 - 1).to(dtype)
        for _ in range(args.warmup):
            S.fft3d(x, -1)
            S.fft3d(x, +1, normalise=True)
    stream.synchronize()
    clocks.start()
    time.sleep(0.3)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    with torch.cuda.stream(stream):
        e0.record(stream)
        for _ in range(args.steps):
            S.fft3d(x, -1)
            S.fft3d(x, +1, normalise=True)
        e1.record(stream)
    stream.synchronize()
    t1 = time.time()
    barrier()
    clocks.window(t0, t1)
    ms = max_over_ranks(e0.elapsed_time(e1))
    time.sleep(0.2)
    clocks.stop()
    alg = 4 * n ** 3 * esz
    gbs = world * alg * args.steps / (ms / 1e3) / 1e9
    # six line passes per forward + inverse, each moving 2 N^3 S bytes
    per_pass = 2 * n ** 3 * esz
    achieved = per_pass / (ms / args.steps / 6 / 1e3) / 1e9
    # e2e: pinned host in, pinned host out
    h = x.cpu().pin_memory()
    out = torch.empty_like(h).pin_memory()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    with torch.cuda.stream(stream):
        s0.record(stream)
        for _ in range(args.steps):
            x.copy_(h, non_blocking=True)
            S.fft3d(x, -1)
            S.fft3d(x, +1, normalise=True)
            out.copy_(x, non_blocking=True)
        s1.record(stream)
    stream.synchronize()
    e2e_ms = max_over_ranks(s0.elapsed_time(s1))
    # the tuned plan's TMA-staged passes record any bounded wait that ran out
    from spectral_upcxx_b200 import _native as NN
    NN.call("sns_fft3d_check", C.c_void_p(stream.cuda_stream))
    return {"metric": "3D FFT forward+inverse GB/s", "value": gbs, "unit": "GB/s",
            "ms_per_step": ms / args.steps, "dtype": "fp32" if esz == 8 else "fp64",
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                         "frac": achieved / hbm, "traffic": None,
                         "kernel": "line pass (avg of 6 per fwd+inv)",
                         "algorithmic_bytes_per_launch": per_pass,
                         "peak_source": f"{peak_src} hbm_gbs"},
            "gpu_launches": 6 * args.steps,
            "e2e": {"value": world * alg * args.steps / (e2e_ms / 1e3) / 1e9, "unit": "GB/s",
                    "h2d_bytes_per_step": n ** 3 * esz, "d2h_bytes_per_step": n ** 3 * esz}}


def ens_bench(S, torch, dev, stream, args, world, rank, hbm, peak_src, clocks, barrier,
              max_over_ranks):
    """Batched ensemble: one graph replay per ensemble step (five launches over
    all boxes).  value = box-steps/s of all ranks; the sequential per-box
    stepping of the same ensemble is timed beside it."""
    from spectral_upcxx_b200 import ic
    r = np.random.default_rng(4 + rank)
    shapes = [(n, n, n) for n, c in ENS_BOXES for _ in range(c)]
    lo, hi = np.log(ENS_NU_RANGE[0]), np.log(ENS_NU_RANGE[1])
    nus = list(np.exp(r.uniform(lo, hi, len(shapes))))
    points = int(sum(np.prod(s) for s in shapes))
    esz = 8
    host_ic = []
    with torch.cuda.stream(stream):
        ens = S.NSEnsemble(shapes, nus, ENS_DT, torch.complex64, tune=True, device=dev)
        for b, s in enumerate(shapes):
            Vd = [x.to(torch.complex64) for x in
                  ic.solenoidal_spectrum_hat(s[0], 1000 * (rank + 1) + b, dev)]
            wd = S.curl(Vd)
            ens.bootstrap(b, Vd, wd)
            host_ic.append(([x.cpu().pin_memory() for x in Vd], [x.cpu().pin_memory() for x in wd]))
        ens.step(args.warmup)
    stream.synchronize()
    nb = len(shapes)
    clocks.start()
    time.sleep(0.3)
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    with torch.cuda.stream(stream):
        e0.record(stream)
        ens.step(args.steps, S.ENS_GRAPH)
        e1.record(stream)
    stream.synchronize()
    t1 = time.time()
    barrier()
    clocks.window(t0, t1)
    ms = max_over_ranks(e0.elapsed_time(e1))
    time.sleep(0.2)
    clocks.stop()
    stats = ens.stats()
    finite = sum(1 for s in stats if np.isfinite(s["energy"]))
    # the same ensemble launched stage by stage, and box by box with the single-box kernels
    alt = {}
    k_alt = max(10, args.steps // 10)
    for name, mode in (("eager", S.ENS_EAGER), ("sequential", S.ENS_SEQUENTIAL)):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ens.step(2, mode)
            a0.record(stream)
            ens.step(k_alt, mode)
            a1.record(stream)
        stream.synchronize()
        alt[name] = max_over_ranks(a0.elapsed_time(a1)) / k_alt
    stage_ms = ens.stage_times(20)
    top = int(np.argmax(stage_ms))
    fields = PASSES[5][1]
    alg = fields[top] * points * esz
    achieved = alg / (stage_ms[top] / 1e3) / 1e9
    step_ms = ms / args.steps
    step_bytes = STEP_FIELDS * points * esz
    # e2e through the public API: upload every box's V0/omega0 from pinned host,
    # bootstrap, K steps each followed by the per-box diagnostics read, download V1
    out_V = [[torch.empty(s, dtype=torch.complex64).pin_memory() for _ in range(3)]
             for s in shapes]
    dev_ic = [([torch.empty(s, dtype=torch.complex64, device=dev) for _ in range(3)],
               [torch.empty(s, dtype=torch.complex64, device=dev) for _ in range(3)])
              for s in shapes]
    barrier()
    torch.cuda.synchronize()
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        s0.record(stream)
        for b in range(nb):
            for a, h in zip(dev_ic[b][0] + dev_ic[b][1], host_ic[b][0] + host_ic[b][1]):
                a.copy_(h, non_blocking=True)
            ens.bootstrap(b, dev_ic[b][0], dev_ic[b][1])
        for _ in range(args.steps):
            ens.step(1, S.ENS_GRAPH)
            ens.stats()  # per-box div.average() monitor (ns.cpp:210), D2H + sync
        for b in range(nb):
            for a, v in zip(out_V[b], ens.state(b)["V1"]):
                a.copy_(v, non_blocking=True)
        s1.record(stream)
    stream.synchronize()
    e2e_ms = max_over_ranks(s0.elapsed_time(s1))
    tuning = ens.tuning()
    ens.close()
    del dev_ic
    torch.cuda.empty_cache()
    return {
        "metric": "NS ensemble box-steps/s (32x32^3 + 24x64^3 + 8x128^3)",
        "value": world * nb * args.steps / (ms / 1e3), "unit": "box-steps/s",
        "ms_per_step": step_ms, "dtype": "fp32 bulk + fp64 reductions", "points": points,
        "ensemble_steps_per_s": world * args.steps / (ms / 1e3),
        "modes_ms_per_ensemble_step": {"graph": step_ms, **alt},
        "speedup_vs_sequential": alt["sequential"] / step_ms,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": None, "kernel": ENS_STAGES[top],
                     "algorithmic_bytes_per_launch": alg, "peak_source": f"{peak_src} hbm_gbs",
                     "step": {"algorithmic_bytes": step_bytes,
                              "achieved_gbs": step_bytes / (step_ms / 1e3) / 1e9,
                              "frac": step_bytes / (step_ms / 1e3) / 1e9 / hbm},
                     "stages": [{"name": nm, "ms": t, "gbs": fields[i] * points * esz / (t / 1e3) / 1e9}
                                for i, (nm, t) in enumerate(zip(ENS_STAGES, stage_ms))]},
        "tuning": [{"threads": t, "line_run_cap": w, "persistent": p} for t, w, p in tuning],
        "gpu_launches": args.steps * 5,
        "diagnostics": {"boxes_finite": finite, "boxes": nb,
                        "energy_min": min(s["energy"] for s in stats),
                        "energy_max": max(s["energy"] for s in stats)},
        "e2e": {"value": world * nb * args.steps / (e2e_ms / 1e3), "unit": "box-steps/s",
                "h2d_bytes_per_step": 6 * points * esz / args.steps,
                "d2h_bytes_per_step": (3 * points * esz + 32 * nb * args.steps) / args.steps,
                "includes": "upload of V0/omega0 of every box from pinned host, bootstrap, K graph "
                            "steps each with the per-box diagnostics read, download of every V1"},
    }


def closure_bench(S, torch, dev, args, world, rank, hbm, peak_src, clocks):
    """The 64^3 closure run against filtered 256^3 DNS: dataset from the
    filtered DNS, GPU training, coarse runs judged by the filtered DNS energy
    spectrum.  value = steps/s of the 64^3 MLP-closure run (device time, K
    steps through a CUDA-event window)."""
    from spectral_upcxx_b200 import closure as CL
    from spectral_upcxx_b200 import ic
    c = CLOSURE
    t0 = time.perf_counter()
    calib = {}
    X, nut, w, s_in, snaps = CL.dns_dataset(S, c["nf"], c["nc"], c["kc"], c["train_seeds"], NU,
                                            DT, c["steps"], c["every"], device=dev, calib=calib)
    t_data = time.perf_counter() - t0
    s_out = float((nut * w).mean() / w.mean())
    model = CL.MLPModel.init(0, s_in=s_in, s_out=s_out, device=dev)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    losses = CL.train(model, X, nut, c["train_steps"], c["batch"], c["lr"], weight=w)
    torch.cuda.synchronize()
    t_train = time.perf_counter() - t0
    samples = X.shape[0]
    del X, nut, w
    torch.cuda.empty_cache()
    # output scale and band of the eddy force fitted a posteriori on the first
    # training seed (not held out), at the coarse time step; the same fit for
    # the Smagorinsky constant and band
    cdt = DT * c["coarse_dt_factor"]
    csteps = c["steps"] // c["coarse_dt_factor"]
    t0 = time.perf_counter()
    calib_errs, band = CL.calibrate(S, model, calib, NU, cdt, csteps, c["kc"])
    smag_errs, (smag_band, cs) = CL.calibrate_smagorinsky(S, calib, NU, cdt, csteps, c["kc"])
    t_cal = time.perf_counter() - t0
    # the textbook Smagorinsky (Cs = 0.17 on every mode) as a further baseline
    extra = {"smagorinsky_cs017_all_modes":
             {"csd2": CL.smagorinsky_cs_delta2(c["cs"], c["kc"]), "band": (0.0, 0.0)}}
    res = CL.evaluate(S, model, c["nf"], c["nc"], c["kc"], c["eval_seeds"], NU, DT, c["steps"],
                      cs=cs, device=dev, band=band, smag_band=smag_band, extra=extra)
    # the same runs with the coarse grid at a larger time step (the cutoff kc
    # relaxes the CFL limit), judged at the same physical time
    res_dt = CL.evaluate(S, model, c["nf"], c["nc"], c["kc"], c["eval_seeds"], NU, DT, c["steps"],
                         cs=cs, device=dev, coarse_dt=cdt, band=band, smag_band=smag_band,
                         extra=extra)
    # device-timed steps/s of the coarse MLP run and of the plain coarse run
    nc = c["nc"]
    Vc0 = CL.truncate([x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(
        c["nf"], c["eval_seeds"][0], dev)], nc, c["kc"])
    timing, launches = {}, {}
    for name in ("mlp", "plain"):
        st = S.NSStepper((nc, nc, nc), NU, DT, torch.complex64, device=dev)
        if name == "mlp":
            st.set_closure(S._native.SNS_CLOSURE_MLP, mlp=model.packed, kc=c["kc"])
            st.set_sgs_band(*band)
        else:
            st.set_closure(S._native.SNS_CLOSURE_NONE, kc=c["kc"])
        st.bootstrap(Vc0, S.curl(Vc0))
        st.step(args.warmup)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        if name == "mlp":
            clocks.start()
            time.sleep(0.3)
        tw0 = time.time()
        e0.record()
        st.step(args.steps)
        e1.record()
        torch.cuda.synchronize()
        if name == "mlp":
            clocks.window(tw0, time.time())
            time.sleep(0.2)
            clocks.stop()
        timing[name] = args.steps / (e0.elapsed_time(e1) / 1e3)
        launches[name] = st.launches_per_step()
        st.close()
    # MLP inference throughput on the tensor cores (64^3 points per call)
    Xi = torch.randn((nc ** 3, 16), device=dev).to(torch.bfloat16)
    for _ in range(3):
        model.infer(Xi)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(50):
        model.infer(Xi)
    e1.record()
    torch.cuda.synchronize()
    ms_inf = e0.elapsed_time(e1) / 50
    flops = 9472.0 * nc ** 3
    tpeak, tsrc = bf16_peak()
    achieved = flops / (ms_inf / 1e3) / 1e12
    return {
        "metric": "closure64 steps/s (MLP eddy-viscosity 64^3 run)",
        "value": world * timing["mlp"], "unit": "steps/s", "ms_per_step": 1000.0 / timing["mlp"],
        "dtype": "fp32 fields + bf16/fp32 MLP", "snapshots": snaps,
        "spectrum_error": {"plain": res["plain"], "smagorinsky": res["smagorinsky"],
                           "mlp": res["mlp"],
                           "smagorinsky_cs017_all_modes": res["smagorinsky_cs017_all_modes"],
                           "shells": f"1..{c['kc'] - 1}", "target": 0.05,
                           "held_out_seeds": c["eval_seeds"],
                           "spectra_first_seed": res["spectra_first_seed"]},
        "closure_fit": {"on": f"training seed {c['train_seeds'][0]}, coarse dt {cdt}",
                        "seconds": t_cal,
                        "mlp_band": band, "mlp_output_scale": model.s_out / s_out,
                        "smagorinsky_band": smag_band, "smagorinsky_cs": cs,
                        "mlp_errors": {f"{k[0]}x{k[1]}": v for k, v in calib_errs.items()},
                        "smagorinsky_errors": {f"{k[0]}x{k[1]}": v for k, v in smag_errs.items()}},
        "throughput": {"mlp_coarse_steps_per_s": timing["mlp"],
                       "plain_coarse_steps_per_s": timing["plain"],
                       "dns_steps_per_s": res["dns_steps_per_s"],
                       "ratio_mlp_vs_dns": timing["mlp"] / res["dns_steps_per_s"],
                       "target_ratio": 20.0,
                       "simulated_time_ratio_at_coarse_dt": timing["mlp"] * cdt /
                       (res["dns_steps_per_s"] * DT)},
        "spectrum_error_at_coarse_dt": {"coarse_dt": cdt, "plain": res_dt["plain"],
                                        "smagorinsky": res_dt["smagorinsky"],
                                        "mlp": res_dt["mlp"],
                                        "smagorinsky_cs017_all_modes":
                                        res_dt["smagorinsky_cs017_all_modes"],
                                        "all_finite": res_dt["all_finite"]},
        "training": {"samples": samples, "steps": c["train_steps"], "batch": c["batch"],
                     "seconds": t_train, "dataset_seconds": t_data,
                     "loss_first": losses[0][1], "loss_last": losses[-1][1],
                     "s_in": s_in, "s_out": s_out},
        "roofline": {"bound": "tensor", "kernel": "MLP inference (k_mlp_infer_tc, tcgen05, 64^3 points)",
                     "achieved": achieved, "unit": "TFLOP/s", "peak": tpeak,
                     "frac": achieved / tpeak, "traffic": None,
                     "peak_source": f"{tsrc} bf16_tflops (burst)",
                     "algorithmic_flops_per_launch": flops},
        "gpu_launches": args.steps * launches["mlp"],
    }


def secondary(S, torch, dev, stream, n, hbm):
    """FP64 NS step, the real-field (half-spectrum) FP32 step, tracer-particle
    moves and 3D-FFT GB/s at n^3 (short runs, device events)."""
    out = {}
    Vh = initial_velocity_hat(n, 7)
    for prec, dtype, esz in (("c128", torch.complex128, 16),):
        with torch.cuda.stream(stream):
            Vd = [torch.from_numpy(x).to(dev, dtype) for x in Vh]
            wd = S.curl(Vd)
            st = S.NSStepper((n, n, n), NU, DT, dtype, device=dev, tune=True)
            st.bootstrap(Vd, wd)
            st.step(3)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st.step(20)
            e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / 20
        out[f"ns{n}_{prec}_steps_per_s"] = 1e3 / ms
        out[f"ns{n}_{prec}_step_frac_of_hbm"] = 30 * n ** 3 * esz / (ms / 1e3) / 1e9 / hbm
        st.close()
        del Vd, wd
    # the same benchmark step on the half spectrum of the (real) field, against
    # the same 30 N^3 S unit of the complex step
    with torch.cuda.stream(stream):
        Vd = [torch.from_numpy(x).to(dev, torch.complex64) for x in Vh]
        wd = S.curl(Vd)
        st = S.NSStepper((n, n, n), NU, DT, torch.complex64, device=dev, real=True, tune=True)
        st.bootstrap(Vd, wd)
        st.step(3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        st.step(50)
        e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / 50
    out[f"ns{n}_c64_real_field_steps_per_s"] = 1e3 / ms
    out[f"ns{n}_c64_real_field_frac_of_30N3S"] = 30 * n ** 3 * 8 / (ms / 1e3) / 1e9 / hbm
    st.close()
    del Vd, wd
    # tracer particles: 2^20 particles through an n^3 complex64 velocity
    g = torch.Generator(device=dev).manual_seed(4)
    with torch.cuda.stream(stream):
        u = [torch.randn((n, n, n), device=dev, generator=g, dtype=torch.complex64)
             for _ in range(3)]
        tr = S.Tracers.uniform(1 << 20, seed=1, device=dev)
        for _ in range(3):
            tr.move(u, 1e-3)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(20):
            tr.move(u, 1e-3)
        e1.record(stream)
    stream.synchronize()
    out["particles_2e20_moves_per_s"] = 20 * (1 << 20) / (e0.elapsed_time(e1) / 1e3)
    del u, tr
    for prec, dtype, esz in (("c64", torch.complex64, 8), ("c128", torch.complex128, 16)):
        g = torch.Generator(device=dev).manual_seed(2)
        with torch.cuda.stream(stream):
            S.fft3d_tune((n, n, n), dtype, device=dev)
            x = torch.complex(torch.rand((n, n, n), device=dev, generator=g, dtype=torch.float64),
                              torch.rand((n, n, n), device=dev, generator=g,
                                         dtype=torch.float64)).to(dtype)
            for _ in range(3):
                S.fft3d(x, -1)
                S.fft3d(x, +1, normalise=True)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(10):
                S.fft3d(x, -1)
                S.fft3d(x, +1, normalise=True)
            e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / 10
        S._native.call("sns_fft3d_check", C.c_void_p(stream.cuda_stream))
        out[f"fft{n}_{prec}_fwd_inv_gbs"] = 4 * n ** 3 * esz / (ms / 1e3) / 1e9
        # comparison row only: the same transform pair through cuFFT (torch.fft)
        with torch.cuda.stream(stream):
            for _ in range(3):
                x = torch.fft.ifftn(torch.fft.fftn(x))
            e0.record(stream)
            for _ in range(10):
                x = torch.fft.ifftn(torch.fft.fftn(x))
            e1.record(stream)
        stream.synchronize()
        ms = e0.elapsed_time(e1) / 10
        out[f"cufft{n}_{prec}_fwd_inv_gbs_comparison"] = 4 * n ** 3 * esz / (ms / 1e3) / 1e9
        del x
    torch.cuda.empty_cache()
    # 3D FFT roofline: a forward + inverse pair is six line passes of 2 N^3 S
    # bytes each (12 N^3 S moved against the 4 N^3 S the GB/s figure counts),
    # so the passes' own rate is 3x that figure, against the copy peak
    for prec, esz in (("c64", 8), ("c128", 16)):
        gbs = out[f"fft{n}_{prec}_fwd_inv_gbs"]
        out[f"fft{n}_{prec}_pass_frac_of_hbm"] = gbs * 3 / hbm
    out.update(ensemble_secondary(S, torch, dev, stream, hbm))
    out.update(closure_secondary(S, torch, dev, stream))
    torch.cuda.empty_cache()
    return out


def ensemble_secondary(S, torch, dev, stream, hbm, steps=20):
    """The ensemble workload (32 x 32^3 + 24 x 64^3 + 8 x 128^3 boxes, nu
    log-uniform in [1/800, 1/100], dt = 1e-3) as one graph replay per ensemble
    step with the default tiles (no tuning run), timed over `steps` steps."""
    from spectral_upcxx_b200 import ic
    r = np.random.default_rng(4)
    shapes = [(m, m, m) for m, c in ENS_BOXES for _ in range(c)]
    lo, hi = np.log(ENS_NU_RANGE[0]), np.log(ENS_NU_RANGE[1])
    nus = list(np.exp(r.uniform(lo, hi, len(shapes))))
    points = int(sum(np.prod(x) for x in shapes))
    with torch.cuda.stream(stream):
        ens = S.NSEnsemble(shapes, nus, ENS_DT, torch.complex64, tune=False, device=dev)
        for b, sh in enumerate(shapes):
            Vd = [x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(sh[0], 1000 + b, dev)]
            ens.bootstrap(b, Vd, S.curl(Vd))
        ens.step(3, S.ENS_GRAPH)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ens.step(steps, S.ENS_GRAPH)
        e1.record(stream)
    stream.synchronize()
    ms = e0.elapsed_time(e1) / steps
    finite = sum(1 for x in ens.stats() if np.isfinite(x["energy"]))
    ens.close()
    return {"ens_64boxes_box_steps_per_s": len(shapes) * 1e3 / ms,
            "ens_64boxes_ensemble_steps_per_s": 1e3 / ms,
            "ens_64boxes_step_frac_of_hbm": STEP_FIELDS * points * 8 / (ms / 1e3) / 1e9 / hbm,
            "ens_64boxes_boxes_finite": finite}


def closure_secondary(S, torch, dev, stream, steps=200):
    """Step rate of the 64^3 coarse run with the MLP eddy-viscosity closure
    (cutoff kc = 21, eddy force on the band 14..20; randomly initialised MLP
    weights -- the step's work does not depend on their values) and of the plain
    coarse run, device-timed."""
    from spectral_upcxx_b200 import closure as CL
    from spectral_upcxx_b200 import ic
    c = CLOSURE
    nc = c["nc"]
    model = CL.MLPModel.init(0, s_in=1.0, s_out=1e-3, device=dev)
    Vc0 = CL.truncate([x.to(torch.complex64) for x in ic.solenoidal_spectrum_hat(
        nc, c["eval_seeds"][0], dev)], nc, c["kc"])
    out = {}
    for name in ("mlp", "plain"):
        with torch.cuda.stream(stream):
            st = S.NSStepper((nc, nc, nc), NU, DT, torch.complex64, device=dev)
            if name == "mlp":
                st.set_closure(S._native.SNS_CLOSURE_MLP, mlp=model.packed, kc=c["kc"])
                st.set_sgs_band(14.0, 20.0)
            else:
                st.set_closure(S._native.SNS_CLOSURE_NONE, kc=c["kc"])
            st.bootstrap(Vc0, S.curl(Vc0))
            st.step(5)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            st.step(steps)
            e1.record(stream)
        stream.synchronize()
        out[f"closure{nc}_{name}_steps_per_s"] = steps / (e0.elapsed_time(e1) / 1e3)
        st.close()
    return out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="ns256_fp32")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    rank, world, local = dist_setup(args)
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_b200(args, rank, world, local)


if __name__ == "__main__":
    sys.exit(main())
