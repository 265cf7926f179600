"""Benchmark of the WaveQ3D engine: ray-steps/s on the sloped Rayleigh workload.

Workload (one bench "step" = one complete propagation of it): linear
gradient profile 1500 + 0.0163 z m/s with Thorp attenuation, bottom sloping
from 200 m at the source to 2000 m at 20 km (boundary_slope), Rayleigh
bottom (1.5, 1.1, 0.5 dB/wavelength), 50 m source, 5 frequencies 100 Hz -
3 kHz, 1801 D/E x 91 AZ rays (wrapping AZ fan), dt 0.05 s for 40 s (800
wave_queue steps), 1024 targets on a 32 x 32 range/depth grid.  Inputs are
synthetic (generated, no data files).

value: whole-job ray-steps/s with the workload resident in HBM, timed with
CUDA events on the engine's stream around the 800 steps.  e2e: the same
metric through the public API with host buffers (queue creation from host
arrays, propagation, eigenray records read back).  roofline: the CPA kernel
(the dominant kernel) in FP64 operations against an FP64 throughput peak
measured on this GPU by bench.py itself.  cpu_baseline: the CPU oracle (a
restatement of the reference's CPU wave_queue) on a bounded sample.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

METRIC = "ray-steps/s"
WORKLOAD = "linear_slope_rayleigh_1801x91_1024tgt_5f_dt0.05_40s"

# algorithmic work of the CPA search per (ray, target) pair and step: the
# reference's distance2 (wave_front.cc:222-236: 15 FP64 operations) plus the
# two time comparisons of detect_eigenrays (wave_queue.cc:386-393)
FLOPS_PER_RAY_TARGET_STEP = 17
# FP64 bytes the CPA kernel must read per interior ray and launch: four
# distance2 terms (rho, theta, phi, sin theta) on three fronts plus on_edge
BYTES_PER_RAY_CPA = 3 * 4 * 8 + 1
# dram__bytes_read.sum + dram__bytes_write.sum of one k_cpa_f32 launch on
# this workload (ncu, launch 301; profiles/fp32c_step_kernels_*.md)
NCU_TRAFFIC_CPA_F32 = 15986688 + 0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--cpu-sample-steps", type=int, default=240,
                    help="wave steps of the CPU samples (240 of 801: eigenrays to targets out to "
                         "about 15 km are built inside the sample)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-reverb", action="store_true",
                    help="skip the reverberation-scale sample (3601 x 181 rays, 4096 targets)")
    ap.add_argument("--no-munk-cpu", action="store_true",
                    help="skip the oracle's full run of the Munk workload (a few seconds)")
    ap.add_argument("--no-gradients", action="store_true", help="skip the gradient workload")
    ap.add_argument("--batch-instances", type=int, default=512,
                    help="instances of the batched gridded workload (0 skips it)")
    ap.add_argument("--profile-workload", default="linear_slope_rayleigh",
                    choices=["linear_slope_rayleigh", "std14", "gridded"],
                    help="workload of --profile-steps (std14: the speed study with 100 targets; "
                         "gridded: one 1801 x 45 ray instance of the batched gridded workload's "
                         "environment, 64 targets, dt 0.05 s)")
    ap.add_argument("--profile-schedule", default="auto", choices=["auto", "side", "inline"],
                    help="reflection schedule of the --profile-steps queue")
    ap.add_argument("--profile-steps", type=int, default=0,
                    help="profiling mode: one queue of the workload, this many wave steps, no output")
    return ap.parse_args()


# ---------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi clock / throttle-reason sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, FileNotFoundError):
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in self.lines:
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- FP64 peak
PEAK_SRC = r"""
#include <cuda_runtime.h>
template <class T>
__global__ void fma_peak(T* out, int iters) {
    T a = threadIdx.x * (T)1e-3, b = (T)1.0000001, c = (T)0.9999999, d = blockIdx.x * (T)1e-6;
    T e = a + (T)1, f = d + (T)2, g = a * (T)0.5, h = d * (T)0.25;
    for (int i = 0; i < iters; ++i) {
        a = a * b + c; d = d * b + c; e = e * b + c; f = f * b + c;
        g = g * b + c; h = h * b + c;
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a + d + e + f + g + h;
}
template <class T>
float run(int iters) {
    T* out; cudaMalloc(&out, 148 * 8 * 256 * sizeof(T));
    cudaEvent_t x, y; cudaEventCreate(&x); cudaEventCreate(&y);
    fma_peak<T><<<148 * 8, 256>>>(out, 100);
    cudaEventRecord(x);
    fma_peak<T><<<148 * 8, 256>>>(out, iters);
    cudaEventRecord(y); cudaEventSynchronize(y);
    float ms = 0; cudaEventElapsedTime(&ms, x, y);
    cudaFree(out); cudaEventDestroy(x); cudaEventDestroy(y);
    return ms;
}
extern "C" float run_peak64(int iters) { return run<double>(iters); }
extern "C" float run_peak32(int iters) { return run<float>(iters); }
"""


def measure_fma_peaks():
    """FP64 and FP32 FMA throughput (TFLOP/s, an FMA counted as 2 flops) of
    this GPU: 6 independent FMA chains per thread, 148 x 8 blocks of 256
    threads.  MEASURED_PEAKS.json carries only HBM and bf16 tensor figures."""
    import ctypes as C
    import tempfile
    out = {"fp64": None, "fp32": None, "source": "measured by bench.py (FMA loop)"}
    try:
        d = tempfile.mkdtemp()
        cu = os.path.join(d, "peak.cu")
        so = os.path.join(d, "peak.so")
        open(cu, "w").write(PEAK_SRC)
        subprocess.check_call(["nvcc", "-O3", "-gencode", "arch=compute_100a,code=sm_100a", "-shared",
                               "-Xcompiler", "-fPIC", "-o", so, cu], stdout=subprocess.DEVNULL,
                              stderr=subprocess.DEVNULL)
        lib = C.CDLL(so)
        for name, key, iters in (("run_peak64", "fp64", 20000), ("run_peak32", "fp32", 40000)):
            fn = getattr(lib, name)
            fn.restype = C.c_float
            ms = fn(iters)
            out[key] = 148 * 8 * 256 * iters * 6 * 2 / (ms / 1e3) / 1e12
    except Exception as e:  # noqa: BLE001
        out["source"] = "unavailable: %s" % e
    return out


# ---------------------------------------------------------------- engine arm
def max_over_ranks(values, dist):
    """Each value's maximum over the ranks (every rank calls this once, in
    the same place); the values themselves with a single process."""
    if dist is None:
        return list(values)
    import torch
    t = torch.tensor(list(values), dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(x) for x in t]


def engine_arm(args, rank, world, dist):
    import underseamodelinglibrary_b200 as u
    from underseamodelinglibrary_b200 import scenarios as S

    sc = S.linear_slope_rayleigh()
    nde, naz = sc["de"].size(), sc["az"].size()
    nt = sc["targets"].size1() * sc["targets"].size2()
    # steps of one propagation: the reference loop "while (time() < 40) step()"
    nsteps, t = 0, 0.0
    while t < sc["time_max"]:
        t += sc["dt"]
        nsteps += 1
    ray_steps = nde * naz * nsteps

    from underseamodelinglibrary_b200 import _abi

    def make(precision=_abi.FP32C):
        return S.build_queue(sc, u.wave_queue, device=0, precision=precision)

    def timed_runs(precision, count):
        """device time (ms) of ``count`` propagations replayed as CUDA
        graphs, queues built first; returns (total ms, launches, eigenrays)"""
        qs = [make(precision) for _ in range(count)]
        for q in qs:
            q.timing(reset=True)
        tot = 0.0
        launches = neig = 0
        for q in qs:
            q.run(sc["time_max"])
            tm = q.timing()
            tot += tm["total_ms"]
            launches += tm["launches"]
            neig += len(q.take_eigenrays())
        return tot, launches, neig

    def kernel_breakdown(precision):
        """per-kernel device ms of one propagation with CUDA events around
        every launch (direct launches, so slower than the graph replay)"""
        q = make(precision)
        q.set_timing(True)
        q.timing(reset=True)
        q.run(sc["time_max"])
        tm = q.timing()
        q.take_eigenrays()
        return {"advance": tm["advance_ms"], "reflect (side stream)": tm["reflect_ms"],
                "cpa": tm["cpa_ms"], "eigenray": tm["eigenray_ms"], "total_with_events": tm["total_ms"]}

    # device-resident timing: queues built (inputs in HBM) before the timer
    for _ in range(args.warmup):
        q = make()
        q.run(sc["time_max"])
        q.take_eigenrays()
        del q
    clocks = ClockSampler(rank)
    clocks.start()
    if dist is not None:
        dist.barrier()
    total_ms, launches, n_eig = timed_runs(_abi.FP32C, args.steps)
    if dist is not None:
        dist.barrier()
    clk = clocks.stop()
    # kernel shares from an event-timed propagation, and the plain FP64 form
    # on the same workload for the FP32C:FP64 ratio
    kern = kernel_breakdown(_abi.FP32C)
    f64_total, _, f64_neig = timed_runs(_abi.FP64, 1)
    kern64 = kernel_breakdown(_abi.FP64)
    cpa_ms = kern["cpa"]
    # the FP32 propagation form: speed, and its eigenrays against the FP64
    # form's on the same workload
    f32_total, _, f32_neig = timed_runs(_abi.FP32, 1)
    from underseamodelinglibrary_b200.eigenrays import form_errors
    q64, q32 = make(_abi.FP64), make(_abi.FP32)
    q64.run(sc["time_max"])
    q32.run(sc["time_max"])
    f32_err = form_errors(q32.take_eigenrays(), q64.take_eigenrays())
    del q64, q32

    # end to end through the public API with host buffers
    e2e_times = []
    h2d = d2h = 0
    for k in range(args.steps):
        t0 = time.perf_counter()
        q = make()
        q.run(sc["time_max"])
        rays = q.take_eigenrays()
        del q
        e2e_times.append(time.perf_counter() - t0)
        nf = sc["freq"].size()
        h2d = 8 * (nf + 2 * nde + 2 * naz + 3 * nt) + 8 * 3
        d2h = len(rays) * (96 + 16 * nf)

    total_s, e2e_s = max_over_ranks([total_ms / 1000.0, sum(e2e_times)], dist)
    value = world * args.steps * ray_steps / total_s
    e2e = world * args.steps * ray_steps / e2e_s

    # roofline of the CPA kernel: algorithmic FP64 operations per launch
    interior = (nde - 2) * ((naz - 1) if _wraps(sc["az"]) else (naz - 2))
    cpa_launch_s = (cpa_ms / 1000.0) / nsteps
    flops_launch = FLOPS_PER_RAY_TARGET_STEP * interior * nt
    achieved = flops_launch / cpa_launch_s / 1e12
    peaks = measure_fma_peaks()
    # the FP32 peak from the clock: 148 SMs x 128 FP32 lanes x 2 flops per
    # FMA x the median SM clock sampled during the timed region
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    fp32_peak = 148 * 128 * 2 * sm_mhz * 1e6 / 1e12
    fp64_peak_clock = 148 * 64 * 2 * sm_mhz * 1e6 / 1e12
    out = {
        "metric": METRIC, "value": value, "unit": "ray-steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64+f32", "data": "synthetic",
        "config": {"workload": WORKLOAD, "rays": nde * naz, "num_de": nde, "num_az": naz,
                   "targets": nt, "frequencies": sc["freq"].size(), "wave_steps": nsteps,
                   "form": "FP32C (FP32-screened CPA, FP64 state)", "parallelism": "replicas" if world > 1 else "single",
                   "l2": "working set (5 fronts, %.0f MB) exceeds L2" % (nde * naz * 5 * 32 * 8 / 1e6)},
        "eigenrays_per_s": world * n_eig / total_s,
        "e2e": {"value": e2e, "unit": "ray-steps/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "fp64_form": {"value": ray_steps / (f64_total / 1000.0), "ms_per_step": f64_total,
                      "kernel_ms": kern64, "eigenrays": f64_neig},
        "fp32_form": {"value": ray_steps / (f32_total / 1000.0), "ms_per_step": f32_total,
                      "vs_fp64_form": f64_total / f32_total, "eigenrays": f32_neig,
                      "form": "FP32 sound speed, gradient and ray derivatives at the altitude offset; "
                              "FP64 state, travel time, distance terms and CPA fit; FP32-screened CPA",
                      "errors_vs_fp64_form": f32_err},
        "eigenrays_per_propagation": n_eig / args.steps,
        "kernel_ms": kern,
        "roofline": {"bound": "fp32", "achieved": achieved,
                     "peak": fp32_peak,
                     "unit": "TFLOP/s",
                     "frac": (achieved / fp32_peak) if fp32_peak else None,
                     "traffic": NCU_TRAFFIC_CPA_F32,
                     "traffic_unit": "bytes per launch (ncu capture)",
                     "kernel": "k_cpa_f32",
                     "peak_source": "clock-derived: 148 SMs x 128 FP32 lanes x 2 x median SM clock %.0f MHz "
                                    "(MEASURED_PEAKS.json has no FP32/FP64 CUDA-core figure)" % sm_mhz,
                     "fp32_fma_loop_tflops": peaks["fp32"],
                     "frac_of_fma_loop": (achieved / peaks["fp32"]) if peaks["fp32"] else None,
                     "fp64_peak": fp64_peak_clock,
                     "fp64_fma_loop_tflops": peaks["fp64"],
                     "fp64_form_cpa_frac_of_fp64_peak": (
                         flops_launch / (kern64["cpa"] / 1000.0 / nsteps) / 1e12 / fp64_peak_clock),
                     "algorithmic_flops_per_launch": flops_launch},
        "roofline_hbm": hbm_roofline(interior, cpa_launch_s),
        "clocks": clk,
    }
    if args.batch_instances > 0:
        out["batched"] = batched_arm(args)
    if not args.no_gradients:
        out["gradients"] = gradient_arm()
    out["std14"] = std14_arm()
    out["munk_flat"] = munk_arm()
    if not args.no_reverb:
        out["reverb_scale_sample"] = reverb_arm()
        out["reverb_batch"] = reverb_batch_arm()
    out["biverbs"] = biverb_arm()
    return out


# the reference's published single-core times of its speed study
# (studies/cmp_speed/cmp_speed_test_20221203.xlsx, WaveQ3D v3.0, Xeon
# E3-1505M v6 @ 3.00 GHz): seconds per propagation by target count
STD14_PUBLISHED_S = {0: 2.576, 100: 4.324, 1000: 19.445}


def std14_arm():
    """The reference's speed study (studies/cmp_speed/cmp_speed.cc): STD14
    grids near Hawaii, 181 x 25 rays, 801 steps of 0.1 s, targets on a
    100 km ring, with an eigenray_collection listener as in the study.
    Device time of the step loop (CUDA-graph replay), FP32C and FP64, next
    to the published single-core CPU time of the same loop."""
    import underseamodelinglibrary_b200 as u
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import _abi
    rows = []
    for nt in (0, 100, 1000):
        sc = S.std14(num_targets=nt)
        row = {"targets": nt, "published_cpu_s": STD14_PUBLISHED_S[nt]}
        for name, prec in (("fp32c", _abi.FP32C), ("fp64", _abi.FP64)):
            best = None
            for _ in range(3):
                q = S.build_queue(sc, u.wave_queue, precision=prec)
                if nt:
                    coll = u.eigenray_collection(sc["freq"], sc["pos"], sc["targets"])
                    q.add_eigenray_listener(coll)
                q.timing(reset=True)
                t0 = time.perf_counter()
                q.run(sc["time_max"])
                wall = time.perf_counter() - t0
                ms = q.timing()["total_ms"]
                best = ms if best is None else min(best, ms)
            row[name + "_ms"] = best
            row[name + "_wall_s_last"] = wall
        row["speedup_fp32c_vs_published_cpu"] = STD14_PUBLISHED_S[nt] / (row["fp32c_ms"] / 1000.0)
        rows.append(row)
    return {"workload": "std14_cmp_speed_181x25_801steps_250Hz", "rays": 181 * 25, "steps": 801,
            "rows": rows}


def munk_arm():
    """The plain FP64 workload: Munk profile, 5000 m flat bottom, source
    1000 m, 10 Hz, 181 x 37 rays, 600 steps of 0.1 s, 100 targets at 500 m.
    Device time of one propagation (CUDA-graph replay, best of 3), FP32C
    and FP64; the oracle's time for the same run is in cpu_baseline."""
    import underseamodelinglibrary_b200 as u
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import _abi
    sc = S.munk_flat()
    out = {"workload": sc["name"] + "_100tgt_600steps_10Hz", "rays": sc["de"].size() * sc["az"].size()}
    for name, prec in (("fp32c", _abi.FP32C), ("fp64", _abi.FP64)):
        best = None
        for _ in range(3):
            q = S.build_queue(sc, u.wave_queue, precision=prec)
            q.timing(reset=True)
            q.run(sc["time_max"])
            ms = q.timing()["total_ms"]
            n_steps, n_eig = q.steps(), len(q.take_eigenrays())
            best = ms if best is None else min(best, ms)
        out[name + "_ms"] = best
        out[name + "_ray_steps_per_s"] = out["rays"] * n_steps / (best / 1000.0)
        out[name + "_eigenrays"] = n_eig
    out["steps"] = n_steps
    return out


def reverb_arm():
    """A bounded sample of the reverberation-scale workload: one of its 16
    source depths (100 m), 3601 x 181 rays, 4096 targets, 32 frequencies,
    the first 10 s (200 steps) of 180 s, eigenverbs off.  Device time of the
    propagation (CUDA-graph replay); the eigenrays are read back after it."""
    import underseamodelinglibrary_b200 as u
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import _abi
    try:
        sc = S.reverb_scale(time_max=10.0)
        rays = sc["de"].size() * sc["az"].size()
        for rep in range(2):
            # the first run also makes this shape's reflection-schedule plan
            t0 = time.perf_counter()
            q = S.build_queue(sc, u.wave_queue, precision=_abi.FP32C, eigenray_capacity=1 << 19)
            t_build = time.perf_counter() - t0
            q.timing(reset=True)
            q.run(sc["time_max"])
            ms = q.timing()["total_ms"]
            n_steps = q.steps()
            n_eig = len(q.take_eigenrays())
            del q
        return {"workload": sc["name"], "sample": "1 of 16 source depths, first 10 s of 180 s, eigenverbs off",
                "rays": rays, "steps": n_steps, "ms_device": ms, "ray_steps_per_s": rays * n_steps / (ms / 1000.0),
                "eigenrays": n_eig, "build_s": t_build, "form": "FP32C"}
    except Exception as e:  # a failure here must not hide the headline line
        return {"error": "%s: %s" % (type(e).__name__, e)}


BIVERB_WORKLOAD = "biverbs_bistatic_footprints_57600x57600_2freq"


def reverb_batch_arm(n_steps=600):
    """The reverberation-scale workload's batch: all 16 source depths
    (20-800 m) in one wq3d_batch_run, 3601 x 181 rays each, 4096 targets,
    32 frequencies, gridded random ocean, Eckart surface, Rayleigh bottom
    (1.8, 1.15, 0.3) with its exact parameter sensitivities, eigenverbs at
    every boundary interaction built and read back (counted per interface),
    FP32C, the first ``n_steps`` steps of 3601.  Device time of the batch."""
    import numpy as np
    import underseamodelinglibrary_b200 as u
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import types as T
    from underseamodelinglibrary_b200 import _abi
    try:
        sc = S.reverb_scale(time_max=(n_steps - 0.5) * 0.05, bottom_loss=u.reflect_loss_rayleigh(1.8, 1.15, 0.3))
        rays = sc["de"].size() * sc["az"].size()
        nf = sc["freq"].size()
        t0 = time.perf_counter()
        qs = []
        for z in np.linspace(20.0, 800.0, 16):
            s1 = dict(sc)
            s1["pos"] = T.wposition1(45.0, -45.0, -float(z))
            q = S.build_queue(s1, u.wave_queue, precision=_abi.FP32C, eigenray_capacity=1 << 17)
            q.enable_sensitivity()
            q.count_eigenverbs(True)
            qs.append(q)
        t_build = time.perf_counter() - t0
        steps, ms = u.run_batch(qs, sc["time_max"])
        n_steps_run = int(sum(steps))
        verbs = [q.eigenverb_counts() for q in qs]
        n_verb = int(sum(sum(v) for v in verbs))
        n_eig = int(sum(len(q.take_eigenrays()) for q in qs))
        del qs
        rec_bytes = 136 + 8 * nf
        return {"workload": sc["name"], "sources": 16,
                "sample": "16 source depths in one batch, first %d of 3601 steps, eigenverbs on, bottom "
                          "sensitivities on" % n_steps,
                "rays_per_source": rays, "steps_total": n_steps_run, "ms_device": ms,
                "ray_steps_per_s": rays * n_steps_run / (ms / 1000.0),
                "eigenrays": n_eig, "eigenverbs": n_verb,
                "eigenverbs_by_interface": [int(sum(v[k] for v in verbs)) for k in range(4)],
                "eigenverbs_per_s": n_verb / (ms / 1000.0),
                "eigenverb_stream_bytes": n_verb * rec_bytes,
                "eigenverb_stream_gb_per_s": n_verb * rec_bytes / (ms / 1000.0) / 1e9,
                "build_s": t_build, "form": "FP32C"}
    except Exception as e:  # noqa: BLE001
        return {"error": "%s: %s" % (type(e).__name__, e)}


def biverb_inputs():
    """Bistatic footprints in the shape of the reference's biverb test
    (biverbs_test.cc:41-77): a source at (0, 0) and a receiver 1.1 km away
    on the surface of 500 m deep isovelocity water, D/E -85..-5.5 deg in
    0.5 deg steps x AZ 0..359 deg in 1 deg steps (57,600 eigenverbs each),
    2 frequencies, -30 dB constant bottom scattering."""
    import numpy as np
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import types as T
    T.set_earth_radius(6371000.0)
    de = np.arange(-85.0, -5.0, 0.5)
    az = np.arange(0.0, 360.0, 1.0)
    src = S.analytic_footprints(0.0, 0.0, 500.0, de, az, 2)
    rcv = S.analytic_footprints(0.007, 0.007, 500.0, de, az, 2)
    return src, rcv, np.array([1000.0, 2000.0])


def biverb_call(lib, fn, src, rcv, freq, num_rcv=None, out=None, out_power=None, capacity=0):
    import ctypes as C
    from underseamodelinglibrary_b200 import _abi
    from underseamodelinglibrary_b200.ocean import scattering_constant
    dp = C.POINTER(C.c_double)
    (s, sp), (r, rp) = src, rcv
    ns, nr = sp.shape[0], rp.shape[0] if num_rcv is None else num_rcv
    count = C.c_size_t()
    desc = scattering_constant(-30.0).desc()
    rc = getattr(lib, fn)(s, sp.ctypes.data_as(dp), ns, r, rp.ctypes.data_as(dp), nr,
                          freq.ctypes.data_as(dp), freq.size, C.byref(desc), 6371000.0, 1.5, 1e-20,
                          out, out_power.ctypes.data_as(dp) if out_power is not None else None,
                          capacity, C.byref(count))
    if rc != 0:
        raise _abi.EngineError(rc, "biverbs")
    return count.value


def biverb_arm():
    """wq3d_biverbs on the bistatic footprint workload, end to end through
    the C ABI: host eigenverbs in, host biverbs out, device buffers made and
    freed inside every call.  The first call counts, and sizes the output;
    then 3 timed calls (wall clock)."""
    import numpy as np
    from underseamodelinglibrary_b200 import _abi
    try:
        lib = _abi.load_engine()
        src, rcv, freq = biverb_inputs()
        n = biverb_call(lib, "wq3d_biverbs", src, rcv, freq)
        out = (_abi.wq3d_biverb * n)()
        power = np.zeros((n, freq.size))
        biverb_call(lib, "wq3d_biverbs", src, rcv, freq, out=out, out_power=power, capacity=n)
        times = []
        for _ in range(3):
            t0 = time.perf_counter()
            biverb_call(lib, "wq3d_biverbs", src, rcv, freq, out=out, out_power=power, capacity=n)
            times.append(time.perf_counter() - t0)
        t = min(times)
        pairs = src[1].shape[0] * rcv[1].shape[0]
        return {"workload": BIVERB_WORKLOAD, "source_eigenverbs": src[1].shape[0],
                "receiver_eigenverbs": rcv[1].shape[0], "pairs": pairs, "biverbs": n,
                "ms_e2e": t * 1000.0, "pairs_per_s": pairs / t, "biverbs_per_s": n / t,
                "timing": "wall clock of the whole C-ABI call, best of 3 (host buffers in and out)"}
    except Exception as e:  # a failure here must not hide the headline line
        return {"error": "%s: %s" % (type(e).__name__, e)}


def gradient_arm():
    """Gradient cost on the differentiable workload (1801 x 91 rays, 2000
    steps of 0.05 s, 64 receivers, 20-node profile grid, Rayleigh bottom):
    the forward pass recorded for the adjoint (checkpoints every 50 steps,
    each eigenray's partials, bottom sensitivities), then one reverse sweep
    for the weighted sum of every eigenray's TL and travel time.
    value = what the gradient adds to a plain forward pass (the recording's
    overhead plus the sweep) / that forward pass; sweep_vs_plain_forward is
    the sweep alone.  All three times are device time in the engine's
    normal mode (chunk graphs, streams overlapped)."""
    from underseamodelinglibrary_b200 import adjoint as A
    import numpy as np
    sc = A.AdjointScenario()
    nodes = A.munk_nodes()
    q = sc.queue(nodes)          # warm-up of the same shapes, whole run (the
    q.run(sc.time_max)           # reflection-schedule plan of this shape)
    del q
    q = sc.queue(nodes)
    q.timing(reset=True)
    q.run(sc.time_max)
    ms_plain = q.timing()["total_ms"]
    del q
    # the bottom-parameter sensitivities alone, to split the recording's cost
    q = sc.queue(nodes)
    q.enable_sensitivity()
    q.timing(reset=True)
    q.run(sc.time_max)
    ms_sens = q.timing()["total_ms"]
    del q
    prop = A.Propagation(sc, nodes, checkpoint=50)
    n = len(prop.eigenrays)
    rng = np.random.default_rng(20261203)
    w_tl, w_t = rng.normal(size=n), rng.normal(size=n)
    prop.vjp(w_tl, w_t)          # first sweep makes the workspace
    g, gb, ms_adj = prop.vjp(w_tl, w_t)
    return {"metric": "adjoint:fwd", "value": (ms_adj + prop.ms_forward - ms_plain) / ms_plain, "unit": "ratio",
            "higher_is_better": False, "ms_forward_recorded": prop.ms_forward, "ms_forward_plain": ms_plain,
            "ms_adjoint": ms_adj, "ms_forward_sensitivities_only": ms_sens,
            "sweep_vs_plain_forward": ms_adj / ms_plain,
            "recording_overhead_vs_plain_forward": (prop.ms_forward - ms_plain) / ms_plain,
            "eigenrays": n, "checkpoint_interval": 50,
            "gradient_norm": float(np.linalg.norm(g)),
            "method": "reverse sweep: checkpoints every 50 steps, recompute per interval, adjoint of AB3, "
                      "reflections and start-up with dual-number step Jacobians; eigenray partials recorded "
                      "in the forward; bottom parameters exact (sensitivity mode)",
            "config": {"workload": "adjoint_munk_grid20_rayleigh_1801x91_2000steps_64rx"}}


def batched_arm(args):
    """Batched solves/s: args.batch_instances uneven instances of the
    gridded workload (own 50x20x20 profile grid and 100x100 bathymetry
    each, 91-1801 D/E x 1-91 AZ rays, 10-120 s, 64 targets, dt 0.05 s),
    FP32C, run together by wq3d_batch_run.  value = instances / (queue
    building + the batch's device time, from its start to its last queue's
    end); the device-only rate is reported beside it."""
    import underseamodelinglibrary_b200 as u
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import _abi
    scs = S.batched_gridded(n_instances=args.batch_instances)
    t0 = time.perf_counter()
    qs = [S.build_queue(sc, u.wave_queue, precision=_abi.FP32C) for sc in scs]
    t_build = time.perf_counter() - t0
    t0 = time.perf_counter()
    steps, ms = u.run_batch(qs, [sc["time_max"] for sc in scs])
    wall = time.perf_counter() - t0
    ray_steps = sum(sc["de"].size() * sc["az"].size() * n for sc, n in zip(scs, steps))
    n_eig = sum(len(q.take_eigenrays()) for q in qs)
    return {"metric": "batched solves/s", "value": len(qs) / (t_build + ms / 1000.0), "unit": "solves/s",
            "value_device_only": len(qs) / (ms / 1000.0),
            "instances": len(qs), "ms_device": ms, "wall_s": wall, "build_s": t_build,
            "ray_steps_per_s": ray_steps / (ms / 1000.0), "ray_steps": ray_steps, "eigenrays": n_eig,
            "config": {"workload": "batched_gridded_%d" % len(qs), "form": "FP32C",
                       "rays_total": sum(sc["de"].size() * sc["az"].size() for sc in scs),
                       "steps_total": sum(steps)}}


def _wraps(az):
    a0, a1 = abs(az[0]), abs(az[az.size() - 1])
    return math.fmod(a0 + 360.0, 360.0) == math.fmod(a1 + 360.0, 360.0)


def hbm_roofline(interior, launch_s):
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    peak = peaks.get("hbm_gbs")
    src = "measured (MEASURED_PEAKS.json)" if peak else "fallback 6650 GB/s"
    peak = peak or 6650.0
    achieved = interior * BYTES_PER_RAY_CPA / launch_s / 1e9
    return {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": None, "peak_source": src}


# ---------------------------------------------------------------- CPU arms
def cpu_sample_scenario(sample_steps):
    """A bounded sample of the same workload: the full 1801-ray D/E fan on
    every 16th AZ column of the 91-ray fan (6 columns), all 1024 targets,
    the first ``sample_steps`` wave_queue steps."""
    from underseamodelinglibrary_b200 import scenarios as S
    from underseamodelinglibrary_b200 import types as T
    sc = S.linear_slope_rayleigh()
    sc["az"] = T.seq_linear(0.0, 64.0, 6)
    sc["time_max"] = sample_steps * sc["dt"] - 0.5 * sc["dt"]
    return sc


def cpu_run(sc, nthreads):
    """Runs ``nthreads`` independent oracle queues concurrently (the
    reference's thread_pool model: one wave_queue per worker)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_binding import OracleQueue
    from underseamodelinglibrary_b200 import scenarios as S
    queues = [S.build_queue(sc, OracleQueue) for _ in range(nthreads)]
    done = [0] * nthreads

    def work(i):
        done[i] = queues[i].run(sc["time_max"])

    th = [threading.Thread(target=work, args=(i,)) for i in range(nthreads)]
    t0 = time.perf_counter()
    for x in th:
        x.start()
    for x in th:
        x.join()
    dt = time.perf_counter() - t0
    rays = sc["de"].size() * sc["az"].size()
    return sum(done) * rays / dt, dt, done[0]


def cpu_baseline(args):
    from underseamodelinglibrary_b200 import scenarios as S
    sc = cpu_sample_scenario(args.cpu_sample_steps)
    v, dt, n = cpu_run(sc, 1)
    out = {"value": v, "unit": "ray-steps/s", "cores": 1, "kind": "port",
           "sample": "oracle (CPU restatement of the reference wave_queue), 1 thread: full 1801-ray "
                     "D/E fan x every 16th AZ column (6 columns), all 1024 targets, first %d of 800 "
                     "steps; %.1f s" % (n, dt)}
    if not args.no_munk_cpu:
        # the whole plain FP64 Munk workload (181 x 37 rays, 600 steps, 100
        # targets), 1 thread
        m = S.munk_flat()
        mv, mdt, mn = cpu_run(m, 1)
        out["munk_flat"] = {"seconds": mdt, "ray_steps_per_s": mv, "steps": mn, "cores": 1,
                            "kind": "port"}
    # the biverb workload's first 4000 receiver eigenverbs against all
    # 57,600 source eigenverbs, 1 thread
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    from oracle_binding import load_oracle
    src, rcv, freq = biverb_inputs()
    k = 4000
    t0 = time.perf_counter()
    nb = biverb_call(load_oracle(), "oracle_biverbs", src, rcv, freq, num_rcv=k)
    dt_b = time.perf_counter() - t0
    out["biverbs"] = {"pairs_per_s": src[1].shape[0] * k / dt_b, "seconds": dt_b, "biverbs": nb,
                      "cores": 1, "kind": "port",
                      "sample": "first %d of %d receiver eigenverbs x all source eigenverbs" % (k, rcv[1].shape[0])}
    return out


def reference_arm(args, rank):
    if rank != 0:
        return None
    ncores = os.cpu_count() or 1
    sc = cpu_sample_scenario(args.cpu_sample_steps)
    for _ in range(args.warmup if args.warmup < 1 else 1):
        cpu_run(cpu_sample_scenario(2), ncores)
    vals = []
    for _ in range(args.steps):
        v, dt, n = cpu_run(sc, ncores)
        vals.append(v)
    value = statistics.mean(vals)
    return {"metric": METRIC, "value": value, "unit": "ray-steps/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": WORKLOAD, "sample": "every 16th AZ column, first %d steps" % n},
            "cpu_baseline": {"value": value, "unit": "ray-steps/s", "cores": ncores, "kind": "port",
                             "sample": "oracle restatement of the reference CPU wave_queue, %d "
                                       "concurrent queues (thread_pool model), full D/E fan x 6 AZ "
                                       "columns, 1024 targets, first %d steps" % (ncores, n)},
            "e2e": {"value": value, "unit": "ray-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch
        import torch.distributed as tdist
        tdist.init_process_group("gloo", timeout=datetime.timedelta(seconds=600))
        dist = tdist
    if args.impl == "reference":
        out = reference_arm(args, rank)
        if out is not None:
            print(json.dumps(out), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return
    if world > 1:
        os.environ["CUDA_VISIBLE_DEVICES"] = str(local)
    if args.profile_steps:
        import underseamodelinglibrary_b200 as u
        from underseamodelinglibrary_b200 import scenarios as S
        from underseamodelinglibrary_b200 import _abi
        if args.profile_workload == "std14":
            sc = S.std14(num_targets=100)
        elif args.profile_workload == "gridded":
            sc = S.gridded_munk(seed=1, num_de=1801, num_az=45, n_targets=64, time_max=60.0, dt=0.05)
        else:
            sc = S.linear_slope_rayleigh()
        q = S.build_queue(sc, u.wave_queue, device=0, precision=_abi.FP32C)
        q.set_reflect_schedule({"auto": _abi.REFLECT_AUTO, "side": _abi.REFLECT_SIDE,
                                "inline": _abi.REFLECT_INLINE}[args.profile_schedule])
        q.step(args.profile_steps)
        print("profile run: %d steps, %d eigenrays" % (q.steps(), len(q.take_eigenrays())))
        return
    out = engine_arm(args, rank, world, dist)
    if rank == 0:
        if not args.no_cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(args)
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
