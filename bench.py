"""Benchmark: RVE voxel-iterations/s of the B200 FFT-homogenization solver.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

A step is one complete solve of the workload's RVE (state reset to the uniform
load, sweeps until the stop rule).  value = voxels x sweeps of all K steps on
all ranks / device time (CUDA events on the solver's stream, max over ranks).
Every sweep counts, FP32 inner sweeps and FP64 defect sweeps alike; the FP64
GPU solver of the same workload is timed as well and reported beside it.

Workloads (synthetic, seeded; the reference project has no dataset):
  thermal128  128^3 steady conduction, ~100 prolate ellipsoids (3a,a,a) with
              random orientation at 30% inclusion fraction, k_incl:k_matrix =
              100:1, mean gradient along z; FP32 sweeps + FP64 refinement to
              residual 1e-8 (default)
  elastic64   64^3 linear elasticity, non-overlapping spheres r = 6 voxels at
              20%, matrix E=3 GPa nu=.35, inclusions E=70 GPa nu=.2,
              macroscopic strain eps_xx = 1e-3; FP64 to residual 1e-6
  batch512    512 seeded two-phase RVEs, N uniform on {32,48,64,96}, penetrable
              spheres of radius N/10 at inclusion fraction uniform in 5-40%,
              stiffness contrast uniform in 2-100 (inclusion E = contrast x 3 GPa,
              nu .2; matrix 3 GPa, .35); 6 unit load cases each -> full C_eff;
              FP32 sweeps + FP64 refinement to residual 1e-6; one multi-RVE
              solve (one graph launch) per grid size, the grid sizes run
              concurrently (a step is the whole batch)
  rec171      microstructure reconstruction (recPlan + runRec(100, 0.8)) on the
              example's 171^3 grid and TPCF; a step is one runRec; value =
              voxels x phase-retrieval passes / device time
  serve       Poisson arrivals of elastic, thermal and J2 solves (1/3 each), N
              log-uniform on [32, 256] rounded to the nearest of {32, 48, 64, 96,
              128, 256} in log scale; elastic as elastic64 (FP32+refine), thermal
              as thermal128 (FP32+refine), J2 as the 256^3 J2 workload with 5
              increments to 0.5% (FP32); residual 1e-6.  Capacity is measured
              with a closed burst first, then offered loads of 0.25x..1.5x that
              capacity are replayed; p50/p99 latency and throughput per load
Multi-GPU: replicas only (one independent solve, or batch, per rank), weak scaling.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "RVE voxel-iters/s at residual 1e-6 (FP32+refine vs FP64)"
UNIT = "voxel-iter/s"

# algorithmic bytes per voxel-iteration (one read + one write of the c-component
# field per 3-D transform direction, the state read and written once, 1-byte
# phase): 6*c*w + 1
def bytes_per_vi(c, w):
    return 6 * c * w + 1


PASS_NAMES = ("z_forward", "y_forward", "x_turnaround", "y_inverse", "z_inverse")
PASS_KERNELS = ("k_zfwd_fast (prologue + z R2C)", "k_ypass_fast<-1>", "k_xturn_fast (x FFT, Green, x IFFT)",
                "k_ypass_fast<+1>", "k_zinv_fast (z C2R + EM update + finalize)")
# two-pass sweeps (per-component operators): the profile's slot 2 is the x
# turnaround, slot 4 the y-z slab pass, the other slots are empty
PASS_NAMES_2 = (None, None, "x_turnaround", None, "yz_slab")
PASS_KERNELS_2 = (None, None, "k_xturn_fast (x FFT, Green, x IFFT)", None,
                  "k_slab<MIX> (y IFFT, z C2R, EM update, polarization, z R2C, y FFT + finalize)")


def pass_bytes(c, w, N, forcing, two_pass=False):
    """Algorithmic bytes per launch of each sweep pass on an N^3 grid with c
    components of w-byte reals: the pass's own inputs and outputs (half
    spectrum N*N*Hzp complex per component, Hzp = N/2+1 rounded up to even;
    state c*V reals; 1-byte phase; the FP32 defect read by the refinement's
    inner sweeps).  Two-pass sweeps: the x turnaround, and the slab pass that
    reads and writes the spectrum and the state once, reads the defect and the
    phase map once per component."""
    V = N ** 3
    hzp = ((N // 2 + 1) + 1) & ~1
    spec = c * N * N * hzp * 2 * w
    state = c * V * w
    forcing_b = c * V * 4 if forcing else 0
    if two_pass:
        return (0, 0, 2 * spec, 0, 2 * spec + 2 * state + c * V + forcing_b)
    zfwd = state + V + spec
    zinv = spec + 2 * state + V + forcing_b
    return (zfwd, 2 * spec, 2 * spec, 2 * spec, zinv)


# DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) from
# the ncu captures summarised in profiles/, keyed (workload, pass, word bytes):
# the five-pass z inverse with a warm cache, the y-z slab pass of the two-pass
# sweep from a --set full capture (cold cache: ncu flushes the caches first)
MEASURED_TRAFFIC = {
    ("thermal128", "z_inverse", 4): (12.0e6, "profiles/thermal128_fp32_sweep_kernels.md"),
    ("thermal128", "yz_slab", 4): (81.8e6, "profiles/thermal128_fp32_two_pass_sweep.md"),
}


WORKLOADS = {
    "thermal128": dict(kind="thermal", N=128, km=1.0, ki=100.0, E=[0.0, 0.0, 1.0], precision="fp32_refine",
                       tol=1e-8, desc="128^3 thermal, 30% ellipsoids (3a,a,a) random orientation, k 100:1, grad z"),
    "elastic64": dict(kind="mech", N=64, E=[1e-3, 0, 0, 0, 0, 0], precision="fp64", tol=1e-6,
                      desc="64^3 elastic, spheres r=6 at 20%, E 70/3 GPa, eps_xx=1e-3"),
    "j2_256": dict(kind="mech", behav="ep", N=256, E=[1e-3, 0, 0, 0, 0, 0], X0=[1, 0, 0, 0, 0, 0], nInc=20,
                   precision="fp32", tol=1e-6,
                   desc="256^3 J2 (E 70 GPa, nu .33, sy 100 MPa, H 1 GPa) with 15% elastic particles (400 GPa, .2), "
                        "log-normal radii 3-10, 20 increments to 2% uniaxial"),
    "batch512": dict(kind="batch", count=512, precision="fp32_refine", tol=1e-6,
                     desc="512 RVEs N in {32,48,64,96}, vf 5-40%, contrast 2-100, 6 load cases each, full C_eff"),
    "elastic2d": dict(kind="2d", N=1024, iterations=25, props=(68.9e9, 0.35, 400e9, 0.23),
                      desc="2-D plane elastic (FFT_Analysis2D), 1024^2, discs at 20%, E 68.9/400 GPa, "
                           "E12 = 0.005, 25 basic-scheme iterations, complex FP64"),
    "rec171": dict(kind="rec", N=171, n=100, beta=0.8, A=25.0, Q=0.4, phi1=0.5, seed=1,
                   desc="microstructure reconstruction (recPlan from a TPCF + runRec(100, 0.8)) on the example's "
                        "171^3 grid and isotropic TPCF f(r) = exp(-r/25) sin(0.4 r)/(0.4 r), phi1 = 0.5; "
                        "complex FP64"),
    "serve": dict(kind="serve", per_level=24, levels=(0.25, 0.5, 1.0, 1.5), tol=1e-6, workers=8,
                  desc="Poisson mix of elastic/thermal/J2 solves, N log-uniform 32..256 (rounded), residual 1e-6"),
}


def make_rve(w, seed=0):
    from mat3d_b200 import rve
    if w["kind"] == "thermal":
        g, meta = rve.ellipsoids(w["N"], vf=0.30, aspect=3.0, n_target=100, seed=seed)
    elif w.get("behav") == "ep":
        g, meta = rve.lognormal_spheres(w["N"], vf=0.15, median=5.0, sigma=0.4, rmin=3.0, rmax=10.0, seed=seed)
    else:
        g, meta = rve.spheres_rsa(w["N"], radius=6.0, vf=0.20, seed=seed)
    return g.ravel().astype(np.int32), meta


# ----------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                smax = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# Reference stop-rule tolerance of the CPU sample per workload: loose enough
# that the reference's loop stops after a handful of sweeps on the full grid
# (thermal128: 5 sweeps; J2: its minimum of 2 in the first increment);
# elastic64 runs the workload's own tolerance (the whole solve).
CPU_SAMPLE_TOL = {"thermal128": 1e-2, "elastic64": 1e-6, "j2_256": 1e30}


def cpu_reference(w, steps, warmup, threads, name):
    """The reference's own solver sources (oracle/_ref) on the host cores, on
    the full workload (grid, microstructure, material): per step one solve with
    the reference's stop rule at CPU_SAMPLE_TOL[name].  The set-up (constructor:
    buffers and FFT plans; material(): tables and the Green operator; setLoad)
    is timed apart and excluded, so `value` is the reference's sweep rate.  Its
    FFT is the project's stand-in for FFTW (oracle/shim/fftw3.h), threaded like
    FFTW over `threads`; the pointwise work is single-threaded, as in the
    reference."""
    from oracle import ref_lib
    rve, _ = make_rve(w)
    N = w["N"]
    V = N ** 3
    if not ref_lib.available():
        return None
    tol = CPU_SAMPLE_TOL.get(name, 1e30)
    ref = ref_lib.RefLib(fft_threads=threads)
    sweeps_all, secs, setup = 0, 0.0, 0.0
    for i in range(warmup + steps):
        if w["kind"] == "thermal":
            r = ref.therm_run((N, N, N), w["km"], w["ki"], rve, np.array(w["E"]), tol, tol)
        elif w.get("behav") == "ep":
            r = ref.mech_run((N, N, N), "ep", MAT_J2, rve, np.array(w["E"], float), np.array(w["X0"], float),
                             tol, tol, 1, 0)
        else:
            r = ref.mech_run((N, N, N), "e", MAT_ELASTIC, rve, np.array(w["E"], float), np.zeros(6), tol, tol, 1, 0)
        su, run_s = ref.last_timing()
        if i >= warmup:
            sweeps_all += r["sweeps"]
            secs += run_s
            setup += su
    what = "first increment of the " if w.get("behav") == "ep" else ""
    return dict(value=V * sweeps_all / secs, sweeps=sweeps_all, seconds=secs, setup_s=setup / max(steps, 1),
                threads=threads,
                sample=f"{steps} x reference solve of the {what}full {N}^3 workload, reference stop rule at {tol:g} "
                       f"({sweeps_all // max(steps, 1)} sweeps each); rate over runAnalysis only, set-up "
                       f"({setup / max(steps, 1):.2f} s per solve: plans, Green operator, load) excluded; FP64; "
                       f"FFT = the project's FFTW stand-in on {threads} threads")


def cpu_baseline_entry(w, name, steps=1):
    """cpu_baseline of the bench line: all host cores, and the reference's own
    setting of 3 FFT threads (src/3d/FFT_analysis3D.cpp:101-102,
    src/3dTherm/FFT_thermal3D.cpp:31-32)."""
    cores = os.cpu_count() or 1
    allc = cpu_reference(w, steps, 0, cores, name)
    if allc is None:
        return None
    as_ref = cpu_reference(w, steps, 0, 3, name)
    return {"value": allc["value"], "unit": UNIT, "cores": cores, "kind": "reference", "sample": allc["sample"],
            "as_reference": {"value": as_ref["value"], "unit": UNIT, "cores": 3, "sample": as_ref["sample"]}}


def cpu_reference_batch(w, steps, warmup, threads):
    """The reference's own solver on the host cores for the batched workload:
    per step, each of the first RVEs of every grid size of the batch (one per
    size) solved for its first load case with the reference's stop rule at
    1e-3; the rate counts runAnalysis only (set-up excluded)."""
    from mat3d_b200 import rve as R
    from oracle import ref_lib
    if not ref_lib.available():
        return None
    ref = ref_lib.RefLib(fft_threads=threads)
    picks, seen = [], set()
    for d in R.batch_rves(w["count"]):
        if d[1] not in seen:
            seen.add(d[1])
            picks.append(d)
    members = [R.batch_member(*d) for d in picks]
    vi, secs = 0, 0.0
    for i in range(warmup + steps):
        for (g, mat, _), d in zip(members, picks):
            N = d[1]
            r = ref.mech_run((N, N, N), "e", mat, g.ravel().astype(np.int32), np.eye(6)[0] * 5e-4, np.zeros(6),
                             1e-3, 1e-3, 1, 0)
            _, run_s = ref.last_timing()
            if i >= warmup:
                vi += N ** 3 * r["sweeps"]
                secs += run_s
    return dict(value=vi / secs, seconds=secs,
                sample=f"{steps} x reference solves of one RVE per grid size {sorted(seen)} of the batch, "
                       f"first load case, reference stop rule at 1e-3; rate over runAnalysis only (set-up "
                       f"excluded); FP64; FFT = the project's FFTW stand-in on {threads} threads")


def disc_rve_2d(N, vf=0.20, seed=0):
    """Seeded 2-D microstructure: overlapping discs of radius N/32 at
    inclusion fraction vf (phase 1 = matrix, 0 = inclusion)."""
    rng = np.random.default_rng(seed)
    g = np.ones((N, N), np.int32)
    r = N / 32.0
    X, Y = np.meshgrid(np.arange(N), np.arange(N), indexing="ij")
    while (g == 0).mean() < vf:
        cx, cy = rng.uniform(0, N, 2)
        dx = (X - cx + N / 2) % N - N / 2
        dy = (Y - cy + N / 2) % N - N / 2
        g[dx * dx + dy * dy <= r * r] = 0
    return g.ravel()


def cpu_reference_2d(w, steps, warmup):
    """The reference's FFT_Analysis2D (oracle/_ref) on the host: each step is
    one full runAnalysis (25 iterations) of the same 2-D workload."""
    from oracle import ref_lib
    if not ref_lib.available():
        return None
    ref = ref_lib.RefLib()
    N = w["N"]
    rve = disc_rve_2d(N)
    E = np.array([0, 0, 0.005], np.complex128)
    secs = 0.0
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        ref.mech2d_run((N, N), np.array(w["props"]), rve, E)
        if i >= warmup:
            secs += time.perf_counter() - t0
    its = steps * w["iterations"]
    return dict(value=N * N * its / secs, seconds=secs,
                sample=f"{steps} x reference runAnalysis of the full {N}^2 workload ({w['iterations']} iterations, "
                       f"set-up included), FP64 complex, single thread")


def run_2d(args, w, rank, world, local):
    """2-D solver: a step is one runAnalysis (w["iterations"] iterations)."""
    import torch
    import torch.distributed as dist

    import mat3d_b200 as m3d

    N = w["N"]
    rve = disc_rve_2d(N, seed=rank)
    E = np.array([0, 0, 0.005], np.complex128)
    s = m3d.Solver2D(N, N)
    s.material(np.array(w["props"]), rve)
    stream = torch.cuda.ExternalStream(s.stream_ptr())

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    for _ in range(args.warmup):
        s.set_load(E)
        s.run(w["iterations"])
    l0 = s.kernel_launches()
    clk = ClockSampler(local)
    clk.start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        s.set_load(E)
        s.run(w["iterations"])
    e1.record(stream)
    barrier()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    launches = s.kernel_launches() - l0
    ms_max = reduce(ms, dist.ReduceOp.MAX if world > 1 else None)
    vi = N * N * w["iterations"] * args.steps
    value = reduce(float(vi), dist.ReduceOp.SUM if world > 1 else None) / (ms_max / 1000.0)
    # e2e: material from the host, run, both fields copied back
    barrier()
    t0 = time.perf_counter()
    for _ in range(max(1, args.steps // 2)):
        s.material(np.array(w["props"]), rve)
        s.set_load(E)
        s.run(w["iterations"])
        s.fields()
    barrier()
    esec = reduce(time.perf_counter() - t0, dist.ReduceOp.MAX if world > 1 else None)
    e2e = reduce(float(N * N * w["iterations"] * max(1, args.steps // 2)),
                 dist.ReduceOp.SUM if world > 1 else None) / esec
    s.close()
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = (json.load(open(peaks_path))["hbm_gbs"], "measured") if os.path.exists(peaks_path) \
        else (6650.0, "fallback")
    # algorithmic bytes per voxel-iteration: pointwise (read eps 48 B + phase 1 B, write
    # sigma and tau 96 B) + three FFT passes reading and writing 3 complex FP64 (96 B each)
    bpv = 48 + 1 + 96 + 3 * 96
    achieved = bpv * vi / (ms / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_2d(w, 1, 0)
    if rank == 0:
        line = {
            "metric": "2-D voxel-iters/s (25-iteration basic scheme, FP64 complex)", "value": value,
            "unit": UNIT, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": args.workload, "desc": w["desc"], "grid": [N, N],
                       "iterations": w["iterations"], "l2": "state (3 complex FP64 fields, 50 MB each) "
                       "exceeds L2 in total; each pass streams 2-3 fields", "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_src, "bytes_per_voxel_iter": bpv,
                         "kernel": "one iteration (pointwise + 3 generic FFT passes)"},
            "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": N * N * 4 + 96,
                    "d2h_bytes_per_step": 2 * 3 * 16 * N * N},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": 1, "kind": "reference",
                                    "sample": cpu["sample"]}
        print(json.dumps(line))


# algorithmic bytes per voxel of each reconstruction pass kernel (complex FP64
# field 16 B, normC 8 B): z forward reads m and writes A; the y passes read and
# write A; the x turnaround reads A and normC and writes A; z inverse reads A and
# the old m (hybrid input-output) and writes m
REC_KERNELS = ("krec_z<Z_FWD>", "krec_y<Y_FWD>", "krec_xturn", "krec_y<Y_INV>", "krec_z<Z_INV>")
REC_BYTES = (32, 32, 40, 32, 48)


def cpu_reference_rec(w, budget_s=40.0):
    """The reference's recPlan / runRec (oracle/_ref) on the host, on the full
    grid: runRec(1) and runRec(3) give the cost of one pass and the fixed part
    (plan set-up, initial field, threshold walk); the value is the rate of the
    full runRec(n) those imply.  The reference transforms with 3 threads
    (fftw_plan_with_nthreads(3))."""
    from oracle import ref_lib
    if not ref_lib.available():
        return None
    from mat3d_b200 import rve as R
    N = w["N"]
    T = R.reconstruction_input((N, N, N), w["A"], w["Q"], w["phi1"])
    ref = ref_lib.RefLib()
    t0 = time.perf_counter()
    ref.rec_run((N, N, N), T, 1, w["beta"], w["seed"])
    t1 = time.perf_counter()
    ref.rec_run((N, N, N), T, 3, w["beta"], w["seed"])
    t3 = time.perf_counter() - t1
    t1 = t1 - t0
    per_pass = max((t3 - t1) / 2, 1e-9)
    fixed = max(t1 - per_pass, 0.0)
    total = fixed + w["n"] * per_pass
    return dict(value=N ** 3 * w["n"] / total, seconds=total, per_pass=per_pass, fixed=fixed,
                sample=f"reference runRec(1) and runRec(3) on the full {N}^3 grid ({t1 + t3:.1f} s): "
                       f"{per_pass:.2f} s per pass, {fixed:.2f} s fixed (set-up + threshold walk), "
                       f"extrapolated to runRec({w['n']})")


def run_rec(args, w, rank, world, local):
    """Reconstruction: a step is one runRec(n, beta) (fresh random field, the
    loop, the threshold walk) on the resident TPCF."""
    import torch
    import torch.distributed as dist

    import mat3d_b200 as m3d
    from mat3d_b200 import rve as R

    N, n, beta = w["N"], w["n"], w["beta"]
    shape = (N, N, N)
    xyz = N ** 3
    T = R.reconstruction_input(shape, w["A"], w["Q"], w["phi1"])
    r = m3d.Reconstruction(T, *shape)
    r.seed(w["seed"] + rank)
    stream = torch.cuda.ExternalStream(r.stream_ptr())

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    for _ in range(args.warmup):
        r.run(n, beta)
    l0 = r.kernel_launches()
    clk = ClockSampler(local)
    clk.start()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    passes = 0
    e0.record(stream)
    for _ in range(args.steps):
        r.run(n, beta)
        passes += r.errors().size
    e1.record(stream)
    barrier()
    clocks = clk.stop()
    ms = e0.elapsed_time(e1)
    launches = r.kernel_launches() - l0
    ms_max = reduce(ms, dist.ReduceOp.MAX if world > 1 else None)
    vp = float(xyz) * passes
    value = reduce(vp, dist.ReduceOp.SUM if world > 1 else None) / (ms_max / 1000.0)
    # per-kernel event times from one host-driven run (same kernels, no graph)
    r.set_profiling(True)
    r.run(n, beta)
    pms, npass = r.profile()
    r.set_profiling(False)
    per_kernel = {REC_KERNELS[k]: 1000.0 * pms[k + 1] / npass for k in range(5)}  # us per launch
    dom = max(range(5), key=lambda k: pms[k + 1])
    dom_us = 1000.0 * pms[dom + 1] / npass
    r.close()
    # e2e: the TPCF from host memory into a new plan, runRec, the field back
    barrier()
    t0 = time.perf_counter()
    e2e_steps = max(1, args.steps // 2)
    ep = 0
    for _ in range(e2e_steps):
        r2 = m3d.Reconstruction(T, *shape)
        r2.seed(w["seed"] + rank)
        r2.run(n, beta)
        ep += r2.errors().size
        r2.field()
        r2.close()
    barrier()
    esec = reduce(time.perf_counter() - t0, dist.ReduceOp.MAX if world > 1 else None)
    e2e = reduce(float(xyz) * ep, dist.ReduceOp.SUM if world > 1 else None) / esec
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = (json.load(open(peaks_path))["hbm_gbs"], "measured") if os.path.exists(peaks_path) \
        else (6650.0, "fallback")
    achieved = REC_BYTES[dom] * xyz / (dom_us * 1e-6) / 1e9
    pass_us = sum(per_kernel.values())
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_rec(w)
    if rank == 0:
        line = {
            "metric": "reconstruction voxel-passes/s (runRec: phase-retrieval passes x voxels, FP64 complex)",
            "value": value, "unit": "voxel-pass/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_max / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "c128", "data": "synthetic",
            "config": {"workload": args.workload, "desc": w["desc"], "grid": list(shape), "n": n, "beta": beta,
                       "passes_per_step": passes / args.steps,
                       "l2": "working set m + A (80 MB each) + normC (40 MB) exceeds L2; each pass streams them",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": None, "peak_source": peak_src, "kernel": REC_KERNELS[dom],
                         "bytes_per_voxel": REC_BYTES[dom], "kernel_us": dom_us, "per_kernel_us": per_kernel,
                         "pass_us": pass_us,
                         "pass_frac": sum(REC_BYTES) * xyz / (pass_us * 1e-6) / 1e9 / peak},
            "e2e": {"value": e2e, "unit": "voxel-pass/s", "h2d_bytes_per_step": 8 * xyz,
                    "d2h_bytes_per_step": 8 * xyz},
            "gpu_launches": launches,
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": "voxel-pass/s", "cores": 3, "kind": "reference",
                                    "sample": cpu["sample"]}
        print(json.dumps(line))


def run_reference_arm(args, w, rank, world):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if w["kind"] == "batch":
        r = cpu_reference_batch(w, args.steps, args.warmup, threads)
    elif w["kind"] == "2d":
        r = cpu_reference_2d(w, args.steps, args.warmup)
    elif w["kind"] == "rec":
        r = cpu_reference_rec(w)
        if r is not None:
            line = {
                "impl": "reference", "metric": "reconstruction voxel-passes/s (runRec: phase-retrieval passes x "
                "voxels, FP64 complex)", "value": r["value"], "unit": "voxel-pass/s", "n_gpus": args.gpus,
                "steps": 1, "warmup": 0, "ms_per_step": 1000 * r["seconds"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "c128", "data": "synthetic",
                "config": {"workload": args.workload, "desc": w["desc"]},
                "cpu_baseline": {"value": r["value"], "unit": "voxel-pass/s", "cores": 3, "kind": "reference",
                                 "sample": r["sample"]},
                "e2e": {"value": r["value"], "unit": "voxel-pass/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            }
            print(json.dumps(line))
            return
    else:
        r = cpu_reference(w, args.steps, args.warmup, threads, args.workload)
    if r is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libmat3d_ref.so not built"}))
        return
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * r["seconds"] / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"]},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": threads, "kind": "reference",
                         "sample": r["sample"]},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ----------------------------------------------------------------------------
def run_batch(args, w, rank, world, local, emit=True):
    """Batched homogenization: a step is the whole batch through m3d_batch_*.
    Returns the bench line (rank 0; printed when `emit`)."""
    import torch
    import torch.distributed as dist

    import mat3d_b200 as m3d
    from mat3d_b200 import rve as R

    desc = R.batch_rves(w["count"], seed0=rank * w["count"])
    t0 = time.perf_counter()
    members = [R.batch_member(*d) for d in desc]
    gen_s = time.perf_counter() - t0

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def reduce(x, op):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=op)
        return float(t.item())

    def make_batch(prec):
        bt = m3d.Batch(m3d.KIND_MECH, prec)
        bt.set_autotune(True)  # schedule per grid size picked by the autotuner (timed inside each step)
        for (g, mat, _), d in zip(members, desc):
            bt.add_mech((d[1],) * 3, mat, g)
        return bt

    def timed(prec, steps, warmup):
        bt = make_batch(prec)
        for _ in range(warmup):
            bt.homogenize(w["tol"])
        barrier()
        dev_ms = wall_ms = 0.0
        vi = sw = n64 = n32 = launches = kl = 0
        for _ in range(steps):
            Ce, _, _ = bt.homogenize(w["tol"])
            st = bt.stats()
            dev_ms += st["device_ms"]
            wall_ms += st["wall_ms"]
            vi += st["voxel_iters"]
            sw += st["sweeps"]
            n64 += st["sweeps_fp64"]
            n32 += st["sweeps_fp32"]
            launches += st["launches"]
            kl += st["kernel_launches"]
        barrier()
        bt.close()
        return dict(dev_ms=dev_ms, wall_ms=wall_ms, vi=vi, sweeps=sw, n64=n64, n32=n32, launches=launches,
                    kl=kl, Ce=Ce, groups=st["groups"], autotuned=st["autotuned"])

    def e2e_run(prec, steps):
        """Through the public API from host arrays: batch creation, adding every
        RVE (phase map and properties copied to the device) and the tensors
        copied back, inside the wall-clock region."""
        barrier()
        t = time.perf_counter()
        vi = 0
        for _ in range(steps):
            bt = make_batch(prec)
            bt.homogenize(w["tol"])
            vi += bt.stats()["voxel_iters"]
            bt.close()
        barrier()
        return vi, time.perf_counter() - t

    clk = ClockSampler(local)
    clk.start()
    res = timed(w["precision"], args.steps, args.warmup)
    clocks = clk.stop()
    ms_max = reduce(res["dev_ms"], dist.ReduceOp.MAX if world > 1 else None)
    vi_tot = reduce(float(res["vi"]), dist.ReduceOp.SUM if world > 1 else None)
    value = vi_tot / (ms_max / 1000.0)
    e2e_steps = max(1, args.steps // 2)
    evi, esec = e2e_run(w["precision"], e2e_steps)
    esec = reduce(esec, dist.ReduceOp.MAX if world > 1 else None)
    e2e_val = reduce(float(evi), dist.ReduceOp.SUM if world > 1 else None) / esec
    steps64 = max(1, args.steps // 2)
    r64 = timed("fp64", steps64, 1)
    ms64 = reduce(r64["dev_ms"], dist.ReduceOp.MAX if world > 1 else None)
    vi64 = reduce(float(r64["vi"]), dist.ReduceOp.SUM if world > 1 else None)
    dC = max(float(np.abs(a - b).max() / np.abs(b).max()) for a, b in zip(res["Ce"], r64["Ce"]))

    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    peak, peak_src = (json.load(open(peaks_path))["hbm_gbs"], "measured") if os.path.exists(peaks_path) \
        else (6650.0, "fallback")
    vox = sum(d[1] ** 3 for d in desc)
    alg = (res["n32"] * bytes_per_vi(6, 4) + res["n64"] * bytes_per_vi(6, 8)) / max(res["sweeps"], 1)
    achieved = vi_tot / world * alg / (res["dev_ms"] / 1000.0) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_batch(w, 1, 0, os.cpu_count() or 1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "batch512" if len(desc) == 512 else f"batch512 (first {len(desc)} RVEs)",
                       "desc": w["desc"], "rves": len(desc),
                       "voxels": vox, "voxel_load_cases": 6 * vox, "precision": w["precision"],
                       "residual_tol": w["tol"], "grid_sizes": sorted({d[1] for d in desc}),
                       "sweeps_per_entry": res["sweeps"] / args.steps / (6 * len(desc)),
                       "fp64_sweeps": res["n64"] / args.steps, "fp32_sweeps": res["n32"] / args.steps,
                       "launches_per_step": res["launches"] / args.steps, "groups": res["groups"],
                       "autotuned_groups": res["autotuned"],
                       "rve_generation_s": gen_s,
                       "l2": "inputs larger than L2 (tens of GB of state per grid-size group)",
                       "parallelism": f"replicas x{world}"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_source": peak_src,
                         "kernel": "whole batch (device time of the graph launches)",
                         "bytes_per_voxel_iter": alg},
            "fp64_solver": {"ms_per_step": ms64 / steps64, "value": vi64 / (ms64 / 1000.0),
                "time_to_solution_ratio": (ms64 / steps64) / (ms_max / args.steps),
                "max_rel_dCeff_vs_fp64": dC},
            "e2e": {"value": e2e_val, "unit": UNIT,
                    "h2d_bytes_per_step": sum(d[1] ** 3 * 4 + 2 * 56 for d in desc),
                    "d2h_bytes_per_step": len(desc) * 2 * 36 * 8},
            "gpu_launches": res["kl"],
            "clocks": clocks,
        }
        if cpu:
            line["cpu_baseline"] = {"value": cpu["value"], "unit": UNIT, "cores": os.cpu_count(),
                                    "kind": "reference", "sample": cpu["sample"]}
        if emit:
            print(json.dumps(line))
        return line
    return None


SERVE_SIZES = (32, 48, 64, 96, 128, 256)
EXTRA_BATCH_COUNT = 128
MAT_ELASTIC = np.array([[70e9, 0.2, 1e30, 0, 1, 0, 1e30], [3e9, 0.35, 1e30, 0, 1, 0, 1e30]])
MAT_J2 = np.array([[400e9, 0.2, 1e30, 0, 1, 0, 1e30], [70e9, 0.33, 100e6, 1e9, 1, 0, 1e30]])


def serve_requests(n, seed):
    """n request descriptors (kind, N) of the serving mix, seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        kind = ("elastic", "thermal", "j2")[rng.integers(3)]
        x = np.exp(rng.uniform(np.log(32), np.log(256)))
        N = min(SERVE_SIZES, key=lambda s: abs(np.log(s) - np.log(x)))
        out.append((kind, N))
    return out


def run_serve(args, w, rank, world, local, emit=True, levels_override=None):
    """Serving: a step is one offered-load level of the sweep.  Returns the
    bench line (rank 0; printed when `emit`)."""
    import torch

    import mat3d_b200 as m3d
    from mat3d_b200 import rve as R

    cache = {}

    def template(kind, N):
        if (kind, N) not in cache:
            if kind == "thermal":
                g, _ = R.ellipsoids(N, vf=0.30, aspect=3.0, n_target=100, seed=N)
            elif kind == "elastic":
                g, _ = R.spheres_rsa(N, radius=6.0, vf=0.20, seed=N)
            else:
                g, _ = R.lognormal_spheres(N, vf=0.15, median=5.0, sigma=0.4, rmin=3.0, rmax=10.0, seed=N)
            cache[(kind, N)] = g.ravel().astype(np.int32)
        return cache[(kind, N)]

    def submit(srv, kind, N):
        ph = template(kind, N)
        if kind == "thermal":
            return srv.submit(m3d.KIND_THERMAL, (N,) * 3, ph, [0, 0, 1.0], km=1.0, ki=100.0,
                              precision="fp32_refine", tol=w["tol"])
        if kind == "elastic":
            return srv.submit(m3d.KIND_MECH, (N,) * 3, ph, [1e-3, 0, 0, 0, 0, 0], mat=MAT_ELASTIC,
                              precision="fp32_refine", tol=w["tol"])
        return srv.submit(m3d.KIND_MECH, (N,) * 3, ph, [0.005 / 5, 0, 0, 0, 0, 0], mat=MAT_J2, behav=m3d.J2,
                          X0=[1, 0, 0, 0, 0, 0], nInc=5, precision="fp32", tol=w["tol"])

    t0 = time.perf_counter()
    for kind in ("elastic", "thermal", "j2"):
        for N in SERVE_SIZES:
            template(kind, N)
    gen_s = time.perf_counter() - t0
    srv = m3d.Server(workers=w["workers"])
    # warm-up: every (kind, N) once, so solvers and graphs exist (resident)
    warm = [submit(srv, k, N) for k in ("elastic", "thermal", "j2") for N in SERVE_SIZES][: max(args.warmup, 1) * 18]
    for t in warm:
        srv.wait(t)
    vox = lambda N: N ** 3

    def replay(descs, rate):
        """Submit descs with exponential inter-arrival times (rate req/s; inf: all at once)."""
        rng = np.random.default_rng(len(descs) + int(rate if np.isfinite(rate) else 0))
        torch.cuda.synchronize()
        start = time.perf_counter()
        tickets, t_next = [], start
        for kind, N in descs:
            if np.isfinite(rate):
                t_next += rng.exponential(1.0 / rate)
                dt = t_next - time.perf_counter()
                if dt > 0:
                    time.sleep(dt)
            tickets.append(submit(srv, kind, N))
        res = [srv.wait(t) for t in tickets]
        span = time.perf_counter() - start
        lat = np.array([r["latency_ms"] for r in res])
        vi = sum(vox(N) * r["sweeps"] for (k, N), r in zip(descs, res))
        bad = sum(1 for r in res if r["status"] not in (m3d.OK, m3d.NOT_CONVERGED))
        per_kind = {}
        for kind in ("elastic", "thermal", "j2"):
            lk = np.array([r["latency_ms"] for (k, _), r in zip(descs, res) if k == kind])
            if lk.size:
                per_kind[kind] = {"n": int(lk.size), "p50_ms": float(np.percentile(lk, 50)),
                                  "p99_ms": float(np.percentile(lk, 99))}
        return dict(span_s=span, p50_ms=float(np.percentile(lat, 50)), p99_ms=float(np.percentile(lat, 99)),
                    mean_ms=float(lat.mean()), req_per_s=len(descs) / span, voxel_iters_per_s=vi / span,
                    failed=bad, n=len(descs), per_kind=per_kind)

    descs = serve_requests(w["per_level"], seed=1000 + rank)
    clk = ClockSampler(local)
    clk.start()
    burst = replay(descs, float("inf"))
    cap = burst["req_per_s"]
    levels = []
    for f in (levels_override or w["levels"][: max(args.steps, 1)]):
        d = serve_requests(w["per_level"], seed=2000 + int(100 * f) + rank)
        r = replay(d, f * cap)
        r.update(offered_x_capacity=f, offered_req_per_s=f * cap)
        levels.append(r)
    clocks = clk.stop()
    st = srv.stats()
    srv.close()
    if rank == 0:
        top = levels[-1] if levels else burst
        line = {
            "metric": "serving p50/p99 latency at residual 1e-6 (and voxel-iters/s)", "value": top["p99_ms"],
            "unit": "ms (p99 latency)", "n_gpus": world, "steps": len(levels), "warmup": len(warm),
            "ms_per_step": 1000 * top["span_s"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": "serve", "desc": w["desc"], "requests_per_level": w["per_level"],
                       "sizes": list(SERVE_SIZES), "rounding": "N log-uniform on [32,256], nearest size in log scale",
                       "j2": "5 increments to 0.5% strain, FP32 sweeps", "workers": w["workers"],
                       "template_generation_s": gen_s, "parallelism": f"replicas x{world}"},
            "serving": {"capacity_burst": burst, "levels": levels, "peak_running": st["peak_running"],
                        "resident_solvers": st["resident_solvers"]},
            "e2e": {"value": top["voxel_iters_per_s"], "unit": UNIT,
                    "h2d_bytes_per_step": sum(4 * N ** 3 for _, N in descs),
                    "d2h_bytes_per_step": len(descs) * 12 * 8},
            "gpu_launches": None,
            "clocks": clocks,
        }
        if emit:
            print(json.dumps(line))
        return line
    return None


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="thermal128", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload only: skip the other configs' summaries")
    ap.add_argument("--profile-passes", action="store_true",
                    help="single-RVE workloads: K solves on the host-driven sweep loop with CUDA events around "
                         "every pass (the launch sequence an ncu capture sees), print the per-pass times; "
                         "batch512: the same for each grid-size group of its first 128 RVEs")
    args = ap.parse_args()
    w = WORKLOADS[args.workload]

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference_arm(args, w, rank, world)
        return

    import torch
    import torch.distributed as dist

    import mat3d_b200 as m3d

    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120))
    if args.profile_passes and w["kind"] == "batch":
        print(json.dumps(profile_batch_groups(args, w)))
        return
    if w["kind"] in ("batch", "serve", "2d", "rec"):
        {"batch": run_batch, "serve": run_serve, "2d": run_2d, "rec": run_rec}[w["kind"]](args, w, rank, world, local)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.profile_passes:
        print(json.dumps(profile_passes(args, w)))
        return
    extras = args.workload == "thermal128" and world == 1 and not args.no_extras
    line = run_single(args, w, args.workload, rank, world, local, emit=not extras)
    if extras:
        line["other_configs"] = run_extras(args, rank, world, local)
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


def profile_batch_groups(args, w):
    """Per-pass CUDA-event times of the batched homogenization's grid-size
    groups: the batch workload's generator with its first EXTRA_BATCH_COUNT
    RVEs, each group one multi-RVE solver (every RVE with its 6 load cases as
    entries) run once with the host-driven loop.  Per group: entry sweeps, the
    launch rounds (trips) and the summed pass times of the FP32 and FP64
    sweeps."""
    import mat3d_b200 as m3d
    from mat3d_b200 import rve as R
    names = ["z_forward", "y_forward", "x_turnaround", "y_inverse", "z_inverse"]
    desc = R.batch_rves(EXTRA_BATCH_COUNT)
    groups = {}
    for d in desc:
        groups.setdefault(d[1], []).append(d)
    out = {"workload": args.workload, "rves": len(desc), "precision": w["precision"], "tol": w["tol"], "groups": {}}
    for N, ds in sorted(groups.items()):
        mem = [R.batch_member(*d) for d in ds]
        s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.ELASTIC, w["precision"], nrve=len(ds), nload=6)
        for r, (g, mat, _) in enumerate(mem):
            s.set_material_mech(mat, g, rve=r)
        s.set_profiling(True)
        s.homogenize(w["tol"])
        p, st = s.profile(), s.stats()
        r = {"rves": len(ds), "entries": 6 * len(ds), "entry_sweeps_fp32": st["sweeps_fp32"],
             "entry_sweeps_fp64": st["sweeps_fp64"]}
        for tag in ("fp32", "fp64"):
            if p[f"n_{tag}"]:
                r[f"trips_{tag}"] = p[f"n_{tag}"]
                r[f"ms_{tag}"] = p[f"ms_{tag}"]
                r[f"pass_ms_{tag}"] = {names[q]: p[f"pass_ms_{tag}"][q] for q in range(5)}
        out["groups"][N] = r
        s.close()
    return out


def profile_passes(args, w):
    """K solves of a single-RVE workload with per-pass CUDA events (host-driven
    loop); per sweep and per pass device times of the FP32 and FP64 sweeps."""
    import mat3d_b200 as m3d
    N = w["N"]
    rve, _ = make_rve(w)
    j2 = w.get("behav") == "ep"
    if w["kind"] == "thermal":
        s = m3d.Solver(m3d.KIND_THERMAL, N, N, N, m3d.ELASTIC, w["precision"], 1)
        s.set_material_thermal(w["km"], w["ki"], rve)
    else:
        s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.J2 if j2 else m3d.ELASTIC, w["precision"], 1)
        s.set_material_mech(MAT_J2 if j2 else MAT_ELASTIC, rve)
    E = np.array(w["E"], float)
    X0 = np.array(w["X0"], float) if "X0" in w else None
    s.set_profiling(True)
    for _ in range(max(args.steps, 1)):
        s.set_load(E, X0)
        s.run(w["tol"], w["tol"], w.get("nInc", 1), m3d.CRIT_RESIDUAL)
    p, st = s.profile(), s.stats()
    names = PASS_NAMES_2 if st["passes_per_sweep"] == 2 else PASS_NAMES
    out = {"workload": args.workload, "solves": max(args.steps, 1), "passes_per_sweep": st["passes_per_sweep"],
           "sweeps_fp32": p["n_fp32"], "sweeps_fp64": p["n_fp64"]}
    for tag, n, ms, pms in (("fp32", p["n_fp32"], p["ms_fp32"], p["pass_ms_fp32"]),
                            ("fp64", p["n_fp64"], p["ms_fp64"], p["pass_ms_fp64"])):
        if n:
            out[f"sweep_us_{tag}"] = 1000 * ms / n
            # the refinement's FP64 defect sweeps run the five passes
            nm = names if (tag == "fp32" or w["precision"] == "fp64") else PASS_NAMES
            out[f"pass_us_{tag}"] = {nm[q]: 1000 * pms[q] / n for q in range(5) if nm[q]}
    s.close()
    return out


def run_extras(args, rank, world, local):
    """The rest of the metric beside the headline line (run after its timed
    region, 1 GPU): serving p50/p99 at 0.5x and 1.0x of the measured capacity,
    the batched homogenization (a stated reduced RVE count), config 0
    (elastic64) and config 2 (j2_256) rates.  Each entry summarises the line
    that `--workload <name>` prints in full."""
    out = {}
    a = argparse.Namespace(**vars(args))
    a.no_cpu_baseline = True

    def keep(line, keys):
        return {k: line[k] for k in keys if k in line}

    t = time.perf_counter()
    a.steps, a.warmup = 2, 1
    ln = run_serve(a, WORKLOADS["serve"], rank, world, local, emit=False, levels_override=(0.5, 1.0))
    if ln:
        sv = ln["serving"]
        out["serve"] = {"capacity_req_per_s": sv["capacity_burst"]["req_per_s"],
                        "capacity_burst": keep(sv["capacity_burst"], ("p50_ms", "p99_ms", "per_kind", "n")),
                        "levels": [keep(l, ("offered_x_capacity", "offered_req_per_s", "p50_ms", "p99_ms", "per_kind",
                                            "req_per_s", "voxel_iters_per_s", "n", "failed")) for l in sv["levels"]],
                        "config": ln["config"], "wall_s": time.perf_counter() - t}
    t = time.perf_counter()
    wb = dict(WORKLOADS["batch512"], count=EXTRA_BATCH_COUNT)
    a.steps, a.warmup = 1, 1
    ln = run_batch(a, wb, rank, world, local, emit=False)
    if ln:
        out["batch"] = {"rves": ln["config"]["rves"], "value": ln["value"], "unit": UNIT,
                        "ms_per_batch": ln["ms_per_step"], "fp64_solver": ln["fp64_solver"],
                        "roofline_frac": ln["roofline"]["frac"], "e2e": ln["e2e"]["value"],
                        "config": ln["config"], "wall_s": time.perf_counter() - t,
                        "note": f"the batch512 workload's generator and settings with its first "
                                f"{EXTRA_BATCH_COUNT} RVEs (bench.py --workload batch512 runs all 512)"}
    for name, steps, warm in (("elastic64", 5, 2), ("j2_256", 1, 0)):
        t = time.perf_counter()
        a.steps, a.warmup = steps, warm
        ln = run_single(a, WORKLOADS[name], name, rank, world, local, emit=False, light=True)
        if ln:
            out[name] = {"value": ln["value"], "unit": UNIT, "ms_per_solve": ln["ms_per_step"],
                         "precision": ln["config"]["precision"], "sweeps_per_solve": ln["config"]["sweeps_per_solve"],
                         "fp64_solver": ln.get("fp64_solver"), "err_vs_fp64": ln.get("err_vs_fp64"),
                         "roofline_solve_frac": ln["roofline_solve"]["frac"], "desc": WORKLOADS[name]["desc"],
                         "wall_s": time.perf_counter() - t}
    return out


def run_single(args, w, name, rank, world, local, emit=True, light=False):
    """One RVE solve per step (thermal128, elastic64, j2_256).  Returns the
    bench line (rank 0; printed when `emit`).  `light`: no per-pass profile
    solve and no end-to-end run (used for the summaries of other configs)."""
    import torch
    import torch.distributed as dist

    import mat3d_b200 as m3d

    N = w["N"]
    V = N ** 3
    c = 3 if w["kind"] == "thermal" else 6
    rve, meta = make_rve(w, seed=rank)
    j2 = w.get("behav") == "ep"
    mat = MAT_J2 if j2 else MAT_ELASTIC
    E = np.array(w["E"], float)
    X0 = np.array(w["X0"], float) if "X0" in w else None
    nInc = w.get("nInc", 1)

    def make_solver(prec):
        if w["kind"] == "thermal":
            s = m3d.Solver(m3d.KIND_THERMAL, N, N, N, m3d.ELASTIC, prec, 1)
            s.set_material_thermal(w["km"], w["ki"], rve)
        else:
            s = m3d.Solver(m3d.KIND_MECH, N, N, N, m3d.J2 if j2 else m3d.ELASTIC, prec, 1)
            s.set_material_mech(mat, rve)
        s.set_load(E, X0)
        return s

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def sum_over_ranks(x):
        if world == 1:
            return x
        t = torch.tensor([x], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.SUM)
        return float(t.item())

    # e2e host buffers in pinned memory: the phase map the step uploads and the
    # field it reads back (written in place by the API, no extra host copy)
    rve_pinned = torch.from_numpy(np.ascontiguousarray(rve, np.int32)).pin_memory().numpy()
    host_out = torch.empty(c * V, dtype=torch.float64).pin_memory().numpy()

    def timed_solves(s, steps, warmup, e2e=False, profile=False):
        """K solves bracketed by barrier + synchronize; CUDA events on the solver stream."""
        stream = torch.cuda.ExternalStream(s.stream_ptr())
        for _ in range(warmup):
            if e2e:
                if w["kind"] == "thermal":
                    s.set_material_thermal(w["km"], w["ki"], rve_pinned)
                else:
                    s.set_material_mech(mat, rve_pinned)
            s.set_load(E, X0)
            s.run(w["tol"], w["tol"], nInc, m3d.CRIT_RESIDUAL)
            if e2e:
                s.field(m3d.FIELD_STRAIN, out=host_out)
        if profile:
            s.set_profiling(True)
        l0 = s.stats()["kernel_launches"]
        barrier()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        sweeps = n64 = n32 = 0
        for _ in range(steps):
            if e2e:
                if w["kind"] == "thermal":
                    s.set_material_thermal(w["km"], w["ki"], rve_pinned)
                else:
                    s.set_material_mech(mat, rve_pinned)
            s.set_load(E, X0)
            s.run(w["tol"], w["tol"], nInc, m3d.CRIT_RESIDUAL)
            if e2e:  # the field copy back overlaps the next step; the last one ends inside the region
                s.field_async(host_out, m3d.FIELD_STRAIN)
            st = s.stats()
            sweeps += st["sweeps"]
            n64 += st["sweeps_fp64"]
            n32 += st["sweeps_fp32"]
        if e2e:
            s.wait_field()
        ev1.record(stream)
        barrier()
        ms = ev0.elapsed_time(ev1)
        prof = s.profile() if profile else None
        if profile:
            s.set_profiling(False)
        launches = s.stats()["kernel_launches"] - l0
        return dict(ms=ms, sweeps=sweeps, n64=n64, n32=n32, st=st, prof=prof, launches=launches)

    # ---- main arm: the workload's precision, device-resident inputs --------
    s = make_solver(w["precision"])
    clk = ClockSampler(local)
    clk.start()
    res = timed_solves(s, args.steps, args.warmup)
    clocks = clk.stop()
    ms_max = max_over_ranks(res["ms"])
    sweeps_tot = sum_over_ranks(res["sweeps"])
    value = V * sweeps_tot / (ms_max / 1000.0)
    # per-sweep device times (events around every sweep; host-driven loop)
    pres = None if light else timed_solves(s, 1, 0, profile=True)

    # ---- e2e through the public API with host buffers -----------------------
    e2e_val = None
    if not light:
        e2e = timed_solves(s, max(2, args.steps // 2), 1, e2e=True)
        e2e_ms = max_over_ranks(e2e["ms"])
        e2e_val = V * sum_over_ranks(e2e["sweeps"]) / (e2e_ms / 1000.0)

    # ---- plain FP64 GPU solver on the same workload (comparison) -----------
    s64 = make_solver("fp64")
    steps64 = 1 if light else max(2, args.steps // 2)
    r64 = timed_solves(s64, steps64, 0 if light else 1)
    ms64 = max_over_ranks(r64["ms"])
    val64 = V * sum_over_ranks(r64["sweeps"]) / (ms64 / 1000.0)

    # ---- roofline: one sweep (5 FFT passes + fused physics) is the unit -----
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        peak = json.load(open(peaks_path))["hbm_gbs"]
        peak_src = "measured"
    else:
        peak, peak_src = 6650.0, "fallback"
    pr = pres["prof"] if pres else {"ms_fp32": 0, "n_fp32": 0, "ms_fp64": 0, "n_fp64": 0,
                                   "pass_ms_fp32": [0] * 5, "pass_ms_fp64": [0] * 5}
    # J2 adds the previous strain and stress and the plastic strain: 8cw + w + 1
    b32, b64 = (8 * c * 4 + 4 + 1, 8 * c * 8 + 8 + 1) if j2 else (bytes_per_vi(c, 4), bytes_per_vi(c, 8))
    # whole timed region: algorithmic bytes of all its sweeps / its device time
    alg_bytes = V * (res["n32"] * b32 + res["n64"] * b64)
    achieved = alg_bytes / (res["ms"] / 1000.0) / 1e9 if res["ms"] > 0 else None
    sweep_fp32_us = 1000 * pr["ms_fp32"] / pr["n_fp32"] if pr["n_fp32"] else None
    sweep_fp64_us = 1000 * pr["ms_fp64"] / pr["n_fp64"] if pr["n_fp64"] else None
    # dominant kernel: the pass with the largest share of the profiled solve's
    # device time (events around every pass), its algorithmic bytes per launch
    # = the pass's own inputs and outputs
    kern = None
    if not j2:
        fp32 = pr["n_fp32"] > 0
        n = pr["n_fp32"] if fp32 else pr["n_fp64"]
        pms = pr["pass_ms_fp32"] if fp32 else pr["pass_ms_fp64"]
        if n and sum(pms) > 0:
            p = int(np.argmax(pms))
            wb = 4 if fp32 else 8
            two = pres["st"]["passes_per_sweep"] == 2
            names, kernels = (PASS_NAMES_2, PASS_KERNELS_2) if two else (PASS_NAMES, PASS_KERNELS)
            forcing = w["precision"] == "fp32_refine" and fp32  # inner sweeps read the FP32 defect
            pb = pass_bytes(c, wb, N, forcing, two)[p]
            us = 1000 * pms[p] / n
            tr = MEASURED_TRAFFIC.get((name, names[p], wb))
            kern = {"bound": "hbm", "kernel": kernels[p], "pass": names[p],
                    "achieved": pb / (us * 1e-6) / 1e9, "peak": peak, "unit": "GB/s",
                    "frac": pb / (us * 1e-6) / 1e9 / peak, "traffic": tr[0] if tr else None,
                    "traffic_source": tr[1] if tr else None, "peak_source": peak_src,
                    "bytes_per_launch": pb, "launch_us": us, "share_of_sweep": pms[p] / sum(pms),
                    "passes_per_sweep": 2 if two else 5,
                    "pass_us": {names[q]: 1000 * pms[q] / n for q in range(5) if names[q]}}

    # ---- error of the timed solve against the FP64 GPU solve at 1e-10 ------
    # (the FP64 GPU solver is pinned to the reference's own solver at these
    # configurations by tests/test_gpu_configs.py)
    err = None
    if w["precision"] != "fp64":
        f_lo = s.field(m3d.FIELD_STRAIN).copy()
        m_lo = s.means()[1]
        # a tighter FP64 reference solve, except in the light summaries, which
        # compare with the FP64 solve just timed (same tolerance)
        ref_tol = w["tol"] if light else 1e-10
        if not light:
            s64.set_load(E, X0)
            s64.run(ref_tol, ref_tol, nInc, m3d.CRIT_RESIDUAL)
        f_hi = s64.field(m3d.FIELD_STRAIN)
        m_hi = s64.means()[1]
        err = {"field_rel_l2": float(np.linalg.norm(f_lo - f_hi) / np.linalg.norm(f_hi)),
               "mean_stress_like_max_rel": float(np.abs(m_lo - m_hi).max() / np.abs(m_hi).max()),
               "against": f"FP64 GPU solve of the same RVE and load to residual {ref_tol:g}",
               "what": ("the last timed-configuration solve's gradient field (rel-L2 over all voxels) and its "
                        "mean flux = the loaded column of K_eff" if w["kind"] == "thermal" else
                        "the last timed-configuration solve's strain field and its mean stress")}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_entry(w, name)

    if rank == 0:
        st = res["st"]
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None,
            "dtype": "f32+f64" if w["precision"] == "fp32_refine" else ("f32" if w["precision"] == "fp32" else "f64"),
            "data": "synthetic",
            "config": {"workload": name, "desc": w["desc"], "grid": [N, N, N],
                       "precision": w["precision"], "residual_tol": w["tol"],
                       "sweeps_per_solve": res["sweeps"] / args.steps,
                       "fp64_sweeps_per_solve": res["n64"] / args.steps,
                       "fp32_sweeps_per_solve": res["n32"] / args.steps,
                       "residual_reached": st["residual"], "rve": meta,
                       "l2": ("a step is one complete solve; its state (FP64 field, FP32 correction and "
                              "defect, spectrum: 152 MB) exceeds L2, the FP32 inner sweeps' own working set "
                              "(78 MB) is reused from L2 by the algorithm")
                             if w["kind"] == "thermal" else
                             ("a step is one complete solve; 64^3 working set is L2-resident by design" if N <= 64
                              else "a step is one complete solve; working set exceeds L2"),
                       "parallelism": f"replicas x{world}"},
            "roofline": kern,
            "roofline_solve": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                               "frac": (achieved / peak) if achieved else None,
                               "peak_source": peak_src,
                               "kernel": "the timed solves (one graph launch each: sweeps of fused FFT passes)",
                               "bytes_per_voxel_iter": {"fp32": b32, "fp64": b64},
                               "sweep_us": {"fp32": sweep_fp32_us, "fp64": sweep_fp64_us}},
            "fp64_solver": {"value": val64, "unit": UNIT, "ms_per_solve": ms64 / steps64,
                            "sweeps_per_solve": r64["sweeps"] / steps64,
                            "time_to_solution_ratio": (ms64 / steps64) / (ms_max / args.steps)},
            "e2e": None if e2e_val is None else {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": 4 * V + 256,
                                                 "d2h_bytes_per_step": c * V * 8,
                                                 "how": "per step: the int32 phase map from pinned host memory "
                                                        "(set_material), the load, the solve, the FP64 field "
                                                        "copied back with m3d_get_field_async (overlapping the "
                                                        "next step; the last copy ends inside the timed region)"},
            "gpu_launches": res["launches"],
            "clocks": clocks,
        }
        if line["roofline"] is None:  # J2 (or no profile): the whole-solve model
            line["roofline"] = dict(line["roofline_solve"], traffic=None)
        if err:
            line["err_vs_fp64"] = err
        if cpu:
            line["cpu_baseline"] = cpu
        if emit:
            print(json.dumps(line))
        return line
    return None


if __name__ == "__main__":
    main()
