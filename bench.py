"""Benchmark of the brute-force reconstruction hot path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload (one "step" = one full reconstruction): 3-D stack of spirals,
64x64x16 image, 4 coils, 16 kz partitions x 4 interleaves x 1024 samples
(M = 65536), field map, exact 3-D phase, TV (lambda 1e-3, 10 reweighting
passes, the reference's -tv default), 16 CG iterations per pass (15 updates,
the reference's cg_num-1).  Inputs are seeded synthetic data (no public
dataset); the k-space data is simulated by this library's exact-phase NUDFT
plus complex Gaussian noise at 40 dB SNR.

Metric: seconds per reconstruction (lower is better).  `value` has every
input resident in HBM; `e2e` goes through the same C-ABI call with pinned
HOST buffers, so the host->device copies of the inputs and the device->host
copy of the image are inside the timed region.  The L2 is flushed (a 256 MiB
write) before every timed step.

Multi-GPU: the path has no exchange step; each rank reconstructs its own
slices (replicas, weak scaling) and `value` = elapsed (max over ranks) /
reconstructions of all ranks.
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
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

BF3D = "bf3d_64x64x16"
METRIC = "s/recon (brute-force 3-D CG, 64x64x16, 4 coils, M=65536, 16 CG x 10 TV)"
UNIT = "s/recon"
CG_NUM, TV_NUM, LAMBDA = 16, 10, 1e-3


def _replicas():
    from __graft_entry__ import load_package
    load_package()
    from impatient_mri_b200 import replicas
    return replicas


def dist_setup():
    """One process per GPU (torchrun environment); NCCL process group for the
    host-side barrier and the max-over-ranks timing only."""
    return _replicas().init(timeout_s=300)


def barrier(ws):
    _replicas().barrier(ws)


def max_over_ranks(v, ws):
    return _replicas().max_over_ranks(v, ws)


class ClockSampler:
    """nvidia-smi clock / throttle sampling during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for n, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


def ncu_traffic(name="nudft_bf3d_64x64x16.md", key="traffic_bytes_per_launch:"):
    """DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum of one ncu
    capture) per launch / application from a committed ncu summary, if any."""
    p = ROOT / "profiles" / name
    if not p.exists():
        return None
    for ln in p.read_text().splitlines():
        if ln.strip().startswith(key):
            try:
                return float(ln.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


def applies_per_recon():
    return TV_NUM * (1 + 2 * (CG_NUM - 1))


GOLDEN = ROOT / "tests" / "golden"


def timed_fixture(name):
    """FP64 results on the timed inputs (tests/golden/gen_timed_golden.py), or
    None when the file is absent."""
    p = GOLDEN / f"{name}_timed.npz"
    return dict(np.load(p)) if p.exists() else None


def case_checksum(case, keys=("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm", "sens", "x_true")):
    import hashlib
    h = hashlib.sha256()
    for k in keys:
        h.update(np.ascontiguousarray(case[k]).tobytes())
    return h.hexdigest()


def rel_l2(a, b):
    a = np.asarray(a, np.complex128).ravel()
    b = np.asarray(b, np.complex128).ravel()
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


# ------------------------------------------------------------ reference --

def cpu_reference_sample(case, sample_k: int, sample_v: int = 512):
    """Times the reference's own CPU NUDFT pair (FP32 + OpenMP build of
    kernels/ftCpu.cpp through parallelFtCpu / parallelIftCpu) on bounded
    samples and extrapolates to one reconstruction: the forward over
    `sample_k` samples against all voxels, the adjoint over all samples for
    `sample_v` voxels (each keeps the loop the reference parallelises whole),
    each scaled to a full apply; a reconstruction is, per TV pass, 1 + (cg_num
    - 1) forward and cg_num - 1 adjoint applies.  The reference brute force has
    only the 2-D phase (z constant), so the per-pair work is the same as the
    3-D formula's but the values are not the 3-D ones."""
    import oracle
    M, N = case["M"], case["N"]
    C = np.asarray(case["sens"]).size // N
    sub = dict(case, kx=case["kx"][:sample_k], ky=case["ky"][:sample_k],
               kz=case["kz"][:sample_k], t=case["t"][:sample_k])
    vsel = np.linspace(0, N - 1, sample_v).astype(np.int64)
    sens = np.asarray(case["sens"]).reshape(C, N)
    adj = dict(case, ix=case["ix"][vsel], iy=case["iy"][vsel], iz=case["iz"][vsel],
               fm=case["fm"][vsel], sens=sens[:, vsel])
    d = np.ones((C, M), np.complex64)
    t0 = time.perf_counter()
    oracle.ref_parallel_ft(case["x_true"], sub, kind="bf32_omp")
    t1 = time.perf_counter()
    oracle.ref_parallel_ift(d, adj, kind="bf32_omp")
    t2 = time.perf_counter()
    f_full, a_full = (t1 - t0) * M / sample_k, (t2 - t1) * N / sample_v
    n_f = TV_NUM * (1 + (CG_NUM - 1))
    n_a = TV_NUM * (CG_NUM - 1)
    return f_full * n_f + a_full * n_a, (f_full, a_full)


# zero-start CG updates to NRMSE <= 1e-3 at the warm-start configuration, measured
# by this build's GPU arm on held-out phantoms (mean 45.25 over 8, 44-47); the
# reference arm runs on the host alone and takes the count from there
WARM_ZERO_UPDATES = 45


def warm_case():
    """The warm-start configuration's trajectory, coils and voxel grid in
    numpy, drawn from the same seeded generator calls as learn.ToepProblem."""
    load_pkg = __import__("__graft_entry__").load_package
    load_pkg()
    from impatient_mri_b200 import synth
    n, C = 512, 32
    rng = np.random.default_rng(1005)
    kx, ky, t = synth.spiral(24, 4096, n / 2 - 0.05, rng)
    sens = np.stack([synth.to_voxel_order(m) for m in synth.coil_maps((n, n), C, rng, ring=True)])
    ix, iy, iz = synth.grid_positions(n, n, 1)
    img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 8, np.random.default_rng(3005)))
    return dict(kx=kx, ky=ky, kz=np.zeros_like(kx), t=t, ix=ix, iy=iy, iz=iz,
                fm=np.zeros(n * n, np.float32), sens=sens.astype(np.complex64), x=img,
                M=kx.size, N=n * n, C=C)


def run_reference_warm(args):
    """Reference arm of the warm-start configuration: the reference's only
    CPU reconstruction is bruteForceCpu, whose CG makes one F and one F^H
    (parallelFtCpu / parallelIftCpu, kernels/parImagingCpu.cpp:84-147) per
    update plus the initial F^H d.  Each step times the reference's FP32
    OpenMP build of both on bounded samples that keep each loop's inner
    dimension whole (the forward over a subset of the samples against all
    voxels, the adjoint over all samples for a subset of the voxels: the
    reference parallelises the inner loop, so shortening it would time
    thread start-up instead of arithmetic), extrapolates each to the full
    problem and to 1 + 2 x 45 applies (45 = zero-start updates to NRMSE <= 1e-3
    on this configuration); the CG vector work (length-N) is below 1e-6 of
    the NUDFT work and not timed."""
    import oracle
    if not oracle.ref_available("bf32_omp"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU build oracle/_ref missing"}))
        return 0
    c = warm_case()
    ks, kv = 64, 256  # forward: samples; adjoint: voxels
    M, N, C = c["M"], c["N"], c["C"]
    fwd = dict(c, kx=c["kx"][:ks], ky=c["ky"][:ks], kz=c["kz"][:ks], t=c["t"][:ks])
    vsel = np.linspace(0, N - 1, kv).astype(np.int64)
    adj = dict(c, ix=c["ix"][vsel], iy=c["iy"][vsel], iz=c["iz"][vsel], fm=c["fm"][vsel],
               sens=c["sens"][:, vsel])
    rng = np.random.default_rng(0)
    d = (rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M)))
    vals, tf, ta = [], [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.ref_parallel_ft(c["x"], fwd, kind="bf32_omp")
        t1 = time.perf_counter()
        oracle.ref_parallel_ift(d, adj, kind="bf32_omp")
        t2 = time.perf_counter()
        f_full, a_full = (t1 - t0) * M / ks, (t2 - t1) * N / kv
        if i >= args.warmup:
            vals.append(a_full * (1 + WARM_ZERO_UPDATES) + f_full * WARM_ZERO_UPDATES)
            tf.append(f_full)
            ta.append(a_full)
    value = float(np.mean(vals))
    cores = os.cpu_count()
    sample = (f"reference parallelFtCpu (FP32, OpenMP {cores} threads) on {ks} of {M} samples x "
              f"{N} voxels x {C} coils and parallelIftCpu on {M} samples x {kv} of {N} voxels x "
              f"{C} coils per step, extrapolated to one full apply each (F {np.mean(tf):.0f} s, "
              f"F^H {np.mean(ta):.0f} s) and to 1 + 2 x {WARM_ZERO_UPDATES} applies per recon "
              f"(zero-start CG to NRMSE <= 1e-3); spread over {len(vals)} steps: "
              f"{min(vals):.0f} .. {max(vals):.0f} s (std {np.std(vals) / value:.1%})")
    line = {"impl": "reference", "metric": WARM_METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{WARM} (plain CG: the reference has no learned part)",
                       "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference_c1(args):
    """Reference arm of the 2-D one-coil configuration: the reference's own
    bruteForceCpu (FP32 OpenMP build), full reconstructions, timed."""
    import oracle
    if not oracle.ref_available("bf32_omp"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU build oracle/_ref missing"}))
        return 0
    fix = timed_fixture(C1)
    load_pkg = __import__("__graft_entry__").load_package
    load_pkg()
    from impatient_mri_b200 import synth
    case = synth.make_case(C1, forward=None)
    if fix is None:
        print(json.dumps({"impl": "reference", "unavailable": "fixture bf2d_64_timed.npz absent"}))
        return 0
    for k_ in ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm", "sens", "kdata"):
        case[k_] = fix[k_]
    o = case["opts"]
    vals = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        oracle.ref_bf_cg(case, kind="bf32_omp", cg_num=o["cg_num"], lam=o["fd_penalizer"],
                         tv=True, tv_num=o["tv_num"])
        if i >= args.warmup:
            vals.append(time.perf_counter() - t0)
    value = float(np.mean(vals))
    line = {"impl": "reference", "metric": C1_METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": C1, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": os.cpu_count(),
                             "kind": "reference",
                             "sample": f"full reference bruteForceCpu recon per step (FP32, "
                                       f"OpenMP), {min(vals):.2f} .. {max(vals):.2f} s"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_reference(args, ws, rank):
    if rank != 0:
        return 0
    if args.workload == WARM:
        return run_reference_warm(args)
    if args.workload == C1:
        return run_reference_c1(args)
    import oracle
    load_pkg = __import__("__graft_entry__").load_package
    load_pkg()
    from impatient_mri_b200 import synth
    case = synth.make_case(BF3D)
    if not oracle.ref_available("bf32_omp"):
        print(json.dumps({"impl": "reference",
                          "unavailable": "reference CPU build oracle/_ref missing"}))
        return 0
    sample_k, sample_v = 8192, 8192
    cores = os.cpu_count()
    vals, fa = [], []
    for i in range(args.warmup + args.steps):
        v, per = cpu_reference_sample(case, sample_k, sample_v)
        if i >= args.warmup:
            vals.append(v)
            fa.append(per)
    value = float(np.mean(vals))
    f_full, a_full = np.mean(fa, axis=0)
    sample = (f"reference parallelFtCpu (FP32, OpenMP {cores} threads) on {sample_k} of "
              f"{case['M']} samples x {case['N']} voxels x 4 coils and parallelIftCpu on all "
              f"samples x {sample_v} voxels per step, each extrapolated to a full apply "
              f"(F {f_full:.1f} s, F^H {a_full:.1f} s), x 160 F + 150 F^H per recon; spread "
              f"over {len(vals)} steps {min(vals):.0f} .. {max(vals):.0f} s; CG vector work "
              f"(length N, < 1e-5 of the NUDFT work) not counted")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": BF3D, "l2": "n/a (CPU)"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ------------------------------------------------------------------ ours --

def run_ours(args, ws, rank, local, emit=True):
    """The brute-force 3-D configuration; emit=False returns the line's dict
    (the headline line nests it) instead of printing it."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import synth
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = pkg.Context(local)

    case = synth.make_case(BF3D, seed=1002 + rank)
    M, N, C = case["M"], case["N"], case["num_coil"]
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32))
    D = {k: f32(case[k]).to(dev) for k in ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm")}
    D["sr"], D["si"] = f32(case["sens"].real).to(dev), f32(case["sens"].imag).to(dev)
    fix = timed_fixture(BF3D)
    if fix is not None and str(fix["checksum"]) != case_checksum(case):
        fix = None  # another seed (rank > 0) or generator: no FP64 result for these inputs
    if fix is not None:
        # k-space data simulated by the FP64 oracle + 40 dB noise (the fixture's)
        y = np.asarray(fix["kdata"], np.complex64).reshape(C, M)
    else:
        # simulated k-space: exact-phase NUDFT of the phantom + 40 dB noise
        yr = torch.zeros(C * M, device=dev)
        yi = torch.zeros(C * M, device=dev)
        pkg.parallelFtGpu(ctx, yr, yi, f32(case["x_true"].real).to(dev),
                          f32(case["x_true"].imag).to(dev), D["kx"], D["ky"], D["kz"], D["ix"],
                          D["iy"], D["iz"], D["fm"], D["t"], M, N, D["sr"], D["si"], C, 1)
        y = yr.cpu().numpy() + 1j * yi.cpu().numpy()
        y = synth.add_noise(y, 40.0, np.random.default_rng(7 + rank)).astype(np.complex64)
    D["yr"], D["yi"] = f32(y.real).to(dev), f32(y.imag).to(dev)
    xr = torch.zeros(N, device=dev)
    xi = torch.zeros(N, device=dev)
    nx, ny, nz = case["dims"]
    opts = pkg.bf_options(cg_num=CG_NUM, fd_penalizer=LAMBDA, tv=True, tv_num=TV_NUM,
                          tv_eps=1e-6, use_z=1, dims=(nx, ny, nz))

    def recon(x_r, x_i, src):
        pkg.bruteForceGpu(ctx, opts, x_r, x_i, src["yr"], src["yi"], src["kx"], src["ky"],
                          src["kz"], src["ix"], src["iy"], src["iz"], src["fm"], src["t"],
                          src["sr"], src["si"], M, N, C, 1)

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    for _ in range(args.warmup):
        xr.zero_(); xi.zero_()
        recon(xr, xi, D)
    torch.cuda.synchronize()

    # ---- device-resident timing (value) ----
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = 0
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            xr.zero_(); xi.zero_()
            flush.fill_(float(s))
            ev[s][0].record()
            recon(xr, xi, D)
            ev[s][1].record()
            launches += ctx.launch_count()
    torch.cuda.synchronize()
    barrier(ws)
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_s = max_over_ranks(sum(step_ms) / 1e3, ws)
    value = total_s / (args.steps * ws)

    # ---- end to end through the C-ABI with pinned host buffers (e2e) ----
    H = {k: v.cpu().pin_memory() for k, v in D.items()}
    hxr = torch.zeros(N).pin_memory()
    hxi = torch.zeros(N).pin_memory()
    h2d = sum(v.numel() * 4 for v in H.values()) + 2 * N * 4
    d2h = 2 * N * 4
    recon(hxr, hxi, H)  # warm
    e2e_ms = []
    barrier(ws)
    torch.cuda.synchronize()
    for s in range(args.steps):
        hxr.zero_(); hxi.zero_()
        flush.fill_(float(s))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        recon(hxr, hxi, H)  # synchronous: returns after the image is back in host memory
        e2e_ms.append((time.perf_counter() - t0) * 1e3)
    barrier(ws)
    e2e_total = max_over_ranks(sum(e2e_ms) / 1e3, ws)
    e2e_value = e2e_total / (args.steps * ws)

    # ---- roofline of the dominant kernel (per-launch CUDA events) ----
    ctx.profile(True)
    xr.zero_(); xi.zero_()
    recon(xr, xi, D)
    prof = ctx.profile_read()
    ctx.profile(False)
    fwd_ms, fwd_n = prof["forward"]
    adj_ms, adj_n = prof["adjoint"]
    avg_launch_s = (fwd_ms + adj_ms) / max(fwd_n + adj_n, 1) / 1e3
    pairs = M * N
    flop_launch = 2.0 * (4 + 4 * C) * pairs  # 3-D phase (4 FMA) + 4 FMA per coil, per pair
    achieved = flop_launch / avg_launch_s / 1e12
    fp32_peak, sfu_peak = pkg.measure_alu_peaks(local)
    nudft_share = (fwd_ms + adj_ms) / 1e3 / value if value > 0 else None

    # error against FP64 on these inputs: the fixture holds the FP64 oracle's
    # image after the first TV pass (15 CG updates, W = 1); the 10-pass FP64
    # run (310 applies of ~78 s on 8 host threads) is not computed
    err = {"timed_config": None,
           "timed_config_note": "10-pass FP64 oracle run not computed (~7 h of host CPU); "
                                "long TV runs amplify rounding perturbations by >1e5"}
    if fix is not None:
        opts1 = pkg.bf_options(cg_num=CG_NUM, fd_penalizer=LAMBDA, tv=True, tv_num=1,
                               tv_eps=1e-6, use_z=1, dims=(nx, ny, nz))
        xr.zero_(); xi.zero_()
        pkg.bruteForceGpu(ctx, opts1, xr, xi, D["yr"], D["yi"], D["kx"], D["ky"], D["kz"],
                          D["ix"], D["iy"], D["iz"], D["fm"], D["t"], D["sr"], D["si"], M, N, C,
                          1)
        x1 = xr.cpu().numpy() + 1j * xi.cpu().numpy()
        err.update(first_tv_pass=rel_l2(x1, fix["x64_tv1"]),
                   first_tv_pass_what="relative L2 of the GPU image after the first TV pass "
                                      "(cg_num 16, lambda 1e-3, W = 1) against the FP64 "
                                      "oracle's on the same inputs (k-space data simulated "
                                      "in FP64 + 40 dB noise)")
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3 * ws, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{BF3D}: 64x64x16, 4 coils, M=65536, cg_num 16, TV 10 "
                               f"passes, lambda 1e-3, 3-D phase",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"replicas x{ws}"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": fp32_peak,
                     "unit": "TFLOP/s", "frac": achieved / fp32_peak,
                     "traffic": ncu_traffic(),
                     "kernel": "k_nudft (forward + adjoint)",
                     "peak_source": "measured FFMA throughput kernel (imp_measure_alu_peaks)",
                     "algorithmic_flop_per_launch": flop_launch,
                     "avg_launch_ms": avg_launch_s * 1e3, "launches": fwd_n + adj_n,
                     "sfu_peak_gops": sfu_peak, "share_of_recon": nudft_share},
        "error_vs_fp64": err,
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            if oracle.ref_available("bf32_omp"):
                v, (f_full, a_full) = cpu_reference_sample(case, 8192, 8192)
                out["cpu_baseline"] = {
                    "value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "reference",
                    "sample": (f"reference parallelFtCpu on 8192 of {M} samples x {N} voxels and "
                               f"parallelIftCpu on {M} samples x 8192 voxels, {C} coils (FP32, "
                               f"OpenMP), each extrapolated to a full apply (F {f_full:.1f} s, "
                               f"F^H {a_full:.1f} s), x 160 F + 150 F^H per recon")}
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                   "kind": "reference", "sample": f"failed: {e}"}
    ctx.close()
    if not emit:
        return out
    if rank == 0:
        print(json.dumps(out))
    return 0


# ------------------------------------------------------------------- C1 --

C1 = "bf2d_64"
C1_METRIC = "s/recon (brute-force 2-D CG, 64x64, 1 coil, M=4096, 8 CG x 10 TV)"


def run_bf2d(args, ws, rank, local):
    """The reference's CPU-runnable case: 2-D 64x64, one coil,
    4 x 1024 spiral (M = 4096), field map, TV lambda 1e-3 with 10 reweighting
    passes (the reference's -tv default) of 8 CG iterations.  Data: this
    library's exact-phase NUDFT of the seeded phantom + 40 dB noise.  The CPU
    baseline is the reference's own bruteForceCpu (FP32 build; 1 thread and the
    OpenMP build on all threads), full runs."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import synth
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = pkg.Context(local)
    case = synth.make_case(C1, seed=1001 + rank)
    fix = timed_fixture(C1) if rank == 0 else None
    if fix is not None:
        # the fixture's inputs: k-space data simulated by the reference's FP64
        # parallelFtCpu + 40 dB noise, with its FP64 and FP32 reconstructions
        for k in ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm", "sens", "x_true"):
            case[k] = fix[k]
    M, N = case["M"], case["N"]
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32))
    D = {k: f32(case[k]).to(dev) for k in ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm")}
    D["sr"], D["si"] = f32(case["sens"].real).to(dev), f32(case["sens"].imag).to(dev)
    if fix is not None:
        y = np.asarray(fix["kdata"], np.complex64).reshape(-1)
    else:
        yr, yi = torch.zeros(M, device=dev), torch.zeros(M, device=dev)
        pkg.parallelFtGpu(ctx, yr, yi, f32(case["x_true"].real).to(dev),
                          f32(case["x_true"].imag).to(dev), D["kx"], D["ky"], D["kz"], D["ix"],
                          D["iy"], D["iz"], D["fm"], D["t"], M, N, D["sr"], D["si"], 1, 0)
        y = yr.cpu().numpy() + 1j * yi.cpu().numpy()
        y = synth.add_noise(y, 40.0, np.random.default_rng(11 + rank)).astype(np.complex64)
    D["yr"], D["yi"] = f32(y.real).to(dev), f32(y.imag).to(dev)
    o = case["opts"]
    opts = pkg.bf_options(cg_num=o["cg_num"], fd_penalizer=o["fd_penalizer"], tv=True,
                          tv_num=o["tv_num"], tv_eps=1e-6)

    def recon(x_r, x_i, s):
        pkg.bruteForceGpu(ctx, opts, x_r, x_i, s["yr"], s["yi"], s["kx"], s["ky"], s["kz"],
                          s["ix"], s["iy"], s["iz"], s["fm"], s["t"], s["sr"], s["si"], M, N, 1,
                          1)

    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    xr, xi = torch.zeros(N, device=dev), torch.zeros(N, device=dev)
    for _ in range(max(args.warmup, 1)):
        xr.zero_(); xi.zero_()
        recon(xr, xi, D)
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = 0
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            xr.zero_(); xi.zero_()
            flush.fill_(float(s))
            ev[s][0].record()
            recon(xr, xi, D)
            ev[s][1].record()
            launches += ctx.launch_count()
    torch.cuda.synchronize()
    barrier(ws)
    value = max_over_ranks(sum(a.elapsed_time(b) for a, b in ev) / 1e3, ws) / (args.steps * ws)
    H = {k: v.cpu().pin_memory() for k, v in D.items()}
    hxr, hxi = torch.zeros(N).pin_memory(), torch.zeros(N).pin_memory()
    h2d = sum(v.numel() * 4 for v in H.values()) + 2 * N * 4
    recon(hxr, hxi, H)
    e2e = []
    for s in range(args.steps):
        hxr.zero_(); hxi.zero_()
        flush.fill_(float(s))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        recon(hxr, hxi, H)
        e2e.append(time.perf_counter() - t0)
    e2e_value = max_over_ranks(float(sum(e2e)), ws) / (args.steps * ws)
    ctx.profile(True)
    xr.zero_(); xi.zero_()
    recon(xr, xi, D)
    prof = ctx.profile_read()
    ctx.profile(False)
    fwd_ms, fwd_n = prof["forward"]
    adj_ms, adj_n = prof["adjoint"]
    avg_launch_s = (fwd_ms + adj_ms) / max(fwd_n + adj_n, 1) / 1e3
    fp32_peak, sfu_peak = pkg.measure_alu_peaks(local)
    # one coil, 2-D phase: 2 MUFU per pair bound the NUDFT (14 FLOP per pair)
    sfu_gops = 2.0 * M * N / avg_launch_s / 1e9
    err = {"timed_config": None, "note": "fixture tests/golden/bf2d_64_timed.npz absent"}
    if fix is not None:
        x = xr.cpu().numpy() + 1j * xi.cpu().numpy()
        err = {"timed_config": rel_l2(x, fix["x64"]),
               "reference_fp32": rel_l2(fix["x32"], fix["x64"]),
               "what": "relative L2 against the reference's own bruteForceCpu FP64 build on "
                       "the timed inputs (cg_num 8, TV 10 passes, lambda 1e-3); "
                       "reference_fp32 = the reference's FP32 build against the same"}
    out = {
        "metric": C1_METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3 * ws, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{C1}: 64x64, 1 coil, 4 x 1024 spiral (M=4096), field map, "
                               f"cg_num 8, TV 10 passes, lambda 1e-3",
                   "l2": "flushed (256 MiB write) before every timed step",
                   "parallelism": f"replicas x{ws}"},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": 2 * N * 4},
        "gpu_launches": launches,
        "roofline": {"bound": "sfu", "achieved": sfu_gops, "peak": sfu_peak, "unit": "Gop/s",
                     "frac": sfu_gops / sfu_peak, "traffic": None,
                     "kernel": "k_nudft (forward + adjoint): 2 MUFU (sin, cos) per pair",
                     "peak_source": "measured MUFU throughput kernel (imp_measure_alu_peaks)",
                     "avg_launch_ms": avg_launch_s * 1e3, "launches": fwd_n + adj_n,
                     "share_of_recon": (fwd_ms + adj_ms) / 1e3 / value if value > 0 else None},
        "error_vs_fp64": err,
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        try:
            import oracle
            cpu_case = dict(case, kdata=y.astype(np.complex64))
            runs = {}
            for kind in ("bf32", "bf32_omp"):
                if oracle.ref_available(kind):
                    t0 = time.perf_counter()
                    oracle.ref_bf_cg(cpu_case, kind=kind, cg_num=o["cg_num"],
                                     lam=o["fd_penalizer"], tv=True, tv_num=o["tv_num"])
                    runs[kind] = time.perf_counter() - t0
            if "bf32_omp" in runs:
                out["cpu_baseline"] = {
                    "value": runs["bf32_omp"], "unit": UNIT, "cores": os.cpu_count(),
                    "kind": "reference",
                    "sample": ("reference bruteForceCpu FP32, full recon: OpenMP on all threads "
                               f"{runs['bf32_omp']:.2f} s, one thread "
                               f"{runs.get('bf32', float('nan')):.2f} s")}
        except Exception as e:  # the baseline is reported, never required
            out["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(),
                                   "kind": "reference", "sample": f"failed: {e}"}
    ctx.close()
    if rank == 0:
        print(json.dumps(out))
    return 0


# ------------------------------------------------------------- Toeplitz --

TOEP = "toep3d_256x256x32"
TOEP_METRIC = ("s/recon (Toeplitz 3-D, 256x256x32, 4 coils, M=2.1M, L=8, Q at OS 2, "
               "20 CG x 10 TV)")


def toep_model_bytes(N, G, C, L1):
    """Algorithmic HBM bytes of one A^H A application: per (coil, segment) the
    Qf_l read (8G) and one read + write of the 2N grid per FFT (2 x 16G), the
    image-side passes (16N), plus the sensitivities (8CN) and CG vectors (48N)."""
    return C * L1 * (8 * G + 32 * G) + C * L1 * 16 * N + 8 * C * N + 48 * N


def toep_fp64_check(pkg, ctx, case, B, opts_fields, dev):
    """FP64 oracle on the Toeplitz configuration's timed inputs (checker leg,
    outside every timed region): one A^H A + lambda D^H D application of a
    random image on Q as the GPU computed it in the last timed step, against the
    FP64 oracle (oracle/toeplitz.py) on the same Q.  An FP64 CG at this size is
    not run: one application takes ~15 s on the host, a TV pass 21 of them."""
    import torch
    from oracle import toeplitz as T
    o = opts_fields
    M, N, C = case["M"], case["N"], case["num_coil"]
    nx, ny, nz = case["dims"]
    L = int(o["ntime_segs"])
    shape = (ny, nx, nz)
    q_shape = tuple(2 * n for n in shape)
    host = lambda t: t.detach().cpu().numpy().astype(np.float64)
    sens = np.asarray(case["sens"], np.complex128).reshape(C, *shape)
    fm = np.asarray(case["fm"], np.float64)
    t = np.asarray(case["t"], np.float64)
    lam = o["fd_penalizer"]
    t0 = time.perf_counter()
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(dev)
    rng = np.random.default_rng(2024)
    pv = rng.standard_normal(N) + 1j * rng.standard_normal(N)
    ar, ai = torch.zeros(N, device=dev), torch.zeros(N, device=dev)
    ops1 = pkg.toeplitz_options(cg_num=1, fd_penalizer=lam, ntime_segs=L)
    pkg.toeplitz_apply(ctx, ops1, ar, ai, f32(pv.real), f32(pv.imag), B["qr"], B["qi"],
                       f32(t), M, f32(fm), f32(sens.real.ravel()), f32(sens.imag.ravel()), C,
                       nx, ny, nz)
    got = host(ar) + 1j * host(ai)
    Q = (host(B["qr"]) + 1j * host(B["qi"])).reshape(L + 1, *q_shape)
    tau, ts0 = T.time_segments(t, L)
    Qf = T.qf_from_q(Q)
    del Q
    ref = (T.aha(pv.reshape(shape), Qf, sens, fm.reshape(shape), tau, ts0)
           + T.dhwd(pv.reshape(shape), np.ones(shape), lam)).ravel()
    return {"one_application": float(np.linalg.norm(got - ref) / np.linalg.norm(ref)),
            "one_application_what": "relative L2 of one A^H A + lambda D^H D application "
                                    "(random image, 4 coils, 9 segments) against FP64 on the "
                                    "GPU-computed Q",
            "timed_config": None,
            "timed_config_note": "FP64 reconstruction not computed (one FP64 application takes "
                                 "~15 s on the host; the recon makes 210); the reconstruction "
                                 "path is checked against the FP64 oracle at smaller sizes in "
                                 "tests/test_toeplitz_gpu.py",
            "checker_s": time.perf_counter() - t0}


def toep_cpu_sample(G_shape, C, L1, applies):
    """Project CPU restatement (not reference code: the reference has no CPU
    Toeplitz path) of one F^H F_l application on the 2N grid with scipy's
    multithreaded FFT, extrapolated to C (L+1) per A^H A and `applies` per recon."""
    import scipy.fft as sf
    rng = np.random.default_rng(0)
    n = tuple(s // 2 for s in G_shape)
    img = (rng.standard_normal(n) + 1j * rng.standard_normal(n)).astype(np.complex64)
    qf = (rng.standard_normal(G_shape) + 1j * rng.standard_normal(G_shape)).astype(np.complex64)
    t0 = time.perf_counter()
    big = np.zeros(G_shape, np.complex64)
    big[tuple(slice(0, s) for s in n)] = img
    f = sf.fftn(big, workers=-1)
    f *= qf
    out = sf.ifftn(f, workers=-1)[tuple(slice(0, s) for s in n)]
    dt = time.perf_counter() - t0
    del out
    return dt * C * L1 * applies, dt


def run_toeplitz(args, ws, rank, local):
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import synth
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = pkg.Context(local)
    case = synth.make_case(TOEP, seed=1003 + rank)
    o = case["opts"]
    M, N, C = case["M"], case["N"], case["num_coil"]
    nx, ny, nz = case["dims"]
    L1 = o["ntime_segs"] + 1
    G = 8 * N
    rng = np.random.default_rng(11 + rank)
    # k-space values: complex Gaussian at the phantom's mean k-space power (the
    # exact simulation, 2.1M x 2.1M x 4 NUDFT pairs, is not part of the step and
    # the Toeplitz timing does not depend on the values)
    kd = ((rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M)))
          * np.sqrt(np.mean(np.abs(case["x_true"]) ** 2) * N / 2)).astype(np.complex64)
    f32 = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32))
    H = {k: f32(case[k]) for k in ("kx", "ky", "kz", "t", "fm")}
    H["sr"], H["si"] = f32(case["sens"].real.ravel()), f32(case["sens"].imag.ravel())
    H["yr"], H["yi"] = f32(kd.real.ravel()), f32(kd.imag.ravel())
    D = {k: v.to(dev) for k, v in H.items()}
    opts = pkg.toeplitz_options(cg_num=o["cg_num"], fd_penalizer=o["fd_penalizer"], tv=o["tv"],
                                tv_num=o["tv_num"], ntime_segs=o["ntime_segs"],
                                gridOS_Q=o["gridOS_Q"], gridOS_FH=o["gridOS_FH"])

    def alloc(where):
        mk = (lambda n: torch.zeros(n, device=dev)) if where == "dev" else (
            lambda n: torch.zeros(n).pin_memory())
        return dict(qr=mk(L1 * G), qi=mk(L1 * G), fr=mk(N), fi=mk(N), xr=mk(N), xi=mk(N))

    def recon(src, out, ev=None):
        """Steps 1-3 of the reference's toeplitz(): Q by gridding, F^H d, CG."""
        if ev: ev[0].record()
        pkg.toeplitz_q(ctx, opts, out["qr"], out["qi"], src["kx"], src["ky"], src["kz"],
                       src["t"], M, nx, ny, nz)
        if ev: ev[1].record()
        pkg.toeplitz_fhd(ctx, opts, out["fr"], out["fi"], src["yr"], src["yi"], src["kx"],
                         src["ky"], src["kz"], src["t"], src["fm"], src["sr"], src["si"], M, C,
                         nx, ny, nz)
        if ev: ev[2].record()
        pkg.toeplitz_recon(ctx, opts, out["xr"], out["xi"], out["fr"], out["fi"], out["qr"],
                           out["qi"], src["t"], M, src["fm"], src["sr"], src["si"], C, nx, ny, nz)
        if ev: ev[3].record()

    B = alloc("dev")
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)
    for _ in range(args.warmup):
        recon(D, B)
    torch.cuda.synchronize()
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(args.steps)]
    launches = 0
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for s in range(args.steps):
            flush.fill_(float(s))
            recon(D, B, evs[s])
            launches += ctx.launch_count()
    torch.cuda.synchronize()
    barrier(ws)
    parts = np.array([[e[i].elapsed_time(e[i + 1]) for i in range(3)] for e in evs])
    step_ms = parts.sum(1)
    value = max_over_ranks(float(step_ms.sum()) / 1e3, ws) / (args.steps * ws)

    # end to end: the same calls with pinned host buffers
    Hb = alloc("host")
    Hs = {k: v.pin_memory() for k, v in H.items()}
    nb = lambda *ks: sum(Hs[k].numel() * 4 for k in ks)
    q_bytes, f_bytes, x_bytes = 2 * L1 * G * 4, 2 * N * 4, 2 * N * 4
    # inputs of the three calls (the trajectory is staged by each call that reads
    # it), plus Q and F^H d going back in for the CG
    h2d = (nb("kx", "ky", "kz", "t") + nb("kx", "ky", "kz", "t", "fm", "sr", "si", "yr", "yi")
           + nb("t", "fm", "sr", "si") + q_bytes + f_bytes)
    d2h = q_bytes + f_bytes + x_bytes  # Q, F^H d and the image come back
    recon(Hs, Hb)
    e2e = []
    barrier(ws)
    for s in range(args.steps):
        flush.fill_(float(s))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        recon(Hs, Hb)
        e2e.append(time.perf_counter() - t0)
    barrier(ws)
    e2e_value = max_over_ranks(float(sum(e2e)), ws) / (args.steps * ws)

    applies = o["tv_num"] * (o["cg_num"] + 1)
    cg_ms = float(np.mean(parts[:, 2]))
    per_apply_s = cg_ms / 1e3 / applies
    model = toep_model_bytes(N, G, C, L1)
    achieved = model / per_apply_s / 1e9
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    out = {
        "metric": TOEP_METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": value * 1e3 * ws, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded trajectory/phantom/coils/field map; Gaussian k-space values)",
        "config": {"workload": f"{TOEP}: 256x256x32, 4 coils, 32 kz x 16 x 4096 (M=2097152), "
                               f"L=8, gridOS_Q 2.0, gridOS_FH 1.5, cg_num 20, TV 10 passes, "
                               f"lambda 1e-3",
                   "l2": "flushed (256 MiB write) before every timed step; grids exceed L2",
                   "parallelism": f"replicas x{ws}"},
        "breakdown_ms": {"q": float(np.mean(parts[:, 0])), "fhd": float(np.mean(parts[:, 1])),
                         "cg": cg_ms},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "traffic": ncu_traffic("toeplitz_apply_toep3d_256x256x32.md",
                                            "traffic_bytes_per_apply:"),
                     "traffic_source": "profiles/toeplitz_apply_toep3d_256x256x32.md: DRAM bytes "
                                       "of the three engine kernels of one application (ncu)",
                     "kernel": "A^H A application inside the CG (pruned FFT engine: k_fwd_pair, "
                               "k_slow with x Qf_l, k_inv_async with the coil sum; CG update), "
                               "per application; bytes = the zero-padded FFT model",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs" if peaks else "fallback",
                     "algorithmic_bytes_per_apply": model, "apply_ms": per_apply_s * 1e3,
                     "applies_per_recon": applies},
        "clocks": clk.summary(),
    }
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["error_vs_fp64"] = toep_fp64_check(pkg, ctx, case, B, opts_fields=o, dev=dev)
        v, dt = toep_cpu_sample((2 * ny, 2 * nx, 2 * nz), C, L1, applies)
        out["cpu_baseline"] = {
            "value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
            "sample": (f"project CPU restatement (the reference has no CPU Toeplitz code): one "
                       f"F^H F_l (pad, scipy FFT, x Qf, IFFT, crop) on the 512x512x64 grid "
                       f"({dt:.2f} s), x{C * L1} per A^H A, x{applies} per recon; gridding "
                       f"of Q and F^H d not counted")}
    ctx.close()
    if rank == 0:
        print(json.dumps(out))
    return 0


def run_toep_apply_only(args, local):
    """A^H A applications of the Toeplitz 3-D geometry through the operator
    C-ABI, with random Q, field map and sensitivities (the small command the
    Toeplitz kernel profiles are taken on)."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    torch.cuda.set_device(local)
    nx, ny, nz = (int(v) for v in args.toep_dims.split(","))
    C, L1 = args.toep_coils, args.toep_segs
    N = nx * ny * nz
    G, M = (8 if nz > 1 else 4) * N, 4096
    g = torch.Generator(device="cuda").manual_seed(5)
    rn = lambda n, s=1.0: torch.randn(n, device="cuda", generator=g) * s
    t = torch.linspace(0.0, 0.01, M, device="cuda")
    fm, sr, si = rn(N, 300.0), rn(C * N), rn(C * N)
    qr, qi, pr, pi = rn(L1 * G), rn(L1 * G), rn(N), rn(N)
    outr, outi = torch.zeros(N, device="cuda"), torch.zeros(N, device="cuda")
    opts = pkg.toeplitz_options(cg_num=1, fd_penalizer=1e-3, ntime_segs=L1 - 1)
    with pkg.Context(local) as ctx:
        for _ in range(max(args.warmup, 1)):
            pkg.toeplitz_apply(ctx, opts, outr, outi, pr, pi, qr, qi, t, M, fm, sr, si, C,
                               nx, ny, nz)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pkg.toeplitz_apply(ctx, opts, outr, outi, pr, pi, qr, qi, t, M, fm, sr, si, C,
                               nx, ny, nz)
        dt = (time.perf_counter() - t0) / max(args.steps, 1)
    print(json.dumps({"toep_apply_only": f"{nx}x{ny}x{nz}, {C} coils, L+1 = {L1}",
                      "ms_per_call_incl_q_load": dt * 1e3}))
    return 0


# ---------------------------------------------------------- warm start --

WARM = "warm512"
WARM_METRIC = ("s/recon to NRMSE<=1e-3 vs converged CG (2-D 512x512, 32 coils, Toeplitz CG): "
               "learned warm start (value) vs zero start")
WEIGHTS = ROOT / "impatient-mri_b200" / "weights" / "unet_warm512.npz"


def run_warm(args, local):
    """Learned warm start at the configuration's size: 2-D 512x512, 32 coils
    on a ring, 24 x 4096 spiral (M = 98304), no field map, CG with the finite-
    difference penalty lambda = 1e-3 lambda_max, 40 dB noise.  Trains the
    U-Net on seeded phantoms with 50-iteration CG labels unless trained
    weights are present, then times CG from the network output and from zero
    on held-out phantoms."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import learn
    torch.cuda.set_device(local)
    ctx = pkg.Context(local)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    t0 = time.perf_counter()
    prob = learn.ToepProblem(pkg, ctx, n=512, C=32, n_il=24, n_s=4096, seed=1005)
    log(f"problem setup {time.perf_counter() - t0:.1f} s, lambda {prob.lam:.4g}")
    trained_here = False
    if WEIGHTS.exists() and not args.retrain:
        params, kappa, meta = learn.load_weights(WEIGHTS)
        train_info = {k: v.tolist() for k, v in meta.items()}
    else:
        t0 = time.perf_counter()
        b, lab, _ = prob.make_pairs(args.train_images, seed=2005)
        t_pairs = time.perf_counter() - t0
        x, y, kappa = learn.normalise(b, lab)
        del b, lab
        net = pkg.UNet(ctx, args.batch, 512, 512, seed=7)
        t0 = time.perf_counter()
        losses = learn.train(net, x, y, epochs=args.epochs, lr=args.lr, log=log)
        t_train = time.perf_counter() - t0
        params = net.get_params()
        net.close()
        del x, y
        train_info = dict(train_images=args.train_images, epochs=args.epochs, lr=args.lr,
                          batch=args.batch, final_loss=losses[-1], pairs_s=t_pairs,
                          train_s=t_train)
        if args.save_weights:
            out = Path(args.save_weights)
            out.parent.mkdir(parents=True, exist_ok=True)
            learn.save_weights(out, params, kappa, train_info)
        trained_here = True
    net1 = pkg.UNet(ctx, 1, 512, 512, seed=7)
    net1.set_params(params)
    bt, _, _ = prob.make_pairs(args.test_images, seed=3005)
    for _ in range(max(args.warmup, 1)):  # warm the graphs and the network
        learn.evaluate(prob, net1, kappa, bt[:1], target=1e-3, kmax=200)
    res = learn.evaluate(prob, net1, kappa, bt, target=1e-3, kmax=200)
    f = lambda k: float(np.mean([r[k] for r in res]))
    line = {
        "metric": WARM_METRIC, "value": f("warm_s"), "unit": UNIT, "n_gpus": 1,
        "steps": len(res), "warmup": args.warmup, "ms_per_step": f("warm_s") * 1e3,
        "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32+bf16",
        "data": "synthetic (seeded ellipse phantoms, ring coils, spiral; 40 dB k-space noise)",
        "config": {"workload": f"{WARM}: 512x512, 32 coils, 24 x 4096 spiral, no field map, "
                               f"FD lambda = 1e-3 lambda_max ({prob.lam:.4g}), U-Net 2->2 ch, "
                               f"4 levels 32-256 ch, BF16", "train": train_info,
                   "trained_in_this_run": trained_here},
        "zero_start": {"s_per_recon": f("zero_s"), "cg_updates": f("zero_iters"),
                       "nrmse": f("zero_nrmse"), "cg_updates_to_residual_1e-4":
                           f("zero_iters_tol")},
        "warm_start": {"s_per_recon": f("warm_s"), "cg_updates": f("warm_iters"),
                       "nrmse": f("warm_nrmse"), "start_nrmse": f("x0_nrmse"),
                       "cg_updates_to_residual_1e-4": f("warm_iters_tol")},
        "speedup": f("zero_s") / f("warm_s"),
    }
    net1.close()
    ctx.close()
    print(json.dumps(line))
    return 0


def fp64_checker(prob, bs, xg, log=None, max_steps=4, tol=1e-11):
    """Checker and CPU baseline of the warm-start line (test infrastructure:
    the FP64 oracle, oracle/toeplitz.py, never inside a timed region).

    For each right-hand side b_i (GPU, [2][N]) and its GPU-converged solution
    xg_i, mixed-precision iterative refinement gives the FP64 solution of the
    same system (A^H A + lambda D^H D) x = b, A^H A from the same Q: the
    residual r = b - A x is evaluated by the FP64 oracle on the host, the
    correction A d = r is solved by the GPU CG in FP32, x += d, until
    |r| / |b| < tol.  Returns (x64 list, info) where info holds the FP64
    residuals reached, the GPU solutions' distances from x64 and the host
    time of one FP64 A^H A application (all host threads)."""
    import torch
    from oracle import toeplitz as T
    n, N, C = prob.n, prob.N, prob.C
    Q = (prob.qr.double().cpu().numpy() + 1j * prob.qi.double().cpu().numpy()).reshape(
        1, 2 * n, 2 * n)
    Qf = T.qf_from_q(Q)
    sens = (prob.sr.double().cpu().numpy() + 1j * prob.si.double().cpu().numpy()).reshape(
        C, n, n)
    fm = np.zeros((n, n))
    tau, t0 = T.time_segments(prob.t.cpu().numpy(), 0)
    ones = np.ones((n, n))
    t_apply = []

    def A64(x):
        t_s = time.perf_counter()
        out = T.aha_coils(x, Qf, sens, fm, tau, t0) + T.dhwd(x, ones, prob.lam)
        t_apply.append(time.perf_counter() - t_s)
        return out

    to_c = lambda v: (v[0].double().cpu().numpy() + 1j * v[1].double().cpu().numpy()).reshape(
        n, n)
    to_g = lambda z: torch.stack([torch.as_tensor(z.real.ravel(), dtype=torch.float32),
                                  torch.as_tensor(z.imag.ravel(), dtype=torch.float32)]).cuda()
    x64s, res, dist, steps = [], [], [], []
    for i in range(bs.shape[0]):
        b = to_c(bs[i])
        nb = np.linalg.norm(b)
        x = to_c(xg[i])
        rel = None
        for k in range(max_steps + 1):
            r = b - A64(x)
            rel = float(np.linalg.norm(r) / nb)
            if rel < tol or k == max_steps:
                break
            s_ = float(np.linalg.norm(r))
            d = torch.zeros(2, N, device="cuda")
            prob.cg(to_g(r / s_), d, 1e-6, 2000)
            x = x + s_ * to_c(d)
        x64s.append(x)
        res.append(rel)
        dist.append(float(np.linalg.norm(to_c(xg[i]) - x) / np.linalg.norm(x)))
        steps.append(k)
        if log:
            log(f"FP64 reference {i}: {k} refinement steps, FP64 residual {rel:.1e}, GPU "
                f"solution {dist[-1]:.1e} from it")
    return x64s, dict(fp64_rel_residual_max=max(res), refinement_steps_max=max(steps),
                      gpu_converged_vs_fp64_max=max(dist),
                      gpu_converged_vs_fp64_mean=float(np.mean(dist)),
                      fp64_apply_s=float(np.median(t_apply)))


def run_headline(args, ws, rank, local):
    """The metric's configuration: learned warm start versus plain zero-start
    CG on the Toeplitz path, 2-D 512x512, 32 ring coils, 24 x 4096 spiral
    (M = 98304), no field map, finite-difference penalty lambda = 1e-3
    lambda_max, 40 dB noise.  One step = one reconstruction of a held-out
    phantom to NRMSE <= 1e-3 against the FP64 solution of the same system;
    `value` = the warm start's seconds per reconstruction (network + CG),
    `zero_start` beside it, both device-timed from resident inputs with the L2
    flushed before each.  The NUDFT half of the metric is the nested `nudft`
    block (the brute-force 3-D configuration and its NUDFT roofline)."""
    import argparse as _ap
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import learn
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    log = lambda m: print(m, file=sys.stderr, flush=True)
    if not WEIGHTS.exists():
        raise SystemExit(f"trained weights missing: {WEIGHTS} (bench.py --workload warm512 "
                         f"--retrain --save-weights ...)")
    params, kappa, meta = learn.load_weights(WEIGHTS)
    ctx = pkg.Context(local)
    prob = learn.ToepProblem(pkg, ctx, n=512, C=32, n_il=24, n_s=4096, seed=1005)
    net1 = pkg.UNet(ctx, 1, 512, 512, seed=7)
    net1.set_params(params)
    K, W = args.steps, args.warmup
    b_all, _ = prob.make_rhs(K + W, seed=3005 + 1000 * rank)
    target, kmax = 1e-3, 300
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=dev)  # 256 MiB > L2

    # GPU-converged solutions (relative residual 1e-6), then the FP64 references
    t0 = time.perf_counter()
    xg = torch.zeros_like(b_all)
    it_conv = [prob.cg(b_all[i], xg[i], 1e-6, 3000) for i in range(K + W)]
    log(f"converged GPU solutions: {time.perf_counter() - t0:.1f} s, updates "
        f"{min(it_conv)}..{max(it_conv)}")
    chk = None
    refs = [xg[i] for i in range(K + W)]
    if not args.no_cpu_baseline:
        t0 = time.perf_counter()
        x64s, chk = fp64_checker(prob, b_all[W:], xg[W:], log=log)
        chk["checker_s"] = time.perf_counter() - t0
        for i, z in enumerate(x64s):
            refs[W + i] = torch.stack([torch.as_tensor(z.real.ravel(), dtype=torch.float32),
                                       torch.as_tensor(z.imag.ravel(),
                                                       dtype=torch.float32)]).to(dev)
    zero = torch.zeros(2, prob.N, device=dev)

    def nr(a, r):
        return float((a - r).norm() / r.norm())

    def k_to_target(i, warm):
        """Fewest CG updates reaching NRMSE <= target (CG's error norm falls
        monotonically; bisection on the update count)."""
        x0 = learn.warm_start(net1, kappa, b_all[i]) if warm else zero
        run = lambda k: learn._cg_k(prob, b_all[i], x0, k)
        if nr(x0, refs[i]) <= target:
            return 0
        if nr(run(kmax), refs[i]) > target:
            return kmax + 1
        lo, hi = 0, kmax
        while hi - lo > 1:
            mid = (lo + hi) // 2
            if nr(run(mid), refs[i]) <= target:
                hi = mid
            else:
                lo = mid
        return hi

    # kernel launches of one network forward (the network's counter is cumulative)
    learn.warm_start(net1, kappa, b_all[0])
    c0 = ctx.launch_count()
    learn.warm_start(net1, kappa, b_all[0])
    net_launches = ctx.launch_count() - c0
    rows = []
    launches = 0
    with ClockSampler(local) as clk:
        for i in range(K + W):
            kz, kw = k_to_target(i, False), k_to_target(i, True)
            tz, xz = learn.timed_run(prob, b_all[i], zero, kz, flush)
            lz = ctx.launch_count()
            tw, xw = learn.timed_run(prob, b_all[i], zero, kw, flush, net1=net1, kappa=kappa)
            lw = ctx.launch_count() + net_launches
            if i < W:
                continue
            launches += lw
            x0w = learn.warm_start(net1, kappa, b_all[i])
            xr_ = zero.clone()
            it_rz = prob.cg(b_all[i], xr_, 1e-4, kmax)
            xr_ = x0w.clone()
            it_rw = prob.cg(b_all[i], xr_, 1e-4, kmax)
            rows.append(dict(kz=kz, kw=kw, tz=tz / 1e3, tw=tw / 1e3, ez=nr(xz, refs[i]),
                             ew=nr(xw, refs[i]), e0=nr(x0w, refs[i]), rz=it_rz, rw=it_rw,
                             lz=lz))
    barrier(ws)
    tz_all = np.array([r["tz"] for r in rows])
    tw_all = np.array([r["tw"] for r in rows])
    value = max_over_ranks(float(tw_all.sum()), ws) / (K * ws)
    zero_v = max_over_ranks(float(tz_all.sum()), ws) / (K * ws)
    speed = tz_all / tw_all

    # end to end through the public API with host buffers: the right-hand side
    # goes up from pinned memory, the network and the CG run, the image comes back
    hb = b_all[W:].cpu().pin_memory()
    hx = torch.zeros(2, prob.N).pin_memory()
    e2e_w, e2e_z = [], []
    for i, r in enumerate(rows):
        for warm, acc in ((True, e2e_w), (False, e2e_z)):
            flush.fill_(2.0)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            bd = hb[i].to(dev, non_blocking=True)
            x = learn.warm_start(net1, kappa, bd) if warm else torch.zeros_like(bd)
            prob.cg(bd, x, 0.0, r["kw"] if warm else r["kz"])
            hx.copy_(x, non_blocking=True)
            torch.cuda.synchronize()
            acc.append(time.perf_counter() - t0)
    e2e_value = max_over_ranks(float(np.sum(e2e_w)), ws) / (K * ws)

    # roofline: one CG update = one A^H A application (+ FD term, vector updates)
    kcg = 40
    x = torch.zeros_like(b_all[0])
    prob.cg(b_all[0], x, 0.0, 4)
    x.zero_()
    flush.fill_(3.0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    prob.cg(b_all[0], x, 0.0, kcg)
    e1.record()
    torch.cuda.synchronize()
    upd_s = e0.elapsed_time(e1) / 1e3 / kcg
    N, G, C = prob.N, 4 * prob.N, prob.C
    model = toep_model_bytes(N, G, C, 1)
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    achieved = model / upd_s / 1e9
    net_ms = []
    for _ in range(5):
        e0.record()
        learn.warm_start(net1, kappa, b_all[0])
        e1.record()
        torch.cuda.synchronize()
        net_ms.append(e0.elapsed_time(e1))
    net1.close()
    ctx.close()

    # the metric's NUDFT half: the brute-force 3-D configuration (few steps)
    a2 = _ap.Namespace(**vars(args))
    a2.steps, a2.warmup, a2.no_cpu_baseline = 3, 1, True
    nud = run_ours(a2, ws, rank, local, emit=False)
    nudft = {"workload": nud["config"]["workload"], "s_per_recon": nud["value"],
             "e2e_s_per_recon": nud["e2e"]["value"], "roofline": nud["roofline"],
             "error_vs_fp64": nud["error_vs_fp64"], "steps": 3, "warmup": 1,
             "gpu_launches": nud["gpu_launches"]}

    f = lambda k: float(np.mean([r[k] for r in rows]))
    line = {
        "metric": WARM_METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": K,
        "warmup": W, "ms_per_step": value * 1e3 * ws, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (BF16 network)",
        "data": "synthetic (seeded ellipse phantoms, ring coils, spiral; 40 dB k-space noise)",
        "config": {"workload": f"{WARM}: 2-D 512x512, 32 coils, 24 x 4096 spiral (M=98304), "
                               f"no field map, Toeplitz CG with FD lambda = 1e-3 lambda_max "
                               f"({prob.lam:.4g}); U-Net 2->2 ch, 4 levels 32-256 ch, BF16; one "
                               f"step = one held-out phantom reconstructed to NRMSE <= 1e-3",
                   "l2": "flushed (256 MiB write) before every timed solve",
                   "parallelism": f"replicas x{ws}",
                   "weights": "impatient-mri_b200/weights/unet_warm512.npz",
                   "train": {k: v.tolist() for k, v in meta.items()},
                   "nrmse_reference": ("FP64 solution of the same system (iterative "
                                       "refinement with FP64 residuals from the FP64 oracle)"
                                       if chk else "GPU CG to relative residual 1e-6")},
        "zero_start": {"s_per_recon": zero_v, "cg_updates": f("kz"), "nrmse": f("ez"),
                       "cg_updates_to_residual_1e-4": f("rz"),
                       "e2e_s_per_recon": float(np.mean(e2e_z))},
        "warm_start": {"s_per_recon": value, "cg_updates": f("kw"), "nrmse": f("ew"),
                       "start_nrmse": f("e0"), "cg_updates_to_residual_1e-4": f("rw"),
                       "network_ms": float(np.median(net_ms))},
        "speedup": zero_v / value,
        "speedup_per_phantom": {"min": float(speed.min()), "median": float(np.median(speed)),
                                "max": float(speed.max()),
                                "warm_faster": int((speed > 1).sum()), "phantoms": K},
        "e2e": {"value": e2e_value, "unit": UNIT,
                "h2d_bytes_per_step": int(hb[0].numel() * 4),
                "d2h_bytes_per_step": int(hx.numel() * 4)},
        "gpu_launches": launches,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm,
                     "traffic": ncu_traffic("toeplitz_apply_warm512.md",
                                            "traffic_bytes_per_apply:"),
                     "traffic_source": "profiles/toeplitz_apply_warm512.md: DRAM bytes of the "
                                       "three engine kernels of one application (ncu)",
                     "kernel": "one CG update (A^H A application: k_fwd_pair, k_slow with x Qf, "
                               "k_inv_async with the coil sum; FD term; vector updates); bytes "
                               "= the zero-padded FFT model of one A^H A application",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else
                                    "fallback 6650 GB/s",
                     "algorithmic_bytes_per_apply": model, "update_ms": upd_s * 1e3},
        "error_vs_fp64": {"warm_start_nrmse_mean": f("ew"),
                          "warm_start_nrmse_max": float(max(r["ew"] for r in rows)),
                          "zero_start_nrmse_max": float(max(r["ez"] for r in rows)),
                          **({k: v for k, v in chk.items()} if chk else
                             {"note": "no FP64 references (--no-cpu-baseline)"})},
        "nudft": nudft,
        "clocks": clk.summary(),
    }
    if chk and rank == 0 and ws == 1:
        per_apply = chk["fp64_apply_s"]
        kz_mean = f("kz")
        line["cpu_baseline"] = {
            "value": per_apply * (kz_mean + 1), "unit": UNIT, "cores": os.cpu_count(),
            "kind": "port",
            "sample": (f"project FP64 CPU restatement of the Toeplitz A^H A + lambda D^H D "
                       f"(oracle/toeplitz.py, scipy FFT on all threads; the reference has no "
                       f"CPU Toeplitz code): median {per_apply:.2f} s per application over the "
                       f"FP64 checker's applications, x (zero-start updates {kz_mean:.1f} + 1)")}
    if rank == 0:
        print(json.dumps(line))
    return 0


# ---------------------------------------------------------- multi-slice --

BATCH = "batch384"
BATCH_METRIC = ("s/recon (brute-force CG, 64 independent 2-D 384x384 slices, 32 coils, "
                "16-32 x 4096-sample spirals per slice, 20 CG iterations)")


def run_batch(args, ws, rank, local):
    """64 independent 384x384 slices with 32 ring coils, each with
    its own seeded spiral of 16..32 interleaves x 4096 samples (uneven M), field
    map and phantom; plain CG, cg_num 20 (19 updates).  The timed job is the
    first `--slices` slices of the seeded 64; with N GPUs each rank takes a
    contiguous share of them (replicas, as the reference's -mgpu) through one
    imp_bruteforce_batch call, and the job time is the maximum over ranks.
    value = that time scaled by the ratio of all 64 slices' sample counts to
    the timed slices' (1 when all 64 are timed; the work per slice is
    proportional to its sample count)."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import synth
    R = _replicas()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = pkg.Context(local)
    n, C, S_total = 384, 32, 64
    S = max(1, min(args.slices, S_total))
    lo, hi = R.slice_range(S, ws, rank)
    rng = np.random.default_rng(1004)
    ix, iy, iz = synth.grid_positions(n, n, 1)
    sens = np.stack([synth.to_voxel_order(m)
                     for m in synth.coil_maps((n, n), C, rng, ring=True)]).astype(np.complex64)
    N = n * n
    f = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).to(dev)
    D = dict(ix=f(ix), iy=f(iy), iz=f(iz), sr=f(sens.real.ravel()), si=f(sens.imag.ravel()))
    kx, ky, tt, fms, kdr, kdi, ms = [], [], [], [], [], [], []
    for s_ in range(S_total):
        il = int(rng.integers(16, 33))
        skx, sky, st = synth.spiral(il, 4096, n / 2 - 0.05, rng)
        img = synth.to_voxel_order(synth.ellipse_phantom((n, n), 8, rng))
        fm = synth.to_voxel_order(synth.field_map((n, n), rng)).astype(np.float32)
        ms.append(skx.size)
        if not lo <= s_ < hi:
            continue
        M = skx.size
        yr = torch.zeros(C * M, device=dev)
        yi = torch.zeros(C * M, device=dev)
        g = dict(kx=f(skx), ky=f(sky), kz=f(np.zeros_like(skx)), t=f(st), fm=f(fm))
        pkg.parallelFtGpu(ctx, yr, yi, f(img.real), f(img.imag), g["kx"], g["ky"], g["kz"],
                          D["ix"], D["iy"], D["iz"], g["fm"], g["t"], M, N, D["sr"], D["si"], C, 0)
        y = yr.cpu().numpy() + 1j * yi.cpu().numpy()
        # per-slice noise seed: the data do not depend on how slices are sharded
        y = synth.add_noise(y, 40.0, np.random.default_rng(5000 + s_)).astype(np.complex64)
        kx.append(skx); ky.append(sky); tt.append(st); fms.append(fm)
        kdr.append(y.real.astype(np.float32)); kdi.append(y.imag.astype(np.float32))
    mine = hi - lo
    if mine:
        k_off = np.cumsum([0] + ms[lo:hi])
        B = dict(kx=f(np.concatenate(kx)), ky=f(np.concatenate(ky)),
                 kz=f(np.zeros(int(k_off[-1]), np.float32)), t=f(np.concatenate(tt)),
                 fm=f(np.concatenate(fms)), kr=f(np.concatenate(kdr)), ki=f(np.concatenate(kdi)))
    xr = torch.zeros(max(mine, 1) * N, device=dev)
    xi = torch.zeros(max(mine, 1) * N, device=dev)
    opts = pkg.bf_options(cg_num=20)

    def recon():
        if not mine:  # more ranks than timed slices: this rank has no work
            return
        xr.zero_(); xi.zero_()
        pkg.bruteForceBatch(ctx, opts, xr, xi, B["kr"], B["ki"], B["kx"], B["ky"], B["kz"],
                            B["t"], k_off, D["ix"], D["iy"], D["iz"], B["fm"], D["sr"], D["si"],
                            N, C)

    for _ in range(max(args.warmup, 1)):
        recon()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    launches = 0
    barrier(ws)
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for s_ in range(args.steps):
            ev[s_][0].record()
            recon()
            ev[s_][1].record()
            launches += ctx.launch_count() if mine else 0
    torch.cuda.synchronize()
    barrier(ws)
    # whole job: every rank's share of the timed slices, time = max over ranks
    ms_step = max_over_ranks(float(np.mean([a.elapsed_time(b) for a, b in ev])), ws)
    launches = int(round(max_over_ranks(float(launches), ws)))
    pairs = float(sum(ms[:S])) * N
    applies = 1 + 2 * 19
    flop = 2.0 * (3 + 4 * C) * pairs * applies
    achieved = flop / (ms_step / 1e3) / 1e12
    fp32_peak, sfu_peak = pkg.measure_alu_peaks(local)
    # 32 coils: one coil group on the tensor-core NUDFT (the multiply-add runs on the
    # tensor pipe); the CUDA cores' binding unit is the SFU, 2 MUFU per pair
    sfu_gops = 2.0 * pairs * applies / (ms_step / 1e3) / 1e9
    scale = float(sum(ms)) / float(sum(ms[:S]))  # work is proportional to the sample count
    if rank != 0:
        ctx.close()
        return 0
    line = {
        "metric": BATCH_METRIC, "value": ms_step / 1e3 * scale, "unit": UNIT, "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": False, "scaling": "strong", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded spirals, phantoms, field maps, ring coils; 40 dB noise)",
        "config": {"workload": f"{BATCH}: {S} of 64 slices timed (sample counts "
                               f"{ms[:S]}); value = that time x {scale:.2f} (all 64 slices' "
                               f"samples / the timed slices' samples); 384x384, 32 coils, "
                               f"cg_num 20, no regularization",
                   "parallelism": f"replicas x{ws}: each GPU one imp_bruteforce_batch call "
                                  "over its contiguous share of the slices (all its slices "
                                  "in lockstep, one launch per CG step)"},
        "gpu_launches": launches,
        "roofline": {"bound": "sfu", "achieved": sfu_gops, "peak": sfu_peak, "unit": "Gop/s",
                     "frac": sfu_gops / sfu_peak, "traffic": None,
                     "kernel": "whole recon (tensor-core NUDFT F and F^H dominate): 2 MUFU "
                               "(sin, cos) per (sample, voxel) pair for all 32 coils, 39 "
                               "applies",
                     "peak_source": "measured MUFU throughput kernel (imp_measure_alu_peaks)",
                     "fp32_equivalent_tflops": achieved,
                     "fp32_equivalent_note": "algorithmic FLOP 2 (3 + 4C) per pair over the "
                                             "measured FFMA peak; above 1 because the "
                                             "multiply-add runs on the tensor pipe",
                     "fp32_equivalent_frac": achieved / fp32_peak},
        "clocks": clk.summary(),
    }
    ctx.close()
    print(json.dumps(line))
    return 0


def run_toeplitz_ref_gpu(args):
    """The reference's own GPU program (oracle/_ref/mriSolver_ref, built from the
    reference sources by oracle/build_ref_gpu.sh) against this build's mriSolver
    on the same input directory and flags (the Toeplitz configuration, written
    in the 1.0 format): wall time of each whole program run, file I/O included,
    and the reference's own printed kernel times."""
    import re
    import tempfile
    from __graft_entry__ import load_package
    load_package()
    from impatient_mri_b200 import io as mio, synth
    ref = ROOT / "oracle" / "_ref" / "mriSolver_ref"
    ours = ROOT / "impatient-mri_b200" / "bin" / "mriSolver"
    if not ref.exists():
        print(json.dumps({"impl": "reference-gpu", "unavailable":
                          "oracle/_ref/mriSolver_ref not built (oracle/build_ref_gpu.sh)"}))
        return 0
    case = synth.make_case(TOEP, seed=1003)
    o = case["opts"]
    M, N, C = case["M"], case["N"], case["num_coil"]
    rng = np.random.default_rng(11)
    kd = ((rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M)))
          * np.sqrt(np.mean(np.abs(case["x_true"]) ** 2) * N / 2)).astype(np.complex64)
    flags = ["-toeplitzGridding", "-ntime_segs", str(o["ntime_segs"]), "-gridOS_Q",
             str(o["gridOS_Q"]), "-gridOS_FH", str(o["gridOS_FH"]), "-cg_num",
             str(args.ref_cg), "-fdp", str(o["fd_penalizer"])]
    if args.ref_tv:
        flags += ["-tv", "-tv_num", str(o["tv_num"])]
    out = {"impl": "reference-gpu", "workload": TOEP, "flags": " ".join(flags)}
    with tempfile.TemporaryDirectory() as d:
        mio.write_dataset(d, "1.0", kx=case["kx"], ky=case["ky"], kz=case["kz"], t=case["t"],
                          ix=case["ix"], iy=case["iy"], iz=case["iz"], fm=case["fm"], kdata=kd,
                          sensi=case["sens"], dims=case["dims"], num_coil=C)
        for name, exe in (("ours", ours), ("reference", ref)):
            t0 = time.perf_counter()
            try:
                r = subprocess.run([str(exe), "-idir", d, *flags], capture_output=True,
                                   text=True, timeout=args.ref_timeout)
                wall = time.perf_counter() - t0
                res = {"wall_s": wall, "rc": r.returncode}
                for key, pat in (("q_ms", r"Q Kernel Time: ([0-9.]+)"),
                                 ("fhd_ms", r"F\^H\(d\) Kernel Time: ([0-9.]+)"),
                                 ("cg_ms", r"CG Execution Time: ([0-9.]+)")):
                    mt = re.search(pat, r.stdout)
                    if mt:
                        res[key] = float(mt.group(1))
                if r.returncode != 0:
                    res["tail"] = (r.stdout + r.stderr)[-400:]
            except subprocess.TimeoutExpired:
                res = {"wall_s": None, "timeout_s": args.ref_timeout}
            out[name] = res
            print(f"{name}: {res}", file=sys.stderr, flush=True)
    print(json.dumps(out))
    return 0


def run_toep_grid_only(args, local):
    """Q and F^H d by gridding for the Toeplitz 3-D geometry (the small command
    the gridding profiles are taken on), timed with CUDA events."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import synth
    torch.cuda.set_device(local)
    case = synth.make_case(TOEP, seed=1003)
    o = case["opts"]
    M, N, C = case["M"], case["N"], case["num_coil"]
    nx, ny, nz = case["dims"]
    L1, G = o["ntime_segs"] + 1, 8 * N
    f = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()
    rng = np.random.default_rng(11)
    kd = (rng.standard_normal((C, M)) + 1j * rng.standard_normal((C, M))).astype(np.complex64)
    D = {k: f(case[k]) for k in ("kx", "ky", "kz", "t", "fm")}
    sr, si = f(case["sens"].real.ravel()), f(case["sens"].imag.ravel())
    yr, yi = f(kd.real.ravel()), f(kd.imag.ravel())
    qr, qi = torch.zeros(L1 * G, device="cuda"), torch.zeros(L1 * G, device="cuda")
    fr, fi = torch.zeros(N, device="cuda"), torch.zeros(N, device="cuda")
    opts = pkg.toeplitz_options(ntime_segs=o["ntime_segs"], gridOS_Q=o["gridOS_Q"],
                                gridOS_FH=o["gridOS_FH"])
    with pkg.Context(local) as ctx:
        def run():
            pkg.toeplitz_q(ctx, opts, qr, qi, D["kx"], D["ky"], D["kz"], D["t"], M, nx, ny, nz)
            pkg.toeplitz_fhd(ctx, opts, fr, fi, yr, yi, D["kx"], D["ky"], D["kz"], D["t"],
                             D["fm"], sr, si, M, C, nx, ny, nz)
        for _ in range(max(args.warmup, 1)):
            run()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            run()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / max(args.steps, 1)
    print(json.dumps({"toep_grid_only": TOEP, "ms_q_plus_fhd": dt * 1e3}))
    return 0


def run_unet_only(args, local):
    """Training steps of the warm start's U-Net at 512x512, batch 8 (the small
    command the U-Net kernel profiles are taken on), timed with CUDA events.
    FLOP = 2 MACs forward + 4 MACs backward per image (data and weight
    gradients), against the measured dense BF16 tensor peak."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import learn
    torch.cuda.set_device(local)
    B, H, W = args.batch, 512, 512
    g = torch.Generator(device="cuda").manual_seed(3)
    x = torch.randn(B, 2, H * W, device="cuda", generator=g)
    t = 0.5 * x
    with pkg.Context(local) as ctx:
        net = pkg.UNet(ctx, B, H, W, seed=1)
        for _ in range(max(args.warmup, 1)):
            net.train_step(x, t, 1e-4)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.steps):
            net.train_step(x, t, 1e-4)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / max(args.steps, 1)
        f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        y = torch.zeros_like(x)
        f0.record()
        for _ in range(args.steps):
            net.forward(x, y)
        f1.record()
        torch.cuda.synchronize()
        ms_f = f0.elapsed_time(f1) / max(args.steps, 1)
        net.close()
    macs = learn.unet_macs(H, W) * B
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (
        ROOT / "MEASURED_PEAKS.json").exists() else {}
    bf16 = float(peaks.get("bf16_tflops", 1590.0))
    tf_train = 6.0 * macs / (ms / 1e3) / 1e12
    tf_fwd = 2.0 * macs / (ms_f / 1e3) / 1e12
    print(json.dumps({"unet_only": f"512x512 batch {B}", "ms_per_train_step": ms,
                      "ms_per_forward": ms_f, "train_tflops": tf_train, "forward_tflops": tf_fwd,
                      "bf16_peak_tflops": bf16, "forward_frac": tf_fwd / bf16,
                      "train_frac": tf_train / bf16}))
    return 0


def run_nudft_only(args, local):
    """Forward + adjoint NUDFT applies of the benchmark geometry through the
    operator C-ABI (the small command the kernel profiles are taken on)."""
    import torch
    from __graft_entry__ import load_package
    pkg = load_package()
    from impatient_mri_b200 import synth
    torch.cuda.set_device(local)
    f = lambda a: torch.as_tensor(np.ascontiguousarray(a, np.float32)).cuda()
    use_z = 1
    if args.nudft_coils:
        # seeded 2-D 256x256 image, M = 65536 random samples, field map, C coils
        C, n, M = args.nudft_coils, 256, 65536
        rng = np.random.default_rng(0)
        N = n * n
        gx = np.linspace(-0.5, 0.5, n, endpoint=False)
        X, Y = np.meshgrid(gx, gx, indexing="ij")
        case = dict(kx=rng.uniform(-n / 2, n / 2, M), ky=rng.uniform(-n / 2, n / 2, M),
                    kz=np.zeros(M), t=rng.uniform(0, 0.02, M), ix=X.ravel(), iy=Y.ravel(),
                    iz=np.zeros(N), fm=rng.uniform(-200, 200, N),
                    sens=rng.standard_normal((C, N)) + 1j * rng.standard_normal((C, N)),
                    x_true=rng.standard_normal(N) + 1j * rng.standard_normal(N))
        use_z = 0
    else:
        case = synth.make_case(BF3D)
        M, N, C = case["M"], case["N"], case["num_coil"]
    g = {k: f(case[k]) for k in ("kx", "ky", "kz", "t", "ix", "iy", "iz", "fm")}
    sr, si = f(case["sens"].real), f(case["sens"].imag)
    xr, xi = f(case["x_true"].real), f(case["x_true"].imag)
    yr = torch.zeros(C * M, device="cuda")
    yi = torch.zeros(C * M, device="cuda")
    with pkg.Context(local) as ctx:
        def pair():
            pkg.parallelFtGpu(ctx, yr, yi, xr, xi, g["kx"], g["ky"], g["kz"], g["ix"], g["iy"],
                              g["iz"], g["fm"], g["t"], M, N, sr, si, C, use_z)
            pkg.parallelIftGpu(ctx, xr, xi, yr, yi, g["kx"], g["ky"], g["kz"], g["ix"],
                               g["iy"], g["iz"], g["fm"], g["t"], M, N, sr, si, C, use_z)
        for _ in range(args.warmup):  # module loading and first-call setup stay out
            pair()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(args.steps):
            pair()
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / max(args.steps, 1)
    what = f"2-D 256x256, M=65536, {C} coils" if args.nudft_coils else BF3D
    print(json.dumps({"nudft_only": what, "ms_per_fwd_adj_pair": dt * 1e3}))
    return 0


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nudft-only", action="store_true",
                    help="only forward + adjoint NUDFT applies (profiling command)")
    ap.add_argument("--nudft-coils", type=int, default=0,
                    help="--nudft-only on a 2-D 256x256, M=65536 case with this many coils")
    ap.add_argument("--toep-grid-only", action="store_true",
                    help="only Toeplitz Q and F^H d gridding (profiling command)")
    ap.add_argument("--unet-only", action="store_true",
                    help="only U-Net training steps at 512x512 (profiling command)")
    ap.add_argument("--toep-apply-only", action="store_true",
                    help="only Toeplitz A^H A applications (profiling command)")
    ap.add_argument("--toep-dims", default="256,256,32",
                    help="--toep-apply-only: image nx,ny,nz")
    ap.add_argument("--toep-coils", type=int, default=4, help="--toep-apply-only: coils")
    ap.add_argument("--toep-segs", type=int, default=9,
                    help="--toep-apply-only: time segments L+1")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference", "reference-gpu"])
    ap.add_argument("--ref-cg", type=int, default=20, help="reference-gpu: cg_num")
    ap.add_argument("--ref-tv", action="store_true", help="reference-gpu: add -tv -tv_num 10")
    ap.add_argument("--ref-timeout", type=int, default=1200)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--slices", type=int, default=64,
                    help="batch384: slices timed (all 64 by default: the configuration)")
    ap.add_argument("--workload", default=WARM, choices=[WARM, BF3D, C1, TOEP, BATCH],
                    help="warm512 (default, the metric: learned warm start vs plain CG at "
                         "512x512 with 32 coils, with the brute-force 3-D NUDFT block), "
                         "bf3d_64x64x16 (brute-force 3-D), bf2d_64 (the 2-D one-coil case), "
                         "the Toeplitz 3-D case, or the 64-slice 384x384 batch")
    ap.add_argument("--retrain", action="store_true", help="warm512: train even if weights exist")
    ap.add_argument("--save-weights", default=None, help="warm512: where to write trained weights")
    ap.add_argument("--train-images", type=int, default=2000)
    ap.add_argument("--test-images", type=int, default=8)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8)
    ap.add_argument("--lr", type=float, default=1e-3)
    args = ap.parse_args()
    ws, rank, local = dist_setup()
    try:
        if args.nudft_only:
            return run_nudft_only(args, local)
        if args.toep_apply_only:
            return run_toep_apply_only(args, local)
        if args.unet_only:
            return run_unet_only(args, local)
        if args.toep_grid_only:
            return run_toep_grid_only(args, local)
        if args.impl == "reference-gpu":
            return run_toeplitz_ref_gpu(args) if rank == 0 else 0
        if args.impl == "reference":
            return run_reference(args, ws, rank)
        if args.workload == TOEP:
            return run_toeplitz(args, ws, rank, local)
        if args.workload == C1:
            return run_bf2d(args, ws, rank, local)
        if args.workload == WARM:
            return run_warm(args, local) if args.retrain else run_headline(args, ws, rank, local)
        if args.workload == BATCH:
            return run_batch(args, ws, rank, local)
        return run_ours(args, ws, rank, local)
    finally:
        _replicas().finalize(ws)


if __name__ == "__main__":
    sys.exit(main())
