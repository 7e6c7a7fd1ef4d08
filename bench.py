#!/usr/bin/env python
"""Benchmark: Stokes solves/s to 1e-9 relative residual on one B200.

Workload: 3D 128^3 periodic variable-viscosity Stokes problem (contrast 100,
inertial alpha = rho/dt with alpha*dx^2/beta0 = 0.1, seeded synthetic
6-mode log-viscosity, N(0,1) mean-removed velocity rhs), block
lower-triangular preconditioner (precon_type 2), visc_type -2.

A step is one full solve.  Reported:
  value   solves/s of the mixed-precision method (FP64 flexible GMRES around
          an FP32 staggered V-cycle + FP32 pressure V-cycle), inputs resident
          in HBM, each solve to |b-Ax|/|b| <= 1e-9 in FP64;
  e2e     the same through the C ABI with host buffers (pinned numpy arrays,
          host->device and device->host copies inside the timed region);
  plain_fp64  the same FGMRES with the FP64 V-cycle (reference arithmetic);
  reference_gmres  the reference's own algorithm (left-preconditioned
          GMRES, FP64) timed on the GPU;
  roofline of the dominant kernel (one Gauss-Seidel smooth of the finest
          level), measured live with CUDA events on the solver's stream;
  cpu_baseline  the CPU oracle (C++ restatement of the reference algorithm):
          one full solve of the same problem on every host thread, plus one
          full 64^3 solve of the same family on one core, rank 0 only;
  learned_stage  the same mixed method with the learned stage (network
          trained on the GPU before the timed region, on 64^3 problems of
          this workload's family, its corrections added as extra FGMRES
          directions, judged by the GMRES residual: dropped for the rest of a
          solve after two network columns that lower the residual estimate by
          less than 10%), and `always_on` with every correction added --
          measured beside `value`, which is the faster mixed configuration
          without it;
  mixed_vs_fp64  relative L2 error of the mixed solution against the FP64 one.

N > 1 GPUs: replicas only (one independent solve per GPU, a different seed
per rank, no collective on the data path); value = total solves / max time.
`--impl reference` times the CPU oracle (the reference Fortran cannot be
built on this machine) on the same workload: every step one full solve.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Stokes solves/s to 1e-9 rel. residual: plain FP64 vs mixed+learned, same B200"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="product", choices=["product", "reference"])
    ap.add_argument("--n", type=int, default=128)
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU-baseline leg")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-stage leg")
    ap.add_argument("--learned-steps", type=int, default=1000, help="training steps (4 pairs each) of the learned stage")
    ap.add_argument("--learned-fields", type=int, default=100)
    return ap.parse_args()


# ------------------------------------------------------------------ clocks
class ClockSampler:
    """nvidia-smi samples every 50 ms.  Entering starts the sampler and waits
    for its first row (nvidia-smi takes longer to start than a short timed
    region lasts), so the rows taken between enter and exit are the timed
    region's; when the region is shorter than one period, the first row
    after it stands in (window "adjacent")."""

    PERIOD_MS = 50

    def __init__(self, device_index: int):
        self.dev = device_index
        self.rows = []
        self._proc = None
        self._lo = self._hi = 0
        self.window = "during"

    def start(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self._proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.dev}", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms",
                 str(self.PERIOD_MS)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except (OSError, FileNotFoundError):
            self._proc = None
            return
        t0 = time.time()
        while not self.rows and time.time() - t0 < 5.0 and self._proc.poll() is None:
            time.sleep(0.005)

    def __enter__(self):
        if self._proc is None:
            self.start()
        self._lo = len(self.rows)
        return self

    def _read(self):
        for line in self._proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        self._hi = len(self.rows)
        if self._proc is None:
            return
        if self._hi == self._lo:
            self.window = "adjacent"
            t0 = time.time()
            while len(self.rows) == self._lo and time.time() - t0 < 1.0 and self._proc.poll() is None:
                time.sleep(0.005)
            self._hi = len(self.rows)
        self._proc.terminate()
        try:
            self._proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self._proc.kill()

    def summary(self):
        rows = self.rows[self._lo:self._hi]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[1]) for r in rows if r[1].replace(".", "").isdigit())
        mx = max((float(r[2]) for r in rows if r[2].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in rows:
            for i, nm in enumerate(names):
                if len(r) > 5 + i and r[5 + i].lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(rows), "window": self.window, "period_ms": self.PERIOD_MS}


# ------------------------------------------------------------------ distributed plumbing
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(world, v, op):
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(world, v):
    """the slowest rank's time (every rank calls it, in the same order)"""
    import torch.distributed as dist
    return _reduce(world, v, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(world, v):
    import torch.distributed as dist
    return _reduce(world, v, dist.ReduceOp.SUM if world > 1 else None)


# ------------------------------------------------------------------ CPU baseline (oracle)
def cpu_solve(prob, knobs_kw: dict, threads: int | None = None):
    """Time one full solve of `prob` by the CPU oracle (the C++ restatement of
    the reference's left-preconditioned GMRES, FP64) with `threads` OpenMP
    threads (None: all).  Returns (seconds, stats)."""
    from oracle import oracle as O
    O.build()
    if threads is not None:
        O.set_threads(threads)
    try:
        t0 = time.perf_counter()
        rc, _, _, _, _, st = O.solve(prob, O.default_knobs(**knobs_kw))
        dt = time.perf_counter() - t0
    finally:
        if threads is not None:
            O.set_threads(omp_threads())
    if rc < 0:
        raise RuntimeError(f"oracle solve failed with status {rc}")
    return dt, st


def omp_threads():
    try:
        return int(os.environ.get("OMP_NUM_THREADS", "")) or os.cpu_count()
    except ValueError:
        return os.cpu_count()


def cpu_model():
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


# ------------------------------------------------------------------ reference arm
def run_reference(args, world, rank):
    """Every step is one full oracle solve of the benchmark problem on all
    host threads (nothing extrapolated)."""
    if rank != 0:
        return
    from lowmachmixtures_b200 import synth
    prob = synth.config_3d_128(0, n=args.n)
    kn = dict(precon_type=2, visc_type=-2)
    times, iters = [], []
    for s in range(args.warmup + args.steps):
        dt, st = cpu_solve(prob, kn)
        if s >= args.warmup:
            times.append(dt)
            iters.append(st["total_iter"])
    solve_s = sum(times) / len(times)
    v = 1.0 / solve_s
    cores = omp_threads()
    sample = (f"one full solve of the {args.n}^3 problem per step (reference GMRES(5) to the reference stop rule, "
              f"{iters[-1]} iterations), {cores} threads of {cpu_model()}")
    line = {
        "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": solve_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
        "config": {"workload": f"stokes_3d_{args.n}^3_inertial_contrast100", "precon_type": 2,
                   "method": "reference GMRES(5), FP64 (CPU oracle restating the Fortran; the Fortran itself "
                             "cannot be built: no Fortran compiler, BoxLib not vendored)"},
        "iterations": iters, "seconds_per_solve": times,
        "cpu_baseline": {"value": v, "unit": "solves/s", "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ product arm
def run_product(args, world, rank, local):
    import numpy as np
    import torch

    from lowmachmixtures_b200 import abi, synth
    from lowmachmixtures_b200 import build as B
    from lowmachmixtures_b200.gmres import StokesSolver

    B.build()
    torch.cuda.set_device(local)
    n = args.n
    prob = synth.config_3d_128(seed=rank, n=n)
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()  # noqa: E731
    d_in = dict(b_u=[dev(a) for a in prob.b_u], b_p=dev(prob.b_p), alpha_fc=[dev(a) for a in prob.alpha_fc],
                beta=dev(prob.beta), beta_ed=[dev(a) for a in prob.beta_ed], gamma=dev(prob.gamma))
    d_xu = [torch.zeros_like(d_in["b_u"][0]) for _ in range(3)]
    d_xp = torch.zeros_like(d_in["b_p"])
    base = dict(precon_type=2, visc_type=-2)
    mixed_kn = abi.make_knobs(**base, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32, orthogonalization=1)
    plain_kn = abi.make_knobs(**base, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP64)
    ref_kn = abi.make_knobs(**base, method=abi.LMM_METHOD_GMRES)

    def solve_dev(s):
        for t in d_xu:
            t.zero_()
        d_xp.zero_()
        return s.solve_device(d_in["b_u"], d_in["b_p"], d_xu, d_xp, d_in["alpha_fc"], d_in["beta"], d_in["beta_ed"],
                              d_in["gamma"], prob.theta_alpha)

    def timed_device(s, steps, warmup, clocks=None):
        ext = torch.cuda.ExternalStream(s.stream_ptr())
        for _ in range(warmup):
            solve_dev(s)
        barrier(world)
        torch.cuda.synchronize()
        l0 = s.lib.lmm_kernel_launches()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        stats = []
        if clocks:
            clocks.__enter__()
        e0.record(ext)
        for _ in range(steps):
            _, _, st = solve_dev(s)
            stats.append(st)
        e1.record(ext)
        torch.cuda.synchronize()
        if clocks:
            clocks.__exit__(None, None, None)
        ms = e0.elapsed_time(e1)
        barrier(world)
        launches = s.lib.lmm_kernel_launches() - l0
        return ms, stats, launches

    mixed = StokesSolver(3, (n, n, n), prob.dx, knobs=mixed_kn, device=local)
    plain = StokesSolver(3, (n, n, n), prob.dx, knobs=plain_kn, device=local)
    refg = StokesSolver(3, (n, n, n), prob.dx, knobs=ref_kn, device=local)

    clocks = ClockSampler(local)
    ms_mixed, st_mixed, launches = timed_device(mixed, args.steps, args.warmup, clocks)
    ms_mixed = max_over_ranks(world, ms_mixed)
    total = sum_over_ranks(world, float(args.steps))
    value = total / (ms_mixed / 1e3)

    ms_plain, st_plain, _ = timed_device(plain, max(2, args.steps // 2), 1)
    ms_plain = max_over_ranks(world, ms_plain)
    plain_steps = max(2, args.steps // 2)
    ms_ref, st_ref, _ = timed_device(refg, max(2, args.steps // 2), 1)
    ms_ref = max_over_ranks(world, ms_ref)

    # e2e through the C ABI with pinned host buffers
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_in = dict(b_u=[pin(a) for a in prob.b_u], b_p=pin(prob.b_p), alpha_fc=[pin(a) for a in prob.alpha_fc],
                beta=pin(prob.beta), beta_ed=[pin(a) for a in prob.beta_ed], gamma=pin(prob.gamma))
    # x is the initial guess in and the solution out: every step gets its own
    # zeroed pinned arrays, prepared before the timed region (a caller's fresh
    # zero initial guess), so no host-side zeroing is timed
    h_x = [([pin(np.zeros(prob.shape)) for _ in range(3)], pin(np.zeros(prob.shape))) for _ in range(args.steps + 1)]

    def solve_host(q):
        h_xu, h_xp = h_x[q]
        return mixed.solve(h_in["b_u"], h_in["b_p"], h_xu, h_xp, h_in["alpha_fc"], h_in["beta"], h_in["beta_ed"],
                           h_in["gamma"], prob.theta_alpha)

    solve_host(args.steps)
    barrier(world)
    torch.cuda.synchronize()
    ext = torch.cuda.ExternalStream(mixed.stream_ptr())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(ext)
    t0 = time.perf_counter()
    for q in range(args.steps):
        solve_host(q)
    t1 = time.perf_counter()
    e1.record(ext)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(world, (t1 - t0) * 1e3)
    e2e_value = total / (ms_e2e / 1e3)
    nf = prob.shape[0] * prob.shape[1] * prob.shape[2]
    # b_u b_p alpha beta beta_ed x0_u x0_p (+ gamma, read only by visc_type +-3)
    h2d = 8 * nf * (3 + 1 + 3 + 1 + 3 + 3 + 1 + (1 if abs(mixed.knobs.visc_type) == 3 else 0))
    d2h = 8 * nf * 4

    # roofline: one Gauss-Seidel smooth of the finest level (6 colour kernels)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    ms_smooth32 = mixed.time_op(1, reps=20)
    ms_smooth64 = plain.time_op(0, reps=20)
    ms_apply64 = plain.time_op(2, reps=20)
    ms_vc32 = mixed.time_op(5, reps=5)
    ms_vc64 = plain.time_op(4, reps=5)
    # algorithmic bytes (the survey's per-cell figures): a smooth w(4F + N + E)
    # = 16 wN (phi r/w, rhs, alpha, beta_cc, 3 edge arrays), stag_applyop
    # w(3F + N + E) = 13 wN (phi, alpha, beta, edges in; L out).  With
    # theta*alpha one value on every face (this workload's constant density)
    # the kernels take it as a scalar: this problem's own minimum has no
    # alpha arrays (13 wN and 10 wN), reported beside the survey's
    a0 = float(np.asarray(prob.alpha_fc[0]).flat[0])
    alpha_uniform = all(bool(np.all(np.asarray(a) == a0)) for a in prob.alpha_fc)
    w_smooth_min, w_apply_min = (13, 10) if alpha_uniform else (16, 13)
    bytes_smooth32 = 16 * 4 * nf
    bytes_smooth64 = 16 * 8 * nf
    bytes_apply64 = 13 * 8 * nf
    gbs = lambda b, ms: b / (ms * 1e-3) / 1e9  # noqa: E731
    roofline = {"bound": "hbm", "kernel": f"gs_colour_fp32 (one full smooth: 6 colour launches in alternating plane order, {n}^3)",
                "achieved": gbs(bytes_smooth32, ms_smooth32), "peak": peak, "unit": "GB/s",
                "frac": gbs(bytes_smooth32, ms_smooth32) / peak, "traffic": None,
                "peak_source": peak_src,
                "algorithmic_bytes": bytes_smooth32, "alpha_uniform": alpha_uniform,
                "problem_min_bytes": w_smooth_min * 4 * nf,
                "frac_of_problem_min": gbs(w_smooth_min * 4 * nf, ms_smooth32) / peak,
                "ms_per_launch": ms_smooth32 / 6.0, "ms_per_smooth": ms_smooth32}
    # the opt-in TMA-staged red/black pair smoother on the same level
    tma_kn = abi.make_knobs(**base, method=abi.LMM_METHOD_FGMRES, precision=abi.LMM_PRECISION_FP32, orthogonalization=1,
                            smoother_tma=1)
    with StokesSolver(3, (n, n, n), prob.dx, knobs=tma_kn, device=local) as tma:
        tma.load_coeffs(d_in["alpha_fc"], d_in["beta"], d_in["beta_ed"], d_in["gamma"], prob.theta_alpha)
        ms_smooth32_tma = tma.time_op(1, reps=20)
    kernels = {
        "gs_smooth_fp32_tma_pair": {"ms": ms_smooth32_tma, "GB/s": gbs(bytes_smooth32, ms_smooth32_tma),
                                    "frac": gbs(bytes_smooth32, ms_smooth32_tma) / peak,
                                    "note": "opt-in (smoother_tma = 1): slower than the colour launches"},
        "gs_smooth_fp64": {"ms": ms_smooth64, "GB/s": gbs(bytes_smooth64, ms_smooth64),
                           "frac": gbs(bytes_smooth64, ms_smooth64) / peak},
        "stag_applyop_fp64": {"ms": ms_apply64, "GB/s": gbs(bytes_apply64, ms_apply64),
                              "frac": gbs(bytes_apply64, ms_apply64) / peak,
                              "frac_of_problem_min": gbs(w_apply_min * 8 * nf, ms_apply64) / peak},
        "vcycle_fp32_ms": ms_vc32, "vcycle_fp64_ms": ms_vc64,
    }

    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_mixed / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64 Krylov + f32 preconditioner", "data": "synthetic",
        "config": {"workload": f"stokes_3d_{n}^3_inertial_contrast100", "n": n, "precon_type": 2, "visc_type": -2,
                   "method": "FGMRES(5) FP64 (classical Gram-Schmidt) + FP32 V-cycles", "rel_tol": 1e-9,
                   "l2": "inputs larger than L2 (device working set > 2 GB per solve)",
                   "parallelism": "replicas" if world > 1 else "single GPU"},
        "iterations": [s["total_iter"] for s in st_mixed],
        "true_rel_residual": [s["norm_resid_true"] / s["norm_b"] for s in st_mixed],
        "plain_fp64": {"value": sum_over_ranks(world, float(plain_steps)) / (ms_plain / 1e3),
                       "ms_per_step": ms_plain / plain_steps, "iterations": [s["total_iter"] for s in st_plain]},
        "reference_gmres_gpu": {"value": sum_over_ranks(world, float(plain_steps)) / (ms_ref / 1e3),
                                "ms_per_step": ms_ref / plain_steps,
                                "iterations": [s["total_iter"] for s in st_ref]},
        "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h},
        "gpu_launches": launches,
        "roofline": roofline,
        "kernels": kernels,
        "autotune": autotune_choices(n),
        "clocks": clocks.summary(),
    }
    if rank == 0 and world == 1 and not args.no_cpu:
        # one full oracle solve of the same problem on every host thread, and
        # one full solve of the 64^3 problem of the same family on one core
        # (a 128^3 solve on one core takes minutes)
        dt, st = cpu_solve(prob, base)
        prob64 = synth.config_3d_128(rank, n=64)
        dt1, st1 = cpu_solve(prob64, base, threads=1)
        dt64, st64 = cpu_solve(prob64, base)
        line["cpu_baseline"] = {
            "value": 1.0 / dt, "unit": "solves/s", "cores": omp_threads(), "kind": "port",
            "sample": (f"one full oracle solve (reference GMRES(5), FP64) of the same {n}^3 problem: {dt:.1f} s, "
                       f"{st['total_iter']} iterations, {omp_threads()} threads of {cpu_model()}"),
            "single_core": {"value": 1.0 / dt1, "unit": "solves/s", "cores": 1, "seconds": dt1,
                            "iterations": st1["total_iter"],
                            "sample": "one full oracle solve of the 64^3 problem of the same family on one core"},
            "all_cores_64": {"value": 1.0 / dt64, "unit": "solves/s", "cores": omp_threads(), "seconds": dt64,
                             "sample": "the same 64^3 solve on every host thread"}}
    # error of the mixed-precision solution against the FP64 one (same inputs;
    # the FP64 path is bit-for-bit the oracle's arithmetic)
    solve_dev(mixed)
    xu_m, xp_m = [t.clone() for t in d_xu], d_xp.clone()
    solve_dev(plain)
    num = sum(float(((a - b) ** 2).sum()) for a, b in zip(xu_m, d_xu))
    den = sum(float((b ** 2).sum()) for b in d_xu)
    pm, pp = xp_m - xp_m.mean(), d_xp - d_xp.mean()
    line["mixed_vs_fp64"] = {"velocity_rel_l2": (num / den) ** 0.5,
                             "pressure_rel_l2_mean_removed": float(((pm - pp) ** 2).sum().sqrt() / (pp ** 2).sum().sqrt())}
    if not args.no_learned:
        line["learned_stage"] = learned_leg(args, prob, n, local, solve_dev, d_in, d_xu, d_xp, world)
    traffic = profiled_traffic("gs_colour_fp32_128")
    if traffic is not None and n == 128:
        # six colour launches per smooth, each captured alone with cold caches
        # (live, consecutive colours of a component share part of it in L2)
        line["roofline"]["traffic"] = traffic * 6
    for s in (mixed, plain, refg):
        s.close()
    if rank == 0:
        print(json.dumps(line), flush=True)


def autotune_choices(n):
    """the block shapes the library's autotuner chose for this grid's levels"""
    from lowmachmixtures_b200 import _native
    lib = _native.load()
    need = lib.lmm_autotune_report(None, 0)
    buf = ctypes.create_string_buffer(need + 1)
    lib.lmm_autotune_report(buf, need + 1)
    return [ln for ln in buf.value.decode().splitlines() if f" {n}x{n}x{n}:" in ln]


def profiled_traffic(key):
    """DRAM bytes per launch of a kernel from the committed ncu summary
    (profiles/traffic.txt: `key bytes_per_launch` lines), or None."""
    try:
        for ln in open(os.path.join(ROOT, "profiles", "traffic.txt")):
            parts = ln.split()
            if len(parts) >= 2 and parts[0] == key:
                return float(parts[1])
    except OSError:
        pass
    return None


def learned_leg(args, prob, n, local, solve_dev, d_in, d_xu, d_xp, world):
    """Train the learned stage (untimed) on 64^3 problems of this workload's
    family (theta alpha dx^2 = 0.1, contrast log-uniform in [10, 1000]), load
    the weights into a network on the bench grid, and time the mixed method
    with the stage judged by the GMRES residual (learned_stage = 4) and with
    it always on (learned_stage = 1)."""
    import torch

    from lowmachmixtures_b200 import learned
    from lowmachmixtures_b200.gmres import StokesSolver
    t0 = time.perf_counter()
    net64, hist, _ = learned.train(n=64, fields=args.learned_fields, steps=args.learned_steps, batch=4, theta_alpha=0.1)
    train_s = time.perf_counter() - t0
    params = net64.params()
    net64.close()
    net = learned.Net((n, n, n), 1, 0)
    net.set_params(params)

    def timed(stage):
        kn = learned.mixed_knobs(learned_stage=stage)
        with StokesSolver(3, (n, n, n), prob.dx, knobs=kn, device=local) as s:
            assert s.lib.lmm_stokes_set_net(s._h, net.h) == 0
            solve_dev(s)
            ext = torch.cuda.ExternalStream(s.stream_ptr())
            steps = max(1, args.steps // 2)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(ext)
            iters = []
            for _ in range(steps):
                _, _, st = solve_dev(s)
                iters.append(st["total_iter"])
            e1.record(ext)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            acc, tried = ctypes.c_int(), ctypes.c_int()
            s.lib.lmm_learned_stats(s._h, ctypes.byref(acc), ctypes.byref(tried))
            rel = st["norm_resid_true"] / st["norm_b"]
        return {"value": steps / (ms / 1e3), "unit": "solves/s", "ms_per_step": ms / steps, "iterations": iters,
                "true_rel_residual": rel, "network_columns_kept": acc.value, "network_corrections": tried.value}

    # the stage as the GMRES residual judges it (learned_stage = 4: network
    # columns dropped for the rest of a solve after two that lower the
    # residual estimate by less than 10%), and always on (learned_stage = 1)
    line = timed(4)
    line["mode"] = "judged (learned_stage = 4)"
    line["always_on"] = timed(1)
    net.close()
    line.update({"train_seconds": train_s, "train_pairs": args.learned_steps * 4, "train_fields": args.learned_fields,
                 "train_grid": "64^3", "loss_first": hist[0], "loss_last": sum(hist[-20:]) / 20})
    return line


def main():
    args = parse()
    if args.impl == "reference":
        # the CPU oracle runs on rank 0 only; other ranks exit without work
        world = int(os.environ.get("WORLD_SIZE", "1"))
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, world, rank)
        return
    world, rank, local = dist_setup(args)
    try:
        run_product(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
