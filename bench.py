#!/usr/bin/env python
"""SIMP iterations/s on a 256x128x128 hex8 cantilever (4,194,304 elements,
12,830,211 DOF), one step = one full SIMP iteration on the device: densities ->
element moduli and the multigrid hierarchy, MGPCG solve of K U = F to relative
residual 1e-8 (cold start, so the residual is relative to ||F||), element energies,
sensitivities, sensitivity filter (r = 1.5), OC bisection and the change test.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Inputs are synthetic: the density field is a sum of 16 random-phase cosines
(seed 2) clipped to [1e-3, 1]; the load is -1 in z on each node of the line
(x = nelx, y = 0..nely, z = 0); the x = 0 face is fixed.  Every vector of the solve is
larger than the 126 MB L2 (12.8M doubles = 103 MB, and a V-cycle streams several),
so no L2 flush is needed between steps.

--impl reference times the CPU restatement of the reference's algorithm (oracle/,
single thread, as the reference's one worker thread) on a bounded sample and reports
the same metric by extrapolation; see cpu_model().
"""
import argparse
import faulthandler
import json
import math
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NELX, NELY, NELZ = 256, 128, 128
METRIC = "SIMP iters/s at 12.8M DOF (256x128x128 hex8), FP64 MGPCG to 1e-8 rel. residual"
UNIT = "SIMP iter/s"
VOLFRAC, PENAL, RMIN, TOL = 0.3, 3.0, 1.5, 1e-8
# MGPCG iterations per SIMP step of this workload, measured by the FP64 GPU path
# (same algorithm as the oracle); used only by the reference arm's extrapolation.
REF_ITERS_PER_STEP = None


def density_field(nelx, nely, nelz, seed=2):
    """rho = clip(0.5 + 0.25 S / sqrt(8), 1e-3, 1), S = sum of 16 cosines
    cos(2 pi (k . c) + phi) with integer k in [1,4]^3, phi ~ U[0, 2 pi), c the element
    centre in unit-cube coordinates; reference element order (x fastest)."""
    rng = np.random.default_rng(seed)
    k = rng.integers(1, 5, size=(16, 3))
    phi = rng.uniform(0, 2 * np.pi, 16)
    cx = (np.arange(nelx) + 0.5) / nelx
    cy = (np.arange(nely) + 0.5) / nely
    cz = (np.arange(nelz) + 0.5) / nelz
    S = np.zeros((nelz, nely, nelx))
    for i in range(16):
        a = 2 * np.pi * k[i, 0] * cx
        b = 2 * np.pi * k[i, 1] * cy
        c = 2 * np.pi * k[i, 2] * cz
        S += np.cos(c[:, None, None] + b[None, :, None] + a[None, None, :] + phi[i])
    return np.clip(0.5 + 0.25 * S / np.sqrt(8), 1e-3, 1.0).astype(np.float32).ravel()


def cantilever_load(nelx, nely, nelz):
    from topologyoptimization_b200 import mesh
    F = np.zeros(mesh.ndof(nelx, nely, nelz))
    for j in range(nely + 1):
        F[3 * mesh.node_id(nelx, j, 0, nely, nelz) + 2] = -1.0
    return F


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:  # noqa: BLE001
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during a region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:  # noqa: BLE001
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:  # noqa: BLE001
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        try:
            for line in open(self.path):
                f = [t.strip() for t in line.split(",")]
                if len(f) < 9:
                    continue
                try:
                    sm.append(float(f[1]))
                    mx.append(float(f[2]))
                except ValueError:
                    continue
                for n, v in zip(names, f[5:9]):
                    if v.lower().startswith("active"):
                        reasons.add(n)
        except Exception:  # noqa: BLE001
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.remove(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def fp64_peak_tflops(torch):
    """Dense FP64 rate of cuBLAS DGEMM (8192^3), best of 5: the FP64 denominator."""
    a = torch.randn(8192, 8192, dtype=torch.float64, device="cuda")
    b = torch.randn_like(a)
    best = 1e9
    for _ in range(6):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    return 2 * 8192 ** 3 / best / 1e12


def cpu_model(t_apply, t_vcycle, t_update, t_post, iters):
    """Time of one SIMP iteration of the single-threaded CPU restatement: hierarchy
    update + iters x (fine apply + V-cycle) + energy/sensitivity/filter/OC (the
    vector updates of CG are O(ndof) and below 1% of an apply)."""
    return t_update + iters * (t_apply + t_vcycle) + t_post


def cpu_sample(iters_per_step):
    """Bounded sample on the host: one fine-grid apply, one V-cycle, one hierarchy
    update and one energy+sensitivity+filter+OC pass at full size (~30-60 s)."""
    from oracle import pyoracle as O
    from topologyoptimization_b200 import mesh
    x = density_field(NELX, NELY, NELZ)
    fixed = mesh.fixed_mask(NELX, NELY, NELZ, "left")
    F = cantilever_load(NELX, NELY, NELZ)
    Ke = O.lk(0.3)
    mg = O.MG(NELX, NELY, NELZ, Ke, fixed)
    t0 = time.perf_counter()
    mg.update(x, PENAL)
    t_update = time.perf_counter() - t0
    t0 = time.perf_counter()
    Ap = mg.apply(F)
    t_apply = time.perf_counter() - t0
    t0 = time.perf_counter()
    mg.vcycle(F)
    t_vcycle = time.perf_counter() - t0
    U = Ap * 1e-3
    t0 = time.perf_counter()
    en = O.element_energy(Ke, NELX, NELY, NELZ, U)
    dc = O.sensitivity(x, x, en, PENAL, 1.0, 1.0, False)
    hs = O.filter_hs(NELX, NELY, NELZ, RMIN)
    dcn = O.filter_sens(NELX, NELY, NELZ, RMIN, hs, x, dc)
    O.oc(x, VOLFRAC, dcn)
    t_post = time.perf_counter() - t0
    del mg
    t = cpu_model(t_apply, t_vcycle, t_update, t_post, iters_per_step)
    return 1.0 / t, dict(t_apply_s=t_apply, t_vcycle_s=t_vcycle, t_update_s=t_update, t_post_s=t_post,
                         iters_per_step=iters_per_step)


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    iters = REF_ITERS_PER_STEP
    if iters is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference arm needs the measured MGPCG "
                                                               "iteration count of this workload"}))
        return 0
    from oracle import pyoracle as O
    from topologyoptimization_b200 import mesh
    x = density_field(NELX, NELY, NELZ)
    fixed = mesh.fixed_mask(NELX, NELY, NELZ, "left")
    F = cantilever_load(NELX, NELY, NELZ)
    mg = O.MG(NELX, NELY, NELZ, O.lk(0.3), fixed)
    t0 = time.perf_counter()
    mg.update(x, PENAL)
    t_update = time.perf_counter() - t0
    t0 = time.perf_counter()
    mg.vcycle(F)
    t_vcycle = time.perf_counter() - t0
    t_post = 0.0  # measured below in the warm-up
    for _ in range(args.warmup):
        mg.apply(F)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        mg.apply(F)
        times.append(time.perf_counter() - t0)
    t_apply = float(np.median(times))
    t_step = cpu_model(t_apply, t_vcycle, t_update, t_post, iters)
    v = 1.0 / t_step
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"SIMP cantilever {NELX}x{NELY}x{NELZ}", "nel": NELX * NELY * NELZ,
                       "ndof": 3 * (NELX + 1) * (NELY + 1) * (NELZ + 1)},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"per step one full-size fine-grid apply ({args.steps} steps, median "
                                       f"{t_apply:.2f} s); one V-cycle {t_vcycle:.2f} s and one hierarchy update "
                                       f"{t_update:.2f} s timed once; SIMP iteration = update + {iters} x "
                                       f"(apply + V-cycle)"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args, rank, world, local_rank):
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", device_id=torch.device("cuda", local_rank))
    nel = NELX * NELY * NELZ
    x0 = density_field(NELX, NELY, NELZ)
    fixed = mesh.fixed_mask(NELX, NELY, NELZ, "left")
    F = cantilever_load(NELX, NELY, NELZ)
    P = Problem(NELX, NELY, NELZ, fixed)
    P.set_load(F)
    torch.cuda.synchronize()
    # caller-owned stream: every torch op below runs on it too, so ordering is explicit
    stream = torch.cuda.Stream()
    P.set_stream(stream)
    so = N.default_solve_opts(precond=N.PREC_MG, max_iter=2000, tol=TOL, warm_start=0, ref_epsilon=0)
    opts = N.SimpOpts(volfrac=VOLFRAC, penal=PENAL, rmin=RMIN, E0=1.0, Emin=1e-9, beta=1.0, use_projection=0,
                      solve=so)

    def barrier():
        if dist is not None:
            dist.barrier()

    # ---- device-resident steps ------------------------------------------------------
    with torch.cuda.stream(stream):
        d_x = torch.from_numpy(x0).cuda()
        for _ in range(args.warmup):
            P.simp_step_dev(d_x, opts)
    torch.cuda.synchronize()
    barrier()
    infos = []
    l0 = N.lib().tpo_launch_count()
    with ClockSampler(local_rank) as clk:
        with torch.cuda.stream(stream):
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for _ in range(args.steps):
                infos.append(P.simp_step_dev(d_x, opts))
            ev1.record(stream)
        torch.cuda.synchronize()
    launches = N.lib().tpo_launch_count() - l0
    t = ev0.elapsed_time(ev1) / 1e3
    barrier()
    t_max = t
    if dist is not None:
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_max = float(tt.item())
    clocks = clk.summary()
    iters = [i.cg_iterations for i in infos]
    value = world * args.steps / t_max

    # ---- end to end through host buffers ------------------------------------------
    x_host = torch.from_numpy(x0.copy()).pin_memory()
    with torch.cuda.stream(stream):
        d_x.copy_(torch.from_numpy(x0))
        for _ in range(args.warmup):
            d_x.copy_(x_host, non_blocking=True)
            P.simp_step_dev(d_x, opts)
            x_host.copy_(d_x)
    torch.cuda.synchronize()
    barrier()
    t0 = time.perf_counter()
    comp = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            d_x.copy_(x_host, non_blocking=True)
        info = P.simp_step_dev(d_x, opts)
        with torch.cuda.stream(stream):
            x_host.copy_(d_x, non_blocking=True)
        stream.synchronize()
        comp.append(info.compliance)
    t_e2e = time.perf_counter() - t0
    if dist is not None:
        tt = torch.tensor([t_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        t_e2e = float(tt.item())
    e2e = {"value": world * args.steps / t_e2e, "unit": UNIT, "h2d_bytes_per_step": 4 * nel,
           "d2h_bytes_per_step": 4 * nel + 8 + 8}

    # ---- dominant kernel: FP64 structured apply ------------------------------------
    ndof = P.ndof
    with torch.cuda.stream(stream):
        u = torch.randn(ndof, dtype=torch.float64, device="cuda")
        out = torch.empty_like(u)
        P.set_densities(d_x, PENAL)
        for _ in range(3):
            P.apply_dev(u, out)
    torch.cuda.synchronize()
    reps = 20
    with torch.cuda.stream(stream):
        a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a0.record(stream)
        for _ in range(reps):
            P.apply_dev(u, out)
        a1.record(stream)
    torch.cuda.synchronize()
    t_apply = a0.elapsed_time(a1) / 1e3 / reps
    alg_bytes = 8 * (2 * ndof + nel)
    torch.cuda.synchronize()
    xs = d_x.double()
    nel_active = int(((1e-9 + xs ** 3 * (1 - 1e-9)) > 1e-6).sum().item())
    flops = 2 * 576 * nel_active
    hbm_peak, peak_kind = measured_peaks()
    achieved = alg_bytes / t_apply / 1e9
    traffic = None
    tp = os.path.join(ROOT, "profiles", "apply_fp64_traffic.json")
    if os.path.exists(tp):
        try:
            traffic = json.load(open(tp))["bytes_per_launch_full_size"]
        except Exception:  # noqa: BLE001
            traffic = None
    fp64_peak = fp64_peak_tflops(torch) if rank == 0 else None
    roofline = {"bound": "hbm", "kernel": "k_apply<double> (node-centric FP64 K*u, 12.8M DOF)",
                "achieved": achieved, "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                "peak_kind": peak_kind, "traffic": traffic, "launch_ms": t_apply * 1e3,
                "algorithmic_bytes": alg_bytes,
                "compute": {"achieved_tflops_fp64": flops / t_apply / 1e12,
                            "peak_tflops_fp64_dgemm": fp64_peak,
                            "frac": (flops / t_apply / 1e12 / fp64_peak) if fp64_peak else None,
                            "note": "FP64 apply is FP64-pipe bound (576 FMA per node); the DGEMM rate "
                                    "measured here is the FP64 denominator"}}

    line = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            del u, out
            torch.cuda.empty_cache()
            v, d = cpu_sample(float(np.mean(iters)))
            cpu = {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": f"oracle (C restatement of the reference, 1 thread) at full size: apply "
                             f"{d['t_apply_s']:.2f} s, V-cycle {d['t_vcycle_s']:.2f} s, update "
                             f"{d['t_update_s']:.2f} s, energy+filter+OC {d['t_post_s']:.2f} s; SIMP iteration "
                             f"= update + {d['iters_per_step']:.1f} x (apply + V-cycle) + post (MGPCG "
                             f"iteration count from this run)"}
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": {"workload": f"SIMP cantilever {NELX}x{NELY}x{NELZ}", "nel": nel,
                           "ndof": ndof, "solver": "FP64 MGPCG, reference hierarchy (6 levels, V(2,2), "
                                                   "omega 0.5, dense Galerkin coarse + 30 sweeps)",
                           "tol": TOL, "parallelism": f"replicas x{world}",
                           "l2": "inputs larger than L2 (103 MB per vector)"},
                "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clocks,
                "solve": {"mgpcg_iters_per_step": iters,
                          "rel_residual_last": infos[-1].rel_residual if infos else None,
                          "compliance_last": comp[-1] if comp else None}}
        print(json.dumps(line))
    P.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    global NELX, NELY, NELZ
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", default=f"{NELX}x{NELY}x{NELZ}",
                    help="elements per axis, e.g. 128x64x64 for a profiling case (default: the benchmark grid)")
    args = ap.parse_args()
    NELX, NELY, NELZ = (int(v) for v in args.grid.lower().split("x"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
