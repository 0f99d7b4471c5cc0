#!/usr/bin/env python
"""SIMP iterations/s on a 256x128x128 hex8 cantilever (4,194,304 elements,
12,830,211 DOF), one step = one full SIMP iteration on the device: densities ->
element moduli and the multigrid hierarchy, MGPCG solve of K U = F to relative
residual 1e-8 (cold start, so the residual is relative to ||F||), element energies,
sensitivities, sensitivity filter (r = 1.5), OC bisection and the change test.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Inputs are synthetic: the density field is a sum of 16 random-phase cosines
(seed 2) clipped to [1e-3, 1]; the load is -1 in z on each node of the line
(x = nelx, y = 0..nely, z = 0); the x = 0 face is fixed.  As in the reference's loop,
the elements under the fixed face and under the loaded line are preserved (start at
density 1, left alone by OC).  Every vector of the solve is
larger than the 126 MB L2 (12.8M doubles = 103 MB, and a V-cycle streams several),
so no L2 flush is needed between steps.

--impl reference times the CPU restatement of the reference's algorithm (oracle/,
single thread, as the reference's one worker thread) on a bounded sample and reports
the same metric by extrapolation: the full-size costs of an apply, a V-cycle, a
hierarchy update and the post-solve pass, times the MG-PCG iteration count of the
reference's solver run to convergence on the 64x32x32 grid of this workload (see
reference_iterations(), reference_model()).

The line also carries the chosen form's error against an FP64 solve to 1e-12 at 12.8M
DOF (chosen_form_error), the 128x64x64 K.u microbenchmark (apply_microbench) and the
batched load-case configuration (batched_load_cases: 8 right-hand sides at 160x80x80,
3 timed block and sequential solves after 3 warm-up, see measure_batched()) and, as
next_rows, the KSP-BDDC solve and the 2D worker timed beside the oracle (measure_ksp_bddc(),
measure_simp2d()).
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
METRIC = "SIMP iters/s at 12.7M DOF: mixed-prec MGPCG vs plain FP64 GPU @1e-8 rel res"
UNIT = "SIMP iter/s"
VOLFRAC, PENAL, RMIN, TOL = 0.3, 3.0, 1.5, 1e-8
# MAX_CG_ITERATIONS of the reference (js/optimizer-worker-3d.js:45), the cap its worker
# gives every MGPCG solve (:3780)
REF_CAP = 400
# grid of the reference arm's converging solve (the iteration count of a multigrid solve
# changes little with the grid; the full-size solve takes hours on one core)
REF_COUNT_GRID = (64, 32, 32)


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


def preserved_elements(nelx, nely, nelz):
    """Elements the SIMP loop keeps solid, as the reference does for its constraint and
    force surfaces (js/optimizer-worker-3d.js:1957-1988): the x = 0 layer under the
    fixed face and the row of elements under the loaded node line (ex = nelx - 1,
    ez = 0).  uint8 mask in reference element order."""
    m = np.zeros(nelx * nely * nelz, np.uint8)
    m.reshape(nelz, nely, nelx)[:, :, 0] = 1
    m.reshape(nelz, nely, nelx)[0, :, nelx - 1] = 1
    return m


def start_design(nelx, nely, nelz):
    """The density field with the preserved elements at full density."""
    x = density_field(nelx, nely, nelz)
    x[preserved_elements(nelx, nely, nelz) == 1] = 1.0
    return x


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


def cpu_model(t_apply, t_vcycle, t_update, t_post, iters):
    """Time of one SIMP iteration of the single-threaded CPU restatement: hierarchy
    update + iters x (fine apply + V-cycle) + energy/sensitivity/filter/OC (the
    vector updates of CG are O(ndof) and below 1% of an apply)."""
    return t_update + iters * (t_apply + t_vcycle) + t_post


def cpu_post_time(O, Ke, x, U):
    """One pass of element energies, sensitivities, sensitivity filter and OC on the
    host (the filter weights are built once per run by the reference, so not here)."""
    hs = O.filter_hs(NELX, NELY, NELZ, RMIN)
    t0 = time.perf_counter()
    en = O.element_energy(Ke, NELX, NELY, NELZ, U)
    dc = O.sensitivity(x, x, en, PENAL, 1.0, 1.0, False)
    dcn = O.filter_sens(NELX, NELY, NELZ, RMIN, hs, x, dc)
    O.oc(x, VOLFRAC, dcn, preserved=preserved_elements(NELX, NELY, NELZ))
    return time.perf_counter() - t0


def reference_iterations():
    """MG-PCG iterations the reference's solver needs on this workload, from a converging
    run: the oracle's ebeMGPCG (the reference's hierarchy: 6 levels, omega 0.5, V(2,2), 30
    coarse sweeps, dense Galerkin <= 3000 DOF; cold start, relative tolerance 1e-8, cap
    2000) on the REF_COUNT_GRID version of this workload (same density-field formula,
    support and line load).  The load is scaled by 1e6 for this count only: the reference
    adds an absolute 1e-12 to pAp and rz (assembly/index.ts:1124-1187), which with unit
    loads stalls its recurrence near 1e-7 before it reaches 1e-8; scaled, the count is the
    one the algorithm needs.  Returns (iterations, seconds, converged)."""
    from oracle import pyoracle as O
    from topologyoptimization_b200 import mesh
    nx, ny, nz = REF_COUNT_GRID
    x = start_design(nx, ny, nz)
    fixed = mesh.fixed_mask(nx, ny, nz, "left")
    F = cantilever_load(nx, ny, nz) * 1e6
    t0 = time.perf_counter()
    mg = O.MG(nx, ny, nz, O.lk(0.3), fixed)
    mg.update(x, PENAL)
    _, it = mg.mgpcg(F, 2000, TOL)
    return it, time.perf_counter() - t0, it < 2000


def reference_costs(apply_reps=1):
    """Per-iteration and per-step costs of the reference's algorithm at full size on one
    host core (the oracle): fine-grid applies (apply_reps of them, each timed), one
    V-cycle, one hierarchy update and one energy + sensitivity + filter + OC pass."""
    from oracle import pyoracle as O
    from topologyoptimization_b200 import mesh
    x = start_design(NELX, NELY, NELZ)
    fixed = mesh.fixed_mask(NELX, NELY, NELZ, "left")
    F = cantilever_load(NELX, NELY, NELZ)
    Ke = O.lk(0.3)
    mg = O.MG(NELX, NELY, NELZ, Ke, fixed)
    t0 = time.perf_counter()
    mg.update(x, PENAL)
    t_update = time.perf_counter() - t0
    t0 = time.perf_counter()
    mg.vcycle(F)
    t_vcycle = time.perf_counter() - t0
    t_apply = []
    for _ in range(max(1, apply_reps)):
        t0 = time.perf_counter()
        Ap = mg.apply(F)
        t_apply.append(time.perf_counter() - t0)
    del mg
    t_post = cpu_post_time(O, Ke, x, Ap * 1e-3)
    return dict(t_apply_s=t_apply, t_vcycle_s=t_vcycle, t_update_s=t_update, t_post_s=t_post)


def reference_model(costs, iters, warmup=0):
    """Seconds per SIMP iteration of the reference's algorithm, extrapolated from the timed
    pieces: update + min(iters, REF_CAP) x (apply + V-cycle) + post."""
    t_apply = float(np.median(costs["t_apply_s"][warmup:] or costs["t_apply_s"]))
    n = min(iters, REF_CAP)
    return cpu_model(t_apply, costs["t_vcycle_s"], costs["t_update_s"], costs["t_post_s"], n), t_apply, n


def reference_sample_text(costs, t_apply, iters, n, t_count, converged, apply_desc):
    cnx, cny, cnz = REF_COUNT_GRID
    capped = f", capped at the reference's {REF_CAP}" if n < iters else ""
    return (f"extrapolated: oracle (C restatement of the reference, 1 thread) at full size, {apply_desc} "
            f"(median {t_apply:.2f} s), one V-cycle {costs['t_vcycle_s']:.2f} s, one hierarchy update "
            f"{costs['t_update_s']:.2f} s, one energy+sensitivity+filter+OC pass {costs['t_post_s']:.2f} s; SIMP "
            f"iteration = update + {n} x (apply + V-cycle) + post, {iters} the MG-PCG iterations of the "
            f"reference's solver run to 1e-8 by the oracle on the {cnx}x{cny}x{cnz} grid of this workload "
            f"({'converged' if converged else 'not converged at 2000'}, {t_count:.1f} s){capped}")


class Replicas:
    """Rank coordination of a replica run (one independent problem per rank, no data
    exchange): a barrier on both sides of a timed region and the maximum of a duration over
    the ranks.  `dist` is torch.distributed (None for one process); `device` is where the
    reduction's tensor lives ("cuda" under NCCL, "cpu" under gloo)."""

    def __init__(self, dist, device):
        self.dist, self.device = dist, device

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()

    def max_over_ranks(self, t):
        if self.dist is None:
            return t
        import torch
        tt = torch.tensor([t], device=self.device, dtype=torch.float64)
        self.dist.all_reduce(tt, op=self.dist.ReduceOp.MAX)
        return float(tt.item())

    @staticmethod
    def job_rate(world, steps, t_max):
        """Whole-job throughput: every rank ran `steps` steps, the slowest took t_max."""
        return world * steps / t_max


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    iters, t_count, converged = reference_iterations()
    costs = reference_costs(apply_reps=args.warmup + args.steps)
    t_step, t_apply, n = reference_model(costs, iters, warmup=args.warmup)
    v = 1.0 / t_step
    line = {"metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_step * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"SIMP cantilever {NELX}x{NELY}x{NELZ}", "nel": NELX * NELY * NELZ,
                       "ndof": 3 * (NELX + 1) * (NELY + 1) * (NELZ + 1)},
            "impl": "reference",
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": reference_sample_text(costs, t_apply, iters, n, t_count, converged,
                                                             f"one fine-grid apply per step ({args.steps} timed "
                                                             f"after {args.warmup} warm-up)")},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def solver_arms(N, levels=6):
    """The solver configurations timed by the bench.  All use the reference's multigrid
    transfers and rediscretised coarse levels with V(2,2) (6 levels).  The chosen form and
    its FP64 comparator smooth the structured levels with the degree-2 Chebyshev
    polynomial on [kappa / 16, kappa], kappa a bound on lambda_max(D^-1 A) (the same
    applies as damped Jacobi, stronger damping of the upper spectrum; the reference's
    omega = 0.5 Jacobi is above the bound's limit once a node is held by a single
    element), damp the dense levels with min(0.5, 1.9 / Gershgorin bound), and solve the
    675-DOF coarsest level directly instead of the reference's 30 sweeps.  `levels` is the
    hierarchy depth of the chosen form (6 for the benchmark grid; a grid 2^k times larger
    per axis needs k more for its coarsest level to stay a dense direct solve)."""
    chosen_mg = dict(coarse_direct=1, safe_omega=1, chebyshev=1, cheb_ratio=16.0, max_levels=levels)
    return {
        # headline: FP64 PCG whose multigrid preconditioner runs in FP32 (every level)
        "mixed": dict(mg=chosen_mg, solve=dict(precision=N.F32_PRECOND, tensor_cores=0)),
        # the same with TF32 tcgen05 applies on the fine level of the V-cycle
        "mixed_tf32_vcycle": dict(mg=chosen_mg, solve=dict(precision=N.F32_PRECOND, tensor_cores=1)),
        # the same with 3xTF32 tcgen05 applies (FP32-class accuracy) on the fine level
        "mixed_3xtf32_vcycle": dict(mg=chosen_mg, solve=dict(precision=N.F32_PRECOND, tensor_cores=3)),
        # FP32 MG-PCG recurrence with FP64 reliable updates (defect correction) at a 0.3 drop
        "mixed_fp32_recurrence": dict(mg=chosen_mg, solve=dict(precision=N.MIXED, inner_tol=0.3, tensor_cores=0)),
        # plain FP64 GPU MG-PCG with the same hierarchy
        "fp64": dict(mg=chosen_mg, solve=dict(precision=N.FP64)),
        # the drop-in: FP64 with the reference's hierarchy (omega 0.5, 30 coarse sweeps)
        "fp64_reference_hierarchy": dict(mg=dict(), solve=dict(precision=N.FP64)),
    }


def time_kernels(torch, P, x0, stream, reps=20):
    """CUDA-event time (s) of one launch of the FP32, TF32 tcgen05 and FP64 fine-grid
    applies of problem P at densities x0, averaged over `reps` back-to-back launches
    on `stream` after 3 warm-up launches.  Launches alternate between two input/output
    pairs (238 MB in FP32 with the moduli, more than the 126 MB L2), so no launch finds
    its input in L2 from the one before."""
    with torch.cuda.stream(stream):
        P.set_densities(torch.from_numpy(x0).cuda(), PENAL)
        u = [torch.randn(P.ndof, dtype=torch.float64, device="cuda") for _ in range(2)]
        out = [torch.empty_like(v) for v in u]
        u32 = [v.float() for v in u]
        o32 = [torch.empty_like(v) for v in u32]
    stream.synchronize()

    def kernel_ms(fn):
        with torch.cuda.stream(stream):
            for i in range(4):
                fn(i & 1)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for i in range(reps):
                fn(i & 1)
            a1.record(stream)
        stream.synchronize()
        return a0.elapsed_time(a1) / reps / 1e3

    t_32 = kernel_ms(lambda i: P.apply_f32_dev(u32[i], o32[i]))
    t_tc = kernel_ms(lambda i: P.apply_tf32_dev(u32[i], o32[i]))
    t_64 = kernel_ms(lambda i: P.apply_dev(u[i], out[i]))
    time_kernels.t_3x = kernel_ms(lambda i: P.apply_3xtf32_dev(u32[i], o32[i]))
    return t_32, t_tc, t_64


def chosen_form_error(torch, P, x0, F, stream, mixed_solve, fp64_solve):
    """Error of the chosen form's solution at the start design against an FP64 solve to
    1e-12 (same hierarchy): max-norm relative error of U, relative error of the compliance
    F.U and max-norm relative error of the compliance sensitivities dc_e = -p x_e^(p-1)
    E0 u_e^T Ke u_e (from the element energies).  The FP64 solve to the same 1e-8 is
    reported beside it: the part of the error the tolerance itself leaves."""
    from topologyoptimization_b200 import _native as N
    xs = torch.from_numpy(x0).cuda()
    x64 = torch.from_numpy(x0.astype(np.float64)).cuda()
    out = {}
    with torch.cuda.stream(stream):
        P.set_densities(xs, PENAL)
        sols = {}
        for name, kw, tol in (("reference", fp64_solve, 1e-12), ("mixed", mixed_solve, TOL), ("fp64", fp64_solve, TOL)):
            o = N.default_solve_opts(precond=N.PREC_MG, max_iter=4000, tol=tol, warm_start=0, ref_epsilon=0, **kw)
            dU = torch.zeros(P.ndof, dtype=torch.float64, device="cuda")
            info = P.solve_dev(dU, o)
            en = torch.empty(P.nel, dtype=torch.float32, device="cuda")
            P.element_energy_dev(dU, en)
            dc = -PENAL * x64 ** (PENAL - 1) * en.double()
            sols[name] = (dU, info, dc)
    stream.synchronize()
    Ur, ir, dcr = sols["reference"]
    for name in ("mixed", "fp64"):
        dU, info, dc = sols[name]
        out[name] = {"u_rel_err": float((dU - Ur).abs().max() / Ur.abs().max()),
                     "compliance_rel_err": abs(info.compliance - ir.compliance) / abs(ir.compliance),
                     "dc_rel_err": float((dc - dcr).abs().max() / dcr.abs().max()),
                     "iterations": info.iterations, "rel_residual": info.rel_residual}
    out["against"] = (f"FP64 MG-PCG to 1e-12 at the start design ({ir.iterations} iterations, residual "
                      f"{ir.rel_residual:.1e})")
    return out


def apply_microbench(torch, reps=20):
    """The matrix-free K.u microbenchmark: 128x64x64 hex8 elements (1,635,075 DOF),
    densities i.i.d. U[1e-3, 1] (seed 0), u i.i.d. N(0, 1) (seed 1) with the x = 0 face's
    DOFs zeroed, penal 3, nu 0.3.  Each apply variant is timed with CUDA events over
    `reps` launches alternating two input/output pairs; GB/s counts the algorithmic bytes
    s (2 ndof + nel); the error is max |Ku - Ku_fp64| / max |Ku_fp64|."""
    from topologyoptimization_b200 import Problem, mesh
    nx, ny, nz = 128, 64, 64
    fixed = mesh.fixed_mask(nx, ny, nz, "left")
    x = np.random.default_rng(0).uniform(1e-3, 1.0, nx * ny * nz).astype(np.float32)
    u = np.random.default_rng(1).standard_normal(mesh.ndof(nx, ny, nz)) * (fixed == 0)
    res = {"workload": f"K.u microbenchmark {nx}x{ny}x{nz}", "ndof": int(len(u))}
    st = torch.cuda.Stream()
    with Problem(nx, ny, nz, fixed) as P, torch.cuda.stream(st):
        P.set_stream(st)
        P.set_densities(x, PENAL)
        nel, ndof = P.nel, P.ndof
        u64 = [torch.from_numpy(u).cuda(), torch.from_numpy(np.roll(u, 3)).cuda()]
        u32 = [v.float() for v in u64]
        o64 = [torch.empty_like(v) for v in u64]
        o32 = [torch.empty_like(v) for v in u32]
        variants = {"fp64": (P.apply_dev, u64, o64, 8), "fp32": (P.apply_f32_dev, u32, o32, 4),
                    "tf32_tcgen05": (P.apply_tf32_dev, u32, o32, 4), "3xtf32_tcgen05": (P.apply_3xtf32_dev, u32, o32, 4)}
        if hasattr(P, "apply_bf16_dev"):
            variants["bf16_tcgen05"] = (P.apply_bf16_dev, u32, o32, 4)
        torch.cuda.synchronize()
        P.apply_dev(u64[0], o64[0])
        torch.cuda.synchronize()
        ref = o64[0].clone()
        for name, (fn, ins, outs, s) in variants.items():
            for i in range(4):
                fn(ins[i & 1], outs[i & 1])
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            for i in range(reps):
                fn(ins[i & 1], outs[i & 1])
            e1.record(st)
            torch.cuda.synchronize()
            t = e0.elapsed_time(e1) / reps / 1e3
            fn(ins[0], outs[0])
            torch.cuda.synchronize()
            err = float((outs[0].double() - ref).abs().max() / ref.abs().max())
            res[name] = {"us": t * 1e6, "gbs": s * (2 * ndof + nel) / t / 1e9, "max_rel_err_vs_fp64": err}
        P.set_stream(None)
    return res


def run_batched(args):
    """--batched: the batched load-case configuration as its own JSON line (see
    measure_batched)."""
    import torch
    torch.cuda.set_device(0)
    dims = (160, 80, 80) if args.grid == "256x128x128" else (NELX, NELY, NELZ)
    print(json.dumps(measure_batched(args.steps, args.warmup, dims)))
    return 0


def measure_batched(steps, warmup, dims):
    """The batched load-case configuration, 160x80x80 hex8 elements (3,168,963 DOF),
    supports at the four corners of the z = 0 face, uniform start density 0.2, 8 unit point
    loads at top-face nodes (position and direction from numpy.random.default_rng(30 + k),
    direction normalize(N(0, I3))).  One step = the 8 solves to 1e-8 (cold start), timed as
    one block solve (tpo_solve_multi_dev) and as 8 sequential single solves, in FP64 and
    with the FP32 multigrid preconditioner, by CUDA events on the current device."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    nx, ny, nz = dims
    nrhs = 8
    fixed = mesh.fixed_mask(nx, ny, nz, "bottom-corners")
    F = np.zeros((nrhs, mesh.ndof(nx, ny, nz)))
    for k in range(nrhs):
        rng = np.random.default_rng(30 + k)
        ix, iy = int(rng.integers(0, nx + 1)), int(rng.integers(0, ny + 1))
        d = rng.standard_normal(3)
        F[k, 3 * mesh.node_id(ix, iy, nz, ny, nz):3 * mesh.node_id(ix, iy, nz, ny, nz) + 3] = d / np.linalg.norm(d)
    x = np.full(nx * ny * nz, 0.2, np.float32)
    P = Problem(nx, ny, nz, fixed, mg=N.default_mg_opts(coarse_direct=1, safe_omega=1, chebyshev=1, cheb_ratio=16.0))
    P.set_densities(x, PENAL)
    dF = torch.from_numpy(F).cuda()
    dU = torch.zeros_like(dF)
    out = {}
    for name, prec in (("fp64", N.FP64), ("mixed", N.F32_PRECOND)):
        opts = N.default_solve_opts(precond=N.PREC_MG, precision=prec, max_iter=2000, tol=TOL, warm_start=0,
                                    ref_epsilon=0)

        def block():
            dU.zero_()
            return P.solve_multi_dev(dF, dU, opts)

        def sequential():
            infos = []
            for k in range(nrhs):
                P.set_load(F[k])
                du = dU[k]
                du.zero_()
                infos.append(P.solve_dev(du, opts))
            return infos

        for label, fn in (("block", block), ("sequential", sequential)):
            for _ in range(warmup):
                fn()
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record()
            for _ in range(steps):
                infos = fn()
            ev1.record()
            torch.cuda.synchronize()
            t = ev0.elapsed_time(ev1) / 1e3 / steps
            out[f"{name}_{label}"] = {"solves_per_s": nrhs / t, "ms_per_8_solves": t * 1e3,
                                      "iterations": [i.iterations for i in infos],
                                      "converged": [i.converged for i in infos]}
    P.close()
    line = {"metric": "solves/s, 8 load cases at 3.17M DOF: block MG-PCG vs 8 sequential solves @1e-8",
            "unit": "solves/s", "n_gpus": 1, "steps": steps, "warmup": warmup, "data": "synthetic",
            "config": {"workload": f"batched load cases {nx}x{ny}x{nz}", "nrhs": nrhs, "bc": "bottom-corners",
                       "density": "uniform 0.2", "solver": "6-level MG V(2,2), Chebyshev smoothing on [kappa/16, kappa], direct coarse solve"},
            "value": out["mixed_block"]["solves_per_s"], "higher_is_better": True,
            "speedup_block_vs_sequential_fp64": out["fp64_block"]["solves_per_s"] / out["fp64_sequential"]["solves_per_s"],
            "speedup_block_vs_sequential_mixed": out["mixed_block"]["solves_per_s"] / out["mixed_sequential"]["solves_per_s"],
            "arms": out}
    return line


def measure_ksp_bddc(torch, dims=(128, 64, 64), iters=100, reps=3, cpu_iters=2):
    """The reference's KSP CG with its BDDC preconditioner (ebeKSP_BDDC, linearSolver
    'petsc') at 128x64x64 (1,635,075 DOF): the bench's density field and cantilever on that
    grid, cold start, the worker's 3 smoother applies, a fixed count of 100 iterations (the
    preconditioner is indefinite, so a run to a tolerance ends at the cap either way).
    GPU: CUDA events around `reps` solves after one warm-up.  CPU: the oracle's
    ebeKSP_BDDC for `cpu_iters` iterations on one core (setup included)."""
    from oracle import pyoracle as O
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    x = start_design(*dims)
    fixed = mesh.fixed_mask(*dims, "left")
    F = cantilever_load(*dims)
    stream = torch.cuda.Stream()
    with Problem(*dims, fixed) as P:
        P.set_stream(stream)
        P.set_densities(x, PENAL)
        P.set_load(F)
        opts = N.default_solve_opts(precond=N.PREC_BDDC, max_iter=iters, tol=1e-30, warm_start=0, ref_epsilon=1,
                                    bddc_smoother_iters=3)
        with torch.cuda.stream(stream):
            dU = torch.zeros(P.ndof, dtype=torch.float64, device="cuda")
        P.solve_dev(dU, opts)
        stream.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            info = P.solve_dev(dU, opts)
        e1.record(stream)
        e1.synchronize()
        t_gpu = e0.elapsed_time(e1) / 1e3 / reps
        gpu_iters = info.iterations
    t0 = time.perf_counter()
    _, cpu_it = O.ksp_bddc(*dims, O.lk(0.3), x, PENAL, fixed, F, cpu_iters, 1e-30)
    t_cpu = time.perf_counter() - t0
    return {"workload": f"KSP-BDDC PCG {dims[0]}x{dims[1]}x{dims[2]} ({mesh.ndof(*dims)} DOF), "
                        f"{iters} iterations, 3 smoother applies",
            "unit": "PCG iterations/s", "gpu": gpu_iters / t_gpu, "gpu_ms_per_iteration": 1e3 * t_gpu / gpu_iters,
            "cpu": cpu_it / t_cpu, "cpu_kind": "port", "cpu_cores": 1,
            "cpu_sample": f"oracle ebeKSP_BDDC, {cpu_it} iterations incl. setup, {t_cpu:.2f} s",
            "gpu_over_cpu": (gpu_iters / t_gpu) / (cpu_it / t_cpu)}


def measure_simp2d(dims=(300, 100), iters=10, cpu_iters=3):
    """The 2D worker (js/optimizer-worker.js) at 300x100 Q4 elements (60,802 DOF): the
    cantilever of its defaults ('left', 'down'), penal 3, no projection, its CG tolerance
    schedule, `iters` iterations through TopologyOptimizerWorker.optimize (wall clock of the
    public call, one device sync per iteration as the worker makes).  CPU: the oracle's 2D
    loop for `cpu_iters` iterations on one core; the CG counts of those iterations are
    compared."""
    from oracle import pyoracle as O
    from topologyoptimization_b200 import mesh
    from topologyoptimization_b200.worker2d import TopologyOptimizerWorker
    nx, ny = dims
    cfg = dict(volumeFraction=0.3, maxIterations=iters, penaltyFactor=3.0, filterRadius=1.5, penalStart=3.0,
               useProjection=False, constraintPosition="left", forceDirection="down")
    w = TopologyOptimizerWorker()
    w.optimize({"nx": nx, "ny": ny}, dict(cfg, maxIterations=2))  # warm-up: module load, first allocation
    t0 = time.perf_counter()
    r = w.optimize({"nx": nx, "ny": ny}, cfg)
    t_gpu = time.perf_counter() - t0
    fixed = mesh.fixed_mask2d(nx, ny, "left")
    F = mesh.load_vector2d(nx, ny, "down")
    pres = np.zeros(nx * ny, np.uint8)
    pres[mesh.constraint_elements2d(nx, ny, "left")] = 1
    pres[mesh.force_elements2d(nx, ny, "down")] = 1
    t0 = time.perf_counter()
    ro = O.simp2d(nx, ny, F, fixed, pres, None, max_iter=cpu_iters, use_projection=0, penal_start=3.0)
    t_cpu = time.perf_counter() - t0
    k = min(cpu_iters, int(r["iterations"]))
    return {"workload": f"2D SIMP cantilever {nx}x{ny} ({mesh.ndof2d(nx, ny)} DOF), {r['iterations']} iterations",
            "unit": "SIMP iter/s", "gpu": r["iterations"] / t_gpu, "cpu": ro["iterations"] / t_cpu,
            "cpu_kind": "port", "cpu_cores": 1, "cpu_sample": f"oracle 2D loop, {ro['iterations']} iterations, "
                                                              f"{t_cpu:.2f} s",
            "cg_iterations": [int(v) for v in r["cgIterations"]],
            "cg_counts_match_oracle": bool(np.array_equal(np.asarray(r["cgIterations"][:k]), ro["cg"][:k])),
            "gpu_over_cpu": (r["iterations"] / t_gpu) / (ro["iterations"] / t_cpu)}


def run_kernels(args):
    """--kernels: only the fine-grid apply kernels of one problem at --grid (the case
    the kernel profiles in profiles/ are captured on)."""
    import torch
    from topologyoptimization_b200 import Problem, mesh
    from topologyoptimization_b200 import _native as N
    torch.cuda.set_device(0)
    x0 = start_design(NELX, NELY, NELZ)
    P = Problem(NELX, NELY, NELZ, mesh.fixed_mask(NELX, NELY, NELZ, "left"), mg=N.default_mg_opts(coarse_direct=1))
    stream = torch.cuda.Stream()
    P.set_stream(stream)
    t_32, t_tc, t_64 = time_kernels(torch, P, x0, stream, reps=args.steps)
    nel, ndof = P.nel, P.ndof
    print(json.dumps({"grid": f"{NELX}x{NELY}x{NELZ}", "nel": nel, "ndof": ndof,
                      "k_apply_w<float>_ms": t_32 * 1e3, "k_apply_tc_ms": t_tc * 1e3,
                      "k_apply_tc_3xtf32_ms": time_kernels.t_3x * 1e3, "k_apply_w<double>_ms": t_64 * 1e3,
                      "gbs_f32": 4 * (2 * ndof + nel) / t_32 / 1e9, "gbs_f64": 8 * (2 * ndof + nel) / t_64 / 1e9}))
    P.close()
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
    x0 = start_design(NELX, NELY, NELZ)
    fixed = mesh.fixed_mask(NELX, NELY, NELZ, "left")
    F = cantilever_load(NELX, NELY, NELZ)
    arms = solver_arms(N, args.levels)
    torch.cuda.synchronize()
    stream = torch.cuda.Stream()  # caller-owned; every torch op below runs on it too
    with torch.cuda.stream(stream):
        d_pres = torch.from_numpy(preserved_elements(NELX, NELY, NELZ)).cuda()

    ranks = Replicas(dist, "cuda")
    barrier, max_over_ranks = ranks.barrier, ranks.max_over_ranks

    problems = {}

    def problem_for(mgkw):
        key = tuple(sorted(mgkw.items()))
        if key not in problems:
            P = Problem(NELX, NELY, NELZ, fixed, mg=N.default_mg_opts(**mgkw))
            P.set_load(F)
            P.set_stream(stream)
            problems[key] = P
        return problems[key]

    def simp_opts(solve_kw):
        so = N.default_solve_opts(precond=N.PREC_MG, max_iter=2000, tol=TOL, warm_start=0, ref_epsilon=0, **solve_kw)
        return N.SimpOpts(volfrac=VOLFRAC, penal=PENAL, rmin=RMIN, E0=1.0, Emin=1e-9, beta=1.0, use_projection=0,
                          guard_sensitivities=1, solve=so)

    def time_arm(name, steps, warmup, clocks=None):
        arm = arms[name]
        P = problem_for(arm["mg"])
        opts = simp_opts(arm["solve"])
        with torch.cuda.stream(stream):
            d_x = torch.from_numpy(x0).cuda()
            for _ in range(warmup):
                P.simp_step_dev(d_x, opts, d_pres)
        stream.synchronize()
        barrier()
        infos = []
        l0 = N.lib().tpo_launch_count()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            for _ in range(steps):
                infos.append(P.simp_step_dev(d_x, opts, d_pres))
            ev1.record(stream)
        stream.synchronize()
        launches = N.lib().tpo_launch_count() - l0
        t = max_over_ranks(ev0.elapsed_time(ev1) / 1e3)
        barrier()
        return dict(value=Replicas.job_rate(world, steps, t), ms_per_step=t / steps * 1e3, launches=launches,
                    iters=[i.cg_iterations for i in infos], converged=[i.converged for i in infos],
                    rel_residual_last=infos[-1].rel_residual,
                    compliance=[i.compliance for i in infos])

    # ---- the headline arm, device-resident, with clock sampling --------------------------
    with ClockSampler(local_rank) as clk:
        head = time_arm("mixed", args.steps, args.warmup)
    clocks = clk.summary()
    wanted = [a.strip() for a in args.arms.split(",")] if args.arms else list(arms)
    others = {k: time_arm(k, args.steps, args.warmup) for k in arms if k != "mixed" and k in wanted}

    # ---- end to end through host buffers (headline arm) --------------------------------
    # tpo_simp_step: the design and the preserved mask go in from pinned host memory and
    # the design comes back every step, inside the C-ABI call
    P = problem_for(arms["mixed"]["mg"])
    opts = simp_opts(arms["mixed"]["solve"])
    x_host = torch.from_numpy(x0.copy()).pin_memory()
    pres_host = torch.from_numpy(preserved_elements(NELX, NELY, NELZ)).pin_memory()
    for _ in range(args.warmup):
        P.simp_step(x_host, opts, pres_host)  # x_host now holds the design after the warm-up steps
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        P.simp_step(x_host, opts, pres_host)
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    e2e = {"value": Replicas.job_rate(world, args.steps, t_e2e), "unit": UNIT, "h2d_bytes_per_step": 5 * nel,
           "d2h_bytes_per_step": 4 * nel + 8 + 8, "call": "tpo_simp_step (host arrays)"}

    # ---- dominant kernels: FP32 apply (mixed), TF32 tcgen05 apply and FP64 apply ----
    ndof = P.ndof
    t_32, t_tc, t_64 = time_kernels(torch, P, x0, stream)
    xs = torch.from_numpy(x0).double()
    nel_active = int(((1e-9 + xs ** 3 * (1 - 1e-9)) > 1e-6).sum().item())
    flops = 2 * 576 * nel_active
    hbm_peak, peak_kind = measured_peaks()
    bytes32 = 4 * (2 * ndof + nel)
    bytes64 = 8 * (2 * ndof + nel)
    # "dense_equiv" rates count the 2 x 576 flops per active element of E_e Ke u_e; the
    # Walsh-basis kernels reach the same result with about 140 operations per element
    roofline = {"bound": "hbm", "kernel": f"k_apply_w<float> (FP32 Walsh-basis structured apply, {ndof / 1e6:.1f}M DOF)",
                "achieved": bytes32 / t_32 / 1e9, "peak": hbm_peak, "unit": "GB/s",
                "frac": bytes32 / t_32 / 1e9 / hbm_peak, "peak_kind": peak_kind,
                "traffic": profile_traffic("apply_w_f32_256x128x128.md"), "launch_ms": t_32 * 1e3,
                "algorithmic_bytes": bytes32, "dense_equiv_fp32_tflops": flops / t_32 / 1e12,
                "other_kernels": {
                    "k_apply_tc": {"launch_ms": t_tc * 1e3, "achieved_gbs": bytes32 / t_tc / 1e9,
                                   "tensor_tflops": flops / t_tc / 1e12,
                                   "traffic": profile_traffic("apply_tc_256x128x128.md")},
                    "k_apply_w<double>": {"launch_ms": t_64 * 1e3, "achieved_gbs": bytes64 / t_64 / 1e9,
                                          "frac_of_hbm": bytes64 / t_64 / 1e9 / hbm_peak,
                                          "dense_equiv_fp64_tflops": flops / t_64 / 1e12,
                                          "traffic": profile_traffic("apply_w_f64_256x128x128.md")}}}

    err = chosen_form_error(torch, problem_for(arms["mixed"]["mg"]), x0, F, stream, arms["mixed"]["solve"],
                            arms["fp64"]["solve"]) if "fp64" in arms else None
    micro = apply_microbench(torch) if not args.no_micro else None
    batched = measure_batched(3, 3, (160, 80, 80)) if rank == 0 and world == 1 and not args.no_batched else None
    rows = None
    if rank == 0 and world == 1 and not args.no_rows:
        rows = {"ksp_bddc": measure_ksp_bddc(torch), "simp2d": measure_simp2d()}

    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            for P_ in problems.values():
                P_.close()
            problems.clear()
            torch.cuda.empty_cache()
            iters, t_count, converged = reference_iterations()
            costs = reference_costs(apply_reps=1)
            t_step, t_apply, n = reference_model(costs, iters)
            cpu = {"value": 1.0 / t_step, "unit": UNIT, "cores": 1, "kind": "port",
                   "sample": reference_sample_text(costs, t_apply, iters, n, t_count, converged,
                                                   "one fine-grid apply")}
        line = {"metric": METRIC, "value": head["value"], "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": head["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64 CG, f32 V-cycle",
                "data": "synthetic",
                "config": {"workload": f"SIMP cantilever {NELX}x{NELY}x{NELZ}", "nel": nel, "ndof": ndof,
                           "solver": f"mixed: FP64 PCG, FP32 multigrid preconditioner ({args.levels} levels, V(2,2) "
                                     "Chebyshev smoothing on [kappa/16, kappa], direct coarse solve)",
                           "tol": TOL, "parallelism": f"replicas x{world}",
                           "l2": f"inputs larger than L2 ({8 * ndof / 1e6:.0f} MB per FP64 vector)",
                           "sensitivity_guard": "rounding-negative element energies clamped at 0"},
                "speedup_vs_fp64": head["value"] / others["fp64"]["value"] if "fp64" in others else None,
                "arms": {"mixed": head, **others},
                "chosen_form_error": err, "apply_microbench": micro, "batched_load_cases": batched, "next_rows": rows,
                "e2e": e2e, "gpu_launches": head["launches"], "roofline": roofline, "cpu_baseline": cpu,
                "clocks": clocks}
        print(json.dumps(line))
    for P_ in problems.values():
        P_.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def profile_traffic(name):
    """DRAM bytes per launch recorded in a profiles/ summary ('traffic_bytes_per_launch:')."""
    path = os.path.join(ROOT, "profiles", name)
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1])
    except OSError:
        pass
    return None


def main():
    global NELX, NELY, NELZ
    faulthandler.enable()
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-micro", action="store_true", help="skip the 128x64x64 K.u microbenchmark")
    ap.add_argument("--no-rows", action="store_true",
                    help="skip the KSP-BDDC and 2D-worker measurements of the main line")
    ap.add_argument("--no-batched", action="store_true",
                    help="skip the batched load-case measurement (8 right-hand sides, 160x80x80) of the main line")
    ap.add_argument("--arms", default="",
                    help="comma list of solver arms timed besides the headline 'mixed' (default: all)")
    ap.add_argument("--batched", action="store_true",
                    help="the batched load-case configuration (8 right-hand sides, 160x80x80): block vs sequential")
    ap.add_argument("--levels", type=int, default=6,
                    help="multigrid levels of the chosen form (7 for 512x256x256)")
    ap.add_argument("--rows", choices=["all", "ksp_bddc", "simp2d"], default=None,
                    help="only the KSP-BDDC and/or 2D-worker measurements (measure_ksp_bddc, measure_simp2d), one JSON line")
    ap.add_argument("--kernels", action="store_true",
                    help="time only the fine-grid apply kernels (FP32, TF32 tcgen05, FP64) at --grid")
    ap.add_argument("--grid", default=f"{NELX}x{NELY}x{NELZ}",
                    help="elements per axis, e.g. 128x64x64 for a profiling case (default: the benchmark grid)")
    args = ap.parse_args()
    NELX, NELY, NELZ = (int(v) for v in args.grid.lower().split("x"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.kernels:
        return run_kernels(args)
    if args.rows:
        import torch
        torch.cuda.set_device(local_rank)
        out = {}
        if args.rows in ("all", "ksp_bddc"):
            out["ksp_bddc"] = measure_ksp_bddc(torch)
        if args.rows in ("all", "simp2d"):
            out["simp2d"] = measure_simp2d()
        print(json.dumps(out))
        return 0
    if args.batched:
        return run_batched(args)
    return run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    sys.exit(main())
