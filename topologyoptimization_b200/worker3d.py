"""TopologyOptimizerWorker3D.optimize on the B200 (js/optimizer-worker-3d.js:1605-2352).

The host keeps only the loop control of the reference's SIMP loop (:2074-2301): penal
continuation, Heaviside beta schedule, the CG tolerance schedule and the stop test.
Each iteration is one tpo_simp_step_dev call (projection, FE solve, element energy,
sensitivity, sensitivity filter, OC bisection, change) with x, U and every
per-element array resident on the device.

Config keys read (same meaning as the reference): volumeFraction, maxIterations,
penaltyFactor, filterRadius, youngsModulus, poissonsRatio, penalStart,
continuationIters, useProjection, betaMax, betaInterval, constraintPosition,
constraintDOFs, forceDirection, forceMagnitude, forceVector, linearSolver
('mgpcg' | 'cg' | 'petsc': the KSP solve with the reference's BDDC preconditioner,
_solveWithWasmKSP_BDDC :3814-3970, cold start), petscPC ('bddc').  Extensions: F (explicit load vector), cgTolerance (fixed CG
tolerance instead of the 1e-3 -> 1e-8 schedule), cgMaxIterations (default 400),
preservedElements / voidElements (element masks), volumetricOutputMode ('on-stop' |
'every-iteration' | 'off', the stress snapshot of :1579-1593), mg (tpo_mg_opts), precision
('fp64' | 'mixed': FP32 MG-PCG with FP64 reliable updates), tensorCores (TF32 fine-level
applies in the mixed solve), guardSensitivities (clamp rounding-negative element
energies at 0; the reference lets them through and OC then produces NaN densities).
"""
import math
import time

import numpy as np

from . import _native as N
from . import mesh
from .problem import Problem

CG_TOL_START = 1e-3
CG_TOL_END = 1e-8
MAX_CG_ITERATIONS = 400


def cg_tolerance(iteration, max_iterations):
    """Tolerance schedule of FE (:4189-4193)."""
    progress = (iteration - 1) / (max_iterations - 1) if max_iterations > 1 else 1.0
    return math.exp(math.log(CG_TOL_START) + progress * (math.log(CG_TOL_END) - math.log(CG_TOL_START)))


class TopologyOptimizerWorker3D:
    def __init__(self):
        self.rmin = 1.5
        self.penal = 3.0
        self.E0 = 1.0
        self.Emin = 1e-9
        self.nu = 0.3
        self.linearSolver = "mgpcg"
        self.cancelled = False
        self._problem = None

    def cancel(self):
        self.cancelled = True

    def optimize(self, model, config, on_message=None):
        import torch

        post = on_message or (lambda m: None)
        nelx, nely, nelz = int(model["nx"]), int(model["ny"]), int(model["nz"])
        nel = nelx * nely * nelz
        volfrac = float(config["volumeFraction"])
        max_iterations = int(config["maxIterations"])
        self.penal = float(config.get("penaltyFactor", self.penal))
        self.rmin = float(config.get("filterRadius", self.rmin))
        if config.get("youngsModulus"):
            self.E0 = float(config["youngsModulus"])
        if config.get("poissonsRatio") is not None:
            self.nu = float(config["poissonsRatio"])
        if config.get("linearSolver"):
            self.linearSolver = config["linearSolver"]
        self.cancelled = False

        fixed = mesh.fixed_mask(nelx, nely, nelz, config.get("constraintPosition", "left"),
                                config.get("constraintDOFs", "all"))
        if config.get("F") is not None:
            F = np.asarray(config["F"], dtype=np.float32)
        else:
            F = mesh.load_vector(nelx, nely, nelz, config.get("forceDirection", "down"),
                                 float(config.get("forceMagnitude", 1.0)), config.get("forceVector"))
        preserved = np.zeros(nel, np.uint8)
        if config.get("preservedElements") is not None:
            preserved[np.asarray(config["preservedElements"], dtype=bool)] = 1
        else:
            preserved[mesh.constraint_elements(nelx, nely, nelz, config.get("constraintPosition", "left"))] = 1
            if config.get("F") is None and config.get("forceVector") is None:
                preserved[mesh.force_elements(nelx, nely, nelz, config.get("forceDirection", "down"))] = 1
        void = np.zeros(nel, np.uint8)
        if config.get("voidElements") is not None:
            void[np.asarray(config["voidElements"], dtype=bool)] = 1

        x = np.full(nel, volfrac, np.float32)
        x[preserved == 1] = 1.0
        x[void == 1] = 0.0

        mg = config.get("mg")
        if self._problem is None or (self._problem.nelx, self._problem.nely, self._problem.nelz) != (nelx, nely, nelz) \
                or not np.array_equal(self._problem.fixed_mask, fixed):
            if self._problem is not None:
                self._problem.close()
            self._problem = Problem(nelx, nely, nelz, fixed, nu=self.nu, mg=mg)
        P = self._problem
        P.set_load(F.astype(np.float64))
        dev = torch.device("cuda")
        d_x = torch.from_numpy(x).to(dev)
        d_pres = torch.from_numpy(preserved).to(dev) if preserved.any() else None
        d_void = torch.from_numpy(void).to(dev) if void.any() else None

        penal_target = self.penal
        penal_start = config.get("penalStart")
        penal_start = min(penal_target, 1.5) if penal_start is None else float(penal_start)
        cont = config.get("continuationIters")
        cont = max(20, max_iterations // 3) if cont is None else int(cont)
        use_proj = config.get("useProjection", True) is not False
        beta_max = float(config.get("betaMax", 64))
        beta_interval = int(config.get("betaInterval", 5))
        cg_cap = int(config.get("cgMaxIterations", MAX_CG_ITERATIONS))
        fixed_tol = config.get("cgTolerance")
        mgpcg = self.linearSolver == "mgpcg"
        bddc = self.linearSolver == "petsc" and config.get("petscPC", "bddc") == "bddc"
        mixed = config.get("precision", "fp64") == "mixed"
        if mixed and not mgpcg:
            raise ValueError("precision='mixed' runs the multigrid-preconditioned solve (linearSolver='mgpcg')")
        guard = int(bool(config.get("guardSensitivities", False)))
        vmode = config.get("volumetricOutputMode")
        vmode = vmode if vmode in ("every-iteration", "off") else "on-stop"
        tensor_cores = int(bool(config.get("tensorCores", False)))
        nfree = int((fixed == 0).sum())

        loop, change, c = 0, 1.0, 0.0
        hist, times, cg_hist = [], [], []
        t_start = time.perf_counter()
        while change > 0.01 and loop < max_iterations:
            if self.cancelled:
                post({"type": "cancelled", "iteration": loop})
                return None
            loop += 1
            t0 = time.perf_counter()
            cur_penal = penal_start + (penal_target - penal_start) * min(1.0, (loop - 1) / cont)
            beta = min(beta_max, 2.0 ** math.floor((loop - 1) / beta_interval)) if use_proj else 1.0
            tol = float(fixed_tol) if fixed_tol is not None else cg_tolerance(loop, max_iterations)
            prec = N.PREC_MG if mgpcg else (N.PREC_BDDC if bddc else N.PREC_JACOBI)
            so = N.default_solve_opts(precond=prec, max_iter=min(nfree, cg_cap),
                                      tol=tol, warm_start=0 if (mgpcg or bddc or loop == 1) else 1,
                                      ref_epsilon=0 if mixed else 1, precision=N.MIXED if mixed else N.FP64,
                                      tensor_cores=tensor_cores)
            opts = N.SimpOpts(volfrac=volfrac, penal=cur_penal, rmin=self.rmin, E0=self.E0, Emin=self.Emin,
                              beta=beta, use_projection=int(use_proj), guard_sensitivities=guard, solve=so)
            info = P.simp_step_dev(d_x, opts, d_pres, d_void)
            c, change = info.compliance, info.change
            dt = (time.perf_counter() - t0) * 1e3
            hist.append(c)
            times.append(dt)
            cg_hist.append(info.cg_iterations)
            vol = self._volumetric(P, nelx, nely, nelz, loop) if vmode == "every-iteration" else None
            post({"type": "progress", "iteration": loop, "compliance": c, "penal": cur_penal, "beta": beta,
                  "timing": {"iterationTime": dt, "avgIterationTime": sum(times) / len(times),
                             "elapsedTime": (time.perf_counter() - t_start) * 1e3},
                  "cgIterations": info.cg_iterations, "volumetricData": vol})
        result = {"densities": d_x.cpu().numpy(), "finalCompliance": c, "iterations": loop,
                  "volumetricData": self._volumetric(P, nelx, nely, nelz, loop) if vmode != "off" and loop else None,
                  "volumeFraction": volfrac, "nx": nelx, "ny": nely, "nz": nelz,
                  "complianceHistory": np.array(hist), "cgIterations": np.array(cg_hist),
                  "timing": {"totalTime": (time.perf_counter() - t_start) * 1e3,
                             "avgIterationTime": sum(times) / max(1, len(times)), "iterationTimes": times}}
        post({"type": "complete", "result": result})
        return result

    @staticmethod
    def _volumetric(P, nx, ny, nz, iteration):
        """_buildVolumetricSnapshot (:1579-1593): the last step's element stress field."""
        stress, mx = P.volumetric_snapshot()
        return {"nx": nx, "ny": ny, "nz": nz, "iteration": iteration, "maxStress": mx, "stress": stress}

    def close(self):
        if self._problem is not None:
            self._problem.close()
            self._problem = None
