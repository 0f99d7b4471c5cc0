"""TopologyOptimizerWorker.optimize of the 2D worker (js/optimizer-worker.js:347-800) on the
B200, restricted to the SIMP hot path (no AMR, manufacturing constraints, genetic optimiser
or UI mesh).

The host keeps the loop control: penal continuation, the Heaviside beta schedule, the CG
tolerance max(CG_TOLERANCE, change * CG_TOLERANCE_COARSE) (:621) and the stop test.  Each
iteration is one tpo_simp2d_step_dev call (projection, FE solve, energies, sensitivities,
2D sensitivity filter, OC, change) with the design and every per-element array resident
on the device.

Config keys read (same meaning as the reference): volumeFraction, maxIterations,
penaltyFactor, filterRadius, youngsModulus, poissonsRatio, penalStart, continuationIters,
useProjection, betaMax, betaInterval, constraintPosition, constraintDOFs, forceDirection,
forceMagnitude, forceVector.  Extensions: F (explicit load vector), preservedElements /
voidElements (element masks in the 2D element order).
"""
import ctypes as C
import math
import time

import numpy as np

from . import _native as N
from . import mesh

CG_TOLERANCE = 1e-8
CG_TOLERANCE_COARSE = 1e-2
MAX_CG_ITERATIONS = 2000


def lk2d(nu=0.3):
    """8x8 quad element matrix (lk(), :1732-1767), row-major, computed by libtpo."""
    Ke = np.empty(64)
    N.check(N.lib().tpo_lk2d(float(nu), N.ptr(Ke)), "tpo_lk2d")
    return Ke


class Problem2D:
    """Device-resident 2D grid (tpo_create2d ... tpo_destroy2d)."""

    def __init__(self, nelx, nely, fixed_mask, Ke=None, nu=0.3):
        self.nelx, self.nely = int(nelx), int(nely)
        self.nel = self.nelx * self.nely
        self.ndof = mesh.ndof2d(self.nelx, self.nely)
        fm = np.ascontiguousarray(fixed_mask, dtype=np.uint8)
        if fm.size != self.ndof:
            raise ValueError(f"fixed_mask has {fm.size} entries, expected {self.ndof}")
        self.fixed_mask = fm
        ke = None if Ke is None else np.ascontiguousarray(Ke, dtype=np.float64)
        h = C.c_void_p()
        N.check(N.lib().tpo_create2d(self.nelx, self.nely, N.ptr(ke), float(nu), N.ptr(fm), C.byref(h)),
                "tpo_create2d")
        self.h = h

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            N.lib().tpo_destroy2d(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001 - interpreter shutdown
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_load(self, F):
        Fa = np.ascontiguousarray(F, dtype=np.float64)
        N.check(N.lib().tpo_set_load2d(self.h, N.ptr(Fa)), "tpo_set_load2d")

    def simp_step_dev(self, d_x, opts, d_preserved=None, d_void=None):
        info = N.SimpInfo2D()
        N.check(N.lib().tpo_simp2d_step_dev(self.h, C.byref(opts), N.ptr(d_x), N.ptr(d_preserved), N.ptr(d_void),
                                            C.byref(info)), "tpo_simp2d_step_dev")
        return info

    def get_u(self):
        U = np.empty(self.ndof)
        N.check(N.lib().tpo_get_u2d(self.h, N.ptr(U)), "tpo_get_u2d")
        return U


class TopologyOptimizerWorker:
    def __init__(self):
        self.rmin = 1.5
        self.penal = 3.0
        self.E0 = 1.0
        self.Emin = 1e-9
        self.nu = 0.3
        self.cancelled = False

    def cancel(self):
        self.cancelled = True

    def optimize(self, model, config, on_message=None):
        import torch

        post = on_message or (lambda m: None)
        nelx, nely = int(model["nx"]), int(model["ny"])
        nel = nelx * nely
        volfrac = float(config["volumeFraction"])
        max_iterations = int(config["maxIterations"])
        self.penal = float(config.get("penaltyFactor", self.penal))
        self.rmin = float(config.get("filterRadius", self.rmin))
        if config.get("youngsModulus"):
            self.E0 = float(config["youngsModulus"])
        if config.get("poissonsRatio") is not None:
            self.nu = float(config["poissonsRatio"])
        self.cancelled = False
        position = config.get("constraintPosition", "left")
        direction = config.get("forceDirection", "down")
        fixed = mesh.fixed_mask2d(nelx, nely, position, config.get("constraintDOFs", "all"))
        if config.get("F") is not None:
            F = np.asarray(config["F"], dtype=np.float32)
        else:
            F = mesh.load_vector2d(nelx, nely, direction, float(config.get("forceMagnitude", 1.0)),
                                   config.get("forceVector"))
        preserved = np.zeros(nel, np.uint8)
        if config.get("preservedElements") is not None:
            preserved[np.asarray(config["preservedElements"], dtype=bool)] = 1
        else:  # the elements under the constraint and force positions (:519-529)
            preserved[mesh.constraint_elements2d(nelx, nely, position)] = 1
            preserved[mesh.force_elements2d(nelx, nely, direction)] = 1
        void = np.zeros(nel, np.uint8)
        if config.get("voidElements") is not None:
            void[np.asarray(config["voidElements"], dtype=bool)] = 1
        x = np.full(nel, volfrac, np.float32)
        x[preserved == 1] = 1.0
        x[void == 1] = 0.0

        penal_target = self.penal
        penal_start = config.get("penalStart")
        penal_start = min(penal_target, 1.5) if penal_start is None else float(penal_start)
        cont = config.get("continuationIters")
        cont = max(20, max_iterations // 3) if cont is None else int(cont)
        use_proj = config.get("useProjection", True) is not False
        beta_max = float(config.get("betaMax", 64))
        beta_interval = int(config.get("betaInterval", 5))

        with Problem2D(nelx, nely, fixed, nu=self.nu) as P:
            P.set_load(F.astype(np.float64))
            dev = torch.device("cuda")
            d_x = torch.from_numpy(x).to(dev)
            d_pres = torch.from_numpy(preserved).to(dev) if preserved.any() else None
            d_void = torch.from_numpy(void).to(dev) if void.any() else None
            loop, change, c = 0, 1.0, 0.0
            hist, times, cg_hist = [], [], []
            t_start = time.perf_counter()
            while change > 0.01 and loop < max_iterations:
                if self.cancelled:
                    post({"type": "cancelled", "iteration": loop})
                    return None
                loop += 1
                t0 = time.perf_counter()
                tol = max(CG_TOLERANCE, change * CG_TOLERANCE_COARSE)
                cur_penal = penal_start + (penal_target - penal_start) * min(1.0, (loop - 1) / cont)
                beta = min(beta_max, 2.0 ** math.floor((loop - 1) / beta_interval)) if use_proj else 1.0
                opts = N.SimpOpts2D(volfrac=volfrac, penal=cur_penal, rmin=self.rmin, E0=self.E0, Emin=self.Emin,
                                    beta=beta, use_projection=int(use_proj), cg_tol=tol,
                                    cg_max_iter=MAX_CG_ITERATIONS)
                info = P.simp_step_dev(d_x, opts, d_pres, d_void)
                c, change = info.compliance, info.change
                dt = (time.perf_counter() - t0) * 1e3
                hist.append(c)
                times.append(dt)
                cg_hist.append(info.cg_iterations)
                post({"type": "progress", "iteration": loop, "compliance": c, "penal": cur_penal, "beta": beta,
                      "timing": {"iterationTime": dt, "avgIterationTime": sum(times) / len(times),
                                 "elapsedTime": (time.perf_counter() - t_start) * 1e3}})
            x_final = d_x.cpu().numpy()
        # densities3D of the completion message (:740-749): the 2D field in x-fastest order
        d3 = x_final.reshape(nelx, nely).T.ravel().copy()
        result = {"densities": d3, "densities2D": x_final, "finalCompliance": c, "iterations": loop,
                  "volumeFraction": volfrac, "nx": nelx, "ny": nely, "nz": 1,
                  "complianceHistory": np.array(hist), "cgIterations": np.array(cg_hist),
                  "timing": {"totalTime": (time.perf_counter() - t_start) * 1e3,
                             "avgIterationTime": sum(times) / max(1, len(times)), "iterationTimes": times}}
        post({"type": "complete", "result": result})
        return result
