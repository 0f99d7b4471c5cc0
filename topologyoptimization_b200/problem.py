"""Device-resident problem handle over libtpo (tpo_create / tpo_* in include/tpo.h).

torch is used only to hold device buffers; every computation runs in libtpo's CUDA
kernels on the handle's stream.
"""
import ctypes as C

import numpy as np

from . import _native as N


def _torch():
    import torch
    return torch


class Problem:
    """One structured hex8 grid with its multigrid hierarchy on the current device."""

    def __init__(self, nelx, nely, nelz, fixed_mask, Ke=None, nu=0.3, mg=None):
        self.nelx, self.nely, self.nelz = int(nelx), int(nely), int(nelz)
        self.nel = self.nelx * self.nely * self.nelz
        self.ndof = 3 * (self.nelx + 1) * (self.nely + 1) * (self.nelz + 1)
        fm = np.ascontiguousarray(fixed_mask, dtype=np.uint8)
        if fm.size != self.ndof:
            raise ValueError(f"fixed_mask has {fm.size} entries, expected {self.ndof}")
        self.fixed_mask = fm
        g = N.Grid(self.nelx, self.nely, self.nelz)
        self.mg_opts = mg if mg is not None else N.default_mg_opts()
        h = C.c_void_p()
        ke = None if Ke is None else np.ascontiguousarray(Ke, dtype=np.float64)
        N.check(N.lib().tpo_create(C.byref(g), N.ptr(ke), float(nu), N.ptr(fm), C.byref(self.mg_opts), C.byref(h)),
                "tpo_create")
        self.h = h
        nl = C.c_int32()
        N.check(N.lib().tpo_sizes(self.h, None, None, C.byref(nl)), "tpo_sizes")
        self.levels = nl.value

    # ---- lifetime -------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            N.lib().tpo_destroy(self.h)
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

    @property
    def stream(self):
        return N.lib().tpo_stream(self.h)

    def set_stream(self, stream):
        """Run on a caller-owned stream (a torch.cuda.Stream or a raw cudaStream_t);
        None returns to the library's own stream."""
        raw = None if stream is None else getattr(stream, "cuda_stream", stream)
        N.check(N.lib().tpo_set_stream(self.h, C.c_void_p(raw) if raw else None), "tpo_set_stream")

    # ---- operators ------------------------------------------------------------------
    def set_densities(self, x, penal, E0=1.0, Emin=1e-9):
        if hasattr(x, "is_cuda") and x.is_cuda:
            x = x.contiguous().float()
            N.check(N.lib().tpo_set_densities_dev(self.h, N.ptr(x), penal, E0, Emin), "tpo_set_densities_dev")
        else:
            xa = np.ascontiguousarray(x, dtype=np.float32)
            N.check(N.lib().tpo_set_densities(self.h, N.ptr(xa), penal, E0, Emin), "tpo_set_densities")

    def set_load(self, F):
        if hasattr(F, "is_cuda") and F.is_cuda:
            F = F.contiguous().double()
            N.check(N.lib().tpo_set_load_dev(self.h, N.ptr(F)), "tpo_set_load_dev")
        else:
            Fa = np.ascontiguousarray(F, dtype=np.float64)
            N.check(N.lib().tpo_set_load(self.h, N.ptr(Fa)), "tpo_set_load")

    def apply(self, u):
        ua = np.ascontiguousarray(u, dtype=np.float64)
        out = np.empty_like(ua)
        N.check(N.lib().tpo_apply(self.h, N.ptr(ua), N.ptr(out)), "tpo_apply")
        return out

    def apply_dev(self, d_u, d_out):
        N.check(N.lib().tpo_apply_dev(self.h, N.ptr(d_u), N.ptr(d_out)), "tpo_apply_dev")

    def apply_f32_dev(self, d_u, d_out):
        N.check(N.lib().tpo_apply_f32_dev(self.h, N.ptr(d_u), N.ptr(d_out)), "tpo_apply_f32_dev")

    def apply_tf32_dev(self, d_u, d_out):
        N.check(N.lib().tpo_apply_tf32_dev(self.h, N.ptr(d_u), N.ptr(d_out)), "tpo_apply_tf32_dev")

    def apply_3xtf32_dev(self, d_u, d_out):
        N.check(N.lib().tpo_apply_3xtf32_dev(self.h, N.ptr(d_u), N.ptr(d_out)), "tpo_apply_3xtf32_dev")

    def apply_bf16_dev(self, d_u, d_out):
        N.check(N.lib().tpo_apply_bf16_dev(self.h, N.ptr(d_u), N.ptr(d_out)), "tpo_apply_bf16_dev")

    def vcycle(self, b):
        ba = np.ascontiguousarray(b, dtype=np.float64)
        out = np.empty_like(ba)
        N.check(N.lib().tpo_vcycle(self.h, N.ptr(ba), N.ptr(out)), "tpo_vcycle")
        return out

    def solve(self, U0=None, opts=None, **kw):
        o = opts if opts is not None else N.default_solve_opts(**kw)
        U = np.zeros(self.ndof) if U0 is None else np.array(U0, dtype=np.float64, copy=True)
        info = N.SolveInfo()
        st = N.lib().tpo_solve(self.h, C.byref(o), N.ptr(U), C.byref(info))
        N.check(st, "tpo_solve", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
        return U, info

    def solve_dev(self, d_U, opts=None, **kw):
        o = opts if opts is not None else N.default_solve_opts(**kw)
        info = N.SolveInfo()
        st = N.lib().tpo_solve_dev(self.h, C.byref(o), N.ptr(d_U), C.byref(info))
        N.check(st, "tpo_solve_dev", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
        return info

    def solve_multi_dev(self, d_F, d_U, opts=None, **kw):
        """Batched solve of nrhs load cases: d_F, d_U are (nrhs, ndof) FP64 device arrays.
        Returns one SolveInfo per right-hand side."""
        o = opts if opts is not None else N.default_solve_opts(**kw)
        nrhs = int(d_F.shape[0])
        infos = (N.SolveInfo * nrhs)()
        st = N.lib().tpo_solve_multi_dev(self.h, C.byref(o), nrhs, N.ptr(d_F), N.ptr(d_U), infos)
        N.check(st, "tpo_solve_multi_dev", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
        return list(infos)

    def level_info(self, li):
        d = np.zeros(5, np.int32)
        N.check(N.lib().tpo_level_info(self.h, int(li), N.ptr(d)), "tpo_level_info")
        return dict(zip(["nelx", "nely", "nelz", "ndof", "dense"], d.tolist()))

    def level_dense(self, li):
        """The dense operator of level li (a Galerkin level), ndof x ndof, on the host."""
        n = self.level_info(li)["ndof"]
        K = np.empty((n, n))
        N.check(N.lib().tpo_level_dense(self.h, int(li), N.ptr(K)), "tpo_level_dense")
        return K

    def volumetric_snapshot(self):
        """(stress float32[nel], max_stress) of the last SIMP step."""
        stress = np.empty(self.nel, np.float32)
        m = C.c_double()
        N.check(N.lib().tpo_volumetric_snapshot(self.h, N.ptr(stress), C.byref(m)), "tpo_volumetric_snapshot")
        return stress, m.value

    def get_u(self):
        U = np.empty(self.ndof)
        N.check(N.lib().tpo_get_u(self.h, N.ptr(U)), "tpo_get_u")
        return U

    # ---- differentiable forward / backward -------------------------------------------
    def set_spring(self, dof, k):
        """Grounded spring k at fine-level DOF `dof` (-1 removes it)."""
        N.check(N.lib().tpo_set_spring(self.h, int(dof), float(k)), "tpo_set_spring")

    def forward_dev(self, d_x, design, opts=None, d_l=None, **kw):
        """xPhys = filter(x), K(xPhys) u = F; returns (J, info) with J = l.u (F.u if d_l is
        None).  d_x: FP64 device design, reference element order."""
        o = opts if opts is not None else N.default_solve_opts(**kw)
        J = C.c_double()
        info = N.SolveInfo()
        st = N.lib().tpo_forward_dev(self.h, C.byref(design), C.byref(o), N.ptr(d_x), N.ptr(d_l), C.byref(J),
                                     C.byref(info))
        N.check(st, "tpo_forward_dev", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
        return J.value, info

    def backward_dev(self, d_grad, opts=None, d_l=None, d_grad_phys=None, **kw):
        """dJ/dx of the last forward_dev into d_grad (FP64 device, nel); returns the adjoint
        solve's info (trivial for the compliance)."""
        o = opts if opts is not None else N.default_solve_opts(**kw)
        info = N.SolveInfo()
        st = N.lib().tpo_backward_dev(self.h, C.byref(o), N.ptr(d_l), N.ptr(d_grad), N.ptr(d_grad_phys),
                                      C.byref(info))
        N.check(st, "tpo_backward_dev", allow=(N.TPO_OK, N.TPO_NOT_CONVERGED))
        return info

    # ---- SIMP pieces (device tensors, reference element order) ----------------------
    def element_energy_dev(self, d_U, d_energy):
        N.check(N.lib().tpo_element_energy_dev(self.h, N.ptr(d_U), N.ptr(d_energy)), "tpo_element_energy_dev")

    def heaviside_dev(self, d_x, beta, d_out):
        N.check(N.lib().tpo_heaviside_dev(self.h, N.ptr(d_x), beta, N.ptr(d_out)), "tpo_heaviside_dev")

    def sensitivity_dev(self, d_x, d_xphys, d_energy, penal, E0, beta, use_projection, d_dc):
        N.check(N.lib().tpo_sensitivity_dev(self.h, N.ptr(d_x), N.ptr(d_xphys), N.ptr(d_energy), penal, E0, beta,
                                            int(use_projection), N.ptr(d_dc)), "tpo_sensitivity_dev")

    def filter_sens_dev(self, rmin, d_x, d_dc, d_dcn):
        N.check(N.lib().tpo_filter_sens_dev(self.h, rmin, N.ptr(d_x), N.ptr(d_dc), N.ptr(d_dcn)),
                "tpo_filter_sens_dev")

    def density_filter_dev(self, radius, d_x, d_out):
        N.check(N.lib().tpo_density_filter_dev(self.h, radius, N.ptr(d_x), N.ptr(d_out)), "tpo_density_filter_dev")

    def density_filter_T_dev(self, radius, d_g, d_out):
        N.check(N.lib().tpo_density_filter_transpose_dev(self.h, radius, N.ptr(d_g), N.ptr(d_out)),
                "tpo_density_filter_transpose_dev")

    def oc_dev(self, d_x, volfrac, d_dc, d_xnew, d_preserved=None, d_void=None):
        lm = C.c_double()
        nb = C.c_int32()
        N.check(N.lib().tpo_oc_dev(self.h, N.ptr(d_x), volfrac, N.ptr(d_dc), N.ptr(d_preserved), N.ptr(d_void),
                                   N.ptr(d_xnew), C.byref(lm), C.byref(nb)), "tpo_oc_dev")
        return lm.value, nb.value

    def oc_update_dev(self, d_x, d_dc, d_xnew, volfrac, move=0.2, max_bisections=1280, d_preserved=None,
                      d_void=None):
        """OC with move limit and bisection cap; returns (change, lmid, bisections)."""
        ch, lm = C.c_double(), C.c_double()
        nb = C.c_int32()
        N.check(N.lib().tpo_oc_update_dev(self.h, N.ptr(d_x), N.ptr(d_dc), N.ptr(d_preserved), N.ptr(d_void),
                                          float(volfrac), float(move), int(max_bisections), N.ptr(d_xnew),
                                          C.byref(ch), C.byref(lm), C.byref(nb)), "tpo_oc_update_dev")
        return ch.value, lm.value, nb.value

    def simp_step(self, x, opts, preserved=None, void=None):
        """tpo_simp_step: one SIMP iteration on host arrays; x (float32, nel, contiguous) is
        updated in place."""
        info = N.SimpInfo()
        N.check(N.lib().tpo_simp_step(self.h, C.byref(opts), N.ptr(x), N.ptr(preserved), N.ptr(void), C.byref(info)),
                "tpo_simp_step")
        return info

    def simp_step_dev(self, d_x, opts, d_preserved=None, d_void=None):
        info = N.SimpInfo()
        N.check(N.lib().tpo_simp_step_dev(self.h, C.byref(opts), N.ptr(d_x), N.ptr(d_preserved), N.ptr(d_void),
                                          C.byref(info)), "tpo_simp_step_dev")
        return info


def lk(nu=0.3):
    """24x24 hex8 element matrix (row-major, 576 doubles) computed by libtpo."""
    Ke = np.empty(576)
    N.check(N.lib().tpo_lk(float(nu), N.ptr(Ke)), "tpo_lk")
    return Ke
