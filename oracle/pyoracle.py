"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` / ``--impl reference`` legs of bench.py, and nowhere else.  The
product library (libtpo.so) never loads this module or the oracle library.
"""
import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")

POSITIONS = {"left": 0, "right": 1, "bottom": 2, "top": 3, "bottom-corners": 4}


def build(force=False):
    src = os.path.join(_HERE, "tpo_oracle.c")
    if force or not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(src):
        subprocess.check_call(["make", "-s", "-C", _HERE])
    return _LIB


class MgOpts(C.Structure):
    _fields_ = [("max_levels", C.c_int), ("galerkin_max_ndof", C.c_int), ("nu1", C.c_int),
                ("nu2", C.c_int), ("omega", C.c_double), ("coarse_iters", C.c_int),
                ("coarse_direct", C.c_int), ("coarse_moduli", C.c_int), ("safe_omega", C.c_int)]


class SimpCfg2D(C.Structure):
    _fields_ = [("nelx", C.c_int), ("nely", C.c_int), ("volfrac", C.c_double), ("penal", C.c_double),
                ("rmin", C.c_double), ("E0", C.c_double), ("Emin", C.c_double), ("nu", C.c_double),
                ("max_iter", C.c_int), ("penal_start", C.c_double), ("continuation_iters", C.c_int),
                ("use_projection", C.c_int), ("beta_max", C.c_double), ("beta_interval", C.c_int)]


class SimpCfg(C.Structure):
    _fields_ = [("nelx", C.c_int), ("nely", C.c_int), ("nelz", C.c_int),
                ("volfrac", C.c_double), ("penal", C.c_double), ("rmin", C.c_double),
                ("E0", C.c_double), ("Emin", C.c_double), ("nu", C.c_double),
                ("max_iter", C.c_int), ("penal_start", C.c_double),
                ("continuation_iters", C.c_int), ("use_projection", C.c_int),
                ("beta_max", C.c_double), ("beta_interval", C.c_int), ("solver", C.c_int),
                ("cg_max_iter", C.c_int), ("cg_tol", C.c_double), ("stop_on_change", C.c_int)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        build()
        _lib = C.CDLL(_LIB)
        _lib.orc_mg_create.restype = C.c_void_p
        _lib.orc_mg_create.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        for fn in ("orc_mg_destroy", "orc_mg_num_levels"):
            getattr(_lib, fn).argtypes = [C.c_void_p]
        _lib.orc_mg_level_info.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        _lib.orc_mg_level_arrays.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_mg_update.argtypes = [C.c_void_p, C.c_void_p, C.c_double, C.c_double, C.c_double]
        _lib.orc_mg_apply_level.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        _lib.orc_mg_vcycle.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_mg_set_spring.argtypes = [C.c_void_p, C.c_longlong, C.c_double]
        _lib.orc_mg_set_spring.restype = None
        _lib.orc_mgpcg.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double]
        _lib.orc_fe_pcg.argtypes = [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_double]
        _lib.orc_lk.argtypes = [C.c_double, C.c_void_p]
        _lib.orc_ebe_pcg.argtypes = [C.c_void_p] * 6 + [C.c_int] * 4 + [C.c_double] * 3 + [C.c_int, C.c_double]
        _lib.orc_oc.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_oc_move.argtypes = [C.c_int, C.c_void_p, C.c_double, C.c_void_p, C.c_void_p, C.c_void_p,
                                     C.c_double, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib.orc_heaviside.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p]
        _lib.orc_sensitivity.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double,
                                         C.c_double, C.c_double, C.c_int, C.c_void_p]
        _lib.orc_filter_hs.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p]
        _lib.orc_filter_sens.argtypes = [C.c_int, C.c_int, C.c_int, C.c_double, C.c_void_p, C.c_void_p,
                                         C.c_void_p, C.c_void_p]
        _lib.orc_density_filter.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double]
        _lib.orc_simp.argtypes = [C.c_void_p] * 10
        _lib.orc_lk2d.argtypes = [C.c_double, C.c_void_p]
        _lib.orc_edofs2d.argtypes = [C.c_int, C.c_int, C.c_void_p]
        _lib.orc_simp2d.argtypes = [C.c_void_p] * 9
        _lib.orc_bddc_partition.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p]
        _lib.orc_ksp_bddc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_double,
                                      C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_double, C.c_int]
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def lk(nu=0.3):
    Ke = np.zeros(576)
    lib().orc_lk(C.c_double(nu), _p(Ke))
    return Ke


def edofs3d(nelx, nely, nelz):
    e = np.zeros(nelx * nely * nelz * 24, np.int32)
    lib().orc_edofs3d(nelx, nely, nelz, _p(e))
    return e


def ndof_of(nelx, nely, nelz):
    return 3 * (nelx + 1) * (nely + 1) * (nelz + 1)


def fixed_mask(nelx, nely, nelz, position="left", dofs=7):
    m = np.zeros(ndof_of(nelx, nely, nelz), np.uint8)
    lib().orc_fixed_dofs(nelx, nely, nelz, POSITIONS[position], dofs, _p(m))
    return m


def constraint_elements(nelx, nely, nelz, position):
    m = np.zeros(nelx * nely * nelz, np.uint8)
    lib().orc_constraint_elements(nelx, nely, nelz, POSITIONS[position], _p(m))
    return m


def apply_a(Ke, edofs, evals, active, p, edof_size=24):
    Ke = np.ascontiguousarray(Ke, np.float64)
    edofs = np.ascontiguousarray(edofs, np.int32)
    evals = np.ascontiguousarray(evals, np.float64)
    active = np.ascontiguousarray(active, np.int32)
    p = np.ascontiguousarray(p, np.float64)
    Ap = np.zeros_like(p)
    lib().orc_apply_a(_p(Ke), _p(edofs), edof_size, _p(evals), _p(active), len(active), _p(p), _p(Ap), len(p))
    return Ap


def dense_matvec(K, p):
    K = np.ascontiguousarray(K, np.float64)
    p = np.ascontiguousarray(p, np.float64)
    out = np.zeros_like(p)
    lib().orc_dense_matvec(_p(K), _p(p), _p(out), len(p))
    return out


def ebe_pcg(dens, Ke, edofs, F, U, freedofs, ndof, Emin, E0, penal, max_iter, tol, edof_size=24):
    dens = np.ascontiguousarray(dens, np.float64)
    F = np.ascontiguousarray(F, np.float64)
    U = np.array(U, np.float64, copy=True)
    freedofs = np.ascontiguousarray(freedofs, np.int32)
    it = lib().orc_ebe_pcg(_p(dens), _p(np.ascontiguousarray(Ke, np.float64)), _p(np.ascontiguousarray(edofs, np.int32)),
                           _p(F), _p(U), _p(freedofs), len(dens), edof_size, ndof, len(freedofs),
                           Emin, E0, penal, max_iter, tol)
    return U, it


def mg_opts(**kw):
    o = MgOpts()
    lib().orc_mg_default_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class MG:
    """Multigrid hierarchy of the reference's MGPrecond3D."""

    def __init__(self, nelx, nely, nelz, Ke, fixed, **opts):
        self.o = mg_opts(**opts)
        self._Ke = np.ascontiguousarray(Ke, np.float64)
        self._fixed = np.ascontiguousarray(fixed, np.uint8)
        self.h = lib().orc_mg_create(nelx, nely, nelz, _p(self._Ke), _p(self._fixed), C.byref(self.o))
        self.ndof = ndof_of(nelx, nely, nelz)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_mg_destroy(self.h)
            self.h = None

    @property
    def num_levels(self):
        return lib().orc_mg_num_levels(self.h)

    def level_info(self, li):
        d = np.zeros(8, np.int32)
        lib().orc_mg_level_info(self.h, li, _p(d))
        return dict(zip(["nelx", "nely", "nelz", "ndof", "nfree", "active", "dense", "nel"], d.tolist()))

    def level_arrays(self, li):
        info = self.level_info(li)
        ev = np.zeros(info["nel"])
        inv = np.zeros(info["ndof"])
        K = np.zeros((info["ndof"], info["ndof"])) if info["dense"] else None
        lib().orc_mg_level_arrays(self.h, li, _p(ev), _p(inv), _p(K))
        return ev, inv, K

    def set_spring(self, dof, k):
        """Grounded spring k at one fine-level DOF (dof = -1 removes it); takes effect in
        the apply at once and in the diagonal at the next update()."""
        lib().orc_mg_set_spring(self.h, int(dof), float(k))

    def update(self, x, penal, E0=1.0, Emin=1e-9):
        x = np.ascontiguousarray(x, np.float32)
        lib().orc_mg_update(self.h, _p(x), penal, E0, Emin)

    def apply(self, p, level=0):
        p = np.ascontiguousarray(p, np.float64)
        out = np.zeros_like(p)
        lib().orc_mg_apply_level(self.h, level, _p(p), _p(out))
        return out

    def vcycle(self, b, x=None):
        b = np.ascontiguousarray(b, np.float64)
        x = np.zeros_like(b) if x is None else np.array(x, np.float64, copy=True)
        lib().orc_mg_vcycle(self.h, _p(b), _p(x))
        return x

    def mgpcg(self, F, max_iter, tol):
        F = np.ascontiguousarray(F, np.float64)
        U = np.zeros_like(F)
        it = lib().orc_mgpcg(self.h, _p(F), _p(U), max_iter, tol)
        return U, it

    def fe_pcg(self, F, U0, max_iter, tol, precond="mg"):
        F = np.ascontiguousarray(F, np.float64)
        U = np.array(U0, np.float64, copy=True)
        it = lib().orc_fe_pcg(self.h, 1 if precond == "mg" else 0, _p(F), _p(U), max_iter, tol)
        return U, it


def bddc_partition(nelx, nely, nelz):
    ns = np.zeros(3, np.int32)
    lib().orc_bddc_partition(nelx, nely, nelz, _p(ns))
    return tuple(int(v) for v in ns)


def ksp_bddc(nelx, nely, nelz, Ke, x, penal, fixed, F, max_iter, tol, smoother_iters=3, E0=1.0, Emin=1e-9):
    """ebeKSP_BDDC as the worker calls it; returns (U, iterations)."""
    U = np.zeros(ndof_of(nelx, nely, nelz))
    it = lib().orc_ksp_bddc(nelx, nely, nelz, _p(np.ascontiguousarray(Ke, np.float64)),
                            _p(np.ascontiguousarray(x, np.float32)), penal, E0, Emin,
                            _p(np.ascontiguousarray(fixed, np.uint8)), _p(np.ascontiguousarray(F, np.float64)),
                            _p(U), max_iter, tol, smoother_iters)
    return U, it


def element_energy(Ke, nelx, nely, nelz, U):
    out = np.zeros(nelx * nely * nelz, np.float32)
    lib().orc_element_energy(_p(np.ascontiguousarray(Ke, np.float64)), nelx, nely, nelz,
                             _p(np.ascontiguousarray(U, np.float64)), _p(out))
    return out


def element_energies_f32(U, KE, edofs, nel, es):
    out = np.zeros(nel, np.float32)
    lib().orc_element_energies_f32(_p(np.ascontiguousarray(U, np.float32)), _p(np.ascontiguousarray(KE, np.float32)),
                                   _p(np.ascontiguousarray(edofs, np.int32)), int(nel), int(es), _p(out))
    return out


def stress(xphys, energy, penal, E0=1.0, Emin=1e-9):
    out = np.zeros(len(xphys), np.float32)
    m = C.c_double()
    lib().orc_stress(_p(np.ascontiguousarray(xphys, np.float32)), _p(np.ascontiguousarray(energy, np.float32)),
                     len(out), C.c_double(penal), C.c_double(E0), C.c_double(Emin), _p(out), C.byref(m))
    return out, m.value


def heaviside(x, beta):
    x = np.ascontiguousarray(x, np.float32)
    out = np.zeros_like(x)
    lib().orc_heaviside(_p(x), len(x), beta, _p(out))
    return out


def sensitivity(x, xphys, energy, penal, E0, beta, use_projection):
    x = np.ascontiguousarray(x, np.float32)
    xphys = np.ascontiguousarray(xphys, np.float32)
    energy = np.ascontiguousarray(energy, np.float32)
    dc = np.zeros_like(x)
    lib().orc_sensitivity(_p(x), _p(xphys), _p(energy), len(x), penal, E0, beta, int(use_projection), _p(dc))
    return dc


def filter_hs(nelx, nely, nelz, rmin):
    hs = np.zeros(nelx * nely * nelz, np.float32)
    lib().orc_filter_hs(nelx, nely, nelz, rmin, _p(hs))
    return hs


def filter_sens(nelx, nely, nelz, rmin, hs, x, dc):
    out = np.zeros(nelx * nely * nelz, np.float32)
    lib().orc_filter_sens(nelx, nely, nelz, rmin, _p(np.ascontiguousarray(hs, np.float32)),
                          _p(np.ascontiguousarray(x, np.float32)), _p(np.ascontiguousarray(dc, np.float32)), _p(out))
    return out


def density_filter(dens, nx, ny, nz, radius):
    dens = np.ascontiguousarray(dens, np.float64)
    out = np.zeros_like(dens)
    lib().orc_density_filter(_p(dens), _p(out), nx, ny, nz, radius)
    return out


def oc(x, volfrac, dc, preserved=None, void=None, move=0.2):
    x = np.ascontiguousarray(x, np.float32)
    dc = np.ascontiguousarray(dc, np.float32)
    xnew = np.zeros_like(x)
    lm = C.c_double(0)
    nb = C.c_int(0)
    lib().orc_oc_move(len(x), _p(x), volfrac, _p(dc), _p(preserved), _p(void), float(move), _p(xnew), C.byref(lm),
                      C.byref(nb))
    return xnew, lm.value, nb.value


def simp(nelx, nely, nelz, F, fixed, preserved=None, void=None, mg=None, **cfg):
    c = SimpCfg(nelx=nelx, nely=nely, nelz=nelz, volfrac=0.3, penal=3.0, rmin=1.5, E0=1.0,
                Emin=1e-9, nu=0.3, max_iter=50, penal_start=-1.0, continuation_iters=-1,
                use_projection=1, beta_max=64.0, beta_interval=5, solver=1, cg_max_iter=400,
                cg_tol=-1.0, stop_on_change=1)
    for k, v in cfg.items():
        setattr(c, k, v)
    n = c.max_iter
    ch, chg = np.zeros(n), np.zeros(n)
    cg = np.zeros(n, np.int32)
    x = np.zeros(nelx * nely * nelz, np.float32)
    o = mg if mg is not None else mg_opts()
    loops = lib().orc_simp(C.byref(c), _p(np.ascontiguousarray(F, np.float32)),
                           _p(np.ascontiguousarray(fixed, np.uint8)), _p(preserved), _p(void),
                           C.byref(o), _p(ch), _p(chg), _p(cg), _p(x))
    return dict(iterations=loops, compliance=ch[:loops], change=chg[:loops], cg=cg[:loops], x=x)


def lk2d(nu=0.3):
    Ke = np.zeros(64)
    lib().orc_lk2d(C.c_double(nu), _p(Ke))
    return Ke


def simp2d(nelx, nely, F, fixed, preserved=None, void=None, **cfg):
    """The 2D worker's loop (orc_simp2d); defaults are the worker's."""
    c = SimpCfg2D(nelx=nelx, nely=nely, volfrac=0.3, penal=3.0, rmin=1.5, E0=1.0, Emin=1e-9, nu=0.3, max_iter=50,
                  penal_start=-1.0, continuation_iters=-1, use_projection=1, beta_max=64.0, beta_interval=5)
    for k, v in cfg.items():
        setattr(c, k, v)
    n = c.max_iter
    ch, chg = np.zeros(n), np.zeros(n)
    cg = np.zeros(n, np.int32)
    x = np.zeros(nelx * nely, np.float32)
    loops = lib().orc_simp2d(C.byref(c), _p(np.ascontiguousarray(F, np.float32)),
                             _p(np.ascontiguousarray(fixed, np.uint8)), _p(preserved), _p(void), _p(ch), _p(chg),
                             _p(cg), _p(x))
    return dict(iterations=loops, compliance=ch[:loops], change=chg[:loops], cg=cg[:loops], x=x)
