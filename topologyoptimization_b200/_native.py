"""ctypes binding of libtpo.so (include/tpo.h).

The library is built in-tree (``python -m topologyoptimization_b200.build``).  Loading
fails loudly when it is missing: there is no CPU fallback for any entry point.
"""
import ctypes as C
import os
import re

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtpo.so")
HEADER = os.path.join(os.path.dirname(HERE), "include", "tpo.h")

TPO_OK = 0
TPO_NOT_CONVERGED = 1
TPO_NONFINITE = 2
TPO_OOM = 3
TPO_BAD_ARG = 4
TPO_CUDA_ERROR = 5
TPO_NO_DEVICE = 6
TPO_TIMEOUT = 7

PREC_JACOBI, PREC_MG, PREC_BDDC = 0, 1, 2
FP64, MIXED, F32_PRECOND = 0, 1, 2


class TpoError(RuntimeError):
    def __init__(self, status, where, message):
        self.status = status
        super().__init__(f"{where}: {status_string(status)} ({status}): {message}")


class Grid(C.Structure):
    _fields_ = [("nelx", C.c_int32), ("nely", C.c_int32), ("nelz", C.c_int32)]


class MgOpts(C.Structure):
    _fields_ = [("max_levels", C.c_int32), ("galerkin_max_ndof", C.c_int32), ("nu1", C.c_int32),
                ("nu2", C.c_int32), ("omega", C.c_double), ("coarse_iters", C.c_int32),
                ("coarse_direct", C.c_int32), ("safe_omega", C.c_int32), ("chebyshev", C.c_int32),
                ("cheb_ratio", C.c_double)]


class SolveOpts(C.Structure):
    _fields_ = [("precond", C.c_int), ("precision", C.c_int), ("max_iter", C.c_int32),
                ("tol", C.c_double), ("warm_start", C.c_int32), ("ref_epsilon", C.c_int32),
                ("inner_tol", C.c_double), ("tensor_cores", C.c_int32), ("bddc_smoother_iters", C.c_int32)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int32), ("outer_iterations", C.c_int32), ("converged", C.c_int32),
                ("rel_residual", C.c_double), ("compliance", C.c_double)]


class SimpOpts(C.Structure):
    _fields_ = [("volfrac", C.c_double), ("penal", C.c_double), ("rmin", C.c_double),
                ("E0", C.c_double), ("Emin", C.c_double), ("beta", C.c_double),
                ("use_projection", C.c_int32), ("guard_sensitivities", C.c_int32), ("solve", SolveOpts)]


class DesignOpts(C.Structure):
    _fields_ = [("penal", C.c_double), ("E0", C.c_double), ("Emin", C.c_double), ("filter_radius", C.c_double)]


class SimpOpts2D(C.Structure):
    _fields_ = [("volfrac", C.c_double), ("penal", C.c_double), ("rmin", C.c_double), ("E0", C.c_double),
                ("Emin", C.c_double), ("beta", C.c_double), ("use_projection", C.c_int32), ("cg_tol", C.c_double),
                ("cg_max_iter", C.c_int32)]


class SimpInfo2D(C.Structure):
    _fields_ = [("compliance", C.c_double), ("change", C.c_double), ("cg_iterations", C.c_int32)]


class SimpInfo(C.Structure):
    _fields_ = [("compliance", C.c_double), ("change", C.c_double), ("cg_iterations", C.c_int32),
                ("converged", C.c_int32), ("rel_residual", C.c_double)]


_lib = None

_P = C.c_void_p
_SIGS = {
    "tpo_status_string": (C.c_char_p, [C.c_int]),
    "tpo_last_error": (C.c_char_p, []),
    "tpo_device_available": (C.c_int, []),
    "tpo_launch_count": (C.c_int64, []),
    "tpo_lk": (C.c_int, [C.c_double, _P]),
    "tpo_apply_a_ebe3d": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int32, _P, _P, C.c_int32]),
    "tpo_dense_matvec": (C.c_int, [_P, _P, _P, C.c_int32]),
    "tpo_element_energies": (C.c_int, [_P, _P, _P, C.c_int32, C.c_int32, C.c_int32, _P]),
    "tpo_ebe_pcg": (C.c_int, [_P, _P, _P, _P, _P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32,
                              C.c_double, C.c_double, C.c_double, C.c_int32, C.c_double, _P]),
    "tpo_default_mg_opts": (None, [_P]),
    "tpo_default_solve_opts": (None, [_P]),
    "tpo_create": (C.c_int, [_P, _P, C.c_double, _P, _P, _P]),
    "tpo_destroy": (C.c_int, [_P]),
    "tpo_sizes": (C.c_int, [_P, _P, _P, _P]),
    "tpo_level_info": (C.c_int, [_P, C.c_int32, _P]),
    "tpo_level_dense": (C.c_int, [_P, C.c_int32, _P]),
    "tpo_set_densities": (C.c_int, [_P, _P, C.c_double, C.c_double, C.c_double]),
    "tpo_set_densities_dev": (C.c_int, [_P, _P, C.c_double, C.c_double, C.c_double]),
    "tpo_set_load": (C.c_int, [_P, _P]),
    "tpo_set_load_dev": (C.c_int, [_P, _P]),
    "tpo_apply": (C.c_int, [_P, _P, _P]),
    "tpo_apply_dev": (C.c_int, [_P, _P, _P]),
    "tpo_apply_f32_dev": (C.c_int, [_P, _P, _P]),
    "tpo_apply_tf32_dev": (C.c_int, [_P, _P, _P]),
    "tpo_apply_3xtf32_dev": (C.c_int, [_P, _P, _P]),
    "tpo_apply_bf16_dev": (C.c_int, [_P, _P, _P]),
    "tpo_vcycle": (C.c_int, [_P, _P, _P]),
    "tpo_solve": (C.c_int, [_P, _P, _P, _P]),
    "tpo_solve_dev": (C.c_int, [_P, _P, _P, _P]),
    "tpo_element_energy_dev": (C.c_int, [_P, _P, _P]),
    "tpo_heaviside_dev": (C.c_int, [_P, _P, C.c_double, _P]),
    "tpo_sensitivity_dev": (C.c_int, [_P, _P, _P, _P, C.c_double, C.c_double, C.c_double, C.c_int32, _P]),
    "tpo_filter_sens_dev": (C.c_int, [_P, C.c_double, _P, _P, _P]),
    "tpo_density_filter_dev": (C.c_int, [_P, C.c_double, _P, _P]),
    "tpo_density_filter_transpose_dev": (C.c_int, [_P, C.c_double, _P, _P]),
    "tpo_oc_dev": (C.c_int, [_P, _P, C.c_double, _P, _P, _P, _P, _P, _P]),
    "tpo_oc_update_dev": (C.c_int, [_P, _P, _P, _P, _P, C.c_double, C.c_double, C.c_int32, _P, _P, _P, _P]),
    "tpo_simp_step_dev": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "tpo_simp_step": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "tpo_get_u": (C.c_int, [_P, _P]),
    "tpo_volumetric_snapshot": (C.c_int, [_P, _P, _P]),
    "tpo_stream": (C.c_void_p, [_P]),
    "tpo_set_stream": (C.c_int, [_P, _P]),
    "tpo_solve_multi_dev": (C.c_int, [_P, _P, C.c_int32, _P, _P, _P]),
    "tpo_set_spring": (C.c_int, [_P, C.c_int64, C.c_double]),
    "tpo_forward_dev": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "tpo_backward_dev": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "tpo_forward": (C.c_int, [_P, _P, _P, _P, _P, _P, _P]),
    "tpo_backward": (C.c_int, [_P, _P, _P, _P, _P]),
    "tpo_mgpcg": (C.c_int, [_P, _P, _P, C.c_int32, C.c_double, _P]),
    "tpo_ksp_bddc": (C.c_int, [_P, _P, _P, C.c_int32, C.c_double, C.c_int32, _P]),
    "tpo_lk2d": (C.c_int, [C.c_double, _P]),
    "tpo_create2d": (C.c_int, [C.c_int32, C.c_int32, _P, C.c_double, _P, _P]),
    "tpo_destroy2d": (C.c_int, [_P]),
    "tpo_set_load2d": (C.c_int, [_P, _P]),
    "tpo_simp2d_step_dev": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "tpo_get_u2d": (C.c_int, [_P, _P]),
    "tpo_apply_static_dev": (C.c_int, [C.c_int32, C.c_int32, C.c_int32, _P, _P, C.c_double, C.c_double,
                                       C.c_double, _P, _P, _P]),
}


def header_functions():
    """Names of every function declared in include/tpo.h."""
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tpo_[a-z0-9_]+)\s*\(", src)))


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"libtpo.so is not built ({LIB_PATH}); run python -m topologyoptimization_b200.build")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def status_string(s):
    try:
        return lib().tpo_status_string(int(s)).decode()
    except Exception:  # noqa: BLE001 - used while formatting another error
        return "status"


def check(status, where, allow=(TPO_OK,)):
    if status not in allow:
        msg = lib().tpo_last_error().decode()
        raise TpoError(status, where, msg)
    return status


def device_available():
    return bool(lib().tpo_device_available())


def default_mg_opts(**kw):
    o = MgOpts()
    lib().tpo_default_mg_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_solve_opts(**kw):
    o = SolveOpts()
    lib().tpo_default_solve_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def ptr(a):
    """Raw address of a numpy array or torch tensor (host or device)."""
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        return C.c_void_p(a.data_ptr())
    return a.ctypes.data_as(C.c_void_p)
