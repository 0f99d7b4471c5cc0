"""libtpo.so loads, exports every entry point include/tpo.h declares, and fails
cleanly (status codes, no crash) where no device is present.  No compute calls."""
import ctypes as C

import numpy as np
import pytest

from topologyoptimization_b200 import _native as N


def test_library_exports_every_header_symbol():
    lib = N.lib()
    names = N.header_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(N._SIGS) == set(names), set(N._SIGS) ^ set(names)


def test_status_strings():
    for s in range(8):
        assert N.status_string(s)
    assert N.status_string(N.TPO_OK) == "ok"


def test_defaults_match_reference_constants():
    mg = N.default_mg_opts()
    # js/optimizer-worker-3d.js:58-64
    assert (mg.max_levels, mg.galerkin_max_ndof, mg.nu1, mg.nu2, mg.omega, mg.coarse_iters) == (6, 3000, 2, 2, 0.5, 30)
    so = N.default_solve_opts()
    assert so.max_iter == 400 and so.tol == 1e-8 and so.ref_epsilon == 1


def test_no_device_paths_fail_cleanly():
    if N.device_available():
        pytest.skip("a device is present; this test covers the no-device path")
    g = N.Grid(2, 2, 2)
    fixed = np.zeros(81, np.uint8)
    h = C.c_void_p()
    st = N.lib().tpo_create(C.byref(g), None, 0.3, N.ptr(fixed), None, C.byref(h))
    assert st == N.TPO_NO_DEVICE
    assert b"device" in N.lib().tpo_last_error()
    Ke = np.zeros(576)
    assert N.lib().tpo_lk(0.3, N.ptr(Ke)) == N.TPO_NO_DEVICE
    from topologyoptimization_b200 import GPUFEASolver
    s = GPUFEASolver()
    assert s.init() is False and s.isAvailable() is False
    with pytest.raises(RuntimeError, match="GPUFEASolver: GPU not available"):
        s.setup({})
    with pytest.raises(RuntimeError, match="not initialized. Call init\\(\\) and setup\\(\\) first."):
        s.solve({})


def test_null_arguments_are_rejected():
    assert N.lib().tpo_lk(0.3, None) == N.TPO_BAD_ARG
    assert N.lib().tpo_destroy(None) == N.TPO_OK
    assert N.lib().tpo_sizes(None, None, None, None) == N.TPO_BAD_ARG
