"""tpo_apply_static_dev: the structured apply that allocates no device memory.

Some callers cannot allocate while they run (a host whose memory pool already holds the
device's free memory, or a loop that cannot afford the device-wide synchronisation of
cudaMalloc/cudaFree); this entry point serves them from a fixed scratch array compiled
into the library.  The GPU test calls it through the C ABI twice in a row, with
different densities and vectors, and compares each result with the problem-handle path
(tpo_set_densities_dev + tpo_apply_dev) on the same inputs.  The file is named so that
pytest collects it last: it also runs after every other test has used the device in the
same process.
"""
import numpy as np
import pytest

from conftest import rel_inf

# (dims, fraction of elements pushed below the 1000 Emin activity threshold)
CASES = [((5, 3, 7), 0.0), ((16, 8, 8), 0.3), ((7, 3, 131), 0.1), ((40, 24, 20), 0.2)]


def _inputs(dims, void_frac, seed):
    from topologyoptimization_b200 import mesh
    rng = np.random.default_rng(seed)
    nel = int(np.prod(dims))
    x = rng.uniform(0.05, 1.0, nel).astype(np.float32)
    x[rng.random(nel) < void_frac] = 1e-3  # E = 1e-9 + 1e-9 (1 - 1e-9) < 1e-6: inactive
    u = rng.standard_normal(mesh.ndof(*dims))
    return x, u


def _static_apply(N, dims, Ke, d_x, d_u, d_out, penal=3.0, E0=1.0, Emin=1e-9):
    return N.lib().tpo_apply_static_dev(int(dims[0]), int(dims[1]), int(dims[2]), N.ptr(Ke), N.ptr(d_x), penal, E0,
                                        Emin, N.ptr(d_u), N.ptr(d_out), None)


@pytest.mark.gpu
@pytest.mark.parametrize("dims,void_frac", CASES)
def test_static_apply_matches_problem_apply(native, dims, void_frac):
    import torch
    from topologyoptimization_b200 import Problem, lk, mesh
    N = native
    Ke = np.ascontiguousarray(lk(0.3))
    fixed = mesh.fixed_mask(*dims, "left")
    got, want = [], []
    with Problem(*dims, fixed) as P:
        for call in range(2):
            x, u = _inputs(dims, void_frac, seed=10 + call)
            d_x = torch.from_numpy(x).cuda()
            d_u = torch.from_numpy(u).cuda()
            d_ref = torch.empty_like(d_u)
            P.set_densities(d_x, 3.0)
            P.apply_dev(d_u, d_ref)
            torch.cuda.synchronize()
            d_out = torch.full_like(d_u, float("nan"))
            st = _static_apply(N, dims, Ke, d_x, d_u, d_out)
            assert st == N.TPO_OK, N.lib().tpo_last_error().decode()
            torch.cuda.synchronize()
            got.append(d_out.cpu().numpy())
            want.append(d_ref.cpu().numpy())
    for g, w in zip(got, want):
        assert np.all(np.isfinite(g))
        assert rel_inf(g, w) < 1e-12
    assert rel_inf(got[0], got[1]) > 1e-3  # the second call did not reuse the first one's moduli


def test_static_apply_rejects_oversize_grid():
    """Argument checks run before any device work: a grid beyond the static scratch is
    refused with TPO_BAD_ARG.  Runs only where no device is visible, so that the dummy
    pointers below can never reach a kernel."""
    from topologyoptimization_b200 import _native as N
    L = N.lib()
    if N.device_available():
        pytest.skip("checked on a host without a device")
    Ke = np.zeros(576)
    dummy = np.zeros(4)
    limit = 1048576
    st = L.tpo_apply_static_dev(1024, 1024, 2, N.ptr(Ke), N.ptr(dummy), 3.0, 1.0, 1e-9, N.ptr(dummy), N.ptr(dummy),
                                None)
    assert st == N.TPO_BAD_ARG
    assert "static scratch" in L.tpo_last_error().decode()
    # a grid just under the limit passes the size check and stops at the device check
    st = L.tpo_apply_static_dev(1024, 1023, 1, N.ptr(Ke), N.ptr(dummy), 3.0, 1.0, 1e-9, N.ptr(dummy), N.ptr(dummy),
                                None)
    assert 1024 * 1023 < limit and st == N.TPO_NO_DEVICE
    st = L.tpo_apply_static_dev(0, 4, 4, N.ptr(Ke), N.ptr(dummy), 3.0, 1.0, 1e-9, N.ptr(dummy), N.ptr(dummy), None)
    assert st == N.TPO_BAD_ARG
    st = L.tpo_apply_static_dev(4, 4, 4, N.ptr(Ke), None, 3.0, 1.0, 1e-9, N.ptr(dummy), N.ptr(dummy), None)
    assert st == N.TPO_BAD_ARG
