"""Writes the fixtures in tests/golden/ from the CPU oracle (oracle/tpo_oracle.c).

    python tests/golden/make_golden.py

The reference (JavaScript + WebAssembly) cannot be executed in this environment, so
the fixtures are the oracle's outputs on seeded inputs.  They freeze the oracle (a
change to it shows up as a fixture diff) and travel with the tests to machines where
the oracle is not rebuilt.  Every fixture records the inputs that produced it.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import pyoracle as O  # noqa: E402


def main():
    Ke = O.lk(0.3)
    np.savez_compressed(os.path.join(HERE, "ke_nu0.3.npz"), Ke=Ke)

    # MGPCG on a 4x4x4 graded block (tests/test-wasm-mgpcg.js scenario 4), tol 1e-6
    dims = (4, 4, 4)
    nel = 64
    x = (0.3 + 0.7 * np.arange(nel) / nel).astype(np.float32)
    fixed = O.fixed_mask(*dims, "bottom-corners")
    F = np.zeros(O.ndof_of(*dims))
    n = (dims[0] // 2) * 25 + (dims[1] // 2) * 5 + dims[2]
    F[3 * n + 1] = -1.0
    mg = O.MG(*dims, Ke, fixed)
    mg.update(x, 3.0)
    U, it = mg.mgpcg(F, 500, 1e-6)
    np.savez_compressed(os.path.join(HERE, "mgpcg_4x4x4_graded.npz"), x=x, F=F, fixed=fixed, U=U, iters=it,
                        tol=1e-6, max_iter=500)

    # apply on 5x3x4 with seeded densities (seed 7) and u ~ N(0,1) (seed 8)
    dims = (5, 3, 4)
    rng = np.random.default_rng(7)
    xa = rng.uniform(1e-3, 1, 60).astype(np.float32)
    E = 1e-9 + xa.astype(np.float64) ** 3 * (1 - 1e-9)
    act = np.flatnonzero(E > 1e-6).astype(np.int32)
    u = np.random.default_rng(8).standard_normal(O.ndof_of(*dims))
    Ku = O.apply_a(Ke, O.edofs3d(*dims), E, act, u)
    np.savez_compressed(os.path.join(HERE, "apply_5x3x4.npz"), x=xa, u=u, Ku=Ku, penal=3.0)

    # 8 SIMP iterations on 12x4x4, cantilever, MGPCG at fixed tol 1e-8, no projection
    dims = (12, 4, 4)
    fixed = O.fixed_mask(*dims, "left")
    F = np.zeros(O.ndof_of(*dims), np.float32)
    for j in range(dims[1] + 1):
        nn = dims[0] * 25 + j * 5
        F[3 * nn + 2] = -1.0
    pres = O.constraint_elements(*dims, "left")
    r = O.simp(*dims, F, fixed, preserved=pres, max_iter=8, solver=1, penal_start=3.0, use_projection=0,
               cg_tol=1e-8, cg_max_iter=400, stop_on_change=1)
    np.savez_compressed(os.path.join(HERE, "simp_12x4x4.npz"), compliance=r["compliance"], change=r["change"],
                        cg=r["cg"], x=r["x"], F=F, fixed=fixed, preserved=pres)

    # The plain SIMP cantilever: 30x10x10, E0 = 1, Emin = 1e-9, nu = 0.3, penal 3 from the
    # start, no projection, volfrac 0.3, sensitivity filter rmin 1.5, x0 = 0.3, 50 OC
    # iterations (move 0.2); x = 0 face fixed, -1 in z on each node of the line
    # (x = 30, y = 0..10, z = 0); Jacobi-PCG (ebePCG, warm start) at the fixed tolerance
    # 1e-8 with a cap of 2000 iterations; the left-face elements preserved.  About a
    # minute of oracle time.
    dims = (30, 10, 10)
    fixed = O.fixed_mask(*dims, "left")
    F = np.zeros(O.ndof_of(*dims), np.float32)
    for j in range(dims[1] + 1):
        nn = dims[0] * (dims[1] + 1) * (dims[2] + 1) + j * (dims[2] + 1)
        F[3 * nn + 2] = -1.0
    pres = O.constraint_elements(*dims, "left")
    r = O.simp(*dims, F, fixed, preserved=pres, max_iter=50, solver=0, penal_start=3.0, use_projection=0,
               cg_tol=1e-8, cg_max_iter=2000, stop_on_change=1, volfrac=0.3, rmin=1.5)
    np.savez_compressed(os.path.join(HERE, "simp_30x10x10_jacobi.npz"), compliance=r["compliance"],
                        change=r["change"], cg=r["cg"], x=r["x"], F=F, fixed=fixed, preserved=pres)

    # The worker's defaults on 16x8x8: tolerance schedule 1e-3 -> 1e-8 over the run,
    # Heaviside projection (beta doubling every 5 iterations), penal continuation from
    # 1.5 to 3 over max(20, maxIter/3) iterations, ebeMGPCG with the reference hierarchy
    # (cap 400), 20 iterations.
    dims = (16, 8, 8)
    fixed = O.fixed_mask(*dims, "left")
    F = np.zeros(O.ndof_of(*dims), np.float32)
    for j in range(dims[1] + 1):
        nn = dims[0] * (dims[1] + 1) * (dims[2] + 1) + j * (dims[2] + 1)
        F[3 * nn + 2] = -1.0
    pres = O.constraint_elements(*dims, "left")
    r = O.simp(*dims, F, fixed, preserved=pres, max_iter=20, solver=1, penal_start=-1.0, continuation_iters=-1,
               use_projection=1, beta_max=64.0, beta_interval=5, cg_tol=-1.0, cg_max_iter=400, stop_on_change=1,
               volfrac=0.3, rmin=1.5)
    np.savez_compressed(os.path.join(HERE, "simp_16x8x8_defaults.npz"), compliance=r["compliance"],
                        change=r["change"], cg=r["cg"], x=r["x"], F=F, fixed=fixed, preserved=pres)
    # The 2D worker (js/optimizer-worker.js): 60x20 and 40x40 cantilevers, x = 0 edge fixed,
    # unit downward load at the bottom-right node ('down'), the constraint and force elements
    # preserved, penal 3 from the start, no projection, the worker's CG tolerance schedule
    # max(1e-8, change * 1e-2) with the absolute test, 40 iterations or the change stop.
    from topologyoptimization_b200 import mesh
    for nx, ny in ((60, 20), (40, 40)):
        fixed = mesh.fixed_mask2d(nx, ny, "left")
        F = mesh.load_vector2d(nx, ny, "down")
        pres = np.zeros(nx * ny, np.uint8)
        pres[mesh.constraint_elements2d(nx, ny, "left")] = 1
        pres[mesh.force_elements2d(nx, ny, "down")] = 1
        r = O.simp2d(nx, ny, F, fixed, pres, None, max_iter=40, use_projection=0, penal_start=3.0)
        np.savez_compressed(os.path.join(HERE, f"simp2d_{nx}x{ny}.npz"), compliance=r["compliance"],
                            change=r["change"], cg=r["cg"], x=r["x"], F=F, fixed=fixed, preserved=pres)
    print("fixtures written to", HERE)


if __name__ == "__main__":
    main()
