"""Writes ke_pattern.h: the sign/magnitude-class pattern of the hex8 element matrix.

    python topologyoptimization_b200/csrc/gen_ke_pattern.py

For the isotropic unit-cube hex8 of lk() (2x2x2 Gauss, local node order
(0,0,0),(1,0,0),(1,1,0),(0,1,0),(0,0,1),(1,0,1),(1,1,1),(0,1,1)), every entry is
+-v[c] for one of a few classes c: entries that are equal or opposite as functions of
the Poisson ratio share a class (the sign of v[c] itself may change with the ratio).  The classes are the common refinement over several
Poisson ratios, so no accidental equality at one ratio merges two classes.  The
structured kernels keep the class values in registers and take (class, sign) of each
entry from this table at compile time.
"""
import os

import numpy as np


def lk(nu):
    f = 1.0 / ((1 + nu) * (1 - 2 * nu))
    C = np.zeros((6, 6))
    C[:3, :3] = f * nu
    np.fill_diagonal(C[:3, :3], f * (1 - nu))
    C[3:, 3:] = np.eye(3) * f * (1 - 2 * nu) / 2
    corners = np.array([[-1, -1, -1], [1, -1, -1], [1, 1, -1], [-1, 1, -1],
                        [-1, -1, 1], [1, -1, 1], [1, 1, 1], [-1, 1, 1]], float)
    K = np.zeros((24, 24))
    g = 1 / np.sqrt(3)
    for xi in (-g, g):
        for eta in (-g, g):
            for zeta in (-g, g):
                q = np.array([xi, eta, zeta])
                dN = np.zeros((8, 3))
                for a, c in enumerate(corners):
                    for k in range(3):
                        t = c[k]
                        for m in range(3):
                            if m != k:
                                t *= 1 + c[m] * q[m]
                        dN[a, k] = t * 0.125
                B = np.zeros((6, 24))
                B[0, 0::3], B[1, 1::3], B[2, 2::3] = dN[:, 0], dN[:, 1], dN[:, 2]
                B[3, 0::3], B[3, 1::3] = dN[:, 1], dN[:, 0]
                B[4, 1::3], B[4, 2::3] = dN[:, 2], dN[:, 1]
                B[5, 0::3], B[5, 2::3] = dN[:, 2], dN[:, 0]
                K += B.T @ C @ B
    return K


def main():
    nus = [0.3, 0.25, 0.41, 0.17]
    W = np.stack([lk(nu) for nu in nus], axis=-1)  # 24 x 24 x R: each entry as a function of nu
    classes = {}
    cls = np.zeros((24, 24), int)
    sign = np.zeros((24, 24), int)
    for i in range(24):
        for j in range(24):
            w = np.round(W[i, j], 10)
            nz = np.flatnonzero(w)
            s_ = 1 if len(nz) == 0 or w[nz[0]] > 0 else -1
            k = tuple(w * s_)
            if k not in classes:
                classes[k] = len(classes)
            cls[i, j] = classes[k]
            sign[i, j] = s_
    n = len(classes)
    rep = [None] * n
    for i in range(24):
        for j in range(24):
            if rep[cls[i, j]] is None:
                rep[cls[i, j]] = i * 24 + j
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ke_pattern.h")
    with open(out, "w") as f:
        f.write("// Generated by gen_ke_pattern.py: sign and magnitude class of every entry of the\n")
        f.write("// hex8 element matrix of lk(); entry (i, j) = kKeSign[i*24+j] * v[kKeClass[i*24+j]].\n")
        f.write("#pragma once\n\nnamespace tpo {\n\n")
        f.write(f"constexpr int kKeClasses = {n};\n")
        f.write("// row-major index of one entry of each class: v[c] = kKeSign[rep] * Ke[rep]\n")
        f.write("constexpr int kKeClassRep[kKeClasses] = {" + ", ".join(map(str, rep)) + "};\n")
        for name, tab in (("kKeClass", cls), ("kKeSign", sign)):
            f.write(f"constexpr signed char {name}[576] = {{\n")
            for i in range(24):
                f.write("    " + ", ".join(str(c) for c in tab[i]) + ",\n")
            f.write("};\n")
        # device-side accessors: constexpr functions with local tables, folded by the
        # compiler when the index is a compile-time constant (fully unrolled loops)
        for fn, tab in (("ke_class", cls), ("ke_sign", sign)):
            f.write(f"__host__ __device__ constexpr int {fn}(int i) {{\n")
            f.write("    constexpr signed char t[576] = {\n")
            for i in range(24):
                f.write("        " + ", ".join(str(c) for c in tab[i]) + ",\n")
            f.write("    };\n    return t[i];\n}\n")
        f.write("\n}  // namespace tpo\n")
    print(f"{n} classes -> {out}")


if __name__ == "__main__":
    main()
