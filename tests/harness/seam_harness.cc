// Test harness: the Node addon's GPUFEASolver call sequence (tpo_seam.h) driven from C++
// on libtpo, with no Node runtime.  Reads one setup from a binary file, then
//   setup(params) -> solve(cold) -> setup(params with densities2) -> solve(warm start =
//   the first solution)
// and writes both results.  Input layout (little endian):
//   int64 nel, ndof; int32 solver_mg, maxIterations; double E0, Emin, penal, tolerance;
//   float KEflat[576]; int32 edofs[nel*24]; float dens[nel]; float dens2[nel];
//   float F[ndof]; uint8 fixed[ndof]
// Output: for each solve, int32 status, iterations, converged; float U[ndof]; double U64[ndof];
// then, for the structured numbering, two SIMP steps from densities2 (seam_simp_step): per
// step int32 status, cg iterations, double compliance, change; then float x[nel].
#include <cstdio>
#include <vector>

#include "tpo_seam.h"

template <typename T>
static bool rd(FILE *f, T *p, size_t n) {
    return std::fread(p, sizeof(T), n, f) == n;
}

int main(int argc, char **argv) {
    if (argc != 3) {
        std::fprintf(stderr, "usage: seam_harness input.bin output.bin\n");
        return 2;
    }
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int64_t nel = 0, ndof = 0;
    int32_t mg = 0, maxit = 0;
    double E0, Emin, penal, tol;
    bool ok = rd(f, &nel, 1) && rd(f, &ndof, 1) && rd(f, &mg, 1) && rd(f, &maxit, 1) && rd(f, &E0, 1) &&
              rd(f, &Emin, 1) && rd(f, &penal, 1) && rd(f, &tol, 1);
    if (!ok || nel < 1 || ndof < 1) return 2;
    std::vector<float> Ke(576), dens(nel), dens2(nel), F(ndof);
    std::vector<int32_t> ed((size_t)nel * 24);
    std::vector<uint8_t> fixed(ndof);
    ok = rd(f, Ke.data(), 576) && rd(f, ed.data(), ed.size()) && rd(f, dens.data(), nel) && rd(f, dens2.data(), nel) &&
         rd(f, F.data(), ndof) && rd(f, fixed.data(), ndof);
    std::fclose(f);
    if (!ok) return 2;

    FILE *o = std::fopen(argv[2], "wb");
    if (!o) return 2;
    tpo_seam::State s;
    tpo_seam::SetupParams q;
    q.KEflat = Ke.data();
    q.edofArray = ed.data();
    q.densities = dens.data();
    q.F = F.data();
    q.fixedMask = fixed.data();
    q.nel = nel;
    q.ndof = ndof;
    q.E0 = E0;
    q.Emin = Emin;
    q.penal = penal;
    q.solver_mg = mg;
    std::vector<float> U(ndof), U2(ndof);
    std::vector<double> U64(ndof), U64b(ndof);
    int rc = 0;
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) q.densities = dens2.data();
        int32_t st = tpo_seam::seam_setup(s, q);
        int32_t it = 0, conv = 0;
        if (st == TPO_OK) {
            int its = 0, cv = 0;
            st = tpo_seam::seam_solve(s, maxit, tol, pass == 1 ? U.data() : nullptr, pass == 0 ? U.data() : U2.data(),
                                      pass == 0 ? U64.data() : U64b.data(), &its, &cv);
            it = its;
            conv = cv;
        }
        if (st != TPO_OK) {
            std::fprintf(stderr, "pass %d: %s\n", pass, s.error.c_str());
            rc = 1;
        }
        std::fwrite(&st, sizeof(st), 1, o);
        std::fwrite(&it, sizeof(it), 1, o);
        std::fwrite(&conv, sizeof(conv), 1, o);
        std::fwrite(pass == 0 ? U.data() : U2.data(), sizeof(float), ndof, o);
        std::fwrite(pass == 0 ? U64.data() : U64b.data(), sizeof(double), ndof, o);
    }
    // then two iterations of the worker's loop on the second setup (structured numbering
    // only): x starts at densities2 and is updated in place
    if (s.structured && rc == 0) {
        tpo_seam::SimpParams sp;
        sp.penal = penal;
        sp.max_iterations = maxit;
        sp.tolerance = 1e-8;
        std::vector<float> x(dens2);
        for (int k = 0; k < 2; k++) {
            double c = 0.0, ch = 0.0;
            int cg = 0;
            int32_t st = tpo_seam::seam_simp_step(s, sp, x.data(), nullptr, nullptr, &c, &ch, &cg);
            if (st != TPO_OK) {
                std::fprintf(stderr, "simp step %d: %s\n", k, s.error.c_str());
                rc = 1;
            }
            std::fwrite(&st, sizeof(st), 1, o);
            std::fwrite(&cg, sizeof(cg), 1, o);
            std::fwrite(&c, sizeof(c), 1, o);
            std::fwrite(&ch, sizeof(ch), 1, o);
        }
        std::fwrite(x.data(), sizeof(float), nel, o);
    }
    tpo_seam::seam_destroy(s);
    std::fclose(o);
    return rc;
}
