/*
 * tpo_oracle.c -- CPU restatement of the reference's 3D SIMP hot path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for libtpo.so, never part of the product.
 * Build: see oracle/Makefile (gcc -O2 -ffp-contract=off, single thread).
 *
 * Citations are file:line in Jozo132/TopologyOptimization.
 */
#include "tpo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* JavaScript Math.max / Math.min: NaN propagates, +0 beats -0 for max. */
static double js_max(double a, double b) {
    if (a != a || b != b) return NAN;
    if (a == b) return signbit(a) ? b : a;
    return a > b ? a : b;
}
static double js_min(double a, double b) {
    if (a != a || b != b) return NAN;
    if (a == b) return signbit(a) ? a : b;
    return a < b ? a : b;
}

/* _powDensity, js/optimizer-worker-3d.js:293-306 */
static double pow_density(double x, double p) {
    if (!isfinite(p) || p != floor(p)) return pow(x, p);
    switch ((int)p) {
    case 0: return 1.0;
    case 1: return x;
    case 2: return x * x;
    case 3: return x * x * x;
    case 4: { double x2 = x * x; return x2 * x2; }
    case 5: { double x2 = x * x; return x2 * x2 * x; }
    case 6: { double x2 = x * x; return x2 * x2 * x2; }
    default: return pow(x, p);
    }
}

/* lk(), js/optimizer-worker-3d.js:3404-3491 (2x2x2 Gauss, unit cube, E = 1). */
void orc_lk(double nu, double *KE) {
    const double E = 1.0;
    double C[6][6];
    memset(C, 0, sizeof C);
    const double fact = E / ((1 + nu) * (1 - 2 * nu));
    C[0][0] = fact * (1 - nu); C[0][1] = fact * nu; C[0][2] = fact * nu;
    C[1][0] = fact * nu; C[1][1] = fact * (1 - nu); C[1][2] = fact * nu;
    C[2][0] = fact * nu; C[2][1] = fact * nu; C[2][2] = fact * (1 - nu);
    C[3][3] = fact * (1 - 2 * nu) / 2;
    C[4][4] = fact * (1 - 2 * nu) / 2;
    C[5][5] = fact * (1 - 2 * nu) / 2;
    for (int i = 0; i < 576; i++) KE[i] = 0.0;
    const double gp[2] = {-1 / sqrt(3.0), 1 / sqrt(3.0)};
    const double gw[2] = {1, 1};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            for (int k = 0; k < 2; k++) {
                const double xi = gp[i], eta = gp[j], zeta = gp[k];
                const double weight = gw[i] * gw[j] * gw[k];
                double dN[8][3] = {
                    {-(1 - eta) * (1 - zeta), -(1 - xi) * (1 - zeta), -(1 - xi) * (1 - eta)},
                    {(1 - eta) * (1 - zeta), -(1 + xi) * (1 - zeta), -(1 + xi) * (1 - eta)},
                    {(1 + eta) * (1 - zeta), (1 + xi) * (1 - zeta), -(1 + xi) * (1 + eta)},
                    {-(1 + eta) * (1 - zeta), (1 - xi) * (1 - zeta), -(1 - xi) * (1 + eta)},
                    {-(1 - eta) * (1 + zeta), -(1 - xi) * (1 + zeta), (1 - xi) * (1 - eta)},
                    {(1 - eta) * (1 + zeta), -(1 + xi) * (1 + zeta), (1 + xi) * (1 - eta)},
                    {(1 + eta) * (1 + zeta), (1 + xi) * (1 + zeta), (1 + xi) * (1 + eta)},
                    {-(1 + eta) * (1 + zeta), (1 - xi) * (1 + zeta), (1 - xi) * (1 + eta)}};
                for (int n = 0; n < 8; n++) {
                    dN[n][0] *= 0.125; dN[n][1] *= 0.125; dN[n][2] *= 0.125;
                }
                const double detJ = 1.0;
                double B[6][24];
                memset(B, 0, sizeof B);
                for (int n = 0; n < 8; n++) {
                    const int col = n * 3;
                    B[0][col] = dN[n][0];
                    B[1][col + 1] = dN[n][1];
                    B[2][col + 2] = dN[n][2];
                    B[3][col] = dN[n][1];
                    B[3][col + 1] = dN[n][0];
                    B[4][col + 1] = dN[n][2];
                    B[4][col + 2] = dN[n][1];
                    B[5][col] = dN[n][2];
                    B[5][col + 2] = dN[n][0];
                }
                double CB[6][24];
                memset(CB, 0, sizeof CB);
                for (int m = 0; m < 6; m++)
                    for (int n = 0; n < 24; n++)
                        for (int p = 0; p < 6; p++) CB[m][n] += C[m][p] * B[p][n];
                for (int m = 0; m < 24; m++)
                    for (int n = 0; n < 24; n++)
                        for (int p = 0; p < 6; p++) KE[m * 24 + n] += B[p][m] * CB[p][n] * detJ * weight;
            }
}

/* _precomputeEdofs3D, js/optimizer-worker-3d.js:1448-1494 (node z fastest, element x fastest). */
void orc_edofs3d(int nelx, int nely, int nelz, int32_t *edofs) {
    const int nny = nely + 1, nnz = nelz + 1;
    for (int elz = 0; elz < nelz; elz++)
        for (int ely = 0; ely < nely; ely++)
            for (int elx = 0; elx < nelx; elx++) {
                const int idx = elx + ely * nelx + elz * nelx * nely;
                const int n[8] = {elx * nny * nnz + ely * nnz + elz,
                                  (elx + 1) * nny * nnz + ely * nnz + elz,
                                  (elx + 1) * nny * nnz + (ely + 1) * nnz + elz,
                                  elx * nny * nnz + (ely + 1) * nnz + elz,
                                  elx * nny * nnz + ely * nnz + (elz + 1),
                                  (elx + 1) * nny * nnz + ely * nnz + (elz + 1),
                                  (elx + 1) * nny * nnz + (ely + 1) * nnz + (elz + 1),
                                  elx * nny * nnz + (ely + 1) * nnz + (elz + 1)};
                for (int a = 0; a < 8; a++)
                    for (int d = 0; d < 3; d++) edofs[(size_t)idx * 24 + a * 3 + d] = 3 * n[a] + d;
            }
}

/* _addNodeDOFs :4429-4434 + getFixedDOFs :4436-4493 */
static int add_node_dofs(uint8_t *fixed, int n, int dofs) {
    int c = 0;
    if (dofs & 1) { fixed[3 * n] = 1; c++; }
    if (dofs & 2) { fixed[3 * n + 1] = 1; c++; }
    if (dofs & 4) { fixed[3 * n + 2] = 1; c++; }
    return c;
}
int orc_fixed_dofs(int nelx, int nely, int nelz, int position, int dofs, uint8_t *fixed) {
    const int nny = nely + 1, nnz = nelz + 1;
    int c = 0;
    switch (position) {
    case 0:
        for (int j = 0; j <= nely; j++)
            for (int k = 0; k <= nelz; k++) c += add_node_dofs(fixed, j * nnz + k, dofs);
        break;
    case 1:
        for (int j = 0; j <= nely; j++)
            for (int k = 0; k <= nelz; k++) c += add_node_dofs(fixed, nelx * nny * nnz + j * nnz + k, dofs);
        break;
    case 2:
        for (int i = 0; i <= nelx; i++)
            for (int k = 0; k <= nelz; k++) c += add_node_dofs(fixed, i * nny * nnz + k, dofs);
        break;
    case 3:
        for (int i = 0; i <= nelx; i++)
            for (int k = 0; k <= nelz; k++) c += add_node_dofs(fixed, i * nny * nnz + nely * nnz + k, dofs);
        break;
    case 4: {
        const int corners[4] = {0, nelx * nny * nnz, nely * nnz, nelx * nny * nnz + nely * nnz};
        for (int q = 0; q < 4; q++) c += add_node_dofs(fixed, corners[q], dofs);
        break;
    }
    default: break;
    }
    return c;
}

/* getConstraintElements :4551-4591 */
void orc_constraint_elements(int nelx, int nely, int nelz, int position, uint8_t *mask) {
    switch (position) {
    case 0:
        for (int ez = 0; ez < nelz; ez++)
            for (int ey = 0; ey < nely; ey++) mask[ey * nelx + ez * nelx * nely] = 1;
        break;
    case 1:
        for (int ez = 0; ez < nelz; ez++)
            for (int ey = 0; ey < nely; ey++) mask[(nelx - 1) + ey * nelx + ez * nelx * nely] = 1;
        break;
    case 2:
        for (int ez = 0; ez < nelz; ez++)
            for (int ex = 0; ex < nelx; ex++) mask[ex + ez * nelx * nely] = 1;
        break;
    case 3:
        for (int ez = 0; ez < nelz; ez++)
            for (int ex = 0; ex < nelx; ex++) mask[ex + (nely - 1) * nelx + ez * nelx * nely] = 1;
        break;
    case 4:
        mask[0] = 1;
        mask[nelx - 1] = 1;
        mask[(nely - 1) * nelx] = 1;
        mask[(nelx - 1) + (nely - 1) * nelx] = 1;
        break;
    default: break;
    }
}

/* applyAEbe3D, assembly/index.ts:403-439 (generalised to edofSize as ebePCG :600-622). */
void orc_apply_a(const double *Ke, const int32_t *edofs, int es, const double *evals,
                 const int32_t *active, int activeCount, const double *p, double *Ap, int ndof) {
    double scratch[24];
    memset(Ap, 0, sizeof(double) * (size_t)ndof);
    for (int ai = 0; ai < activeCount; ai++) {
        const int e = active[ai];
        const double E = evals[e];
        const int32_t *ed = edofs + (size_t)e * es;
        for (int j = 0; j < es; j++) scratch[j] = p[ed[j]];
        for (int i = 0; i < es; i++) {
            double sum = 0.0;
            for (int j = 0; j < es; j++) sum += Ke[i * es + j] * scratch[j];
            Ap[ed[i]] = Ap[ed[i]] + E * sum;
        }
    }
}

/* denseMatVecRaw, assembly/index.ts:450-464 */
void orc_dense_matvec(const double *K, const double *p, double *Ap, int n) {
    for (int i = 0; i < n; i++) {
        double s = 0.0;
        for (int j = 0; j < n; j++) s += K[(size_t)i * n + j] * p[j];
        Ap[i] = s;
    }
}

/* ebePCG, assembly/index.ts:504-733.  Returns the reference's iteration value: the
 * iteration index at convergence, else cgMax (also when it converged on the last pass). */
int orc_ebe_pcg(const double *dens, const double *Ke, const int32_t *edofs, const double *F,
                double *U, const int32_t *freedofs, int nel, int es, int ndof, int nfree,
                double Emin, double E0, double penal, int maxIter, double tol) {
    const double EPS = 1e-12;
    const double dE = E0 - Emin;
    const double skip = Emin * 1000.0;
    double *ev = malloc(sizeof(double) * (size_t)nel);
    int32_t *act = malloc(sizeof(int32_t) * (size_t)nel);
    double *diag = calloc((size_t)ndof, sizeof(double));
    double *Uf = malloc(sizeof(double) * (size_t)nfree), *r = malloc(sizeof(double) * (size_t)nfree);
    double *z = malloc(sizeof(double) * (size_t)nfree), *p = malloc(sizeof(double) * (size_t)nfree);
    double *Ap = malloc(sizeof(double) * (size_t)nfree), *inv = malloc(sizeof(double) * (size_t)nfree);
    double *pf = malloc(sizeof(double) * (size_t)ndof), *apf = malloc(sizeof(double) * (size_t)ndof);
    int na = 0;
    for (int e = 0; e < nel; e++) {
        const double s = Emin + pow(dens[e], penal) * dE;
        ev[e] = s;
        if (s > skip) act[na++] = e;
    }
    for (int ai = 0; ai < na; ai++) {
        const int e = act[ai];
        for (int i = 0; i < es; i++) {
            const int gi = edofs[(size_t)e * es + i];
            diag[gi] = diag[gi] + ev[e] * Ke[i * es + i];
        }
    }
    for (int i = 0; i < nfree; i++) {
        const double d = diag[freedofs[i]];
        inv[i] = d > 1e-30 ? 1.0 / d : 0.0;
    }
    for (int i = 0; i < nfree; i++) Uf[i] = U[freedofs[i]];
    memset(pf, 0, sizeof(double) * (size_t)ndof);
    for (int i = 0; i < nfree; i++) pf[freedofs[i]] = Uf[i];
    orc_apply_a(Ke, edofs, es, ev, act, na, pf, apf, ndof);
    for (int i = 0; i < nfree; i++) r[i] = F[freedofs[i]] - apf[freedofs[i]];
    double rz = 0.0, r0 = 0.0;
    for (int i = 0; i < nfree; i++) {
        const double zi = inv[i] * r[i];
        z[i] = zi; p[i] = zi;
        rz += r[i] * zi;
        r0 += r[i] * r[i];
    }
    const double tolSq = tol * tol * (r0 > 1e-30 ? r0 : 1e-30);
    const int cgMax = maxIter < nfree ? maxIter : nfree;
    int ret = cgMax;
    for (int it = 0; it < cgMax; it++) {
        double rn = 0.0;
        for (int i = 0; i < nfree; i++) rn += r[i] * r[i];
        if (rn < tolSq) { ret = it; goto done; }
        memset(pf, 0, sizeof(double) * (size_t)ndof);
        for (int i = 0; i < nfree; i++) pf[freedofs[i]] = p[i];
        orc_apply_a(Ke, edofs, es, ev, act, na, pf, apf, ndof);
        for (int i = 0; i < nfree; i++) Ap[i] = apf[freedofs[i]];
        double pAp = 0.0;
        for (int i = 0; i < nfree; i++) pAp += p[i] * Ap[i];
        const double alpha = rz / (pAp + EPS);
        double rzn = 0.0;
        for (int i = 0; i < nfree; i++) {
            const double ri = r[i] - alpha * Ap[i];
            const double zi = inv[i] * ri;
            Uf[i] = Uf[i] + alpha * p[i];
            r[i] = ri;
            z[i] = zi;
            rzn += ri * zi;
        }
        const double beta = rzn / (rz + EPS);
        for (int i = 0; i < nfree; i++) p[i] = z[i] + beta * p[i];
        rz = rzn;
    }
done:
    memset(U, 0, sizeof(double) * (size_t)ndof);
    for (int i = 0; i < nfree; i++) U[freedofs[i]] = Uf[i];
    free(ev); free(act); free(diag); free(Uf); free(r); free(z); free(p); free(Ap); free(inv);
    free(pf); free(apf);
    return ret;
}

/* ========================================================================== */
/* Geometric multigrid: MGPrecond3D (js/optimizer-worker-3d.js:317-1025) and   */
/* the WASM core mgApplyA / mgSmooth / mgVcycle / ebeMGPCG                      */
/* (assembly/index.ts:773-1193).                                                */
/* ========================================================================== */
typedef struct {
    int nelx, nely, nelz, nel, ndof, nfree;
    int32_t *edofs;
    uint8_t *fixed;
    int32_t *free;
    float *dens;
    double *E, *diag, *invDiag, *Au, *res, *b, *x;
    int32_t *active;
    int activeCount;
    double *denseK;   /* ndof*ndof or NULL */
    double *chol;     /* coarsest only, coarse_direct: dense lower factor */
    double omega;     /* Jacobi damping of this level */
} orc_level;

struct orc_mg {
    orc_mg_opts o;
    double Ke[576];
    int nl;
    orc_level L[16];
    double *cg[4];
    long long sdof; /* grounded spring k at one fine-level DOF (-1: none), an extension */
    double sk;
};

void orc_mg_default_opts(orc_mg_opts *o) {
    o->max_levels = 6;
    o->galerkin_max_ndof = 3000;
    o->nu1 = 2;
    o->nu2 = 2;
    o->omega = 0.5;
    o->coarse_iters = 30;
    o->coarse_direct = 0;
    o->coarse_moduli = 0;
    o->safe_omega = 0;
}

static void make_level(orc_level *l, int nx, int ny, int nz, const uint8_t *fixed) {
    memset(l, 0, sizeof *l);
    l->nelx = nx; l->nely = ny; l->nelz = nz;
    l->nel = nx * ny * nz;
    l->ndof = 3 * (nx + 1) * (ny + 1) * (nz + 1);
    l->edofs = malloc(sizeof(int32_t) * (size_t)l->nel * 24);
    orc_edofs3d(nx, ny, nz, l->edofs);
    l->fixed = malloc((size_t)l->ndof);
    memcpy(l->fixed, fixed, (size_t)l->ndof);
    int nf = 0;
    for (int i = 0; i < l->ndof; i++) nf += !fixed[i];
    l->nfree = nf;
    l->free = malloc(sizeof(int32_t) * (size_t)(nf ? nf : 1));
    nf = 0;
    for (int i = 0; i < l->ndof; i++) if (!fixed[i]) l->free[nf++] = i;
    l->dens = calloc((size_t)l->nel, sizeof(float));
    l->E = calloc((size_t)l->nel, sizeof(double));
    l->active = calloc((size_t)l->nel, sizeof(int32_t));
    size_t nd = (size_t)l->ndof;
    l->diag = calloc(nd, 8); l->invDiag = calloc(nd, 8);
    l->Au = calloc(nd, 8); l->res = calloc(nd, 8); l->b = calloc(nd, 8); l->x = calloc(nd, 8);
}

/* _downsampleFixedMaskBy2 :384-406 (injection from fine node min(2c, nF-1)). */
static uint8_t *downsample_fixed(const uint8_t *ff, int nxe, int nye, int nze, int cxe, int cye, int cze) {
    const int nxF = nxe + 1, nyF = nye + 1, nzF = nze + 1;
    const int nxC = cxe + 1, nyC = cye + 1, nzC = cze + 1;
    uint8_t *fc = calloc((size_t)3 * nxC * nyC * nzC, 1);
    for (int cz = 0; cz < nzC; cz++) {
        const int fz = 2 * cz < nzF - 1 ? 2 * cz : nzF - 1;
        for (int cy = 0; cy < nyC; cy++) {
            const int fy = 2 * cy < nyF - 1 ? 2 * cy : nyF - 1;
            for (int cx = 0; cx < nxC; cx++) {
                const int fx = 2 * cx < nxF - 1 ? 2 * cx : nxF - 1;
                const int nF = fx * nyF * nzF + fy * nzF + fz;
                const int nC = cx * nyC * nzC + cy * nzC + cz;
                for (int d = 0; d < 3; d++) fc[3 * nC + d] = ff[3 * nF + d];
            }
        }
    }
    return fc;
}

/* ensure() :408-442 */
orc_mg *orc_mg_create(int nelx, int nely, int nelz, const double *Ke, const uint8_t *fixedMask,
                      const orc_mg_opts *opts) {
    orc_mg *mg = calloc(1, sizeof *mg);
    if (opts) mg->o = *opts; else orc_mg_default_opts(&mg->o);
    mg->sdof = -1;
    memcpy(mg->Ke, Ke, sizeof mg->Ke);
    make_level(&mg->L[0], nelx, nely, nelz, fixedMask);
    mg->nl = 1;
    int cx = nelx, cy = nely, cz = nelz;
    for (int li = 1; li < mg->o.max_levels && li < 16; li++) {
        const int nx = cx / 2, ny = cy / 2, nz = cz / 2;
        if (nx < 2 || ny < 2 || nz < 2) break;
        uint8_t *fc = downsample_fixed(mg->L[li - 1].fixed, cx, cy, cz, nx, ny, nz);
        make_level(&mg->L[li], nx, ny, nz, fc);
        free(fc);
        mg->nl++;
        cx = nx; cy = ny; cz = nz;
    }
    const size_t nd = (size_t)mg->L[0].ndof;
    for (int i = 0; i < 4; i++) mg->cg[i] = calloc(nd, 8);
    return mg;
}

void orc_mg_destroy(orc_mg *mg) {
    if (!mg) return;
    for (int li = 0; li < mg->nl; li++) {
        orc_level *l = &mg->L[li];
        free(l->edofs); free(l->fixed); free(l->free); free(l->dens); free(l->E); free(l->active);
        free(l->diag); free(l->invDiag); free(l->Au); free(l->res); free(l->b); free(l->x);
        free(l->denseK); free(l->chol);
    }
    for (int i = 0; i < 4; i++) free(mg->cg[i]);
    free(mg);
}

int orc_mg_num_levels(const orc_mg *mg) { return mg->nl; }

void orc_mg_level_info(const orc_mg *mg, int li, int *d) {
    const orc_level *l = &mg->L[li];
    d[0] = l->nelx; d[1] = l->nely; d[2] = l->nelz; d[3] = l->ndof; d[4] = l->nfree;
    d[5] = l->activeCount; d[6] = l->denseK != NULL; d[7] = l->nel;
}

void orc_mg_level_arrays(const orc_mg *mg, int li, double *evals, double *invDiag, double *denseK) {
    const orc_level *l = &mg->L[li];
    if (evals) memcpy(evals, l->E, sizeof(double) * (size_t)l->nel);
    if (invDiag) memcpy(invDiag, l->invDiag, sizeof(double) * (size_t)l->ndof);
    if (denseK && l->denseK) memcpy(denseK, l->denseK, sizeof(double) * (size_t)l->ndof * l->ndof);
}

/* _updateOperatorLevel :753-796 */
static void update_operator_level(orc_mg *mg, orc_level *l, double penal, double E0, double Emin) {
    const double dE = E0 - Emin, skip = Emin * 1000;
    int ac = 0;
    for (int e = 0; e < l->nel; e++) {
        const double E = Emin + pow_density((double)l->dens[e], penal) * dE;
        l->E[e] = E;
        if (E > skip) l->active[ac++] = e;
    }
    l->activeCount = ac;
    memset(l->diag, 0, sizeof(double) * (size_t)l->ndof);
    for (int ai = 0; ai < ac; ai++) {
        const int e = l->active[ai];
        for (int i = 0; i < 24; i++) {
            const int g = l->edofs[(size_t)e * 24 + i];
            l->diag[g] += l->E[e] * mg->Ke[i * 24 + i];
        }
    }
    if (l == &mg->L[0] && mg->sdof >= 0) l->diag[mg->sdof] += mg->sk;
    memset(l->invDiag, 0, sizeof(double) * (size_t)l->ndof);
    for (int i = 0; i < l->nfree; i++) {
        const int d = l->free[i];
        l->invDiag[d] = l->diag[d] > 1e-30 ? 1.0 / l->diag[d] : 0.0;
    }
}

void orc_mg_set_spring(orc_mg *mg, long long dof, double k) {
    mg->sdof = dof;
    mg->sk = dof >= 0 ? k : 0.0;
}

/* _restrictEvalAvg :702-739 */
static void restrict_eval_avg(orc_mg *mg, const orc_level *f, orc_level *c, double Emin) {
    const int nxF = f->nelx, nyF = f->nely, nzF = f->nelz;
    const int nxC = c->nelx, nyC = c->nely, nzC = c->nelz;
    const double skip = Emin * 1000;
    int ac = 0, idx = 0;
    for (int cz = 0; cz < nzC; cz++)
        for (int cy = 0; cy < nyC; cy++)
            for (int cx = 0; cx < nxC; cx++, idx++) {
                double sum = 0;
                int count = 0;
                for (int dz = 0; dz < 2; dz++) {
                    const int fz = 2 * cz + dz;
                    if (fz >= nzF) continue;
                    for (int dy = 0; dy < 2; dy++) {
                        const int fy = 2 * cy + dy;
                        if (fy >= nyF) continue;
                        for (int dx = 0; dx < 2; dx++) {
                            const int fx = 2 * cx + dx;
                            if (fx >= nxF) continue;
                            const double Ef = f->E[fx + fy * nxF + fz * nxF * nyF];
                            sum += (mg->o.coarse_moduli && !(Ef > skip)) ? 0.0 : Ef;
                            count++;
                        }
                    }
                }
                const double E = count > 0 ? (sum / count) * 2.0 : 0;
                c->E[idx] = E;
                if (E > skip) c->active[ac++] = idx;
            }
    c->activeCount = ac;
    memset(c->diag, 0, sizeof(double) * (size_t)c->ndof);
    for (int ai = 0; ai < ac; ai++) {
        const int e = c->active[ai];
        for (int i = 0; i < 24; i++) c->diag[c->edofs[(size_t)e * 24 + i]] += c->E[e] * mg->Ke[i * 24 + i];
    }
    memset(c->invDiag, 0, sizeof(double) * (size_t)c->ndof);
    for (int i = 0; i < c->nfree; i++) {
        const int d = c->free[i];
        const double v = c->diag[d];
        c->invDiag[d] = v > 1e-30 ? 1.0 / v : 0.0;
    }
    free(c->denseK);
    c->denseK = NULL;
}

/* The volumetric stress field of the SIMP loop (js/optimizer-worker-3d.js:2175-2184):
 * stiffness = Emin + Math.pow(xPhys, penal) (E0 - Emin), stress = stiffness * energy stored
 * into a Float32Array, max over the double values starting at 0 (:2178, :2184). */
void orc_stress(const float *xPhys, const float *energy, int n, double penal, double E0, double Emin,
                float *stress, double *max_stress) {
    double mx = 0.0;
    for (int e = 0; e < n; e++) {
        const double stiffness = Emin + pow((double)xPhys[e], penal) * (E0 - Emin);
        const double sv = stiffness * (double)energy[e];
        stress[e] = (float)sv;
        if (sv > mx) mx = sv;
    }
    *max_stress = mx;
}

/* GPUCompute.computeElementEnergies (js/gpu-compute.js:187-303): the WGSL kernel's
 * arithmetic restated in C, float32 throughout, loop order i then j, negative indices
 * skipped (-ffp-contract=off keeps every product and sum rounded to float). */
void orc_element_energies_f32(const float *U, const float *KE, const int32_t *edofs, int nel, int es,
                              float *energies) {
    for (int el = 0; el < nel; el++) {
        const size_t off = (size_t)el * es;
        float energy = 0.0f;
        for (int i = 0; i < es; i++) {
            const int di = edofs[off + i];
            if (di < 0) continue;
            const float ui = U[di];
            for (int j = 0; j < es; j++) {
                const int dj = edofs[off + j];
                if (dj < 0) continue;
                energy = energy + ui * KE[i * es + j] * U[dj];
            }
        }
        energies[el] = energy;
    }
}

/* _buildProlongMap :585-625 */
static void prolong_map(const orc_level *f, const orc_level *c, int32_t *pN, double *pW, uint8_t *pC) {
    const int nxF = f->nelx + 1, nyF = f->nely + 1, nzF = f->nelz + 1;
    const int nxC = c->nelx + 1, nyC = c->nely + 1, nzC = c->nelz + 1;
    for (int fz = 0; fz < nzF; fz++) {
        const int cz0 = (fz >> 1) < nzC - 1 ? (fz >> 1) : nzC - 1;
        const int cz1 = cz0 + 1 < nzC - 1 ? cz0 + 1 : nzC - 1;
        const double tz = (cz0 != cz1 && (fz & 1)) ? 0.5 : 0.0;
        for (int fy = 0; fy < nyF; fy++) {
            const int cy0 = (fy >> 1) < nyC - 1 ? (fy >> 1) : nyC - 1;
            const int cy1 = cy0 + 1 < nyC - 1 ? cy0 + 1 : nyC - 1;
            const double ty = (cy0 != cy1 && (fy & 1)) ? 0.5 : 0.0;
            for (int fx = 0; fx < nxF; fx++) {
                const int cx0 = (fx >> 1) < nxC - 1 ? (fx >> 1) : nxC - 1;
                const int cx1 = cx0 + 1 < nxC - 1 ? cx0 + 1 : nxC - 1;
                const double tx = (cx0 != cx1 && (fx & 1)) ? 0.5 : 0.0;
                const int nF = fx * nyF * nzF + fy * nzF + fz;
                const int cxa[2] = {cx0, cx1}, cya[2] = {cy0, cy1}, cza[2] = {cz0, cz1};
                const double wxa[2] = {1 - tx, tx}, wya[2] = {1 - ty, ty}, wza[2] = {1 - tz, tz};
                int cnt = 0;
                for (int dz = 0; dz < 2; dz++)
                    for (int dy = 0; dy < 2; dy++)
                        for (int dx = 0; dx < 2; dx++) {
                            const double w = wxa[dx] * wya[dy] * wza[dz];
                            if (w > 0) {
                                pN[nF * 8 + cnt] = cxa[dx] * nyC * nzC + cya[dy] * nzC + cza[dz];
                                pW[nF * 8 + cnt] = w;
                                cnt++;
                            }
                        }
                pC[nF] = (uint8_t)cnt;
            }
        }
    }
}

/* _diagFromDense :742-751 */
static void diag_from_dense(orc_level *l) {
    const int n = l->ndof;
    memset(l->diag, 0, sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) l->diag[i] = l->denseK[(size_t)i * n + i];
    memset(l->invDiag, 0, sizeof(double) * (size_t)n);
    for (int ii = 0; ii < l->nfree; ii++) {
        const int d = l->free[ii];
        l->invDiag[d] = l->diag[d] > 1e-30 ? 1.0 / l->diag[d] : 0;
    }
}

/* _assembleGalerkinFromElements :628-662 */
static void galerkin_from_elements(orc_mg *mg, int li) {
    const orc_level *f = &mg->L[li - 1];
    orc_level *c = &mg->L[li];
    const int n = c->ndof;
    const int nnF = (f->nelx + 1) * (f->nely + 1) * (f->nelz + 1);
    free(c->denseK);
    c->denseK = calloc((size_t)n * n, 8);
    int32_t *pN = calloc((size_t)nnF * 8, 4);
    double *pW = calloc((size_t)nnF * 8, 8);
    uint8_t *pC = calloc((size_t)nnF, 1);
    prolong_map(f, c, pN, pW, pC);
    double *K = c->denseK;
    for (int ai = 0; ai < f->activeCount; ai++) {
        const int e = f->active[ai];
        const double E = f->E[e];
        for (int i = 0; i < 24; i++) {
            const int fdI = f->edofs[(size_t)e * 24 + i], nI = fdI / 3, dI = fdI % 3;
            for (int j = i; j < 24; j++) {
                const double kij = E * mg->Ke[i * 24 + j];
                if (kij == 0) continue;
                const int fdJ = f->edofs[(size_t)e * 24 + j], nJ = fdJ / 3, dJ = fdJ % 3;
                for (int pi = 0; pi < pC[nI]; pi++) {
                    const int cr = 3 * pN[nI * 8 + pi] + dI;
                    const double wi = pW[nI * 8 + pi];
                    for (int pj = 0; pj < pC[nJ]; pj++) {
                        const int cc = 3 * pN[nJ * 8 + pj] + dJ;
                        const double val = wi * kij * pW[nJ * 8 + pj];
                        K[(size_t)cr * n + cc] += val;
                        if (i != j) K[(size_t)cc * n + cr] += val;
                    }
                }
            }
        }
    }
    free(pN); free(pW); free(pC);
    diag_from_dense(c);
}

/* _assembleGalerkinFromMatrix :665-699 */
static void galerkin_from_matrix(orc_mg *mg, int li) {
    const orc_level *f = &mg->L[li - 1];
    orc_level *c = &mg->L[li];
    const int nF = f->ndof, nC = c->ndof;
    const int nnF = (f->nelx + 1) * (f->nely + 1) * (f->nelz + 1);
    int32_t *pN = calloc((size_t)nnF * 8, 4);
    double *pW = calloc((size_t)nnF * 8, 8);
    uint8_t *pC = calloc((size_t)nnF, 1);
    prolong_map(f, c, pN, pW, pC);
    double *P = calloc((size_t)nF * nC, 8);
    for (int nf = 0; nf < nnF; nf++)
        for (int pi = 0; pi < pC[nf]; pi++)
            for (int d = 0; d < 3; d++) P[(size_t)(3 * nf + d) * nC + (3 * pN[nf * 8 + pi] + d)] = pW[nf * 8 + pi];
    double *T = calloc((size_t)nF * nC, 8);
    const double *Kf = f->denseK;
    for (int i = 0; i < nF; i++)
        for (int j = 0; j < nC; j++) {
            double s = 0;
            for (int k = 0; k < nF; k++) s += Kf[(size_t)i * nF + k] * P[(size_t)k * nC + j];
            T[(size_t)i * nC + j] = s;
        }
    free(c->denseK);
    c->denseK = calloc((size_t)nC * nC, 8);
    for (int i = 0; i < nC; i++)
        for (int j = 0; j < nC; j++) {
            double s = 0;
            for (int k = 0; k < nF; k++) s += P[(size_t)k * nC + i] * T[(size_t)k * nC + j];
            c->denseK[(size_t)i * nC + j] = s;
        }
    free(P); free(T); free(pN); free(pW); free(pC);
    diag_from_dense(c);
}

/* Dense Cholesky of the coarsest operator restricted to its free, non-singular DOFs
 * (rows/columns of fixed or zero-diagonal DOFs are replaced by identity).  Used only
 * by the coarse_direct option (an extension); the reference has no direct
 * coarse solve. */
static void coarse_factor(orc_mg *mg) {
    orc_level *c = &mg->L[mg->nl - 1];
    const int n = c->ndof;
    free(c->chol);
    double *A = calloc((size_t)n * n, 8);
    if (c->denseK) {
        memcpy(A, c->denseK, sizeof(double) * (size_t)n * n);
    } else {
        for (int ai = 0; ai < c->activeCount; ai++) {
            const int e = c->active[ai];
            for (int i = 0; i < 24; i++)
                for (int j = 0; j < 24; j++)
                    A[(size_t)c->edofs[(size_t)e * 24 + i] * n + c->edofs[(size_t)e * 24 + j]] +=
                        c->E[e] * mg->Ke[i * 24 + j];
        }
    }
    for (int i = 0; i < n; i++) {
        if (c->invDiag[i] == 0.0) {
            for (int j = 0; j < n; j++) { A[(size_t)i * n + j] = 0; A[(size_t)j * n + i] = 0; }
            A[(size_t)i * n + i] = 1.0;
        }
    }
    /* Cholesky, lower triangle.  A pivot (Schur complement) at or below 1e-10 of its
     * row's diagonal is a singular direction (a floating island of active elements) up
     * to rounding: it is replaced by 1, which decouples it.  The relative test makes the
     * decision independent of the sign of rounding noise in an exactly singular pivot. */
    for (int j = 0; j < n; j++) {
        const double ajj = A[(size_t)j * n + j];
        double d = ajj;
        for (int k = 0; k < j; k++) d -= A[(size_t)j * n + k] * A[(size_t)j * n + k];
        if (!(d > 1e-10 * ajj)) d = 1.0;
        const double ljj = sqrt(d);
        A[(size_t)j * n + j] = ljj;
        for (int i = j + 1; i < n; i++) {
            double s = A[(size_t)i * n + j];
            for (int k = 0; k < j; k++) s -= A[(size_t)i * n + k] * A[(size_t)j * n + k];
            A[(size_t)i * n + j] = s / ljj;
        }
    }
    c->chol = A;
}

static void coarse_solve(const orc_level *c, const double *b, double *x) {
    const int n = c->ndof;
    const double *L = c->chol;
    for (int i = 0; i < n; i++) {
        double s = c->invDiag[i] == 0.0 ? 0.0 : b[i];
        for (int k = 0; k < i; k++) s -= L[(size_t)i * n + k] * x[k];
        x[i] = s / L[(size_t)i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double s = x[i];
        for (int k = i + 1; k < n; k++) s -= L[(size_t)k * n + i] * x[k];
        x[i] = s / L[(size_t)i * n + i];
    }
    for (int i = 0; i < n; i++) if (c->invDiag[i] == 0.0) x[i] = 0.0;
}

/* Damping under safe_omega (an extension, not in the reference): damped Jacobi
 * converges iff omega * lambda_max(D^-1 A) < 2.  For a rediscretised level
 * lambda_max(D^-1 A) <= lambda_max(diag(Ke)^-1 Ke) = kappa; for a dense level the
 * Gershgorin row bound max_i sum_j |A_ij| / A_ii over free rows with a positive diagonal. */
static double ke_kappa(const double *Ke) {
    double a[24][24];
    for (int i = 0; i < 24; i++)
        for (int j = 0; j < 24; j++) a[i][j] = Ke[i * 24 + j] / sqrt(Ke[i * 24 + i] * Ke[j * 24 + j]);
    /* power iteration on the shifted matrix a + I (positive semidefinite + I): converges to
       the largest eigenvalue; 20000 steps on a 24x24 matrix */
    double v[24], w[24], lam = 0.0;
    for (int i = 0; i < 24; i++) v[i] = 1.0 + 0.01 * i;
    for (int it = 0; it < 20000; it++) {
        double nrm = 0.0;
        for (int i = 0; i < 24; i++) {
            double t = v[i];
            for (int j = 0; j < 24; j++) t += a[i][j] * v[j];
            w[i] = t;
            nrm += t * t;
        }
        nrm = sqrt(nrm);
        double num = 0.0, den = 0.0;
        for (int i = 0; i < 24; i++) { num += v[i] * w[i]; den += v[i] * v[i]; }
        lam = num / den - 1.0;
        for (int i = 0; i < 24; i++) v[i] = w[i] / nrm;
    }
    return lam;
}

static double dense_jacobi_bound(const orc_level *l) {
    const int n = l->ndof;
    double g = 0.0;
    for (int i = 0; i < n; i++) {
        const double d = l->denseK[(size_t)i * n + i];
        if (l->fixed[i] || !(d > 1e-30)) continue;
        double s = 0.0;
        for (int j = 0; j < n; j++) s += fabs(l->denseK[(size_t)i * n + j]);
        if (s / d > g) g = s / d;
    }
    return g;
}

/* updateFromFine :558-582 */
void orc_mg_update(orc_mg *mg, const float *xFine, double penal, double E0, double Emin) {
    orc_level *L0 = &mg->L[0];
    memcpy(L0->dens, xFine, sizeof(float) * (size_t)L0->nel);
    update_operator_level(mg, L0, penal, E0, Emin);
    for (int li = 1; li < mg->nl; li++) {
        orc_level *c = &mg->L[li];
        if (c->ndof <= mg->o.galerkin_max_ndof) {
            if (mg->L[li - 1].denseK) galerkin_from_matrix(mg, li);
            else galerkin_from_elements(mg, li);
        } else {
            restrict_eval_avg(mg, &mg->L[li - 1], c, Emin);
        }
    }
    const double kappa = mg->o.safe_omega ? ke_kappa(mg->Ke) : 0.0;
    for (int li = 0; li < mg->nl; li++) {
        orc_level *l = &mg->L[li];
        l->omega = mg->o.omega;
        if (!mg->o.safe_omega) continue;
        const double g = l->denseK ? dense_jacobi_bound(l) : kappa;
        if (g > 0.0 && 1.9 / g < l->omega) l->omega = 1.9 / g;
    }
    if (mg->o.coarse_direct) coarse_factor(mg);
}

/* mgApplyA, assembly/index.ts:773-817 */
void orc_mg_apply_level(orc_mg *mg, int li, const double *p, double *Ap) {
    orc_level *l = &mg->L[li];
    if (l->denseK) {
        orc_dense_matvec(l->denseK, p, Ap, l->ndof);
        return;
    }
    orc_apply_a(mg->Ke, l->edofs, 24, l->E, l->active, l->activeCount, p, Ap, l->ndof);
    if (li == 0 && mg->sdof >= 0) Ap[mg->sdof] += mg->sk * p[mg->sdof];
}

/* mgSmooth, assembly/index.ts:820-834 */
static void mg_smooth(orc_mg *mg, int li, const double *b, double *x) {
    orc_level *l = &mg->L[li];
    orc_mg_apply_level(mg, li, x, l->Au);
    for (int ii = 0; ii < l->nfree; ii++) {
        const int d = l->free[ii];
        const double r = b[d] - l->Au[d];
        x[d] = x[d] + l->omega * l->invDiag[d] * r;
    }
}

/* per-dimension transfer: c0 = min(f>>1, nC-1), c1 = min(c0+1, nC-1), t = 0.5 iff c0 != c1 and f odd */
static void transfer_1d(int f, int nC, int *c0, int *c1, double *w0, double *w1) {
    *c0 = (f >> 1) < nC - 1 ? (f >> 1) : nC - 1;
    *c1 = *c0 + 1 < nC - 1 ? *c0 + 1 : nC - 1;
    const double t = (*c0 != *c1 && (f & 1)) ? 0.5 : 0.0;
    *w0 = 1.0 - t;
    *w1 = t;
}

/* mgVcycle, assembly/index.ts:837-1048 */
static void mg_vcycle(orc_mg *mg, int li, const double *b, double *x) {
    orc_level *l = &mg->L[li];
    const int last = li == mg->nl - 1;
    if (last && mg->o.coarse_direct) {
        coarse_solve(l, b, x);
        return;
    }
    for (int s = 0; s < mg->o.nu1; s++) mg_smooth(mg, li, b, x);
    orc_mg_apply_level(mg, li, x, l->Au);
    memset(l->res, 0, sizeof(double) * (size_t)l->ndof);
    for (int ii = 0; ii < l->nfree; ii++) {
        const int d = l->free[ii];
        l->res[d] = b[d] - l->Au[d];
    }
    if (last) {
        for (int s = 0; s < mg->o.coarse_iters; s++) mg_smooth(mg, li, b, x);
        return;
    }
    orc_level *c = &mg->L[li + 1];
    const int nxF = l->nelx + 1, nyF = l->nely + 1, nzF = l->nelz + 1;
    const int nxC = c->nelx + 1, nyC = c->nely + 1, nzC = c->nelz + 1;
    double *bC = c->b, *xC = c->x;
    memset(bC, 0, sizeof(double) * (size_t)c->ndof);
    for (int fz = 0; fz < nzF; fz++) {
        int cz[2]; double wz[2];
        transfer_1d(fz, nzC, &cz[0], &cz[1], &wz[0], &wz[1]);
        for (int fy = 0; fy < nyF; fy++) {
            int cy[2]; double wy[2];
            transfer_1d(fy, nyC, &cy[0], &cy[1], &wy[0], &wy[1]);
            for (int fx = 0; fx < nxF; fx++) {
                int cx[2]; double wx[2];
                transfer_1d(fx, nxC, &cx[0], &cx[1], &wx[0], &wx[1]);
                const int nF = fx * nyF * nzF + fy * nzF + fz;
                const double r0 = l->res[3 * nF], r1 = l->res[3 * nF + 1], r2 = l->res[3 * nF + 2];
                /* corner order 000,100,010,110,001,101,011,111 as :886-968 */
                for (int q = 0; q < 8; q++) {
                    const int dx = q & 1, dy = (q >> 1) & 1, dz = (q >> 2) & 1;
                    const double w = wx[dx] * wy[dy] * wz[dz];
                    if (w > 0) {
                        const int c3 = 3 * (cx[dx] * nyC * nzC + cy[dy] * nzC + cz[dz]);
                        bC[c3] = bC[c3] + w * r0;
                        bC[c3 + 1] = bC[c3 + 1] + w * r1;
                        bC[c3 + 2] = bC[c3 + 2] + w * r2;
                    }
                }
            }
        }
    }
    for (int i = 0; i < c->ndof; i++) if (c->fixed[i]) bC[i] = 0.0;
    memset(xC, 0, sizeof(double) * (size_t)c->ndof);
    mg_vcycle(mg, li + 1, bC, xC);
    for (int fz = 0; fz < nzF; fz++) {
        int cz[2]; double wz[2];
        transfer_1d(fz, nzC, &cz[0], &cz[1], &wz[0], &wz[1]);
        for (int fy = 0; fy < nyF; fy++) {
            int cy[2]; double wy[2];
            transfer_1d(fy, nyC, &cy[0], &cy[1], &wy[0], &wy[1]);
            for (int fx = 0; fx < nxF; fx++) {
                int cx[2]; double wx[2];
                transfer_1d(fx, nxC, &cx[0], &cx[1], &wx[0], &wx[1]);
                const int nF = fx * nyF * nzF + fy * nzF + fz;
                for (int d = 0; d < 3; d++) {
                    const int fi = 3 * nF + d;
                    if (l->fixed[fi]) continue;
                    double val = 0.0;
                    int first = 1;
                    for (int q = 0; q < 8; q++) {
                        const int dx = q & 1, dy = (q >> 1) & 1, dz = (q >> 2) & 1;
                        const double w = wx[dx] * wy[dy] * wz[dz];
                        const double term = xC[3 * (cx[dx] * nyC * nzC + cy[dy] * nzC + cz[dz]) + d] * w;
                        if (first) { val = term; first = 0; } else val = val + term;
                    }
                    x[fi] = x[fi] + val;
                }
            }
        }
    }
    for (int s = 0; s < mg->o.nu2; s++) mg_smooth(mg, li, b, x);
}

void orc_mg_vcycle(orc_mg *mg, const double *b, double *x) { mg_vcycle(mg, 0, b, x); }

/* ebeMGPCG, assembly/index.ts:1076-1193 (cold start). */
int orc_mgpcg(orc_mg *mg, const double *F, double *U, int maxIter, double tol) {
    const double EPS = 1e-12;
    const orc_level *l0 = &mg->L[0];
    const int n = l0->ndof;
    const uint8_t *fm = l0->fixed;
    double *r = mg->cg[0], *z = mg->cg[1], *p = mg->cg[2], *Ap = mg->cg[3];
    memset(U, 0, sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) r[i] = fm[i] ? 0.0 : F[i];
    memset(z, 0, sizeof(double) * (size_t)n);
    mg_vcycle(mg, 0, r, z);
    for (int i = 0; i < n; i++) if (fm[i]) z[i] = 0.0;
    memcpy(p, z, sizeof(double) * (size_t)n);
    double rz = 0.0, r0 = 0.0;
    for (int i = 0; i < n; i++) { rz += r[i] * z[i]; r0 += r[i] * r[i]; }
    const double tolSq = tol * tol * (r0 > 1e-30 ? r0 : 1e-30);
    for (int it = 0; it < maxIter; it++) {
        double rn = 0.0;
        for (int i = 0; i < n; i++) rn += r[i] * r[i];
        if (rn < tolSq) return it;
        orc_mg_apply_level(mg, 0, p, Ap);
        for (int i = 0; i < n; i++) if (fm[i]) Ap[i] = 0.0;
        double pAp = 0.0;
        for (int i = 0; i < n; i++) pAp += p[i] * Ap[i];
        const double alpha = rz / (pAp + EPS);
        for (int i = 0; i < n; i++) {
            U[i] = U[i] + alpha * p[i];
            r[i] = r[i] - alpha * Ap[i];
        }
        memset(z, 0, sizeof(double) * (size_t)n);
        mg_vcycle(mg, 0, r, z);
        for (int i = 0; i < n; i++) if (fm[i]) z[i] = 0.0;
        double rzn = 0.0;
        for (int i = 0; i < n; i++) rzn += r[i] * z[i];
        const double beta = rzn / (rz + EPS);
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rzn;
    }
    return maxIter;
}

/* FE() JS PCG, js/optimizer-worker-3d.js:4189-4371 (full space, warm start, fixed DOFs
 * masked).  precond 0 = Jacobi (_computeFullDiagonal :4401-4417), 1 = MG (apply :1021).
 * Returns cgIters as the reference counts it (iterations actually performed). */
int orc_fe_pcg(orc_mg *mg, int precond, const double *F, double *U, int maxIter, double tol) {
    const double EPS = 1e-12;
    orc_level *l0 = &mg->L[0];
    const int n = l0->ndof;
    const uint8_t *fm = l0->fixed;
    double *r = mg->cg[0], *z = mg->cg[1], *p = mg->cg[2], *Ap = mg->cg[3];
    double *inv = calloc((size_t)n, 8);
    for (int i = 0; i < n; i++) if (!fm[i] && l0->diag[i] > 1e-30) inv[i] = 1.0 / l0->diag[i];
    for (int i = 0; i < n; i++) if (fm[i]) U[i] = 0;
    orc_mg_apply_level(mg, 0, U, r);
    for (int i = 0; i < n; i++) r[i] = F[i] - r[i];
    for (int i = 0; i < n; i++) if (fm[i]) r[i] = 0;
    if (precond == 1) { memset(z, 0, 8 * (size_t)n); mg_vcycle(mg, 0, r, z); }
    else for (int i = 0; i < n; i++) z[i] = inv[i] * r[i];
    for (int i = 0; i < n; i++) if (fm[i]) z[i] = 0;
    memcpy(p, z, 8 * (size_t)n);
    double rz = 0;
    for (int i = 0; i < n; i++) rz += r[i] * z[i];
    double r0 = 0;
    for (int i = 0; i < n; i++) r0 += r[i] * r[i];
    const double tolSq = tol * tol * (r0 > 1e-30 ? r0 : 1e-30);
    int cgIters = 0;
    for (int it = 0; it < maxIter; it++) {
        double rn = 0;
        for (int i = 0; i < n; i++) rn += r[i] * r[i];
        if (rn < tolSq) break;
        cgIters = it + 1;
        orc_mg_apply_level(mg, 0, p, Ap);
        for (int i = 0; i < n; i++) if (fm[i]) Ap[i] = 0;
        double pAp = 0;
        for (int i = 0; i < n; i++) pAp += p[i] * Ap[i];
        const double alpha = rz / (pAp + EPS);
        for (int i = 0; i < n; i++) { U[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        if (precond == 1) { memset(z, 0, 8 * (size_t)n); mg_vcycle(mg, 0, r, z); }
        else for (int i = 0; i < n; i++) z[i] = inv[i] * r[i];
        for (int i = 0; i < n; i++) if (fm[i]) z[i] = 0;
        double rzn = 0;
        for (int i = 0; i < n; i++) rzn += r[i] * z[i];
        const double beta = rzn / (rz + EPS);
        for (int i = 0; i < n; i++) p[i] = z[i] + beta * p[i];
        rz = rzn;
    }
    free(inv);
    return cgIters;
}

/* ========================================================================== */
/* KSP CG + "BDDC": KSPSolver._buildSubdomains / _updateBDDC                   */
/* (js/optimizer-worker-3d.js:1141-1231), _solveWithWasmKSP_BDDC (:3814-3970)  */
/* and ebeKSP_BDDC / bddcApply / bddcApplyA (assembly/index.ts:1204-1517).     */
/* ========================================================================== */
void orc_bddc_partition(int nelx, int nely, int nelz, int ns[3]) {
    const long long total = (long long)nelx * nely * nelz;
    double tgt = ceil(cbrt((double)total / 100.0));
    if (tgt > 64) tgt = 64;
    if (tgt < 8) tgt = 8;
    const double nx = nelx, ny = nely, nz = nelz;
    const double fx = round(cbrt(tgt * (nx * nx) / (ny * nz)));
    const double fy = round(cbrt(tgt * (ny * ny) / (nx * nz)));
    const double fz = round(cbrt(tgt * (nz * nz) / (nx * ny)));
    ns[0] = (int)(fx < nx ? fx : nx);
    ns[1] = (int)(fy < ny ? fy : ny);
    ns[2] = (int)(fz < nz ? fz : nz);
    for (int a = 0; a < 3; a++) if (ns[a] < 2) ns[a] = 2; /* KSP_BDDC_MIN_SUBDOMAINS */
}

typedef struct {
    int n;            /* DOFs touched */
    int32_t *dofs;    /* sorted */
    double *lid;      /* local inverse diagonal, ndof entries */
} orc_sub;

/* bddcApplyA :1227-1255: y = sum over active e of E_e Ke x_e (y zeroed first) */
static void bddc_apply_a(const double *Ke, const int32_t *edofs, const double *ev, const int32_t *act, int na,
                         const double *x, double *y, int ndof) {
    orc_apply_a(Ke, edofs, 24, ev, act, na, x, y, ndof);
}

int orc_ksp_bddc(int nelx, int nely, int nelz, const double *Ke, const float *x, double penal, double E0,
                 double Emin, const uint8_t *fixed, const double *F, double *U, int maxIter, double tol,
                 int smootherIters) {
    const double EPS = 1e-12;
    const int nel = nelx * nely * nelz;
    const int nny = nely + 1, nnz = nelz + 1;
    const int ndof = 3 * (nelx + 1) * nny * nnz;
    int32_t *edofs = malloc(sizeof(int32_t) * (size_t)nel * 24);
    orc_edofs3d(nelx, nely, nelz, edofs);
    /* E_vals with Math.pow (:3825-3830 and KSPSolver.updateOperators :1110-1116) */
    double *ev = malloc(8 * (size_t)nel);
    int32_t *act = malloc(4 * (size_t)nel);
    int na = 0;
    for (int e = 0; e < nel; e++) {
        const double E = Emin + pow((double)x[e], penal) * (E0 - Emin);
        ev[e] = E;
        if (E > Emin * 1000.0) act[na++] = e;
    }
    double *diag = calloc((size_t)ndof, 8), *inv = calloc((size_t)ndof, 8);
    for (int ai = 0; ai < na; ai++) {
        const int e = act[ai];
        for (int i = 0; i < 24; i++) diag[edofs[(size_t)e * 24 + i]] += ev[e] * Ke[i * 24 + i];
    }
    for (int i = 0; i < ndof; i++) if (!fixed[i] && diag[i] > 1e-30) inv[i] = 1.0 / diag[i];
    /* _buildSubdomains: blocks in (sz, sy, sx) order, empty blocks dropped */
    int ns[3];
    orc_bddc_partition(nelx, nely, nelz, ns);
    const int maxsub = ns[0] * ns[1] * ns[2];
    orc_sub *subs = calloc((size_t)maxsub, sizeof(orc_sub));
    uint8_t *coarse = calloc((size_t)ndof, 1);
    uint8_t *mark = calloc((size_t)ndof, 1);
    double *ldiag = malloc(8 * (size_t)ndof);
    int nsub = 0;
    for (int sz = 0; sz < ns[2]; sz++) {
        const int z0 = (int)floor((double)sz * nelz / ns[2]), z1 = (int)floor((double)(sz + 1) * nelz / ns[2]);
        for (int sy = 0; sy < ns[1]; sy++) {
            const int y0 = (int)floor((double)sy * nely / ns[1]), y1 = (int)floor((double)(sy + 1) * nely / ns[1]);
            for (int sx = 0; sx < ns[0]; sx++) {
                const int x0 = (int)floor((double)sx * nelx / ns[0]), x1 = (int)floor((double)(sx + 1) * nelx / ns[0]);
                if (x1 <= x0 || y1 <= y0 || z1 <= z0) continue;
                orc_sub *sb = &subs[nsub++];
                /* corner nodes -> coarse DOFs (clamped) */
                const int cxs[2] = {x0, x1}, cys[2] = {y0, y1}, czs[2] = {z0, z1};
                for (int a = 0; a < 2; a++)
                    for (int b = 0; b < 2; b++)
                        for (int cc = 0; cc < 2; cc++) {
                            const int cx = cxs[cc] < nelx ? cxs[cc] : nelx, cy = cys[b] < nely ? cys[b] : nely;
                            const int cz = czs[a] < nelz ? czs[a] : nelz;
                            const int node = cx * nny * nnz + cy * nnz + cz;
                            coarse[3 * node] = coarse[3 * node + 1] = coarse[3 * node + 2] = 1;
                        }
                /* _updateBDDC: DOFs touched, local diagonal over every element of the block */
                memset(mark, 0, (size_t)ndof);
                memset(ldiag, 0, 8 * (size_t)ndof);
                int cnt = 0;
                for (int ez = z0; ez < z1; ez++)
                    for (int ey = y0; ey < y1; ey++)
                        for (int ex = x0; ex < x1; ex++) {
                            const int e = ex + ey * nelx + ez * nelx * nely;
                            for (int i = 0; i < 24; i++) {
                                const int d = edofs[(size_t)e * 24 + i];
                                if (!mark[d]) { mark[d] = 1; cnt++; }
                            }
                            if (ev[e] < 1e-30) continue;
                            for (int i = 0; i < 24; i++) ldiag[edofs[(size_t)e * 24 + i]] += ev[e] * Ke[i * 24 + i];
                        }
                sb->n = cnt;
                sb->dofs = malloc(4 * (size_t)cnt);
                sb->lid = calloc((size_t)ndof, 8);
                int k = 0;
                for (int d = 0; d < ndof; d++)
                    if (mark[d]) {
                        sb->dofs[k++] = d;
                        if (!fixed[d] && ldiag[d] > 1e-30) sb->lid[d] = 1.0 / ldiag[d];
                    }
            }
        }
    }
    int32_t *cmap = malloc(4 * (size_t)ndof);
    int ncoarse = 0;
    for (int d = 0; d < ndof; d++) if (coarse[d]) cmap[ncoarse++] = d;
    double *r = calloc((size_t)ndof, 8), *z = calloc((size_t)ndof, 8), *p = calloc((size_t)ndof, 8);
    double *Ap = calloc((size_t)ndof, 8), *lc = calloc((size_t)ndof, 8), *w = calloc((size_t)ndof, 8);
    double *cc = calloc((size_t)ndof, 8);
    /* bddcApply :1264-1353 */
#define BDDC_APPLY()                                                                                   \
    do {                                                                                               \
        memset(z, 0, 8 * (size_t)ndof);                                                                \
        memset(w, 0, 8 * (size_t)ndof);                                                                \
        for (int si = 0; si < nsub; si++)                                                              \
            for (int li = 0; li < subs[si].n; li++) {                                                  \
                const int gi = subs[si].dofs[li];                                                      \
                z[gi] = z[gi] + subs[si].lid[gi] * r[gi];                                              \
                w[gi] = w[gi] + 1.0;                                                                   \
            }                                                                                          \
        for (int i = 0; i < ndof; i++) if (w[i] > 1e-12) z[i] = z[i] / w[i];                          \
        for (int sw = 1; sw < smootherIters; sw++) {                                                   \
            bddc_apply_a(Ke, edofs, ev, act, na, z, lc, ndof);                                         \
            for (int i = 0; i < ndof; i++) { const double res = r[i] - lc[i]; z[i] = z[i] + inv[i] * res; } \
        }                                                                                              \
        memset(cc, 0, 8 * (size_t)ndof);                                                               \
        if (ncoarse > 0) {                                                                             \
            bddc_apply_a(Ke, edofs, ev, act, na, z, lc, ndof);                                         \
            for (int ci = 0; ci < ncoarse; ci++) {                                                     \
                const int gi = cmap[ci];                                                               \
                cc[gi] = inv[gi] * (r[gi] - lc[gi]);                                                   \
            }                                                                                          \
        }                                                                                              \
        for (int i = 0; i < ndof; i++) z[i] = z[i] + cc[i];                                            \
        for (int i = 0; i < ndof; i++) if (fixed[i]) z[i] = 0.0;                                       \
    } while (0)
    /* ebeKSP_BDDC :1386-1516 */
    memset(U, 0, 8 * (size_t)ndof);
    for (int i = 0; i < ndof; i++) r[i] = fixed[i] ? 0.0 : F[i];
    BDDC_APPLY();
    memcpy(p, z, 8 * (size_t)ndof);
    double rz = 0.0, r0 = 0.0;
    for (int i = 0; i < ndof; i++) { rz += r[i] * z[i]; r0 += r[i] * r[i]; }
    const double tolSq = tol * tol * (r0 > 1e-30 ? r0 : 1e-30);
    int ret = maxIter;
    for (int it = 0; it < maxIter; it++) {
        double rn = 0.0;
        for (int i = 0; i < ndof; i++) rn += r[i] * r[i];
        if (rn < tolSq) { ret = it; break; }
        bddc_apply_a(Ke, edofs, ev, act, na, p, Ap, ndof);
        for (int i = 0; i < ndof; i++) if (fixed[i]) Ap[i] = 0.0;
        double pAp = 0.0;
        for (int i = 0; i < ndof; i++) pAp += p[i] * Ap[i];
        const double alpha = rz / (pAp + EPS);
        for (int i = 0; i < ndof; i++) { U[i] = U[i] + alpha * p[i]; r[i] = r[i] - alpha * Ap[i]; }
        BDDC_APPLY();
        double rzn = 0.0;
        for (int i = 0; i < ndof; i++) rzn += r[i] * z[i];
        const double beta = rzn / (rz + EPS);
        for (int i = 0; i < ndof; i++) p[i] = z[i] + beta * p[i];
        rz = rzn;
    }
#undef BDDC_APPLY
    for (int si = 0; si < nsub; si++) { free(subs[si].dofs); free(subs[si].lid); }
    free(subs); free(coarse); free(mark); free(ldiag); free(cmap);
    free(r); free(z); free(p); free(Ap); free(lc); free(w); free(cc);
    free(edofs); free(ev); free(act); free(diag); free(inv);
    return ret;
}

/* ========================================================================== */
/* SIMP pieces                                                                 */
/* ========================================================================== */

/* element energy loop :2163-2173 with _computeElementEnergyFlat :1561-1571 (unit Ke,
 * every element), stored into a Float32Array. */
void orc_element_energy(const double *Ke, int nelx, int nely, int nelz, const double *U, float *energy) {
    const int nny = nely + 1, nnz = nelz + 1;
    double Ue[24];
    for (int elz = 0; elz < nelz; elz++)
        for (int ely = 0; ely < nely; ely++)
            for (int elx = 0; elx < nelx; elx++) {
                const int e = elx + ely * nelx + elz * nelx * nely;
                const int n[8] = {elx * nny * nnz + ely * nnz + elz,
                                  (elx + 1) * nny * nnz + ely * nnz + elz,
                                  (elx + 1) * nny * nnz + (ely + 1) * nnz + elz,
                                  elx * nny * nnz + (ely + 1) * nnz + elz,
                                  elx * nny * nnz + ely * nnz + (elz + 1),
                                  (elx + 1) * nny * nnz + ely * nnz + (elz + 1),
                                  (elx + 1) * nny * nnz + (ely + 1) * nnz + (elz + 1),
                                  elx * nny * nnz + (ely + 1) * nnz + (elz + 1)};
                for (int a = 0; a < 8; a++)
                    for (int d = 0; d < 3; d++) Ue[a * 3 + d] = U[3 * n[a] + d];
                double en = 0;
                for (int i = 0; i < 24; i++) {
                    const double ui = Ue[i];
                    for (int j = 0; j < 24; j++) en += ui * Ke[i * 24 + j] * Ue[j];
                }
                energy[e] = (float)en;
            }
}

/* _heavisideProject :3500-3509 (eta = 0.5) */
void orc_heaviside(const float *x, int n, double beta, float *xPhys) {
    const double eta = 0.5;
    const double tb = tanh(beta * eta), tb1 = tanh(beta * (1 - eta));
    const double den = tb + tb1;
    for (int i = 0; i < n; i++) xPhys[i] = (float)((tb + tanh(beta * ((double)x[i] - eta))) / den);
}

/* sensitivity :2175-2192 (note E0, not E0 - Emin) */
void orc_sensitivity(const float *x, const float *xPhys, const float *energy, int n, double penal,
                     double E0, double beta, int useProj, float *dc) {
    const double tb = tanh(beta * 0.5);
    const double hden = 2 * tb;
    for (int e = 0; e < n; e++) {
        const double en = energy[e];
        const double dcp = -penal * pow((double)xPhys[e], penal - 1) * E0 * en;
        const double th = tanh(beta * ((double)x[e] - 0.5));
        const double dpdx = useProj ? beta * (1 - th * th) / hden : 1.0;
        dc[e] = (float)(dcp * dpdx);
    }
}

/* prepareFilter :3006-3050 -- Hs accumulated into a Float32Array in triplet order. */
void orc_filter_hs(int nelx, int nely, int nelz, double rmin, float *Hs) {
    const int R = (int)floor(rmin);
    memset(Hs, 0, sizeof(float) * (size_t)nelx * nely * nelz);
    for (int i = 0; i < nelx; i++)
        for (int j = 0; j < nely; j++)
            for (int m = 0; m < nelz; m++) {
                const int e1 = i + j * nelx + m * nelx * nely;
                for (int k = (i - R > 0 ? i - R : 0); k <= (i + R < nelx - 1 ? i + R : nelx - 1); k++)
                    for (int l = (j - R > 0 ? j - R : 0); l <= (j + R < nely - 1 ? j + R : nely - 1); l++)
                        for (int nn = (m - R > 0 ? m - R : 0); nn <= (m + R < nelz - 1 ? m + R : nelz - 1); nn++) {
                            const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l) + (m - nn) * (m - nn)));
                            if (dist <= rmin) Hs[e1] = (float)((double)Hs[e1] + js_max(0, rmin - dist));
                        }
            }
}

/* filterSensitivities :3052-3064 -- dcn accumulated into a Float32Array. */
void orc_filter_sens(int nelx, int nely, int nelz, double rmin, const float *Hs, const float *x,
                     const float *dc, float *dcn) {
    const int R = (int)floor(rmin);
    const int nel = nelx * nely * nelz;
    memset(dcn, 0, sizeof(float) * (size_t)nel);
    for (int i = 0; i < nelx; i++)
        for (int j = 0; j < nely; j++)
            for (int m = 0; m < nelz; m++) {
                const int e1 = i + j * nelx + m * nelx * nely;
                for (int k = (i - R > 0 ? i - R : 0); k <= (i + R < nelx - 1 ? i + R : nelx - 1); k++)
                    for (int l = (j - R > 0 ? j - R : 0); l <= (j + R < nely - 1 ? j + R : nely - 1); l++)
                        for (int nn = (m - R > 0 ? m - R : 0); nn <= (m + R < nelz - 1 ? m + R : nelz - 1); nn++) {
                            const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l) + (m - nn) * (m - nn)));
                            if (dist <= rmin) {
                                const int e2 = k + l * nelx + nn * nelx * nely;
                                const double s = js_max(0, rmin - dist);
                                dcn[e1] = (float)((double)dcn[e1] + s * (double)x[e2] * (double)dc[e2]);
                            }
                        }
            }
    for (int i = 0; i < nel; i++)
        dcn[i] = (float)((double)dcn[i] / ((double)Hs[i] * js_max(1e-3, (double)x[i])));
}

/* applyDensityFilter, assembly/index.ts:224-273 */
void orc_density_filter(const double *dens, double *out, int nx, int ny, int nz, double radius) {
    const int r = (int)ceil(radius);
    const double r2 = radius * radius;
    for (int ez = 0; ez < nz; ez++)
        for (int ey = 0; ey < ny; ey++)
            for (int ex = 0; ex < nx; ex++) {
                double sum = 0.0, sw = 0.0;
                const int z0 = ez - r > 0 ? ez - r : 0, z1 = ez + r < nz - 1 ? ez + r : nz - 1;
                const int y0 = ey - r > 0 ? ey - r : 0, y1 = ey + r < ny - 1 ? ey + r : ny - 1;
                const int x0 = ex - r > 0 ? ex - r : 0, x1 = ex + r < nx - 1 ? ex + r : nx - 1;
                for (int kz = z0; kz <= z1; kz++)
                    for (int ky = y0; ky <= y1; ky++)
                        for (int kx = x0; kx <= x1; kx++) {
                            const double dx = ex - kx, dy = ey - ky, dz = ez - kz;
                            const double d2 = dx * dx + dy * dy + dz * dz;
                            if (d2 <= r2) {
                                const double w = radius - sqrt(d2);
                                sum += w * dens[kx + ky * nx + kz * nx * ny];
                                sw += w;
                            }
                        }
                out[ex + ey * nx + ez * nx * ny] = sum / sw;
            }
}

/* OC :3066-3101 (move 0.2, bisection on [0, 1e9] to 1e-3 relative). */
void orc_oc(int nel, const float *x, double volfrac, const float *dc, const uint8_t *pres,
            const uint8_t *voidm, float *xnew, double *lmid_out, int *nb_out) {
    orc_oc_move(nel, x, volfrac, dc, pres, voidm, 0.2, xnew, lmid_out, nb_out);
}

/* The same bisection with the move limit as a parameter (the reference fixes it at 0.2). */
void orc_oc_move(int nel, const float *x, double volfrac, const float *dc, const uint8_t *pres,
                 const uint8_t *voidm, double move, float *xnew, double *lmid_out, int *nb_out) {
    double l1 = 0, l2 = 1e9, lmid = 0;
    int nb = 0;
    while ((l2 - l1) / (l2 + l1) > 1e-3) {
        lmid = 0.5 * (l2 + l1);
        for (int i = 0; i < nel; i++) {
            if (pres && pres[i]) xnew[i] = 1.0f;
            else if (voidm && voidm[i]) xnew[i] = 0.0f;
            else {
                const double xi = x[i];
                const double Be = -(double)dc[i] / lmid;
                xnew[i] = (float)js_max(0.0, js_max(xi - move, js_min(1.0, js_min(xi + move, xi * sqrt(Be)))));
            }
        }
        double s = 0;
        for (int i = 0; i < nel; i++) s += xnew[i];
        if (s > volfrac * nel) l1 = lmid; else l2 = lmid;
        nb++;
    }
    if (lmid_out) *lmid_out = lmid;
    if (nb_out) *nb_out = nb;
}

/* optimize() SIMP loop :1943-2301 restricted to the hot path (no AMR, no manufacturing
 * constraints, no UI mesh). */
int orc_simp(const orc_simp_cfg *cfg, const float *F32, const uint8_t *fixedMask,
             const uint8_t *pres, const uint8_t *voidm, const orc_mg_opts *mgopts,
             double *c_hist, double *ch_hist, int *cg_hist, float *x_out) {
    const int nelx = cfg->nelx, nely = cfg->nely, nelz = cfg->nelz;
    const int nel = nelx * nely * nelz;
    const int ndof = 3 * (nelx + 1) * (nely + 1) * (nelz + 1);
    double Ke[576];
    orc_lk(cfg->nu, Ke);
    int32_t *edofs = malloc(sizeof(int32_t) * (size_t)nel * 24);
    orc_edofs3d(nelx, nely, nelz, edofs);
    int nfree = 0;
    for (int i = 0; i < ndof; i++) nfree += !fixedMask[i];
    int32_t *freed = malloc(sizeof(int32_t) * (size_t)nfree);
    nfree = 0;
    for (int i = 0; i < ndof; i++) if (!fixedMask[i]) freed[nfree++] = i;
    double *F = malloc(8 * (size_t)ndof), *U = calloc((size_t)ndof, 8), *Uprev = calloc((size_t)ndof, 8);
    for (int i = 0; i < ndof; i++) F[i] = F32[i];
    float *bufA = malloc(4 * (size_t)nel), *bufB = malloc(4 * (size_t)nel);
    float *x = bufA, *xnew = bufB, *xold = malloc(4 * (size_t)nel);
    float *xPhys = malloc(4 * (size_t)nel), *en = malloc(4 * (size_t)nel), *dc = malloc(4 * (size_t)nel);
    float *dcn = malloc(4 * (size_t)nel), *Hs = malloc(4 * (size_t)nel);
    double *dens64 = malloc(8 * (size_t)nel);
    for (int i = 0; i < nel; i++) x[i] = (float)cfg->volfrac;
    for (int i = 0; i < nel; i++) if (pres && pres[i]) x[i] = 1.0f;
    for (int i = 0; i < nel; i++) if (voidm && voidm[i]) x[i] = 0.0f;
    orc_filter_hs(nelx, nely, nelz, cfg->rmin, Hs);
    orc_mg *mg = orc_mg_create(nelx, nely, nelz, Ke, fixedMask, mgopts);
    const double pT = cfg->penal;
    const double pS = cfg->penal_start >= 0 ? cfg->penal_start : (pT < 1.5 ? pT : 1.5);
    const int contI = cfg->continuation_iters >= 0 ? cfg->continuation_iters
                                                   : (20 > cfg->max_iter / 3 ? 20 : cfg->max_iter / 3);
    int loop = 0;
    double change = 1;
    while ((!cfg->stop_on_change || change > 0.01) && loop < cfg->max_iter) {
        loop++;
        memcpy(xold, x, 4 * (size_t)nel);
        const double fr = (double)(loop - 1) / contI;
        const double cp = pS + (pT - pS) * (fr < 1.0 ? fr : 1.0);
        double beta = 1;
        if (cfg->use_projection) {
            beta = pow(2, floor((double)(loop - 1) / cfg->beta_interval));
            if (cfg->beta_max < beta) beta = cfg->beta_max;
            orc_heaviside(x, nel, beta, xPhys);
        } else {
            memcpy(xPhys, x, 4 * (size_t)nel);
        }
        double tol;
        if (cfg->cg_tol > 0) tol = cfg->cg_tol;
        else {
            const double prog = cfg->max_iter > 1 ? (double)(loop - 1) / (cfg->max_iter - 1) : 1;
            tol = exp(log(1e-3) + prog * (log(1e-8) - log(1e-3)));
        }
        const int cgmax = nfree < cfg->cg_max_iter ? nfree : cfg->cg_max_iter;
        int its = 0;
        if (cfg->solver == 0) {
            for (int i = 0; i < nel; i++) dens64[i] = xPhys[i];
            if (loop > 1) memcpy(U, Uprev, 8 * (size_t)ndof); else memset(U, 0, 8 * (size_t)ndof);
            its = orc_ebe_pcg(dens64, Ke, edofs, F, U, freed, nel, 24, ndof, nfree, cfg->Emin, cfg->E0,
                              cp, cgmax, tol);
        } else if (cfg->solver == 1) {
            orc_mg_update(mg, xPhys, cp, cfg->E0, cfg->Emin);
            its = orc_mgpcg(mg, F, U, cgmax, tol);
        } else if (cfg->solver == 4) {
            /* linearSolver 'petsc': _solveWithWasmKSP_BDDC (:3814-3970), U filled with 0
             * (:3922-3923), KSP_BDDC_SMOOTHER_ITERS = 3 (:1031) */
            memset(U, 0, 8 * (size_t)ndof);
            its = orc_ksp_bddc(nelx, nely, nelz, Ke, xPhys, cp, cfg->E0, cfg->Emin, fixedMask, F, U, cgmax, tol, 3);
        } else {
            orc_mg_update(mg, xPhys, cp, cfg->E0, cfg->Emin);
            if (loop > 1) memcpy(U, Uprev, 8 * (size_t)ndof); else memset(U, 0, 8 * (size_t)ndof);
            its = orc_fe_pcg(mg, cfg->solver == 3 ? 1 : 0, F, U, cgmax, tol);
        }
        memcpy(Uprev, U, 8 * (size_t)ndof);
        double c = 0;
        for (int i = 0; i < ndof; i++) c += F[i] * U[i];
        orc_element_energy(Ke, nelx, nely, nelz, U, en);
        orc_sensitivity(x, xPhys, en, nel, cp, cfg->E0, beta, cfg->use_projection, dc);
        orc_filter_sens(nelx, nely, nelz, cfg->rmin, Hs, x, dc, dcn);
        orc_oc(nel, x, cfg->volfrac, dcn, pres, voidm, xnew, NULL, NULL);
        change = 0;
        for (int i = 0; i < nel; i++) {
            const double d = fabs((double)xnew[i] - (double)xold[i]);
            change = js_max(change, d);
        }
        float *t = x; x = xnew; xnew = t;
        if (c_hist) c_hist[loop - 1] = c;
        if (ch_hist) ch_hist[loop - 1] = change;
        if (cg_hist) cg_hist[loop - 1] = its;
    }
    if (x_out) memcpy(x_out, x, 4 * (size_t)nel);
    orc_mg_destroy(mg);
    free(edofs); free(freed); free(F); free(U); free(Uprev); free(bufA); free(bufB); free(xold);
    free(xPhys); free(en); free(dc); free(dcn); free(Hs); free(dens64);
    return loop;
}

/* ========================================================================== */
/* The 2D worker: TopologyOptimizerWorker.optimize (js/optimizer-worker.js      */
/* :347-800) restricted to the hot path (no AMR, constraints or UI mesh).      */
/* ========================================================================== */
void orc_lk2d(double nu, double *Ke) {
    /* lk() :1732-1767 */
    const double k[8] = {1.0 / 2 - nu / 6, 1.0 / 8 + nu / 8, -1.0 / 4 - nu / 12, -1.0 / 8 + 3 * nu / 8,
                         -1.0 / 4 + nu / 12, -1.0 / 8 - nu / 8, nu / 6, 1.0 / 8 - 3 * nu / 8};
    static const int ord[8][8] = {{0, 1, 2, 3, 4, 5, 6, 7}, {1, 0, 7, 6, 5, 4, 3, 2}, {2, 7, 0, 5, 6, 3, 4, 1},
                                  {3, 6, 5, 0, 7, 2, 1, 4}, {4, 5, 6, 7, 0, 1, 2, 3}, {5, 4, 3, 2, 1, 0, 7, 6},
                                  {6, 3, 4, 1, 2, 7, 0, 5}, {7, 2, 1, 4, 3, 6, 5, 0}};
    for (int i = 0; i < 8; i++)
        for (int j = 0; j < 8; j++) Ke[i * 8 + j] = k[ord[i][j]] * (1 / (1 - nu * nu));
}

void orc_edofs2d(int nelx, int nely, int32_t *ed) {
    /* _precomputeEdofs2D :247-268 */
    for (int ely = 0; ely < nely; ely++)
        for (int elx = 0; elx < nelx; elx++) {
            const int o = (ely + elx * nely) * 8;
            const int n1 = (nely + 1) * elx + ely, n2 = (nely + 1) * (elx + 1) + ely;
            ed[o] = 2 * n1; ed[o + 1] = 2 * n1 + 1; ed[o + 2] = 2 * n2; ed[o + 3] = 2 * n2 + 1;
            ed[o + 4] = 2 * n2 + 2; ed[o + 5] = 2 * n2 + 3; ed[o + 6] = 2 * n1 + 2; ed[o + 7] = 2 * n1 + 3;
        }
}

/* prepareFilter :1391-1429 (triplets in (i, j, k, l) order; Hs in a Float32Array) and
 * filterSensitivities :1431-1443 (dcn in a Float32Array). */
void orc_filter_hs2d(int nelx, int nely, double rmin, float *Hs) {
    const int R = (int)floor(rmin);
    for (int e = 0; e < nelx * nely; e++) Hs[e] = 0.0f;
    for (int i = 0; i < nelx; i++)
        for (int j = 0; j < nely; j++) {
            const int e1 = i * nely + j;
            for (int k = (i - R > 0 ? i - R : 0); k <= (i + R < nelx - 1 ? i + R : nelx - 1); k++)
                for (int l = (j - R > 0 ? j - R : 0); l <= (j + R < nely - 1 ? j + R : nely - 1); l++) {
                    const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l)));
                    if (dist <= rmin) Hs[e1] = (float)((double)Hs[e1] + js_max(0, rmin - dist));
                }
        }
}
void orc_filter_sens2d(int nelx, int nely, double rmin, const float *Hs, const float *x, const float *dc, float *dcn) {
    const int R = (int)floor(rmin);
    const int nel = nelx * nely;
    for (int e = 0; e < nel; e++) dcn[e] = 0.0f;
    for (int i = 0; i < nelx; i++)
        for (int j = 0; j < nely; j++) {
            const int e1 = i * nely + j;
            for (int k = (i - R > 0 ? i - R : 0); k <= (i + R < nelx - 1 ? i + R : nelx - 1); k++)
                for (int l = (j - R > 0 ? j - R : 0); l <= (j + R < nely - 1 ? j + R : nely - 1); l++) {
                    const double dist = sqrt((double)((i - k) * (i - k) + (j - l) * (j - l)));
                    if (dist <= rmin) {
                        const int e2 = k * nely + l;
                        dcn[e1] = (float)((double)dcn[e1] + js_max(0, rmin - dist) * (double)x[e2] * (double)dc[e2]);
                    }
                }
        }
    for (int e = 0; e < nel; e++) dcn[e] = (float)((double)dcn[e] / ((double)Hs[e] * js_max(1e-3, (double)x[e])));
}

int orc_simp2d(const orc_simp2d_cfg *cfg, const float *F32, const uint8_t *fixed, const uint8_t *pres,
               const uint8_t *voidm, double *c_hist, double *ch_hist, int *cg_hist, float *x_out) {
    const int nelx = cfg->nelx, nely = cfg->nely, nel = nelx * nely, ndof = 2 * (nelx + 1) * (nely + 1);
    const double CG_TOL = 1e-8, CG_TOL_COARSE = 1e-2, EPS = 1e-12;
    const int MAX_CG = 2000;
    double Ke[64];
    orc_lk2d(cfg->nu, Ke);
    int32_t *ed = malloc(4 * (size_t)nel * 8);
    orc_edofs2d(nelx, nely, ed);
    int nfree = 0;
    for (int i = 0; i < ndof; i++) nfree += !fixed[i];
    int32_t *freed = malloc(4 * (size_t)(nfree > 0 ? nfree : 1));
    nfree = 0;
    for (int i = 0; i < ndof; i++) if (!fixed[i]) freed[nfree++] = i;
    float *x = malloc(4 * (size_t)nel), *xold = malloc(4 * (size_t)nel), *xPhys = malloc(4 * (size_t)nel);
    float *en = malloc(4 * (size_t)nel), *dc = malloc(4 * (size_t)nel), *dcn = malloc(4 * (size_t)nel);
    float *xnew = malloc(4 * (size_t)nel), *Hs = malloc(4 * (size_t)nel);
    double *ev = malloc(8 * (size_t)nel), *diag = malloc(8 * (size_t)ndof), *inv = malloc(8 * (size_t)(nfree + 1));
    int32_t *act = malloc(4 * (size_t)nel);
    double *U = malloc(8 * (size_t)ndof), *pf = malloc(8 * (size_t)ndof), *apf = malloc(8 * (size_t)ndof);
    double *Uf = malloc(8 * (size_t)(nfree + 1)), *r = malloc(8 * (size_t)(nfree + 1)), *z = malloc(8 * (size_t)(nfree + 1));
    double *p = malloc(8 * (size_t)(nfree + 1)), *Ap = malloc(8 * (size_t)(nfree + 1));
    for (int e = 0; e < nel; e++) x[e] = (float)cfg->volfrac;
    if (pres) for (int e = 0; e < nel; e++) if (pres[e]) x[e] = 1.0f;
    if (voidm) for (int e = 0; e < nel; e++) if (voidm[e]) x[e] = 0.0f;
    orc_filter_hs2d(nelx, nely, cfg->rmin, Hs);
    const double penalTarget = cfg->penal;
    const double penalStart = cfg->penal_start >= 0 ? cfg->penal_start : (penalTarget < 1.5 ? penalTarget : 1.5);
    const int contIters = cfg->continuation_iters >= 0 ? cfg->continuation_iters
                                                       : (cfg->max_iter / 3 > 20 ? cfg->max_iter / 3 : 20);
    int loop = 0;
    double change = 1.0;
    while (change > 0.01 && loop < cfg->max_iter) {
        loop++;
        memcpy(xold, x, 4 * (size_t)nel);
        const double tolerance = CG_TOL > change * CG_TOL_COARSE ? CG_TOL : change * CG_TOL_COARSE;
        const double t = (double)(loop - 1) / contIters;
        const double penal = penalStart + (penalTarget - penalStart) * (t < 1.0 ? t : 1.0);
        double beta = 1.0;
        if (cfg->use_projection) {
            beta = pow(2, floor((double)(loop - 1) / cfg->beta_interval));
            if (beta > cfg->beta_max) beta = cfg->beta_max;
        }
        const float *xp = x;
        if (cfg->use_projection) { orc_heaviside(x, nel, beta, xPhys); xp = xPhys; }
        /* FE / solveCG */
        int na = 0;
        for (int e = 0; e < nel; e++) {
            const double E = cfg->Emin + pow((double)xp[e], penal) * (cfg->E0 - cfg->Emin);
            ev[e] = E;
            if (E > cfg->Emin * 1000) act[na++] = e;
        }
        memset(diag, 0, 8 * (size_t)ndof);
        for (int ai = 0; ai < na; ai++) {
            const int e = act[ai];
            for (int i = 0; i < 8; i++) diag[ed[e * 8 + i]] = diag[ed[e * 8 + i]] + ev[e] * Ke[i * 8 + i];
        }
        for (int i = 0; i < nfree; i++) { const double d = diag[freed[i]]; inv[i] = d > 1e-30 ? 1.0 / d : 0.0; }
        for (int i = 0; i < nfree; i++) { Uf[i] = 0.0; r[i] = F32[freed[i]]; }
        double rz = 0.0;
        for (int i = 0; i < nfree; i++) { z[i] = inv[i] * r[i]; p[i] = z[i]; rz += r[i] * z[i]; }
        const int maxIter = nfree < MAX_CG ? nfree : MAX_CG;
        const double tolSq = tolerance * tolerance;
        int its = maxIter;
        for (int it = 0; it < maxIter; it++) {
            double rn = 0.0;
            for (int i = 0; i < nfree; i++) rn += r[i] * r[i];
            if (rn < tolSq) { its = it; break; }
            memset(pf, 0, 8 * (size_t)ndof);
            for (int i = 0; i < nfree; i++) pf[freed[i]] = p[i];
            orc_apply_a(Ke, ed, 8, ev, act, na, pf, apf, ndof);
            for (int i = 0; i < nfree; i++) Ap[i] = apf[freed[i]];
            double pAp = 0.0;
            for (int i = 0; i < nfree; i++) pAp += p[i] * Ap[i];
            const double alpha = rz / (pAp + EPS);
            double rzn = 0.0;
            for (int i = 0; i < nfree; i++) {
                Uf[i] += alpha * p[i];
                r[i] -= alpha * Ap[i];
                z[i] = inv[i] * r[i];
                rzn += r[i] * z[i];
            }
            const double b = rzn / (rz + EPS);
            for (int i = 0; i < nfree; i++) p[i] = z[i] + b * p[i];
            rz = rzn;
        }
        memset(U, 0, 8 * (size_t)ndof);
        for (int i = 0; i < nfree; i++) U[freed[i]] = Uf[i];
        double c = 0.0;
        for (int i = 0; i < ndof; i++) c += F32[i] * U[i];
        /* energies and sensitivities :633-653 */
        for (int e = 0; e < nel; e++) {
            double Ue[8], energy = 0.0;
            for (int i = 0; i < 8; i++) Ue[i] = U[ed[e * 8 + i]];
            for (int i = 0; i < 8; i++) {
                const double ui = Ue[i];
                for (int j = 0; j < 8; j++) energy += ui * Ke[i * 8 + j] * Ue[j];
            }
            en[e] = (float)energy;
        }
        orc_sensitivity(x, xp, en, nel, penal, cfg->E0, beta, cfg->use_projection, dc);
        orc_filter_sens2d(nelx, nely, cfg->rmin, Hs, x, dc, dcn);
        orc_oc(nel, x, cfg->volfrac, dcn, pres, voidm, xnew, NULL, NULL);
        change = 0.0;
        for (int e = 0; e < nel; e++) change = js_max(change, fabs((double)xnew[e] - (double)xold[e]));
        memcpy(x, xnew, 4 * (size_t)nel);
        c_hist[loop - 1] = c;
        ch_hist[loop - 1] = change;
        cg_hist[loop - 1] = its;
    }
    memcpy(x_out, x, 4 * (size_t)nel);
    free(ed); free(freed); free(x); free(xold); free(xPhys); free(en); free(dc); free(dcn); free(xnew); free(Hs);
    free(ev); free(diag); free(inv); free(act); free(U); free(pf); free(apf); free(Uf); free(r); free(z); free(p); free(Ap);
    return loop;
}
