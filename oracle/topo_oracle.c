/*
 * CPU restatement of GPU-TO's MGCG solve (the MATLAB MEX mgcg1) and of the
 * element-level pieces of the top3D125 design loop.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product.  The product
 * never links or calls this file; only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it.
 *
 * It restates, in this project's own code, the algorithm of
 *   Cantilever/TOP3D125MGCGCUDA/mgcg1.cu  (the GPU MEX; its semantics are
 *                                          followed where the two builds differ)
 *   Cantilever/omp/mgcg1.c                (the OpenMP MEX, compiled unmodified
 *                                          into oracle/_ref as the pin)
 * Every routine cites the reference lines it follows.  All arithmetic is FP64.
 */
#include "topo_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* grid helpers                                                              */
/* ------------------------------------------------------------------------ */

/* Local element node a -> (x,y,z) offsets (mgcg1.c:621-624). */
static const int LX[8] = {0, 1, 1, 0, 0, 1, 1, 0};
static const int LY[8] = {0, 0, 1, 1, 0, 0, 1, 1};
static const int LZ[8] = {0, 0, 0, 0, 1, 1, 1, 1};

/* Inverse of the table above: local index of offset (x,y,z). */
static inline int local_index(int x, int y, int z) { return 4 * z + (y == 0 ? x : 3 - x); }

typedef struct {
    int nx, ny, nz;    /* elements per direction */
    long nnod, ndof, nel;
} grid_t;

static grid_t make_grid(int nelx, int nely, int nelz)
{
    grid_t g;
    g.nx = nelx;
    g.ny = nely;
    g.nz = nelz;
    g.nnod = (long)(nelx + 1) * (nely + 1) * (nelz + 1);
    g.ndof = 3 * g.nnod;
    g.nel = (long)nelx * nely * nelz;
    return g;
}

static inline long node_id(const grid_t *g, int i, int j, int k)
{
    return ((long)(g->nz + 1) * (g->ny + 1)) * i + (long)(g->ny + 1) * k + j;
}

static inline long elem_id(const grid_t *g, int i, int j, int k)
{
    return ((long)g->nz * g->ny) * i + (long)g->ny * k + j;
}

/* ------------------------------------------------------------------------ */
/* element matrices (mgcg1.c:1370-1533, mgcg1.cu:2000-2040)                  */
/* ------------------------------------------------------------------------ */

/* Strain-displacement matrix at natural point (s,e,t) for an hx*hy*hz hex,
 * Voigt rows xx, yy, zz, xy, yz, zx (the row order of mgcg1.c:1421-1531). */
static void strain_matrix(double s, double e, double t, double hx, double hy, double hz,
                          double B[6][24])
{
    memset(B, 0, sizeof(double) * 6 * 24);
    const double nat[3] = {s, e, t};
    for (int a = 0; a < 8; ++a) {
        const double xa = 2 * LX[a] - 1, ya = 2 * LY[a] - 1, za = 2 * LZ[a] - 1;
        const double fx = 1 + xa * nat[0], fy = 1 + ya * nat[1], fz = 1 + za * nat[2];
        /* d/dx of (1/8) fx fy fz, with dx = (hx/2) ds */
        const double dx = 0.25 * xa * fy * fz / hx;
        const double dy = 0.25 * ya * fx * fz / hy;
        const double dz = 0.25 * za * fx * fy / hz;
        B[0][3 * a + 0] = dx;
        B[1][3 * a + 1] = dy;
        B[2][3 * a + 2] = dz;
        B[3][3 * a + 0] = dy;
        B[3][3 * a + 1] = dx;
        B[4][3 * a + 1] = dz;
        B[4][3 * a + 2] = dy;
        B[5][3 * a + 0] = dz;
        B[5][3 * a + 2] = dx;
    }
}

/* Isotropic elasticity matrix for E = 1 (mgcg1.c:1390-1418 defD). */
static void elasticity(double nu, double D[6][6])
{
    memset(D, 0, sizeof(double) * 36);
    const double c = 1.0 / ((1.0 + nu) * (1.0 - 2.0 * nu));
    for (int p = 0; p < 3; ++p)
        for (int q = 0; q < 3; ++q) D[p][q] = c * (p == q ? 1.0 - nu : nu);
    for (int p = 3; p < 6; ++p) D[p][p] = c * (1.0 - 2.0 * nu) / 2.0;
}

void or_hex8_gauss_parts(double nu, double hx, double hy, double hz, double *Kg)
{
    const double gp[2] = {-1.0 / sqrt(3.0), 1.0 / sqrt(3.0)};
    const double w = hx * hy * hz / 8.0; /* |J| times the unit Gauss weight */
    double D[6][6], B[6][24], DB[6][24];
    elasticity(nu, D);
    for (int ix = 0; ix < 2; ++ix)
        for (int iz = 0; iz < 2; ++iz)
            for (int iy = 0; iy < 2; ++iy) {
                const int g = 4 * ix + 2 * iz + iy;
                strain_matrix(gp[ix], gp[iy], gp[iz], hx, hy, hz, B);
                for (int p = 0; p < 6; ++p)
                    for (int n = 0; n < 24; ++n) {
                        double acc = 0.0;
                        for (int q = 0; q < 6; ++q) acc += D[p][q] * B[q][n];
                        DB[p][n] = acc;
                    }
                double *K = Kg + (long)g * 576;
                /* symmetric by construction: compute the lower triangle, mirror */
                for (int m = 0; m < 24; ++m)
                    for (int n = 0; n <= m; ++n) {
                        double acc = 0.0;
                        for (int p = 0; p < 6; ++p) acc += B[p][m] * DB[p][n];
                        K[m * 24 + n] = K[n * 24 + m] = w * acc;
                    }
            }
}

void or_hex8_stiffness(double nu, double hx, double hy, double hz, double *Ke)
{
    double Kg[8 * 576];
    or_hex8_gauss_parts(nu, hx, hy, hz, Kg);
    for (int m = 0; m < 576; ++m) {
        double acc = 0.0;
        for (int g = 0; g < 8; ++g) acc += Kg[g * 576 + m];
        Ke[m] = acc;
    }
}

/* ------------------------------------------------------------------------ */
/* operators                                                                 */
/* ------------------------------------------------------------------------ */

/* A level's operator: either CX-scaled Ke (the fine level) or one 24x24
 * element matrix per element (coarse levels, full storage). */
typedef struct {
    grid_t g;
    const double *Ke;  /* fine level: 576 */
    const double *CX;  /* fine level: nel */
    double *Ael;       /* coarse level: nel*576 */
} op_t;

static inline const double *elem_matrix(const op_t *op, long e, double *scratch)
{
    if (op->Ael) return op->Ael + e * 576;
    const double c = op->CX[e];
    for (int m = 0; m < 576; ++m) scratch[m] = c * op->Ke[m];
    return scratch;
}

/* r = f - A u, or r = A u when f == NULL.  Node-centred gather over the
 * up-to-8 elements around each node (mgcg1.cu:941-997, 1208-1324). */
static void op_residual(const op_t *op, const double *f, const double *u, double *r)
{
    const grid_t *g = &op->g;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i <= g->nx; ++i)
        for (int k = 0; k <= g->nz; ++k)
            for (int j = 0; j <= g->ny; ++j) {
                const long n = node_id(g, i, j, k);
                double acc[3] = {0.0, 0.0, 0.0};
                for (int ei = i - 1; ei <= i; ++ei) {
                    if (ei < 0 || ei >= g->nx) continue;
                    for (int ek = k - 1; ek <= k; ++ek) {
                        if (ek < 0 || ek >= g->nz) continue;
                        for (int ej = j - 1; ej <= j; ++ej) {
                            if (ej < 0 || ej >= g->ny) continue;
                            const long e = elem_id(g, ei, ej, ek);
                            const int a = local_index(i - ei, j - ej, k - ek);
                            const double *K = op->Ael ? op->Ael + e * 576 : op->Ke;
                            const double c = op->Ael ? 1.0 : op->CX[e];
                            double t[3] = {0.0, 0.0, 0.0};
                            for (int b = 0; b < 8; ++b) {
                                const long nb = node_id(g, ei + LX[b], ej + LY[b], ek + LZ[b]);
                                for (int q = 0; q < 3; ++q) {
                                    const double ub = u[3 * nb + q];
                                    for (int d = 0; d < 3; ++d)
                                        t[d] += K[(3 * a + d) * 24 + 3 * b + q] * ub;
                                }
                            }
                            for (int d = 0; d < 3; ++d) acc[d] += c * t[d];
                        }
                    }
                }
                for (int d = 0; d < 3; ++d)
                    r[3 * n + d] = f ? f[3 * n + d] - acc[d] : acc[d];
            }
}

void or_apply_fine(const double *Ke, const double *CX, const double *u, double *r,
                   int nelx, int nely, int nelz)
{
    op_t op = {make_grid(nelx, nely, nelz), Ke, CX, NULL};
    op_residual(&op, NULL, u, r);
}

/* Operator diagonal (mgcg1.cu:1404-1487 prepADc / prepAD0c). */
static void op_diagonal(const op_t *op, double *diag)
{
    const grid_t *g = &op->g;
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i <= g->nx; ++i)
        for (int k = 0; k <= g->nz; ++k)
            for (int j = 0; j <= g->ny; ++j) {
                const long n = node_id(g, i, j, k);
                double acc[3] = {0.0, 0.0, 0.0};
                for (int ei = i - 1; ei <= i; ++ei) {
                    if (ei < 0 || ei >= g->nx) continue;
                    for (int ek = k - 1; ek <= k; ++ek) {
                        if (ek < 0 || ek >= g->nz) continue;
                        for (int ej = j - 1; ej <= j; ++ej) {
                            if (ej < 0 || ej >= g->ny) continue;
                            const long e = elem_id(g, ei, ej, ek);
                            const int a = local_index(i - ei, j - ej, k - ek);
                            for (int d = 0; d < 3; ++d) {
                                const int m = 3 * a + d;
                                acc[d] += op->Ael ? op->Ael[e * 576 + m * 24 + m]
                                                  : op->CX[e] * op->Ke[m * 24 + m];
                            }
                        }
                    }
                }
                for (int d = 0; d < 3; ++d) diag[3 * n + d] = acc[d];
            }
}

/* Level-1 operator: 2h element whose Gauss point g is weighted by the
 * density of the fine sub-element containing it (mgcg1.cu:2042-2070 coarseAe2c). */
static void build_quadrature_level(const grid_t *gc, const double *CXfine, const double *Kg,
                                   double *Ael)
{
    const grid_t gf = make_grid(2 * gc->nx, 2 * gc->ny, 2 * gc->nz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < gc->nx; ++i)
        for (int k = 0; k < gc->nz; ++k)
            for (int j = 0; j < gc->ny; ++j) {
                double *A = Ael + elem_id(gc, i, j, k) * 576;
                for (int m = 0; m < 576; ++m) A[m] = 0.0;
                for (int ix = 0; ix < 2; ++ix)
                    for (int iz = 0; iz < 2; ++iz)
                        for (int iy = 0; iy < 2; ++iy) {
                            const double c = CXfine[elem_id(&gf, 2 * i + ix, 2 * j + iy, 2 * k + iz)];
                            const double *K = Kg + (4 * ix + 2 * iz + iy) * 576;
                            for (int m = 0; m < 576; ++m) A[m] += c * K[m];
                        }
            }
}

/* Trilinear prolongation weight of the coarse node at local (ax,ay,az) onto
 * the point (px,py,pz) in {0,1,2}^3 of the fine 3x3x3 node patch (the
 * 1, 1/2, 1/4, 1/8 weights of mgcg1.c:1093-1100 and top3D125mgcg.m:248-280). */
static inline double tri_weight(int ax, int ay, int az, int px, int py, int pz)
{
    const double wx = 1.0 - 0.5 * abs(px - 2 * ax);
    const double wy = 1.0 - 0.5 * abs(py - 2 * ay);
    const double wz = 1.0 - 0.5 * abs(pz - 2 * az);
    return (wx > 0 && wy > 0 && wz > 0) ? wx * wy * wz : 0.0;
}

/* Galerkin coarse element matrices P^T A_fine P over each 2x2x2 block of
 * fine elements (mgcg1.cu:1678-1743 coarseAe3c). */
static void build_galerkin_level(const grid_t *gc, const double *Afine, double *Ael)
{
    const grid_t gf = make_grid(2 * gc->nx, 2 * gc->ny, 2 * gc->nz);
    /* Pc[c][b][a]: weight of coarse local node a on child c's local node b */
    static double Pc[8][8][8];
    static int ready = 0;
#pragma omp critical(pc_init)
    if (!ready) {
        for (int c = 0; c < 8; ++c)
            for (int b = 0; b < 8; ++b)
                for (int a = 0; a < 8; ++a)
                    Pc[c][b][a] = tri_weight(LX[a], LY[a], LZ[a], LX[c] + LX[b], LY[c] + LY[b],
                                             LZ[c] + LZ[b]);
        ready = 1;
    }
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < gc->nx; ++i)
        for (int k = 0; k < gc->nz; ++k)
            for (int j = 0; j < gc->ny; ++j) {
                double *A = Ael + elem_id(gc, i, j, k) * 576;
                double T[24 * 24];
                for (int m = 0; m < 576; ++m) A[m] = 0.0;
                for (int c = 0; c < 8; ++c) {
                    const double *K =
                        Afine + elem_id(&gf, 2 * i + LX[c], 2 * j + LY[c], 2 * k + LZ[c]) * 576;
                    /* T = K Pc  (rows: child dofs, cols: coarse dofs) */
                    for (int bp = 0; bp < 24; ++bp)
                        for (int a = 0; a < 8; ++a)
                            for (int q = 0; q < 3; ++q) {
                                double acc = 0.0;
                                for (int b = 0; b < 8; ++b)
                                    acc += K[bp * 24 + 3 * b + q] * Pc[c][b][a];
                                T[bp * 24 + 3 * a + q] = acc;
                            }
                    /* A += Pc^T T */
                    for (int a = 0; a < 8; ++a)
                        for (int p = 0; p < 3; ++p)
                            for (int n = 0; n < 24; ++n) {
                                double acc = 0.0;
                                for (int b = 0; b < 8; ++b)
                                    acc += Pc[c][b][a] * T[(3 * b + p) * 24 + n];
                                A[(3 * a + p) * 24 + n] += acc;
                            }
                }
                /* exact symmetry, as the packed storage of mgcg1.cu implies */
                for (int m = 0; m < 24; ++m)
                    for (int n = 0; n < m; ++n) {
                        const double s = 0.5 * (A[m * 24 + n] + A[n * 24 + m]);
                        A[m * 24 + n] = A[n * 24 + m] = s;
                    }
            }
}

/* Dirichlet penalty on the coarsest element matrices (mgcg1.cu:1368-1402
 * CorrCsAc, same as mgcg1.c:918-953).  For a fixed dof at node (i,j,k) and
 * each element (i+di, j+dj, k+dk), di,dj,dk in {-1,0}, the reference writes
 * 1e10 on the diagonal of the element-local node at offset (-di, 1+dj, -dk):
 * its lookup table is mirrored in y relative to the true local index
 * (-di, -dj, -dk).  The same entries are penalised here. */
static void coarsest_penalty(const grid_t *g, const unsigned char *fixmask, double *Ael)
{
    for (int i = 0; i <= g->nx; ++i)
        for (int k = 0; k <= g->nz; ++k)
            for (int j = 0; j <= g->ny; ++j) {
                const long n = node_id(g, i, j, k);
                for (int d = 0; d < 3; ++d) {
                    if (!(fixmask[n] & (1u << d))) continue;
                    for (int di = -1; di <= 0; ++di)
                        for (int dk = -1; dk <= 0; ++dk)
                            for (int dj = -1; dj <= 0; ++dj) {
                                const int ei = i + di, ej = j + dj, ek = k + dk;
                                if (ei < 0 || ei >= g->nx || ej < 0 || ej >= g->ny || ek < 0 ||
                                    ek >= g->nz)
                                    continue;
                                const int a = local_index(-di, 1 + dj, -dk);
                                const int m = 3 * a + d;
                                Ael[elem_id(g, ei, ej, ek) * 576 + m * 24 + m] = 1e10;
                            }
                }
            }
}

/* Dense assembly of the coarsest operator (mgcg1.cu:1747-1806 assembAc). */
static void assemble_dense(const grid_t *g, const double *Ael, double *AQ)
{
    const long n = g->ndof;
    memset(AQ, 0, sizeof(double) * n * n);
    for (int i = 0; i < g->nx; ++i)
        for (int k = 0; k < g->nz; ++k)
            for (int j = 0; j < g->ny; ++j) {
                const double *A = Ael + elem_id(g, i, j, k) * 576;
                for (int a = 0; a < 8; ++a) {
                    const long na = node_id(g, i + LX[a], j + LY[a], k + LZ[a]);
                    for (int b = 0; b < 8; ++b) {
                        const long nb = node_id(g, i + LX[b], j + LY[b], k + LZ[b]);
                        for (int p = 0; p < 3; ++p)
                            for (int q = 0; q < 3; ++q)
                                AQ[(3 * na + p) * n + 3 * nb + q] += A[(3 * a + p) * 24 + 3 * b + q];
                    }
                }
            }
}

/* Textbook Cholesky A = L L^T, L stored in the lower triangle (column-by-
 * column, inner products), returns 0 or the 1-based index of a bad pivot. */
static int cholesky(long n, double *A)
{
    for (long j = 0; j < n; ++j) {
        double s = A[j * n + j];
        for (long k = 0; k < j; ++k) s -= A[j * n + k] * A[j * n + k];
        if (!(s > 0.0)) return (int)(j + 1);
        const double d = sqrt(s);
        A[j * n + j] = d;
#pragma omp parallel for schedule(static) if (n - j > 256)
        for (long i = j + 1; i < n; ++i) {
            double t = A[i * n + j];
            for (long k = 0; k < j; ++k) t -= A[i * n + k] * A[j * n + k];
            A[i * n + j] = t / d;
        }
    }
    return 0;
}

static void cholesky_solve(long n, const double *L, const double *b, double *x)
{
    for (long i = 0; i < n; ++i) {
        double s = b[i];
        for (long k = 0; k < i; ++k) s -= L[i * n + k] * x[k];
        x[i] = s / L[i * n + i];
    }
    for (long i = n - 1; i >= 0; --i) {
        double s = x[i];
        for (long k = i + 1; k < n; ++k) s -= L[k * n + i] * x[k];
        x[i] = s / L[i * n + i];
    }
}

/* Full-weighting restriction F_c = P^T R_f (mgcg1.cu:792-831 rstrFc). */
static void restrict_fw(const grid_t *gc, const double *rf, double *fc)
{
    const grid_t gf = make_grid(2 * gc->nx, 2 * gc->ny, 2 * gc->nz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i <= gc->nx; ++i)
        for (int k = 0; k <= gc->nz; ++k)
            for (int j = 0; j <= gc->ny; ++j) {
                double acc[3] = {0.0, 0.0, 0.0};
                for (int di = -1; di <= 1; ++di) {
                    const int fi = 2 * i + di;
                    if (fi < 0 || fi > gf.nx) continue;
                    for (int dk = -1; dk <= 1; ++dk) {
                        const int fk = 2 * k + dk;
                        if (fk < 0 || fk > gf.nz) continue;
                        for (int dj = -1; dj <= 1; ++dj) {
                            const int fj = 2 * j + dj;
                            if (fj < 0 || fj > gf.ny) continue;
                            const double w = ldexp(1.0, -(abs(di) + abs(dj) + abs(dk)));
                            const long nf = node_id(&gf, fi, fj, fk);
                            for (int d = 0; d < 3; ++d) acc[d] += w * rf[3 * nf + d];
                        }
                    }
                }
                const long nc = node_id(gc, i, j, k);
                for (int d = 0; d < 3; ++d) fc[3 * nc + d] = acc[d];
            }
}

/* u_f += P u_c, trilinear (mgcg1.cu:1587-1641 interpc). */
static void prolong_add(const grid_t *gf, const double *uc, double *uf)
{
    const grid_t gc = make_grid(gf->nx / 2, gf->ny / 2, gf->nz / 2);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i <= gf->nx; ++i)
        for (int k = 0; k <= gf->nz; ++k)
            for (int j = 0; j <= gf->ny; ++j) {
                const int ci[2] = {i / 2, (i + 1) / 2};
                const int cj[2] = {j / 2, (j + 1) / 2};
                const int ck[2] = {k / 2, (k + 1) / 2};
                const int ni = (i & 1) ? 2 : 1, nj = (j & 1) ? 2 : 1, nk = (k & 1) ? 2 : 1;
                const double w = 1.0 / (ni * nj * nk);
                double acc[3] = {0.0, 0.0, 0.0};
                for (int a = 0; a < ni; ++a)
                    for (int c = 0; c < nk; ++c)
                        for (int b = 0; b < nj; ++b) {
                            const long nc = node_id(&gc, ci[a], cj[b], ck[c]);
                            for (int d = 0; d < 3; ++d) acc[d] += uc[3 * nc + d];
                        }
                const long nf = node_id(gf, i, j, k);
                for (int d = 0; d < 3; ++d) uf[3 * nf + d] += w * acc[d];
            }
}

static void zero_fixed(const grid_t *g, const unsigned char *mask, double *v)
{
    for (long n = 0; n < g->nnod; ++n)
        if (mask[n])
            for (int d = 0; d < 3; ++d)
                if (mask[n] & (1u << d)) v[3 * n + d] = 0.0;
}

static double dot(long n, const double *a, const double *b)
{
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
}

/* ------------------------------------------------------------------------ */
/* multigrid hierarchy and V-cycle (mgcg1.cu:326-651)                        */
/* ------------------------------------------------------------------------ */

typedef struct {
    int nl;
    or_opts o;
    grid_t g[16];
    op_t op[16];
    unsigned char *mask[16];
    double *diag[16], *U[16], *F[16], *R[16];
    double *Ael[16];
    double *CXr[16];  /* mgcg9 hierarchy: re-discretised element scales */
    double *L;  /* coarsest Cholesky factor */
} mg_t;

static void mg_free(mg_t *mg)
{
    for (int l = 0; l < mg->nl; ++l) {
        free(mg->mask[l]);
        free(mg->diag[l]);
        free(mg->R[l]);
        if (l > 0) {
            free(mg->U[l]);
            free(mg->F[l]);
            free(mg->Ael[l]);
            free(mg->CXr[l]);
        }
    }
    free(mg->L);
}

/* Fixed-dof bitmask per node from the 1-based dof list (mgcg1.cu:1326-1331
 * ZeroBCc).  Coarse levels keep the dofs of fine nodes with even (i,j,k)
 * (mgcg1.cu:747-790 rstrFDc). */
static int mg_build(mg_t *mg, const double *Ke0, const double *CX, const double *fixed1b, int nfd,
                    int nelx, int nely, int nelz, int nl, const or_opts *o)
{
    memset(mg, 0, sizeof(*mg));
    mg->nl = nl;
    mg->o = *o;
    for (int l = 0; l < nl; ++l) mg->g[l] = make_grid(nelx >> l, nely >> l, nelz >> l);
    mg->mask[0] = calloc(mg->g[0].nnod, 1);
    for (int n = 0; n < nfd; ++n) {
        const long dof = (long)fixed1b[n] - 1;
        if (dof < 0 || dof >= mg->g[0].ndof) return 1;
        mg->mask[0][dof / 3] |= (unsigned char)(1u << (dof % 3));
    }
    for (int l = 1; l < nl; ++l) {
        const grid_t *gc = &mg->g[l], *gf = &mg->g[l - 1];
        mg->mask[l] = calloc(gc->nnod, 1);
        for (int i = 0; i <= gc->nx; ++i)
            for (int k = 0; k <= gc->nz; ++k)
                for (int j = 0; j <= gc->ny; ++j)
                    mg->mask[l][node_id(gc, i, j, k)] =
                        mg->mask[l - 1][node_id(gf, 2 * i, 2 * j, 2 * k)];
    }
    double Kg[8 * 576];
    or_hex8_gauss_parts(o->nu, 2.0, 2.0, 2.0, Kg);
    for (int l = 0; l < nl; ++l) {
        grid_t *g = &mg->g[l];
        mg->op[l].g = *g;
        if (l == 0) {
            mg->op[0].Ke = Ke0;
            mg->op[0].CX = CX;
        } else if (o->coarse) {
            /* mgcg9.cu:753-781 formCXc: CX_l = 2 * mean of the 8 children */
            const grid_t *gf = &mg->g[l - 1];
            const double *CXf = (l == 1) ? CX : mg->CXr[l - 1];
            mg->CXr[l] = malloc(sizeof(double) * g->nel);
            for (int i = 0; i < g->nx; ++i)
                for (int k = 0; k < g->nz; ++k)
                    for (int j = 0; j < g->ny; ++j) {
                        double s = 0.0;
                        for (int a = 0; a < 2; ++a)
                            for (int b = 0; b < 2; ++b)
                                for (int c = 0; c < 2; ++c) s += CXf[elem_id(gf, 2 * i + a, 2 * j + c, 2 * k + b)];
                        mg->CXr[l][elem_id(g, i, j, k)] = 2.0 * (s / 8.0);
                    }
            mg->op[l].Ke = Ke0;
            mg->op[l].CX = mg->CXr[l];
            mg->U[l] = calloc(g->ndof, sizeof(double));
            mg->F[l] = calloc(g->ndof, sizeof(double));
        } else {
            mg->Ael[l] = malloc(sizeof(double) * 576 * g->nel);
            if (l == 1)
                build_quadrature_level(g, CX, Kg, mg->Ael[l]);
            else
                build_galerkin_level(g, mg->Ael[l - 1], mg->Ael[l]);
            mg->op[l].Ael = mg->Ael[l];
            mg->U[l] = calloc(g->ndof, sizeof(double));
            mg->F[l] = calloc(g->ndof, sizeof(double));
        }
        mg->R[l] = calloc(g->ndof, sizeof(double));
        mg->diag[l] = calloc(g->ndof, sizeof(double));
        if (l == nl - 1 && o->coarse) {
            if (g->ndof >= 20000) return 2;
            /* mgcg9.cu:1243-1300 assembAQc and :1005-1028 CorrCsAQc: the
             * re-discretised operator, then zero rows/columns and 1e10 on
             * every fixed dof */
            const double *CXc = (l == 0) ? CX : mg->CXr[l];
            double *Ael = malloc(sizeof(double) * 576 * g->nel);
            for (long e = 0; e < g->nel; ++e)
                for (int m = 0; m < 576; ++m) Ael[e * 576 + m] = CXc[e] * Ke0[m];
            mg->L = malloc(sizeof(double) * g->ndof * g->ndof);
            assemble_dense(g, Ael, mg->L);
            free(Ael);
            const long N = g->ndof;
            for (long r = 0; r < N; ++r)
                for (long q = 0; q < N; ++q) {
                    const int fr = (mg->mask[l][r / 3] >> (r % 3)) & 1, fq = (mg->mask[l][q / 3] >> (q % 3)) & 1;
                    if (fr || fq) mg->L[r * N + q] = (r == q) ? 1e10 : 0.0;
                }
            if (cholesky(g->ndof, mg->L)) return 3;
        } else if (l == nl - 1) {
            if (l > 0) coarsest_penalty(g, mg->mask[l], mg->Ael[l]);
            if (g->ndof > 20000) return 2;
            mg->L = malloc(sizeof(double) * g->ndof * g->ndof);
            if (l == 0) {
                /* single-level hierarchy: dense fine operator with identity rows
                 * for fixed dofs (the reference would run plain CG here) */
                double *Ael = malloc(sizeof(double) * 576 * g->nel);
                for (long e = 0; e < g->nel; ++e)
                    for (int m = 0; m < 576; ++m) Ael[e * 576 + m] = CX[e] * Ke0[m];
                coarsest_penalty(g, mg->mask[0], Ael);
                assemble_dense(g, Ael, mg->L);
                free(Ael);
            } else {
                assemble_dense(g, mg->Ael[l], mg->L);
            }
            if (cholesky(g->ndof, mg->L)) return 3;
        }
        op_diagonal(&mg->op[l], mg->diag[l]);
    }
    return 0;
}

static void jacobi_update(long n, double omega, const double *diag, const double *r, double *u)
{
    /* U = (1-w) U + w (R + D U)/D, in the reference's form (mgcg1.cu:1199-1206) */
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; ++i) u[i] = (1.0 - omega) * u[i] + omega * (r[i] + diag[i] * u[i]) / diag[i];
}

static void mg_vcycle(mg_t *mg, double *f0, double *u0)
{
    const int nl = mg->nl;
    const or_opts *o = &mg->o;
    mg->F[0] = f0;
    mg->U[0] = u0;
    for (int l = 0; l < nl; ++l) {
        const grid_t *g = &mg->g[l];
        if (l > 0) {
            restrict_fw(g, mg->R[l - 1], mg->F[l]);
            zero_fixed(g, mg->mask[l], mg->F[l]);
        }
        if (l < nl - 1) {
            const double *D = mg->diag[l];
            double *U = mg->U[l], *F = mg->F[l], *R = mg->R[l];
#pragma omp parallel for schedule(static)
            for (long i = 0; i < g->ndof; ++i) U[i] = o->prerelax * F[i] / D[i];
            for (int s = 0; s < o->nswp; ++s) {
                op_residual(&mg->op[l], F, U, R);
                zero_fixed(g, mg->mask[l], R);
                jacobi_update(g->ndof, o->omega, D, R, U);
            }
            op_residual(&mg->op[l], F, U, R);
            zero_fixed(g, mg->mask[l], R);
        } else {
            cholesky_solve(g->ndof, mg->L, mg->F[l], mg->U[l]);
        }
    }
    for (int l = nl - 2; l >= 0; --l) {
        const grid_t *g = &mg->g[l];
        double *U = mg->U[l], *F = mg->F[l], *R = mg->R[l];
        prolong_add(g, mg->U[l + 1], U);
        zero_fixed(g, mg->mask[l], U);
        for (int s = 0; s < o->nswp; ++s) {
            op_residual(&mg->op[l], F, U, R);
            zero_fixed(g, mg->mask[l], R);
            jacobi_update(g->ndof, o->omega, mg->diag[l], R, U);
        }
    }
}

void or_default_opts(or_opts *o)
{
    o->nswp = 3;
    o->omega = 0.48;
    o->prerelax = 0.7;
    o->nu = 0.3;
    o->coarse = 0;
}

static int check_args(int nelx, int nely, int nelz, int nl)
{
    if (nl < 1 || nl > 15 || nelx < 1 || nely < 1 || nelz < 1) return 1;
    const int m = 1 << (nl - 1);
    if (nelx % m || nely % m || nelz % m) return 1;
    return 0;
}

int or_vcycle_apply(const double *Ke0, const double *CX, const double *fixed1b, int nfd,
                    int nelx, int nely, int nelz, int nl, const or_opts *opts,
                    const double *r, double *z)
{
    or_opts o;
    if (!opts) or_default_opts(&o);
    else o = *opts;
    if (check_args(nelx, nely, nelz, nl)) return 1;
    mg_t mg;
    int st = mg_build(&mg, Ke0, CX, fixed1b, nfd, nelx, nely, nelz, nl, &o);
    if (!st) {
        const long ndof = mg.g[0].ndof;
        double *f = malloc(sizeof(double) * ndof);
        memcpy(f, r, sizeof(double) * ndof);
        mg_vcycle(&mg, f, z);
        free(f);
    }
    mg_free(&mg);
    return st;
}

int or_mgcg1(const double *Ke0, const double *F, double *U, const double *CX,
             const double *fixed1b, int nfd, int nelx, int nely, int nelz, int nl,
             double tol, int maxit, const or_opts *opts, double *relres, int *nit,
             double *res_history)
{
    or_opts o;
    if (!opts) or_default_opts(&o);
    else o = *opts;
    if (check_args(nelx, nely, nelz, nl) || maxit < 0) return 1;
    mg_t mg;
    int st = mg_build(&mg, Ke0, CX, fixed1b, nfd, nelx, nely, nelz, nl, &o);
    if (st) {
        mg_free(&mg);
        return st;
    }
    const grid_t *g = &mg.g[0];
    const long n = g->ndof;
    double *R = malloc(sizeof(double) * n), *P = malloc(sizeof(double) * n);
    double *Q = malloc(sizeof(double) * n), *Z = malloc(sizeof(double) * n);

    /* mgcg1.cu:235-286 */
    memset(U, 0, sizeof(double) * n);
    memcpy(R, F, sizeof(double) * n);
    const double res0 = sqrt(dot(n, F, F));
    mg_vcycle(&mg, R, P);
    memcpy(Z, P, sizeof(double) * n);
    double rho_p = dot(n, R, Z);
    double rel = 1.0;
    int it;
    for (it = 0; it < maxit; ++it) {
        op_residual(&mg.op[0], NULL, P, Q);
        zero_fixed(g, mg.mask[0], Q);
        const double alpha = rho_p / dot(n, P, Q);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) {
            U[i] += alpha * P[i];
            R[i] -= alpha * Q[i];
        }
        mg_vcycle(&mg, R, Z);
        const double rho = dot(n, R, Z);
        const double beta = rho / rho_p;
#pragma omp parallel for schedule(static)
        for (long i = 0; i < n; ++i) P[i] = Z[i] + beta * P[i];
        rho_p = rho;
        rel = sqrt(dot(n, R, R)) / res0;
        if (res_history) res_history[it] = rel;
        if (rel < tol) break;
    }
    for (long i = 1; i < n; i += 3) U[i] = -U[i];
    *relres = rel;
    *nit = it;
    free(R);
    free(P);
    free(Q);
    free(Z);
    mg_free(&mg);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* design-loop pieces                                                        */
/* ------------------------------------------------------------------------ */

void or_element_energy(const double *Ke, const double *U, double *ce, int nelx, int nely,
                       int nelz)
{
    const grid_t g = make_grid(nelx, nely, nelz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nelx; ++i)
        for (int k = 0; k < nelz; ++k)
            for (int j = 0; j < nely; ++j) {
                double ue[24];
                for (int a = 0; a < 8; ++a) {
                    const long na = node_id(&g, i + LX[a], j + LY[a], k + LZ[a]);
                    for (int d = 0; d < 3; ++d) ue[3 * a + d] = U[3 * na + d];
                }
                double s = 0.0;
                for (int m = 0; m < 24; ++m) {
                    double t = 0.0;
                    for (int q = 0; q < 24; ++q) t += Ke[m * 24 + q] * ue[q];
                    s += ue[m] * t;
                }
                ce[elem_id(&g, i, j, k)] = s;
            }
}

/* MATLAB 'symmetric' padding: mirror including the edge sample. */
static inline int mirror(int i, int n)
{
    while (i < 0 || i >= n) {
        if (i < 0) i = -1 - i;
        if (i >= n) i = 2 * n - 1 - i;
    }
    return i;
}

double or_filter3d(const double *in, double *out, int nelx, int nely, int nelz, double rmin)
{
    const int R = (int)ceil(rmin) - 1;
    const int W = 2 * R + 1;
    double *h = malloc(sizeof(double) * W * W * W);
    double hsum = 0.0;
    for (int a = -R; a <= R; ++a)
        for (int b = -R; b <= R; ++b)
            for (int c = -R; c <= R; ++c) {
                const double v = rmin - sqrt((double)(a * a + b * b + c * c));
                const double w = v > 0 ? v : 0.0;
                h[((a + R) * W + (b + R)) * W + (c + R)] = w;
                hsum += w;
            }
    const grid_t g = make_grid(nelx, nely, nelz);
#pragma omp parallel for collapse(2) schedule(static)
    for (int i = 0; i < nelx; ++i)
        for (int k = 0; k < nelz; ++k)
            for (int j = 0; j < nely; ++j) {
                double acc = 0.0;
                for (int a = -R; a <= R; ++a) {
                    const int ii = mirror(i + a, nelx);
                    for (int c = -R; c <= R; ++c) {
                        const int kk = mirror(k + c, nelz);
                        for (int b = -R; b <= R; ++b) {
                            const int jj = mirror(j + b, nely);
                            acc += h[((a + R) * W + (b + R)) * W + (c + R)] * in[elem_id(&g, ii, jj, kk)];
                        }
                    }
                }
                out[elem_id(&g, i, j, k)] = acc;
            }
    free(h);
    return hsum;
}
