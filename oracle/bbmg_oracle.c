/*
 * bbmg_oracle.c -- CPU restatement of NGA2's black-box multigrid solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle and the timed CPU
 * baseline.  Only tests/, __graft_entry__.smoke() and bench.py's CPU legs load
 * it; the product library (nga2_b200/) never links or calls it.
 *
 * It restates src/solver/bbmg_class.f90 (Dendy black-box MG with Shapira's
 * lumping, 8-colour Gauss-Seidel, Galerkin RAP, V/W cycle, optional PCG) for a
 * single rank, where every MPI halo exchange (vsync/msync, bbmg_class.f90:
 * 1388-1724) reduces to the periodic copy of the one-cell overlap and every
 * MPI_ALLREDUCE reduces to the local value.  The ILS parameterisation and the
 * 7-point -> 27-point operator scatter follow src/solver/ils_class.f90:184-198
 * and 244-256.  LAPACK DGESV (bbmg_class.f90:913) is restated as an unblocked
 * LU with row partial pivoting (first maximum on ties) followed by the
 * column-oriented unit-lower and upper triangular solves.  With
 * pin_singular = 0 the DGESV behaviour is kept exactly (a pivot that is
 * exactly zero returns the right-hand side unchanged; a round-off pivot is
 * divided by).  With pin_singular = 1 (the default, and what the CUDA solver
 * does) the unknown of a round-off pivot is set to zero instead; this only
 * changes singular (periodic / all-Neumann) coarse problems, where DGESV's
 * division injects an arbitrary null-space component.
 *
 * Parity status: the reference has no tests or golden vectors for this path
 * and cannot be compiled here (Fortran + MPI + LAPACK), so the restatement is
 * pinned by known answers instead: the exact FFT solution of the periodic
 * constant-coefficient problem, the algebraic identities R = P^T and
 * A_c = R A P, and scipy's LAPACK dgesv on the coarse matrix.
 *
 * Data layout mirrors the reference: per level, arrays span the one-cell
 * overlap (Fortran i = 0..nx+1, i fastest), operators are stored
 * array-of-structures with the 3x3x3 stencil contiguous per cell
 * (opr(-1:1,-1:1,-1:1,i,j,k)), prolongation with its 2x2x2 weights contiguous.
 * Floating-point sums run in the reference's column-major element order.
 */
#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_EPS DBL_EPSILON /* epsilon(1.0_WP), bbmg_class.f90:880 */
#define ORC_MAXLVL 32

typedef struct {
    int nx, ny, nz;       /* interior sizes (imin=1 .. imax=nx) */
    int nxo, nyo, nzo;    /* sizes with the one-cell overlap */
    long ncell, ncello;
    double *opr;    /* 27 per cell */
    double *c2f;    /* 8 per cell, levels < nlvl */
    double *f2c;    /* 27 per cell, levels > 1 */
    double *oprc2f; /* 27 per cell, levels < nlvl */
    double *v, *f, *r;
} olvl;

typedef struct {
    int xper, yper, zper;
    int nlvl, nlvl_alloc;
    olvl lvl[ORC_MAXLVL + 1]; /* 1-based like the reference */
    /* parameters (bbmg_class.f90:91-98) */
    double max_res;
    int max_ite, ncycle, relax_pre, relax_post, ncell_coarsest;
    int use_direct_solve, use_krylov;
    /* direct solver (bbmg_class.f90:80-83) */
    int np, lu_info;
    int pin_singular; /* 1: unknowns with a round-off pivot are set to zero */
    int *piv, *pinned;
    double *OP, *LU, *rhs;
    /* solver information */
    double my_res0, my_res;
    int my_ite;
    /* Krylov work vectors (bbmg_class.f90:105-106) */
    double *res, *pp, *zz, *Ap, *sol;
    double alpha, beta, rho1, rho2;
} obbmg;

/* ---- indexing -------------------------------------------------------- */
static inline long IX(const olvl *L, int i, int j, int k) {
    return ((long)k * L->nyo + j) * L->nxo + i;
}
static inline int O27(int li, int lj, int lk) { return (li + 1) + 3 * (lj + 1) + 9 * (lk + 1); }
static inline int C8(int pi, int pj, int pk) { return pi + 2 * pj + 4 * pk; }

/* integer division by two rounding up, bbmg_class.f90:147-151 */
static inline int odiv(int n) { return n / 2 + n % 2; }

/* parity with periodic wrap, bbmg_class.f90:155-181 */
static inline int pmod1(int per, int i, int n) {
    if (per) return 1 - ((((i + n - 1) % n) + 1) % 2);
    return 1 - (i % 2);
}
static inline int pmodx(const obbmg *b, int i, int n) { return pmod1(b->xper, i, b->lvl[n].nx); }
static inline int pmody(const obbmg *b, int i, int n) { return pmod1(b->yper, i, b->lvl[n].ny); }
static inline int pmodz(const obbmg *b, int i, int n) { return pmod1(b->zper, i, b->lvl[n].nz); }

static inline double fsign(double a, double b) { return copysign(fabs(a), b); }

/* ---- overlap synchronisation (vsync/msync on one rank) ---------------- */
/* Periodic directions copy the opposite interior layer into the overlap, in
 * the order x, y, z over the full extent of the other directions, as the
 * reference's exchanges do (bbmg_class.f90:1401-1553).  Non-periodic
 * overlaps are left untouched. */
static void osync(const obbmg *b, const olvl *L, double *A, int nc) {
    const int nxo = L->nxo, nyo = L->nyo, nzo = L->nzo;
    if (b->xper) {
        for (int k = 0; k < nzo; k++)
            for (int j = 0; j < nyo; j++) {
                memcpy(A + IX(L, nxo - 1, j, k) * nc, A + IX(L, 1, j, k) * nc, sizeof(double) * nc);
                memcpy(A + IX(L, 0, j, k) * nc, A + IX(L, nxo - 2, j, k) * nc, sizeof(double) * nc);
            }
    }
    if (b->yper) {
        for (int k = 0; k < nzo; k++)
            for (int i = 0; i < nxo; i++) {
                memcpy(A + IX(L, i, nyo - 1, k) * nc, A + IX(L, i, 1, k) * nc, sizeof(double) * nc);
                memcpy(A + IX(L, i, 0, k) * nc, A + IX(L, i, nyo - 2, k) * nc, sizeof(double) * nc);
            }
    }
    if (b->zper) {
        for (int j = 0; j < nyo; j++)
            for (int i = 0; i < nxo; i++) {
                memcpy(A + IX(L, i, j, nzo - 1) * nc, A + IX(L, i, j, 1) * nc, sizeof(double) * nc);
                memcpy(A + IX(L, i, j, 0) * nc, A + IX(L, i, j, nzo - 2) * nc, sizeof(double) * nc);
            }
    }
}

/* ---- construction (bbmg_class.f90:185-369, 575-600; ils_class.f90:184-198) */
static void free_level(olvl *L) {
    free(L->opr); free(L->c2f); free(L->f2c); free(L->oprc2f);
    free(L->v); free(L->f); free(L->r);
    memset(L, 0, sizeof(*L));
}

void orc_destroy(obbmg *b) {
    if (!b) return;
    for (int n = 1; n <= b->nlvl_alloc; n++) free_level(&b->lvl[n]);
    free(b->piv); free(b->pinned); free(b->OP); free(b->LU); free(b->rhs);
    free(b->res); free(b->pp); free(b->zz); free(b->Ap); free(b->sol);
    free(b);
}

obbmg *orc_create(int nx, int ny, int nz, int xper, int yper, int zper,
                  int max_ite, double max_res, int ncycle, int relax_pre, int relax_post,
                  int ncell_coarsest, int use_direct_solve, int use_krylov) {
    if (nx < 1 || ny < 1 || nz < 1) return NULL;
    obbmg *b = (obbmg *)calloc(1, sizeof(obbmg));
    if (!b) return NULL;
    b->xper = xper; b->yper = yper; b->zper = zper;
    /* level count, bbmg_class.f90:231-238 */
    int lx = 1, ly = 1, lz = 1;
    while (nx > (1 << (lx - 1))) lx++;
    while (ny > (1 << (ly - 1))) ly++;
    while (nz > (1 << (lz - 1))) lz++;
    int n1 = lx == 1 ? INT_MAX : lx, n2 = ly == 1 ? INT_MAX : ly, n3 = lz == 1 ? INT_MAX : lz;
    int nl = n1 < n2 ? n1 : n2; nl = nl < n3 ? nl : n3;
    if (lx == 1 && ly == 1 && lz == 1) nl = 1;
    if (nl > ORC_MAXLVL) nl = ORC_MAXLVL;
    b->nlvl = nl;
    /* sizes, bbmg_class.f90:242-334 */
    b->lvl[1].nx = nx; b->lvl[1].ny = ny; b->lvl[1].nz = nz;
    for (int n = 2; n <= nl; n++) {
        b->lvl[n].nx = odiv(b->lvl[n - 1].nx);
        b->lvl[n].ny = odiv(b->lvl[n - 1].ny);
        b->lvl[n].nz = odiv(b->lvl[n - 1].nz);
    }
    for (int n = 1; n <= nl; n++) {
        olvl *L = &b->lvl[n];
        L->nxo = L->nx + 2; L->nyo = L->ny + 2; L->nzo = L->nz + 2;
        L->ncell = (long)L->nx * L->ny * L->nz;
        L->ncello = (long)L->nxo * L->nyo * L->nzo;
    }
    /* the constructor truncates with the default ncell_coarsest=0
       (bbmg_class.f90:96,336-341), so storage exists for every level */
    b->nlvl_alloc = nl;
    for (int n = 1; n <= nl; n++) {
        olvl *L = &b->lvl[n];
        long c = L->ncello;
        if (n < nl) { L->c2f = calloc(c * 8, sizeof(double)); L->oprc2f = calloc(c * 27, sizeof(double)); }
        if (n > 1) L->f2c = calloc(c * 27, sizeof(double));
        L->opr = calloc(c * 27, sizeof(double));
        L->v = calloc(c, sizeof(double)); L->f = calloc(c, sizeof(double)); L->r = calloc(c, sizeof(double));
        if (!L->opr || !L->v || !L->f || !L->r || (n < nl && (!L->c2f || !L->oprc2f)) || (n > 1 && !L->f2c)) {
            orc_destroy(b); return NULL;
        }
    }
    b->max_ite = max_ite; b->max_res = max_res; b->ncycle = ncycle;
    b->relax_pre = relax_pre; b->relax_post = relax_post; b->ncell_coarsest = ncell_coarsest;
    b->use_direct_solve = use_direct_solve; b->use_krylov = use_krylov;
    b->pin_singular = 1;
    /* initialize, bbmg_class.f90:584-598 */
    for (int n = 1; n <= b->nlvl; n++)
        if (b->lvl[n].ncell <= b->ncell_coarsest) { b->nlvl = n; break; }
    if (b->use_krylov) {
        long c = b->lvl[1].ncello;
        b->sol = calloc(c, sizeof(double)); b->res = calloc(c, sizeof(double));
        b->Ap = calloc(c, sizeof(double)); b->pp = calloc(c, sizeof(double)); b->zz = calloc(c, sizeof(double));
        if (!b->sol || !b->res || !b->Ap || !b->pp || !b->zz) { orc_destroy(b); return NULL; }
    }
    return b;
}

int orc_nlvl(const obbmg *b) { return b->nlvl; }
void orc_level_dims(const obbmg *b, int n, int *dims) {
    dims[0] = b->lvl[n].nx; dims[1] = b->lvl[n].ny; dims[2] = b->lvl[n].nz;
}

/* ---- operator input (ils_class.f90:244-256) ---------------------------- */
/* opr is (nst, nx+2g, ny+2g, nz+2g) in Fortran order with g overlap layers;
 * stc is (nst,3) in C order [st][dim].  Interior entries are scattered into
 * the 27-point layout, adding in stencil order. */
void orc_set_operator(obbmg *b, int nst, const int *stc, const double *opr, int g) {
    olvl *L = &b->lvl[1];
    long sx = (long)nst, sy = sx * (L->nx + 2 * g), sz = sy * (L->ny + 2 * g);
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++) {
                double *o = L->opr + IX(L, i, j, k) * 27;
                for (int s = 0; s < 27; s++) o[s] = 0.0;
                const double *src = opr + (long)(k - 1 + g) * sz + (long)(j - 1 + g) * sy + (long)(i - 1 + g) * sx;
                for (int st = 0; st < nst; st++) {
                    int q = O27(stc[3 * st], stc[3 * st + 1], stc[3 * st + 2]);
                    o[q] = o[q] + src[st];
                }
            }
}

/* ---- setup: prolongation (bbmg_class.f90:966-1197) --------------------- */
void orc_recompute_prolongation(obbmg *b, int n) {
    olvl *L = &b->lvl[n];
    const double ratio = 10.0;
    /* sweep 1: identity and lines */
    for (int fk = 0; fk < L->nzo; fk++)
        for (int fj = 0; fj < L->nyo; fj++)
            for (int fi = 0; fi < L->nxo; fi++) {
                int n1 = pmodx(b, fi, n), n2 = pmody(b, fj, n), n3 = pmodz(b, fk, n);
                double *c = L->c2f + IX(L, fi, fj, fk) * 8;
                const double *o = L->opr + IX(L, fi, fj, fk) * 27;
                for (int s = 0; s < 8; s++) c[s] = 0.0;
                int sum = n1 + n2 + n3;
                if (sum == 0) {
                    c[C8(0, 0, 0)] = 1.0;
                } else if (sum == 1) {
                    double o1[3] = {0.0, 0.0, 0.0}; /* opr1d(-1:1) at o1[l+1] */
                    for (int lk = -1; lk <= 1; lk++)
                        for (int lj = -1; lj <= 1; lj++)
                            for (int li = -1; li <= 1; li++) {
                                double a = o[O27(li, lj, lk)];
                                int l, ax;
                                if (n1 == 1) { ax = O27(li, 0, 0); l = li; }
                                else if (n2 == 1) { ax = O27(0, lj, 0); l = lj; }
                                else { ax = O27(0, 0, lk); l = lk; }
                                if (ratio * fabs(o[ax]) >= fabs(a)) o1[l + 1] = o1[l + 1] + a;
                                else o1[1] = o1[1] + a;
                            }
                    o1[1] = fsign(fmax(fabs(o1[1]), ORC_EPS), o1[1]);
                    c[C8(0, 0, 0)] = -o1[0] / o1[1];
                    if (n1 == 1) c[C8(1, 0, 0)] = -o1[2] / o1[1];
                    else if (n2 == 1) c[C8(0, 1, 0)] = -o1[2] / o1[1];
                    else c[C8(0, 0, 1)] = -o1[2] / o1[1];
                }
            }
    /* sweep 2: faces */
    for (int fk = 0; fk < L->nzo; fk++)
        for (int fj = 0; fj < L->nyo; fj++)
            for (int fi = 0; fi < L->nxo; fi++) {
                int n1 = pmodx(b, fi, n), n2 = pmody(b, fj, n), n3 = pmodz(b, fk, n);
                if (n1 + n2 + n3 != 2) continue;
                double *c = L->c2f + IX(L, fi, fj, fk) * 8;
                const double *o = L->opr + IX(L, fi, fj, fk) * 27;
                double o2[3][3] = {{0}}; /* opr2d(a,b) at o2[a+1][b+1] */
                if (n1 == 0) { /* yz-plane */
                    if (fj == 0 || fj == L->nyo - 1 || fk == 0 || fk == L->nzo - 1) continue;
                    for (int lk = -1; lk <= 1; lk++)
                        for (int lj = -1; lj <= 1; lj++)
                            for (int li = -1; li <= 1; li++) {
                                double a = o[O27(li, lj, lk)];
                                if (ratio * fabs(o[O27(0, lj, lk)]) >= fabs(a)) o2[lj + 1][lk + 1] = o2[lj + 1][lk + 1] + a;
                                else o2[1][1] = o2[1][1] + a;
                            }
                    o2[1][1] = fsign(fmax(fabs(o2[1][1]), ORC_EPS), o2[1][1]);
                    for (int lk = -1; lk <= 1; lk++)
                        for (int lj = -1; lj <= 1; lj++) {
                            if (lj == 0 && lk == 0) continue;
                            for (int pk = 0; pk <= 1 - abs(lk); pk++)
                                for (int pj = 0; pj <= 1 - abs(lj); pj++) {
                                    int sj = (lj + 1) / 2 + pj, sk = (lk + 1) / 2 + pk;
                                    const double *cn = L->c2f + IX(L, fi, fj + lj, fk + lk) * 8;
                                    c[C8(0, sj, sk)] = c[C8(0, sj, sk)] - o2[lj + 1][lk + 1] / o2[1][1] * cn[C8(0, pj, pk)];
                                }
                        }
                } else if (n2 == 0) { /* zx-plane */
                    if (fk == 0 || fk == L->nzo - 1 || fi == 0 || fi == L->nxo - 1) continue;
                    for (int lk = -1; lk <= 1; lk++)
                        for (int lj = -1; lj <= 1; lj++)
                            for (int li = -1; li <= 1; li++) {
                                double a = o[O27(li, lj, lk)];
                                if (ratio * fabs(o[O27(li, 0, lk)]) >= fabs(a)) o2[li + 1][lk + 1] = o2[li + 1][lk + 1] + a;
                                else o2[1][1] = o2[1][1] + a;
                            }
                    o2[1][1] = fsign(fmax(fabs(o2[1][1]), ORC_EPS), o2[1][1]);
                    for (int lk = -1; lk <= 1; lk++)
                        for (int li = -1; li <= 1; li++) {
                            if (li == 0 && lk == 0) continue;
                            for (int pk = 0; pk <= 1 - abs(lk); pk++)
                                for (int pi = 0; pi <= 1 - abs(li); pi++) {
                                    int si = (li + 1) / 2 + pi, sk = (lk + 1) / 2 + pk;
                                    const double *cn = L->c2f + IX(L, fi + li, fj, fk + lk) * 8;
                                    c[C8(si, 0, sk)] = c[C8(si, 0, sk)] - o2[li + 1][lk + 1] / o2[1][1] * cn[C8(pi, 0, pk)];
                                }
                        }
                } else { /* xy-plane */
                    if (fi == 0 || fi == L->nxo - 1 || fj == 0 || fj == L->nyo - 1) continue;
                    for (int lk = -1; lk <= 1; lk++)
                        for (int lj = -1; lj <= 1; lj++)
                            for (int li = -1; li <= 1; li++) {
                                double a = o[O27(li, lj, lk)];
                                if (ratio * fabs(o[O27(li, lj, 0)]) >= fabs(a)) o2[li + 1][lj + 1] = o2[li + 1][lj + 1] + a;
                                else o2[1][1] = o2[1][1] + a;
                            }
                    o2[1][1] = fsign(fmax(fabs(o2[1][1]), ORC_EPS), o2[1][1]);
                    for (int lj = -1; lj <= 1; lj++)
                        for (int li = -1; li <= 1; li++) {
                            if (li == 0 && lj == 0) continue;
                            for (int pj = 0; pj <= 1 - abs(lj); pj++)
                                for (int pi = 0; pi <= 1 - abs(li); pi++) {
                                    int si = (li + 1) / 2 + pi, sj = (lj + 1) / 2 + pj;
                                    const double *cn = L->c2f + IX(L, fi + li, fj + lj, fk) * 8;
                                    c[C8(si, sj, 0)] = c[C8(si, sj, 0)] - o2[li + 1][lj + 1] / o2[1][1] * cn[C8(pi, pj, 0)];
                                }
                        }
                }
            }
    /* sweep 3: cube centres, interior only */
    for (int fk = 1; fk <= L->nz; fk++)
        for (int fj = 1; fj <= L->ny; fj++)
            for (int fi = 1; fi <= L->nx; fi++) {
                int n1 = pmodx(b, fi, n), n2 = pmody(b, fj, n), n3 = pmodz(b, fk, n);
                if (n1 + n2 + n3 != 3) continue;
                double *c = L->c2f + IX(L, fi, fj, fk) * 8;
                const double *o = L->opr + IX(L, fi, fj, fk) * 27;
                double d = fsign(fmax(fabs(o[O27(0, 0, 0)]), ORC_EPS), o[O27(0, 0, 0)]);
                for (int lk = -1; lk <= 1; lk++)
                    for (int lj = -1; lj <= 1; lj++)
                        for (int li = -1; li <= 1; li++) {
                            if (li == 0 && lj == 0 && lk == 0) continue;
                            const double *cn = L->c2f + IX(L, fi + li, fj + lj, fk + lk) * 8;
                            for (int pk = 0; pk <= 1 - abs(lk); pk++)
                                for (int pj = 0; pj <= 1 - abs(lj); pj++)
                                    for (int pi = 0; pi <= 1 - abs(li); pi++) {
                                        int si = (li + 1) / 2 + pi, sj = (lj + 1) / 2 + pj, sk = (lk + 1) / 2 + pk;
                                        c[C8(si, sj, sk)] = c[C8(si, sj, sk)] - o[O27(li, lj, lk)] / d * cn[C8(pi, pj, pk)];
                                    }
                        }
            }
    osync(b, L, L->c2f, 8);
}

/* ---- setup: restriction (bbmg_class.f90:1201-1231) --------------------- */
void orc_recompute_restriction(obbmg *b, int n) {
    olvl *L = &b->lvl[n], *F = &b->lvl[n - 1];
    memset(L->f2c, 0, sizeof(double) * 27 * L->ncello);
    for (int ck = 1; ck <= L->nz; ck++)
        for (int cj = 1; cj <= L->ny; cj++)
            for (int ci = 1; ci <= L->nx; ci++) {
                int fi = 2 * ci - 1, fj = 2 * cj - 1, fk = 2 * ck - 1;
                double *w = L->f2c + IX(L, ci, cj, ck) * 27;
                for (int rk = -pmodz(b, fk - 1, n - 1); rk <= pmodz(b, fk + 1, n - 1); rk++)
                    for (int rj = -pmody(b, fj - 1, n - 1); rj <= pmody(b, fj + 1, n - 1); rj++)
                        for (int ri = -pmodx(b, fi - 1, n - 1); ri <= pmodx(b, fi + 1, n - 1); ri++) {
                            int pi = (1 - ri) / 2, pj = (1 - rj) / 2, pk = (1 - rk) / 2;
                            w[O27(ri, rj, rk)] = F->c2f[IX(F, fi + ri, fj + rj, fk + rk) * 8 + C8(pi, pj, pk)];
                        }
            }
    osync(b, L, L->f2c, 27);
}

/* ---- setup: Galerkin operator (bbmg_class.f90:1235-1303) --------------- */
void orc_recompute_operator(obbmg *b, int n) {
    olvl *L = &b->lvl[n], *F = &b->lvl[n - 1];
    memset(F->oprc2f, 0, sizeof(double) * 27 * F->ncello);
    for (int fk = 1; fk <= F->nz; fk++)
        for (int fj = 1; fj <= F->ny; fj++)
            for (int fi = 1; fi <= F->nx; fi++) {
                double *q = F->oprc2f + IX(F, fi, fj, fk) * 27;
                const double *o = F->opr + IX(F, fi, fj, fk) * 27;
                int px0 = pmodx(b, fi, n - 1), py0 = pmody(b, fj, n - 1), pz0 = pmodz(b, fk, n - 1);
                for (int lk = -1; lk <= 1; lk++)
                    for (int lj = -1; lj <= 1; lj++)
                        for (int li = -1; li <= 1; li++) {
                            int pxl = pmodx(b, fi + li, n - 1), pyl = pmody(b, fj + lj, n - 1), pzl = pmodz(b, fk + lk, n - 1);
                            const double *cn = F->c2f + IX(F, fi + li, fj + lj, fk + lk) * 8;
                            for (int pk = 0; pk <= pzl; pk++)
                                for (int pj = 0; pj <= pyl; pj++)
                                    for (int pi = 0; pi <= pxl; pi++) {
                                        int si = pi + (1 - px0) * (li < 0 ? li : 0) + (1 - pxl) * (li > 0 ? li : 0);
                                        int sj = pj + (1 - py0) * (lj < 0 ? lj : 0) + (1 - pyl) * (lj > 0 ? lj : 0);
                                        int sk = pk + (1 - pz0) * (lk < 0 ? lk : 0) + (1 - pzl) * (lk > 0 ? lk : 0);
                                        q[O27(si, sj, sk)] = q[O27(si, sj, sk)] + o[O27(li, lj, lk)] * cn[C8(pi, pj, pk)];
                                    }
                        }
            }
    osync(b, F, F->oprc2f, 27);
    memset(L->opr, 0, sizeof(double) * 27 * L->ncello);
    for (int ck = 1; ck <= L->nz; ck++)
        for (int cj = 1; cj <= L->ny; cj++)
            for (int ci = 1; ci <= L->nx; ci++) {
                int fi = 2 * ci - 1, fj = 2 * cj - 1, fk = 2 * ck - 1;
                double *o = L->opr + IX(L, ci, cj, ck) * 27;
                const double *w = L->f2c + IX(L, ci, cj, ck) * 27;
                for (int rk = -pmodz(b, fk - 1, n - 1); rk <= pmodz(b, fk + 1, n - 1); rk++)
                    for (int rj = -pmody(b, fj - 1, n - 1); rj <= pmody(b, fj + 1, n - 1); rj++)
                        for (int ri = -pmodx(b, fi - 1, n - 1); ri <= pmodx(b, fi + 1, n - 1); ri++) {
                            const double *q = F->oprc2f + IX(F, fi + ri, fj + rj, fk + rk) * 27;
                            for (int lk = -1 + pmodz(b, fk + rk, n - 1); lk <= 1; lk++)
                                for (int lj = -1 + pmody(b, fj + rj, n - 1); lj <= 1; lj++)
                                    for (int li = -1 + pmodx(b, fi + ri, n - 1); li <= 1; li++) {
                                        /* (r-1)/2 with Fortran truncation toward zero */
                                        int si = (ri - 1) / 2 + li, sj = (rj - 1) / 2 + lj, sk = (rk - 1) / 2 + lk;
                                        o[O27(si, sj, sk)] = o[O27(si, sj, sk)] + w[O27(ri, rj, rk)] * q[O27(li, lj, lk)];
                                    }
                        }
            }
    osync(b, L, L->opr, 27);
}

/* ---- setup: dense coarsest problem (bbmg_class.f90:1307-1385) ---------- */
/* unblocked LU with row partial pivoting; A is column-major n x n */
static int lu_factor(int n, double *A, int *piv) {
    int info = 0;
    for (int j = 0; j < n; j++) {
        int p = j;
        double amax = fabs(A[(long)j * n + j]);
        for (int i = j + 1; i < n; i++) {
            double a = fabs(A[(long)j * n + i]);
            if (a > amax) { amax = a; p = i; }
        }
        piv[j] = p;
        if (A[(long)j * n + p] != 0.0) {
            if (p != j)
                for (int c = 0; c < n; c++) {
                    double t = A[(long)c * n + j]; A[(long)c * n + j] = A[(long)c * n + p]; A[(long)c * n + p] = t;
                }
            double d = A[(long)j * n + j];
            for (int i = j + 1; i < n; i++) A[(long)j * n + i] = A[(long)j * n + i] / d;
        } else if (info == 0) {
            info = j + 1;
        }
        for (int c = j + 1; c < n; c++) {
            double u = A[(long)c * n + j];
            for (int i = j + 1; i < n; i++) A[(long)c * n + i] = A[(long)c * n + i] - A[(long)j * n + i] * u;
        }
    }
    return info;
}

static void lu_solve(int n, const double *A, const int *piv, const int *pinned, double *x) {
    for (int j = 0; j < n; j++) {
        int p = piv[j];
        if (p != j) { double t = x[j]; x[j] = x[p]; x[p] = t; }
    }
    for (int k = 0; k < n; k++) {
        if (x[k] != 0.0)
            for (int i = k + 1; i < n; i++) x[i] = x[i] - x[k] * A[(long)k * n + i];
    }
    for (int k = n - 1; k >= 0; k--) {
        if (pinned && pinned[k]) { x[k] = 0.0; continue; }
        if (x[k] != 0.0) {
            x[k] = x[k] / A[(long)k * n + k];
            for (int i = 0; i < k; i++) x[i] = x[i] - x[k] * A[(long)k * n + i];
        }
    }
}

void orc_recompute_direct(obbmg *b) {
    olvl *L = &b->lvl[b->nlvl];
    b->np = (int)L->ncell;
    int np = b->np;
    free(b->piv); free(b->OP); free(b->LU); free(b->rhs);
    b->piv = calloc(np, sizeof(int));
    b->OP = calloc((long)np * np, sizeof(double));
    b->LU = calloc((long)np * np, sizeof(double));
    b->rhs = calloc(np, sizeof(double));
    const int nx = L->nx, ny = L->ny;
    for (int k1 = 1; k1 <= L->nz; k1++)
        for (int j1 = 1; j1 <= L->ny; j1++)
            for (int i1 = 1; i1 <= L->nx; i1++) {
                int ind1 = i1 + (j1 - 1) * nx + (k1 - 1) * nx * ny;
                const double *o = L->opr + IX(L, i1, j1, k1) * 27;
                for (int sk = -1; sk <= 1; sk++) {
                    int k2 = k1 + sk;
                    if (k2 == L->nz + 1) { if (!b->zper) continue; k2 = 1; }
                    if (k2 == 0) { if (!b->zper) continue; k2 = L->nz; }
                    for (int sj = -1; sj <= 1; sj++) {
                        int j2 = j1 + sj;
                        if (j2 == L->ny + 1) { if (!b->yper) continue; j2 = 1; }
                        if (j2 == 0) { if (!b->yper) continue; j2 = L->ny; }
                        for (int si = -1; si <= 1; si++) {
                            int i2 = i1 + si;
                            if (i2 == L->nx + 1) { if (!b->xper) continue; i2 = 1; }
                            if (i2 == 0) { if (!b->xper) continue; i2 = L->nx; }
                            int ind2 = i2 + (j2 - 1) * nx + (k2 - 1) * nx * ny;
                            long e = (long)(ind2 - 1) * np + (ind1 - 1);
                            b->OP[e] = b->OP[e] + o[O27(si, sj, sk)];
                        }
                    }
                }
            }
    /* the reference factors a fresh copy at every call (bbmg_class.f90:912-913);
       the factorisation is deterministic, so it is done once here */
    memcpy(b->LU, b->OP, sizeof(double) * (long)np * np);
    b->lu_info = lu_factor(np, b->LU, b->piv);
    /* A periodic or all-Neumann problem makes the coarsest matrix singular;
       its LU then ends with a pivot of round-off size.  Dividing by it (what
       DGESV does) injects an arbitrarily large null-space component; with
       pin_singular the unknown of every pivot below 1000*np*eps*max|pivot|
       (three decades above the round-off level: with density contrasts of
       1e3 the round-off pivot reaches ~1e-14 of the largest, genuine ones
       stay above ~1e-3) is set to zero instead, i.e. the consistent part of
       the system is solved. */
    free(b->pinned);
    b->pinned = calloc(np, sizeof(int));
    double umax = 0.0;
    for (int k = 0; k < np; k++) umax = fmax(umax, fabs(b->LU[(long)k * np + k]));
    double tol = 1000.0 * (double)np * ORC_EPS * umax;
    for (int k = 0; k < np; k++) b->pinned[k] = b->pin_singular && fabs(b->LU[(long)k * np + k]) <= tol;
}

/* ---- update (bbmg_class.f90:932-962) ----------------------------------- */
void orc_update(obbmg *b) {
    olvl *L = &b->lvl[1];
    for (int k = 0; k < L->nzo; k++)
        for (int j = 0; j < L->nyo; j++)
            for (int i = 0; i < L->nxo; i++) {
                if (i >= 1 && i <= L->nx && j >= 1 && j <= L->ny && k >= 1 && k <= L->nz) continue;
                double *o = L->opr + IX(L, i, j, k) * 27;
                for (int s = 0; s < 27; s++) o[s] = 0.0;
                o[O27(0, 0, 0)] = 1.0;
            }
    osync(b, L, L->opr, 27);
    for (int n = 2; n <= b->nlvl; n++) {
        orc_recompute_prolongation(b, n - 1);
        orc_recompute_restriction(b, n);
        orc_recompute_operator(b, n);
    }
    orc_recompute_direct(b);
}

/* ---- solve-phase kernels ------------------------------------------------ */
static inline double stencil27(const double *o, const olvl *L, const double *A, int i, int j, int k) {
    double s = 0.0;
    for (int lk = -1; lk <= 1; lk++)
        for (int lj = -1; lj <= 1; lj++)
            for (int li = -1; li <= 1; li++)
                s = s + o[O27(li, lj, lk)] * A[IX(L, i + li, j + lj, k + lk)];
    return s;
}

/* bbmg_class.f90:831-844 */
void orc_get_residual(obbmg *b, int n) {
    olvl *L = &b->lvl[n];
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++) {
                long c = IX(L, i, j, k);
                L->r[c] = L->f[c] - stencil27(L->opr + c * 27, L, L->v, i, j, k);
            }
    osync(b, L, L->r, 1);
}

/* bbmg_class.f90:848-887 */
static void orc_relax_vec(obbmg *b, double *A, const double *B, int n, int dir) {
    olvl *L = &b->lvl[n];
    int c0 = dir > 0 ? 1 : 8, c1 = dir > 0 ? 8 : 1, cd = dir > 0 ? 1 : -1;
    for (int col = c0; cd > 0 ? col <= c1 : col >= c1; col += cd) {
        int pz = ((col - 1) / 4) % 2, py = ((col - 1) / 2) % 2, px = (col - 1) % 2;
        for (int k = 1 + pz; k <= L->nz; k += 2)
            for (int j = 1 + py; j <= L->ny; j += 2)
                for (int i = 1 + px; i <= L->nx; i += 2) {
                    long c = IX(L, i, j, k);
                    const double *o = L->opr + c * 27;
                    A[c] = 0.0;
                    A[c] = stencil27(o, L, A, i, j, k);
                    A[c] = (B[c] - A[c]) / (o[O27(0, 0, 0)] + ORC_EPS);
                }
        osync(b, L, A, 1);
    }
}
void orc_relax(obbmg *b, int n, int dir) { orc_relax_vec(b, b->lvl[n].v, b->lvl[n].f, n, dir); }

/* prolongation application, bbmg_class.f90:779-801 */
static void orc_c2f_vec(obbmg *b, const double *Ac, int nc, double *Af, int nf) {
    olvl *C = &b->lvl[nc], *F = &b->lvl[nf];
    for (int fk = 1; fk <= F->nz; fk++)
        for (int fj = 1; fj <= F->ny; fj++)
            for (int fi = 1; fi <= F->nx; fi++) {
                int ci = (fi + 1) / 2, cj = (fj + 1) / 2, ck = (fk + 1) / 2;
                const double *w = F->c2f + IX(F, fi, fj, fk) * 8;
                double s = 0.0;
                for (int pk = 0; pk <= 1; pk++)
                    for (int pj = 0; pj <= 1; pj++)
                        for (int pi = 0; pi <= 1; pi++)
                            s = s + w[C8(pi, pj, pk)] * Ac[IX(C, ci + pi, cj + pj, ck + pk)];
                Af[IX(F, fi, fj, fk)] = s;
            }
    osync(b, F, Af, 1);
}
void orc_c2f(obbmg *b, int nc) { orc_c2f_vec(b, b->lvl[nc].v, nc, b->lvl[nc - 1].r, nc - 1); }

/* restriction application, bbmg_class.f90:805-827 */
static void orc_f2c_vec(obbmg *b, const double *Af, int nf, double *Ac, int nc) {
    olvl *C = &b->lvl[nc], *F = &b->lvl[nf];
    for (int ck = 1; ck <= C->nz; ck++)
        for (int cj = 1; cj <= C->ny; cj++)
            for (int ci = 1; ci <= C->nx; ci++) {
                int fi = 2 * ci - 1, fj = 2 * cj - 1, fk = 2 * ck - 1;
                const double *w = C->f2c + IX(C, ci, cj, ck) * 27;
                double s = 0.0;
                for (int rk = -1; rk <= 1; rk++)
                    for (int rj = -1; rj <= 1; rj++)
                        for (int ri = -1; ri <= 1; ri++)
                            s = s + w[O27(ri, rj, rk)] * Af[IX(F, fi + ri, fj + rj, fk + rk)];
                Ac[IX(C, ci, cj, ck)] = s;
            }
    osync(b, C, Ac, 1);
}
void orc_f2c(obbmg *b, int nf) { orc_f2c_vec(b, b->lvl[nf].r, nf, b->lvl[nf + 1].f, nf + 1); }

/* bbmg_class.f90:891-927 */
void orc_direct_solve(obbmg *b) {
    olvl *L = &b->lvl[b->nlvl];
    const int nx = L->nx, ny = L->ny;
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++)
                b->rhs[i - 1 + (j - 1) * nx + (k - 1) * nx * ny] = L->f[IX(L, i, j, k)];
    if (b->lu_info == 0 || b->pin_singular) lu_solve(b->np, b->LU, b->piv, b->pinned, b->rhs);
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++)
                L->v[IX(L, i, j, k)] = b->rhs[i - 1 + (j - 1) * nx + (k - 1) * nx * ny];
    osync(b, L, L->v, 1);
}

/* bbmg_class.f90:732-776 */
void orc_cycle(obbmg *b, int n) {
    olvl *L = &b->lvl[n];
    if (n > 1) memset(L->v, 0, sizeof(double) * L->ncello);
    if (n == b->nlvl) {
        if (b->use_direct_solve) orc_direct_solve(b);
        else {
            int dir = 1;
            for (int i = 0; i < b->relax_pre + b->relax_post; i++) { orc_relax(b, n, dir); dir = -dir; }
        }
        return;
    }
    int dir = 1;
    for (int i = 0; i < b->relax_pre; i++) { orc_relax(b, n, dir); dir = -dir; }
    orc_get_residual(b, n);
    orc_f2c(b, n);
    for (int i = 0; i < b->ncycle; i++) orc_cycle(b, n + 1);
    orc_c2f(b, n + 1);
    for (long c = 0; c < L->ncello; c++) L->v[c] = L->v[c] + L->r[c];
    for (int i = 0; i < b->relax_post; i++) { orc_relax(b, n, dir); dir = -dir; }
}

/* maximum of |A| over the interior; a NaN anywhere makes the result NaN */
static double maxabs_interior(const olvl *L, const double *A) {
    double m = 0.0;
    int bad = 0;
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++) {
                double a = fabs(A[IX(L, i, j, k)]);
                if (a != a) bad = 1;
                else if (a > m) m = a;
            }
    return bad ? NAN : m;
}
static double dot_interior(const olvl *L, const double *A, const double *B) {
    double s = 0.0;
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++) {
                long c = IX(L, i, j, k);
                s = s + A[c] * B[c];
            }
    return s;
}

/* bbmg_class.f90:643-703 */
static void orc_cgsolve(obbmg *b) {
    olvl *L = &b->lvl[1];
    long nc = L->ncello;
    memcpy(b->res, L->r, sizeof(double) * nc);
    memcpy(b->sol, L->v, sizeof(double) * nc);
    for (int n = 1; n <= b->max_ite; n++) {
        memcpy(L->f, b->res, sizeof(double) * nc);
        osync(b, L, L->f, 1);
        memset(L->v, 0, sizeof(double) * nc);
        orc_cycle(b, 1);
        memcpy(b->zz, L->v, sizeof(double) * nc);
        b->rho2 = b->rho1;
        b->rho1 = dot_interior(L, b->zz, b->res);
        b->beta = (n == 1) ? 0.0 : b->rho1 / b->rho2;
        for (long c = 0; c < nc; c++) b->pp[c] = b->zz[c] + b->beta * b->pp[c];
        osync(b, L, b->pp, 1);
        for (int k = 1; k <= L->nz; k++)
            for (int j = 1; j <= L->ny; j++)
                for (int i = 1; i <= L->nx; i++) {
                    long c = IX(L, i, j, k);
                    b->Ap[c] = stencil27(L->opr + c * 27, L, b->pp, i, j, k);
                }
        b->alpha = b->rho1 / dot_interior(L, b->pp, b->Ap);
        for (long c = 0; c < nc; c++) b->sol[c] = b->sol[c] + b->alpha * b->pp[c];
        for (long c = 0; c < nc; c++) b->res[c] = b->res[c] - b->alpha * b->Ap[c];
        b->my_res = maxabs_interior(L, b->res) / b->my_res0;
        b->my_ite = n;
        if (b->my_res <= b->max_res) break;
    }
    memcpy(L->v, b->sol, sizeof(double) * nc);
}

/* bbmg_class.f90:707-728 */
static void orc_mgsolve(obbmg *b) {
    olvl *L = &b->lvl[1];
    for (int n = 1; n <= b->max_ite; n++) {
        orc_cycle(b, 1);
        orc_get_residual(b, 1);
        b->my_res = maxabs_interior(L, L->r) / b->my_res0;
        b->my_ite = n;
        if (b->my_res <= b->max_res) break;
    }
}

/* bbmg_class.f90:604-639 */
void orc_bbmg_solve(obbmg *b) {
    olvl *L = &b->lvl[1];
    for (int k = 0; k < L->nzo; k++)
        for (int j = 0; j < L->nyo; j++)
            for (int i = 0; i < L->nxo; i++) {
                if (i >= 1 && i <= L->nx && j >= 1 && j <= L->ny && k >= 1 && k <= L->nz) continue;
                L->f[IX(L, i, j, k)] = 0.0;
                L->v[IX(L, i, j, k)] = 0.0;
            }
    osync(b, L, L->f, 1);
    osync(b, L, L->v, 1);
    orc_get_residual(b, 1);
    b->my_res0 = maxabs_interior(L, L->r);
    if (b->my_res0 == 0.0) { b->my_ite = 0; b->my_res = 0.0; return; }
    if (b->use_krylov) orc_cgsolve(b);
    else orc_mgsolve(b);
}

/* ils%solve bbmg branch (ils_class.f90:674-700, 740-743, 780-788).
 * rhs/sol are interior arrays (nx,ny,nz), i fastest. */
void orc_solve(obbmg *b, const double *rhs, double *sol, int *it, double *rerr) {
    olvl *L = &b->lvl[1];
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++) {
                long e = ((long)(k - 1) * L->ny + (j - 1)) * L->nx + (i - 1);
                L->f[IX(L, i, j, k)] = rhs[e];
                L->v[IX(L, i, j, k)] = sol[e];
            }
    orc_bbmg_solve(b);
    *it = b->my_ite;
    *rerr = b->my_res;
    for (int k = 1; k <= L->nz; k++)
        for (int j = 1; j <= L->ny; j++)
            for (int i = 1; i <= L->nx; i++) {
                long e = ((long)(k - 1) * L->ny + (j - 1)) * L->nx + (i - 1);
                sol[e] = L->v[IX(L, i, j, k)];
            }
}

/* ---- array access for tests -------------------------------------------- */
/* which: 0=opr(27) 1=c2f(8) 2=f2c(27) 3=oprc2f(27) 4=v 5=f 6=r.  Arrays are
 * copied with the overlap, cell-major (k, j, i) and the coefficient index
 * fastest. Returns the number of doubles, or -1 if absent. */
static double *orc_array(obbmg *b, int n, int which, int *ncoef) {
    olvl *L = &b->lvl[n];
    switch (which) {
    case 0: *ncoef = 27; return L->opr;
    case 1: *ncoef = 8; return L->c2f;
    case 2: *ncoef = 27; return L->f2c;
    case 3: *ncoef = 27; return L->oprc2f;
    case 4: *ncoef = 1; return L->v;
    case 5: *ncoef = 1; return L->f;
    case 6: *ncoef = 1; return L->r;
    }
    return NULL;
}
long orc_get(obbmg *b, int n, int which, double *out) {
    int nc = 0;
    if (n < 1 || n > b->nlvl_alloc) return -1;
    double *a = orc_array(b, n, which, &nc);
    if (!a) return -1;
    long cnt = b->lvl[n].ncello * nc;
    if (out) memcpy(out, a, sizeof(double) * cnt);
    return cnt;
}
long orc_put(obbmg *b, int n, int which, const double *in) {
    int nc = 0;
    if (n < 1 || n > b->nlvl_alloc) return -1;
    double *a = orc_array(b, n, which, &nc);
    if (!a) return -1;
    long cnt = b->lvl[n].ncello * nc;
    memcpy(a, in, sizeof(double) * cnt);
    return cnt;
}
int orc_direct_info(const obbmg *b, int *np) { *np = b->np; return b->lu_info; }
long orc_get_direct(const obbmg *b, double *OP, double *LU, int *piv) {
    long nn = (long)b->np * b->np;
    if (OP) memcpy(OP, b->OP, sizeof(double) * nn);
    if (LU) memcpy(LU, b->LU, sizeof(double) * nn);
    if (piv) memcpy(piv, b->piv, sizeof(int) * b->np);
    return nn;
}
/* dense solve with the stored factorisation (the direct_solve arithmetic) */
void orc_direct_apply(const obbmg *b, double *x) {
    if (b->lu_info == 0 || b->pin_singular) lu_solve(b->np, b->LU, b->piv, b->pinned, x);
}
void orc_set_pin_singular(obbmg *b, int pin) { b->pin_singular = pin; }
int orc_npinned(const obbmg *b) {
    int c = 0;
    for (int k = 0; k < b->np; k++) c += b->pinned ? b->pinned[k] : 0;
    return c;
}
void orc_set_params(obbmg *b, int max_ite, double max_res) { b->max_ite = max_ite; b->max_res = max_res; }
