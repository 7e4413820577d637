/*
 * oracle.c -- FP64 CPU restatement of the cpsFDTD time step (see oracle.h).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA product, never part of it.
 *
 * Arithmetic is written so that C's left-to-right association reproduces the
 * reference expressions term by term; compile with -ffp-contract=off so that
 * no fused multiply-add changes a rounding.  Loops are parallelised with
 * OpenMP over independent cells only, so results do not depend on the thread
 * count.
 */
#include "oracle.h"
#include "cells.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* Material indices with fixed meaning in the E update (BasicFDTD.cpp:34-38) */
#define ID_DISPERSIVE 2
#define ID_PEC 4

enum { EX = 0, EY, EZ, HX, HY, HZ };
enum { FX1 = 0, FX2, FY1, FY2, FZ1, FZ2 };

typedef struct {
    int on;
    int np[6];
    double *bE[6], *cE[6], *bH[6], *cH[6];
    double *qe[6][2]; /* psi of H differences, applied to E (reference QH**) */
    double *qh[6][2]; /* psi of E differences, applied to H (reference QE**) */
    double cpmlE, cpmlH;
    int literal; /* 1: cpmlE/cpmlH for every cell (CPML.cpp:524-525); 0: each cell's curl coefficient */
} pml_t;

typedef struct {
    int u1, u2, v1, v2; /* inclusive table ranges */
    double *dE, *pE, *dH, *pH;
} face_t;

typedef struct {
    int on;
    int Nt;
    double *einc, *hinc;
    int i1, i2, j1, j2, k1, k2;
    face_t face[6];
    double cE[6][2]; /* signed coefficient of E1/E2 correction per face */
    double cH[6][2]; /* signed coefficient of H1/H2 correction per face */
} tfsf_t;

typedef struct {
    int comp;
    int64_t idx;
    int n;
    double *wave;
} src_t;

typedef struct {
    int npts;
    int64_t *idx;
    double *sample; /* [npts][6] */
    int nfreq;
    uint32_t mask;
    int ncomp;
    int comps[6];
    double *omega;
    double *acc; /* [npts][ncomp][nfreq][2] */
} port_t;

struct orc {
    int nx, ny, nz;
    double dx, dy, dz, dt;
    int64_t sx, sy; /* strides of i and j in the [i][j][k] layout */
    int64_t ncell;
    double *F[6];
    uint8_t *id;
    int nmedia;
    double *aE, *bE, *aH, *bH;
    /* stretched-coordinate arrays, names as Structure.h:82-83 */
    double *cExy, *cEyx, *cEzx, *cExz, *cEzy, *cEyz;
    double *cHxy, *cHyx, *cHzx, *cHxz, *cHzy, *cHyz;
    int64_t step;
    pml_t pml;
    dl_t dl;
    gain_t gain;
    three_t three;
    tfsf_t tfsf;
    int nsrc;
    src_t *src;
    int nport;
    port_t *port;
};

#define IDX(o, i, j, k) ((int64_t)(i) * (o)->sx + (int64_t)(j) * (o)->sy + (int64_t)(k))

static void *zalloc(size_t n) { return calloc(n ? n : 1, 1); }

int orc_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

orc *orc_create(int nx, int ny, int nz, double dx, double dy, double dz, double dt)
{
    if (nx < 2 || ny < 2 || nz < 2) return NULL;
    orc *o = (orc *)zalloc(sizeof(orc));
    o->nx = nx; o->ny = ny; o->nz = nz;
    o->dx = dx; o->dy = dy; o->dz = dz; o->dt = dt;
    o->sy = nz + 1;
    o->sx = (int64_t)(ny + 1) * (nz + 1);
    o->ncell = (int64_t)(nx + 1) * o->sx;
    for (int c = 0; c < 6; ++c) o->F[c] = (double *)zalloc(sizeof(double) * o->ncell);
    o->id = (uint8_t *)zalloc(o->ncell);
    /* Structure.cpp:411-445: stretch arrays start at 1/delta */
    o->cEyz = (double *)zalloc(sizeof(double) * nx); o->cEzy = (double *)zalloc(sizeof(double) * nx);
    o->cHyz = (double *)zalloc(sizeof(double) * nx); o->cHzy = (double *)zalloc(sizeof(double) * nx);
    o->cExz = (double *)zalloc(sizeof(double) * ny); o->cEzx = (double *)zalloc(sizeof(double) * ny);
    o->cHxz = (double *)zalloc(sizeof(double) * ny); o->cHzx = (double *)zalloc(sizeof(double) * ny);
    o->cExy = (double *)zalloc(sizeof(double) * nz); o->cEyx = (double *)zalloc(sizeof(double) * nz);
    o->cHxy = (double *)zalloc(sizeof(double) * nz); o->cHyx = (double *)zalloc(sizeof(double) * nz);
    double t = 1.0 / dx;
    for (int i = 0; i < nx; ++i) o->cEyz[i] = o->cEzy[i] = o->cHyz[i] = o->cHzy[i] = t;
    t = 1.0 / dy;
    for (int i = 0; i < ny; ++i) o->cExz[i] = o->cEzx[i] = o->cHxz[i] = o->cHzx[i] = t;
    t = 1.0 / dz;
    for (int i = 0; i < nz; ++i) o->cEyx[i] = o->cExy[i] = o->cHyx[i] = o->cHxy[i] = t;
    o->step = 1;
    return o;
}

void orc_destroy(orc *o)
{
    if (!o) return;
    for (int c = 0; c < 6; ++c) free(o->F[c]);
    free(o->id);
    free(o->aE); free(o->bE); free(o->aH); free(o->bH);
    double *st[12] = {o->cExy, o->cEyx, o->cEzx, o->cExz, o->cEzy, o->cEyz,
                      o->cHxy, o->cHyx, o->cHzx, o->cHxz, o->cHzy, o->cHyz};
    for (int s = 0; s < 12; ++s) free(st[s]);
    for (int f = 0; f < 6; ++f) {
        free(o->pml.bE[f]); free(o->pml.cE[f]); free(o->pml.bH[f]); free(o->pml.cH[f]);
        for (int q = 0; q < 2; ++q) { free(o->pml.qe[f][q]); free(o->pml.qh[f][q]); }
        free(o->tfsf.face[f].dE); free(o->tfsf.face[f].pE);
        free(o->tfsf.face[f].dH); free(o->tfsf.face[f].pH);
    }
    free(o->dl.cell); free(o->dl.state);
    free(o->gain.cell); free(o->gain.state);
    free(o->three.cell); free(o->three.state);
    free(o->tfsf.einc); free(o->tfsf.hinc);
    for (int s = 0; s < o->nsrc; ++s) free(o->src[s].wave);
    free(o->src);
    for (int p = 0; p < o->nport; ++p) {
        free(o->port[p].idx); free(o->port[p].sample);
        free(o->port[p].omega); free(o->port[p].acc);
    }
    free(o->port);
    free(o);
}

/* Structure.cpp:446-451 */
int orc_set_media(orc *o, int n, const double *epsR, const double *muR,
                  const double *sig, const double *sigM)
{
    if (n < 1 || n > 256) return 1;
    o->nmedia = n;
    o->aE = (double *)zalloc(sizeof(double) * 256); o->bE = (double *)zalloc(sizeof(double) * 256);
    o->aH = (double *)zalloc(sizeof(double) * 256); o->bH = (double *)zalloc(sizeof(double) * 256);
    const double dt = o->dt;
    for (int i = 0; i < n; ++i) {
        o->aE[i] = (2.0 * K_EPS0 * epsR[i] - sig[i] * dt) / (2.0 * K_EPS0 * epsR[i] + sig[i] * dt);
        o->bE[i] = (2.0 * dt) / (2.0 * K_EPS0 * epsR[i] + sig[i] * dt);
        o->aH[i] = (2.0 * K_MU0 * muR[i] - sigM[i] * dt) / (2.0 * K_MU0 * muR[i] + sigM[i] * dt);
        o->bH[i] = (2.0 * dt) / (2.0 * K_MU0 * muR[i] + sigM[i] * dt);
    }
    return 0;
}

int orc_set_ids(orc *o, const uint8_t *ids)
{
    memcpy(o->id, ids, o->ncell);
    return 0;
}

/* ---------------------------------------------------------------- CPML --- */

/* Grading of an E-side (integer-node) layer: CPML.cpp:139-183.  Index 0 is the
 * outer boundary node for the first end and the inner node for the second end. */
static void pml_grade_e(double *kappa, double *b, double *c, int first, int np, double dt,
                        double del, double m, double ma, double sigmax, double kapmax,
                        double alpmax)
{
    double *sigma = (double *)zalloc(sizeof(double) * (np + 1));
    double *alpha = (double *)zalloc(sizeof(double) * (np + 1));
    for (int i = 1; i <= np + 1; ++i) {
        double ps, pa;
        if (first) {
            ps = pow(((double)np + 1.0 - i) / ((double)np), m);
            pa = pow(((double)i - 1.0) / ((double)np), ma);
        } else {
            ps = pow(((double)i - 1.0) / np, m);
            pa = pow(((double)np + 1.0 - i) / np, ma);
        }
        sigma[i - 1] = sigmax * ps;
        kappa[i - 1] = 1.0 + (kapmax - 1.0) * ps;
        alpha[i - 1] = alpmax * pa;
    }
    for (int i = 0; i <= np; ++i) {
        b[i] = exp(-(sigma[i] / kappa[i] + alpha[i]) * dt / K_EPS0);
        if ((sigma[i] == 0.0) && (alpha[i] == 0.0))
            c[i] = 0.0;
        else
            c[i] = sigma[i] * (b[i] - 1.0) / (sigma[i] + kappa[i] * alpha[i]) / kappa[i] / del;
    }
    free(sigma);
    free(alpha);
}

/* Grading of an H-side (half-node) layer: CPML.cpp:185-229.  The reference
 * leaves b/c[np-1] unset (its loop stops at np-2); here every entry, including
 * np-1, uses the same formula. */
static void pml_grade_h(double *kappa, double *b, double *c, int first, int np, double dt,
                        double del, double m, double ma, double sigmax, double kapmax,
                        double alpmax)
{
    double *sigma = (double *)zalloc(sizeof(double) * np);
    double *alpha = (double *)zalloc(sizeof(double) * np);
    for (int i = 1; i <= np; ++i) {
        double ps, pa;
        if (first) {
            ps = pow(((np - i + 0.5) / np), m);
            pa = pow(((i - 0.5) / np), ma);
        } else {
            ps = pow(((i - 0.5) / np), m);
            pa = pow(((np - i + 0.5) / np), ma);
        }
        sigma[i - 1] = sigmax * ps;
        kappa[i - 1] = 1.0 + (kapmax - 1.0) * ps;
        alpha[i - 1] = alpmax * pa;
    }
    for (int i = 0; i < np; ++i) {
        b[i] = exp(-(sigma[i] / kappa[i] + alpha[i]) * dt / K_EPS0);
        if ((sigma[i] == 0.0) && (alpha[i] == 0.0))
            c[i] = 0.0;
        else
            c[i] = sigma[i] * (b[i] - 1.0) / (sigma[i] + kappa[i] * alpha[i]) / kappa[i] / del;
    }
    free(sigma);
    free(alpha);
}

/* CPML::InitializeCPML, CPML.cpp:231-527.  npml = {x1,x2,y1,y2,z1,z2}; both
 * ends of an axis must be equal (the reference folds the second-end kappa
 * with the first-end count, CPML.cpp:374,402,430,459,487,515). */
int orc_pml_init(orc *o, const int32_t npml[6], double m, double malp, double kapmax,
                 double sig_ratio, double alpmax, int literal)
{
    pml_t *P = &o->pml;
    P->literal = literal;
    for (int a = 0; a < 3; ++a) {
        if (npml[2 * a] != npml[2 * a + 1]) return 1;
        if (npml[2 * a] < 1) return 1;
    }
    if (npml[0] * 2 >= o->nx || npml[2] * 2 >= o->ny || npml[4] * 2 >= o->nz) return 1;
    for (int f = 0; f < 6; ++f) P->np[f] = npml[f];
    const double eta0 = sqrt(K_MU0 / K_EPS0);
    const double del[3] = {o->dx, o->dy, o->dz};
    double *cE1[3] = {o->cEzy, o->cEzx, o->cExy}, *cE2[3] = {o->cEyz, o->cExz, o->cEyx};
    double *cH1[3] = {o->cHzy, o->cHzx, o->cHxy}, *cH2[3] = {o->cHyz, o->cHxz, o->cHyx};
    const int nax[3] = {o->nx, o->ny, o->nz};
    for (int a = 0; a < 3; ++a) {
        const double sigmax = sig_ratio * (0.8 * (m + 1) / (del[a] * eta0));
        for (int end = 0; end < 2; ++end) {
            const int f = 2 * a + end, np = P->np[f];
            double *kap = (double *)zalloc(sizeof(double) * (np + 1));
            P->bE[f] = (double *)zalloc(sizeof(double) * (np + 1));
            P->cE[f] = (double *)zalloc(sizeof(double) * (np + 1));
            pml_grade_e(kap, P->bE[f], P->cE[f], end == 0, np, o->dt, del[a], m, malp, sigmax,
                        kapmax, alpmax);
            if (end == 0) {
                for (int i = 0; i <= np; ++i) { cE1[a][i] = cE1[a][i] / kap[i]; cE2[a][i] = cE2[a][i] / kap[i]; }
            } else {
                const int base = nax[a] - np;
                for (int i = 0; i < np; ++i) {
                    cE1[a][base + i] = cE1[a][base + i] / kap[i];
                    cE2[a][base + i] = cE2[a][base + i] / kap[i];
                }
            }
            free(kap);
        }
    }
    for (int a = 0; a < 3; ++a) {
        const double sigmax = sig_ratio * (0.8 * (m + 1) / (del[a] * eta0));
        for (int end = 0; end < 2; ++end) {
            const int f = 2 * a + end, np = P->np[f];
            double *kap = (double *)zalloc(sizeof(double) * np);
            P->bH[f] = (double *)zalloc(sizeof(double) * np);
            P->cH[f] = (double *)zalloc(sizeof(double) * np);
            pml_grade_h(kap, P->bH[f], P->cH[f], end == 0, np, o->dt, del[a], m, malp, sigmax,
                        kapmax, alpmax);
            const int base = end == 0 ? 0 : nax[a] - np;
            for (int i = 0; i < np; ++i) {
                cH1[a][base + i] = cH1[a][base + i] / kap[i];
                cH2[a][base + i] = cH2[a][base + i] / kap[i];
            }
            free(kap);
        }
    }
    /* psi storage: x slabs [s][0..ny][0..nz], y slabs [0..nx][s][0..nz],
     * z slabs [0..nx][0..ny][s], s in [0, np] */
    for (int f = 0; f < 6; ++f) {
        const int np = P->np[f];
        int64_t n;
        if (f < 2) n = (int64_t)(np + 1) * (o->ny + 1) * (o->nz + 1);
        else if (f < 4) n = (int64_t)(o->nx + 1) * (np + 1) * (o->nz + 1);
        else n = (int64_t)(o->nx + 1) * (o->ny + 1) * (np + 1);
        for (int q = 0; q < 2; ++q) {
            P->qe[f][q] = (double *)zalloc(sizeof(double) * n);
            P->qh[f][q] = (double *)zalloc(sizeof(double) * n);
        }
    }
    P->cpmlE = o->dt / K_EPS0;
    P->cpmlH = o->bH[0];
    P->on = 1;
    return 0;
}

/* psi slab index for face f at global (i,j,k) with slab-local s */
static inline int64_t qidx(const orc *o, int f, int s, int i, int j, int k)
{
    const int np = o->pml.np[f];
    if (f < 2) return ((int64_t)s * (o->ny + 1) + j) * (o->nz + 1) + k;
    if (f < 4) return ((int64_t)i * (np + 1) + s) * (o->nz + 1) + k;
    return ((int64_t)i * (o->ny + 1) + j) * (np + 1) + s;
}

/* Coefficient of a cell's psi term: with literal the reference's single
 * cpmlE = dt/eps0 and cpmlH = bH[0] (CPML.cpp:524-525); otherwise the cell's
 * own curl coefficient -- bE of its medium (C3 on Drude-Lorentz cells), bH
 * of its medium -- which equals the literal values in eps_r = mu_r = 1 media. */
static inline double pml_ce(const orc *o, int64_t g)
{
    if (o->pml.literal) return o->pml.cpmlE;
    const int id = o->id[g];
    return (id == ID_DISPERSIVE && o->dl.on) ? o->dl.C3 : o->bE[id];
}

static inline double pml_ch(const orc *o, int64_t g)
{
    return o->pml.literal ? o->pml.cpmlH : o->bH[o->id[g]];
}

/* CPML::UpdateCPMLEFields, CPML.cpp:529-607 */
void orc_op_e_pml(orc *o)
{
    pml_t *P = &o->pml;
    if (!P->on) return;
    double *Ex = o->F[EX], *Ey = o->F[EY], *Ez = o->F[EZ];
    const double *Hx = o->F[HX], *Hy = o->F[HY], *Hz = o->F[HZ];
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int end = 0; end < 2; ++end) { /* x slabs */
        const int f = FX1 + end, np = P->np[f];
        const double *b = P->bE[f], *c = P->cE[f];
        double *q0 = P->qe[f][0], *q1 = P->qe[f][1];
#pragma omp parallel for schedule(static)
        for (int s = 0; s < np; ++s) {
            const int cs = end == 0 ? s + 1 : s;            /* coefficient index */
            const int i = end == 0 ? s + 1 : nx - np + s;   /* global i */
            for (int j = 1; j < ny; ++j)
                for (int k = 1; k < nz; ++k) {
                    const int64_t g = IDX(o, i, j, k), q = qidx(o, f, cs, i, j, k);
                    q0[q] = b[cs] * q0[q] + c[cs] * (Hz[g] - Hz[g - o->sx]);
                    Ey[g] = Ey[g] - q0[q] * pml_ce(o, g);
                    q1[q] = b[cs] * q1[q] + c[cs] * (Hy[g] - Hy[g - o->sx]);
                    Ez[g] = Ez[g] + q1[q] * pml_ce(o, g);
                }
        }
    }
    for (int end = 0; end < 2; ++end) { /* y slabs */
        const int f = FY1 + end, np = P->np[f];
        const double *b = P->bE[f], *c = P->cE[f];
        double *q0 = P->qe[f][0], *q1 = P->qe[f][1];
#pragma omp parallel for schedule(static)
        for (int i = 1; i < nx; ++i)
            for (int s = 0; s < np; ++s) {
                const int cs = end == 0 ? s + 1 : s;
                const int j = end == 0 ? s + 1 : ny - np + s;
                for (int k = 1; k < nz; ++k) {
                    const int64_t g = IDX(o, i, j, k), q = qidx(o, f, cs, i, j, k);
                    q0[q] = b[cs] * q0[q] + c[cs] * (Hx[g] - Hx[g - o->sy]);
                    Ez[g] = Ez[g] - q0[q] * pml_ce(o, g);
                    q1[q] = b[cs] * q1[q] + c[cs] * (Hz[g] - Hz[g - o->sy]);
                    Ex[g] = Ex[g] + q1[q] * pml_ce(o, g);
                }
            }
    }
    for (int end = 0; end < 2; ++end) { /* z slabs */
        const int f = FZ1 + end, np = P->np[f];
        const double *b = P->bE[f], *c = P->cE[f];
        double *q0 = P->qe[f][0], *q1 = P->qe[f][1];
#pragma omp parallel for schedule(static)
        for (int i = 1; i < nx; ++i)
            for (int j = 1; j < ny; ++j)
                for (int s = 0; s < np; ++s) {
                    const int cs = end == 0 ? s + 1 : s;
                    const int k = end == 0 ? s + 1 : nz - np + s;
                    const int64_t g = IDX(o, i, j, k), q = qidx(o, f, cs, i, j, k);
                    q0[q] = b[cs] * q0[q] + c[cs] * (Hy[g] - Hy[g - 1]);
                    Ex[g] = Ex[g] - q0[q] * pml_ce(o, g);
                    q1[q] = b[cs] * q1[q] + c[cs] * (Hx[g] - Hx[g - 1]);
                    Ey[g] = Ey[g] + q1[q] * pml_ce(o, g);
                }
    }
}

/* CPML::UpdateCPMLHFields, CPML.cpp:609-689 */
void orc_op_h_pml(orc *o)
{
    pml_t *P = &o->pml;
    if (!P->on) return;
    const double *Ex = o->F[EX], *Ey = o->F[EY], *Ez = o->F[EZ];
    double *Hx = o->F[HX], *Hy = o->F[HY], *Hz = o->F[HZ];
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    for (int end = 0; end < 2; ++end) {
        const int f = FX1 + end, np = P->np[f];
        const double *b = P->bH[f], *c = P->cH[f];
        double *q0 = P->qh[f][0], *q1 = P->qh[f][1];
#pragma omp parallel for schedule(static)
        for (int s = 0; s < np; ++s) {
            const int i = end == 0 ? s : nx - np + s;
            for (int j = 0; j < ny; ++j)
                for (int k = 0; k < nz; ++k) {
                    const int64_t g = IDX(o, i, j, k), q = qidx(o, f, s, i, j, k);
                    q0[q] = b[s] * q0[q] + c[s] * (Ez[g + o->sx] - Ez[g]);
                    Hy[g] = Hy[g] + q0[q] * pml_ch(o, g);
                    q1[q] = b[s] * q1[q] + c[s] * (Ey[g + o->sx] - Ey[g]);
                    Hz[g] = Hz[g] - q1[q] * pml_ch(o, g);
                }
        }
    }
    for (int end = 0; end < 2; ++end) {
        const int f = FY1 + end, np = P->np[f];
        const double *b = P->bH[f], *c = P->cH[f];
        double *q0 = P->qh[f][0], *q1 = P->qh[f][1];
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int s = 0; s < np; ++s) {
                const int j = end == 0 ? s : ny - np + s;
                for (int k = 0; k < nz; ++k) {
                    const int64_t g = IDX(o, i, j, k), q = qidx(o, f, s, i, j, k);
                    q0[q] = b[s] * q0[q] + c[s] * (Ex[g + o->sy] - Ex[g]);
                    Hz[g] = Hz[g] - q0[q] * pml_ch(o, g);
                    q1[q] = b[s] * q1[q] + c[s] * (Ez[g + o->sy] - Ez[g]);
                    Hx[g] = Hx[g] + q1[q] * pml_ch(o, g);
                }
            }
    }
    for (int end = 0; end < 2; ++end) {
        const int f = FZ1 + end, np = P->np[f];
        const double *b = P->bH[f], *c = P->cH[f];
        double *q0 = P->qh[f][0], *q1 = P->qh[f][1];
#pragma omp parallel for schedule(static)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int s = 0; s < np; ++s) {
                    const int k = end == 0 ? s : nz - np + s;
                    const int64_t g = IDX(o, i, j, k), q = qidx(o, f, s, i, j, k);
                    q0[q] = b[s] * q0[q] + c[s] * (Ey[g + 1] - Ey[g]);
                    Hx[g] = Hx[g] - q0[q] * pml_ch(o, g);
                    q1[q] = b[s] * q1[q] + c[s] * (Ex[g + 1] - Ex[g]);
                    Hy[g] = Hy[g] + q1[q] * pml_ch(o, g);
                }
    }
}

/* ---------------------------------------------------------- Yee bulk --- */

/* BasicHFieldUpdate, BasicFDTD.cpp:67-84 */
void orc_op_h_bulk(orc *o)
{
    const double *Ex = o->F[EX], *Ey = o->F[EY], *Ez = o->F[EZ];
    double *Hx = o->F[HX], *Hy = o->F[HY], *Hz = o->F[HZ];
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    const int64_t sx = o->sx, sy = o->sy;
#pragma omp parallel for schedule(static)
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k) {
                const int64_t g = IDX(o, i, j, k);
                const int id = o->id[g];
                const double aH = o->aH[id], bH = o->bH[id];
                Hx[g] = aH * Hx[g] - bH * (Ez[g + sy] - Ez[g]) * o->cHxz[j] + bH * (Ey[g + 1] - Ey[g]) * o->cHxy[k];
                Hy[g] = aH * Hy[g] - bH * (Ex[g + 1] - Ex[g]) * o->cHyx[k] + bH * (Ez[g + sx] - Ez[g]) * o->cHyz[i];
                Hz[g] = aH * Hz[g] + bH * (Ex[g + sy] - Ex[g]) * o->cHzx[j] - bH * (Ey[g + sx] - Ey[g]) * o->cHzy[i];
            }
}

/* BasicEFieldUpdate, BasicFDTD.cpp:25-47 */
void orc_op_e_bulk(orc *o)
{
    double *Ex = o->F[EX], *Ey = o->F[EY], *Ez = o->F[EZ];
    const double *Hx = o->F[HX], *Hy = o->F[HY], *Hz = o->F[HZ];
    const int nx = o->nx, ny = o->ny, nz = o->nz;
    const int64_t sx = o->sx, sy = o->sy;
#pragma omp parallel for schedule(static)
    for (int i = 1; i < nx; ++i)
        for (int j = 1; j < ny; ++j)
            for (int k = 1; k < nz; ++k) {
                const int64_t g = IDX(o, i, j, k);
                const int id = o->id[g];
                if (id == ID_PEC) {
                    Ex[g] = 0.0; Ey[g] = 0.0; Ez[g] = 0.0;
                } else if (id != ID_DISPERSIVE) {
                    const double aE = o->aE[id], bE = o->bE[id];
                    Ex[g] = aE * Ex[g] + bE * (Hz[g] - Hz[g - sy]) * o->cExz[j] - bE * (Hy[g] - Hy[g - 1]) * o->cExy[k];
                    Ey[g] = aE * Ey[g] + bE * (Hx[g] - Hx[g - 1]) * o->cEyx[k] - bE * (Hz[g] - Hz[g - sx]) * o->cEyz[i];
                    Ez[g] = aE * Ez[g] + bE * (Hy[g] - Hy[g - sx]) * o->cEzy[i] - bE * (Hx[g] - Hx[g - sy]) * o->cEzx[j];
                }
            }
}

/* ------------------------------------------------------ Drude-Lorentz --- */

int orc_dl_init(orc *o, double sigma, double epsInf, int nD, const double *fD, const double *gD,
                int nL, const double *fL, const double *dL, const double *depsL, int literal)
{
    dl_t *D = &o->dl;
    if (nD < 0 || nL < 0 || nD > MAXP || nL > MAXP) return 1;
    dl_coeffs(D, o->dt, sigma, epsInf, nD, fD, gD, nL, fL, dL, depsL, literal);
    int64_t n = 0;
    for (int i = 1; i < o->nx; ++i)
        for (int j = 1; j < o->ny; ++j)
            for (int k = 1; k < o->nz; ++k)
                if (o->id[IDX(o, i, j, k)] == ID_DISPERSIVE) ++n;
    D->ncell = n;
    D->cell = (int64_t *)zalloc(sizeof(int64_t) * n);
    D->stride = nD + 2 * nL + 1;
    D->state = (double *)zalloc(sizeof(double) * n * 3 * D->stride);
    n = 0;
    for (int i = 1; i < o->nx; ++i)
        for (int j = 1; j < o->ny; ++j)
            for (int k = 1; k < o->nz; ++k)
                if (o->id[IDX(o, i, j, k)] == ID_DISPERSIVE) D->cell[n++] = IDX(o, i, j, k);
    D->on = 1;
    return 0;
}

/* 3-D form of Drude_Lorentz::EFieldUpdate for ID==2 cells; the curl terms
 * are those of BasicFDTD.cpp:39-41 with bE replaced by C3. */
void orc_op_dl(orc *o)
{
    dl_t *D = &o->dl;
    if (!D->on) return;
    double *Ex = o->F[EX], *Ey = o->F[EY], *Ez = o->F[EZ];
    const double *Hx = o->F[HX], *Hy = o->F[HY], *Hz = o->F[HZ];
    const int64_t sx = o->sx, sy = o->sy;
    const double C3 = D->C3;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < D->ncell; ++c) {
        const int64_t g = D->cell[c];
        const int i = (int)(g / sx), j = (int)((g / sy) % (o->ny + 1)), k = (int)(g % sy);
        double *st = D->state + c * 3 * D->stride;
        const double cx = C3 * (Hz[g] - Hz[g - sy]) * o->cExz[j] - C3 * (Hy[g] - Hy[g - 1]) * o->cExy[k];
        const double cy = C3 * (Hx[g] - Hx[g - 1]) * o->cEyx[k] - C3 * (Hz[g] - Hz[g - sx]) * o->cEyz[i];
        const double cz = C3 * (Hy[g] - Hy[g - sx]) * o->cEzy[i] - C3 * (Hx[g] - Hx[g - sy]) * o->cEzx[j];
        Ex[g] = dl_component(D, o->dt, Ex[g], cx, st);
        Ey[g] = dl_component(D, o->dt, Ey[g], cy, st + D->stride);
        Ez[g] = dl_component(D, o->dt, Ez[g], cz, st + 2 * D->stride);
    }
}

/* -------------------------------------------------- four-level gain --- */

int orc_gain_init(orc *o, int gain_id, double lambda_a, double lambda_b, double gamma_a,
                  double gamma_b, double t30, double t32, double t21, double t10, double N_0,
                  double pump_rate)
{
    gain_t *G = &o->gain;
    if (gain_id < 0 || gain_id > 255 || gain_id == ID_DISPERSIVE || gain_id == ID_PEC) return 1;
    G->gain_id = gain_id;
    gain_coeffs(G, o->dt, o->dx, o->dy, lambda_a, lambda_b, gamma_a, gamma_b, t30, t32, t21, t10,
                N_0, pump_rate);
    int64_t n = 0;
    for (int i = 1; i < o->nx; ++i)
        for (int j = 1; j < o->ny; ++j)
            for (int k = 1; k < o->nz; ++k)
                if (o->id[IDX(o, i, j, k)] == gain_id) ++n;
    G->ncell = n;
    G->cell = (int64_t *)zalloc(sizeof(int64_t) * n);
    G->state = (double *)zalloc(sizeof(double) * n * GAIN_WORDS);
    n = 0;
    for (int i = 1; i < o->nx; ++i)
        for (int j = 1; j < o->ny; ++j)
            for (int k = 1; k < o->nz; ++k)
                if (o->id[IDX(o, i, j, k)] == gain_id) {
                    gain_site_init(G->state + n * GAIN_WORDS);
                    G->cell[n++] = IDX(o, i, j, k);
                }
    G->on = 1;
    return 0;
}

void orc_op_gain_p(orc *o)
{
    gain_t *G = &o->gain;
    if (!G->on) return;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < G->ncell; ++c) {
        const int64_t g = G->cell[c];
        const double E[3] = {o->F[EX][g], o->F[EY][g], o->F[EZ][g]};
        gain_site_p(G, G->state + c * GAIN_WORDS, E, 3);
    }
}

void orc_op_gain_e(orc *o)
{
    gain_t *G = &o->gain;
    if (!G->on) return;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < G->ncell; ++c) {
        const int64_t g = G->cell[c];
        double E[3] = {o->F[EX][g], o->F[EY][g], o->F[EZ][g]};
        gain_site_e(G, G->state + c * GAIN_WORDS, E, 3);
        o->F[EX][g] = E[0]; o->F[EY][g] = E[1]; o->F[EZ][g] = E[2];
    }
}

void orc_op_gain_n(orc *o)
{
    gain_t *G = &o->gain;
    if (!G->on) return;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < G->ncell; ++c) {
        const int64_t g = G->cell[c];
        const double E[3] = {o->F[EX][g], o->F[EY][g], o->F[EZ][g]};
        gain_site_n(G, G->state + c * GAIN_WORDS, E, 3);
    }
}

int orc_gain_populations(const orc *o, double *out)
{
    const gain_t *G = &o->gain;
    if (!G->on) return 1;
    for (int64_t c = 0; c < G->ncell; ++c)
        for (int q = 0; q < 4; ++q) out[c * 4 + q] = G->state[c * GAIN_WORDS + GS_N + q];
    return 0;
}

/* ------------------------------------------------- three-level gain --- */

/* ThreeLevel::ThreeLevel (ThreeLevel.cpp:29-209) with the "cells" placement:
 * the E-range cells of ID gain_id (the reference's extra site past the list,
 * :147-149, sits at (Nx, Ny) where E stays zero, and is left out) */
int orc_three_init(orc *o, int gain_id, double lambda_a, double lambda_b, double gamma_a, double gamma_b,
                   double t20, double t21, double t10, double N_0, int literal)
{
    three_t *T3 = &o->three;
    if (gain_id < 0 || gain_id > 255 || gain_id == ID_DISPERSIVE || gain_id == ID_PEC || o->gain.on) return 1;
    T3->gain_id = gain_id;
    three_coeffs(T3, o->dt, lambda_a, lambda_b, gamma_a, gamma_b, t20, t21, t10, N_0, literal);
    int64_t n = 0;
    for (int i = 1; i < o->nx; ++i)
        for (int j = 1; j < o->ny; ++j)
            for (int k = 1; k < o->nz; ++k)
                if (o->id[IDX(o, i, j, k)] == gain_id) ++n;
    T3->ncell = n;
    T3->cell = (int64_t *)zalloc(sizeof(int64_t) * n);
    T3->state = (double *)zalloc(sizeof(double) * n * THREE_WORDS);
    n = 0;
    for (int i = 1; i < o->nx; ++i)
        for (int j = 1; j < o->ny; ++j)
            for (int k = 1; k < o->nz; ++k)
                if (o->id[IDX(o, i, j, k)] == gain_id) {
                    three_site_init(T3->state + n * THREE_WORDS, N_0);
                    T3->cell[n++] = IDX(o, i, j, k);
                }
    T3->on = 1;
    return 0;
}

void orc_op_three_p(orc *o)
{
    three_t *T3 = &o->three;
    if (!T3->on) return;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < T3->ncell; ++c) {
        const int64_t g = T3->cell[c];
        const double E[3] = {o->F[EX][g], o->F[EY][g], o->F[EZ][g]};
        three_site_p(T3, T3->state + c * THREE_WORDS, E, 3);
    }
}

void orc_op_three_e(orc *o)
{
    three_t *T3 = &o->three;
    if (!T3->on) return;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < T3->ncell; ++c) {
        const int64_t g = T3->cell[c];
        double E[3] = {o->F[EX][g], o->F[EY][g], o->F[EZ][g]};
        three_site_e(T3, T3->state + c * THREE_WORDS, E, 3);
        o->F[EX][g] = E[0]; o->F[EY][g] = E[1]; o->F[EZ][g] = E[2];
    }
}

void orc_op_three_n(orc *o)
{
    three_t *T3 = &o->three;
    if (!T3->on) return;
#pragma omp parallel for schedule(static)
    for (int64_t c = 0; c < T3->ncell; ++c) {
        const int64_t g = T3->cell[c];
        const double E[3] = {o->F[EX][g], o->F[EY][g], o->F[EZ][g]};
        three_site_n(T3, T3->state + c * THREE_WORDS, E, 3);
    }
}

/* N0 N1 N2 per site, sites in [i][j][k] order */
int orc_three_populations(const orc *o, double *out)
{
    const three_t *T3 = &o->three;
    if (!T3->on) return 1;
    for (int64_t c = 0; c < T3->ncell; ++c)
        for (int q = 0; q < 3; ++q) out[c * 3 + q] = T3->state[c * THREE_WORDS + TS_N0 + q];
    return 0;
}

int64_t orc_count_cells(const orc *o, int which)
{
    return which == 0 ? o->dl.ncell : which == 1 ? o->gain.ncell : o->three.ncell;
}

/* ------------------------------------------------------------- TF/SF --- */

/* Gaussian-beam profile and retarded delay of one boundary point:
 * the per-point block repeated through TF_SF.cpp:148-887. */
static void tfsf_point(double x, double y, double z, double kx, double ky, double kz,
                       double kabs, double w0, double z0, double zR, double l0, double dt,
                       double *delay, double *profile)
{
    const double r2 = x * x + y * y + z * z;
    double r_dot_k = (x * kx + y * ky + z * kz) / kabs;
    const double rho2 = r2 - r_dot_k * r_dot_k;
    r_dot_k = r_dot_k - z0;
    const double wz = w0 * sqrt(1 + r_dot_k * r_dot_k / (zR * zR));
    *profile = exp(-rho2 / wz / wz);
    *delay = ((x * kx + y * ky + z * kz) / K_C - l0) / dt;
}

/* Incident waveform tables, TF_SF.cpp:898-955 */
static void tfsf_tables(double *einc, double *hinc, int Nt, double lambda, double dlambda,
                        double dt, int cwmode)
{
    const double nu = K_C / lambda;
    const double T = 1.0 / nu;
    const int nT = (int)(T / dt);
    const double dnu = K_C / (lambda - dlambda / 2.0) - K_C / (lambda + dlambda / 2.0);
    const double domega = 2.0 * K_PI * dnu;
    const double sig = domega * domega / (16 * log(2));
    if (cwmode) {
        const int nd = 5 * nT;
        for (int n = 0; n < nd && n <= Nt; ++n) {
            einc[n] = exp(-((n * dt) - 5.0 * T) * ((n * dt) - 5 * T) / (4.0 * T * T)) * sin(2.0 * K_PI * nu * (n * dt));
            hinc[n] = exp(-((n * dt + dt / 2.0) - 5.0 * T) * ((n * dt + dt / 2.0) - 5 * T) / (4.0 * T * T)) * sin(2.0 * K_PI * nu * (n * dt + dt / 2.0));
        }
        for (int n = nd; n <= Nt; ++n) {
            einc[n] = sin(2.0 * K_PI * nu * (n * dt));
            hinc[n] = sin(2.0 * K_PI * nu * (n * dt + dt / 2.0));
        }
    } else {
        const double t0 = 5 * T;
        for (int n = 0; n <= Nt; ++n) {
            einc[n] = exp(-sig * ((double)n * dt - t0) * ((double)n * dt - t0)) * sin(2.0 * K_PI * nu * ((double)n * dt - t0));
            hinc[n] = exp(-sig * ((double)n * dt + dt / 2.0 - t0) * ((double)n * dt + dt / 2.0 - t0)) * sin(2.0 * K_PI * nu * ((double)n * dt + dt / 2.0 - t0));
        }
    }
}

int orc_tfsf_init(orc *o, const orc_tfsf_params *p)
{
    tfsf_t *S = &o->tfsf;
    const double dx = o->dx, dy = o->dy, dz = o->dz, dt = o->dt;
    const double theta = p->theta_deg * K_PI / 180.0, phi = p->phi_deg * K_PI / 180.0;
    const double psi = p->psi_deg * K_PI / 180.0, E0 = p->E0;
    const int i0 = p->i0, j0 = p->j0, k0 = p->k0;
    S->i1 = p->n_x1; S->i2 = o->nx - p->n_x2;
    S->j1 = p->n_y1; S->j2 = o->ny - p->n_y2;
    S->k1 = p->n_z1; S->k2 = o->nz - p->n_z2;
    const int i1 = S->i1, i2 = S->i2, j1 = S->j1, j2 = S->j2, k1 = S->k1, k2 = S->k2;
    if (i1 < 1 || j1 < 1 || k1 < 1 || i2 + 1 > o->nx - 1 || j2 + 1 > o->ny - 1 || k2 + 1 > o->nz - 1 ||
        i2 <= i1 || j2 <= j1 || k2 <= k1 || p->Nt < 1)
        return 1;
    const double eta0 = sqrt(K_MU0 / K_EPS0);
    /* Taflove polarisation, TF_SF.cpp:112-117 */
    const double E0x = E0 * (cos(psi) * sin(phi) - sin(psi) * cos(theta) * cos(phi));
    const double E0y = E0 * (-cos(psi) * cos(phi) - sin(psi) * cos(theta) * sin(phi));
    const double E0z = E0 * sin(psi) * sin(theta);
    const double H0x = E0 / eta0 * (sin(psi) * sin(phi) + cos(psi) * cos(theta) * cos(phi));
    const double H0y = E0 / eta0 * (-sin(psi) * cos(phi) + cos(psi) * cos(theta) * sin(phi));
    const double H0z = -E0 / eta0 * cos(psi) * sin(theta);
    const double kx = sin(theta) * cos(phi), ky = sin(theta) * sin(phi), kz = cos(theta);
    const double kabs = sqrt(kx * kx + ky * ky + kz * kz);
    /* earliest corner delay, TF_SF.cpp:124-138 */
    const int ci[2] = {i1, i2}, cj[2] = {j1, j2}, ck[2] = {k1, k2};
    double l0 = 0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) {
                const double v = (kx * (ci[a] - i0) * dx + ky * (cj[b] - j0) * dy + kz * (ck[c] - k0) * dz) / K_C;
                if ((a | b | c) == 0 || l0 > v) l0 = v;
            }
    const double zR = K_PI * p->w0 * p->w0 / p->lambda;
    /* face tables: y faces (u=i, v=k), x faces (u=j, v=k), z faces (u=i, v=j) */
    for (int f = 0; f < 6; ++f) {
        face_t *F = &S->face[f];
        const int ax = f / 2; /* 0: x faces, 1: y faces, 2: z faces (FX1..FZ2) */
        if (ax == 0) { F->u1 = j1; F->u2 = j2; F->v1 = k1; F->v2 = k2; }
        else if (ax == 1) { F->u1 = i1; F->u2 = i2; F->v1 = k1; F->v2 = k2; }
        else { F->u1 = i1; F->u2 = i2; F->v1 = j1; F->v2 = j2; }
        const int nu = F->u2 - F->u1 + 1, nv = F->v2 - F->v1 + 1;
        F->dE = (double *)zalloc(sizeof(double) * nu * nv); F->pE = (double *)zalloc(sizeof(double) * nu * nv);
        F->dH = (double *)zalloc(sizeof(double) * nu * nv); F->pH = (double *)zalloc(sizeof(double) * nu * nv);
        const int far = f & 1;
        for (int u = F->u1; u <= F->u2; ++u)
            for (int v = F->v1; v <= F->v2; ++v) {
                double xE, yE, zE, xH, yH, zH;
                if (ax == 0) {
                    const int i = far ? i2 : i1, j = u, k = v;
                    xE = dx * (far ? (i - i0 + 0.5) : (i - i0 - 0.5)); yE = dy * (j - j0); zE = dz * (k - k0);
                    xH = dx * (i - i0); yH = yE; zH = zE;
                } else if (ax == 1) {
                    const int i = u, j = far ? j2 : j1, k = v;
                    xE = dx * (i - i0); yE = dy * (far ? (j - j0 + 0.5) : (j - j0 - 0.5)); zE = dz * (k - k0);
                    xH = xE; yH = dy * (j - j0); zH = zE;
                } else {
                    const int i = u, j = v, k = far ? k2 : k1;
                    xE = dx * (i - i0); yE = dy * (j - j0); zE = dz * (far ? (k - k0 + 0.5) : (k - k0 - 0.5));
                    xH = xE; yH = yE; zH = dz * (k - k0);
                }
                const int64_t t = (int64_t)(u - F->u1) * nv + (v - F->v1);
                tfsf_point(xE, yE, zE, kx, ky, kz, kabs, p->w0, p->z0, zR, l0, dt, &F->dE[t], &F->pE[t]);
                tfsf_point(xH, yH, zH, kx, ky, kz, kabs, p->w0, p->z0, zR, l0, dt, &F->dH[t], &F->pH[t]);
            }
    }
    const double CEx = dt / (K_EPS0 * dx), CEy = dt / (K_EPS0 * dy), CEz = dt / (K_EPS0 * dz);
    const double CHx = dt / (K_MU0 * dx), CHy = dt / (K_MU0 * dy), CHz = dt / (K_MU0 * dz);
    /* signed coefficients, TF_SF.cpp:988-1089 (E) and 1201-1300 (H).
     * E1/H1 and E2/H2 components per face: x faces (Ey|Hz, Ez|Hy),
     * y faces (Ex|Hz, Ez|Hx), z faces (Ex|Hy, Ey|Hx). */
    S->cE[FX1][0] = CEx * H0z;  S->cE[FX1][1] = -(CEx * H0y);
    S->cE[FX2][0] = -(CEx * H0z); S->cE[FX2][1] = CEx * H0y;
    S->cE[FY1][0] = -(CEy * H0z); S->cE[FY1][1] = CEy * H0x;
    S->cE[FY2][0] = CEy * H0z;  S->cE[FY2][1] = -(CEy * H0x);
    S->cE[FZ1][0] = CEz * H0y;  S->cE[FZ1][1] = -(CEz * H0x);
    S->cE[FZ2][0] = -(CEz * H0y); S->cE[FZ2][1] = CEz * H0x;
    S->cH[FX1][0] = CHx * E0y;  S->cH[FX1][1] = -(CHx * E0z);
    S->cH[FX2][0] = -(CHx * E0y); S->cH[FX2][1] = CHx * E0z;
    S->cH[FY1][0] = -(CHy * E0x); S->cH[FY1][1] = CHy * E0z;
    S->cH[FY2][0] = CHy * E0x;  S->cH[FY2][1] = -(CHy * E0z);
    S->cH[FZ1][0] = CHz * E0x;  S->cH[FZ1][1] = -(CHz * E0y);
    S->cH[FZ2][0] = -(CHz * E0x); S->cH[FZ2][1] = CHz * E0y;
    S->Nt = p->Nt;
    free(S->einc); free(S->hinc);
    S->einc = (double *)zalloc(sizeof(double) * (p->Nt + 2));
    S->hinc = (double *)zalloc(sizeof(double) * (p->Nt + 2));
    tfsf_tables(S->einc, S->hinc, p->Nt, p->lambda, p->dlambda, dt, p->cwmode);
    S->on = 1;
    return 0;
}

int orc_tfsf_set_tables(orc *o, int n, const double *einc, const double *hinc)
{
    tfsf_t *S = &o->tfsf;
    if (!S->on || n != S->Nt + 1) return 1;
    memcpy(S->einc, einc, sizeof(double) * n);
    memcpy(S->hinc, hinc, sizeof(double) * n);
    return 0;
}

int orc_tfsf_tables(const orc *o, double *einc, double *hinc)
{
    const tfsf_t *S = &o->tfsf;
    if (!S->on) return 1;
    memcpy(einc, S->einc, sizeof(double) * (S->Nt + 1));
    memcpy(hinc, S->hinc, sizeof(double) * (S->Nt + 1));
    return 0;
}

/* TF_SF::Einc_onPoint / Hinc_onPoint, TF_SF.cpp:966-986.  Indices past the
 * end of the table read 0 (the reference reads beyond its allocation). */
static inline double tfsf_lookup(const double *tab, int Nt, double retarded)
{
    if (retarded <= 0) return 0.0;
    const double fl = floor(retarded);
    const double resid = retarded - fl;
    const long n = (long)fl;
    const double a = n <= Nt ? tab[n] : 0.0;
    const double b = n + 1 <= Nt ? tab[n + 1] : 0.0;
    return ((1.0 - resid) * a + resid * b);
}

/* target component and ranges of correction `which` (0: E1/H1, 1: E2/H2) on
 * face f: component index, whether it spans the closed u range, closed v range */
static void tfsf_target(int f, int which, int isH, int *comp)
{
    static const int cE[3][2] = {{EY, EZ}, {EX, EZ}, {EX, EY}};
    static const int cH[3][2] = {{HZ, HY}, {HZ, HX}, {HY, HX}};
    *comp = isH ? cH[f / 2][which] : cE[f / 2][which];
}

/* Apply the E (isH=0) or H (isH=1) corrections of all faces, in the
 * reference's face order y1, y2, x1, x2, z1, z2. */
static void tfsf_apply(orc *o, int n, int isH)
{
    tfsf_t *S = &o->tfsf;
    if (!S->on) return;
    static const int order[6] = {FY1, FY2, FX1, FX2, FZ1, FZ2};
    for (int oi = 0; oi < 6; ++oi) {
        const int f = order[oi], ax = f / 2, far = f & 1;
        const face_t *F = &S->face[f];
        const int nv = F->v2 - F->v1 + 1;
        for (int which = 0; which < 2; ++which) {
            int comp;
            tfsf_target(f, which, isH, &comp);
            /* E1 covers u in [u1,u2), v in [v1,v2]; E2 covers [u1,u2] x [v1,v2).
             * H on x faces covers only [u1,u2) x [v1,v2): the reference applies
             * the x-face H strips with unset point members (TF_SF.cpp:1244-1251,
             * 1260-1267), which read as zero. */
            int ue = which == 0 ? F->u2 - 1 : F->u2;
            int ve = which == 0 ? F->v2 : F->v2 - 1;
            if (isH && ax == 0) { ue = F->u2 - 1; ve = F->v2 - 1; }
            const double coef = isH ? S->cH[f][which] : S->cE[f][which];
            double *fld = o->F[comp];
            const double *tab = isH ? S->einc : S->hinc;
            const double *dl = isH ? F->dH : F->dE, *pr = isH ? F->pH : F->pE;
            for (int u = F->u1; u <= ue; ++u)
                for (int v = F->v1; v <= ve; ++v) {
                    int i, j, k;
                    if (ax == 0) { i = far ? S->i2 : S->i1; j = u; k = v; if (isH) i += far ? 1 : -1; }
                    else if (ax == 1) { i = u; j = far ? S->j2 : S->j1; k = v; if (isH) j += far ? 1 : -1; }
                    else { i = u; j = v; k = far ? S->k2 : S->k1; if (isH) k += far ? 1 : -1; }
                    const int64_t t = (int64_t)(u - F->u1) * nv + (v - F->v1);
                    const int64_t g = IDX(o, i, j, k);
                    fld[g] = fld[g] + coef * tfsf_lookup(tab, S->Nt, (double)n - dl[t]) * pr[t];
                }
        }
    }
}

void orc_op_tfsf_h(orc *o, int n) { tfsf_apply(o, n, 1); }
void orc_op_tfsf_e(orc *o, int n) { tfsf_apply(o, n, 0); }

/* ------------------------------------------------------ point sources --- */

int orc_source_add(orc *o, int comp, int i, int j, int k, const double *wave, int nwave)
{
    if (comp < 0 || comp > 5 || i < 0 || j < 0 || k < 0 || i > o->nx || j > o->ny || k > o->nz || nwave < 1)
        return 1;
    o->src = (src_t *)realloc(o->src, sizeof(src_t) * (o->nsrc + 1));
    src_t *s = &o->src[o->nsrc++];
    s->comp = comp; s->idx = IDX(o, i, j, k); s->n = nwave;
    s->wave = (double *)zalloc(sizeof(double) * nwave);
    memcpy(s->wave, wave, sizeof(double) * nwave);
    return 0;
}

/* Additive source F += wave[n], as the commented injection at main.cpp:284-286 */
void orc_op_sources(orc *o, int n)
{
    for (int s = 0; s < o->nsrc; ++s) {
        const src_t *S = &o->src[s];
        if (n >= 0 && n < S->n) o->F[S->comp][S->idx] = o->F[S->comp][S->idx] + S->wave[n];
    }
}

/* -------------------------------------------------------------- ports --- */

int orc_port_add(orc *o, int npts, const int32_t *ijk)
{
    if (npts < 1) return -1;
    for (int p = 0; p < npts; ++p) {
        const int i = ijk[3 * p], j = ijk[3 * p + 1], k = ijk[3 * p + 2];
        if (i < 0 || j < 0 || k < 0 || i > o->nx || j > o->ny || k > o->nz) return -1;
    }
    o->port = (port_t *)realloc(o->port, sizeof(port_t) * (o->nport + 1));
    port_t *P = &o->port[o->nport];
    memset(P, 0, sizeof(*P));
    P->npts = npts;
    P->idx = (int64_t *)zalloc(sizeof(int64_t) * npts);
    P->sample = (double *)zalloc(sizeof(double) * npts * 6);
    for (int p = 0; p < npts; ++p) P->idx[p] = IDX(o, ijk[3 * p], ijk[3 * p + 1], ijk[3 * p + 2]);
    return o->nport++;
}

int orc_port_set_dft(orc *o, int port, int nfreq, const double *freq_hz, uint32_t comp_mask)
{
    if (port < 0 || port >= o->nport || nfreq < 1 || (comp_mask & 63u) == 0) return 1;
    port_t *P = &o->port[port];
    P->nfreq = nfreq;
    P->mask = comp_mask & 63u;
    P->ncomp = 0;
    for (int c = 0; c < 6; ++c)
        if (P->mask & (1u << c)) P->comps[P->ncomp++] = c;
    free(P->omega); free(P->acc);
    P->omega = (double *)zalloc(sizeof(double) * nfreq);
    for (int f = 0; f < nfreq; ++f) P->omega[f] = 2.0 * K_PI * freq_hz[f];
    P->acc = (double *)zalloc(sizeof(double) * (size_t)P->npts * P->ncomp * nfreq * 2);
    return 0;
}

/* Update_Fields_on_Port (Ports.cpp:88-99, 342-353), then the running DFT:
 * acc += s * exp(-i w t), t = n dt for E and (n - 1/2) dt for H. */
void orc_op_ports(orc *o, int n)
{
    for (int p = 0; p < o->nport; ++p) {
        port_t *P = &o->port[p];
        for (int q = 0; q < P->npts; ++q)
            for (int c = 0; c < 6; ++c) P->sample[q * 6 + c] = o->F[c][P->idx[q]];
        if (!P->nfreq) continue;
#pragma omp parallel for schedule(static)
        for (int q = 0; q < P->npts; ++q)
            for (int ci = 0; ci < P->ncomp; ++ci) {
                const int c = P->comps[ci];
                const double t = c < 3 ? (double)n * o->dt : ((double)n - 0.5) * o->dt;
                const double s = P->sample[q * 6 + c];
                double *acc = P->acc + ((size_t)q * P->ncomp + ci) * P->nfreq * 2;
                for (int f = 0; f < P->nfreq; ++f) {
                    const double ph = P->omega[f] * t;
                    acc[2 * f] += s * cos(ph);
                    acc[2 * f + 1] -= s * sin(ph);
                }
            }
    }
}

int orc_port_read(const orc *o, int port, double *out)
{
    if (port < 0 || port >= o->nport) return 1;
    memcpy(out, o->port[port].sample, sizeof(double) * 6 * o->port[port].npts);
    return 0;
}

int orc_port_dft_read(const orc *o, int port, double *out)
{
    if (port < 0 || port >= o->nport || !o->port[port].nfreq) return 1;
    const port_t *P = &o->port[port];
    memcpy(out, P->acc, sizeof(double) * (size_t)P->npts * P->ncomp * P->nfreq * 2);
    return 0;
}

/* --------------------------------------------------------- time step --- */

void orc_set_step(orc *o, int64_t n) { o->step = n; }
int64_t orc_get_step(const orc *o) { return o->step; }

/* One step in the order of main.cpp:267-344 with the TF/SF, gain and source
 * calls at their (commented) positions. */
void orc_step(orc *o, int nsteps)
{
    for (int s = 0; s < nsteps; ++s) {
        const int n = (int)o->step;
        orc_op_h_bulk(o);
        orc_op_tfsf_h(o, n);
        orc_op_h_pml(o);
        orc_op_e_bulk(o);
        orc_op_dl(o);
        orc_op_gain_p(o);
        orc_op_gain_e(o);
        orc_op_gain_n(o);
        orc_op_three_p(o);
        orc_op_three_e(o);
        orc_op_three_n(o);
        orc_op_tfsf_e(o, n);
        orc_op_sources(o, n);
        orc_op_e_pml(o);
        orc_op_ports(o, n);
        o->step++;
    }
}

int orc_get_field(const orc *o, int comp, double *out)
{
    if (comp < 0 || comp > 5) return 1;
    memcpy(out, o->F[comp], sizeof(double) * o->ncell);
    return 0;
}

int orc_set_field(orc *o, int comp, const double *in)
{
    if (comp < 0 || comp > 5) return 1;
    memcpy(o->F[comp], in, sizeof(double) * o->ncell);
    return 0;
}

/* which: 0..11 = cExy cEyx cEzx cExz cEzy cEyz cHxy cHyx cHzx cHxz cHzy cHyz */
int orc_get_stretch(const orc *o, int which, double *out)
{
    const double *a[12] = {o->cExy, o->cEyx, o->cEzx, o->cExz, o->cEzy, o->cEyz,
                           o->cHxy, o->cHyx, o->cHzx, o->cHxz, o->cHzy, o->cHyz};
    const int n[12] = {o->nz, o->nz, o->ny, o->ny, o->nx, o->nx, o->nz, o->nz, o->ny, o->ny, o->nx, o->nx};
    if (which < 0 || which > 11) return 1;
    memcpy(out, a[which], sizeof(double) * n[which]);
    return 0;
}

/* ------------------------------------------------------- 2-D TE pins --- */

/* Runs the 2-D TE problem that oracle/ref2d_harness.cpp runs through the
 * reference classes: per step a TE H update, a source on Hz, the E update
 * (Drude_Lorentz::EFieldUpdate's whole-grid form when use_dl, else a plain
 * TE update), then the gain P -> E -> N updates on ID==5 sites. */
int orc2d_run(int nx, int ny, double dx, double dy, double dt, const uint8_t *ids2d, int nmedia,
              const double *epsR, const double *muR, const double *sig, const double *sigM,
              int use_dl, double dl_sigma, double dl_epsInf, int nD, const double *fD,
              const double *gD, int nL, const double *fL, const double *dL, const double *depsL,
              int dl_literal, int use_gain, const double *gp, int si, int sj, const double *wave,
              int nsteps, double *Ex, double *Ey, double *Hz)
{
    const int64_t n2 = (int64_t)(nx + 1) * (ny + 1);
#define I2(i, j) ((int64_t)(i) * (ny + 1) + (j))
    double aE[256], bE[256], aH[256], bH[256];
    if (nmedia < 1 || nmedia > 256) return 1;
    for (int m = 0; m < nmedia; ++m) {
        aE[m] = (2.0 * K_EPS0 * epsR[m] - sig[m] * dt) / (2.0 * K_EPS0 * epsR[m] + sig[m] * dt);
        bE[m] = (2.0 * dt) / (2.0 * K_EPS0 * epsR[m] + sig[m] * dt);
        aH[m] = (2.0 * K_MU0 * muR[m] - sigM[m] * dt) / (2.0 * K_MU0 * muR[m] + sigM[m] * dt);
        bH[m] = (2.0 * dt) / (2.0 * K_MU0 * muR[m] + sigM[m] * dt);
    }
    const double cx = 1.0 / dx, cy = 1.0 / dy;
    memset(Ex, 0, sizeof(double) * n2); memset(Ey, 0, sizeof(double) * n2); memset(Hz, 0, sizeof(double) * n2);
    dl_t D; memset(&D, 0, sizeof(D));
    double *dls = NULL;
    if (use_dl) {
        dl_coeffs(&D, dt, dl_sigma, dl_epsInf, nD, fD, gD, nL, fL, dL, depsL, dl_literal);
        D.stride = nD + 2 * nL + 1;
        dls = (double *)zalloc(sizeof(double) * n2 * 2 * D.stride);
    }
    gain_t G; memset(&G, 0, sizeof(G));
    three_t T3; memset(&T3, 0, sizeof(T3));
    int64_t ng = 0;
    int64_t *gcell = NULL;
    double *gst = NULL;
    const int words = use_gain == 2 ? THREE_WORDS : GAIN_WORDS;
    if (use_gain == 2) {
        /* gp: lambda_a lambda_b gamma_a gamma_b t20 t21 t10 N_0 literal */
        three_coeffs(&T3, dt, gp[0], gp[1], gp[2], gp[3], gp[4], gp[5], gp[6], gp[7], (int)gp[8]);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                if (ids2d[I2(i, j)] == 5) ++ng;
        gcell = (int64_t *)zalloc(sizeof(int64_t) * (ng + 1));
        gst = (double *)zalloc(sizeof(double) * (ng + 1) * THREE_WORDS);
        ng = 0;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                if (ids2d[I2(i, j)] == 5) { three_site_init(gst + ng * THREE_WORDS, gp[7]); gcell[ng++] = I2(i, j); }
    } else if (use_gain) {
        gain_coeffs(&G, dt, dx, dy, gp[0], gp[1], gp[2], gp[3], gp[4], gp[5], gp[6], gp[7], gp[8], gp[9]);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                if (ids2d[I2(i, j)] == 5) ++ng;
        gcell = (int64_t *)zalloc(sizeof(int64_t) * (ng + 1));
        gst = (double *)zalloc(sizeof(double) * (ng + 1) * GAIN_WORDS);
        ng = 0;
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                if (ids2d[I2(i, j)] == 5) { gain_site_init(gst + ng * GAIN_WORDS); gcell[ng++] = I2(i, j); }
    }
    for (int n = 0; n < nsteps; ++n) {
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                const int id = ids2d[I2(i, j)];
                Hz[I2(i, j)] = aH[id] * Hz[I2(i, j)] + bH[id] * (Ex[I2(i, j + 1)] - Ex[I2(i, j)]) * cy - bH[id] * (Ey[I2(i + 1, j)] - Ey[I2(i, j)]) * cx;
            }
        Hz[I2(si, sj)] = Hz[I2(si, sj)] + wave[n];
        int64_t dlc = 0;
        for (int i = 1; i < nx; ++i)
            for (int j = 1; j < ny; ++j) {
                const int64_t g = I2(i, j);
                const int id = ids2d[g];
                if (use_dl && id == ID_DISPERSIVE) {
                    double *st = dls + dlc * 2 * D.stride;
                    Ex[g] = dl_component(&D, dt, Ex[g], D.C3 * (Hz[g] - Hz[g - 1]) * cy, st);
                    Ey[g] = dl_component(&D, dt, Ey[g], -(D.C3 * (Hz[g] - Hz[g - (ny + 1)]) * cx), st + D.stride);
                    ++dlc;
                } else if (id == ID_PEC) {
                    Ex[g] = 0.0; Ey[g] = 0.0;
                } else {
                    Ex[g] = aE[id] * Ex[g] + bE[id] * (Hz[g] - Hz[g - 1]) * cy;
                    Ey[g] = aE[id] * Ey[g] - bE[id] * (Hz[g] - Hz[g - (ny + 1)]) * cx;
                }
            }
        if (use_dl) { /* boundary lines of Drude_Lorentz.cpp:219-226 */
            for (int j = 1; j < ny; ++j) Ex[I2(0, j)] = aE[0] * Ex[I2(0, j)] + bE[0] * (Hz[I2(0, j)] - Hz[I2(0, j - 1)]) * cy;
            for (int i = 1; i < nx; ++i) Ey[I2(i, 0)] = aE[0] * Ey[I2(i, 0)] - bE[0] * (Hz[I2(i, 0)] - Hz[I2(i - 1, 0)]) * cx;
        }
        if (use_gain == 2) {
            for (int64_t c = 0; c < ng; ++c) {
                double E[3] = {Ex[gcell[c]], Ey[gcell[c]], 0.0};
                three_site_p(&T3, gst + c * words, E, 2);
            }
            for (int64_t c = 0; c < ng; ++c) {
                double E[3] = {Ex[gcell[c]], Ey[gcell[c]], 0.0};
                three_site_e(&T3, gst + c * words, E, 2);
                Ex[gcell[c]] = E[0]; Ey[gcell[c]] = E[1];
            }
            for (int64_t c = 0; c < ng; ++c) {
                double E[3] = {Ex[gcell[c]], Ey[gcell[c]], 0.0};
                three_site_n(&T3, gst + c * words, E, 2);
            }
        } else if (use_gain) {
            for (int64_t c = 0; c < ng; ++c) {
                double E[3] = {Ex[gcell[c]], Ey[gcell[c]], 0.0};
                gain_site_p(&G, gst + c * GAIN_WORDS, E, 2);
            }
            for (int64_t c = 0; c < ng; ++c) {
                double E[3] = {Ex[gcell[c]], Ey[gcell[c]], 0.0};
                gain_site_e(&G, gst + c * GAIN_WORDS, E, 2);
                Ex[gcell[c]] = E[0]; Ey[gcell[c]] = E[1];
            }
            for (int64_t c = 0; c < ng; ++c) {
                double E[3] = {Ex[gcell[c]], Ey[gcell[c]], 0.0};
                gain_site_n(&G, gst + c * GAIN_WORDS, E, 2);
            }
        }
    }
    free(dls); free(gcell); free(gst);
#undef I2
    return 0;
}
