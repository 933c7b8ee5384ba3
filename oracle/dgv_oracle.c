/*
 * dgv_oracle.c -- CPU FP64 restatement of the reference's collision hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see dgv_oracle.h).  Every routine follows the
 * reference routine cited beside it operation by operation, including the
 * left-to-right evaluation order of Fortran expressions, so that floating-point
 * results can be compared tightly.  Compiled with -ffp-contract=off so that the
 * compiler does not fuse multiply-adds the Fortran source writes separately.
 *
 * Parity unpinned against reference outputs (the Fortran cannot be built here
 * and the reference has no golden vectors); see dgv_oracle.h for the
 * invariants that pin it instead.
 */
#include "dgv_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PI_REF 3.141592653589793238462643 /* pi25DT, dgvtools_mod.f90:386 */

struct dgvo_ctx {
    dgvo_grid_desc d;
    int32_t P, Nc;
    int64_t N;
    double *gu, *gv, *gw;                 /* 1-D grids, M+1 points          */
    double *xu, *wu, *xv, *wv, *xw, *ww;  /* Gauss nodes / weights per axis */
    double *clu, *cru, *clv, *crv, *clw, *crw;
    int32_t *cug, *cvg, *cwg;             /* cell integer coordinates       */
    double *nu, *nv, *nw, *nwt;           /* node coordinates and weights   */
    int32_t *npc, *nui, *nvi, *nwi;       /* parent cell, local indices     */
    int32_t ccell;                        /* canonical cell                 */
    /* A-arrays, reference layout, 0-based */
    int64_t nnz;
    int32_t *capphi;
    double *A;
    int32_t *xi, *xi1;
    /* shift tables, SetCellsUGINdsSftArrs */
    int32_t *dui, *dvi, *dwi, *phican;
    int64_t *Ashift;
};

/* ------------------------------------------------------------------------- */
/* Gauss-Legendre nodes on [-1,1], ascending.  Newton iteration on the        */
/* three-term Legendre recurrence; the reference takes the same rule from     */
/* Numerical Recipes' GauLeg (gaussian_mod.f90:4-54, called miscset.f90:80-100).*/
void dgvo_gauss_legendre(int n, double *x, double *w)
{
    if (n == 1) { x[0] = 0.0; w[0] = 2.0; return; }   /* miscset.f90:77-78 */
    int half = (n + 1) / 2;
    for (int i = 0; i < half; i++) {
        double z = cos(PI_REF * (i + 0.75) / (n + 0.5));
        double dp = 0.0;
        for (int it = 0; it < 100; it++) {
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1; p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
            double dz = p1 / dp;
            z -= dz;
            if (fabs(dz) < 1e-16) break;
        }
        {   /* one more evaluation at the converged root for the weight */
            double p0 = 1.0, p1 = z;
            for (int k = 2; k <= n; k++) {
                double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
                p0 = p1; p1 = p2;
            }
            dp = n * (z * p1 - p0) / (z * z - 1.0);
        }
        x[i] = -z;
        x[n - 1 - i] = z;
        w[i] = 2.0 / ((1.0 - z * z) * dp * dp);
        w[n - 1 - i] = w[i];
    }
    if (n % 2 == 1) x[n / 2] = 0.0;
}

/* uniform 1-D grid, OldCreateUmesh (miscset.f90:433-470, uniform branch) */
static void make_grid(int M, double L, double R, double *g)
{
    for (int i = 0; i <= M; i++) g[i] = L + (R - L) / (double)M * (double)i;
}

/* finduiviwi (dgvtools_mod.f90:300-338) for one axis: 1-based index of the
 * right end point of the interval containing x, 0 if x is off the grid.  The
 * v and w loops of the reference bound the index by size(ugrid) and
 * size(wgrid) respectively; `bound` carries that size. */
static int find_axis(const double *g, int npts, int bound, double x)
{
    const double eps = 10e-11; /* epsill = 10d-11 */
    if (x < g[0] - eps || x > g[npts - 1] + eps) return 0;
    int i = 1;
    while (x >= g[i - 1] - eps && i < bound) i++;
    return i;
}

int32_t dgvo_find_cell(const dgvo_ctx *c, double u, double v, double w)
{
    const dgvo_grid_desc *d = &c->d;
    int ui = find_axis(c->gu, d->Mu + 1, d->Mu + 1, u);
    int vi = find_axis(c->gv, d->Mv + 1, d->Mu + 1, v); /* size(ugrid), as in the reference */
    int wi = find_axis(c->gw, d->Mw + 1, d->Mw + 1, w);
    if (ui * vi * wi == 0) return -1;
    /* celli = (ui-2)*Mv*Mw + (vi-2)*Mw + (wi-2) + 1, dgvtools_mod.f90:1227 */
    return (ui - 2) * d->Mv * d->Mw + (vi - 2) * d->Mw + (wi - 2);
}

dgvo_ctx *dgvo_create(const dgvo_grid_desc *d)
{
    if (d->su < 1 || d->sv < 1 || d->sw < 1 || d->Mu < 1 || d->Mv < 1 || d->Mw < 1) return NULL;
    dgvo_ctx *c = (dgvo_ctx *)calloc(1, sizeof(dgvo_ctx));
    c->d = *d;
    c->P = d->su * d->sv * d->sw;
    c->Nc = d->Mu * d->Mv * d->Mw;
    c->N = (int64_t)c->P * c->Nc;
    c->gu = malloc(sizeof(double) * (d->Mu + 1));
    c->gv = malloc(sizeof(double) * (d->Mv + 1));
    c->gw = malloc(sizeof(double) * (d->Mw + 1));
    make_grid(d->Mu, d->u_L, d->u_R, c->gu);
    make_grid(d->Mv, d->v_L, d->v_R, c->gv);
    make_grid(d->Mw, d->w_L, d->w_R, c->gw);
    c->xu = malloc(sizeof(double) * d->su); c->wu = malloc(sizeof(double) * d->su);
    c->xv = malloc(sizeof(double) * d->sv); c->wv = malloc(sizeof(double) * d->sv);
    c->xw = malloc(sizeof(double) * d->sw); c->ww = malloc(sizeof(double) * d->sw);
    dgvo_gauss_legendre(d->su, c->xu, c->wu);
    dgvo_gauss_legendre(d->sv, c->xv, c->wv);
    dgvo_gauss_legendre(d->sw, c->xw, c->ww);
    int Nc = c->Nc;
    c->clu = malloc(sizeof(double) * Nc); c->cru = malloc(sizeof(double) * Nc);
    c->clv = malloc(sizeof(double) * Nc); c->crv = malloc(sizeof(double) * Nc);
    c->clw = malloc(sizeof(double) * Nc); c->crw = malloc(sizeof(double) * Nc);
    c->cug = malloc(sizeof(int32_t) * Nc); c->cvg = malloc(sizeof(int32_t) * Nc);
    c->cwg = malloc(sizeof(int32_t) * Nc);
    /* FillCellsArrsDGV (miscset.f90:882-937): u outer, v, w inner */
    int m = 0;
    for (int iu = 0; iu < d->Mu; iu++)
        for (int iv = 0; iv < d->Mv; iv++)
            for (int iw = 0; iw < d->Mw; iw++) {
                c->clu[m] = c->gu[iu]; c->cru[m] = c->gu[iu + 1];
                c->clv[m] = c->gv[iv]; c->crv[m] = c->gv[iv + 1];
                c->clw[m] = c->gw[iw]; c->crw[m] = c->gw[iw + 1];
                /* SetCellsUGINdsSftArrs enumerates the same order (miscset.f90:1245-1277) */
                c->cug[m] = iu; c->cvg[m] = iv; c->cwg[m] = iw;
                m++;
            }
    int64_t N = c->N;
    c->nu = malloc(sizeof(double) * N); c->nv = malloc(sizeof(double) * N);
    c->nw = malloc(sizeof(double) * N); c->nwt = malloc(sizeof(double) * N);
    c->npc = malloc(sizeof(int32_t) * N); c->nui = malloc(sizeof(int32_t) * N);
    c->nvi = malloc(sizeof(int32_t) * N); c->nwi = malloc(sizeof(int32_t) * N);
    /* SetNodesDGV (miscset.f90:1112-1183) */
    int64_t jm = 0;
    for (int ic = 0; ic < Nc; ic++) {
        for (int iu = 0; iu < d->su; iu++) {
            double ru = c->xu[iu] * (c->cru[ic] - c->clu[ic]) / 2.0 + (c->cru[ic] + c->clu[ic]) / 2.0;
            double qu = c->wu[iu];
            for (int iv = 0; iv < d->sv; iv++) {
                double rv = c->xv[iv] * (c->crv[ic] - c->clv[ic]) / 2.0 + (c->crv[ic] + c->clv[ic]) / 2.0;
                double qv = c->wv[iv];
                for (int iw = 0; iw < d->sw; iw++) {
                    double rw = c->xw[iw] * (c->crw[ic] - c->clw[ic]) / 2.0 + (c->crw[ic] + c->clw[ic]) / 2.0;
                    double qw = c->ww[iw];
                    c->npc[jm] = ic;
                    c->nu[jm] = ru; c->nv[jm] = rv; c->nw[jm] = rw;
                    c->nwt[jm] = qu * qv * qw * (c->cru[ic] - c->clu[ic]) * (c->crv[ic] - c->clv[ic]) *
                                 (c->crw[ic] - c->clw[ic]) / 8.0;
                    c->nui[jm] = iu; c->nvi[jm] = iv; c->nwi[jm] = iw;
                    jm++;
                }
            }
        }
    }
    /* the canonical cell is the one containing v = 0 (miscmpiset.f90:553,588) */
    c->ccell = dgvo_find_cell(c, 0.0, 0.0, 0.0);
    return c;
}

static void free_A(dgvo_ctx *c)
{
    free(c->capphi); free(c->A); free(c->xi); free(c->xi1);
    free(c->dui); free(c->dvi); free(c->dwi); free(c->phican); free(c->Ashift);
    c->capphi = NULL; c->A = NULL; c->xi = c->xi1 = NULL;
    c->dui = c->dvi = c->dwi = c->phican = NULL; c->Ashift = NULL;
    c->nnz = 0;
}

void dgvo_destroy(dgvo_ctx *c)
{
    if (!c) return;
    free_A(c);
    free(c->gu); free(c->gv); free(c->gw);
    free(c->xu); free(c->wu); free(c->xv); free(c->wv); free(c->xw); free(c->ww);
    free(c->clu); free(c->cru); free(c->clv); free(c->crv); free(c->clw); free(c->crw);
    free(c->cug); free(c->cvg); free(c->cwg);
    free(c->nu); free(c->nv); free(c->nw); free(c->nwt);
    free(c->npc); free(c->nui); free(c->nvi); free(c->nwi);
    free(c);
}

int64_t dgvo_num_nodes(const dgvo_ctx *c) { return c->N; }
int32_t dgvo_nodes_per_cell(const dgvo_ctx *c) { return c->P; }
int32_t dgvo_num_cells(const dgvo_ctx *c) { return c->Nc; }
int32_t dgvo_canonical_cell(const dgvo_ctx *c) { return c->ccell; }

void dgvo_get_nodes(const dgvo_ctx *c, double *u, double *v, double *w, double *gwts,
                    int32_t *pcell, int32_t *ui, int32_t *vi, int32_t *wi)
{
    size_t n = (size_t)c->N;
    if (u) memcpy(u, c->nu, n * sizeof(double));
    if (v) memcpy(v, c->nv, n * sizeof(double));
    if (w) memcpy(w, c->nw, n * sizeof(double));
    if (gwts) memcpy(gwts, c->nwt, n * sizeof(double));
    if (pcell) memcpy(pcell, c->npc, n * sizeof(int32_t));
    if (ui) memcpy(ui, c->nui, n * sizeof(int32_t));
    if (vi) memcpy(vi, c->nvi, n * sizeof(int32_t));
    if (wi) memcpy(wi, c->nwi, n * sizeof(int32_t));
}

void dgvo_get_cells(const dgvo_ctx *c, int32_t *ugi, int32_t *vgi, int32_t *wgi,
                    double *lu, double *ru, double *lv, double *rv, double *lw, double *rw)
{
    size_t n = (size_t)c->Nc;
    if (ugi) memcpy(ugi, c->cug, n * sizeof(int32_t));
    if (vgi) memcpy(vgi, c->cvg, n * sizeof(int32_t));
    if (wgi) memcpy(wgi, c->cwg, n * sizeof(int32_t));
    if (lu) memcpy(lu, c->clu, n * sizeof(double));
    if (ru) memcpy(ru, c->cru, n * sizeof(double));
    if (lv) memcpy(lv, c->clv, n * sizeof(double));
    if (rv) memcpy(rv, c->crv, n * sizeof(double));
    if (lw) memcpy(lw, c->clw, n * sizeof(double));
    if (rw) memcpy(rw, c->crw, n * sizeof(double));
}

/* ------------------------------------------------------------------------- */
/* SetCellsUGINdsSftArrs (miscset.f90:1202-1311)                              */
static void build_shift_tables(dgvo_ctx *c)
{
    int64_t N = c->N;
    int32_t cc = c->ccell;
    int32_t gov = c->d.sv, gow = c->d.sw;
    c->dui = malloc(sizeof(int32_t) * N); c->dvi = malloc(sizeof(int32_t) * N);
    c->dwi = malloc(sizeof(int32_t) * N); c->phican = malloc(sizeof(int32_t) * N);
    c->Ashift = malloc(sizeof(int64_t) * N);
    /* prefix sums of capphi give Ashift = sum(A_capphi(1:phishift-1)) */
    int64_t *pre = malloc(sizeof(int64_t) * (N + 1));
    pre[0] = 0;
    for (int64_t k = 0; k < N; k++) pre[k + 1] = pre[k] + c->capphi[k];
    int64_t my_cshift = (int64_t)cc * c->P;
    for (int64_t i = 0; i < N; i++) {
        int32_t pc = c->npc[i];
        c->dui[i] = c->cug[pc] - c->cug[cc];
        c->dvi[i] = c->cvg[pc] - c->cvg[cc];
        c->dwi[i] = c->cwg[pc] - c->cwg[cc];
        int64_t phishift = my_cshift + (int64_t)c->nui[i] * gov * gow + (int64_t)c->nvi[i] * gow + c->nwi[i];
        c->phican[i] = (int32_t)phishift;
        c->Ashift[i] = pre[phishift];
    }
    free(pre);
}

int dgvo_set_A(dgvo_ctx *c, const int32_t *capphi, int64_t nnz, const double *A,
               const int32_t *xi, const int32_t *xi1, int one_based)
{
    free_A(c);
    if (c->ccell < 0) return 1;
    int64_t N = c->N, tot = 0;
    for (int64_t k = 0; k < N; k++) { if (capphi[k] < 0) return 2; tot += capphi[k]; }
    if (tot != nnz) return 3;
    int off = one_based ? 1 : 0;
    for (int64_t j = 0; j < nnz; j++) {
        int64_t a = (int64_t)xi[j] - off, b = (int64_t)xi1[j] - off;
        if (a < 0 || a >= N || b < 0 || b >= N) return 4;
    }
    c->nnz = nnz;
    c->capphi = malloc(sizeof(int32_t) * N);
    memcpy(c->capphi, capphi, sizeof(int32_t) * N);
    c->A = malloc(sizeof(double) * (nnz ? nnz : 1));
    c->xi = malloc(sizeof(int32_t) * (nnz ? nnz : 1));
    c->xi1 = malloc(sizeof(int32_t) * (nnz ? nnz : 1));
    memcpy(c->A, A, sizeof(double) * nnz);
    for (int64_t j = 0; j < nnz; j++) { c->xi[j] = xi[j] - off; c->xi1[j] = xi1[j] - off; }
    build_shift_tables(c);
    return 0;
}

void dgvo_get_shift_tables(const dgvo_ctx *c, int32_t *dui, int32_t *dvi, int32_t *dwi,
                           int32_t *phican, int64_t *Ashift)
{
    size_t n = (size_t)c->N;
    if (dui) memcpy(dui, c->dui, n * sizeof(int32_t));
    if (dvi) memcpy(dvi, c->dvi, n * sizeof(int32_t));
    if (dwi) memcpy(dwi, c->dwi, n * sizeof(int32_t));
    if (phican) memcpy(phican, c->phican, n * sizeof(int32_t));
    if (Ashift) memcpy(Ashift, c->Ashift, n * sizeof(int64_t));
}

/* ------------------------------------------------------------------------- */
/* Shifted flat index of node k when its cell is moved by (du,dv,dw); -1 when */
/* the moved cell leaves the grid.  This is the bounds check and the address  */
/* arithmetic of collision_mod.f90:196-215.                                   */
static inline int64_t shifted_index(const dgvo_ctx *c, int32_t k, int32_t du, int32_t dv, int32_t dw)
{
    const dgvo_grid_desc *d = &c->d;
    int32_t kc = c->npc[k];
    int32_t iu = c->cug[kc] + du;
    if (iu < 0 || iu >= d->Mu) return -1;
    int32_t iv = c->cvg[kc] + dv;
    if (iv < 0 || iv >= d->Mv) return -1;
    int32_t iw = c->cwg[kc] + dw;
    if (iw < 0 || iw >= d->Mw) return -1;
    return ((int64_t)iu * d->Mw * d->Mv + (int64_t)iv * d->Mw + iw) * c->P +
           (int64_t)c->nui[k] * d->sw * d->sv + (int64_t)c->nvi[k] * d->sw + c->nwi[k];
}

/* EvalCollisionPeriodicAPlus_DGV (collision_mod.f90:143-229) for one node */
static double aplus_node(const dgvo_ctx *c, const double *f, int64_t iphi)
{
    int64_t Ashift = c->Ashift[iphi];
    int32_t phicap = c->capphi[c->phican[iphi]];
    int32_t du = c->dui[iphi], dv = c->dvi[iphi], dw = c->dwi[iphi];
    double acc = 0.0;
    for (int32_t j = 0; j < phicap; j++) {
        int64_t a = shifted_index(c, c->xi[Ashift + j], du, dv, dw);
        if (a < 0) continue;
        int64_t b = shifted_index(c, c->xi1[Ashift + j], du, dv, dw);
        if (b < 0) continue;
        acc = acc + 2.0 * f[a] * f[b] * c->A[Ashift + j];
    }
    return acc / c->nwt[iphi];
}

void dgvo_collide_aplus(const dgvo_ctx *c, const double *f, double *fc,
                        const int64_t *nodes, int64_t nnodes, int nthreads)
{
    if (!nodes) nnodes = c->N;
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int64_t t = 0; t < nnodes; t++) {
        int64_t iphi = nodes ? nodes[t] : t;
        fc[iphi] = aplus_node(c, f, iphi);
    }
    (void)nthreads;
}

/* EvalCollisionPeriodicA_DGV (collision_mod.f90:29-129): the same Q through
 * compacted scratch arrays fxi, fxi1, Aphi */
void dgvo_collide_a(const dgvo_ctx *c, const double *f, double *fc)
{
    int32_t maxcap = 0;
    for (int64_t k = 0; k < c->N; k++) if (c->capphi[k] > maxcap) maxcap = c->capphi[k];
    double *fxi = malloc(sizeof(double) * (maxcap + 1));
    double *fxi1 = malloc(sizeof(double) * (maxcap + 1));
    double *Aphi = malloc(sizeof(double) * (maxcap + 1));
    for (int64_t iphi = 0; iphi < c->N; iphi++) {
        int64_t Ashift = c->Ashift[iphi];
        int32_t phicap = c->capphi[c->phican[iphi]];
        int32_t du = c->dui[iphi], dv = c->dvi[iphi], dw = c->dwi[iphi];
        int32_t k = 0;
        for (int32_t j = 0; j < phicap; j++) {
            int64_t a = shifted_index(c, c->xi[Ashift + j], du, dv, dw);
            if (a < 0) continue;
            int64_t b = shifted_index(c, c->xi1[Ashift + j], du, dv, dw);
            if (b < 0) continue;
            fxi[k] = f[a]; fxi1[k] = f[b]; Aphi[k] = c->A[Ashift + j];
            k++;
        }
        double s = 0.0;
        for (int32_t j = 0; j < k; j++) s += Aphi[j] * fxi[j] * fxi1[j];
        fc[iphi] = 2.0 * s / c->nwt[iphi];
    }
    free(fxi); free(fxi1); free(Aphi);
}

/* IphiDGV (dgvtools_mod.f90:847-877): no shifts, every node's own records */
void dgvo_iphi(const dgvo_ctx *c, const double *f, double kappa, double *iphi)
{
    int64_t act = 0;
    for (int64_t i = 0; i < c->N; i++) {
        double s = 0.0;
        for (int64_t j = act; j < act + c->capphi[i]; j++) s = s + c->A[j] * f[c->xi[j]] * f[c->xi1[j]];
        iphi[i] = 2.0 * s / c->nwt[i] * kappa;
        act += c->capphi[i];
    }
}

/* EvalCollisionPeriodicMixedTermsA_DGV (collision_mod.f90:244-332) */
void dgvo_mixed_terms(const dgvo_ctx *c, const double *f, const double *fm, double *fc, int nthreads)
{
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 16) num_threads(nthreads)
#endif
    for (int64_t iphi = 0; iphi < c->N; iphi++) {
        int64_t Ashift = c->Ashift[iphi];
        int32_t phicap = c->capphi[c->phican[iphi]];
        int32_t du = c->dui[iphi], dv = c->dvi[iphi], dw = c->dwi[iphi];
        double acc = 0.0;
        for (int32_t j = 0; j < phicap; j++) {
            int64_t a = shifted_index(c, c->xi[Ashift + j], du, dv, dw);
            if (a < 0) continue;
            int64_t b = shifted_index(c, c->xi1[Ashift + j], du, dv, dw);
            if (b < 0) continue;
            acc = acc + (fm[a] * f[b] + f[a] * fm[b]) * c->A[Ashift + j];
        }
        fc[iphi] = 2.0 * acc / c->nwt[iphi];
    }
    (void)nthreads;
}

/* PrepareFMA_DGV (collision_mod.f90:377-464), fmA column-major */
void dgvo_prepare_fma(const dgvo_ctx *c, const double *fm, double *fmA)
{
    int64_t N = c->N;
    memset(fmA, 0, sizeof(double) * (size_t)N * (size_t)N);
    for (int64_t iphi = 0; iphi < N; iphi++) {
        int64_t Ashift = c->Ashift[iphi];
        int32_t phicap = c->capphi[c->phican[iphi]];
        int32_t du = c->dui[iphi], dv = c->dvi[iphi], dw = c->dwi[iphi];
        double *col = fmA + (size_t)N * (size_t)iphi;
        for (int32_t j = 0; j < phicap; j++) {
            int64_t a = shifted_index(c, c->xi[Ashift + j], du, dv, dw);
            if (a < 0) continue;
            int64_t b = shifted_index(c, c->xi1[Ashift + j], du, dv, dw);
            if (b < 0) continue;
            col[a] = col[a] + fm[b] * c->A[Ashift + j];
            col[b] = col[b] + fm[a] * c->A[Ashift + j];
        }
        for (int64_t k = 0; k < N; k++) col[k] = col[k] / c->nwt[iphi];
    }
}

/* EvalCollisionLinear (collision_mod.f90:346-359): fc = 2*MATMUL(f,fmA) */
void dgvo_eval_linear(const dgvo_ctx *c, const double *fmA, const double *f, double *fc)
{
    int64_t N = c->N;
    for (int64_t i = 0; i < N; i++) {
        const double *col = fmA + (size_t)N * (size_t)i;
        double s = 0.0;
        for (int64_t k = 0; k < N; k++) s += f[k] * col[k];
        fc[i] = 2.0 * s;
    }
}

/* g = J^T v with J = dQ/df; the derivative of the APlus loop term by term */
void dgvo_vjp(const dgvo_ctx *c, const double *f, const double *v, double *g, int nthreads)
{
    int64_t N = c->N;
    int nt = 1;
#ifdef _OPENMP
    nt = nthreads > 0 ? nthreads : omp_get_max_threads();
#endif
    double *buf = calloc((size_t)nt * (size_t)N, sizeof(double));
#ifdef _OPENMP
#pragma omp parallel num_threads(nt)
#endif
    {
        int tid = 0;
#ifdef _OPENMP
        tid = omp_get_thread_num();
#endif
        double *gl = buf + (size_t)tid * (size_t)N;
#ifdef _OPENMP
#pragma omp for schedule(static)
#endif
        for (int64_t iphi = 0; iphi < N; iphi++) {
            int64_t Ashift = c->Ashift[iphi];
            int32_t phicap = c->capphi[c->phican[iphi]];
            int32_t du = c->dui[iphi], dv = c->dvi[iphi], dw = c->dwi[iphi];
            double ci = 2.0 * v[iphi] / c->nwt[iphi];
            for (int32_t j = 0; j < phicap; j++) {
                int64_t a = shifted_index(c, c->xi[Ashift + j], du, dv, dw);
                if (a < 0) continue;
                int64_t b = shifted_index(c, c->xi1[Ashift + j], du, dv, dw);
                if (b < 0) continue;
                double t = ci * c->A[Ashift + j];
                gl[a] += t * f[b];
                gl[b] += t * f[a];
            }
        }
    }
    for (int64_t k = 0; k < N; k++) {
        double s = 0.0;
        for (int t = 0; t < nt; t++) s += buf[(size_t)t * (size_t)N + k];
        g[k] = s;
    }
    free(buf);
}

/* ------------------------------------------------------------------------- */
/* SpatialOperSH_DGV, run_mode 0 (spat_oper_mod.f90:48-66)                   */
void dgvo_spatial_oper(const dgvo_ctx *c, const double *f, double *fcol, double dt,
                       double kappa, int nthreads)
{
    dgvo_collide_aplus(c, f, fcol, NULL, 0, nthreads);
    double coef = kappa * dt; /* (mol_diam/L_inf)**2*N_inf*dt */
    for (int64_t i = 0; i < c->N; i++) fcol[i] = fcol[i] * coef;
}

/* Regime state of SpatialOperSH_DGV (run_mode, fm; spat_oper_mod.f90:28-68) */
struct dgvo_regime {
    int run_mode;
    double decomp_lev, linear_lev, last_L1;
    double *fm;
};

dgvo_regime *dgvo_regime_create(const dgvo_ctx *c, double decomp_lev, double linear_lev)
{
    dgvo_regime *r = calloc(1, sizeof(dgvo_regime));
    r->decomp_lev = decomp_lev;
    r->linear_lev = linear_lev;
    r->last_L1 = -1.0;
    r->fm = calloc((size_t)c->N, sizeof(double));
    return r;
}

void dgvo_regime_free(dgvo_regime *r)
{
    if (!r) return;
    free(r->fm);
    free(r);
}

int dgvo_regime_mode(const dgvo_regime *r, double *last_L1)
{
    if (last_L1) *last_L1 = r->last_L1;
    return r->run_mode;
}

/* CheckSolutionMode_DGV (spat_oper_mod.f90:195-272): the local Maxwellian of
 * f, the relative L1 distance to it, the run_mode switch and the refresh of
 * fm (PrepareFMA_DGV: here fm itself -- the linear part is evaluated as the
 * mixed terms at fm, equal to 2*MATMUL(Df, fmA)); Df = f - fm */
static void check_mode(const dgvo_ctx *c, dgvo_regime *r, const double *f, double *Df)
{
    int64_t N = c->N, i;
    double m[5];
    dgvo_moments(c, f, m);
    double *fmn = malloc(sizeof(double) * N);
    dgvo_maxwellian(c, m[4], m[1], m[2], m[3], m[0], fmn);
    double L1 = 0.0;
    for (i = 0; i < N; i++) L1 = L1 + fabs(f[i] - fmn[i]) * c->nwt[i];
    L1 = L1 / m[0];
    r->last_L1 = L1;
    if (L1 < r->decomp_lev) {
        double L1fm;
        switch (r->run_mode) {
        case 0:
            memcpy(r->fm, fmn, sizeof(double) * N);
            r->run_mode = L1 < r->linear_lev ? 2 : 1;
            break;
        case 1:
        case 2:
            L1fm = 0.0;
            for (i = 0; i < N; i++) L1fm = L1fm + fabs(r->fm[i] - fmn[i]) * c->nwt[i];
            L1fm = L1fm / m[0];
            if (L1fm > r->linear_lev / 2.0) memcpy(r->fm, fmn, sizeof(double) * N);
            if (r->run_mode == 1 && L1 < r->linear_lev) r->run_mode = 2;
            else if (r->run_mode == 2 && L1 > r->linear_lev) r->run_mode = 1;
            break;
        }
        for (i = 0; i < N; i++) Df[i] = f[i] - r->fm[i];
    } else {
        r->run_mode = 0;
    }
    free(fmn);
}

/* SpatialOperSH_DGV (spat_oper_mod.f90:28-68) with its run modes: 0 Q(f),
 * 1 L(Df) + Q(Df), 2 L(Df); times kappa*dt.  r == NULL: mode 0 always. */
void dgvo_spatial_oper_regime(const dgvo_ctx *c, dgvo_regime *r, const double *f, double *fcol, double dt,
                              double kappa, int nthreads)
{
    if (!r) {
        dgvo_spatial_oper(c, f, fcol, dt, kappa, nthreads);
        return;
    }
    int64_t N = c->N, i;
    double *Df = malloc(sizeof(double) * N), *scr = malloc(sizeof(double) * N);
    check_mode(c, r, f, Df);
    switch (r->run_mode) {
    case 0:
        dgvo_collide_aplus(c, f, fcol, NULL, 0, nthreads);
        break;
    case 1:
        dgvo_mixed_terms(c, Df, r->fm, scr, nthreads);
        dgvo_collide_aplus(c, Df, fcol, NULL, 0, nthreads);
        for (i = 0; i < N; i++) fcol[i] = fcol[i] + scr[i];
        break;
    default:
        dgvo_mixed_terms(c, Df, r->fm, fcol, nthreads);
        break;
    }
    double coef = kappa * dt;
    for (i = 0; i < N; i++) fcol[i] = fcol[i] * coef;
    free(Df);
    free(scr);
}

/* TimeIntegratorORK_SH_DGV (time_integr_mod.f90:26-152) */
int dgvo_rk_step(const dgvo_ctx *c, int order, double *f, double *frhs1, double dt,
                 double kappa, int nthreads)
{
    return dgvo_rk_step_regime(c, NULL, order, f, frhs1, dt, kappa, nthreads);
}

int dgvo_rk_step_regime(const dgvo_ctx *c, dgvo_regime *reg, int order, double *f, double *frhs1, double dt,
                        double kappa, int nthreads)
{
    int64_t N = c->N;
    if (order < 1 || order > 5) return 1;
    double *t0 = malloc(sizeof(double) * N), *ft2 = malloc(sizeof(double) * N);
    double *ft3 = malloc(sizeof(double) * N), *ft4 = malloc(sizeof(double) * N);
    int64_t i;
    switch (order) {
    case 1:
        dgvo_spatial_oper_regime(c, reg, f, frhs1, dt, kappa, nthreads);
        for (i = 0; i < N; i++) f[i] = f[i] + frhs1[i];
        break;
    case 2: /* :55-59 */
        dgvo_spatial_oper_regime(c, reg, f, frhs1, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] * 2 / 3.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft2, dt, kappa, nthreads);
        for (i = 0; i < N; i++) f[i] = f[i] + frhs1[i] / 4.0 + ft2[i] * 3.0 / 4;
        break;
    case 3: /* :76-82 */
        dgvo_spatial_oper_regime(c, reg, f, frhs1, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] / 2.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft2, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + ft2[i] * 3.0 / 4;
        dgvo_spatial_oper_regime(c, reg, t0, ft3, dt, kappa, nthreads);
        for (i = 0; i < N; i++) f[i] = f[i] + frhs1[i] * 2 / 9.0 + ft2[i] * 3.0 / 9.0 + ft3[i] * 4 / 9.0;
        break;
    case 4: /* :95-104 */
        dgvo_spatial_oper_regime(c, reg, f, frhs1, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] / 2.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft2, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] / 4.0 + ft2[i] / 4.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft3, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] - ft2[i] + ft3[i] * 2;
        dgvo_spatial_oper_regime(c, reg, t0, ft2, dt, kappa, nthreads);
        for (i = 0; i < N; i++) f[i] = f[i] + frhs1[i] / 6.0 + ft3[i] * 2 / 3.0 + ft2[i] / 6.0;
        break;
    case 5: /* :122-146 */
        dgvo_spatial_oper_regime(c, reg, f, frhs1, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] / 2.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft2, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] / 4.0 + ft2[i] / 4.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft3, dt, kappa, nthreads);
        for (i = 0; i < N; i++) t0[i] = f[i] - ft2[i] + ft3[i] * 2.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft4, dt, kappa, nthreads);
        for (i = 0; i < N; i++) ft3[i] = -ft2[i] / 5.0 + ft3[i] * 546 / 625.0;
        for (i = 0; i < N; i++) t0[i] = f[i] + frhs1[i] * 7.0 / 27.0 + ft2[i] * 10.0 / 27.0 + ft4[i] / 27.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft2, dt, kappa, nthreads);
        for (i = 0; i < N; i++)
            t0[i] = f[i] + frhs1[i] * 28.0 / 625.0 + ft3[i] + ft4[i] * 54 / 625.0 - ft2[i] * 378 / 625.0;
        dgvo_spatial_oper_regime(c, reg, t0, ft3, dt, kappa, nthreads);
        for (i = 0; i < N; i++)
            f[i] = f[i] + frhs1[i] / 24.0 + ft4[i] * 5.0 / 48.0 + ft2[i] * 27.0 / 56.0 + ft3[i] * 125 / 336.0;
        break;
    }
    for (i = 0; i < N; i++) frhs1[i] = frhs1[i] / dt; /* :151 */
    free(t0); free(ft2); free(ft3); free(ft4);
    return 0;
}

/* TimeIntegratorMTS_SH_DGV (time_integr_mod.f90:314-364) */
int dgvo_ab_step(const dgvo_ctx *c, int order, double *f, double *frhs, double dt,
                 double kappa, int nthreads)
{
    int64_t N = c->N, i;
    if (order < 1 || order > 5) return 1;
    double *r1 = frhs, *r2 = frhs + N, *r3 = frhs + 2 * N, *r4 = frhs + 3 * N, *r5 = frhs + 4 * N;
    /* push the right-side history (f1..f4 are not used by the update) */
    if (order >= 5) memcpy(r5, r4, sizeof(double) * N);
    if (order >= 4) memcpy(r4, r3, sizeof(double) * N);
    if (order >= 3) memcpy(r3, r2, sizeof(double) * N);
    if (order >= 2) memcpy(r2, r1, sizeof(double) * N);
    dgvo_spatial_oper(c, f, r1, dt, kappa, nthreads);
    switch (order) {
    case 1:
        for (i = 0; i < N; i++) f[i] = f[i] + r1[i];
        break;
    case 2:
        for (i = 0; i < N; i++) f[i] = f[i] + r1[i] * 3.0 / 2.0 - dt * r2[i] / 2.0;
        break;
    case 3:
        for (i = 0; i < N; i++)
            f[i] = f[i] + r1[i] * 23.0 / 12.0 - dt * r2[i] * 4 / 3.0 + dt * r3[i] * 5.0 / 12.0;
        break;
    case 4:
        for (i = 0; i < N; i++)
            f[i] = f[i] + r1[i] * 55.0 / 24.0 - dt * r2[i] * 59.0 / 24.0 + dt * r3[i] * 37.0 / 24.0 -
                   dt * r4[i] * 3.0 / 8;
        break;
    case 5:
        for (i = 0; i < N; i++)
            f[i] = f[i] + r1[i] * (1901.0 / 720.0) - dt * r2[i] * (2774.0 / 720.0) +
                   dt * r3[i] * (2616.0 / 720.0) - dt * r4[i] * (1274.0 / 720.0) +
                   dt * r5[i] * (251.0 / 720.0);
        break;
    }
    for (i = 0; i < N; i++) r1[i] = r1[i] / dt; /* :363 */
    return 0;
}

/* PrepareMTS_SH_DGV (time_integr_mod.f90:443-569): rkmts-1 RK steps of order
 * rkmts, pushing the right-side history before each */
int dgvo_prepare_ab(const dgvo_ctx *c, int order, double *f, double *frhs, double dt,
                    double kappa, int nthreads)
{
    int64_t N = c->N;
    if (order < 1 || order > 5) return 1;
    double *r1 = frhs, *r2 = frhs + N, *r3 = frhs + 2 * N, *r4 = frhs + 3 * N;
    for (int i = 2; i <= order; i++) {
        switch (order) { /* :524-533 */
        case 3: memcpy(r2, r1, sizeof(double) * N); break;
        case 4: memcpy(r3, r2, sizeof(double) * N); memcpy(r2, r1, sizeof(double) * N); break;
        case 5:
            memcpy(r4, r3, sizeof(double) * N); memcpy(r3, r2, sizeof(double) * N);
            memcpy(r2, r1, sizeof(double) * N);
            break;
        default: break;
        }
        dgvo_rk_step(c, order, f, r1, dt, kappa, nthreads);
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* MassCheckRec (dgvtools_mod.f90:1437-1458)                                 */
void dgvo_moments(const dgvo_ctx *c, const double *f, double *out5)
{
    int64_t N = c->N, i;
    double n = 0, su = 0, sv = 0, sw = 0, st = 0;
    for (i = 0; i < N; i++) n += f[i] * c->nwt[i];
    for (i = 0; i < N; i++) su += f[i] * c->nwt[i] * c->nu[i];
    for (i = 0; i < N; i++) sv += f[i] * c->nwt[i] * c->nv[i];
    for (i = 0; i < N; i++) sw += f[i] * c->nwt[i] * c->nw[i];
    double ub = su / n, vb = sv / n, wb = sw / n;
    for (i = 0; i < N; i++) {
        double du = c->nu[i] - ub, dv = c->nv[i] - vb, dw = c->nw[i] - wb;
        st += f[i] * c->nwt[i] * (du * du + dv * dv + dw * dw);
    }
    out5[0] = n; out5[1] = ub; out5[2] = vb; out5[3] = wb;
    out5[4] = st / n / 3.0 * 2.0;
}

/* maxwelveldist (distributions_mod.f90:83-95) */
void dgvo_maxwellian(const dgvo_ctx *c, double T, double u0, double v0, double w0,
                     double n, double *f)
{
    double beta = sqrt(PI_REF * T) * (PI_REF * T);
    double tt = T > 0.0000001 ? T : 0.0000001;
    for (int64_t i = 0; i < c->N; i++) {
        double du = c->nu[i] - u0, dv = c->nv[i] - v0, dw = c->nw[i] - w0;
        f[i] = n * exp(-(du * du + dv * dv + dw * dw) / tt) / beta;
    }
}

/* L2(w)-orthogonal projection removing the five collision-invariant moments */
void dgvo_project_conservative(const dgvo_ctx *c, double *q)
{
    int64_t N = c->N;
    double G[5][5] = {{0}}, m[5] = {0};
    for (int64_t i = 0; i < N; i++) {
        double u = c->nu[i], v = c->nv[i], w = c->nw[i];
        double psi[5] = {1.0, u, v, w, u * u + v * v + w * w};
        for (int a = 0; a < 5; a++) {
            m[a] += c->nwt[i] * psi[a] * q[i];
            for (int b = 0; b < 5; b++) G[a][b] += c->nwt[i] * psi[a] * psi[b];
        }
    }
    /* Gaussian elimination with partial pivoting on the 5x5 Gram system */
    double M[5][6];
    for (int a = 0; a < 5; a++) { for (int b = 0; b < 5; b++) M[a][b] = G[a][b]; M[a][5] = m[a]; }
    for (int k = 0; k < 5; k++) {
        int piv = k;
        for (int r = k + 1; r < 5; r++) if (fabs(M[r][k]) > fabs(M[piv][k])) piv = r;
        if (piv != k) for (int b = 0; b < 6; b++) { double t = M[k][b]; M[k][b] = M[piv][b]; M[piv][b] = t; }
        for (int r = k + 1; r < 5; r++) {
            double fct = M[r][k] / M[k][k];
            for (int b = k; b < 6; b++) M[r][b] -= fct * M[k][b];
        }
    }
    double lam[5];
    for (int k = 4; k >= 0; k--) {
        double s = M[k][5];
        for (int b = k + 1; b < 5; b++) s -= M[k][b] * lam[b];
        lam[k] = s / M[k][k];
    }
    for (int64_t i = 0; i < N; i++) {
        double u = c->nu[i], v = c->nv[i], w = c->nw[i];
        q[i] -= lam[0] + lam[1] * u + lam[2] * v + lam[3] * w + lam[4] * (u * u + v * v + w * w);
    }
}

/* ------------------------------------------------------------------------- */
/* SetA_DGV and its helpers (dgvtools_mod.f90:377-681, 938-1122)              */

/* lagrbasfun (dgvtools_mod.f90:31-56) */
static double lagrbasfun(int i, double x, const double *kappa, int n)
{
    double y = 1.0;
    for (int j = 0; j < i; j++) y = y * (kappa[j] - x) / (kappa[j] - kappa[i]);
    for (int j = i + 1; j < n; j++) y = y * (kappa[j] - x) / (kappa[j] - kappa[i]);
    return y;
}

/* EvalLagrBasisFunByNdsDGblzmEZ (dgvtools_mod.f90:232-289).  mode 0: the
 * commented "rem to restore" lines put back (cell test + Lagrange product with
 * y starting at 1); modes 1..5: y = 1, u, v, w, u^2+v^2+w^2 everywhere, the
 * shipped known-answer configuration (:267-274). */
static double basis_ez(const dgvo_ctx *c, double u, double v, double w, int32_t i, int mode)
{
    switch (mode) {
    case 1: return 1.0;
    case 2: return u;
    case 3: return v;
    case 4: return w;
    case 5: return u * u + v * v + w * w;
    default: break;
    }
    int32_t cp = c->npc[i];
    double lu = c->clu[cp], ru = c->cru[cp], lv = c->clv[cp], rv = c->crv[cp];
    double lw = c->clw[cp], rw = c->crw[cp];
    if (u < lu || ru < u || v < lv || rv < v || w < lw || rw < w) return 0.0;
    double y = 1.0;
    double unor = (u - (ru + lu) / 2.0) / (ru - lu) * 2.0;
    y = y * lagrbasfun(c->nui[i], unor, c->xu, c->d.su);
    double vnor = (v - (rv + lv) / 2.0) / (rv - lv) * 2.0;
    y = y * lagrbasfun(c->nvi[i], vnor, c->xv, c->d.sv);
    double wnor = (w - (rw + lw) / 2.0) / (rw - lw) * 2.0;
    y = y * lagrbasfun(c->nwi[i], wnor, c->xw, c->d.sw);
    return y;
}

typedef struct {
    const dgvo_ctx *c;
    int32_t i1;
    int mode;
    double xiu, xiv, xiw, xi1u, xi1v, xi1w;
    double ugu, ugv, ugw, ugux2, ugvx2, ugwx2, ugux3, ugvx3, ugwx3, g1, g2, dsph;
    double varphi_xi, varphi_xi1;
    double ires_e, ErrEps;
    double sinchi, coschi;
} pair_state;

/* EvalPhiPostCollIntegrand (dgvtools_mod.f90:938-975) */
static double post_coll_integrand(const pair_state *s, double epsil)
{
    double sinchicoseps = cos(epsil) * s->sinchi / s->g1;
    double sinchisineps = sin(epsil) * s->sinchi / s->g2;
    double ku = s->ugu * s->coschi - s->ugux2 * sinchicoseps - s->ugux3 * sinchisineps;
    double kv = s->ugv * s->coschi - s->ugvx2 * sinchicoseps - s->ugvx3 * sinchisineps;
    double kw = s->ugw * s->coschi - s->ugwx2 * sinchicoseps - s->ugwx3 * sinchisineps;
    double xiupr = ((s->xiu + s->xi1u) + s->dsph * ku) / 2.0;
    double xi1upr = ((s->xiu + s->xi1u) - s->dsph * ku) / 2.0;
    double xivpr = ((s->xiv + s->xi1v) + s->dsph * kv) / 2.0;
    double xi1vpr = ((s->xiv + s->xi1v) - s->dsph * kv) / 2.0;
    double xiwpr = ((s->xiw + s->xi1w) + s->dsph * kw) / 2.0;
    double xi1wpr = ((s->xiw + s->xi1w) - s->dsph * kw) / 2.0;
    double z = basis_ez(s->c, xiupr, xivpr, xiwpr, s->i1, s->mode) +
               basis_ez(s->c, xi1upr, xi1vpr, xi1wpr, s->i1, s->mode) - s->varphi_xi - s->varphi_xi1;
    return z;
}

typedef double (*integrand_fn)(pair_state *s, double x);

/* The adaptive Simpson scheme shared by the chi loop (dgvtools_mod.f90:532-637)
 * and A_IntEpsilon (:1013-1119): n0 initial cells on [0, len]; cells whose
 * three samples sum below 1e-15 in magnitude are dropped; a marked cell is
 * halved and its two-panel Simpson sum accepted when the error indicator
 * |q1+q2-q|/15/h is at most err; the whole pass stops once the running
 * estimate of the remaining integral is at most err. */
static double adaptive_simpson(pair_state *s, integrand_fn fn, double len, int n0, double err,
                               double int_init, int ncap)
{
    if (n0 > ncap) n0 = ncap; /* warning branch of the reference: the mesh is capped */
    size_t cap = (size_t)ncap;
    double *nd1 = calloc(2 * cap, sizeof(double)), *nd2 = calloc(2 * cap, sizeof(double));
    double *fn1 = calloc(3 * cap, sizeof(double)), *fn2 = calloc(3 * cap, sizeof(double));
    int *rf1 = calloc(cap, sizeof(int)), *rf2 = calloc(cap, sizeof(int));
    int n1 = n0;
    for (int d = 1; d <= n1; d++) {
        nd1[2 * (d - 1)] = (d - 1) * len / (double)n1;
        nd1[2 * d - 1] = d * len / (double)n1;
    }
    for (int d = 1; d <= n1; d++) {
        if (d > 1 && nd1[2 * d - 2] == nd1[2 * d - 3]) fn1[3 * d - 3] = fn1[3 * d - 4];
        else fn1[3 * d - 3] = fn(s, nd1[2 * d - 2]);
        fn1[3 * d - 1] = fn(s, nd1[2 * d - 1]);
        fn1[3 * d - 2] = fn(s, (nd1[2 * d - 2] + nd1[2 * d - 1]) / 2.0);
        rf1[d - 1] = 1;
    }
    double total = 0.0, my_int = int_init;
    int flag = 1;
    while (flag) {
        flag = 0;
        memset(nd2, 0, 2 * cap * sizeof(double));
        memset(fn2, 0, 3 * cap * sizeof(double));
        memset(rf2, 0, cap * sizeof(int));
        int e = 0;
        if (my_int > err) {
            my_int = 0.0;
            for (int d = 1; d <= n1; d++) {
                double fa = fn1[3 * d - 3], fm = fn1[3 * d - 2], fb = fn1[3 * d - 1];
                if (!(fabs(fa) + fabs(fm) + fabs(fb) > 1.0e-15 && rf1[d - 1] == 1)) continue;
                if (e > ncap - 2) { /* the reference stops here; report as NaN */
                    total = NAN; flag = 0; goto done;
                }
                double a = nd1[2 * d - 2], b = nd1[2 * d - 1];
                nd2[2 * e] = a; fn2[3 * e] = fa;
                nd2[2 * e + 3] = b; fn2[3 * e + 5] = fb;
                nd2[2 * e + 1] = (a + b) / 2;
                nd2[2 * e + 2] = nd2[2 * e + 1];
                fn2[3 * e + 2] = fm; fn2[3 * e + 3] = fm;
                fn2[3 * e + 1] = fn(s, (nd2[2 * e + 1] + nd2[2 * e]) / 2.0);
                fn2[3 * e + 4] = fn(s, (nd2[2 * e + 3] + nd2[2 * e + 2]) / 2.0);
                double quad = (fa + 4 * fm + fb) * (b - a) / 6;
                double quad1 = (fn2[3 * e] + 4 * fn2[3 * e + 1] + fn2[3 * e + 2]) * (nd2[2 * e + 1] - nd2[2 * e]) / 6;
                double quad2 = (fn2[3 * e + 3] + 4 * fn2[3 * e + 4] + fn2[3 * e + 5]) * (nd2[2 * e + 3] - nd2[2 * e + 2]) / 6;
                double es = fabs(quad1 + quad2 - quad) / 15 / (b - a);
                my_int = my_int + fabs(quad1) + fabs(quad2);
                if (es > err) {
                    flag = 1; rf2[e] = 1; rf2[e + 1] = 1;
                } else {
                    rf2[e] = 0; rf2[e + 1] = 0;
                    total = total + quad1 + quad2;
                }
                e += 2;
            }
        }
        double *t;
        t = nd1; nd1 = nd2; nd2 = t;
        t = fn1; fn1 = fn2; fn2 = t;
        int *ti = rf1; rf1 = rf2; rf2 = ti;
        n1 = e;
    }
done:
    free(nd1); free(nd2); free(fn1); free(fn2); free(rf1); free(rf2);
    return total;
}

static double eps_integrand(pair_state *s, double eps) { return post_coll_integrand(s, eps); }

/* A_IntEpsilon (dgvtools_mod.f90:988-1122) */
static double int_epsilon(pair_state *s, double chi)
{
    s->sinchi = sin(chi);
    s->coschi = cos(chi);
    int n0 = (int)floor(PI_REF * s->dsph * s->sinchi / s->ires_e) + 1;
    double r = adaptive_simpson(s, eps_integrand, 2 * PI_REF, n0, s->ErrEps, 10 * s->ErrEps, 10000);
    return r * s->sinchi;
}

static void pair_setup(pair_state *s, const dgvo_ctx *c, int32_t i1, int32_t i2, int32_t i3, int mode)
{
    s->c = c; s->i1 = i1; s->mode = mode;
    s->xiu = c->nu[i2]; s->xiv = c->nv[i2]; s->xiw = c->nw[i2];
    s->xi1u = c->nu[i3]; s->xi1v = c->nv[i3]; s->xi1w = c->nw[i3];
    s->varphi_xi = basis_ez(c, s->xiu, s->xiv, s->xiw, i1, mode);
    s->varphi_xi1 = basis_ez(c, s->xi1u, s->xi1v, s->xi1w, i1, mode);
    double du = s->xiu - s->xi1u, dv = s->xiv - s->xi1v, dw = s->xiw - s->xi1w;
    s->dsph = sqrt(du * du + dv * dv + dw * dw);
    s->ugu = (s->xiu - s->xi1u) / s->dsph;
    s->ugv = (s->xiv - s->xi1v) / s->dsph;
    s->ugw = (s->xiw - s->xi1w) / s->dsph;
    double ugu = s->ugu, ugv = s->ugv, ugw = s->ugw;
    /* two vectors orthogonal to g (dgvtools_mod.f90:497-525) */
    if (fabs(ugw - ugv) + fabs(ugu - ugw) + fabs(ugv - ugu) < 1.0e-6) {
        s->ugux2 = ugv; s->ugvx2 = -ugu; s->ugwx2 = 0;
        s->ugux3 = ugu * ugw; s->ugvx3 = ugv * ugw; s->ugwx3 = -(ugu * ugu) - (ugv * ugv);
        s->g1 = sqrt(s->ugux2 * s->ugux2 + s->ugvx2 * s->ugvx2);
        s->g2 = sqrt(s->ugux3 * s->ugux3 + s->ugvx3 * s->ugvx3 + s->ugwx3 * s->ugwx3);
    } else {
        s->ugux2 = (ugw - ugv); s->ugvx2 = (ugu - ugw); s->ugwx2 = (ugv - ugu);
        s->ugux3 = ((ugv * ugv) - (ugv) * (ugu) - (ugw) * (ugu) + (ugw * ugw));
        s->ugvx3 = ((ugw * ugw) - (ugw) * (ugv) - (ugu) * (ugv) + (ugu * ugu));
        s->ugwx3 = ((ugu * ugu) - (ugu) * (ugw) - (ugv) * (ugw) + (ugv * ugv));
        s->g1 = sqrt(s->ugux2 * s->ugux2 + s->ugvx2 * s->ugvx2 + s->ugwx2 * s->ugwx2);
        s->g2 = sqrt(s->ugux3 * s->ugux3 + s->ugvx3 * s->ugvx3 + s->ugwx3 * s->ugwx3);
    }
}

static double chi_integrand(pair_state *s, double chi) { return int_epsilon(s, chi); }

/* integral over chi of A_IntEpsilon for one pair (dgvtools_mod.f90:532-637) */
static double pair_integral(pair_state *s, double ires_t, double ErrChi)
{
    int n0 = (int)floor(PI_REF * s->dsph / ires_t / 2.0) + 1;
    return adaptive_simpson(s, chi_integrand, PI_REF, n0, ErrChi, 100 * ErrChi, 10000);
}

/* reference prefilter: collision sphere vs circumscribed sphere of the cell
 * (dgvtools_mod.f90:484-531) */
static inline int prefilter_pass(const double *uu, const double *vv, const double *ww, double dphi,
                                 double Trad, double xiu, double xiv, double xiw, double xi1u,
                                 double xi1v, double xi1w, double *dsph_out)
{
    double a = xiu - xi1u, b = xiv - xi1v, cc = xiw - xi1w;
    double dsph = sqrt(a * a + b * b + cc * cc);
    double p = xiu + xi1u - uu[0] - uu[1], q = xiv + xi1v - vv[0] - vv[1], r = xiw + xi1w - ww[0] - ww[1];
    double dist2 = sqrt(p * p + q * q + r * r);
    *dsph_out = dsph;
    if ((dist2 > dsph + dphi) || (dist2 + dphi < dsph) || (dsph > Trad)) return 0;
    return 1;
}

double dgvo_seta_pair_integral(const dgvo_ctx *c, int32_t i1, int32_t i2, int32_t i3,
                               double ErrChi, double ErrEps, int basis_mode)
{
    int32_t pci = c->npc[i1];
    double hu = c->cru[pci] - c->clu[pci], hv = c->crv[pci] - c->clv[pci], hw = c->crw[pci] - c->clw[pci];
    double hmax = hu > hv ? hu : hv;
    if (hw > hmax) hmax = hw;
    pair_state s;
    pair_setup(&s, c, i1, i2, i3, basis_mode);
    s.ires_e = hmax / 32;
    s.ErrEps = ErrEps;
    return pair_integral(&s, hmax / 32, ErrChi);
}

int64_t dgvo_seta(const dgvo_ctx *c, int32_t i1, double Trad, double ErrChi, double ErrEps,
                  double min_sens, int basis_mode, int nthreads, double **Aout, int32_t **xiout,
                  int32_t **xi1out)
{
    int64_t ni = c->N;
    int32_t pci = c->npc[i1];
    double uu[2] = {c->clu[pci], c->cru[pci]}, vv[2] = {c->clv[pci], c->crv[pci]};
    double ww[2] = {c->clw[pci], c->crw[pci]};
    double dphi = sqrt((uu[1] - uu[0]) * (uu[1] - uu[0]) + (vv[1] - vv[0]) * (vv[1] - vv[0]) +
                       (ww[1] - ww[0]) * (ww[1] - ww[0]));
    double hmax = uu[1] - uu[0];
    if (vv[1] - vv[0] > hmax) hmax = vv[1] - vv[0];
    if (ww[1] - ww[0] > hmax) hmax = ww[1] - ww[0];
    double ires_t = hmax / 32, ires_e = ires_t;
    /* per-i2 record lists, concatenated in i2 order: the serial order of the
     * reference loop */
    int64_t *cnt = calloc((size_t)ni, sizeof(int64_t));
    double **av = calloc((size_t)ni, sizeof(double *));
    int32_t **bv = calloc((size_t)ni, sizeof(int32_t *));
#ifdef _OPENMP
    if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
#endif
    for (int64_t i2 = 0; i2 < ni; i2++) {
        int64_t capn = 16, n = 0;
        double *a = malloc(sizeof(double) * capn);
        int32_t *b = malloc(sizeof(int32_t) * capn);
        for (int64_t i3 = i2 + 1; i3 < ni; i3++) {
            double dsph;
            if (!prefilter_pass(uu, vv, ww, dphi, Trad, c->nu[i2], c->nv[i2], c->nw[i2], c->nu[i3],
                                c->nv[i3], c->nw[i3], &dsph))
                continue;
            pair_state s;
            pair_setup(&s, c, i1, (int32_t)i2, (int32_t)i3, basis_mode);
            s.ires_e = ires_e;
            s.ErrEps = ErrEps;
            double Atemp = pair_integral(&s, ires_t, ErrChi);
            if (fabs(Atemp) > min_sens) {
                Atemp = Atemp * c->nwt[i3];
                Atemp = Atemp * c->nwt[i2];
                double d8 = s.dsph / 8.0;
                if (n == capn) {
                    capn *= 2;
                    a = realloc(a, sizeof(double) * capn);
                    b = realloc(b, sizeof(int32_t) * capn);
                }
                a[n] = Atemp * d8;
                b[n] = (int32_t)i3;
                n++;
            }
        }
        cnt[i2] = n; av[i2] = a; bv[i2] = b;
    }
    (void)nthreads;
    int64_t tot = 0;
    for (int64_t i2 = 0; i2 < ni; i2++) tot += cnt[i2];
    double *A = malloc(sizeof(double) * (tot ? tot : 1));
    int32_t *X = malloc(sizeof(int32_t) * (tot ? tot : 1)), *X1 = malloc(sizeof(int32_t) * (tot ? tot : 1));
    int64_t k = 0;
    for (int64_t i2 = 0; i2 < ni; i2++) {
        for (int64_t j = 0; j < cnt[i2]; j++) { A[k] = av[i2][j]; X[k] = (int32_t)i2; X1[k] = bv[i2][j]; k++; }
        free(av[i2]); free(bv[i2]);
    }
    free(cnt); free(av); free(bv);
    *Aout = A; *xiout = X; *xi1out = X1;
    return tot;
}

/* ------------------------------------------------------------------------- */
/* Synthetic records                                                          */
static inline uint64_t splitmix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

double dgvo_synth_value(uint64_t seed, int32_t p, int32_t i2, int32_t i3, double w2, double w3,
                        double dsph)
{
    uint64_t k = ((uint64_t)(uint32_t)p << 48) ^ ((uint64_t)(uint32_t)i2 << 24) ^ (uint64_t)(uint32_t)i3;
    uint64_t h = splitmix64(k ^ splitmix64(seed));
    double u = (double)(h >> 11) * (1.0 / 9007199254740992.0); /* [0,1) */
    u = 2.0 * u - 1.0;
    return w2 * w3 * (dsph / 8.0) * u;
}

/* exact test: does the sphere with diameter |xi - xi1| through xi and xi1
 * meet the closed box [lo,hi]? (surface intersects iff dmin <= r <= dmax) */
static inline int sphere_meets_box(const double *lo, const double *hi, double mu, double mv, double mw,
                                   double r)
{
    double m[3] = {mu, mv, mw}, dmin = 0.0, dmax = 0.0;
    for (int k = 0; k < 3; k++) {
        double a = lo[k] - m[k], b = m[k] - hi[k];
        double t = a > 0.0 ? a : (b > 0.0 ? b : 0.0);
        dmin += t * t;
        double fa = fabs(m[k] - lo[k]), fb = fabs(m[k] - hi[k]);
        double fm = fa > fb ? fa : fb;
        dmax += fm * fm;
    }
    double r2 = r * r;
    return (r2 >= dmin) && (r2 <= dmax);
}

int64_t dgvo_synth_A(const dgvo_ctx *c, uint64_t seed, double Trad, int support_mode, int32_t p_only,
                     int32_t **capphi_out, double **Aout, int32_t **xiout, int32_t **xi1out)
{
    int64_t N = c->N;
    int32_t P = c->P, cc = c->ccell;
    double uu[2] = {c->clu[cc], c->cru[cc]}, vv[2] = {c->clv[cc], c->crv[cc]}, ww[2] = {c->clw[cc], c->crw[cc]};
    double dphi = sqrt((uu[1] - uu[0]) * (uu[1] - uu[0]) + (vv[1] - vv[0]) * (vv[1] - vv[0]) +
                       (ww[1] - ww[0]) * (ww[1] - ww[0]));
    double lo[3] = {uu[0], vv[0], ww[0]}, hi[3] = {uu[1], vv[1], ww[1]};
    /* pass 1: the p-independent pair list */
    int64_t *cnt = calloc((size_t)N + 1, sizeof(int64_t));
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int64_t i2 = 0; i2 < N; i2++) {
        int64_t n = 0;
        for (int64_t i3 = i2 + 1; i3 < N; i3++) {
            double dsph;
            if (!prefilter_pass(uu, vv, ww, dphi, Trad, c->nu[i2], c->nv[i2], c->nw[i2], c->nu[i3],
                                c->nv[i3], c->nw[i3], &dsph))
                continue;
            if (support_mode == 1 &&
                !sphere_meets_box(lo, hi, (c->nu[i2] + c->nu[i3]) / 2.0, (c->nv[i2] + c->nv[i3]) / 2.0,
                                  (c->nw[i2] + c->nw[i3]) / 2.0, dsph / 2.0))
                continue;
            n++;
        }
        cnt[i2] = n;
    }
    int64_t *off = malloc(sizeof(int64_t) * ((size_t)N + 1));
    off[0] = 0;
    for (int64_t i = 0; i < N; i++) off[i + 1] = off[i] + cnt[i];
    int64_t npairs = off[N];
    int32_t *pb = malloc(sizeof(int32_t) * (npairs ? npairs : 1));
    double *pd = malloc(sizeof(double) * (npairs ? npairs : 1));
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int64_t i2 = 0; i2 < N; i2++) {
        int64_t k = off[i2];
        for (int64_t i3 = i2 + 1; i3 < N; i3++) {
            double dsph;
            if (!prefilter_pass(uu, vv, ww, dphi, Trad, c->nu[i2], c->nv[i2], c->nw[i2], c->nu[i3],
                                c->nv[i3], c->nw[i3], &dsph))
                continue;
            if (support_mode == 1 &&
                !sphere_meets_box(lo, hi, (c->nu[i2] + c->nu[i3]) / 2.0, (c->nv[i2] + c->nv[i3]) / 2.0,
                                  (c->nw[i2] + c->nw[i3]) / 2.0, dsph / 2.0))
                continue;
            pb[k] = (int32_t)i3; pd[k] = dsph; k++;
        }
    }
    /* one basis function (p_only) or all of them; with P = 1 both are p = 0 */
    const int single = p_only >= 0 && p_only < P;
    int32_t np_ = single ? 1 : P;
    int64_t nnz = npairs * np_;
    int32_t *capphi = calloc((size_t)N, sizeof(int32_t));
    double *A = malloc(sizeof(double) * (nnz ? nnz : 1));
    int32_t *X = malloc(sizeof(int32_t) * (nnz ? nnz : 1)), *X1 = malloc(sizeof(int32_t) * (nnz ? nnz : 1));
    for (int32_t t = 0; t < np_; t++) capphi[(int64_t)cc * P + (single ? p_only : t)] = (int32_t)npairs;
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int32_t t = 0; t < np_; t++) {
        int32_t p = single ? p_only : t;
        int64_t base = (int64_t)t * npairs;
        for (int64_t i2 = 0; i2 < N; i2++)
            for (int64_t k = off[i2]; k < off[i2 + 1]; k++) {
                int32_t i3 = pb[k];
                A[base + k] = dgvo_synth_value(seed, p, (int32_t)i2, i3, c->nwt[i2], c->nwt[i3], pd[k]);
                X[base + k] = (int32_t)i2;
                X1[base + k] = i3;
            }
    }
    free(cnt); free(off); free(pb); free(pd);
    *capphi_out = capphi; *Aout = A; *xiout = X; *xi1out = X1;
    return nnz;
}

void dgvo_free(void *p) { free(p); }
