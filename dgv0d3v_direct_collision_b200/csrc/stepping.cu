// stepping.cu -- moments, equilibrium, conservation projection and the
// Runge-Kutta / Adams-Bashforth drivers around the collision operator.
// Compiled with -fmad=false: every stage combination evaluates the reference
// expression with the same operations in the same order (divisions by the
// literal constants included), so the stepping adds no rounding of its own
// beyond the reference's.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "dgv_internal.h"

namespace dgv {

// ---------------------------------------------------------------------------
// deterministic weighted sums: NPART fixed CTAs per VDF, fixed-order trees
constexpr int NPART = 32;
constexpr int RED_THREADS = 256;

// Sums over nodes of w_i * x_i * psi_k(v_i) for psi = 1, u, v, w, |v - ub|^2
// (kind 0: x = f, used by the moments; with center = ubar for the second
// pass) or psi = 1, u, v, w, |v|^2 (kind 1, used by the projection).
__global__ void k_wsum5(const double *x, const double *nu, const double *nv, const double *nw, const double *nwt,
                        long long N, const double *center, double *part)
{
    const int v = blockIdx.y, b = blockIdx.x;
    const double *xv = x + (size_t)v * N;
    double cu = 0, cv = 0, cw = 0;
    if (center) { cu = center[v * 3]; cv = center[v * 3 + 1]; cw = center[v * 3 + 2]; }
    double s[5] = {0, 0, 0, 0, 0};
    for (long long i = (long long)b * RED_THREADS + threadIdx.x; i < N; i += (long long)NPART * RED_THREADS) {
        double fw = xv[i] * nwt[i];
        double u = nu[i], vv = nv[i], w = nw[i];
        s[0] += fw;
        s[1] += fw * u;
        s[2] += fw * vv;
        s[3] += fw * w;
        double du = u - cu, dv = vv - cv, dw = w - cw;
        s[4] += fw * (du * du + dv * dv + dw * dw);
    }
    __shared__ double sh[5][RED_THREADS];
    for (int k = 0; k < 5; k++) sh[k][threadIdx.x] = s[k];
    __syncthreads();
    for (int off = RED_THREADS / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off)
            for (int k = 0; k < 5; k++) sh[k][threadIdx.x] += sh[k][threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x < 5) part[((size_t)v * NPART + b) * 5 + threadIdx.x] = sh[threadIdx.x][0];
}

// projection: q -= lam0 + lam1 u + lam2 v + lam3 w + lam4 |v|^2 with
// lam = G^{-1} m, m the invariant moments of q (fixed-order sum of partials)
struct Gram {
    double inv[25];
};

__global__ void k_project_apply(double *q, const double *nu, const double *nv, const double *nw, long long N,
                                const double *part, Gram g)
{
    const int v = blockIdx.y;
    __shared__ double lam[5];
    if (threadIdx.x == 0) {
        double m[5] = {0, 0, 0, 0, 0};
        for (int b = 0; b < NPART; b++)
            for (int k = 0; k < 5; k++) m[k] += part[((size_t)v * NPART + b) * 5 + k];
        for (int a = 0; a < 5; a++) {
            double s = 0;
            for (int k = 0; k < 5; k++) s += g.inv[a * 5 + k] * m[k];
            lam[a] = s;
        }
    }
    __syncthreads();
    double *qv = q + (size_t)v * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x) {
        double u = nu[i], vv = nv[i], w = nw[i];
        qv[i] -= lam[0] + lam[1] * u + lam[2] * vv + lam[3] * w + lam[4] * (u * u + vv * vv + w * w);
    }
}

static int ensure_red(Ctx *c, int nvdf)
{
    return ensure_buffer(c, &c->d_red, &c->red_bytes, ((size_t)nvdf * NPART * 5 + (size_t)nvdf * 3) * sizeof(double));
}

int project_device(Ctx *c, double *d_q, int nvdf)
{
    const Grid &g = c->grid;
    int rc = ensure_red(c, nvdf);
    if (rc) return rc;
    k_wsum5<<<dim3(NPART, nvdf), RED_THREADS, 0, c->stream>>>(d_q, c->d_nu, c->d_nv, c->d_nw, c->d_nwt, g.N, nullptr,
                                                            c->d_red);
    DGV_CUDA(c, cudaGetLastError());
    Gram gr;
    std::memcpy(gr.inv, c->gram_inv, sizeof(gr.inv));
    k_project_apply<<<dim3(64, nvdf), 256, 0, c->stream>>>(d_q, c->d_nu, c->d_nv, c->d_nw, g.N, c->d_red, gr);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 2);
    return DGV_OK;
}

// MassCheckRec (dgvtools_mod.f90:1437-1458): n, ubar, vbar, wbar, T
int moments_device(Ctx *c, const double *d_f, int nvdf, double *h_out)
{
    const Grid &g = c->grid;
    int rc = ensure_red(c, nvdf);
    if (rc) return rc;
    std::vector<double> part((size_t)nvdf * NPART * 5);
    k_wsum5<<<dim3(NPART, nvdf), RED_THREADS, 0, c->stream>>>(d_f, c->d_nu, c->d_nv, c->d_nw, c->d_nwt, g.N, nullptr,
                                                            c->d_red);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaMemcpyAsync(part.data(), c->d_red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    std::vector<double> center((size_t)nvdf * 3);
    for (int v = 0; v < nvdf; v++) {
        double s[5] = {0, 0, 0, 0, 0};
        for (int b = 0; b < NPART; b++)
            for (int k = 0; k < 4; k++) s[k] += part[((size_t)v * NPART + b) * 5 + k];
        h_out[v * 5 + 0] = s[0];
        for (int k = 1; k < 4; k++) h_out[v * 5 + k] = s[k] / s[0];
        for (int k = 0; k < 3; k++) center[(size_t)v * 3 + k] = h_out[v * 5 + 1 + k];
    }
    double *d_center = c->d_red + (size_t)nvdf * NPART * 5;
    DGV_CUDA(c, cudaMemcpyAsync(d_center, center.data(), center.size() * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    k_wsum5<<<dim3(NPART, nvdf), RED_THREADS, 0, c->stream>>>(d_f, c->d_nu, c->d_nv, c->d_nw, c->d_nwt, g.N, d_center,
                                                            c->d_red);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaMemcpyAsync(part.data(), c->d_red, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    for (int v = 0; v < nvdf; v++) {
        double st = 0;
        for (int b = 0; b < NPART; b++) st += part[((size_t)v * NPART + b) * 5 + 4];
        h_out[v * 5 + 4] = st / h_out[v * 5 + 0] / 3.0 * 2.0;
    }
    return DGV_OK;
}

// maxwelveldist (distributions_mod.f90:83-95)
__global__ void k_maxwellian(double *f, const double *nu, const double *nv, const double *nw, long long N, double T,
                             double u0, double v0, double w0, double n)
{
    const double pi = 3.141592653589793238462643;
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    double beta = sqrt(pi * T) * (pi * T);
    double tt = T > 0.0000001 ? T : 0.0000001;
    double du = nu[i] - u0, dv = nv[i] - v0, dw = nw[i] - w0;
    f[i] = n * exp(-(du * du + dv * dv + dw * dw) / tt) / beta;
}

int maxwellian_device(Ctx *c, double T, double u0, double v0, double w0, double n, double *d_f)
{
    long long N = c->grid.N;
    k_maxwellian<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(d_f, c->d_nu, c->d_nv, c->d_nw, N, T, u0, v0, w0, n);
    DGV_CUDA(c, cudaGetLastError());
    return DGV_OK;
}

// ---------------------------------------------------------------------------
// Stage combinations of TimeIntegratorORK_SH_DGV (time_integr_mod.f90:40-151)
// and TimeIntegratorMTS_SH_DGV (:325-363), written as in the reference.
enum StageOp {
    RK2_T2, RK2_F,                                   // :55-57
    RK3_T2, RK3_T3, RK3_F,                           // :76-82
    RK4_T2, RK4_T3, RK4_T4, RK4_F,                   // :97-104
    RK5_T2, RK5_T3, RK5_T4, RK5_FT3, RK5_T5, RK5_T6, RK5_F,  // :124-146
    RK1_F, DIV_DT,
    AB1_F, AB2_F, AB3_F, AB4_F, AB5_F
};

struct StageArgs {
    const double *f, *r1, *t2, *t3, *t4, *h2, *h3, *h4, *h5;
    double *out;
    long long n;
    double dt;
    int op;
};

__global__ void k_stage(StageArgs a)
{
    long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= a.n) return;
    const double dt = a.dt;
    double f = a.f ? a.f[i] : 0.0, r1 = a.r1 ? a.r1[i] : 0.0;
    double t2 = a.t2 ? a.t2[i] : 0.0, t3 = a.t3 ? a.t3[i] : 0.0, t4 = a.t4 ? a.t4[i] : 0.0;
    double y = 0.0;
    switch (a.op) {
    case RK1_F: y = f + r1; break;
    case RK2_T2: y = f + r1 * 2 / 3.0; break;
    case RK2_F: y = f + r1 / 4.0 + t2 * 3.0 / 4; break;
    case RK3_T2: y = f + r1 / 2.0; break;
    case RK3_T3: y = f + t2 * 3.0 / 4; break;
    case RK3_F: y = f + r1 * 2 / 9.0 + t2 * 3.0 / 9.0 + t3 * 4 / 9.0; break;
    case RK4_T2: y = f + r1 / 2.0; break;
    case RK4_T3: y = f + r1 / 4.0 + t2 / 4.0; break;
    case RK4_T4: y = f - t2 + t3 * 2; break;
    case RK4_F: y = f + r1 / 6.0 + t3 * 2 / 3.0 + t2 / 6.0; break;
    case RK5_T2: y = f + r1 / 2.0; break;
    case RK5_T3: y = f + r1 / 4.0 + t2 / 4.0; break;
    case RK5_T4: y = f - t2 + t3 * 2.0; break;
    case RK5_FT3: y = -t2 / 5.0 + t3 * 546 / 625.0; break;
    case RK5_T5: y = f + r1 * 7.0 / 27.0 + t2 * 10.0 / 27.0 + t4 / 27.0; break;
    case RK5_T6: y = f + r1 * 28.0 / 625.0 + t3 + t4 * 54 / 625.0 - t2 * 378 / 625.0; break;
    case RK5_F: y = f + r1 / 24.0 + t4 * 5.0 / 48.0 + t2 * 27.0 / 56.0 + t3 * 125 / 336.0; break;
    case DIV_DT: y = r1 / dt; break;
    case AB1_F: y = f + r1; break;
    case AB2_F: y = f + r1 * 3.0 / 2.0 - dt * a.h2[i] / 2.0; break;
    case AB3_F: y = f + r1 * 23.0 / 12.0 - dt * a.h2[i] * 4 / 3.0 + dt * a.h3[i] * 5.0 / 12.0; break;
    case AB4_F:
        y = f + r1 * 55.0 / 24.0 - dt * a.h2[i] * 59.0 / 24.0 + dt * a.h3[i] * 37.0 / 24.0 - dt * a.h4[i] * 3.0 / 8;
        break;
    case AB5_F:
        y = f + r1 * (1901.0 / 720.0) - dt * a.h2[i] * (2774.0 / 720.0) + dt * a.h3[i] * (2616.0 / 720.0) -
            dt * a.h4[i] * (1274.0 / 720.0) + dt * a.h5[i] * (251.0 / 720.0);
        break;
    }
    a.out[i] = y;
}

// the stage combination over the nb VDFs of a batch (nb * N entries; the
// coefficients do not depend on the VDF)
static int stage_nb(Ctx *c, int nb, int op, double *out, const double *f, const double *r1,
                    const double *t2 = nullptr, const double *t3 = nullptr, const double *t4 = nullptr,
                    double dt = 1.0, const double *h2 = nullptr, const double *h3 = nullptr,
                    const double *h4 = nullptr, const double *h5 = nullptr)
{
    StageArgs a;
    a.f = f; a.r1 = r1; a.t2 = t2; a.t3 = t3; a.t4 = t4; a.h2 = h2; a.h3 = h3; a.h4 = h4; a.h5 = h5;
    a.out = out; a.n = (long long)nb * c->grid.N; a.dt = dt; a.op = op;
    k_stage<<<(unsigned)((a.n + 255) / 256), 256, 0, c->stream>>>(a);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 1);
    return DGV_OK;
}

static int stage(Ctx *c, int op, double *out, const double *f, const double *r1, const double *t2 = nullptr,
                 const double *t3 = nullptr, const double *t4 = nullptr, double dt = 1.0,
                 const double *h2 = nullptr, const double *h3 = nullptr, const double *h4 = nullptr,
                 const double *h5 = nullptr)
{
    return stage_nb(c, 1, op, out, f, r1, t2, t3, t4, dt, h2, h3, h4, h5);
}

// the RK temporaries, for batches of up to nb VDFs; growing them releases
// the graphs that captured the old ones
static int ensure_tmp(Ctx *c, int nb = 1)
{
    const size_t need = (size_t)nb * (size_t)c->grid.N;
    if (c->tmp_n >= need && c->d_tmp[0]) return DGV_OK;
    release_graphs(c);
    for (auto &p : c->d_tmp) { if (p) cudaFree(p); p = nullptr; }
    c->tmp_n = 0;
    for (auto &p : c->d_tmp) DGV_CUDA(c, cudaMalloc(&p, sizeof(double) * need));
    c->tmp_n = need;
    return DGV_OK;
}

#define TRY(x)                 \
    do {                       \
        int rc_ = (x);         \
        if (rc_) return rc_;   \
    } while (0)

// SpatialOperSH_DGV (spat_oper_mod.f90:28-68), run_mode 0: Q scaled by kappa*dt
// sum_i |a_i - b_i| w_i: NPART fixed CTAs, fixed-order trees
__global__ void k_wl1(const double *a, const double *b, const double *w, long long N, double *part)
{
    double s = 0.0;
    for (long long i = (long long)blockIdx.x * RED_THREADS + threadIdx.x; i < N; i += (long long)NPART * RED_THREADS)
        s = s + fabs(a[i] - b[i]) * w[i];
    __shared__ double sh[RED_THREADS];
    sh[threadIdx.x] = s;
    __syncthreads();
    for (int off = RED_THREADS / 2; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
        __syncthreads();
    }
    if (threadIdx.x == 0) part[blockIdx.x] = sh[0];
}

// y = (a - b), or y = (a + b) * s, or y = a * s
__global__ void k_regime_combine(double *y, const double *a, const double *b, double s, int op, long long N)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    if (op == 0) y[i] = a[i] - b[i];
    else if (op == 1) y[i] = (a[i] + b[i]) * s;
    else y[i] = a[i] * s;
}

static int wl1(Ctx *c, const double *a, const double *b, double *out)
{
    TRY(ensure_red(c, 1));
    k_wl1<<<NPART, RED_THREADS, 0, c->stream>>>(a, b, c->d_nwt, c->grid.N, c->d_red);
    DGV_CUDA(c, cudaGetLastError());
    double part[NPART];
    DGV_CUDA(c, cudaMemcpyAsync(part, c->d_red, sizeof(part), cudaMemcpyDeviceToHost, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    double s = 0.0;
    for (int b2 = 0; b2 < NPART; b2++) s += part[b2];
    *out = s;
    return DGV_OK;
}

static int combine(Ctx *c, double *y, const double *a, const double *b, double s, int op)
{
    const long long N = c->grid.N;
    k_regime_combine<<<(unsigned)((N + 255) / 256), 256, 0, c->stream>>>(y, a, b, s, op, N);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 1);
    return DGV_OK;
}

// SpatialOperSH_DGV (spat_oper_mod.f90:28-68) with CheckSolutionMode_DGV
// (:195-272): the local Maxwellian fMN of f and the relative L1 distance
// sum |f - fMN| w / n decide the run mode -- 0 far from equilibrium: Q(f);
// 1 (distance < decomp_lev): L(Df) + Q(Df); 2 (distance < linear_lev): L(Df)
// only, Df = f - fm, L the linearised operator at fm (the mixed terms at fm,
// = 2 MATMUL(Df, fmA) of EvalCollisionLinear).  fm is replaced by fMN when a
// mode is entered from 0 or when it has drifted more than linear_lev/2 from
// fMN.  All times kappa*dt.  With decomp_lev = 0 the mode stays 0 (plain Q).
int spatial_device(Ctx *c, const double *x, double *out, double dt, int precision)
{
    const double coef = c->grid.d.kappa * dt;
    if (!(c->decomp_lev > 0.0)) return collide_device(c, x, out, 1, precision, coef);
    const size_t nb = sizeof(double) * (size_t)c->grid.N;
    TRY(ensure_buffer(c, &c->d_fmn, &c->fmn_bytes, nb));
    TRY(ensure_buffer(c, &c->d_dfr, &c->dfr_bytes, nb));
    TRY(ensure_buffer(c, &c->d_rgt, &c->rgt_bytes, nb));
    if (!c->d_fm) DGV_CUDA(c, cudaMalloc(&c->d_fm, nb));
    double m[5];
    TRY(moments_device(c, x, 1, m));
    TRY(maxwellian_device(c, m[4], m[1], m[2], m[3], m[0], c->d_fmn));
    double L1 = 0.0;
    TRY(wl1(c, x, c->d_fmn, &L1));
    L1 = L1 / m[0];
    c->last_L1 = L1;
    if (L1 < c->decomp_lev) {
        bool refresh = false;
        if (c->run_mode == 0) {
            refresh = true;
            c->run_mode = L1 < c->linear_lev ? 2 : 1;
        } else {
            double L1fm = 0.0;
            TRY(wl1(c, c->d_fm, c->d_fmn, &L1fm));
            L1fm = L1fm / m[0];
            if (L1fm > c->linear_lev / 2.0) refresh = true;
            if (c->run_mode == 1 && L1 < c->linear_lev) c->run_mode = 2;
            else if (c->run_mode == 2 && L1 > c->linear_lev) c->run_mode = 1;
        }
        if (refresh) DGV_CUDA(c, cudaMemcpyAsync(c->d_fm, c->d_fmn, nb, cudaMemcpyDeviceToDevice, c->stream));
        TRY(combine(c, c->d_dfr, x, c->d_fm, 0.0, 0));
    } else {
        c->run_mode = 0;
    }
    if (c->run_mode == 0) return collide_device(c, x, out, 1, precision, coef);
    const bool proj = c->project;
    c->project = false;
    int rc = jvp_device(c, c->d_fm, c->d_dfr, c->run_mode == 1 ? c->d_rgt : out, DGV_PREC_F64);
    if (!rc && c->run_mode == 1) {
        rc = collide_device(c, c->d_dfr, out, 1, precision, 1.0);
        if (!rc) rc = combine(c, out, out, c->d_rgt, coef, 1);  // (Q(Df) + L(Df)) * kappa dt
    } else if (!rc) {
        rc = combine(c, out, out, nullptr, coef, 2);
    }
    c->project = proj;
    if (rc) return rc;
    if (proj) return project_device(c, out, 1);
    return DGV_OK;
}

static int spatial(Ctx *c, const double *x, double *out, double dt, int precision)
{
    return spatial_device(c, x, out, dt, precision);
}

// one RK step of the given order for nb VDFs; d_r1 receives frhs1 (already
// divided by dt).  A batch evaluates Q of all its VDFs in one call per stage
// (run modes are per VDF and need nb = 1).
static int rk_body(Ctx *c, double *f, double *r1, double dt, int order, int precision, int nb = 1)
{
    double *t0 = c->d_tmp[0], *t2 = c->d_tmp[1], *t3 = c->d_tmp[2], *t4 = c->d_tmp[3];
    auto spatial = [c, nb](const double *x, double *out, double dt_, int prec) {
        return nb == 1 ? spatial_device(c, x, out, dt_, prec)
                       : collide_device(c, x, out, nb, prec, c->grid.d.kappa * dt_);
    };
    auto stage = [c, nb](int op, double *out, const double *f_, const double *r1_, const double *t2_ = nullptr,
                         const double *t3_ = nullptr, const double *t4_ = nullptr, double dt_ = 1.0) {
        return stage_nb(c, nb, op, out, f_, r1_, t2_, t3_, t4_, dt_);
    };
    switch (order) {
    case 1:
        TRY(spatial(f, r1, dt, precision));
        TRY(stage(RK1_F, f, f, r1));
        break;
    case 2:
        TRY(spatial(f, r1, dt, precision));
        TRY(stage(RK2_T2, t0, f, r1));
        TRY(spatial(t0, t2, dt, precision));
        TRY(stage(RK2_F, f, f, r1, t2));
        break;
    case 3:
        TRY(spatial(f, r1, dt, precision));
        TRY(stage(RK3_T2, t0, f, r1));
        TRY(spatial(t0, t2, dt, precision));
        TRY(stage(RK3_T3, t0, f, r1, t2));
        TRY(spatial(t0, t3, dt, precision));
        TRY(stage(RK3_F, f, f, r1, t2, t3));
        break;
    case 4:
        TRY(spatial(f, r1, dt, precision));
        TRY(stage(RK4_T2, t0, f, r1));
        TRY(spatial(t0, t2, dt, precision));
        TRY(stage(RK4_T3, t0, f, r1, t2));
        TRY(spatial(t0, t3, dt, precision));
        TRY(stage(RK4_T4, t0, f, r1, t2, t3));
        TRY(spatial(t0, t2, dt, precision));  // the 4th stage reuses ft2 (:102)
        TRY(stage(RK4_F, f, f, r1, t2, t3));
        break;
    case 5:
        TRY(spatial(f, r1, dt, precision));
        TRY(stage(RK5_T2, t0, f, r1));
        TRY(spatial(t0, t2, dt, precision));
        TRY(stage(RK5_T3, t0, f, r1, t2));
        TRY(spatial(t0, t3, dt, precision));
        TRY(stage(RK5_T4, t0, f, r1, t2, t3));
        TRY(spatial(t0, t4, dt, precision));
        TRY(stage(RK5_FT3, t3, nullptr, nullptr, t2, t3));
        TRY(stage(RK5_T5, t0, f, r1, t2, t3, t4));
        TRY(spatial(t0, t2, dt, precision));  // ft5 kept in ft2 (:136)
        TRY(stage(RK5_T6, t0, f, r1, t2, t3, t4));
        TRY(spatial(t0, t3, dt, precision));  // ft6 kept in ft3 (:140)
        TRY(stage(RK5_F, f, f, r1, t2, t3, t4));
        break;
    default:
        return set_err(c, DGV_EINVAL, "step_rk: order must be 1..5");
    }
    TRY(stage(DIV_DT, r1, nullptr, r1, nullptr, nullptr, nullptr, dt));
    return DGV_OK;
}

// The first call for a given (order, buffers, dt, precision) runs eagerly: it
// settles the autotuned chunk counts and grows every work buffer.  The second
// call captures the whole step into a CUDA graph; later calls replay it.
struct RkGraphKey {
    double *f, *r1;
    double dt;
    int order, precision, project, nb;
    bool operator<(const RkGraphKey &o) const
    {
        return std::memcmp(this, &o, sizeof(*this)) < 0;
    }
};
struct RkGraph {
    int calls = 0;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;  // kernels in the graph, counted while capturing
};
static std::map<const Ctx *, std::map<RkGraphKey, RkGraph>> g_graphs;
static std::recursive_mutex g_graphs_mu;  // contexts on different host threads share the cache

void release_group_graphs(const Ctx *c);

void release_graphs(const Ctx *c)
{
    release_group_graphs(c);
    std::lock_guard<std::recursive_mutex> lk(g_graphs_mu);
    auto it = g_graphs.find(c);
    if (it == g_graphs.end()) return;
    for (auto &kv : it->second)
        if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
    g_graphs.erase(it);
}

int rk_step_device(Ctx *c, double *d_f, double *d_frhs1, double dt, int order, int precision, int nb)
{
    if (order < 1 || order > 5) return set_err(c, DGV_EINVAL, "step_rk: order must be 1..5");
    if (nb < 1) return set_err(c, DGV_EINVAL, "step_rk: batch must hold at least one VDF");
    if (nb > 1 && c->decomp_lev > 0.0)
        return set_err(c, DGV_EUNSUP, "step_rk: run modes (dgv_set_regime) are per VDF; batches need them off");
    TRY(ensure_tmp(c, nb));
    double *r1 = d_frhs1 ? d_frhs1 : c->d_tmp[4];
    // with run modes the mode check synchronises on the host at every stage:
    // no graph capture
    if (c->decomp_lev > 0.0) return rk_body(c, d_f, r1, dt, order, precision);
    RkGraphKey key;
    std::memset(&key, 0, sizeof(key));
    key.f = d_f; key.r1 = r1; key.dt = dt; key.order = order; key.precision = precision; key.project = c->project;
    key.nb = nb;
    std::unique_lock<std::recursive_mutex> lk(g_graphs_mu);
    RkGraph &gr = g_graphs[c][key];
    if (gr.exec) {
        DGV_CUDA(c, cudaGraphLaunch(gr.exec, c->stream));
        count_launches(c, gr.launches);
        return DGV_OK;
    }
    if (gr.calls++ == 0) return rk_body(c, d_f, r1, dt, order, precision, nb);
    const long long before = c->kt_all;
    cudaGraph_t graph = nullptr;
    DGV_CUDA(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    int rc = rk_body(c, d_f, r1, dt, order, precision, nb);
    cudaError_t e = cudaStreamEndCapture(c->stream, &graph);
    if (rc) { if (graph) cudaGraphDestroy(graph); return rc; }
    if (e != cudaSuccess) return set_err(c, DGV_ECUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_err(c, DGV_ECUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    // looked up again: a buffer that grew while capturing released the cache
    RkGraph &g2 = g_graphs[c][key];
    if (g2.exec) cudaGraphExecDestroy(g2.exec);
    g2.exec = exec;
    g2.calls = 2;
    g2.launches = c->kt_all - before;
    DGV_CUDA(c, cudaGraphLaunch(exec, c->stream));
    return DGV_OK;
}

// ---------------------------------------------------------------------------
// Adams-Bashforth: d_hist[0..4] = frhs1..frhs5 (newest first)
static int ensure_hist(Ctx *c)
{
    for (auto &p : c->d_hist)
        if (!p) {
            DGV_CUDA(c, cudaMalloc(&p, sizeof(double) * (size_t)c->grid.N));
            DGV_CUDA(c, cudaMemsetAsync(p, 0, sizeof(double) * (size_t)c->grid.N, c->stream));
        }
    return DGV_OK;
}

// push the right-side history down by one for an order-k method:
// frhs_k = frhs_{k-1}, ..., frhs2 = frhs1 (pointer rotation)
static void push_hist(Ctx *c, int k)
{
    if (k < 2) return;
    double *last = c->d_hist[k - 1];
    for (int j = k - 1; j >= 1; j--) c->d_hist[j] = c->d_hist[j - 1];
    c->d_hist[0] = last;
}

int ab_prepare_device(Ctx *c, double *d_f, double dt, int order, int precision)
{
    if (order < 1 || order > 5) return set_err(c, DGV_EINVAL, "prepare_ab: order must be 1..5");
    TRY(ensure_tmp(c));
    TRY(ensure_hist(c));
    c->ab_order = order;
    // PrepareMTS_SH_DGV (time_integr_mod.f90:519-566): order-1 RK steps,
    // pushing frhs2..frhs(order-1) before each (for order 2 nothing is pushed)
    for (int i = 2; i <= order; i++) {
        if (order >= 3) push_hist(c, order - 1);
        TRY(rk_body(c, d_f, c->d_hist[0], dt, order, precision));
    }
    return DGV_OK;
}

// The multistep state a solution file keeps (WriteSol_DGV,
// readwrite.f90:1756-1800): the method order and frhs1..frhs(order-1),
// already divided by dt, newest first; host copies.
int ab_history_get(Ctx *c, int *order, std::vector<double> &frhs)
{
    *order = c->ab_order;
    const size_t N = (size_t)c->grid.N;
    frhs.assign(c->ab_order > 1 ? (size_t)(c->ab_order - 1) * N : 0, 0.0);
    for (int j = 0; j + 1 < c->ab_order; j++)
        DGV_CUDA(c, cudaMemcpyAsync(frhs.data() + (size_t)j * N, c->d_hist[j], N * sizeof(double),
                                    cudaMemcpyDeviceToHost, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    return DGV_OK;
}

int ab_history_set(Ctx *c, int order, const double *frhs)
{
    if (order < 1 || order > 5) return set_err(c, DGV_EINVAL, "solution file: method order outside 1..5");
    TRY(ensure_tmp(c));
    TRY(ensure_hist(c));
    const size_t N = (size_t)c->grid.N;
    for (int j = 0; j + 1 < order; j++)
        DGV_CUDA(c, cudaMemcpyAsync(c->d_hist[j], frhs + (size_t)j * N, N * sizeof(double), cudaMemcpyHostToDevice,
                                    c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    c->ab_order = order;
    return DGV_OK;
}

int ab_step_device(Ctx *c, double *d_f, double dt, int precision)
{
    int order = c->ab_order;
    if (order < 1) return set_err(c, DGV_ESTATE, "step_ab: call dgv_prepare_ab first");
    TRY(ensure_tmp(c));
    push_hist(c, order);
    double *r1 = c->d_hist[0];
    TRY(spatial(c, d_f, r1, dt, precision));
    static const int ops[6] = {0, AB1_F, AB2_F, AB3_F, AB4_F, AB5_F};
    TRY(stage(c, ops[order], d_f, d_f, r1, nullptr, nullptr, nullptr, dt, c->d_hist[1], c->d_hist[2], c->d_hist[3],
              c->d_hist[4]));
    TRY(stage(c, DIV_DT, r1, nullptr, r1, nullptr, nullptr, nullptr, dt));
    return DGV_OK;
}

}  // namespace dgv
