// api.cu -- the extern "C" entry points of libdgv_b200.so (include/dgv_b200.h).
// Host pointers are staged through device buffers owned by the context;
// device pointers are used in place.  No entry point aborts: failures return
// a status code and leave a message for dgv_last_error.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <new>

#include "dgv_internal.h"

namespace dgv {

void release_graphs(const Ctx *c);
int vjp_device(Ctx *c, const double *d_f, const double *d_v, double *d_g, int precision);

int set_err(Ctx *c, int code, const std::string &msg)
{
    if (c) c->err = msg;
    return code;
}

// Grows a device work buffer.  A reallocation moves the buffer, so every CUDA
// graph captured on this context (which holds the old address) is released
// first and re-captured on demand.
int ensure_buffer(Ctx *c, double **p, size_t *have, size_t need_bytes)
{
    if (*have >= need_bytes && *p) return DGV_OK;
    release_graphs(c);
    if (*p) {
        cudaStreamSynchronize(c->stream);
        cudaFree(*p);
        *p = nullptr;
        *have = 0;
    }
    cudaError_t e = cudaMalloc((void **)p, need_bytes ? need_bytes : 8);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return set_err(c, DGV_ENOMEM, std::string("device allocation of ") + std::to_string(need_bytes) +
                                          " bytes failed: " + cudaGetErrorString(e));
    }
    *have = need_bytes;
    return DGV_OK;
}

int ensure_errflag(Ctx *c)
{
    if (c->d_err) return DGV_OK;
    DGV_CUDA(c, cudaHostAlloc((void **)&c->h_err, sizeof(int), cudaHostAllocMapped));
    *(volatile int *)c->h_err = 0;
    DGV_CUDA(c, cudaHostGetDevicePointer((void **)&c->d_err, c->h_err, 0));
    return DGV_OK;
}

// After the stream has synchronised: report (and clear) a bounded device wait
// that gave up.
int check_errflag(Ctx *c)
{
    if (c->h_err && *(volatile int *)c->h_err) {
        *(volatile int *)c->h_err = 0;
        return set_err(c, DGV_ETIMEOUT, "a bounded device wait in a collision kernel gave up; results discarded");
    }
    return DGV_OK;
}

// Where an array lives: *dev = true for memory of the context's device (or
// managed memory), false for host memory; device memory of another GPU is
// refused (a kernel of this context cannot read it safely).
int classify_ptr(Ctx *c, const void *p, bool *dev)
{
    cudaPointerAttributes at;
    *dev = false;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return DGV_OK;
    }
    if (at.type == cudaMemoryTypeManaged) {
        *dev = true;
    } else if (at.type == cudaMemoryTypeDevice) {
        if (at.device != c->device)
            return set_err(c, DGV_EINVAL, "an array lives on device " + std::to_string(at.device) +
                                              ", the context on device " + std::to_string(c->device));
        *dev = true;
    }
    return DGV_OK;
}

// Inverse of the Gram matrix G_ab = sum_i w_i psi_a psi_b of the invariants
static int gram_inverse(Ctx *c)
{
    const Grid &g = c->grid;
    double G[5][10] = {{0}};
    for (long long i = 0; i < g.N; i++) {
        double u = g.nu[i], v = g.nv[i], w = g.nw[i];
        double psi[5] = {1.0, u, v, w, u * u + v * v + w * w};
        for (int a = 0; a < 5; a++)
            for (int b = 0; b < 5; b++) G[a][b] += g.nwt[i] * psi[a] * psi[b];
    }
    for (int a = 0; a < 5; a++) G[a][5 + a] = 1.0;
    for (int k = 0; k < 5; k++) {
        int piv = k;
        for (int r = k + 1; r < 5; r++)
            if (std::fabs(G[r][k]) > std::fabs(G[piv][k])) piv = r;
        if (G[piv][k] == 0.0) return set_err(c, DGV_EINVAL, "grid: singular invariant Gram matrix");
        if (piv != k)
            for (int b = 0; b < 10; b++) std::swap(G[k][b], G[piv][b]);
        double d = G[k][k];
        for (int b = 0; b < 10; b++) G[k][b] /= d;
        for (int r = 0; r < 5; r++)
            if (r != k) {
                double fct = G[r][k];
                for (int b = 0; b < 10; b++) G[r][b] -= fct * G[k][b];
            }
    }
    for (int a = 0; a < 5; a++)
        for (int b = 0; b < 5; b++) c->gram_inv[a * 5 + b] = G[a][5 + b];
    return DGV_OK;
}

KTimer::KTimer(Ctx *ctx) : c(ctx)
{
    if (!c->ktiming) return;
    cudaStreamCaptureStatus st = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(c->stream, &st) != cudaSuccess || st != cudaStreamCaptureStatusNone) return;
    if (!c->kt_pool.empty()) {
        ev = c->kt_pool.back();
        c->kt_pool.pop_back();
    } else if (cudaEventCreate(&ev.first) != cudaSuccess || cudaEventCreate(&ev.second) != cudaSuccess) {
        return;
    }
    on = cudaEventRecord(ev.first, c->stream) == cudaSuccess;
}

void KTimer::stop(long long nlaunch)
{
    if (!on) return;
    if (cudaEventRecord(ev.second, c->stream) == cudaSuccess) {
        c->kt_pending.push_back(ev);
        c->kt_launches += nlaunch;
    }
    on = false;
}

void count_launches(Ctx *c, long long n)
{
    c->kt_all += n;
}

void free_ktimers(Ctx *c)
{
    for (auto *v : {&c->kt_pending, &c->kt_pool})
        for (auto &pr : *v) {
            if (pr.first) cudaEventDestroy(pr.first);
            if (pr.second) cudaEventDestroy(pr.second);
        }
    c->kt_pending.clear();
    c->kt_pool.clear();
}

static void destroy_ctx(Ctx *c)
{
    cudaSetDevice(c->device);
    release_graphs(c);
    free_ktimers(c);
    free_layout(c->lay);
    double *bufs[] = {c->d_nu, c->d_nv, c->d_nw, c->d_nwt, c->d_partial, c->d_in, c->d_out, c->d_red, c->d_fm,
                      c->d_tcF, c->d_tcQ, c->d_glm, c->d_fg, c->d_tc2done, c->d_fmn, c->d_dfr, c->d_rgt};
    for (double *p : bufs)
        if (p) cudaFree(p);
    for (double *p : c->d_tmp)
        if (p) cudaFree(p);
    for (double *p : c->d_hist)
        if (p) cudaFree(p);
    if (c->h_err) cudaFreeHost(c->h_err);
    if (c->own_stream) cudaStreamDestroy(c->own_stream);
}

// Stage an input array: device pointers pass through, host arrays are copied
// into the context's input buffer at offset `slot` (in doubles).
// Grows the input staging buffer to `need_doubles`, keeping its contents.
// Growth moves the buffer: pointers handed out by stage_in before it are
// invalid afterwards, so calls that stage several inputs reserve the total
// first.
static int reserve_in(Ctx *c, size_t need_doubles)
{
    const size_t need = need_doubles * sizeof(double);
    if (c->in_bytes >= need) return DGV_OK;
    release_graphs(c);  // the move invalidates captured graphs
    double *nb = nullptr;
    DGV_CUDA(c, cudaMalloc(&nb, need));
    if (c->d_in) {
        DGV_CUDA(c, cudaMemcpyAsync(nb, c->d_in, c->in_bytes, cudaMemcpyDeviceToDevice, c->stream));
        DGV_CUDA(c, cudaStreamSynchronize(c->stream));
        cudaFree(c->d_in);
    }
    c->d_in = nb;
    c->in_bytes = need;
    return DGV_OK;
}

static int stage_in(Ctx *c, const double *p, size_t n, size_t slot, const double **d)
{
    bool dev = false;
    int rc = classify_ptr(c, p, &dev);
    if (rc) return rc;
    if (dev) { *d = p; return DGV_OK; }
    rc = reserve_in(c, slot + n);
    if (rc) return rc;
    DGV_CUDA(c, cudaMemcpyAsync(c->d_in + slot, p, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    *d = c->d_in + slot;
    return DGV_OK;
}

static int out_ptr(Ctx *c, double *p, size_t n, double **d, bool *host)
{
    bool dev = false;
    int rc = classify_ptr(c, p, &dev);
    if (rc) return rc;
    if (dev) { *d = p; *host = false; return DGV_OK; }
    rc = ensure_buffer(c, &c->d_out, &c->out_bytes, n * sizeof(double));
    if (rc) return rc;
    *d = c->d_out;
    *host = true;
    return DGV_OK;
}

static int finish(Ctx *c, double *host_dst, const double *d_src, size_t n, bool host)
{
    if (host) DGV_CUDA(c, cudaMemcpyAsync(host_dst, d_src, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (host || !c->async) {
        DGV_CUDA(c, cudaStreamSynchronize(c->stream));
        return check_errflag(c);
    }
    return DGV_OK;
}

}  // namespace dgv

using namespace dgv;

#define CTX_CHECK(ctx)                                   \
    do {                                                 \
        if (!(ctx)) return DGV_EINVAL;                   \
        (ctx)->c.err.clear();                            \
        if (cudaSetDevice((ctx)->c.device) != cudaSuccess) \
            return set_err(&(ctx)->c, DGV_ECUDA, "cudaSetDevice failed"); \
    } while (0)

#define TRY(x)               \
    do {                     \
        int rc_ = (x);       \
        if (rc_) return rc_; \
    } while (0)

extern "C" {

int dgv_ctx_create(const dgv_grid_desc *desc, int device, dgv_ctx **out)
{
    if (!desc || !out) return DGV_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return DGV_ECUDA;
    }
    if (cudaSetDevice(device) != cudaSuccess) return DGV_ECUDA;
    dgv_ctx *h = new (std::nothrow) dgv_ctx();
    if (!h) return DGV_ENOMEM;
    Ctx *c = &h->c;
    c->device = device;
    int rc = build_grid(*desc, c->grid, c->err);
    if (rc) { delete h; return rc; }
    rc = gram_inverse(c);
    if (rc) { delete h; return rc; }
    if (cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking) != cudaSuccess) { delete h; return DGV_ECUDA; }
    c->stream = c->own_stream;
    const Grid &g = c->grid;
    size_t nb = sizeof(double) * (size_t)g.N;
    double **dst[4] = {&c->d_nu, &c->d_nv, &c->d_nw, &c->d_nwt};
    const std::vector<double> *src[4] = {&g.nu, &g.nv, &g.nw, &g.nwt};
    for (int k = 0; k < 4; k++) {
        if (cudaMalloc(dst[k], nb) != cudaSuccess || cudaMemcpy(*dst[k], src[k]->data(), nb, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            destroy_ctx(c);
            delete h;
            return DGV_ENOMEM;
        }
    }
    if (ensure_errflag(c)) {
        destroy_ctx(c);
        delete h;
        return DGV_ECUDA;
    }
    noalloc_prepare(c);
    *out = h;
    return DGV_OK;
}

int dgv_ctx_destroy(dgv_ctx *ctx)
{
    if (!ctx) return DGV_EINVAL;
    destroy_ctx(&ctx->c);
    delete ctx;
    return DGV_OK;
}

const char *dgv_last_error(const dgv_ctx *ctx) { return ctx ? ctx->c.err.c_str() : "null context"; }

int dgv_set_stream(dgv_ctx *ctx, void *stream)
{
    CTX_CHECK(ctx);
    ctx->c.stream = stream ? (cudaStream_t)stream : ctx->c.own_stream;
    return DGV_OK;
}

int dgv_set_async(dgv_ctx *ctx, int async_flag)
{
    CTX_CHECK(ctx);
    ctx->c.async = async_flag != 0;
    return DGV_OK;
}

int dgv_set_option(dgv_ctx *ctx, int option, int64_t value)
{
    CTX_CHECK(ctx);
    switch (option) {
    case DGV_OPT_PROJECT: ctx->c.project = value != 0; return DGV_OK;
    case DGV_OPT_NCHUNKS:
        if (value < 0 || value > 65535) return set_err(&ctx->c, DGV_EINVAL, "nchunks out of range");
        ctx->c.nchunks_opt = (int)value;
        return DGV_OK;
    case DGV_OPT_KTIMING: ctx->c.ktiming = value != 0; return DGV_OK;
    case DGV_OPT_TCSETMB:
        if (value < 1 || value > 4096) return set_err(&ctx->c, DGV_EINVAL, "records per launch must be 1..4096 MB");
        ctx->c.tc_set_mb = (int)value;
        ctx->c.tc_user_launch = true;
        release_graphs(&ctx->c);
        return DGV_OK;
    case DGV_OPT_TCTILES:
        if (value != 1 && value != 2) return set_err(&ctx->c, DGV_EINVAL, "VDF tiles per CTA must be 1 or 2");
        ctx->c.tc_tiles_per_cta = (int)value;
        ctx->c.tc_user_launch = true;
        release_graphs(&ctx->c);
        return DGV_OK;
    case DGV_OPT_TCFORM:
        if (value != 1 && value != 2) return set_err(&ctx->c, DGV_EINVAL, "tensor-core form must be 1 or 2");
        ctx->c.tc_form = (int)value;
        release_graphs(&ctx->c);
        return DGV_OK;
    case DGV_OPT_WAIT_LIMIT_US:
        if (value < 0 || value > 60000000) return set_err(&ctx->c, DGV_EINVAL, "wait limit must be 0..60e6 us");
        ctx->c.wait_limit_us = value;
        release_graphs(&ctx->c);
        return DGV_OK;
    case DGV_OPT_TEST_WITHHOLD:
        ctx->c.test_withhold = value != 0;
        return DGV_OK;
    case DGV_OPT_TCPERSIST:
        if (value != 0 && value != 1) return set_err(&ctx->c, DGV_EINVAL, "persistent launches: 0 or 1");
        ctx->c.tc_persistent = (int)value;
        ctx->c.tc_user_launch = true;
        release_graphs(&ctx->c);
        return DGV_OK;
    case DGV_OPT_FGLOBAL:
        if (value != 0 && value != 1) return set_err(&ctx->c, DGV_EINVAL, "f placement must be 0 (auto) or 1 (global)");
        ctx->c.f_global = (int)value;
        ctx->c.tuned.clear();  // chunk counts were chosen for the other placement
        release_graphs(&ctx->c);
        return DGV_OK;
    case DGV_OPT_TCAUTOTUNE:
        ctx->c.tc_autotune = value != 0;
        if (!value) {  // back to the fixed defaults (unless the caller set them)
            ctx->c.tc_tuned.clear();
            ctx->c.tc_tuned_adj.clear();
            if (!ctx->c.tc_user_launch) {
                ctx->c.tc_tiles_per_cta = 2;
                ctx->c.tc_set_mb = 48;
                ctx->c.tc_persistent = 0;
            }
        }
        release_graphs(&ctx->c);
        return DGV_OK;
    default: return set_err(&ctx->c, DGV_EINVAL, "unknown option");
    }
}

int dgv_get_option(dgv_ctx *ctx, int option, int64_t *value)
{
    CTX_CHECK(ctx);
    const Ctx &c = ctx->c;
    if (!value) return set_err(&ctx->c, DGV_EINVAL, "get_option: NULL value");
    switch (option) {
    case DGV_OPT_PROJECT: *value = c.project ? 1 : 0; return DGV_OK;
    case DGV_OPT_NCHUNKS: *value = c.nchunks_opt; return DGV_OK;
    case DGV_OPT_KTIMING: *value = c.ktiming ? 1 : 0; return DGV_OK;
    case DGV_OPT_TCFORM: *value = c.tc_form; return DGV_OK;
    case DGV_OPT_TCTILES: *value = c.tc_tiles_per_cta; return DGV_OK;
    case DGV_OPT_TCSETMB: *value = c.tc_set_mb; return DGV_OK;
    case DGV_OPT_WAIT_LIMIT_US: *value = c.wait_limit_us; return DGV_OK;
    case DGV_OPT_TCAUTOTUNE: *value = c.tc_autotune ? 1 : 0; return DGV_OK;
    case DGV_OPT_TEST_WITHHOLD: *value = c.test_withhold ? 1 : 0; return DGV_OK;
    case DGV_OPT_FGLOBAL: *value = c.f_global; return DGV_OK;
    case DGV_OPT_TCPERSIST: *value = c.tc_persistent; return DGV_OK;
    default: return set_err(&ctx->c, DGV_EINVAL, "unknown option");
    }
}

int dgv_release_layouts(dgv_ctx *ctx, int mask, int64_t *freed_bytes)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (mask & ~(DGV_LAYOUT_F32 | DGV_LAYOUT_TC_CHUNK | DGV_LAYOUT_TC_BLOCK | DGV_LAYOUT_TC_ADJ))
        return set_err(c, DGV_EINVAL, "release_layouts: unknown layout bits");
    size_t free0 = 0, free1 = 0, total = 0;
    DGV_CUDA(c, cudaMemGetInfo(&free0, &total));
    int rc = release_layouts(c, mask);
    if (rc) return rc;
    DGV_CUDA(c, cudaMemGetInfo(&free1, &total));
    if (freed_bytes) *freed_bytes = (int64_t)free1 - (int64_t)free0;
    return DGV_OK;
}

int dgv_kernel_stats(dgv_ctx *ctx, double *ms, int64_t *launches, int64_t *all_launches, int reset)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    DGV_CUDA(c, cudaSetDevice(c->device));
    for (auto &pr : c->kt_pending) {
        float t = 0.f;
        DGV_CUDA(c, cudaEventSynchronize(pr.second));
        DGV_CUDA(c, cudaEventElapsedTime(&t, pr.first, pr.second));
        c->kt_ms += t;
        c->kt_pool.push_back(pr);
    }
    c->kt_pending.clear();
    if (ms) *ms = c->kt_ms;
    if (launches) *launches = c->kt_launches;
    if (all_launches) *all_launches = c->kt_all;
    if (reset) {
        c->kt_ms = 0.0;
        c->kt_launches = 0;
        c->kt_all = 0;
    }
    return DGV_OK;
}

int dgv_set_regime(dgv_ctx *ctx, double decomp_lev, double linear_lev)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (decomp_lev < 0.0 || linear_lev < 0.0) return set_err(c, DGV_EINVAL, "set_regime: levels must be >= 0");
    release_graphs(c);
    c->decomp_lev = decomp_lev;
    c->linear_lev = linear_lev;
    c->run_mode = 0;
    c->last_L1 = -1.0;
    return DGV_OK;
}

int dgv_regime_info(const dgv_ctx *ctx, int32_t *run_mode, double *last_L1)
{
    if (!ctx) return DGV_EINVAL;
    if (run_mode) *run_mode = ctx->c.run_mode;
    if (last_L1) *last_L1 = ctx->c.last_L1;
    return DGV_OK;
}

int dgv_grid_info(const dgv_ctx *ctx, int64_t *N, int32_t *P, int32_t *Nc, int32_t *ccell)
{
    if (!ctx) return DGV_EINVAL;
    const Grid &g = ctx->c.grid;
    if (N) *N = g.N;
    if (P) *P = g.P;
    if (Nc) *Nc = g.Nc;
    if (ccell) *ccell = g.ccell;
    return DGV_OK;
}

int dgv_nodes(const dgv_ctx *ctx, double *u, double *v, double *w, double *gwts)
{
    if (!ctx) return DGV_EINVAL;
    const Grid &g = ctx->c.grid;
    size_t nb = sizeof(double) * (size_t)g.N;
    if (u) std::memcpy(u, g.nu.data(), nb);
    if (v) std::memcpy(v, g.nv.data(), nb);
    if (w) std::memcpy(w, g.nw.data(), nb);
    if (gwts) std::memcpy(gwts, g.nwt.data(), nb);
    return DGV_OK;
}

int dgv_load_A(dgv_ctx *ctx, int64_t nnz, const int32_t *capphi, const double *A, const int32_t *A_xi,
               const int32_t *A_xi1, int one_based)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    release_graphs(c);
    free_layout(c->lay);
    c->tuned.clear();
    return layout_from_reference(c, nnz, capphi, A, A_xi, A_xi1, one_based);
}

int dgv_generate_A_synthetic(dgv_ctx *ctx, uint64_t seed, double Trad, int support_mode)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    release_graphs(c);
    c->tuned.clear();
    return layout_synthetic(c, seed, Trad, support_mode);
}

int dgv_compute_A(dgv_ctx *ctx, double Trad, double ErrChi, double ErrEps, double min_sens, int basis_mode)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    DGV_CUDA(c, cudaSetDevice(c->device));
    release_graphs(c);
    TRY(layout_seta(c, Trad, ErrChi, ErrEps, min_sens, basis_mode));
    return DGV_OK;
}

int dgv_A_info(const dgv_ctx *ctx, int64_t *nrecords, int64_t *npairs, int64_t *nblocks, double *record_shifts)
{
    if (!ctx) return DGV_EINVAL;
    const Layout &L = ctx->c.lay;
    if (nrecords) *nrecords = L.nrecords;
    if (npairs) *npairs = L.npairs;
    if (nblocks) *nblocks = L.nblocks;
    if (record_shifts) *record_shifts = L.record_shifts;
    return DGV_OK;
}

int dgv_export_A(const dgv_ctx *ctx, int64_t *nnz_out, int32_t *capphi, double *A, int32_t *A_xi, int32_t *A_xi1)
{
    if (!ctx || !nnz_out) return DGV_EINVAL;
    Ctx *c = const_cast<Ctx *>(&ctx->c);
    if (cudaSetDevice(c->device) != cudaSuccess) return DGV_ECUDA;
    long long n = 0;
    int rc = layout_export(c, &n, capphi, A, A_xi, A_xi1);
    *nnz_out = n;
    return rc;
}

int dgv_collide_batched(dgv_ctx *ctx, int32_t nb, const double *f, double *q, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (nb < 1 || !f || !q) return set_err(c, DGV_EINVAL, "collide: need nb >= 1 and non-NULL arrays");
    size_t n = (size_t)nb * (size_t)c->grid.N;
    const double *df;
    double *dq;
    bool host = false;
    TRY(stage_in(c, f, n, 0, &df));
    TRY(out_ptr(c, q, n, &dq, &host));
    TRY(collide_device(c, df, dq, nb, precision, 1.0));
    return finish(c, q, dq, n, host);
}

int dgv_collide_cells(dgv_ctx *ctx, int32_t nb, const double *f, double *q, int32_t cell0, int32_t cell1,
                      int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (nb < 1 || !f || !q) return set_err(c, DGV_EINVAL, "collide_cells: need nb >= 1 and non-NULL arrays");
    if (cell0 < 0 || cell1 > c->grid.Nc || cell0 >= cell1)
        return set_err(c, DGV_ERANGE, "collide_cells: cell range outside [0, Nc) or empty");
    size_t n = (size_t)nb * (size_t)c->grid.N;
    size_t nout = (size_t)nb * (size_t)(cell1 - cell0) * (size_t)c->grid.P;
    const double *df;
    double *dq;
    bool host = false;
    TRY(stage_in(c, f, n, 0, &df));
    TRY(out_ptr(c, q, nout, &dq, &host));
    TRY(collide_cells_device(c, df, dq, nb, precision, cell0, cell1));
    return finish(c, q, dq, nout, host);
}

int dgv_collide(dgv_ctx *ctx, const double *f, double *q, int64_t n, int precision)
{
    if (!ctx) return DGV_EINVAL;
    if (n != ctx->c.grid.N) return set_err(&ctx->c, DGV_EINVAL, "collide: n must equal the number of nodes");
    return dgv_collide_batched(ctx, 1, f, q, precision);
}

int dgv_spatial_oper(dgv_ctx *ctx, const double *f, double *fcol, double dt, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f || !fcol) return set_err(c, DGV_EINVAL, "spatial_oper: NULL array");
    size_t n = (size_t)c->grid.N;
    const double *df;
    double *dq;
    bool host = false;
    TRY(stage_in(c, f, n, 0, &df));
    TRY(out_ptr(c, fcol, n, &dq, &host));
    TRY(spatial_device(c, df, dq, dt, precision));
    return finish(c, fcol, dq, n, host);
}

// f is advanced in place; host f is staged in and copied back
int dgv_step_rk(dgv_ctx *ctx, double *f, double *frhs1, double dt, int order, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f) return set_err(c, DGV_EINVAL, "step_rk: NULL f");
    size_t n = (size_t)c->grid.N;
    bool fdev = false, rdev = false;
    TRY(classify_ptr(c, f, &fdev));
    if (frhs1) TRY(classify_ptr(c, frhs1, &rdev));
    bool rhost = frhs1 && !rdev;
    if (!fdev || rhost) TRY(ensure_buffer(c, &c->d_out, &c->out_bytes, 2 * n * sizeof(double)));
    double *df = fdev ? f : c->d_out;
    double *dr = rhost ? c->d_out + n : frhs1;
    if (!fdev) DGV_CUDA(c, cudaMemcpyAsync(df, f, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TRY(rk_step_device(c, df, dr, dt, order, precision));
    if (!fdev) DGV_CUDA(c, cudaMemcpyAsync(f, df, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (rhost) DGV_CUDA(c, cudaMemcpyAsync(frhs1, dr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (!fdev || rhost || !c->async) {
        DGV_CUDA(c, cudaStreamSynchronize(c->stream));
        return check_errflag(c);
    }
    return DGV_OK;
}

// nb VDFs advanced in place; host arrays are staged in and copied back
int dgv_step_rk_batched(dgv_ctx *ctx, int32_t nb, double *f, double *frhs1, double dt, int order, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f || nb < 1) return set_err(c, DGV_EINVAL, "step_rk_batched: need nb >= 1 and a non-NULL f");
    const size_t n = (size_t)nb * (size_t)c->grid.N;
    bool fdev = false, rdev = false;
    TRY(classify_ptr(c, f, &fdev));
    if (frhs1) TRY(classify_ptr(c, frhs1, &rdev));
    const bool rhost = frhs1 && !rdev;
    if (!fdev || rhost) TRY(ensure_buffer(c, &c->d_out, &c->out_bytes, 2 * n * sizeof(double)));
    double *df = fdev ? f : c->d_out;
    double *dr = rhost ? c->d_out + n : frhs1;
    if (!fdev) DGV_CUDA(c, cudaMemcpyAsync(df, f, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    TRY(rk_step_device(c, df, dr, dt, order, precision, nb));
    if (!fdev) DGV_CUDA(c, cudaMemcpyAsync(f, df, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (rhost) DGV_CUDA(c, cudaMemcpyAsync(frhs1, dr, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (!fdev || rhost || !c->async) {
        DGV_CUDA(c, cudaStreamSynchronize(c->stream));
        return check_errflag(c);
    }
    return DGV_OK;
}

static int ab_common(dgv_ctx *ctx, double *f, double dt, int order, int precision, bool prepare)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f) return set_err(c, DGV_EINVAL, "AB: NULL f");
    size_t n = (size_t)c->grid.N;
    bool fdev = false;
    TRY(classify_ptr(c, f, &fdev));
    double *df = f;
    if (!fdev) {
        TRY(ensure_buffer(c, &c->d_out, &c->out_bytes, n * sizeof(double)));
        df = c->d_out;
        DGV_CUDA(c, cudaMemcpyAsync(df, f, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    TRY(prepare ? ab_prepare_device(c, df, dt, order, precision) : ab_step_device(c, df, dt, precision));
    if (!fdev) DGV_CUDA(c, cudaMemcpyAsync(f, df, n * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    if (!fdev || !c->async) {
        DGV_CUDA(c, cudaStreamSynchronize(c->stream));
        return check_errflag(c);
    }
    return DGV_OK;
}

int dgv_prepare_ab(dgv_ctx *ctx, double *f, double dt, int order, int precision)
{
    return ab_common(ctx, f, dt, order, precision, true);
}

int dgv_step_ab(dgv_ctx *ctx, double *f, double dt, int precision)
{
    return ab_common(ctx, f, dt, 0, precision, false);
}

int dgv_moments(dgv_ctx *ctx, const double *f, double out[5])
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f || !out) return set_err(c, DGV_EINVAL, "moments: NULL array");
    const double *df;
    TRY(stage_in(c, f, (size_t)c->grid.N, 0, &df));
    return moments_device(c, df, 1, out);
}

int dgv_maxwellian(dgv_ctx *ctx, double T, double u0, double v0, double w0, double n, double *f)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f) return set_err(c, DGV_EINVAL, "maxwellian: NULL array");
    size_t N = (size_t)c->grid.N;
    double *df;
    bool host = false;
    TRY(out_ptr(c, f, N, &df, &host));
    TRY(maxwellian_device(c, T, u0, v0, w0, n, df));
    return finish(c, f, df, N, host);
}

int dgv_project(dgv_ctx *ctx, double *q, int32_t nb)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!q || nb < 1) return set_err(c, DGV_EINVAL, "project: need nb >= 1 and a non-NULL array");
    size_t n = (size_t)nb * (size_t)c->grid.N;
    bool dev = false;
    TRY(classify_ptr(c, q, &dev));
    double *dq = q;
    if (!dev) {
        TRY(ensure_buffer(c, &c->d_out, &c->out_bytes, n * sizeof(double)));
        dq = c->d_out;
        DGV_CUDA(c, cudaMemcpyAsync(dq, q, n * sizeof(double), cudaMemcpyHostToDevice, c->stream));
    }
    TRY(project_device(c, dq, nb));
    return finish(c, q, dq, n, !dev);
}

int dgv_jvp(dgv_ctx *ctx, const double *f, const double *df, double *q, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f || !df || !q) return set_err(c, DGV_EINVAL, "jvp: NULL array");
    size_t n = (size_t)c->grid.N;
    const double *d1, *d2;
    double *dq;
    bool host = false;
    TRY(reserve_in(c, 2 * n));  // both inputs staged: no move between them
    TRY(stage_in(c, f, n, 0, &d1));
    TRY(stage_in(c, df, n, n, &d2));
    TRY(out_ptr(c, q, n, &dq, &host));
    TRY(jvp_device(c, d1, d2, dq, precision));
    return finish(c, q, dq, n, host);
}

int dgv_vjp(dgv_ctx *ctx, const double *f, const double *v, double *g, int precision)
{
    return dgv_vjp_batched(ctx, 1, f, v, g, precision);
}

int dgv_vjp_batched(dgv_ctx *ctx, int32_t nb, const double *f, const double *v, double *g, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!f || !v || !g || nb < 1) return set_err(c, DGV_EINVAL, "vjp: need nb >= 1 and non-NULL arrays");
    if (precision != DGV_PREC_F64 && precision != DGV_PREC_TC)
        return set_err(c, DGV_EUNSUP, "vjp: FP64 (DGV_PREC_F64) or tensor cores (DGV_PREC_TC) only");
    const size_t N = (size_t)c->grid.N, n = (size_t)nb * N;
    const double *d1, *d2;
    double *dg;
    bool host = false;
    TRY(reserve_in(c, 2 * n));  // both inputs staged: no move between them
    TRY(stage_in(c, f, n, 0, &d1));
    TRY(stage_in(c, v, n, n, &d2));
    TRY(out_ptr(c, g, n, &dg, &host));
    if (precision == DGV_PREC_TC) {
        TRY(vjp_tc_device(c, d1, d2, dg, nb));
    } else {
        for (int32_t b = 0; b < nb; b++) TRY(vjp_device(c, d1 + b * N, d2 + b * N, dg + b * N, precision));
    }
    return finish(c, g, dg, n, host);
}

int dgv_prepare_linear(dgv_ctx *ctx, const double *fm)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!fm) return set_err(c, DGV_EINVAL, "prepare_linear: NULL array");
    size_t n = (size_t)c->grid.N;
    if (!c->d_fm) DGV_CUDA(c, cudaMalloc(&c->d_fm, n * sizeof(double)));
    DGV_CUDA(c, cudaMemcpyAsync(c->d_fm, fm, n * sizeof(double), cudaMemcpyDefault, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    return DGV_OK;
}

int dgv_apply_linear(dgv_ctx *ctx, const double *df, double *q, int precision)
{
    CTX_CHECK(ctx);
    Ctx *c = &ctx->c;
    if (!c->d_fm) return set_err(c, DGV_ESTATE, "apply_linear: call dgv_prepare_linear first");
    if (!df || !q) return set_err(c, DGV_EINVAL, "apply_linear: NULL array");
    size_t n = (size_t)c->grid.N;
    const double *d2;
    double *dq;
    bool host = false;
    TRY(stage_in(c, df, n, n, &d2));
    TRY(out_ptr(c, q, n, &dq, &host));
    TRY(jvp_device(c, c->d_fm, d2, dq, precision));
    return finish(c, q, dq, n, host);
}

}  // extern "C"
