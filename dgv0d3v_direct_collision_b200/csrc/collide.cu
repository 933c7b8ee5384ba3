// collide.cu -- the collision operator Q(f,f) on the device pair layout.
//
// Q_i = 2/w_i * sum_{records j of canonical basis fn p(i)} A_j f[xi_j + d_i] f[xi1_j + d_i]
// over the records whose shifted cells stay in the grid (collision_mod.f90:186-227).
//
// Kernel organisation (one CTA = one chunk of cell-pair blocks x one slice of
// output cells x one VDF):
//   * f of the VDF is staged once into shared memory, local-major
//     f_s[l*Nc + cell], so that the 32 lanes of a warp (32 consecutive output
//     cells D) gather 32 consecutive words: conflict-free;
//   * every thread owns one output cell D and keeps the P sums of its P
//     output nodes (D, p) in registers;
//   * a block's pairs are streamed with warp-uniform broadcast loads of their
//     rows (two shared-memory offsets + P values); for each pair the thread
//     forms prod = f_s[o1+D]*f_s[o2+D] once and does P multiply-adds, one per
//     canonical basis function -- the record structure is the same for every
//     p, so the two gathers are shared by P records;
//   * the block-level box test replaces the per-record bounds checks; warps
//     with no valid lane skip the block;
//   * per-chunk partial sums go to a scratch buffer and a second kernel adds
//     the chunks in a fixed order, divides by the node weight and scales:
//     results are deterministic run to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>

#include "dgv_internal.h"

namespace dgv {

struct CollideArgs {
    const double *f;        // [nvdf][N]
    const double *f2;       // second argument for the bilinear (JVP) form, or nullptr
    double *partial;        // [nvdf][nchunks][P][Nc]
    const BlockInfo *blk;
    const char *rows;
    const int *bounds;      // [nchunks+1]
    long long N;
    int Nc, Mv, Mw, nchunks, dcta, rowb;
};

// -------------------------------------------------------------------------
// FP64
template <int PV>
__global__ void __launch_bounds__(384, 1) k_collide_f64(CollideArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *f_s = reinterpret_cast<double *>(smem_raw);
    const int vdf = blockIdx.x, slice = blockIdx.y, chunk = blockIdx.z;
    const double *f = a.f + (size_t)vdf * a.N;
    for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
        int cell = (int)(i / PV), l = (int)(i - (long long)cell * PV);
        f_s[l * a.Nc + cell] = __ldg(f + i);
    }
    __syncthreads();
    constexpr int RD = ((1 + PV) + 1) / 2 * 2;
    const int D = slice * a.dcta + threadIdx.x;
    const bool inD = (int)threadIdx.x < a.dcta && D < a.Nc;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    double acc[PV];
#pragma unroll
    for (int j = 0; j < PV; j++) acc[j] = 0.0;
    const int b0 = a.bounds[chunk], b1 = a.bounds[chunk + 1];
    for (int b = b0; b < b1; ++b) {
        const BlockInfo bi = a.blk[b];
        const bool valid = inD && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] &&
                           Dw >= bi.lo[2] && Dw <= bi.hi[2];
        if (!__any_sync(0xffffffffu, valid)) continue;
        const double2 *row = reinterpret_cast<const double2 *>(a.rows + (size_t)bi.start * a.rowb);
        for (int k = 0; k < bi.count; ++k, row += RD / 2) {
            double rv[RD];
#pragma unroll
            for (int t = 0; t < RD / 2; t++) {
                double2 x = __ldg(row + t);
                rv[2 * t] = x.x;
                rv[2 * t + 1] = x.y;
            }
            if (valid) {
                long long o = __double_as_longlong(rv[0]);
                int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
                double prod = f_s[o1 + D] * f_s[o2 + D];
#pragma unroll
                for (int j = 0; j < PV; j++) acc[j] = fma(rv[1 + j], prod, acc[j]);
            }
        }
    }
    if (inD) {
        double *out = a.partial + ((size_t)vdf * a.nchunks + chunk) * PV * a.Nc;
#pragma unroll
        for (int j = 0; j < PV; j++) out[(size_t)j * a.Nc + D] = acc[j];
    }
}

// -------------------------------------------------------------------------
// FP32 products with compensated accumulation.  Within a group of at most
// 16 pairs the P partial sums run in FP32; each group sum is then added to a
// (sum, correction) pair with Knuth's branch-free two-sum, so the rounding of
// the long accumulation is carried along instead of lost.
__device__ __forceinline__ void two_sum_acc(float &s, float &c, float x)
{
    float t = s + x;
    float bp = t - s;
    float err = (s - (t - bp)) + (x - bp);
    s = t;
    c += err;
}

template <int PV>
__global__ void __launch_bounds__(384, 1) k_collide_f32c(CollideArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    float *f_s = reinterpret_cast<float *>(smem_raw);
    const int vdf = blockIdx.x, slice = blockIdx.y, chunk = blockIdx.z;
    const double *f = a.f + (size_t)vdf * a.N;
    for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
        int cell = (int)(i / PV), l = (int)(i - (long long)cell * PV);
        f_s[l * a.Nc + cell] = __double2float_rn(__ldg(f + i));
    }
    __syncthreads();
    constexpr int RW = ((2 + PV) + 3) / 4 * 4;
    const int D = slice * a.dcta + threadIdx.x;
    const bool inD = (int)threadIdx.x < a.dcta && D < a.Nc;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    float s[PV], cmp[PV], part[PV];
#pragma unroll
    for (int j = 0; j < PV; j++) { s[j] = 0.f; cmp[j] = 0.f; part[j] = 0.f; }
    const int b0 = a.bounds[chunk], b1 = a.bounds[chunk + 1];
    for (int b = b0; b < b1; ++b) {
        const BlockInfo bi = a.blk[b];
        const bool valid = inD && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] &&
                           Dw >= bi.lo[2] && Dw <= bi.hi[2];
        if (!__any_sync(0xffffffffu, valid)) continue;
        const float4 *row = reinterpret_cast<const float4 *>(a.rows + (size_t)bi.start * a.rowb);
        int n = 0;
        for (int k = 0; k < bi.count; ++k, row += RW / 4) {
            float rv[RW];
#pragma unroll
            for (int t = 0; t < RW / 4; t++) {
                float4 x = __ldg(row + t);
                rv[4 * t] = x.x; rv[4 * t + 1] = x.y; rv[4 * t + 2] = x.z; rv[4 * t + 3] = x.w;
            }
            if (valid) {
                int o1 = __float_as_int(rv[0]), o2 = __float_as_int(rv[1]);
                float prod = f_s[o1 + D] * f_s[o2 + D];
#pragma unroll
                for (int j = 0; j < PV; j++) part[j] = fmaf(rv[2 + j], prod, part[j]);
                if (++n == 16) {
#pragma unroll
                    for (int j = 0; j < PV; j++) { two_sum_acc(s[j], cmp[j], part[j]); part[j] = 0.f; }
                    n = 0;
                }
            }
        }
        if (valid && n) {
#pragma unroll
            for (int j = 0; j < PV; j++) { two_sum_acc(s[j], cmp[j], part[j]); part[j] = 0.f; }
        }
    }
    if (inD) {
        double *out = a.partial + ((size_t)vdf * a.nchunks + chunk) * PV * a.Nc;
#pragma unroll
        for (int j = 0; j < PV; j++) out[(size_t)j * a.Nc + D] = (double)s[j] + (double)cmp[j];
    }
}

// -------------------------------------------------------------------------
// Bilinear form for the Jacobian-vector product: prod = f(a) g(b) + g(a) f(b)
// (collision_mod.f90:290-292).  The second argument is gathered from global
// memory (L1/L2) so that the shared copy of f still fits at large grids.
template <int PV>
__global__ void __launch_bounds__(384, 1) k_bilinear_f64(CollideArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *f_s = reinterpret_cast<double *>(smem_raw);
    const int vdf = blockIdx.x, slice = blockIdx.y, chunk = blockIdx.z;
    const double *f = a.f + (size_t)vdf * a.N;
    const double *g = a.f2 + (size_t)vdf * a.N;
    for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
        int cell = (int)(i / PV), l = (int)(i - (long long)cell * PV);
        f_s[l * a.Nc + cell] = __ldg(f + i);
    }
    __syncthreads();
    constexpr int RD = ((1 + PV) + 1) / 2 * 2;
    const int D = slice * a.dcta + threadIdx.x;
    const bool inD = (int)threadIdx.x < a.dcta && D < a.Nc;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    double acc[PV];
#pragma unroll
    for (int j = 0; j < PV; j++) acc[j] = 0.0;
    const int b0 = a.bounds[chunk], b1 = a.bounds[chunk + 1];
    for (int b = b0; b < b1; ++b) {
        const BlockInfo bi = a.blk[b];
        const bool valid = inD && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] &&
                           Dw >= bi.lo[2] && Dw <= bi.hi[2];
        if (!__any_sync(0xffffffffu, valid)) continue;
        const double2 *row = reinterpret_cast<const double2 *>(a.rows + (size_t)bi.start * a.rowb);
        for (int k = 0; k < bi.count; ++k, row += RD / 2) {
            double rv[RD];
#pragma unroll
            for (int t = 0; t < RD / 2; t++) {
                double2 x = __ldg(row + t);
                rv[2 * t] = x.x;
                rv[2 * t + 1] = x.y;
            }
            if (valid) {
                long long o = __double_as_longlong(rv[0]);
                int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
                // global node index of the gathered shared-memory word o + D
                int q1 = o1 + D, q2 = o2 + D;
                int l1 = q1 / a.Nc, l2 = q2 / a.Nc;
                long long i1 = (long long)(q1 - l1 * a.Nc) * PV + l1;
                long long i2 = (long long)(q2 - l2 * a.Nc) * PV + l2;
                double prod = f_s[q1] * __ldg(g + i2) + __ldg(g + i1) * f_s[q2];
#pragma unroll
                for (int j = 0; j < PV; j++) acc[j] = fma(rv[1 + j], prod, acc[j]);
            }
        }
    }
    if (inD) {
        double *out = a.partial + ((size_t)vdf * a.nchunks + chunk) * PV * a.Nc;
#pragma unroll
        for (int j = 0; j < PV; j++) out[(size_t)j * a.Nc + D] = acc[j];
    }
}

// q[v][D*P+p] = scale * (2 * sum_chunks partial[v][chunk][p][D]) / w[D*P+p]
__global__ void k_reduce_chunks(const double *partial, const double *w, double *q, int nchunks, int P, int Nc,
                                long long N, int nvdf, double scale)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long tot = (long long)nvdf * N;
    if (idx >= tot) return;
    int v = (int)(idx / N);
    long long r = idx - (long long)v * N;
    int p = (int)(r / Nc), D = (int)(r - (long long)p * Nc);  // D fastest: coalesced partial reads
    const double *src = partial + ((size_t)v * nchunks * P + p) * Nc + D;
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++) s += src[(size_t)ch * P * Nc];
    long long i = (long long)D * P + p;
    double val = 2.0 * s / w[i];
    if (scale != 1.0) val = val * scale;
    q[(size_t)v * N + i] = val;
}

// -------------------------------------------------------------------------
typedef void (*KernelFn)(CollideArgs);

static KernelFn pick_kernel(int P, int precision, bool bilinear)
{
    if (bilinear) {
        switch (P) {
        case 1: return k_bilinear_f64<1>;
        case 8: return k_bilinear_f64<8>;
        case 27: return k_bilinear_f64<27>;
        default: return nullptr;
        }
    }
    if (precision == DGV_PREC_F64) {
        switch (P) {
        case 1: return k_collide_f64<1>;
        case 8: return k_collide_f64<8>;
        case 27: return k_collide_f64<27>;
        default: return nullptr;
        }
    }
    switch (P) {
    case 1: return k_collide_f32c<1>;
    case 8: return k_collide_f32c<8>;
    case 27: return k_collide_f32c<27>;
    default: return nullptr;
    }
}

struct LaunchShape {
    int dcta, slices, threads;
    size_t smem;
};

static LaunchShape shape_for(const Ctx *c, int precision)
{
    const Grid &g = c->grid;
    LaunchShape s;
    int nc32 = (g.Nc + 31) / 32 * 32;
    s.dcta = std::min(nc32, 384);
    s.slices = (g.Nc + s.dcta - 1) / s.dcta;
    s.threads = s.dcta;
    s.smem = (size_t)g.N * (precision == DGV_PREC_F64 ? sizeof(double) : sizeof(float));
    return s;
}

static int run_collide(Ctx *c, const double *d_f, const double *d_f2, double *d_q, int nvdf, int precision,
                       double scale, int nchunks)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    const bool bilinear = d_f2 != nullptr;
    KernelFn fn = pick_kernel(g.P, precision, bilinear);
    if (!fn) return set_err(c, DGV_EUNSUP, "collide: this build supports 1, 8 or 27 nodes per cell");
    LaunchShape sh = shape_for(c, bilinear ? DGV_PREC_F64 : precision);
    int maxsm = 0;
    DGV_CUDA(c, cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    if (sh.smem > (size_t)maxsm)
        return set_err(c, DGV_EUNSUP, "collide: f of one VDF does not fit in shared memory for this grid");
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    nchunks = std::max(1, std::min<int>(nchunks, (int)std::max<long long>(1, L.nblocks)));
    int *d_bounds = nullptr;
    int rc = get_chunks(c, nchunks, &d_bounds);
    if (rc) return rc;
    size_t need = (size_t)nvdf * nchunks * g.P * g.Nc * sizeof(double);
    rc = ensure_buffer(c, &c->d_partial, &c->partial_bytes, need);
    if (rc) return rc;
    CollideArgs a;
    a.f = d_f; a.f2 = d_f2; a.partial = c->d_partial; a.blk = L.blk;
    a.rows = (const char *)((precision == DGV_PREC_F64 || bilinear) ? L.rows64 : L.rows32);
    a.rowb = (precision == DGV_PREC_F64 || bilinear) ? L.RD64 * 8 : L.RW32 * 4;
    a.bounds = d_bounds; a.N = g.N; a.Nc = g.Nc; a.Mv = g.d.Mv; a.Mw = g.d.Mw;
    a.nchunks = nchunks; a.dcta = sh.dcta;
    if (nchunks > 65535) return set_err(c, DGV_EINVAL, "collide: at most 65535 chunks");
    // VDF fastest: the CTAs resident at one time work on the same chunk of
    // rows for different VDFs, so each row is fetched from HBM once and then
    // served from L2
    fn<<<dim3(nvdf, sh.slices, nchunks), sh.threads, sh.smem, c->stream>>>(a);
    DGV_CUDA(c, cudaGetLastError());
    long long tot = (long long)nvdf * g.N;
    k_reduce_chunks<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->d_partial, c->d_nwt, d_q, nchunks, g.P,
                                                                             g.Nc, g.N, nvdf, scale);
    DGV_CUDA(c, cudaGetLastError());
    return DGV_OK;
}

// Chunk count.  Many VDFs: the smallest count whose last wave of CTAs is at
// least 90% full (one CTA per SM: the shared copy of f takes most of it).
// Few VDFs: measured -- each candidate is timed once and the fastest kept.
static int choose_chunks(Ctx *c, const double *d_f, const double *d_f2, double *d_q, int nvdf, int precision)
{
    if (c->nchunks_opt > 0) return c->nchunks_opt;
    const Grid &g = c->grid;
    LaunchShape sh = shape_for(c, precision);
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    long long units = (long long)nvdf * sh.slices;
    if (units >= 2LL * nsm) {
        for (int k = 1; k <= 8; k++) {
            long long ctas = units * k;
            long long waves = (ctas + nsm - 1) / nsm;
            if ((double)ctas / (double)(waves * nsm) >= 0.9) return k;
        }
        return 8;
    }
    long long key = ((long long)precision << 40) ^ ((long long)(d_f2 != nullptr) << 39) ^ nvdf;
    auto it = c->tuned.find(key);
    if (it != c->tuned.end()) return it->second;
    int base = (int)std::max<long long>(1, (long long)nsm / units);
    int cand[4] = {base, 2 * base, 4 * base, 8 * base};
    float best_ms = 1e30f;
    int best = cand[1];
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int t = 0; t < 4; t++) {
        if (run_collide(c, d_f, d_f2, d_q, nvdf, precision, 1.0, cand[t])) break;  // warm-up
        cudaEventRecord(e0, c->stream);
        run_collide(c, d_f, d_f2, d_q, nvdf, precision, 1.0, cand[t]);
        cudaEventRecord(e1, c->stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best_ms) { best_ms = ms; best = cand[t]; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->tuned[key] = best;
    (void)g;
    return best;
}

int collide_device(Ctx *c, const double *d_f, double *d_q, int nvdf, int precision, double scale)
{
    if (!c->lay.blk) return set_err(c, DGV_ESTATE, "collide: no A-arrays loaded");
    if (precision != DGV_PREC_F64 && precision != DGV_PREC_F32C)
        return set_err(c, DGV_EINVAL, "collide: unknown precision");
    int nch = choose_chunks(c, d_f, nullptr, d_q, nvdf, precision);
    int rc = run_collide(c, d_f, nullptr, d_q, nvdf, precision, scale, nch);
    if (rc) return rc;
    if (c->project) return project_device(c, d_q, nvdf);
    return DGV_OK;
}

int jvp_device(Ctx *c, const double *d_f, const double *d_df, double *d_q, int precision)
{
    if (!c->lay.blk) return set_err(c, DGV_ESTATE, "jvp: no A-arrays loaded");
    (void)precision;
    int nch = choose_chunks(c, d_f, d_df, d_q, 1, DGV_PREC_F64);
    // the bilinear kernel sums 2/w * A * (f g + g f) / 2 * 2: the reduce
    // kernel's factor 2 is the reference's "2*fc/w" (collision_mod.f90:326)
    return run_collide(c, d_f, d_df, d_q, 1, DGV_PREC_F64, 1.0, nch);
}

}  // namespace dgv
