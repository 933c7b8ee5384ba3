// collide.cu -- the collision operator Q(f,f) on the device pair layout.
//
// Q_i = 2/w_i * sum_{records j of canonical basis fn p(i)} A_j f[xi_j + d_i] f[xi1_j + d_i]
// over the records whose shifted cells stay in the grid (collision_mod.f90:186-227).
//
// Kernel organisation (one CTA = one chunk of cell-pair blocks x one slice of
// output cells x one VDF):
//   * f of the VDF is staged once into shared memory, local-major
//     f_s[l*Nc + cell], so that the 32 lanes of a warp (32 consecutive output
//     cells D) gather 32 consecutive words: conflict-free; on grids whose f
//     does not fit (FP64: more than ~26 000 nodes), the gathers read a
//     local-major copy in global memory instead (GF: 256 contiguous bytes per
//     warp and gather, served by L1 and L2);
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
#include <type_traits>

#include "dgv_internal.h"
#include "pipeline.cuh"

namespace dgv {

enum CollideMode { MODE_F64 = 0, MODE_F32C = 1, MODE_BILINEAR = 2 };
constexpr int P_SLICE = 25;  // basis functions per CTA for grids of more than 27 nodes per cell

struct CollideArgs {
    const double *f;        // [nvdf][N]
    const double *f2;       // second argument for the bilinear (JVP) form, or nullptr
    double *partial;        // [nvdf][nchunks][P][Nc]
    const BlockInfo *blk;
    const char *rows;
    const int *bounds;      // [nchunks+1]
    int *err;               // raised by a bounded wait that gave up
    long long N;
    int Nc, Mv, Mw, nchunks, dcta, rowb;
    int cell0, cell1;       // output cells evaluated: [cell0, cell1)
    int nst, sp;            // pipeline stages, pairs per stage
    int off_f, off_hdr, off_bar;  // shared-memory layout (bytes)
    int Pt, npsl;           // nodes per cell; slices of PV basis functions per cell (1 unless sliced)
    const void *fg;         // GF: local-major copies of f, [nvdf][Pt*Nc] of the kernel's type
    unsigned long long wait_ns;  // limit of every bounded wait
};

// Knuth's branch-free two-sum: s + c carries x exactly
__device__ __forceinline__ void two_sum_acc(float &s, float &c, float x)
{
    float t = s + x;
    float bp = t - s;
    float err = (s - (t - bp)) + (x - bp);
    s = t;
    c += err;
}

// Shared memory: [NST stages of SP rows][f_s: local-major copy of f][stage
// headers][full/empty mbarriers].  Warp 0 is the producer (its lane 0 issues
// the bulk copies); the other warps are consumers, one output cell each.
//   MODE_F64      acc_p += v_p * f(a) f(b)                       (FP64)
//   MODE_F32C     FP32 products; groups of <= 16 pairs summed in FP32 and
//                 added to (sum, correction) with two-sum
//   MODE_BILINEAR acc_p += v_p * (f(a) g(b) + g(a) f(b)), g gathered from
//                 global memory (the Jacobian-vector product)
//
// SL (sliced, for many nodes per cell, e.g. P = 125): a CTA serves the PV
// basis functions p in [ps*PV, ps*PV + PV) of its output cells (ps =
// blockIdx.y % npsl), reading them from the full rows with scalar loads; the
// node stride is the runtime Pt.
// GF (f in global memory): the gathers read a.fg, a local-major copy of f made
// by k_f_local_major, instead of a shared-memory copy.
template <int PV, int MODE, bool SL = false, bool GF = false>
__global__ void __launch_bounds__(384, 1) k_collide_pipe(CollideArgs a)
{
    using T = typename std::conditional<MODE == MODE_F32C, float, double>::type;
    extern __shared__ __align__(128) unsigned char smem[];
    const size_t stage_bytes = (size_t)a.sp * a.rowb;
    unsigned char *stages = smem;
    T *f_s = reinterpret_cast<T *>(smem + a.off_f);
    StageHdr *hdr = reinterpret_cast<StageHdr *>(smem + a.off_hdr);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + a.off_bar);
    uint64_t *empty = full + a.nst;
    const int vdf = blockIdx.x, slice = SL ? blockIdx.y / a.npsl : blockIdx.y, chunk = blockIdx.z;
    const int PT = SL ? a.Pt : PV;                    // nodes per cell
    const int pofs = SL ? (blockIdx.y % a.npsl) * PV : 0;  // first basis function of the slice
    const int nconsumer_warps = a.dcta / 32;
    if (threadIdx.x == 0) {
        for (int s = 0; s < a.nst; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], nconsumer_warps);
        }
        fence_mbar_init();
    }
    const T *fgv = GF ? reinterpret_cast<const T *>(a.fg) + (size_t)vdf * a.N : nullptr;
    // f at local-major index q (l*Nc + cell)
    auto fat = [&](int q) -> T {
        if constexpr (GF) return __ldg(fgv + q);
        else return f_s[q];
    };
    if constexpr (!GF) {
        const double *f = a.f + (size_t)vdf * a.N;
        for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
            int cell = (int)(i / PT), l = (int)(i - (long long)cell * PT);
            f_s[l * a.Nc + cell] = (T)__ldg(f + i);
        }
    }
    __syncthreads();
    const int b0 = a.bounds[chunk], b1 = a.bounds[chunk + 1];
    const int d0 = a.cell0 + slice * a.dcta, d1 = min(a.cell1, d0 + a.dcta);

    if (threadIdx.x < 32) {  // producer: warp 0
        produce_rows(a.blk, b0, b1, a.Mv, a.Mw, d0, d1, a.rows, a.rowb, stages, a.sp, a.nst, hdr, full, empty, a.err,
                     a.wait_ns);
        return;
    }

    // ---------------- consumers: one output cell D per thread ----------------
    const int tc = threadIdx.x - 32, lane = threadIdx.x & 31;
    const int D = d0 + tc;
    const bool inD = tc < a.dcta && D < d1;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    const double *g = (MODE == MODE_BILINEAR) ? a.f2 + (size_t)vdf * a.N : nullptr;
    T acc[PV];
    float cmp[MODE == MODE_F32C ? PV : 1], part[MODE == MODE_F32C ? PV : 1];
#pragma unroll
    for (int j = 0; j < PV; j++) acc[j] = (T)0;
    if constexpr (MODE == MODE_F32C) {
#pragma unroll
        for (int j = 0; j < PV; j++) { cmp[j] = 0.f; part[j] = 0.f; }
    }
    int npend = 0;  // pairs in the open FP32 group
    int cur = -1;
    bool valid = false;
    constexpr int RD = ((1 + PV) + 1) / 2 * 2;  // FP64 row, doubles
    constexpr int RW = ((2 + PV) + 3) / 4 * 4;  // FP32 row, words
    for (int it = 0;; it++) {
        const int s = it % a.nst;
        if (!mbar_wait(&full[s], (it / a.nst) & 1, a.err, a.wait_ns)) break;
        const StageHdr h = hdr[s];
        if (h.block < 0) break;
        if (h.block != cur) {
            if constexpr (MODE == MODE_F32C) {
                if (valid && npend) {
#pragma unroll
                    for (int j = 0; j < PV; j++) { two_sum_acc(acc[j], cmp[j], part[j]); part[j] = 0.f; }
                    npend = 0;
                }
            }
            cur = h.block;
            const BlockInfo bi = a.blk[cur];
            valid = inD && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] && Dw >= bi.lo[2] &&
                    Dw <= bi.hi[2];
        }
        if (__any_sync(0xffffffffu, valid) && valid) {
            const unsigned char *st = stages + s * stage_bytes;
            // software pipeline over the stage's pairs: the gathers of pair k+1
            // are issued before the multiply-adds of pair k, so their latency
            // overlaps arithmetic
            if constexpr (MODE == MODE_F32C) {
                const int *ow = reinterpret_cast<const int *>(st);
                const int rws = a.rowb / 4;
                float pa = fat(ow[0] + D), pb = fat(ow[1] + D);
                for (int k = 0; k < h.n; k++) {
                    const float prod = pa * pb;
                    if (k + 1 < h.n) {
                        pa = fat(ow[(k + 1) * rws] + D);
                        pb = fat(ow[(k + 1) * rws + 1] + D);
                    }
                    if constexpr (SL) {
                        const float *rowf = reinterpret_cast<const float *>(st + (size_t)k * a.rowb) + 2 + pofs;
#pragma unroll
                        for (int j = 0; j < PV; j++) part[j] = fmaf(rowf[j], prod, part[j]);
                    } else {
                        const float4 *row = reinterpret_cast<const float4 *>(st + (size_t)k * a.rowb);
                        float rv[RW];
#pragma unroll
                        for (int t = 0; t < RW / 4; t++) {
                            float4 x = row[t];
                            rv[4 * t] = x.x; rv[4 * t + 1] = x.y; rv[4 * t + 2] = x.z; rv[4 * t + 3] = x.w;
                        }
#pragma unroll
                        for (int j = 0; j < PV; j++) part[j] = fmaf(rv[2 + j], prod, part[j]);
                    }
                    if (++npend == 16) {
#pragma unroll
                        for (int j = 0; j < PV; j++) { two_sum_acc(acc[j], cmp[j], part[j]); part[j] = 0.f; }
                        npend = 0;
                    }
                }
            } else {
                const int *ow = reinterpret_cast<const int *>(st);
                const int rws = a.rowb / 4;
                int q1 = ow[0] + D, q2 = ow[1] + D;
                double pa = fat(q1), pb = fat(q2);
                double ga = 0.0, gb = 0.0;
                if constexpr (MODE == MODE_BILINEAR) {
                    const int l1 = q1 / a.Nc, l2 = q2 / a.Nc;
                    ga = __ldg(g + (long long)(q1 - l1 * a.Nc) * PT + l1);
                    gb = __ldg(g + (long long)(q2 - l2 * a.Nc) * PT + l2);
                }
                for (int k = 0; k < h.n; k++) {
                    double prod;
                    if constexpr (MODE == MODE_BILINEAR) prod = pa * gb + ga * pb;
                    else prod = pa * pb;
                    if (k + 1 < h.n) {
                        q1 = ow[(k + 1) * rws] + D;
                        q2 = ow[(k + 1) * rws + 1] + D;
                        pa = fat(q1);
                        pb = fat(q2);
                        if constexpr (MODE == MODE_BILINEAR) {
                            const int l1 = q1 / a.Nc, l2 = q2 / a.Nc;
                            ga = __ldg(g + (long long)(q1 - l1 * a.Nc) * PT + l1);
                            gb = __ldg(g + (long long)(q2 - l2 * a.Nc) * PT + l2);
                        }
                    }
                    // values v[0..P-1] start at byte 8 of the row; each 16-byte
                    // load is consumed at once to keep few values live
                    if constexpr (SL) {
                        const double *rowd = reinterpret_cast<const double *>(st + (size_t)k * a.rowb) + 1 + pofs;
#pragma unroll
                        for (int j = 0; j < PV; j++) acc[j] = fma(rowd[j], prod, acc[j]);
                    } else {
                        const double2 *row2 = reinterpret_cast<const double2 *>(st + (size_t)k * a.rowb);
                        acc[0] = fma(row2[0].y, prod, acc[0]);
#pragma unroll
                        for (int t = 1; t < RD / 2; t++) {
                            const double2 x = row2[t];
                            if (2 * t - 1 < PV) acc[2 * t - 1] = fma(x.x, prod, acc[2 * t - 1]);
                            if (2 * t < PV) acc[2 * t] = fma(x.y, prod, acc[2 * t]);
                        }
                    }
                }
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
    if constexpr (MODE == MODE_F32C) {
        if (valid && npend) {
#pragma unroll
            for (int j = 0; j < PV; j++) { two_sum_acc(acc[j], cmp[j], part[j]); part[j] = 0.f; }
        }
    }
    if (inD) {
        double *out = a.partial + ((size_t)vdf * a.nchunks + chunk) * PT * a.Nc + (size_t)pofs * a.Nc;
#pragma unroll
        for (int j = 0; j < PV; j++) {
            double v = (double)acc[j];
            if constexpr (MODE == MODE_F32C) v += (double)cmp[j];
            if (!SL || pofs + j < PT) out[(size_t)j * a.Nc + D] = v;
        }
    }
}

// q[v][D*P+p - cell0*P] = scale * (2 * sum_chunks partial[v][chunk][p][D]) / w[D*P+p]
// for the output cells D in [cell0, cell1)
__global__ void k_reduce_chunks(const double *partial, const double *w, double *q, int nchunks, int P, int Nc,
                                int cell0, int cell1, int nvdf, double scale)
{
    const int ncell = cell1 - cell0;
    const long long len = (long long)ncell * P;
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nvdf * len) return;
    int v = (int)(idx / len);
    long long r = idx - (long long)v * len;
    int p = (int)(r / ncell), D = cell0 + (int)(r - (long long)p * ncell);  // D fastest: coalesced partial reads
    const double *src = partial + ((size_t)v * nchunks * P + p) * Nc + D;
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++) s += src[(size_t)ch * P * Nc];
    long long i = (long long)D * P + p;
    double val = 2.0 * s / w[i];
    if (scale != 1.0) val = val * scale;
    q[(size_t)v * len + (i - (long long)cell0 * P)] = val;
}

// -------------------------------------------------------------------------
typedef void (*KernelFn)(CollideArgs);

template <bool GF>
static KernelFn pick_kernel_gf(int P, int mode)
{
#define DGV_PICK(PV)                                                           \
    case PV:                                                                   \
        if (mode == MODE_F64) return k_collide_pipe<PV, MODE_F64, false, GF>;   \
        if (mode == MODE_F32C) return k_collide_pipe<PV, MODE_F32C, false, GF>; \
        return k_collide_pipe<PV, MODE_BILINEAR, false, GF>;
    switch (P) {
        DGV_PICK(1)
        DGV_PICK(8)
        DGV_PICK(27)
    case 125:  // slices of 25 basis functions per CTA
        if (mode == MODE_F64) return k_collide_pipe<P_SLICE, MODE_F64, true, GF>;
        if (mode == MODE_F32C) return k_collide_pipe<P_SLICE, MODE_F32C, true, GF>;
        return k_collide_pipe<P_SLICE, MODE_BILINEAR, true, GF>;
    default: return nullptr;
    }
#undef DGV_PICK
}

static KernelFn pick_kernel(int P, int mode, bool gf)
{
    return gf ? pick_kernel_gf<true>(P, mode) : pick_kernel_gf<false>(P, mode);
}

// out[v][l*Nc + cell] = (T) f[v][cell*P + l]: the local-major copies the GF
// kernels gather from (reads coalesced; writes strided by Nc)
template <typename T>
__global__ void k_f_local_major(const double *f, T *out, long long N, int Nc, int P, int nvdf)
{
    const long long tot = (long long)nvdf * N;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const long long v = i / N, r = i - v * N;
        const int cell = (int)(r / P), l = (int)(r - (long long)cell * P);
        out[v * N + (long long)l * Nc + cell] = (T)f[i];
    }
}

// basis functions per CTA of the sliced kernels, and the slices of a grid
static int p_slices(int P) { return P > 27 ? (P + P_SLICE - 1) / P_SLICE : 1; }

// FP32 rows from the FP64 rows: offsets copied, values rounded to nearest
// (as the layout builders write them)
__global__ void k_rows32_from64(const double *rows64, int RD64, float *rows32, int RW32, int P,
                                       long long npairs)
{
    const long long tot = npairs * RW32;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < tot; i += (long long)gridDim.x * blockDim.x) {
        const long long k = i / RW32;
        const int w = (int)(i - k * RW32);
        const double *r = rows64 + (size_t)k * RD64;
        float x = 0.f;
        if (w < 2) {
            int o[2];
            memcpy(o, r, 8);
            x = __int_as_float(o[w]);
        } else if (w - 2 < P) {
            x = __double2float_rn(r[1 + (w - 2)]);
        }
        rows32[i] = x;
    }
}

int ensure_rows32(Ctx *c)
{
    Layout &L = c->lay;
    if (L.rows32 || !L.rows64) return DGV_OK;
    const size_t bytes = (size_t)std::max<long long>(1, L.npairs) * L.RW32 * sizeof(float);
    cudaError_t e = cudaMalloc(&L.rows32, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        L.rows32 = nullptr;
        return set_err(c, DGV_ENOMEM, "FP32 rows: no room on the device");
    }
    if (L.npairs) {
        k_rows32_from64<<<148 * 8, 256, 0, c->stream>>>((const double *)L.rows64, L.RD64, (float *)L.rows32, L.RW32,
                                                      c->grid.P, L.npairs);
        DGV_CUDA(c, cudaGetLastError());
        count_launches(c, 1);
    }
    return DGV_OK;
}

int f_local_major(Ctx *c, const double *d_f, int nvdf, bool f32, const void **out)
{
    const Grid &g = c->grid;
    int rc = ensure_buffer(c, &c->d_fg, &c->fg_bytes, (size_t)nvdf * g.N * (f32 ? sizeof(float) : sizeof(double)));
    if (rc) return rc;
    const long long tot = (long long)nvdf * g.N;
    const unsigned nblk = (unsigned)std::min<long long>((tot + 255) / 256, 148LL * 16);
    if (f32)
        k_f_local_major<float><<<nblk, 256, 0, c->stream>>>(d_f, reinterpret_cast<float *>(c->d_fg), g.N, g.Nc, g.P,
                                                            nvdf);
    else
        k_f_local_major<double><<<nblk, 256, 0, c->stream>>>(d_f, c->d_fg, g.N, g.Nc, g.P, nvdf);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 1);
    *out = c->d_fg;
    return DGV_OK;
}

struct LaunchShape {
    int dcta, slices, threads, nst, sp, off_f, off_hdr, off_bar;
    size_t smem;
    bool gf;  // f gathered from a local-major copy in global memory
};

// Pipeline geometry: consumers = one warp per 32 output cells (<= 384), plus
// the producer warp; the stage ring takes what shared memory the copy of f
// leaves, up to 64 KiB, in 6 stages.  f goes to global memory (GF) when its
// shared copy and a ring of at least 4 rows per stage do not fit, or when
// DGV_OPT_FGLOBAL asks for it.
static int shape_for(Ctx *c, int mode, LaunchShape &s, int ncell)
{
    const Grid &g = c->grid;
    const Layout &L = c->lay;
    int maxsm = 0;
    DGV_CUDA(c, cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    // at most 11 consumer warps + the producer: 12 warps = 3 per SM
    // sub-partition, which leaves 170 registers per thread (no spills)
    s.slices = (ncell + 351) / 352;
    s.dcta = ((ncell + s.slices - 1) / s.slices + 31) / 32 * 32;
    s.threads = 32 + s.dcta;
    const int rowb = mode == MODE_F32C ? L.RW32 * 4 : L.RD64 * 8;
    size_t fbytes = (size_t)g.N * (mode == MODE_F32C ? sizeof(float) : sizeof(double));
    const int nst = 6;
    const size_t tail = 16 + (size_t)nst * sizeof(StageHdr) + 2 * nst * sizeof(uint64_t) + 16;
    s.gf = c->f_global == 1 || fbytes + tail + (size_t)nst * 4 * rowb > (size_t)maxsm;
    if (s.gf) fbytes = 0;
    if (fbytes + tail + (size_t)nst * 4 * rowb > (size_t)maxsm)
        return set_err(c, DGV_EUNSUP, "collide: the row ring does not fit in shared memory");
    if (g.N > INT32_MAX / 2)  // local-major indices of the gathers are ints
        return set_err(c, DGV_EUNSUP, "collide: grid too large");
    size_t ring = std::min<size_t>(64 * 1024, (size_t)maxsm - fbytes - tail);
    s.nst = nst;
    s.sp = (int)std::min<size_t>(256, ring / ((size_t)nst * rowb));
    s.off_f = s.nst * s.sp * rowb;
    s.off_hdr = (int)((s.off_f + fbytes + 15) / 16 * 16);
    s.off_bar = s.off_hdr + s.nst * (int)sizeof(StageHdr);
    s.smem = (size_t)s.off_bar + 2 * s.nst * sizeof(uint64_t);
    return DGV_OK;
}

static int run_collide(Ctx *c, const double *d_f, const double *d_f2, double *d_q, int nvdf, int precision,
                       double scale, int nchunks, int cell0, int cell1)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    const int mode = d_f2 ? MODE_BILINEAR : (precision == DGV_PREC_F64 ? MODE_F64 : MODE_F32C);
    LaunchShape sh;
    int rc = shape_for(c, mode, sh, cell1 - cell0);
    if (rc) return rc;
    if (mode == MODE_F32C && (rc = ensure_rows32(c))) return rc;  // rebuilt if released
    KernelFn fn = pick_kernel(g.P, mode, sh.gf);
    if (!fn) return set_err(c, DGV_EUNSUP, "collide: this build supports 1, 8, 27 or 125 nodes per cell");
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sh.smem));
    nchunks = std::max(1, std::min<int>(nchunks, (int)std::max<long long>(1, L.nblocks)));
    if (nchunks > 65535) return set_err(c, DGV_EINVAL, "collide: at most 65535 chunks");
    int *d_bounds = nullptr;
    rc = get_chunks(c, nchunks, &d_bounds);
    if (rc) return rc;
    size_t need = (size_t)nvdf * nchunks * g.P * g.Nc * sizeof(double);
    rc = ensure_buffer(c, &c->d_partial, &c->partial_bytes, need);
    if (rc) return rc;
    rc = ensure_errflag(c);
    if (rc) return rc;
    CollideArgs a;
    a.f = d_f; a.f2 = d_f2; a.partial = c->d_partial; a.blk = L.blk; a.err = c->d_err;
    a.rows = (const char *)(mode == MODE_F32C ? L.rows32 : L.rows64);
    a.rowb = mode == MODE_F32C ? L.RW32 * 4 : L.RD64 * 8;
    a.bounds = d_bounds; a.N = g.N; a.Nc = g.Nc; a.Mv = g.d.Mv; a.Mw = g.d.Mw;
    a.nchunks = nchunks; a.dcta = sh.dcta; a.nst = sh.nst; a.sp = sh.sp;
    a.cell0 = cell0; a.cell1 = cell1;
    a.off_f = sh.off_f; a.off_hdr = sh.off_hdr; a.off_bar = sh.off_bar;
    a.Pt = g.P; a.npsl = p_slices(g.P);
    a.wait_ns = wait_limit_ns(c);
    a.fg = nullptr;
    if (sh.gf && (rc = f_local_major(c, d_f, nvdf, mode == MODE_F32C, &a.fg))) return rc;
    // VDF fastest: the CTAs resident at one time work on the same chunk of
    // rows for different VDFs, so each row is fetched from HBM once and then
    // served from L2
    KTimer kt(c);
    fn<<<dim3(nvdf, sh.slices * a.npsl, nchunks), sh.threads, sh.smem, c->stream>>>(a);
    kt.stop(1);
    DGV_CUDA(c, cudaGetLastError());
    const long long tot_out = (long long)nvdf * (cell1 - cell0) * g.P;
    k_reduce_chunks<<<(unsigned)((tot_out + 255) / 256), 256, 0, c->stream>>>(c->d_partial, c->d_nwt, d_q, nchunks,
                                                                                 g.P, g.Nc, cell0, cell1, nvdf, scale);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 2);
    return DGV_OK;
}

// Chunk count.  Batches that fill at least a quarter of the SMs: the smallest
// count giving at least 8 waves of CTAs (work per chunk varies; more, smaller
// CTAs balance it) whose last wave is at least 90% full (one CTA per SM: the
// shared copy of f takes most of it).  Smaller batches: measured -- each
// candidate is timed once and the fastest kept.
static int choose_chunks(Ctx *c, const double *d_f, const double *d_f2, double *d_q, int nvdf, int precision,
                         int cell0, int cell1)
{
    if (c->nchunks_opt > 0) return c->nchunks_opt;
    const Grid &g = c->grid;
    LaunchShape sh;
    int rc0 = shape_for(c, d_f2 ? MODE_BILINEAR : (precision == DGV_PREC_F64 ? MODE_F64 : MODE_F32C), sh,
                        cell1 - cell0);
    if (rc0) return 1;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device);
    long long units = (long long)nvdf * sh.slices * p_slices(c->grid.P);
    if (units * 4 >= nsm) {
        for (int k = 1; k <= 64; k++) {
            long long ctas = units * k;
            long long waves = (ctas + nsm - 1) / nsm;
            if (waves >= 8 && (double)ctas / (double)(waves * nsm) >= 0.9) return k;
        }
        return 64;
    }
    long long key = ((long long)precision << 56) ^ ((long long)(d_f2 != nullptr) << 55) ^
                    ((long long)cell0 << 38) ^ ((long long)cell1 << 21) ^ nvdf;
    auto it = c->tuned.find(key);
    if (it != c->tuned.end()) return it->second;
    int base = (int)std::max<long long>(1, (long long)nsm / units);
    int cand[4] = {2 * base, 4 * base, 8 * base, 16 * base};
    float best_ms = 1e30f;
    int best = cand[1];
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int t = 0; t < 4; t++) {
        if (run_collide(c, d_f, d_f2, d_q, nvdf, precision, 1.0, cand[t], cell0, cell1)) break;  // warm-up
        cudaEventRecord(e0, c->stream);
        run_collide(c, d_f, d_f2, d_q, nvdf, precision, 1.0, cand[t], cell0, cell1);
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
    if (precision == DGV_PREC_TC) return collide_tc_device(c, d_f, d_q, nvdf, scale);
    if (precision != DGV_PREC_F64 && precision != DGV_PREC_F32C)
        return set_err(c, DGV_EINVAL, "collide: unknown precision");
    int nch = choose_chunks(c, d_f, nullptr, d_q, nvdf, precision, 0, c->grid.Nc);
    int rc = run_collide(c, d_f, nullptr, d_q, nvdf, precision, scale, nch, 0, c->grid.Nc);
    if (rc) return rc;
    if (c->project) return project_device(c, d_q, nvdf);
    return DGV_OK;
}

int collide_cells_device(Ctx *c, const double *d_f, double *d_q, int nvdf, int precision, int cell0, int cell1)
{
    if (!c->lay.blk) return set_err(c, DGV_ESTATE, "collide: no A-arrays loaded");
    if (precision != DGV_PREC_F64 && precision != DGV_PREC_F32C)
        return set_err(c, DGV_EUNSUP, "collide_cells: FP64 or FP32-compensated only");
    if (cell0 < 0 || cell1 > c->grid.Nc || cell0 >= cell1)
        return set_err(c, DGV_ERANGE, "collide_cells: cell range outside [0, Nc) or empty");
    int nch = choose_chunks(c, d_f, nullptr, d_q, nvdf, precision, cell0, cell1);
    return run_collide(c, d_f, nullptr, d_q, nvdf, precision, 1.0, nch, cell0, cell1);
}

int jvp_device(Ctx *c, const double *d_f, const double *d_df, double *d_q, int precision)
{
    if (!c->lay.blk) return set_err(c, DGV_ESTATE, "jvp: no A-arrays loaded");
    if (precision != DGV_PREC_F64) return set_err(c, DGV_EUNSUP, "jvp: the mixed-terms kernel computes in FP64 only");
    int nch = choose_chunks(c, d_f, d_df, d_q, 1, DGV_PREC_F64, 0, c->grid.Nc);
    // the bilinear kernel sums 2/w * A * (f g + g f) / 2 * 2: the reduce
    // kernel's factor 2 is the reference's "2*fc/w" (collision_mod.f90:326)
    return run_collide(c, d_f, d_df, d_q, 1, DGV_PREC_F64, 1.0, nch, 0, c->grid.Nc);
}

}  // namespace dgv
