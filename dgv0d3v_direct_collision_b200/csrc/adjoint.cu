// adjoint.cu -- vector-Jacobian product of the collision operator.
//
// Q_i = 2/w_i sum_j A_j f(a_j) f(b_j)  (a_j, b_j: shifted xi, xi1 of record j)
// g_k = sum_i v_i dQ_i/df_k = sum_i c_i sum_j A_j (delta_{k,a_j} f(b_j) + delta_{k,b_j} f(a_j)),
// c_i = 2 v_i / w_i.  The adjoint of collision_mod.f90:213-216; at a
// Maxwellian fm it equals 2*fmA*v (collision_mod.f90:448-449, 357).
//
// Same traversal as the forward kernel: a thread owns an output cell D and
// keeps its P cotangent weights c_(D,p) in registers; for every pair it forms
// vA = sum_p A_p c_p (P multiply-adds, the forward's cost) and scatters
// vA*f(b) to g(a) and vA*f(a) to g(b) with FP64 atomic adds (so the summation
// order, and the last bits of g, vary from run to run).  The scatter goes to a
// local-major copy g_lm[l*Nc + cell] -- the layout of the shared copy of f,
// so its indices are the gather offsets o1+D, o2+D -- where the 32 lanes of
// a warp (32 consecutive cells) hit 256 contiguous bytes instead of 32 lines
// P doubles apart; k_lm_to_nodes writes g in node order afterwards.  On grids
// whose f does not fit in shared memory (or with DGV_OPT_FGLOBAL) the gathers
// read a local-major copy of f in global memory instead (GF).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "dgv_internal.h"
#include "pipeline.cuh"

namespace dgv {

struct VjpArgs {
    const double *f, *v, *w;
    double *g;
    const BlockInfo *blk;
    const char *rows;
    const int *bounds;
    int *err;
    long long N;
    int Nc, Mv, Mw, dcta, rowb, nst, sp, off_f, off_hdr, off_bar;
    int Pt, npsl;  // nodes per cell; slices of PV basis functions (1 unless sliced)
    const double *fg;  // GF: local-major copy of f
    unsigned long long wait_ns;  // limit of every bounded wait
};

// Same shared-memory row pipeline as the forward kernel (pipeline.cuh).
// SL (sliced, for many nodes per cell): a CTA forms vA over the PV basis
// functions of its slice only (blockIdx.y % npsl) and scatters that part;
// the scatters of the slices add up to the full adjoint.
template <int PV, bool SL = false, bool GF = false>
__global__ void __launch_bounds__(384, 1) k_vjp_pipe(VjpArgs a)
{
    extern __shared__ __align__(128) unsigned char smem[];
    const size_t stage_bytes = (size_t)a.sp * a.rowb;
    unsigned char *stages = smem;
    double *f_s = reinterpret_cast<double *>(smem + a.off_f);
    StageHdr *hdr = reinterpret_cast<StageHdr *>(smem + a.off_hdr);
    uint64_t *full = reinterpret_cast<uint64_t *>(smem + a.off_bar);
    uint64_t *empty = full + a.nst;
    const int slice = SL ? blockIdx.y / a.npsl : blockIdx.y, chunk = blockIdx.z;
    const int PT = SL ? a.Pt : PV;                         // nodes per cell
    const int pofs = SL ? (blockIdx.y % a.npsl) * PV : 0;  // first basis function of the slice
    if (threadIdx.x == 0) {
        for (int s = 0; s < a.nst; s++) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], a.dcta / 32);
        }
        fence_mbar_init();
    }
    auto fat = [&](int q) -> double {
        if constexpr (GF) return __ldg(a.fg + q);
        else return f_s[q];
    };
    if constexpr (!GF) {
        for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
            int cell = (int)(i / PT), l = (int)(i - (long long)cell * PT);
            f_s[l * a.Nc + cell] = __ldg(a.f + i);
        }
    }
    __syncthreads();
    const int b0 = a.bounds[chunk], b1 = a.bounds[chunk + 1];
    const int d0 = slice * a.dcta, d1 = min(a.Nc, d0 + a.dcta);
    if (threadIdx.x < 32) {  // producer: warp 0
        produce_rows(a.blk, b0, b1, a.Mv, a.Mw, d0, d1, a.rows, a.rowb, stages, a.sp, a.nst, hdr, full, empty, a.err,
                     a.wait_ns);
        return;
    }
    const int tc = threadIdx.x - 32, lane = threadIdx.x & 31;
    const int D = d0 + tc;
    const bool inD = tc < a.dcta && D < a.Nc;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    double cw[PV];
#pragma unroll
    for (int j = 0; j < PV; j++) {
        long long i = (long long)D * PT + pofs + j;
        cw[j] = (inD && pofs + j < PT) ? 2.0 * a.v[i] / a.w[i] : 0.0;
    }
    constexpr int RD = ((1 + PV) + 1) / 2 * 2;
    int cur = -1;
    bool valid = false;
    for (int it = 0;; it++) {
        const int s = it % a.nst;
        if (!mbar_wait(&full[s], (it / a.nst) & 1, a.err, a.wait_ns)) break;
        const StageHdr h = hdr[s];
        if (h.block < 0) break;
        if (h.block != cur) {
            cur = h.block;
            const BlockInfo bi = a.blk[cur];
            valid = inD && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] && Dw >= bi.lo[2] &&
                    Dw <= bi.hi[2];
        }
        if (__any_sync(0xffffffffu, valid) && valid) {
            const unsigned char *st = stages + s * stage_bytes;
#pragma unroll 2
            for (int k = 0; k < h.n; k++) {
                double vA = 0.0;
                long long o;
                if constexpr (SL) {
                    const double *rowd = reinterpret_cast<const double *>(st + (size_t)k * a.rowb);
                    o = __double_as_longlong(rowd[0]);
#pragma unroll
                    for (int j = 0; j < PV; j++) vA = fma(rowd[1 + pofs + j], cw[j], vA);
                } else {
                    const double2 *row = reinterpret_cast<const double2 *>(st + (size_t)k * a.rowb);
                    double rv[RD];
#pragma unroll
                    for (int t = 0; t < RD / 2; t++) {
                        double2 x = row[t];
                        rv[2 * t] = x.x;
                        rv[2 * t + 1] = x.y;
                    }
                    o = __double_as_longlong(rv[0]);
#pragma unroll
                    for (int j = 0; j < PV; j++) vA = fma(rv[1 + j], cw[j], vA);
                }
                const int q1 = (int)(unsigned)(o & 0xffffffffLL) + D, q2 = (int)(o >> 32) + D;
                atomicAdd(a.g + q1, vA * fat(q2));
                atomicAdd(a.g + q2, vA * fat(q1));
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(&empty[s]);
    }
}

// g[cell*P + l] = g_lm[l*Nc + cell]
__global__ void k_lm_to_nodes(const double *g_lm, double *g, long long N, int Nc, int P)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= N) return;
    const int cell = (int)(i / P), l = (int)(i - (long long)cell * P);
    g[i] = g_lm[(size_t)l * Nc + cell];
}

typedef void (*VjpFn)(VjpArgs);

int vjp_device(Ctx *c, const double *d_f, const double *d_v, double *d_g, int precision)
{
    if (precision != DGV_PREC_F64) return set_err(c, DGV_EUNSUP, "vjp: this kernel computes in FP64 only");
    if (!c->lay.blk) return set_err(c, DGV_ESTATE, "vjp: no A-arrays loaded");
    const Grid &g = c->grid;
    const Layout &L = c->lay;
    if (g.N > INT32_MAX / 2) return set_err(c, DGV_EUNSUP, "vjp: grid too large");
    const int npsl = g.P > 27 ? (g.P + 24) / 25 : 1;
    int maxsm = 0, nsm = 148;
    DGV_CUDA(c, cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    DGV_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const int slices = (g.Nc + 351) / 352;
    const int dcta = ((g.Nc + slices - 1) / slices + 31) / 32 * 32;
    const int rowb = L.RD64 * 8, nst = 6;
    size_t fbytes = (size_t)g.N * sizeof(double);
    const size_t tail = 16 + nst * sizeof(StageHdr) + 2 * nst * sizeof(uint64_t) + 16;
    const bool gf = c->f_global == 1 || fbytes + tail + (size_t)nst * 4 * rowb > (size_t)maxsm;
    if (gf) fbytes = 0;
    if (fbytes + tail + (size_t)nst * 4 * rowb > (size_t)maxsm)
        return set_err(c, DGV_EUNSUP, "vjp: the row ring does not fit in shared memory");
    VjpFn fn = nullptr;
#define DGV_VJP_PICK(...) fn = gf ? k_vjp_pipe<__VA_ARGS__, true> : k_vjp_pipe<__VA_ARGS__, false>
    switch (g.P) {
    case 1: DGV_VJP_PICK(1, false); break;
    case 8: DGV_VJP_PICK(8, false); break;
    case 27: DGV_VJP_PICK(27, false); break;
    case 125: DGV_VJP_PICK(25, true); break;  // slices of 25 basis functions per CTA
    default: return set_err(c, DGV_EUNSUP, "vjp: this build supports 1, 8, 27 or 125 nodes per cell");
    }
#undef DGV_VJP_PICK
    const size_t ring = std::min<size_t>(64 * 1024, (size_t)maxsm - fbytes - tail);
    const int sp = (int)std::min<size_t>(256, ring / ((size_t)nst * rowb));
    VjpArgs a;
    a.off_f = nst * sp * rowb;
    a.off_hdr = (int)((a.off_f + fbytes + 15) / 16 * 16);
    a.off_bar = a.off_hdr + nst * (int)sizeof(StageHdr);
    const size_t smem = (size_t)a.off_bar + 2 * nst * sizeof(uint64_t);
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nchunks = std::max(1, std::min<int>(2 * nsm / slices, (int)std::max<long long>(1, L.nblocks)));
    int *d_bounds = nullptr;
    int rc = get_chunks(c, nchunks, &d_bounds);
    if (rc) return rc;
    rc = ensure_errflag(c);
    if (rc) return rc;
    rc = ensure_buffer(c, &c->d_glm, &c->glm_bytes, sizeof(double) * (size_t)g.N);
    if (rc) return rc;
    DGV_CUDA(c, cudaMemsetAsync(c->d_glm, 0, sizeof(double) * (size_t)g.N, c->stream));
    a.f = d_f; a.v = d_v; a.w = c->d_nwt; a.g = c->d_glm; a.blk = L.blk; a.rows = (const char *)L.rows64;
    a.bounds = d_bounds; a.err = c->d_err; a.N = g.N; a.Nc = g.Nc; a.Mv = g.d.Mv; a.Mw = g.d.Mw; a.dcta = dcta;
    a.rowb = rowb; a.nst = nst; a.sp = sp; a.Pt = g.P; a.npsl = npsl;
    a.wait_ns = wait_limit_ns(c);
    a.fg = nullptr;
    if (gf) {
        const void *fg = nullptr;
        if ((rc = f_local_major(c, d_f, 1, false, &fg))) return rc;
        a.fg = static_cast<const double *>(fg);
    }
    fn<<<dim3(1, slices * npsl, nchunks), 32 + dcta, smem, c->stream>>>(a);
    DGV_CUDA(c, cudaGetLastError());
    k_lm_to_nodes<<<(unsigned)((g.N + 255) / 256), 256, 0, c->stream>>>(c->d_glm, d_g, g.N, g.Nc, g.P);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 2);
    return DGV_OK;
}

}  // namespace dgv
