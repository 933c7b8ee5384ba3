// collide_tc.cu -- batched Q(f,f) on the 5th-generation tensor cores.
//
// Per cell-pair block (c1,c2) and output cell D the operator is a product of
// two small matrices:  Q[(D,b), p] += sum_k  P[(D,b), k] * V[k, p],
//   P[(D,b), k] = f_b(c1+D-ccell, l1_k) * f_b(c2+D-ccell, l2_k)   (k = pair)
//   V[k, p]     = A value of canonical basis function p for pair k.
// One tcgen05.mma tile has M = 128 rows = 4 consecutive output cells x 32
// VDFs, N = 32 basis functions (P <= 32, zero-padded), K = 16 pairs.
//
// Precision: P and V are split into fp16 hi + lo parts (x = hi + lo + O(2^-24 x))
// after exact power-of-two scaling (per VDF for f, one global factor for A).
// hi*hi is accumulated by the tensor core in FP32 over one 64-pair chunk
// (4 MMAs); hi*lo + lo*hi (2^-11 smaller) in a second accumulator over the
// whole block.  The epilogue adds chunk results in FP32 and each block total
// into a (sum, correction) pair with two-sum, so the long accumulation over
// all blocks is compensated; at the end of a launch the pair is added in FP64
// to the output accumulator in global memory.
//
// Warp roles (448 threads, one CTA per SM):
//   warp 0      producer: TMA bulk copies of the V chunk records into a ring
//   warp 1      allocates tensor memory; lane 0 issues the MMAs
//   warps 2-9   generators: P tiles (split fp16) into shared memory
//   warps 10-13 epilogue: per-block compensated flush, final FP64 add
// Every wait is bounded (%globaltimer); a timeout raises the error flag, each
// role still reaches the final barrier, in-flight copies and MMAs are
// drained, and tensor memory is freed before the CTA exits.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dgv_internal.h"
#include "pipeline.cuh"

namespace dgv {

constexpr int TC_KCH = 64;                        // pairs per chunk record
constexpr int TC_TILE_B = 32 * TC_KCH * 2;        // one 32 x 64 fp16 tile (4 KiB)
constexpr int TC_REC = 2 * TC_TILE_B + TC_KCH * 2;  // hi tile, lo tile, (l1,l2) bytes
constexpr int TC_ROWS = 128;
constexpr int TC_ATILE = TC_ROWS * TC_KCH * 2;    // 128 x 64 fp16 (16 KiB)
constexpr int TC_NSTB = 4;                        // V ring stages
constexpr int TC_THREADS = 448;
constexpr int TC_GEN_WARPS = 8;
constexpr int TC_EPI_WARPS = 4;

// ----------------------------------------------------------------------------
// tcgen05 helpers (sm_100a)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo)
{
    // K-major, no swizzle: core matrices of 8 rows x 16 bytes; lbo = stride of
    // core matrices along K, sbo = stride of 8-row groups; version 1
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | (1ULL << 46);
}

__device__ __forceinline__ void umma_f16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc)
        : "memory");
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void fence_async_shared() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const float *v)
{
    uint32_t r[16];
#pragma unroll
    for (int i = 0; i < 16; i++) r[i] = __float_as_uint(v[i]);
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], "
        "{%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(taddr),
        "r"(r[0]), "r"(r[1]), "r"(r[2]), "r"(r[3]), "r"(r[4]), "r"(r[5]), "r"(r[6]), "r"(r[7]), "r"(r[8]),
        "r"(r[9]), "r"(r[10]), "r"(r[11]), "r"(r[12]), "r"(r[13]), "r"(r[14]), "r"(r[15])
        : "memory");
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}

// bounded wait whose outcome is the same for every lane of the warp (the
// warp-collective tensor-memory instructions that follow need a converged warp)
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, int *err)
{
    const bool ok = mbar_wait(bar, parity, err);
    return __all_sync(0xffffffffu, ok);
}

// split x into fp16 hi + lo (two values at a time)
__device__ __forceinline__ void split2(float x0, float x1, uint32_t &hi, uint32_t &lo)
{
    __half2 h = __floats2half2_rn(x0, x1);
    float2 hf = __half22float2(h);
    __half2 l = __floats2half2_rn(x0 - hf.x, x1 - hf.y);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = *reinterpret_cast<uint32_t *>(&l);
}

struct TcArgs {
    const float *F;           // [nbt][Nc][P][32] scaled f, zero for padded VDFs
    const unsigned char *V;   // chunk records
    const int *chunk_start;   // [nblocks+1]
    const BlockInfo *blk;
    double *qacc;             // [(D*P+p)*NV + vdf]
    const double *inv_scale;  // [NV]
    int *err;
    int b0, b1;               // block range of this launch
    int Nc, P, Mv, Mw, ccell, NV, nvdf;
};

__device__ __forceinline__ bool dgroup_meets(const BlockInfo &bi, int D0, int Nc, int Mv, int Mw)
{
    for (int d = 0; d < 4; d++) {
        int D = D0 + d;
        if (D >= Nc) break;
        int Du = D / (Mv * Mw), Dv = (D / Mw) % Mv, Dw = D % Mw;
        if (Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] && Dw >= bi.lo[2] &&
            Dw <= bi.hi[2])
            return true;
    }
    return false;
}

// 512 in the launch bound caps registers at 128 per thread: with 14 warps,
// two of the four SM sub-partitions hold 4 warps each.
//
// Tensor memory (256 columns): hi*hi accumulators of chunks (double
// buffered, columns 0-31 / 32-63), hi*lo + lo*hi accumulators of blocks
// (64-95 / 96-127), compensated sum and correction (128-159 / 160-191).
// The hi*hi chain of a chunk is only 4 MMAs long and the small terms get
// their own chain, so few roundings of the tensor-core accumulator reach
// the result; chunk sums are added in FP32 (round to nearest) and block sums
// with two-sum.
__global__ void __launch_bounds__(512, 1) k_collide_tc(TcArgs a)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *abuf = smem;                                // 2 x (hi, lo) A tiles
    unsigned char *vring = smem + 4 * TC_ATILE;                // TC_NSTB x TC_REC
    uint64_t *bars = reinterpret_cast<uint64_t *>(vring + TC_NSTB * TC_REC);
    uint64_t *b_full = bars, *b_empty = bars + TC_NSTB;
    uint64_t *a_full = bars + 2 * TC_NSTB, *a_empty = a_full + 2;
    uint64_t *h_full = a_empty + 2, *h_empty = h_full + 2;     // chunk accumulators
    uint64_t *l_full = h_empty + 2, *l_empty = l_full + 2;     // block accumulators
    uint64_t *drain = l_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bt = blockIdx.x, D0 = blockIdx.y * 4;
    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_NSTB; s++) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            mbar_init(&a_full[s], TC_GEN_WARPS);
            mbar_init(&a_empty[s], 1);
            mbar_init(&h_full[s], 1);
            mbar_init(&h_empty[s], TC_EPI_WARPS);
            mbar_init(&l_full[s], 1);
            mbar_init(&l_empty[s], TC_EPI_WARPS);
        }
        mbar_init(drain, 1);
        fence_mbar_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 256;" ::"r"(smem_u32(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // instruction descriptor: FP32 accumulator, fp16 A and B, both K-major,
    // N = 32, M = 128
    const uint32_t idesc = (1u << 4) | ((uint32_t)(32 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);

    if (warp == 0) {
        // ---------------- producer ----------------
        if (lane == 0) {
            int g = 0;
            bool ok = true;
            for (int b = a.b0; b < a.b1 && ok; b++) {
                const BlockInfo bi = a.blk[b];
                if (!dgroup_meets(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
                const int c0 = a.chunk_start[b], c1 = a.chunk_start[b + 1];
                for (int c = c0; c < c1; c++, g++) {
                    const int s = g % TC_NSTB;
                    if (!mbar_wait(&b_empty[s], ((g / TC_NSTB) & 1) ^ 1, a.err)) { ok = false; break; }
                    mbar_arrive_expect_tx(&b_full[s], TC_REC);
                    bulk_g2s(vring + s * TC_REC, a.V + (size_t)c * TC_REC, TC_REC, &b_full[s]);
                }
            }
            if (!ok)  // let the copies already issued land
                for (int j = g > TC_NSTB ? g - TC_NSTB : 0; j < g; j++)
                    mbar_wait(&b_full[j % TC_NSTB], (j / TC_NSTB) & 1, a.err);
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int g = 0, q = 0;
            bool ok = true;
            for (int b = a.b0; b < a.b1 && ok; b++) {
                const BlockInfo bi = a.blk[b];
                if (!dgroup_meets(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
                const int c0 = a.chunk_start[b], c1 = a.chunk_start[b + 1];
                const int lb = q & 1;
                if (!mbar_wait(&l_empty[lb], ((q >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                const uint32_t dlo = tmem + (uint32_t)(64 + lb * 32);
                for (int c = c0; c < c1; c++, g++) {
                    const int s = g % TC_NSTB, x = g & 1;
                    if (!mbar_wait(&b_full[s], (g / TC_NSTB) & 1, a.err)) { ok = false; break; }
                    if (!mbar_wait(&a_full[x], (g >> 1) & 1, a.err)) { ok = false; break; }
                    if (!mbar_wait(&h_empty[x], ((g >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t dhi = tmem + (uint32_t)(x * 32);
                    const uint32_t vb = smem_u32(vring + s * TC_REC);
                    const uint32_t ah = smem_u32(abuf + (2 * x) * TC_ATILE), al = smem_u32(abuf + (2 * x + 1) * TC_ATILE);
#pragma unroll
                    for (int t = 0; t < TC_KCH / 16; t++) {
                        const uint32_t ko = t * 256;  // two core matrices (K = 16) per step
                        const uint64_t dAh = umma_desc(ah + ko, 128, 1024), dAl = umma_desc(al + ko, 128, 1024);
                        const uint64_t dBh = umma_desc(vb + ko, 128, 1024), dBl = umma_desc(vb + TC_TILE_B + ko, 128, 1024);
                        umma_f16(dhi, dAh, dBh, idesc, t == 0 ? 0u : 1u);
                        umma_f16(dlo, dAh, dBl, idesc, (c == c0 && t == 0) ? 0u : 1u);
                        umma_f16(dlo, dAl, dBh, idesc, 1u);
                    }
                    umma_commit(&a_empty[x]);
                    umma_commit(&b_empty[s]);
                    umma_commit(&h_full[x]);
                }
                if (!ok) break;
                umma_commit(&l_full[lb]);
                q++;
            }
            // every MMA issued so far completes before tensor memory is freed
            umma_commit(drain);
            mbar_wait(drain, 0, a.err);
        }
        __syncwarp();
    } else if (warp < 2 + TC_GEN_WARPS) {
        // ---------------- generators ----------------
        const int gi = warp - 2, d = gi & 3, kh = gi >> 2;  // output cell slot, half of the chunk
        const int D = D0 + d, row = d * 32 + lane;
        const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
        const float *Fb = a.F + (size_t)bt * a.Nc * a.P * 32 + lane;
        int g = 0;
        bool ok = true;
        for (int b = a.b0; b < a.b1 && ok; b++) {
            const BlockInfo bi = a.blk[b];
            if (!dgroup_meets(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
            const bool valid = D < a.Nc && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] &&
                               Dw >= bi.lo[2] && Dw <= bi.hi[2];
            const float *F1 = Fb + (size_t)(bi.c1 + D - a.ccell) * a.P * 32;
            const float *F2 = Fb + (size_t)(bi.c2 + D - a.ccell) * a.P * 32;
            const int c0 = a.chunk_start[b], c1 = a.chunk_start[b + 1];
            for (int c = c0; c < c1; c++, g++) {
                const int s = g % TC_NSTB, x = g & 1;
                if (!mbar_wait_warp(&b_full[s], (g / TC_NSTB) & 1, a.err)) { ok = false; break; }
                if (!mbar_wait_warp(&a_empty[x], ((g >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                const unsigned char *idx = vring + s * TC_REC + 2 * TC_TILE_B;
                unsigned char *ah = abuf + (2 * x) * TC_ATILE, *al = abuf + (2 * x + 1) * TC_ATILE;
#pragma unroll
                for (int kgl = 0; kgl < 4; kgl++) {
                    const int kg = kh * 4 + kgl;
                    uint32_t hi[4], lo[4];
                    if (valid) {
                        float x8[8];
#pragma unroll
                        for (int j = 0; j < 8; j++) {
                            const int k = kg * 8 + j;
                            const int l1 = idx[2 * k], l2 = idx[2 * k + 1];
                            x8[j] = __ldg(F1 + l1 * 32) * __ldg(F2 + l2 * 32);
                        }
#pragma unroll
                        for (int j = 0; j < 4; j++) split2(x8[2 * j], x8[2 * j + 1], hi[j], lo[j]);
                    } else {
#pragma unroll
                        for (int j = 0; j < 4; j++) { hi[j] = 0u; lo[j] = 0u; }
                    }
                    // core matrix (row/8, kg): 8 rows x 16 bytes
                    const int off = ((row >> 3) * 8 + kg) * 128 + (row & 7) * 16;
                    *reinterpret_cast<uint4 *>(ah + off) = make_uint4(hi[0], hi[1], hi[2], hi[3]);
                    *reinterpret_cast<uint4 *>(al + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
                }
                fence_async_shared();  // generic-proxy writes -> visible to the tensor core
                __syncwarp();
                if (lane == 0) mbar_arrive(&a_full[x]);
            }
        }
    } else if (warp < 2 + TC_GEN_WARPS + TC_EPI_WARPS) {
        // ---------------- epilogue ----------------
        const int quarter = warp & 3, r = quarter * 32 + lane;  // tensor memory lane = tile row
        const uint32_t tl = tmem + ((uint32_t)(quarter * 32) << 16);
        float run[32];  // FP32 sum of the chunks of the current block
#pragma unroll
        for (int i = 0; i < 32; i++) run[i] = 0.f;
#pragma unroll
        for (int h = 0; h < 4; h++) tmem_st16(tl + 128 + 16 * h, run);
        int g = 0, q = 0;
        bool ok = true;
        for (int b = a.b0; b < a.b1 && ok; b++) {
            const BlockInfo bi = a.blk[b];
            if (!dgroup_meets(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
            const int c0 = a.chunk_start[b], c1 = a.chunk_start[b + 1];
            for (int c = c0; c < c1; c++, g++) {
                const int x = g & 1;
                if (!mbar_wait_warp(&h_full[x], (g >> 1) & 1, a.err)) { ok = false; break; }
                tc_fence_after();
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float v[16];
                    tmem_ld16(tl + x * 32 + 16 * h, v);
#pragma unroll
                    for (int i = 0; i < 16; i++) run[16 * h + i] += v[i];
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&h_empty[x]);
            }
            if (!ok) break;
            const int lb = q & 1;
            if (!mbar_wait_warp(&l_full[lb], (q >> 1) & 1, a.err)) { ok = false; break; }
            tc_fence_after();
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float v[16], sm[16], cm[16];
                tmem_ld16(tl + 64 + lb * 32 + 16 * h, v);
                tmem_ld16(tl + 128 + 16 * h, sm);
                tmem_ld16(tl + 160 + 16 * h, cm);
#pragma unroll
                for (int i = 0; i < 16; i++) {  // two-sum of sum + block total
                    const float xb = run[16 * h + i] + v[i];
                    const float t = sm[i] + xb, bp = t - sm[i];
                    cm[i] += (sm[i] - (t - bp)) + (xb - bp);
                    sm[i] = t;
                    run[16 * h + i] = 0.f;
                }
                tmem_st16(tl + 128 + 16 * h, sm);
                tmem_st16(tl + 160 + 16 * h, cm);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&l_empty[lb]);
            q++;
        }
        if (ok) {
            const int d = r >> 5, vdf = bt * 32 + (r & 31);
            const int D = D0 + d;
            const bool mine = D < a.Nc && vdf < a.nvdf;
            const double sc = mine ? a.inv_scale[vdf] : 0.0;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float sm[16], cm[16];
                tmem_ld16(tl + 128 + 16 * h, sm);
                tmem_ld16(tl + 160 + 16 * h, cm);
                if (mine)
                    for (int i = 0; i < 16; i++) {
                        const int p = 16 * h + i;
                        if (p < a.P) {
                            double *dst = a.qacc + ((size_t)D * a.P + p) * a.NV + vdf;
                            *dst += ((double)sm[i] + (double)cm[i]) * sc;
                        }
                    }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 256;" ::"r"(tmem) : "memory");
}

// ----------------------------------------------------------------------------
// chunk records: per block, ceil(count/64) records of {V hi tile, V lo tile,
// (l1,l2) bytes}; tiles K-major without swizzle: element (p, k) at byte
// ((p/8)*8 + k/8)*128 + (p%8)*16 + (k%8)*2
__global__ void k_tc_build(const BlockInfo *blk, const double *rows64, int RD64, const int *chunk_start, int P,
                           int Nc, int ccell, float vscale, unsigned char *V)
{
    const BlockInfo bi = blk[blockIdx.x];
    const int c0 = chunk_start[blockIdx.x], c1 = chunk_start[blockIdx.x + 1];
    for (int t = threadIdx.x; t < (c1 - c0) * TC_KCH; t += blockDim.x) {
        const int c = t / TC_KCH, k = t % TC_KCH, pr = c * TC_KCH + k;
        unsigned char *rec = V + (size_t)(c0 + c) * TC_REC;
        int l1 = 0, l2 = 0;
        const bool real = pr < bi.count;
        const double *row = rows64 + (size_t)(bi.start + (real ? pr : 0)) * RD64;
        if (real) {
            long long o = __double_as_longlong(row[0]);
            int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
            l1 = (o1 - (bi.c1 - ccell)) / Nc;
            l2 = (o2 - (bi.c2 - ccell)) / Nc;
        }
        rec[2 * TC_TILE_B + 2 * k] = (unsigned char)l1;
        rec[2 * TC_TILE_B + 2 * k + 1] = (unsigned char)l2;
        for (int p = 0; p < 32; p++) {
            float x = (real && p < P) ? (float)(row[1 + p] * (double)vscale) : 0.f;
            __half h = __float2half_rn(x);
            __half l = __float2half_rn(x - __half2float(h));
            const int off = ((p >> 3) * 8 + (k >> 3)) * 128 + (p & 7) * 16 + (k & 7) * 2;
            *reinterpret_cast<__half *>(rec + off) = h;
            *reinterpret_cast<__half *>(rec + TC_TILE_B + off) = l;
        }
    }
}

__global__ void k_absmax_rows(const double *rows64, long long npairs, int RD64, int P, unsigned long long *out)
{
    double m = 0.0;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npairs * P;
         i += (long long)gridDim.x * blockDim.x) {
        long long pr = i / P;
        int p = (int)(i - pr * P);
        m = fmax(m, fabs(rows64[pr * RD64 + 1 + p]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// per-VDF scale 2^e (max |f| -> 2^6) and the scaled, b-minor copy of f
__global__ void k_tc_fprep(const double *f, long long N, int nvdf, double vinv, float *F, double *inv_scale,
                           int Nc, int P, int NV)
{
    const int v = blockIdx.x;
    __shared__ double red[32];
    double m = 0.0;
    if (v < nvdf)
        for (long long i = threadIdx.x; i < N; i += blockDim.x) m = fmax(m, fabs(f[(size_t)v * N + i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x < 32) {
        m = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.0;
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0) red[0] = m;
    }
    __syncthreads();
    m = red[0];
    int e = 0;
    if (m > 0.0) {
        frexp(m, &e);  // m = f * 2^e, f in [0.5, 1)
        e = 6 - e;
    }
    const double s = ldexp(1.0, e);
    if (threadIdx.x == 0) inv_scale[v] = ldexp(1.0, -2 * e) * vinv;
    const int bt = v / 32, lb = v % 32;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) {
        const int cell = (int)(i / P), l = (int)(i - (long long)cell * P);
        const double x = v < nvdf ? f[(size_t)v * N + i] * s : 0.0;
        F[(((size_t)bt * Nc + cell) * P + l) * 32 + lb] = (float)x;
    }
}

// q[v][D*P+p] = scale * 2 * qacc[(D*P+p)*NV + v] / w[D*P+p]
__global__ void k_tc_final(const double *qacc, const double *w, double *q, long long N, int nvdf, int NV, double scale)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nvdf * N) return;
    const int v = (int)(idx % nvdf);
    const long long i = idx / nvdf;
    double val = 2.0 * qacc[i * NV + v] / w[i];
    if (scale != 1.0) val = val * scale;
    q[(size_t)v * N + i] = val;
}

// ----------------------------------------------------------------------------
static int tc_prepare(Ctx *c)
{
    Layout &L = c->lay;
    if (L.tc_V) return DGV_OK;
    const Grid &g = c->grid;
    std::vector<int> cs(L.nblocks + 1, 0);
    for (long long b = 0; b < L.nblocks; b++) cs[b + 1] = cs[b] + (L.h_blk[b].count + TC_KCH - 1) / TC_KCH;
    const long long nch = cs[L.nblocks];
    unsigned long long *d_max = nullptr;
    DGV_CUDA(c, cudaMalloc(&d_max, sizeof(unsigned long long)));
    DGV_CUDA(c, cudaMemsetAsync(d_max, 0, sizeof(unsigned long long), c->stream));
    k_absmax_rows<<<1184, 256, 0, c->stream>>>((const double *)L.rows64, L.npairs, L.RD64, g.P, d_max);
    DGV_CUDA(c, cudaGetLastError());
    unsigned long long hm = 0;
    DGV_CUDA(c, cudaMemcpyAsync(&hm, d_max, sizeof(hm), cudaMemcpyDeviceToHost, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d_max);
    double vmax;
    std::memcpy(&vmax, &hm, sizeof(vmax));
    int e = 0;
    if (vmax > 0.0) {
        std::frexp(vmax, &e);
        e = 14 - e;
    }
    L.tc_vscale = std::ldexp(1.0, e);
    DGV_CUDA(c, cudaMalloc(&L.tc_chunk_start, sizeof(int) * (L.nblocks + 1)));
    DGV_CUDA(c, cudaMemcpy(L.tc_chunk_start, cs.data(), sizeof(int) * (L.nblocks + 1), cudaMemcpyHostToDevice));
    DGV_CUDA(c, cudaMalloc(&L.tc_V, (size_t)std::max<long long>(1, nch) * TC_REC));
    if (L.nblocks)
        k_tc_build<<<(unsigned)L.nblocks, 256, 0, c->stream>>>(L.blk, (const double *)L.rows64, L.RD64,
                                                                L.tc_chunk_start, g.P, g.Nc, g.ccell,
                                                                (float)L.tc_vscale, (unsigned char *)L.tc_V);
    DGV_CUDA(c, cudaGetLastError());
    L.tc_chunk_host = cs;
    // block sets of about 48 MB of chunk records each (their values stay in L2)
    L.tc_sets.clear();
    L.tc_sets.push_back(0);
    const long long per_set = (48LL << 20) / TC_REC;
    long long acc = 0;
    for (long long b = 0; b < L.nblocks; b++) {
        acc += cs[b + 1] - cs[b];
        if (acc >= per_set) { L.tc_sets.push_back((int)(b + 1)); acc = 0; }
    }
    if (L.tc_sets.back() != (int)L.nblocks) L.tc_sets.push_back((int)L.nblocks);
    return DGV_OK;
}

int collide_tc_device(Ctx *c, const double *d_f, double *d_q, int nvdf, double scale)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    if (!L.blk) return set_err(c, DGV_ESTATE, "collide: no A-arrays loaded");
    if (g.P > 32) return set_err(c, DGV_EUNSUP, "tensor-core path: at most 32 nodes per cell");
    int rc = tc_prepare(c);
    if (rc) return rc;
    rc = ensure_errflag(c);
    if (rc) return rc;
    const int nbt = (nvdf + 31) / 32, NV = nbt * 32;
    const size_t fbytes = (size_t)nbt * g.Nc * g.P * 32 * sizeof(float);
    const size_t qbytes = (size_t)g.N * NV * sizeof(double);
    rc = ensure_buffer(c, &c->d_tcF, &c->tcF_bytes, fbytes + NV * sizeof(double));
    if (rc) return rc;
    rc = ensure_buffer(c, &c->d_tcQ, &c->tcQ_bytes, qbytes);
    if (rc) return rc;
    float *F = reinterpret_cast<float *>(c->d_tcF);
    double *inv = reinterpret_cast<double *>(reinterpret_cast<char *>(c->d_tcF) + fbytes);
    k_tc_fprep<<<NV, 256, 0, c->stream>>>(d_f, g.N, nvdf, 1.0 / L.tc_vscale, F, inv, g.Nc, g.P, NV);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaMemsetAsync(c->d_tcQ, 0, qbytes, c->stream));
    const size_t smem = 4 * (size_t)TC_ATILE + (size_t)TC_NSTB * TC_REC + (2 * TC_NSTB + 16) * sizeof(uint64_t) + 16;
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)k_collide_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    TcArgs a;
    a.F = F; a.V = (const unsigned char *)L.tc_V; a.chunk_start = L.tc_chunk_start; a.blk = L.blk;
    a.qacc = c->d_tcQ; a.inv_scale = inv; a.err = c->d_err;
    a.Nc = g.Nc; a.P = g.P; a.Mv = g.d.Mv; a.Mw = g.d.Mw; a.ccell = g.ccell; a.NV = NV; a.nvdf = nvdf;
    const dim3 grid(nbt, (g.Nc + 3) / 4);
    for (size_t s = 0; s + 1 < L.tc_sets.size(); s++) {
        a.b0 = L.tc_sets[s];
        a.b1 = L.tc_sets[s + 1];
        k_collide_tc<<<grid, TC_THREADS, smem, c->stream>>>(a);
        DGV_CUDA(c, cudaGetLastError());
    }
    long long tot = (long long)nvdf * g.N;
    k_tc_final<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->d_tcQ, c->d_nwt, d_q, g.N, nvdf, NV, scale);
    DGV_CUDA(c, cudaGetLastError());
    if (c->project) return project_device(c, d_q, nvdf);
    return DGV_OK;
}

}  // namespace dgv
