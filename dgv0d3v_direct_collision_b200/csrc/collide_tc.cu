// collide_tc.cu -- batched Q(f,f) on the 5th-generation tensor cores.
//
// Per cell-pair block (c1,c2) and output cell D the operator is a product of
// two small matrices:  Q[(D,b), p] += sum_k  P[(D,b), k] * V[k, p],
//   P[(D,b), k] = f_b(c1+D-ccell, l1_k) * f_b(c2+D-ccell, l2_k)   (k = pair)
//   V[k, p]     = A value of canonical basis function p for pair k.
// One tcgen05.mma tile has M = 128 rows = NDG consecutive output cells x VB
// VDFs (VB = 128, 64 or 32 by batch size), N = 32 basis functions (P <= 32,
// zero-padded), K = 16 pairs.  A CTA owns one row tile for the blocks of one
// launch; its A-values arrive as 64-pair chunk records (TMA bulk copies,
// shared by every CTA of the launch through L2), and the f values of the
// block's 2 x NDG cells are staged in shared memory once per block.
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
//   warp 0      producer: TMA bulk copies of f slices and V chunk records
//   warp 1      allocates tensor memory; lane 0 issues the MMAs
//   warps 2-9   generators: warp w writes k-group w (8 pairs) of the P tiles
//               (split fp16) for all 128 rows
//   warps 10-13 epilogue: chunk and block sums, final FP64 add
// Every wait is bounded (%globaltimer); a timeout raises the error flag, each
// role still reaches the final barrier, in-flight copies and MMAs are
// drained, and tensor memory is freed before the CTA exits.
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "dgv_internal.h"
#include "pipeline.cuh"

namespace dgv {

constexpr int TC_KCH = 64;                          // pairs per chunk record
constexpr int TC_TILE_B = 32 * TC_KCH * 2;          // one 32 x 64 fp16 tile (4 KiB)
constexpr int TC_REC = 2 * TC_TILE_B + TC_KCH * 2;  // hi tile, lo tile, (l1,l2) bytes
constexpr int TC_ROWS = 128;
constexpr int TC_ATILE = TC_ROWS * TC_KCH * 2;      // 128 x 64 fp16 (16 KiB)
constexpr int TC_NSTB = 6;                          // V ring stages
constexpr int TC_THREADS = 448;
constexpr int TC_GEN_WARPS = 8;
constexpr int TC_EPI_WARPS = 4;
static_assert(TC_GEN_WARPS * 8 == TC_KCH, "one generator warp per k-group of 8 pairs");

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
    const float *F;           // [nbt][Nc][P][VB] scaled f, zero for padded VDFs
    const unsigned char *V;   // chunk records
    const int *chunk_start;   // [nblocks+1]
    const BlockInfo *blk;
    const int *order;         // row-tile order of this launch (heaviest first)
    double *qacc;             // [(D*P+p)*NV + vdf]
    const double *inv_scale;  // [NV]
    int *err;
    int b0, b1;               // block range of this launch
    int Nc, P, Mv, Mw, ccell, NV, nvdf, nbt;
    int off_f, fslot;         // shared-memory offset and size of one f slot
};

template <int NDG>
__device__ __forceinline__ bool dgroup_meets(const BlockInfo &bi, int D0, int Nc, int Mv, int Mw)
{
#pragma unroll
    for (int d = 0; d < NDG; d++) {
        const int D = D0 + d;
        if (D >= Nc) break;
        const int Du = D / (Mv * Mw), Dv = (D / Mw) % Mv, Dw = D % Mw;
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
template <int VB>
__global__ void __launch_bounds__(512, 1) k_collide_tc(TcArgs a)
{
    constexpr int NDG = TC_ROWS / VB;  // output cells per row tile
    constexpr int NJ = VB / 32;        // VDF groups of 32 per output cell
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *abuf = smem;                   // 2 x (hi, lo) A tiles
    unsigned char *vring = smem + 4 * TC_ATILE;   // TC_NSTB x TC_REC
    float *fs = reinterpret_cast<float *>(smem + a.off_f);  // 2 slots x {side 1, side 2}
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + a.off_f + 2 * a.fslot);
    uint64_t *b_full = bars, *b_empty = bars + TC_NSTB;
    uint64_t *a_full = bars + 2 * TC_NSTB, *a_empty = a_full + 2;
    uint64_t *h_full = a_empty + 2, *h_empty = h_full + 2;  // chunk accumulators
    uint64_t *l_full = h_empty + 2, *l_empty = l_full + 2;  // block accumulators
    uint64_t *f_full = l_empty + 2, *f_empty = f_full + 2;  // f slots
    uint64_t *drain = f_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bt = blockIdx.x % a.nbt, D0 = a.order[blockIdx.x / a.nbt] * NDG;
    const int cell_floats = a.P * VB;  // one cell of one VDF tile
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
            mbar_init(&f_full[s], 1);
            mbar_init(&f_empty[s], TC_GEN_WARPS);
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
            int g = 0, q = 0;
            bool ok = true;
            const float *Fbt = a.F + (size_t)bt * a.Nc * cell_floats;
            for (int b = a.b0; b < a.b1 && ok; b++) {
                const BlockInfo bi = a.blk[b];
                if (!dgroup_meets<NDG>(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
                // f of cells c1 + D - ccell and c2 + D - ccell, D in the tile,
                // clipped to the grid (cells outside are never read)
                const int fb = q & 1;
                if (!mbar_wait(&f_empty[fb], ((q >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                int lo[2], hi[2];
                uint32_t tx = 0;
                for (int sd = 0; sd < 2; sd++) {
                    const int cs = (sd ? bi.c2 : bi.c1) + D0 - a.ccell;
                    lo[sd] = max(cs, 0);
                    hi[sd] = min(cs + NDG, a.Nc);
                    if (hi[sd] > lo[sd]) tx += (uint32_t)((hi[sd] - lo[sd]) * cell_floats * 4);
                }
                if (tx) {
                    mbar_arrive_expect_tx(&f_full[fb], tx);
                    for (int sd = 0; sd < 2; sd++) {
                        if (hi[sd] <= lo[sd]) continue;
                        const int cs = (sd ? bi.c2 : bi.c1) + D0 - a.ccell;
                        float *dst = fs + (size_t)(2 * fb + sd) * NDG * cell_floats + (size_t)(lo[sd] - cs) * cell_floats;
                        bulk_g2s(dst, Fbt + (size_t)lo[sd] * cell_floats, (uint32_t)((hi[sd] - lo[sd]) * cell_floats * 4),
                                 &f_full[fb]);
                    }
                } else {
                    mbar_arrive(&f_full[fb]);
                }
                q++;
                const int c0 = a.chunk_start[b], c1 = a.chunk_start[b + 1];
                for (int c = c0; c < c1; c++, g++) {
                    const int s = g % TC_NSTB;
                    if (!mbar_wait(&b_empty[s], ((g / TC_NSTB) & 1) ^ 1, a.err)) { ok = false; break; }
                    mbar_arrive_expect_tx(&b_full[s], TC_REC);
                    bulk_g2s(vring + s * TC_REC, a.V + (size_t)c * TC_REC, TC_REC, &b_full[s]);
                }
            }
            if (!ok) {  // let the copies already issued land
                for (int j = g > TC_NSTB ? g - TC_NSTB : 0; j < g; j++)
                    mbar_wait(&b_full[j % TC_NSTB], (j / TC_NSTB) & 1, a.err);
                for (int j = q > 2 ? q - 2 : 0; j < q; j++) mbar_wait(&f_full[j & 1], (j >> 1) & 1, a.err);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int g = 0, q = 0;
            bool ok = true;
            for (int b = a.b0; b < a.b1 && ok; b++) {
                const BlockInfo bi = a.blk[b];
                if (!dgroup_meets<NDG>(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
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
        const int kg = warp - 2;  // k-group of this warp: pairs 8 kg .. 8 kg + 7 of a chunk
        int Dc[NDG];
#pragma unroll
        for (int d = 0; d < NDG; d++) Dc[d] = D0 + d;
        int g = 0, q = 0;
        bool ok = true;
        for (int b = a.b0; b < a.b1 && ok; b++) {
            const BlockInfo bi = a.blk[b];
            if (!dgroup_meets<NDG>(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
            bool valid[NDG];
#pragma unroll
            for (int d = 0; d < NDG; d++) {
                const int D = Dc[d];
                const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
                valid[d] = D < a.Nc && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] &&
                           Dw >= bi.lo[2] && Dw <= bi.hi[2];
            }
            const int fb = q & 1;
            if (!mbar_wait_warp(&f_full[fb], (q >> 1) & 1, a.err)) { ok = false; break; }
            const float *f1 = fs + (size_t)(2 * fb) * NDG * cell_floats + lane;
            const float *f2 = f1 + (size_t)NDG * cell_floats;
            const int c0 = a.chunk_start[b], c1 = a.chunk_start[b + 1];
            for (int c = c0; c < c1; c++, g++) {
                const int s = g % TC_NSTB, x = g & 1;
                if (!mbar_wait_warp(&b_full[s], (g / TC_NSTB) & 1, a.err)) { ok = false; break; }
                if (!mbar_wait_warp(&a_empty[x], ((g >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                const uint4 iv = *reinterpret_cast<const uint4 *>(vring + s * TC_REC + 2 * TC_TILE_B + 16 * kg);
                const uint32_t w4[4] = {iv.x, iv.y, iv.z, iv.w};
                int o1[8], o2[8];  // f offsets (floats) of the 8 pairs
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const uint32_t wd = w4[j >> 1] >> (16 * (j & 1));
                    o1[j] = (int)(wd & 0xffu) * VB;
                    o2[j] = (int)((wd >> 8) & 0xffu) * VB;
                }
                unsigned char *ah = abuf + (2 * x) * TC_ATILE, *al = abuf + (2 * x + 1) * TC_ATILE;
#pragma unroll
                for (int d = 0; d < NDG; d++) {
                    const float *p1 = f1 + d * cell_floats, *p2 = f2 + d * cell_floats;
#pragma unroll
                    for (int jj = 0; jj < NJ; jj++) {
                        const int row = d * VB + jj * 32 + lane;
                        uint32_t hi[4], lo[4];
                        if (valid[d]) {
                            float x8[8];
#pragma unroll
                            for (int j = 0; j < 8; j++) x8[j] = p1[o1[j] + jj * 32] * p2[o2[j] + jj * 32];
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
                }
                fence_async_shared();  // generic-proxy writes -> visible to the tensor core
                __syncwarp();
                if (lane == 0) mbar_arrive(&a_full[x]);
            }
            __syncwarp();
            if (lane == 0) mbar_arrive(&f_empty[fb]);  // this warp's reads of the f slot are done
            q++;
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
            if (!dgroup_meets<NDG>(bi, D0, a.Nc, a.Mv, a.Mw)) continue;
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
            const int d = r / VB, vdf = bt * VB + (r % VB);
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

// per-VDF scale 2^e (max |f| -> [32, 64)) and the scaled copy of f in VDF
// tiles of VB: F[((bt*Nc + cell)*P + l)*VB + v%VB]
__global__ void k_tc_fprep(const double *f, long long N, int nvdf, double vinv, float *F, double *inv_scale,
                           int Nc, int P, int VB)
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
    const int bt = v / VB, lb = v % VB;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) {
        const int cell = (int)(i / P), l = (int)(i - (long long)cell * P);
        const double x = v < nvdf ? f[(size_t)v * N + i] * s : 0.0;
        F[(((size_t)bt * Nc + cell) * P + l) * VB + lb] = (float)x;
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
        e = 14 - e;  // largest |value| -> [2^13, 2^14): fp16 hi parts stay finite
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
    // block sets of about 48 MB of chunk records each: one launch per set, its
    // records stay in L2 while every row tile reads them
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

// Row-tile order per launch: tiles (groups of NDG output cells) sorted by the
// chunk records they consume, heaviest first, so the last wave of CTAs is
// short.  One array of nsets x ngroups on the device, built once per NDG.
static int tc_order(Ctx *c, int NDG, const int **d_order)
{
    Layout &L = c->lay;
    auto it = L.tc_order.find(NDG);
    if (it != L.tc_order.end()) { *d_order = it->second; return DGV_OK; }
    const Grid &g = c->grid;
    const int ng = (g.Nc + NDG - 1) / NDG, nsets = (int)L.tc_sets.size() - 1;
    std::vector<int> all((size_t)nsets * ng);
    std::vector<long long> work(ng);
    std::vector<int> stamp(ng, -1);
    for (int s = 0; s < nsets; s++) {
        std::fill(work.begin(), work.end(), 0);
        for (int b = L.tc_sets[s]; b < L.tc_sets[s + 1]; b++) {
            const BlockInfo &bi = L.h_blk[b];
            const int ch = L.tc_chunk_host[b + 1] - L.tc_chunk_host[b];
            for (int u = bi.lo[0]; u <= bi.hi[0]; u++)
                for (int v = bi.lo[1]; v <= bi.hi[1]; v++)
                    for (int w = bi.lo[2]; w <= bi.hi[2]; w++) {
                        const int grp = ((u * g.d.Mv + v) * g.d.Mw + w) / NDG;
                        if (stamp[grp] != b) { stamp[grp] = b; work[grp] += ch; }
                    }
        }
        int *o = all.data() + (size_t)s * ng;
        std::iota(o, o + ng, 0);
        std::stable_sort(o, o + ng, [&](int x, int y) { return work[x] > work[y]; });
    }
    int *d = nullptr;
    DGV_CUDA(c, cudaMalloc(&d, sizeof(int) * all.size()));
    DGV_CUDA(c, cudaMemcpy(d, all.data(), sizeof(int) * all.size(), cudaMemcpyHostToDevice));
    L.tc_order[NDG] = d;
    *d_order = d;
    return DGV_OK;
}

template <int VB>
static int launch_tc(Ctx *c, TcArgs &a, const int *d_order, int ng)
{
    const size_t smem = (size_t)a.off_f + 2 * (size_t)a.fslot + (2 * TC_NSTB + 20) * sizeof(uint64_t) + 16;
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)k_collide_tc<VB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    const Layout &L = c->lay;
    for (size_t s = 0; s + 1 < L.tc_sets.size(); s++) {
        a.b0 = L.tc_sets[s];
        a.b1 = L.tc_sets[s + 1];
        a.order = d_order + s * ng;
        k_collide_tc<VB><<<(unsigned)(a.nbt * ng), TC_THREADS, smem, c->stream>>>(a);
        DGV_CUDA(c, cudaGetLastError());
    }
    return DGV_OK;
}

int collide_tc_device(Ctx *c, const double *d_f, double *d_q, int nvdf, double scale)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    if (!L.blk) return set_err(c, DGV_ESTATE, "collide: no A-arrays loaded");
    if (g.P > 32) return set_err(c, DGV_EUNSUP, "tensor-core path: at most 32 nodes per cell");
    if (nvdf < 1) return set_err(c, DGV_EINVAL, "collide: batch must hold at least one VDF");
    int rc = tc_prepare(c);
    if (rc) return rc;
    rc = ensure_errflag(c);
    if (rc) return rc;
    // VDFs per row tile: all 128 rows of a tile on one output cell when the
    // batch fills them, else 2 or 4 consecutive cells
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32), NDG = TC_ROWS / VB;
    const int nbt = (nvdf + VB - 1) / VB, NV = nbt * VB, ng = (g.Nc + NDG - 1) / NDG;
    const size_t fbytes = (size_t)nbt * g.Nc * g.P * VB * sizeof(float);
    const size_t qbytes = (size_t)g.N * NV * sizeof(double);
    rc = ensure_buffer(c, &c->d_tcF, &c->tcF_bytes, fbytes + NV * sizeof(double));
    if (rc) return rc;
    rc = ensure_buffer(c, &c->d_tcQ, &c->tcQ_bytes, qbytes);
    if (rc) return rc;
    const int *d_order = nullptr;
    rc = tc_order(c, NDG, &d_order);
    if (rc) return rc;
    float *F = reinterpret_cast<float *>(c->d_tcF);
    double *inv = reinterpret_cast<double *>(reinterpret_cast<char *>(c->d_tcF) + fbytes);
    k_tc_fprep<<<NV, 256, 0, c->stream>>>(d_f, g.N, nvdf, 1.0 / L.tc_vscale, F, inv, g.Nc, g.P, VB);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaMemsetAsync(c->d_tcQ, 0, qbytes, c->stream));
    TcArgs a;
    a.F = F; a.V = (const unsigned char *)L.tc_V; a.chunk_start = L.tc_chunk_start; a.blk = L.blk;
    a.order = nullptr; a.qacc = c->d_tcQ; a.inv_scale = inv; a.err = c->d_err;
    a.Nc = g.Nc; a.P = g.P; a.Mv = g.d.Mv; a.Mw = g.d.Mw; a.ccell = g.ccell; a.NV = NV; a.nvdf = nvdf; a.nbt = nbt;
    a.off_f = 4 * TC_ATILE + TC_NSTB * TC_REC;                 // 16-byte aligned
    a.fslot = 2 * NDG * g.P * VB * (int)sizeof(float);         // both sides of one block
    switch (VB) {
    case 128: rc = launch_tc<128>(c, a, d_order, ng); break;
    case 64: rc = launch_tc<64>(c, a, d_order, ng); break;
    default: rc = launch_tc<32>(c, a, d_order, ng); break;
    }
    if (rc) return rc;
    long long tot = (long long)nvdf * g.N;
    k_tc_final<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->d_tcQ, c->d_nwt, d_q, g.N, nvdf, NV, scale);
    DGV_CUDA(c, cudaGetLastError());
    if (c->project) return project_device(c, d_q, nvdf);
    return DGV_OK;
}

}  // namespace dgv
