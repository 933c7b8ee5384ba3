// collide_tc.cu -- batched Q(f,f) on the 5th-generation tensor cores.
//
// Two forms share this file: the chunk form described here (products of
// f-values formed per pair on the CUDA cores, DGV_OPT_TCFORM = 1) and the
// block form further down (dense per-block value matrices on the tensor core,
// the default for 8 or 27 nodes per cell).
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
constexpr int TC_REC = 2 * TC_TILE_B + TC_KCH * 4;  // hi tile, lo tile, f offsets of the pairs
constexpr int TC_ROWS = 128;
constexpr int TC_NSTB = 4;                          // V ring stages
constexpr int TC_NA = 4;                            // A tile stages
constexpr int TC_ATILE = TC_ROWS * TC_KCH * 2;      // 128 x 64 fp16 (16 KiB)
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

// registers written by the tcgen05.ld forms below are valid after tmem_wait_ld()
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// the same wait with the 32 registers of one load as operands: no use of them
// can be scheduled before it
__device__ __forceinline__ void tmem_wait_ld32(uint32_t *r)
{
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]), "+r"(r[15]),
                   "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]), "+r"(r[22]), "+r"(r[23]),
                   "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]), "+r"(r[29]), "+r"(r[30]), "+r"(r[31])
                 :
                 : "memory");
}

// 32 consecutive columns of this warp's lane quarter in one instruction (no wait)
__device__ __forceinline__ void tmem_ld32_nowait(uint32_t taddr, uint32_t *r)
{
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                 : "=r"(r[0]),"=r"(r[1]),"=r"(r[2]),"=r"(r[3]),"=r"(r[4]),"=r"(r[5]),"=r"(r[6]),"=r"(r[7]),"=r"(r[8]),"=r"(r[9]),"=r"(r[10]),"=r"(r[11]),"=r"(r[12]),"=r"(r[13]),"=r"(r[14]),"=r"(r[15]),"=r"(r[16]),"=r"(r[17]),"=r"(r[18]),"=r"(r[19]),"=r"(r[20]),"=r"(r[21]),"=r"(r[22]),"=r"(r[23]),"=r"(r[24]),"=r"(r[25]),"=r"(r[26]),"=r"(r[27]),"=r"(r[28]),"=r"(r[29]),"=r"(r[30]),"=r"(r[31])
                 : "r"(taddr));
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

// two FP32 products with one packed instruction (round to nearest, as FMUL)
__device__ __forceinline__ float2 fmul2(float2 a, float2 b)
{
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mul.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}

// bounded wait whose outcome is the same for every lane of the warp (the
// warp-collective tensor-memory instructions that follow need a converged warp)
__device__ __forceinline__ bool mbar_wait_warp(uint64_t *bar, uint32_t parity, int *err,
                                               unsigned long long limit_ns = WAIT_LIMIT_NS)
{
    const bool ok = mbar_wait(bar, parity, err, limit_ns);
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

// One entry of a row tile's work list: a block whose valid output-cell box
// meets the tile, with its chunk records and the tile cells it is valid for.
struct __align__(16) TcItem {
    int chunk0;  // first chunk record
    int nch;     // chunk records (bits 0-15) | valid cell slots of the tile << 16
    int c1, c2;  // cells of the block, canonical frame
};

struct TcArgs {
    const float *F;           // [nbt][Nc][P][VB] scaled f, zero for padded VDFs
    const unsigned char *V;   // chunk records
    const TcItem *items;      // work lists of this launch
    const int *item_start;    // [ntiles + 1] into items, tiles in launch order
    const int *tile_of;       // row-tile index (group of NDG cells) in launch order
    double *qacc;             // [(D*P+p)*NV + vdf]
    const double *inv_scale;  // [NV]
    int *err;
    int Nc, P, ccell, NV, nvdf, nbt;
    int off_f, fslot;         // shared-memory offset and size of one f slot
};

// 512 in the launch bound caps registers at 128 per thread: with 14 warps,
// two of the four SM sub-partitions hold 4 warps each.
//
// Tensor memory (256 columns): per chunk (double buffered, 64 columns each)
// hi*hi in the first 32 columns and hi*lo + lo*hi in the next 32; the
// compensated sum and its correction in columns 128-159 / 160-191.
template <int VB>
__global__ void __launch_bounds__(512, 1) k_collide_tc(TcArgs a)
{
    constexpr int NDG = TC_ROWS / VB;  // output cells per row tile
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char *abuf = smem;                          // TC_NA x (hi, lo) A tiles
    unsigned char *vring = smem + 2 * TC_NA * TC_ATILE;  // TC_NSTB x TC_REC
    float *fs = reinterpret_cast<float *>(smem + a.off_f);  // 2 slots x {side 1, side 2}
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + a.off_f + 2 * a.fslot);
    uint64_t *b_full = bars, *b_empty = bars + TC_NSTB;
    uint64_t *a_full = bars + 2 * TC_NSTB, *a_empty = a_full + TC_NA;
    uint64_t *h_full = a_empty + TC_NA, *h_empty = h_full + 2;  // chunk accumulators
    uint64_t *f_full = h_empty + 2, *f_empty = f_full + 2;      // f slots
    uint64_t *drain = f_empty + 2;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(drain + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int bt = blockIdx.x % a.nbt, ti = blockIdx.x / a.nbt;
    const int D0 = a.tile_of[ti] * NDG;
    const int i0 = a.item_start[ti], i1 = a.item_start[ti + 1];
    const int cell_floats = a.P * VB;  // one cell of one VDF tile
    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_NSTB; s++) {
            mbar_init(&b_full[s], 1);
            mbar_init(&b_empty[s], 1);
        }
        for (int s = 0; s < TC_NA; s++) {
            mbar_init(&a_full[s], TC_GEN_WARPS);
            mbar_init(&a_empty[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            mbar_init(&h_full[s], 1);
            mbar_init(&h_empty[s], TC_EPI_WARPS);
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

    if (warp == 0) {
        // ---------------- producer ----------------
        if (lane == 0) {
            int g = 0, q = 0;
            bool ok = true;
            const float *Fbt = a.F + (size_t)bt * a.Nc * cell_floats;
            for (int it = i0; it < i1 && ok; it++) {
                const TcItem e = a.items[it];
                // f of cells c1 + D - ccell and c2 + D - ccell, D in the tile,
                // clipped to the grid (cells outside are never read)
                const int fb = q & 1;
                if (!mbar_wait(&f_empty[fb], ((q >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                int lo[2], hi[2];
                uint32_t tx = 0;
                for (int sd = 0; sd < 2; sd++) {
                    const int cs = (sd ? e.c2 : e.c1) + D0 - a.ccell;
                    lo[sd] = max(cs, 0);
                    hi[sd] = min(cs + NDG, a.Nc);
                    if (hi[sd] > lo[sd]) tx += (uint32_t)((hi[sd] - lo[sd]) * cell_floats * 4);
                }
                if (tx) {
                    mbar_arrive_expect_tx(&f_full[fb], tx);
                    for (int sd = 0; sd < 2; sd++) {
                        if (hi[sd] <= lo[sd]) continue;
                        const int cs = (sd ? e.c2 : e.c1) + D0 - a.ccell;
                        float *dst = fs + (size_t)(2 * fb + sd) * NDG * cell_floats + (size_t)(lo[sd] - cs) * cell_floats;
                        bulk_g2s(dst, Fbt + (size_t)lo[sd] * cell_floats, (uint32_t)((hi[sd] - lo[sd]) * cell_floats * 4),
                                 &f_full[fb]);
                    }
                } else {
                    mbar_arrive(&f_full[fb]);
                }
                q++;
                const int nch = e.nch & 0xffff;
                for (int c = 0; c < nch; c++, g++) {
                    const int s = g % TC_NSTB;
                    if (!mbar_wait(&b_empty[s], ((g / TC_NSTB) & 1) ^ 1, a.err)) { ok = false; break; }
                    mbar_arrive_expect_tx(&b_full[s], TC_REC);
                    bulk_g2s(vring + s * TC_REC, a.V + (size_t)(e.chunk0 + c) * TC_REC, TC_REC, &b_full[s]);
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
            // instruction descriptors: FP32 accumulator, fp16 A and B, both
            // K-major, M = 128, N = 64 (B hi and lo tiles: hi*hi and hi*lo in
            // one instruction) or N = 32 (B hi tile: lo*hi)
            const uint32_t id64 = (1u << 4) | ((uint32_t)(64 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
            const uint32_t id32 = (1u << 4) | ((uint32_t)(32 >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
            const uint64_t dA0 = umma_desc(smem_u32(abuf), 128, 1024);
            const uint64_t dV0 = umma_desc(smem_u32(vring), 128, 1024);
            int g = 0;
            bool ok = true;
            for (int it = i0; it < i1 && ok; it++) {
                const int nch = a.items[it].nch & 0xffff;
                for (int c = 0; c < nch; c++, g++) {
                    const int s = g % TC_NSTB, xa = g % TC_NA, xh = g & 1;
                    if (!mbar_wait(&b_full[s], (g / TC_NSTB) & 1, a.err)) { ok = false; break; }
                    if (!mbar_wait(&a_full[xa], (g / TC_NA) & 1, a.err)) { ok = false; break; }
                    if (!mbar_wait(&h_empty[xh], ((g >> 1) & 1) ^ 1, a.err)) { ok = false; break; }
                    tc_fence_after();
                    const uint32_t dacc = tmem + (uint32_t)(xh * 64);
                    // descriptor start addresses are in 16-byte units
                    const uint64_t dAh = dA0 + (uint64_t)((2 * xa) * TC_ATILE >> 4);
                    const uint64_t dAl = dA0 + (uint64_t)((2 * xa + 1) * TC_ATILE >> 4);
                    const uint64_t dB = dV0 + (uint64_t)(s * TC_REC >> 4);
#pragma unroll
                    for (int t = 0; t < TC_KCH / 16; t++) {  // K = 16: two core matrices (256 B) per step
                        umma_f16(dacc, dAh + 16 * t, dB + 16 * t, id64, t == 0 ? 0u : 1u);
                        umma_f16(dacc + 32, dAl + 16 * t, dB + 16 * t, id32, 1u);
                    }
                    umma_commit(&a_empty[xa]);
                    umma_commit(&b_empty[s]);
                    umma_commit(&h_full[xh]);
                }
            }
            // every MMA issued so far completes before tensor memory is freed
            umma_commit(drain);
            mbar_wait(drain, 0, a.err);
        }
        __syncwarp();
    } else if (warp < 2 + TC_GEN_WARPS) {
        // ---------------- generators ----------------
        // Lane l owns tile rows jj*32 + l (jj = 0..3): output cell slot
        // l / (VB/4) and the 4 consecutive VDFs 4*(l % (VB/4)) + jj, so one
        // 16-byte shared load gives the f values of all 4 rows.
        const int kg = warp - 2;  // k-group of this warp: pairs 8 kg .. 8 kg + 7 of a chunk
        constexpr int LPC = VB / 4;                             // lanes per output cell
        constexpr int SH = VB == 128 ? 0 : (VB == 64 ? 1 : 2);  // offsets are stored for VB = 128
        const int dl = lane / LPC, vq = lane % LPC;
        int g = 0, q = 0;
        bool ok = true;
        for (int it = i0; it < i1 && ok; it++) {
            const TcItem e = a.items[it];
            const bool valid = (e.nch >> (16 + dl)) & 1;
            const int fb = q & 1;
            if (!mbar_wait_warp(&f_full[fb], (q >> 1) & 1, a.err)) { ok = false; break; }
            // rows of cells outside the block's box read stale (in-bounds) shared
            // memory and are zeroed below
            const float *f1 = fs + (size_t)(2 * fb) * NDG * cell_floats + (size_t)dl * cell_floats + 4 * vq;
            const float *f2 = f1 + (size_t)NDG * cell_floats;
            const int nch = e.nch & 0xffff;
            for (int c = 0; c < nch; c++, g++) {
                const int s = g % TC_NSTB, xa = g % TC_NA;
                if (!mbar_wait_warp(&b_full[s], (g / TC_NSTB) & 1, a.err)) { ok = false; break; }
                if (!mbar_wait_warp(&a_empty[xa], ((g / TC_NA) & 1) ^ 1, a.err)) { ok = false; break; }
                const uint4 *ip = reinterpret_cast<const uint4 *>(vring + s * TC_REC + 2 * TC_TILE_B + 32 * kg);
                const uint4 i0v = ip[0], i1v = ip[1];
                const uint32_t w8[8] = {i0v.x, i0v.y, i0v.z, i0v.w, i1v.x, i1v.y, i1v.z, i1v.w};
                float xv[8][4];
                float4 a1 = make_float4(0.f, 0.f, 0.f, 0.f);
                uint32_t prev = 0xffffffffu;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const uint32_t o1 = (w8[j] & 0xffffu) >> SH, o2 = (w8[j] >> 16) >> SH;
                    if (o1 != prev) {  // pairs are sorted by l1: reuse the last f1 load
                        a1 = *reinterpret_cast<const float4 *>(f1 + o1);
                        prev = o1;
                    }
                    const float4 a2 = *reinterpret_cast<const float4 *>(f2 + o2);
                    const float2 p01 = fmul2(make_float2(a1.x, a1.y), make_float2(a2.x, a2.y));
                    const float2 p23 = fmul2(make_float2(a1.z, a1.w), make_float2(a2.z, a2.w));
                    xv[j][0] = p01.x; xv[j][1] = p01.y; xv[j][2] = p23.x; xv[j][3] = p23.y;
                }
                unsigned char *ah = abuf + (2 * xa) * TC_ATILE, *al = abuf + (2 * xa + 1) * TC_ATILE;
#pragma unroll
                for (int jj = 0; jj < 4; jj++) {
                    const int row = jj * 32 + lane;
                    uint32_t hi[4], lo[4];
#pragma unroll
                    for (int j = 0; j < 4; j++) split2(xv[2 * j][jj], xv[2 * j + 1][jj], hi[j], lo[j]);
                    if (!valid) {
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
                if (lane == 0) mbar_arrive(&a_full[xa]);
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
        int g = 0;
        bool ok = true;
        for (int it = i0; it < i1 && ok; it++) {
            const int nch = a.items[it].nch & 0xffff;
            for (int c = 0; c < nch; c++, g++) {
                const int xh = g & 1;
                if (!mbar_wait_warp(&h_full[xh], (g >> 1) & 1, a.err)) { ok = false; break; }
                tc_fence_after();
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float vh[16], vl[16];
                    tmem_ld16(tl + xh * 64 + 16 * h, vh);
                    tmem_ld16(tl + xh * 64 + 32 + 16 * h, vl);
#pragma unroll
                    for (int i = 0; i < 16; i++) run[16 * h + i] += vh[i] + vl[i];
                }
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&h_empty[xh]);
            }
            if (!ok) break;
#pragma unroll
            for (int h = 0; h < 2; h++) {  // two-sum of the block total into (sum, correction)
                float sm[16], cm[16];
                tmem_ld16(tl + 128 + 16 * h, sm);
                tmem_ld16(tl + 160 + 16 * h, cm);
#pragma unroll
                for (int i = 0; i < 16; i++) {
                    const float xb = run[16 * h + i];
                    const float t = sm[i] + xb, bp = t - sm[i];
                    cm[i] += (sm[i] - (t - bp)) + (xb - bp);
                    sm[i] = t;
                    run[16 * h + i] = 0.f;
                }
                tmem_st16(tl + 128 + 16 * h, sm);
                tmem_st16(tl + 160 + 16 * h, cm);
            }
        }
        if (ok) {
            // tile row r = jj*32 + l: cell slot l / (VB/4), VDF 4*(l % (VB/4)) + jj
            const int l = r & 31, jj = r >> 5;
            const int d = l / (VB / 4), vdf = bt * VB + 4 * (l % (VB / 4)) + jj;
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
// per pair the f offsets l1*128 | l2*128 << 16}; tiles K-major without swizzle: element (p, k) at byte
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
        // f offsets (floats) of the two factors in a 128-VDF tile slice
        *reinterpret_cast<uint32_t *>(rec + 2 * TC_TILE_B + 4 * k) = (uint32_t)(l1 * 128) | ((uint32_t)(l2 * 128) << 16);
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
                           int Nc, int P, int VB, int pw)
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
    if (threadIdx.x == 0) inv_scale[v] = ldexp(1.0, -pw * e) * vinv;  // f enters the result pw times
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
// power-of-two scale of the A values: the largest |value| -> [2^13, 2^14), so
// fp16 hi parts stay finite
static int tc_value_scale(Ctx *c, double *scale)
{
    const Layout &L = c->lay;
    const Grid &g = c->grid;
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
    *scale = std::ldexp(1.0, e);
    return DGV_OK;
}

static int tc_prepare(Ctx *c)
{
    Layout &L = c->lay;
    if (L.tc_V) return DGV_OK;
    const Grid &g = c->grid;
    std::vector<int> cs(L.nblocks + 1, 0);
    for (long long b = 0; b < L.nblocks; b++) cs[b + 1] = cs[b] + (L.h_blk[b].count + TC_KCH - 1) / TC_KCH;
    const long long nch = cs[L.nblocks];
    int rc = tc_value_scale(c, &L.tc_vscale);
    if (rc) return rc;
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

// Work lists, built once per cells-per-tile NDG and form: for every launch
// (block set) and row tile (NDG consecutive output cells), the blocks whose
// valid box meets the tile, in block order, with the tile cells each is valid
// for.  Tiles of a launch are ordered by their work, heaviest first, so the
// last wave of CTAs is short.  An item carries first[b] (the block's first
// chunk record, or the block index) and count[b] (its chunk records, or 1).
struct TcLists {
    TcItem *items = nullptr;
    int *item_start = nullptr;  // per set: ntiles + 1 entries
    int *tile_of = nullptr;     // per set: ntiles entries
};

// Adds the items of one block for one owner-cell shift: every output cell D
// of the block's box maps to the owner cell T = D + shift (linear indices;
// exact, the box keeps both shifted cells inside the grid); owner cells of a
// tile are consecutive, so an item is pushed once per (tile, id) and the
// owner cells it serves are set as bits.
// An item's nch holds `low` (chunk form: its chunk records; block form: the
// block's mask of nodes l1) and the owner-cell bits from bit `vshift` (16 in
// the chunk form, 27 in the block form); `weight` is its work for the tile
// ordering and the plan.
static void tc_items_for_block(const Grid &g, const BlockInfo &bi, int NDG, int shift, int id, int low, int vshift,
                               long long weight, int fc1, int fc2, std::vector<std::vector<TcItem>> &per,
                               std::vector<long long> &work)
{
    int last = -1;
    for (int u = bi.lo[0]; u <= bi.hi[0]; u++)
        for (int v = bi.lo[1]; v <= bi.hi[1]; v++)
            for (int w = bi.lo[2]; w <= bi.hi[2]; w++) {
                const int T = (u * g.d.Mv + v) * g.d.Mw + w + shift, grp = T / NDG;
                if (grp != last) {  // same tile as the last cell or new
                    if (per[grp].empty() || per[grp].back().chunk0 != id) {
                        per[grp].push_back(TcItem{id, low, fc1, fc2});
                        work[grp] += weight;
                    }
                    last = grp;
                }
                per[grp].back().nch |= 1 << (vshift + T % NDG);
            }
}

constexpr int T2_N_ = 256;  // column group width of the block form (T2_N below)

// columns the MMAs of one block-form item issue: groups of 256, the last
// rounded up to 16
__host__ __device__ inline int t2_issued_cols(int ncol)
{
    const int ng = (ncol + T2_N_ - 1) / T2_N_;
    return (ng - 1) * T2_N_ + ((ncol - (ng - 1) * T2_N_) + 15) / 16 * 16;
}

// mode 0: items of the chunk form (owner = output cell D; first/count = the
// blocks' chunk records); mode 1: items of the block form's collision
// operator (owner = output cell D; chunk0 = the block's first record group,
// nch = its mask of nodes l1); mode 2: items of the block-form adjoint (owner
// = target cell T, two scatters per block, see k_collide_tc2)
static int tc_work_lists(Ctx *c, int NDG, int key, const std::vector<int> &sets, const std::vector<int> &first,
                         const std::vector<int> &count, TcLists *out, int mode = 0)
{
    Layout &L = c->lay;
    auto it = L.tc_lists.find(key);
    if (it != L.tc_lists.end()) {
        out->items = reinterpret_cast<TcItem *>(it->second[0]);
        out->item_start = reinterpret_cast<int *>(it->second[1]);
        out->tile_of = reinterpret_cast<int *>(it->second[2]);
        return DGV_OK;
    }
    const Grid &g = c->grid;
    const int ng = (g.Nc + NDG - 1) / NDG, nsets = (int)sets.size() - 1;
    std::vector<TcItem> items;
    std::vector<int> start((size_t)nsets * (ng + 1)), tile_of((size_t)nsets * ng);
    std::vector<std::vector<TcItem>> per(ng);
    std::vector<long long> work(ng);
    long long wsum = 0;
    for (int s = 0; s < nsets; s++) {
        for (auto &v : per) v.clear();
        std::fill(work.begin(), work.end(), 0);
        for (int b = sets[s]; b < sets[s + 1]; b++) {
            const BlockInfo &bi = L.h_blk[b];
            if (mode == 0) {
                tc_items_for_block(g, bi, NDG, 0, first[b], count[b], 16, count[b], bi.c1, bi.c2, per, work);
            } else if (mode == 1) {
                const int msk = (int)L.tc2_mask[b];
                tc_items_for_block(g, bi, NDG, 0, (int)L.tc2_goff[b], msk, 27,
                                   t2_issued_cols(__builtin_popcount(msk) * g.P), bi.c1, bi.c2, per, work);
            } else {
                const int o1 = bi.c1 - g.ccell, o2 = bi.c2 - g.ccell;
                const int m1 = (int)L.tc2_mask[b], m2 = (int)L.tc2_mask[L.nblocks + b];
                // pass 1 (W, to the c1 side): side cells T - o1, F16 cells T - o1 + o2
                tc_items_for_block(g, bi, NDG, o1, (int)L.tc2_goff[b], m1, 27,
                                   t2_issued_cols(__builtin_popcount(m1) * g.P), g.ccell - o1, g.ccell + o2 - o1,
                                   per, work);
                // pass 2 (W2, to the c2 side): side cells T - o2, F16 cells T - o2 + o1
                tc_items_for_block(g, bi, NDG, o2, (int)L.tc2_goff2[b] | (1 << 30), m2, 27,
                                   t2_issued_cols(__builtin_popcount(m2) * g.P), g.ccell - o2, g.ccell + o1 - o2,
                                   per, work);
            }
        }
        for (long long wv : work) wsum += wv;
        int *o = tile_of.data() + (size_t)s * ng;
        std::iota(o, o + ng, 0);
        std::stable_sort(o, o + ng, [&](int x, int y) { return work[x] > work[y]; });
        int *st = start.data() + (size_t)s * (ng + 1);
        for (int t = 0; t < ng; t++) {
            st[t] = (int)items.size();
            items.insert(items.end(), per[o[t]].begin(), per[o[t]].end());
        }
        st[ng] = (int)items.size();
    }
    if (items.size() > (size_t)INT32_MAX) return set_err(c, DGV_EUNSUP, "tensor-core path: work list too long");
    void *d[3] = {nullptr, nullptr, nullptr};
    DGV_CUDA(c, cudaMalloc(&d[0], sizeof(TcItem) * std::max<size_t>(1, items.size())));
    DGV_CUDA(c, cudaMalloc(&d[1], sizeof(int) * start.size()));
    DGV_CUDA(c, cudaMalloc(&d[2], sizeof(int) * tile_of.size()));
    if (!items.empty()) DGV_CUDA(c, cudaMemcpy(d[0], items.data(), sizeof(TcItem) * items.size(), cudaMemcpyHostToDevice));
    DGV_CUDA(c, cudaMemcpy(d[1], start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice));
    DGV_CUDA(c, cudaMemcpy(d[2], tile_of.data(), sizeof(int) * tile_of.size(), cudaMemcpyHostToDevice));
    L.tc_lists[key] = {d[0], d[1], d[2]};
    L.tc_list_work[key] = wsum;
    L.tc_list_items[key] = (long long)items.size();
    out->items = reinterpret_cast<TcItem *>(d[0]);
    out->item_start = reinterpret_cast<int *>(d[1]);
    out->tile_of = reinterpret_cast<int *>(d[2]);
    return DGV_OK;
}

static int tc_lists(Ctx *c, int NDG, TcLists *out)
{
    const Layout &L = c->lay;
    std::vector<int> first(L.nblocks), count(L.nblocks);
    for (long long b = 0; b < L.nblocks; b++) {
        first[b] = L.tc_chunk_host[b];
        count[b] = L.tc_chunk_host[b + 1] - L.tc_chunk_host[b];
    }
    return tc_work_lists(c, NDG, NDG, L.tc_sets, first, count, out);
}

// ============================================================================
// Block form.  The values of a cell-pair block (c1, c2) form a dense matrix
//   W[l2, (l1, p)] = V[pair (l1, l2), p]   (0 where the block has no pair),
// so that for output cell D and VDF b
//   Q[(D,b), p] += sum_l1 f_b(c1+D, l1) * G[(D,b), (l1, p)],   G = F2 W,
//   F2[(D,b), l2] = f_b(c2+D, l2).
// G is a tensor-core product per block: M = 128 rows, K = 32 nodes l2
// (zero-padded), N = P*P columns (l1, p) in groups of 256; F2 and W are split
// into fp16 hi + lo and hi*hi, hi*lo and lo*hi go into one FP32 accumulator.
// The CUDA cores then contract each group of G with f(c1+D) in FP32 and add the
// block total into a (sum, correction) pair with two-sum, in registers.  The
// per-pair products of the chunk form become columns of G: the CUDA cores do
// P*P multiply-adds per row and block instead of forming and splitting one
// product per pair and row.
//
// A CTA owns one row tile (NDG output cells x VB VDFs) for two consecutive
// VDF tiles, so each block's W crosses from L2 once for 256 rows.
// Warp roles (320 threads, one CTA per SM):
//   warp 0     producer: TMA bulk copies of f (both tiles) and W groups
//   warp 1     allocates all 512 tensor-memory columns; lane 0 issues MMAs
//   warps 2-9  epilogue: warp w serves VDF tile (w-2)/4, tensor-memory lanes
//              32*(w%4) .. +31 (one row per thread)
// Tensor memory: two accumulators of 256 columns, used alternately by the
// (group, VDF tile) jobs.  Measured on B200: an M = 128 MMA costs ~130 cycles
// at N = 128 whether A comes from shared or tensor memory, and about the same
// at N = 256, so the wide groups halve the MMA time of a block.  Every wait is
// bounded, as in the chunk form.
constexpr int T2_N = 256;                     // columns (l1, p) per group
constexpr int T2_K = 32;                      // nodes l2 per block, zero-padded
constexpr int T2_TILE = T2_N * T2_K * 2;      // one fp16 tile (16 KiB)
constexpr int T2_GREC = 2 * T2_TILE;          // hi and lo tiles of one group
constexpr int T2_NSTW = 3;                    // W ring stages
constexpr int T2_ATILE = TC_ROWS * T2_K * 2;  // 128 rows x 32 fp16 (8 KiB)
constexpr int T2_EPI_WARPS = 8;
// slot header, after the side tile of the slot's first VDF tile: the item's
// column count, for each rank jj of its mask the offset (floats) l*VB of the
// node l in the side tile (-1 past the mask's nodes), and the item's nch;
// written by the producer before it arms the slot
constexpr int T2_HDR = 128;
constexpr int T2_THREADS = 32 * (2 + T2_EPI_WARPS);

__host__ __device__ constexpr int t2_groups(int P) { return (P * P + T2_N - 1) / T2_N; }

// column groups of a collision-operator item: its block's mask of nodes l1
// is in the low 27 bits of nch
template <int P>
__device__ __forceinline__ int t2_item_groups(int nch)
{
    return (__popc((unsigned)nch & 0x7ffffffu) * P + T2_N - 1) / T2_N;
}

// byte offset of element (row, k) of a K-major tile without swizzle, K = 32:
// core matrices of 8 rows x 16 bytes, four along K (128 B apart), row groups
// of 8 512 B apart
__host__ __device__ __forceinline__ int t2_off(int row, int k)
{
    return ((row >> 3) * 4 + (k >> 3)) * 128 + (row & 7) * 16 + (k & 7) * 2;
}

// per block the masks of the nodes l1 (mask[b]) and l2 (mask[nblocks + b])
// its pairs use
__global__ void k_tc2_mask(const BlockInfo *blk, const double *rows64, int RD64, int Nc, int ccell, unsigned *mask,
                           long long nblocks)
{
    const BlockInfo bi = blk[blockIdx.x];
    unsigned m1 = 0u, m2 = 0u;
    for (int k = threadIdx.x; k < bi.count; k += blockDim.x) {
        const long long o = __double_as_longlong(rows64[(size_t)(bi.start + k) * RD64]);
        const int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
        m1 |= 1u << ((o1 - (bi.c1 - ccell)) / Nc);
        m2 |= 1u << ((o2 - (bi.c2 - ccell)) / Nc);
    }
    m1 = __reduce_or_sync(0xffffffffu, m1);
    m2 = __reduce_or_sync(0xffffffffu, m2);
    __shared__ unsigned sm[2][32];
    if ((threadIdx.x & 31) == 0) { sm[0][threadIdx.x >> 5] = m1; sm[1][threadIdx.x >> 5] = m2; }
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned r1 = 0u, r2 = 0u;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) { r1 |= sm[0][w]; r2 |= sm[1][w]; }
        mask[blockIdx.x] = r1;
        mask[nblocks + blockIdx.x] = r2;
    }
}

// one record per block: groups of {W hi tile, W lo tile}, group g holding
// columns n in [256 g, 256 g + 256) as tile rows, compacted to the nodes of
// one of the block's masks: arrangement 0 (the collision operator and the
// adjoint's pass to the c1 side) n = rank(l1)*P + p, K = l2, mask of the
// nodes l1; arrangement 1 (the adjoint's pass to the c2 side) n = rank(l2)*P +
// p, K = l1, mask of the nodes l2.  The block's record holds goff[b+1] -
// goff[b] = ceil(popc(mask) P / 256) groups from group goff[b] on.
__global__ void k_tc2_build(const BlockInfo *blk, const double *rows64, int RD64, int P, int Nc, int ccell,
                            float vscale, unsigned char *W, int arr, const unsigned *mask, const long long *goff)
{
    const BlockInfo bi = blk[blockIdx.x];
    const int NG = (int)(goff[blockIdx.x + 1] - goff[blockIdx.x]);
    const unsigned msk = mask[blockIdx.x];
    unsigned char *rec = W + (size_t)goff[blockIdx.x] * T2_GREC;
    uint4 *r4 = reinterpret_cast<uint4 *>(rec);
    for (int t = threadIdx.x; t < NG * T2_GREC / 16; t += blockDim.x) r4[t] = make_uint4(0u, 0u, 0u, 0u);
    __syncthreads();
    for (int t = threadIdx.x; t < bi.count * P; t += blockDim.x) {
        const int k = t / P, p = t - k * P;
        const double *row = rows64 + (size_t)(bi.start + k) * RD64;
        const long long o = __double_as_longlong(row[0]);
        const int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
        const int l1 = (o1 - (bi.c1 - ccell)) / Nc, l2 = (o2 - (bi.c2 - ccell)) / Nc;
        const int lc = arr == 0 ? l1 : l2, lk = arr == 0 ? l2 : l1;
        const int n = __popc(msk & ((1u << lc) - 1u)) * P + p, g = n / T2_N;
        const float x = (float)(row[1 + p] * (double)vscale);
        const __half h = __float2half_rn(x);
        const __half l = __float2half_rn(x - __half2float(h));
        unsigned char *dst = rec + (size_t)g * T2_GREC + t2_off(n - g * T2_N, lk);
        *reinterpret_cast<__half *>(dst) = h;
        *reinterpret_cast<__half *>(dst + T2_TILE) = l;
    }
}

// F16[((bt*2 + h)*Nc + cell) * VB*64 + t2_off(v, l)]: per VDF tile and cell a
// tile of VB rows (VDFs) x 32 nodes, h = 0 hi / 1 lo parts of the scaled FP32
// copy F[((bt*Nc + cell)*P + l)*VB + v]; nodes l >= P are zero
constexpr int T2_MAXG = 4;  // grids of one launch (mixed-grid batches)

// Per call, for the grids of one launch (one, or the members of a mixed-grid
// group): per VDF slot v (one CTA; slots past nvdf are zero rows) the
// power-of-two scale of f (max |f| -> [32, 64)), the scaled FP32 side tile
// F[bt][cell][l][lb] and its split fp16 operand tiles (hi, lo) in the MMA's
// A layout, nodes l >= P zero; inv_scale[v] undoes the scale in the result
// (f enters it pw times).
struct Tc2PrepGrid {
    const double *f;
    float *F;
    unsigned char *F16;
    double *inv_scale;
    long long N;
    int nvdf, NV, Nc, P, VB, pw;
    double vinv;
};
struct Tc2PrepLaunch {
    Tc2PrepGrid g[T2_MAXG];
    int ngrids;
    int vbase[T2_MAXG + 1];  // first CTA of each grid
};

__global__ void k_tc2_prep(const __grid_constant__ Tc2PrepLaunch A)
{
    int gi = 0;
    while (gi + 1 < A.ngrids && (int)blockIdx.x >= A.vbase[gi + 1]) gi++;
    const Tc2PrepGrid &G = A.g[gi];
    const int v = blockIdx.x - A.vbase[gi];
    __shared__ double red[32];
    double m = 0.0;
    if (v < G.nvdf)
        for (long long i = threadIdx.x; i < G.N; i += blockDim.x) m = fmax(m, fabs(G.f[(size_t)v * G.N + i]));
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
    const double sc = ldexp(1.0, e);
    if (threadIdx.x == 0) G.inv_scale[v] = ldexp(1.0, -G.pw * e) * G.vinv;
    const int bt = v / G.VB, lb = v % G.VB, P = G.P;
    const size_t tile = (size_t)G.VB * T2_K * 2;
    for (long long i = threadIdx.x; i < (long long)G.Nc * T2_K; i += blockDim.x) {
        const int cell = (int)(i / T2_K), l = (int)(i % T2_K);
        float x = 0.f;
        if (l < P) {
            x = v < G.nvdf ? (float)(G.f[(size_t)v * G.N + (size_t)cell * P + l] * sc) : 0.f;
            G.F[(((size_t)bt * G.Nc + cell) * P + l) * G.VB + lb] = x;
        }
        const __half h = __float2half_rn(x);
        const __half lo = __float2half_rn(x - __half2float(h));
        unsigned char *base = G.F16 + ((size_t)(2 * bt) * G.Nc + cell) * tile + t2_off(lb, l);
        *reinterpret_cast<__half *>(base) = h;
        *reinterpret_cast<__half *>(base + (size_t)G.Nc * tile) = lo;
    }
}

// q[v][i] = scale * 2 * qacc[i*NV + v] / w[i] for the grids of one launch
struct Tc2FinalGrid {
    const double *qacc, *w;
    double *q;
    long long N;
    int nvdf, NV;
    double scale;
};
struct Tc2FinalLaunch {
    Tc2FinalGrid g[T2_MAXG];
    int ngrids;
    long long ebase[T2_MAXG + 1];  // first output element of each grid
};

__global__ void k_tc2_final(const __grid_constant__ Tc2FinalLaunch A)
{
    const long long tot = A.ebase[A.ngrids];
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < tot;
         idx += (long long)gridDim.x * blockDim.x) {
        int gi = 0;
        while (gi + 1 < A.ngrids && idx >= A.ebase[gi + 1]) gi++;
        const Tc2FinalGrid &G = A.g[gi];
        const long long k = idx - A.ebase[gi];
        const int v = (int)(k % G.nvdf);
        const long long i = k / G.nvdf;
        double val = 2.0 * G.qacc[i * G.NV + v] / G.w[i];
        if (G.scale != 1.0) val = val * G.scale;
        G.q[(size_t)v * G.N + i] = val;
    }
}

struct Tc2Args {
    const float *F;            // [nbt][Nc][P][VB] FP32 side factor: scaled f (forward) or c = 2v/w (adjoint)
    const unsigned char *F16;  // [nbt][hi, lo][Nc][VB x 32 tile]
    const unsigned char *W;    // block records
    const unsigned char *W2;   // adjoint: the records of its pass to the c2 side (items with 1 << 30)
    const TcItem *items;       // work lists (chunk0 = first record group, | 1 << 30 for W2)
    const int *item_start;     // per block set: [ng + 1]
    const int *tile_of;        // per block set: row-tile index in work order [ng]
    double *qacc;              // [(D*P+p)*NV + vdf]
    const double *inv_scale;   // [NV]
    int *err;
    int *done;   // persistent launches: per (row tile, VDF-tile pair, epilogue warp) the sets added to qacc
    int Nc, ccell, NV, nvdf, nbt, nbp;
    int tpc;     // VDF tiles per CTA (1 or 2)
    int ng;      // row tiles
};


// One launch of the block form.  Its work is a sequence of units, unit
// ubase[g] + (s*ng + t)*nbp + bp serving, for grid g, block set s, the t-th
// row tile of that set's order (heaviest first) and the VDF tiles
// tpc*bp .. tpc*bp + tpc-1.
//   one launch per block set: CTA b serves unit b;
//   persistent (one launch for all sets and grids, one CTA per SM): each CTA's
//   producer takes the next unit from a counter (atomicAdd: units are handed
//   out in increasing order, balanced like the hardware's CTA dispatch) and
//   passes it to the MMA thread and the epilogue warps through a two-entry
//   queue in shared memory; the FP64 sums of a unit go into qacc after those
//   of the same rows' previous set (per-warp flags in done), so the additions
//   happen in the same order as with one launch per set and the results are
//   the same bit for bit.  A unit's predecessor has a smaller index, so it was
//   handed out earlier to a resident CTA: the waits on the flags end.
struct Tc2Launch {
    Tc2Args g[T2_MAXG];
    int ngrids;
    int ubase[T2_MAXG + 1];
    int *counter;  // persistent: the next unit to hand out (starts at 0); nullptr: unit = blockIdx.x
    int tpcmax;    // persistent: the VDF tiles every unit of the launch holds (the host launches persistent
                   // kernels only when all units hold the same number)
    int region;  // bytes per VDF tile in an item slot: A hi, A lo, side (FP32), slot header
    unsigned long long wait_ns;  // limit of every bounded wait
    int withhold;  // test of the bounded waits: CTA 0 withholds its first W copy
};

struct T2Unit {
    int gi, s, bp, tile, i0, i1, bt0, nb2;
};

// MG: the launch serves several grids (the unit's grid is looked up); else grid 0
template <bool MG>
__device__ __forceinline__ T2Unit t2_unit(const Tc2Launch &L, int u)
{
    T2Unit r;
    r.gi = 0;
    if constexpr (MG)
        while (r.gi + 1 < L.ngrids && u >= L.ubase[r.gi + 1]) r.gi++;
    const Tc2Args &a = L.g[MG ? r.gi : 0];
    int v = u - L.ubase[r.gi];
    const int per = a.nbp * a.ng;
    r.s = v / per;
    v -= r.s * per;
    r.bp = v % a.nbp;
    const int ti = v / a.nbp;
    r.tile = a.tile_of[(size_t)r.s * a.ng + ti];
    r.i0 = a.item_start[(size_t)r.s * (a.ng + 1) + ti];
    r.i1 = a.item_start[(size_t)r.s * (a.ng + 1) + ti + 1];
    r.bt0 = a.tpc * r.bp;
    r.nb2 = min(a.tpc, a.nbt - r.bt0);
    return r;
}

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(int *p, int v)
{
    asm volatile("st.release.gpu.global.b32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// bounded wait until *flag >= target (another CTA's release); like mbar_wait
// it gives up after limit_ns (raising err) or when err is raised elsewhere
__device__ __forceinline__ bool flag_wait(const int *flag, int target, int *err, unsigned long long limit_ns)
{
    if (ld_acquire_gpu(flag) >= target) return true;
    const unsigned long long t0 = globaltimer_ns();
    unsigned long long tcheck = t0;
    while (ld_acquire_gpu(flag) < target) {
        __nanosleep(256);
        const unsigned long long t = globaltimer_ns();
        if (t - t0 > limit_ns) {
            *(volatile int *)err = 1;
            return false;
        }
        if (t - tcheck > 1000000ULL) {
            tcheck = t;
            if (*(volatile int *)err) return false;
        }
    }
    return true;
}

// two-sum of x into (S, Cc), two nodes per packed operation: each half rounds
// like the scalar operation and x - y is fma(y, -1, x) (one rounding, as the
// subtraction), so the results are those of the scalar two-sum; x = 0 leaves
// (S, Cc) unchanged
__device__ __forceinline__ void two_sum2(float2 &S, float2 &Cc, float2 x)
{
    const float2 m1 = make_float2(-1.f, -1.f);
    const float2 t = __fadd2_rn(S, x);
    const float2 bpv = __ffma2_rn(S, m1, t);                       // t - S
    const float2 e1 = __ffma2_rn(__ffma2_rn(bpv, m1, t), m1, S);  // S - (t - bpv)
    const float2 e2 = __ffma2_rn(bpv, m1, x);                      // x - bpv
    Cc = __fadd2_rn(Cc, __fadd2_rn(e1, e2));
    S = t;
}

// MODE 0: Q(f,f), a CTA owns output cells D and an item (block c1, c2) reads
//         F16 tiles of cells c2 + D and the FP32 side tile of cells c1 + D;
//         per row acc[p] += f(c1+D, l1) G[(l1, p)].
// MODE 1: the adjoint g = J(f)^T v (block form of the VJP), a CTA owns
//         target cells T; an item is one of the two scatters of a block:
//           W  (pass 1, to the c1 side): G = f(c2+D) W,  D = T - c1,
//           W2 (pass 2, to the c2 side): G = f(c1+D) W2, D = T - c2,
//         (W2: the block's values with the roles of its two nodes swapped,
//         compacted to the nodes l2 of the block's second mask); the item's
//         c1/c2 fields hold ccell + (side cell - T) and ccell + (F16 cell -
//         T); the side tile is c = 2v/w at cells D, and per row each node l
//         of the mask gets sum_p c(D, p) G[(rank(l), p)].
// Both modes: an item's nch holds the block's node mask (low 27 bits) and the
// owner cells it serves (bits 27..30), chunk0 its first record group.
// The three roles walk the same units and items in the same order; their
// counters of items, W groups and (group, VDF tile) jobs run on across units.
template <int VB, int P, int MODE, bool MG>
__global__ void __launch_bounds__(T2_THREADS, 1) k_collide_tc2(const __grid_constant__ Tc2Launch L)
{
    constexpr int NDG = TC_ROWS / VB;
    constexpr int NG = t2_groups(P);
    extern __shared__ __align__(1024) unsigned char smem[];
    const int region = L.region;
    unsigned char *wring = smem;                      // T2_NSTW x T2_GREC
    unsigned char *slots = smem + T2_NSTW * T2_GREC;  // 2 item slots x 2 VDF tiles x region
    uint64_t *bars = reinterpret_cast<uint64_t *>(slots + 4 * region);
    uint64_t *w_full = bars, *w_empty = bars + T2_NSTW;
    uint64_t *s_full = w_empty + T2_NSTW, *s_empty = s_full + 2;
    uint64_t *c_full = s_empty + 2, *c_empty = c_full + 2;
    uint64_t *drain = c_empty + 4;
    uint64_t *uq_full = drain + 1, *uq_empty = uq_full + 2;  // unit queue
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(uq_empty + 2);
    volatile int *uq = reinterpret_cast<volatile int *>(tmem_slot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int total = L.ubase[L.ngrids];
    int *const err0 = L.g[0].err;
    // VDF tiles this CTA's units hold: its one unit's (one launch per set), or
    // the launch's (persistent: the same in every unit); the epilogue warps of
    // the other tile leave at once, as if the CTA had been launched without them
    const int nbw = L.counter ? L.tpcmax : (blockIdx.x < (unsigned)total ? t2_unit<MG>(L, blockIdx.x).nb2 : 1);
    if (threadIdx.x == 0) {
        for (int s = 0; s < T2_NSTW; s++) {
            mbar_init(&w_full[s], 1);
            mbar_init(&w_empty[s], 1);
        }
        for (int s = 0; s < 2; s++) {
            mbar_init(&s_full[s], 1);
            mbar_init(&s_empty[s], 1 + 4 * nbw);  // the MMA commit + the epilogue warps of the CTA's tiles
        }
        for (int s = 0; s < 2; s++) {
            mbar_init(&c_full[s], 1);
            mbar_init(&c_empty[s], 4);  // the epilogue warps of the job's tile
        }
        mbar_init(drain, 1);
        for (int s = 0; s < 2; s++) {
            mbar_init(&uq_full[s], 1);
            mbar_init(&uq_empty[s], 1 + 4 * nbw);  // the MMA thread + the epilogue warps of the CTA's tiles
        }
        fence_mbar_init();
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_slot))
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot;
    // zero the item slots once: the copies of an item skip cells outside the
    // grid, so rows of such cells read what the slot held before -- zeros or
    // finite values of earlier items, which the zero side factors of rows an
    // item does not serve turn into exact zeros
    for (int t = threadIdx.x; t < region / 4; t += blockDim.x)  // 4 slots of `region` bytes, 16 B per store
        reinterpret_cast<uint4 *>(slots)[t] = make_uint4(0u, 0u, 0u, 0u);
    fence_async_shared();  // visible to the tensor core and ordered before the copies
    if (warp >= 2) {
        // zero all 512 columns once (warps 2-5 the first 256, 6-9 the rest, each
        // its lane quarter): an item's last column group may be narrower than
        // the 32-column loads of the epilogue, whose extra columns then hold
        // zeros or finite values of earlier jobs, times a zero factor
        const float z[16] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        const uint32_t tq = tmem + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(((warp - 2) >> 2) * 256);
#pragma unroll 1
        for (int cz = 0; cz < 256; cz += 16) tmem_st16(tq + (uint32_t)cz, z);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();

    if (warp == 0) {
        // ---------------- producer ----------------
        if (lane == 0) {
            int q = 0, gw = 0;
            bool ok = true;
            const size_t tile = (size_t)VB * T2_K * 2;
            for (int k = 0; ok; k++) {
                int u = k == 0 ? (int)blockIdx.x : total;
                if (L.counter) {
                    // hand the next unit to the other roles (a unit >= total ends them)
                    const int slot = k & 1;
                    if (!mbar_wait(&uq_empty[slot], ((k >> 1) & 1) ^ 1, err0, L.wait_ns)) { ok = false; break; }
                    u = atomicAdd(L.counter, 1);
                    uq[slot] = u;
                    mbar_arrive(&uq_full[slot]);
                }
                if (u >= total) break;
                const T2Unit un = t2_unit<MG>(L, u);
                const Tc2Args &a = L.g[MG ? un.gi : 0];
                const int D0 = un.tile * NDG;
                for (int it = un.i0; it < un.i1; it++) {
                    const TcItem e = a.items[it];
                    const int s = q & 1;
                    if (!mbar_wait(&s_empty[s], ((q >> 1) & 1) ^ 1, a.err, L.wait_ns)) { ok = false; break; }
                    // f of cells c1 + D - ccell (FP32) and c2 + D - ccell (fp16
                    // tiles), D in the row tile, clipped to the grid
                    const int cs1 = e.c1 + D0 - a.ccell, cs2 = e.c2 + D0 - a.ccell;
                    const int lo1 = max(cs1, 0), hi1 = min(cs1 + NDG, a.Nc);
                    const int lo2 = max(cs2, 0), hi2 = min(cs2 + NDG, a.Nc);
                    {
                        int *hd = reinterpret_cast<int *>(slots + (size_t)(2 * s) * region + 2 * T2_ATILE +
                                                          NDG * P * VB * 4);
                        const unsigned msk = (unsigned)e.nch & 0x7ffffffu;
                        int k = 0;
                        for (int l = 0; l < P; l++)
                            if ((msk >> l) & 1u) hd[1 + k++] = l * VB;
                        hd[0] = k * P;
                        for (; k < P; k++) hd[1 + k] = -1;
                        hd[1 + P] = e.nch;
                    }
                    uint32_t tx = 0;
                    if (hi1 > lo1) tx += (uint32_t)(un.nb2 * (hi1 - lo1) * P * VB * 4);
                    if (hi2 > lo2) tx += (uint32_t)(un.nb2 * 2 * (hi2 - lo2) * tile);
                    if (tx) {
                        mbar_arrive_expect_tx(&s_full[s], tx);
                        for (int j = 0; j < un.nb2; j++) {
                            const int bt = un.bt0 + j;
                            unsigned char *reg = slots + (size_t)(2 * s + j) * region;
                            if (hi2 > lo2) {
                                const unsigned char *src = a.F16 + ((size_t)(2 * bt) * a.Nc + lo2) * tile;
                                const uint32_t nb = (uint32_t)((hi2 - lo2) * tile);
                                bulk_g2s(reg + (lo2 - cs2) * tile, src, nb, &s_full[s]);
                                bulk_g2s(reg + T2_ATILE + (lo2 - cs2) * tile, src + (size_t)a.Nc * tile, nb,
                                         &s_full[s]);
                            }
                            if (hi1 > lo1)
                                bulk_g2s(reg + 2 * T2_ATILE + (size_t)(lo1 - cs1) * P * VB * 4,
                                         a.F + ((size_t)bt * a.Nc + lo1) * P * VB, (uint32_t)((hi1 - lo1) * P * VB * 4),
                                         &s_full[s]);
                        }
                    } else {
                        mbar_arrive(&s_full[s]);
                    }
                    q++;
                    // the item's compacted record: groups from chunk0 & 0x3fffffff
                    // of W, or of W2 for the adjoint's pass to the c2 side
                    const int ngb = t2_item_groups<P>(e.nch);
                    const unsigned char *wrec =
                        ((MODE == 1 && (e.chunk0 >> 30)) ? a.W2 : a.W) + (size_t)(e.chunk0 & 0x3fffffff) * T2_GREC;
                    for (int g = 0; g < ngb; g++, gw++) {
                        const int st = gw % T2_NSTW;
                        if (!mbar_wait(&w_empty[st], ((gw / T2_NSTW) & 1) ^ 1, a.err, L.wait_ns)) {
                            ok = false;
                            break;
                        }
                        if (L.withhold && blockIdx.x == 0 && gw == 0) continue;  // the stage nothing completes
                        mbar_arrive_expect_tx(&w_full[st], T2_GREC);
                        bulk_g2s(wring + st * T2_GREC, wrec + (size_t)g * T2_GREC, T2_GREC, &w_full[st]);
                    }
                    if (!ok) break;
                }
            }
            if (!ok) {  // let the copies already issued land
                for (int j = gw > T2_NSTW ? gw - T2_NSTW : 0; j < gw; j++)
                    mbar_wait(&w_full[j % T2_NSTW], (j / T2_NSTW) & 1, err0, L.wait_ns);
                for (int j = q > 2 ? q - 2 : 0; j < q; j++) mbar_wait(&s_full[j & 1], (j >> 1) & 1, err0, L.wait_ns);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            // FP32 accumulator, fp16 A and B, both K-major, M = 128, N = 256;
            // an item's last group holds ncol - 256 (ngb-1) columns: its MMAs
            // use N rounded up to 16
            const uint32_t idesc = (1u << 4) | ((uint32_t)(T2_N >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
            int q = 0, gw = 0, J = 0;
            bool ok = true;
            for (int k = 0; ok; k++) {
                int u = k == 0 ? (int)blockIdx.x : total;
                if (L.counter) {
                    const int slot = k & 1;
                    if (!mbar_wait(&uq_full[slot], (k >> 1) & 1, err0, L.wait_ns)) { ok = false; break; }
                    u = uq[slot];
                    mbar_arrive(&uq_empty[slot]);
                }
                if (u >= total) break;
                const T2Unit un = t2_unit<MG>(L, u);
                int *const err = L.g[MG ? un.gi : 0].err;
                for (int it = un.i0; it < un.i1 && ok; it++) {
                    const int s = q & 1;
                    if (!mbar_wait(&s_full[s], (q >> 1) & 1, err, L.wait_ns)) { ok = false; break; }
                    const int ncol = *reinterpret_cast<const int *>(slots + (size_t)(2 * s) * region + 2 * T2_ATILE +
                                                                     NDG * P * VB * 4);
                    const int ngb = (ncol + T2_N - 1) / T2_N;
                    const int nlast = ((ncol - (ngb - 1) * T2_N) + 15) / 16 * 16;
                    const uint32_t idesc_last =
                        (1u << 4) | ((uint32_t)(nlast >> 3) << 17) | ((uint32_t)(TC_ROWS >> 4) << 24);
                    for (int g = 0; g < ngb && ok; g++, gw++) {
                        const int st = gw % T2_NSTW;
                        if (!mbar_wait(&w_full[st], (gw / T2_NSTW) & 1, err, L.wait_ns)) { ok = false; break; }
                        const uint64_t dWh = umma_desc(smem_u32(wring + st * T2_GREC), 128, 512);
                        const uint64_t dWl = umma_desc(smem_u32(wring + st * T2_GREC + T2_TILE), 128, 512);
                        const uint32_t id = g == ngb - 1 ? idesc_last : idesc;
                        for (int j = 0; j < un.nb2; j++, J++) {
                            const int cs = J & 1;
                            if (!mbar_wait(&c_empty[cs], ((J >> 1) & 1) ^ 1, err, L.wait_ns)) { ok = false; break; }
                            tc_fence_after();
                            unsigned char *reg = slots + (size_t)(2 * s + j) * region;
                            const uint64_t dAh = umma_desc(smem_u32(reg), 128, 512);
                            const uint64_t dAl = umma_desc(smem_u32(reg + T2_ATILE), 128, 512);
                            const uint32_t dacc = tmem + (uint32_t)(cs * T2_N);
#pragma unroll
                            for (int t = 0; t < T2_K / 16; t++) {  // K = 16 per instruction: 256 B along K
                                umma_f16(dacc, dAh + 16 * t, dWh + 16 * t, id, t ? 1u : 0u);
                                umma_f16(dacc, dAh + 16 * t, dWl + 16 * t, id, 1u);
                                umma_f16(dacc, dAl + 16 * t, dWh + 16 * t, id, 1u);
                            }
                            umma_commit(&c_full[cs]);
                        }
                        if (!ok) break;
                        umma_commit(&w_empty[st]);
                    }
                    if (!ok) break;
                    umma_commit(&s_empty[s]);
                    q++;
                }
            }
            // every MMA issued so far completes before tensor memory is freed
            umma_commit(drain);
            mbar_wait(drain, 0, err0, L.wait_ns);
        }
        __syncwarp();
    } else if ((warp - 2) / 4 < nbw) {
        // ---------------- epilogue ----------------
        // warp w serves VDF tile (w-2)/4 of every unit of the CTA
        const int j = (warp - 2) / 4, quarter = warp & 3, r = quarter * 32 + lane;
        const uint32_t tl = tmem + ((uint32_t)(quarter * 32) << 16);
        const int d = r / VB, v = r % VB;
        int q = 0, Jb = 0;  // items consumed; (group, VDF tile) jobs of the items before
        bool ok = true;
        for (int k = 0; ok; k++) {
            int u = k == 0 ? (int)blockIdx.x : total;
            if (L.counter) {
                const int slot = k & 1;
                if (!mbar_wait_warp(&uq_full[slot], (k >> 1) & 1, err0, L.wait_ns)) { ok = false; break; }
                u = uq[slot];
                __syncwarp();
                if (lane == 0) mbar_arrive(&uq_empty[slot]);
            }
            if (u >= total) break;
            int nb2, i0, i1;
            int *err;
            {
                const T2Unit un = t2_unit<MG>(L, u);
                nb2 = un.nb2;
                i0 = un.i0;
                i1 = un.i1;
                err = L.g[MG ? un.gi : 0].err;
            }
            // (sum, correction) per node, nodes (2i, 2i+1) in the halves of one
            // float2, so that the item folds run in packed FP32x2 operations
            constexpr int P2 = (P + 1) / 2;
            float2 S2[P2], Cc2[P2], acc2[MODE == 0 ? P2 : 1];
#pragma unroll
            for (int i = 0; i < P2; i++) {
                S2[i] = make_float2(0.f, 0.f);
                Cc2[i] = make_float2(0.f, 0.f);
            }
#pragma unroll
            for (int i = 0; i < (MODE == 0 ? P2 : 1); i++) acc2[i] = make_float2(0.f, 0.f);  // MODE 0: the item's sums
            for (int it = i0; it < i1; it++) {
                const int s = q & 1;
                if (!mbar_wait_warp(&s_full[s], (q >> 1) & 1, err, L.wait_ns)) { ok = false; break; }
                const float *f1s = reinterpret_cast<const float *>(slots + (size_t)(2 * s + j) * region + 2 * T2_ATILE) +
                                   d * P * VB + v;
                const int *hoff =
                    reinterpret_cast<const int *>(slots + (size_t)(2 * s) * region + 2 * T2_ATILE + NDG * P * VB * 4) +
                    1;
                const int nch = hoff[P];
                const bool valid = (nch >> (27 + d)) & 1;
                const unsigned msk = (unsigned)nch & 0x7ffffffu;
                const int nl = __popc(msk), ncol = nl * P, ngb = (ncol + T2_N - 1) / T2_N;
                // Columns n = jj*P + p, jj = the rank of a node of the item's mask.
                // MODE 0: side = f(c1 + D, l1) of the jj-th node l1 (its offset from
                //         the slot header; 0 past the mask's nodes),
                //         acc[p] += side * G[n].
                // MODE 1: side = c(D, p) (all P live), the sum over p of each jj is
                //         complete after its P consecutive columns and is kept in
                //         stg[jj] (local memory: its read index is the rank of a
                //         node); after the item each node l of the mask adds
                //         stg[rank(l)] into its (sum, correction).
                constexpr int NR = 3;  // MODE 1: interleaved partial sums over p (6 or 9 chains measured slower)
                float f1[P], stg[MODE == 1 ? P : 1], run[NR];
#pragma unroll
                for (int l = 0; l < P; l++) {
                    if constexpr (MODE == 1) {
                        f1[l] = f1s[l * VB];
                    } else {
                        // loaded before the column loop (the TMEM waits order all
                        // shared-memory loads, so loads inside it would stall); a
                        // row the item does not serve gets zero factors, so its
                        // columns add exact zeros
                        const int o = hoff[l];
                        f1[l] = (valid && o >= 0) ? f1s[o] : 0.f;
                    }
                }
                // one 32-column load per wait (two per wait, with the side factors
                // and sums live, would spill)
                constexpr int LW = 32;
#pragma unroll
                for (int g = 0; g < NG; g++) {
                    if (g >= ngb) break;
                    const int J = Jb + g * nb2 + j, cs = J & 1;
                    if (!mbar_wait_warp(&c_full[cs], (J >> 1) & 1, err, L.wait_ns)) { ok = false; break; }
                    tc_fence_after();
#pragma unroll
                    for (int hh = 0; hh < T2_N / LW; hh++) {
                        if (g * T2_N + LW * hh >= P * P || g * T2_N + LW * hh >= ncol) break;
                        uint32_t G[LW];
                        tmem_ld32_nowait(tl + (uint32_t)(cs * T2_N + LW * hh), G);
                        tmem_wait_ld32(G);
#pragma unroll
                        for (int i = 0; i < LW; i++) {
                            const int n = g * T2_N + LW * hh + i;
                            if (n < P * P) {
                                if constexpr (MODE == 0) {
                                    float &a = ((n % P) & 1) ? acc2[(n % P) / 2].y : acc2[(n % P) / 2].x;
                                    a = fmaf(f1[n / P], __uint_as_float(G[i]), a);
                                } else {
                                    // NR interleaved partial sums over p
                                    const int pp = n % P, rr = pp % NR;
                                    run[rr] = pp < NR ? f1[pp] * __uint_as_float(G[i])
                                                      : fmaf(f1[pp], __uint_as_float(G[i]), run[rr]);
                                    if (pp == P - 1) {
                                        float t = run[0];
#pragma unroll
                                        for (int k = 1; k < (P < NR ? P : NR); k++) t += run[k];
                                        stg[n / P] = t;
                                    }
                                }
                            }
                        }
                    }
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&c_empty[cs]);
                }
                if (!ok) break;
                Jb += ngb * nb2;
                __syncwarp();
                if (lane == 0) mbar_arrive(&s_empty[s]);  // this warp's reads of the slot are done
                if constexpr (MODE == 1) {
                    // after the slot is released: the node totals come from
                    // registers and local memory only
                    if (valid) {
                        // two-sum of the node totals into (sum, correction);
                        // nodes outside the mask add exact zeros
#pragma unroll
                        for (int i = 0; i < P2; i++) {
                            float x[2];
#pragma unroll
                            for (int e = 0; e < 2; e++) {
                                const int p = 2 * i + e;
                                x[e] = (p < P && ((msk >> p) & 1u)) ? stg[__popc(msk & ((1u << p) - 1u))] : 0.f;
                            }
                            two_sum2(S2[i], Cc2[i], make_float2(x[0], x[1]));
                        }
                    }
                }
                if constexpr (MODE == 0) {
                    // the item's total two-summed into (sum, correction); a row
                    // the item does not serve adds exact zeros (zero side factors)
#pragma unroll
                    for (int i = 0; i < P2; i++) {
                        two_sum2(S2[i], Cc2[i], acc2[i]);
                        acc2[i] = make_float2(0.f, 0.f);
                    }
                }
                q++;
            }
            if (!ok) continue;
            // the unit's sums into qacc; persistent launches first wait until the
            // same rows' previous block set is in
            const T2Unit un = t2_unit<MG>(L, u);
            const Tc2Args &a = L.g[MG ? un.gi : 0];
            int *flag = a.done ? a.done + ((size_t)un.tile * a.nbp + un.bp) * T2_EPI_WARPS + (warp - 2) : nullptr;
            if (flag) {
                bool fok = true;
                if (lane == 0) fok = flag_wait(flag, un.s, a.err, L.wait_ns);
                if (!__shfl_sync(0xffffffffu, fok ? 1 : 0, 0)) { ok = false; continue; }
            }
            const int D = un.tile * NDG + d, vdf = (un.bt0 + j) * VB + v;
            if (D < a.Nc && vdf < a.nvdf) {
                const double sc = MODE == 0 ? a.inv_scale[vdf] : 1.0;  // the adjoint scales in k_tc_vjp_final
#pragma unroll
                for (int p = 0; p < P; p++) {
                    double *dst = a.qacc + ((size_t)D * P + p) * a.NV + vdf;
                    const float sv = (p & 1) ? S2[p / 2].y : S2[p / 2].x, cv = (p & 1) ? Cc2[p / 2].y : Cc2[p / 2].x;
                    *dst += ((double)sv + (double)cv) * sc;
                }
            }
            if (flag) {
                __syncwarp();  // the warp's additions are ordered before lane 0's release
                if (lane == 0) st_release_gpu(flag, un.s + 1);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 1)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
}

// Block records of the collision operator, compacted to the nodes l1 each
// block uses: a mask per block (device pass over the pairs), the blocks'
// group offsets on the host, then the records.
static int tc2_prepare(Ctx *c)
{
    Layout &L = c->lay;
    if (L.tc2_W) return DGV_OK;
    const Grid &g = c->grid;
    int rc = tc_value_scale(c, &L.tc2_vscale);
    if (rc) return rc;
    const long long nb = L.nblocks;
    L.tc2_mask.assign(2 * (size_t)nb, 0u);
    L.tc2_goff.assign((size_t)nb + 1, 0);
    unsigned *d_mask = nullptr;
    long long *d_goff = nullptr;
    DGV_CUDA(c, cudaMalloc(&d_mask, sizeof(unsigned) * std::max<long long>(1, 2 * nb)));
    if (nb) {
        k_tc2_mask<<<(unsigned)nb, 128, 0, c->stream>>>(L.blk, (const double *)L.rows64, L.RD64, g.Nc, g.ccell, d_mask,
                                                         nb);
        DGV_CUDA(c, cudaGetLastError());
        DGV_CUDA(c, cudaMemcpyAsync(L.tc2_mask.data(), d_mask, sizeof(unsigned) * 2 * nb, cudaMemcpyDeviceToHost,
                                    c->stream));
        DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    }
    for (long long b = 0; b < nb; b++)
        L.tc2_goff[b + 1] = L.tc2_goff[b] + (__builtin_popcount(L.tc2_mask[b]) * g.P + T2_N - 1) / T2_N;
    const size_t bytes = (size_t)std::max<long long>(1, L.tc2_goff[nb]) * T2_GREC;
    cudaError_t e = cudaMalloc(&L.tc2_W, bytes);
    if (e != cudaSuccess || cudaMalloc(&d_goff, sizeof(long long) * (nb + 1)) != cudaSuccess) {
        cudaGetLastError();
        if (L.tc2_W) cudaFree(L.tc2_W);
        L.tc2_W = nullptr;
        cudaFree(d_mask);
        return set_err(c, DGV_ENOMEM, "tensor-core block form: no room for the block records");
    }
    DGV_CUDA(c, cudaMemcpyAsync(d_goff, L.tc2_goff.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice,
                                c->stream));
    if (nb)
        k_tc2_build<<<(unsigned)nb, 256, 0, c->stream>>>(L.blk, (const double *)L.rows64, L.RD64, g.P, g.Nc, g.ccell,
                                                          (float)L.tc2_vscale, (unsigned char *)L.tc2_W, 0, d_mask,
                                                          d_goff);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d_mask);
    cudaFree(d_goff);
    return DGV_OK;
}

// Block sets of about c->tc_set_mb MB of records, one launch each; a changed
// size drops the block-form work lists built for the old sets.
static void tc2_sets(Ctx *c)
{
    Layout &L = c->lay;
    if (L.tc2_set_mb == c->tc_set_mb && !L.tc2_sets.empty()) return;
    for (auto it = L.tc_lists.begin(); it != L.tc_lists.end();) {
        if (it->first >= 256) {
            for (void *p : it->second) cudaFree(p);
            L.tc_list_work.erase(it->first);
            L.tc_list_items.erase(it->first);
            it = L.tc_lists.erase(it);
        } else {
            ++it;
        }
    }
    // about tc_set_mb MB of the collision operator's (compacted) records per set
    L.tc2_sets.clear();
    L.tc2_sets.push_back(0);
    const long long per_set = std::max<long long>(1, ((long long)c->tc_set_mb << 20) / T2_GREC);
    long long acc = 0;
    for (long long b = 0; b < L.nblocks; b++) {
        acc += L.tc2_goff[b + 1] - L.tc2_goff[b];
        if (acc >= per_set && b + 1 < L.nblocks) {
            L.tc2_sets.push_back((int)(b + 1));
            acc = 0;
        }
    }
    if (L.tc2_sets.back() != (int)L.nblocks) L.tc2_sets.push_back((int)L.nblocks);
    L.tc2_set_mb = c->tc_set_mb;
    L.tc2_sets_adj.clear();
}

// The adjoint's launches: about tc_set_mb MB of records per launch counting
// both record sets its items read (W for the pass to the c1 side, W2 for
// the pass to the c2 side), so that a launch's records stay in L2 as the
// collision operator's do.  Built after tc2_sets and the adjoint's records.
static void tc2_sets_adjoint(Ctx *c)
{
    Layout &L = c->lay;
    if (!L.tc2_sets_adj.empty()) return;
    L.tc2_sets_adj.push_back(0);
    const long long per_set = std::max<long long>(1, ((long long)c->tc_set_mb << 20) / T2_GREC);
    long long acc = 0;
    for (long long b = 0; b < L.nblocks; b++) {
        acc += (L.tc2_goff[b + 1] - L.tc2_goff[b]) + (L.tc2_goff2[b + 1] - L.tc2_goff2[b]);
        if (acc >= per_set && b + 1 < L.nblocks) {
            L.tc2_sets_adj.push_back((int)(b + 1));
            acc = 0;
        }
    }
    if (L.tc2_sets_adj.back() != (int)L.nblocks) L.tc2_sets_adj.push_back((int)L.nblocks);
}

// the wait limit of the launches, and the one-shot test switch (DGV_OPT_TEST_WITHHOLD:
// CTA 0 of the first launch arms no copy for its first W stage, so the waits on
// that stage run out and the call reports DGV_ETIMEOUT)
static void tc2_wait_args(Ctx *c, Tc2Launch &Lh)
{
    Lh.wait_ns = wait_limit_ns(c);
    Lh.withhold = c->test_withhold ? 1 : 0;
    c->test_withhold = false;
}

// a persistent launch needs every unit to hold the same number of VDF tiles:
// the epilogue warps of a tile that some units lack would run ahead of the
// tensor-memory accumulators' phases (their parity could then not tell a
// later phase from a completed one)
static bool t2_uniform(const Tc2Args &a)
{
    return a.nbt <= a.tpc || a.nbt % a.tpc == 0;
}

// persistent launches: the order flags (row tile x VDF-tile pair x epilogue
// warp) and, after them, the unit counter
static size_t t2_flag_bytes(const Tc2Args &a)
{
    return sizeof(int) * ((size_t)a.ng * a.nbp * T2_EPI_WARPS + 1);
}

// bytes per VDF tile in an item slot: A hi, A lo, the FP32 side tile, the slot header
static int t2_region(int P, int VB)
{
    return (2 * T2_ATILE + (TC_ROWS / VB) * P * VB * 4 + T2_HDR + 1023) / 1024 * 1024;
}

static size_t t2_smem(int region)
{
    return (size_t)T2_NSTW * T2_GREC + 4 * (size_t)region + (2 * T2_NSTW + 17) * sizeof(uint64_t) + 16;
}

// the launch of a block-form kernel: one unit per CTA (grid = units), or
// persistent (grid = one CTA per SM, launched cooperatively so that all CTAs
// are resident at once: a CTA may wait for another's flag)
template <int VB, int P, int MODE, bool MG = false>
static int t2_launch(Ctx *c, const Tc2Launch &Lh, bool persistent, cudaStream_t stream)
{
    const int total = Lh.ubase[Lh.ngrids];
    if (total <= 0) return DGV_OK;
    const size_t smem = t2_smem(Lh.region);
    auto fn = k_collide_tc2<VB, P, MODE, MG>;
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (!persistent) {
        fn<<<(unsigned)total, T2_THREADS, smem, stream>>>(Lh);
        DGV_CUDA(c, cudaGetLastError());
        return DGV_OK;
    }
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.blockDim = dim3(T2_THREADS);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    {
        int nsm = 148, per_sm = 0;
        DGV_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
        DGV_CUDA(c, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, (const void *)fn, T2_THREADS, smem));
        if (per_sm < 1) return set_err(c, DGV_EUNSUP, "block form: the kernel does not fit on an SM");
        cfg.gridDim = dim3((unsigned)std::min<long long>(total, (long long)nsm * per_sm));
        attr[0].id = cudaLaunchAttributeCooperative;
        attr[0].val.cooperative = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    DGV_CUDA(c, cudaLaunchKernelEx(&cfg, fn, Lh));
    return DGV_OK;
}

// The block form's launches over the block sets of one grid: one launch per
// set (c->tc_persistent = 0, or a batch whose VDF-tile pairs do not all hold
// the same number of tiles), or one persistent launch over all sets, whose
// per-warp order flags (row tile x VDF-tile pair x epilogue warp) start at 0.
template <int VB, int P, int MODE = 0>
static int launch_tc2(Ctx *c, Tc2Args &a, const TcLists &tl, const std::vector<int> &sets, int region)
{
    Tc2Launch Lh;
    std::memset(&Lh, 0, sizeof(Lh));
    Lh.ngrids = 1;
    Lh.region = region;
    Lh.tpcmax = std::min(a.tpc, a.nbt);
    tc2_wait_args(c, Lh);
    const int nsets = (int)sets.size() - 1, per = a.nbp * a.ng;
    KTimer kt(c);
    if (c->tc_persistent && t2_uniform(a)) {
        const size_t fb = t2_flag_bytes(a);
        int rc = ensure_buffer(c, &c->d_tc2done, &c->tc2done_bytes, fb);
        if (rc) return rc;
        DGV_CUDA(c, cudaMemsetAsync(c->d_tc2done, 0, fb, c->stream));
        a.item_start = tl.item_start;
        a.tile_of = tl.tile_of;
        a.done = reinterpret_cast<int *>(c->d_tc2done);
        Lh.counter = a.done + (size_t)a.ng * a.nbp * T2_EPI_WARPS;
        Lh.g[0] = a;
        Lh.ubase[1] = nsets * per;
        if ((rc = t2_launch<VB, P, MODE>(c, Lh, true, c->stream))) return rc;
        kt.stop(1);
        count_launches(c, 1);
        return DGV_OK;
    }
    a.done = nullptr;
    Lh.ubase[1] = per;
    for (int s = 0; s < nsets; s++) {
        a.item_start = tl.item_start + (size_t)s * (a.ng + 1);
        a.tile_of = tl.tile_of + (size_t)s * a.ng;
        Lh.g[0] = a;
        int rc = t2_launch<VB, P, MODE>(c, Lh, false, c->stream);
        if (rc) return rc;
        Lh.withhold = 0;  // the test withholds in the first launch only
    }
    kt.stop(nsets);
    count_launches(c, nsets);
    return DGV_OK;
}

template <int P, int MODE = 0>
static int launch_tc2_vb(Ctx *c, Tc2Args &a, const TcLists &tl, int VB, const std::vector<int> &sets, int region)
{
    switch (VB) {
    case 128: return launch_tc2<128, P, MODE>(c, a, tl, sets, region);
    case 64: return launch_tc2<64, P, MODE>(c, a, tl, sets, region);
    default: return launch_tc2<32, P, MODE>(c, a, tl, sets, region);
    }
}

// the tuned launch choice of this batch class, if the context has one (and the
// caller set none of the options)
static void tc2_use_tuned(Ctx *c, int nvdf)
{
    if (!c->tc_autotune || c->tc_user_launch) return;
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32), nbt = (nvdf + VB - 1) / VB;
    auto it = c->tc_tuned.find(VB * 2 + (nbt > 1 ? 1 : 0));
    if (it == c->tc_tuned.end()) return;
    c->tc_tiles_per_cta = it->second.tiles;
    c->tc_set_mb = it->second.set_mb;
    c->tc_persistent = it->second.persistent;
}

// One block-form evaluation in three parts: tc2_begin (records, sets, work
// lists, buffers; f in the tile layouts; sums zeroed), the launches, tc2_end
// (FP64 sums / w, scale, projection).
struct Tc2Call {
    Tc2Args a;
    TcLists tl;
    Tc2PrepGrid prep;
    int VB = 0, region = 0;
};

// the f preparation of the grids of one launch (one CTA per VDF slot)
static int tc2_launch_prep(Ctx *c, const Tc2PrepGrid *gs, int n, cudaStream_t stream)
{
    Tc2PrepLaunch A;
    std::memset(&A, 0, sizeof(A));
    A.ngrids = n;
    for (int i = 0; i < n; i++) {
        A.g[i] = gs[i];
        A.vbase[i + 1] = A.vbase[i] + gs[i].NV;
    }
    k_tc2_prep<<<(unsigned)A.vbase[n], 256, 0, stream>>>(A);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 1);
    return DGV_OK;
}

// the final step (FP64 sums / w x scale into q) of the grids of one launch
static int tc2_launch_final(Ctx *c, const Tc2FinalGrid *gs, int n, cudaStream_t stream)
{
    Tc2FinalLaunch A;
    std::memset(&A, 0, sizeof(A));
    A.ngrids = n;
    for (int i = 0; i < n; i++) {
        A.g[i] = gs[i];
        A.ebase[i + 1] = A.ebase[i] + (long long)gs[i].nvdf * gs[i].N;
    }
    const long long tot = A.ebase[n];
    k_tc2_final<<<(unsigned)std::min<long long>((tot + 255) / 256, 148LL * 32), 256, 0, stream>>>(A);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 1);
    return DGV_OK;
}

// launch_prep = false: the caller launches the f preparation (k.prep) with
// those of other grids
static int tc2_begin(Ctx *c, const double *d_f, int nvdf, Tc2Call &k, cudaStream_t stream, bool launch_prep)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    int rc = tc2_prepare(c);
    if (rc) return rc;
    tc2_sets(c);
    rc = ensure_errflag(c);
    if (rc) return rc;
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32), NDG = TC_ROWS / VB;
    const int nbt = (nvdf + VB - 1) / VB, NV = nbt * VB, ng = (g.Nc + NDG - 1) / NDG;
    const size_t fbytes = (size_t)nbt * g.Nc * g.P * VB * sizeof(float);
    const size_t f16bytes = (size_t)nbt * 2 * g.Nc * VB * T2_K * 2;
    const size_t qbytes = (size_t)g.N * NV * sizeof(double);
    rc = ensure_buffer(c, &c->d_tcF, &c->tcF_bytes, fbytes + f16bytes + NV * sizeof(double));
    if (rc) return rc;
    rc = ensure_buffer(c, &c->d_tcQ, &c->tcQ_bytes, qbytes);
    if (rc) return rc;
    {
        std::vector<int> first, count;
        rc = tc_work_lists(c, NDG, 256 + NDG, L.tc2_sets, first, count, &k.tl, 1);
        if (rc) return rc;
    }
    float *F = reinterpret_cast<float *>(c->d_tcF);
    unsigned char *F16 = reinterpret_cast<unsigned char *>(c->d_tcF) + fbytes;
    double *inv = reinterpret_cast<double *>(F16 + f16bytes);
    k.prep = Tc2PrepGrid{d_f, F, F16, inv, g.N, nvdf, NV, g.Nc, g.P, VB, 2, 1.0 / L.tc2_vscale};
    DGV_CUDA(c, cudaMemsetAsync(c->d_tcQ, 0, qbytes, stream));
    if (launch_prep && (rc = tc2_launch_prep(c, &k.prep, 1, stream))) return rc;
    Tc2Args &a = k.a;
    std::memset(&a, 0, sizeof(a));
    a.F = F; a.F16 = F16; a.W = (const unsigned char *)L.tc2_W; a.W2 = nullptr; a.items = k.tl.items;
    a.qacc = c->d_tcQ; a.inv_scale = inv; a.err = c->d_err;
    a.Nc = g.Nc; a.ccell = g.ccell; a.NV = NV; a.nvdf = nvdf; a.nbt = nbt;
    a.tpc = c->tc_tiles_per_cta;
    a.nbp = (nbt + a.tpc - 1) / a.tpc;
    a.ng = ng;
    k.VB = VB;
    k.region = t2_region(g.P, VB);
    // the order flags of persistent launches, allocated here on every call so
    // that a captured call (graphs of RK steps and of mixed-grid groups) finds
    // them in place
    return ensure_buffer(c, &c->d_tc2done, &c->tc2done_bytes, t2_flag_bytes(a));
}

static Tc2FinalGrid tc2_final_of(Ctx *c, double *d_q, int nvdf, int NV, double scale)
{
    return Tc2FinalGrid{c->d_tcQ, c->d_nwt, d_q, c->grid.N, nvdf, NV, scale};
}

static int tc2_end(Ctx *c, double *d_q, int nvdf, int NV, double scale)
{
    const Tc2FinalGrid fg = tc2_final_of(c, d_q, nvdf, NV, scale);
    int rc = tc2_launch_final(c, &fg, 1, c->stream);
    if (rc) return rc;
    if (c->project) return project_device(c, d_q, nvdf);
    return DGV_OK;
}

static int collide_tc2_body(Ctx *c, const double *d_f, double *d_q, int nvdf, double scale)
{
    Tc2Call k;
    int rc = tc2_begin(c, d_f, nvdf, k, c->stream, true);
    if (rc) return rc;
    const std::vector<int> &sets = c->lay.tc2_sets;
    rc = c->grid.P == 27 ? launch_tc2_vb<27>(c, k.a, k.tl, k.VB, sets, k.region)
                         : launch_tc2_vb<8>(c, k.a, k.tl, k.VB, sets, k.region);
    if (rc) return rc;
    return tc2_end(c, d_q, nvdf, k.a.NV, scale);
}

// Mixed-grid batch (dgv_collide_group) in one persistent launch: members of
// the block form with the same nodes per cell and VDF tile size (at most
// T2_MAXG of them).  On the origin stream: one launch prepares every
// member's f tiles, the persistent launch serves every member's units (grid
// after grid, each in set order with its own order flags), one launch writes
// every member's Q; a member's conservation projection, if on, runs on its
// own stream (after fork2; join[n + i] brings it back).  The members' tuned
// launch choices (VDF tiles per CTA, records per launch) are kept.
int collide_tc2_group(Ctx *const *cs, const double *const *f, double *const *q, const int *nb, int n,
                      cudaStream_t origin, cudaEvent_t fork2, const cudaEvent_t *join)
{
    Ctx *c0 = cs[0];
    if (n < 1 || n > T2_MAXG) return set_err(c0, DGV_EUNSUP, "collide_group: persistent launch serves 1-4 grids");
    const int P = cs[0]->grid.P, VB = nb[0] > 64 ? 128 : (nb[0] > 32 ? 64 : 32);
    for (int i = 0; i < n; i++) {
        const int VBi = nb[i] > 64 ? 128 : (nb[i] > 32 ? 64 : 32);
        if (cs[i]->grid.P != P || (P != 27 && P != 8) || cs[i]->tc_form != 2 || VBi != VB || !cs[i]->lay.tc2_W)
            return set_err(c0, DGV_EUNSUP, "collide_group: members differ in nodes per cell, form or VDF tile");
    }
    for (int i = 0; i < n; i++) tc2_use_tuned(cs[i], nb[i]);
    Tc2Launch Lh;
    std::memset(&Lh, 0, sizeof(Lh));
    Lh.ngrids = n;
    // every unit of the launch must hold the same number of VDF tiles (checked
    // before any work is queued)
    for (int i = 0; i < n; i++) {
        Tc2Args t;
        std::memset(&t, 0, sizeof(t));
        t.nbt = (nb[i] + VB - 1) / VB;
        t.tpc = cs[i]->tc_tiles_per_cta;
        const int tpm = std::min(t.tpc, t.nbt);
        if (!t2_uniform(t) || (i > 0 && tpm != Lh.tpcmax))
            return set_err(c0, DGV_EUNSUP, "collide_group: the members' units hold different numbers of VDF tiles");
        Lh.tpcmax = tpm;
    }
    tc2_wait_args(c0, Lh);
    int units = 0;
    std::vector<int> NVs(n);
    std::vector<Tc2PrepGrid> preps(n);
    for (int i = 0; i < n; i++) {
        Ctx *c = cs[i];
        Tc2Call k;
        int rc = tc2_begin(c, f[i], nb[i], k, origin, false);
        if (rc) return rc;
        DGV_CUDA(c, cudaMemsetAsync(c->d_tc2done, 0, t2_flag_bytes(k.a), origin));
        k.a.item_start = k.tl.item_start;
        k.a.tile_of = k.tl.tile_of;
        k.a.done = reinterpret_cast<int *>(c->d_tc2done);
        if (i == 0) Lh.counter = k.a.done + (size_t)k.a.ng * k.a.nbp * T2_EPI_WARPS;  // the launch's unit counter
        Lh.g[i] = k.a;
        Lh.region = k.region;
        Lh.ubase[i] = units;
        units += ((int)c->lay.tc2_sets.size() - 1) * k.a.nbp * k.a.ng;
        NVs[i] = k.a.NV;
        preps[i] = k.prep;
    }
    {
        const int rc = tc2_launch_prep(c0, preps.data(), n, origin);
        if (rc) return rc;
    }
    Lh.ubase[n] = units;
    int rc;
    if (n > 1) {
        switch (VB) {
        case 128: rc = P == 27 ? t2_launch<128, 27, 0, true>(c0, Lh, true, origin)
                               : t2_launch<128, 8, 0, true>(c0, Lh, true, origin); break;
        case 64: rc = P == 27 ? t2_launch<64, 27, 0, true>(c0, Lh, true, origin)
                              : t2_launch<64, 8, 0, true>(c0, Lh, true, origin); break;
        default: rc = P == 27 ? t2_launch<32, 27, 0, true>(c0, Lh, true, origin)
                              : t2_launch<32, 8, 0, true>(c0, Lh, true, origin); break;
        }
    } else {
        switch (VB) {
        case 128: rc = P == 27 ? t2_launch<128, 27, 0>(c0, Lh, true, origin)
                               : t2_launch<128, 8, 0>(c0, Lh, true, origin); break;
        case 64: rc = P == 27 ? t2_launch<64, 27, 0>(c0, Lh, true, origin)
                              : t2_launch<64, 8, 0>(c0, Lh, true, origin); break;
        default: rc = P == 27 ? t2_launch<32, 27, 0>(c0, Lh, true, origin)
                              : t2_launch<32, 8, 0>(c0, Lh, true, origin); break;
        }
    }
    if (rc) return rc;
    count_launches(c0, 1);
    std::vector<Tc2FinalGrid> finals(n);
    for (int i = 0; i < n; i++) finals[i] = tc2_final_of(cs[i], q[i], nb[i], NVs[i], 1.0);
    if ((rc = tc2_launch_final(c0, finals.data(), n, origin))) return rc;
    // each member's conservation projection, if it has it on, on its stream
    DGV_CUDA(c0, cudaEventRecord(fork2, origin));
    for (int i = 0; i < n; i++) {
        Ctx *c = cs[i];
        if (!c->project) continue;
        if (c->stream != origin) DGV_CUDA(c, cudaStreamWaitEvent(c->stream, fork2, 0));
        if ((rc = project_device(c, q[i], nb[i]))) return rc;
        if (c->stream != origin) {
            DGV_CUDA(c, cudaEventRecord(join[n + i], c->stream));
            DGV_CUDA(c0, cudaStreamWaitEvent(origin, join[n + i], 0));
        }
    }
    return DGV_OK;
}

// The block form's launch choices, tuned on the first evaluation of each
// batch class (VDF tile size; one or several VDF tiles): VDF tiles per CTA (two
// let a block's records cross from L2 once per 256 rows, one gives twice the
// CTAs), block records per launch (the records one launch streams should stay
// in L2 while all its CTAs read them) and one launch per set or one persistent
// launch (no tail of short CTAs at the end of each set).  Per records size one
// evaluation warms up (work lists), then each choice is evaluated once, timed
// with CUDA events on the context stream; the fastest is kept for the context.
// Not while the stream is being captured (the current choice serves), and not
// when the caller set any of the three options.
static int tc2_autotune(Ctx *c, const double *d_f, double *d_q, int nvdf, double scale)
{
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32);
    const int nbt = (nvdf + VB - 1) / VB;
    const int key = VB * 2 + (nbt > 1 ? 1 : 0);
    auto it = c->tc_tuned.find(key);
    if (it != c->tc_tuned.end()) {
        c->tc_tiles_per_cta = it->second.tiles;
        c->tc_set_mb = it->second.set_mb;
        c->tc_persistent = it->second.persistent;
        return DGV_OK;
    }
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    DGV_CUDA(c, cudaStreamIsCapturing(c->stream, &cap));
    if (cap != cudaStreamCaptureStatusNone) return DGV_OK;
    const bool kt = c->ktiming;
    const long long kt_all = c->kt_all;
    c->ktiming = false;
    // records per launch up to 48 MB: with the f tiles and the FP64
    // accumulators a launch touches (~84 MB at 27^3 x 256), its working set
    // then (nearly) stays in the 126 MB L2; 96 MB sets ran as fast but read
    // their records ~10x from DRAM (measured)
    const int tiles[2] = {2, 1}, mbs[2] = {24, 48};
    float best_ms = 1e30f;
    Ctx::TcChoice best{c->tc_tiles_per_cta, c->tc_set_mb, c->tc_persistent};
    int rc = DGV_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DGV_CUDA(c, cudaEventCreate(&e0));
    DGV_CUDA(c, cudaEventCreate(&e1));
    for (int mb : mbs) {
        c->tc_set_mb = mb;
        c->tc_tiles_per_cta = 2;
        c->tc_persistent = 0;
        if ((rc = collide_tc2_body(c, d_f, d_q, nvdf, scale))) break;  // warm-up: sets and work lists
        for (int t : tiles) {
            if (t > 1 && nbt < 2) continue;
            const bool uniform = nbt <= t || nbt % t == 0;  // else persistent falls back to per-set launches
            for (int pe = 0; pe < (uniform ? 2 : 1); pe++) {
                c->tc_tiles_per_cta = t;
                c->tc_persistent = pe;
                cudaEventRecord(e0, c->stream);
                if ((rc = collide_tc2_body(c, d_f, d_q, nvdf, scale))) break;
                cudaEventRecord(e1, c->stream);
                if (cudaEventSynchronize(e1) != cudaSuccess) {
                    rc = set_err(c, DGV_ECUDA, "autotune: event failed");
                    break;
                }
                if ((rc = check_errflag(c))) break;
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best_ms) {
                    best_ms = ms;
                    best = Ctx::TcChoice{t, mb, pe};
                }
            }
            if (rc) break;
        }
        if (rc) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    c->ktiming = kt;
    c->kt_all = kt_all;
    c->tc_tiles_per_cta = best.tiles;
    c->tc_set_mb = best.set_mb;
    c->tc_persistent = best.persistent;
    if (rc) return rc;
    c->tc_tuned[key] = best;
    return DGV_OK;
}

static int collide_tc2_device(Ctx *c, const double *d_f, double *d_q, int nvdf, double scale)
{
    if (c->tc_autotune && !c->tc_user_launch) {
        const int rc = tc2_autotune(c, d_f, d_q, nvdf, scale);
        if (rc) return rc;
    }
    return collide_tc2_body(c, d_f, d_q, nvdf, scale);
}

// ----------------------------------------------------------------------------
// Block-form adjoint (VJP): g = J(f)^T v for a batch, on the tensor cores.
// With c_i = 2 v_i / w_i and Q_i = (2/w_i) sum_j A_j f(a_j) f(b_j), the
// adjoint of collision_mod.f90:213-216 scatters c_i A_j f(b_j) to a_j and
// c_i A_j f(a_j) to b_j.  Per block and output cell D these are
//   g(c1+D, l1) += sum_p c(D,p) G1[(D,b), (p,l1)], G1 = F2 W1 (the forward's
//                  product, columns reordered p-major),
//   g(c2+D, l2) += sum_p c(D,p) G2[(D,b), (p,l2)], G2 = F1 W2 (the block's
//                  values with the two nodes' roles swapped),
// so the kernel is the forward's with target-cell ownership (MODE 1).

// per-VDF power-of-two scale of c = 2 v / w (max |c| -> [32, 64)) and the
// scaled FP32 copy in the layout of F; inv_c[v] = the inverse scale
__global__ void k_tc_cprep(const double *vv, const double *w, long long N, int nvdf, float *C, double *inv_c, int Nc,
                           int P, int VB)
{
    const int v = blockIdx.x;
    __shared__ double red[32];
    double m = 0.0;
    if (v < nvdf)
        for (long long i = threadIdx.x; i < N; i += blockDim.x) m = fmax(m, fabs(2.0 * vv[(size_t)v * N + i] / w[i]));
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
        frexp(m, &e);
        e = 6 - e;
    }
    const double sc = ldexp(1.0, e);
    if (threadIdx.x == 0) inv_c[v] = ldexp(1.0, -e);
    const int bt = v / VB, lb = v % VB;
    for (long long i = threadIdx.x; i < N; i += blockDim.x) {
        const int cell = (int)(i / P), l = (int)(i - (long long)cell * P);
        const double x = v < nvdf ? 2.0 * vv[(size_t)v * N + i] / w[i] * sc : 0.0;
        C[(((size_t)bt * Nc + cell) * P + l) * VB + lb] = (float)x;
    }
}

// g[v][i] = gacc[i*NV + v] * inv_f[v] * inv_c[v]
__global__ void k_tc_vjp_final(const double *gacc, const double *inv_f, const double *inv_c, double *g, long long N,
                               int nvdf, int NV)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nvdf * N) return;
    const int v = (int)(idx % nvdf);
    const long long i = idx / nvdf;
    g[(size_t)v * N + i] = gacc[i * NV + v] * inv_f[v] * inv_c[v];
}

// the adjoint's second record set W2 (arrangement 1 of k_tc2_build, compacted
// to the blocks' masks of nodes l2), built on the first adjoint call with the
// value scale of W; the pass to the c1 side reads W itself
static int tc2_prepare_adjoint(Ctx *c)
{
    Layout &L = c->lay;
    if (L.tc2_Wv) return DGV_OK;
    const Grid &g = c->grid;
    const long long nb = L.nblocks;
    L.tc2_goff2.assign((size_t)nb + 1, 0);
    for (long long b = 0; b < nb; b++)
        L.tc2_goff2[b + 1] = L.tc2_goff2[b] + (__builtin_popcount(L.tc2_mask[nb + b]) * g.P + T2_N - 1) / T2_N;
    unsigned *d_mask = nullptr;
    long long *d_goff = nullptr;
    cudaError_t e = cudaMalloc(&L.tc2_Wv, (size_t)std::max<long long>(1, L.tc2_goff2[nb]) * T2_GREC);
    if (e != cudaSuccess || cudaMalloc(&d_mask, sizeof(unsigned) * std::max<long long>(1, nb)) != cudaSuccess ||
        cudaMalloc(&d_goff, sizeof(long long) * (nb + 1)) != cudaSuccess) {
        cudaGetLastError();
        if (L.tc2_Wv) cudaFree(L.tc2_Wv);
        if (d_mask) cudaFree(d_mask);
        L.tc2_Wv = nullptr;
        return set_err(c, DGV_ENOMEM, "tensor-core adjoint: no room for its block records");
    }
    DGV_CUDA(c, cudaMemcpyAsync(d_mask, L.tc2_mask.data() + nb, sizeof(unsigned) * nb, cudaMemcpyHostToDevice,
                                c->stream));
    DGV_CUDA(c, cudaMemcpyAsync(d_goff, L.tc2_goff2.data(), sizeof(long long) * (nb + 1), cudaMemcpyHostToDevice,
                                c->stream));
    if (nb)
        k_tc2_build<<<(unsigned)nb, 256, 0, c->stream>>>(L.blk, (const double *)L.rows64, L.RD64, g.P, g.Nc, g.ccell,
                                                          (float)L.tc2_vscale, (unsigned char *)L.tc2_Wv, 1, d_mask,
                                                          d_goff);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d_mask);
    cudaFree(d_goff);
    return DGV_OK;
}

static int vjp_tc_body(Ctx *c, const double *d_f, const double *d_v, double *d_g, int nvdf)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    if (!L.blk) return set_err(c, DGV_ESTATE, "vjp: no A-arrays loaded");
    if (g.P != 27 && g.P != 8)
        return set_err(c, DGV_EUNSUP, "tensor-core adjoint: grids of 8 or 27 nodes per cell");
    if (nvdf < 1) return set_err(c, DGV_EINVAL, "vjp: batch must hold at least one VDF");
    int rc = tc2_prepare(c);
    if (rc) return rc;
    if ((rc = tc2_prepare_adjoint(c))) return rc;
    tc2_sets(c);
    tc2_sets_adjoint(c);
    if ((rc = ensure_errflag(c))) return rc;
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32), NDG = TC_ROWS / VB;
    const int nbt = (nvdf + VB - 1) / VB, NV = nbt * VB, ng = (g.Nc + NDG - 1) / NDG;
    const size_t fbytes = (size_t)nbt * g.Nc * g.P * VB * sizeof(float);
    const size_t f16bytes = (size_t)nbt * 2 * g.Nc * VB * T2_K * 2;
    const size_t gbytes = (size_t)g.N * NV * sizeof(double);
    rc = ensure_buffer(c, &c->d_tcF, &c->tcF_bytes, 2 * fbytes + f16bytes + 2 * NV * sizeof(double));
    if (rc) return rc;
    rc = ensure_buffer(c, &c->d_tcQ, &c->tcQ_bytes, gbytes);
    if (rc) return rc;
    TcLists tl;
    {
        std::vector<int> first, count;
        rc = tc_work_lists(c, NDG, 512 + NDG, L.tc2_sets_adj, first, count, &tl, 2);
        if (rc) return rc;
    }
    float *F = reinterpret_cast<float *>(c->d_tcF);
    unsigned char *F16 = reinterpret_cast<unsigned char *>(c->d_tcF) + fbytes;
    float *Cf = reinterpret_cast<float *>(F16 + f16bytes);
    double *inv_f = reinterpret_cast<double *>(reinterpret_cast<unsigned char *>(Cf) + fbytes);
    double *inv_c = inv_f + NV;
    {
        const Tc2PrepGrid pg{d_f, F, F16, inv_f, g.N, nvdf, NV, g.Nc, g.P, VB, 1, 1.0 / L.tc2_vscale};
        if ((rc = tc2_launch_prep(c, &pg, 1, c->stream))) return rc;
    }
    k_tc_cprep<<<NV, 256, 0, c->stream>>>(d_v, c->d_nwt, g.N, nvdf, Cf, inv_c, g.Nc, g.P, VB);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaMemsetAsync(c->d_tcQ, 0, gbytes, c->stream));
    Tc2Args a;
    std::memset(&a, 0, sizeof(a));
    a.F = Cf; a.F16 = F16; a.W = (const unsigned char *)L.tc2_W; a.W2 = (const unsigned char *)L.tc2_Wv;
    a.items = tl.items; a.qacc = c->d_tcQ; a.inv_scale = nullptr;
    a.err = c->d_err; a.Nc = g.Nc; a.ccell = g.ccell; a.NV = NV; a.nvdf = nvdf; a.nbt = nbt;
    a.tpc = c->tc_tiles_per_cta;
    a.nbp = (nbt + a.tpc - 1) / a.tpc;
    a.ng = ng;
    const int region = t2_region(g.P, VB);
    rc = g.P == 27 ? launch_tc2_vb<27, 1>(c, a, tl, VB, L.tc2_sets_adj, region)
                   : launch_tc2_vb<8, 1>(c, a, tl, VB, L.tc2_sets_adj, region);
    if (rc) return rc;
    const long long tot = (long long)nvdf * g.N;
    k_tc_vjp_final<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->d_tcQ, inv_f, inv_c, d_g, g.N, nvdf, NV);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 2);  // k_tc_cprep, k_tc_vjp_final (k_tc2_prep counted above)
    return DGV_OK;
}

// The adjoint uses the collision operator's tuned VDF tiles per CTA and
// records per launch (its sets hold that many MB of W and W2 records
// together); one launch per set or one persistent launch is chosen on its
// own first call per batch class (evaluated once each after a warm-up, CUDA
// events on the context stream), unless the caller set DGV_OPT_TCPERSIST.
int vjp_tc_device(Ctx *c, const double *d_f, const double *d_v, double *d_g, int nvdf)
{
    tc2_use_tuned(c, nvdf);
    if (!c->tc_autotune || c->tc_user_launch) return vjp_tc_body(c, d_f, d_v, d_g, nvdf);
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32), nbt = (nvdf + VB - 1) / VB;
    const int key = VB * 2 + (nbt > 1 ? 1 : 0);
    const int saved = c->tc_persistent;
    int pers = 0, rc = DGV_OK;
    auto it = c->tc_tuned_adj.find(key);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    DGV_CUDA(c, cudaStreamIsCapturing(c->stream, &cap));
    if (it != c->tc_tuned_adj.end()) {
        pers = it->second;
    } else if (cap == cudaStreamCaptureStatusNone) {
        const bool kt = c->ktiming;
        const long long kt_all = c->kt_all;
        c->ktiming = false;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        DGV_CUDA(c, cudaEventCreate(&e0));
        DGV_CUDA(c, cudaEventCreate(&e1));
        float best = 1e30f;
        c->tc_persistent = 0;
        rc = vjp_tc_body(c, d_f, d_v, d_g, nvdf);  // warm-up: adjoint records, sets, work lists
        for (int pe = 0; pe < 2 && !rc; pe++) {
            c->tc_persistent = pe;
            cudaEventRecord(e0, c->stream);
            if ((rc = vjp_tc_body(c, d_f, d_v, d_g, nvdf))) break;
            cudaEventRecord(e1, c->stream);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                rc = set_err(c, DGV_ECUDA, "autotune: event failed");
                break;
            }
            if ((rc = check_errflag(c))) break;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) { best = ms; pers = pe; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c->ktiming = kt;
        c->kt_all = kt_all;
        if (rc) { c->tc_persistent = saved; return rc; }
        c->tc_tuned_adj[key] = pers;
    }
    c->tc_persistent = pers;
    rc = vjp_tc_body(c, d_f, d_v, d_g, nvdf);
    c->tc_persistent = saved;
    return rc;
}

template <int VB>
static int launch_tc(Ctx *c, TcArgs &a, const TcLists &tl, int ng)
{
    const size_t smem = (size_t)a.off_f + 2 * (size_t)a.fslot + (2 * TC_NSTB + 2 * TC_NA + 10) * sizeof(uint64_t) + 16;
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)k_collide_tc<VB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)smem));
    const Layout &L = c->lay;
    KTimer kt(c);
    for (size_t s = 0; s + 1 < L.tc_sets.size(); s++) {
        a.item_start = tl.item_start + s * (ng + 1);
        a.tile_of = tl.tile_of + s * ng;
        k_collide_tc<VB><<<(unsigned)(a.nbt * ng), TC_THREADS, smem, c->stream>>>(a);
        DGV_CUDA(c, cudaGetLastError());
    }
    kt.stop((long long)L.tc_sets.size() - 1);
    count_launches(c, (long long)L.tc_sets.size() - 1);
    return DGV_OK;
}

// Work plan of one tensor-core evaluation of nvdf VDFs in the current form:
// kernel launches, work items (block x row tile, or chunk x row tile) summed
// over the VDF tiles, and the FLOPs the MMAs issue (dense tiles, all three
// split products).  Builds the records and lists if they do not exist yet.
int tc_plan(Ctx *c, int nvdf, long long *launches, long long *items, double *flop)
{
    const Grid &g = c->grid;
    Layout &L = c->lay;
    if (!L.blk) return set_err(c, DGV_ESTATE, "tc_plan: no A-arrays loaded");
    if (g.P > 32 || nvdf < 1) return set_err(c, DGV_EINVAL, "tc_plan: no tensor-core plan for this grid or batch");
    const int VB = nvdf > 64 ? 128 : (nvdf > 32 ? 64 : 32), NDG = TC_ROWS / VB;
    const long long nbt = (nvdf + VB - 1) / VB;
    TcLists tl;
    int rc;
    bool block = c->tc_form == 2 && (g.P == 27 || g.P == 8);
    if (block && (rc = tc2_prepare(c))) {
        if (rc != DGV_ENOMEM) return rc;
        c->err.clear();
        block = false;  // as collide_tc_device: the chunk form serves
    }
    if (block) {
        if (c->tc_autotune && !c->tc_user_launch) {  // the choice tuned for this batch class, if any
            auto it = c->tc_tuned.find(VB * 2 + (nbt > 1 ? 1 : 0));
            if (it != c->tc_tuned.end()) {
                c->tc_tiles_per_cta = it->second.tiles;
                c->tc_set_mb = it->second.set_mb;
                c->tc_persistent = it->second.persistent;
            }
        }
        tc2_sets(c);
        std::vector<int> first, count;
        if ((rc = tc_work_lists(c, NDG, 256 + NDG, L.tc2_sets, first, count, &tl, 1))) return rc;
        // per item and VDF tile: 2 K steps x 3 split products over its issued columns
        const long long cols = L.tc_list_work[256 + NDG];
        const int tpc = c->tc_tiles_per_cta;
        const bool uniform = nbt <= tpc || nbt % tpc == 0;
        *launches = c->tc_persistent && uniform ? 1 : (long long)L.tc2_sets.size() - 1;
        *items = L.tc_list_items[256 + NDG] * nbt;
        *flop = (double)cols * nbt * 6.0 * 2.0 * TC_ROWS * 16;
    } else {
        if ((rc = tc_prepare(c))) return rc;
        if ((rc = tc_lists(c, NDG, &tl))) return rc;
        const long long w = L.tc_list_work[NDG];
        *launches = (long long)L.tc_sets.size() - 1;
        *items = w * nbt;  // chunk x row tile
        *flop = (double)w * nbt * 4.0 * 2.0 * TC_ROWS * 16 * (64 + 32);
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
    if (c->tc_form == 2 && (g.P == 27 || g.P == 8)) {
        // the block records need ~2x the room of the chunk records: when they
        // do not fit, the chunk form serves the call
        const int rc2 = collide_tc2_device(c, d_f, d_q, nvdf, scale);
        if (rc2 != DGV_ENOMEM || L.tc2_W) return rc2;
        c->err.clear();
    }
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
    TcLists tl;
    rc = tc_lists(c, NDG, &tl);
    if (rc) return rc;
    float *F = reinterpret_cast<float *>(c->d_tcF);
    double *inv = reinterpret_cast<double *>(reinterpret_cast<char *>(c->d_tcF) + fbytes);
    k_tc_fprep<<<NV, 256, 0, c->stream>>>(d_f, g.N, nvdf, 1.0 / L.tc_vscale, F, inv, g.Nc, g.P, VB, 2);
    DGV_CUDA(c, cudaGetLastError());
    DGV_CUDA(c, cudaMemsetAsync(c->d_tcQ, 0, qbytes, c->stream));
    TcArgs a;
    a.F = F; a.V = (const unsigned char *)L.tc_V; a.items = tl.items; a.item_start = nullptr; a.tile_of = nullptr;
    a.qacc = c->d_tcQ; a.inv_scale = inv; a.err = c->d_err;
    a.Nc = g.Nc; a.P = g.P; a.ccell = g.ccell; a.NV = NV; a.nvdf = nvdf; a.nbt = nbt;
    a.off_f = 2 * TC_NA * TC_ATILE + TC_NSTB * TC_REC;  // 16-byte aligned
    a.fslot = 2 * NDG * g.P * VB * (int)sizeof(float);  // both sides of one block
    switch (VB) {
    case 128: rc = launch_tc<128>(c, a, tl, ng); break;
    case 64: rc = launch_tc<64>(c, a, tl, ng); break;
    default: rc = launch_tc<32>(c, a, tl, ng); break;
    }
    if (rc) return rc;
    long long tot = (long long)nvdf * g.N;
    k_tc_final<<<(unsigned)((tot + 255) / 256), 256, 0, c->stream>>>(c->d_tcQ, c->d_nwt, d_q, g.N, nvdf, NV, scale);
    DGV_CUDA(c, cudaGetLastError());
    count_launches(c, 2);  // k_tc_fprep, k_tc_final
    if (c->project) return project_device(c, d_q, nvdf);
    return DGV_OK;
}

}  // namespace dgv

extern "C" int dgv_tc_plan(dgv_ctx *ctx, int32_t nvdf, int64_t *launches, int64_t *items, double *tensor_flop)
{
    if (!ctx) return DGV_EINVAL;
    dgv::Ctx *c = &ctx->c;
    c->err.clear();
    DGV_CUDA(c, cudaSetDevice(c->device));
    long long l = 0, it = 0;
    double fl = 0.0;
    int rc = dgv::tc_plan(c, nvdf, &l, &it, &fl);
    if (rc) return rc;
    if (launches) *launches = l;
    if (items) *items = it;
    if (tensor_flop) *tensor_flop = fl;
    return DGV_OK;
}
