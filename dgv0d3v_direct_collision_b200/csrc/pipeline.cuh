// pipeline.cuh -- shared-memory row pipeline for the CUDA-core kernels.
//
// One producer warp streams the A-rows of the blocks a CTA needs into a ring
// of NST shared-memory stages with TMA bulk copies (cp.async.bulk, one
// contiguous run of rows per stage, completion counted on an mbarrier); the
// consumer warps wait on a stage's "full" barrier, compute, and arrive on its
// "empty" barrier so the producer can refill it.  Every wait is bounded: after
// a limit of device time (WAIT_LIMIT_NS unless the context sets another) the
// waiter raises the kernel's error flag and gives up, so a logic error ends the
// kernel with a status instead of hanging the GPU.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace dgv {

// a wait gives up after this many nanoseconds of device time (%globaltimer)
constexpr unsigned long long WAIT_LIMIT_NS = 4000000000ULL;

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait for the completion of the phase with the given parity.  While
// waiting it also looks at the error flag about once a millisecond, so once
// one wait has given up the other waits of the launch (and of launches queued
// behind it) give up within a millisecond instead of each running its limit.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *err,
                                          unsigned long long limit_ns = WAIT_LIMIT_NS)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    unsigned long long tcheck = t0;
    while (!mbar_try_wait(bar, parity)) {
        const unsigned long long t = globaltimer_ns();
        if (t - t0 > limit_ns) {
            *(volatile int *)err = 1;  // host-mapped flag, read after the stream synchronises
            return false;
        }
        if (t - tcheck > 1000000ULL) {
            tcheck = t;
            if (*(volatile int *)err) return false;
        }
    }
    return true;
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// global -> shared bulk copy (16-byte aligned addresses, size multiple of 16)
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

struct StageHdr {
    int block;  // block index, -1 = end of stream
    int first;  // first pair of the stage within the block
    int n;      // pairs in the stage
    int pad;
};

// Does the valid output-cell box of a block meet the linear cell range
// [d0, d1)?  Conservative: compares the linear extent of the box.
__device__ __forceinline__ bool box_meets_range(const signed char *lo, const signed char *hi, int Mv, int Mw, int d0,
                                                int d1)
{
    int a = (lo[0] * Mv + lo[1]) * Mw + lo[2];
    int b = (hi[0] * Mv + hi[1]) * Mw + hi[2];
    return a < d1 && b >= d0;
}

// Producer side of the pipeline, run by all 32 lanes of one warp: streams, in
// block order, the rows of every block in [b0, b1) whose box meets the cell
// range [d0, d1), at most sp pairs per stage, then posts an end-of-stream
// header.  The lanes test 32 blocks at a time (a CTA's chunk can hold millions
// of one-pair blocks, e.g. on grids of one node per cell, of which its slice of
// output cells meets few); lane 0 waits on the stages and issues the copies.
// On the normal path the consumers wait on every stage, so nothing is left in
// flight when they finish.  If a wait gives up, the producer stops issuing and
// waits (bounded) for the copies it already issued, so no copy can land in the
// shared memory of a CTA that has exited.
template <typename BlockT>
__device__ __forceinline__ void produce_rows(const BlockT *blk, int b0, int b1, int Mv, int Mw, int d0, int d1,
                                             const char *rows, int rowb, unsigned char *stages, int sp, int nst,
                                             StageHdr *hdr, uint64_t *full, uint64_t *empty, int *err,
                                             unsigned long long wait_ns)
{
    const size_t stage_bytes = (size_t)sp * rowb;
    const int lane = threadIdx.x & 31;
    int it = 0;  // stages issued (lane 0)
    bool ok = true;
    for (int base = b0; base < b1 && ok; base += 32) {
        const int b = base + lane;
        bool meet = false;
        long long start = 0;
        int count = 0;
        if (b < b1) {
            const BlockT bi = blk[b];
            meet = box_meets_range(bi.lo, bi.hi, Mv, Mw, d0, d1);
            start = bi.start;
            count = bi.count;
        }
        unsigned m = __ballot_sync(0xffffffffu, meet);
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            const long long st = __shfl_sync(0xffffffffu, start, j);
            const int cnt = __shfl_sync(0xffffffffu, count, j), bj = base + j;
            if (lane == 0) {
                for (int off = 0; off < cnt; off += sp) {
                    const int n = min(sp, cnt - off), s = it % nst;
                    if (!mbar_wait(&empty[s], ((it / nst) & 1) ^ 1, err, wait_ns)) { ok = false; break; }
                    hdr[s] = StageHdr{bj, off, n, 0};
                    mbar_arrive_expect_tx(&full[s], (uint32_t)(n * rowb));
                    bulk_g2s(stages + s * stage_bytes, rows + (size_t)(st + off) * rowb, (uint32_t)(n * rowb),
                             &full[s]);
                    it++;
                }
            }
            ok = __shfl_sync(0xffffffffu, ok, 0);
            if (!ok) break;
        }
    }
    if (lane != 0) return;
    if (ok) {
        const int s = it % nst;
        if (mbar_wait(&empty[s], ((it / nst) & 1) ^ 1, err, wait_ns)) {
            hdr[s] = StageHdr{-1, 0, 0, 0};
            mbar_arrive(&full[s]);
            return;
        }
    }
    // the most recent use of each slot is the one still possibly in flight
    for (int j = it > nst ? it - nst : 0; j < it; j++) mbar_wait(&full[j % nst], (j / nst) & 1, err, wait_ns);
}

}  // namespace dgv
