// synth.cu -- seeded synthetic A-arrays generated directly in the device pair
// layout.  Compiled with -fmad=false: the prefilter distances and the record
// values use exactly the multiply/add sequence of their definition, so the
// records are reproducible bit for bit on any IEEE machine.
//
// Record structure (the part that drives cost and must be realistic): the
// pairs xi < xi1 that pass the prefilter of SetA_DGV (dgvtools_mod.f90:527,
// collision sphere vs. circumscribed sphere of the canonical cell, cutoff
// Trad) and, for support_mode 1, whose collision sphere actually meets the
// canonical cell -- outside that set the SetA integral is identically zero.
// The structure does not depend on the basis function p, so every pair
// carries one record per canonical basis function.
// Values: A = w_xi * w_xi1 * (|g|/8) * u with u in [-1,1) from a splitmix64
// hash of (seed, p, xi, xi1): the reference's scaling (dgvtools_mod.f90:654-659)
// with a seeded stand-in for the collision integral.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "dgv_internal.h"

namespace dgv {

struct SynthArgs {
    const double *nu, *nv, *nw, *nwt;
    double lo[3], hi[3], uu[2], vv[2], ww[2], dphi, Trad;
    unsigned long long seed;
    int support, P, Nc, ccell;
};

__device__ __forceinline__ unsigned long long splitmix64(unsigned long long x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

__device__ __forceinline__ double synth_value(unsigned long long seed, int p, int i2, int i3, double w2,
                                              double w3, double dsph)
{
    unsigned long long k = ((unsigned long long)(unsigned)p << 48) ^ ((unsigned long long)(unsigned)i2 << 24) ^
                           (unsigned long long)(unsigned)i3;
    unsigned long long h = splitmix64(k ^ splitmix64(seed));
    double u = (double)(h >> 11) * (1.0 / 9007199254740992.0);
    u = 2.0 * u - 1.0;
    return w2 * w3 * (dsph / 8.0) * u;
}

// prefilter (and exact support test) for nodes a < b; returns dsph or -1
__device__ __forceinline__ double pair_passes(const SynthArgs &s, int a, int b)
{
    double xiu = s.nu[a], xiv = s.nv[a], xiw = s.nw[a];
    double xi1u = s.nu[b], xi1v = s.nv[b], xi1w = s.nw[b];
    double da = xiu - xi1u, db = xiv - xi1v, dc = xiw - xi1w;
    double dsph = sqrt(da * da + db * db + dc * dc);
    double p = xiu + xi1u - s.uu[0] - s.uu[1];
    double q = xiv + xi1v - s.vv[0] - s.vv[1];
    double r = xiw + xi1w - s.ww[0] - s.ww[1];
    double dist2 = sqrt(p * p + q * q + r * r);
    if ((dist2 > dsph + s.dphi) || (dist2 + s.dphi < dsph) || (dsph > s.Trad)) return -1.0;
    if (s.support == 1) {
        double m[3] = {(xiu + xi1u) / 2.0, (xiv + xi1v) / 2.0, (xiw + xi1w) / 2.0};
        double rad = dsph / 2.0, dmin = 0.0, dmax = 0.0;
        for (int k = 0; k < 3; k++) {
            double aa = s.lo[k] - m[k], bb = m[k] - s.hi[k];
            double t = aa > 0.0 ? aa : (bb > 0.0 ? bb : 0.0);
            dmin += t * t;
            double fa = fabs(m[k] - s.lo[k]), fb = fabs(m[k] - s.hi[k]);
            double fm = fa > fb ? fa : fb;
            dmax += fm * fm;
        }
        double r2 = rad * rad;
        if (!((r2 >= dmin) && (r2 <= dmax))) return -1.0;
    }
    return dsph;
}

// one CTA per candidate cell pair (c1 = blockIdx.y <= c2 = blockIdx.x)
__global__ void k_synth_count(SynthArgs s, int *counts)
{
    int c2 = blockIdx.x, c1 = blockIdx.y;
    if (c2 < c1) return;
    int P = s.P, n = 0;
    for (int t = threadIdx.x; t < P * P; t += blockDim.x) {
        int l1 = t / P, l2 = t - l1 * P;
        if (c1 == c2 && l2 <= l1) continue;
        if (pair_passes(s, c1 * P + l1, c2 * P + l2) >= 0.0) n++;
    }
    __shared__ int red[32];
    for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        int tot = 0;
        for (int w = 0; w < (int)(blockDim.x + 31) / 32; w++) tot += red[w];
        counts[(size_t)c1 * s.Nc + c2] = tot;
    }
}

// one CTA per non-empty block; pairs written in (l1,l2) order, in chunks of
// blockDim.x candidate pairs (a multiple of 32) with a running base
__global__ void k_synth_fill(SynthArgs s, const BlockInfo *blk, double *rows64, int RD64, float *rows32,
                             int RW32)
{
    const BlockInfo b = blk[blockIdx.x];
    const int P = s.P;
    __shared__ int wsum[32];
    __shared__ int chunk_base;
    if (threadIdx.x == 0) chunk_base = 0;
    __syncthreads();
    for (int t0 = 0; t0 < P * P; t0 += blockDim.x) {
        const int t = t0 + (int)threadIdx.x;
        const int l1 = t / P, l2 = t - l1 * P;
        double dsph = -1.0;
        if (t < P * P && !(b.c1 == b.c2 && l2 <= l1)) dsph = pair_passes(s, b.c1 * P + l1, b.c2 * P + l2);
        const bool pass = dsph >= 0.0;
        // exclusive rank of this pair among passing pairs, in thread order
        const unsigned m = __ballot_sync(0xffffffffu, pass);
        const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
        const int rank = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) wsum[w] = __popc(m);
        __syncthreads();
        int base = chunk_base;
        for (int k = 0; k < w; k++) base += wsum[k];
        if (pass) {
            const long long k = b.start + base + rank;
            const int a = b.c1 * P + l1, bb = b.c2 * P + l2;
            int o[2] = {l1 * s.Nc + (b.c1 - s.ccell), l2 * s.Nc + (b.c2 - s.ccell)};
            double *r = rows64 + (size_t)k * RD64;
            float *r32 = rows32 + (size_t)k * RW32;
            double slot;
            memcpy(&slot, o, 8);
            r[0] = slot;
            r32[0] = __int_as_float(o[0]);
            r32[1] = __int_as_float(o[1]);
            const double w2 = s.nwt[a], w3 = s.nwt[bb];
            for (int p = 0; p < P; p++) {
                const double v = synth_value(s.seed, p, a, bb, w2, w3, dsph);
                r[1 + p] = v;
                r32[2 + p] = __double2float_rn(v);
            }
            for (int p = 1 + P; p < RD64; p++) r[p] = 0.0;
            for (int p = 2 + P; p < RW32; p++) r32[p] = 0.0f;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int tot = 0;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += wsum[k];
            chunk_base += tot;
        }
        __syncthreads();
    }
}

int layout_synthetic(Ctx *c, unsigned long long seed, double Trad, int support_mode)
{
    const Grid &g = c->grid;
    const int P = g.P, Nc = g.Nc;
    if (P > 255) return set_err(c, DGV_EUNSUP, "synthetic A: at most 255 nodes per cell");
    if (support_mode != 0 && support_mode != 1) return set_err(c, DGV_EINVAL, "synthetic A: support_mode is 0 or 1");
    if (!(Trad > 0.0)) return set_err(c, DGV_EINVAL, "synthetic A: Trad must be positive");
    SynthArgs s;
    s.nu = c->d_nu; s.nv = c->d_nv; s.nw = c->d_nw; s.nwt = c->d_nwt;
    int cc = g.ccell;
    s.uu[0] = g.lu[cc]; s.uu[1] = g.ru[cc];
    s.vv[0] = g.lv[cc]; s.vv[1] = g.rv[cc];
    s.ww[0] = g.lw[cc]; s.ww[1] = g.rw[cc];
    s.lo[0] = s.uu[0]; s.lo[1] = s.vv[0]; s.lo[2] = s.ww[0];
    s.hi[0] = s.uu[1]; s.hi[1] = s.vv[1]; s.hi[2] = s.ww[1];
    {
        volatile double a = s.uu[1] - s.uu[0], b = s.vv[1] - s.vv[0], d = s.ww[1] - s.ww[0];
        volatile double a2 = a * a, b2 = b * b, d2 = d * d;
        volatile double sum = a2 + b2;
        sum = sum + d2;
        s.dphi = std::sqrt((double)sum);
    }
    s.Trad = Trad; s.seed = seed; s.support = support_mode; s.P = P; s.Nc = Nc; s.ccell = cc;
    int *d_counts = nullptr;
    size_t ncand = (size_t)Nc * Nc;
    DGV_CUDA(c, cudaMalloc(&d_counts, ncand * sizeof(int)));
    DGV_CUDA(c, cudaMemsetAsync(d_counts, 0, ncand * sizeof(int), c->stream));
    int thr = P * P < 128 ? 128 : (P * P < 256 ? 256 : 512);
    k_synth_count<<<dim3(Nc, Nc), thr, 0, c->stream>>>(s, d_counts);
    DGV_CUDA(c, cudaGetLastError());
    std::vector<int> counts(ncand);
    DGV_CUDA(c, cudaMemcpyAsync(counts.data(), d_counts, ncand * sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    cudaFree(d_counts);
    free_layout(c->lay);
    Layout &L = c->lay;
    L.RD64 = ((1 + P) + 1) / 2 * 2;
    L.RW32 = ((2 + P) + 3) / 4 * 4;
    std::vector<BlockInfo> blk;
    long long npairs = 0;
    double record_shifts = 0.0;
    for (int c1 = 0; c1 < Nc; c1++)
        for (int c2 = c1; c2 < Nc; c2++) {
            int n = counts[(size_t)c1 * Nc + c2];
            if (!n) continue;
            BlockInfo b;
            std::memset(&b, 0, sizeof(b));
            b.start = npairs; b.count = n; b.c1 = c1; b.c2 = c2;
            int a[3] = {g.cell_u(c1), g.cell_v(c1), g.cell_w(c1)};
            int e[3] = {g.cell_u(c2), g.cell_v(c2), g.cell_w(c2)};
            int ccx[3] = {g.ccu, g.ccv, g.ccw}, M[3] = {g.d.Mu, g.d.Mv, g.d.Mw};
            double vol = 1.0;
            for (int k = 0; k < 3; k++) {
                int mn = a[k] < e[k] ? a[k] : e[k], mx = a[k] > e[k] ? a[k] : e[k];
                int lo = ccx[k] - mn > 0 ? ccx[k] - mn : 0;
                int hi = ccx[k] + M[k] - 1 - mx < M[k] - 1 ? ccx[k] + M[k] - 1 - mx : M[k] - 1;
                b.lo[k] = (signed char)lo; b.hi[k] = (signed char)hi;
                vol *= (double)(hi - lo + 1);
            }
            record_shifts += (double)n * P * vol;
            blk.push_back(b);
            npairs += n;
        }
    L.npairs = npairs;
    L.nblocks = (long long)blk.size();
    L.nrecords = npairs * P;
    L.record_shifts = record_shifts;
    L.h_blk = blk;
    L.h_work.resize(blk.size());
    for (size_t b = 0; b < blk.size(); b++) {
        double vol = 1.0;
        for (int k = 0; k < 3; k++) vol *= (double)(blk[b].hi[k] - blk[b].lo[k] + 1);
        L.h_work[b] = (double)blk[b].count * vol + 64.0;
    }
    DGV_CUDA(c, cudaMalloc(&L.blk, std::max<size_t>(1, blk.size()) * sizeof(BlockInfo)));
    DGV_CUDA(c, cudaMalloc(&L.rows64, std::max<long long>(1, npairs) * L.RD64 * sizeof(double)));
    DGV_CUDA(c, cudaMalloc(&L.rows32, std::max<long long>(1, npairs) * L.RW32 * sizeof(float)));
    if (!blk.empty()) {
        DGV_CUDA(c, cudaMemcpyAsync(L.blk, blk.data(), blk.size() * sizeof(BlockInfo), cudaMemcpyHostToDevice, c->stream));
        const int fthr = std::min(1024, ((P * P + 31) / 32) * 32);
        k_synth_fill<<<(unsigned)blk.size(), fthr, 0, c->stream>>>(s, L.blk, (double *)L.rows64, L.RD64,
                                                                    (float *)L.rows32, L.RW32);
        DGV_CUDA(c, cudaGetLastError());
    }
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    return DGV_OK;
}

}  // namespace dgv
