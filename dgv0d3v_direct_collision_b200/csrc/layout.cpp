// layout.cpp -- conversion of reference-layout A-arrays (commvar.f90:157-167)
// into the device pair layout, export back to the reference layout, and the
// work partition of the block list.
//
// Reference layout: records of node k are A(Ashift_k+1 .. Ashift_k+capphi_k)
// with Ashift_k = sum(capphi(1:k-1)) (miscset.f90:1307).  Only nodes of the
// canonical cell are ever read by EvalCollisionPeriodicAPlus_DGV
// (collision_mod.f90:186-188: records are addressed through nodes_phican).
//
// Pair layout: a record (xi, xi1, A) of canonical basis function p becomes
// value v[p] of the unordered pair {xi, xi1}; the product f(xi)f(xi1) under a
// cell shift is symmetric in the two velocities, so (xi, xi1) and (xi1, xi)
// are the same pair.  Pairs are grouped by their cell pair (c1 <= c2) and
// sorted by (c1, c2, l1, l2); duplicate records of one p are summed.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "dgv_internal.h"

namespace dgv {

void free_layout(Layout &L)
{
    if (L.blk) cudaFree(L.blk);
    if (L.rows64) cudaFree(L.rows64);
    if (L.rows32) cudaFree(L.rows32);
    for (auto &kv : L.chunks) cudaFree(kv.second);
    if (L.tc_V) cudaFree(L.tc_V);
    if (L.tc_chunk_start) cudaFree(L.tc_chunk_start);
    if (L.tc2_W) cudaFree(L.tc2_W);
    if (L.tc2_Wv) cudaFree(L.tc2_Wv);
    for (auto &kv : L.tc_lists)
        for (void *p : kv.second) cudaFree(p);
    L = Layout();
}

// Frees the device layouts of `mask` (DGV_LAYOUT_*); each is rebuilt on its
// next use (FP32 rows from the FP64 rows by ensure_rows32, the tensor-core
// records by their prepare functions).  Graphs holding launches that read
// them are released first.
int release_layouts(Ctx *c, int mask)
{
    Layout &L = c->lay;
    release_graphs(c);
    DGV_CUDA(c, cudaStreamSynchronize(c->stream));
    auto drop_lists = [&](int lo, int hi) {  // work lists keyed in [lo, hi)
        for (auto it = L.tc_lists.begin(); it != L.tc_lists.end();) {
            if (it->first >= lo && it->first < hi) {
                for (void *q : it->second) cudaFree(q);
                L.tc_list_work.erase(it->first);
                L.tc_list_items.erase(it->first);
                it = L.tc_lists.erase(it);
            } else {
                ++it;
            }
        }
    };
    if ((mask & DGV_LAYOUT_F32) && L.rows32) {
        cudaFree(L.rows32);
        L.rows32 = nullptr;
    }
    if (mask & DGV_LAYOUT_TC_CHUNK) {
        if (L.tc_V) cudaFree(L.tc_V);
        if (L.tc_chunk_start) cudaFree(L.tc_chunk_start);
        L.tc_V = nullptr;
        L.tc_chunk_start = nullptr;
        L.tc_chunk_host.clear();
        L.tc_sets.clear();
        drop_lists(0, 256);
    }
    if (mask & (DGV_LAYOUT_TC_BLOCK | DGV_LAYOUT_TC_ADJ)) {
        if (L.tc2_Wv) cudaFree(L.tc2_Wv);
        L.tc2_Wv = nullptr;
        L.tc2_goff2.clear();
        L.tc2_sets_adj.clear();
        drop_lists(512, 1 << 30);
    }
    if (mask & DGV_LAYOUT_TC_BLOCK) {
        if (L.tc2_W) cudaFree(L.tc2_W);
        L.tc2_W = nullptr;
        L.tc2_mask.clear();
        L.tc2_goff.clear();
        L.tc2_sets.clear();
        L.tc2_set_mb = 0;
        drop_lists(256, 512);
    }
    return DGV_OK;
}

static inline void box_for(const Grid &g, int c1, int c2, BlockInfo &b)
{
    int a[3] = {g.cell_u(c1), g.cell_v(c1), g.cell_w(c1)};
    int e[3] = {g.cell_u(c2), g.cell_v(c2), g.cell_w(c2)};
    int cc[3] = {g.ccu, g.ccv, g.ccw};
    int M[3] = {g.d.Mu, g.d.Mv, g.d.Mw};
    for (int k = 0; k < 3; k++) {
        int mn = std::min(a[k], e[k]), mx = std::max(a[k], e[k]);
        int lo = std::max(0, cc[k] - mn), hi = std::min(M[k] - 1, cc[k] + M[k] - 1 - mx);
        b.lo[k] = (signed char)lo;
        b.hi[k] = (signed char)hi;
    }
}

static inline double box_volume(const BlockInfo &b)
{
    double v = 1.0;
    for (int k = 0; k < 3; k++) v *= (double)(b.hi[k] - b.lo[k] + 1 > 0 ? b.hi[k] - b.lo[k] + 1 : 0);
    return v;
}

// Row sizes: FP64 rows hold one 8-byte slot for (o1, o2) then P doubles,
// padded to a 16-byte multiple; FP32 rows hold (o1, o2) then P floats,
// padded to a 16-byte multiple.
static void row_sizes(int P, int &RD64, int &RW32)
{
    RD64 = ((1 + P) + 1) / 2 * 2;
    RW32 = ((2 + P) + 3) / 4 * 4;
}

// Uploads host rows and blocks and finishes the Layout bookkeeping.
static int upload_layout(Ctx *c, std::vector<BlockInfo> &blk, std::vector<double> &rows64,
                         long long npairs, long long nrecords, double record_shifts)
{
    Layout &L = c->lay;
    const Grid &g = c->grid;
    int P = g.P;
    std::vector<float> rows32((size_t)npairs * L.RW32, 0.0f);
    for (long long k = 0; k < npairs; k++) {
        const double *r = rows64.data() + (size_t)k * L.RD64;
        float *s = rows32.data() + (size_t)k * L.RW32;
        std::memcpy(s, r, 8);  // o1, o2
        for (int p = 0; p < P; p++) s[2 + p] = (float)r[1 + p];
    }
    L.npairs = npairs;
    L.nblocks = (long long)blk.size();
    L.nrecords = nrecords;
    L.record_shifts = record_shifts;
    L.h_blk = blk;
    L.h_work.resize(blk.size());
    for (size_t b = 0; b < blk.size(); b++) L.h_work[b] = (double)blk[b].count * box_volume(blk[b]) + 64.0;
    size_t bb = std::max<size_t>(1, blk.size()) * sizeof(BlockInfo);
    size_t r64 = std::max<size_t>(1, rows64.size()) * sizeof(double);
    size_t r32 = std::max<size_t>(1, rows32.size()) * sizeof(float);
    DGV_CUDA(c, cudaMalloc(&L.blk, bb));
    DGV_CUDA(c, cudaMalloc(&L.rows64, r64));
    DGV_CUDA(c, cudaMalloc(&L.rows32, r32));
    if (!blk.empty()) DGV_CUDA(c, cudaMemcpy(L.blk, blk.data(), blk.size() * sizeof(BlockInfo), cudaMemcpyHostToDevice));
    if (!rows64.empty()) DGV_CUDA(c, cudaMemcpy(L.rows64, rows64.data(), rows64.size() * sizeof(double), cudaMemcpyHostToDevice));
    if (!rows32.empty()) DGV_CUDA(c, cudaMemcpy(L.rows32, rows32.data(), rows32.size() * sizeof(float), cudaMemcpyHostToDevice));
    return DGV_OK;
}

int layout_from_reference(Ctx *c, long long nnz, const int32_t *capphi, const double *A,
                          const int32_t *xi, const int32_t *xi1, int one_based)
{
    const Grid &g = c->grid;
    const long long N = g.N;
    const int P = g.P, Nc = g.Nc;
    if (nnz < 0) return set_err(c, DGV_EINVAL, "load_A: negative record count");
    if (!capphi || (nnz > 0 && (!A || !xi || !xi1)))
        return set_err(c, DGV_EINVAL, "load_A: NULL array");
    std::vector<long long> pre(N + 1, 0);
    for (long long k = 0; k < N; k++) {
        if (capphi[k] < 0) return set_err(c, DGV_EINVAL, "load_A: negative A_capphi entry");
        pre[k + 1] = pre[k] + capphi[k];
    }
    if (pre[N] != nnz)
        return set_err(c, DGV_EINVAL, "load_A: sum(A_capphi) differs from the record count");
    const int off = one_based ? 1 : 0;
    const long long k0 = (long long)g.ccell * P;
    // keys of the canonical-cell records
    const unsigned long long PP = (unsigned long long)P * P;
    long long ncan = pre[k0 + P] - pre[k0];
    std::vector<unsigned long long> keys;
    keys.reserve((size_t)ncan);
    for (int p = 0; p < P; p++)
        for (long long j = pre[k0 + p]; j < pre[k0 + p + 1]; j++) {
            long long a = (long long)xi[j] - off, b = (long long)xi1[j] - off;
            if (a < 0 || a >= N || b < 0 || b >= N)
                return set_err(c, DGV_ERANGE, "load_A: A_xi/A_xi1 index outside the node range");
            if (a > b) std::swap(a, b);
            unsigned long long key = ((unsigned long long)(a / P) * Nc + (unsigned long long)(b / P)) * PP +
                                     (unsigned long long)(a % P) * P + (unsigned long long)(b % P);
            keys.push_back(key);
        }
    std::vector<unsigned long long> pairs(keys);
    std::sort(pairs.begin(), pairs.end());
    pairs.erase(std::unique(pairs.begin(), pairs.end()), pairs.end());
    const long long npairs = (long long)pairs.size();
    Layout &L = c->lay;
    row_sizes(P, L.RD64, L.RW32);
    std::vector<double> rows64((size_t)npairs * L.RD64, 0.0);
    // pair offsets and blocks
    std::vector<BlockInfo> blk;
    for (long long k = 0; k < npairs; k++) {
        unsigned long long key = pairs[k];
        int l2 = (int)(key % P), l1 = (int)((key / P) % P);
        unsigned long long cp = key / PP;
        int c2 = (int)(cp % Nc), c1 = (int)(cp / Nc);
        int32_t o[2] = {l1 * Nc + (c1 - g.ccell), l2 * Nc + (c2 - g.ccell)};
        std::memcpy(rows64.data() + (size_t)k * L.RD64, o, 8);
        if (blk.empty() || blk.back().c1 != c1 || blk.back().c2 != c2) {
            BlockInfo b;
            std::memset(&b, 0, sizeof(b));
            b.start = k; b.count = 0; b.c1 = c1; b.c2 = c2;
            box_for(g, c1, c2, b);
            blk.push_back(b);
        }
        blk.back().count++;
    }
    // values; the record order within one p is kept for duplicate sums
    size_t t = 0;
    double record_shifts = 0.0;
    std::vector<double> pair_vol((size_t)npairs, 0.0);
    for (const auto &b : blk)
        for (long long k = b.start; k < b.start + b.count; k++) pair_vol[(size_t)k] = box_volume(b);
    for (int p = 0; p < P; p++)
        for (long long j = pre[k0 + p]; j < pre[k0 + p + 1]; j++, t++) {
            long long k = std::lower_bound(pairs.begin(), pairs.end(), keys[t]) - pairs.begin();
            double *r = rows64.data() + (size_t)k * L.RD64;
            r[1 + p] += A[j];
            record_shifts += pair_vol[(size_t)k];
        }
    return upload_layout(c, blk, rows64, npairs, ncan, record_shifts);
}

int layout_export(Ctx *c, long long *nnz_out, int32_t *capphi, double *A, int32_t *xi,
                  int32_t *xi1)
{
    const Grid &g = c->grid;
    const Layout &L = c->lay;
    const int P = g.P;
    std::vector<double> rows((size_t)L.npairs * L.RD64);
    if (L.npairs)
        DGV_CUDA(c, cudaMemcpy(rows.data(), L.rows64, rows.size() * sizeof(double), cudaMemcpyDeviceToHost));
    long long nnz = 0;
    std::vector<long long> cnt(P, 0);
    for (long long k = 0; k < L.npairs; k++)
        for (int p = 0; p < P; p++)
            if (rows[(size_t)k * L.RD64 + 1 + p] != 0.0) { cnt[p]++; nnz++; }
    *nnz_out = nnz;
    if (!capphi || !A || !xi || !xi1) return DGV_OK;
    std::memset(capphi, 0, sizeof(int32_t) * (size_t)g.N);
    for (int p = 0; p < P; p++) capphi[(long long)g.ccell * P + p] = (int32_t)cnt[p];
    long long j = 0;
    for (int p = 0; p < P; p++)
        for (const auto &b : L.h_blk)
            for (long long k = b.start; k < b.start + b.count; k++) {
                const double *r = rows.data() + (size_t)k * L.RD64;
                double v = r[1 + p];
                if (v == 0.0) continue;
                int32_t o[2];
                std::memcpy(o, r, 8);
                int l1 = (o[0] - (b.c1 - g.ccell)) / g.Nc, l2 = (o[1] - (b.c2 - g.ccell)) / g.Nc;
                A[j] = v;
                xi[j] = b.c1 * P + l1;
                xi1[j] = b.c2 * P + l2;
                j++;
            }
    return DGV_OK;
}

// Contiguous block ranges of about equal work (pairs x valid shifts).
int get_chunks(Ctx *c, int nchunks, int **d_bounds)
{
    Layout &L = c->lay;
    auto it = L.chunks.find(nchunks);
    if (it != L.chunks.end()) { *d_bounds = it->second; return DGV_OK; }
    std::vector<int> bounds(nchunks + 1, (int)L.nblocks);
    double tot = 0.0;
    for (double w : L.h_work) tot += w;
    bounds[0] = 0;
    double acc = 0.0;
    int ch = 1;
    for (long long b = 0; b < L.nblocks && ch < nchunks; b++) {
        acc += L.h_work[b];
        while (ch < nchunks && acc >= tot * ch / nchunks) bounds[ch++] = (int)(b + 1);
    }
    int *d = nullptr;
    DGV_CUDA(c, cudaMalloc(&d, sizeof(int) * (nchunks + 1)));
    DGV_CUDA(c, cudaMemcpy(d, bounds.data(), sizeof(int) * (nchunks + 1), cudaMemcpyHostToDevice));
    L.chunks[nchunks] = d;
    *d_bounds = d;
    return DGV_OK;
}

}  // namespace dgv
