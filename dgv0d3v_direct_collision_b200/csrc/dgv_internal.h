// dgv_internal.h -- context, device layout and kernel entry points shared by
// the sources of libdgv_b200.so.  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/dgv_b200.h"

namespace dgv {

// One cell-pair block of the pair layout.  Records of the reference are
// regrouped by the (canonical-frame) cells c1 <= c2 of their two velocities;
// for an output cell D the block contributes iff both shifted cells
// c1 + D - ccell and c2 + D - ccell stay inside the grid, i.e. iff D lies in
// the box [lo, hi] (per axis).  This is the per-record bounds test of
// collision_mod.f90:196-211 hoisted to the block.
struct __align__(16) BlockInfo {
    long long start;   // first pair of the block
    int count;         // pairs in the block
    int c1, c2;        // linear cell indices, canonical frame
    signed char lo[3]; // valid output-cell box, inclusive
    signed char hi[3];
    short pad;
};
static_assert(sizeof(BlockInfo) == 32, "BlockInfo layout");

// Host-side grid (own restatement of the reference's uniform mesh).
struct Grid {
    dgv_grid_desc d;
    int P = 0, Nc = 0;
    long long N = 0;
    int ccell = -1, ccu = 0, ccv = 0, ccw = 0;
    std::vector<double> gu, gv, gw;          // 1-D grids
    std::vector<double> xu, wu, xv, wv, xw, ww;  // Gauss-Legendre rules
    std::vector<double> lu, ru, lv, rv, lw, rw;  // cell bounds
    std::vector<double> nu, nv, nw, nwt;     // node coordinates and weights
    int cell_u(int c) const { return c / (d.Mv * d.Mw); }
    int cell_v(int c) const { return (c / d.Mw) % d.Mv; }
    int cell_w(int c) const { return c % d.Mw; }
};
int build_grid(const dgv_grid_desc &d, Grid &g, std::string &err);

// Device copy of the A-arrays in the pair layout.
//   rows64[pair] = { int32 o1, int32 o2, double v[P], pad }  (RD64 doubles)
//   rows32[pair] = { int32 o1, int32 o2, float v[P], pad }   (RW32 words)
// o1 = l1*Nc + (c1 - ccell), o2 = l2*Nc + (c2 - ccell): for output cell D the
// two factors are f_s[o1 + D] and f_s[o2 + D] in the local-major shared copy
// f_s[l*Nc + cell] of f.  v[p] is the A value of canonical basis function p
// for the pair (0 where the reference has no record).
struct Layout {
    long long nrecords = 0, npairs = 0, nblocks = 0;
    double record_shifts = 0;  // sum over records of valid shifts
    int RD64 = 0, RW32 = 0;    // row length in doubles / 32-bit words
    BlockInfo *blk = nullptr;  // device
    void *rows64 = nullptr;    // device
    void *rows32 = nullptr;    // device
    std::vector<BlockInfo> h_blk;     // host copy
    std::vector<double> h_work;       // per block: pairs x valid shifts
    // work partitions: nchunks -> device array of nchunks+1 block bounds
    std::map<int, int *> chunks;
    // tensor-core form (built on first use): per block ceil(count/64) chunk
    // records of split-fp16 value tiles, their first record per block, the
    // power-of-two value scale, and the block sets of one launch each
    void *tc_V = nullptr;            // device
    int *tc_chunk_start = nullptr;   // device, nblocks+1
    double tc_vscale = 1.0;
    std::vector<int> tc_chunk_host;
    std::vector<int> tc_sets;
    // block form (built on first use): per block the dense split-fp16 tiles
    // W[l2][(l1, p)] of its values, the value scale, and the block sets
    void *tc2_W = nullptr;  // device
    void *tc2_Wv = nullptr;  // device: the adjoint's second record set (built on first use)
    double tc2_vscale = 1.0;
    std::vector<int> tc2_sets;
    std::vector<int> tc2_sets_adj;  // the adjoint's launches (both of its record sets per launch)
    int tc2_set_mb = 0;  // record megabytes per set the sets were built for
    // device work lists {items, item starts, tile order}, keyed by cells per
    // tile (chunk form) or 256 + cells per tile (block form)
    std::map<int, std::vector<void *>> tc_lists;
    std::map<int, long long> tc_list_work;   // per key: sum of the items' work (chunk records / issued columns)
    std::map<int, long long> tc_list_items;  // per key: number of items
    // block form: per block the masks of its nodes l1 (entries 0..nblocks-1)
    // and l2 (nblocks..2 nblocks-1; bit l set if the block has a pair with
    // node l) and the first record group of the block's compacted records in
    // W (tc2_goff) and in the adjoint's W2 (tc2_goff2); nblocks + 1 entries,
    // host
    std::vector<uint32_t> tc2_mask;
    std::vector<long long> tc2_goff, tc2_goff2;
};
void free_layout(Layout &L);

struct Ctx {
    int device = 0;
    Grid grid;
    Layout lay;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    bool async = false;
    bool project = false;
    int nchunks_opt = 0;
    std::string err;
    // device copies of node tables
    double *d_nu = nullptr, *d_nv = nullptr, *d_nw = nullptr, *d_nwt = nullptr;
    double gram_inv[25];  // inverse Gram matrix of the invariants, FP64
    // device work buffers (grown on demand)
    double *d_partial = nullptr;
    size_t partial_bytes = 0;
    double *d_in = nullptr, *d_out = nullptr;  // staging for host pointers
    size_t in_bytes = 0, out_bytes = 0;
    double *d_tmp[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    size_t tmp_n = 0;
    double *d_red = nullptr;  // reduction scratch
    size_t red_bytes = 0;
    // tensor-core path: scaled fp32 copy of f (+ per-VDF scales), FP64 sums
    double *d_tcF = nullptr, *d_tcQ = nullptr;
    size_t tcF_bytes = 0, tcQ_bytes = 0;
    // CUDA-core kernels with f in global memory: local-major copies f[v][l*Nc + cell]
    double *d_fg = nullptr;
    size_t fg_bytes = 0;
    // VJP: local-major accumulator g_lm[l*Nc + cell]
    double *d_glm = nullptr;
    size_t glm_bytes = 0;
    // Adams-Bashforth history: right sides frhs1..frhs5 (newest first)
    double *d_hist[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
    int ab_order = 0;
    // linearisation point
    double *d_fm = nullptr;
    // run modes of SpatialOperSH_DGV (CheckSolutionMode_DGV): off while
    // decomp_lev == 0; the local Maxwellian, Df = f - fm and a scratch array
    double decomp_lev = 0.0, linear_lev = 0.0, last_L1 = -1.0;
    int run_mode = 0;
    double *d_fmn = nullptr, *d_dfr = nullptr, *d_rgt = nullptr;
    size_t fmn_bytes = 0, dfr_bytes = 0, rgt_bytes = 0;
    // error flag raised by a bounded device wait that gave up: pinned host
    // memory mapped into the device (h_err and d_err alias the same int)
    int *h_err = nullptr, *d_err = nullptr;
    // autotuned chunk counts keyed by (precision, nvdf bucket)
    std::map<long long, int> tuned;
    // kernel timing (DGV_OPT_KTIMING): event pairs around the collision
    // kernel's launches, summed on request; launch counters
    bool ktiming = false;
    int tc_form = 2;  // DGV_OPT_TCFORM: 1 chunk form, 2 block form (8 or 27 nodes per cell)
    int tc_tiles_per_cta = 2;  // DGV_OPT_TCTILES: VDF tiles per CTA in the block form
    int tc_set_mb = 48;        // DGV_OPT_TCSETMB: block form, MB of records per launch
    long long wait_limit_us = 0;  // DGV_OPT_WAIT_LIMIT_US: bounded waits of the block form (0 = 4 s)
    int f_global = 0;             // DGV_OPT_FGLOBAL: 1 = CUDA-core kernels gather f from global memory
    bool tc_autotune = true;      // DGV_OPT_TCAUTOTUNE: tune tiles per CTA and records per launch
    int tc_persistent = 0;     // DGV_OPT_TCPERSIST: block form, 1 = one persistent launch over all block sets
    bool tc_user_launch = false;  // the caller set DGV_OPT_TCTILES, _TCSETMB or _TCPERSIST: no tuning
    struct TcChoice {
        int tiles, set_mb, persistent;
    };
    std::map<int, TcChoice> tc_tuned;  // per batch class: the tuned launch choice
    std::map<int, int> tc_tuned_adj;   // per batch class: the adjoint's persistent-launch choice
    double *d_tc2done = nullptr;       // persistent block-form launches: order flags (ints)
    size_t tc2done_bytes = 0;
    bool test_withhold = false;   // DGV_OPT_TEST_WITHHOLD: the next block-form launch withholds one copy
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> kt_pending, kt_pool;
    long long kt_launches = 0, kt_all = 0;
    double kt_ms = 0.0;
};

// Brackets the launches of the collision kernel on the context stream with
// CUDA events when kernel timing is on (not while the stream is captured).
struct KTimer {
    Ctx *c;
    std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
    bool on = false;
    explicit KTimer(Ctx *ctx);
    void stop(long long nlaunch);
};
void count_launches(Ctx *c, long long n);
void free_ktimers(Ctx *c);

// error helpers
int set_err(Ctx *c, int code, const std::string &msg);
#define DGV_CUDA(c, call)                                                        \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess)                                                   \
            return dgv::set_err((c), DGV_ECUDA,                                  \
                                std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

int ensure_buffer(Ctx *c, double **p, size_t *have, size_t need_bytes);
// frees the layouts of a DGV_LAYOUT_* mask (rebuilt on their next use)
int release_layouts(Ctx *c, int mask);
// the FP32 rows, rebuilt from the FP64 rows after a release
int ensure_rows32(Ctx *c);
// local-major copies f[v][l*Nc + cell] of nvdf VDFs (FP32 or FP64) in the
// context's buffer, for the CUDA-core kernels that gather f from global memory
int f_local_major(Ctx *c, const double *d_f, int nvdf, bool f32, const void **out);
// the limit of the kernels' bounded waits (DGV_OPT_WAIT_LIMIT_US, else 4 s)
inline unsigned long long wait_limit_ns(const Ctx *c)
{
    return c->wait_limit_us > 0 ? (unsigned long long)c->wait_limit_us * 1000ULL : 4000000000ULL;
}
// *dev = true for memory of c's device (or managed), false for host memory;
// DGV_EINVAL for device memory of another GPU
int classify_ptr(Ctx *c, const void *p, bool *dev);
// loads the no-allocation path's static work array on c's device (the
// runtime loads modules lazily), so that it is reserved from context creation
void noalloc_prepare(Ctx *c);
void release_graphs(const Ctx *c);
int ensure_errflag(Ctx *c);
int check_errflag(Ctx *c);

// layout construction
int layout_from_reference(Ctx *c, long long nnz, const int32_t *capphi, const double *A,
                          const int32_t *xi, const int32_t *xi1, int one_based);
int layout_synthetic(Ctx *c, unsigned long long seed, double Trad, int support_mode);
int layout_seta(Ctx *c, double Trad, double ErrChi, double ErrEps, double min_sens, int basis_mode);
int layout_export(Ctx *c, long long *nnz_out, int32_t *capphi, double *A, int32_t *xi,
                  int32_t *xi1);
int get_chunks(Ctx *c, int nchunks, int **d_bounds);

// kernels (device pointers, ctx stream)
int collide_device(Ctx *c, const double *d_f, double *d_q, int nvdf, int precision,
                   double scale);
int collide_tc_device(Ctx *c, const double *d_f, double *d_q, int nvdf, double scale);
int collide_cells_device(Ctx *c, const double *d_f, double *d_q, int nvdf, int precision, int cell0, int cell1);
int jvp_device(Ctx *c, const double *d_f, const double *d_df, double *d_q, int precision);
int vjp_device(Ctx *c, const double *d_f, const double *d_v, double *d_g, int precision);
int vjp_tc_device(Ctx *c, const double *d_f, const double *d_v, double *d_g, int nvdf);
int moments_device(Ctx *c, const double *d_f, int nvdf, double *h_out);
int project_device(Ctx *c, double *d_q, int nvdf);
int maxwellian_device(Ctx *c, double T, double u0, double v0, double w0, double n, double *d_f);
int rk_step_device(Ctx *c, double *d_f, double *d_frhs1, double dt, int order, int precision, int nb = 1);
int spatial_device(Ctx *c, const double *d_f, double *d_out, double dt, int precision);
int ab_prepare_device(Ctx *c, double *d_f, double dt, int order, int precision);
int ab_step_device(Ctx *c, double *d_f, double dt, int precision);
int ab_history_get(Ctx *c, int *order, std::vector<double> &frhs);
int ab_history_set(Ctx *c, int order, const double *frhs);

}  // namespace dgv

struct dgv_ctx {
    dgv::Ctx c;
};
