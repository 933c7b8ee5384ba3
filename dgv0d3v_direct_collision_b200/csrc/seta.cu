// seta.cu -- the A-array precompute (SetA_DGV, dgvtools_mod.f90:377-681,
// with A_IntEpsilon :988-1122 and EvalPhiPostCollIntegrand :938-975) on the
// device.
//
// For a canonical basis function phi (node i1 of the canonical cell) and a
// pair of velocities xi < xi1, the record value is
//   A = w(xi) w(xi1) |g|/8 * int_0^pi sin(chi) int_0^2pi
//         [phi(xi') + phi(xi1') - phi(xi) - phi(xi1)] d eps d chi
// (post-collision velocities xi', xi1' on the sphere over the pair), each
// integral by the reference's adaptive Simpson scheme: n0 uniform cells,
// every cell with a non-zero sample halved and its two-panel Simpson sum
// accepted when |q1+q2-q|/15/h <= err, otherwise refined on the next level;
// a level is only processed while the sum of |q1|+|q2| over the previous
// level exceeds err.  The records kept are those with |A| > min_sens.
//
// Device organisation: the pair layout (cell-pair blocks) is built first with
// the reference prefilter and the exact sphere-cell test (outside it the
// integrand vanishes identically, A = 0); then one warp per (pair, basis
// function) evaluates the two nested integrals.  The chi integral is run by
// the whole warp in the reference's cell order; each chi sample is an eps
// integral whose cells are spread over the 32 lanes.  The first two levels
// of each scheme are fused (all initial cells with a non-zero sample are
// refined on level 1), so only cells marked for a further level are stored:
// in per-warp lists in global scratch.  Sums within a level are reduced
// across lanes, so their rounding order differs from the serial loop.
// Compiled with -fmad=false, as the oracle is compiled without contraction.
// The integrand, the basis function and the eps integral are real calls, not
// inlined copies: inlined at every call site the kernel outgrew the
// instruction cache (warps stalled on instruction fetch, 0.07 IPC).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "dgv_internal.h"

namespace dgv {

namespace {

constexpr double PI_SETA = 3.141592653589793238462643;  // pi25DT (dgvtools_mod.f90:386)
constexpr int SETA_NCAP = 10000;                          // cell cap of the reference's scheme
constexpr int SETA_WARPS = 8;                             // warps per CTA

struct Cell {
    double a, b, fa, fm, fb;
};

// Gauss-Legendre nodes on [-1, 1] per axis (kept out of the kernel's
// parameter block: indexed in loops, they would otherwise be copied to local
// memory)
__constant__ double c_xu[8], c_xv[8], c_xw[8];

struct SetaArgs {
    const int2 *pairs;  // (xi, xi1) node indices of every row of the layout
    long long npairs;
    int P;
    const double *nu, *nv, *nw, *nwt;
    double lu, ru, lv, rv, lw, rw;  // canonical cell
    int su, sv, sw;
    int ccell;
    double ires, err_chi, err_eps, min_sens;
    int mode;  // 0: Lagrange basis; 1..5: invariants 1, u, v, w, |v|^2
    double *rows64;
    int RD64;
    unsigned long long *next;  // work counter
    Cell *scratch;             // 4 lists of SETA_NCAP cells per warp
    int *nan_flag;
};

struct PairState {
    double xiu, xiv, xiw, xi1u, xi1v, xi1w;
    double ugu, ugv, ugw, ugux2, ugvx2, ugwx2, ugux3, ugvx3, ugwx3, g1, g2, dsph;
    double varphi;  // phi(xi) + phi(xi1)
    int pu, pv, pw;
};

// lagrbasfun (dgvtools_mod.f90:31-56)
__device__ double lagr(int i, double x, const double *kap, int n)
{
    double y = 1.0;
    for (int j = 0; j < i; j++) y = y * (kap[j] - x) / (kap[j] - kap[i]);
    for (int j = i + 1; j < n; j++) y = y * (kap[j] - x) / (kap[j] - kap[i]);
    return y;
}

// EvalLagrBasisFunByNdsDGblzmEZ (dgvtools_mod.f90:232-289) with the
// commented cell test and Lagrange product put back (mode 0), or a collision
// invariant (modes 1..5, the known-answer configuration of :267-274)
__device__ __noinline__ double basis(const SetaArgs &a, const PairState &s, double u, double v, double w)
{
    switch (a.mode) {
    case 1: return 1.0;
    case 2: return u;
    case 3: return v;
    case 4: return w;
    case 5: return u * u + v * v + w * w;
    default: break;
    }
    if (u < a.lu || a.ru < u || v < a.lv || a.rv < v || w < a.lw || a.rw < w) return 0.0;
    double y = 1.0;
    double unor = (u - (a.ru + a.lu) / 2.0) / (a.ru - a.lu) * 2.0;
    y = y * lagr(s.pu, unor, c_xu, a.su);
    double vnor = (v - (a.rv + a.lv) / 2.0) / (a.rv - a.lv) * 2.0;
    y = y * lagr(s.pv, vnor, c_xv, a.sv);
    double wnor = (w - (a.rw + a.lw) / 2.0) / (a.rw - a.lw) * 2.0;
    y = y * lagr(s.pw, wnor, c_xw, a.sw);
    return y;
}

// EvalPhiPostCollIntegrand (dgvtools_mod.f90:938-975)
__device__ __noinline__ double integrand(const SetaArgs &a, const PairState &s, double sinchi, double coschi,
                                         double epsil)
{
    double sinchicoseps = cos(epsil) * sinchi / s.g1;
    double sinchisineps = sin(epsil) * sinchi / s.g2;
    double ku = s.ugu * coschi - s.ugux2 * sinchicoseps - s.ugux3 * sinchisineps;
    double kv = s.ugv * coschi - s.ugvx2 * sinchicoseps - s.ugvx3 * sinchisineps;
    double kw = s.ugw * coschi - s.ugwx2 * sinchicoseps - s.ugwx3 * sinchisineps;
    double xiupr = ((s.xiu + s.xi1u) + s.dsph * ku) / 2.0;
    double xi1upr = ((s.xiu + s.xi1u) - s.dsph * ku) / 2.0;
    double xivpr = ((s.xiv + s.xi1v) + s.dsph * kv) / 2.0;
    double xi1vpr = ((s.xiv + s.xi1v) - s.dsph * kv) / 2.0;
    double xiwpr = ((s.xiw + s.xi1w) + s.dsph * kw) / 2.0;
    double xi1wpr = ((s.xiw + s.xi1w) - s.dsph * kw) / 2.0;
    return basis(a, s, xiupr, xivpr, xiwpr) + basis(a, s, xi1upr, xi1vpr, xi1wpr) - s.varphi;
}

__device__ __forceinline__ double warp_sum(double x)
{
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}

// Simpson test of one cell with its two quarter-point samples; returns the
// refine flag and adds to the level's sums
__device__ __forceinline__ bool simpson_cell(double a, double b, double fa, double fm, double fb, double fq1, double fq3,
                                             double err, double &total, double &my_int)
{
    const double mid = (a + b) / 2;
    const double quad = (fa + 4 * fm + fb) * (b - a) / 6;
    const double quad1 = (fa + 4 * fq1 + fm) * (mid - a) / 6;
    const double quad2 = (fm + 4 * fq3 + fb) * (b - mid) / 6;
    const double es = fabs(quad1 + quad2 - quad) / 15 / (b - a);
    my_int = my_int + fabs(quad1) + fabs(quad2);
    if (es > err) return true;
    total = total + quad1 + quad2;
    return false;
}

// A_IntEpsilon (dgvtools_mod.f90:988-1122): warp-cooperative; every lane
// returns the same value
__device__ __noinline__ double eps_integral(const SetaArgs &a, const PairState &s, double chi, Cell *lst0, Cell *lst1)
{
    const int lane = threadIdx.x & 31;
    __syncwarp();  // every lane is done reading the lists of the previous call
    const double sinchi = sin(chi), coschi = cos(chi);
    int n1 = (int)floor(PI_SETA * s.dsph * sinchi / a.ires) + 1;
    if (n1 > SETA_NCAP) n1 = SETA_NCAP;
    const double len = 2 * PI_SETA, err = a.err_eps;
    double total = 0.0, my_int = 0.0, carry = 0.0;
    int nmark = 0, nnz = 0;
    bool overflow = false;
    // levels 0 and 1: initial cells, every cell with a non-zero sample halved
    for (int base = 0; base < n1; base += 32) {
        const int d = base + lane;
        const bool act = d < n1;
        double ca = 0, cb = 0, fa = 0, fm = 0, fb = 0;
        if (act) {
            ca = (double)d * len / (double)n1;
            cb = (double)(d + 1) * len / (double)n1;
            fb = integrand(a, s, sinchi, coschi, cb);
            fm = integrand(a, s, sinchi, coschi, (ca + cb) / 2.0);
        }
        const double left = __shfl_up_sync(0xffffffffu, fb, 1);
        if (act) fa = lane ? left : (d == 0 ? integrand(a, s, sinchi, coschi, ca) : carry);
        carry = __shfl_sync(0xffffffffu, fb, 31);
        const bool nz = act && (fabs(fa) + fabs(fm) + fabs(fb) > 1.0e-15);
        bool ref = false;
        double fq1 = 0, fq3 = 0;
        const double mid = (ca + cb) / 2;
        if (nz) {
            fq1 = integrand(a, s, sinchi, coschi, (mid + ca) / 2.0);
            fq3 = integrand(a, s, sinchi, coschi, (cb + mid) / 2.0);
            ref = simpson_cell(ca, cb, fa, fm, fb, fq1, fq3, err, total, my_int);
        }
        const unsigned mnz = __ballot_sync(0xffffffffu, nz), mref = __ballot_sync(0xffffffffu, ref);
        nnz += __popc(mnz);
        if (ref) {
            const int pos = nmark + 2 * __popc(mref & ((1u << lane) - 1u));
            if (pos + 1 < SETA_NCAP) {
                lst0[pos] = Cell{ca, mid, fa, fq1, fm};
                lst0[pos + 1] = Cell{mid, cb, fm, fq3, fb};
            }
        }
        nmark += 2 * __popc(mref);
    }
    if (2 * nnz > SETA_NCAP) overflow = true;  // the reference's cap: children counter beyond ncap - 2
    __syncwarp();                              // list writes visible to every lane
    total = warp_sum(total);
    my_int = warp_sum(my_int);
    Cell *cur = lst0, *nxt = lst1;
    while (!overflow && nmark > 0 && my_int > err) {
        double tl = 0.0, ml = 0.0;
        int nm2 = 0, nnz2 = 0;
        for (int base = 0; base < nmark; base += 32) {
            const int k = base + lane;
            const bool act = k < nmark;
            Cell c{0, 0, 0, 0, 0};
            if (act) c = cur[k];
            const bool nz = act && (fabs(c.fa) + fabs(c.fm) + fabs(c.fb) > 1.0e-15);
            bool ref = false;
            double fq1 = 0, fq3 = 0;
            const double mid = (c.a + c.b) / 2;
            if (nz) {
                fq1 = integrand(a, s, sinchi, coschi, (mid + c.a) / 2.0);
                fq3 = integrand(a, s, sinchi, coschi, (c.b + mid) / 2.0);
                ref = simpson_cell(c.a, c.b, c.fa, c.fm, c.fb, fq1, fq3, err, tl, ml);
            }
            const unsigned mnz = __ballot_sync(0xffffffffu, nz), mref = __ballot_sync(0xffffffffu, ref);
            nnz2 += __popc(mnz);
            if (ref) {
                const int pos = nm2 + 2 * __popc(mref & ((1u << lane) - 1u));
                if (pos + 1 < SETA_NCAP) {
                    nxt[pos] = Cell{c.a, mid, c.fa, fq1, c.fm};
                    nxt[pos + 1] = Cell{mid, c.b, c.fm, fq3, c.fb};
                }
            }
            nm2 += 2 * __popc(mref);
        }
        __syncwarp();
        if (2 * nnz2 > SETA_NCAP) overflow = true;
        total += warp_sum(tl);
        my_int = warp_sum(ml);
        nmark = nm2;
        Cell *t = cur;
        cur = nxt;
        nxt = t;
    }
    if (overflow) return nan("");
    return total * sinchi;
}

// the chi integral of one pair (dgvtools_mod.f90:532-637): cells in the
// reference's order, each sample an eps integral
__device__ double pair_integral(const SetaArgs &a, const PairState &s, Cell *warp_scratch)
{
    Cell *e0 = warp_scratch, *e1 = warp_scratch + SETA_NCAP;
    Cell *c0 = warp_scratch + 2 * SETA_NCAP, *c1 = warp_scratch + 3 * SETA_NCAP;
    const int lane = threadIdx.x & 31;
    int n1 = (int)floor(PI_SETA * s.dsph / a.ires / 2.0) + 1;
    if (n1 > SETA_NCAP) n1 = SETA_NCAP;
    const double len = PI_SETA, err = a.err_chi;
    double total = 0.0, my_int = 0.0, fprev = 0.0;
    int nmark = 0, nnz = 0;
    for (int d = 0; d < n1; d++) {
        const double ca = (double)d * len / (double)n1, cb = (double)(d + 1) * len / (double)n1;
        const double fa = d == 0 ? eps_integral(a, s, ca, e0, e1) : fprev;
        const double fb = eps_integral(a, s, cb, e0, e1);
        const double fm = eps_integral(a, s, (ca + cb) / 2.0, e0, e1);
        fprev = fb;
        if (!(fabs(fa) + fabs(fm) + fabs(fb) > 1.0e-15)) continue;
        if (++nnz > SETA_NCAP / 2) return nan("");
        const double mid = (ca + cb) / 2;
        const double fq1 = eps_integral(a, s, (mid + ca) / 2.0, e0, e1);
        const double fq3 = eps_integral(a, s, (cb + mid) / 2.0, e0, e1);
        if (simpson_cell(ca, cb, fa, fm, fb, fq1, fq3, err, total, my_int)) {
            if (lane == 0) {
                c0[nmark] = Cell{ca, mid, fa, fq1, fm};
                c0[nmark + 1] = Cell{mid, cb, fm, fq3, fb};
            }
            nmark += 2;
        }
    }
    __syncwarp();
    Cell *cur = c0, *nxt = c1;
    while (nmark > 0 && my_int > err) {
        my_int = 0.0;
        int nm2 = 0, nnz2 = 0;
        for (int k = 0; k < nmark; k++) {
            const Cell c = cur[k];
            if (!(fabs(c.fa) + fabs(c.fm) + fabs(c.fb) > 1.0e-15)) continue;
            if (++nnz2 > SETA_NCAP / 2) return nan("");
            const double mid = (c.a + c.b) / 2;
            const double fq1 = eps_integral(a, s, (mid + c.a) / 2.0, e0, e1);
            const double fq3 = eps_integral(a, s, (c.b + mid) / 2.0, e0, e1);
            if (simpson_cell(c.a, c.b, c.fa, c.fm, c.fb, fq1, fq3, err, total, my_int)) {
                if (lane == 0) {
                    nxt[nm2] = Cell{c.a, mid, c.fa, fq1, c.fm};
                    nxt[nm2 + 1] = Cell{mid, c.b, c.fm, fq3, c.fb};
                }
                nm2 += 2;
            }
        }
        __syncwarp();
        nmark = nm2;
        Cell *t = cur;
        cur = nxt;
        nxt = t;
    }
    return total;
}

__global__ void __launch_bounds__(32 * SETA_WARPS, 1) k_seta(SetaArgs a)
{
    const int lane = threadIdx.x & 31;
    const long long warp_global = (long long)blockIdx.x * SETA_WARPS + (threadIdx.x >> 5);
    Cell *ws = a.scratch + warp_global * 4 * SETA_NCAP;
    const unsigned long long nitems = (unsigned long long)a.npairs * a.P;
    for (;;) {
        unsigned long long item = 0;
        if (lane == 0) item = atomicAdd(a.next, 1ULL);
        item = __shfl_sync(0xffffffffu, item, 0);
        if (item >= nitems) break;
        const long long k = (long long)(item / a.P);
        const int p = (int)(item - (unsigned long long)k * a.P);
        const int2 pr = a.pairs[k];
        PairState s;
        s.pu = p / (a.sv * a.sw);
        s.pv = (p / a.sw) % a.sv;
        s.pw = p % a.sw;
        s.xiu = a.nu[pr.x]; s.xiv = a.nv[pr.x]; s.xiw = a.nw[pr.x];
        s.xi1u = a.nu[pr.y]; s.xi1v = a.nv[pr.y]; s.xi1w = a.nw[pr.y];
        s.varphi = basis(a, s, s.xiu, s.xiv, s.xiw) + basis(a, s, s.xi1u, s.xi1v, s.xi1w);
        const double du = s.xiu - s.xi1u, dv = s.xiv - s.xi1v, dw = s.xiw - s.xi1w;
        s.dsph = sqrt(du * du + dv * dv + dw * dw);
        s.ugu = (s.xiu - s.xi1u) / s.dsph;
        s.ugv = (s.xiv - s.xi1v) / s.dsph;
        s.ugw = (s.xiw - s.xi1w) / s.dsph;
        const double ugu = s.ugu, ugv = s.ugv, ugw = s.ugw;
        // two vectors orthogonal to g (dgvtools_mod.f90:497-525)
        if (fabs(ugw - ugv) + fabs(ugu - ugw) + fabs(ugv - ugu) < 1.0e-6) {
            s.ugux2 = ugv; s.ugvx2 = -ugu; s.ugwx2 = 0;
            s.ugux3 = ugu * ugw; s.ugvx3 = ugv * ugw; s.ugwx3 = -(ugu * ugu) - (ugv * ugv);
            s.g1 = sqrt(s.ugux2 * s.ugux2 + s.ugvx2 * s.ugvx2);
            s.g2 = sqrt(s.ugux3 * s.ugux3 + s.ugvx3 * s.ugvx3 + s.ugwx3 * s.ugwx3);
        } else {
            s.ugux2 = (ugw - ugv); s.ugvx2 = (ugu - ugw); s.ugwx2 = (ugv - ugu);
            s.ugux3 = ((ugv * ugv) - (ugv) * (ugu) - (ugw) * (ugu) + (ugw * ugw));
            s.ugvx3 = ((ugw * ugw) - (ugw) * (ugv) - (ugu) * (ugv) + (ugu * ugu));
            s.ugwx3 = ((ugu * ugu) - (ugu) * (ugw) - (ugv) * (ugw) + (ugv * ugv));
            s.g1 = sqrt(s.ugux2 * s.ugux2 + s.ugvx2 * s.ugvx2 + s.ugwx2 * s.ugwx2);
            s.g2 = sqrt(s.ugux3 * s.ugux3 + s.ugvx3 * s.ugvx3 + s.ugwx3 * s.ugwx3);
        }
        double Atemp = pair_integral(a, s, ws);
        double out = 0.0;
        if (Atemp != Atemp) {
            if (lane == 0) atomicExch(a.nan_flag, 1);
        } else if (fabs(Atemp) > a.min_sens) {
            Atemp = Atemp * a.nwt[pr.y];
            Atemp = Atemp * a.nwt[pr.x];
            out = Atemp * (s.dsph / 8.0);
        }
        if (lane == 0) a.rows64[(size_t)k * a.RD64 + 1 + p] = out;
    }
}

// (xi, xi1) of every row of the layout
__global__ void k_seta_pairs(const BlockInfo *blk, const double *rows64, int RD64, int P, int Nc, int ccell, int2 *pairs)
{
    const BlockInfo b = blk[blockIdx.x];
    for (int k = threadIdx.x; k < b.count; k += blockDim.x) {
        const long long o = __double_as_longlong(rows64[(size_t)(b.start + k) * RD64]);
        const int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
        const int l1 = (o1 - (b.c1 - ccell)) / Nc, l2 = (o2 - (b.c2 - ccell)) / Nc;
        pairs[b.start + k] = make_int2(b.c1 * P + l1, b.c2 * P + l2);
    }
}

// FP32 rows from the FP64 rows; non-zero value counts and record-shifts per block
__global__ void k_seta_finish(const BlockInfo *blk, const double *rows64, int RD64, float *rows32, int RW32, int P,
                              unsigned long long *nrec, double *rshift)
{
    const BlockInfo b = blk[blockIdx.x];
    __shared__ int cnt;
    if (threadIdx.x == 0) cnt = 0;
    __syncthreads();
    int mine = 0;
    for (long long t = threadIdx.x; t < (long long)b.count * P; t += blockDim.x) {
        const long long k = b.start + t / P;
        const int p = (int)(t % P);
        const double v = rows64[(size_t)k * RD64 + 1 + p];
        rows32[(size_t)k * RW32 + 2 + p] = __double2float_rn(v);
        mine += v != 0.0;
    }
    atomicAdd(&cnt, mine);
    __syncthreads();
    if (threadIdx.x == 0 && cnt) {
        double vol = 1.0;
        for (int d = 0; d < 3; d++) vol *= (double)(b.hi[d] - b.lo[d] + 1);
        atomicAdd(nrec, (unsigned long long)cnt);
        atomicAdd(rshift, (double)cnt * vol);
    }
}

}  // namespace

int layout_seta(Ctx *c, double Trad, double ErrChi, double ErrEps, double min_sens, int basis_mode)
{
    const Grid &g = c->grid;
    if (g.d.su > 8 || g.d.sv > 8 || g.d.sw > 8) return set_err(c, DGV_EUNSUP, "compute_A: at most 8 nodes per cell axis");
    if (!(ErrChi > 0.0) || !(ErrEps > 0.0) || min_sens < 0.0)
        return set_err(c, DGV_EINVAL, "compute_A: ErrChi, ErrEps must be positive and min_sens non-negative");
    if (basis_mode < 0 || basis_mode > 5) return set_err(c, DGV_EINVAL, "compute_A: basis_mode is 0..5");
    // pair layout of every pair whose collision sphere meets the canonical cell
    int rc = layout_synthetic(c, 0, Trad, 1);
    if (rc) return rc;
    Layout &L = c->lay;
    const int cc = g.ccell;
    SetaArgs a;
    std::memset(&a, 0, sizeof(a));
    a.npairs = L.npairs; a.P = g.P;
    a.nu = c->d_nu; a.nv = c->d_nv; a.nw = c->d_nw; a.nwt = c->d_nwt;
    a.lu = g.lu[cc]; a.ru = g.ru[cc]; a.lv = g.lv[cc]; a.rv = g.rv[cc]; a.lw = g.lw[cc]; a.rw = g.rw[cc];
    {
        double xu[8] = {0}, xv[8] = {0}, xw[8] = {0};
        for (int i = 0; i < g.d.su; i++) xu[i] = g.xu[i];
        for (int i = 0; i < g.d.sv; i++) xv[i] = g.xv[i];
        for (int i = 0; i < g.d.sw; i++) xw[i] = g.xw[i];
        DGV_CUDA(c, cudaMemcpyToSymbolAsync(c_xu, xu, sizeof(xu), 0, cudaMemcpyHostToDevice, c->stream));
        DGV_CUDA(c, cudaMemcpyToSymbolAsync(c_xv, xv, sizeof(xv), 0, cudaMemcpyHostToDevice, c->stream));
        DGV_CUDA(c, cudaMemcpyToSymbolAsync(c_xw, xw, sizeof(xw), 0, cudaMemcpyHostToDevice, c->stream));
    }
    a.su = g.d.su; a.sv = g.d.sv; a.sw = g.d.sw; a.ccell = cc;
    double hmax = std::max(a.ru - a.lu, std::max(a.rv - a.lv, a.rw - a.lw));
    a.ires = hmax / 32;
    a.err_chi = ErrChi; a.err_eps = ErrEps; a.min_sens = min_sens; a.mode = basis_mode;
    a.rows64 = (double *)L.rows64; a.RD64 = L.RD64;
    if (L.npairs == 0) return DGV_OK;
    int nsm = 148;
    DGV_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    const int nblk = nsm;  // one CTA of 8 warps per SM (up to 255 registers a thread)
    const size_t scratch = (size_t)nblk * SETA_WARPS * 4 * SETA_NCAP * sizeof(Cell);
    int2 *pairs = nullptr;
    unsigned long long *ctr = nullptr;
    Cell *ws = nullptr;
    DGV_CUDA(c, cudaMalloc(&pairs, sizeof(int2) * (size_t)L.npairs));
    DGV_CUDA(c, cudaMalloc(&ctr, 2 * sizeof(unsigned long long) + 2 * sizeof(double) + 16));
    DGV_CUDA(c, cudaMalloc(&ws, scratch));
    DGV_CUDA(c, cudaMemsetAsync(ctr, 0, 2 * sizeof(unsigned long long) + 2 * sizeof(double) + 16, c->stream));
    k_seta_pairs<<<(unsigned)L.nblocks, 256, 0, c->stream>>>(L.blk, (const double *)L.rows64, L.RD64, g.P, g.Nc, cc, pairs);
    cudaError_t e = cudaGetLastError();
    int *nan_flag = reinterpret_cast<int *>(ctr + 1);
    unsigned long long *nrec = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(ctr) + 16);
    double *rshift = reinterpret_cast<double *>(reinterpret_cast<char *>(ctr) + 24);
    if (e == cudaSuccess) {
        a.pairs = pairs; a.next = ctr; a.scratch = ws; a.nan_flag = nan_flag;
        k_seta<<<nblk, 32 * SETA_WARPS, 0, c->stream>>>(a);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) {
        k_seta_finish<<<(unsigned)L.nblocks, 256, 0, c->stream>>>(L.blk, (const double *)L.rows64, L.RD64,
                                                                   (float *)L.rows32, L.RW32, g.P, nrec, rshift);
        e = cudaGetLastError();
    }
    unsigned long long host[4] = {0, 0, 0, 0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, ctr, 32, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(pairs);
    cudaFree(ctr);
    cudaFree(ws);
    if (e != cudaSuccess) return set_err(c, DGV_ECUDA, std::string("compute_A: ") + cudaGetErrorString(e));
    int nanf = 0;
    std::memcpy(&nanf, &host[1], sizeof(int));
    if (nanf) return set_err(c, DGV_ERANGE, "compute_A: an integral exceeded the reference's cell cap (10000)");
    L.nrecords = (long long)host[2];
    double rs;
    std::memcpy(&rs, &host[3], sizeof(double));
    L.record_shifts = rs;
    return DGV_OK;
}

}  // namespace dgv
