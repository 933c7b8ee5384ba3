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
// vA*f(b) to g(a) and vA*f(a) to g(b) with FP64 atomic adds.
#include <cuda_runtime.h>

#include <algorithm>

#include "dgv_internal.h"

namespace dgv {

struct VjpArgs {
    const double *f, *v, *w;
    double *g;
    const BlockInfo *blk;
    const char *rows;
    const int *bounds;
    long long N;
    int Nc, Mv, Mw, dcta, rowb;
};

template <int PV>
__global__ void __launch_bounds__(384, 1) k_vjp_scatter(VjpArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *f_s = reinterpret_cast<double *>(smem_raw);
    const int chunk = blockIdx.x, slice = blockIdx.y;
    for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
        int cell = (int)(i / PV), l = (int)(i - (long long)cell * PV);
        f_s[l * a.Nc + cell] = __ldg(a.f + i);
    }
    __syncthreads();
    constexpr int RD = ((1 + PV) + 1) / 2 * 2;
    const int D = slice * a.dcta + threadIdx.x;
    const bool inD = (int)threadIdx.x < a.dcta && D < a.Nc;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    double cw[PV];
#pragma unroll
    for (int j = 0; j < PV; j++) {
        long long i = (long long)D * PV + j;
        cw[j] = inD ? 2.0 * a.v[i] / a.w[i] : 0.0;
    }
    const int b0 = a.bounds[chunk], b1 = a.bounds[chunk + 1];
    for (int b = b0; b < b1; ++b) {
        const BlockInfo bi = a.blk[b];
        const bool valid = inD && Du >= bi.lo[0] && Du <= bi.hi[0] && Dv >= bi.lo[1] && Dv <= bi.hi[1] &&
                           Dw >= bi.lo[2] && Dw <= bi.hi[2];
        if (!__any_sync(0xffffffffu, valid)) continue;
        const double2 *row = reinterpret_cast<const double2 *>(a.rows + (size_t)bi.start * a.rowb);
        for (int k = 0; k < bi.count; ++k, row += RD / 2) {
            double rv[RD];
#pragma unroll
            for (int t = 0; t < RD / 2; t++) {
                double2 x = __ldg(row + t);
                rv[2 * t] = x.x;
                rv[2 * t + 1] = x.y;
            }
            if (valid) {
                long long o = __double_as_longlong(rv[0]);
                int q1 = (int)(unsigned)(o & 0xffffffffLL) + D, q2 = (int)(o >> 32) + D;
                double vA = 0.0;
#pragma unroll
                for (int j = 0; j < PV; j++) vA = fma(rv[1 + j], cw[j], vA);
                int l1 = q1 / a.Nc, l2 = q2 / a.Nc;
                long long i1 = (long long)(q1 - l1 * a.Nc) * PV + l1;
                long long i2 = (long long)(q2 - l2 * a.Nc) * PV + l2;
                atomicAdd(a.g + i1, vA * f_s[q2]);
                atomicAdd(a.g + i2, vA * f_s[q1]);
            }
        }
    }
}

typedef void (*VjpFn)(VjpArgs);

int vjp_device(Ctx *c, const double *d_f, const double *d_v, double *d_g, int precision)
{
    (void)precision;
    if (!c->lay.blk) return set_err(c, DGV_ESTATE, "vjp: no A-arrays loaded");
    const Grid &g = c->grid;
    VjpFn fn = nullptr;
    switch (g.P) {
    case 1: fn = k_vjp_scatter<1>; break;
    case 8: fn = k_vjp_scatter<8>; break;
    case 27: fn = k_vjp_scatter<27>; break;
    default: return set_err(c, DGV_EUNSUP, "vjp: this build supports 1, 8 or 27 nodes per cell");
    }
    int nc32 = (g.Nc + 31) / 32 * 32;
    int dcta = std::min(nc32, 384), slices = (g.Nc + dcta - 1) / dcta;
    size_t smem = (size_t)g.N * sizeof(double);
    int maxsm = 0, nsm = 148;
    DGV_CUDA(c, cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    DGV_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    if (smem > (size_t)maxsm) return set_err(c, DGV_EUNSUP, "vjp: f does not fit in shared memory for this grid");
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int nchunks = std::max(1, std::min<int>(2 * nsm / slices, (int)std::max<long long>(1, c->lay.nblocks)));
    int *d_bounds = nullptr;
    int rc = get_chunks(c, nchunks, &d_bounds);
    if (rc) return rc;
    DGV_CUDA(c, cudaMemsetAsync(d_g, 0, sizeof(double) * (size_t)g.N, c->stream));
    VjpArgs a;
    a.f = d_f; a.v = d_v; a.w = c->d_nwt; a.g = d_g; a.blk = c->lay.blk; a.rows = (const char *)c->lay.rows64;
    a.bounds = d_bounds; a.N = g.N; a.Nc = g.Nc; a.Mv = g.d.Mv; a.Mw = g.d.Mw; a.dcta = dcta;
    a.rowb = c->lay.RD64 * 8;
    fn<<<dim3(nchunks, slices, 1), dcta, smem, c->stream>>>(a);
    DGV_CUDA(c, cudaGetLastError());
    return DGV_OK;
}

}  // namespace dgv
