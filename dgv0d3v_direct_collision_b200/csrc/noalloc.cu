// noalloc.cu -- dgv_collide_f64_noalloc: Q(f,f) in FP64 without any device
// allocation inside the call.
//
// Who needs it: programs that settle their device memory once, at start-up,
// and must not allocate afterwards -- a driver that hands all free memory to
// its own pool allocator (a framework's caching allocator, or a Fortran code
// that sizes every array before the time loop), or a process running under a
// fixed per-process memory budget on a shared GPU.  For them a cudaMalloc in
// the middle of the time loop either fails outright or stalls the device with
// an implicit synchronisation.  The regular entry points grow their work
// buffers on demand with cudaMalloc; this one never does.
//
// The work buffer of the FP64 collision kernel (the per-chunk partial sums
// that the fixed-order reduction adds up) lives instead in the file-scope
// array below, whose size is fixed at build time: 32 MiB on every GPU on which
// a context is created.  The CUDA runtime loads a library's device code and
// data lazily, so dgv_ctx_create loads this array on its device at once (a
// pool allocator set up after the context cannot take its room); it stays
// until the process exits.  In host code the array's name is only a stand-in
// for the device symbol, so every call asks the runtime for its device
// address (cudaGetSymbolAddress) with the context's device current and passes
// that pointer to the kernels.
#include <cuda_runtime.h>

#include <algorithm>
#include <string>

#include "dgv_internal.h"

namespace dgv {

// capacity of the shared work array, in doubles (2^22 doubles = 32 MiB)
constexpr long long NOALLOC_SCRATCH_DOUBLES = 1LL << 22;
static __device__ __align__(256) double g_noalloc_scratch[NOALLOC_SCRATCH_DOUBLES];

// Device address of g_noalloc_scratch on c's device (current), looked up on
// every call: cheap once the module is loaded, and still right after the host
// program reset the device (which unloads it).
static int noalloc_scratch(Ctx *c, double **out)
{
    double *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress((void **)&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        cudaGetLastError();
        return set_err(c, DGV_ECUDA, std::string("no-alloc scratch: cudaGetSymbolAddress failed: ") +
                                         cudaGetErrorString(e));
    }
    *out = p;
    return DGV_OK;
}

struct NoAllocArgs {
    const double *f;
    double *partial;  // [nvdf][nchunks][P][Nc] inside the static array
    const BlockInfo *blk;
    const char *rows;
    long long N, nblocks;
    int Nc, Mv, Mw, nchunks, dcta, rowb;
};

// The FP64 collision kernel with its block range computed in place (chunk k
// takes blocks [k*nblocks/nchunks, (k+1)*nblocks/nchunks)) instead of read from
// a separately allocated table.
template <int PV>
__global__ void __launch_bounds__(384, 1) k_collide_f64_noalloc(NoAllocArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    double *f_s = reinterpret_cast<double *>(smem_raw);
    const int vdf = blockIdx.x, slice = blockIdx.y, chunk = blockIdx.z;
    const double *f = a.f + (size_t)vdf * a.N;
    for (long long i = threadIdx.x; i < a.N; i += blockDim.x) {
        int cell = (int)(i / PV), l = (int)(i - (long long)cell * PV);
        f_s[l * a.Nc + cell] = __ldg(f + i);
    }
    __syncthreads();
    constexpr int RD = ((1 + PV) + 1) / 2 * 2;
    const int D = slice * a.dcta + threadIdx.x;
    const bool inD = (int)threadIdx.x < a.dcta && D < a.Nc;
    const int Du = D / (a.Mv * a.Mw), Dv = (D / a.Mw) % a.Mv, Dw = D % a.Mw;
    double acc[PV];
#pragma unroll
    for (int j = 0; j < PV; j++) acc[j] = 0.0;
    const long long b0 = a.nblocks * chunk / a.nchunks, b1 = a.nblocks * (chunk + 1) / a.nchunks;
    for (long long b = b0; b < b1; ++b) {
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
                int o1 = (int)(unsigned)(o & 0xffffffffLL), o2 = (int)(o >> 32);
                double prod = f_s[o1 + D] * f_s[o2 + D];
#pragma unroll
                for (int j = 0; j < PV; j++) acc[j] = fma(rv[1 + j], prod, acc[j]);
            }
        }
    }
    // every (vdf, chunk, p, D < Nc) entry the reduction reads is written here,
    // so the array needs no clearing between calls
    if (inD) {
        double *out = a.partial + ((size_t)vdf * a.nchunks + chunk) * PV * a.Nc;
#pragma unroll
        for (int j = 0; j < PV; j++) out[(size_t)j * a.Nc + D] = acc[j];
    }
}

__global__ void k_reduce_noalloc(const double *partial, const double *w, double *q, int nchunks, int P, int Nc,
                                 long long N, int nvdf)
{
    long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= (long long)nvdf * N) return;
    int v = (int)(idx / N);
    long long r = idx - (long long)v * N;
    int p = (int)(r / Nc), D = (int)(r - (long long)p * Nc);
    const double *src = partial + ((size_t)v * nchunks * P + p) * Nc + D;
    double s = 0.0;
    for (int ch = 0; ch < nchunks; ch++) s += src[(size_t)ch * P * Nc];
    long long i = (long long)D * P + p;
    q[(size_t)v * N + i] = 2.0 * s / w[i];
}

typedef void (*NoAllocFn)(NoAllocArgs);

static NoAllocFn noalloc_kernel(int P)
{
    switch (P) {
    case 1: return k_collide_f64_noalloc<1>;
    case 8: return k_collide_f64_noalloc<8>;
    case 27: return k_collide_f64_noalloc<27>;
    default: return nullptr;
    }
}

// Called by dgv_ctx_create with the device current: loads the module holding
// the static array (reserving its 32 MiB now rather than at the first call)
// and raises the kernel's shared-memory limit.  Failures are not fatal to the
// context; the first no-alloc call reports them.
void noalloc_prepare(Ctx *c)
{
    double *p = nullptr;
    if (noalloc_scratch(c, &p)) c->err.clear();
    NoAllocFn fn = noalloc_kernel(c->grid.P);
    const size_t smem = (size_t)c->grid.N * sizeof(double);
    int maxsm = 0;
    if (fn && cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device) == cudaSuccess &&
        smem <= (size_t)maxsm)
        cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    cudaGetLastError();
}

static int collide_noalloc(Ctx *c, const double *f, double *q, int nb, cudaStream_t st)
{
    const Grid &g = c->grid;
    const Layout &L = c->lay;
    if (!L.blk) return set_err(c, DGV_ESTATE, "collide_noalloc: no A-arrays loaded");
    if (nb < 1 || !f || !q) return set_err(c, DGV_EINVAL, "collide_noalloc: need nb >= 1 and non-NULL arrays");
    bool fdev = false, qdev = false;
    int rc = classify_ptr(c, f, &fdev);
    if (rc) return rc;
    if ((rc = classify_ptr(c, q, &qdev))) return rc;
    if (!fdev || !qdev)
        return set_err(c, DGV_EINVAL, "collide_noalloc: f and q must be device (or managed) memory of the context's device");
    NoAllocFn fn = noalloc_kernel(g.P);
    if (!fn) return set_err(c, DGV_EUNSUP, "collide_noalloc: 1, 8 or 27 nodes per cell");
    const long long per_chunk = (long long)nb * g.N;  // doubles of partials per chunk
    if (per_chunk > NOALLOC_SCRATCH_DOUBLES)
        return set_err(c, DGV_EINVAL,
                       "collide_noalloc: nb*N = " + std::to_string(per_chunk) +
                           " exceeds the fixed work array of " + std::to_string(NOALLOC_SCRATCH_DOUBLES) +
                           " doubles (32 MiB); pass fewer VDFs per call");
    int nsm = 148, maxsm = 0;
    DGV_CUDA(c, cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, c->device));
    DGV_CUDA(c, cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, c->device));
    const int nc32 = (g.Nc + 31) / 32 * 32;
    const int dcta = std::min(nc32, 384), slices = (g.Nc + dcta - 1) / dcta;
    const size_t smem = (size_t)g.N * sizeof(double);
    if (smem > (size_t)maxsm) return set_err(c, DGV_EUNSUP, "collide_noalloc: f does not fit in shared memory");
    long long want = std::max<long long>(1, 2LL * nsm / ((long long)nb * slices));
    long long fit = NOALLOC_SCRATCH_DOUBLES / per_chunk;
    int nchunks = (int)std::max<long long>(1, std::min<long long>({want, fit, std::max<long long>(1, L.nblocks), 65535LL}));
    double *scratch = nullptr;
    rc = noalloc_scratch(c, &scratch);
    if (rc) return rc;
    DGV_CUDA(c, cudaFuncSetAttribute((const void *)fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    NoAllocArgs a;
    a.f = f; a.partial = scratch; a.blk = L.blk; a.rows = (const char *)L.rows64;
    a.N = g.N; a.nblocks = L.nblocks; a.Nc = g.Nc; a.Mv = g.d.Mv; a.Mw = g.d.Mw;
    a.nchunks = nchunks; a.dcta = dcta; a.rowb = L.RD64 * 8;
    fn<<<dim3(nb, slices, nchunks), dcta, smem, st>>>(a);
    DGV_CUDA(c, cudaGetLastError());
    long long tot = (long long)nb * g.N;
    k_reduce_noalloc<<<(unsigned)((tot + 255) / 256), 256, 0, st>>>(scratch, c->d_nwt, q, nchunks, g.P, g.Nc, g.N,
                                                                     nb);
    DGV_CUDA(c, cudaGetLastError());
    if (!c->async) DGV_CUDA(c, cudaStreamSynchronize(st));
    return DGV_OK;
}

}  // namespace dgv

extern "C" int dgv_collide_f64_noalloc(dgv_ctx *ctx, const double *f, double *q, int32_t nb, void *stream)
{
    if (!ctx) return DGV_EINVAL;
    dgv::Ctx *c = &ctx->c;
    c->err.clear();
    if (cudaSetDevice(c->device) != cudaSuccess) return dgv::set_err(c, DGV_ECUDA, "cudaSetDevice failed");
    return dgv::collide_noalloc(c, f, q, nb, stream ? (cudaStream_t)stream : c->stream);
}
