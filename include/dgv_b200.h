/*
 * dgv_b200.h -- C-ABI of the B200 collision library (libdgv_b200.so).
 *
 * Drop-in boundary for the hot path of the DG-velocity Boltzmann solver: the
 * direct evaluation of the collision integral Q(f,f) and the Runge-Kutta /
 * Adams-Bashforth stepping that calls it.  Every entry point is `extern "C"`,
 * takes plain pointers and sizes, returns an int status (never aborts) and is
 * bind(C)-compatible for a Fortran ISO_C_BINDING interface.  Each declaration
 * names the reference routine (file:line) it replaces.
 *
 * Conventions
 *   - A context (dgv_ctx) owns one uniform velocity grid, the device copy of
 *     the collision-information A-arrays and all device work buffers.  It is
 *     not thread-safe; use one context per host thread.
 *   - Node arrays (f, q, ...) have N = Mu*Mv*Mw*su*sv*sw entries in the
 *     reference's node order: cell-major (u outer, v, w inner), then the local
 *     node (ui, vi, wi) with wi fastest (miscset.f90:882-937, 1112-1183).
 *   - Array pointers may be host memory (copied through device staging
 *     buffers inside the call) or device memory (used in place); the library
 *     asks the CUDA runtime which.  With host pointers every call is
 *     synchronous; with device pointers the work is ordered on the context's
 *     stream and the call returns after it completes, unless dgv_set_async(1).
 *   - Node indices passed in (A_xi, A_xi1) are 1-based when one_based != 0,
 *     as the reference stores them.
 */
#ifndef DGV_B200_H
#define DGV_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DGV_OK 0
#define DGV_EINVAL 1   /* bad size, layout or argument                       */
#define DGV_ERANGE 2   /* an index points outside the grid                    */
#define DGV_ECUDA 3    /* a CUDA runtime call failed                          */
#define DGV_ETIMEOUT 4 /* a bounded device wait gave up                       */
#define DGV_ENOMEM 5   /* device or host allocation failed                    */
#define DGV_ESTATE 6   /* call out of order (e.g. no A-arrays loaded yet)     */
#define DGV_EUNSUP 7   /* configuration this build does not support           */

/* arithmetic of the collision kernel */
#define DGV_PREC_F64 0  /* plain FP64 gather-multiply-accumulate               */
#define DGV_PREC_F32C 1 /* FP32 products, compensated (two-sum) accumulation   */
#define DGV_PREC_TC 2   /* tensor cores (tcgen05): split-fp16 hi+lo products,  */
                        /* FP32 accumulation, compensated per-block flush,     */
                        /* FP64 final sums; at most 32 nodes per cell          */

/* options for dgv_set_option */
#define DGV_OPT_PROJECT 1  /* 1: apply the FP64 conservation projection to Q  */
#define DGV_OPT_NCHUNKS 2  /* work chunks per VDF (0 = autotune)             */
#define DGV_OPT_KTIMING 3  /* 1: time the collision kernel with CUDA events   */
                           /* on the context stream (read: dgv_kernel_stats)  */
#define DGV_OPT_TCFORM 4   /* tensor-core form: 2 (default) = dense cell-pair */
                           /* blocks (f(c2) x W on the tensor core, then      */
                           /* f(c1) on the CUDA cores; grids of 8 or 27 nodes */
                           /* per cell, others use form 1), 1 = pair chunks   */
                           /* (products formed per pair on the CUDA cores)    */
#define DGV_OPT_TCTILES 5  /* block form: VDF tiles of 128 per CTA, 2 (one W  */
                           /* read from L2 per 256 rows, one accumulator per  */
                           /* tile) or 1 (two accumulators per tile)          */
#define DGV_OPT_TCSETMB 6  /* block form: MB of block records per kernel     */
                           /* launch (default 48; a launch's records are read */
                           /* by all its CTAs, so they should stay in L2)     */
#define DGV_OPT_WAIT_LIMIT_US 7  /* microseconds after which a bounded wait   */
                                 /* of a collision kernel (block form, FP64,  */
                                 /* FP32-compensated, mixed terms, adjoint)   */
                                 /* gives up (0 = 4 s); the call then returns */
                                 /* DGV_ETIMEOUT                              */
#define DGV_OPT_TCAUTOTUNE 9      /* block form: 1 (default) = on the first    */
                                 /* evaluation of each batch class, time VDF  */
                                 /* tiles per CTA x records per launch x      */
                                 /* persistent or not, keep the fastest; 0 =  */
                                 /* the options' values (setting _TCTILES,    */
                                 /* _TCSETMB or _TCPERSIST also switches the  */
                                 /* tuning off)                               */
#define DGV_OPT_TCPERSIST 11     /* block form: 1 = one persistent launch (one */
                                 /* CTA per SM) over all sets of records,     */
                                 /* each set's sums added in set order; 0 =   */
                                 /* one launch per set (same results, bit for */
                                 /* bit)                                      */
#define DGV_OPT_FGLOBAL 10        /* CUDA-core kernels (FP64, FP32-compensated, */
                                 /* mixed terms, FP64 adjoint): 0 (default) = */
                                 /* f of a VDF staged in shared memory when   */
                                 /* it fits, else gathered from a local-major */
                                 /* copy in global memory (L1/L2); 1 = always */
                                 /* the global copy                           */
#define DGV_OPT_TEST_WITHHOLD 8  /* 1: test of the bounded waits: the next    */
                                 /* block-form call leaves one of its copies  */
                                 /* unissued, so its waits run out and it     */
                                 /* returns DGV_ETIMEOUT; resets itself       */

/* layouts for dgv_release_layouts */
#define DGV_LAYOUT_F32 1      /* FP32 rows of the pair layout (FP32-compensated Q) */
#define DGV_LAYOUT_TC_CHUNK 2 /* records of the tensor-core chunk form          */
#define DGV_LAYOUT_TC_BLOCK 4 /* records of the block form and of its adjoint   */
#define DGV_LAYOUT_TC_ADJ 8   /* only the adjoint's second record set           */

typedef struct dgv_ctx dgv_ctx;

/* Uniform velocity grid (SetDGVblzmmesh + Set3DCellsR_DGVblzm + SetNodesDGV,
 * miscset.f90:210-431, 544-597, 1112-1183) and the dimensionless collision
 * scale kappa = (mol_diam/L_inf)^2 * N_inf (spat_oper_mod.f90:65). */
typedef struct {
    int32_t su, sv, sw;  /* Gauss-Legendre nodes per cell per axis */
    int32_t Mu, Mv, Mw;  /* cells per axis                        */
    double u_L, u_R, v_L, v_R, w_L, w_R;
    double kappa;
} dgv_grid_desc;

/* -- context ------------------------------------------------------------ */
/* Builds the grid, nodes, weights and the canonical cell (the cell holding
 * v = 0, FindCellContainsPoint_DGV dgvtools_mod.f90:1175-1247) on `device`.
 * Replaces the setup sequence of DGVblzmPL.f90:75-105. */
int dgv_ctx_create(const dgv_grid_desc *desc, int device, dgv_ctx **out);
int dgv_ctx_destroy(dgv_ctx *ctx);
/* message of the last failing call on this context ("" if none) */
const char *dgv_last_error(const dgv_ctx *ctx);
/* run on a caller-owned cudaStream_t (NULL = the context's own stream) */
int dgv_set_stream(dgv_ctx *ctx, void *stream);
/* 1: device-pointer calls return without synchronising the stream */
int dgv_set_async(dgv_ctx *ctx, int async_flag);
int dgv_set_option(dgv_ctx *ctx, int option, int64_t value);
/* No counterpart in the reference (configuration query): the current value
 * of an option (for DGV_OPT_TCTILES / DGV_OPT_TCSETMB: the choice the
 * autotuner made for the last batch class evaluated) */
int dgv_get_option(dgv_ctx *ctx, int option, int64_t *value);
/* Frees device layouts the caller does not need (DGV_LAYOUT_* mask): the FP32
 * rows (7 GB at 27^3, built when A is loaded), the records of either
 * tensor-core form (built on first use: 8 GB chunk, 12 GB block, 12 GB more for
 * the block form's adjoint at 27^3).  Each is rebuilt on its next use, with the
 * same values (FP32 rows from the FP64 rows, records from the pair layout);
 * CUDA graphs of the context are released.  *freed_bytes (may be NULL) gets
 * the change in the device's free memory.  No counterpart in the reference. */
int dgv_release_layouts(dgv_ctx *ctx, int mask, int64_t *freed_bytes);
/* No counterpart in the reference (measurement hook): summed device time in
 * ms and launch count of the collision kernel (k_collide_tc / k_collide_pipe)
 * over the calls made since the last reset while DGV_OPT_KTIMING was on,
 * and the number of kernels of this library those calls launched.
 * Synchronises on the recorded events; reset != 0 clears the sums. */
int dgv_kernel_stats(dgv_ctx *ctx, double *ms, int64_t *launches, int64_t *all_launches, int reset);
/* No counterpart in the reference (measurement hook): the work plan of one
 * DGV_PREC_TC evaluation of nvdf VDFs in the current tensor-core form --
 * kernel launches, work items summed over the VDF tiles, and the FLOPs the
 * MMAs issue (dense tiles, all split products), for tensor-pipe rooflines.
 * Builds the device records and work lists if they do not exist yet. */
int dgv_tc_plan(dgv_ctx *ctx, int32_t nvdf, int64_t *launches, int64_t *items, double *tensor_flop);
/* N, P = su*sv*sw, number of cells, canonical cell (0-based) */
int dgv_grid_info(const dgv_ctx *ctx, int64_t *N, int32_t *P, int32_t *Nc, int32_t *ccell);
/* host copies of nodes_u/_v/_w/_gwts (miscset.f90:1112-1183); any may be NULL */
int dgv_nodes(const dgv_ctx *ctx, double *u, double *v, double *w, double *gwts);

/* -- A-arrays ------------------------------------------------------------- */
/* Uploads A-arrays in the reference layout (commvar.f90:157-167, as read by
 * ReadAarraysDGV readwrite.f90:1066-1118): capphi[N] records per node,
 * records of node k contiguous in node order; A[nnz], A_xi[nnz], A_xi1[nnz].
 * Only the records of canonical-cell nodes are used, as in
 * EvalCollisionPeriodicAPlus_DGV (collision_mod.f90:186-188).  Converts them
 * once to the device pair layout; replaces ReadAarrays* + the A part of
 * SetCellsUGINdsSftArrs (miscset.f90:1202-1311). */
int dgv_load_A(dgv_ctx *ctx, int64_t nnz, const int32_t *capphi, const double *A,
               const int32_t *A_xi, const int32_t *A_xi1, int one_based);
/* Generates synthetic A-arrays on the device with the reference's record
 * structure: every pair xi<xi1 that passes the SetA_DGV prefilter
 * (dgvtools_mod.f90:527, cutoff Trad) and, for support_mode 1, whose
 * collision sphere meets the canonical cell, one record per canonical basis
 * function with value w_xi*w_xi1*|g|/8*u, u = splitmix64 hash of
 * (seed, p, xi, xi1) in [-1,1).  No reference counterpart: a seeded stand-in
 * for A-arrays that take hours to precompute. */
int dgv_generate_A_synthetic(dgv_ctx *ctx, uint64_t seed, double Trad, int support_mode);
/* Computes the A-arrays on the device: SetA_DGV (dgvtools_mod.f90:377-681,
 * with A_IntEpsilon :988-1122 and EvalPhiPostCollIntegrand :938-975) for every
 * basis function of the canonical cell -- nested adaptive Simpson integrals
 * over the collision sphere of every pair xi < xi1 passing the prefilter
 * (cutoff Trad), tolerances ErrChi (chi) and ErrEps (eps), records with
 * |A| > min_sens kept.  basis_mode 0 is the Lagrange basis with the
 * commented lines of :254-287 restored; 1..5 put the collision invariants
 * 1, u, v, w, |v|^2 in place of the basis function (the known-answer test
 * of :267-274: every record ~ 0).  Replaces the precompute whose output
 * ReadAarraysDGV reads. */
int dgv_compute_A(dgv_ctx *ctx, double Trad, double ErrChi, double ErrEps, double min_sens, int basis_mode);
/* counts of the loaded A-arrays: records, distinct (xi,xi1) pairs, cell-pair
 * blocks, and record-shift visits per Q evaluation */
int dgv_A_info(const dgv_ctx *ctx, int64_t *nrecords, int64_t *npairs, int64_t *nblocks,
               double *record_shifts);
/* Copies the loaded A-arrays back in the reference layout, 0-based, records
 * of each canonical basis function grouped by cell pair; nnz_out receives the
 * count.  Pass NULL arrays to query the size. */
int dgv_export_A(const dgv_ctx *ctx, int64_t *nnz_out, int32_t *capphi, double *A,
                 int32_t *A_xi, int32_t *A_xi1);

/* -- A-array files (the reference's on-disk operator) --------------------- */
/* Reads the A-arrays of an operator file (WriteAarraysDGV's format,
 * readwrite.f90:1459-1484: a Fortran unformatted sequential file of the
 * records (mm, nn) and (A_capphi, A, A_xi, A_xi1, A_phi), gfortran record
 * framing, subrecords for records over 2^31-9 bytes), or of a chunked
 * operator split over nfiles files (ReadAarraysChnksDGV,
 * readwrite.f90:1130-1243: A_capphi summed, records concatenated in file
 * order), and loads them into the context as dgv_load_A does. */
int dgv_read_A_files(dgv_ctx *ctx, const char *const *paths, int32_t nfiles);
/* Writes the loaded A-arrays as one operator file in that format
 * (WriteAarraysDGV, readwrite.f90:1459-1484); max_subrecord = 0 for
 * gfortran's limit, a smaller positive value splits records sooner. */
int dgv_write_A_file(dgv_ctx *ctx, const char *path, int64_t max_subrecord);
/* The same reader without a context or a GPU (ReadAarraysChnksDGV,
 * readwrite.f90:1130-1243): fills caller arrays, indices 1-based as stored;
 * NULL arrays query nnz_out only.  Errors: dgv_file_error(). */
int dgv_read_A_arrays(const char *const *paths, int32_t nfiles, int32_t N, int64_t *nnz_out,
                      int32_t *capphi, double *A, int32_t *A_xi, int32_t *A_xi1);
/* The same writer from caller arrays (WriteAarraysDGV, readwrite.f90:1459-1484),
 * indices 1-based; A_phi is derived from capphi. */
int dgv_write_A_arrays(const char *path, int32_t N, int64_t nnz, const int32_t *capphi, const double *A,
                       const int32_t *A_xi, const int32_t *A_xi1, int64_t max_subrecord);
/* message of the last failing dgv_read_A_arrays / dgv_write_A_arrays on this
 * thread (the file routines of readwrite.f90:1066-1484 stop on errors) */
const char *dgv_file_error(void);

/* -- collision operator --------------------------------------------------- */
/* q = Q(f,f) (EvalCollisionPeriodicAPlus_DGV, collision_mod.f90:143-229);
 * n must equal N. */
int dgv_collide(dgv_ctx *ctx, const double *f, double *q, int64_t n, int precision);
/* nb VDFs stored contiguously, f[nb][N] -> q[nb][N] */
int dgv_collide_batched(dgv_ctx *ctx, int32_t nb, const double *f, double *q, int precision);
/* One mixed batch over n velocity grids (one context per grid, all on one
 * device): q[k][nb[k]][N_k] = Q(f[k]) on ctxs[k]'s grid, device pointers
 * only.  The members run on their contexts' streams, forked from and joined
 * back to `stream` (NULL = ctxs[0]'s stream).  The first call for a member
 * list runs eagerly, the second captures the group in one CUDA graph, later
 * calls replay it with one launch; a context whose buffers or A-arrays change
 * drops the graphs it belongs to.  Errors are reported on ctxs[0].  The
 * reference evaluates each VDF with EvalCollisionPeriodicAPlus_DGV
 * (collision_mod.f90:143-229) on one grid per run. */
int dgv_collide_group(int32_t n, dgv_ctx *const *ctxs, const int32_t *nb, const double *const *f,
                      double *const *q, int precision, void *stream);
/* fcol = kappa*dt*Q(f,f) (SpatialOperSH_DGV, spat_oper_mod.f90:28-68); with
 * run modes switched on (dgv_set_regime) the mode of CheckSolutionMode_DGV
 * decides: Q(f), L(Df) + Q(Df) or L(Df), Df = f - fm */
int dgv_spatial_oper(dgv_ctx *ctx, const double *f, double *fcol, double dt, int precision);
/* Switches on the run modes of SpatialOperSH_DGV for dgv_spatial_oper and the
 * RK / AB steps (CheckSolutionMode_DGV, spat_oper_mod.f90:195-272, levels
 * decomp_lev and linear_lev of commvar): relative L1 distance of f to its
 * local Maxwellian below decomp_lev -> decomposition (mode 1), below
 * linear_lev -> linearised (mode 2), else the full operator (mode 0).
 * decomp_lev = 0 switches them off.  Resets the mode to 0; the mode's
 * linearisation point fm is also the one dgv_apply_linear uses.  RK steps
 * are not captured into graphs while modes are on. */
int dgv_set_regime(dgv_ctx *ctx, double decomp_lev, double linear_lev);
/* current run_mode and the last relative L1 distance (-1 before the first
 * check), as CheckSolutionMode_DGV (spat_oper_mod.f90:195-272) and
 * KeepTrackL1_err_DGV record them */
int dgv_regime_info(const dgv_ctx *ctx, int32_t *run_mode, double *last_L1);
/* Q on the output cells [cell0, cell1) only: q[nb][(cell1-cell0)*P], node
 * order within the range.  The MPI split of output nodes over ranks
 * (miscmpiset.f90:195-200, 1017-1098; each rank's share of the loop of
 * collision_mod.f90:186-227): one rank of a sharded single-VDF run evaluates
 * its cells and the slices are gathered.  FP64 or FP32-compensated; no
 * conservation projection (it needs the whole Q). */
int dgv_collide_cells(dgv_ctx *ctx, int32_t nb, const double *f, double *q, int32_t cell0, int32_t cell1,
                      int precision);
/* No counterpart in the reference.  q = Q(f,f) in FP64, as dgv_collide_batched,
 * for callers that cannot allocate device memory once they are running -- a
 * driver that gives all free memory to its own pool allocator at start-up, or
 * a process held to a fixed memory budget on a shared GPU, where a cudaMalloc
 * in the time loop would fail or stall the device.  This call allocates
 * nothing: f and q are caller-owned device arrays [nb][N] of the context's
 * device, and the kernel's partial sums go to a static 32 MiB device array.
 * The CUDA runtime loads device data lazily, so dgv_ctx_create loads that
 * array on its device: create the context before a pool allocator takes the
 * free memory; the 32 MiB stay reserved until the process exits.  Each call
 * looks up the array's device address (no allocation); after the host program
 * resets the device, make the next call outside any stream capture (the
 * lookup reloads the array).  Limit: nb*N <= 4194304 (2^22) doubles, else
 * DGV_EINVAL.  All calls share the array and leave their partial sums in it:
 * calls that overlap on the GPU (other streams or host threads) race, so
 * serialise them.  No conservation projection.  stream NULL = the context's
 * stream. */
int dgv_collide_f64_noalloc(dgv_ctx *ctx, const double *f, double *q, int32_t nb, void *stream);

/* -- time integration ------------------------------------------------------ */
/* One optimal Runge-Kutta step of order 1..5 in place on f
 * (TimeIntegratorORK_SH_DGV, time_integr_mod.f90:26-152).  frhs1 (may be NULL)
 * receives the first-stage right side divided by dt, as the reference leaves
 * it in commvar's frhs1. */
int dgv_step_rk(dgv_ctx *ctx, double *f, double *frhs1, double dt, int order, int precision);
/* One RK step of order 1..5 for nb VDFs stored contiguously (f[nb][N], in
 * place; frhs1 [nb][N] or NULL): TimeIntegratorORK_SH_DGV
 * (time_integr_mod.f90:26-152) applied to every VDF, with each stage's Q of
 * the whole batch evaluated in one call (the tensor-core path evaluates it
 * in one pass); captured into a CUDA graph from the second call with the
 * same arrays, as dgv_step_rk.  Run modes (dgv_set_regime) are per VDF:
 * with them on, nb > 1 gives DGV_EUNSUP. */
int dgv_step_rk_batched(dgv_ctx *ctx, int32_t nb, double *f, double *frhs1, double dt, int order, int precision);
/* Adams-Bashforth start-up: order-1 RK steps of that order, filling the
 * right-side history kept in the context (PrepareMTS_SH_DGV, time_integr_mod.f90:443-569). */
int dgv_prepare_ab(dgv_ctx *ctx, double *f, double dt, int order, int precision);
/* One Adams-Bashforth step of the order given to dgv_prepare_ab
 * (TimeIntegratorMTS_SH_DGV, time_integr_mod.f90:314-364). */
int dgv_step_ab(dgv_ctx *ctx, double *f, double dt, int precision);
/* Writes a solution file (WriteSol_DGV, readwrite.f90:1756-1796): Fortran
 * unformatted sequential records (e_time, dt), (rkmts), (N) and
 * (f, f1..f(rkmts-1), frhs1..frhs(rkmts-1)), rkmts = the order given to
 * dgv_prepare_ab (1 before it), frhs* = the context's Adams-Bashforth right
 * sides.  f1..f4 are written as zeros: the multistep formulas never read
 * them.  f may be a host or a device pointer. */
int dgv_write_solution(dgv_ctx *ctx, const char *path, const double *f, double e_time, double dt);
/* Reads such a file (RestartSolutionDGV, readwrite.f90:2389-2513) into f
 * (host or device) and the context's Adams-Bashforth history, so that
 * dgv_step_ab continues with order rkmts; e_time / dt may be NULL.  A file
 * whose N differs from the grid's is refused, as the reference refuses it. */
int dgv_read_solution(dgv_ctx *ctx, const char *path, double *f, double *e_time, double *dt);
/* The same solution files without a context or a GPU (WriteSol_DGV,
 * readwrite.f90:1756-1796): arrays holds f, f1..f(rkmts-1),
 * frhs1..frhs(rkmts-1), (2 rkmts - 1) N doubles.  Errors: dgv_file_error(). */
int dgv_write_solution_arrays(const char *path, int32_t N, int32_t rkmts, double e_time, double dt,
                              const double *arrays);
/* (RestartSolutionDGV, readwrite.f90:2485-2507) any output may be NULL;
 * call with arrays = NULL first to learn N and rkmts. */
int dgv_read_solution_arrays(const char *path, int32_t *N, int32_t *rkmts, double *e_time, double *dt,
                             double *arrays);

/* -- moments, equilibrium, conservation ----------------------------------- */
/* out = n, ubar, vbar, wbar, T (MassCheckRec, dgvtools_mod.f90:1437-1458) */
int dgv_moments(dgv_ctx *ctx, const double *f, double out[5]);
/* f = n exp(-|v-u0|^2/T)/(pi T)^{3/2} at every node (maxwelveldist,
 * distributions_mod.f90:83-95) */
int dgv_maxwellian(dgv_ctx *ctx, double T, double u0, double v0, double w0, double n,
                   double *f);
/* In place, FP64: removes from q its components along the collision
 * invariants 1,u,v,w,|v|^2 in the quadrature inner product, so that the
 * moments the reference monitors (dgvtools_mod.f90:1680-1691) vanish. */
int dgv_project(dgv_ctx *ctx, double *q, int32_t nb);

/* -- derivatives ----------------------------------------------------------- */
/* q = 2/w * sum A (f(xi) df(xi1) + df(xi) f(xi1)): the Jacobian-vector product
 * of Q at f (EvalCollisionPeriodicMixedTermsA_DGV, collision_mod.f90:244-332).
 * FP64 only: other precisions give DGV_EUNSUP (as dgv_apply_linear). */
int dgv_jvp(dgv_ctx *ctx, const double *f, const double *df, double *q, int precision);
/* g = J(f)^T v: the vector-Jacobian product of Q at f; g_k = sum_i v_i dQ_i/df_k.
 * Adjoint of collision_mod.f90:213-216; equals 2*fmA*v at a Maxwellian
 * (collision_mod.f90:448-449, 357).  precision DGV_PREC_F64 or DGV_PREC_TC
 * (as dgv_vjp_batched); DGV_PREC_F32C gives DGV_EUNSUP. */
int dgv_vjp(dgv_ctx *ctx, const double *f, const double *v, double *g, int precision);
/* The same for nb VDFs stored contiguously: g[b] = J(f[b])^T v[b].
 * DGV_PREC_F64: the FP64 kernel per VDF.  DGV_PREC_TC: all VDFs in one pass
 * of the block form on the tensor cores (8 or 27 nodes per cell): per
 * cell-pair block the forward's product f(c2) W and the product f(c1) W'
 * (the block's values with the two nodes' roles swapped), both contracted
 * with c = 2v/w; split-fp16 operands, FP32 accumulation with compensated
 * block sums, FP64 final sums.  The first call builds the adjoint's block
 * records: twice the device memory of the forward's.  The reference has no
 * adjoint: this is the transpose of the loop of collision_mod.f90:186-227,
 * and 2*fmA*v of collision_mod.f90:448-449 at a Maxwellian. */
int dgv_vjp_batched(dgv_ctx *ctx, int32_t nb, const double *f, const double *v, double *g, int precision);
/* Stores the linearisation point fm (PrepareFMA_DGV, collision_mod.f90:377-464).
 * The dense N x N fmA is not materialised; dgv_apply_linear is matrix-free. */
int dgv_prepare_linear(dgv_ctx *ctx, const double *fm);
/* q = 2*MATMUL(df, fmA) at the stored fm (EvalCollisionLinear,
 * collision_mod.f90:346-359) */
int dgv_apply_linear(dgv_ctx *ctx, const double *df, double *q, int precision);

#ifdef __cplusplus
}
#endif
#endif /* DGV_B200_H */
