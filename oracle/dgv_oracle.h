/*
 * dgv_oracle.h -- CPU FP64 restatement of the reference's collision hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker: it is called by
 * tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg.  The
 * product (dgv0d3v_direct_collision_b200) never links, imports or calls it.
 *
 * Parity status: the reference (Fortran 90 + MPI) cannot be compiled here (no
 * Fortran compiler, no MPI headers) and ships no tests, fixtures or golden
 * vectors, so this restatement is "parity unpinned" against reference outputs.
 * It is pinned instead by invariants the reference itself relies on:
 *   - the collision-invariant known-answer test of SetA_DGV
 *     (dgvtools_mod.f90:254-287: with phi replaced by 1,u,v,w,|v|^2 every
 *     A-record vanishes),
 *   - agreement of the two reference Q routines it restates
 *     (collision_mod.f90:29-129 vs :143-229) and of the unshifted
 *     IphiDGV (dgvtools_mod.f90:847-877) on canonical-cell nodes,
 *   - agreement with an independent pure-Python loop restatement
 *     (tests/golden/make_golden.py) whose outputs are committed as fixtures.
 *
 * Indices are 0-based everywhere in this API unless an argument says
 * otherwise; the reference's are 1-based.
 */
#ifndef DGV_ORACLE_H
#define DGV_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t su, sv, sw;       /* Gauss nodes per cell per axis (reference su,sv,sw) */
    int32_t Mu, Mv, Mw;       /* cells per axis (reference Mu,Mv,Mw)                */
    double u_L, u_R, v_L, v_R, w_L, w_R;
} dgvo_grid_desc;

typedef struct dgvo_ctx dgvo_ctx;

dgvo_ctx *dgvo_create(const dgvo_grid_desc *d);
void dgvo_destroy(dgvo_ctx *c);

/* sizes: N nodes, P = su*sv*sw nodes per cell, Nc cells, canonical cell */
int64_t dgvo_num_nodes(const dgvo_ctx *c);
int32_t dgvo_nodes_per_cell(const dgvo_ctx *c);
int32_t dgvo_num_cells(const dgvo_ctx *c);
int32_t dgvo_canonical_cell(const dgvo_ctx *c);

/* node tables (miscset.f90:1112-1183): coordinates, weights, parent cell, local indices */
void dgvo_get_nodes(const dgvo_ctx *c, double *u, double *v, double *w, double *gwts,
                    int32_t *pcell, int32_t *ui, int32_t *vi, int32_t *wi);
/* cell integer coordinates (miscset.f90:1245-1277) and bounds */
void dgvo_get_cells(const dgvo_ctx *c, int32_t *ugi, int32_t *vgi, int32_t *wgi,
                    double *lu, double *ru, double *lv, double *rv, double *lw, double *rw);
/* Gauss-Legendre rule on [-1,1] (replaces GauLeg, gaussian_mod.f90:4) */
void dgvo_gauss_legendre(int n, double *x, double *w);
/* cell containing a point, -1 if none (dgvtools_mod.f90:1175-1247) */
int32_t dgvo_find_cell(const dgvo_ctx *c, double u, double v, double w);

/* A-arrays in the reference layout (commvar.f90:157-167).  capphi has N entries
 * (one per node); records of node k are contiguous and ordered by node.  Builds
 * the shift tables of SetCellsUGINdsSftArrs (miscset.f90:1202-1311). */
int dgvo_set_A(dgvo_ctx *c, const int32_t *capphi, int64_t nnz, const double *A,
               const int32_t *xi, const int32_t *xi1, int one_based);
void dgvo_get_shift_tables(const dgvo_ctx *c, int32_t *dui, int32_t *dvi, int32_t *dwi,
                           int32_t *phican, int64_t *Ashift);

/* Q (collision_mod.f90:143-229).  nodes==NULL evaluates every node; otherwise
 * only the listed nodes (fc has N entries, unlisted entries left untouched). */
void dgvo_collide_aplus(const dgvo_ctx *c, const double *f, double *fc,
                        const int64_t *nodes, int64_t nnodes, int nthreads);
/* same Q through compacted scratch arrays (collision_mod.f90:29-129) */
void dgvo_collide_a(const dgvo_ctx *c, const double *f, double *fc);
/* unshifted moments of Q for the basis functions that own records, scaled by kappa
 * (dgvtools_mod.f90:847-877) */
void dgvo_iphi(const dgvo_ctx *c, const double *f, double kappa, double *iphi);
/* cross term 2/w sum A (fm(xi) f(xi1) + f(xi) fm(xi1)) (collision_mod.f90:244-332) */
void dgvo_mixed_terms(const dgvo_ctx *c, const double *f, const double *fm, double *fc,
                      int nthreads);
/* dense linearised operator fmA (N x N, column-major: fmA[k + N*i]) (collision_mod.f90:377-464) */
void dgvo_prepare_fma(const dgvo_ctx *c, const double *fm, double *fmA);
/* fc = 2 * MATMUL(f, fmA) (collision_mod.f90:346-359) */
void dgvo_eval_linear(const dgvo_ctx *c, const double *fmA, const double *f, double *fc);
/* vector-Jacobian product g_k = sum_i v_i dQ_i/df_k, restated from the same loop */
void dgvo_vjp(const dgvo_ctx *c, const double *f, const double *v, double *g, int nthreads);

/* SpatialOperSH_DGV, run_mode 0 (spat_oper_mod.f90:28-68): fcol = Q * kappa * dt */
/* SpatialOperSH_DGV with CheckSolutionMode_DGV's run modes (spat_oper_mod.f90:28-68, 195-272) */
typedef struct dgvo_regime dgvo_regime;
dgvo_regime *dgvo_regime_create(const dgvo_ctx *c, double decomp_lev, double linear_lev);
void dgvo_regime_free(dgvo_regime *r);
int dgvo_regime_mode(const dgvo_regime *r, double *last_L1);
void dgvo_spatial_oper_regime(const dgvo_ctx *c, dgvo_regime *r, const double *f, double *fcol, double dt,
                              double kappa, int nthreads);
int dgvo_rk_step_regime(const dgvo_ctx *c, dgvo_regime *r, int order, double *f, double *frhs1, double dt,
                        double kappa, int nthreads);
void dgvo_spatial_oper(const dgvo_ctx *c, const double *f, double *fcol, double dt,
                       double kappa, int nthreads);
/* TimeIntegratorORK_SH_DGV (time_integr_mod.f90:26-152): one step of RK1..RK5.
 * f is advanced in place; frhs1 receives the first-stage right side / dt. */
int dgvo_rk_step(const dgvo_ctx *c, int order, double *f, double *frhs1, double dt,
                 double kappa, int nthreads);
/* TimeIntegratorMTS_SH_DGV (time_integr_mod.f90:314-364).  frhs holds 5 history
 * vectors of N entries (frhs1..frhs5, newest first); advanced in place. */
int dgvo_ab_step(const dgvo_ctx *c, int order, double *f, double *frhs, double dt,
                 double kappa, int nthreads);
/* PrepareMTS_SH_DGV (time_integr_mod.f90:443-569): order-1 RK start-up steps */
int dgvo_prepare_ab(const dgvo_ctx *c, int order, double *f, double *frhs, double dt,
                    double kappa, int nthreads);

/* MassCheckRec (dgvtools_mod.f90:1437-1458): out = n, ubar, vbar, wbar, T */
void dgvo_moments(const dgvo_ctx *c, const double *f, double *out5);
/* maxwelveldist (distributions_mod.f90:83-95) at every node */
void dgvo_maxwellian(const dgvo_ctx *c, double T, double u0, double v0, double w0,
                     double n, double *f);
/* L2(w) projection of q onto the complement of span{1,u,v,w,|v|^2}: after it
 * sum_i w_i psi(v_i) q_i = 0 for the five collision invariants */
void dgvo_project_conservative(const dgvo_ctx *c, double *q);

/* SetA_DGV (dgvtools_mod.f90:377-681, 938-1122) for one basis function i1
 * (0-based node index).  basis_mode 0 = Lagrange basis function restored
 * (dgvtools_mod.f90:254-287 "rem to restore" lines, equivalently :115-210);
 * 1..5 = the collision invariants 1,u,v,w,|v|^2 listed at :267-274.
 * Records are returned through malloc'd arrays (free with dgvo_free). */
int64_t dgvo_seta(const dgvo_ctx *c, int32_t i1, double Trad, double ErrChi,
                  double ErrEps, double min_sens, int basis_mode, int nthreads,
                  double **A, int32_t **xi, int32_t **xi1);
/* the raw chi-integral of SetA for a single pair (no weights, no |g|/8) */
double dgvo_seta_pair_integral(const dgvo_ctx *c, int32_t i1, int32_t i2, int32_t i3,
                               double ErrChi, double ErrEps, int basis_mode);

/* Synthetic A-arrays with the real index structure: for every canonical basis
 * function p (node ccell*P+p, in order) every pair i2<i3 that passes the
 * reference prefilter (dgvtools_mod.f90:527) and, when support_mode==1, whose
 * collision sphere surface meets the canonical cell, gets one record with
 * value  w_i2 * w_i3 * |g|/8 * u,  u = hash(seed,p,i2,i3) in [-1,1).
 * p_only >= 0 generates the records of that basis function only.
 * Returns nnz; arrays malloc'd (0-based xi/xi1, capphi has N entries). */
int64_t dgvo_synth_A(const dgvo_ctx *c, uint64_t seed, double Trad, int support_mode, int32_t p_only,
                     int32_t **capphi, double **A, int32_t **xi, int32_t **xi1);
/* the synthetic value for one record (shared definition with the GPU generator) */
double dgvo_synth_value(uint64_t seed, int32_t p, int32_t i2, int32_t i3, double w2,
                        double w3, double dsph);
void dgvo_free(void *p);

#ifdef __cplusplus
}
#endif
#endif
