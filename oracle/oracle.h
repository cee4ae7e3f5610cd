/*
 * THE ORACLE -- test infrastructure, not product code.
 *
 * A C++ FP64 CPU restatement of the density-fitting path of pysisyphus-addons.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load it, and only as the checker (or the timed CPU baseline), never as the
 * thing measured or shipped. The product library (libpa_b200.so) never links
 * or calls it.
 *
 * The drivers follow the reference's loop, screening, layout and threshold
 * semantics (file:line citations in oracle.cpp). The integral values follow
 * from the mathematics: contracted spherical Gaussian ERIs by the
 * Obara-Saika vertical recurrence plus the Head-Gordon-Pople horizontal
 * recurrence -- a different scheme from the McMurchie-Davidson kernels of the
 * CUDA library, so agreement between the two is a genuine cross-check.
 *
 * All arrays are column-major (Fortran order) exactly as the reference's
 * bind(c) wrappers expect; basis pointers are 1-based.
 */
#pragma once
#ifdef __cplusplus
extern "C" {
#endif

/* Boys-function mode: 0 = exact (series / asymptotic, ~1e-16 relative),
 * 1 = reference-compatible (5-point Neville on a 0.01 grid for x < 27,
 *     asymptotic formula for x >= 27; common/integrals/boys.f90:88-97). */
void oracle_set_boys_mode(int mode);
int oracle_get_boys_mode(void);
void oracle_set_threads(int nthreads);
/* 1: skip the metric (inv_chol + dtrmm) in the 2d/4d and std drivers (raw tensors). */
void oracle_set_skip_metric(int skip);
/* Adds shift * I to (P|Q) before its Cholesky factorization (default 0: the
 * reference's behaviour). For auxiliary bases that are linearly dependent to
 * machine precision, where dpotrf fails. */
void oracle_set_metric_shift(double shift);
// 0: schwarz_estimate (default), 1: qvl_estimate in the Coulomb contraction.
void oracle_set_screening(int mode);
/* 1: keep the bra Schwarz vector of the last orbital basis and reuse it while
 * the basis is unchanged (timing aid for sampled CPU baselines; default 0). */
void oracle_set_reuse_screening(int reuse);
int oracle_get_threads(void);
/* Optional BLAS/LAPACK (Fortran calling convention) used by inv_chol / dtrmm /
 * dgemm, exactly as the reference calls them; naive loops when unset. */
void oracle_register_lapack(void* dpotrf, void* dtrtri, void* dtrmm, void* dgemm);

void oracle_boys(int nmax, double x, double* out);
double oracle_erfinv(double x);
void oracle_contracted_center(int na, const double* axs, const double* das, const double* A,
                              int nb, const double* bxs, const double* dbs, const double* B,
                              double* R);

/* Contracted spherical ERI block (ab|cd), order (ma, mb, mc, md) with md fastest.
 * Shells are given raw (coefficients refer to normalized primitives and are
 * renormalized like common/normalization.f90). A shell with L < 0 is a unit
 * s function with exponent 0 (used for 2- and 3-center integrals). */
int oracle_eri_block(int La, int na, const double* ea, const double* ca, const double* A,
                     int Lb, int nb, const double* eb, const double* cb, const double* B,
                     int Lc, int nc, const double* ec, const double* cc, const double* C,
                     int Ld, int nd, const double* ed, const double* cd, const double* D,
                     double* out);

/* Mirrors of the reference's C-ABI (same argument lists). */
void oracle_init(void);
void oracle_int_schwarz_aux(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                            const double* bas_data, double* integrals);
void oracle_int_schwarz_bra(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                            const double* bas_data, double* integrals);
void oracle_int2c2e_metric(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                           const double* bas_data, int naux, double* metric);
void oracle_contract_coulomb_densities_2d(
    int nshells, int ndata, const int* bas_centers, const int* bas_spec, const double* bas_data,
    int nshells_aux, int ndata_aux, const int* bas_centers_aux, const int* bas_spec_aux,
    const double* bas_data_aux, int ndens, int nbfs, const double* densities, int naux,
    double* df_tensor);
void oracle_contract_coulomb_densities_4d(
    int nshells, int ndata, const int* bas_centers, const int* bas_spec, const double* bas_data,
    int nshells_aux, int ndata_aux, const int* bas_centers_aux, const int* bas_spec_aux,
    const double* bas_data_aux, int ndens, int nbfs, const double* densities, int nstates,
    double* coulomb_tensor);
void oracle_intor_eri2c(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                        const double* bas_data, int nshells_aux, int ndata_aux,
                        const int* bas_centers_aux, const int* bas_spec_aux,
                        const double* bas_data_aux, int nbfs, double* eri2c);
void oracle_intor_df1c(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                       const double* bas_data, int nshells_aux, int ndata_aux,
                       const int* bas_centers_aux, const int* bas_spec_aux,
                       const double* bas_data_aux, int nbfs, int nbfs_aux, double* df1c);
void oracle_intor_df2c_mo(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                          const double* bas_data, int nshells_aux, int ndata_aux,
                          const int* bas_centers_aux, const int* bas_spec_aux,
                          const double* bas_data_aux, int nbfs, int nmos, const double* mo_tensor,
                          int nbfs_aux, double* df2c_mo);

/* Statistics of the last 3c2e driver call: computed and skipped shell triples,
 * spherical integrals of computed triples, and phase times (seconds). */
typedef struct {
  long long ntriplets, nskipped, nints;
  double t_screener, t_metric, t_chol, t_3c, t_trmm, t_total;
} OracleStats;
void oracle_last_stats(OracleStats* out);

/* Extended-precision (long double) Cholesky factor of M and Y = L^-1 B, for
 * checking FP64 solves of ill-conditioned metrics. Returns 0 or the 1-based
 * column of the first non-positive pivot; L_out may be NULL. */
int oracle_chol_solve_ld(int n, const double* M, int nrhs, const double* B, double* Y,
                         double* L_out);
/* ||L L^T - M||_F / ||M||_F in long double (L: lower triangle of Lc). */
double oracle_chol_backward_error_ld(int n, const double* M, const double* Lc);

/* Mirror of f_eval_densities (grid/grid_wrapper.f90:12-38): densities on grid
 * points from Cartesian AO density matrices (ndens, nbfs, nbfs), column-major
 * grid3d(3, npoints), output grid_densities(ndens, npoints). */
void oracle_eval_densities(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                           const double* bas_data, int npoints, const double* grid3d, int ndens, int nbfs,
                           const double* densities, double* grid_densities, int blk_size, double thresh);
/* Records of the estimator study benchmark_int3c2e (intor/benchmark.f90:15-132):
 * (schwarz_estimate, qvl_estimate, ||(ab|c)||_2, distance) per non-concentric,
 * non-small pair and auxiliary shell, in the reference's loop order. Returns
 * their number; writes at most cap. */
long long oracle_int3c2e_estimates(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                                   const double* bas_data, int nshells_aux, int ndata_aux,
                                   const int* bas_centers_aux, const int* bas_spec_aux,
                                   const double* bas_data_aux, long long cap, double* records,
                                   long long* nskipped);
/* Mirror of f_eval_prim_density (gdma/prim_dens.f90:100-259). */
void oracle_eval_prim_density(int nprims, int npoints, int nbfs, const int* ls_inds, const double* primdata,
                              const double* coords3d, const double* P, double sw, double* rho);

#ifdef __cplusplus
}
#endif
