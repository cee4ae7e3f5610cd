/*
 * pa_b200.h -- C-ABI of libpa_b200.so, the B200 (sm_100a) implementation of
 * the density-fitting path of pysisyphus-addons.
 *
 * The f_* entry points keep the argument lists of the reference's bind(c)
 * Fortran wrappers (file:line below, within the reference project), so a
 * caller that binds those symbols (Cython `cdef extern`, ctypes, cffi) can
 * link this library instead:
 *   - all scalars are int32 passed by value;
 *   - all arrays are column-major (Fortran order) host arrays;
 *   - bas_centers (nshells x 3) and bas_spec (nshells x 5) hold 1-based
 *     pointers into bas_data, packed as described in common/shells.f90:97-187;
 *   - outputs are written in place; the library keeps no reference to any
 *     argument after the call returns.
 * Differences from the reference: every entry point returns an int status
 * (PA_OK = 0; a caller that declared the function void ignores it) instead of
 * terminating the process (`error stop`) or silently ignoring LAPACK errors,
 * and pa_last_error() describes the last failure of the calling thread.
 *
 * The pa_* entry points are additions: options, statistics, and a
 * device-resident variant of the path that takes device pointers and a CUDA
 * stream (cudaStream_t passed as void*).
 */
#ifndef PA_B200_H
#define PA_B200_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. */
#define PA_OK 0
#define PA_ERR_ARG 1        /* invalid argument (sizes, pointers, layout)        */
#define PA_ERR_LMAX 2       /* angular momentum above the compiled maximum       */
#define PA_ERR_NOT_SPD 3    /* metric (P|Q) not positive definite (dpotrf info>0) */
#define PA_ERR_CUDA 4       /* CUDA runtime error                                 */
#define PA_ERR_TIMEOUT 5    /* a bounded device-side wait gave up                 */
#define PA_ERR_NO_DEVICE 6  /* no usable CUDA device                              */
#define PA_ERR_SCRATCH 7    /* request exceeds a fixed scratch capacity           */

/* Compiled angular-momentum limits (reference defaults, meson.options:1-4). */
#define PA_LMAX_ORBITAL 4
#define PA_LMAX_AUX 5

/* Boys-function modes. */
#define PA_BOYS_EXACT 0     /* ~1e-16 relative                                    */
#define PA_BOYS_REFERENCE 1 /* behaviour of common/integrals/boys.f90 (default)    */

/* Precision forms of the three-center contraction. */
#define PA_PRECISION_FP64 0  /* FP64 throughout (default)                          */
#define PA_PRECISION_MIXED 1 /* FP32 recurrences for triplets below a Schwarz bound */

/* Triplet estimates of the density-fitting screening. */
#define PA_SCREEN_SCHWARZ 0 /* Q_ab Q_c (schwarz_estimate, default)                */
#define PA_SCREEN_QVL 1     /* qvl_estimate, common/screening.f90:267-299          */

/* Density layouts for the pa_* entry points. */
#define PA_LAYOUT_FORTRAN 0 /* (ndens, nbf, nbf) column-major: d fastest          */
#define PA_LAYOUT_C 1       /* (ndens, nbf, nbf) row-major: last index fastest    */

/* ------------------------------------------------------------------------ */
/* Reference-compatible entry points                                         */
/* ------------------------------------------------------------------------ */

/* Replaces f_init, common/integrals/init.f90:13-27: one-time set-up (device
 * tables on the current device). Optional; every entry point calls it. */
int f_init(void);

/* Replaces f_int_schwarz_aux, intor/intor_wrapper.f90:12-24:
 * integrals[c] = sqrt(||(c|c)||_F) for every shell c. */
int f_int_schwarz_aux(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                      const double* bas_data, double* integrals);

/* Replaces f_int_schwarz_bra, intor/intor_wrapper.f90:26-38:
 * integrals[a(a+1)/2 + b] = sqrt(||(ab|ab)||_F), 0-based a >= b. */
int f_int_schwarz_bra(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                      const double* bas_data, double* integrals);

/* Replaces f_contract_coulomb_densities_2d, diabatization/intor_wrapper.f90:12-43:
 * df_tensor(naux, ndens) = L^-1 sum_(a>=b) (ab|P) [D + (a!=b) D^T]. */
int f_contract_coulomb_densities_2d(int nshells, int ndata, const int* bas_centers,
                                    const int* bas_spec, const double* bas_data, int nshells_aux,
                                    int ndata_aux, const int* bas_centers_aux,
                                    const int* bas_spec_aux, const double* bas_data_aux,
                                    int ndens, int nbfs, const double* densities, int naux,
                                    double* df_tensor);

/* Replaces f_contract_coulomb_densities_4d, diabatization/intor_wrapper.f90:45-76:
 * coulomb_tensor(nstates, nstates, nstates, nstates), ndens = nstates(nstates+1)/2. */
int f_contract_coulomb_densities_4d(int nshells, int ndata, const int* bas_centers,
                                    const int* bas_spec, const double* bas_data, int nshells_aux,
                                    int ndata_aux, const int* bas_centers_aux,
                                    const int* bas_spec_aux, const double* bas_data_aux,
                                    int ndens, int nbfs, const double* densities, int nstates,
                                    double* coulomb_tensor);

/* Replaces f_intor_eri2c, std/intor_wrapper.f90:12-35: eri2c(nbfs, nbfs) = T T^T
 * with T = (mu mu|P) L^-T. */
int f_intor_eri2c(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                  const double* bas_data, int nshells_aux, int ndata_aux,
                  const int* bas_centers_aux, const int* bas_spec_aux,
                  const double* bas_data_aux, int nbfs, double* eri2c_tensor);

/* Replaces f_intor_df1c, std/intor_wrapper.f90:37-61: df1c(nbfs, nbfs_aux) =
 * (mu mu|P) L^-T. */
int f_intor_df1c(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                 const double* bas_data, int nshells_aux, int ndata_aux,
                 const int* bas_centers_aux, const int* bas_spec_aux, const double* bas_data_aux,
                 int nbfs, int nbfs_aux, double* df1c_tensor);

/* Replaces f_intor_df2c_mo, std/intor_wrapper.f90:63-88: df2c_mo(nmos(nmos+1)/2,
 * nbfs_aux) = MO-pair-packed (pq|P) L^-T for mo_tensor(nbfs, nmos). */
int f_intor_df2c_mo(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                    const double* bas_data, int nshells_aux, int ndata_aux,
                    const int* bas_centers_aux, const int* bas_spec_aux,
                    const double* bas_data_aux, int nbfs, int nmos, const double* mo_tensor,
                    int nbfs_aux, double* df2c_mo_tensor);

/* ------------------------------------------------------------------------ */
/* Additions                                                                 */
/* ------------------------------------------------------------------------ */

/* Message of the last failure on the calling thread ("" if none). */
const char* pa_last_error(void);

/* Options (process-wide). Boys mode: PA_BOYS_REFERENCE (default) or
 * PA_BOYS_EXACT. Screening threshold: default (double)1e-10f, the reference's
 * REAL(4) literal (diabatization/intor.f90:140). */
int pa_set_boys_mode(int mode);
int pa_get_boys_mode(void);
int pa_set_screen_threshold(double thresh);
/* 1: return the raw contraction sum_(a>=b) (ab|P) Dsym without the metric
 * solve L^-1 (the first half of the density fit); 0 (default): full path. */
int pa_set_skip_metric(int skip);
/* Adds shift * I to (P|Q) before its Cholesky factorization in every
 * density-fitting entry point (default 0: the reference's behaviour). An
 * option for auxiliary bases that are linearly dependent to machine precision
 * (dpotrf fails; the reference then continues with a broken factor, its info
 * being ignored, common/linalg.f90:78). */
int pa_set_metric_shift(double shift);
/* Precision form of the density-fitting contraction (process-wide):
 * PA_PRECISION_FP64 (default) or PA_PRECISION_MIXED, in which shell triplets
 * with Schwarz bound Q_ab * Q_c < fp32_thresh (e.g. 1e-6) evaluate the Boys
 * function (below T = 27 / 30), the Hermite recurrence and the solid-harmonic
 * contraction in FP32. pa_set_mixed_kernels picks how: 0 (default) inside the
 * FP64 class kernels, whose density product stays FP64; 1 on separate
 * weak-triplet kernels whose density product is a split-BF16 tensor-core
 * product (three BF16 slices per operand, six slice products, FP32
 * accumulation over one step, FP64 across steps), the other triplets on the
 * FP64 kernels. Both keep the accumulation across triplets in FP64. The
 * reference is FP64 only. */
int pa_set_precision(int mode, double fp32_thresh);
int pa_set_mixed_kernels(int mode);
int pa_get_mixed_kernels(void);
/* Grid of the three-center class launches (process-wide): 0 (default) =
 * persistent blocks that pull work items until none is left, 1 = one block
 * per work item. */
int pa_set_class_grid(int mode);
/* The f_* entry points keep the device copies (with the shell-pair lists) of
 * the last 8 bases they were given, for later calls with byte-identical basis
 * arrays on the same device; pa_basis_cache_clear frees them. pa_get_device
 * gives the CUDA device of the calling thread, on which calls run. */
int pa_basis_cache_clear(void);
int pa_get_device(int* device);
/* Granularity of the three-center work queue: work items per SM and shell
 * class; 0 (default) picks it from the system size (2 at 40 atoms, 8 at 200).
 * Finer items shorten the tail of each class launch and cost more partial
 * sums. */
int pa_set_items_per_sm(int items);
int pa_get_precision(void);
/* Triplet estimate of the density-fitting contraction (process-wide):
 * PA_SCREEN_SCHWARZ (default) is schwarz_estimate, the reference's active line
 * (diabatization/intor.f90:138); PA_SCREEN_QVL is qvl_estimate
 * (common/screening.f90:267-299), the commented-out alternative at :137:
 * beyond the sum of the extents of the bra distribution and the auxiliary
 * shell, Q_ab pi sqrt(2) beta_c / ((zeta_a + zeta_b)^(1/4) R^(L_c + 1))
 * replaces Q_ab Q_c. Applies to the Coulomb-tensor entry points and
 * pa_count_triplets; the std tensors always use the Schwarz estimate, as the
 * reference does. */
int pa_set_screening(int mode);
int pa_get_screening(void);

/* Statistics of the last density-fitting call on this process. */
typedef struct {
  long long ntriplets;       /* shell triplets a >= b, c                       */
  long long nskipped;        /* screened out (-1 when not counted)             */
  long long nints;           /* spherical integrals of computed triplets (-1)  */
  double ms_total;           /* device time of the whole path (CUDA events)    */
  double ms_screen;          /* unit set-up, Schwarz vectors, class sorting    */
  double ms_bra;             /* density folding of the bra units               */
  double ms_metric;          /* metric (P|Q) and its Cholesky factor           */
  double ms_3c;              /* three-center contraction and its reduction     */
  double ms_solve;           /* L^-1 df and the Coulomb-tensor assembly        */
  int kernel_launches;       /* kernels launched by the library in the call    */
  int launches_3c;           /* of which three-center contraction kernels      */
} pa_stats;
int pa_get_stats(pa_stats* out);
/* Profiling aid (no counterpart in the reference): with on = 1 the
 * three-center class launches of the single-molecule path run one after
 * another on one stream, each bracketed by CUDA events; pa_get_class_times
 * then gives (L_ab, L_c, ms) of every class run of the last call (up to cap
 * entries) and returns their number. */
int pa_set_class_timing(int on);
int pa_get_class_times(int cap, int* lab, int* lc, double* ms);
/* Tile-shape variants of the three-center class kernels (no counterpart in
 * the reference; its OpenMP loop has no tiles). Each class (L_ab = la + lb in
 * 0..2*PA_LMAX_ORBITAL, L_c in 0..PA_LMAX_AUX) has variants 0..PA_TILE_VARIANTS-1:
 *   0: the largest auxiliary tile that fits two blocks per SM (default);
 *   1: the tile, at least half as large, that keeps the most lanes of the
 *      block busy while the integrals are built;
 *   2: three blocks per SM for classes with L_ab + L_c > 5.
 * Results agree to rounding between variants. The selection is process-wide
 * and read at the start of each call. pa_tile_shape gives, for one variant,
 * out[0] = auxiliary shells per tile, out[1] = bra units per step, out[2] =
 * lanes per triplet, out[3] = blocks per SM, out[4] = shared memory bytes per
 * block. pa_load_tile_table applies a table of "L_ab L_c variant" lines (#
 * comments; NULL = the default table); the library applies its default table
 * once per process before the first call: $PA_B200_TILE_TABLE when set (empty
 * = none), else df3c_tiles.txt beside the library, when present. The package's
 * autotuner (pysisyphus_addons.tune) writes such tables. */
#define PA_TILE_VARIANTS 3
int pa_set_tile_variant(int lab, int lc, int variant);
int pa_get_tile_variant(int lab, int lc, int* variant);
int pa_tile_shape(int lab, int lc, int variant, int* out);
int pa_load_tile_table(const char* path, int* napplied);

/* Device-resident path. A pa_basis holds an unpacked, normalized basis on the
 * host and its copy in device memory of the current device. */
typedef struct pa_basis_s* pa_basis;
int pa_basis_create(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                    const double* bas_data, int lmax_allowed, pa_basis* out);
int pa_basis_destroy(pa_basis basis);
int pa_basis_info(pa_basis basis, int* nshells, int* nsph, int* lmax);

/* df(naux, ndens), column-major, = L^-1 (ab|P) D; d_densities and d_df are
 * device pointers; stream is a cudaStream_t (0 = default stream). Synchronous:
 * returns after the result is complete (errors are reported here). */
int pa_df_2d(pa_basis orbital, pa_basis aux, int ndens, int nbf, const double* d_densities,
             int layout, double* d_df, void* stream);
/* Coulomb tensor (nstates^4, column-major) from device densities. */
int pa_df_4d(pa_basis orbital, pa_basis aux, int ndens, int nbf, const double* d_densities,
             int layout, int nstates, double* d_coulomb, void* stream);
/* Batched form: the Coulomb tensors of nmol molecules in one call. Molecule m
 * has the bases orbital[m] / aux[m], ndens[m] = nstates[m] (nstates[m] + 1) / 2
 * device densities d_densities[m] (in `layout`) and the device output
 * d_coulomb[m] (nstates[m]^4, column-major). Every molecule's screening,
 * density folding and metric chain run concurrently; the three-center work of
 * all molecules runs as one persistent launch per shell-triplet class, fed by
 * the class's queue of work items (molecules by decreasing work, each heavy
 * first). With use_graph = 1 the whole sequence is recorded once as a CUDA
 * graph and replayed by later calls with the same handles, sizes, pointers and
 * options (the last batch is kept per device). Synchronous: returns after the
 * tensors are complete; work already queued on `stream` is waited for first. */
int pa_df_4d_batch(int nmol, const pa_basis* orbital, const pa_basis* aux, const int* ndens,
                   const double* const* d_densities, int layout, const int* nstates,
                   double* const* d_coulomb, int use_graph, void* stream);

/* Host-buffer variants of f_contract_coulomb_densities_{2d,4d} with an explicit
 * density layout (PA_LAYOUT_C avoids a transposed host copy). */
int pa_contract_coulomb_densities_2d(pa_basis orbital, pa_basis aux, int ndens, int nbf,
                                     const double* densities, int layout, double* df_tensor);
int pa_contract_coulomb_densities_4d(pa_basis orbital, pa_basis aux, int ndens, int nbf,
                                     const double* densities, int layout, int nstates,
                                     double* coulomb_tensor);

/* Device-resident sTDDFT tensors (std/intor.f90); outputs column-major on the
 * device, synchronous on `stream`:
 *   pa_std_df1c:    d_out(nbf, naux)  = (mu mu|P) L^-T            (intor_df1c)
 *   pa_std_eri2c:   d_out(nbf, nbf)   = df1c df1c^T                (intor_eri2c)
 *   pa_std_df2c_mo: d_out(nmos(nmos+1)/2, naux) = packed (pq|P) L^-T for the MO
 *                   coefficients d_mo(nbf, nmos)                   (intor_df2c_mo) */
int pa_std_df1c(pa_basis orbital, pa_basis aux, double* d_out, void* stream);
int pa_std_eri2c(pa_basis orbital, pa_basis aux, double* d_out, void* stream);
int pa_std_df2c_mo(pa_basis orbital, pa_basis aux, int nmos, const double* d_mo, double* d_out,
                   void* stream);

/* Screening statistics for a basis pair: number of shell triplets that pass
 * the Schwarz test and their spherical integral count (runs the Schwarz
 * kernels; host-side counting). */
int pa_count_triplets(pa_basis orbital, pa_basis aux, long long* ntriplets, long long* ncomputed,
                      long long* nints);

/* Building blocks exposed for tests: Boys values F_0..F_nmax(T) for n
 * arguments on the device (results copied to host), and the metric (P|Q). */
int pa_boys_eval(int mode, int nmax, int n, const double* T, double* out);
int pa_metric(pa_basis aux, double* metric);
/* Host-buffer Cholesky solve on the device, the linear algebra of
 * inv_chol + dtrmm (common/linalg.f90:60-82, diabatization/intor.f90:198):
 * the lower triangle of A (n x n, column-major) is replaced by L with
 * A = L L^T (entries above the diagonal are left as they were), and B
 * (n x nrhs) by L^-1 B. PA_ERR_NOT_SPD when A is not positive definite. */
int pa_cholesky_solve(int n, double* A, int nrhs, double* B);

/* Diagnostic of the precision form's density product (no counterpart in the
 * reference, which has no tensor-core path): C (m x n) = A (m x k) B^T
 * (B: n x k), all row-major host arrays, computed by one block with the
 * split-BF16 tcgen05 product of the weak-triplet three-center kernels (three
 * BF16 slices per operand, six slice products accumulated in FP32 in tensor
 * memory). 1 <= m <= 128, 1 <= n <= 48, 1 <= k <= 128. Synchronous. */
int pa_split_product_check(int m, int n, int k, const double* A, const double* B, double* C);

/* The estimator study (replaces intor/benchmark_wrapper.f90:13-37,
 * f_benchmark_int3c2e, same arguments): prints the basis sizes, the time and
 * the number of shell triplets the QVL estimate skips, and writes
 * int_estimates.bin (4 doubles per record) in the working directory.
 * pa_int3c2e_estimates gives the records themselves: (schwarz_estimate,
 * qvl_estimate, ||(ab|c)||_2, distance of the pair's contracted center to the
 * auxiliary center) for every shell pair a >= b that is not concentric and
 * whose Schwarz value exceeds 1e-10, and every auxiliary shell c, in the
 * reference's loop order (intor/benchmark.f90:82-118); records == NULL
 * returns only *nrecords and *nskipped (records with qvl_estimate < 1e-10). */
int f_benchmark_int3c2e(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                        const double* bas_data, int nshells_aux, int ndata_aux, const int* bas_centers_aux,
                        const int* bas_spec_aux, const double* bas_data_aux);
int pa_int3c2e_estimates(pa_basis orbital, pa_basis aux, long long cap, double* records, long long* nrecords,
                         long long* nskipped);

/* Densities on grid points (replaces grid/grid_wrapper.f90:12-38,
 * f_eval_densities, same arguments): grid3d(3, npoints) column-major,
 * densities(ndens, nbfs, nbfs) Cartesian AO density matrices in pysisyphus
 * order (nbfs = the basis' Cartesian size), grid_densities(ndens, npoints)
 * written. Points in consecutive blocks of blk_size (1..4096); a function pair
 * contributes to a block when |f D mean_nu mean_mu| >= thresh
 * (grid/grid.f90:236-258). Shells up to g (PA_ERR_LMAX above, where the
 * reference writes NaN). Host buffers; synchronous. */
int f_eval_densities(int nshells, int ndata, const int* bas_centers, const int* bas_spec,
                     const double* bas_data, int npoints, const double* grid3d, int ndens, int nbfs,
                     const double* densities, double* grid_densities, int blk_size, double thresh);
/* Density of the primitive pairs with exponent sum below `sw` on grid points
 * (replaces gdma/prim_dens.f90:100-259, f_eval_prim_density, same arguments):
 * ls_inds(2, nprims) = (L, 0-based Cartesian start), primdata(5, nprims) =
 * (coefficient, exponent, x, y, z), coords3d(3, npoints), P(nbfs, nbfs),
 * rho(npoints) written. L up to 4 (the reference's g prefactors fill 14 of
 * the 15 components; these are all 15). Host buffers; synchronous. */
int f_eval_prim_density(int nprims, int npoints, int nbfs, const int* ls_inds, const double* primdata,
                        const double* coords3d, const double* P, double sw, double* rho);

/* The metric half of contract_coulomb_densities_2d / _4d on device buffers
 * (common/linalg.f90:60-82 inv_chol, diabatization/intor.f90:198 dtrmm and
 * :204-270 the tensor): (P|Q) of `aux` (+ the metric shift), its Cholesky
 * factor, d_df = L^-1 d_raw (naux x ndens, column-major) and, with nstates > 0,
 * the Coulomb tensor (nstates^4, column-major) into d_coulomb. d_raw is the
 * screened three-center contraction, e.g. gathered from auxiliary-shell shards
 * (pa_df_2d with the metric skipped, on a sub-basis of consecutive auxiliary
 * shells per rank); it is read only. Synchronous on `stream`. No counterpart
 * entry point in the reference, whose driver does these steps inline. */
int pa_df_solve(pa_basis aux, int ndens, const double* d_raw, double* d_df, int nstates, double* d_coulomb,
                void* stream);

/* Allocation-free variant of pa_cholesky_solve on device buffers. This entry
 * point has no counterpart in the reference.
 *
 * Who it is for: callers that cannot allocate device memory at call time --
 * applications whose GPU memory is handed out entirely by another allocator
 * (e.g. a framework's caching allocator that reserved the device up front),
 * and code that must not call cudaMalloc / cudaFree because those calls can
 * synchronize the whole device and stall unrelated work. It calls no
 * cudaMalloc, cudaFree, memory pool or allocating library routine; its
 * scratch memory is one fixed array of PA_NOALLOC_SCRATCH_DOUBLES doubles
 * (8 MiB) in the library's device image, which every GPU that loads the
 * library holds until the process exits.
 *
 * d_A (n x n, column-major, device): its lower triangle is replaced by L with
 * A = L L^T (entries above the diagonal are left as they were). d_B (n x nrhs,
 * device) is read only; d_X (n x nrhs, device) receives L^-1 B. d_X may be d_B
 * (B is copied to the scratch array first) but must not overlap d_A
 * (PA_ERR_ARG). stream is a cudaStream_t (0 = default stream). The call is
 * synchronous: it reads a status word back to the host and waits for `stream`
 * before it returns. Limit: 4096 * ceil(n / 64) + n * nrhs + 32 <=
 * PA_NOALLOC_SCRATCH_DOUBLES (e.g. n = 2240 with nrhs up to 404), else
 * PA_ERR_SCRATCH before any device work. PA_ERR_NOT_SPD as for
 * pa_cholesky_solve. A CUDA error already pending from the caller's earlier
 * work is reported (PA_ERR_CUDA) and left pending.
 *
 * Every call looks up the array's device address in the current context
 * (cudaGetSymbolAddress, with the device current); the first call on a device
 * also loads the library's device code there, so make that first call before
 * any stream capture. All calls in the process share the one array per device:
 * calls that overlap on the GPU (concurrent streams or host threads) race on
 * it and must be serialized by the caller. */
#define PA_NOALLOC_SCRATCH_DOUBLES (1 << 20)
int pa_cholesky_solve_noalloc(int n, double* d_A, int nrhs, const double* d_B, double* d_X,
                              void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PA_B200_H */
