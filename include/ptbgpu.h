/*
 * ptbgpu.h -- C-ABI of the B200 density-matrix step for PTB.
 *
 * Drop-in boundary for the Fortran SCF driver (twoscf, source/pgtb.f90:345-670):
 * every entry point takes host pointers in the reference's packed layout
 * (FP64, 1-based ij = i(i-1)/2 + j for j <= i: column i, rows <= i;
 * source/solve.f:149-200) and default Fortran integers as int64_t (the
 * reference builds with -i8, source/Makefile:35-37).  The library copies in
 * and out; it keeps no caller pointer after a call returns.
 *
 * Every function returns 0 on success or one of the PTBGPU_E* codes below;
 * ptbgpu_last_error() returns the message of the last failure on a context.
 * A context is not re-entrant: one host thread drives it at a time.
 */
#ifndef PTBGPU_H
#define PTBGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define PTBGPU_OK               0
#define PTBGPU_EINVAL           1   /* bad argument (size, mode, null pointer)          */
#define PTBGPU_ECUDA            2   /* CUDA runtime / cuBLAS / cuSOLVER failure           */
#define PTBGPU_ENOTSPD          3   /* overlap (sub)matrix not positive definite          */
#define PTBGPU_ENAN             4   /* NaN during an iteration ("error stop" in the ref.) */
#define PTBGPU_EITER            5   /* iteration cap reached without convergence          */
#define PTBGPU_ENOTIMPL         6   /* mode the reference stops on ("not implemented")     */
#define PTBGPU_ETIMEOUT         7   /* a bounded device-side wait gave up                 */
#define PTBGPU_ENOMEM           8   /* device allocation failed                           */

/* ---- mode codes (source/purification_settings.f90:6-27) ---------------- */
#define PTBGPU_MODE_FULL                 1
#define PTBGPU_MODE_SUBMATRIX            2
#define PTBGPU_COLUMNS_SINGLE            1
#define PTBGPU_COLUMNS_ATOMS             2
#define PTBGPU_COLUMNS_FULL_MATRIX       3
#define PTBGPU_COLUMNS_KMEANS            4
#define PTBGPU_SUBMATRIX_SIGN            1
#define PTBGPU_SUBMATRIX_SYGV            2
#define PTBGPU_TYPE_MCWEENY              1
#define PTBGPU_TYPE_PADE                 2
#define PTBGPU_TYPE_NEWTON               3
#define PTBGPU_TYPE_DIAG                 4
#define PTBGPU_METRIC_INV                1
#define PTBGPU_METRIC_INV_SQRT           2
#define PTBGPU_METRIC_SQRT               3

/* ---- precision of the trace-correcting purification -------------------- */
#define PTBGPU_PREC_FP64                 0  /* every product in FP64 (comparator path)      */
#define PTBGPU_PREC_MIXED                1  /* bf16x3 tensor-core iterations + FP64 refinement */

typedef struct ptbgpu_ctx ptbgpu_ctx;

/* POD mirror of tPurificationSet (source/purification_settings.f90:29-86). */
typedef struct {
    int64_t mode;               /* 1 full, 2 submatrix                    */
    int64_t type;               /* 1 mcweeny, 2 pade, 3 newton, 4 diag    */
    int64_t cycles;             /* purification cycles (default 40)       */
    int64_t prlvl;              /* print level (default 1)                */
    int64_t nel;                /* electrons (set by the caller)          */
    int64_t submatrix_mode;     /* 1 sign, 2 sygv                         */
    int64_t submatrix_columns;  /* 1..4                                   */
    int64_t metric_type;        /* 1 inv, 2 inv_sqrt, 3 sqrt              */
    int64_t metric_cycles;      /* default 50                             */
    int64_t metric_iterative;   /* logical                                */
    int64_t chempot_cycles;     /* default 60                             */
    double  chempot_guess;      /* default -1.5                           */
    double  chempot_increment;  /* default 0.1                            */
} ptbgpu_pur_settings;

/* Options that have no counterpart in the reference's argument lists. */
typedef struct {
    double  filter;             /* >0: zero |A_ij| < filter in H and S first (source/pgtb.f90:567-585) */
    int64_t precision;          /* PTBGPU_PREC_*                                  */
    int64_t print_level;        /* 0 silent, 1 the reference's progress lines     */
    int64_t max_iter;           /* cap on trace-correcting iterations (0 = 100)   */
    double  electronic_temp;    /* solve2 Fermi temperature in K (0 = 300)        */
    double  glob_par15;         /* solve2 orbital-energy shift for mode >= 2      */
    double  glob_par17;
    int64_t split3_iters;       /* PREC_MIXED: leading iterations whose products use the
                                   three-plane bf16 split (~24 bits); 0 = all, -1 = none
                                   (the default: the refinement rounds make them unnecessary) */
    int64_t fp64_slices;        /* PREC_MIXED: 6..8 -> the FP64 products around the purification
                                   (orthogonalisation, cleanup, commutator, back-transform) run on
                                   the int8 tensor cores with that many 7-bit slices per operand;
                                   0 -> cuBLAS/cuSOLVER FP64 */
    int64_t refine_rounds;      /* PREC_MIXED: cap on the refinement rounds (Newton steps on the
                                   occupied subspace after the tensor-core purification); 0 = 4 */
    double  refine_tol;         /* PREC_MIXED: another round runs while the error predicted after
                                   the last one (orthonormal basis) exceeds this; 0 = 1e-7 */
} ptbgpu_opts;

/* What a call reports back (all optional for the caller). */
typedef struct {
    double  mu;                 /* chemical potential (Eh) / last bisection midpoint  */
    double  nel;                /* electron count of the result, tr(PS)              */
    double  band_energy;        /* tr(PH) with the filtered H                        */
    double  idempotency_ref;    /* |sum(1/2 PSP - P)| as source/metrics.f90:356      */
    double  idempotency_frob;   /* ||1/2 PSP - P||_F                                 */
    int64_t nsm;                /* number of submatrices                             */
    int64_t sum_dims;           /* sum of submatrix dimensions                       */
    int64_t max_dim;            /* largest submatrix dimension                       */
    int64_t iterations;         /* purification iterations (all passes)              */
    int64_t mu_iterations;      /* chemical-potential steps                          */
    int64_t info;               /* first nonzero LAPACK-style info, 0 otherwise      */
    double  ms_total;           /* device time of the call (CUDA events)             */
    double  ms_h2d;
    double  ms_solve;
    double  ms_d2h;
    double  flops;              /* algorithmic FLOPs of the call                     */
    double  ms_tc_sp2;          /* summed device time of the SP2 tensor-core products */
    int64_t n_tc_sp2;           /* their launches                                     */
    double  ms_tc_full;         /* summed device time of the general tensor-core products */
    int64_t n_tc_full;
    int64_t kernel_launches;    /* launches of this library's own kernels in the call */
    double  ms_oz;              /* summed device time of the int8-sliced FP64 products */
    int64_t n_oz;
    double  oz_ops;             /* int8 multiply-adds x 2 those products executed (slice pairs, all tiles) */
    double  tc_flops;           /* bf16 flops the tcgen05 split products executed (all planes, all tiles) */
    int64_t refine_rounds;      /* PREC_MIXED: refinement rounds run                                   */
    int64_t fp64_fallback;      /* PREC_MIXED: 1 if the refinement could not reach refine_tol (gap too
                                   small for the bf16 trajectory) and the purification was redone in FP64 */
} ptbgpu_stats;

/* ---- lifecycle ---------------------------------------------------------- */
/* Replaces nothing in the reference (its accel_lib context, source/cuda_context.f90:1-24,
 * is an unbuilt stub).  One context per device and host thread. */
int  ptbgpu_init(int device, ptbgpu_ctx** ctx);
int  ptbgpu_finalize(ptbgpu_ctx* ctx);
int  ptbgpu_last_error(const ptbgpu_ctx* ctx, char* buf, size_t len);
void ptbgpu_default_settings(ptbgpu_pur_settings* s);   /* type-bound defaults, purification_settings.f90:29-86 */
void ptbgpu_default_opts(ptbgpu_opts* o);
/* No counterpart in the reference: device name and the CUDA runtime, driver,
 * cuBLAS and cuSOLVER versions the context is bound to, as one text line. */
int  ptbgpu_runtime_info(const ptbgpu_ctx* ctx, char* buf, size_t len);

/* ---- matrix utilities --------------------------------------------------- */
/* filter_matrix_sym(A, n, filter), source/pgtb.f90:1532-1547: in place on a
 * host packed array, |A_ij| < filter -> 0. */
int ptbgpu_filter_packed(ptbgpu_ctx* ctx, int64_t n, double* Apk, double filter);

/* check_density / get_nel / band_structure / idempotent
 * (source/metrics.f90:144-179, 202-230, 253-277, 316-360) on packed host data;
 * Hpk may be NULL.  Fills st->nel, band_energy, idempotency_*. */
int ptbgpu_check_density(ptbgpu_ctx* ctx, int64_t ndim, const double* Ppk, const double* Spk,
                         const double* Hpk, ptbgpu_stats* st);

/* ---- the density-matrix step -------------------------------------------- */
/* sm_stupid_simple(ndim,nelref,Hvec,Svec,Pvec,n,xyz,aoat,submatrix_columns,submatrix_mode),
 * source/sm.f90:34-409.  partition (nat entries, 1-based cluster per atom) is
 * required for columns mode 4 in place of the reference's k-means; NULL otherwise.
 * Filtering (opts->filter) is applied to copies of H and S first. */
int ptbgpu_sm_density(ptbgpu_ctx* ctx, int64_t ndim, int64_t nelref,
                      const double* Hpk, const double* Spk, double* Ppk,
                      int64_t nat, const double* xyz, const int64_t* aoat,
                      int64_t submatrix_columns, int64_t submatrix_mode,
                      const int64_t* partition, const ptbgpu_opts* opts, ptbgpu_stats* st);

/* purification(pur, ndim, H, S, P) -> purification_wrapper, source/purification.f90:28-80:
 * metric, chemical-potential search and the selected purification type in FP64. */
int ptbgpu_purify(ptbgpu_ctx* ctx, const ptbgpu_pur_settings* pur, int64_t ndim,
                  const double* Hpk, const double* Spk, double* Ppk,
                  const ptbgpu_opts* opts, ptbgpu_stats* st);

/* Trace-correcting (SP2) purification, the B200 fast path for the dense
 * density step; replaces the mu search of purification_search
 * (source/purification.f90:232-353) with trace correction.  nel must be even.
 * opts->precision selects FP64 or bf16x3 + FP64 refinement. */
int ptbgpu_tc_purify(ptbgpu_ctx* ctx, int64_t ndim, int64_t nel,
                     const double* Hpk, const double* Spk, double* Ppk,
                     const ptbgpu_opts* opts, ptbgpu_stats* st);

/* Same with device-resident packed arrays (no host copies); stream is a
 * cudaStream_t or NULL for the context's own stream. */
int ptbgpu_tc_purify_device(ptbgpu_ctx* ctx, int64_t ndim, int64_t nel,
                            const double* dHpk, const double* dSpk, double* dPpk,
                            const ptbgpu_opts* opts, ptbgpu_stats* st);

/* ptbgpu_tc_purify over ninst independent systems (system i: ndim[i], nel[i],
 * Hpk[i], Spk[i] in, Ppk[i] out), as the PTB driver would loop over many
 * molecules (the density step of source/pgtb.f90:599-618 once per system).  `workers` host
 * threads (0 = 4), each with its own worker context and stream on ctx's
 * device, take systems largest first, so that small systems overlap on the
 * GPU.  st may be NULL or point to ninst stats; wall_ms (may be NULL) gets the
 * host wall time of the whole batch.  The first failing system's status is
 * returned and named in ptbgpu_last_error(ctx); systems not yet started are
 * skipped then.  Worker contexts are kept for later batches and released by
 * ptbgpu_finalize(ctx). */
int ptbgpu_tc_purify_batch(ptbgpu_ctx* ctx, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                           const double* const* Hpk, const double* const* Spk, double* const* Ppk,
                           int64_t workers, const ptbgpu_opts* opts, ptbgpu_stats* st, double* wall_ms);

/* The density step of many independent systems in one launch of the library's
 * FP64 eigensolver: per system the filtered generalized eigenproblem
 * H_k U = S_k U e and P_k = 2 sum_{i < nel_k/2} u_i u_i^T (the dense projector
 * at T = 0, i.e. the reference's solve2, source/pgtb.f90:1066-1170, without the
 * Fermi smearing), P_k formed in the same launch; nel_k must be even (closed
 * shell: an odd count is EINVAL).  Systems up to order 1024 run
 * one CTA each in a persistent launch (largest first), larger ones (up to 12032)
 * one thread-block cluster each, beside them.  opts->filter is applied to H and
 * S (filter_matrix_sym).  Per-system stats carry flops; wall_ms the host time of
 * the call.  ENOTSPD names the first system whose S is not positive definite. */
int ptbgpu_eig_density_batch(ptbgpu_ctx* ctx, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                             const double* const* Hpk, const double* const* Spk, double* const* Ppk,
                             const ptbgpu_opts* opts, ptbgpu_stats* st, double* wall_ms);

/* The same systems purified together: bucketed by ndim rounded up to 256 and
 * padded within a bucket (decoupled padding: unit overlap, orthogonalised
 * diagonal at the system's upper spectral bound), stacked, and every step run
 * as one launch over all systems of a bucket (split-bf16 tcgen05 products over
 * the stacked planes, batched cuBLAS / cuSOLVER for the FP64 steps, per-system
 * branch and stop decisions on the device).  Results agree with
 * ptbgpu_tc_purify to the same tolerances (not bit for bit: the padded FP64
 * steps round differently).  A system the grouped path cannot finish is redone
 * by ptbgpu_tc_purify in FP64 (stats.fp64_fallback).  Per-system stats carry
 * iterations, refinement rounds and flops; wall_ms the host time of the call. */
int ptbgpu_tc_purify_grouped(ptbgpu_ctx* ctx, int64_t ninst, const int64_t* ndim, const int64_t* nel,
                             const double* const* Hpk, const double* const* Spk, double* const* Ppk,
                             const ptbgpu_opts* opts, ptbgpu_stats* st, double* wall_ms);

/* solve2(mode,ndim,nel,nopen,homo,et,focc,H,S,P,e,U,fail), source/pgtb.f90:1066-1170:
 * dense generalized eigensolve + Fermi smearing, the check-mode oracle.
 * e (ndim) and focc (ndim) may be NULL. */
int ptbgpu_solve2(ptbgpu_ctx* ctx, int64_t mode, int64_t ndim, int64_t nel, int64_t nopen,
                  const double* Hpk, const double* Spk, double* Ppk, double* e, double* focc,
                  const ptbgpu_opts* opts, ptbgpu_stats* st);

/* tr(PS) and tr(PH) (the nel and band_energy of ptbgpu_check_density) of
 * device-resident packed P, S, H without allocating any device memory and
 * without a context: for callers that own all device memory themselves (a
 * Fortran SCF driver with its own pool, a device already full with the
 * matrices of a large box) or cannot afford the device-wide synchronisation of
 * cudaMalloc/cudaFree.  No counterpart in the reference.  out (host, 2 doubles)
 * = {tr(PS), tr(PH)}; dHpk may be NULL (out[1] = 0).  Working memory is a
 * fixed 1 MB array in the library's device image: ndim <= 65536, larger sizes
 * are rejected with PTBGPU_EINVAL.  The CUDA runtime loads device code lazily
 * by default, so the first call on a device places this code and its 1 MB
 * array there and looks up the array's device address: a caller that will run
 * with the device full makes its first call early (or sets
 * CUDA_MODULE_LOADING=EAGER), and makes it before any stream capture.  After a
 * cudaDeviceReset of a device the kept address is stale: do not call again on
 * that device.  Calls share the array: calls whose kernels overlap on the GPU
 * race.  stream is a cudaStream_t (NULL: the legacy default stream); the call
 * returns after the stream has finished.  The caller's current device is the
 * same after the call as before.  err (may be NULL) receives the message of a
 * failure. */
int ptbgpu_density_traces_noalloc(int device, int64_t ndim, const double* dPpk, const double* dSpk,
                                  const double* dHpk, double* out, void* stream, char* err, size_t errlen);

/* The submatrix method in phases, for splitting one step over ranks (each rank
 * one device; no counterpart in the reference, which runs sm_stupid_simple on
 * one node).  The submatrices are independent; only the chemical-potential
 * bisection couples them, through the electron count, one scalar per step:
 *   ptbgpu_sm_plan     filter, grouping, pattern scan and maps on the whole
 *                      system (every rank, identical); dims(ndim) receives the
 *                      nsm submatrix dimensions (what a size-balanced assignment
 *                      of submatrices to ranks needs);
 *   ptbgpu_sm_prepare  gather, reduction, eigensolve and fe weights of this
 *                      rank's submatrices (0-based indices);
 *   ptbgpu_sm_nel      this rank's electron count at mu (sum over ranks = the
 *                      nel of source/sm.f90:322-340);
 *   ptbgpu_sm_finish   this rank's owned columns of P at mu, zeros elsewhere,
 *                      packed (the sum over ranks is the reference's P).
 * One rank preparing every submatrix and bisecting on the host reproduces
 * ptbgpu_sm_density exactly.  The plan stays on the context until the next
 * plan or ptbgpu_finalize. */
int ptbgpu_sm_plan(ptbgpu_ctx* ctx, int64_t ndim, const double* Hpk, const double* Spk, int64_t nat,
                   const double* xyz, const int64_t* aoat, int64_t submatrix_columns, int64_t submatrix_mode,
                   const int64_t* partition, const ptbgpu_opts* opts, int64_t* nsm, int64_t* dims);
int ptbgpu_sm_prepare(ptbgpu_ctx* ctx, int64_t nlocal, const int64_t* ids, ptbgpu_stats* st);
int ptbgpu_sm_nel(ptbgpu_ctx* ctx, double mu, double* nel);
int ptbgpu_sm_finish(ptbgpu_ctx* ctx, int64_t ndim, double mu, double* Ppk);

/* Columns mode 4 grouping, source/sm.f90:127-154 + clustering_kmeans :459-514
 * + KMPP source/kmpp.f: k-means++ on the atom positions for 1..min(64, nat)
 * clusters, keeping the partition with the least sum over submatrices of
 * dim^2.5 (dim from the H > 0 / S > 0 index-set test on the filtered H, S).
 * The reference's generator is global Fortran state shared by an OpenMP loop;
 * here each cluster count draws from its own splitmix64 stream derived from
 * `seed`, so the partition is reproducible.  partition(nat) receives 1-based
 * cluster ids (the input ptbgpu_sm_density takes in mode 4); nsm and effort
 * (may be NULL) the chosen count and its cost.  ptbgpu_sm_density in mode 4
 * with partition == NULL runs this with seed 42. */
int ptbgpu_kmeans_partition(ptbgpu_ctx* ctx, int64_t ndim, const double* Hpk, const double* Spk, int64_t nat,
                            const double* xyz, const int64_t* aoat, uint64_t seed, const ptbgpu_opts* opts,
                            int64_t* partition, int64_t* nsm, double* effort);

/* ---- population analysis on the produced P ------------------------------ */
/* mlpop14(nao, s, s34, s14), source/mlpop.f:142-190: s34 = S^(1-x) and s14 = S^x
 * in REAL*4 (nao x nao, column-major) from an FP32 eigen-decomposition of the
 * packed FP64 overlap Spk; x is mull_loew14 (source/parcom.f90:26: 1/3). */
int ptbgpu_mlpop14(ptbgpu_ctx* ctx, int64_t nao, const double* Spk, double x, float* s34, float* s14);
/* The same with device-resident Spk and device outputs. */
int ptbgpu_mlpop14_device(ptbgpu_ctx* ctx, int64_t nao, const double* dSpk, double x, float* d_s34,
                          float* d_s14);
/* mlpop2(n, nao, p, s1, s2, q, qsh), source/mlpop.f:198-235: atomic populations
 * q(n) and shell populations qsh(10, n) (Fortran order) from the diagonal of
 * s2 P s1, with P packed FP64 and s1 = S^(1-x), s2 = S^x REAL*4 column-major.
 * aoat(nao) (AO -> atom) and shell2ao(nao) (AO -> shell of its atom), 1-based,
 * are the bascom module arrays the Fortran routine reads.  The diagonal is
 * formed from one int8-sliced product (6 slices, exact int32 sums), more
 * accurate than the reference's REAL*4 ssymm + sgemm. */
int ptbgpu_mlpop2(ptbgpu_ctx* ctx, int64_t n, int64_t nao, const double* Ppk, const float* s1, const float* s2,
                  const int64_t* aoat, const int64_t* shell2ao, double* q, double* qsh, ptbgpu_stats* st);
/* The same with P (e.g. left on the device by ptbgpu_tc_purify_device), s1 and
 * s2 device-resident; aoat, shell2ao, q and qsh are host arrays. */
int ptbgpu_mlpop2_device(ptbgpu_ctx* ctx, int64_t n, int64_t nao, const double* dPpk, const float* d_s1,
                         const float* d_s2, const int64_t* aoat, const int64_t* shell2ao, double* q, double* qsh,
                         ptbgpu_stats* st);

/* ---- kernel-level entry points (parity tests and benchmarks) ------------ */
/* C = X * X for a symmetric n x n FP64 matrix X (row-major), computed with the
 * bf16x3 tcgen05 kernel (hi/lo split, FP32 accumulation); C is FP32 row-major. */
int ptbgpu_symsq_bf16x3(ptbgpu_ctx* ctx, int64_t n, const double* X, float* C);
/* The same with the three-plane split (hi, mid, lo) and six products, ~24-bit operands. */
int ptbgpu_symsq_bf16x6(ptbgpu_ctx* ctx, int64_t n, const double* X, float* C);
/* Either split with an explicit kernel: planes 2 or 3; kblock 32 or 64 (one CTA,
 * that K block), 1032 or 1064 (two planes only: the CTA-pair cta_group::2
 * kernel with K block 32 or 64), or 0 (the autotuned choice). */
int ptbgpu_symsq_split(ptbgpu_ctx* ctx, int64_t n, int64_t planes, int64_t kblock, const double* X, float* C,
                       double* ms);   /* ms (may be NULL): device time of the product launch(es) */
/* C = A * B for n x n FP64 row-major host matrices, on the int8 tensor cores
 * with `slices` (6..8) 7-bit slices per operand row and an int32-exact K loop;
 * kblock 32 or 64 bytes (0 = default); variant 0 default (5 for 6 to 8
 * slices unless kblock is 64, else 1), 1 A slices read from shared memory by
 * every MMA, 2 A slices copied into tensor memory once per K step, 3 variant 1
 * on a CTA pair (256-row tiles, cta_group::2), 4 128-column tiles with the
 * accumulator groups summed in two passes over K (kblock 0 or 32), 5 variant 4
 * on a CTA pair (256 x 128 tiles), all bit-identical.  tri_a / tri_b: 0 full, 1 lower, 2 upper
 * triangular (the other part is read as zero and its K blocks are skipped);
 * symmetric != 0: only the upper triangle of C is computed and mirrored.
 * n <= (2^31 - 1) / (slices * 127^2) rounded down to a multiple of 128.
 * ms (may be NULL) receives the device time of the product kernel. */
/* The tile list that ptbgpu_oz_gemm's product launches for the same n, slices,
 * kblock and variant (host logic only: no context, no device).  a_tri / b_tri
 * mask the rows of the two K-major operands (rows of A and of B^T): 0 none,
 * 1 k <= i, 2 k >= i.  symmetric != 0: only tiles touching the upper triangle.
 * Writes min(cap, count) tiles as int32 {row block (pair row block for the
 * CTA-pair variants), column block, k0, k1} into tiles, the count into
 * *ntiles, and info[0] = the resolved variant, info[1] = columns per tile,
 * info[2] = CTAs launched, info[3] = rows per tile entry.  No counterpart in
 * the reference. */
int ptbgpu_oz_tiles(int64_t n, int64_t slices, int64_t kblock, int64_t variant, int64_t a_tri, int64_t b_tri,
                    int64_t symmetric, int32_t* tiles, int64_t cap, int64_t* ntiles, int64_t* info);
int ptbgpu_oz_gemm(ptbgpu_ctx* ctx, int64_t n, int64_t slices, int64_t kblock, int64_t variant, int64_t tri_a,
                   int64_t tri_b, int64_t symmetric, const double* A, const double* B, double* C, double* ms);

/* The batched FP64 generalized eigensolver of the submatrix method on dense
 * host problems (kernel-level entry for tests and measurements; it replaces the
 * per-submatrix la_sygvd and the S_k U product of source/sm.f90:296-310).
 * Orders up to 1024 run one CTA per problem in a persistent launch, larger ones
 * one thread-block cluster per problem.  nprob problems of orders dims[k]
 * (1..10240): H and S hold their column-major dims[k]^2 blocks one after
 * another; owned holds nown[k] (0-based, local) owned indices per problem, one
 * list after another.  Out: e and fe (sum of dims each, per problem in the
 * solver's order, not sorted): the eigenvalues of H c = e S c and the weights
 * fe_j = sum_c (S U)_{c,j} U_{c,j} over the owned rows c.  With Pcols non-NULL
 * also the owned columns of P = U occ U^T with occ = 2 / 1 / 0 for e < / = / > mu
 * (dims[k] x nown[k] column-major per problem, one after another).  ENOTSPD
 * if an S block is not positive definite. */
int ptbgpu_sygv_batched(ptbgpu_ctx* ctx, int64_t nprob, const int64_t* dims, const double* H, const double* S,
                        const int64_t* nown, const int64_t* owned, double mu, double* e, double* fe,
                        double* Pcols);

/* ---- consumer of P in the next SCF iteration ---------------------------- */
/* The iteration-2 XC long-range damping of twoscf (source/pgtb.f90:482-513) on
 * the packed arrays: xab(lin(a,b)) = (1 + erf(-1.8 (rab - r)/r))/2 with
 * r = rad(a) + rad(b) over atom pairs, then Hpk(k) += Ppk(k) (hao(i) + hao(j))
 * xab(lin(aoat(j), aoat(i))) for j < i and Hpk(k) += 2 Ppk(k) xdiag(i) hao(i)
 * xab(lin(aoat(i), aoat(i))) on the diagonal.  rad(nat) is the special radius
 * shell_cnf3(10,at) + (cn - avcn(at)) shell_resp(10,at,1); hao(ndim) is
 * shell_cnf2(shell2ao(i), at(aoat(i))) * gq(aoat(i)); xdiag(ndim) is
 * shell_xi(8, at(aoat(i))); rab is the packed atom-pair distance array
 * (nat(nat+1)/2).  aoat(i) outside 1..nat -> PTBGPU_EINVAL.  ms_update (may be
 * NULL) gets the device time of the AO-pair update. */
int ptbgpu_xc_damping(ptbgpu_ctx* ctx, int64_t nat, int64_t ndim, const int64_t* aoat, const double* rab,
                      const double* rad, const double* hao, const double* xdiag, const double* Ppk, double* Hpk,
                      double* ms_update);
/* The same with Ppk and Hpk device-resident (e.g. P left on the device by
 * ptbgpu_tc_purify_device, H to be passed on to the next density step);
 * aoat, rab, rad, hao, xdiag are host arrays.  dPpk and dHpk must start on a
 * 16-byte boundary (PTBGPU_EINVAL otherwise). */
int ptbgpu_xc_damping_device(ptbgpu_ctx* ctx, int64_t nat, int64_t ndim, const int64_t* aoat, const double* rab,
                             const double* rad, const double* hao, const double* xdiag, const double* dPpk,
                             double* dHpk, double* ms_update);

/* ---- self-test ------------------------------------------------------------ */
/* No counterpart in the reference.  Runs one bounded device wait on a flag that
 * nothing sets, with a limit of limit_us (1..2e6) microseconds, through the
 * same error path as the library's kernels' waits: returns PTBGPU_ETIMEOUT with
 * a message naming the site, and leaves the context usable.  For testing the
 * failure path without faulting or hanging a GPU. */
int ptbgpu_selftest_bounded_wait(ptbgpu_ctx* ctx, int64_t limit_us);

#ifdef __cplusplus
}
#endif
#endif /* PTBGPU_H */
