/*
 * iccg.h -- C ABI of iccg_b200, a Blackwell (sm_100a) implementation of the
 * preconditioned conjugate-gradient hot path of stomo0511/ICCG.
 *
 * Plain C types only: ints, doubles, pointers and sizes.  Every function
 * returns an int status (ICCG_OK = 0) unless stated otherwise; no C++
 * exception crosses this boundary.  A context (iccg_ctx) owns one CUDA stream
 * and the device-resident matrix, schedule, preconditioner and work vectors
 * of one linear system.  A context is not thread-safe; use one per thread or
 * per system.  Any number of contexts may live on one device.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * stomo0511/ICCG).  The CRS layout is the reference's (crs_io.hpp:10-49):
 * 0-based int32 rowptr[n+1], int32 colind[nnz] (ascending within a row),
 * double val[nnz].  The schedule arrays are the reference's ColorSchedule
 * (color.hpp:9-22).
 */
#ifndef ICCG_H
#define ICCG_H

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define ICCG_OK 0
#define ICCG_ERR_ARG (-1)           /* bad size / index / pointer              */
#define ICCG_ERR_DIAG (-2)          /* IC(0): diagonal missing   (ic0.cpp:52)  */
#define ICCG_ERR_PIVOT_ZERO (-3)    /* IC(0): |L_jj| < 1e-30     (ic0.cpp:86)  */
#define ICCG_ERR_PIVOT_NONPOS (-4)  /* IC(0): pivot <= 0         (ic0.cpp:104) */
#define ICCG_ERR_IO (-5)            /* malformed or unreadable file            */
#define ICCG_ERR_NOMEM (-6)         /* host or device allocation failed        */
#define ICCG_ERR_CUDA (-7)          /* CUDA runtime error                      */
#define ICCG_ERR_STATE (-8)         /* call order (e.g. apply before build)    */
#define ICCG_ERR_SCHEDULE (-9)      /* schedule violates a dependency          */
#define ICCG_ERR_NONFINITE (-10)    /* NaN/Inf in a CG scalar                  */

/* ---- enums ------------------------------------------------------------- */
#define ICCG_PRECOND_NONE 0      /* Identity  (precond.hpp:8-17)           */
#define ICCG_PRECOND_JACOBI 1    /* Jacobi    (precond.hpp:19-45)          */
#define ICCG_PRECOND_IC0 2       /* IC0       (ic0.hpp:11-76)              */

#define ICCG_SCHED_NONE 0        /* natural order (iccg_crs)               */
#define ICCG_SCHED_MC 1          /* ColorSchedule::MC_NODE                 */
#define ICCG_SCHED_ABMC 2        /* ColorSchedule::ABMC_BLOCK              */

#define ICCG_STORE_FP64 0        /* A and L stored in FP64                 */
#define ICCG_STORE_FP32 1        /* A and L stored in FP32, FP64 vectors   */

#define ICCG_MODE_PLAIN 0        /* one kernel per reference operation,
                                    scalars checked on the host each
                                    iteration (the plain FP64 GPU path)    */
#define ICCG_MODE_FUSED 1        /* fused kernels, device-side scalars,
                                    iterations replayed as a CUDA graph    */

/* CG result (cg_crs.cpp:82-86) plus what the reference prints afterwards. */
typedef struct {
    int iters;               /* CGResult::iters                           */
    int converged;           /* CGResult::converged                       */
    int status;              /* 0 converged, 1 breakdown, 2 max_iter      */
    int n_replacements;      /* FP64 residual replacements performed      */
    double rel_resid;        /* CGResult::rel_resid (recurrence)          */
    double true_rel_resid;   /* ||b - A x|| / ||b|| in FP64 (cg_crs.cpp:518-528) */
    double solve_ms;         /* device time of the solve (CUDA events)    */
} iccg_result;

typedef struct {
    int mode;          /* ICCG_MODE_PLAIN or ICCG_MODE_FUSED                  */
    int storage;       /* ICCG_STORE_FP64 or ICCG_STORE_FP32                  */
    int rr_interval;   /* FP64 residual replacement every k iterations
                          (FP32 storage only; 0 = off; default 50)           */
    int graph_iters;   /* FUSED: iterations per graph launch (default 16)    */
} iccg_solve_opts;

typedef struct iccg_ctx iccg_ctx;
typedef struct iccg_crs iccg_crs;

/* ======================================================================= */
/* Host-side CRS objects and file formats                                   */
/* ======================================================================= */

/* read_matrix_market_crs (crs_io.hpp:52, crs_io.cpp:73-159) */
int iccg_mm_read(const char* path, iccg_crs** out);
/* writes A (full) as MatrixMarket coordinate real; symmetric=1 writes the
   lower triangle with a `symmetric` header */
int iccg_mm_write(const char* path, int n, const int* rowptr, const int* colind,
                  const double* val, int symmetric);
/* wraps caller arrays into a new CRS object (copies) */
int iccg_crs_create(int n, const int* rowptr, const int* colind, const double* val,
                    iccg_crs** out);
int iccg_crs_dims(const iccg_crs* a, int* n, int* nnz);
int iccg_crs_copy(const iccg_crs* a, int* rowptr, int* colind, double* val);
void iccg_crs_free(iccg_crs* a);

/* ReadColorFile_1Based (color.cpp:14-47)        kind 0
   ReadBlockFile_1Based (block.cpp:15-51)        kind 1
   ReadBlockColorFile_1Based (block.cpp:53-89)   kind 2
   out[n_expected] receives 0-based ids, *k_out the count in the header. */
int iccg_read_assignment(int kind, const char* path, int n_expected, int* out, int* k_out);
/* writes the same formats (1-based), k = header count */
int iccg_write_assignment(const char* path, int n, const int* values0, int k);

/* ======================================================================= */
/* Orderings and schedules (bit-exact with the reference)                   */
/* ======================================================================= */

/* BuildPermutationByColor (color.cpp:50-63) */
int iccg_perm_by_color(int n, const int* color, int* new_of_old);
/* BuildPermutationByBlockColor (block.cpp:92-114) */
int iccg_perm_by_block_color(int n, int nb, const int* block_of_old, const int* block_color,
                             int* new_of_old);
/* Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141).  cap >= number of
   entries with j <= i in the input; *out_nnz receives the result size. */
int iccg_ptap_lower(int n, const int* rowptr, const int* colind, const double* val,
                    const int* new_of_old, int cap, int* out_rowptr, int* out_colind,
                    double* out_val, int* out_nnz);
/* expand_lower_to_full (crs_io.hpp:56, crs_io.cpp:163-227) */
int iccg_expand_lower_nnz(int n, const int* rowptr, const int* colind, int* out_nnz);
int iccg_expand_lower_to_full(int n, const int* rowptr, const int* colind, const double* val,
                              int* out_rowptr, int* out_colind, double* out_val);
/* Permute_PtAP_LowerCRS_to_LowerCRS (color.cpp:66-141) followed by
   expand_lower_to_full (crs_io.cpp:163-227), the caller's A_run
   (cg_crs.cpp:419-421), computed on CUDA device `device`: host arrays in,
   the full permuted matrix into out_rowptr[n+1], out_colind[cap],
   out_val[cap]; *out_nnz receives its size (also when cap is too small, with
   ICCG_ERR_ARG).  The same bits as iccg_ptap_lower + iccg_expand_lower_to_full:
   each output entry is one input value when no (i, j) pair repeats; inputs
   that repeat a pair (whose sums depend on the order) or give output rows of
   more than 256 entries are computed by those host routines instead, and
   *on_device (may be NULL) receives 0.  2 * nnz of the input bounds the
   output size. */
int iccg_ptap_full_gpu(int device, int n, const int* rowptr, const int* colind, const double* val,
                       const int* new_of_old, int cap, int* out_rowptr, int* out_colind, double* out_val,
                       int* out_nnz, int* on_device);
/* BuildColorPtrRows_FromPermutationAndColor (color.cpp:164-197) */
int iccg_color_schedule(int n, const int* color, int nc, const int* new_of_old,
                        int* color_ptr, int* rows_of_color);
/* BuildABMCSchedule (block.cpp:116-174) */
int iccg_abmc_schedule(int n, const int* new_of_old, const int* block_of_old,
                       const int* block_color, int nb, int nc, int* color_ptr_blk,
                       int* blocks_of_color, int* block_ptr, int* rows_of_block);
/* DebugCheck_InterBlockSameColorEdges (cg_crs.cpp:171-224): returns the total
   count (>= 0) or ICCG_ERR_ARG; per-color counts into by_color[nc] if given. */
long long iccg_check_interblock_same_color(int n, const int* rowptr, const int* colind,
                                           const int* block_of_old, const int* block_color,
                                           int nb, int nc, long long* by_color);
/* DebugCheck_ScheduleHazards_OnLower (cg_crs.cpp:259-336): same-color j<i
   dependencies in the lower pattern of the permuted matrix. */
long long iccg_check_schedule_hazards(int n, const int* rowptr, const int* colind,
                                      const int* new_of_old, const int* color_old,
                                      const int* block_of_old, long long* same_block,
                                      long long* cross_block);

/* ======================================================================= */
/* Problem generators (no counterpart in the reference, whose inputs come   */
/* from SuiteSparse and an external igraph tool, run_*.sh, check_igraph.cpp) */
/* ======================================================================= */

#define ICCG_GEN_2D5 0   /* 5-point, diag 2(wx+wy), off -wx/-wy               */
#define ICCG_GEN_3D7 1   /* 7-point, diag 2(wx+wy+wz), off -wx/-wy/-wz         */
int iccg_gen_stencil(int kind, int nx, int ny, int nz, double wx, double wy, double wz,
                     iccg_crs** out);
/* 27-point cell-centred diffusion on nx*ny*nz cells; coefficients are the
   harmonic means of exp(sigma*g), g a unit-variance Gaussian field smoothed
   by a 3-cell box filter, sigma set so max/min of the field = contrast. */
int iccg_gen_diffusion27(int nx, int ny, int nz, double contrast, unsigned long long seed,
                         iccg_crs** out);
/* symmetrised k-nearest-neighbour graph Laplacian of npts uniform points in
   the unit square, weights 1/dist, plus diag_shift * I */
int iccg_gen_knn_laplacian(int npts, int k, double diag_shift, unsigned long long seed,
                           iccg_crs** out);
/* x[i] ~ U(-1,1) from splitmix64(seed): ((u >> 11) * 2^-53) * 2 - 1 */
int iccg_gen_uniform(int n, unsigned long long seed, double* out);
/* y = A x on the host in CSR order with spmv's rounding (cg_crs.cpp:68-77:
   product and sum rounded separately); used to form b = A x* */
int iccg_host_spmv(int n, const int* rowptr, const int* colind, const double* val, const double* x, double* y);
/* greedy node coloring in natural order (smallest free color) */
int iccg_color_greedy(int n, const int* rowptr, const int* colind, int* color, int* nc);
/* ABMC blocking: method 0 = consecutive ids, 1 = breadth-first aggregation */
int iccg_block_partition(int n, const int* rowptr, const int* colind, int block_size,
                         int method, int* block_of_old, int* nb);
/* greedy coloring of the block quotient graph in block-id order */
int iccg_color_blocks(int n, const int* rowptr, const int* colind, const int* block_of_old,
                      int nb, int* block_color, int* nc);

/* ======================================================================= */
/* Device context                                                           */
/* ======================================================================= */

int iccg_ctx_create(int device, iccg_ctx** out);
int iccg_ctx_destroy(iccg_ctx* ctx);
/* message of the last failing call on this context (never NULL) */
const char* iccg_ctx_last_error(const iccg_ctx* ctx);
/* message of the last failing context-free call on this thread */
const char* iccg_last_error(void);
/* the context's cudaStream_t, as void* */
void* iccg_ctx_stream(iccg_ctx* ctx);
/* number of kernels this context has launched so far (graph nodes count
   once per replay) */
long long iccg_ctx_launch_count(const iccg_ctx* ctx);
/* bytes of device memory held by this context */
long long iccg_ctx_device_bytes(const iccg_ctx* ctx);
/* context options.
   ICCG_OPT_TILED (default 1): 1 runs the lane-interleaved kernels (an
   internal row order with 32 independent units per warp, SELL-32 storage);
   0 forces the CSR kernels (one thread per row / per unit).
   ICCG_OPT_SWEEP (default 0), lane-interleaved substitutions: 0 uses the
   staged kernel (batches of rows copied into shared memory) where a batch
   fits shared memory, 1 forces the per-slice two-phase kernel.
   ICCG_OPT_PDL (default 1): 1 launches kernels with programmatic dependent
   launch: the per-iteration kernels let the next launch start once their
   main loop is done, so it is placed while their tail (the reduction) runs;
   every kernel still waits for its predecessor's results.  0 launches each
   kernel after its predecessor has finished.
   ICCG_OPT_STAGE_KB (default 0): shared memory, in KB, that two stage
   buffers of the staged kernel may fill (batches are sized for two, so they
   also fit the default single buffer); 0 takes the device's opt-in maximum
   per block.  Smaller batches leave room for
   more resident CTAs per SM.  A level with a group of units that alone
   exceeds it runs on the per-slice kernel.  Setting it re-plans the
   batches of a built preconditioner.
   ICCG_OPT_STAGE_BUFS (default 1): stage buffers per CTA of the staged
   kernel; 1 refills a CTA's one buffer after each batch, 2 copies the next
   batch into a second buffer while the current one is worked on.  One
   buffer halves a CTA's shared memory, so twice as many CTAs share an SM
   and overlap each other's copies; on the 128^3 system that was faster.
   Every choice gives the same bits with FP64 storage.
   ICCG_OPT_PERSIST (default 0): 1 runs each IC(0) apply -- both
   substitution sweeps, every level -- as one persistent launch in which
   CTAs take the staged batches from a ticket counter and wait only for the
   batches whose rows they read; in a fused solve the same launch also does
   the CG update x += alpha p, r -= alpha Ap and r.r.  0 launches one kernel
   per level (ICCG_OPT_SWEEP chooses which).  It applies where every level
   is staged.  FP64 results are the same bits either way.
   ICCG_OPT_FUSE_UPDATE (default 0), lane-interleaved fused solves with the
   per-level kernels: 1 does the CG update x += alpha p, r -= alpha Ap and
   the r.r reduction inside the forward sweep's launches (where every
   forward level runs the chain-only or single-buffered staged kernel), so
   the update needs no launch and r is not read back; 0 launches the update
   on its own.  Iterations with a residual replacement always update on
   their own.  The fused form stages r and Ap with each batch, writes the new
   r back, and leaves x += alpha p to the p update (k_xpay); the same bits
   as the update on its own.  On the 128^3 ABMC system it is slower
   (22.50 against 21.78 ms mixed, 34.85 against 32.66 ms FP64): the
   chain-only forward level, latency-bound, loses more than the launch and
   the bytes saved; it is kept as an option.
   ICCG_OPT_DEFER_X (default 0), fused solves: x += alpha p is done by the p
   update (p = z + beta p), which reads p anyway, instead of by the r update:
   8 bytes per row less per iteration.  A solve that stops between the two
   gets the pending x update before its true residual.  Iterations with an
   FP64 residual replacement update x with r.  The same bits either way;
   measured slightly slower on the 128^3 ABMC system (21.26 against 21.15 ms
   mixed, 32.39 against 32.00 ms FP64), so it is kept as an option.
   ICCG_OPT_SPMV_PACK (default 1), lane-interleaved FP32 SpMV: the matrix
   entries are read as one 8-byte word of value and column instead of two
   4-byte loads (an extra packed copy of A's FP32 values and columns).  The
   same bits either way.
   ICCG_OPT_STAGE_ROWS (default 256, 32 to 8192): the staged sweep's batches
   hold up to 16 unit groups and this many rows (a single larger group is one
   batch); more rows give more chains per CTA and larger stage buffers, fewer
   CTAs per SM.  The same bits for any value.  256 against 512: the 96^3
   27-point multicolor solve 23.95 -> 22.12 ms mixed and 25.17 -> 23.95 ms
   FP64, ABMC B=8 20.76 -> 20.47 and 40.63 -> 39.53 ms, the 128^3 7-point
   ABMC B=16 solve unchanged (its batches are single 512-row groups).
   ICCG_OPT_SPMV_TPR (default 1; 2 or 4), FP32 storage: threads per row of
   the SpMV, for matrices with long rows.  Each of the TPR threads sums every
   TPR-th entry of the row and the partial sums are added in a fixed order:
   deterministic, but not the single CSR-order sum of 1 thread per row, so
   FP32-storage results change in their last bits (FP64 storage always uses
   one thread per row and the reference's order).
   ICCG_OPT_EARLY (default 1; 0 to 3): loads before the wait on the previous
   launch, per storage (bit 0: FP32 storage, bit 1: FP64).  With programmatic
   dependent launch each hot kernel lets the next launch in right after its
   own wait, and before its wait loads what the launch just before cannot
   write: the SpMV's first slice of A, the sweeps' first batch of L (and the
   input rows / r where they are older), the update's r, x, p and the p
   update's p, x for each thread's first two pairs.  Staged sweep levels of
   fewer than two CTAs per SM run without it.  The same bits either
   way.  The 128^3 ABMC mixed solve 21.15 -> 19.95 ms and the 96^3 27-point
   multicolor one 21.18 -> 19.54 ms; the FP64 fused solve 32.2 -> 33.3 ms, so
   FP64 storage keeps it off by default.
   ICCG_OPT_UPDATE_CHAIN (default 0): where the first forward level is
   chain-only (every row's one in-unit entry is the previous step of its
   unit), the CG update kernel also does that level: x += alpha p for every
   row, r -= alpha Ap, and the level's chains from the new r, in one launch
   (k_update_chain).  The same bits.  Slower on the systems measured (128^3
   ABMC mixed 19.91 -> 20.39 ms, FP64 32.00 -> 32.38; 96^3 27-point
   multicolor mixed 19.56 -> 19.72), so off by default; the tuner tries it. */
#define ICCG_OPT_TILED 0
#define ICCG_OPT_SWEEP 1
#define ICCG_OPT_PDL 2
#define ICCG_OPT_STAGE_KB 3
#define ICCG_OPT_STAGE_BUFS 4
#define ICCG_OPT_PERSIST 5
#define ICCG_OPT_FUSE_UPDATE 6
#define ICCG_OPT_DEFER_X 7
#define ICCG_OPT_SPMV_PACK 8
#define ICCG_OPT_STAGE_ROWS 9
#define ICCG_OPT_SPMV_TPR 10
#define ICCG_OPT_EARLY 11
#define ICCG_OPT_UPDATE_CHAIN 12
int iccg_ctx_set_option(iccg_ctx* ctx, int option, long long value);

/* Uploads A_run (the matrix conjugate_gradient runs on, cg_crs.cpp:442-447):
   full symmetric CRS with ascending columns.  Keeps an FP64 copy and, on
   first FP32-storage use, an FP32 copy of the values. */
int iccg_matrix_upload(iccg_ctx* ctx, int n, const int* rowptr, const int* colind,
                       const double* val);

/* ColorSchedule with mode MC_NODE (color.hpp:9-13, cg_crs.cpp:468-471) */
int iccg_schedule_mc(iccg_ctx* ctx, int nc, const int* color_ptr, const int* rows_of_color);
/* ColorSchedule with mode ABMC_BLOCK (color.hpp:15-21, cg_crs.cpp:474-481) */
int iccg_schedule_abmc(iccg_ctx* ctx, int nc, int nb, const int* color_ptr_blk,
                       const int* blocks_of_color, const int* block_ptr,
                       const int* rows_of_block);
/* sched == nullptr: natural-order substitutions (ic0.cpp:368) */
int iccg_schedule_none(iccg_ctx* ctx);

/* Preconditioner construction: Identity(A) / Jacobi(A) / IC0(A, shift)
   (precond.hpp:10, precond.hpp:23-36, ic0.cpp:6-12).  IC(0) is factored on
   the device in the schedule's order.  auto_shift != 0: on a non-positive
   pivot the factorisation restarts with shift = max(2*shift, 1e-3*max|a_ii|)
   (at most 40 restarts) instead of failing (the reference throws,
   ic0.cpp:104-113).  The shift is added to every pivot, as the reference's
   shift argument is (ic0.cpp:103).  The factor is
   stored in FP64 and, for FP32-storage solves, also rounded to FP32. */
int iccg_precond_build(iccg_ctx* ctx, int kind, double shift, int auto_shift);
/* the shift the last IC(0) build ended with */
double iccg_precond_shift(const iccg_ctx* ctx);

/* Precond::apply(r, z, sched) (precond.hpp:12, precond.hpp:38, ic0.hpp:34,
   ic0.cpp:366-393) with host vectors; storage selects FP64 or FP32 factor. */
int iccg_precond_apply(iccg_ctx* ctx, const double* r, double* z, int storage);
/* same with device pointers on the context's stream */
int iccg_precond_apply_dev(iccg_ctx* ctx, const double* r, double* z, int storage);

/* exports the device IC(0) factor in the reference's layout: L (CRS, lower +
   diagonal, ic0.hpp:41-44) and L^T (CSC of L, ic0.hpp:46-48).  nnzL via
   iccg_precond_nnz. */
int iccg_precond_nnz(const iccg_ctx* ctx, int* nnzL);
int iccg_precond_export(iccg_ctx* ctx, int* Lp, int* Li, double* Lx, int* Up, int* Ui,
                        double* Ux);

/* spmv (cg_crs.cpp:54-79), host vectors / device vectors */
int iccg_spmv(iccg_ctx* ctx, const double* x, double* y, int storage);
int iccg_spmv_dev(iccg_ctx* ctx, const double* x, double* y, int storage);

/* dot / nrm2 (cg_crs.cpp:33-50) on device vectors, evaluated in double-double
   and rounded once to double */
int iccg_dot_dev(iccg_ctx* ctx, int n, const double* a, const double* b, double* out);

/* iccg_dot_dev without a context and without any device allocation.  No
   counterpart in the reference: it exists for callers that cannot call
   cudaMalloc (a host whose allocator has reserved the device memory for its
   own pool, or a latency-bound loop in which the device-wide
   synchronisation of cudaMalloc/cudaFree is not allowed).
   a, b: n doubles in device memory; out: one double in device memory,
   written asynchronously on `stream` (a cudaStream_t, NULL = default
   stream).  The same double-double evaluation as iccg_dot_dev; each block
   of 4096 elements is summed by one CTA, so the result depends only on the
   inputs.  Its scratch is a fixed static device array (64 KiB) inside the
   library, which limits n to ICCG_NOALLOC_MAX_N; larger n is rejected with
   ICCG_ERR_ARG (message via iccg_last_error).
   The first call on each device does a set-up (finds the scratch address
   and clears its counter, synchronising `stream`); make it before any
   stream capture.  Calls that overlap in time on one device (two host
   threads, or two streams running concurrently) share the scratch and race:
   serialise them.  The scratch address found by that set-up is kept for the
   life of the process: after cudaDeviceReset (or any teardown of the
   device's primary context) the library's device image is loaded anew, and
   this entry point must not be called on that device again. */
#define ICCG_NOALLOC_MAX_N 16777216
int iccg_dot_dev_noalloc(int n, const double* a, const double* b, double* out, void* stream);

/* conjugate_gradient<Precond> (cg_crs.cpp:89-162) on A_run with the built
   preconditioner and schedule.  x holds x0 on entry and the solution on
   return.  opts may be NULL (FUSED, FP64, rr 50, graph 8). */
int iccg_solve(iccg_ctx* ctx, const double* b, double* x, int max_iter, double tol,
               const iccg_solve_opts* opts, iccg_result* res);
int iccg_solve_dev(iccg_ctx* ctx, const double* b, double* x, int max_iter, double tol,
                   const iccg_solve_opts* opts, iccg_result* res);

/* per-kernel-class device time of the last solve run with profiling on:
   class 0 SpMV, 1 forward sweep, 2 backward sweep, 3 vector/reduction
   kernels, 4 residual replacement, 5 persistent IC(0) apply (both sweeps,
   and in a fused solve the CG update).  enable != 0 brackets every launch of
   the following solves with CUDA events (launches are not graphed then). */
int iccg_profile_enable(iccg_ctx* ctx, int enable);
int iccg_profile_read(iccg_ctx* ctx, int cls, double* total_ms, long long* launches);

/* The substitution kernel that each level (color) of the IC(0) sweeps runs
   on, for storage ICCG_STORE_FP64 / ICCG_STORE_FP32 and the forward (fwd != 0)
   or backward sweep: kinds[l] = 0 chain-only, 1 staged, 2 per-slice
   two-phase, 3 one-phase (units of more than 64 rows), 4 CSR (untiled
   path), 5 the persistent apply (all levels in one launch); grids[l] =
   CTAs launched.  *nlevels receives the level count and
   at most cap entries are written.  Sets up the FP32 copies on first use,
   as a solve would.  No counterpart in the reference (its sweeps have one
   OpenMP form, ic0.cpp:194-339). */
int iccg_sweep_plan(iccg_ctx* ctx, int storage, int fwd, int* kinds, int* grids, int cap, int* nlevels);

/* ---------------------------------------------------------------------------
   Batched solves: many independent conjugate_gradient runs (cg_crs.cpp:89-162)
   advanced together, one kernel launch per CG step for all of them.  The
   reference solves one system per call (main_abmc.cpp, main_piccg.cpp); a
   caller with many systems loops over it.  No counterpart in the reference.

   A batch holds systems: contexts with a matrix, a schedule and a built IC(0)
   preconditioner (the caller keeps ownership; a context must stay alive and
   unchanged while the batch solves with it, and is not used by other calls
   meanwhile).  Every level of each system's sweeps must fit the staged
   substitution kernel (iccg_sweep_plan kind 1 or 0), which holds for the
   multicolor and ABMC schedules of the 7- and 27-point problems.

   iccg_batch_solve runs nsolve solves (no session solve may be in flight:
   see iccg_batch_open below): solve s is system system[s] (an index
   returned by iccg_batch_add_system) with the right-hand side b[s] and the
   initial guess / solution x[s] (host arrays of that system's n doubles, A_run
   order).  Each solve gives the same iterations, status, residuals and the
   same bits of x as iccg_solve on its context alone with the same opts, in
   any batch (mode must be ICCG_MODE_FUSED).  res[s].solve_ms is the device
   time from the start of the batch to the iteration at which solve s stopped;
   iccg_batch_device_ms gives the whole batch's device time.  Solves of one
   system are best placed next to each other: each level's matrix data is
   then read from DRAM once for all of them.
   --------------------------------------------------------------------------- */
typedef struct iccg_batch iccg_batch;
int iccg_batch_create(int device, iccg_batch** out);
int iccg_batch_destroy(iccg_batch* batch);
const char* iccg_batch_last_error(const iccg_batch* batch);
long long iccg_batch_launch_count(const iccg_batch* batch);
long long iccg_batch_device_bytes(const iccg_batch* batch);
double iccg_batch_device_ms(const iccg_batch* batch);
int iccg_batch_add_system(iccg_batch* batch, iccg_ctx* ctx, int* index);
int iccg_batch_clear(iccg_batch* batch);
int iccg_batch_solve(iccg_batch* batch, int nsolve, const int* system, const double* const* b,
                     double* const* x, int max_iter, double tol, const iccg_solve_opts* opts,
                     iccg_result* res);
/* A system whose solves have all been retired leaves the batch; its index
   may be given to a later iccg_batch_add_system. */
int iccg_batch_remove_system(iccg_batch* batch, int index);

/* Continuous batching (a serving loop): solves enter and leave while others
   run.  iccg_batch_open starts a session of `slots` solve slots with the
   given options (storage, rr_interval, graph_iters; mode must be FUSED); no
   solve may be in flight.  iccg_batch_submit admits a solve of system
   `system` into a free slot (*slot receives it): b and x0 (x0 NULL = zeros)
   are copied before it returns; its start-up (r0, z0, p0) runs with the next
   step.  iccg_batch_step advances every running solve graph_iters
   iterations in one graph launch (each CG kernel one launch over all of
   them), waits for it, and writes up to cap slots whose solves stopped and
   were not reported before into stopped[] (*nstopped of them; the rest come
   with the next calls); *nrunning (may be NULL) receives the solves still
   running or waiting to start.  iccg_batch_retire copies the solutions of
   n stopped solves into x[i] (host, n doubles of the solve's system, A_run
   order), fills res[i] (solve_ms: device time from admission to the stop)
   and frees their slots.  A solve gives the same bits, iterations and
   residuals as iccg_solve on its context alone, whatever runs beside it. */
int iccg_batch_open(iccg_batch* batch, int slots, const iccg_solve_opts* opts);
int iccg_batch_submit(iccg_batch* batch, int system, const double* b, const double* x0, int max_iter,
                      double tol, int* slot);
int iccg_batch_step(iccg_batch* batch, int* stopped, int cap, int* nstopped, int* nrunning);
int iccg_batch_retire(iccg_batch* batch, int n, const int* slots, double* const* x, iccg_result* res);

/* free and total device memory of `device` (cudaMemGetInfo), for admission
   by free device memory */
int iccg_device_memory(int device, long long* free_bytes, long long* total_bytes);

#ifdef __cplusplus
}
#endif
#endif /* ICCG_H */
