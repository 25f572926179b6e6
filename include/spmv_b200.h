/*
 * spmv_b200.h - C ABI of the B200 (sm_100a) implementation of libspmv's hot
 * path: the distributed CSR product (spmv::Matrix), the ghost map and halo
 * exchange (spmv::L2GMap) and conjugate gradients (spmv::cg).
 *
 * Conventions
 *  - Every entry point returns an int status (SPMV_SUCCESS == 0).  On failure
 *    spmv_last_error() returns the message of the calling thread's last error;
 *    where the reference throws std::runtime_error, the message is the same
 *    string (e.g. "Ghosts must be sorted", L2GMap.cpp:35).
 *  - The reference is an MPI library: one rank holds one row block.  Here one
 *    spmv_comm is a *virtual communicator* of `size` ranks that all live on one
 *    GPU.  Calls that are collective in the reference (L2GMap construction,
 *    update, reverse_update, cg) take the arrays of all ranks at once: an
 *    argument declared `T const* x` with the comment "[size]" holds one entry
 *    per rank, in rank order.
 *  - Vectors are passed per rank as plain pointers.  With SPMV_MEMORY_HOST the
 *    call copies them to the device, runs the kernels and copies results back
 *    before returning.  With SPMV_MEMORY_DEVICE they are device pointers and
 *    the call is ordered on the communicator's CUDA stream.
 *  - The library owns device copies of matrices and maps; callers own every
 *    buffer they pass in.  There is no CPU compute path: every product,
 *    gather, scatter-add and solver step runs as a CUDA kernel.
 */
#ifndef SPMV_B200_H
#define SPMV_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SPMV_B200_VERSION_MAJOR 0
#define SPMV_B200_VERSION_MINOR 1

/* Largest number of virtual ranks (row-block partitions) per communicator. */
#define SPMV_MAX_PARTS 64

typedef enum spmv_status {
  SPMV_SUCCESS = 0,
  SPMV_ERROR_INVALID_ARGUMENT = 1, /* bad sizes, unsorted ghosts, ...       */
  SPMV_ERROR_CUDA = 2,             /* a CUDA runtime call failed           */
  SPMV_ERROR_OUT_OF_MEMORY = 3,
  SPMV_ERROR_NO_DEVICE = 4,        /* device work on a host-only comm      */
  SPMV_ERROR_BREAKDOWN = 5,        /* CG: p.Ap is zero or not finite       */
  SPMV_ERROR_NOT_SUPPORTED = 6,    /* dtype / option not implemented       */
  SPMV_ERROR_INTERNAL = 7
} spmv_status;

/* Scalar type of a matrix or vector; replaces spmv::mpi_type<T>()
 * (mpi_type.h:11-33). */
typedef enum spmv_dtype {
  SPMV_FLOAT64 = 0,
  SPMV_FLOAT32 = 1,
  SPMV_COMPLEX64 = 2,  /* std::complex<float>: matrices, products, maps */
  SPMV_COMPLEX128 = 3  /* std::complex<double>: matrices, products, maps */
} spmv_dtype;

typedef enum spmv_memory {
  SPMV_MEMORY_HOST = 0,
  SPMV_MEMORY_DEVICE = 1
} spmv_memory;

/* SpMV kernel family used by a matrix (see spmv_matrix_set_kernel). */
typedef enum spmv_kernel {
  SPMV_KERNEL_AUTO = 0,   /* chosen from row-length statistics          */
  SPMV_KERNEL_VECTOR = 1, /* vector CSR: a W-lane group per row          */
  SPMV_KERNEL_MERGE = 2,  /* merge-path, load balanced for skewed rows   */
  SPMV_KERNEL_SELL = 3,   /* sliced ELLPACK (32-row slices), warp per slice */
  SPMV_KERNEL_STAGED = 4  /* sliced ELLPACK streamed through shared memory by
                             bulk asynchronous copies (warp-specialised)  */
} spmv_kernel;

/* Fields of the communication pattern of one rank of an L2GMap.  They are
 * the members of the same names in the reference (L2GMap.h:80-91). */
typedef enum spmv_pattern_field {
  SPMV_PATTERN_NEIGHBOURS = 0,
  SPMV_PATTERN_SEND_COUNT = 1,
  SPMV_PATTERN_RECV_COUNT = 2,
  SPMV_PATTERN_SEND_OFFSET = 3,
  SPMV_PATTERN_RECV_OFFSET = 4,
  SPMV_PATTERN_INDEXBUF = 5
} spmv_pattern_field;

typedef struct spmv_comm_s* spmv_comm;
typedef struct spmv_l2gmap_s* spmv_l2gmap;
typedef struct spmv_matrix_s* spmv_matrix;

/* ------------------------------------------------------------------------ */
/* Errors and version                                                        */
/* ------------------------------------------------------------------------ */

/* Message of the calling thread's last failed call ("" if none). */
const char* spmv_last_error(void);
int spmv_get_version(int* major, int* minor);

/* ------------------------------------------------------------------------ */
/* Virtual communicator.  Replaces the MPI_Comm argument of the reference    */
/* (L2GMap.h:29, Matrix.h:59, cg.h:27).                                      */
/* ------------------------------------------------------------------------ */

/* device >= 0: ranks live on that CUDA device; `stream` is a cudaStream_t to
 * order work on (NULL: the library creates its own non-blocking stream).
 * device == -1: a host-only communicator; maps and matrices can be built and
 * inspected, device work fails with SPMV_ERROR_NO_DEVICE. */
int spmv_comm_create(int device, void* stream, int size, spmv_comm* comm);
int spmv_comm_destroy(spmv_comm comm);
int spmv_comm_size(spmv_comm comm, int* size);
int spmv_comm_device(spmv_comm comm, int* device);
int spmv_comm_stream(spmv_comm comm, void** stream);
int spmv_comm_synchronize(spmv_comm comm);

/* ------------------------------------------------------------------------ */
/* L2GMap (reference: L2GMap.h:14-97, L2GMap.cpp:15-199)                     */
/* ------------------------------------------------------------------------ */

/* Collective construction (L2GMap::L2GMap, L2GMap.cpp:15-122) for all ranks:
 * local_size[size], ghosts[size][num_ghosts[r]] (global indices, sorted
 * ascending, none in the rank's own range).  Errors: "Ghosts must be sorted"
 * (L2GMap.cpp:35), "Ghost index in local range" (L2GMap.cpp:45). */
int spmv_l2gmap_create(spmv_comm comm, const int64_t* local_size,
                       const int64_t* const* ghosts, const int64_t* num_ghosts,
                       spmv_l2gmap* map);
int spmv_l2gmap_destroy(spmv_l2gmap map);
/* L2GMap::local_size, num_ghosts, global_size, global_offset
 * (L2GMap.cpp:187-199). */
int spmv_l2gmap_local_size(spmv_l2gmap map, int rank, int32_t* out);
int spmv_l2gmap_num_ghosts(spmv_l2gmap map, int rank, int32_t* out);
int spmv_l2gmap_global_size(spmv_l2gmap map, int64_t* out);
int spmv_l2gmap_global_offset(spmv_l2gmap map, int rank, int64_t* out);
/* L2GMap::global_to_local (L2GMap.cpp:172-185).  An index neither owned by
 * nor ghosted on `rank` is an error (the reference's behaviour there is
 * undefined). */
int spmv_l2gmap_global_to_local(spmv_l2gmap map, int rank,
                                int64_t global_index, int32_t* out);
/* L2GMap::ghosts (L2GMap.h:75).  *ghosts stays valid while the map lives. */
int spmv_l2gmap_ghosts(spmv_l2gmap map, int rank, const int64_t** ghosts,
                       int32_t* n);
/* One array of the rank's communication pattern (L2GMap.h:80-91), exactly as
 * the reference computes it, including send_offset already shifted by
 * local_size (L2GMap.cpp:120-121).  *data stays valid while the map lives. */
int spmv_l2gmap_pattern(spmv_l2gmap map, int rank, spmv_pattern_field field,
                        const int32_t** data, int32_t* n);
/* L2GMap::update<T> (L2GMap.cpp:126-150): for all ranks at once, copy each
 * owner's values into the ghost slots of the ranks that ghost them.
 * vecs[size], each of length local_size + num_ghosts.  Bit-exact copy. */
int spmv_l2gmap_update(spmv_l2gmap map, spmv_dtype dtype, spmv_memory memory,
                       void* const* vecs);
/* L2GMap::reverse_update<T> (L2GMap.cpp:152-170): add every ghost slot into
 * its owner's entry, in the reference's order (neighbour rank order, then
 * ghost order), so results are bitwise those of the reference loop. */
int spmv_l2gmap_reverse_update(spmv_l2gmap map, spmv_dtype dtype,
                               spmv_memory memory, void* const* vecs);

/* ------------------------------------------------------------------------ */
/* Matrix (reference: Matrix.h:23-81, Matrix.cpp:13-211)                     */
/* ------------------------------------------------------------------------ */

/* Matrix::Matrix (Matrix.cpp:13-22) plus the inspector step mkl_init
 * (Matrix.cpp:34-51): copies in every rank's local CSR block (0-based,
 * int32 row pointers and column indices, columns [0, ncols) with the
 * col_map's ghosts after its owned range).  nrows[size], ncols[size],
 * rowptr[size][nrows[r]+1], colind[size][nnz], values[size][nnz] of `dtype`
 * (float64, float32, complex128 or complex64 - the reference's four
 * instantiations, Matrix.cpp:441-444; complex values interleaved re, im).
 * row_map may be NULL (then rows have no map, and spmv_cg is refused).
 * Complex matrices support mult and transpmult (plain transpose, result of
 * ncols entries as in the generic path, Matrix.cpp:206-211); the solvers,
 * SpMM and the adjoint sampling are real only. */
int spmv_matrix_create_csr(spmv_comm comm, spmv_dtype dtype,
                           spmv_l2gmap col_map, spmv_l2gmap row_map,
                           const int32_t* nrows, const int32_t* ncols,
                           const int32_t* const* rowptr,
                           const int32_t* const* colind,
                           const void* const* values, spmv_matrix* A);
int spmv_matrix_destroy(spmv_matrix A);
/* Matrix::create_matrix (Matrix.cpp:213-438) for every rank: rank r's block
 * has nrows_local[r] owned rows followed by n_row_ghosts[r] ghost rows
 * (global indices row_ghosts[r][i], rows other ranks own), and columns
 * numbered owned first (ncols_local[r]) then col_ghosts[r] (sorted global
 * indices); rowptr[r] has nrows_local[r] + n_row_ghosts[r] + 1 entries.
 * Ghost rows are added into their owners' rows (entries with the same row
 * and column summed in the reference's triplet order: the owner's rows
 * first, then received rows by ascending sender), the owners' ghost columns
 * grow by the columns those rows bring (ascending), and each row ends in
 * ascending column order.  Returns the assembled matrix and its two maps
 * (row map without ghosts); the caller destroys all three.  Ranges are the
 * prefix sums of nrows_local and ncols_local. */
int spmv_matrix_create_assembled(spmv_comm comm, spmv_dtype dtype, const int64_t* nrows_local,
                                 const int64_t* ncols_local, const int32_t* const* rowptr,
                                 const int32_t* const* colind, const void* const* values,
                                 const int64_t* const* row_ghosts, const int64_t* n_row_ghosts,
                                 const int64_t* const* col_ghosts,
                                 const int64_t* n_col_ghosts, spmv_l2gmap* col_map,
                                 spmv_l2gmap* row_map, spmv_matrix* A);
/* Matrix::operator* (Matrix.cpp:158-166, 199-204): y[r] = A[r] x[r] for all
 * ranks in one launch.  x[r] has ncols[r] entries (owned, then ghosts: run
 * spmv_l2gmap_update first, as the reference's callers do), y[r] nrows[r]. */
int spmv_matrix_mult(spmv_matrix A, spmv_memory memory, const void* const* x,
                     void* const* y);
/* Matrix::transpmult (Matrix.cpp:168-176, 206-211): y[r] = A[r]^T x[r];
 * x[r] has nrows[r] entries, y[r] ncols[r] (ghost tail included: follow with
 * spmv_l2gmap_reverse_update, as restrictmain.cpp:60-66 does). */
int spmv_matrix_transpmult(spmv_matrix A, spmv_memory memory,
                           const void* const* x, void* const* y);
int spmv_matrix_dtype(spmv_matrix A, spmv_dtype* dtype);
int spmv_matrix_rows(spmv_matrix A, int rank, int32_t* nrows);
int spmv_matrix_cols(spmv_matrix A, int rank, int32_t* ncols);
int spmv_matrix_nnz(spmv_matrix A, int rank, int64_t* nnz);
/* Matrix::mat() (Matrix.h:51-53): the host copy of rank's CSR block. */
int spmv_matrix_csr(spmv_matrix A, int rank, const int32_t** rowptr,
                    const int32_t** colind, const void** values);
/* Matrix::col_map()/row_map() (Matrix.h:45-48). */
int spmv_matrix_col_map(spmv_matrix A, spmv_l2gmap* map);
int spmv_matrix_row_map(spmv_matrix A, spmv_l2gmap* map);
/* Replace the values of every rank (same sparsity pattern).  values[size]. */
int spmv_matrix_set_values(spmv_matrix A, spmv_memory memory,
                           const void* const* values);
/* Allocation-free product y[r] = A[r] x[r] (no counterpart in the reference).
 *
 * For callers that must not allocate device memory while they run: an
 * application whose device memory is handed out by its own allocator or pool,
 * sized at start-up, cannot have a library call cudaMalloc behind its back (the
 * call fails when the pool already holds the memory, and cudaMalloc/cudaFree
 * can stall the whole device in the middle of a time-critical loop).
 * spmv_matrix_mult's merge-path kernel keeps per-CTA partial row sums in a
 * buffer the library allocates on first use; this entry point runs the same
 * merge-path kernels with those partial sums in a fixed device array that is
 * part of the library (192 KiB, kept on every device that loads the library
 * until the process exits), so a call allocates nothing.
 *  - x and y are device pointers, one per rank, as for spmv_matrix_mult with
 *    SPMV_MEMORY_DEVICE; the work is ordered on the communicator's stream.
 *  - Limit: rows + nonzeros over all ranks of at most 33,554,432 (16384 tiles
 *    of 2048); a larger matrix is rejected with SPMV_ERROR_INVALID_ARGUMENT.
 *  - The first call on a device looks up the array's device address, once per
 *    device; make that first call before any stream capture.  The address is
 *    kept for the life of the process: after cudaDeviceReset (which also ends
 *    every handle of this library on that device) do not call it again.
 *  - All calls share the one array, which keeps what the last call left in it
 *    (each call writes every slot before reading it, so nothing needs
 *    clearing); calls that overlap on the GPU, e.g. from two streams of the
 *    same device, race on it and must not be issued.
 *  - Results equal spmv_matrix_mult's within rounding (FP64: 1e-12 of
 *    (|A||x|) per row); bitwise when that matrix also uses the merge-path
 *    kernel. */
int spmv_matrix_mult_noalloc(spmv_matrix A, const void* const* x,
                             void* const* y);
/* Kernel choice.  width: lanes per row for SPMV_KERNEL_VECTOR (1..32, a
 * power of two), loads in flight per lane for SPMV_KERNEL_SELL (1..16, a
 * power of two), gathers in flight per lane for SPMV_KERNEL_STAGED (4, 5, 7,
 * 8 or 9; 5, 7 and 9 suit stencils whose rows have a multiple of that many
 * entries: 5-, 7- and 27-point);
 * 0 = from statistics; block: threads per CTA (0 = default; the staged
 * product always runs 416-thread CTAs, which get_kernel and the tuner
 * report). */
int spmv_matrix_set_kernel(spmv_matrix A, spmv_kernel kernel, int width,
                           int block);
int spmv_matrix_get_kernel(spmv_matrix A, spmv_kernel* kernel, int* width,
                           int* block);

typedef struct spmv_tune_result {
  spmv_kernel kernel;  /* chosen kernel family                               */
  int width;           /* lanes per row (vector) or loads per lane (SELL)    */
  int block;           /* threads per CTA                                    */
  double us;           /* time of one product with that choice, microseconds */
  int candidates;      /* configurations timed (0: taken from the cache)     */
} spmv_tune_result;

/* Autotuner (no counterpart in the reference; mkl_sparse_optimize,
 * Matrix.cpp:43, is the reference's analysis step): times the product over
 * candidate kernels, widths and block sizes on this matrix, `reps` launches
 * each, and keeps the fastest for mult and for the solvers.  Allocates scratch
 * vectors for the timing.  With the environment variable SPMV_B200_TUNE_CACHE
 * naming a file, results are cached there by matrix statistics. */
int spmv_matrix_autotune(spmv_matrix A, int reps, spmv_tune_result* best);

/* ------------------------------------------------------------------------ */
/* Conjugate gradients (reference: cg.h:27-29, cg.cpp:11-83)                 */
/* ------------------------------------------------------------------------ */

typedef struct spmv_cg_info {
  int iterations;          /* k as returned by spmv::cg                    */
  int status;              /* SPMV_SUCCESS or SPMV_ERROR_BREAKDOWN          */
  double rnorm0;           /* ||b||^2                                       */
  double rnorm;            /* last recursive ||r||^2                        */
} spmv_cg_info;

/* spmv::cg (cg.cpp:11-83): unpreconditioned CG from x0 = 0 on all ranks at
 * once, stopping when ||r||^2/||b||^2 < rtol^2 or after max_its iterations.
 * b[size] (row_map local_size entries each; b_rows[size] gives their lengths
 * for the "b.rows() != A.rows()" check, or NULL to skip it), x[size] out
 * (col_map local_size + num_ghosts entries each; the ghost tail is zero, as
 * in the reference).  FP64 only.  Each iteration runs as one CUDA graph body
 * under a device-side while loop; there is no host round trip per iteration.
 * Differences from the reference: b == 0 returns x = 0 after 0 iterations
 * (the reference divides 0 by 0), and p.Ap == 0 or non-finite stops with
 * SPMV_ERROR_BREAKDOWN (the reference carries NaN to max_its). */
int spmv_cg(spmv_matrix A, spmv_memory memory, const double* const* b,
            const int64_t* b_rows, double* const* x, int max_its, double rtol,
            int* num_its);
/* As spmv_cg, filling *info (may be NULL). */
int spmv_cg_ex(spmv_matrix A, spmv_memory memory, const double* const* b,
               const int64_t* b_rows, double* const* x, int max_its,
               double rtol, spmv_cg_info* info);

/* ------------------------------------------------------------------------ */
/* Mixed-precision CG (no counterpart in the reference; builds on spmv::cg)   */
/* ------------------------------------------------------------------------ */

/* The product a solver of this matrix runs (chosen by timing when the
 * solver's workspace was built): solver 0 = spmv_cg, 1 = the FP32 inner
 * product of spmv_cg_mixed, 2 = its FP64 residual product.  kernel is
 * SPMV_KERNEL_VECTOR (width = lanes per row) or SPMV_KERNEL_SELL (width =
 * loads in flight per lane); index_bits is 32 (global column indices) or 16
 * (offsets from the row); us is the plain product's timed duration.  Fails
 * when that solver has not run on the matrix.  No reference counterpart. */
int spmv_matrix_solver_product(spmv_matrix A, int solver, spmv_kernel* kernel,
                               int* width, int* index_bits, double* us);

/* How spmv_cg runs on this matrix (chosen by timing when its workspace was
 * built): *fused = 0 for a CUDA graph of three kernels per iteration, 1 for
 * one cooperative launch per solve with *ctas_per_sm persistent CTAs per SM
 * and the residual held in shared memory (*r_shared = 1) or global memory,
 * 2 for the same launch in the merged-update form (two grid syncs per
 * iteration instead of three).
 * Fails when spmv_cg has not run on the matrix.  No reference counterpart. */
int spmv_matrix_cg_form(spmv_matrix A, int* fused, int* ctas_per_sm, int* r_shared);

/* The same for spmv_cg_mixed: *fused = 0 for its CUDA graph (three kernels
 * per inner iteration, three more per refinement), 1 for one cooperative
 * launch per solve (the FP32 residual in shared memory when *r_shared = 1).
 * Fails when spmv_cg_mixed has not run on the matrix.  No reference
 * counterpart. */
int spmv_matrix_cg_mixed_form(spmv_matrix A, int* fused, int* ctas_per_sm, int* r_shared);

typedef struct spmv_ir_info {
  int iterations;   /* inner FP32 CG iterations                             */
  int refinements;  /* FP64 true-residual recomputations                    */
  int status;       /* SPMV_SUCCESS or SPMV_ERROR_BREAKDOWN                 */
  int converged;    /* 1 if ||b - A x|| / ||b|| < rtol was confirmed in FP64 */
  double relres;    /* that FP64 relative residual, at the last refinement  */
} spmv_ir_info;

/* Solves A x = b (A FP64, SPD) to ||b - A x|| / ||b|| < rtol, checked in FP64,
 * with FP32 inner CG iterations on an FP32 copy of A (made on first use) and
 * FP64 refinement: FP64 solution, FP64 true residual b - A x, FP64 dot-product
 * accumulation and FP64 alpha/beta.  Arguments as spmv_cg; max_its bounds the
 * inner iterations.  Runs as one CUDA graph launch. */
int spmv_cg_mixed(spmv_matrix A, spmv_memory memory, const double* const* b,
                  const int64_t* b_rows, double* const* x, int max_its,
                  double rtol, spmv_ir_info* info);

/* ------------------------------------------------------------------------ */
/* Several right-hand sides (no counterpart in the reference)                */
/* ------------------------------------------------------------------------ */

/* Y[r] = A[r] X[r] for nrhs (1..32) right-hand sides at once, reading A once:
 * X[r] is ncols[r] x nrhs and Y[r] nrows[r] x nrhs, row-major (the nrhs values
 * of one row contiguous). */
int spmv_matrix_mult_block(spmv_matrix A, int nrhs, spmv_memory memory,
                           const void* const* x, void* const* y);
/* Block CG: nrhs (1..32) independent CG solves (the recurrence of spmv::cg,
 * cg.cpp:11-83, per column, each with its own stopping test) sharing one
 * product per iteration.  b[r] is local_size x nrhs, x[r] (local_size +
 * num_ghosts) x nrhs (ghost rows zero), row-major; info[nrhs] may be NULL. */
int spmv_cg_block(spmv_matrix A, int nrhs, spmv_memory memory,
                  const double* const* b, double* const* x, int max_its,
                  double rtol, spmv_cg_info* info);

/* ------------------------------------------------------------------------ */
/* Batched solves (no counterpart in the reference; builds on spmv::cg)      */
/* ------------------------------------------------------------------------ */

typedef struct spmv_batch_s* spmv_batch;

typedef struct spmv_batch_info {
  int iterations;   /* inner CG iterations of this right-hand side           */
  int refinements;  /* FP64 true-residual recomputations                     */
  int status;       /* SPMV_SUCCESS or SPMV_ERROR_BREAKDOWN                  */
  int converged;    /* 1 if ||b - A x|| / ||b|| < rtol was confirmed in FP64  */
  double relres;    /* that FP64 relative residual                           */
} spmv_batch_info;

/* Inner precision of a batched solve. */
typedef enum spmv_batch_precision {
  SPMV_BATCH_MIXED = 0,  /* FP32 inner CG, FP64 refinement (reliable updates)  */
  SPMV_BATCH_FP64 = 1    /* FP64 CG; the stopping test is confirmed by one
                            FP64 residual                                       */
} spmv_batch_precision;

/* Launch shape of the batched kernel (0 in a field of spmv_batch_set_config:
 * keep the current value). */
typedef struct spmv_batch_config {
  int ctas_per_sm;   /* CTAs of 512 threads per SM: 1 or 2                     */
  int tile_rows;     /* rows a warp takes at a time: 128, 256 or 512           */
  int rhs_lanes;     /* lanes per block row in the block products: 32 (one
                        right-hand side per lane) or 16 (two per lane)         */
  int window;        /* 2: the products stage the band of the gathered vector
                        a CTA reads in shared memory; 1: they gather through
                        L1 (0 in spmv_batch_set_config: keep)                 */
  double us;         /* autotune: time of the timed solve, microseconds        */
  int candidates;    /* autotune: configurations timed (0: from the cache)     */
} spmv_batch_config;

/* nsys independent SPD systems of sizes n[i] (square CSR blocks with
 * symmetric patterns, FP64 values) for spmv_batch_solve (no counterpart in
 * the reference; each solve is spmv::cg's recurrence, cg.cpp:50-80, on
 * Matrix::operator*, Matrix.cpp:199-204).  Copies in.  At creation each
 * system is renumbered once (reverse Cuthill-McKee, rows sorted by length in
 * windows of 1024) and stored as SELL-32 slices with FP32 and FP64 values
 * and 16-bit column offsets when every offset fits (else 32-bit columns);
 * the solves map b in and x out.  At most 8191 systems. */
int spmv_batch_create(spmv_comm comm, int nsys, const int32_t* n,
                      const int32_t* const* rowptr,
                      const int32_t* const* colind,
                      const double* const* values, spmv_batch* batch);
int spmv_batch_destroy(spmv_batch batch);
/* System `system` also takes a block of nrhs (1..32) right-hand sides in
 * spmv_batch_solve_ex, solved in the same launch with one product per
 * iteration for all its columns (its matrix read once per iteration). */
int spmv_batch_set_block(spmv_batch batch, int system, int nrhs);
/* Launch shape of the solves of one precision; see spmv_batch_config.
 * spmv_batch_autotune times the candidates (ctas_per_sm x tile_rows x
 * rhs_lanes) on short solves of this batch in that precision and keeps the
 * fastest; with SPMV_B200_TUNE_CACHE naming a file the choice is cached by
 * batch statistics and precision. */
int spmv_batch_set_config(spmv_batch batch, spmv_batch_precision precision,
                          const spmv_batch_config* config);
int spmv_batch_get_config(spmv_batch batch, spmv_batch_precision precision,
                          spmv_batch_config* config);
int spmv_batch_autotune(spmv_batch batch, spmv_batch_precision precision,
                        spmv_batch_config* best);
/* Storage statistics: rows, nonzeros and stored SELL entries (padding
 * included) over all systems, and the bits per stored column index. */
int spmv_batch_stats(spmv_batch batch, int64_t* rows, int64_t* nnz,
                     int64_t* stored, int* index_bits);
/* Solves every system A_i x_i = b_i to ||b_i - A_i x_i|| / ||b_i|| < rtol
 * (confirmed in FP64) and, when the batch has a block and bblock/xblock are
 * not NULL, A_s X = B for the block's system s (bblock and xblock n_s x nrhs,
 * row-major), all in one cooperative launch: every CG iteration of every
 * system and block column runs in lockstep, each recurrence with its own
 * alpha, beta and stopping test; a system stops iterating when it has
 * converged.  precision: SPMV_BATCH_MIXED (FP32 inner iterations, FP64
 * refinement, as spmv_cg_mixed) or SPMV_BATCH_FP64.  b[nsys], x[nsys];
 * info[nsys] and block_info[nrhs] may be NULL.  max_its bounds each
 * recurrence's inner iterations. */
int spmv_batch_solve_ex(spmv_batch batch, spmv_memory memory,
                        spmv_batch_precision precision,
                        const double* const* b, double* const* x,
                        const double* bblock, double* xblock, int max_its,
                        double rtol, spmv_batch_info* info,
                        spmv_batch_info* block_info);
/* spmv_batch_solve_ex with SPMV_BATCH_MIXED and no block. */
int spmv_batch_solve(spmv_batch batch, spmv_memory memory,
                     const double* const* b, double* const* x, int max_its,
                     double rtol, spmv_batch_info* info);

/* ------------------------------------------------------------------------ */
/* Adjoint of x = A^{-1} b (no counterpart in the reference)                 */
/* ------------------------------------------------------------------------ */

/* out[r][k] = scale * lambda[r][row(k)] * x[r][col(k)] for every stored entry
 * k of rank r's block, in the block's entry order.  With lambda the adjoint
 * solution (A^T lambda = dL/dx; spmv_cg on A for symmetric A) and scale = -1
 * this is dL/dA on A's sparsity pattern; dL/db is lambda itself.  lambda[r]
 * has nrows[r] entries, x[r] ncols[r] (owned then ghosts: update it first),
 * out[r] nnz[r]; all of the matrix dtype. */
int spmv_matrix_sample_outer(spmv_matrix A, spmv_memory memory, double scale,
                             const void* const* lambda, const void* const* x,
                             void* const* out);

/* ------------------------------------------------------------------------ */
/* PETSc binary files (reference: read_petsc.h:18-32, read_petsc.cpp)       */
/* ------------------------------------------------------------------------ */

/* owner_ranges (read_petsc.cpp:13-30, CreateA.cpp:12-29): ranges[size + 1]
 * splitting n items over size ranks, the first n % size ranks one larger. */
int spmv_owner_ranges(int size, int64_t n, int64_t* ranges);

/* spmv::read_petsc_binary (read_petsc.cpp:32-191) for every rank of comm at
 * once: a PETSc binary matrix file (32-bit indices, big endian) split by
 * owner_ranges over rows and columns.  Rank r's columns are numbered owned
 * first, then its ghosts in ascending global order; entries within a row are
 * in ascending local column order.  Returns the FP64 matrix and its two maps
 * (row map without ghosts); the caller destroys all three.  Errors: "Could
 * not open file", "Bad signature in PETSc Matrix file", and (where the
 * reference reads out of range) truncated files, row lengths that do not sum
 * to nnz and column indices outside [0, ncols). */
int spmv_petsc_read_matrix(spmv_comm comm, const char* filename, spmv_l2gmap* col_map,
                           spmv_l2gmap* row_map, spmv_matrix* A);

/* Length of a PETSc binary vector file ("Bad signature in PETSc Vector
 * file" if it is not one). */
int spmv_petsc_vector_size(const char* filename, int64_t* n);

/* spmv::read_petsc_binary_vector (read_petsc.cpp:193-260) for every rank:
 * values[r] (host) receives the rank's owner_ranges(size, n) block. */
int spmv_petsc_read_vector(spmv_comm comm, const char* filename, double* const* values);

#ifdef __cplusplus
}
#endif

#endif /* SPMV_B200_H */
