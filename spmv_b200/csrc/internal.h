// Internal declarations of libspmv_b200: handle structs, error plumbing and
// the kernel-launch interfaces shared between the translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "spmv_b200.h"

namespace spmvb {

// ---------------------------------------------------------------------------
// Errors.  Every entry point converts an spmvb::Error (or std::exception) into
// a status code and stores the message for spmv_last_error().
// ---------------------------------------------------------------------------
struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

[[noreturn]] inline void fail(int status, const std::string& msg) {
  throw Error(status, msg);
}
inline void require(bool ok, const std::string& msg) {
  if (!ok) fail(SPMV_ERROR_INVALID_ARGUMENT, msg);
}

void set_last_error(const std::string& msg);
// Debug log (stderr) when SPMV_B200_DEBUG is set in the environment.
void debug_log(const std::string& msg);
// For calls whose failure must not abort the caller (frees, destroys): a
// failure is logged and the runtime's pending error is cleared, so it cannot
// be reported later by an unrelated call.
void soft_check(cudaError_t e, const char* what);

#define SPMVB_CUDA(call)                                                     \
  do {                                                                       \
    cudaError_t e_ = (call);                                                 \
    if (e_ != cudaSuccess)                                                   \
      ::spmvb::fail(e_ == cudaErrorMemoryAllocation ? SPMV_ERROR_OUT_OF_MEMORY \
                                                    : SPMV_ERROR_CUDA,       \
                    std::string(#call) + ": " + cudaGetErrorString(e_));     \
  } while (0)

// Runs `body` and turns exceptions into a status code.
template <class F>
int guard(F&& body) {
  try {
    body();
    return SPMV_SUCCESS;
  } catch (const Error& e) {
    set_last_error(e.what());
    return e.status;
  } catch (const std::bad_alloc&) {
    set_last_error("spmv: host allocation failed");
    return SPMV_ERROR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return SPMV_ERROR_INTERNAL;
  }
}

inline size_t dtype_size(spmv_dtype t) {
  switch (t) {
    case SPMV_FLOAT64: return 8;
    case SPMV_FLOAT32: return 4;
    case SPMV_COMPLEX64: return 8;
    case SPMV_COMPLEX128: return 16;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: unknown dtype");
}

// ---------------------------------------------------------------------------
// Device buffer (RAII, cudaMalloc/cudaFree on the owning device).
// ---------------------------------------------------------------------------
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  DevBuf(DevBuf&& o) noexcept : ptr(o.ptr), bytes(o.bytes) {
    o.ptr = nullptr;
    o.bytes = 0;
  }
  DevBuf& operator=(DevBuf&& o) noexcept {
    if (this != &o) {
      release();
      ptr = o.ptr;
      bytes = o.bytes;
      o.ptr = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevBuf() { release(); }
  void release() {
    if (ptr) soft_check(cudaFree(ptr), "cudaFree");
    ptr = nullptr;
    bytes = 0;
  }
  // Grows (never shrinks) to at least `n` bytes; contents are not kept.
  void reserve(size_t n) {
    if (n <= bytes) return;
    release();
    if (n == 0) return;
    SPMVB_CUDA(cudaMalloc(&ptr, n));
    bytes = n;
  }
  template <class T>
  T* as() const { return static_cast<T*>(ptr); }
};

// Selects the communicator's device for the lifetime of the guard.
struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev);
  ~DeviceGuard();
};

}  // namespace spmvb

// ---------------------------------------------------------------------------
// Handles
// ---------------------------------------------------------------------------
struct spmv_comm_s {
  int device = -1;          // -1: host-only
  int size = 0;             // number of virtual ranks
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  int num_sms = 0;
  // References: the caller's handle plus one per live map or matrix, so the
  // communicator outlives everything created on it, whatever the order of
  // the destroy calls.
  int refs = 1;
  // Staging buffers for SPMV_MEMORY_HOST calls.
  spmvb::DevBuf stage_in, stage_out;
  // Device word a staged product sets when one of its bounded waits timed
  // out (checked and cleared by spmv_comm_synchronize).
  spmvb::DevBuf wait_err;
  int* wait_flag() {
    if (!wait_err.ptr) {
      wait_err.reserve(sizeof(int));
      SPMVB_CUDA(cudaMemset(wait_err.ptr, 0, sizeof(int)));
    }
    return wait_err.as<int>();
  }
  void require_device() const {
    if (device < 0)
      spmvb::fail(SPMV_ERROR_NO_DEVICE,
                  "spmv: communicator has no CUDA device");
  }
};

namespace spmvb {

// Launch with programmatic stream serialization (see pdl_wait in
// kernels.cuh): the kernel must call pdl_wait() before touching global memory.
inline void launch_pdl(const void* fn, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                       void** args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  SPMVB_CUDA(cudaLaunchKernelExC(&cfg, fn, args));
}

// Communication pattern of one rank, as L2GMap.cpp:15-122 computes it.
struct RankMap {
  int64_t local_size = 0;
  std::vector<int64_t> ghosts;
  std::vector<int32_t> neighbours, send_count, recv_count, send_offset,
      recv_offset, indexbuf;
};

// Device tables derived from the pattern.
struct HaloTables {
  bool built = false;
  int64_t n_update = 0;   // ghost slots over all ranks
  int64_t n_targets = 0;  // distinct (rank, owned index) reverse targets
  int64_t n_contrib = 0;  // reverse contributions
  DevBuf upd_ranks;       // int32: (dst_rank << 16) | src_rank
  DevBuf upd_dst;         // int32 dst index in dst rank's vector
  DevBuf upd_src;         // int32 src index in src rank's vector
  DevBuf rev_tgt_rank;    // int32
  DevBuf rev_tgt_idx;     // int32
  DevBuf rev_ptr;         // int32 [n_targets+1]
  DevBuf rev_src_rank;    // int32 [n_contrib]
  DevBuf rev_src_idx;     // int32 [n_contrib]
};

}  // namespace spmvb

struct spmv_l2gmap_s {
  spmv_comm comm = nullptr;
  int refs = 1;  // caller's handle plus one per matrix using the map
  std::vector<int64_t> ranges;           // [size+1]
  std::vector<spmvb::RankMap> rank;      // [size]
  spmvb::HaloTables halo;
  int64_t vec_len(int r) const {
    return rank[r].local_size + (int64_t)rank[r].ghosts.size();
  }
};

namespace spmvb {

// One rank's block of a concatenated CSR on the device.
struct DevPart {
  int32_t nrows = 0, ncols = 0;
  int64_t nnz = 0;
  int64_t rp_off = 0;   // offset of this rank's rowptr in the concatenation
  int64_t nz_off = 0;   // offset of this rank's entries (aligned to 4)
  // SELL-32 layout of the same block (when built).
  int64_t sl_off = 0;   // offset of this rank's slice offsets
  int64_t sz_off = 0;   // offset of this rank's SELL entries
  int64_t snnz = 0;     // SELL entries including padding
};

// A device CSR (all ranks concatenated) plus the derived column arrays.
struct DevCsr {
  std::vector<DevPart> parts;
  int64_t rp_total = 0, nz_total = 0;   // allocated lengths (with padding)
  DevBuf rowptr;        // int32
  DevBuf cols;          // int32: rank-local column indices
  DevBuf vals;          // scalar of the matrix dtype
  DevBuf cols_global;   // int32: global column indices (fused-halo layout)
  DevBuf vals32;        // float copy of FP64 values (mixed precision)
  DevBuf merge_carry;   // per-CTA carries of the merge-path product
  // SELL-32 copy (sliced ELLPACK, padding columns are -1), built when the
  // kernel choice is SELL: slice offsets (int32, per rank relative to the
  // rank's first SELL entry, nslices+1 each), columns, values, and the
  // fused-halo / FP32 variants.
  bool sell_built = false;
  int64_t sl_total = 0, sz_total = 0;
  DevBuf sell_off, sell_cols, sell_vals, sell_cols_global, sell_vals32;
  // 16-bit column offsets for the fused-halo layout (d16): entry j of
  // global row g has column g + d16[j], built with cols_global when every
  // offset lies in [-32767, 32767]; the SELL copy pads with -32768.
  bool d16 = false;
  DevBuf d16_global, sell_d16_global;
  // Host copy of the SELL slice offsets (all ranks, as in sell_off) and the
  // staged-traversal tile tables, one per bytes per entry (6, 8, 10, 12):
  // ok is false when some slice is too wide for one stage.
  std::vector<int32_t> h_sell_off;
  struct StagedTable {
    bool built = false, ok = false;
    int ntiles = 0;
    DevBuf desc;
    // Host copy of each tile's rank, first slice and slice count.
    struct Rows {
      int32_t rank, s0, nslices;
    };
    std::vector<Rows> rows;
  } staged[4];
  // Row statistics (over all ranks).
  double mean_row = 0;
  int64_t max_row = 0;
  int64_t sell_padded = 0;   // SELL-32 entries (with padding) over all ranks
};

}  // namespace spmvb

struct CgWorkspace;  // cg.cu
struct IrWorkspace;  // ir.cu

struct spmv_matrix_s {
  spmv_comm comm = nullptr;
  spmv_dtype dtype = SPMV_FLOAT64;
  spmv_l2gmap col_map = nullptr, row_map = nullptr;
  // Host copies (Matrix::mat()).
  std::vector<std::vector<int32_t>> h_rowptr, h_colind;
  std::vector<std::vector<unsigned char>> h_vals;
  std::vector<int32_t> nrows, ncols;
  // Device plans.
  spmvb::DevCsr fwd;            // A
  spmvb::DevCsr trn;            // A^T, built on first transpmult
  bool trn_built = false;
  std::vector<std::vector<int32_t>> h_trn_rowptr;  // A^T's row pointers (SELL build)
  // Kernel choice.
  spmv_kernel kernel = SPMV_KERNEL_AUTO;
  int width = 0, block = 0;
  // Set by spmv_matrix_set_kernel with an explicit kernel: the solvers'
  // products then use that kind (and width) too.  The autotuner's choice is
  // for mult; the solvers time their own products.
  bool kernel_set = false;
  std::unique_ptr<CgWorkspace, void (*)(CgWorkspace*)> cg{nullptr, nullptr};
  std::unique_ptr<IrWorkspace, void (*)(IrWorkspace*)> ir{nullptr, nullptr};
};

namespace spmvb {

// ---------------------------------------------------------------------------
// Kernel-launch interfaces (implemented in the .cu files)
// ---------------------------------------------------------------------------
struct SpmvLaunch {
  const DevCsr* csr;
  const int32_t* cols;                 // csr->cols or csr->cols_global
  spmv_dtype dtype;
  const void* const* x;                // [nparts] device pointers
  void* const* y;                      // [nparts]
  spmv_kernel kernel;
  int width, block;
  int num_sms;
  DevBuf* carry;                       // merge-path scratch (per matrix)
  int* err = nullptr;                  // staged product: timed-out wait flag
};
void launch_spmv(const SpmvLaunch& L, cudaStream_t stream);
void launch_merge(const SpmvLaunch& L, cudaStream_t stream, DevBuf& carry);
// Kernel family for a matrix: the caller's choice, or from row statistics:
// merge-path when the longest row is far above the mean, SELL-32 when its
// padding is small (allow_sell: the SELL copy can exist for this CSR), else
// vector CSR.  A SELL request where SELL cannot be used gives vector CSR.
spmv_kernel pick_kernel(spmv_kernel requested, const DevCsr& C, bool allow_sell = true);
// Lanes per row picked from the mean row length (vector kernel).
int auto_width(double mean_row, spmv_dtype dtype);
int max_blocks_for(int num_sms, int BS);
// SELL-32 layout (sell.cu): built on the device from the device CSR.
int64_t sell_padded_size(const std::vector<int32_t>& rowptr, int32_t nrows,
                         std::vector<int32_t>* soff);
void build_sell(spmv_matrix A, DevCsr& C, cudaStream_t stream);
// After new values: re-scatter them into the SELL copy (same pattern).
void refresh_sell_values(spmv_matrix A);
void launch_sell(const SpmvLaunch& L, const int32_t* sell_cols, cudaStream_t stream);
// SELL copies of the fused-halo columns and of the FP32 values.
void build_sell_global(spmv_matrix A);
void build_sell_vals32(spmv_matrix A);
// SELL launch table (the PartArg's rowptr field carries the slice offsets).
struct SpmvArgs;
// Plain products over a prepared launch table (vector CSR / SELL).  d16:
// the table's cols are 16-bit offsets (see use_d16); keep: the solvers' L2
// policies (vectors kept, matrix streamed).  Either needs BS = 256.
void launch_vector_args(const SpmvArgs& a, spmv_dtype dtype, int W, int BS,
                        cudaStream_t s, bool d16 = false);
void launch_sell_args(const SpmvArgs& a, spmv_dtype dtype, int U, int BS,
                      cudaStream_t s, bool d16 = false, bool keep = false);
int fill_sell_args(SpmvArgs& a, const DevCsr& C, const int32_t* cols,
                   const void* vals, size_t es, const void* const* x,
                   void* const* y, const void* const* xown, int BS, int max_blocks);
// Points a fused-halo launch table (vector CSR when !sell, else SELL) at the
// 16-bit offsets; the kernels reinterpret the cols field.
void use_d16(SpmvArgs& a, const DevCsr& C, bool sell);
// Whether the solvers may use 16-bit offsets (SPMV_B200_D16=0 turns them off).
bool d16_enabled();
// The solvers' product over the fused-halo layout: vector CSR (w lanes per
// row) or SELL-32 (w loads in flight per lane), with 32-bit columns or
// 16-bit offsets.
enum class ProductKind : int {
  Vector = 0,  // vector CSR, w lanes per row
  Sell = 1,    // SELL-32 from registers, w loads in flight per lane
  Staged = 2,  // SELL-32 staged in shared memory by bulk copies, w gathers per lane
};
// Threads per CTA of the staged product (12 consumer warps and a producer
// warp; a block size given with SPMV_KERNEL_STAGED is not used).
constexpr int kStagedThreads = 416;
// Gathers in flight per lane of the staged product: 4, 8, or a stencil's
// exact row width 5 or 7 (one unmasked chunk per slice).
inline int staged_width(int w) {
  return w == 9 ? 9 : w >= 8 ? 8 : (w == 7 || w == 5) ? w : 4;
}
// The staged width that divides a stencil's longest row exactly (9, 7 or 5,
// so its full slices take the unmasked path), or 0.
inline int exact_staged_width(int64_t max_row) {
  for (int u : {9, 7, 5})
    if (max_row > 0 && max_row % u == 0 && max_row <= 4 * u) return u;
  return 0;
}
struct SolverProduct {
  ProductKind kind = ProductKind::Vector;
  int w = 0;
  bool d16 = false;
  float us = 0.f;
  bool sell_layout() const { return kind != ProductKind::Vector; }
};
// Launches the solver's own product kernel for a candidate over a prepared
// launch table (the kernel's graph-only side effects compiled out).
using ProductLauncher =
    std::function<void(const SolverProduct&, const SpmvArgs&, cudaStream_t)>;
// Times `launch` for each candidate (x: global input, y: global output, of
// dtype dt; xown_rows: each rank's xown = its rows of x) and returns the
// fastest.  A kernel set on the matrix restricts the candidates to that kind
// and width.
SolverProduct choose_solver_product(spmv_matrix A, spmv_dtype dt, const void* x, void* y,
                                    bool xown_rows, const ProductLauncher& launch);
// Fused (cooperative, persistent) solver kernels: each CTA owns a contiguous
// run of a staged tile table and so a contiguous range of global rows.
struct FusedCta {
  int32_t t0, t1;  // tiles [t0, t1)
  int32_t g0, g1;  // global rows [g0, g1)
};
// Splits the tiles of `t` into `grid` contiguous runs of about n / grid rows
// each; returns the longest run's row count.
int64_t fused_ctas(spmv_matrix A, const DevCsr::StagedTable& t, int grid,
                   std::vector<FusedCta>& out);
struct FusedPlan {
  const void* fn = nullptr;
  int grid = 0, block = 0, smem = 0;
  int cps = 0;      // CTAs per SM
  bool rs = false;  // a vector of the CTA's rows kept in shared memory
  bool merged = false;  // spmv_cg's merged-update form (two grid syncs per iteration)
  std::vector<FusedCta> ctas;
};
// A plan for kernel `fn` of `block` threads at `cps` CTAs per SM over the
// tiles of `t`: `stage_smem` bytes of stage buffers plus `rs_bytes` per row
// of the longest run in shared memory; false when it does not fit.
bool fused_plan(spmv_matrix A, const DevCsr::StagedTable& t, const void* fn, int block,
                int cps, int64_t stage_smem, int rs_bytes, FusedPlan& plan);
// Bound of each grid wait of a fused solve: 2 s, or SPMV_B200_WAIT_LIMIT_NS.
unsigned long long fused_wait_ns();
// The products chosen by the built solver workspaces (fails if none).
SolverProduct cg_product(spmv_matrix A);
// How the built CG workspace runs a solve (fails if none).
struct CgForm {
  bool fused = false;
  int cps = 0;
  bool rs = false;
  bool merged = false;  // two grid syncs per iteration (spmv_cg's fused form only)
};
CgForm cg_form(spmv_matrix A);
CgForm ir_form(spmv_matrix A);  // spmv_cg_mixed's
SolverProduct ir_product(spmv_matrix A, bool fp32);
// Builds the SELL copies the solvers may time (when SELL is applicable).
void prepare_solver_layouts(spmv_matrix A, bool fp32);
// The staged tile table of the forward SELL layout for `entry_bytes` bytes per
// entry (value + index) and `max_entries` entries per tile (built once).
const DevCsr::StagedTable& staged_table(DevCsr& C, int entry_bytes, int max_entries);
// Grid (persistent: at most the resident CTAs) and dynamic shared memory of
// a staged launch of `fn` over `ntiles` tiles; sets the function's shared
// memory limit.
struct StagedShape {
  int grid = 0, smem = 0;
};
StagedShape staged_shape(const void* fn, int entry_bytes, int ntiles, int num_sms);
// Plain staged product over the forward SELL layout (falls back to SELL-32
// from registers when a slice is too wide for a stage).
void launch_staged(const SpmvLaunch& L, cudaStream_t stream);

void build_halo_tables(spmv_l2gmap map);
void launch_update(spmv_l2gmap map, spmv_dtype dtype, void* const* vecs,
                   cudaStream_t stream);
void launch_reverse_update(spmv_l2gmap map, spmv_dtype dtype,
                           void* const* vecs, cudaStream_t stream);

// Build the L2GMap pattern on the host (all ranks).
void build_pattern(spmv_l2gmap map, const int64_t* local_size,
                   const int64_t* const* ghosts, const int64_t* num_ghosts);

// Drop one reference, freeing the object with the last one.
void release_comm(spmv_comm comm);
void release_map(spmv_l2gmap map);

void upload_csr(spmv_matrix A);
void build_transpose(spmv_matrix A);
void build_global_cols(spmv_matrix A);

// CG in the fused-halo (global) layout: cg_rhs/cg_solution are the device
// vectors of length global_size that cg_run reads b from and leaves x in.
double* cg_rhs(spmv_matrix A);
double* cg_solution(spmv_matrix A);
void cg_run(spmv_matrix A, int max_its, double rtol, spmv_cg_info* info);
void destroy_cg_workspace(CgWorkspace* w);

// Mixed-precision CG (ir.cu): same layout as cg_*; the FP32 copy of the
// values is made on first use.
void ensure_vals32(spmv_matrix A);
double* ir_rhs(spmv_matrix A);
double* ir_solution(spmv_matrix A);
void ir_run(spmv_matrix A, int max_its, double rtol, spmv_ir_info* info);
void destroy_ir_workspace(IrWorkspace* w);

// Solver argument checks and global-layout copies (api.cpp).
void check_solve_args(spmv_matrix A, spmv_memory memory, const double* const* b,
                      const int64_t* b_rows, double* const* x);
void copy_rhs_in(spmv_matrix A, spmv_memory memory, const double* const* b, double* db);
void copy_solution_out(spmv_matrix A, spmv_memory memory, const double* dx,
                       double* const* x);

// Multi-right-hand-side product and block CG (block.cu); blocks are row-major
// with leading dimension k.
void launch_spmm(spmv_matrix A, int k, const void* const* x, void* const* y,
                 cudaStream_t stream);
void block_cg(spmv_matrix A, int k, const double* d_b, double* d_x, int max_its,
              double rtol, spmv_cg_info* info);



// out[r][k] = scale * lambda[r][row(k)] * x[r][col(k)] (adjoint.cu).
void launch_sample_outer(spmv_matrix A, double scale, const void* const* lambda,
                         const void* const* x, void* const* out,
                         cudaStream_t stream);

}  // namespace spmvb
