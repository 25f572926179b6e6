// CSR sparse matrix-vector product for sm_100a (Matrix::operator* and
// transpmult of the reference, Matrix.cpp:158-211).
//
// Vector-CSR kernel: a group of W lanes (W = 1..32) computes one row.  Each
// lane walks the row in 16-byte steps (double2/int2 or float4/int4 loads of
// values and column indices), starting from the row start rounded down to the
// vector width; entries outside [start, end) are masked, never multiplied.
// The group reduces with shuffles.  All ranks of a communicator run in one
// launch: the CTA index selects the rank through a table in kernel
// parameters, and each CTA strides over the rank's row tiles (BS/W rows per
// tile), so the grid is sized to the GPU rather than to the matrix.  W follows
// the mean row length so that one pass of 16-byte loads covers a typical row.
#include <algorithm>
#include <cstdlib>
#include <string>
#include <cmath>

#include "internal.h"
#include "spmv_kernel.cuh"
#include "sell_staged.cuh"

namespace spmvb {

int auto_width(double mean_row, spmv_dtype dtype) {
  // Entries per 16-byte load.
  const int N = dtype == SPMV_FLOAT32 ? 4 : (dtype == SPMV_COMPLEX128 ? 1 : 2);
  // Slots one pass must cover: the row plus up to N-1 entries of the
  // alignment head.
  const double slots = mean_row + (N - 1);
  int w = 1;
  while (w < 32 && w * N < slots) w <<= 1;
  return w;
}

int fill_spmv_args(SpmvArgs& a, const DevCsr& csr, const int32_t* cols,
                   size_t es, const void* const* x, void* const* y,
                   const void* const* xown, int rows_per_tile,
                   int max_blocks) {
  a.nparts = int(csr.parts.size());
  int64_t tiles_total = 0;
  for (const DevPart& D : csr.parts)
    tiles_total += (int64_t(D.nrows) + rows_per_tile - 1) / rows_per_tile;
  int blocks = 0;
  int64_t row0 = 0;
  for (int p = 0; p < a.nparts; ++p) {
    const DevPart& D = csr.parts[p];
    PartArg& P = a.part[p];
    P.row0 = int32_t(row0);
    row0 += D.nrows;
    P.rowptr = csr.rowptr.as<int32_t>() + D.rp_off;
    P.cols = cols + D.nz_off;
    P.vals = static_cast<const char*>(csr.vals.ptr) + D.nz_off * es;
    P.x = x[p];
    P.y = y[p];
    P.xown = xown ? xown[p] : nullptr;
    P.nrows = D.nrows;
    P.block_begin = blocks;
    const int64_t tiles = (int64_t(D.nrows) + rows_per_tile - 1) / rows_per_tile;
    int64_t nb = tiles;
    if (tiles_total > max_blocks)
      nb = std::max<int64_t>(tiles > 0 ? 1 : 0,
                             (tiles * max_blocks + tiles_total - 1) / tiles_total);
    P.ntiles = int32_t(tiles);
    P.nblocks = int32_t(nb);
    blocks += int(nb);
  }
  a.nblocks = blocks;
  return blocks;
}

namespace {

template <typename T, int BS, bool D16 = false>
void launch_vector(const SpmvArgs& a, int W, cudaStream_t s) {
  const dim3 grid(a.nblocks), block(BS);
  switch (W) {
    case 1: spmv_vector_kernel<T, 1, BS, D16><<<grid, block, 0, s>>>(a); break;
    case 2: spmv_vector_kernel<T, 2, BS, D16><<<grid, block, 0, s>>>(a); break;
    case 4: spmv_vector_kernel<T, 4, BS, D16><<<grid, block, 0, s>>>(a); break;
    case 8: spmv_vector_kernel<T, 8, BS, D16><<<grid, block, 0, s>>>(a); break;
    case 16: spmv_vector_kernel<T, 16, BS, D16><<<grid, block, 0, s>>>(a); break;
    case 32: spmv_vector_kernel<T, 32, BS, D16><<<grid, block, 0, s>>>(a); break;
    default: fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: width must be 1..32, a power of two");
  }
}

template <typename T>
void launch_vector_bs(const SpmvArgs& a, int W, int BS, cudaStream_t s) {
  switch (BS) {
    case 128: launch_vector<T, 128>(a, W, s); break;
    case 256: launch_vector<T, 256>(a, W, s); break;
    case 512: launch_vector<T, 512>(a, W, s); break;
    default: fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: block must be 128, 256 or 512");
  }
}

}  // namespace

void launch_vector_args(const SpmvArgs& a, spmv_dtype dtype, int W, int BS,
                        cudaStream_t s, bool d16) {
  if (a.nblocks == 0) return;
  if (d16) {
    require(BS == 256, "spmv: 16-bit offset products run 256 threads per CTA");
    if (dtype == SPMV_FLOAT64)
      launch_vector<double, 256, true>(a, W, s);
    else
      launch_vector<float, 256, true>(a, W, s);
  } else if (dtype == SPMV_FLOAT64)
    launch_vector_bs<double>(a, W, BS, s);
  else
    launch_vector_bs<float>(a, W, BS, s);
  SPMVB_CUDA(cudaGetLastError());
}

void prepare_solver_layouts(spmv_matrix A, bool fp32) {
  build_global_cols(A);
  if (fp32) ensure_vals32(A);
  const bool sell_ok = pick_kernel(SPMV_KERNEL_AUTO, A->fwd) == SPMV_KERNEL_SELL;
  const bool want = A->kernel_set
                        ? (A->kernel == SPMV_KERNEL_SELL || A->kernel == SPMV_KERNEL_STAGED)
                        : sell_ok;
  if (want) {
    build_sell_global(A);
    if (fp32) build_sell_vals32(A);
  }
}

SolverProduct choose_solver_product(spmv_matrix A, spmv_dtype dt, const void* x, void* y,
                                    bool xown_rows, const ProductLauncher& launch) {
  const DevCsr& C = A->fwd;
  spmv_comm comm = A->comm;
  const int P = comm->size;
  const bool f32 = dt == SPMV_FLOAT32;
  const size_t es = f32 ? sizeof(float) : sizeof(double);
  const void* sell_vals = f32 ? C.sell_vals32.ptr : C.sell_vals.ptr;
  const bool have_sell = C.sell_cols_global.ptr != nullptr && sell_vals != nullptr;

  std::vector<SolverProduct> cands;
  const bool only = A->kernel_set;
  const spmv_kernel k = A->kernel;
  const bool want_vec = !only || !have_sell || (k != SPMV_KERNEL_SELL && k != SPMV_KERNEL_STAGED);
  const bool want_sell = have_sell && (!only || k == SPMV_KERNEL_SELL);
  const bool want_staged = have_sell && (!only || k == SPMV_KERNEL_STAGED);
  std::vector<bool> d16s{false};
  if (C.d16) d16s.push_back(true);
  for (bool d : d16s) {
    if (want_vec) {
      std::vector<int> ws;
      if (only && k == SPMV_KERNEL_VECTOR && A->width > 0) {
        ws.push_back(A->width);
      } else {
        const int aw = auto_width(C.mean_row, dt);
        for (int w : {aw / 2, aw, aw * 2})
          if (w >= 1 && w <= 32 && std::find(ws.begin(), ws.end(), w) == ws.end())
            ws.push_back(w);
      }
      for (int w : ws) cands.push_back({ProductKind::Vector, w, d, 0.f});
    }
    if (want_sell) {
      if (only && A->width > 0)
        cands.push_back({ProductKind::Sell, std::min(A->width, 16), d, 0.f});
      else
        for (int u : {2, 4, 8}) cands.push_back({ProductKind::Sell, u, d, 0.f});
    }
    if (want_staged) {
      const int eb = int(es) + (d ? 2 : 4);
      if (staged_table(A->fwd, eb, SolverStaged::max_entries(eb)).ok) {
        if (only && A->width > 0) {
          cands.push_back({ProductKind::Staged, staged_width(A->width), d, 0.f});
        } else {
          for (int u : {4, 8}) cands.push_back({ProductKind::Staged, u, d, 0.f});
          // A stencil whose longest row is a multiple of 9, 7 or 5 entries:
          // its full slices take the unmasked path.
          if (exact_staged_width(C.max_row) > 0)
            cands.push_back({ProductKind::Staged, exact_staged_width(C.max_row), d, 0.f});
        }
      }
    }
  }
  require(!cands.empty(), "spmv: no product kernel applies to this matrix");
  // SPMV_B200_SOLVER_PRODUCT=<vector|sell|staged>:<width>:<16|32> keeps only that
  // candidate (for profilers, whose serialised replays distort the timing).
  if (const char* pin = std::getenv("SPMV_B200_SOLVER_PRODUCT")) {
    static const char* kinds[] = {"vector", "sell", "staged"};
    std::vector<SolverProduct> kept;
    for (const SolverProduct& cd : cands) {
      const std::string name = std::string(kinds[int(cd.kind)]) + ":" + std::to_string(cd.w) +
                               ":" + (cd.d16 ? "16" : "32");
      if (name == pin) kept.push_back(cd);
    }
    require(!kept.empty(), "spmv: SPMV_B200_SOLVER_PRODUCT names no candidate of this matrix");
    cands = kept;
  }

  const spmv_l2gmap rm = A->row_map;
  std::vector<const void*> xs(P), own(P);
  std::vector<void*> ys(P);
  for (int r = 0; r < P; ++r) {
    xs[r] = x;
    own[r] = static_cast<const char*>(x) + rm->ranges[r] * es;
    ys[r] = static_cast<char*>(y) + rm->ranges[r] * es;
  }
  const void* const* xown = xown_rows ? own.data() : nullptr;
  const int mb = max_blocks_for(comm->num_sms, 256);
  cudaStream_t s = comm->stream;
  cudaEvent_t e0, e1;
  SPMVB_CUDA(cudaEventCreate(&e0));
  SPMVB_CUDA(cudaEventCreate(&e1));
  SolverProduct best = cands.front();
  best.us = 1e30f;
  static const char* names[] = {"vector", "sell", "staged"};
  try {
    for (SolverProduct& cd : cands) {
      SpmvArgs a;
      if (cd.sell_layout()) {
        fill_sell_args(a, C, C.sell_cols_global.as<int32_t>(), sell_vals, es, xs.data(),
                       ys.data(), xown, 256, mb);
      } else {
        fill_spmv_args(a, C, C.cols_global.as<int32_t>(), es, xs.data(), ys.data(), xown,
                       256 / cd.w, mb);
        if (f32)
          for (int r = 0; r < P; ++r)
            a.part[r].vals = C.vals32.as<float>() + C.parts[r].nz_off;
      }
      if (cd.d16) use_d16(a, C, cd.sell_layout());
      auto run = [&] { launch(cd, a, s); };
      run();
      constexpr int reps = 5;
      SPMVB_CUDA(cudaEventRecord(e0, s));
      for (int i = 0; i < reps; ++i) run();
      SPMVB_CUDA(cudaEventRecord(e1, s));
      SPMVB_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      SPMVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      cd.us = ms * 1000.f / reps;
      if (cd.us < best.us) best = cd;
      debug_log(std::string("solver product ") + (f32 ? "f32 " : "f64 ") +
                names[int(cd.kind)] + " " + std::to_string(cd.w) +
                (cd.d16 ? " d16 " : " d32 ") + std::to_string(cd.us) + " us");
    }
  } catch (...) {
    soft_check(cudaEventDestroy(e0), "cudaEventDestroy");
    soft_check(cudaEventDestroy(e1), "cudaEventDestroy");
    throw;
  }
  soft_check(cudaEventDestroy(e0), "cudaEventDestroy");
  soft_check(cudaEventDestroy(e1), "cudaEventDestroy");
  // 16-bit offsets within 3% of the same kernel with 32-bit columns count as
  // a tie and win it: they stream fewer bytes, which pays inside a solver
  // (whose other phases share the SMs and L2) even where the bare product
  // runs equally fast (c2 fused CG: 44.6 us per iteration against 47.6).
  if (!best.d16)
    for (const SolverProduct& cd : cands)
      if (cd.d16 && cd.kind == best.kind && cd.w == best.w && cd.us <= 1.03f * best.us) {
        best = cd;
        break;
      }
  return best;
}

spmv_kernel pick_kernel(spmv_kernel requested, const DevCsr& C, bool allow_sell) {
  if (requested == SPMV_KERNEL_SELL || requested == SPMV_KERNEL_STAGED)
    return allow_sell ? requested : SPMV_KERNEL_VECTOR;
  if (requested != SPMV_KERNEL_AUTO) return requested;
  const double skew_limit = std::max(64.0, 8.0 * C.mean_row);
  if (double(C.max_row) > skew_limit) return SPMV_KERNEL_MERGE;
  int64_t nnz = 0;
  for (const DevPart& D : C.parts) nnz += D.nnz;
  if (allow_sell && nnz > 0 && C.sell_padded > 0 && C.sell_padded <= nnz + nnz / 4)
    return SPMV_KERNEL_SELL;
  return SPMV_KERNEL_VECTOR;
}

int max_blocks_for(int num_sms, int BS) {
  // One wave of resident CTAs (2048 threads per SM), times two so that a
  // CTA finishing early finds work without waiting for the tail.
  return std::max(1, num_sms) * (2048 / BS) * 2;
}

void launch_spmv(const SpmvLaunch& L0, cudaStream_t stream) {
  SpmvLaunch L = L0;
  const bool cplx = L.dtype == SPMV_COMPLEX64 || L.dtype == SPMV_COMPLEX128;
  const int BS = L.block > 0 ? L.block : 256;
  require(BS == 128 || BS == 256 || BS == 512,
          "spmv: block must be 128, 256 or 512");
  spmv_kernel k = pick_kernel(L.kernel, *L.csr, L.csr->sell_built);
  // Complex products run SELL-32 or vector CSR (merge-path and the staged
  // pipeline are real only).
  if (cplx && k == SPMV_KERNEL_MERGE) k = SPMV_KERNEL_VECTOR;
  if (cplx && k == SPMV_KERNEL_STAGED) k = SPMV_KERNEL_SELL;
  // A width belongs to the kernel it was chosen for (lanes per row, loads or
  // gathers in flight); a fallback to another kernel uses its own default.
  const bool same_kind = k == L.kernel || L.kernel == SPMV_KERNEL_AUTO;
  if (!same_kind) L.width = 0;
  if (k == SPMV_KERNEL_MERGE) {
    require(L.carry != nullptr, "spmv: merge-path product needs a carry buffer");
    launch_merge(L, stream, *L.carry);
    return;
  }
  if (k == SPMV_KERNEL_SELL) {
    launch_sell(L, L.csr->sell_cols.as<int32_t>(), stream);
    return;
  }
  if (k == SPMV_KERNEL_STAGED) {
    launch_staged(L, stream);
    return;
  }
  const int W = L.width > 0 ? L.width : auto_width(L.csr->mean_row, L.dtype);
  require(W >= 1 && W <= 32 && (W & (W - 1)) == 0,
          "spmv: width must be 1..32, a power of two");
  SpmvArgs a;
  const size_t es = dtype_size(L.dtype);
  fill_spmv_args(a, *L.csr, L.cols, es, L.x, L.y, nullptr, BS / W,
                 max_blocks_for(L.num_sms, BS));
  if (a.nblocks == 0) return;
  switch (L.dtype) {
    case SPMV_FLOAT64: launch_vector_bs<double>(a, W, BS, stream); break;
    case SPMV_FLOAT32: launch_vector_bs<float>(a, W, BS, stream); break;
    case SPMV_COMPLEX128: launch_vector_bs<c128>(a, W, BS, stream); break;
    case SPMV_COMPLEX64: launch_vector_bs<c64>(a, W, BS, stream); break;
  }
  SPMVB_CUDA(cudaGetLastError());
}

}  // namespace spmvb
