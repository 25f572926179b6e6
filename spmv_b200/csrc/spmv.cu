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
#include <cmath>

#include "internal.h"
#include "spmv_kernel.cuh"

namespace spmvb {

int auto_width(double mean_row, spmv_dtype dtype) {
  const int N = dtype == SPMV_FLOAT32 ? 4 : 2;
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

spmv_kernel pick_kernel(spmv_kernel requested, const DevCsr& C, bool allow_sell) {
  if (requested == SPMV_KERNEL_SELL) return allow_sell ? SPMV_KERNEL_SELL : SPMV_KERNEL_VECTOR;
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

void launch_spmv(const SpmvLaunch& L, cudaStream_t stream) {
  require(L.dtype == SPMV_FLOAT64 || L.dtype == SPMV_FLOAT32,
          "spmv: only float64 and float32 products are implemented");
  const int W = L.width > 0 ? L.width : auto_width(L.csr->mean_row, L.dtype);
  const int BS = L.block > 0 ? L.block : 256;
  require(W >= 1 && W <= 32 && (W & (W - 1)) == 0,
          "spmv: width must be 1..32, a power of two");
  require(BS == 128 || BS == 256 || BS == 512,
          "spmv: block must be 128, 256 or 512");
  const spmv_kernel k = pick_kernel(L.kernel, *L.csr, L.csr->sell_built);
  if (k == SPMV_KERNEL_MERGE) {
    require(L.carry != nullptr, "spmv: merge-path product needs a carry buffer");
    launch_merge(L, stream, *L.carry);
    return;
  }
  if (k == SPMV_KERNEL_SELL) {
    launch_sell(L, L.csr->sell_cols.as<int32_t>(), stream);
    return;
  }
  SpmvArgs a;
  const size_t es = dtype_size(L.dtype);
  fill_spmv_args(a, *L.csr, L.cols, es, L.x, L.y, nullptr, BS / W,
                 max_blocks_for(L.num_sms, BS));
  if (a.nblocks == 0) return;
  if (L.dtype == SPMV_FLOAT64)
    launch_vector_bs<double>(a, W, BS, stream);
  else
    launch_vector_bs<float>(a, W, BS, stream);
  SPMVB_CUDA(cudaGetLastError());
}

}  // namespace spmvb
