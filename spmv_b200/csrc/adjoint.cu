// Adjoint of x = A^{-1} b (no counterpart in the reference).
//
// For a loss L(x) with g = dL/dx, the adjoint solve A^T lambda = g (A is SPD
// here, so the same CG) gives dL/db = lambda and dL/dA_ij = -lambda_i x_j.
// Only the stored entries of A are parameters, so the gradient with respect
// to A's values is the outer product -lambda x^T sampled on A's pattern:
//
//   out[k] = scale * lambda[row(k)] * x[col(k)]      for every stored entry k
//
// with scale = -1 for the gradient.  One group of W lanes per row, as in the
// product: the row's lambda is loaded once, x is gathered per entry, and the
// output is written in the matrix's own entry order (coalesced).
#include "internal.h"
#include "spmv_kernel.cuh"

namespace spmvb {

namespace {

// Launch table: x = column-space vectors, xown = lambda, y = output values.
template <typename T, int W, int BS>
__global__ void __launch_bounds__(BS)
    sample_outer_kernel(const __grid_constant__ SpmvArgs a, T scale) {
  const int p = find_part(a, blockIdx.x);
  const PartArg& P = a.part[p];
  const T* __restrict__ x = static_cast<const T*>(P.x);
  const T* __restrict__ lam = static_cast<const T*>(P.xown);
  T* __restrict__ out = static_cast<T*>(P.y);
  const int group = int(threadIdx.x) / W, lane = int(threadIdx.x) % W;
  for (int tile = int(blockIdx.x) - P.block_begin; tile < P.ntiles;
       tile += P.nblocks) {
    const int row = tile * (BS / W) + group;
    if (row >= P.nrows) continue;
    const int s = __ldg(P.rowptr + row), e = __ldg(P.rowptr + row + 1);
    const T l = scale * __ldg(lam + row);
    for (int j = s + lane; j < e; j += W) out[j] = l * __ldg(x + __ldg(P.cols + j));
  }
}

}  // namespace

void launch_sample_outer(spmv_matrix A, double scale, const void* const* lambda,
                         const void* const* x, void* const* out,
                         cudaStream_t stream) {
  const DevCsr& C = A->fwd;
  const size_t es = dtype_size(A->dtype);
  const int P = A->comm->size;
  constexpr int BS = 256;
  const int W = auto_width(C.mean_row, A->dtype);
  SpmvArgs a;
  // y carries the per-rank output base; fill_spmv_args offsets only the
  // matrix arrays, so rank r's entries are out[r][0 .. nnz_r).
  std::vector<void*> outs(out, out + P);
  fill_spmv_args(a, C, C.cols.as<int32_t>(), es, x, outs.data(), lambda, BS / W,
                 max_blocks_for(A->comm->num_sms, BS));
  if (a.nblocks == 0) return;
  const dim3 grid(a.nblocks);
#define SPMVB_SAMPLE(T)                                                              \
  switch (W) {                                                                       \
    case 1: sample_outer_kernel<T, 1, BS><<<grid, BS, 0, stream>>>(a, T(scale)); break; \
    case 2: sample_outer_kernel<T, 2, BS><<<grid, BS, 0, stream>>>(a, T(scale)); break; \
    case 4: sample_outer_kernel<T, 4, BS><<<grid, BS, 0, stream>>>(a, T(scale)); break; \
    case 8: sample_outer_kernel<T, 8, BS><<<grid, BS, 0, stream>>>(a, T(scale)); break; \
    case 16: sample_outer_kernel<T, 16, BS><<<grid, BS, 0, stream>>>(a, T(scale)); break; \
    default: sample_outer_kernel<T, 32, BS><<<grid, BS, 0, stream>>>(a, T(scale)); break; \
  }
  if (A->dtype == SPMV_FLOAT64) {
    SPMVB_SAMPLE(double)
  } else {
    SPMVB_SAMPLE(float)
  }
#undef SPMVB_SAMPLE
  SPMVB_CUDA(cudaGetLastError());
}

}  // namespace spmvb
