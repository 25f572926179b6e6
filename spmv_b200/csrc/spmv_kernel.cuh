// The vector-CSR row kernel, shared by the plain product (spmv.cu) and the
// CG product with its p.Ap epilogue (cg.cu).
#pragma once

#include "kernels.cuh"

namespace spmvb {

struct DevCsr;
// Fills the per-rank table of one launch over `csr` (spmv.cu).  Returns the
// number of CTAs; each covers tiles of `rows_per_tile` rows.
int fill_spmv_args(SpmvArgs& a, const DevCsr& csr, const int32_t* cols,
                   size_t es, const void* const* x, void* const* y,
                   const void* const* xown, int rows_per_tile,
                   int max_blocks);

// Dot product of one CSR row with x, computed by a group of W lanes.  The
// result is identical in every lane of the group.
template <typename T, int W>
__device__ __forceinline__ T row_dot(const int32_t* __restrict__ cols,
                                     const T* __restrict__ vals,
                                     const T* __restrict__ x, int s, int e,
                                     int lane) {
  using VT = VecT<T>;
  constexpr int N = VT::N;
  T sum = T(0);
  for (int j = (s & ~(N - 1)) + lane * N; j < e; j += W * N) {
    const typename VT::V v =
        ld_stream(reinterpret_cast<const typename VT::V*>(vals + j));
    const typename VT::C c =
        ld_stream(reinterpret_cast<const typename VT::C*>(cols + j));
#pragma unroll
    for (int u = 0; u < N; ++u) {
      const int jj = j + u;
      if (jj >= s && jj < e) sum += comp(v, u) * ld_gather(x + comp(c, u));
    }
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1)
    sum += __shfl_xor_sync(0xffffffffu, sum, o, W);
  return sum;
}

// Visits every row of the CTA's rank: f(row, A_row . x) in lane 0 of each
// group.  Returns nothing; the callback accumulates what it needs.
template <typename T, int W, int BS, class F>
__device__ __forceinline__ void for_rows(const SpmvArgs& a, F&& f) {
  const int p = find_part(a, blockIdx.x);
  const PartArg& P = a.part[p];
  const int32_t* __restrict__ cols = P.cols;
  const T* __restrict__ vals = static_cast<const T*>(P.vals);
  const T* __restrict__ x = static_cast<const T*>(P.x);
  const int group = int(threadIdx.x) / W, lane = int(threadIdx.x) % W;
  for (int tile = int(blockIdx.x) - P.block_begin; tile < P.ntiles;
       tile += P.nblocks) {
    const int row = tile * (BS / W) + group;
    int s = 0, e = 0;
    if (row < P.nrows) {
      s = __ldg(P.rowptr + row);
      e = __ldg(P.rowptr + row + 1);
    }
    const T sum = row_dot<T, W>(cols, vals, x, s, e, lane);
    if (lane == 0 && row < P.nrows) f(P, row, sum);
  }
}

template <typename T, int W, int BS>
__global__ void __launch_bounds__(BS)
    spmv_vector_kernel(const __grid_constant__ SpmvArgs a) {
  for_rows<T, W, BS>(a, [](const PartArg& P, int row, T sum) {
    static_cast<T*>(P.y)[row] = sum;
  });
}

}  // namespace spmvb
