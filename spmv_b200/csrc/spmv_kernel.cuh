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

// Gathers: g(P, c) returns entry c of the vector a rank's product reads.
// XGather loads the PartArg's x (KEEP: with the L2 evict-last policy, for
// solver vectors re-read every iteration); a solver may pass its own (the
// CG product forms p = r + beta p_old on the fly).
template <typename T, bool KEEP = false>
struct XGather {
  uint64_t pol;
  __device__ __forceinline__ XGather() : pol(KEEP ? l2_policy_keep() : 0) {}
  __device__ __forceinline__ T operator()(const PartArg& P, int c) const {
    const T* x = static_cast<const T*>(P.x);
    if constexpr (KEEP)
      return ld_pol(x + c, pol);
    else
      return ld_gather(x + c);
  }
};

// Dot product of one CSR row with the gathered vector, computed by a group
// of W lanes.  The result is identical in every lane of the group.
template <typename T, int W, class G>
__device__ __forceinline__ T row_dot(const int32_t* __restrict__ cols,
                                     const T* __restrict__ vals, const PartArg& P,
                                     const G& gx, int s, int e, int lane) {
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
      if (jj >= s && jj < e) sum += comp(v, u) * gx(P, comp(c, u));
    }
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) sum += shfl_xor(sum, o, W);
  return sum;
}

// As row_dot, with each column stored as a 16-bit offset from the row's
// global index g (column = g + offset; the solvers' fused-halo layout, where
// all offsets of a matrix fit in 16 bits).  N offsets load as one 4- or
// 8-byte vector beside the N values.
template <typename T>
struct Vec16;
template <>
struct Vec16<double> {
  using C = short2;
};
template <>
struct Vec16<float> {
  using C = short4;
};
__device__ __forceinline__ int comp(const short2& v, int i) { return i == 0 ? v.x : v.y; }
__device__ __forceinline__ int comp(const short4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

template <typename T, int W, class G>
__device__ __forceinline__ T row_dot16(const int16_t* __restrict__ offs,
                                       const T* __restrict__ vals, const PartArg& P,
                                       const G& gx, int g, int s, int e, int lane) {
  using VT = VecT<T>;
  constexpr int N = VT::N;
  T sum = T(0);
  for (int j = (s & ~(N - 1)) + lane * N; j < e; j += W * N) {
    const typename VT::V v =
        ld_stream(reinterpret_cast<const typename VT::V*>(vals + j));
    const typename Vec16<T>::C c =
        ld_stream(reinterpret_cast<const typename Vec16<T>::C*>(offs + j));
#pragma unroll
    for (int u = 0; u < N; ++u) {
      const int jj = j + u;
      if (jj >= s && jj < e) sum += comp(v, u) * gx(P, g + comp(c, u));
    }
  }
#pragma unroll
  for (int o = W / 2; o > 0; o >>= 1) sum += shfl_xor(sum, o, W);
  return sum;
}

// Visits every row of the CTA's rank: f(row, A_row . x) in lane 0 of each
// group.  Returns nothing; the callback accumulates what it needs.  D16:
// the PartArg's cols field points to 16-bit row offsets (see row_dot16).
template <typename T, int W, int BS, bool D16 = false, class F, class G = XGather<T>>
__device__ __forceinline__ void for_rows(const SpmvArgs& a, F&& f, const G& gx = G()) {
  const int p = find_part(a, blockIdx.x);
  const PartArg& P = a.part[p];
  const int32_t* __restrict__ cols = P.cols;
  const T* __restrict__ vals = static_cast<const T*>(P.vals);
  const int group = int(threadIdx.x) / W, lane = int(threadIdx.x) % W;
  for (int tile = int(blockIdx.x) - P.block_begin; tile < P.ntiles;
       tile += P.nblocks) {
    const int row = tile * (BS / W) + group;
    int s = 0, e = 0;
    if (row < P.nrows) {
      s = __ldg(P.rowptr + row);
      e = __ldg(P.rowptr + row + 1);
    }
    T sum;
    if constexpr (D16)
      sum = row_dot16<T, W>(reinterpret_cast<const int16_t*>(cols), vals, P, gx,
                            P.row0 + row, s, e, lane);
    else
      sum = row_dot<T, W>(cols, vals, P, gx, s, e, lane);
    if (lane == 0 && row < P.nrows) f(P, row, sum);
  }
}

// SELL-32 (sliced ELLPACK) traversal.  A rank's rows are cut into slices of
// 32; slice s holds w_s = its longest row's length columns, stored column by
// column: entry k of row 32s+l is at soff[s] + 32k + l (soff = the
// PartArg's rowptr field here).  Short rows are padded with column -1.  One
// warp takes one slice, lane l its row 32s+l, so every load of the warp is a
// contiguous 256-byte (FP64) or 128-byte run, and each lane issues U value and
// U column loads before it needs any of them.  A row is summed in storage
// order (k ascending), the order of the sequential CSR loop.
//
// KEEP (the solvers): matrix loads carry an L2 evict-first policy and the
// default gathers an evict-last one, so vectors re-read every iteration stay
// in L2 while the matrix streams through it.  D16: 16-bit offsets from the row's
// global index instead of 32-bit columns, -32768 marking padding.
template <typename T, int BS, int U, bool KEEP = false, bool D16 = false, class F,
          class G = XGather<T, KEEP>>
__device__ __forceinline__ void sell_for_rows(const SpmvArgs& a, F&& f, const G& gx = G()) {
  uint64_t stream = 0;
  if (KEEP) stream = l2_policy_stream();
  const int p = find_part(a, blockIdx.x);
  const PartArg& P = a.part[p];
  const int32_t* __restrict__ soff = P.rowptr;
  const int32_t* __restrict__ cols = P.cols;
  const T* __restrict__ vals = static_cast<const T*>(P.vals);
  const int warp = int(threadIdx.x) >> 5, lane = int(threadIdx.x) & 31;
  const int nslices = (P.nrows + 31) >> 5;
  for (int tile = int(blockIdx.x) - P.block_begin; tile < P.ntiles;
       tile += P.nblocks) {
    const int slice = tile * (BS / 32) + warp;
    if (slice >= nslices) continue;  // uniform across the warp
    const int o = __ldg(soff + slice);
    const int w = (__ldg(soff + slice + 1) - o) >> 5;
    const int g = P.row0 + slice * 32 + lane;  // global row (D16 base)
    T sum = T(0);
    for (int k0 = 0; k0 < w; k0 += U) {
      // All U column and value loads first, then the U gathers, then the
      // sums: each lane has 2U independent loads in flight, then U more.
      // (The two index forms test padding differently: a 16-bit offset by
      // its sentinel, a 32-bit column by its sign.  Both were measured
      // against alternatives on the 7-point stencil; the compiler schedules
      // the two forms best written this way.)
      T v[U];
      int c[U];
      bool ok[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        if (k0 + u < w) {
          const int idx = o + (k0 + u) * 32 + lane;
          if (D16) {
            const int16_t* offs = reinterpret_cast<const int16_t*>(cols);
            const int d = KEEP ? ld_pol(offs + idx, stream) : int(ld_stream(offs + idx));
            ok[u] = d != -32768;
            c[u] = g + d;
          } else {
            c[u] = KEEP ? ld_pol(cols + idx, stream) : ld_stream(cols + idx);
          }
          if constexpr (KEEP)
            v[u] = ld_pol(vals + idx, stream);
          else
            v[u] = ld_stream(vals + idx);
        } else {
          v[u] = T(0);
          c[u] = D16 ? 0 : -1;
          ok[u] = false;
        }
        if (!D16) ok[u] = c[u] >= 0;
      }
      T xv[U];
#pragma unroll
      for (int u = 0; u < U; ++u) xv[u] = ok[u] ? gx(P, c[u]) : T(0);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (ok[u]) sum += v[u] * xv[u];
    }
    const int row = slice * 32 + lane;
    if (row < P.nrows) f(P, row, sum);
  }
}

template <typename T, int BS, int U, bool D16 = false, bool KEEP = false>
__global__ void __launch_bounds__(BS)
    spmv_sell_kernel(const __grid_constant__ SpmvArgs a) {
  sell_for_rows<T, BS, U, KEEP, D16>(a, [](const PartArg& P, int row, T sum) {
    static_cast<T*>(P.y)[row] = sum;
  });
}

template <typename T, int W, int BS, bool D16 = false>
__global__ void __launch_bounds__(BS)
    spmv_vector_kernel(const __grid_constant__ SpmvArgs a) {
  for_rows<T, W, BS, D16>(a, [](const PartArg& P, int row, T sum) {
    static_cast<T*>(P.y)[row] = sum;
  });
}

}  // namespace spmvb
