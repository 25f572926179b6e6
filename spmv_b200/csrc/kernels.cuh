// Device-side building blocks shared by the kernels: kernel-parameter tables,
// vector types, cache-hinted loads and deterministic block reductions.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "spmv_b200.h"

namespace spmvb {

// Per-rank descriptor of one launch over a concatenated CSR.  A launch covers
// all ranks; rank p owns CTAs [block_begin, block_begin + nblocks), which
// stride over its ntiles row tiles.
struct PartArg {
  const int32_t* rowptr;   // rank's row pointers (nrows+1), relative to vals
  const int32_t* cols;     // rank's column indices
  const void* vals;        // rank's values
  const void* x;           // input vector the column indices refer to
  void* y;                 // output rows
  const void* xown;        // this rank's own entries of x (row-aligned)
  int32_t nrows;
  int32_t block_begin;
  int32_t nblocks;
  int32_t ntiles;
  int32_t row0;            // global index of the rank's first row (16-bit
  int32_t pad;             // column offsets are relative to the global row)
};

struct SpmvArgs {
  int32_t nparts;
  int32_t nblocks;
  PartArg part[SPMV_MAX_PARTS];
};

// Pointer per rank, for the halo kernels.
struct PtrTable {
  void* p[SPMV_MAX_PARTS];
};

template <typename T>
struct VecT;
template <>
struct VecT<double> {
  static constexpr int N = 2;  // 16-byte value loads
  using V = double2;
  using C = int2;
};
template <>
struct VecT<float> {
  static constexpr int N = 4;
  using V = float4;
  using C = int4;
};

__device__ __forceinline__ double comp(const double2& v, int i) {
  return i == 0 ? v.x : v.y;
}
__device__ __forceinline__ float comp(const float4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}
__device__ __forceinline__ int comp(const int2& v, int i) {
  return i == 0 ? v.x : v.y;
}
__device__ __forceinline__ int comp(const int4& v, int i) {
  return i == 0 ? v.x : (i == 1 ? v.y : (i == 2 ? v.z : v.w));
}

// Complex scalar with the layout of std::complex<F> (re, im).  The product
// rounds as std::complex's does for finite values without FMA contraction:
// re = a.re b.re - a.im b.im, im = a.re b.im + a.im b.re, each product and
// sum rounded separately (the library is compiled with -fmad=false).
template <typename F>
struct alignas(2 * sizeof(F)) Cplx {
  F re, im;
  Cplx() = default;
  __host__ __device__ constexpr Cplx(F r, F i = F(0)) : re(r), im(i) {}
};
template <typename F>
__device__ __forceinline__ Cplx<F> operator*(const Cplx<F>& a, const Cplx<F>& b) {
  return Cplx<F>(a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re);
}
template <typename F>
__device__ __forceinline__ Cplx<F> operator+(const Cplx<F>& a, const Cplx<F>& b) {
  return Cplx<F>(a.re + b.re, a.im + b.im);
}
template <typename F>
__device__ __forceinline__ Cplx<F>& operator+=(Cplx<F>& a, const Cplx<F>& b) {
  a.re += b.re;
  a.im += b.im;
  return a;
}
using c64 = Cplx<float>;
using c128 = Cplx<double>;

// Streaming loads for matrix data (read once per product): evict-first.
template <typename V>
__device__ __forceinline__ V ld_stream(const V* p) {
  return __ldcs(p);
}
__device__ __forceinline__ c128 ld_stream(const c128* p) {
  const double2 v = __ldcs(reinterpret_cast<const double2*>(p));
  return c128(v.x, v.y);
}
__device__ __forceinline__ c64 ld_stream(const c64* p) {
  const float2 v = __ldcs(reinterpret_cast<const float2*>(p));
  return c64(v.x, v.y);
}
// Read-only cached load for gathered vector entries.
template <typename T>
__device__ __forceinline__ T ld_gather(const T* p) {
  return __ldg(p);
}
__device__ __forceinline__ c128 ld_gather(const c128* p) {
  const double2 v = __ldg(reinterpret_cast<const double2*>(p));
  return c128(v.x, v.y);
}
__device__ __forceinline__ c64 ld_gather(const c64* p) {
  const float2 v = __ldg(reinterpret_cast<const float2*>(p));
  return c64(v.x, v.y);
}

// Vector widths of the vector-CSR loads for complex values: one complex
// double or two complex floats per 16-byte load.
struct alignas(16) c64x2 {
  c64 a, b;
};
__device__ __forceinline__ c64x2 ld_stream(const c64x2* p) {
  const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
  return c64x2{c64(v.x, v.y), c64(v.z, v.w)};
}
template <>
struct VecT<c128> {
  static constexpr int N = 1;
  using V = c128;
  using C = int;
};
template <>
struct VecT<c64> {
  static constexpr int N = 2;
  using V = c64x2;
  using C = int2;
};
__device__ __forceinline__ c128 comp(const c128& v, int) { return v; }
__device__ __forceinline__ int comp(int v, int) { return v; }
__device__ __forceinline__ c64 comp(const c64x2& v, int i) { return i == 0 ? v.a : v.b; }

// Butterfly shuffle within groups of W lanes (real and complex).
template <typename T>
__device__ __forceinline__ T shfl_xor(T v, int o, int W) {
  return __shfl_xor_sync(0xffffffffu, v, o, W);
}
template <typename F>
__device__ __forceinline__ Cplx<F> shfl_xor(Cplx<F> v, int o, int W) {
  return Cplx<F>(__shfl_xor_sync(0xffffffffu, v.re, o, W),
                 __shfl_xor_sync(0xffffffffu, v.im, o, W));
}

// L2 cache policies (per-instruction hints; no device setting is touched).
// Solver vectors are re-read every iteration and fit in L2 with room to
// spare, the matrix is streamed once per iteration: vector accesses carry an
// evict-last policy, matrix loads an evict-first one, so the matrix stream
// does not push the vectors out.
__device__ __forceinline__ uint64_t l2_policy_keep() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_stream() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ double ld_pol(const double* a, uint64_t pol) {
  double v;
  asm volatile("ld.global.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ float ld_pol(const float* a, uint64_t pol) {
  float v;
  asm volatile("ld.global.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ int ld_pol(const int* a, uint64_t pol) {
  int v;
  asm volatile("ld.global.L2::cache_hint.s32 %0, [%1], %2;" : "=r"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ int ld_pol(const int16_t* a, uint64_t pol) {
  short v;
  asm volatile("ld.global.L2::cache_hint.s16 %0, [%1], %2;" : "=h"(v) : "l"(a), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_pol(double* a, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(a), "d"(v), "l"(pol)
               : "memory");
}
__device__ __forceinline__ void st_pol(float* a, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(a), "f"(v), "l"(pol)
               : "memory");
}

// Programmatic dependent launch.  A kernel launched with the
// programmatic-stream-serialization attribute may start before the kernel
// ahead of it on the stream has finished; pdl_wait() (griddepcontrol.wait)
// blocks until that kernel has completed and its memory operations are
// visible, so a kernel that calls it before its first global-memory access
// behaves exactly as with an ordinary launch and gains only the overlap of
// its launch with the previous kernel's tail.  pdl_launch_dependents() lets
// the next such kernel be scheduled early.  Both are no-ops without the
// attribute.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() {
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Rank owning CTA `b` of a launch (ranks' CTA ranges are ascending).
__device__ __forceinline__ int find_part(const SpmvArgs& a, int b) {
  int lo = 0, hi = a.nparts - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (a.part[mid].block_begin <= b)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Sum over the CTA; the result is valid in thread 0.  The order of additions
// depends only on blockDim, so results are reproducible run to run.
template <int BS>
__device__ __forceinline__ double block_sum(double v, double* smem) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (lane == 0) smem[warp] = v;
  __syncthreads();
  if (warp == 0) {
    v = lane < (BS >> 5) ? smem[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  }
  __syncthreads();
  return v;
}

// Single-pass grid reduction: every CTA stores its partial; the last CTA to
// arrive (atomic ticket) sums all partials in index order and returns true in
// all of its threads with the total in *total (valid in thread 0).  The
// ticket counter is reset by the last CTA so the kernel can be relaunched.
// No CTA waits for another: there is no spin loop.
template <int BS>
__device__ __forceinline__ bool grid_sum(double part, double* partials,
                                         unsigned int* ticket, double* total,
                                         double* smem) {
  __shared__ bool s_last;
  if (threadIdx.x == 0) {
    partials[blockIdx.x] = part;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double v = 0.0;
  for (unsigned int i = threadIdx.x; i < gridDim.x; i += BS)
    v += __ldcg(partials + i);
  v = block_sum<BS>(v, smem);
  if (threadIdx.x == 0) {
    *total = v;
    *ticket = 0u;
  }
  return true;
}

// Two sums at once (same scheme as grid_sum; partials holds 2 per CTA).
template <int BS>
__device__ __forceinline__ bool grid_sum2(double a, double b, double* partials,
                                          unsigned int* ticket, double* ta,
                                          double* tb, double* smem) {
  __shared__ bool s_last;
  a = block_sum<BS>(a, smem);
  b = block_sum<BS>(b, smem);
  if (threadIdx.x == 0) {
    partials[2 * blockIdx.x] = a;
    partials[2 * blockIdx.x + 1] = b;
    __threadfence();
    const unsigned int t = atomicAdd(ticket, 1u);
    s_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!s_last) return false;
  __threadfence();
  double va = 0.0, vb = 0.0;
  for (unsigned int i = threadIdx.x; i < gridDim.x; i += BS) {
    va += __ldcg(partials + 2 * i);
    vb += __ldcg(partials + 2 * i + 1);
  }
  va = block_sum<BS>(va, smem);
  vb = block_sum<BS>(vb, smem);
  if (threadIdx.x == 0) {
    *ta = va;
    *tb = vb;
    *ticket = 0u;
  }
  return true;
}

// ---------------------------------------------------------------------------
// Grid barrier and grid sum for cooperative launches (every CTA resident),
// over the first NT threads of each CTA (named barrier 1; the CTA's other
// warps do not take part).  `count` is zero at launch; the e-th barrier of
// the launch waits for count = e * gridDim.x.  Waits are bounded by
// `limit_ns` of global time: a barrier that does not complete in time, or
// sees *err raised, raises *err and returns false (CTAs that have already
// passed fail at their next barrier).
__device__ __forceinline__ void named_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// One thread per CTA, after a CTA barrier: arrival is a release (the CTA's
// writes before the barrier are visible to any CTA that sees the count),
// the wait an acquire.
__device__ __forceinline__ bool grid_arrive_wait(unsigned long long* count,
                                                 unsigned long long target, int* err,
                                                 unsigned long long limit_ns) {
  asm volatile("red.release.gpu.global.add.u64 [%0], %1;" ::"l"(count), "l"(1ull) : "memory");
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (uint32_t i = 0;; ++i) {
    unsigned long long c;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(c) : "l"(count) : "memory");
    if (c >= target) return true;
    if (*static_cast<volatile int*>(err)) return false;
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > limit_ns) break;
    if (i >= 64) __nanosleep(32);
  }
  atomicExch(err, 1);
  return false;
}

template <int NT>
struct GridSum {
  double red[NT / 32];
  double total;
  int ok;
};

// Barrier only.  All NT threads call it; returns the same verdict in all.
template <int NT>
__device__ __forceinline__ bool coop_grid_barrier(unsigned long long* count,
                                                  unsigned long long target, int* err,
                                                  unsigned long long limit_ns, GridSum<NT>& s) {
  named_sync(1, NT);
  if (threadIdx.x == 0) s.ok = grid_arrive_wait(count, target, err, limit_ns);
  named_sync(1, NT);
  return s.ok != 0;
}

// Warp sums of v into s.red (then a barrier of the NT threads).
template <int NT>
__device__ __forceinline__ void warp_partials(double v, GridSum<NT>& s) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) s.red[threadIdx.x >> 5] = v;
  named_sync(1, NT);
}

// s.red summed in warp order (one thread).
template <int NT>
__device__ __forceinline__ double sum_partials(const GridSum<NT>& s) {
  double t = 0.0;
#pragma unroll 4
  for (int w = 0; w < NT / 32; ++w) t += s.red[w];
  return t;
}

// Sum of v over the NT threads of every CTA.  Each CTA publishes its partial
// (warp sums, then warps in index order) in parts[blockIdx.x]; after the
// barrier every CTA reads all partials at once (thread i takes partials i,
// i + NT, ...) and reduces them in the same fixed order, so all CTAs hold
// the same total.
template <int NT>
__device__ __forceinline__ bool coop_grid_sum(double v, double* parts, unsigned long long* count,
                                              unsigned long long target, int* err,
                                              unsigned long long limit_ns, GridSum<NT>& s,
                                              double* total) {
  warp_partials<NT>(v, s);
  if (threadIdx.x == 0) {
    __stcg(parts + blockIdx.x, sum_partials<NT>(s));
    s.ok = grid_arrive_wait(count, target, err, limit_ns);
  }
  named_sync(1, NT);
  if (!s.ok) return false;
  double t = 0.0;
  for (unsigned int i = threadIdx.x; i < gridDim.x; i += unsigned(NT)) t += __ldcg(parts + i);
  warp_partials<NT>(t, s);
  if (threadIdx.x == 0) s.total = sum_partials<NT>(s);
  named_sync(1, NT);
  *total = s.total;
  return true;
}

// N sums at once, the same way: parts holds N partials per CTA (CTA b's at
// parts[N b .. N b + N - 1]); every CTA gets the same N totals.
template <int NT, int N>
struct GridSumN {
  double red[N][NT / 32];
  double total[N];
  int ok;
};

template <int NT, int N>
__device__ __forceinline__ bool coop_grid_sum_n(const double (&v)[N], double* parts,
                                                unsigned long long* count,
                                                unsigned long long target, int* err,
                                                unsigned long long limit_ns, GridSumN<NT, N>& s,
                                                double (&total)[N]) {
  const int warp = int(threadIdx.x) >> 5, lane = int(threadIdx.x) & 31;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double x = v[j];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) s.red[j][warp] = x;
  }
  named_sync(1, NT);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; ++w) t += s.red[j][w];
      __stcg(parts + N * blockIdx.x + j, t);
    }
    s.ok = grid_arrive_wait(count, target, err, limit_ns);
  }
  named_sync(1, NT);
  if (!s.ok) return false;
#pragma unroll
  for (int j = 0; j < N; ++j) {
    double t = 0.0;
    for (unsigned int i = threadIdx.x; i < gridDim.x; i += unsigned(NT))
      t += __ldcg(parts + N * i + j);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) s.red[j][warp] = t;
  }
  named_sync(1, NT);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int j = 0; j < N; ++j) {
      double t = 0.0;
      for (int w = 0; w < NT / 32; ++w) t += s.red[j][w];
      s.total[j] = t;
    }
  }
  named_sync(1, NT);
#pragma unroll
  for (int j = 0; j < N; ++j) total[j] = s.total[j];
  return true;
}

}  // namespace spmvb
