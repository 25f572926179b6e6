// Ghost exchange between the virtual ranks of one GPU: L2GMap::update and
// L2GMap::reverse_update of the reference (L2GMap.cpp:126-170).
//
// update is one gather over every ghost slot of every rank: the slot receives
// the owner's entry, a bit-exact copy (the reference packs the owner values
// and moves them with MPI_Neighbor_alltoallv, L2GMap.cpp:137-147).
//
// reverse_update is one thread per distinct (rank, owned index) target: it
// loads the target once, adds its contributors in the reference's order
// (neighbour rank order, then the neighbour's ghost order, L2GMap.cpp:168-169)
// and stores once.  No atomics, so the result is bitwise the reference's.
#include "internal.h"
#include "kernels.cuh"

namespace spmvb {

namespace {

// Element types moved by the halo kernels.  Complex values are added
// component-wise.
struct C64 {
  float re, im;
};
struct C128 {
  double re, im;
};
__device__ __forceinline__ double addv(double a, double b) { return a + b; }
__device__ __forceinline__ float addv(float a, float b) { return a + b; }
__device__ __forceinline__ C64 addv(C64 a, C64 b) {
  return {a.re + b.re, a.im + b.im};
}
__device__ __forceinline__ C128 addv(C128 a, C128 b) {
  return {a.re + b.re, a.im + b.im};
}

template <typename T>
__global__ void update_kernel(const __grid_constant__ PtrTable v,
                              const int32_t* __restrict__ ranks,
                              const int32_t* __restrict__ dst,
                              const int32_t* __restrict__ src, int64_t n) {
  // Launched programmatically: wait for the previous kernel's writes (x may
  // have just been produced).  Once a CTA has issued its part of the gather
  // the product that usually follows may be scheduled (it waits for this
  // kernel's completion before reading anything).
  pdl_wait();
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x) {
    const int rr = ranks[i];
    const T val = static_cast<const T*>(v.p[rr & 0xffff])[src[i]];
    static_cast<T*>(v.p[rr >> 16])[dst[i]] = val;
  }
  pdl_launch_dependents();
}

template <typename T>
__global__ void reverse_kernel(const __grid_constant__ PtrTable v,
                               const int32_t* __restrict__ tgt_rank,
                               const int32_t* __restrict__ tgt_idx,
                               const int32_t* __restrict__ ptr,
                               const int32_t* __restrict__ src_rank,
                               const int32_t* __restrict__ src_idx,
                               int64_t n) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n;
       t += int64_t(gridDim.x) * blockDim.x) {
    T* out = static_cast<T*>(v.p[tgt_rank[t]]) + tgt_idx[t];
    T acc = *out;
    for (int32_t c = ptr[t]; c < ptr[t + 1]; ++c)
      acc = addv(acc, static_cast<const T*>(v.p[src_rank[c]])[src_idx[c]]);
    *out = acc;
  }
}

int grid_for(int64_t n, int threads, int num_sms) {
  const int64_t want = (n + threads - 1) / threads;
  const int64_t cap = int64_t(num_sms) * 16;
  return int(std::max<int64_t>(1, std::min(want, cap)));
}

PtrTable table_of(spmv_l2gmap map, void* const* vecs) {
  PtrTable t{};
  for (int r = 0; r < map->comm->size; ++r) t.p[r] = vecs[r];
  return t;
}

}  // namespace

void launch_update(spmv_l2gmap map, spmv_dtype dtype, void* const* vecs,
                   cudaStream_t stream) {
  build_halo_tables(map);
  const HaloTables& H = map->halo;
  if (H.n_update == 0) return;
  const PtrTable t = table_of(map, vecs);
  const int threads = 256;
  const int grid = grid_for(H.n_update, threads, map->comm->num_sms);
  const int32_t* rk = H.upd_ranks.as<int32_t>();
  const int32_t* d = H.upd_dst.as<int32_t>();
  const int32_t* s = H.upd_src.as<int32_t>();
  int64_t n = H.n_update;
  void* args[] = {const_cast<PtrTable*>(&t), &rk, &d, &s, &n};
  const void* fn = nullptr;
  switch (dtype) {
    case SPMV_FLOAT64: fn = (const void*)update_kernel<double>; break;
    case SPMV_FLOAT32: fn = (const void*)update_kernel<float>; break;
    case SPMV_COMPLEX64: fn = (const void*)update_kernel<C64>; break;
    case SPMV_COMPLEX128: fn = (const void*)update_kernel<C128>; break;
  }
  launch_pdl(fn, dim3(grid), dim3(threads), 0, stream, args);
  SPMVB_CUDA(cudaGetLastError());
}

void launch_reverse_update(spmv_l2gmap map, spmv_dtype dtype,
                           void* const* vecs, cudaStream_t stream) {
  build_halo_tables(map);
  const HaloTables& H = map->halo;
  if (H.n_targets == 0) return;
  const PtrTable t = table_of(map, vecs);
  const int threads = 256;
  const int grid = grid_for(H.n_targets, threads, map->comm->num_sms);
  const int32_t* tr = H.rev_tgt_rank.as<int32_t>();
  const int32_t* ti = H.rev_tgt_idx.as<int32_t>();
  const int32_t* pt = H.rev_ptr.as<int32_t>();
  const int32_t* sr = H.rev_src_rank.as<int32_t>();
  const int32_t* si = H.rev_src_idx.as<int32_t>();
  switch (dtype) {
    case SPMV_FLOAT64: reverse_kernel<double><<<grid, threads, 0, stream>>>(t, tr, ti, pt, sr, si, H.n_targets); break;
    case SPMV_FLOAT32: reverse_kernel<float><<<grid, threads, 0, stream>>>(t, tr, ti, pt, sr, si, H.n_targets); break;
    case SPMV_COMPLEX64: reverse_kernel<C64><<<grid, threads, 0, stream>>>(t, tr, ti, pt, sr, si, H.n_targets); break;
    case SPMV_COMPLEX128: reverse_kernel<C128><<<grid, threads, 0, stream>>>(t, tr, ti, pt, sr, si, H.n_targets); break;
  }
  SPMVB_CUDA(cudaGetLastError());
}

}  // namespace spmvb
