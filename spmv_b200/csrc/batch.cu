// Batched mixed-precision CG: many independent SPD systems of uneven size in
// one persistent launch (no counterpart in the reference; it builds on
// spmv::cg, cg.cpp:11-83, and on the refinement scheme of ir.cu).
//
// Work queue: systems are visited largest first (by nonzeros) so the long
// solves start early.  A thread-block cluster of CL CTAs (on CL SMs) pops one
// system at a time from an atomic counter; its CTAs split the system's rows
// into CL contiguous parts and run, per iteration,
//
//   A   y = A32 p on own rows, p.y partial                 | cluster barrier
//   B   alpha; d += alpha p, r -= alpha y, r.r partial     | cluster barrier
//   C   (refinement, see ir.cu) x += d, d = 0              | cluster barrier
//       r = fl32(b - A64 x), ||b - A x||^2 (FP64), r.r, r.p | cluster barrier
//   D   p = r + beta (p - c r)                             | cluster barrier
//
// Partial sums go to a slot in each CTA's shared memory; after the barrier
// every CTA reads the CL slots through distributed shared memory in rank
// order and forms the same total, so every CTA takes the same branch and
// meets the same barriers: the control flow is uniform across the cluster by
// construction, and each loop is bounded by max_its.  Vectors live in global
// memory (each system's rows are read by its own cluster only).  The
// convergence test ||b - A x|| / ||b|| < rtol is made on the FP64 residual.
#include <cooperative_groups.h>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "internal.h"
#include "spmv_kernel.cuh"

namespace cgx = cooperative_groups;

struct spmv_batch_s {
  spmv_comm comm = nullptr;
  int nsys = 0;
  std::vector<int32_t> n;          // rows per system
  std::vector<int64_t> row_off;    // first row of each system (global rows)
  std::vector<int64_t> nz_off;     // first entry of each system
  std::vector<int64_t> rp_off;     // first row pointer of each system
  int64_t rows = 0, nnz = 0;
  double mean_row = 0;
  spmvb::DevBuf d_n, d_row_off, d_nz_off, d_rp_off, d_order, rowptr, cols, vals64,
      vals32, b, x, r, p, y, d, counter, results;
  int cluster = 1;                 // CTAs per system (1, 2, 4 or 8)
};

namespace spmvb {

namespace {

constexpr int BBS = 512;  // threads per CTA

struct BatchResult {
  int iterations, refinements, status, converged;
  double relres;
};

struct BatchArgs {
  const int32_t* n;
  const int64_t* row_off;
  const int64_t* nz_off;
  const int64_t* rp_off;
  const int32_t* order;
  const int32_t* rowptr;
  const int32_t* cols;
  const double* vals64;
  const float* vals32;
  const double* b;
  double* x;
  float* r;
  float* p;
  float* y;
  float* d;
  unsigned int* counter;
  BatchResult* res;
  int nsys;
  int kmax;
  double rtol2;
  double delta2;
};

// Sum of v over the CTA (valid in all threads).
__device__ __forceinline__ double cta_sum(double v, double* smem) {
  v = block_sum<BBS>(v, smem);
  if (threadIdx.x == 0) smem[32] = v;
  __syncthreads();
  const double t = smem[32];
  __syncthreads();
  return t;
}

// Cluster-wide sums of NV values: each CTA publishes its CTA sums in
// slot[0..NV), the barrier makes them visible, and every CTA adds the CL
// slots in rank order.  A second barrier keeps the slots from being
// overwritten before every CTA has read them.
template <int CL, int NV>
__device__ __forceinline__ void cluster_sums(double (&v)[NV], double* slot,
                                             double* smem) {
#pragma unroll
  for (int i = 0; i < NV; ++i) v[i] = cta_sum(v[i], smem);
  if (CL == 1) return;
  cgx::cluster_group cl = cgx::this_cluster();
  if (threadIdx.x == 0)
#pragma unroll
    for (int i = 0; i < NV; ++i) slot[i] = v[i];
  cl.sync();
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    double t = 0.0;
    for (int c = 0; c < CL; ++c) t += cl.map_shared_rank(slot, c)[i];
    v[i] = t;
  }
  cl.sync();
}

template <int CL>
__device__ __forceinline__ void cluster_barrier() {
  if (CL == 1)
    __syncthreads();
  else
    cgx::this_cluster().sync();
}

// y_i = sum_j A_ij v_j over rows [r0, r1) of one system: W lanes per row.
template <typename T, typename V, int W, class F>
__device__ __forceinline__ void sys_rows(const int32_t* __restrict__ rp,
                                         const int32_t* __restrict__ cols,
                                         const T* __restrict__ vals,
                                         const V* __restrict__ v, int r0, int r1,
                                         F&& f) {
  const int group = int(threadIdx.x) / W, lane = int(threadIdx.x) % W;
  for (int base = r0; base < r1; base += BBS / W) {
    const int row = base + group;
    T sum = T(0);
    if (row < r1) {
      const int s = rp[row], e = rp[row + 1];
      for (int j = s + lane; j < e; j += W) sum += vals[j] * T(v[cols[j]]);
    }
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o, W);
    if (lane == 0 && row < r1) f(row, sum);
  }
}

template <int CL, int W>
__global__ void __launch_bounds__(BBS) batch_cg_kernel(const __grid_constant__ BatchArgs a) {
  __shared__ double smem[40];
  __shared__ double slot[8];
  __shared__ int s_sys;
  const unsigned int crank = CL == 1 ? 0u : cgx::this_cluster().block_rank();

  for (;;) {
    // Pop the next system (rank 0 of the cluster), share it.
    if (crank == 0 && threadIdx.x == 0) {
      const unsigned int t = atomicAdd(a.counter, 1u);
      s_sys = t < unsigned(a.nsys) ? a.order[t] : -1;
    }
    cluster_barrier<CL>();
    int sys;
    if (CL == 1) {
      sys = s_sys;
    } else {
      sys = *cgx::this_cluster().map_shared_rank(&s_sys, 0);
    }
    cluster_barrier<CL>();  // s_sys may be overwritten only after all read it
    if (sys < 0) return;

    const int n = a.n[sys];
    const int64_t ro = a.row_off[sys], zo = a.nz_off[sys];
    const int32_t* rp = a.rowptr + a.rp_off[sys];
    const int32_t* cols = a.cols + zo;
    const double* v64 = a.vals64 + zo;
    const float* v32 = a.vals32 + zo;
    const double* b = a.b + ro;
    double* x = a.x + ro;
    float* r = a.r + ro;
    float* p = a.p + ro;
    float* y = a.y + ro;
    float* d = a.d + ro;
    const int r0 = int(int64_t(n) * crank / CL), r1 = int(int64_t(n) * (crank + 1) / CL);

    // Init: x = 0, d = 0, r = p = fl32(b); ||b||^2, r.r.
    double s2[2] = {0.0, 0.0};
    for (int i = r0 + threadIdx.x; i < r1; i += BBS) {
      const double bi = b[i];
      const float ri = float(bi);
      x[i] = 0.0;
      d[i] = 0.0f;
      r[i] = ri;
      p[i] = ri;
      s2[0] += bi * bi;
      s2[1] += double(ri) * double(ri);
    }
    cluster_sums<CL, 2>(s2, slot, smem);
    const double rr0 = s2[0];
    double rr = s2[1], rr_max = s2[1], rr_true = rr0;
    int k = 0, refinements = 0, status = SPMV_SUCCESS, converged = rr0 == 0.0;
    bool go = a.kmax > 0 && rr0 > 0.0 && isfinite(rr0);

    while (go) {
      // A: y = A32 p, p.y.
      double s1[1] = {0.0};
      sys_rows<float, float, W>(rp, cols, v32, p, r0, r1, [&](int row, float sum) {
        y[row] = sum;
        s1[0] += double(p[row]) * double(sum);
      });
      cluster_sums<CL, 1>(s1, slot, smem);
      const double pap = s1[0];
      if (pap == 0.0 || !isfinite(pap)) {
        status = SPMV_ERROR_BREAKDOWN;
        break;
      }
      const double alpha = rr / pap;
      // B: d += alpha p, r -= alpha y, r.r.
      const float af = float(alpha);
      s1[0] = 0.0;
      for (int i = r0 + threadIdx.x; i < r1; i += BBS) {
        d[i] = d[i] + af * p[i];
        const float ri = r[i] - af * y[i];
        r[i] = ri;
        s1[0] += double(ri) * double(ri);
      }
      cluster_sums<CL, 1>(s1, slot, smem);
      const double rr_new = s1[0];
      ++k;
      rr_max = fmax(rr_max, rr_new);
      const bool refine = rr_new < a.delta2 * rr_max || rr_new / rr0 < a.rtol2 ||
                          k >= a.kmax || !isfinite(rr_new);
      double beta = rr_new / rr, c = 0.0;
      const double rr_prev = rr;
      rr = rr_new;
      if (refine) {
        // C: fold the correction, true residual in FP64, resync r.
        for (int i = r0 + threadIdx.x; i < r1; i += BBS) {
          x[i] = x[i] + double(d[i]);
          d[i] = 0.0f;
        }
        cluster_barrier<CL>();
        double s3[3] = {0.0, 0.0, 0.0};  // ||r64||^2, r32.r32, r32.p
        sys_rows<double, double, W>(rp, cols, v64, x, r0, r1, [&](int row, double sum) {
          const double ri = b[row] - sum;
          const float rf = float(ri);
          r[row] = rf;
          s3[0] += ri * ri;
          s3[1] += double(rf) * double(rf);
          s3[2] += double(rf) * double(p[row]);
        });
        cluster_sums<CL, 3>(s3, slot, smem);
        ++refinements;
        rr_true = s3[0];
        rr_max = s3[1];
        if (rr_true / rr0 < a.rtol2) converged = 1;
        if (!isfinite(rr_true)) status = SPMV_ERROR_BREAKDOWN;
        beta = s3[1] / rr_prev;
        rr = s3[1];
        c = s3[1] > 0.0 ? s3[2] / s3[1] : 0.0;
      }
      if (converged || status != SPMV_SUCCESS || k >= a.kmax) break;
      // D: p = r + beta (p - c r).
      const float bf = float(beta), cf = float(c);
      for (int i = r0 + threadIdx.x; i < r1; i += BBS) {
        const float ri = r[i];
        p[i] = ri + bf * (p[i] - cf * ri);
      }
      cluster_barrier<CL>();
    }
    if (crank == 0 && threadIdx.x == 0) {
      BatchResult& R = a.res[sys];
      R.iterations = k;
      R.refinements = refinements;
      R.status = status;
      R.converged = converged;
      R.relres = rr0 > 0.0 ? sqrt(rr_true / rr0) : 0.0;
    }
    cluster_barrier<CL>();
  }
}

template <int CL>
void launch_batch(const BatchArgs& args, int W, int clusters, cudaStream_t s) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(clusters * CL);
  cfg.blockDim = dim3(BBS);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = CL;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  switch (W) {
    case 4: SPMVB_CUDA(cudaLaunchKernelEx(&cfg, batch_cg_kernel<CL, 4>, args)); break;
    case 8: SPMVB_CUDA(cudaLaunchKernelEx(&cfg, batch_cg_kernel<CL, 8>, args)); break;
    case 16: SPMVB_CUDA(cudaLaunchKernelEx(&cfg, batch_cg_kernel<CL, 16>, args)); break;
    default: SPMVB_CUDA(cudaLaunchKernelEx(&cfg, batch_cg_kernel<CL, 32>, args)); break;
  }
}

}  // namespace

void batch_solve(spmv_batch B, const double* d_b, double* d_x, int max_its, double rtol,
                 spmv_batch_info* info) {
  spmv_comm comm = B->comm;
  cudaStream_t s = comm->stream;
  const int64_t rows = std::max<int64_t>(B->rows, 1);
  B->r.reserve(4 * rows);
  B->p.reserve(4 * rows);
  B->y.reserve(4 * rows);
  B->d.reserve(4 * rows);
  B->counter.reserve(sizeof(unsigned int));
  B->results.reserve(sizeof(BatchResult) * std::max(B->nsys, 1));
  SPMVB_CUDA(cudaMemsetAsync(B->counter.ptr, 0, sizeof(unsigned int), s));
  BatchArgs a;
  a.n = B->d_n.as<int32_t>();
  a.row_off = B->d_row_off.as<int64_t>();
  a.nz_off = B->d_nz_off.as<int64_t>();
  a.rp_off = B->d_rp_off.as<int64_t>();
  a.order = B->d_order.as<int32_t>();
  a.rowptr = B->rowptr.as<int32_t>();
  a.cols = B->cols.as<int32_t>();
  a.vals64 = B->vals64.as<double>();
  a.vals32 = B->vals32.as<float>();
  a.b = d_b;
  a.x = d_x;
  a.r = B->r.as<float>();
  a.p = B->p.as<float>();
  a.y = B->y.as<float>();
  a.d = B->d.as<float>();
  a.counter = B->counter.as<unsigned int>();
  a.res = B->results.as<BatchResult>();
  a.nsys = B->nsys;
  a.kmax = max_its;
  a.rtol2 = rtol * rtol;
  a.delta2 = 0.01;
  // Lanes per row from the mean row length (FP32 values).
  int W = 4;
  while (W < 32 && W < B->mean_row) W <<= 1;
  const int CL = B->cluster;
  // Persistent grid: as many clusters as fit at once (two CTAs per SM).
  const int clusters = std::max(1, (comm->num_sms * 2) / CL);
  switch (CL) {
    case 1: launch_batch<1>(a, W, clusters, s); break;
    case 2: launch_batch<2>(a, W, clusters, s); break;
    case 4: launch_batch<4>(a, W, clusters, s); break;
    case 8: launch_batch<8>(a, W, clusters, s); break;
    default: fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: batch cluster size must be 1, 2, 4 or 8");
  }
  std::vector<BatchResult> res(B->nsys);
  if (B->nsys > 0)
    SPMVB_CUDA(cudaMemcpyAsync(res.data(), B->results.ptr, sizeof(BatchResult) * B->nsys,
                               cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
  if (info)
    for (int i = 0; i < B->nsys; ++i) {
      info[i].iterations = res[i].iterations;
      info[i].refinements = res[i].refinements;
      info[i].status = res[i].status;
      info[i].converged = res[i].converged;
      info[i].relres = res[i].relres;
    }
}

}  // namespace spmvb

using namespace spmvb;

extern "C" {

int spmv_batch_create(spmv_comm comm, int nsys, const int32_t* n,
                      const int32_t* const* rowptr, const int32_t* const* colind,
                      const double* const* values, spmv_batch* out) {
  return guard([&] {
    require(comm != nullptr && out != nullptr, "spmv: NULL argument");
    *out = nullptr;
    require(nsys >= 0, "spmv: negative system count");
    require(nsys == 0 || (n && rowptr && colind && values), "spmv: NULL CSR array");
    comm->require_device();
    std::unique_ptr<spmv_batch_s> B(new spmv_batch_s);
    B->comm = comm;
    B->nsys = nsys;
    B->n.assign(n, n + nsys);
    std::vector<int32_t> rp_all;
    std::vector<int32_t> ci_all;
    std::vector<double> v64;
    std::vector<float> v32;
    for (int s = 0; s < nsys; ++s) {
      const int32_t m = n[s];
      require(m >= 0, "spmv: negative system size");
      require(rowptr[s] && rowptr[s][0] == 0, "spmv: row pointers must start at 0");
      for (int32_t i = 0; i < m; ++i)
        require(rowptr[s][i + 1] >= rowptr[s][i], "spmv: row pointers must be non-decreasing");
      const int64_t nz = rowptr[s][m];
      require(nz == 0 || (colind[s] && values[s]), "spmv: NULL column or value array");
      for (int64_t j = 0; j < nz; ++j)
        require(colind[s][j] >= 0 && colind[s][j] < m, "spmv: column index out of range");
      B->row_off.push_back(B->rows);
      B->nz_off.push_back(int64_t(ci_all.size()));
      B->rp_off.push_back(int64_t(rp_all.size()));
      rp_all.insert(rp_all.end(), rowptr[s], rowptr[s] + m + 1);
      ci_all.insert(ci_all.end(), colind[s], colind[s] + nz);
      v64.insert(v64.end(), values[s], values[s] + nz);
      B->rows += m;
    }
    B->nnz = int64_t(ci_all.size());
    B->mean_row = B->rows > 0 ? double(B->nnz) / double(B->rows) : 0.0;
    v32.assign(v64.begin(), v64.end());
    // Visit order: most nonzeros first.
    std::vector<int32_t> order(nsys);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const int64_t na = rowptr[a][n[a]], nb = rowptr[b][n[b]];
      return na > nb;
    });
    DeviceGuard dg(comm->device);
    auto up = [](DevBuf& buf, const void* src, size_t bytes) {
      buf.reserve(std::max<size_t>(bytes, 16));
      if (bytes) SPMVB_CUDA(cudaMemcpy(buf.ptr, src, bytes, cudaMemcpyHostToDevice));
    };
    up(B->d_n, B->n.data(), sizeof(int32_t) * nsys);
    up(B->d_row_off, B->row_off.data(), sizeof(int64_t) * nsys);
    up(B->d_nz_off, B->nz_off.data(), sizeof(int64_t) * nsys);
    up(B->d_rp_off, B->rp_off.data(), sizeof(int64_t) * nsys);
    up(B->d_order, order.data(), sizeof(int32_t) * nsys);
    up(B->rowptr, rp_all.data(), sizeof(int32_t) * rp_all.size());
    up(B->cols, ci_all.data(), sizeof(int32_t) * ci_all.size());
    up(B->vals64, v64.data(), sizeof(double) * v64.size());
    up(B->vals32, v32.data(), sizeof(float) * v32.size());
    B->b.reserve(sizeof(double) * std::max<int64_t>(B->rows, 1));
    B->x.reserve(sizeof(double) * std::max<int64_t>(B->rows, 1));
    ++comm->refs;
    *out = B.release();
  });
}

int spmv_batch_destroy(spmv_batch B) {
  return guard([&] {
    if (!B) return;
    spmv_comm comm = B->comm;
    {
      DeviceGuard dg(comm->device);
      delete B;
    }
    release_comm(comm);
  });
}

int spmv_batch_set_cluster(spmv_batch B, int cluster) {
  return guard([&] {
    require(B != nullptr, "spmv: NULL batch");
    require(cluster == 1 || cluster == 2 || cluster == 4 || cluster == 8,
            "spmv: batch cluster size must be 1, 2, 4 or 8");
    B->cluster = cluster;
  });
}

int spmv_batch_solve(spmv_batch B, spmv_memory memory, const double* const* b,
                     double* const* x, int max_its, double rtol,
                     spmv_batch_info* info) {
  return guard([&] {
    require(B != nullptr, "spmv: NULL batch");
    require(b != nullptr && x != nullptr, "spmv: NULL vector array");
    require(memory == SPMV_MEMORY_HOST || memory == SPMV_MEMORY_DEVICE,
            "spmv: unknown memory kind");
    spmv_comm comm = B->comm;
    DeviceGuard dg(comm->device);
    cudaStream_t s = comm->stream;
    const cudaMemcpyKind in = memory == SPMV_MEMORY_HOST ? cudaMemcpyHostToDevice
                                                         : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind outk = memory == SPMV_MEMORY_HOST ? cudaMemcpyDeviceToHost
                                                           : cudaMemcpyDeviceToDevice;
    for (int i = 0; i < B->nsys; ++i) {
      if (B->n[i] == 0) continue;
      require(b[i] != nullptr && x[i] != nullptr, "spmv: NULL vector");
      SPMVB_CUDA(cudaMemcpyAsync(B->b.as<double>() + B->row_off[i], b[i],
                                 sizeof(double) * B->n[i], in, s));
    }
    batch_solve(B, B->b.as<double>(), B->x.as<double>(), max_its, rtol, info);
    for (int i = 0; i < B->nsys; ++i)
      if (B->n[i] > 0)
        SPMVB_CUDA(cudaMemcpyAsync(x[i], B->x.as<double>() + B->row_off[i],
                                   sizeof(double) * B->n[i], outk, s));
    SPMVB_CUDA(cudaStreamSynchronize(s));
    if (info)
      for (int i = 0; i < B->nsys; ++i)
        if (info[i].status == SPMV_ERROR_BREAKDOWN)
          fail(SPMV_ERROR_BREAKDOWN, "spmv batch: breakdown in system " + std::to_string(i));
  });
}

}  // extern "C"
