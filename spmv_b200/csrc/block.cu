// Multi-right-hand-side product and block CG (no counterpart in the
// reference; builds on Matrix::operator* and spmv::cg, cg.cpp:11-83).
//
// Vectors of k right-hand sides are stored row-major (n x k, leading
// dimension k), so the k values of one row are contiguous.  The SpMM gives a
// row a group of K lanes (K = k rounded up to a power of two, at most 32):
// every lane reads the row's column indices and values (the same addresses,
// one broadcast transaction) and lane l accumulates right-hand side l from a
// contiguous run of X.  A is read once for all k right-hand sides.
//
// Block CG runs k independent CG recurrences that share each product: the
// SpMM's epilogue forms the k dot products p_l . (A p)_l, and every column has
// its own alpha, beta, convergence test (cg.cpp:78) and breakdown flag; a
// converged column stops changing.  The loop ends when every column has
// converged or broken down, or after max_its iterations, as one CUDA graph
// with a device-side while loop (same structure as cg.cu).
#include <algorithm>
#include <cmath>

#include "internal.h"
#include "spmv_kernel.cuh"

namespace spmvb {

namespace {

constexpr int BBS = 256;
constexpr int MAXK = 32;

// Rows of one launch: group of K lanes per row, lane = right-hand side.
template <typename T, int K, class F>
__device__ __forceinline__ void spmm_rows(const SpmvArgs& a, int k, F&& f) {
  const int p = find_part(a, blockIdx.x);
  const PartArg& P = a.part[p];
  const int32_t* __restrict__ cols = P.cols;
  const T* __restrict__ vals = static_cast<const T*>(P.vals);
  const T* __restrict__ x = static_cast<const T*>(P.x);
  const int group = int(threadIdx.x) / K, lane = int(threadIdx.x) % K;
  const bool on = lane < k;
  for (int tile = int(blockIdx.x) - P.block_begin; tile < P.ntiles; tile += P.nblocks) {
    const int row = tile * (BBS / K) + group;
    if (row >= P.nrows) continue;
    const int s = __ldg(P.rowptr + row), e = __ldg(P.rowptr + row + 1);
    T acc = T(0);
    int j = s;
    for (; j + 4 <= e; j += 4) {
      int c[4];
      T v[4], xv[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        c[u] = __ldg(cols + j + u);
        v[u] = __ldg(vals + j + u);
      }
#pragma unroll
      for (int u = 0; u < 4; ++u) xv[u] = on ? __ldg(x + int64_t(c[u]) * k + lane) : T(0);
#pragma unroll
      for (int u = 0; u < 4; ++u) acc += v[u] * xv[u];
    }
    for (; j < e; ++j) {
      const int c = __ldg(cols + j);
      const T v = __ldg(vals + j);
      if (on) acc += v * __ldg(x + int64_t(c) * k + lane);
    }
    if (on) f(P, row, lane, acc);
  }
}

template <typename T, int K>
__global__ void __launch_bounds__(BBS)
    spmm_kernel(const __grid_constant__ SpmvArgs a, int k) {
  spmm_rows<T, K>(a, k, [&](const PartArg& P, int row, int lane, T acc) {
    static_cast<T*>(P.y)[int64_t(row) * k + lane] = acc;
  });
}

// ---------------------------------------------------------------------------
// Block CG state and kernels
// ---------------------------------------------------------------------------
struct BcgState {
  double rr0[MAXK], rr[MAXK], pap[MAXK], alpha[MAXK], beta[MAXK];
  int active[MAXK], status[MAXK], its[MAXK];
  int k, kmax, nrhs, pad;
  double rtol2;
  unsigned int t0, t1, t2, pad2;
};

struct BcgPtrs {
  const double* b;
  double* x;
  double* r;
  double* p;
  double* y;
  double* partials;  // [CTAs][MAXK]
  BcgState* st;
  int64_t n;
  int nrhs;
};

// Per-column sums: thread t contributes v to column col (-1: nothing).  The
// CTA's column sums go to partials[blockIdx.x][col] (threads in index order);
// the last CTA to arrive sums each column's partials in CTA order.
__device__ bool column_sums(double v, int col, const BcgPtrs& c, unsigned int* ticket,
                            double* out /*[MAXK]*/) {
  __shared__ double s[BBS];
  __shared__ int sc[BBS];
  __shared__ bool last;
  s[threadIdx.x] = v;
  sc[threadIdx.x] = col;
  __syncthreads();
  if (threadIdx.x < MAXK) {
    double t = 0.0;
    if (int(threadIdx.x) < c.nrhs)
      for (int i = 0; i < BBS; ++i)
        if (sc[i] == int(threadIdx.x)) t += s[i];
    c.partials[blockIdx.x * MAXK + threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    last = atomicAdd(ticket, 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (!last) return false;
  __threadfence();
  if (threadIdx.x < MAXK) {
    double t = 0.0;
    for (unsigned int b = 0; b < gridDim.x; ++b) t += __ldcg(c.partials + b * MAXK + threadIdx.x);
    out[threadIdx.x] = t;
  }
  __syncthreads();
  if (threadIdx.x == 0) *ticket = 0u;
  return true;
}

#define BCG_LOOP(i) \
  for (int64_t i = blockIdx.x * int64_t(BBS) + threadIdx.x; i < c.n * c.nrhs; i += int64_t(gridDim.x) * BBS)

// The elementwise kernels give thread t the entries t, t + G, ... with G a
// multiple of nrhs (the grid stride), so a thread always sees the same
// right-hand side col = t % nrhs.
__global__ void __launch_bounds__(BBS) bcg_init(const BcgPtrs c, cudaGraphConditionalHandle h) {
  __shared__ double tot[MAXK];
  const int col = int((blockIdx.x * int64_t(BBS) + threadIdx.x) % c.nrhs);
  double acc = 0.0;
  BCG_LOOP(i) {
    const double bi = c.b[i];
    c.r[i] = bi;
    c.p[i] = bi;
    c.x[i] = 0.0;
    acc += bi * bi;
  }
  if (column_sums(acc, col, c, &c.st->t0, tot) && threadIdx.x == 0) {
    BcgState* st = c.st;
    int any = 0;
    for (int l = 0; l < c.nrhs; ++l) {
      st->rr0[l] = tot[l];
      st->rr[l] = tot[l];
      st->active[l] = tot[l] > 0.0 && isfinite(tot[l]);
      st->status[l] = SPMV_SUCCESS;
      st->its[l] = 0;
      any |= st->active[l];
    }
    st->k = 0;
    cudaGraphSetConditional(h, (any && st->kmax > 0) ? 1u : 0u);
  }
}

template <int K>
__global__ void __launch_bounds__(BBS)
    bcg_spmm_dot(const __grid_constant__ SpmvArgs a, const BcgPtrs c,
                 cudaGraphConditionalHandle h) {
  __shared__ double tot[MAXK];
  if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
  double acc = 0.0;
  // K lanes per row and BBS % K == 0, so this thread's lane (= column) is
  // fixed: threadIdx.x % K.
  spmm_rows<double, K>(a, c.nrhs, [&](const PartArg& P, int row, int lane, double v) {
    static_cast<double*>(P.y)[int64_t(row) * c.nrhs + lane] = v;
    acc += static_cast<const double*>(P.xown)[int64_t(row) * c.nrhs + lane] * v;
  });
  const int lane = int(threadIdx.x) % K;
  if (column_sums(acc, lane < c.nrhs ? lane : -1, c, &c.st->t1, tot) && threadIdx.x == 0) {
    BcgState* st = c.st;
    for (int l = 0; l < c.nrhs; ++l) {
      st->pap[l] = tot[l];
      if (!st->active[l]) {
        st->alpha[l] = 0.0;
        continue;
      }
      if (tot[l] == 0.0 || !isfinite(tot[l])) {
        st->status[l] = SPMV_ERROR_BREAKDOWN;
        st->active[l] = 0;
        st->alpha[l] = 0.0;
      } else {
        st->alpha[l] = st->rr[l] / tot[l];
      }
    }
  }
}

__global__ void __launch_bounds__(BBS)
    bcg_update_xr(const BcgPtrs c, cudaGraphConditionalHandle h) {
  __shared__ double tot[MAXK];
  const int col = int((blockIdx.x * int64_t(BBS) + threadIdx.x) % c.nrhs);
  const BcgState* st = c.st;
  const bool act = st->active[col];
  const double alpha = st->alpha[col];
  double acc = 0.0;
  if (act) {
    BCG_LOOP(i) {
      c.x[i] = c.x[i] + alpha * c.p[i];
      const double ri = c.r[i] - alpha * c.y[i];
      c.r[i] = ri;
      acc += ri * ri;
    }
  }
  if (column_sums(acc, col, c, &c.st->t2, tot) && threadIdx.x == 0) {
    BcgState* s = c.st;
    s->k += 1;
    int any = 0;
    for (int l = 0; l < c.nrhs; ++l) {
      if (!s->active[l]) {
        s->beta[l] = 0.0;
        continue;
      }
      s->its[l] = s->k;
      s->beta[l] = tot[l] / s->rr[l];
      s->rr[l] = tot[l];
      if (tot[l] / s->rr0[l] < s->rtol2) s->active[l] = 0;
      any |= s->active[l];
    }
    cudaGraphSetConditional(h, (any && s->k < s->kmax) ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(BBS) bcg_update_p(const BcgPtrs c) {
  const int col = int((blockIdx.x * int64_t(BBS) + threadIdx.x) % c.nrhs);
  // A column that converged in this iteration still had its beta set; one
  // that was already inactive has beta 0 and p = r is harmless (unused).
  const double beta = c.st->beta[col];
  BCG_LOOP(i) c.p[i] = c.r[i] + beta * c.p[i];
}

}  // namespace

// y[r] (nrows x k) = A[r] x[r] (ncols x k) for all ranks, device pointers.
void launch_spmm(spmv_matrix A, int k, const void* const* x, void* const* y,
                 cudaStream_t stream) {
  require(k >= 1 && k <= MAXK, "spmv: block products take 1..32 right-hand sides");
  require(A->dtype == SPMV_FLOAT64 || A->dtype == SPMV_FLOAT32,
          "spmv: only float64 and float32 products are implemented");
  int K = 1;
  while (K < k) K <<= 1;
  SpmvArgs a;
  fill_spmv_args(a, A->fwd, A->fwd.cols.as<int32_t>(), dtype_size(A->dtype), x, y,
                 nullptr, BBS / K, max_blocks_for(A->comm->num_sms, BBS));
  if (a.nblocks == 0) return;
#define SPMVB_SPMM(T)                                                             \
  switch (K) {                                                                    \
    case 1: spmm_kernel<T, 1><<<a.nblocks, BBS, 0, stream>>>(a, k); break;        \
    case 2: spmm_kernel<T, 2><<<a.nblocks, BBS, 0, stream>>>(a, k); break;        \
    case 4: spmm_kernel<T, 4><<<a.nblocks, BBS, 0, stream>>>(a, k); break;        \
    case 8: spmm_kernel<T, 8><<<a.nblocks, BBS, 0, stream>>>(a, k); break;        \
    case 16: spmm_kernel<T, 16><<<a.nblocks, BBS, 0, stream>>>(a, k); break;      \
    default: spmm_kernel<T, 32><<<a.nblocks, BBS, 0, stream>>>(a, k); break;      \
  }
  if (A->dtype == SPMV_FLOAT64) {
    SPMVB_SPMM(double)
  } else {
    SPMVB_SPMM(float)
  }
#undef SPMVB_SPMM
  SPMVB_CUDA(cudaGetLastError());
}

// Block CG in the fused-halo layout over row-major n x k blocks; d_b, d_x
// are global-layout device blocks.
void block_cg(spmv_matrix A, int k, const double* d_b, double* d_x, int max_its,
              double rtol, spmv_cg_info* info) {
  require(k >= 1 && k <= MAXK, "spmv: block CG takes 1..32 right-hand sides");
  spmv_comm comm = A->comm;
  build_global_cols(A);
  const int64_t n = A->row_map->ranges.back();
  const int P = comm->size;
  DevBuf r, p, y, partials, state;
  const size_t bytes = sizeof(double) * std::max<int64_t>(n * k, 1);
  r.reserve(bytes);
  p.reserve(bytes);
  y.reserve(bytes);
  state.reserve(sizeof(BcgState));
  SPMVB_CUDA(cudaMemset(state.ptr, 0, sizeof(BcgState)));
  int K = 1;
  while (K < k) K <<= 1;
  std::vector<const void*> xs(P), own(P);
  std::vector<void*> ys(P);
  for (int q = 0; q < P; ++q) {
    const int64_t off = A->row_map->ranges[q] * k;
    xs[q] = p.as<double>();
    own[q] = p.as<double>() + off;
    ys[q] = y.as<double>() + off;
  }
  SpmvArgs a;
  fill_spmv_args(a, A->fwd, A->fwd.cols_global.as<int32_t>(), sizeof(double), xs.data(),
                 ys.data(), own.data(), BBS / K, max_blocks_for(comm->num_sms, BBS));
  // Elementwise grid: a multiple of k threads so each thread keeps one column.
  const int ew_threads = BBS;
  int ew_grid = std::max(1, comm->num_sms) * (2048 / BBS);
  while ((int64_t(ew_grid) * ew_threads) % k) ++ew_grid;
  partials.reserve(sizeof(double) * MAXK * std::max(a.nblocks, ew_grid));
  BcgPtrs c;
  c.b = d_b;
  c.x = d_x;
  c.r = r.as<double>();
  c.p = p.as<double>();
  c.y = y.as<double>();
  c.partials = partials.as<double>();
  c.st = state.as<BcgState>();
  c.n = n;
  c.nrhs = k;
  BcgState host{};
  host.kmax = max_its;
  host.nrhs = k;
  host.rtol2 = rtol * rtol;
  cudaStream_t s = comm->stream;
  SPMVB_CUDA(cudaMemcpyAsync(&c.st->k, &host.k, sizeof(int) * 4, cudaMemcpyHostToDevice, s));
  SPMVB_CUDA(cudaMemcpyAsync(&c.st->rtol2, &host.rtol2, sizeof(double),
                             cudaMemcpyHostToDevice, s));

  using K1 = void (*)(SpmvArgs, BcgPtrs, cudaGraphConditionalHandle);
  K1 k1;
  switch (K) {
    case 1: k1 = bcg_spmm_dot<1>; break;
    case 2: k1 = bcg_spmm_dot<2>; break;
    case 4: k1 = bcg_spmm_dot<4>; break;
    case 8: k1 = bcg_spmm_dot<8>; break;
    case 16: k1 = bcg_spmm_dot<16>; break;
    default: k1 = bcg_spmm_dot<32>; break;
  }
  cudaGraph_t g = nullptr;
  cudaGraphExec_t ge = nullptr;
  cudaGraphConditionalHandle h;
  SPMVB_CUDA(cudaGraphCreate(&g, 0));
  try {
    SPMVB_CUDA(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    auto add = [&](cudaGraphNode_t* node, cudaGraph_t gg, const cudaGraphNode_t* dep,
                   size_t nd, void* fn, int grid, void** args) {
      cudaKernelNodeParams kp{};
      kp.func = fn;
      kp.gridDim = dim3(grid);
      kp.blockDim = dim3(BBS);
      kp.kernelParams = args;
      SPMVB_CUDA(cudaGraphAddKernelNode(node, gg, dep, nd, &kp));
    };
    cudaGraphNode_t n0, nl, b1, b2, b3;
    void* a0[] = {&c, &h};
    add(&n0, g, nullptr, 0, (void*)bcg_init, ew_grid, a0);
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    SPMVB_CUDA(cudaGraphAddNode(&nl, g, &n0, 1, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    void* a1[] = {&a, &c, &h};
    add(&b1, body, nullptr, 0, (void*)k1, a.nblocks, a1);
    void* a2[] = {&c, &h};
    add(&b2, body, &b1, 1, (void*)bcg_update_xr, ew_grid, a2);
    void* a3[] = {&c};
    add(&b3, body, &b2, 1, (void*)bcg_update_p, ew_grid, a3);
    SPMVB_CUDA(cudaGraphInstantiate(&ge, g, 0));
    SPMVB_CUDA(cudaGraphLaunch(ge, s));
    SPMVB_CUDA(cudaMemcpyAsync(&host, c.st, sizeof(BcgState), cudaMemcpyDeviceToHost, s));
    SPMVB_CUDA(cudaStreamSynchronize(s));
  } catch (...) {
    if (ge) cudaGraphExecDestroy(ge);
    cudaGraphDestroy(g);
    throw;
  }
  soft_check(cudaGraphExecDestroy(ge), "cudaGraphExecDestroy");
  soft_check(cudaGraphDestroy(g), "cudaGraphDestroy");
  if (info)
    for (int l = 0; l < k; ++l) {
      info[l].iterations = host.its[l];
      info[l].status = host.status[l];
      info[l].rnorm0 = host.rr0[l];
      info[l].rnorm = host.rr[l];
    }
}

}  // namespace spmvb

using namespace spmvb;

extern "C" {

int spmv_matrix_mult_block(spmv_matrix A, int nrhs, spmv_memory memory,
                           const void* const* x, void* const* y) {
  return guard([&] {
    require(A != nullptr, "spmv: Matrix is NULL");
    require(x != nullptr && y != nullptr, "spmv: vector array is NULL");
    require(nrhs >= 1 && nrhs <= MAXK, "spmv: block products take 1..32 right-hand sides");
    spmv_comm comm = A->comm;
    comm->require_device();
    DeviceGuard dg(comm->device);
    cudaStream_t s = comm->stream;
    if (memory == SPMV_MEMORY_DEVICE) {
      launch_spmm(A, nrhs, x, y, s);
      return;
    }
    require(memory == SPMV_MEMORY_HOST, "spmv: unknown memory kind");
    const int P = comm->size;
    const size_t es = dtype_size(A->dtype);
    std::vector<int64_t> xo(P), yo(P);
    int64_t xt = 0, yt = 0;
    for (int r = 0; r < P; ++r) {
      xo[r] = xt;
      yo[r] = yt;
      xt += (int64_t(A->ncols[r]) * nrhs * es + 255) / 256 * 256;
      yt += (int64_t(A->nrows[r]) * nrhs * es + 255) / 256 * 256;
    }
    comm->stage_in.reserve(std::max<int64_t>(xt, 256));
    comm->stage_out.reserve(std::max<int64_t>(yt, 256));
    std::vector<const void*> dx(P);
    std::vector<void*> dy(P);
    for (int r = 0; r < P; ++r) {
      dx[r] = comm->stage_in.as<char>() + xo[r];
      dy[r] = comm->stage_out.as<char>() + yo[r];
      const size_t bytes = size_t(A->ncols[r]) * nrhs * es;
      if (bytes)
        SPMVB_CUDA(cudaMemcpyAsync(const_cast<void*>(dx[r]), x[r], bytes,
                                   cudaMemcpyHostToDevice, s));
    }
    launch_spmm(A, nrhs, dx.data(), dy.data(), s);
    for (int r = 0; r < P; ++r) {
      const size_t bytes = size_t(A->nrows[r]) * nrhs * es;
      if (bytes) SPMVB_CUDA(cudaMemcpyAsync(y[r], dy[r], bytes, cudaMemcpyDeviceToHost, s));
    }
    SPMVB_CUDA(cudaStreamSynchronize(s));
  });
}

int spmv_cg_block(spmv_matrix A, int nrhs, spmv_memory memory, const double* const* b,
                  double* const* x, int max_its, double rtol, spmv_cg_info* info) {
  return guard([&] {
    require(nrhs >= 1 && nrhs <= MAXK, "spmv: block CG takes 1..32 right-hand sides");
    check_solve_args(A, memory, b, nullptr, x);
    spmv_comm comm = A->comm;
    DeviceGuard dg(comm->device);
    cudaStream_t s = comm->stream;
    spmv_l2gmap rm = A->row_map, cm = A->col_map;
    const int P = comm->size;
    const int64_t n = rm->ranges.back();
    DevBuf db, dxb;
    db.reserve(sizeof(double) * std::max<int64_t>(n * nrhs, 1));
    dxb.reserve(sizeof(double) * std::max<int64_t>(n * nrhs, 1));
    const cudaMemcpyKind in = memory == SPMV_MEMORY_HOST ? cudaMemcpyHostToDevice
                                                         : cudaMemcpyDeviceToDevice;
    const cudaMemcpyKind outk = memory == SPMV_MEMORY_HOST ? cudaMemcpyDeviceToHost
                                                           : cudaMemcpyDeviceToDevice;
    for (int r = 0; r < P; ++r) {
      const int64_t M = rm->rank[r].local_size;
      if (M == 0) continue;
      require(b[r] != nullptr, "spmv::cg - Error: b is NULL");
      SPMVB_CUDA(cudaMemcpyAsync(db.as<double>() + rm->ranges[r] * nrhs, b[r],
                                 sizeof(double) * M * nrhs, in, s));
    }
    std::vector<spmv_cg_info> local(nrhs);
    block_cg(A, nrhs, db.as<double>(), dxb.as<double>(), max_its, rtol, local.data());
    for (int r = 0; r < P; ++r) {
      const int64_t M = rm->rank[r].local_size;
      const int64_t G = int64_t(cm->rank[r].ghosts.size());
      if (M + G == 0) continue;
      require(x[r] != nullptr, "spmv::cg - Error: x is NULL");
      if (M > 0)
        SPMVB_CUDA(cudaMemcpyAsync(x[r], dxb.as<double>() + rm->ranges[r] * nrhs,
                                   sizeof(double) * M * nrhs, outk, s));
      if (G > 0) {
        if (memory == SPMV_MEMORY_HOST)
          std::fill(x[r] + M * nrhs, x[r] + (M + G) * nrhs, 0.0);
        else
          SPMVB_CUDA(cudaMemsetAsync(x[r] + M * nrhs, 0, sizeof(double) * G * nrhs, s));
      }
    }
    SPMVB_CUDA(cudaStreamSynchronize(s));
    if (info) std::copy(local.begin(), local.end(), info);
    for (int l = 0; l < nrhs; ++l)
      if (local[l].status == SPMV_ERROR_BREAKDOWN)
        fail(SPMV_ERROR_BREAKDOWN, "spmv::cg - Error: breakdown in right-hand side " +
                                       std::to_string(l));
  });
}

}  // extern "C"
