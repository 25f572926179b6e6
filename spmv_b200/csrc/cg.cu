// Conjugate gradients on the device (spmv::cg, cg.cpp:11-83).
//
// The solve runs in the fused-halo layout: all ranks' rows form one global
// vector and the column indices are global, so the product reads the owners'
// entries of p directly instead of first copying them into ghost slots (the
// values read are the ones L2GMap::update would have copied, so the result is
// the same).  One iteration is three kernels:
//
//   K1  y = A p and p.y           (SpMV with a dot-product epilogue; the last
//                                  CTA forms alpha = rnorm_old / p.y)
//   K2  x += alpha p, r -= alpha y, r.r
//                                 (the last CTA forms beta, counts the
//                                  iteration, tests convergence and sets the
//                                  graph's loop condition)
//   K3  p = p beta + r
//
// The three kernels form the body of a CUDA-graph while node; an init kernel
// before it sets r = p = b, x = 0 and rnorm0.  A whole solve is one graph
// launch with no host round trip per iteration.  Reductions are single pass
// (per-CTA partials, the last CTA to arrive sums them in index order), so
// results are reproducible run to run.  Vector updates are compiled without
// FMA contraction (-fmad=false), matching the separate multiply and add of
// the reference's Eigen expressions.
#include <algorithm>
#include <cmath>

#include "internal.h"
#include "spmv_kernel.cuh"

struct CgState {
  double rnorm0, rnorm_old, rnorm_new, alpha, beta, pdoty, rtol2, pad0;
  int k, kmax, status, pad1;
  unsigned int ticket0, ticket1, ticket2, pad2;
};

struct CgWorkspace {
  int64_t n = 0;
  int W = 0, BS = 256;
  bool sell = false;  // K1 over the SELL-32 copy (W = loads per lane)
  bool d16 = false;   // K1 reads 16-bit column offsets
  spmvb::DevBuf b, x, r, p, y, partials, state;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle handle = 0;
  CgState host{};
  ~CgWorkspace() {
    if (exec) spmvb::soft_check(cudaGraphExecDestroy(exec), "cudaGraphExecDestroy");
    if (graph) spmvb::soft_check(cudaGraphDestroy(graph), "cudaGraphDestroy");
  }
};

namespace spmvb {

namespace {

constexpr int EW_BS = 256;  // threads per CTA of the vector kernels

struct CgPtrs {
  const double* b;
  double* x;
  double* r;
  double* p;
  double* y;
  double* partials;
  CgState* st;
  int64_t n;
};

__global__ void __launch_bounds__(EW_BS)
    cg_init(const CgPtrs c, cudaGraphConditionalHandle h) {
  __shared__ double smem[32];
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  for (int64_t i = blockIdx.x * int64_t(EW_BS) + threadIdx.x; i < c.n;
       i += int64_t(gridDim.x) * EW_BS) {
    const double bi = c.b[i];
    st_pol(c.r + i, bi, keep);
    st_pol(c.p + i, bi, keep);
    st_pol(c.x + i, 0.0, keep);
    acc += bi * bi;
  }
  const double part = block_sum<EW_BS>(acc, smem);
  double total;
  if (grid_sum<EW_BS>(part, c.partials, &c.st->ticket0, &total, smem) &&
      threadIdx.x == 0) {
    CgState* st = c.st;
    st->rnorm0 = total;
    st->rnorm_old = total;
    st->rnorm_new = total;
    st->k = 0;
    st->status = SPMV_SUCCESS;
    // b == 0 (or non-finite): nothing to iterate on.
    const bool go = st->kmax > 0 && total > 0.0 && isfinite(total);
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

// K1 epilogue: the grid-wide p.y, alpha and the breakdown test.
template <int BS>
__device__ __forceinline__ void cg_dot_finish(double acc, const CgPtrs& c,
                                              double* smem) {
  const double part = block_sum<BS>(acc, smem);
  double total;
  if (grid_sum<BS>(part, c.partials, &c.st->ticket1, &total, smem) &&
      threadIdx.x == 0) {
    CgState* st = c.st;
    st->pdoty = total;
    if (total == 0.0 || !isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
    st->alpha = st->rnorm_old / total;
  }
}

// K1 over the SELL-32 copy (U loads in flight per lane).
template <int U, int BS, bool D16>
__global__ void __launch_bounds__(BS)
    cg_spmv_dot_sell(const __grid_constant__ SpmvArgs a, const CgPtrs c,
                     cudaGraphConditionalHandle h) {
  __shared__ double smem[32];
  if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  sell_for_rows<double, BS, U, true, D16>(a, [&](const PartArg& P, int row, double sum) {
    st_pol(static_cast<double*>(P.y) + row, sum, keep);
    acc += ld_pol(static_cast<const double*>(P.xown) + row, keep) * sum;
  });
  cg_dot_finish<BS>(acc, c, smem);
}

template <int W, int BS, bool D16>
__global__ void __launch_bounds__(BS)
    cg_spmv_dot(const __grid_constant__ SpmvArgs a, const CgPtrs c,
                cudaGraphConditionalHandle h) {
  __shared__ double smem[32];
  // Default the loop condition to "stop"; K2 sets it to continue.  If K2's
  // last-CTA step ever failed to run, the loop would end, never spin.
  if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
  double acc = 0.0;
  for_rows<double, W, BS, D16>(a, [&](const PartArg& P, int row, double sum) {
    static_cast<double*>(P.y)[row] = sum;
    acc += static_cast<const double*>(P.xown)[row] * sum;
  });
  const double part = block_sum<BS>(acc, smem);
  double total;
  if (grid_sum<BS>(part, c.partials, &c.st->ticket1, &total, smem) &&
      threadIdx.x == 0) {
    CgState* st = c.st;
    st->pdoty = total;
    if (total == 0.0 || !isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
    st->alpha = st->rnorm_old / total;
  }
}

__global__ void __launch_bounds__(EW_BS)
    cg_update_xr(const CgPtrs c, cudaGraphConditionalHandle h) {
  __shared__ double smem[32];
  const bool ok = c.st->status == SPMV_SUCCESS;
  const double alpha = c.st->alpha;
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  if (ok) {
    for (int64_t i = blockIdx.x * int64_t(EW_BS) + threadIdx.x; i < c.n;
         i += int64_t(gridDim.x) * EW_BS) {
      st_pol(c.x + i, ld_pol(c.x + i, keep) + alpha * ld_pol(c.p + i, keep), keep);
      const double ri = ld_pol(c.r + i, keep) - alpha * ld_pol(c.y + i, keep);
      st_pol(c.r + i, ri, keep);
      acc += ri * ri;
    }
  }
  const double part = block_sum<EW_BS>(acc, smem);
  double total;
  if (grid_sum<EW_BS>(part, c.partials, &c.st->ticket2, &total, smem) &&
      threadIdx.x == 0) {
    CgState* st = c.st;
    st->k += 1;
    bool go = false;
    if (st->status == SPMV_SUCCESS) {
      st->rnorm_new = total;
      st->beta = total / st->rnorm_old;
      st->rnorm_old = total;
      const bool converged = total / st->rnorm0 < st->rtol2;
      go = !converged && st->k < st->kmax;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

__global__ void __launch_bounds__(EW_BS) cg_update_p(const CgPtrs c) {
  if (c.st->status != SPMV_SUCCESS) return;
  const double beta = c.st->beta;
  const uint64_t keep = l2_policy_keep();
  for (int64_t i = blockIdx.x * int64_t(EW_BS) + threadIdx.x; i < c.n;
       i += int64_t(gridDim.x) * EW_BS)
    st_pol(c.p + i, ld_pol(c.p + i, keep) * beta + ld_pol(c.r + i, keep), keep);
}

using DotFn = void (*)(SpmvArgs, CgPtrs, cudaGraphConditionalHandle);
template <bool D16>
DotFn dot_kernel(int W) {
  switch (W) {
    case 1: return cg_spmv_dot<1, 256, D16>;
    case 2: return cg_spmv_dot<2, 256, D16>;
    case 4: return cg_spmv_dot<4, 256, D16>;
    case 8: return cg_spmv_dot<8, 256, D16>;
    case 16: return cg_spmv_dot<16, 256, D16>;
    case 32: return cg_spmv_dot<32, 256, D16>;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: width must be 1..32, a power of two");
}

template <bool D16>
DotFn dot_kernel_sell(int U) {
  switch (U) {
    case 1: return cg_spmv_dot_sell<1, 256, D16>;
    case 2: return cg_spmv_dot_sell<2, 256, D16>;
    case 4: return cg_spmv_dot_sell<4, 256, D16>;
    case 8: return cg_spmv_dot_sell<8, 256, D16>;
    case 16: return cg_spmv_dot_sell<16, 256, D16>;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: SELL width must be 1, 2, 4, 8 or 16");
}

void add_kernel(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* dep,
                size_t ndep, void* fn, int grid, int block, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = fn;
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(block);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  kp.extra = nullptr;
  SPMVB_CUDA(cudaGraphAddKernelNode(node, g, dep, ndep, &kp));
}

void build_graph(spmv_matrix A, CgWorkspace& w) {
  spmv_comm comm = A->comm;
  const int P = comm->size;
  const int W = w.W, BS = w.BS;

  // Product over the global layout: every rank reads p (global) and writes
  // its own rows of y.
  std::vector<const void*> xs(P), xown(P);
  std::vector<void*> ys(P);
  const spmv_l2gmap rm = A->row_map;
  for (int r = 0; r < P; ++r) {
    xs[r] = w.p.as<double>();
    xown[r] = w.p.as<double>() + rm->ranges[r];
    ys[r] = w.y.as<double>() + rm->ranges[r];
  }
  SpmvArgs sa;
  if (w.sell)
    fill_sell_args(sa, A->fwd, A->fwd.sell_cols_global.as<int32_t>(),
                   A->fwd.sell_vals.ptr, sizeof(double), xs.data(), ys.data(),
                   xown.data(), BS, max_blocks_for(comm->num_sms, BS));
  else
    fill_spmv_args(sa, A->fwd, A->fwd.cols_global.as<int32_t>(), sizeof(double),
                   xs.data(), ys.data(), xown.data(), BS / W,
                   max_blocks_for(comm->num_sms, BS));
  if (w.d16) use_d16(sa, A->fwd, w.sell);
  const int ew_grid = std::max(1, comm->num_sms) * (2048 / EW_BS);
  w.partials.reserve(sizeof(double) * std::max(sa.nblocks, ew_grid));

  CgPtrs c;
  c.b = w.b.as<double>();
  c.x = w.x.as<double>();
  c.r = w.r.as<double>();
  c.p = w.p.as<double>();
  c.y = w.y.as<double>();
  c.partials = w.partials.as<double>();
  c.st = w.state.as<CgState>();
  c.n = w.n;

  SPMVB_CUDA(cudaGraphCreate(&w.graph, 0));
  SPMVB_CUDA(cudaGraphConditionalHandleCreate(&w.handle, w.graph, 0,
                                              cudaGraphCondAssignDefault));
  cudaGraphNode_t n_init, n_loop;
  {
    void* args[] = {&c, &w.handle};
    add_kernel(&n_init, w.graph, nullptr, 0, (void*)cg_init, ew_grid, EW_BS,
               args);
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = w.handle;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  SPMVB_CUDA(cudaGraphAddNode(&n_loop, w.graph, &n_init, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];

  cudaGraphNode_t k1 = nullptr, k2 = nullptr, k3 = nullptr;
  if (sa.nblocks > 0) {
    void* args[] = {&sa, &c, &w.handle};
    const DotFn fn = w.sell ? (w.d16 ? dot_kernel_sell<true>(W) : dot_kernel_sell<false>(W))
                            : (w.d16 ? dot_kernel<true>(W) : dot_kernel<false>(W));
    add_kernel(&k1, body, nullptr, 0, (void*)fn, sa.nblocks, BS, args);
  }
  {
    void* args[] = {&c, &w.handle};
    add_kernel(&k2, body, k1 ? &k1 : nullptr, k1 ? 1 : 0, (void*)cg_update_xr,
               ew_grid, EW_BS, args);
  }
  {
    void* args[] = {&c};
    add_kernel(&k3, body, &k2, 1, (void*)cg_update_p, ew_grid, EW_BS, args);
  }
  SPMVB_CUDA(cudaGraphInstantiate(&w.exec, w.graph, 0));
}

}  // namespace

void destroy_cg_workspace(CgWorkspace* w) { delete w; }

CgWorkspace& cg_workspace(spmv_matrix A) {
  if (!A->cg) {
    build_global_cols(A);
    std::unique_ptr<CgWorkspace, void (*)(CgWorkspace*)> w(
        new CgWorkspace, destroy_cg_workspace);
    const int64_t n = A->row_map->ranges.back();
    w->n = n;
    const size_t bytes = sizeof(double) * std::max<int64_t>(n, 1);
    w->b.reserve(bytes);
    w->x.reserve(bytes);
    w->r.reserve(bytes);
    w->p.reserve(bytes);
    w->y.reserve(bytes);
    w->state.reserve(sizeof(CgState));
    SPMVB_CUDA(cudaMemset(w->state.ptr, 0, sizeof(CgState)));
    w->sell = pick_kernel(A->kernel, A->fwd) == SPMV_KERNEL_SELL;
    if (w->sell) build_sell_global(A);
    w->d16 = A->fwd.d16;
    w->W = A->width > 0 ? A->width
                        : (w->sell ? 8 : auto_width(A->fwd.mean_row, SPMV_FLOAT64));
    w->BS = 256;
    build_graph(A, *w);
    A->cg = std::move(w);
  }
  return *A->cg;
}

double* cg_rhs(spmv_matrix A) { return cg_workspace(A).b.as<double>(); }
double* cg_solution(spmv_matrix A) { return cg_workspace(A).x.as<double>(); }

void cg_run(spmv_matrix A, int max_its, double rtol, spmv_cg_info* info) {
  CgWorkspace& w = cg_workspace(A);
  cudaStream_t s = A->comm->stream;
  // kmax and rtol^2 for this solve (cg.cpp:49).
  w.host.kmax = max_its;
  w.host.rtol2 = rtol * rtol;
  CgState* st = w.state.as<CgState>();
  SPMVB_CUDA(cudaMemcpyAsync(&st->kmax, &w.host.kmax, sizeof(int),
                             cudaMemcpyHostToDevice, s));
  SPMVB_CUDA(cudaMemcpyAsync(&st->rtol2, &w.host.rtol2, sizeof(double),
                             cudaMemcpyHostToDevice, s));
  SPMVB_CUDA(cudaGraphLaunch(w.exec, s));
  SPMVB_CUDA(cudaMemcpyAsync(&w.host, st, sizeof(CgState),
                             cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
  if (info) {
    info->iterations = w.host.k;
    info->status = w.host.status;
    info->rnorm0 = w.host.rnorm0;
    info->rnorm = w.host.rnorm_new;
  }
}

}  // namespace spmvb
