// Mixed-precision CG: FP32 inner iterations, FP64 refinement (no counterpart
// in the reference; it builds on spmv::cg, cg.cpp:11-83).
//
// The inner iteration is CG on an FP32 copy of A with FP32 vectors r, p, y
// and an FP32 correction d; every dot product is accumulated in FP64 and
// alpha, beta are FP64.  A refinement step ("reliable update") runs whenever
// the FP32 residual norm has dropped 10x below the largest value since the
// last refinement, when the FP32 recursion claims convergence, and at the
// iteration cap:
//
//   x += d (FP64), d = 0
//   r64 = b - A x             FP64 product and FP64 norm: the true residual
//   stop if ||r64||^2 / ||b||^2 < rtol^2
//   r = fl32(r64); p -= (r.p / r.r) r          (re-orthogonalise p)
//
// and CG continues with p = r + beta p, beta = ||r_new||^2 / ||r_old||^2.
// Carrying p across refinements keeps the Krylov information, so the inner
// iteration count stays close to FP64 CG's while each inner iteration moves
// FP32 data (van der Vorst & Ye, "Residual replacement strategies for Krylov
// subspace iterative methods", SISC 2000; Clark et al., "Solving lattice QCD
// systems of equations using mixed precision solvers on GPUs", 2010).
//
// Graph: init -> WHILE { K1 FP32 product + p.y; K2 d/r update, r.r, decide
// refinement; IF(refine) { fold x; FP64 residual; resync r, p.r } ; K3 p }.
#include <algorithm>
#include <cmath>

#include "internal.h"
#include "spmv_kernel.cuh"

struct IrState {
  double rr0, rr, rr_new, rr_max, alpha, beta, pap, c, rtol2, delta2, rr_true;
  double rr_prev;
  int k, kmax, status, converged, refine, refinements, k_guard, pad1;
  unsigned int t0, t1, t2, t3, t4, pad2[3];
};

struct IrWorkspace {
  int64_t n = 0;
  int W32 = 0, W64 = 0;
  bool sell32 = false, sell64 = false;  // products over the SELL-32 copies
  bool d16 = false;                     // products read 16-bit column offsets
  spmvb::DevBuf b, x, r64, r, p, y, d, partials, state;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle h_loop = 0, h_ref = 0;
  IrState host{};
  ~IrWorkspace() {
    if (exec) spmvb::soft_check(cudaGraphExecDestroy(exec), "cudaGraphExecDestroy");
    if (graph) spmvb::soft_check(cudaGraphDestroy(graph), "cudaGraphDestroy");
  }
};

namespace spmvb {

namespace {

constexpr int EW = 256;

struct IrPtrs {
  const double* b;
  double* x;
  double* r64;
  float* r;
  float* p;
  float* y;
  float* d;
  double* partials;
  IrState* st;
  int64_t n;
};

#define IR_LOOP(i)                                                      \
  for (int64_t i = blockIdx.x * int64_t(EW) + threadIdx.x; i < c.n;   \
       i += int64_t(gridDim.x) * EW)

__global__ void __launch_bounds__(EW) ir_init(const IrPtrs c, cudaGraphConditionalHandle h) {
  __shared__ double smem[32];
  double bb = 0.0, rr = 0.0;
  IR_LOOP(i) {
    const double bi = c.b[i];
    const float ri = float(bi);
    c.r[i] = ri;
    c.p[i] = ri;
    c.d[i] = 0.0f;
    c.x[i] = 0.0;
    bb += bi * bi;
    rr += double(ri) * double(ri);
  }
  double tb, tr;
  if (grid_sum2<EW>(bb, rr, c.partials, &c.st->t0, &tb, &tr, smem) && threadIdx.x == 0) {
    IrState* st = c.st;
    st->rr0 = tb;
    st->rr = tr;
    st->rr_max = tr;
    st->rr_true = tb;
    st->c = 0.0;
    st->k = 0;
    st->k_guard = 0;
    st->status = SPMV_SUCCESS;
    st->converged = 0;
    st->refinements = 0;
    const bool go = st->kmax > 0 && tb > 0.0 && isfinite(tb);
    if (!go) st->converged = tb == 0.0 ? 1 : 0;
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

// Row traversal of the products: vector CSR (W lanes per row) or SELL-32
// (W loads in flight per lane); D16: 16-bit column offsets.
template <typename T, int W, bool SELL, bool D16, class F>
__device__ __forceinline__ void rows_of(const SpmvArgs& a, F&& f) {
  if constexpr (SELL)
    sell_for_rows<T, 256, W, true, D16>(a, f);  // vectors kept in L2, matrix streamed
  else
    for_rows<T, W, 256, D16>(a, f);
}

// K1: y = A32 p (FP32 row sums), p.y accumulated in FP64.
template <int W, bool SELL, bool D16>
__global__ void __launch_bounds__(256)
    ir_spmv_dot(const __grid_constant__ SpmvArgs a, const IrPtrs c,
                cudaGraphConditionalHandle h_loop) {
  __shared__ double smem[32];
  if (blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_loop, 0u);
  double acc = 0.0;
  const uint64_t keep = l2_policy_keep();
  rows_of<float, W, SELL, D16>(a, [&](const PartArg& P, int row, float sum) {
    st_pol(static_cast<float*>(P.y) + row, sum, keep);
    acc += double(ld_pol(static_cast<const float*>(P.xown) + row, keep)) * double(sum);
  });
  const double part = block_sum<256>(acc, smem);
  double total;
  if (grid_sum<256>(part, c.partials, &c.st->t1, &total, smem) && threadIdx.x == 0) {
    IrState* st = c.st;
    st->pap = total;
    if (total == 0.0 || !isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
    st->alpha = st->rr / total;
  }
}

// K2: d += alpha p, r -= alpha y, r.r; decides whether to refine.
__global__ void __launch_bounds__(EW)
    ir_update(const IrPtrs c, cudaGraphConditionalHandle h_ref) {
  __shared__ double smem[32];
  const bool ok = c.st->status == SPMV_SUCCESS;
  const float alpha = float(c.st->alpha);
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  if (ok) {
    IR_LOOP(i) {
      st_pol(c.d + i, ld_pol(c.d + i, keep) + alpha * ld_pol(c.p + i, keep), keep);
      const float ri = ld_pol(c.r + i, keep) - alpha * ld_pol(c.y + i, keep);
      st_pol(c.r + i, ri, keep);
      acc += double(ri) * double(ri);
    }
  }
  const double part = block_sum<EW>(acc, smem);
  double total;
  if (grid_sum<EW>(part, c.partials, &c.st->t2, &total, smem) && threadIdx.x == 0) {
    IrState* st = c.st;
    st->k += 1;
    bool refine = false;
    if (st->status == SPMV_SUCCESS) {
      st->rr_new = total;
      st->rr_max = fmax(st->rr_max, total);
      refine = total < st->delta2 * st->rr_max || total / st->rr0 < st->rtol2 ||
               st->k >= st->kmax || !isfinite(total);
      st->rr_prev = st->rr;
      st->beta = total / st->rr;
      st->rr = total;
    }
    st->c = 0.0;
    st->refine = refine ? 1 : 0;
    cudaGraphSetConditional(h_ref, refine ? 1u : 0u);
  }
}

// Refinement 1: fold the FP32 correction into the FP64 solution.
__global__ void __launch_bounds__(EW) ir_fold(const IrPtrs c) {
  IR_LOOP(i) {
    c.x[i] = c.x[i] + double(c.d[i]);
    c.d[i] = 0.0f;
  }
}

// Refinement 2: r64 = b - A x in FP64, and its norm.
template <int W, bool SELL, bool D16>
__global__ void __launch_bounds__(256)
    ir_residual(const __grid_constant__ SpmvArgs a, const IrPtrs c) {
  __shared__ double smem[32];
  double acc = 0.0;
  rows_of<double, W, SELL, D16>(a, [&](const PartArg& P, int row, double sum) {
    const int64_t g = static_cast<const double*>(P.y) - c.r64 + row;
    const double ri = c.b[g] - sum;
    c.r64[g] = ri;
    acc += ri * ri;
  });
  const double part = block_sum<256>(acc, smem);
  double total;
  if (grid_sum<256>(part, c.partials, &c.st->t3, &total, smem) && threadIdx.x == 0) {
    IrState* st = c.st;
    st->rr_true = total;
    st->refinements += 1;
    st->rr_max = total;
    if (total / st->rr0 < st->rtol2) st->converged = 1;
    if (!isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
  }
}

// Refinement 3: r = fl32(r64); r.r and r.p (FP64) for beta and the
// re-orthogonalisation coefficient.
__global__ void __launch_bounds__(EW) ir_resync(const IrPtrs c) {
  __shared__ double smem[32];
  double rr = 0.0, rp = 0.0;
  IR_LOOP(i) {
    const float ri = float(c.r64[i]);
    c.r[i] = ri;
    rr += double(ri) * double(ri);
    rp += double(ri) * double(c.p[i]);
  }
  double trr, trp;
  if (grid_sum2<EW>(rr, rp, c.partials, &c.st->t4, &trr, &trp, smem) &&
      threadIdx.x == 0) {
    IrState* st = c.st;
    // beta with the replaced residual over ||r||^2 before this step.
    st->beta = trr / st->rr_prev;
    st->rr = trr;
    st->c = trp / trr;
  }
}

// K3: p = r + beta (p - c r); sets the loop condition.
__global__ void __launch_bounds__(EW)
    ir_update_p(const IrPtrs c, cudaGraphConditionalHandle h_loop) {
  const IrState* st = c.st;
  const bool stop = st->status != SPMV_SUCCESS || st->converged;
  if (!stop) {
    const float beta = float(st->beta);
    const float cc = float(st->c);
    const uint64_t keep = l2_policy_keep();
    IR_LOOP(i) {
      const float ri = ld_pol(c.r + i, keep);
      st_pol(c.p + i, ri + beta * (ld_pol(c.p + i, keep) - cc * ri), keep);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    IrState* s = c.st;
    s->k_guard += 1;
    const bool go = !stop && s->k < s->kmax && s->k_guard < s->kmax;
    cudaGraphSetConditional(h_loop, go ? 1u : 0u);
  }
}

__global__ void to_float(const double* __restrict__ in, float* __restrict__ out,
                         int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

using K1 = void (*)(SpmvArgs, IrPtrs, cudaGraphConditionalHandle);
using KR = void (*)(SpmvArgs, IrPtrs);

// SELL widths are loads in flight per lane (1..16), vector widths lanes per
// row (1..32).
template <bool SELL, bool D16>
K1 pick_k1(int W) {
  switch (W) {
    case 1: return ir_spmv_dot<1, SELL, D16>;
    case 2: return ir_spmv_dot<2, SELL, D16>;
    case 4: return ir_spmv_dot<4, SELL, D16>;
    case 8: return ir_spmv_dot<8, SELL, D16>;
    case 16: return ir_spmv_dot<16, SELL, D16>;
    case 32: if (!SELL) return ir_spmv_dot<32, SELL, D16>;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: unsupported product width");
}
template <bool SELL, bool D16>
KR pick_kr(int W) {
  switch (W) {
    case 1: return ir_residual<1, SELL, D16>;
    case 2: return ir_residual<2, SELL, D16>;
    case 4: return ir_residual<4, SELL, D16>;
    case 8: return ir_residual<8, SELL, D16>;
    case 16: return ir_residual<16, SELL, D16>;
    case 32: if (!SELL) return ir_residual<32, SELL, D16>;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: unsupported product width");
}
template <class Fn>
Fn pick4(bool sell, bool d16, int W, Fn (*ss)(int), Fn (*sp)(int), Fn (*vs)(int),
         Fn (*vp)(int)) {
  return sell ? (d16 ? ss(W) : sp(W)) : (d16 ? vs(W) : vp(W));
}

void add_kernel(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* dep,
                size_t ndep, void* fn, int grid, int block, void** args) {
  cudaKernelNodeParams kp{};
  kp.func = fn;
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(block);
  kp.kernelParams = args;
  SPMVB_CUDA(cudaGraphAddKernelNode(node, g, dep, ndep, &kp));
}

void build_ir_graph(spmv_matrix A, IrWorkspace& w) {
  spmv_comm comm = A->comm;
  const int P = comm->size;
  const spmv_l2gmap rm = A->row_map;
  // FP32 product over p (global layout), FP64 residual product over x.
  std::vector<const void*> xs32(P), own32(P), xs64(P);
  std::vector<void*> ys32(P), ys64(P);
  for (int r = 0; r < P; ++r) {
    xs32[r] = w.p.as<float>();
    own32[r] = w.p.as<float>() + rm->ranges[r];
    ys32[r] = w.y.as<float>() + rm->ranges[r];
    xs64[r] = w.x.as<double>();
    ys64[r] = w.r64.as<double>() + rm->ranges[r];
  }
  const DevCsr& C = A->fwd;
  SpmvArgs a32, a64;
  const int mb = max_blocks_for(comm->num_sms, 256);
  auto fill32 = [&](SpmvArgs& a, bool sell, int W) {
    if (sell) {
      fill_sell_args(a, C, C.sell_cols_global.as<int32_t>(), C.sell_vals32.ptr,
                     sizeof(float), xs32.data(), ys32.data(), own32.data(), 256, mb);
    } else {
      fill_spmv_args(a, C, C.cols_global.as<int32_t>(), sizeof(float), xs32.data(),
                     ys32.data(), own32.data(), 256 / W, mb);
      for (int r = 0; r < P; ++r)
        a.part[r].vals = C.vals32.as<float>() + C.parts[r].nz_off;
    }
    if (w.d16) use_d16(a, C, sell);
  };
  // The FP32 product is chosen by timing the plain FP32 kernels on the
  // matrix (the FP64 choice does not carry over: FP32 rows are half the
  // bytes, and the best lane count and layout differ).
  {
    struct Cand {
      bool sell;
      int w;
    };
    std::vector<Cand> cands;
    for (int wv : {2, 4, 8, 16}) cands.push_back({false, wv});
    if (C.sell_vals32.ptr)
      for (int u : {4, 8}) cands.push_back({true, u});
    cudaStream_t s = comm->stream;
    cudaEvent_t e0, e1;
    SPMVB_CUDA(cudaEventCreate(&e0));
    SPMVB_CUDA(cudaEventCreate(&e1));
    double best = 1e300;
    for (const Cand& cd : cands) {
      SpmvArgs t;
      fill32(t, cd.sell, cd.w);
      auto run = [&] {
        cd.sell ? launch_sell_args(t, SPMV_FLOAT32, cd.w, 256, s, w.d16)
                : launch_vector_args(t, SPMV_FLOAT32, cd.w, 256, s, w.d16);
      };
      run();
      SPMVB_CUDA(cudaEventRecord(e0, s));
      for (int i = 0; i < 5; ++i) run();
      SPMVB_CUDA(cudaEventRecord(e1, s));
      SPMVB_CUDA(cudaEventSynchronize(e1));
      float ms = 0.f;
      SPMVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (ms < best) {
        best = ms;
        w.sell32 = cd.sell;
        w.W32 = cd.w;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
  }
  fill32(a32, w.sell32, w.W32);
  if (w.sell64)
    fill_sell_args(a64, C, C.sell_cols_global.as<int32_t>(), C.sell_vals.ptr,
                   sizeof(double), xs64.data(), ys64.data(), nullptr, 256, mb);
  else
    fill_spmv_args(a64, C, C.cols_global.as<int32_t>(), sizeof(double), xs64.data(),
                   ys64.data(), nullptr, 256 / w.W64, mb);
  if (w.d16) use_d16(a64, C, w.sell64);
  const int ew_grid = std::max(1, comm->num_sms) * (2048 / EW);
  w.partials.reserve(sizeof(double) * 2 * std::max({a32.nblocks, a64.nblocks, ew_grid}));

  IrPtrs c;
  c.b = w.b.as<double>();
  c.x = w.x.as<double>();
  c.r64 = w.r64.as<double>();
  c.r = w.r.as<float>();
  c.p = w.p.as<float>();
  c.y = w.y.as<float>();
  c.d = w.d.as<float>();
  c.partials = w.partials.as<double>();
  c.st = w.state.as<IrState>();
  c.n = w.n;

  const K1 k1 = pick4<K1>(w.sell32, w.d16, w.W32, pick_k1<true, true>, pick_k1<true, false>,
                         pick_k1<false, true>, pick_k1<false, false>);
  const KR kr = pick4<KR>(w.sell64, w.d16, w.W64, pick_kr<true, true>, pick_kr<true, false>,
                          pick_kr<false, true>, pick_kr<false, false>);

  SPMVB_CUDA(cudaGraphCreate(&w.graph, 0));
  SPMVB_CUDA(cudaGraphConditionalHandleCreate(&w.h_loop, w.graph, 0,
                                              cudaGraphCondAssignDefault));
  cudaGraphNode_t n_init, n_loop;
  {
    void* args[] = {&c, &w.h_loop};
    add_kernel(&n_init, w.graph, nullptr, 0, (void*)ir_init, ew_grid, EW, args);
  }
  cudaGraphNodeParams lp{};
  lp.type = cudaGraphNodeTypeConditional;
  lp.conditional.handle = w.h_loop;
  lp.conditional.type = cudaGraphCondTypeWhile;
  lp.conditional.size = 1;
  SPMVB_CUDA(cudaGraphAddNode(&n_loop, w.graph, &n_init, 1, &lp));
  cudaGraph_t body = lp.conditional.phGraph_out[0];

  SPMVB_CUDA(cudaGraphConditionalHandleCreate(&w.h_ref, body, 0, 0));
  cudaGraphNode_t b1, b2, b_if, b3;
  {
    void* args[] = {&a32, &c, &w.h_loop};
    add_kernel(&b1, body, nullptr, 0, (void*)k1, a32.nblocks, 256, args);
  }
  {
    void* args[] = {&c, &w.h_ref};
    add_kernel(&b2, body, &b1, 1, (void*)ir_update, ew_grid, EW, args);
  }
  cudaGraphNodeParams ip{};
  ip.type = cudaGraphNodeTypeConditional;
  ip.conditional.handle = w.h_ref;
  ip.conditional.type = cudaGraphCondTypeIf;
  ip.conditional.size = 1;
  SPMVB_CUDA(cudaGraphAddNode(&b_if, body, &b2, 1, &ip));
  cudaGraph_t rbody = ip.conditional.phGraph_out[0];
  {
    cudaGraphNode_t r1, r2, r3;
    void* a1[] = {&c};
    add_kernel(&r1, rbody, nullptr, 0, (void*)ir_fold, ew_grid, EW, a1);
    void* a2[] = {&a64, &c};
    add_kernel(&r2, rbody, &r1, 1, (void*)kr, a64.nblocks, 256, a2);
    void* a3[] = {&c};
    add_kernel(&r3, rbody, &r2, 1, (void*)ir_resync, ew_grid, EW, a3);
  }
  {
    void* args[] = {&c, &w.h_loop};
    add_kernel(&b3, body, &b_if, 1, (void*)ir_update_p, ew_grid, EW, args);
  }
  SPMVB_CUDA(cudaGraphInstantiate(&w.exec, w.graph, 0));
}

}  // namespace

void destroy_ir_workspace(IrWorkspace* w) { delete w; }

void ensure_vals32(spmv_matrix A) {
  DevCsr& C = A->fwd;
  if (C.vals32.ptr) return;
  require(A->dtype == SPMV_FLOAT64, "spmv: FP32 copy needs an FP64 matrix");
  C.vals32.reserve(sizeof(float) * C.nz_total);
  to_float<<<std::max(1, A->comm->num_sms) * 8, 256, 0, A->comm->stream>>>(
      C.vals.as<double>(), C.vals32.as<float>(), C.nz_total);
  SPMVB_CUDA(cudaGetLastError());
}

IrWorkspace& ir_workspace(spmv_matrix A) {
  if (!A->ir) {
    build_global_cols(A);
    ensure_vals32(A);
    std::unique_ptr<IrWorkspace, void (*)(IrWorkspace*)> w(new IrWorkspace,
                                                            destroy_ir_workspace);
    const int64_t n = A->row_map->ranges.back();
    w->n = n;
    const size_t n1 = std::max<int64_t>(n, 1);
    w->b.reserve(8 * n1);
    w->x.reserve(8 * n1);
    w->r64.reserve(8 * n1);
    w->r.reserve(4 * n1);
    w->p.reserve(4 * n1);
    w->y.reserve(4 * n1);
    w->d.reserve(4 * n1);
    w->state.reserve(sizeof(IrState));
    SPMVB_CUDA(cudaMemset(w->state.ptr, 0, sizeof(IrState)));
    // FP64 residual: the matrix's own kernel choice.  FP32 product: timed
    // in build_ir_graph over vector CSR and (when its padding is small)
    // SELL.
    w->sell64 = pick_kernel(A->kernel, A->fwd) == SPMV_KERNEL_SELL;
    if (w->sell64)
      w->W64 = A->width > 0 ? std::min(A->width, 16) : 8;
    else
      w->W64 = auto_width(A->fwd.mean_row, SPMV_FLOAT64);
    if (pick_kernel(SPMV_KERNEL_AUTO, A->fwd) == SPMV_KERNEL_SELL || w->sell64) {
      build_sell_global(A);
      build_sell_vals32(A);
    }
    w->W32 = auto_width(A->fwd.mean_row, SPMV_FLOAT32);
    w->d16 = A->fwd.d16;
    build_ir_graph(A, *w);
    A->ir = std::move(w);
  }
  return *A->ir;
}

double* ir_rhs(spmv_matrix A) { return ir_workspace(A).b.as<double>(); }
double* ir_solution(spmv_matrix A) { return ir_workspace(A).x.as<double>(); }

void ir_run(spmv_matrix A, int max_its, double rtol, spmv_ir_info* info) {
  IrWorkspace& w = ir_workspace(A);
  cudaStream_t s = A->comm->stream;
  IrState* st = w.state.as<IrState>();
  w.host.kmax = max_its;
  w.host.rtol2 = rtol * rtol;
  w.host.delta2 = 0.01;  // refine when ||r|| fell 10x below its recent maximum
  SPMVB_CUDA(cudaMemcpyAsync(&st->kmax, &w.host.kmax, sizeof(int),
                             cudaMemcpyHostToDevice, s));
  SPMVB_CUDA(cudaMemcpyAsync(&st->rtol2, &w.host.rtol2, 2 * sizeof(double),
                             cudaMemcpyHostToDevice, s));
  SPMVB_CUDA(cudaGraphLaunch(w.exec, s));
  SPMVB_CUDA(cudaMemcpyAsync(&w.host, st, sizeof(IrState), cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
  if (info) {
    info->iterations = w.host.k;
    info->refinements = w.host.refinements;
    info->status = w.host.status;
    info->converged = w.host.converged;
    info->relres = w.host.rr0 > 0 ? std::sqrt(w.host.rr_true / w.host.rr0) : 0.0;
  }
}

}  // namespace spmvb
