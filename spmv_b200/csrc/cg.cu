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
//   K2  r -= alpha y, r.r         (the last CTA forms beta, counts the
//                                  iteration, tests convergence and sets the
//                                  graph's loop condition)
//   K3  x += alpha p, p = p beta + r
//                                 (x is updated where p is read anyway: 10
//                                  vector passes per iteration instead of 11;
//                                  the arithmetic is the reference's)
//
// The three kernels form the body of a CUDA-graph while node; an init kernel
// before it sets r = p = b, x = 0 and rnorm0.  (Programmatic dependent
// launch of K2 and K3 was measured on the 7-point stencil and gained
// nothing.)  A whole solve is one graph
// launch with no host round trip per iteration.  Reductions are single pass
// (per-CTA partials, the last CTA to arrive sums them in index order), so
// results are reproducible run to run for a given product kernel.  Vector
// updates are compiled without FMA contraction (-fmad=false), matching the
// separate multiply and add of the reference's Eigen expressions.
//
// K1's product is chosen per matrix by timing each candidate K1 (outside the
// graph, with the loop-condition write compiled out): vector CSR, SELL-32
// from registers, or SELL-32 staged through shared memory by bulk copies,
// each with 32-bit columns or 16-bit offsets.  (Forming p inside K1, where
// the product gathers it, saves K3's pass over p and r but doubles the
// gathers; measured on the 7-point stencil it was slower.)
#include <algorithm>
#include <cmath>
#include <type_traits>

#include "internal.h"
#include "sell_staged.cuh"
#include "spmv_kernel.cuh"

struct CgState {
  double rnorm0, rnorm_old, rnorm_new, alpha, beta, pdoty, rtol2, pad0;
  int k, kmax, status, stage_err;
  unsigned int ticket0, ticket1, ticket2, pad2;
};

struct CgWorkspace {
  int64_t n = 0;
  spmvb::SolverProduct product;
  spmvb::DevBuf b, x, r, p, y, partials, state;
  const spmvb::StagedDesc* tiles = nullptr;
  int ntiles = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle h_loop = 0;
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
  const StagedDesc* tiles;  // staged product only
  int ntiles;
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
    st->stage_err = 0;
    // b == 0 (or non-finite): nothing to iterate on.
    const bool go = st->kmax > 0 && total > 0.0 && isfinite(total);
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

// K1 body shared by the traversals: rows(f) visits every row; the product
// gathers p (the launch table's x) with the L2 keep policy.
template <int BS, class Rows>
__device__ __forceinline__ void cg_k1(const CgPtrs& c, Rows&& rows) {
  __shared__ double smem[32];
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  rows([&](const PartArg& P, int row, double sum) {
    const int g = P.row0 + row;
    st_pol(c.y + g, sum, keep);
    acc += ld_pol(c.p + g, keep) * sum;
  });
  const double part = block_sum<BS>(acc, smem);
  double total;
  if (grid_sum<BS>(part, c.partials, &c.st->ticket1, &total, smem) && threadIdx.x == 0) {
    CgState* st = c.st;
    st->pdoty = total;
    if (total == 0.0 || !isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
    st->alpha = st->rnorm_old / total;
  }
}

// K1 kernels.  H: the graph form, which first defaults the loop condition
// to "stop" (K2 sets it to continue; if K2's last-CTA step ever failed to
// run, the loop would end, never spin); !H: the same kernel for timing.
template <int W, bool D16, bool H>
__global__ void __launch_bounds__(256)
    cg_k1_vector(const __grid_constant__ SpmvArgs a, const CgPtrs c,
                 cudaGraphConditionalHandle h) {
  if (H && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
  cg_k1<256>(c, [&](auto&& f) { for_rows<double, W, 256, D16>(a, f, XGather<double, true>()); });
}

template <int U, bool D16, bool H>
__global__ void __launch_bounds__(256)
    cg_k1_sell(const __grid_constant__ SpmvArgs a, const CgPtrs c,
               cudaGraphConditionalHandle h) {
  if (H && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
  cg_k1<256>(c, [&](auto&& f) { sell_for_rows<double, 256, U, true, D16>(a, f); });
}

template <int U, bool D16, bool H>
__global__ void __launch_bounds__(SolverStaged::BS)
    cg_k1_staged(const __grid_constant__ SpmvArgs a, const CgPtrs c,
                 cudaGraphConditionalHandle h) {
  if (H && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h, 0u);
  using CI = typename std::conditional<D16, int16_t, int32_t>::type;
  cg_k1<SolverStaged::BS>(c, [&](auto&& f) {
    sell_staged_rows<SolverStaged, double, CI, U>(a, c.tiles, c.ntiles, &c.st->stage_err, f,
                                                  XGather<double, true>());
  });
}

// K2: r -= alpha y, r.r; beta, the iteration count and the convergence
// test.  Sets `h` to continue (1) or stop (0).
__global__ void __launch_bounds__(EW_BS)
    cg_update_r(const CgPtrs c, cudaGraphConditionalHandle h) {
  __shared__ double smem[32];
  const bool ok = c.st->status == SPMV_SUCCESS;
  const double alpha = c.st->alpha;
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  if (ok) {
    for (int64_t i = blockIdx.x * int64_t(EW_BS) + threadIdx.x; i < c.n;
         i += int64_t(gridDim.x) * EW_BS) {
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
      go = !converged && st->k < st->kmax && st->stage_err == 0;
    }
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

// K3: x += alpha p, p = p beta + r (with this iteration's alpha and beta;
// skipped, like K2's update, after a breakdown).
__global__ void __launch_bounds__(EW_BS) cg_update_xp(const CgPtrs c) {
  if (c.st->status != SPMV_SUCCESS) return;
  const double alpha = c.st->alpha;
  const double beta = c.st->beta;
  const uint64_t keep = l2_policy_keep();
  for (int64_t i = blockIdx.x * int64_t(EW_BS) + threadIdx.x; i < c.n;
       i += int64_t(gridDim.x) * EW_BS) {
    const double pi = ld_pol(c.p + i, keep);
    st_pol(c.x + i, ld_pol(c.x + i, keep) + alpha * pi, keep);
    st_pol(c.p + i, pi * beta + ld_pol(c.r + i, keep), keep);
  }
}

using K1Fn = void (*)(SpmvArgs, CgPtrs, cudaGraphConditionalHandle);

template <bool D16, bool H>
K1Fn k1_vector(int W) {
  switch (W) {
    case 1: return cg_k1_vector<1, D16, H>;
    case 2: return cg_k1_vector<2, D16, H>;
    case 4: return cg_k1_vector<4, D16, H>;
    case 8: return cg_k1_vector<8, D16, H>;
    case 16: return cg_k1_vector<16, D16, H>;
    case 32: return cg_k1_vector<32, D16, H>;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: width must be 1..32, a power of two");
}

template <bool D16, bool H>
K1Fn k1_sell(int U) {
  switch (U) {
    case 1: return cg_k1_sell<1, D16, H>;
    case 2: return cg_k1_sell<2, D16, H>;
    case 4: return cg_k1_sell<4, D16, H>;
    case 8: return cg_k1_sell<8, D16, H>;
    case 16: return cg_k1_sell<16, D16, H>;
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: SELL width must be 1, 2, 4, 8 or 16");
}

template <bool D16, bool H>
K1Fn k1_staged(int U) {
  switch (staged_width(U)) {
    case 8: return cg_k1_staged<8, D16, H>;
    case 7: return cg_k1_staged<7, D16, H>;
    case 5: return cg_k1_staged<5, D16, H>;
    default: return cg_k1_staged<4, D16, H>;
  }
}

template <bool H>
K1Fn k1_fn_h(const SolverProduct& sp) {
  switch (sp.kind) {
    case ProductKind::Vector: return sp.d16 ? k1_vector<true, H>(sp.w) : k1_vector<false, H>(sp.w);
    case ProductKind::Sell: return sp.d16 ? k1_sell<true, H>(sp.w) : k1_sell<false, H>(sp.w);
    case ProductKind::Staged: return sp.d16 ? k1_staged<true, H>(sp.w) : k1_staged<false, H>(sp.w);
  }
  fail(SPMV_ERROR_INTERNAL, "spmv: unknown product kind");
}

// K1 for a product choice; handle: the graph form (sets the loop condition).
K1Fn k1_fn(const SolverProduct& sp, bool handle) {
  return handle ? k1_fn_h<true>(sp) : k1_fn_h<false>(sp);
}

// Launch shape of K1: vector/SELL use the launch table's CTAs (256 threads);
// staged runs persistent CTAs with its stage buffers in dynamic shared memory.
struct K1Shape {
  int grid, block, smem;
};
K1Shape k1_shape(const SolverProduct& sp, const SpmvArgs& a, int ntiles, int num_sms) {
  if (sp.kind != ProductKind::Staged) return {a.nblocks, 256, 0};
  const int eb = 8 + (sp.d16 ? 2 : 4);
  const StagedShape sh = staged_shape((const void*)k1_fn(sp, false), eb, ntiles, num_sms);
  // The graph form has the same resources; give it the same limit.
  SPMVB_CUDA(cudaFuncSetAttribute((const void*)k1_fn(sp, true),
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, sh.smem));
  return {sh.grid, SolverStaged::BS, sh.smem};
}

CgPtrs cg_ptrs(CgWorkspace& w) {
  CgPtrs c;
  c.b = w.b.as<double>();
  c.x = w.x.as<double>();
  c.r = w.r.as<double>();
  c.p = w.p.as<double>();
  c.y = w.y.as<double>();
  c.partials = w.partials.as<double>();
  c.st = w.state.as<CgState>();
  c.n = w.n;
  c.tiles = w.tiles;
  c.ntiles = w.ntiles;
  return c;
}

void add_kernel(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* dep,
                size_t ndep, void* fn, int grid, int block, int smem, void** args) {
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeKernel;
  np.kernel.func = fn;
  np.kernel.gridDim = dim3(grid);
  np.kernel.blockDim = dim3(block);
  np.kernel.sharedMemBytes = unsigned(smem);
  np.kernel.kernelParams = args;
  np.kernel.extra = nullptr;
  SPMVB_CUDA(cudaGraphAddNode(node, g, dep, ndep, &np));
}

// The staged tile table a product uses (FP64 values).
const DevCsr::StagedTable& cg_tiles(spmv_matrix A, const SolverProduct& sp) {
  const int eb = 8 + (sp.d16 ? 2 : 4);
  return staged_table(A->fwd, eb, SolverStaged::max_entries(eb));
}

// Launch table of K1 over the global layout for a product.  K1 takes its
// vectors from CgPtrs; the table supplies the matrix and the row ranges.
SpmvArgs k1_args(spmv_matrix A, CgWorkspace& w, const SolverProduct& sp) {
  spmv_comm comm = A->comm;
  const int P = comm->size;
  const spmv_l2gmap rm = A->row_map;
  std::vector<const void*> xs(P), xown(P);
  std::vector<void*> ys(P);
  for (int r = 0; r < P; ++r) {
    xs[r] = w.p.as<double>();
    xown[r] = w.p.as<double>() + rm->ranges[r];
    ys[r] = w.y.as<double>() + rm->ranges[r];
  }
  SpmvArgs sa;
  const int mb = max_blocks_for(comm->num_sms, 256);
  if (sp.sell_layout())
    fill_sell_args(sa, A->fwd, A->fwd.sell_cols_global.as<int32_t>(), A->fwd.sell_vals.ptr,
                   sizeof(double), xs.data(), ys.data(), xown.data(), 256, mb);
  else
    fill_spmv_args(sa, A->fwd, A->fwd.cols_global.as<int32_t>(), sizeof(double), xs.data(),
                   ys.data(), xown.data(), 256 / sp.w, mb);
  if (sp.d16) use_d16(sa, A->fwd, sp.sell_layout());
  return sa;
}

void build_graph(spmv_matrix A, CgWorkspace& w) {
  spmv_comm comm = A->comm;
  SpmvArgs sa = k1_args(A, w, w.product);
  const int ew_grid = std::max(1, comm->num_sms) * (2048 / EW_BS);
  const K1Shape k1s = k1_shape(w.product, sa, w.ntiles, comm->num_sms);
  w.partials.reserve(sizeof(double) * std::max(k1s.grid, ew_grid));
  CgPtrs c = cg_ptrs(w);

  SPMVB_CUDA(cudaGraphCreate(&w.graph, 0));
  SPMVB_CUDA(cudaGraphConditionalHandleCreate(&w.h_loop, w.graph, 0,
                                              cudaGraphCondAssignDefault));
  cudaGraphNode_t n_init, n_loop;
  {
    void* args[] = {&c, &w.h_loop};
    add_kernel(&n_init, w.graph, nullptr, 0, (void*)cg_init, ew_grid, EW_BS, 0, args);
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = w.h_loop;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  SPMVB_CUDA(cudaGraphAddNode(&n_loop, w.graph, &n_init, 1, &cp));
  cudaGraph_t body = cp.conditional.phGraph_out[0];

  cudaGraphNode_t k1 = nullptr, k2;
  if (sa.nblocks > 0) {
    void* args[] = {&sa, &c, &w.h_loop};
    add_kernel(&k1, body, nullptr, 0, (void*)k1_fn(w.product, true), k1s.grid, k1s.block,
               k1s.smem, args);
  }
  {
    void* args[] = {&c, &w.h_loop};
    add_kernel(&k2, body, k1 ? &k1 : nullptr, k1 ? 1 : 0, (void*)cg_update_r, ew_grid, EW_BS,
               0, args);
  }
  {
    cudaGraphNode_t k3;
    void* args[] = {&c};
    add_kernel(&k3, body, &k2, 1, (void*)cg_update_xp, ew_grid, EW_BS, 0, args);
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
    SPMVB_CUDA(cudaMemset(w->p.ptr, 0, bytes));
    spmv_comm comm = A->comm;
    // Partials for any K1 grid: the launch table's (at most max_blocks_for)
    // or a persistent staged grid (at most a few CTAs per SM).
    w->partials.reserve(sizeof(double) *
                        std::max(max_blocks_for(comm->num_sms, 256),
                                 std::max(1, comm->num_sms) * 32));
    // K1's product: the candidate whose K1 (timed outside the graph) is
    // fastest on this matrix.
    prepare_solver_layouts(A, false);
    CgWorkspace& ws = *w;
    const SolverProduct sp = choose_solver_product(
        A, SPMV_FLOAT64, ws.p.ptr, ws.y.ptr, true,
        [&](const SolverProduct& cd, const SpmvArgs& a, cudaStream_t s) {
          int ntiles = 0;
          if (cd.kind == ProductKind::Staged) {
            const DevCsr::StagedTable& t = cg_tiles(A, cd);
            ws.tiles = t.desc.as<StagedDesc>();
            ws.ntiles = ntiles = t.ntiles;
          }
          CgPtrs c = cg_ptrs(ws);
          const K1Shape sh = k1_shape(cd, a, ntiles, comm->num_sms);
          cudaGraphConditionalHandle none = 0;
          void* args[] = {const_cast<SpmvArgs*>(&a), &c, &none};
          SPMVB_CUDA(cudaLaunchKernel((void*)k1_fn(cd, false), dim3(sh.grid), dim3(sh.block),
                                      args, size_t(sh.smem), s));
        });
    ws.product = sp;
    ws.tiles = nullptr;
    ws.ntiles = 0;
    if (sp.kind == ProductKind::Staged) {
      const DevCsr::StagedTable& t = cg_tiles(A, sp);
      ws.tiles = t.desc.as<StagedDesc>();
      ws.ntiles = t.ntiles;
    }
    build_graph(A, ws);
    A->cg = std::move(w);
  }
  return *A->cg;
}

SolverProduct cg_product(spmv_matrix A) {
  require(A->cg != nullptr, "spmv: spmv_cg has not run on this matrix");
  return A->cg->product;
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
  if (w.host.stage_err)
    fail(SPMV_ERROR_CUDA, "spmv::cg - a staged product's bounded wait timed out");
  if (info) {
    info->iterations = w.host.k;
    info->status = w.host.status;
    info->rnorm0 = w.host.rnorm0;
    info->rnorm = w.host.rnorm_new;
  }
}

}  // namespace spmvb
