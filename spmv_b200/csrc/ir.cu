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
#include <cstdlib>
#include <string>

#include <type_traits>

#include "internal.h"
#include "sell_staged.cuh"
#include "spmv_kernel.cuh"

struct IrState {
  double rr0, rr, rr_new, rr_max, alpha, beta, pap, c, rtol2, delta2, rr_true;
  double rr_prev;
  int k, kmax, status, converged, refine, refinements, k_guard, stage_err;
  unsigned int t0, t1, t2, t3, t4, pad2[3];
};

struct IrWorkspace {
  int64_t n = 0;
  spmvb::SolverProduct p32, p64;        // FP32 inner and FP64 residual products
  const spmvb::StagedDesc* tiles32 = nullptr;  // staged tile tables (if staged)
  const spmvb::StagedDesc* tiles64 = nullptr;
  int ntiles32 = 0, ntiles64 = 0;
  spmvb::DevBuf b, x, r64, r, p, y, d, partials, state;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaGraphConditionalHandle h_loop = 0, h_ref = 0;
  // Fused form (one cooperative launch per solve), when chosen.
  bool fused = false;
  const void* fused_fn = nullptr;
  int fused_grid = 0, fused_block = 0, fused_smem = 0, fused_cps = 0;
  bool fused_rs = false;
  spmvb::DevBuf bar, fpartials, ctas;
  spmvb::SpmvArgs fa32, fa64;  // FP32 product over p, FP64 SELL over x
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
  const StagedDesc* tiles32;  // staged products only
  const StagedDesc* tiles64;
  int ntiles32, ntiles64;
  unsigned long long* bar;     // fused solve: grid barrier counter
  unsigned long long wait_ns;  // fused solve: bound of each grid wait
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
    st->stage_err = 0;
    const bool go = st->kmax > 0 && tb > 0.0 && isfinite(tb);
    if (!go) st->converged = tb == 0.0 ? 1 : 0;
    cudaGraphSetConditional(h, go ? 1u : 0u);
  }
}

// Row traversal of the products, by kind (ProductKind): 0 vector CSR (W
// lanes per row), 1 SELL-32 from registers (W loads in flight per lane), 2
// SELL-32 staged through shared memory (W gathers in flight per lane);
// D16: 16-bit column offsets.  SELL kinds keep the vectors in L2 and stream
// the matrix.
template <int KIND>
__host__ __device__ constexpr int kind_bs() {
  return KIND == 2 ? SolverStaged::BS : 256;
}

template <typename T, int W, int KIND, bool D16, class F>
__device__ __forceinline__ void rows_of(const SpmvArgs& a, const StagedDesc* tiles, int ntiles,
                                        int* err, F&& f) {
  if constexpr (KIND == 1) {
    sell_for_rows<T, 256, W, true, D16>(a, f);
  } else if constexpr (KIND == 2) {
    using CI = typename std::conditional<D16, int16_t, int32_t>::type;
    sell_staged_rows<SolverStaged, T, CI, W>(a, tiles, ntiles, err, f, XGather<T, true>());
  } else {
    for_rows<T, W, 256, D16>(a, f);
  }
}

// K1: y = A32 p (FP32 row sums), p.y accumulated in FP64.  !H: the same
// kernel outside the graph (no loop condition), for timing candidates.
template <int W, int KIND, bool D16, bool H>
__device__ __forceinline__ void ir_spmv_dot_body(const SpmvArgs& a, const IrPtrs& c,
                                                 cudaGraphConditionalHandle h_loop) {
  constexpr int BS = kind_bs<KIND>();
  __shared__ double smem[32];
  if (H && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional(h_loop, 0u);
  double acc = 0.0;
  const uint64_t keep = l2_policy_keep();
  rows_of<float, W, KIND, D16>(a, c.tiles32, c.ntiles32, &c.st->stage_err,
                               [&](const PartArg& P, int row, float sum) {
    st_pol(static_cast<float*>(P.y) + row, sum, keep);
    acc += double(ld_pol(static_cast<const float*>(P.xown) + row, keep)) * double(sum);
  });
  const double part = block_sum<BS>(acc, smem);
  double total;
  if (grid_sum<BS>(part, c.partials, &c.st->t1, &total, smem) && threadIdx.x == 0) {
    IrState* st = c.st;
    st->pap = total;
    if (total == 0.0 || !isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
    st->alpha = st->rr / total;
  }
}

// Launch bounds: the vector and SELL forms keep the compiler's own register
// choice; the staged form is compiled for its 3 resident CTAs per SM.
template <int W, int KIND, bool D16, bool H>
__global__ void __launch_bounds__(256)
    ir_spmv_dot(const __grid_constant__ SpmvArgs a, const IrPtrs c,
                cudaGraphConditionalHandle h_loop) {
  ir_spmv_dot_body<W, KIND, D16, H>(a, c, h_loop);
}
template <int W, bool D16, bool H>
__global__ void __launch_bounds__(SolverStaged::BS, SolverStaged::MINB)
    ir_spmv_dot_staged(const __grid_constant__ SpmvArgs a, const IrPtrs c,
                       cudaGraphConditionalHandle h_loop) {
  ir_spmv_dot_body<W, 2, D16, H>(a, c, h_loop);
}

// K2: r -= alpha y, r.r; decides whether to refine.  (The correction
// update d += alpha p is made where p is read anyway: by K3, or by the fold
// when this iteration refines.)
__global__ void __launch_bounds__(EW)
    ir_update(const IrPtrs c, cudaGraphConditionalHandle h_ref) {
  __shared__ double smem[32];
  const bool ok = c.st->status == SPMV_SUCCESS;
  const float alpha = float(c.st->alpha);
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  if (ok) {
    IR_LOOP(i) {
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

// Refinement 1: fold the FP32 correction, with this iteration's alpha p,
// into the FP64 solution.
__global__ void __launch_bounds__(EW) ir_fold(const IrPtrs c) {
  const float alpha = float(c.st->alpha);
  IR_LOOP(i) {
    const float di = c.d[i] + alpha * c.p[i];
    c.x[i] = c.x[i] + double(di);
    c.d[i] = 0.0f;
  }
}

// Refinement 2: r64 = b - A x in FP64, and its norm.
template <int W, int KIND, bool D16>
__device__ __forceinline__ void ir_residual_body(const SpmvArgs& a, const IrPtrs& c) {
  constexpr int BS = kind_bs<KIND>();
  __shared__ double smem[32];
  double acc = 0.0;
  rows_of<double, W, KIND, D16>(a, c.tiles64, c.ntiles64, &c.st->stage_err,
                                [&](const PartArg& P, int row, double sum) {
    const int64_t g = static_cast<const double*>(P.y) - c.r64 + row;
    const double ri = c.b[g] - sum;
    c.r64[g] = ri;
    acc += ri * ri;
  });
  const double part = block_sum<BS>(acc, smem);
  double total;
  if (grid_sum<BS>(part, c.partials, &c.st->t3, &total, smem) && threadIdx.x == 0) {
    IrState* st = c.st;
    st->rr_true = total;
    st->refinements += 1;
    st->rr_max = total;
    if (total / st->rr0 < st->rtol2) st->converged = 1;
    if (!isfinite(total)) st->status = SPMV_ERROR_BREAKDOWN;
  }
}

template <int W, int KIND, bool D16>
__global__ void __launch_bounds__(256)
    ir_residual(const __grid_constant__ SpmvArgs a, const IrPtrs c) {
  ir_residual_body<W, KIND, D16>(a, c);
}
template <int W, bool D16>
__global__ void __launch_bounds__(SolverStaged::BS, SolverStaged::MINB)
    ir_residual_staged(const __grid_constant__ SpmvArgs a, const IrPtrs c) {
  ir_residual_body<W, 2, D16>(a, c);
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

// K3: d += alpha p (unless the fold did it), p = r + beta (p - c r); sets
// the loop condition.
__global__ void __launch_bounds__(EW)
    ir_update_p(const IrPtrs c, cudaGraphConditionalHandle h_loop) {
  const IrState* st = c.st;
  const bool stop = st->status != SPMV_SUCCESS || st->converged;
  if (!stop) {
    const float alpha = float(st->alpha);
    const float beta = float(st->beta);
    const float cc = float(st->c);
    const bool fold_d = st->refine == 0;
    const uint64_t keep = l2_policy_keep();
    IR_LOOP(i) {
      const float ri = ld_pol(c.r + i, keep);
      const float pi = ld_pol(c.p + i, keep);
      if (fold_d) st_pol(c.d + i, ld_pol(c.d + i, keep) + alpha * pi, keep);
      st_pol(c.p + i, ri + beta * (pi - cc * ri), keep);
    }
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    IrState* s = c.st;
    s->k_guard += 1;
    const bool go = !stop && s->k < s->kmax && s->k_guard < s->kmax && s->stage_err == 0;
    cudaGraphSetConditional(h_loop, go ? 1u : 0u);
  }
}

// ---------------------------------------------------------------------------
// Fused solve: the whole mixed-precision CG (init, inner iterations and the
// refinements) as one cooperative launch of persistent CTAs, each owning a
// contiguous run of the FP32 product's staged tiles and so a contiguous
// range of global rows; grid barriers between the phases.  Per inner
// iteration, with exactly the graph form's arithmetic:
//
//   A  y = A32 p (the staged FP32 traversal), p.y in FP64  -> alpha
//   B  r -= alpha y, r.r; the refinement test              -> beta ...
//   (refining: x += d + alpha p, d = 0 -> barrier; r = fl32(b - A x) with
//    the FP64 product over the CTA's slices (SELL-32 from global memory,
//    storage order); ||b - A x||, r.r, r.p                  -> beta, c)
//   C  d += alpha p (unless refined), p = r + beta (p - c r) -> barrier
//
// RS: the CTA's rows of r (FP32) stay in shared memory for the whole solve.
// The refinement's FP64 residual is written straight into r (the graph form
// keeps it in r64 first: the same values).
struct IrScalars {
  double rr0, rr, rr_new, rr_max, alpha, beta, pap, c, rtol2, delta2, rr_true, rr_prev;
  int k, kmax, status, converged, refine, refinements, k_guard, go;
};

// Phase A for one consumer thread: returns its share of p.y.
template <class CFG, int U, typename CI>
__device__ __forceinline__ double ir_fused_product(const SpmvArgs& a, int count, uint64_t q_base,
                                                   StagedLoop<CFG>& pipe,
                                                   const unsigned char* smem, int* err,
                                                   float* __restrict__ y,
                                                   const float* __restrict__ p) {
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  staged_loop_consume<CFG, float, CI, U>(
      a, count, q_base, pipe, smem, err,
      [&](const PartArg& P, int row, float sum) {
        const int g = P.row0 + row;
        st_pol(y + g, sum, keep);
        acc += double(ld_pol(p + g, keep)) * double(sum);
      },
      XGather<float, true>());
  return acc;
}

// The refinement's FP64 residual over the CTA's slices (tiles t0..t1 of
// the FP32 table: the same slices in the FP64 SELL arrays), one warp per
// slice, each row summed in storage order; f(g, r64, exists) by every lane
// of the warp for each slice (exists: the lane's row is a row of the rank).
template <int NW, int U, bool D16, class F>
__device__ __forceinline__ void ir_fused_residual(const SpmvArgs& a,
                                                  const StagedDesc* __restrict__ tiles, int t0,
                                                  int t1, const double* __restrict__ x,
                                                  const double* __restrict__ b, F&& f) {
  using CI = typename std::conditional<D16, int16_t, int32_t>::type;
  const int warp = int(threadIdx.x) >> 5, lane = int(threadIdx.x) & 31;
  int q = warp;
  for (int t = t0; t < t1; ++t) {
    const StagedDesc* d = tiles + t;
    const int ns = __ldg(&d->nslices);
    if (q >= ns) {
      q -= ns;
      continue;
    }
    const PartArg& P = a.part[__ldg(&d->rank)];
    const int s0 = __ldg(&d->s0);
    const int32_t* __restrict__ soff = P.rowptr;
    const CI* __restrict__ cols = reinterpret_cast<const CI*>(P.cols);
    const double* __restrict__ vals = static_cast<const double*>(P.vals);
    for (; q < ns; q += NW) {
      const int slice = s0 + q;
      const int o = __ldg(soff + slice);
      const int w = (__ldg(soff + slice + 1) - o) >> 5;
      const int row = slice * 32 + lane;
      const int g = P.row0 + row;
      double sum = 0.0;
      for (int k0 = 0; k0 < w; k0 += U) {
        double v[U], xv[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const bool in = k0 + u < w;
          const int idx = o + (k0 + u) * 32 + lane;
          const int ci = in ? int(cols[idx]) : 0;
          ok[u] = in && (D16 ? ci != -32768 : ci >= 0);
          v[u] = in ? vals[idx] : 0.0;
          xv[u] = ok[u] ? x[D16 ? g + ci : ci] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) sum += v[u] * xv[u];
      }
      const bool exists = row < P.nrows;
      f(g, exists ? b[g] - sum : 0.0, exists);
    }
    q -= ns;
  }
}

template <class CFG, int U, bool D16, bool RS>
__global__ void __launch_bounds__(CFG::BS, CFG::MINB)
    ir_fused(const __grid_constant__ SpmvArgs a32, const __grid_constant__ SpmvArgs a64,
             const IrPtrs c, const FusedCta* __restrict__ ctas) {
  using CI = typename std::conditional<D16, int16_t, int32_t>::type;
  constexpr int NT = CFG::NC * 32;
  constexpr int STAGES_BYTES = CFG::smem_bytes(4 + int(sizeof(CI)));
  // Rows per thread in flight in the vector phases (B and C) and entries
  // per lane in flight in the refinement's residual: as many as the shape's
  // registers hold without spilling.
  constexpr int V = CFG::MINB == 3 ? 1 : 4;
  constexpr int UR = CFG::MINB == 3 ? 4 : 6;
  extern __shared__ __align__(128) unsigned char staged_smem[];
  __shared__ StagedLoop<CFG> pipe;
  __shared__ GridSumN<NT, 1> gs1;
  __shared__ GridSumN<NT, 2> gs2;
  __shared__ GridSumN<NT, 3> gs3;
  __shared__ GridSum<NT> gsb;
  __shared__ double racc[CFG::NC][3];
  __shared__ FusedCta me;
  __shared__ IrScalars sv;

  const int tid = int(threadIdx.x);
  if (tid == 0) {
    me = ctas[blockIdx.x];
    staged_loop_init(pipe);
  }
  __syncthreads();
  int* err = &c.st->stage_err;
  if (tid >= NT) {
    if (tid == NT)
      staged_loop_produce<CFG, float, CI>(a32, c.tiles32 + me.t0, me.t1 - me.t0, pipe,
                                          staged_smem, err);
    return;
  }
  auto r_at = [&](int g) -> float& {
    return RS ? reinterpret_cast<float*>(staged_smem + STAGES_BYTES)[g - me.g0] : c.r[g];
  };
  // Grid syncs (sums and plain barriers) are numbered 1, 2, ...; sync e
  // completes when the counter reaches e * gridDim.x.  A sum at sync e
  // publishes into partial array e & 1 (3 per CTA): the array was last read
  // before sync e - 1 at the latest, which every CTA has passed.
  unsigned long long epoch = 0;
  auto parts = [&](unsigned long long e) { return c.partials + (e & 1) * 3 * gridDim.x; };
  auto sum1 = [&](double v, double& total) -> bool {
    double in[1] = {v}, out[1] = {0.0};
    ++epoch;
    const bool okk = coop_grid_sum_n<NT, 1>(in, parts(epoch), c.bar, epoch * gridDim.x, err,
                                            c.wait_ns, gs1, out);
    total = out[0];
    return okk;
  };
  auto barrier = [&]() {
    ++epoch;
    return coop_grid_barrier<NT>(c.bar, epoch * gridDim.x, err, c.wait_ns, gsb);
  };
  const uint64_t keep = l2_policy_keep();
  bool ok = true;

  // Init (ir_init): r = p = fl32(b), d = 0, x = 0; ||b||^2 and ||r||^2.
  {
    double bb = 0.0, rr = 0.0;
    for (int g = me.g0 + tid; g < me.g1; g += NT) {
      const double bi = c.b[g];
      const float ri = float(bi);
      r_at(g) = ri;
      c.p[g] = ri;
      c.d[g] = 0.0f;
      c.x[g] = 0.0;
      bb += bi * bi;
      rr += double(ri) * double(ri);
    }
    double in[2] = {bb, rr}, out[2] = {0.0, 0.0};
    ++epoch;
    ok = coop_grid_sum_n<NT, 2>(in, parts(epoch), c.bar, epoch * gridDim.x, err, c.wait_ns,
                                gs2, out);
    if (tid == 0) {
      sv.kmax = *static_cast<volatile int*>(&c.st->kmax);
      sv.rtol2 = *static_cast<volatile double*>(&c.st->rtol2);
      sv.delta2 = *static_cast<volatile double*>(&c.st->delta2);
      sv.rr0 = out[0];
      sv.rr = out[1];
      sv.rr_max = out[1];
      sv.rr_true = out[0];
      sv.rr_new = sv.alpha = sv.beta = sv.pap = sv.rr_prev = 0.0;
      sv.c = 0.0;
      sv.k = sv.k_guard = sv.refinements = sv.refine = 0;
      sv.status = SPMV_SUCCESS;
      sv.converged = 0;
      sv.go = ok && sv.kmax > 0 && out[0] > 0.0 && isfinite(out[0]);
      if (!sv.go && ok) sv.converged = out[0] == 0.0 ? 1 : 0;
    }
    named_sync(1, NT);
  }
  int it = 0;
  while (sv.go) {
    // A (ir_spmv_dot): y = A32 p, p.y.
    const int count = me.t1 - me.t0;
    double pap = 0.0;
    const bool okA = sum1(ir_fused_product<CFG, U, CI>(a32, count, uint64_t(it) * uint64_t(count),
                                                        pipe, staged_smem, err, c.y, c.p),
                          pap);
    ++it;
    if (!okA) {
      ok = false;
      break;
    }
    if (tid == 0) {
      sv.pap = pap;
      if (pap == 0.0 || !isfinite(pap)) sv.status = SPMV_ERROR_BREAKDOWN;
      sv.alpha = sv.rr / pap;
    }
    named_sync(1, NT);
    // B (ir_update): r -= alpha y, r.r; the refinement test.
    const bool good = sv.status == SPMV_SUCCESS;
    const float alpha32 = float(sv.alpha);
    double acc = 0.0;
    if (good) {
      const int g1 = me.g1;
      for (int g0 = me.g0 + tid; g0 < g1; g0 += V * NT) {
        float yv[V];
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) yv[u] = ld_pol(c.y + g, keep);
        }
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            const float ri = r_at(g) - alpha32 * yv[u];
            r_at(g) = ri;
            acc += double(ri) * double(ri);
          }
        }
      }
    }
    double total = 0.0;
    if (!sum1(acc, total)) {
      ok = false;
      break;
    }
    if (tid == 0) {
      sv.k += 1;
      bool refine = false;
      if (sv.status == SPMV_SUCCESS) {
        sv.rr_new = total;
        sv.rr_max = fmax(sv.rr_max, total);
        refine = total < sv.delta2 * sv.rr_max || total / sv.rr0 < sv.rtol2 ||
                 sv.k >= sv.kmax || !isfinite(total);
        sv.rr_prev = sv.rr;
        sv.beta = total / sv.rr;
        sv.rr = total;
      }
      sv.c = 0.0;
      sv.refine = refine ? 1 : 0;
    }
    named_sync(1, NT);
    if (sv.refine) {
      // Fold (ir_fold): x += d + alpha p, d = 0.
      for (int g = me.g0 + tid; g < me.g1; g += NT) {
        const float di = c.d[g] + alpha32 * c.p[g];
        c.x[g] = c.x[g] + double(di);
        c.d[g] = 0.0f;
      }
      if (!barrier()) {
        ok = false;
        break;
      }
      // Residual and resync (ir_residual, ir_resync): r = fl32(b - A x).
      // ||b - A x||^2, r.r and r.p: summed per slice across the warp and
      // kept per warp in shared memory (no accumulators live across the
      // gathers), then handed to the grid sum by each warp's lane 0.
      const int warp = tid >> 5, lane = tid & 31;
      if (lane == 0) racc[warp][0] = racc[warp][1] = racc[warp][2] = 0.0;
      __syncwarp();
      ir_fused_residual<CFG::NC, UR, D16>(
          a64, c.tiles32, me.t0, me.t1, c.x, c.b, [&](int g, double r64, bool exists) {
            const float ri = float(r64);
            double v0 = 0.0, v1 = 0.0, v2 = 0.0;
            if (exists) {
              r_at(g) = ri;
              v0 = r64 * r64;
              v1 = double(ri) * double(ri);
              v2 = double(ri) * double(c.p[g]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
              v0 += __shfl_xor_sync(0xffffffffu, v0, o);
              v1 += __shfl_xor_sync(0xffffffffu, v1, o);
              v2 += __shfl_xor_sync(0xffffffffu, v2, o);
            }
            if (lane == 0) {
              racc[warp][0] += v0;
              racc[warp][1] += v1;
              racc[warp][2] += v2;
            }
          });
      __syncwarp();
      double t3[3] = {0.0, 0.0, 0.0};
      if (lane == 0) {
        t3[0] = racc[warp][0];
        t3[1] = racc[warp][1];
        t3[2] = racc[warp][2];
      }
      double o3[3];
      ++epoch;
      if (!coop_grid_sum_n<NT, 3>(t3, parts(epoch), c.bar, epoch * gridDim.x, err, c.wait_ns,
                                  gs3, o3)) {
        ok = false;
        break;
      }
      if (tid == 0) {
        sv.rr_true = o3[0];
        sv.refinements += 1;
        sv.rr_max = o3[0];
        if (o3[0] / sv.rr0 < sv.rtol2) sv.converged = 1;
        if (!isfinite(o3[0])) sv.status = SPMV_ERROR_BREAKDOWN;
        sv.beta = o3[1] / sv.rr_prev;
        sv.rr = o3[1];
        sv.c = o3[2] / o3[1];
      }
      named_sync(1, NT);
    }
    // C (ir_update_p): d += alpha p (unless folded), p = r + beta (p - c r).
    const bool stop = sv.status != SPMV_SUCCESS || sv.converged;
    if (!stop) {
      const float beta32 = float(sv.beta);
      const float cc = float(sv.c);
      const bool fold_d = sv.refine == 0;
      const int g1 = me.g1;
      for (int g0 = me.g0 + tid; g0 < g1; g0 += V * NT) {
        float pv[V], dv[V];
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            pv[u] = ld_pol(c.p + g, keep);
            dv[u] = fold_d ? ld_pol(c.d + g, keep) : 0.0f;
          }
        }
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            const float ri = r_at(g);
            if (fold_d) st_pol(c.d + g, dv[u] + alpha32 * pv[u], keep);
            st_pol(c.p + g, ri + beta32 * (pv[u] - cc * ri), keep);
          }
        }
      }
    }
    if (tid == 0) {
      sv.k_guard += 1;
      sv.go = !stop && sv.k < sv.kmax && sv.k_guard < sv.kmax;
    }
    named_sync(1, NT);
    if (!sv.go) break;
    if (!barrier()) {  // A gathers p
      ok = false;
      break;
    }
  }
  if (tid == 0) {
    pipe.stop = 1;
    if (ok && blockIdx.x == 0) {
      IrState* st = c.st;
      st->rr0 = sv.rr0;
      st->rr = sv.rr;
      st->rr_new = sv.rr_new;
      st->rr_max = sv.rr_max;
      st->alpha = sv.alpha;
      st->beta = sv.beta;
      st->pap = sv.pap;
      st->c = sv.c;
      st->rr_true = sv.rr_true;
      st->rr_prev = sv.rr_prev;
      st->k = sv.k;
      st->status = sv.status;
      st->converged = sv.converged;
      st->refine = sv.refine;
      st->refinements = sv.refinements;
      st->k_guard = sv.k_guard;
    }
  }
}

using IrFusedFn = void (*)(SpmvArgs, SpmvArgs, IrPtrs, const FusedCta*);
using IrFusedTwo = StagedCfg<12, 3, 16384, 2>;
using IrFusedThree = StagedCfg<12, 4, 16384, 3>;

template <class CFG, bool D16, bool RS>
IrFusedFn ir_fused_fn_u(int U) {
  switch (staged_width(U)) {
    case 9: return ir_fused<CFG, 9, D16, RS>;
    case 8: return ir_fused<CFG, 8, D16, RS>;
    case 7: return ir_fused<CFG, 7, D16, RS>;
    case 5: return ir_fused<CFG, 5, D16, RS>;
    default: return ir_fused<CFG, 4, D16, RS>;
  }
}
template <class CFG, bool RS>
IrFusedFn ir_fused_fn(const SolverProduct& p) {
  return p.d16 ? ir_fused_fn_u<CFG, true, RS>(p.w) : ir_fused_fn_u<CFG, false, RS>(p.w);
}

__global__ void to_float(const double* __restrict__ in, float* __restrict__ out,
                         int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

using K1 = void (*)(SpmvArgs, IrPtrs, cudaGraphConditionalHandle);
using KR = void (*)(SpmvArgs, IrPtrs);

// Widths: vector CSR lanes per row (1..32), SELL-32 loads in flight per
// lane (1..16), staged gathers in flight per lane (4 or 8).
template <int KIND, bool D16, bool H>
K1 pick_k1(int W) {
  if constexpr (KIND == 2) {
    switch (staged_width(W)) {
      case 8: return ir_spmv_dot_staged<8, D16, H>;
      case 9: return ir_spmv_dot_staged<9, D16, H>;
      case 7: return ir_spmv_dot_staged<7, D16, H>;
      case 5: return ir_spmv_dot_staged<5, D16, H>;
      default: return ir_spmv_dot_staged<4, D16, H>;
    }
  } else {
    switch (W) {
      case 1: return ir_spmv_dot<1, KIND, D16, H>;
      case 2: return ir_spmv_dot<2, KIND, D16, H>;
      case 4: return ir_spmv_dot<4, KIND, D16, H>;
      case 8: return ir_spmv_dot<8, KIND, D16, H>;
      case 16: return ir_spmv_dot<16, KIND, D16, H>;
      case 32: if (KIND == 0) return ir_spmv_dot<32, KIND, D16, H>;
    }
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: unsupported product width");
}
template <int KIND, bool D16>
KR pick_kr(int W) {
  if constexpr (KIND == 2) {
    switch (staged_width(W)) {
      case 8: return ir_residual_staged<8, D16>;
      case 9: return ir_residual_staged<9, D16>;
      case 7: return ir_residual_staged<7, D16>;
      case 5: return ir_residual_staged<5, D16>;
      default: return ir_residual_staged<4, D16>;
    }
  } else {
    switch (W) {
      case 1: return ir_residual<1, KIND, D16>;
      case 2: return ir_residual<2, KIND, D16>;
      case 4: return ir_residual<4, KIND, D16>;
      case 8: return ir_residual<8, KIND, D16>;
      case 16: return ir_residual<16, KIND, D16>;
      case 32: if (KIND == 0) return ir_residual<32, KIND, D16>;
    }
  }
  fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: unsupported product width");
}
template <bool H>
K1 k1_fn_h(const SolverProduct& p) {
  switch (p.kind) {
    case ProductKind::Vector: return p.d16 ? pick_k1<0, true, H>(p.w) : pick_k1<0, false, H>(p.w);
    case ProductKind::Sell: return p.d16 ? pick_k1<1, true, H>(p.w) : pick_k1<1, false, H>(p.w);
    case ProductKind::Staged: return p.d16 ? pick_k1<2, true, H>(p.w) : pick_k1<2, false, H>(p.w);
  }
  fail(SPMV_ERROR_INTERNAL, "spmv: unknown product kind");
}
K1 k1_fn(const SolverProduct& p, bool handle) {
  return handle ? k1_fn_h<true>(p) : k1_fn_h<false>(p);
}
KR kr_fn(const SolverProduct& p) {
  switch (p.kind) {
    case ProductKind::Vector: return p.d16 ? pick_kr<0, true>(p.w) : pick_kr<0, false>(p.w);
    case ProductKind::Sell: return p.d16 ? pick_kr<1, true>(p.w) : pick_kr<1, false>(p.w);
    case ProductKind::Staged: return p.d16 ? pick_kr<2, true>(p.w) : pick_kr<2, false>(p.w);
  }
  fail(SPMV_ERROR_INTERNAL, "spmv: unknown product kind");
}

// Bytes per entry of a product's matrix stream (value + index).
int entry_bytes(const SolverProduct& p, bool fp32) {
  return (fp32 ? 4 : 8) + (p.d16 ? 2 : 4);
}
const DevCsr::StagedTable& ir_tiles(spmv_matrix A, const SolverProduct& p, bool fp32) {
  const int eb = entry_bytes(p, fp32);
  return staged_table(A->fwd, eb, SolverStaged::max_entries(eb));
}

// Launch shape of a product kernel: vector/SELL use the launch table's CTAs
// (256 threads); staged runs persistent CTAs with dynamic shared memory.
struct KShape {
  int grid, block, smem;
};
KShape k_shape(const void* fn, const void* fn_graph, const SolverProduct& p, bool fp32,
               const SpmvArgs& a, int ntiles, int num_sms) {
  if (p.kind != ProductKind::Staged) return {a.nblocks, 256, 0};
  const StagedShape sh = staged_shape(fn, entry_bytes(p, fp32), ntiles, num_sms);
  if (fn_graph && fn_graph != fn)
    SPMVB_CUDA(cudaFuncSetAttribute(fn_graph, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    sh.smem));
  return {sh.grid, SolverStaged::BS, sh.smem};
}

IrPtrs ir_ptrs(IrWorkspace& w) {
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
  c.tiles32 = w.tiles32;
  c.tiles64 = w.tiles64;
  c.ntiles32 = w.ntiles32;
  c.ntiles64 = w.ntiles64;
  c.bar = w.bar.as<unsigned long long>();
  c.wait_ns = fused_wait_ns();
  return c;
}

void add_kernel(cudaGraphNode_t* node, cudaGraph_t g, const cudaGraphNode_t* dep,
                size_t ndep, void* fn, int grid, int block, void** args, int smem = 0) {
  cudaKernelNodeParams kp{};
  kp.func = fn;
  kp.gridDim = dim3(grid);
  kp.blockDim = dim3(block);
  kp.sharedMemBytes = unsigned(smem);
  kp.kernelParams = args;
  SPMVB_CUDA(cudaGraphAddKernelNode(node, g, dep, ndep, &kp));
}

// Launch tables of the FP32 product over p and the FP64 residual product
// over x (global layout).
void ir_args(spmv_matrix A, IrWorkspace& w, const SolverProduct& p, bool fp32, SpmvArgs& a) {
  spmv_comm comm = A->comm;
  const int P = comm->size;
  const spmv_l2gmap rm = A->row_map;
  std::vector<const void*> xs(P), own(P);
  std::vector<void*> ys(P);
  for (int r = 0; r < P; ++r) {
    if (fp32) {
      xs[r] = w.p.as<float>();
      own[r] = w.p.as<float>() + rm->ranges[r];
      ys[r] = w.y.as<float>() + rm->ranges[r];
    } else {
      xs[r] = w.x.as<double>();
      ys[r] = w.r64.as<double>() + rm->ranges[r];
    }
  }
  const DevCsr& C = A->fwd;
  const int mb = max_blocks_for(comm->num_sms, 256);
  const size_t es = fp32 ? sizeof(float) : sizeof(double);
  const void* const* xown = fp32 ? own.data() : nullptr;
  if (p.sell_layout()) {
    fill_sell_args(a, C, C.sell_cols_global.as<int32_t>(),
                   fp32 ? C.sell_vals32.ptr : C.sell_vals.ptr, es, xs.data(), ys.data(), xown,
                   256, mb);
  } else {
    fill_spmv_args(a, C, C.cols_global.as<int32_t>(), es, xs.data(), ys.data(), xown,
                   256 / p.w, mb);
    if (fp32)
      for (int r = 0; r < P; ++r) a.part[r].vals = C.vals32.as<float>() + C.parts[r].nz_off;
  }
  if (p.d16) use_d16(a, C, p.sell_layout());
}

void build_ir_graph(spmv_matrix A, IrWorkspace& w) {
  spmv_comm comm = A->comm;
  SpmvArgs a32, a64;
  ir_args(A, w, w.p32, true, a32);
  ir_args(A, w, w.p64, false, a64);
  const K1 k1 = k1_fn(w.p32, true);
  const KR kr = kr_fn(w.p64);
  const KShape s1 = k_shape((const void*)k1_fn(w.p32, false), (const void*)k1, w.p32, true, a32,
                            w.ntiles32, comm->num_sms);
  const KShape sr = k_shape((const void*)kr, nullptr, w.p64, false, a64, w.ntiles64,
                            comm->num_sms);
  const int ew_grid = std::max(1, comm->num_sms) * (2048 / EW);
  w.partials.reserve(sizeof(double) * 2 * std::max({s1.grid, sr.grid, ew_grid}));
  IrPtrs c = ir_ptrs(w);

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
    add_kernel(&b1, body, nullptr, 0, (void*)k1, s1.grid, s1.block, args, s1.smem);
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
    add_kernel(&r2, rbody, &r1, 1, (void*)kr, sr.grid, sr.block, a2, sr.smem);
    void* a3[] = {&c};
    add_kernel(&r3, rbody, &r2, 1, (void*)ir_resync, ew_grid, EW, a3);
  }
  {
    void* args[] = {&c, &w.h_loop};
    add_kernel(&b3, body, &b_if, 1, (void*)ir_update_p, ew_grid, EW, args);
  }
  SPMVB_CUDA(cudaGraphInstantiate(&w.exec, w.graph, 0));
}

// Fused plans over the FP32 product's tiles: shape CFG (CFG::MINB CTAs per
// SM), the CTA's rows of r in shared memory (RS) or in global memory.
template <class CFG, bool RS>
bool ir_plan(spmv_matrix A, const IrWorkspace& w, FusedPlan& plan) {
  static_assert(CFG::max_entries(6) == SolverStaged::max_entries(6) &&
                    CFG::max_entries(8) == SolverStaged::max_entries(8),
                "the fused shape uses the solver product's tiles");
  const int eb = entry_bytes(w.p32, true);
  return fused_plan(A, ir_tiles(A, w.p32, true), (const void*)ir_fused_fn<CFG, RS>(w.p32),
                    CFG::BS, CFG::MINB, CFG::smem_bytes(eb), RS ? 4 : 0, plan);
}

void ir_use_plan(IrWorkspace& w, const FusedPlan& plan) {
  w.fused = true;
  w.fused_fn = plan.fn;
  w.fused_grid = plan.grid;
  w.fused_block = plan.block;
  w.fused_smem = plan.smem;
  w.fused_cps = plan.cps;
  w.fused_rs = plan.rs;
  w.fpartials.reserve(sizeof(double) * 6 * size_t(plan.grid));  // 2 arrays of 3 per CTA
  w.ctas.reserve(sizeof(FusedCta) * plan.ctas.size());
  SPMVB_CUDA(cudaMemcpy(w.ctas.ptr, plan.ctas.data(), sizeof(FusedCta) * plan.ctas.size(),
                        cudaMemcpyHostToDevice));
}

// One solve as ir_run enqueues it: kmax, rtol^2, delta^2 and the error
// flag, then the fused launch or the graph.
void ir_enqueue(IrWorkspace& w, cudaStream_t s) {
  IrState* st = w.state.as<IrState>();
  SPMVB_CUDA(cudaMemcpyAsync(&st->kmax, &w.host.kmax, sizeof(int), cudaMemcpyHostToDevice, s));
  SPMVB_CUDA(cudaMemcpyAsync(&st->rtol2, &w.host.rtol2, 2 * sizeof(double),
                             cudaMemcpyHostToDevice, s));
  if (w.fused) {
    const size_t g = size_t(w.fused_grid);
    require(w.fpartials.bytes >= 6 * g * sizeof(double) &&
                w.ctas.bytes >= g * sizeof(FusedCta) && w.tiles32 != nullptr,
            "spmv: fused mixed CG buffers smaller than its grid");
    SPMVB_CUDA(cudaMemsetAsync(&st->stage_err, 0, sizeof(int), s));
    SPMVB_CUDA(cudaMemsetAsync(w.bar.ptr, 0, sizeof(unsigned long long), s));
    IrPtrs c = ir_ptrs(w);
    c.partials = w.fpartials.as<double>();
    const FusedCta* ctas = w.ctas.as<FusedCta>();
    void* args[] = {&w.fa32, &w.fa64, &c, &ctas};
    const cudaError_t e = cudaLaunchCooperativeKernel(
        w.fused_fn, dim3(w.fused_grid), dim3(w.fused_block), args, size_t(w.fused_smem), s);
    if (e != cudaErrorCooperativeLaunchTooLarge) {
      SPMVB_CUDA(e);
      return;
    }
    // The grid no longer fits on the device at once: this solve and the
    // later ones run in the graph form (the refused launch ran nothing).
    (void)cudaGetLastError();
    w.fused = false;
  }
  SPMVB_CUDA(cudaGraphLaunch(w.exec, s));
}

__global__ void ir_fill(double* v, int64_t n, double value) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    v[i] = value;
}

// Device time of a solve of `its` inner iterations in the current form
// (b = 1, no convergence test can pass, delta2 = 0: no refinement but the
// one the iteration cap forces), best of three.
float ir_time(IrWorkspace& w, cudaStream_t s, int its) {
  w.host.kmax = its;
  w.host.rtol2 = 0.0;
  w.host.delta2 = 0.0;
  cudaEvent_t e0, e1;
  SPMVB_CUDA(cudaEventCreate(&e0));
  SPMVB_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    SPMVB_CUDA(cudaEventRecord(e0, s));
    ir_enqueue(w, s);
    SPMVB_CUDA(cudaEventRecord(e1, s));
    SPMVB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SPMVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best = std::min(best, ms);
  }
  SPMVB_CUDA(cudaEventDestroy(e0));
  SPMVB_CUDA(cudaEventDestroy(e1));
  SPMVB_CUDA(cudaMemcpy(&w.host, w.state.ptr, sizeof(IrState), cudaMemcpyDeviceToHost));
  if (w.host.stage_err)
    fail(SPMV_ERROR_CUDA, "spmv: a bounded wait of the fused mixed CG solve timed out");
  return best;
}

// Chooses between the graph form and the fused plans that fit (the FP32
// product must be staged) by timing each: s = device time per inner
// iteration (a 40-iteration solve less an 8-iteration one, over 32) and
// F = the rest of the 8-iteration solve (launch, init and the refinement the
// cap forces), scored s + F / 100: solves to 1e-10 refine about once per
// 50..250 inner iterations.  The candidates are two
// CTAs per SM of 3 stages with r in shared or global memory, or three of 4
// stages (the graph form's product shape) with r in global memory.
// SPMV_B200_CG_MIXED_FUSED: "0" keeps the graph form; "2:smem", "2:global"
// or "3:global" forces that plan, failing if it does not fit.
void ir_choose_form(spmv_matrix A, IrWorkspace& w) {
  w.fused = false;
  if (w.p32.kind != ProductKind::Staged || w.n == 0) return;
  const char* env = std::getenv("SPMV_B200_CG_MIXED_FUSED");
  const std::string mode = env ? env : "";
  if (mode == "0") return;
  spmv_comm comm = A->comm;
  int coop = 0;
  SPMVB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, comm->device));
  if (!coop) return;
  if (!ir_tiles(A, w.p32, true).ok) return;
  w.bar.reserve(sizeof(unsigned long long));
  ir_args(A, w, w.p32, true, w.fa32);
  SolverProduct s64 = w.p32;  // the FP64 residual walks the same SELL slices
  ir_args(A, w, s64, false, w.fa64);
  if (!mode.empty()) {
    FusedPlan p;
    bool fits = false;
    if (mode == "2:smem") fits = ir_plan<IrFusedTwo, true>(A, w, p);
    else if (mode == "2:global") fits = ir_plan<IrFusedTwo, false>(A, w, p);
    else if (mode == "3:global") fits = ir_plan<IrFusedThree, false>(A, w, p);
    require(fits, "spmv: SPMV_B200_CG_MIXED_FUSED must be 0 or a fused plan that fits this "
                  "matrix (2:smem, 2:global, 3:global)");
    ir_use_plan(w, p);
    return;
  }
  std::vector<FusedPlan> plans;
  {
    FusedPlan p1, p2, p3;
    if (ir_plan<IrFusedTwo, true>(A, w, p1)) plans.push_back(std::move(p1));
    if (ir_plan<IrFusedTwo, false>(A, w, p2)) plans.push_back(std::move(p2));
    if (ir_plan<IrFusedThree, false>(A, w, p3)) plans.push_back(std::move(p3));
  }
  if (plans.empty()) return;
  cudaStream_t s = comm->stream;
  SPMVB_CUDA(cudaDeviceSynchronize());
  ir_fill<<<std::max(1, comm->num_sms) * 4, 256, 0, s>>>(w.b.as<double>(), w.n, 1.0);
  SPMVB_CUDA(cudaGetLastError());
  auto score = [&](const char* name) {
    const float t8 = ir_time(w, s, 8), t40 = ir_time(w, s, 40);
    const float per_it = (t40 - t8) / 32.f, fixed = t8 - 8.f * per_it;
    debug_log(std::string("cg_mixed form ") + name + ": " + std::to_string(per_it * 1e3f) +
              " us per inner iteration, " + std::to_string(fixed * 1e3f) +
              " us per solve + refinement");
    return per_it + fixed / 100.f;
  };
  float best = score("graph");
  int pick = -1;
  for (size_t i = 0; i < plans.size(); ++i) {
    ir_use_plan(w, plans[i]);
    const std::string name = "fused " + std::to_string(plans[i].cps) +
                             (plans[i].rs ? ":smem" : ":global");
    const float t = score(name.c_str());
    if (!w.fused) continue;  // the plan's launch was refused (graph form ran)
    if (t < best) {
      best = t;
      pick = int(i);
    }
  }
  w.fused = false;
  if (pick >= 0) ir_use_plan(w, plans[size_t(pick)]);
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
    SPMVB_CUDA(cudaMemset(w->p.ptr, 0, 4 * n1));
    SPMVB_CUDA(cudaMemset(w->x.ptr, 0, 8 * n1));
    // Each product (FP32 inner, FP64 residual) is the candidate whose own
    // kernel (timed outside the graph) is fastest on this matrix; the FP64
    // choice does not carry over, FP32 rows being half the bytes.
    prepare_solver_layouts(A, true);
    w->partials.reserve(sizeof(double) * 2 *
                        std::max(max_blocks_for(A->comm->num_sms, 256),
                                 std::max(1, A->comm->num_sms) * 32));
    IrWorkspace& ws = *w;
    const int nsm = A->comm->num_sms;
    auto use_tiles = [&](const SolverProduct& p, bool fp32) {
      const StagedDesc* t = nullptr;
      int nt = 0;
      if (p.kind == ProductKind::Staged) {
        const DevCsr::StagedTable& tab = ir_tiles(A, p, fp32);
        t = tab.desc.as<StagedDesc>();
        nt = tab.ntiles;
      }
      (fp32 ? ws.tiles32 : ws.tiles64) = t;
      (fp32 ? ws.ntiles32 : ws.ntiles64) = nt;
    };
    auto launch = [&](const void* fn, const SolverProduct& p, bool fp32, const SpmvArgs& a,
                      cudaStream_t s) {
      use_tiles(p, fp32);
      IrPtrs c = ir_ptrs(ws);
      const KShape sh = k_shape(fn, nullptr, p, fp32, a, fp32 ? ws.ntiles32 : ws.ntiles64, nsm);
      cudaGraphConditionalHandle none = 0;
      void* args[] = {const_cast<SpmvArgs*>(&a), &c, &none};
      SPMVB_CUDA(cudaLaunchKernel(fn, dim3(sh.grid), dim3(sh.block), args, size_t(sh.smem), s));
    };
    ws.p32 = choose_solver_product(
        A, SPMV_FLOAT32, ws.p.ptr, ws.y.ptr, true,
        [&](const SolverProduct& cd, const SpmvArgs& a, cudaStream_t s) {
          launch((const void*)k1_fn(cd, false), cd, true, a, s);
        });
    ws.p64 = choose_solver_product(
        A, SPMV_FLOAT64, ws.x.ptr, ws.r64.ptr, false,
        [&](const SolverProduct& cd, const SpmvArgs& a, cudaStream_t s) {
          launch((const void*)kr_fn(cd), cd, false, a, s);
        });
    use_tiles(ws.p32, true);
    use_tiles(ws.p64, false);
    build_ir_graph(A, *w);
    ir_choose_form(A, *w);
    A->ir = std::move(w);
  }
  return *A->ir;
}

CgForm ir_form(spmv_matrix A) {
  require(A->ir != nullptr, "spmv: spmv_cg_mixed has not run on this matrix");
  const IrWorkspace& w = *A->ir;
  CgForm f;
  f.fused = w.fused;
  f.cps = w.fused ? w.fused_cps : 0;
  f.rs = w.fused && w.fused_rs;
  return f;
}

SolverProduct ir_product(spmv_matrix A, bool fp32) {
  require(A->ir != nullptr, "spmv: spmv_cg_mixed has not run on this matrix");
  return fp32 ? A->ir->p32 : A->ir->p64;
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
  ir_enqueue(w, s);
  SPMVB_CUDA(cudaMemcpyAsync(&w.host, st, sizeof(IrState), cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
  if (w.host.stage_err)
    fail(SPMV_ERROR_CUDA, "spmv: a bounded wait on the device timed out");
  if (info) {
    info->iterations = w.host.k;
    info->refinements = w.host.refinements;
    info->status = w.host.status;
    info->converged = w.host.converged;
    info->relres = w.host.rr0 > 0 ? std::sqrt(w.host.rr_true / w.host.rr0) : 0.0;
  }
}

}  // namespace spmvb
