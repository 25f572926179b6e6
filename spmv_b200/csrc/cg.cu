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
//
// With a staged product the whole solve can instead run as one cooperative
// launch (cg_fused below: the same three phases per iteration separated by
// grid barriers, the residual held in shared memory); the workspace times
// both forms on the matrix and keeps the faster.
#include <algorithm>
#include <cmath>
#include <cstddef>
#include <cstdlib>
#include <string>
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
  // Fused solve (one cooperative launch; see cg_fused).
  bool fused = false;
  const void* fused_fn = nullptr;
  int fused_grid = 0, fused_block = 0, fused_smem = 0, fused_cps = 0;
  bool fused_rs = false;
  bool fused_mg = false;  // the merged-update form
  spmvb::DevBuf bar, partials2, ctas;
  spmvb::SpmvArgs fused_args;
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
  unsigned long long* bar;  // fused solve: grid barrier counter
  double* partials2;        // fused solve: second reduction's partials
  unsigned long long wait_ns;  // fused solve: bound of each grid wait
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
__global__ void __launch_bounds__(SolverStaged::BS, SolverStaged::MINB)
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

// ---------------------------------------------------------------------------
// Fused solve: the whole of cg (init and every iteration) as one cooperative
// launch of persistent CTAs, each owning a contiguous run of the staged
// tiles and so a contiguous range [g0, g1) of the global rows.  Per
// iteration, with grid barriers between the phases:
//
//   A  y = A p over the CTA's tiles (the staged traversal; its producer warp
//      keeps streaming the same tiles pass after pass, so the next pass's
//      first tiles land during B and C), p.y          -> barrier, alpha
//   B  r -= alpha y on the CTA's rows, r.r           -> barrier, beta,
//      count, convergence test (identical in every CTA)
//   C  x += alpha p, p = p beta + r on the CTA's rows -> barrier (A gathers p)
//      (in the last iteration x only)
//
// RS: r lives in shared memory for the whole solve (only this CTA's rows
// ever read it), so it never crosses HBM.  The arithmetic of every vector
// element is the graph form's; the two dot products are summed in a
// different grouping (per-CTA partials over the CTA's rows).
// Phase A of the fused solve for one consumer thread: one pass of the staged
// traversal, y = A p, returning this thread's share of p.y.
template <class CFG, int U, typename CI>
__device__ __forceinline__ double cg_fused_product(const SpmvArgs& a, int count, uint64_t q_base,
                                                StagedLoop<CFG>& pipe,
                                                const unsigned char* smem, int* err,
                                                double* __restrict__ y,
                                                const double* __restrict__ p) {
  const uint64_t keep = l2_policy_keep();
  double acc = 0.0;
  staged_loop_consume<CFG, double, CI, U>(
      a, count, q_base, pipe, smem, err,
      [&](const PartArg& P, int row, double sum) {
        const int g = P.row0 + row;
        st_pol(y + g, sum, keep);
        acc += ld_pol(p + g, keep) * sum;
      },
      XGather<double, true>());
  return acc;
}

// Phase A of the merged-update form: y = A p, and this thread's shares of
// p.y, r.y and y.y (r_at(g): r of the CTA's row g, final for this iteration).
struct Sums3 {
  double py, ry, yy;
};
template <class CFG, int U, typename CI, class RAt>
__device__ __forceinline__ Sums3 cg_fused_product3(const SpmvArgs& a, int count, uint64_t q_base,
                                                   StagedLoop<CFG>& pipe,
                                                   const unsigned char* smem, int* err,
                                                   double* __restrict__ y,
                                                   const double* __restrict__ p, RAt&& r_at) {
  const uint64_t keep = l2_policy_keep();
  Sums3 acc{0.0, 0.0, 0.0};
  staged_loop_consume<CFG, double, CI, U>(
      a, count, q_base, pipe, smem, err,
      [&](const PartArg& P, int row, double sum) {
        const int g = P.row0 + row;
        st_pol(y + g, sum, keep);
        acc.py += ld_pol(p + g, keep) * sum;
        acc.ry += r_at(g) * sum;
        acc.yy += sum * sum;
      },
      XGather<double, true>());
  return acc;
}

// Solver scalars of the fused solve (one copy per CTA, in shared memory,
// written by thread 0 between barriers).
struct FusedScalars {
  double rnorm0, rnorm_old, rnorm_new, alpha, beta, pdoty, rtol2;
  int kmax, k, status, go;
};

// The fused solve after its CTA's set-up, for the NT consumer threads (the
// CTA's first NT): init, then per iteration phase A = product(k) (this
// thread's share of p.y after y = A p over the CTA's rows), B and C with the
// grid barriers between; V rows per thread in flight in the vector phases;
// r_at(g): r of the CTA's global row g.  Thread 0 of CTA 0 writes the final
// state.  Returns false when a bounded wait failed (the error flag is
// raised).
template <int NT, int V, class RAt, class Product>
__device__ __forceinline__ bool cg_fused_solve(const CgPtrs& c, const FusedCta& me,
                                               GridSum<NT>& gs, FusedScalars& sv, RAt&& r_at,
                                               Product&& product) {
  const int tid = int(threadIdx.x);
  auto grid_sum = [&](double v, double* parts, unsigned long long epoch, double* total) {
    return coop_grid_sum<NT>(v, parts, c.bar, epoch * gridDim.x, &c.st->stage_err, c.wait_ns,
                             gs, total);
  };
  // Init: r = p = b, x = 0, rnorm0 = b.b.  Barrier epochs: 1 for the init,
  // 3j+2, 3j+3, 3j+4 for phases A, B, C of iteration j.
  double acc = 0.0;
  {
    const uint64_t keep = l2_policy_keep();
    const int g1 = me.g1;
    for (int g = me.g0 + tid; g < g1; g += NT) {
      const double bi = c.b[g];
      r_at(g) = bi;
      st_pol(c.p + g, bi, keep);
      st_pol(c.x + g, 0.0, keep);
      acc += bi * bi;
    }
  }
  double rnorm0 = 0.0;
  bool ok = grid_sum(acc, c.partials2, 1, &rnorm0);
  if (tid == 0) {
    sv.rtol2 = *static_cast<volatile double*>(&c.st->rtol2);
    sv.kmax = *static_cast<volatile int*>(&c.st->kmax);
    sv.rnorm0 = sv.rnorm_old = sv.rnorm_new = rnorm0;
    sv.alpha = sv.beta = sv.pdoty = 0.0;
    sv.k = 0;
    sv.status = SPMV_SUCCESS;
    sv.go = ok && sv.kmax > 0 && rnorm0 > 0.0 && isfinite(rnorm0);
  }
  named_sync(1, NT);
  int k = 0;
  while (sv.go) {
    // A: y = A p, p.y.
    acc = product(k);
    double pdoty = 0.0;
    if (!grid_sum(acc, c.partials, 3ull * unsigned(k) + 2, &pdoty)) {
      ok = false;
      break;
    }
    const bool broke = pdoty == 0.0 || !isfinite(pdoty);

    // B: r -= alpha y, r.r (skipped after a breakdown; r is read when used).
    acc = 0.0;
    if (!broke) {
      const double alpha = sv.rnorm_old / pdoty;
      const uint64_t keep = l2_policy_keep();
      const int g1 = me.g1;
      for (int g0 = me.g0 + tid; g0 < g1; g0 += V * NT) {
        double yv[V];
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) yv[u] = ld_pol(c.y + g, keep);
        }
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            const double ri = r_at(g) - alpha * yv[u];
            r_at(g) = ri;
            acc += ri * ri;
          }
        }
      }
    }
    double rr = 0.0;
    if (!grid_sum(acc, c.partials2, 3ull * unsigned(k) + 3, &rr)) {
      ok = false;
      break;
    }
    // alpha, beta, the count and the convergence test (one thread; every
    // CTA computes the same from the same totals).
    if (tid == 0) {
      sv.k = k + 1;
      sv.pdoty = pdoty;
      sv.alpha = sv.rnorm_old / pdoty;
      if (broke) {
        sv.status = SPMV_ERROR_BREAKDOWN;
        sv.go = false;
      } else {
        sv.rnorm_new = rr;
        sv.beta = rr / sv.rnorm_old;
        sv.rnorm_old = rr;
        const bool converged = rr / sv.rnorm0 < sv.rtol2;
        sv.go = !converged && k + 1 < sv.kmax;
      }
    }
    named_sync(1, NT);
    k += 1;
    if (broke) break;

    // C: x += alpha p (this iteration's alpha and p), then, unless the solve
    // stops here, p = p beta + r.
    {
      const double alpha = sv.alpha, beta = sv.beta;
      const bool go = sv.go;
      const uint64_t keep = l2_policy_keep();
      const int g1 = me.g1;
      for (int g0 = me.g0 + tid; g0 < g1; g0 += V * NT) {
        double pv[V], xv[V];
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            pv[u] = ld_pol(c.p + g, keep);
            xv[u] = ld_pol(c.x + g, keep);
          }
        }
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            st_pol(c.x + g, xv[u] + alpha * pv[u], keep);
            if (go) st_pol(c.p + g, pv[u] * beta + r_at(g), keep);
          }
        }
      }
      if (!go) break;
    }
    if (!coop_grid_barrier<NT>(c.bar, (3ull * unsigned(k) + 1) * gridDim.x, &c.st->stage_err,
                               c.wait_ns, gs)) {
      ok = false;
      break;
    }
  }
  if (tid == 0 && ok && blockIdx.x == 0) {
    CgState* st = c.st;
    st->rnorm0 = sv.rnorm0;
    st->rnorm_old = sv.rnorm_old;
    st->rnorm_new = sv.rnorm_new;
    st->alpha = sv.alpha;
    st->beta = sv.beta;
    st->pdoty = sv.pdoty;
    st->k = sv.k;
    st->status = sv.status;
  }
  return ok;
}

// The merged-update form of the fused solve: two grid syncs per iteration
// instead of three.  Entering iteration k, r_k, p_k and x_k are final and
// each CTA holds its share of rr_k = r_k.r_k, summed when r_k was formed.
//   A  y = A p_k with p.y, r.y and y.y in the product's epilogue; one grid
//      sum of the four with rr_k.  Every CTA then stops when k > 0 and
//      rr_k / rr_0 < rtol^2 (x = x_k after k iterations: cg.cpp's test after
//      its k-th update) or when k = kmax; otherwise alpha = rr_k / p.y and
//      beta = rr' / rr_k with rr' = rr_k - 2 alpha r.y + alpha^2 y.y, which
//      is r_{k+1}.r_{k+1} in exact arithmetic.  rr' is formed from this
//      iteration's true rr_k, so its rounding does not carry over: the
//      stopping test and the next alpha use the true r.r summed in C.
//   C  r -= alpha y, x += alpha p, p = p beta + r on the CTA's rows (the same
//      arithmetic per element as the three-sync form), and the CTA's share
//      of r.r -> grid barrier (A gathers p).
// The solve runs one product more than the three-sync form: the one whose
// sums carry the final r.r.
template <int NT, int V, class RAt, class Product>
__device__ __forceinline__ bool cg_fused_solve_merged(const CgPtrs& c, const FusedCta& me,
                                                      GridSum<NT>& gs, GridSumN<NT, 4>& g4,
                                                      FusedScalars& sv, RAt&& r_at,
                                                      Product&& product) {
  const int tid = int(threadIdx.x);
  // Init: r = p = b, x = 0, rr_0 = b.b.  Barrier epochs: 1 for the init,
  // 2k + 2 for iteration k's sum and 2k + 3 for its closing barrier.
  double rr_part = 0.0;
  {
    const uint64_t keep = l2_policy_keep();
    const int g1 = me.g1;
    for (int g = me.g0 + tid; g < g1; g += NT) {
      const double bi = c.b[g];
      r_at(g) = bi;
      st_pol(c.p + g, bi, keep);
      st_pol(c.x + g, 0.0, keep);
      rr_part += bi * bi;
    }
  }
  double rnorm0 = 0.0;
  bool ok = coop_grid_sum<NT>(rr_part, c.partials2, c.bar, gridDim.x, &c.st->stage_err,
                              c.wait_ns, gs, &rnorm0);
  if (tid == 0) {
    sv.rtol2 = *static_cast<volatile double*>(&c.st->rtol2);
    sv.kmax = *static_cast<volatile int*>(&c.st->kmax);
    sv.rnorm0 = sv.rnorm_old = sv.rnorm_new = rnorm0;
    sv.alpha = sv.beta = sv.pdoty = 0.0;
    sv.k = 0;
    sv.status = SPMV_SUCCESS;
    sv.go = ok && sv.kmax > 0 && rnorm0 > 0.0 && isfinite(rnorm0);
  }
  named_sync(1, NT);
  int k = 0;
  while (sv.go) {
    // A: y = A p, the four sums.
    const Sums3 s3 = product(k);
    const double in[4] = {s3.py, s3.ry, s3.yy, rr_part};
    double tot[4];
    if (!coop_grid_sum_n<NT, 4>(in, c.partials, c.bar, (2ull * unsigned(k) + 2) * gridDim.x,
                                &c.st->stage_err, c.wait_ns, g4, tot)) {
      ok = false;
      break;
    }
    // The stopping test, alpha and beta (one thread; every CTA computes the
    // same from the same totals).
    if (tid == 0) {
      const double rr = tot[3];
      if (k > 0) {
        sv.rnorm_new = rr;
        sv.rnorm_old = rr;
      }
      if ((k > 0 && rr / sv.rnorm0 < sv.rtol2) || k >= sv.kmax) {
        sv.go = false;
      } else {
        const double py = tot[0];
        sv.k = k + 1;
        sv.pdoty = py;
        sv.alpha = rr / py;
        if (py == 0.0 || !isfinite(py)) {
          sv.status = SPMV_ERROR_BREAKDOWN;
          sv.go = false;
        } else {
          const double a = sv.alpha;
          const double rr1 = rr - 2.0 * a * tot[1] + a * a * tot[2];
          sv.beta = rr1 / rr;
        }
      }
    }
    named_sync(1, NT);
    if (!sv.go) break;

    // C: r -= alpha y, x += alpha p, p = p beta + r, this CTA's r.r.
    {
      const double alpha = sv.alpha, beta = sv.beta;
      const uint64_t keep = l2_policy_keep();
      const int g1 = me.g1;
      rr_part = 0.0;
      for (int g0 = me.g0 + tid; g0 < g1; g0 += V * NT) {
        double yv[V], pv[V], xv[V];
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            yv[u] = ld_pol(c.y + g, keep);
            pv[u] = ld_pol(c.p + g, keep);
            xv[u] = ld_pol(c.x + g, keep);
          }
        }
#pragma unroll
        for (int u = 0; u < V; ++u) {
          const int g = g0 + u * NT;
          if (g < g1) {
            const double ri = r_at(g) - alpha * yv[u];
            r_at(g) = ri;
            rr_part += ri * ri;
            st_pol(c.x + g, xv[u] + alpha * pv[u], keep);
            st_pol(c.p + g, pv[u] * beta + ri, keep);
          }
        }
      }
    }
    if (!coop_grid_barrier<NT>(c.bar, (2ull * unsigned(k) + 3) * gridDim.x, &c.st->stage_err,
                               c.wait_ns, gs)) {
      ok = false;
      break;
    }
    ++k;
  }
  if (tid == 0 && ok && blockIdx.x == 0) {
    CgState* st = c.st;
    st->rnorm0 = sv.rnorm0;
    st->rnorm_old = sv.rnorm_old;
    st->rnorm_new = sv.rnorm_new;
    st->alpha = sv.alpha;
    st->beta = sv.beta;
    st->pdoty = sv.pdoty;
    st->k = sv.k;
    st->status = sv.status;
  }
  return ok;
}

// MG: the merged-update form (two grid syncs per iteration), else three.
template <class CFG, int U, bool D16, bool RS, bool MG>
__global__ void __launch_bounds__(CFG::BS, CFG::MINB)
    cg_fused(const __grid_constant__ SpmvArgs a, const CgPtrs c,
             const FusedCta* __restrict__ ctas) {
  using CI = typename std::conditional<D16, int16_t, int32_t>::type;
  constexpr int NT = CFG::NC * 32;
  constexpr int STAGES_BYTES = CFG::smem_bytes(8 + int(sizeof(CI)));
  // Rows per thread in flight in the vector phases: as many as the shape's
  // registers hold without spilling.
  constexpr int V = CFG::MINB == 2 ? 4 : CFG::MINB == 3 ? 1 : 2;
  extern __shared__ __align__(128) unsigned char staged_smem[];
  __shared__ StagedLoop<CFG> pipe;
  __shared__ GridSum<NT> gs;
  // The CTA's tiles and rows, and the solver scalars: kept in shared memory,
  // out of the registers the product phase needs.
  __shared__ FusedCta me;
  __shared__ FusedScalars sv;

  const int tid = int(threadIdx.x);
  if (tid == 0) {
    me = ctas[blockIdx.x];
    staged_loop_init(pipe);
  }
  __syncthreads();
  if (tid >= NT) {
    if (tid == NT)
      staged_loop_produce<CFG, double, CI>(a, c.tiles + me.t0, me.t1 - me.t0, pipe,
                                           staged_smem, &c.st->stage_err);
    return;
  }
  // r of global row g (this CTA's rows only when RS).
  auto r_at = [&](int g) -> double& {
    return RS ? reinterpret_cast<double*>(staged_smem + STAGES_BYTES)[g - me.g0] : c.r[g];
  };
  if constexpr (MG) {
    __shared__ GridSumN<NT, 4> g4;
    // One row per thread in flight in the merged update (measured on c2 at
    // two CTAs per SM: 41.1 us per iteration, against 42.9 with two rows and
    // 43.2 with four).
    constexpr int VM = CFG::MINB == 2 ? 1 : V;
    cg_fused_solve_merged<NT, VM>(c, me, gs, g4, sv, r_at, [&](int k) {
      const int count = me.t1 - me.t0;
      return cg_fused_product3<CFG, U, CI>(a, count, uint64_t(k) * uint64_t(count), pipe,
                                           staged_smem, &c.st->stage_err, c.y, c.p, r_at);
    });
  } else {
    cg_fused_solve<NT, V>(c, me, gs, sv, r_at, [&](int k) {
      const int count = me.t1 - me.t0;
      return cg_fused_product<CFG, U, CI>(a, count, uint64_t(k) * uint64_t(count), pipe,
                                          staged_smem, &c.st->stage_err, c.y, c.p);
    });
  }
  if (tid == 0) pipe.stop = 1;
}

using FusedFn = void (*)(SpmvArgs, CgPtrs, const FusedCta*);

// Fused shapes: one CTA per SM (28 consumer warps, 6 stages) or two
// (12 consumer warps, 3 stages each), the rest of shared memory holding r;
// with r in global memory, two CTAs of 6 stages, or three of 4 (the graph
// form's product shape, 48 registers per thread).
using CgFusedOne = StagedCfg<28, 6, 16384>;
using CgFusedTwo = StagedCfg<12, 3, 16384, 2>;
using CgFusedTwoDeep = StagedCfg<12, 6, 16384, 2>;
using CgFusedThree = StagedCfg<12, 4, 16384, 3>;

template <class CFG, bool D16, bool RS, bool MG>
FusedFn fused_fn_u(int U) {
  switch (staged_width(U)) {
    case 8: return cg_fused<CFG, 8, D16, RS, MG>;
    case 9: return cg_fused<CFG, 9, D16, RS, MG>;
    case 7: return cg_fused<CFG, 7, D16, RS, MG>;
    case 5: return cg_fused<CFG, 5, D16, RS, MG>;
    default: return cg_fused<CFG, 4, D16, RS, MG>;
  }
}

template <class CFG, bool RS, bool MG = false>
FusedFn fused_fn(const SolverProduct& sp) {
  return sp.d16 ? fused_fn_u<CFG, true, RS, MG>(sp.w) : fused_fn_u<CFG, false, RS, MG>(sp.w);
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
    case 9: return cg_k1_staged<9, D16, H>;
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
  c.bar = w.bar.as<unsigned long long>();
  c.partials2 = w.partials2.as<double>();
  c.wait_ns = fused_wait_ns();
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

// Staged product: shape CFG (CFG::MINB CTAs per SM).
template <class CFG, bool RS, bool MG = false>
bool plan_fused(spmv_matrix A, const SolverProduct& sp, FusedPlan& plan) {
  static_assert(CFG::max_entries(10) == SolverStaged::max_entries(10) &&
                    CFG::max_entries(12) == SolverStaged::max_entries(12),
                "fused shapes use the solver product's tiles");
  const int eb = 8 + (sp.d16 ? 2 : 4);
  if (!fused_plan(A, cg_tiles(A, sp), (const void*)fused_fn<CFG, RS, MG>(sp), CFG::BS,
                  CFG::MINB, CFG::smem_bytes(eb), RS ? 8 : 0, plan))
    return false;
  plan.merged = MG;
  return true;
}

void use_plan(CgWorkspace& w, FusedPlan& plan) {
  w.fused = true;
  w.fused_fn = plan.fn;
  w.fused_grid = plan.grid;
  w.fused_block = plan.block;
  w.fused_smem = plan.smem;
  w.fused_cps = plan.cps;
  w.fused_rs = plan.rs;
  w.fused_mg = plan.merged;
  // One partial per CTA in each reduction's array (four in partials for the
  // merged form).  partials is baked into the graph form's kernels and never
  // reallocated: it was sized for more CTAs than any plan has.
  require(w.partials.bytes >= sizeof(double) * size_t(plan.grid) * (plan.merged ? 4 : 1),
          "spmv: fused CG grid larger than its partials array");
  w.partials2.reserve(sizeof(double) * size_t(plan.grid));
  w.ctas.reserve(sizeof(FusedCta) * plan.ctas.size());
  SPMVB_CUDA(cudaMemcpy(w.ctas.ptr, plan.ctas.data(), sizeof(FusedCta) * plan.ctas.size(),
                        cudaMemcpyHostToDevice));
}

// One solve as enqueued by cg_run (kmax, rtol^2 and the error flag first).
void enqueue_solve(CgWorkspace& w, cudaStream_t s) {
  CgState* st = w.state.as<CgState>();
  static_assert(offsetof(CgState, stage_err) + sizeof(int) - offsetof(CgState, rtol2) == 32,
                "rtol2 .. stage_err are one contiguous block");
  SPMVB_CUDA(cudaMemcpyAsync(&st->rtol2, &w.host.rtol2, 32, cudaMemcpyHostToDevice, s));
  if (w.fused) {
    const size_t g = size_t(w.fused_grid);
    require(w.partials.bytes >= g * sizeof(double) && w.partials2.bytes >= g * sizeof(double) &&
                w.ctas.bytes >= g * sizeof(FusedCta) && w.tiles != nullptr,
            "spmv: fused CG buffers smaller than its grid");
    SPMVB_CUDA(cudaMemsetAsync(w.bar.ptr, 0, sizeof(unsigned long long), s));
    CgPtrs c = cg_ptrs(w);
    const FusedCta* ctas = w.ctas.as<FusedCta>();
    void* args[] = {&w.fused_args, &c, &ctas};
    const cudaError_t e = cudaLaunchCooperativeKernel(
        w.fused_fn, dim3(w.fused_grid), dim3(w.fused_block), args, size_t(w.fused_smem), s);
    if (e != cudaErrorCooperativeLaunchTooLarge) {
      SPMVB_CUDA(e);
      return;
    }
    // The grid no longer fits on the device at once (a context given fewer
    // SMs than the plan was made for): this solve and the later ones run in
    // the graph form.  The error is a refused launch; nothing ran.
    (void)cudaGetLastError();
    w.fused = false;
  }
  SPMVB_CUDA(cudaGraphLaunch(w.exec, s));
}

__global__ void cg_fill(double* v, int64_t n, double value) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    v[i] = value;
}

// Device time of `its` iterations of the current form (b = 1, no
// convergence test can pass), best of three.
float time_iterations(CgWorkspace& w, cudaStream_t s, int its) {
  w.host.kmax = its;
  w.host.rtol2 = 0.0;
  w.host.stage_err = 0;
  cudaEvent_t e0, e1;
  SPMVB_CUDA(cudaEventCreate(&e0));
  SPMVB_CUDA(cudaEventCreate(&e1));
  float best = 1e30f;
  for (int rep = 0; rep < 4; ++rep) {
    SPMVB_CUDA(cudaEventRecord(e0, s));
    enqueue_solve(w, s);
    SPMVB_CUDA(cudaEventRecord(e1, s));
    SPMVB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SPMVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    if (rep > 0) best = std::min(best, ms);
  }
  SPMVB_CUDA(cudaEventDestroy(e0));
  SPMVB_CUDA(cudaEventDestroy(e1));
  SPMVB_CUDA(cudaMemcpy(&w.host, w.state.ptr, sizeof(CgState), cudaMemcpyDeviceToHost));
  if (w.host.stage_err)
    fail(SPMV_ERROR_CUDA, "spmv::cg - a bounded wait of the fused solve timed out");
  return best;
}

// Chooses between the graph form and the fused plans that fit, by timing 32
// iterations of each on b = 1 (the fused form needs a staged product):
// r in shared memory with one or two CTAs per SM (when the CTAs' rows fit),
// or r in global memory with two CTAs of 6 stages or three of 4; and the
// merged-update form (two grid syncs per iteration) of the 2-CTA shared and
// 3-CTA global plans, whose one extra product per solve weighs 1/32 here.
// SPMV_B200_CG_FUSED: "0" keeps the graph form; "<cps>:<smem|global>[:m]"
// forces that plan (1:smem, 2:smem, 1:global, 2:global, 3:global, 2:smem:m,
// 3:global:m), failing if it does not fit.
void choose_form(spmv_matrix A, CgWorkspace& w) {
  w.fused = false;
  const SolverProduct& sp = w.product;
  if (sp.kind != ProductKind::Staged || w.n == 0) return;
  const char* env = std::getenv("SPMV_B200_CG_FUSED");
  const std::string mode = env ? env : "";
  if (mode == "0") return;
  spmv_comm comm = A->comm;
  int coop = 0;
  SPMVB_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, comm->device));
  if (!coop) return;
  // The fused kernel streams the product's tile table.
  const DevCsr::StagedTable& tiles = cg_tiles(A, sp);
  if (!tiles.ok) return;
  w.tiles = tiles.desc.as<StagedDesc>();
  w.ntiles = tiles.ntiles;
  w.bar.reserve(sizeof(unsigned long long));
  w.fused_args = k1_args(A, w, w.product);

  if (!mode.empty()) {
    FusedPlan p;
    bool fits = false;
    if (mode == "1:smem") fits = plan_fused<CgFusedOne, true>(A, sp, p);
    else if (mode == "2:smem") fits = plan_fused<CgFusedTwo, true>(A, sp, p);
    else if (mode == "1:global") fits = plan_fused<CgFusedOne, false>(A, sp, p);
    else if (mode == "2:global") fits = plan_fused<CgFusedTwoDeep, false>(A, sp, p);
    else if (mode == "3:global") fits = plan_fused<CgFusedThree, false>(A, sp, p);
    else if (mode == "2:smem:m") fits = plan_fused<CgFusedTwo, true, true>(A, sp, p);
    else if (mode == "3:global:m") fits = plan_fused<CgFusedThree, false, true>(A, sp, p);
    require(fits, "spmv: SPMV_B200_CG_FUSED must be 0 or a fused plan that fits this matrix "
                  "(1:smem, 2:smem, 1:global, 2:global, 3:global, 2:smem:m, 3:global:m)");
    use_plan(w, p);
    return;
  }
  std::vector<FusedPlan> plans;
  {
    FusedPlan p1, p2, p3, p4, p5, p6;
    if (plan_fused<CgFusedOne, true>(A, sp, p1)) plans.push_back(std::move(p1));
    if (plan_fused<CgFusedTwo, true>(A, sp, p2)) plans.push_back(std::move(p2));
    if (plan_fused<CgFusedTwoDeep, false>(A, sp, p3)) plans.push_back(std::move(p3));
    if (plan_fused<CgFusedThree, false>(A, sp, p4)) plans.push_back(std::move(p4));
    if (plan_fused<CgFusedTwo, true, true>(A, sp, p5)) plans.push_back(std::move(p5));
    if (plan_fused<CgFusedThree, false, true>(A, sp, p6)) plans.push_back(std::move(p6));
  }
  if (plans.empty()) return;
  cudaStream_t s = A->comm->stream;
  const int its = 32;
  SPMVB_CUDA(cudaDeviceSynchronize());
  cg_fill<<<std::max(1, comm->num_sms) * 4, 256, 0, s>>>(w.b.as<double>(), w.n, 1.0);
  SPMVB_CUDA(cudaGetLastError());
  float best = time_iterations(w, s, its);
  int pick = -1;
  for (size_t i = 0; i < plans.size(); ++i) {
    use_plan(w, plans[i]);
    const float t = time_iterations(w, s, its);
    if (!w.fused) continue;  // the plan's launch was refused (graph form ran)
    if (t < best) {
      best = t;
      pick = int(i);
    }
  }
  w.fused = false;
  if (pick >= 0) use_plan(w, plans[size_t(pick)]);
}

}  // namespace

// Fused solve plans.  The tiles are split into `grid` contiguous runs of
// about n / grid rows each (tile starts are row boundaries, so each run
// covers a contiguous range of global rows); returns the longest run.
int64_t fused_ctas(spmv_matrix A, const DevCsr::StagedTable& t, int grid,
                   std::vector<FusedCta>& out) {
  const std::vector<int64_t>& ranges = A->row_map->ranges;
  const int T = t.ntiles;
  const int64_t n = ranges.back();
  std::vector<int64_t> start(size_t(T) + 1);
  for (int k = 0; k < T; ++k) {
    const DevCsr::StagedTable::Rows& r = t.rows[size_t(k)];
    start[size_t(k)] =
        std::min<int64_t>(ranges[size_t(r.rank)] + int64_t(r.s0) * 32, ranges[size_t(r.rank) + 1]);
  }
  start[size_t(T)] = n;
  out.assign(size_t(grid), FusedCta{});
  int kb = 0;
  int64_t longest = 0;
  for (int b = 0; b < grid; ++b) {
    const int64_t target = n * (b + 1) / grid;
    const int ke = b + 1 == grid
                       ? T
                       : int(std::lower_bound(start.begin() + kb, start.end(), target) -
                             start.begin());
    out[size_t(b)] = {kb, ke, int32_t(start[size_t(kb)]), int32_t(start[size_t(ke)])};
    longest = std::max(longest, start[size_t(ke)] - start[size_t(kb)]);
    kb = ke;
  }
  return longest;
}


bool fused_plan(spmv_matrix A, const DevCsr::StagedTable& t, const void* fn, int block,
                int cps, int64_t stage_smem, int rs_bytes, FusedPlan& plan) {
  if (!fn || !t.ok) return false;
  spmv_comm comm = A->comm;
  const int grid = std::max(1, comm->num_sms) * cps;
  std::vector<FusedCta> ctas;
  const int64_t longest = fused_ctas(A, t, grid, ctas);
  const int64_t smem = stage_smem + (longest * rs_bytes + 15) / 16 * 16;
  int optin = 0;
  SPMVB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin,
                                    comm->device));
  cudaFuncAttributes fa{};
  SPMVB_CUDA(cudaFuncGetAttributes(&fa, fn));
  if (smem + int64_t(fa.sharedSizeBytes) > optin) return false;
  SPMVB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int nb = 0;
  SPMVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, block, size_t(smem)));
  if (nb < cps) return false;
  plan.fn = fn;
  plan.grid = grid;
  plan.block = block;
  plan.smem = int(smem);
  plan.cps = cps;
  plan.rs = rs_bytes > 0;
  plan.ctas = std::move(ctas);
  return true;
}

// A healthy grid wait is microseconds; tests set the limit low to make one
// run out on purpose.
unsigned long long fused_wait_ns() {
  unsigned long long ns = 2000000000ull;
  if (const char* lim = std::getenv("SPMV_B200_WAIT_LIMIT_NS"))
    ns = std::strtoull(lim, nullptr, 10);
  return ns;
}

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
    choose_form(A, ws);
    A->cg = std::move(w);
  }
  return *A->cg;
}

SolverProduct cg_product(spmv_matrix A) {
  require(A->cg != nullptr, "spmv: spmv_cg has not run on this matrix");
  return A->cg->product;
}

CgForm cg_form(spmv_matrix A) {
  require(A->cg != nullptr, "spmv: spmv_cg has not run on this matrix");
  const CgWorkspace& w = *A->cg;
  CgForm f;
  f.fused = w.fused;
  f.cps = w.fused ? w.fused_cps : 0;
  f.rs = w.fused && w.fused_rs;
  f.merged = w.fused && w.fused_mg;
  return f;
}

double* cg_rhs(spmv_matrix A) { return cg_workspace(A).b.as<double>(); }
double* cg_solution(spmv_matrix A) { return cg_workspace(A).x.as<double>(); }

void cg_run(spmv_matrix A, int max_its, double rtol, spmv_cg_info* info) {
  CgWorkspace& w = cg_workspace(A);
  cudaStream_t s = A->comm->stream;
  // kmax and rtol^2 for this solve (cg.cpp:49).
  w.host.kmax = max_its;
  w.host.rtol2 = rtol * rtol;
  w.host.stage_err = 0;
  CgState* st = w.state.as<CgState>();
  enqueue_solve(w, s);
  SPMVB_CUDA(cudaMemcpyAsync(&w.host, st, sizeof(CgState),
                             cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
  if (w.host.stage_err)
    fail(SPMV_ERROR_CUDA, "spmv::cg - a bounded wait on the device timed out");
  if (info) {
    info->iterations = w.host.k;
    info->status = w.host.status;
    info->rnorm0 = w.host.rnorm0;
    info->rnorm = w.host.rnorm_new;
  }
}

}  // namespace spmvb
