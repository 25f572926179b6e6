// Autotuner for the product kernel of a matrix (spmv_matrix_autotune).
//
// Candidates: vector CSR at half, equal and twice the statistics' lane count,
// SELL-32 at 2..16 loads in flight per lane (when its padding is at most 2x
// the nonzeros), each at 128, 256 and 512 threads per CTA; the staged SELL-32
// product at 4 and 8 gathers in flight per lane (its CTA shape is fixed); and
// merge-path.
// Every candidate runs once untimed (building any layout it needs), then
// `reps` times between two CUDA events on the communicator's stream; the
// fastest becomes the matrix's kernel for mult (the solvers time their own
// products over the fused-halo layout).  With SPMV_B200_TUNE_CACHE naming a file, results are cached
// there by matrix statistics (dtype, ranks, rows, nonzeros, longest row,
// SELL padding) and a later matrix with the same statistics skips the timing.
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>

#include "internal.h"

namespace spmvb {

namespace {

std::string tune_key(spmv_matrix A) {
  const DevCsr& C = A->fwd;
  int64_t rows = 0, nnz = 0;
  for (const DevPart& D : C.parts) {
    rows += D.nrows;
    nnz += D.nnz;
  }
  std::ostringstream k;
  k << "v1:" << int(A->dtype) << ":" << C.parts.size() << ":" << rows << ":" << nnz
    << ":" << C.max_row << ":" << C.sell_padded;
  return k.str();
}

bool cache_lookup(const std::string& key, spmv_tune_result* r) {
  const char* path = std::getenv("SPMV_B200_TUNE_CACHE");
  if (!path) return false;
  std::ifstream f(path);
  std::string k;
  int kernel, width, block;
  double us;
  while (f >> k >> kernel >> width >> block >> us)
    if (k == key) {
      r->kernel = spmv_kernel(kernel);
      r->width = width;
      r->block = block;
      r->us = us;
      r->candidates = 0;
      return true;
    }
  return false;
}

void cache_store(const std::string& key, const spmv_tune_result& r) {
  const char* path = std::getenv("SPMV_B200_TUNE_CACHE");
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  f << key << " " << int(r.kernel) << " " << r.width << " " << r.block << " " << r.us
    << "\n";
}

}  // namespace

void autotune(spmv_matrix A, int reps, spmv_tune_result* best) {
  spmv_comm comm = A->comm;
  comm->require_device();
  require(reps >= 1, "spmv: autotune needs reps >= 1");
  DeviceGuard dg(comm->device);
  const std::string key = tune_key(A);
  spmv_tune_result r{};
  if (cache_lookup(key, &r)) {
    A->kernel = r.kernel;
    A->width = r.width;
    A->block = r.kernel == SPMV_KERNEL_STAGED ? 0 : r.block;
    A->kernel_set = false;
    A->cg.reset();
    A->ir.reset();
    if (best) *best = r;
    return;
  }
  const DevCsr& C = A->fwd;
  const int P = comm->size;
  const size_t es = dtype_size(A->dtype);
  // Scratch vectors (zero-filled; the traffic does not depend on values).
  std::vector<int64_t> xo(P), yo(P);
  int64_t xt = 0, yt = 0;
  for (int p = 0; p < P; ++p) {
    xo[p] = xt;
    yo[p] = yt;
    xt += (C.parts[p].ncols + 63) / 64 * 64;
    yt += (C.parts[p].nrows + 63) / 64 * 64;
  }
  DevBuf xbuf, ybuf;
  xbuf.reserve(std::max<int64_t>(xt, 64) * es);
  ybuf.reserve(std::max<int64_t>(yt, 64) * es);
  SPMVB_CUDA(cudaMemset(xbuf.ptr, 0, std::max<int64_t>(xt, 64) * es));
  std::vector<const void*> xs(P);
  std::vector<void*> ys(P);
  for (int p = 0; p < P; ++p) {
    xs[p] = xbuf.as<char>() + xo[p] * es;
    ys[p] = ybuf.as<char>() + yo[p] * es;
  }
  struct Cand {
    spmv_kernel k;
    int w, bs;
  };
  std::vector<Cand> cands;
  const int wa = auto_width(C.mean_row, A->dtype);
  for (int bs : {128, 256, 512}) {
    for (int w : {wa / 2, wa, wa * 2})
      if (w >= 1 && w <= 32 && w * 32 >= 32 && bs / w >= 1)
        cands.push_back({SPMV_KERNEL_VECTOR, w, bs});
    int64_t nnz = 0;
    for (const DevPart& D : C.parts) nnz += D.nnz;
    if (C.sell_padded <= 2 * std::max<int64_t>(nnz, 1))
      for (int u : {2, 4, 8, 16}) cands.push_back({SPMV_KERNEL_SELL, u, bs});
  }
  // Staged and merge-path products are real only.
  const bool cplx = A->dtype == SPMV_COMPLEX64 || A->dtype == SPMV_COMPLEX128;
  if (!cplx) {
    int64_t nnz = 0;
    for (const DevPart& D : C.parts) nnz += D.nnz;
    if (C.sell_padded <= 2 * std::max<int64_t>(nnz, 1))
      for (int u : {4, 8}) cands.push_back({SPMV_KERNEL_STAGED, u, 0});
    if (C.sell_padded <= 2 * std::max<int64_t>(nnz, 1) && exact_staged_width(C.max_row) > 0)
      cands.push_back({SPMV_KERNEL_STAGED, exact_staged_width(C.max_row), 0});
    cands.push_back({SPMV_KERNEL_MERGE, 0, 256});
  }

  cudaStream_t s = comm->stream;
  cudaEvent_t e0, e1;
  SPMVB_CUDA(cudaEventCreate(&e0));
  SPMVB_CUDA(cudaEventCreate(&e1));
  double best_us = 1e300;
  Cand best_c = cands.front();
  for (const Cand& c : cands) {
    if (c.k == SPMV_KERNEL_SELL || c.k == SPMV_KERNEL_STAGED) build_sell(A, A->fwd, s);
    SpmvLaunch L{};
    L.csr = &A->fwd;
    L.cols = C.cols.as<int32_t>();
    L.dtype = A->dtype;
    L.kernel = c.k;
    L.width = c.w;
    L.block = c.bs;
    L.num_sms = comm->num_sms;
    L.carry = &A->fwd.merge_carry;
    L.err = comm->wait_flag();
    L.x = xs.data();
    L.y = ys.data();
    launch_spmv(L, s);
    SPMVB_CUDA(cudaEventRecord(e0, s));
    for (int i = 0; i < reps; ++i) launch_spmv(L, s);
    SPMVB_CUDA(cudaEventRecord(e1, s));
    SPMVB_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    SPMVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    const double us = 1e3 * ms / reps;
    debug_log("autotune " + std::to_string(int(c.k)) + " w=" + std::to_string(c.w) +
              " bs=" + std::to_string(c.bs) + ": " + std::to_string(us) + " us");
    if (us < best_us) {
      best_us = us;
      best_c = c;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  A->kernel = best_c.k;
  A->width = best_c.w;
  A->block = best_c.bs;
  A->kernel_set = false;
  A->cg.reset();
  A->ir.reset();
  r.kernel = best_c.k;
  r.width = best_c.w;
  // Threads per CTA the chosen kernel runs (the staged product's own shape).
  r.block = best_c.k == SPMV_KERNEL_STAGED ? kStagedThreads : best_c.bs;
  r.us = best_us;
  r.candidates = int(cands.size());
  cache_store(key, r);
  if (best) *best = r;
}

}  // namespace spmvb

extern "C" int spmv_matrix_autotune(spmv_matrix A, int reps, spmv_tune_result* best) {
  return spmvb::guard([&] {
    spmvb::require(A != nullptr, "spmv: Matrix is NULL");
    spmvb::autotune(A, reps, best);
  });
}
