// Batched solves: API, device layout, launch and autotuner (no counterpart
// in the reference; the recurrences are spmv::cg's, cg.cpp:50-80, on the
// product of Matrix::operator*, Matrix.cpp:199-204).  The kernel is
// batch_kernel.cuh, the host planning batch_plan.cpp.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>

#include "batch.h"

using spmvb::bat::BW;
using spmvb::bat::LaunchCfg;
using spmvb::bat::NSUM;
using spmvb::bat::Plan;
using spmvb::bat::Slot;
using spmvb::bat::Unit;
using spmvb::bat::UnitState;

struct spmv_batch_s {
  spmv_comm comm = nullptr;
  Plan plan;                      // host view (the big arrays are released after upload)
  int nsys = 0;
  // Block of right-hand sides.
  int block_sys = -1, block_nrhs = 0;
  int32_t block_n = 0, block_npad = 0;
  int64_t block_nnz = 0;
  LaunchCfg cfg[2] = {LaunchCfg{}, LaunchCfg{2, 8, 1, 0}};  // per precision (mixed, FP64)
  int gmax = 0;                   // CTAs of the largest grid (partials are sized for it)
  spmvb::DevBuf units, soff, sbound, vals32, vals64, idx, perm;
  spmvb::DevBuf v32, v64;         // r, p, y, d in FP32 / FP64 (4 x rows_pad)
  spmvb::DevBuf x, b;             // FP64, rows_pad
  spmvb::DevBuf brp, bcol, bval32, bval64, bperm;
  spmvb::DevBuf bv32, bv64, bx, bb;  // block vectors (npad x BW)
  spmvb::DevBuf slots, ust, tickets, parts, bar, err;
  spmvb::DevBuf uptr;             // b and x pointer tables (2 x nsys)
  spmvb::DevBuf stage;            // host-memory solves: b and x staged here
  spmvb::DevBuf prof;             // phase timeline (SPMV_B200_BATCH_PROFILE)
  std::vector<int64_t> part_off;  // per unit
};

namespace spmvb {
namespace bat {
namespace {

unsigned long long wait_ns() {
  unsigned long long ns = 2000000000ull;
  if (const char* lim = std::getenv("SPMV_B200_WAIT_LIMIT_NS")) ns = std::strtoull(lim, nullptr, 10);
  return ns;
}

int tile_slices_of(int tile_rows) { return tile_rows / 32; }

constexpr int kProfCap = 1 << 16;
// Refinement test of the mixed solves: refine when the FP32 residual norm has
// fallen 100x below its largest value since the last refinement (the
// reliable-update criterion with delta = 0.01; squared norms compared).
constexpr double kDelta2 = 1e-4;
// Rows of p the product phase stages per CTA (64 KB in FP32, kept as a ring
// across a pass's chunks; 88 KB in FP64: two CTAs per SM still fit).
constexpr int kWinRows32 = 16384;
static_assert((kWinRows32 & (kWinRows32 - 1)) == 0, "the FP32 window is a ring of 2^k rows");
constexpr int kWinRows64 = 11264;

// With SPMV_B200_BATCH_PROFILE naming a file, each solve appends one line:
// the time between consecutive grid barriers summed per phase (init, A, B,
// C, D), in microseconds, with the number of barriers of each.
void write_profile(spmv_batch B, const char* tag) {
  const char* path = std::getenv("SPMV_B200_BATCH_PROFILE");
  if (!path || !B->prof.ptr) return;
  std::vector<unsigned long long> h(2 * kProfCap + 16 + 3 * 1024);
  SPMVB_CUDA(cudaMemcpy(h.data(), B->prof.ptr, sizeof(unsigned long long) * h.size(),
                        cudaMemcpyDeviceToHost));
  double us[6] = {0, 0, 0, 0, 0, 0};
  int cnt[6] = {0, 0, 0, 0, 0, 0};
  unsigned long long prev = h[1];
  for (int e = 1; e < kProfCap; ++e) {
    const unsigned long long t = h[2 * e + 1];
    if (t == 0) break;
    const int code = int(h[2 * e]);
    if (code >= 0 && code < 6) {
      us[code] += 1e-3 * double(t - prev);
      cnt[code] += 1;
    }
    prev = t;
  }
  std::ofstream f(path, std::ios::app);
  f << "{\"solve\": \"" << tag << "\", \"init_us\": " << us[1] << ", \"A_us\": " << us[2]
    << ", \"B_us\": " << us[3] << ", \"C_us\": " << us[4] << ", \"D_us\": " << us[5]
    << ", \"iterations\": " << cnt[2] << ", \"refining_iterations\": " << cnt[5];
  // Product phase, summed over CTAs and iterations (divide by the CTA-phase
  // count for a mean per CTA and phase): window bounds, window load, tiles.
  const unsigned long long* sub = h.data() + 2 * kProfCap;
  const double n = sub[5] ? double(sub[5]) : 1.0;
  f << ", \"A_cta_mean_us\": {\"bounds\": " << 1e-3 * sub[0] / n << ", \"load\": "
    << 1e-3 * sub[1] / n << ", \"tiles\": " << 1e-3 * sub[2] / n << ", \"total\": "
    << 1e-3 * sub[3] / n << ", \"max_total\": " << 1e-3 * sub[4] << "}";
  // Per-CTA time in phases A, B, C (microseconds, summed over the solve).
  const unsigned long long* pc = sub + 16;
  const char* names[3] = {"A", "B", "C"};
  for (int ph = 0; ph < 3; ++ph) {
    f << ", \"cta_" << names[ph] << "_us\": [";
    for (int c = 0; c < 2 * B->comm->num_sms && c < 1024; ++c)
      f << (c ? ", " : "") << int64_t(1e-3 * pc[ph * 1024 + c]);
    f << "]";
  }
  f << "}\n";
}

void upload(DevBuf& buf, const void* src, size_t bytes) {
  buf.reserve(std::max<size_t>(bytes, 16));
  if (bytes) SPMVB_CUDA(cudaMemcpy(buf.ptr, src, bytes, cudaMemcpyHostToDevice));
}

int nunits_of(const spmv_batch_s* B, bool with_block) { return B->nsys + (with_block ? 1 : 0); }

// Unit table (singles, then the block when the batch has one).
void build_units(spmv_batch B) {
  const Plan& P = B->plan;
  const int nu = nunits_of(B, B->block_sys >= 0);
  std::vector<Unit> U(std::max(nu, 1));
  B->part_off.assign(nu, 0);
  int64_t off = 0;
  for (int i = 0; i < B->nsys; ++i) {
    Unit& u = U[i];
    u.row0 = P.row0[i];
    u.slice0 = P.slice0[i];
    u.n = P.n[i];
    u.nslices = (P.n[i] + 31) / 32;
    u.kind = 0;
    u.slot0 = i;
    u.sys = i;
    u.pad = 0;
    u.part_off = off;
    B->part_off[i] = off;
    off += int64_t(B->gmax) * NSUM;
  }
  if (B->block_sys >= 0) {
    Unit& u = U[B->nsys];
    u.row0 = 0;
    u.slice0 = 0;
    u.n = B->block_n;
    u.nslices = B->block_npad;
    u.kind = 1;
    u.slot0 = B->nsys;
    u.sys = B->block_sys;
    u.pad = 0;
    u.part_off = off;
    B->part_off[B->nsys] = off;
    off += int64_t(B->gmax) * NSUM * BW;
  }
  upload(B->units, U.data(), sizeof(Unit) * U.size());
  B->parts.reserve(sizeof(double) * std::max<int64_t>(off, 1));
  const int nslot = B->nsys + (B->block_sys >= 0 ? BW : 0);
  B->slots.reserve(sizeof(Slot) * std::max(nslot, 1));
  B->ust.reserve(sizeof(UnitState) * std::max(nu, 1));
  B->tickets.reserve(sizeof(unsigned int) * std::max(nu, 1));
  SPMVB_CUDA(cudaMemset(B->tickets.ptr, 0, sizeof(unsigned int) * std::max(nu, 1)));
}

// Device layout of one solve precision (vectors allocated on first use).
template <typename T>
void vectors(spmv_batch B, T*& r, T*& p, T*& y, T*& d, T*& rB, T*& pB, T*& yB, T*& dB) {
  const int64_t n = std::max<int64_t>(B->plan.rows_pad, 32);
  DevBuf& v = sizeof(T) == 4 ? B->v32 : B->v64;
  if (!v.ptr) {
    v.reserve(4 * sizeof(T) * size_t(n));
    SPMVB_CUDA(cudaMemset(v.ptr, 0, 4 * sizeof(T) * size_t(n)));
  }
  T* base = v.as<T>();
  r = base;
  p = base + n;
  y = base + 2 * n;
  d = base + 3 * n;
  rB = pB = yB = dB = nullptr;
  if (B->block_sys >= 0) {
    const int64_t nb = int64_t(std::max(B->block_npad, 16)) * BW;
    DevBuf& bv = sizeof(T) == 4 ? B->bv32 : B->bv64;
    if (!bv.ptr) {
      bv.reserve(4 * sizeof(T) * size_t(nb));
      SPMVB_CUDA(cudaMemset(bv.ptr, 0, 4 * sizeof(T) * size_t(nb)));
    }
    T* bb = bv.as<T>();
    rB = bb;
    pB = bb + nb;
    yB = bb + 2 * nb;
    dB = bb + 3 * nb;
  }
}

struct SolveIo {
  const double* const* b_user;  // device pointer table
  double* const* x_user;
  const double* B_user;
  double* X_user;
  bool with_block;
};

template <typename T, typename CI>
void fill_args(spmv_batch B, Args<T, CI>& a, const SolveIo& io, int kmax, double rtol,
               double delta2, const LaunchCfg& cfg, bool dry) {
  a = Args<T, CI>{};
  a.units = B->units.as<Unit>();
  a.nunits = nunits_of(B, io.with_block);
  a.kmax = kmax;
  a.rtol2 = rtol * rtol;
  a.delta2 = delta2;
  a.tile_slices = cfg.tile_slices;
  // Tile weights against a single unit's tile (8), per phase, from per-CTA
  // phase times on the batched k-NN workload: in FP32 a block tile costs
  // 0.5x a single tile in the product, 1.5x in the alpha update, 1.25x in
  // the p update; a refinement tile (FP64 product and three sums) 48x a
  // p-update tile.
  a.w = sizeof(T) == 4 ? Weights{4, 12, 10, 128, 384} : Weights{8, 8, 10, 128, 384};
  a.nrhs = io.with_block ? B->block_nrhs : 0;
  a.soff = B->soff.as<int64_t>();
  a.sbound = B->sbound.as<int2>();
  a.win_cap = cfg.window ? (sizeof(T) == 4 ? kWinRows32 : kWinRows64) : 0;
  a.vals = sizeof(T) == 4 ? reinterpret_cast<const T*>(B->vals32.ptr)
                          : reinterpret_cast<const T*>(B->vals64.ptr);
  a.vals64 = B->vals64.as<double>();
  a.idx = B->idx.as<CI>();
  a.perm = B->perm.as<int32_t>();
  if (!dry) vectors<T>(B, a.r, a.p, a.y, a.d, a.rB, a.pB, a.yB, a.dB);
  a.x = B->x.as<double>();
  a.b = B->b.as<double>();
  if (B->block_sys >= 0) {
    a.brp = B->brp.as<int32_t>();
    a.bcol = B->bcol.as<int32_t>();
    a.bval = sizeof(T) == 4 ? reinterpret_cast<const T*>(B->bval32.ptr)
                            : reinterpret_cast<const T*>(B->bval64.ptr);
    a.bval64 = B->bval64.as<double>();
    a.bperm = B->bperm.as<int32_t>();
    a.xB = B->bx.as<double>();
    a.bB = B->bb.as<double>();
  }
  a.b_user = io.b_user;
  a.x_user = io.x_user;
  a.B_user = io.B_user;
  a.X_user = io.X_user;
  a.slots = B->slots.as<Slot>();
  a.ust = B->ust.as<UnitState>();
  a.tickets = B->tickets.as<unsigned int>();
  a.parts = B->parts.as<double>();
  a.bar = B->bar.as<unsigned long long>();
  a.err = B->err.as<int>();
  a.limit_ns = wait_ns();
  a.prof = nullptr;
  a.prof_cap = 0;
  if (!dry && std::getenv("SPMV_B200_BATCH_PROFILE")) {
    B->prof.reserve(sizeof(unsigned long long) * (2 * kProfCap + 16 + 3 * 1024));
    SPMVB_CUDA(cudaMemsetAsync(B->prof.ptr, 0,
                               sizeof(unsigned long long) * (2 * kProfCap + 16 + 3 * 1024),
                               B->comm->stream));
    a.prof = B->prof.as<unsigned long long>();
    a.prof_cap = kProfCap;
  }
}

// One launch of the lockstep kernel; false when the shape cannot be resident.
bool run(spmv_batch B, spmv_batch_precision prec, const SolveIo& io, int kmax, double rtol,
         const LaunchCfg& cfg, bool dry) {
  spmv_comm comm = B->comm;
  cudaStream_t s = comm->stream;
  const int nu = nunits_of(B, io.with_block);
  if (!dry) {
    SPMVB_CUDA(cudaMemsetAsync(B->bar.ptr, 0, sizeof(unsigned long long), s));
    SPMVB_CUDA(cudaMemsetAsync(B->err.ptr, 0, sizeof(int), s));
    SPMVB_CUDA(cudaMemsetAsync(B->tickets.ptr, 0, sizeof(unsigned int) * std::max(nu, 1), s));
  }
  const bool d16 = B->plan.fits16;
  if (prec == SPMV_BATCH_MIXED) {
    if (d16) {
      Args<float, int16_t> a;
      fill_args(B, a, io, kmax, rtol, kDelta2, cfg, dry);
      return launch_f32(&a, true, cfg, comm->num_sms, s, dry);
    }
    Args<float, int32_t> a;
    fill_args(B, a, io, kmax, rtol, 0.01, cfg, dry);
    return launch_f32(&a, false, cfg, comm->num_sms, s, dry);
  }
  if (d16) {
    Args<double, int16_t> a;
    fill_args(B, a, io, kmax, rtol, 0.0, cfg, dry);
    return launch_f64(&a, true, cfg, comm->num_sms, s, dry);
  }
  Args<double, int32_t> a;
  fill_args(B, a, io, kmax, rtol, 0.0, cfg, dry);
  return launch_f64(&a, false, cfg, comm->num_sms, s, dry);
}

// The configured shape, or 1 CTA per SM when 2 do not fit.
LaunchCfg resident_cfg(spmv_batch B, spmv_batch_precision prec, LaunchCfg c, const SolveIo& io) {
  for (;;) {
    if (run(B, prec, io, 0, 1.0, c, true)) return c;
    if (c.cps <= 1) fail(SPMV_ERROR_CUDA, "spmv batch: the kernel cannot be made resident");
    c.cps = 1;
  }
}

std::string tune_key(spmv_batch B, int prec) {
  std::ostringstream k;
  k << "batch:v4:" << prec << ":" << B->nsys << ":" << B->plan.rows_pad << ":" << B->plan.nnz_total << ":"
    << B->plan.entries << ":" << (B->plan.fits16 ? 16 : 32) << ":" << B->block_nrhs << ":"
    << B->block_n;
  return k.str();
}

bool cache_lookup(const std::string& key, LaunchCfg& c, double& us) {
  const char* path = std::getenv("SPMV_B200_TUNE_CACHE");
  if (!path) return false;
  std::ifstream f(path);
  std::string line;
  while (std::getline(f, line)) {
    std::istringstream is(line);
    std::string k;
    LaunchCfg t;
    double u = 0;
    if ((is >> k >> t.cps >> t.tile_slices >> t.rhs_rows >> t.window >> u) && k == key) {
      c = t;
      us = u;
      return true;
    }
  }
  return false;
}

void cache_store(const std::string& key, const LaunchCfg& c, double us) {
  const char* path = std::getenv("SPMV_B200_TUNE_CACHE");
  if (!path) return;
  std::ofstream f(path, std::ios::app);
  f << key << " " << c.cps << " " << c.tile_slices << " " << c.rhs_rows << " " << c.window << " "
    << us << "\n";
}

void check_err(spmv_batch B) {
  int err = 0;
  SPMVB_CUDA(cudaMemcpy(&err, B->err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
  if (err) fail(SPMV_ERROR_CUDA, "spmv batch: a bounded grid wait on the device timed out");
}

}  // namespace
}  // namespace bat
}  // namespace spmvb

using namespace spmvb;
using namespace spmvb::bat;

extern "C" {

int spmv_batch_create(spmv_comm comm, int nsys, const int32_t* n,
                      const int32_t* const* rowptr, const int32_t* const* colind,
                      const double* const* values, spmv_batch* out) {
  return guard([&] {
    require(comm != nullptr && out != nullptr, "spmv: NULL argument");
    *out = nullptr;
    require(nsys >= 0, "spmv: negative system count");
    require(nsys < MAX_UNITS, "spmv batch: at most 8191 systems");
    require(nsys == 0 || (n && rowptr && colind && values), "spmv: NULL CSR array");
    comm->require_device();
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
    }
    std::unique_ptr<spmv_batch_s> B(new spmv_batch_s);
    B->comm = comm;
    B->nsys = nsys;
    plan_batch(nsys, n, rowptr, colind, values, B->plan);
    Plan& P = B->plan;
    require(P.nslices < (int64_t(1) << 31), "spmv batch: too many rows");
    DeviceGuard dg(comm->device);
    upload(B->soff, P.soff.data(), sizeof(int64_t) * P.soff.size());
    upload(B->sbound, P.sbound.data(), sizeof(int32_t) * P.sbound.size());
    upload(B->vals32, P.vals32.data(), sizeof(float) * P.vals32.size());
    upload(B->vals64, P.vals64.data(), sizeof(double) * P.vals64.size());
    if (P.fits16)
      upload(B->idx, P.off16.data(), sizeof(int16_t) * P.off16.size());
    else
      upload(B->idx, P.col32.data(), sizeof(int32_t) * P.col32.size());
    upload(B->perm, P.perm.data(), sizeof(int32_t) * P.perm.size());
    // The host copies of the big arrays are not needed again.
    std::vector<float>().swap(P.vals32);
    std::vector<double>().swap(P.vals64);
    std::vector<int16_t>().swap(P.off16);
    std::vector<int32_t>().swap(P.col32);
    std::vector<int32_t>().swap(P.perm);
    std::vector<int64_t>().swap(P.soff);
    std::vector<int32_t>().swap(P.sbound);
    const int64_t rows = std::max<int64_t>(P.rows_pad, 32);
    B->x.reserve(sizeof(double) * rows);
    B->b.reserve(sizeof(double) * rows);
    SPMVB_CUDA(cudaMemset(B->x.ptr, 0, sizeof(double) * rows));
    SPMVB_CUDA(cudaMemset(B->b.ptr, 0, sizeof(double) * rows));
    B->bar.reserve(sizeof(unsigned long long));
    B->err.reserve(sizeof(int));
    B->uptr.reserve(sizeof(void*) * 2 * std::max(nsys, 1));
    B->gmax = 2 * std::max(comm->num_sms, 1);
    build_units(B.get());
    // The block's CSR is built from the system when a block is declared.
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

int spmv_batch_set_block(spmv_batch B, int system, int nrhs) {
  return guard([&] {
    require(B != nullptr, "spmv: NULL batch");
    require(system >= 0 && system < B->nsys, "spmv batch: block system out of range");
    require(nrhs >= 1 && nrhs <= BW, "spmv batch: a block takes 1..32 right-hand sides");
    spmv_comm comm = B->comm;
    comm->require_device();
    DeviceGuard dg(comm->device);
    const Plan& P = B->plan;
    const int32_t m = P.n[system];
    const int64_t ns = (m + 31) / 32;
    // The system's SELL slices, read back: the block's CSR is the same matrix
    // in the same (planned) row order.  Padding entries have value 0 and are
    // dropped, as is any stored zero (it adds nothing to a product).
    std::vector<int64_t> soff(ns + 1);
    SPMVB_CUDA(cudaMemcpy(soff.data(), B->soff.as<int64_t>() + P.slice0[system],
                          sizeof(int64_t) * (ns + 1), cudaMemcpyDeviceToHost));
    const int64_t e0 = soff[0], ne = soff[ns] - e0;
    std::vector<double> v64(ne);
    std::vector<int32_t> col(ne);
    if (ne) {
      SPMVB_CUDA(cudaMemcpy(v64.data(), B->vals64.as<double>() + e0, sizeof(double) * ne,
                            cudaMemcpyDeviceToHost));
      if (P.fits16) {
        std::vector<int16_t> off(ne);
        SPMVB_CUDA(cudaMemcpy(off.data(), B->idx.as<int16_t>() + e0, sizeof(int16_t) * ne,
                              cudaMemcpyDeviceToHost));
        for (int64_t sl = 0; sl < ns; ++sl)
          for (int64_t e = soff[sl]; e < soff[sl + 1]; ++e) {
            const int64_t row = 32 * sl + ((e - soff[sl]) & 31);
            col[e - e0] = int32_t(row + off[e - e0]);
          }
      } else {
        SPMVB_CUDA(cudaMemcpy(col.data(), B->idx.as<int32_t>() + e0, sizeof(int32_t) * ne,
                              cudaMemcpyDeviceToHost));
      }
    }
    const int32_t npad = (m + 63) / 64 * 64;  // whole block tiles at every tile size
    std::vector<int32_t> rp(npad + 1, 0), bc;
    std::vector<double> bv64;
    std::vector<float> bv32;
    for (int32_t row = 0; row < npad; ++row) {
      if (row < m) {
        const int64_t sl = row / 32, l = row % 32;
        const int64_t w = (soff[sl + 1] - soff[sl]) / 32;
        for (int64_t k = 0; k < w; ++k) {
          const int64_t e = soff[sl] - e0 + 32 * k + l;
          if (v64[e] == 0.0) continue;
          bc.push_back(col[e]);
          bv64.push_back(v64[e]);
          bv32.push_back(float(v64[e]));
        }
      }
      rp[row + 1] = int32_t(bc.size());
    }
    std::vector<int32_t> bperm(npad, -1);
    for (int32_t i = 0; i < m; ++i) bperm[i] = P.sys_perm[system][i];
    upload(B->brp, rp.data(), sizeof(int32_t) * rp.size());
    upload(B->bcol, bc.data(), sizeof(int32_t) * bc.size());
    upload(B->bval64, bv64.data(), sizeof(double) * bv64.size());
    upload(B->bval32, bv32.data(), sizeof(float) * bv32.size());
    upload(B->bperm, bperm.data(), sizeof(int32_t) * bperm.size());
    B->bv32.release();
    B->bv64.release();
    const size_t nb = size_t(std::max(npad, 16)) * BW;
    B->bx.reserve(sizeof(double) * nb);
    B->bb.reserve(sizeof(double) * nb);
    SPMVB_CUDA(cudaMemset(B->bx.ptr, 0, sizeof(double) * nb));
    SPMVB_CUDA(cudaMemset(B->bb.ptr, 0, sizeof(double) * nb));
    B->block_sys = system;
    B->block_nrhs = nrhs;
    B->block_n = m;
    B->block_npad = npad;
    B->block_nnz = int64_t(bc.size());
    build_units(B);
  });
}

int spmv_batch_set_config(spmv_batch B, spmv_batch_precision prec, const spmv_batch_config* c) {
  return guard([&] {
    require(B != nullptr && c != nullptr, "spmv: NULL argument");
    require(prec == SPMV_BATCH_MIXED || prec == SPMV_BATCH_FP64, "spmv batch: unknown precision");
    LaunchCfg& cfg = B->cfg[prec];
    if (c->ctas_per_sm) {
      require(c->ctas_per_sm == 1 || c->ctas_per_sm == 2, "spmv batch: ctas_per_sm must be 1 or 2");
      cfg.cps = c->ctas_per_sm;
    }
    if (c->tile_rows) {
      require(c->tile_rows == 128 || c->tile_rows == 256 || c->tile_rows == 512,
              "spmv batch: tile_rows must be 128, 256 or 512");
      cfg.tile_slices = tile_slices_of(c->tile_rows);
    }
    if (c->rhs_lanes) {
      require(c->rhs_lanes == 32 || c->rhs_lanes == 16, "spmv batch: rhs_lanes must be 32 or 16");
      cfg.rhs_rows = 32 / c->rhs_lanes;
    }
    if (c->window) {
      require(c->window == 1 || c->window == 2, "spmv batch: window must be 1 (off) or 2 (on)");
      cfg.window = c->window == 2;
    }
  });
}

int spmv_batch_get_config(spmv_batch B, spmv_batch_precision prec, spmv_batch_config* c) {
  return guard([&] {
    require(B != nullptr && c != nullptr, "spmv: NULL argument");
    require(prec == SPMV_BATCH_MIXED || prec == SPMV_BATCH_FP64, "spmv batch: unknown precision");
    const LaunchCfg& cfg = B->cfg[prec];
    c->ctas_per_sm = cfg.cps;
    c->tile_rows = 32 * cfg.tile_slices;
    c->rhs_lanes = 32 / cfg.rhs_rows;
    c->window = cfg.window ? 2 : 1;
    c->us = 0.0;
    c->candidates = 0;
  });
}

int spmv_batch_stats(spmv_batch B, int64_t* rows, int64_t* nnz, int64_t* stored,
                     int* index_bits) {
  return guard([&] {
    require(B != nullptr, "spmv: NULL batch");
    int64_t r = 0;
    for (int32_t v : B->plan.n) r += v;
    if (rows) *rows = r;
    if (nnz) *nnz = B->plan.nnz_total;
    if (stored) *stored = B->plan.entries;
    if (index_bits) *index_bits = B->plan.fits16 ? 16 : 32;
  });
}

int spmv_batch_autotune(spmv_batch B, spmv_batch_precision prec, spmv_batch_config* best) {
  return guard([&] {
    require(B != nullptr, "spmv: NULL batch");
    require(prec == SPMV_BATCH_MIXED || prec == SPMV_BATCH_FP64, "spmv batch: unknown precision");
    spmv_comm comm = B->comm;
    comm->require_device();
    DeviceGuard dg(comm->device);
    cudaStream_t s = comm->stream;
    const std::string key = tune_key(B, int(prec));
    LaunchCfg pick;
    double pick_us = 0.0;
    int tried = 0;
    if (!cache_lookup(key, pick, pick_us)) {
      // One fixed pseudo-random right-hand side in [-1, 1) shared by every
      // system (splitmix64 of the row index; a vector of ones would not do:
      // it is an eigenvector of a graph Laplacian plus a diagonal shift, so
      // CG would stop after one iteration), solutions into scratch (every
      // system writes its own rows of one shared scratch vector, which
      // nothing reads).
      const bool blk = B->block_sys >= 0;
      int32_t nmax = 1;
      for (int32_t v : B->plan.n) nmax = std::max(nmax, v);
      const int64_t nbl = blk ? int64_t(B->block_n) * B->block_nrhs : 0;
      DevBuf rhs, scratch, tab;
      const size_t len = size_t(std::max<int64_t>(nmax, nbl));
      rhs.reserve(sizeof(double) * len);
      scratch.reserve(sizeof(double) * len);
      std::vector<double> h(len);
      for (size_t i = 0; i < len; ++i) {
        uint64_t z = (uint64_t(i) + 1) * 0x9E3779B97F4A7C15ull;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        z ^= z >> 31;
        h[i] = double(z >> 11) * 0x1.0p-52 - 1.0;
      }
      SPMVB_CUDA(cudaMemcpy(rhs.ptr, h.data(), sizeof(double) * len, cudaMemcpyHostToDevice));
      std::vector<const void*> ptrs(2 * std::max(B->nsys, 1));
      for (int i = 0; i < B->nsys; ++i) {
        ptrs[i] = rhs.ptr;
        ptrs[B->nsys + i] = scratch.ptr;
      }
      tab.reserve(sizeof(void*) * ptrs.size());
      SPMVB_CUDA(cudaMemcpy(tab.ptr, ptrs.data(), sizeof(void*) * ptrs.size(),
                            cudaMemcpyHostToDevice));
      SolveIo io;
      io.b_user = reinterpret_cast<const double* const*>(tab.ptr);
      io.x_user = reinterpret_cast<double* const*>(tab.as<void*>() + B->nsys);
      io.B_user = blk ? rhs.as<double>() : nullptr;
      io.X_user = blk ? scratch.as<double>() : nullptr;
      io.with_block = blk;
      cudaEvent_t e0, e1;
      SPMVB_CUDA(cudaEventCreate(&e0));
      SPMVB_CUDA(cudaEventCreate(&e1));
      double best_us = 1e300;
      const int kmax = 64;
      for (int cps : {2, 1})
        for (int ts : {4, 8, 16})
          for (int rr : {1, 2})
            for (int win : {1, 0}) {
            if (rr == 2 && !blk) continue;
            LaunchCfg c;
            c.cps = cps;
            c.tile_slices = ts;
            c.rhs_rows = rr;
            c.window = win;
            if (!run(B, prec, io, kmax, 1e-30, c, true)) continue;
            run(B, prec, io, kmax, 1e-30, c, false);
            double us = 1e300;
            for (int rep = 0; rep < 2; ++rep) {
              SPMVB_CUDA(cudaEventRecord(e0, s));
              run(B, prec, io, kmax, 1e-30, c, false);
              SPMVB_CUDA(cudaEventRecord(e1, s));
              SPMVB_CUDA(cudaEventSynchronize(e1));
              float ms = 0.f;
              SPMVB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
              us = std::min(us, 1e3 * double(ms));
            }
            check_err(B);
            ++tried;
            if (us < best_us) {
              best_us = us;
              pick = c;
            }
          }
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      require(tried > 0, "spmv batch: no launch shape can be made resident");
      pick_us = best_us;
      cache_store(key, pick, pick_us);
    }
    B->cfg[prec] = pick;
    if (best) {
      best->ctas_per_sm = pick.cps;
      best->tile_rows = 32 * pick.tile_slices;
      best->rhs_lanes = 32 / pick.rhs_rows;
      best->window = pick.window ? 2 : 1;
      best->us = pick_us;
      best->candidates = tried;
    }
  });
}

int spmv_batch_solve_ex(spmv_batch B, spmv_memory memory, spmv_batch_precision precision,
                        const double* const* b, double* const* x, const double* bblock,
                        double* xblock, int max_its, double rtol, spmv_batch_info* info,
                        spmv_batch_info* block_info) {
  return guard([&] {
    require(B != nullptr, "spmv: NULL batch");
    require(B->nsys == 0 || (b != nullptr && x != nullptr), "spmv: NULL vector array");
    require(memory == SPMV_MEMORY_HOST || memory == SPMV_MEMORY_DEVICE,
            "spmv: unknown memory kind");
    require(precision == SPMV_BATCH_MIXED || precision == SPMV_BATCH_FP64,
            "spmv batch: unknown precision");
    require(max_its >= 0, "spmv batch: negative iteration bound");
    spmv_comm comm = B->comm;
    comm->require_device();
    DeviceGuard dg(comm->device);
    cudaStream_t s = comm->stream;
    const bool blk = B->block_sys >= 0 && bblock != nullptr && xblock != nullptr;
    const Plan& P = B->plan;
    const int ns = B->nsys;
    for (int i = 0; i < ns; ++i)
      if (P.n[i] > 0) require(b[i] != nullptr && x[i] != nullptr, "spmv: NULL vector");
    // The caller's vectors as device pointers (host vectors staged).
    std::vector<const void*> ptrs(2 * std::max(ns, 1), nullptr);
    const double* Bd = bblock;
    double* Xd = xblock;
    int64_t tot = 0;
    for (int i = 0; i < ns; ++i) tot += P.n[i];
    const int64_t nbl = blk ? int64_t(B->block_n) * B->block_nrhs : 0;
    if (memory == SPMV_MEMORY_HOST) {
      B->stage.reserve(sizeof(double) * size_t(std::max<int64_t>(2 * (tot + nbl), 2)));
      double* st = B->stage.as<double>();
      int64_t o = 0;
      for (int i = 0; i < ns; ++i) {
        ptrs[i] = st + o;
        ptrs[ns + i] = st + tot + nbl + o;
        if (P.n[i] > 0)
          SPMVB_CUDA(cudaMemcpyAsync(st + o, b[i], sizeof(double) * P.n[i],
                                     cudaMemcpyHostToDevice, s));
        o += P.n[i];
      }
      if (blk) {
        Bd = st + tot;
        Xd = st + tot + nbl + tot;
        SPMVB_CUDA(cudaMemcpyAsync(const_cast<double*>(Bd), bblock, sizeof(double) * nbl,
                                   cudaMemcpyHostToDevice, s));
      }
    } else {
      for (int i = 0; i < ns; ++i) {
        ptrs[i] = b[i];
        ptrs[ns + i] = x[i];
      }
    }
    SPMVB_CUDA(cudaMemcpyAsync(B->uptr.ptr, ptrs.data(), sizeof(void*) * ptrs.size(),
                               cudaMemcpyHostToDevice, s));
    SolveIo io;
    io.b_user = reinterpret_cast<const double* const*>(B->uptr.ptr);
    io.x_user = reinterpret_cast<double* const*>(B->uptr.as<void*>() + ns);
    io.B_user = blk ? Bd : nullptr;
    io.X_user = blk ? Xd : nullptr;
    io.with_block = blk;
    const LaunchCfg cfg = resident_cfg(B, precision, B->cfg[precision], io);
    require(run(B, precision, io, max_its, rtol, cfg, false),
            "spmv batch: the kernel cannot be made resident");
    const int nslot = ns + (blk ? BW : 0);
    std::vector<Slot> sl(std::max(nslot, 1));
    if (nslot)
      SPMVB_CUDA(cudaMemcpyAsync(sl.data(), B->slots.ptr, sizeof(Slot) * nslot,
                                 cudaMemcpyDeviceToHost, s));
    if (memory == SPMV_MEMORY_HOST) {
      const double* st = B->stage.as<double>();
      int64_t o = 0;
      for (int i = 0; i < ns; ++i) {
        if (P.n[i] > 0)
          SPMVB_CUDA(cudaMemcpyAsync(x[i], st + tot + nbl + o, sizeof(double) * P.n[i],
                                     cudaMemcpyDeviceToHost, s));
        o += P.n[i];
      }
      if (blk)
        SPMVB_CUDA(cudaMemcpyAsync(xblock, Xd, sizeof(double) * nbl, cudaMemcpyDeviceToHost, s));
    }
    SPMVB_CUDA(cudaStreamSynchronize(s));
    check_err(B);
    write_profile(B, precision == SPMV_BATCH_MIXED ? "mixed" : "fp64");
    auto fill = [](const Slot& q, spmv_batch_info& o) {
      o.iterations = q.its;
      o.refinements = q.refs;
      o.status = q.status;
      o.converged = q.converged;
      o.relres = q.rr0 > 0.0 ? std::sqrt(q.rr_true / q.rr0) : 0.0;
    };
    if (info)
      for (int i = 0; i < ns; ++i) fill(sl[i], info[i]);
    if (block_info && blk)
      for (int l = 0; l < B->block_nrhs; ++l) fill(sl[ns + l], block_info[l]);
    for (int i = 0; i < ns; ++i)
      if (sl[i].status == SPMV_ERROR_BREAKDOWN)
        fail(SPMV_ERROR_BREAKDOWN, "spmv batch: breakdown in system " + std::to_string(i));
    if (blk)
      for (int l = 0; l < B->block_nrhs; ++l)
        if (sl[ns + l].status == SPMV_ERROR_BREAKDOWN)
          fail(SPMV_ERROR_BREAKDOWN,
               "spmv batch: breakdown in block column " + std::to_string(l));
  });
}

int spmv_batch_solve(spmv_batch B, spmv_memory memory, const double* const* b,
                     double* const* x, int max_its, double rtol, spmv_batch_info* info) {
  return spmv_batch_solve_ex(B, memory, SPMV_BATCH_MIXED, b, x, nullptr, nullptr, max_its,
                             rtol, info, nullptr);
}

}  // extern "C"
