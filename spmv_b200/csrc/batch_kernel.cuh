// Lockstep batched CG: every system of a batch (and the block of right-hand
// sides of one system) iterates in the same persistent cooperative launch,
// one CG iteration of all units per pass of its loop (no counterpart in the
// reference; each recurrence is spmv::cg's, cg.cpp:50-80, with the FP32-inner
// / FP64-refinement scheme of the mixed solver).
//
// Per lockstep iteration k, over the units still iterating:
//   A  y = A p (inner precision), partial p.y             | grid barrier
//   B  alpha; d += alpha p, r -= alpha y, partial r.r      | grid barrier
//   C  units that refine: r = fl(b - A64 (x + d)) (FP64), ||r64||^2, r.r, r.p
//      the others: p = r + beta p                          | grid barrier
//   D  (only when some unit refined) x += d, d = 0, p = r + beta (p - c r)
//                                                          | grid barrier
// Work is split by tiles (32 x tile_slices rows of a unit, or tile_slices
// block rows): the active units' tiles are listed in unit order with a
// per-phase cost weight, and CTA c takes the tiles whose weight position
// falls in [c W / G, (c + 1) W / G) -- every CTA streams an equal share of
// the whole batch in every phase, whatever the unit sizes.  Inside a CTA the
// warps deal its tiles round robin.
//
// Reductions: a warp sums each of its tiles (fixed shuffle tree) into a
// running sum per unit, the CTA adds its warps' sums in warp order and
// publishes one partial per (unit, CTA); the CTA that completes a unit's tile
// count (atomic ticket) adds the partials in CTA order and updates the unit's
// recurrences (alpha, beta, refinement and stopping decisions).  Every CTA
// reads those decisions after the next grid barrier, so the control flow is
// the same in all CTAs by construction.  The order of every sum depends only
// on the launch configuration and the batch, so solves are reproducible run
// to run.
//
// The grid barrier spins only in a cooperative launch (every CTA resident),
// one thread per CTA, bounded by `limit_ns` of global time; a CTA that times
// out or sees the error flag raises it and returns, and the others leave at
// their next barrier.
#pragma once

#include <algorithm>

#include "batch.h"
#include "kernels.cuh"

namespace spmvb {
namespace bat {

enum { PH_INIT = 0, PH_A = 1, PH_C = 3, PH_D = 4, PH_FINAL = 5, PH_B = 2 };

constexpr int U = 8;  // gathers in flight per lane in the products

// Relative cost of one tile of a phase (in units of a single-unit tile of a
// vector phase).  The FP64 refinement product reads the FP64 matrix and two
// gathered vectors per entry; the block's refinement product reads its matrix
// once for all its columns.
// A block tile holds BT_MUL x tile_slices block rows (32 x that many
// elements, as many as a single-unit tile of the vector phases).  The
// weights were set by timing the batched workload's phases: the refinement
// product is latency-bound (two gathered vectors per entry), and block tiles
// four times as long were slower in every phase.
constexpr int BT_MUL = 1;
// Weights in eighths of a single unit's tile in the same phase; the
// refinement tiles' and the block's weights come with the launch (they
// differ between the precisions), measured per CTA on the batched workload.
__device__ __forceinline__ int tile_weight(const Weights& w, int ph, int kind, bool refine) {
  if (ph == PH_C && refine) return kind == 0 ? w.one_c2 : w.blk_c2;
  if (kind == 0) return 8;
  return ph == PH_A ? w.blk_a : ph == PH_B ? w.blk_b : ph == PH_C ? w.blk_c : 8;
}
__device__ __forceinline__ int tile_rows_of(const Unit& un, int tile_slices) {
  return un.kind == 0 ? tile_slices : BT_MUL * tile_slices;
}
// Tiles of a unit: 32 x tile_slices rows (single units, nslices slices) or
// BT_MUL x tile_slices block rows (the block, nslices rows).
__device__ __forceinline__ int unit_tiles(const Unit& un, int tile_slices) {
  const int tr = tile_rows_of(un, tile_slices);
  return (un.nslices + tr - 1) / tr;
}

// Slices in one chunk of a product unit: NW tiles of at most 16 slices.
constexpr int CH_MAX = 16 * NW;

struct Smem {
  double sums[MAXQ][NW][NSUM];
  int q_list[MAXQ], q_ja[MAXQ], q_jb[MAXQ], q_t[MAXQ], q_ref[MAXQ], q_kind[MAXQ];
  int q_cf[MAXQ], q_ns[MAXQ];
  int q_pos[MAXQ + 1];
  long long scan[NW];
  long long tot;
  int wmin[NW], wmax[NW];
  int nq, next_i, nref, ok, blk_last;
  // The current chunk of a product unit: its slices' entry offsets, the
  // hand-out counter, and each slice's sums.
  long long ch_off[CH_MAX + 1];
  double ch_part[NSUM][CH_MAX];
  int ch_next;
  // Global rows [ring_lo, ring_hi] of p held in the FP32 window (empty when
  // ring_lo > ring_hi); valid within one pass of the product phase.
  long long ring_lo, ring_hi;
};

// Dynamic shared memory: the unit list (2 ints per unit), then a region that
// holds the product's window of p and, at other times, the block unit's
// per-warp column sums.
extern __shared__ __align__(16) unsigned char bat_dyn[];
__device__ __forceinline__ size_t win_offset(int nunits) {
  return (size_t(2) * sizeof(int) * size_t(nunits) + 15) & ~size_t(15);
}
__device__ __forceinline__ double (*block_sums(int nunits))[NSUM][BW] {
  return reinterpret_cast<double (*)[NSUM][BW]>(bat_dyn + win_offset(nunits));
}

// ---------------------------------------------------------------------------
// Small vector helpers.
// ---------------------------------------------------------------------------
template <typename T>
struct Four {
  T v[4];
};
__device__ __forceinline__ Four<float> ld4(const float* p) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  return Four<float>{{t.x, t.y, t.z, t.w}};
}
__device__ __forceinline__ Four<double> ld4(const double* p) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  return Four<double>{{a.x, a.y, b.x, b.y}};
}
__device__ __forceinline__ void st4(float* p, const Four<float>& f) {
  *reinterpret_cast<float4*>(p) = make_float4(f.v[0], f.v[1], f.v[2], f.v[3]);
}
__device__ __forceinline__ void st4(double* p, const Four<double>& f) {
  *reinterpret_cast<double2*>(p) = make_double2(f.v[0], f.v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(f.v[2], f.v[3]);
}

// R consecutive elements (R = 1, 2, 4), aligned to R elements.
template <typename T, int R>
__device__ __forceinline__ void ldR(const T* p, T (&o)[R]) {
  if constexpr (R == 4) {
    const Four<T> f = ld4(p);
#pragma unroll
    for (int i = 0; i < 4; ++i) o[i] = f.v[i];
  } else if constexpr (R == 2) {
    if constexpr (sizeof(T) == 4) {
      const float2 t = *reinterpret_cast<const float2*>(p);
      o[0] = t.x;
      o[1] = t.y;
    } else {
      const double2 t = *reinterpret_cast<const double2*>(p);
      o[0] = t.x;
      o[1] = t.y;
    }
  } else {
    o[0] = *p;
  }
}
template <typename T, int R>
__device__ __forceinline__ void stR(T* p, const T (&v)[R]) {
  if constexpr (R == 4) {
    Four<T> f;
#pragma unroll
    for (int i = 0; i < 4; ++i) f.v[i] = v[i];
    st4(p, f);
  } else if constexpr (R == 2) {
    if constexpr (sizeof(T) == 4)
      *reinterpret_cast<float2*>(p) = make_float2(v[0], v[1]);
    else
      *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  } else {
    *p = v[0];
  }
}

__device__ __forceinline__ double warp_total(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Column index of a gathered entry.
template <typename CI>
__device__ __forceinline__ int64_t gcol(int c, int64_t row, int64_t row0) {
  if constexpr (sizeof(CI) == 2)
    return row + c;
  else
    return row0 + c;
}
__device__ __forceinline__ int ldidx(const int16_t* p) { return int(__ldcs(p)); }
__device__ __forceinline__ int ldidx(const int32_t* p) { return __ldcs(p); }

// ---------------------------------------------------------------------------
// Grid barrier over all threads of every CTA.
// ---------------------------------------------------------------------------
// With a.prof set, CTA 0 records after each barrier the phase that ended
// (code) and %globaltimer: prof[2 e] = code, prof[2 e + 1] = time.
__device__ __forceinline__ unsigned long long gtimer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

template <typename T, typename CI>
__device__ __forceinline__ bool gbar(const Args<T, CI>& a, unsigned long long& epoch, Smem& sm,
                                     int code) {
  ++epoch;
  __syncthreads();
  if (threadIdx.x == 0) {
    sm.ok = grid_arrive_wait(a.bar, epoch * gridDim.x, a.err, a.limit_ns) ? 1 : 0;
    if (a.prof && blockIdx.x == 0 && epoch < unsigned(a.prof_cap)) {
      a.prof[2 * epoch] = code;
      a.prof[2 * epoch + 1] = gtimer();
    }
  }
  __syncthreads();
  return sm.ok != 0;
}

// ---------------------------------------------------------------------------
// Unit lists: the units `inc` admits, in unit order, with the exclusive
// prefix of their weights (tiles x tile weight).  Every CTA builds the same
// list from the same global state.  Returns the count; sm.tot >> 20 is the
// total weight.
// ---------------------------------------------------------------------------
template <class Inc>
__device__ __forceinline__ int build_list(int nunits, int* lu, int* lw, Smem& sm, Inc&& inc) {
  const int per = (nunits + NT - 1) / NT;
  const int u0 = int(threadIdx.x) * per, u1 = min(nunits, u0 + per);
  long long mine = 0;
  for (int u = u0; u < u1; ++u) {
    int w = 0;
    if (inc(u, w)) mine += (static_cast<long long>(w) << 20) | 1;
  }
  const int lane = int(threadIdx.x) & 31, warp = int(threadIdx.x) >> 5;
  long long incl = mine;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const long long v = __shfl_up_sync(0xffffffffu, incl, o);
    if (lane >= o) incl += v;
  }
  if (lane == 31) sm.scan[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    long long v = lane < NW ? sm.scan[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const long long t = __shfl_up_sync(0xffffffffu, v, o);
      if (lane >= o) v += t;
    }
    if (lane < NW) sm.scan[lane] = v;
    if (lane == NW - 1) sm.tot = v;
  }
  __syncthreads();
  const long long excl = incl - mine + (warp > 0 ? sm.scan[warp - 1] : 0);
  int c = int(excl & 0xFFFFF);
  long long wacc = excl >> 20;
  for (int u = u0; u < u1; ++u) {
    int w = 0;
    if (inc(u, w)) {
      lu[c] = u;
      lw[c] = int(wacc);
      ++c;
      wacc += w;
    }
  }
  __syncthreads();
  return int(sm.tot & 0xFFFFF);
}

__device__ __forceinline__ long long cta_of(long long x, long long W, int G) {
  return ((x + 1) * G + W - 1) / W - 1;
}
__device__ __forceinline__ int tiles_from(long long num, int wt, int T) {
  if (num <= 0) return 0;
  const long long t = (num + wt - 1) / wt;
  return int(t < T ? t : T);
}

// ---------------------------------------------------------------------------
// Tile bodies.  Single-unit bodies return the tile's sums in every lane;
// block bodies return column `lane`'s sums in lane `lane`.
// ---------------------------------------------------------------------------
template <typename T, typename CI>
struct Ctx {
  const Args<T, CI>& a;
  int k;
  uint64_t keep, strm;
};

// The tile's slice offsets, one per lane (lane l: soff of slice s0 + l; the
// tile has at most 16 slices, so lanes 0..16 cover its ends).
__device__ __forceinline__ int64_t tile_soff(const int64_t* soff, int64_t sg0, int n) {
  const int lane = int(threadIdx.x) & 31;
  return lane <= n ? soff[sg0 + lane] : 0;
}

// Bulk L2 prefetch of a tile's entries [e0, e1) (values and indices, each a
// contiguous run in the SELL layout; e0 and e1 are multiples of 32 entries,
// so both runs start on 64-byte boundaries and are multiples of 64 bytes
// long).  One lane issues it; the whole run streams from DRAM while the
// warp works through the tile's first slices.
template <typename V, typename CI>
__device__ __forceinline__ void prefetch_tile(const V* vals, const CI* idx, int64_t e0,
                                              int64_t e1) {
  if ((threadIdx.x & 31) != 0 || e1 <= e0) return;
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(vals + e0),
               "r"(unsigned((e1 - e0) * int64_t(sizeof(V))))
               : "memory");
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(idx + e0),
               "r"(unsigned((e1 - e0) * int64_t(sizeof(CI))))
               : "memory");
}

// A, single: y = A p over the chunk's slices [c_lo, c_hi) of the unit
// (offsets staged in sm.ch_off), p.y of each slice into sm.ch_part.  The
// CTA's warps take the slices in order from a shared counter (warp w starts
// with slice w), so the warps in flight work on neighbouring slices, whose
// gathers share lines, and no warp is left with the wide slices of the
// length-sorted windows while the others wait at the chunk's end.  Up to UA
// entries per lane are in flight (FP32: 14, one round for most k-NN rows;
// FP64: 8), and each slice's tail (the warp's p.y reduction, the claim of
// the next slice) overlaps the next slice's loads.
// WIN: p is read from the CTA's shared-memory window, whose element 0 is
// p[wbase] (global row index); the window covers every column of the slices.
template <typename T, typename CI, bool WIN>
__device__ __noinline__ void tileA1(const Ctx<T, CI>& x, const Unit& u, int c_lo, int c_hi,
                                    int64_t wbase, Smem& sm) {
  // Entries per lane in flight: FP32 14 (a remainder of at most 2 takes a
  // short batch), FP64 8; sizes at which the batch, the next slice's state
  // and the pending sum stay in registers.
  constexpr int UA = sizeof(T) == 4 ? 14 : 8;
  constexpr int UT = sizeof(T) == 4 ? 2 : 0;
  const Args<T, CI>& a = x.a;
  // FP32: the window is a ring of win_cap (a power of two) rows, row g at
  // g & (win_cap - 1); FP64: rows from wbase on.
  constexpr bool RING = sizeof(T) == 4;
  const T* pw = reinterpret_cast<const T*>(bat_dyn + win_offset(a.nunits)) - (RING ? 0 : wbase);
  const int64_t wmask = RING ? int64_t(a.win_cap - 1) : int64_t(-1);
  const int lane = int(threadIdx.x) & 31;
  const T* __restrict__ vals = a.vals;
  const CI* __restrict__ idx = a.idx;
  const T* __restrict__ pv_ = a.p;
  const int n = c_hi - c_lo;
  int i = int(threadIdx.x) >> 5;
  if (i >= n) return;
  // The next slice is claimed, and the previous slice's p.y reduced across
  // the warp, while this slice's first loads are in flight.
  int nxt = 0;
  if (lane == 0) nxt = atomicAdd(&sm.ch_next, 1);
  int64_t e0 = sm.ch_off[i];
  int w = int((sm.ch_off[i + 1] - e0) >> 5);
  double pend = 0.0;
  int pend_i = -1;
  auto settle = [&]() {
    if (pend_i >= 0) {
      const double t = warp_total(pend);
      if (lane == 0) sm.ch_part[0][pend_i] = t;
      pend_i = -1;
    }
  };
  for (;;) {
    const int64_t row = u.row0 + 32 * int64_t(c_lo + i) + lane;
    const T* vp = vals + e0 + lane;
    const CI* ip = idx + e0 + lane;
    T acc = T(0);
    // Every lane loads UA entries (past the slice's width it repeats the last
    // one, so no predicate stays live across the loads and the batch fits the
    // registers); only the slice's own entries gather p.
    for (int k0 = 0; k0 < w; k0 += UA) {
      if (UT > 0 && w - k0 <= UT) {
        T v[UT > 0 ? UT : 1];
        int c[UT > 0 ? UT : 1];
#pragma unroll
        for (int q = 0; q < UT; ++q) {
          const int kk = min(k0 + q, w - 1);
          v[q] = __ldcs(vp + 32 * kk);
          c[q] = ldidx(ip + 32 * kk);
        }
        settle();
#pragma unroll
        for (int q = 0; q < UT; ++q)
          if (k0 + q < w) {
            const int64_t gc = gcol<CI>(c[q], row, u.row0);
            acc += v[q] * (WIN ? pw[gc & wmask] : ld_pol(pv_ + gc, x.keep));
          }
        break;
      }
      T v[UA];
      int c[UA];
#pragma unroll
      for (int q = 0; q < UA; ++q) {
        const int kk = min(k0 + q, w - 1);
        v[q] = __ldcs(vp + 32 * kk);
        c[q] = ldidx(ip + 32 * kk);
      }
      settle();
#pragma unroll
      for (int q = 0; q < UA; ++q)
        if (k0 + q < w) {
          const int64_t gc = gcol<CI>(c[q], row, u.row0);
          acc += v[q] * (WIN ? pw[gc & wmask] : ld_pol(pv_ + gc, x.keep));
        }
    }
    settle();
    st_pol(a.y + row, acc, x.keep);
    const T pv = WIN ? pw[row & wmask] : ld_pol(pv_ + row, x.keep);
    pend = double(pv) * double(acc);
    pend_i = i;
    i = __shfl_sync(0xffffffffu, nxt, 0);
    if (i >= n) break;
    if (lane == 0) nxt = atomicAdd(&sm.ch_next, 1);
    e0 = sm.ch_off[i];
    w = int((sm.ch_off[i + 1] - e0) >> 5);
  }
  settle();
}

// C, single, refining: r = fl(b - A64 (x + d)); ||r64||^2, r.r, r.p per
// slice of the chunk [c_lo, c_hi) (handed out like the product's).
// WIN: x + d (FP64) is read from the CTA's shared-memory window.
constexpr int UC1 = 8;
template <typename T, typename CI, bool WIN>
__device__ __noinline__ void tileC1(const Ctx<T, CI>& x, const Unit& u, int c_lo, int c_hi,
                                    int64_t wbase, Smem& sm) {
  const Args<T, CI>& a = x.a;
  const double* xw = reinterpret_cast<const double*>(bat_dyn + win_offset(a.nunits)) - wbase;
  const int lane = int(threadIdx.x) & 31;
  const double* __restrict__ vals = a.vals64;
  const CI* __restrict__ idx = a.idx;
  const int n = c_hi - c_lo;
  int i = int(threadIdx.x) >> 5;
  while (i < n) {
    int nxt = 0;
    if (lane == 0) nxt = atomicAdd(&sm.ch_next, 1);
    const int64_t e0 = sm.ch_off[i];
    const int w = int((sm.ch_off[i + 1] - e0) >> 5);
    const int64_t row = u.row0 + 32 * int64_t(c_lo + i) + lane;
    const double* vp = vals + e0 + lane;
    const CI* ip = idx + e0 + lane;
    double acc = 0.0;
    for (int k0 = 0; k0 < w; k0 += UC1) {
      double v[UC1];
      int c[UC1];
#pragma unroll
      for (int q = 0; q < UC1; ++q) {
        const int kk = min(k0 + q, w - 1);
        v[q] = __ldcs(vp + 32 * kk);
        c[q] = ldidx(ip + 32 * kk);
      }
#pragma unroll
      for (int q = 0; q < UC1; ++q)
        if (k0 + q < w) {
          const int64_t cc = gcol<CI>(c[q], row, u.row0);
          acc += v[q] * (WIN ? xw[cc] : ld_pol(a.x + cc, x.keep) + double(ld_pol(a.d + cc, x.keep)));
        }
    }
    const double r64 = ld_pol(a.b + row, x.keep) - acc;
    const T rf = T(r64);
    st_pol(a.r + row, rf, x.keep);
    const T pv = ld_pol(a.p + row, x.keep);
    const double t0 = warp_total(r64 * r64);
    const double t1 = warp_total(double(rf) * double(rf));
    const double t2 = warp_total(double(rf) * double(pv));
    if (lane == 0) {
      sm.ch_part[0][i] = t0;
      sm.ch_part[1][i] = t1;
      sm.ch_part[2][i] = t2;
    }
    i = __shfl_sync(0xffffffffu, nxt, 0);
  }
}

// Rows of a single-unit tile for the vector phases: 4 consecutive rows per
// lane per step, 128 rows per warp step.  The bodies copy the vector
// pointers into __restrict__ locals so a step's loads can be issued before
// the previous step's stores.
#define BAT_ROWS4(i)                                                                 \
  const int64_t beg_ = u.row0 + 32 * int64_t(j) * a.tile_slices;                     \
  const int64_t end_ = u.row0 + 32 * int64_t(min(u.nslices, (j + 1) * a.tile_slices)); \
  _Pragma("unroll 2") for (int64_t i = beg_ + 4 * (int(threadIdx.x) & 31); i < end_; i += 128)

template <typename T, typename CI>
__device__ __noinline__ void tileB1(const Ctx<T, CI>& x, const Unit& u, int j, double* ts) {
  const Args<T, CI>& a = x.a;
  const T af = T(__ldcg(&a.slots[u.slot0].alpha));
  T* __restrict__ dd = a.d;
  T* __restrict__ rr = a.r;
  const T* __restrict__ pp = a.p;
  const T* __restrict__ yy = a.y;
  double t = 0.0;
  BAT_ROWS4(i) {
    const Four<T> p = ld4(pp + i), y = ld4(yy + i);
    Four<T> r = ld4(rr + i), d = ld4(dd + i);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      d.v[e] = d.v[e] + af * p.v[e];
      r.v[e] = r.v[e] - af * y.v[e];
      t += double(r.v[e]) * double(r.v[e]);
    }
    st4(dd + i, d);
    st4(rr + i, r);
  }
  ts[0] = warp_total(t);
}

// C, single, not refining: p = r + beta p.
template <typename T, typename CI>
__device__ __noinline__ void tileP1(const Ctx<T, CI>& x, const Unit& u, int j) {
  const Args<T, CI>& a = x.a;
  const T bf = T(__ldcg(&a.slots[u.slot0].beta));
  T* __restrict__ pp = a.p;
  const T* __restrict__ rr = a.r;
  BAT_ROWS4(i) {
    const Four<T> r = ld4(rr + i);
    Four<T> p = ld4(pp + i);
#pragma unroll
    for (int e = 0; e < 4; ++e) p.v[e] = r.v[e] + bf * p.v[e];
    st4(pp + i, p);
  }
}

// D, single (a refined unit): x += d, d = 0; p = r + beta (p - c r) while
// the recurrence continues.
template <typename T, typename CI>
__device__ __noinline__ void tileD1(const Ctx<T, CI>& x, const Unit& u, int j) {
  const Args<T, CI>& a = x.a;
  const Slot* sl = a.slots + u.slot0;
  const bool act = __ldcg(&sl->active) != 0;
  const T bf = T(__ldcg(&sl->beta)), cf = T(__ldcg(&sl->c));
  T* __restrict__ dd = a.d;
  double* __restrict__ xx = a.x;
  T* __restrict__ pp = a.p;
  const T* __restrict__ rr = a.r;
  BAT_ROWS4(i) {
    Four<T> d = ld4(dd + i);
    Four<double> xv = ld4(xx + i);
    Four<T> p, r;
    if (act) {
      p = ld4(pp + i);
      r = ld4(rr + i);
    }
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      xv.v[e] = xv.v[e] + double(d.v[e]);
      d.v[e] = T(0);
    }
    st4(xx + i, xv);
    st4(dd + i, d);
    if (act) {
#pragma unroll
      for (int e = 0; e < 4; ++e) p.v[e] = r.v[e] + bf * (p.v[e] - cf * r.v[e]);
      st4(pp + i, p);
    }
  }
}

// Init, single: b in the planned order, x = d = 0, r = p = fl(b);
// ||b||^2, r.r.
template <typename T, typename CI>
__device__ __noinline__ void tileI1(const Ctx<T, CI>& x, const Unit& u, int j, double* ts) {
  const Args<T, CI>& a = x.a;
  const double* __restrict__ bu = a.b_user[u.sys];
  const int32_t* __restrict__ perm = a.perm;
  double* __restrict__ bb = a.b;
  double* __restrict__ xx = a.x;
  T* __restrict__ dd = a.d;
  T* __restrict__ rr = a.r;
  T* __restrict__ pp = a.p;
  double t0 = 0.0, t1 = 0.0;
  BAT_ROWS4(i) {
    Four<double> bv, zx;
    Four<T> rv, zt;
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int pr = perm[i + e];
      const double bi = pr >= 0 ? bu[pr] : 0.0;
      bv.v[e] = bi;
      rv.v[e] = T(bi);
      zx.v[e] = 0.0;
      zt.v[e] = T(0);
      t0 += bi * bi;
      t1 += double(rv.v[e]) * double(rv.v[e]);
    }
    st4(bb + i, bv);
    st4(xx + i, zx);
    st4(dd + i, zt);
    st4(rr + i, rv);
    st4(pp + i, rv);
  }
  ts[0] = warp_total(t0);
  ts[1] = warp_total(t1);
}

template <typename T, typename CI>
__device__ __noinline__ void tileF1(const Ctx<T, CI>& x, const Unit& u, int j) {
  const Args<T, CI>& a = x.a;
  double* __restrict__ xu = a.x_user[u.sys];
  const int32_t* __restrict__ perm = a.perm;
  const double* __restrict__ xx = a.x;
  const T* __restrict__ dd = a.d;
  BAT_ROWS4(i) {
    const Four<double> xv = ld4(xx + i);
    const Four<T> d = ld4(dd + i);
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const int pr = perm[i + e];
      if (pr >= 0) xu[pr] = xv.v[e] + double(d.v[e]);
    }
  }
}

// ---- block tiles ----------------------------------------------------------
// Vector phases: 4 block rows per warp step, lane l takes row l / 8 of the
// step and columns 4 (l % 8) .. 4 (l % 8) + 3 (one 16-byte access per
// vector).  Column sums are combined over the step's rows and moved to
// lane = column at the end.
#define BAT_BROWS(e)                                                      \
  const int r0_ = j * BT_MUL * a.tile_slices,                                   \
            r1_ = min(u.nslices, r0_ + BT_MUL * a.tile_slices);                   \
  _Pragma("unroll 2") for (int64_t e = int64_t(r0_ + (int(threadIdx.x) & 31) / 8) * BW + \
                                       4 * ((int(threadIdx.x) & 31) % 8);                  \
                           e < int64_t(r1_) * BW; e += 4 * BW)

__device__ __forceinline__ int bcol0() { return 4 * ((int(threadIdx.x) & 31) % 8); }

__device__ __forceinline__ void bsums_to_column(double (&v)[4]) {
#pragma unroll
  for (int o = 8; o < 32; o <<= 1)
#pragma unroll
    for (int r = 0; r < 4; ++r) v[r] += __shfl_xor_sync(0xffffffffu, v[r], o);
}

// Column sums held 4 per lane (lane l < 8: columns 4 l .. 4 l + 3) moved to
// lane = column.
__device__ __forceinline__ double to_column4(const double (&v)[4]) {
  const int lane = int(threadIdx.x) & 31;
  double out = 0.0;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const double t = __shfl_sync(0xffffffffu, v[r], lane / 4);
    if (lane % 4 == r) out = t;
  }
  return out;
}

template <typename T, typename CI>
__device__ __noinline__ void tileB2(const Ctx<T, CI>& x, const Unit& u, int j, double* ts) {
  const Args<T, CI>& a = x.a;
  const int c0 = bcol0();
  T af[4];
  bool act[4];
  double al[4];
  int ac[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {  // all the loads first: one round trip
    const Slot* sl = a.slots + u.slot0 + c0 + r;
    ac[r] = __ldcg(&sl->active);
    al[r] = __ldcg(&sl->alpha);
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    act[r] = ac[r] != 0;
    af[r] = act[r] ? T(al[r]) : T(0);
  }
  T* __restrict__ dd = a.dB;
  T* __restrict__ rr = a.rB;
  const T* __restrict__ pp = a.pB;
  const T* __restrict__ yy = a.yB;
  double t[4] = {0.0, 0.0, 0.0, 0.0};
  BAT_BROWS(e) {
    const Four<T> p = ld4(pp + e), y = ld4(yy + e);
    Four<T> r = ld4(rr + e), d = ld4(dd + e);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      d.v[c] = d.v[c] + af[c] * p.v[c];
      r.v[c] = r.v[c] - af[c] * y.v[c];
      t[c] += double(r.v[c]) * double(r.v[c]);
    }
    st4(dd + e, d);
    st4(rr + e, r);
  }
  bsums_to_column(t);
  ts[0] = to_column4(t);
}

// C, block, no column refines: p = r + beta p for the active columns.
template <typename T, typename CI>
__device__ __noinline__ void tileP2(const Ctx<T, CI>& x, const Unit& u, int j) {
  const Args<T, CI>& a = x.a;
  const int c0 = bcol0();
  T bf[4];
  bool act[4];
  double be[4];
  int ac[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const Slot* sl = a.slots + u.slot0 + c0 + r;
    ac[r] = __ldcg(&sl->active);
    be[r] = __ldcg(&sl->beta);
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    act[r] = ac[r] != 0;
    bf[r] = T(be[r]);
  }
  T* __restrict__ pp = a.pB;
  const T* __restrict__ rr = a.rB;
  BAT_BROWS(e) {
    const Four<T> r = ld4(rr + e);
    Four<T> p = ld4(pp + e);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (act[c]) p.v[c] = r.v[c] + bf[c] * p.v[c];
    st4(pp + e, p);
  }
}

template <typename T, typename CI>
__device__ __noinline__ void tileD2(const Ctx<T, CI>& x, const Unit& u, int j) {
  const Args<T, CI>& a = x.a;
  const int c0 = bcol0();
  T bf[4], cf[4];
  bool ref[4], act[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const Slot* sl = a.slots + u.slot0 + c0 + r;
    ref[r] = __ldcg(&sl->refine_at) == x.k;
    act[r] = __ldcg(&sl->active) != 0;
    bf[r] = T(__ldcg(&sl->beta));
    cf[r] = T(__ldcg(&sl->c));
  }
  T* __restrict__ dd = a.dB;
  double* __restrict__ xx = a.xB;
  T* __restrict__ pp = a.pB;
  const T* __restrict__ rr = a.rB;
  BAT_BROWS(e) {
    Four<T> d = ld4(dd + e), p = ld4(pp + e);
    const Four<T> r = ld4(rr + e);
    Four<double> xv = ld4(xx + e);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (ref[c]) {
        xv.v[c] = xv.v[c] + double(d.v[c]);
        d.v[c] = T(0);
        if (act[c]) p.v[c] = r.v[c] + bf[c] * (p.v[c] - cf[c] * r.v[c]);
      }
    st4(xx + e, xv);
    st4(dd + e, d);
    st4(pp + e, p);
  }
}

template <typename T, typename CI>
__device__ __noinline__ void tileI2(const Ctx<T, CI>& x, const Unit& u, int j, double* ts) {
  const Args<T, CI>& a = x.a;
  const int c0 = bcol0();
  const int32_t* __restrict__ bperm = a.bperm;
  const double* __restrict__ bu = a.B_user;
  double* __restrict__ bb = a.bB;
  double* __restrict__ xx = a.xB;
  T* __restrict__ dd = a.dB;
  T* __restrict__ rr = a.rB;
  T* __restrict__ pp = a.pB;
  double t0[4] = {0.0, 0.0, 0.0, 0.0}, t1[4] = {0.0, 0.0, 0.0, 0.0};
  BAT_BROWS(e) {
    const int row = int(e / BW);
    const int pr = bperm[row];
    Four<double> bv, zx;
    Four<T> rv, zt;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const double bi = (pr >= 0 && c0 + c < a.nrhs) ? bu[int64_t(pr) * a.nrhs + c0 + c] : 0.0;
      bv.v[c] = bi;
      rv.v[c] = T(bi);
      zx.v[c] = 0.0;
      zt.v[c] = T(0);
      t0[c] += bi * bi;
      t1[c] += double(rv.v[c]) * double(rv.v[c]);
    }
    st4(bb + e, bv);
    st4(xx + e, zx);
    st4(dd + e, zt);
    st4(rr + e, rv);
    st4(pp + e, rv);
  }
  bsums_to_column(t0);
  bsums_to_column(t1);
  ts[0] = to_column4(t0);
  ts[1] = to_column4(t1);
}

template <typename T, typename CI>
__device__ __noinline__ void tileF2(const Ctx<T, CI>& x, const Unit& u, int j) {
  const Args<T, CI>& a = x.a;
  const int c0 = bcol0();
  const int32_t* __restrict__ bperm = a.bperm;
  double* __restrict__ xu = a.X_user;
  const double* __restrict__ xx = a.xB;
  const T* __restrict__ dd = a.dB;
  BAT_BROWS(e) {
    const int pr = bperm[int(e / BW)];
    if (pr < 0) continue;
    const Four<double> xv = ld4(xx + e);
    const Four<T> d = ld4(dd + e);
#pragma unroll
    for (int c = 0; c < 4; ++c)
      if (c0 + c < a.nrhs) xu[int64_t(pr) * a.nrhs + c0 + c] = xv.v[c] + double(d.v[c]);
  }
}

// Column sums held R per lane (lanes l < KW of segment 0 after the segment
// combine) moved to lane = column.
template <int R>
__device__ __forceinline__ double to_column(const double (&v)[R]) {
  const int lane = int(threadIdx.x) & 31;
  double out = 0.0;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const double t = __shfl_sync(0xffffffffu, v[r], lane / R);
    if (lane % R == r) out = t;
  }
  return out;
}

// A, block: Y = A P for the tile's rows, R rows per warp step (32 / R lanes
// per row, R columns per lane); p.y per column.
template <typename T, typename CI, int R>
__device__ __noinline__ void tileA2(const Ctx<T, CI>& x, const Unit& u, int j, double* ts) {
  const Args<T, CI>& a = x.a;
  constexpr int KW = 32 / R;
  const int lane = int(threadIdx.x) & 31, seg = lane / KW, cl = lane % KW, c0 = cl * R;
  const int r0 = j * BT_MUL * a.tile_slices, r1 = min(u.nslices, r0 + BT_MUL * a.tile_slices);
  const T* __restrict__ pB = a.pB;
  double py[R];
#pragma unroll
  for (int r = 0; r < R; ++r) py[r] = 0.0;
  for (int rb = r0; rb < r1; rb += R) {
    const int row = rb + seg;
    const int s = a.brp[row], len = a.brp[row + 1] - s;
    int maxlen = len;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
    T acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = T(0);
    for (int j0 = 0; j0 < maxlen; j0 += KW) {
      const bool have = j0 + cl < len;
      const int cj = have ? __ldcs(a.bcol + s + j0 + cl) : 0;
      const T vj = have ? __ldcs(a.bval + s + j0 + cl) : T(0);
      const int cnt = min(KW, maxlen - j0);
      for (int t0 = 0; t0 < cnt; t0 += U) {
        int c[U];
        T v[U];
        T g[U][R];
#pragma unroll
        for (int q = 0; q < U; ++q) {
          c[q] = __shfl_sync(0xffffffffu, cj, (t0 + q) % KW, KW);
          v[q] = __shfl_sync(0xffffffffu, vj, (t0 + q) % KW, KW);
        }
        // Every index is a valid row (0 for a missing entry, another entry's
        // column past cnt), so the gathers need no predicate; the sum takes
        // the first cnt.
#pragma unroll
        for (int q = 0; q < U; ++q) ldR<T, R>(pB + int64_t(c[q]) * BW + c0, g[q]);
#pragma unroll
        for (int q = 0; q < U; ++q)
          if (t0 + q < cnt)
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] += v[q] * g[q][r];
      }
    }
    stR<T, R>(a.yB + int64_t(row) * BW + c0, acc);
    T pv[R];
    ldR<T, R>(pB + int64_t(row) * BW + c0, pv);
#pragma unroll
    for (int r = 0; r < R; ++r) py[r] += double(pv[r]) * double(acc[r]);
  }
#pragma unroll
  for (int o = KW; o < 32; o <<= 1)
#pragma unroll
    for (int r = 0; r < R; ++r) py[r] += __shfl_xor_sync(0xffffffffu, py[r], o);
  ts[0] = to_column<R>(py);
}

// C, block (some column refines): refining columns r = fl(b - A64 (x + d))
// with their three sums; the other active columns p = r + beta p.
template <typename T, typename CI, int R>
__device__ __noinline__ void tileC2(const Ctx<T, CI>& x, const Unit& u, int j, double* ts) {
  const Args<T, CI>& a = x.a;
  constexpr int KW = 32 / R;
  constexpr int UC = 4;  // entries in flight (each R doubles of x and R of d)
  const int lane = int(threadIdx.x) & 31, seg = lane / KW, cl = lane % KW, c0 = cl * R;
  const int r0 = j * BT_MUL * a.tile_slices, r1 = min(u.nslices, r0 + BT_MUL * a.tile_slices);
  bool ref[R], act[R];
  T bf[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const Slot* sl = a.slots + u.slot0 + c0 + r;
    ref[r] = __ldcg(&sl->refine_at) == x.k;
    act[r] = __ldcg(&sl->active) != 0;
    bf[r] = T(__ldcg(&sl->beta));
  }
  double t0[R], t1[R], t2[R];
#pragma unroll
  for (int r = 0; r < R; ++r) t0[r] = t1[r] = t2[r] = 0.0;
  for (int rb = r0; rb < r1; rb += R) {
    const int row = rb + seg;
    const int s = a.brp[row], len = a.brp[row + 1] - s;
    int maxlen = len;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxlen = max(maxlen, __shfl_xor_sync(0xffffffffu, maxlen, o));
    double acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0.0;
    for (int j0 = 0; j0 < maxlen; j0 += KW) {
      const bool have = j0 + cl < len;
      const int cj = have ? __ldcs(a.bcol + s + j0 + cl) : 0;
      const double vj = have ? __ldcs(a.bval64 + s + j0 + cl) : 0.0;
      const int cnt = min(KW, maxlen - j0);
      for (int t0i = 0; t0i < cnt; t0i += UC) {
        int c[UC];
        double v[UC], gx[UC][R];
        T gd[UC][R];
#pragma unroll
        for (int q = 0; q < UC; ++q) {
          c[q] = __shfl_sync(0xffffffffu, cj, (t0i + q) % KW, KW);
          v[q] = __shfl_sync(0xffffffffu, vj, (t0i + q) % KW, KW);
        }
#pragma unroll
        for (int q = 0; q < UC; ++q) {
          ldR<double, R>(a.xB + int64_t(c[q]) * BW + c0, gx[q]);
          ldR<T, R>(a.dB + int64_t(c[q]) * BW + c0, gd[q]);
        }
#pragma unroll
        for (int q = 0; q < UC; ++q)
          if (t0i + q < cnt)
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] += v[q] * (gx[q][r] + double(gd[q][r]));
      }
    }
    const int64_t e = int64_t(row) * BW + c0;
    double bv[R];
    T rv[R], pv[R];
    ldR<double, R>(a.bB + e, bv);
    ldR<T, R>(a.rB + e, rv);
    ldR<T, R>(a.pB + e, pv);
    T rn[R], pn[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
      rn[r] = rv[r];
      pn[r] = pv[r];
      if (ref[r]) {
        const double r64 = bv[r] - acc[r];
        rn[r] = T(r64);
        t0[r] += r64 * r64;
        t1[r] += double(rn[r]) * double(rn[r]);
        t2[r] += double(rn[r]) * double(pv[r]);
      } else if (act[r]) {
        pn[r] = rv[r] + bf[r] * pv[r];
      }
    }
    stR<T, R>(a.rB + e, rn);
    stR<T, R>(a.pB + e, pn);
  }
#pragma unroll
  for (int o = KW; o < 32; o <<= 1)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      t0[r] += __shfl_xor_sync(0xffffffffu, t0[r], o);
      t1[r] += __shfl_xor_sync(0xffffffffu, t1[r], o);
      t2[r] += __shfl_xor_sync(0xffffffffu, t2[r], o);
    }
  ts[0] = to_column<R>(t0);
  ts[1] = to_column<R>(t1);
  ts[2] = to_column<R>(t2);
}

// ---------------------------------------------------------------------------
// Recurrence updates, made by the CTA that completes a unit's reduction
// (single units: lane 0 for slot0; block: lane l for column l).
// ---------------------------------------------------------------------------
// Slot fields go through L2 (another CTA may have written them since this
// SM last read them).  All lanes of the warp call it; `own` lanes update
// their slot (lane 0 for a single unit, every lane for the block's
// columns).  The block's columns refine together: when one of them is due,
// every active column takes the FP64 residual in the same iteration, since
// the block's refinement product serves all its columns at once.
template <typename T, typename CI>
__device__ __forceinline__ void update_slot(const Ctx<T, CI>& x, int ph, Slot* gsl, bool own,
                                            bool blk, const double* tot, bool& act,
                                            bool& refine) {
  const Args<T, CI>& a = x.a;
  Slot L;
  act = false;
  refine = false;
  if (own) {
    const double* src = reinterpret_cast<const double*>(gsl);
    double* dst = reinterpret_cast<double*>(&L);
#pragma unroll
    for (int i = 0; i < int(sizeof(Slot) / sizeof(double)); ++i) dst[i] = __ldcg(src + i);
  }
  if (own && ph == PH_INIT) {
    const double rr0 = tot[0];
    L.rr0 = rr0;
    L.rr = tot[1];
    L.rr_max = tot[1];
    L.rr_true = rr0;
    L.rr_prev = 0.0;
    L.alpha = L.beta = L.c = 0.0;
    L.its = 0;
    L.refs = 0;
    L.status = SPMV_SUCCESS;
    L.converged = rr0 == 0.0;
    L.refine_at = -1;
    act = a.kmax > 0 && rr0 > 0.0 && isfinite(rr0);
    L.active = act;
  } else if (own && L.active) {
    act = true;
    if (ph == PH_A) {
      const double pap = tot[0];
      if (pap == 0.0 || !isfinite(pap)) {
        L.status = SPMV_ERROR_BREAKDOWN;
        L.active = 0;
        act = false;
      } else {
        L.alpha = L.rr / pap;
      }
    } else if (ph == PH_B) {
      const double rr_new = tot[0];
      const int its = L.its + 1;
      L.its = its;
      const double rr_max = fmax(L.rr_max, rr_new);
      L.rr_max = rr_max;
      refine = rr_new < a.delta2 * rr_max || rr_new / L.rr0 < a.rtol2 || its >= a.kmax ||
               !isfinite(rr_new);
      L.beta = rr_new / L.rr;
      L.c = 0.0;
      L.rr_prev = L.rr;
      L.rr = rr_new;
    } else if (ph == PH_C && L.refine_at == x.k) {
      L.refs += 1;
      L.rr_true = tot[0];
      L.rr_max = tot[1];
      bool stop = false;
      if (tot[0] / L.rr0 < a.rtol2) {
        L.converged = 1;
        stop = true;
      }
      if (!isfinite(tot[0])) {
        L.status = SPMV_ERROR_BREAKDOWN;
        stop = true;
      }
      L.beta = tot[1] / L.rr_prev;
      L.rr = tot[1];
      L.c = tot[1] > 0.0 ? tot[2] / tot[1] : 0.0;
      if (L.its >= a.kmax) stop = true;
      if (stop) {
        L.active = 0;
        act = false;
      }
      refine = true;
    }
  }
  if (ph == PH_B) {
    if (blk && __ballot_sync(0xffffffffu, refine) != 0u && act) refine = true;
    if (own && refine) L.refine_at = x.k;
  }
  if (own) {
    const double* src = reinterpret_cast<const double*>(&L);
    double* dst = reinterpret_cast<double*>(gsl);
#pragma unroll
    for (int i = 0; i < int(sizeof(Slot) / sizeof(double)); ++i) __stcg(dst + i, src[i]);
  }
}

// ---------------------------------------------------------------------------
// Copies fl64(x + d)[row0 + wlo, row0 + wlo + wsize) into the window (the
// refinement product's operand).
template <typename T, typename CI>
__device__ __forceinline__ void load_window_xd(const Args<T, CI>& a, const Unit& un, int wlo,
                                               int wsize) {
  double* win = reinterpret_cast<double*>(bat_dyn + win_offset(a.nunits));
  const double* xs = a.x + un.row0 + wlo;
  const T* ds = a.d + un.row0 + wlo;
  for (int i0 = 4 * int(threadIdx.x); i0 < wsize; i0 += 4 * 2 * NT) {
    Four<double> xv[2];
    Four<T> dv[2];
#pragma unroll
    for (int u = 0; u < 2; ++u)
      if (i0 + u * 4 * NT < wsize) {
        xv[u] = ld4(xs + i0 + u * 4 * NT);
        dv[u] = ld4(ds + i0 + u * 4 * NT);
      }
#pragma unroll
    for (int u = 0; u < 2; ++u)
      if (i0 + u * 4 * NT < wsize) {
#pragma unroll
        for (int e = 0; e < 4; ++e) xv[u].v[e] = xv[u].v[e] + double(dv[u].v[e]);
        st4(win + i0 + u * 4 * NT, xv[u]);
      }
  }
}

// One phase over a unit list.
// ---------------------------------------------------------------------------
template <int PH, typename T, typename CI, int R>
__device__ __forceinline__ void unit_info(const Args<T, CI>& a, int k, int u, int& ntiles,
                                          int& wt, int& kind, bool& refine) {
  const Unit& un = a.units[u];
  kind = un.kind;
  ntiles = unit_tiles(un, a.tile_slices);
  refine = false;
  if (PH == PH_C) refine = __ldcg(&a.ust[u].refine_at) == k;
  wt = tile_weight(a.w, PH, kind, refine);
}

template <int PH>
struct NSumOf {
  static constexpr int value = PH == PH_INIT ? 2 : (PH == PH_A || PH == PH_B) ? 1 : PH == PH_C ? 3 : 0;
};

// Window of p for a chunk of a unit's slices [s_lo, s_hi): the smallest and
// largest column the chunk reads (and its own rows).  All NT threads; the
// result is valid in all.
template <typename T, typename CI>
__device__ __forceinline__ bool chunk_window(const Args<T, CI>& a, const Unit& un, int s_lo,
                                             int s_hi, Smem& sm, int& wlo, int& wsize, int cap) {
  const int lane = int(threadIdx.x) & 31, warp = int(threadIdx.x) >> 5;
  int lo = 32 * s_lo, hi = 32 * s_hi - 1;
  for (int t = s_lo + int(threadIdx.x); t <= s_hi; t += NT) {
    sm.ch_off[t - s_lo] = a.soff[un.slice0 + t];
    if (t == s_hi) break;
    const int2 b = a.sbound[un.slice0 + t];
    lo = min(lo, b.x);
    hi = max(hi, b.y);
  }
  if (threadIdx.x == 0) sm.ch_next = NW;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xffffffffu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xffffffffu, hi, o));
  }
  if (lane == 0) {
    sm.wmin[warp] = lo;
    sm.wmax[warp] = hi;
  }
  __syncthreads();
  lo = sm.wmin[0];
  hi = sm.wmax[0];
#pragma unroll
  for (int w = 1; w < NW; ++w) {
    lo = min(lo, sm.wmin[w]);
    hi = max(hi, sm.wmax[w]);
  }
  wlo = lo & ~3;
  wsize = ((hi + 1 - wlo) + 3) & ~3;
  return wsize <= cap;
}

// Copies p[row0 + wlo, row0 + wlo + wsize) into the window (16-byte steps:
// row0 is a multiple of 32 and wlo of 4).  FP32: the window is a ring (row g
// at g & (win_cap - 1)) and only the rows it does not hold yet are copied;
// sm.ring_lo/ring_hi are read here and updated by the caller after the
// barrier that follows.
template <typename T, typename CI>
__device__ __forceinline__ void load_window(const Args<T, CI>& a, const Unit& un, int wlo,
                                            int wsize, const Smem& sm) {
  T* win = reinterpret_cast<T*>(bat_dyn + win_offset(a.nunits));
  auto copy = [&](int64_t g0, int64_t g1, int64_t mask, int64_t base) {
    // Rows [g0, g1) (multiples of 4) to win[(g - base) & mask].
    const T* src = a.p + g0;
    const int64_t n = g1 - g0;
    for (int64_t i0 = 4 * int64_t(threadIdx.x); i0 < n; i0 += 4 * 4 * NT) {
      Four<T> v[4];
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (i0 + u * 4 * NT < n) v[u] = ld4(src + i0 + u * 4 * NT);
#pragma unroll
      for (int u = 0; u < 4; ++u)
        if (i0 + u * 4 * NT < n) st4(win + ((g0 + i0 + u * 4 * NT - base) & mask), v[u]);
    }
  };
  const int64_t g0 = un.row0 + wlo, g1 = g0 + wsize;
  if (sizeof(T) != 4) {
    copy(g0, g1, int64_t(-1), g0);
    return;
  }
  const int64_t mask = int64_t(a.win_cap - 1);
  const int64_t r0 = sm.ring_lo, r1 = sm.ring_hi + 1;
  if (r0 >= r1 || r1 <= g0 || r0 >= g1) {
    copy(g0, g1, mask, 0);
  } else {
    if (g0 < r0) copy(g0, r0, mask, 0);
    if (r1 < g1) copy(r1, g1, mask, 0);
  }
}

// The recurrence update of a unit whose sums are complete (acc: per lane for
// the block's columns, in every lane for a single unit), by one warp.
template <int PH, typename T, typename CI>
__device__ __forceinline__ void finish_unit(const Ctx<T, CI>& x, int u, const Unit& un, bool blk,
                                            const double* acc) {
  const Args<T, CI>& a = x.a;
  const int lane = int(threadIdx.x) & 31;
  bool act = false, refine = false;
  update_slot(x, PH, a.slots + un.slot0 + (blk ? lane : 0), blk || lane == 0, blk, acc, act,
              refine);
  const unsigned am = __ballot_sync(0xffffffffu, act);
  const unsigned rm = __ballot_sync(0xffffffffu, refine);
  if (lane == 0) {
    if (PH == PH_INIT) {
      a.ust[u].active = am != 0;
      a.ust[u].refine_at = -1;
    } else if (PH == PH_A || PH == PH_C) {
      a.ust[u].active = am != 0;
    } else if (PH == PH_B) {
      if (rm) a.ust[u].refine_at = x.k;
    }
    a.tickets[u] = 0u;
    __threadfence();
  }
}

// One phase over a unit list.  CTA c (of the G' = min(G, W) CTAs that take
// part) covers weight positions [c W / G', (c + 1) W / G'); every CTA whose
// range overlaps a unit's tile starts -- the CTAs cta_of(first tile) ..
// cta_of(last tile), each of them non-empty -- publishes one partial per sum
// for that unit (zero when none of the unit's tiles starts in its range) and
// takes a ticket; the one that completes the count adds the partials in CTA
// order.
template <int PH, typename T, typename CI, int R>
__device__ void run_phase(const Ctx<T, CI>& x, int cnt, long long W, const int* lu,
                          const int* lw, Smem& sm) {
  constexpr int NS = NSumOf<PH>::value;
  constexpr int NS1 = NS > 0 ? NS : 1;
  const Args<T, CI>& a = x.a;
  if (cnt == 0 || W <= 0) return;
  // With a.prof, each CTA adds its time in phases A, B and C (per CTA).
  struct CtaClock {
    unsigned long long* slot;
    unsigned long long t0;
    __device__ ~CtaClock() {
      if (slot) atomicAdd(slot, gtimer() - t0);
    }
  } cta_clock{(a.prof && threadIdx.x == 0 && (PH == PH_A || PH == PH_B || PH == PH_C))
                  ? a.prof + 2 * a.prof_cap + 16 + (PH == PH_A ? 0 : PH == PH_B ? 1 : 2) * 1024 +
                        blockIdx.x
                  : nullptr,
              gtimer()};
  const int G = int(W < (long long)gridDim.x ? W : (long long)gridDim.x), cta = int(blockIdx.x);
  if (cta >= G) return;
  const long long Lr = (long long)cta * W / G, Rr = (long long)(cta + 1) * W / G;
  const int lane = int(threadIdx.x) & 31, warp = int(threadIdx.x) >> 5;
  double (*bsum)[NSUM][BW] = block_sums(a.nunits);
  // First list entry whose weight span reaches Lr.
  int i0 = 0;
  {
    int lo = 0, hi = cnt - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (lw[mid] <= Lr)
        lo = mid;
      else
        hi = mid - 1;
    }
    i0 = lo;
  }
  while (i0 < cnt && lw[i0] < Rr) {
    // The window region also holds the block's sums: the ring of p starts
    // empty in every pass.
    if (threadIdx.x == 0) {
      sm.ring_lo = 1;
      sm.ring_hi = 0;
    }
    // Pass table: up to MAXQ consecutive entries this CTA reports for.
    if (warp == 0) {
      int nq = 0, pos = 0, i = i0;
      while (nq < MAXQ && i < cnt && lw[i] < Rr) {
        const int idx = i + lane;
        int ja = 0, jb = 0, T_ = 0, wt = 1, kind = 0;
        bool ref = false;
        long long cf = 0, cl = -1;
        const bool in = idx < cnt && lw[idx] < Rr;
        if (in) {
          unit_info<PH, T, CI, R>(a, x.k, lu[idx], T_, wt, kind, ref);
          ja = tiles_from(Lr - lw[idx], wt, T_);
          jb = tiles_from(Rr - lw[idx], wt, T_);
          cf = cta_of(lw[idx], W, G);
          cl = cta_of(lw[idx] + (long long)(T_ - 1) * wt, W, G);
        }
        const bool has = in && cta <= cl;
        const unsigned m = __ballot_sync(0xffffffffu, has);
        const unsigned inm = __ballot_sync(0xffffffffu, in);
        const int before = __popc(m & ((1u << lane) - 1));
        const int cntl = has ? jb - ja : 0;
        int incl = cntl;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
          const int v = __shfl_up_sync(0xffffffffu, incl, o);
          if (lane >= o) incl += v;
        }
        const int slot = nq + before;
        const bool keep = has && slot < MAXQ;
        const unsigned km = __ballot_sync(0xffffffffu, keep);
        if (keep) {
          sm.q_list[slot] = idx;
          sm.q_ja[slot] = ja;
          sm.q_jb[slot] = jb;
          sm.q_t[slot] = T_;
          sm.q_ref[slot] = ref;
          sm.q_kind[slot] = kind;
          sm.q_cf[slot] = int(cf);
          sm.q_ns[slot] = int(cl - cf + 1);
          sm.q_pos[slot] = pos + incl - cntl;
        }
        if (km != m) {
          const int first_cut = __ffs(m & ~km) - 1;
          pos += __shfl_sync(0xffffffffu, incl - cntl, first_cut);
          nq = MAXQ;
          i = i + first_cut;
          break;
        }
        pos += __shfl_sync(0xffffffffu, incl, 31);
        nq += __popc(km);
        const int scanned = 32 - __clz(inm);
        i += scanned;
        if (scanned < 32) break;
      }
      if (lane == 0) {
        sm.nq = nq;
        sm.q_pos[nq] = pos;
        sm.next_i = i;
      }
    }
    __syncthreads();
    const int nq = sm.nq;
    if (NS > 0) {
      for (int t = int(threadIdx.x); t < nq * NW * NSUM; t += NT) (&sm.sums[0][0][0])[t] = 0.0;
      if (PH != PH_A && PH != PH_C)
        for (int t = int(threadIdx.x); t < NW * NSUM * BW; t += NT)
          (&bsum[0][0][0])[t] = 0.0;
      __syncthreads();
    }
    double run[NS1];
    int a_end = 0;  // phase A: end of the current chunk's slices
    auto flush = [&](int qq) {
      if (NS == 0) return;
      if (sm.q_kind[qq] == 0) {
        if (lane == 0)
#pragma unroll
          for (int s = 0; s < NS1; ++s) sm.sums[qq][warp][s] = run[s];
      } else {
#pragma unroll
        for (int s = 0; s < NS1; ++s) bsum[warp][s][lane] = run[s];
      }
    };
    auto body = [&](const Unit& un, int qq, int j, int64_t wbase, bool win) {
      double ts[NSUM] = {0.0, 0.0, 0.0};
      if (un.kind == 0) {
        if (PH == PH_INIT) tileI1(x, un, j, ts);
        if (PH == PH_A) {
          // j: the chunk's first slice; its slices [j, a_end) are handed out
          // to the warps, their sums left in sm.ch_part.
          if (win)
            tileA1<T, CI, true>(x, un, j, a_end, wbase, sm);
          else
            tileA1<T, CI, false>(x, un, j, a_end, 0, sm);
        }
        if (PH == PH_B) tileB1(x, un, j, ts);
        if (PH == PH_C) {
          if (sm.q_ref[qq]) {
            if (win)
              tileC1<T, CI, true>(x, un, j, a_end, wbase, sm);
            else
              tileC1<T, CI, false>(x, un, j, a_end, 0, sm);
          } else {
            tileP1(x, un, j);
          }
        }
        if (PH == PH_D) tileD1(x, un, j);
        if (PH == PH_FINAL) tileF1(x, un, j);
      } else {
        if (PH == PH_INIT) tileI2(x, un, j, ts);
        if (PH == PH_A) tileA2<T, CI, R>(x, un, j, ts);
        if (PH == PH_B) tileB2(x, un, j, ts);
        if (PH == PH_C) {
          if (sm.q_ref[qq])
            tileC2<T, CI, R>(x, un, j, ts);
          else
            tileP2(x, un, j);
        }
        if (PH == PH_D) tileD2(x, un, j);
        if (PH == PH_FINAL) tileF2(x, un, j);
      }
#pragma unroll
      for (int s = 0; s < NS1; ++s) run[s] += ts[s];
    };
    if (PH == PH_A || PH == PH_C) {
      // Product units in chunks of NW tiles: the chunk's slices are dealt
      // round robin to the warps, and (single units) the chunk's window of
      // the gathered vector is staged in shared memory first.  In phase C
      // the other units' tiles go one per warp in the same loop.
      const bool prof = PH == PH_A && a.prof != nullptr && threadIdx.x == 0;
      unsigned long long t_a = prof ? gtimer() : 0, t_w = 0, t_l = 0, t_b = 0;
      for (int qq = 0; qq < nq; ++qq) {
        const Unit un = a.units[lu[sm.q_list[qq]]];
#pragma unroll
        for (int s = 0; s < NS1; ++s) run[s] = 0.0;
        if (un.kind != 0) {
          __syncthreads();
          for (int t = int(threadIdx.x); t < NW * NSUM * BW; t += NT) (&bsum[0][0][0])[t] = 0.0;
          if (threadIdx.x == 0) {
            sm.ring_lo = 1;
            sm.ring_hi = 0;
          }
          __syncthreads();
        }
        for (int c0 = sm.q_ja[qq]; c0 < sm.q_jb[qq]; c0 += NW) {
          const int c1 = min(sm.q_jb[qq], c0 + NW);
          bool win = false;
          int wlo = 0, wsize = 0;
          unsigned long long t0 = prof ? gtimer() : 0, t1 = t0, t2 = t0;
          const bool chunked = un.kind == 0 && (PH == PH_A || sm.q_ref[qq]);
          if (chunked) {
            const int cap = PH == PH_A ? a.win_cap : a.win_cap * int(sizeof(T)) / 8;
            win = chunk_window(a, un, c0 * a.tile_slices,
                               min(un.nslices, c1 * a.tile_slices), sm, wlo, wsize, cap);
            if (prof) t1 = gtimer();
            if (win) {
              if (PH == PH_A)
                load_window(a, un, wlo, wsize, sm);
              else
                load_window_xd(a, un, wlo, wsize);
            }
            __syncthreads();
            if (PH == PH_A && win && threadIdx.x == 0) {
              sm.ring_lo = un.row0 + wlo;
              sm.ring_hi = un.row0 + wlo + wsize - 1;
            }
            if (prof) t2 = gtimer();
          }
          if (chunked) {
            // The chunk's slices, handed out to the warps; then warp 0 adds
            // their sums in slice order (the same order on every run).
            const int c_lo = c0 * a.tile_slices;
            a_end = min(un.nslices, c1 * a.tile_slices);
            if (c_lo + warp < a_end) body(un, qq, c_lo, un.row0 + wlo, win);
            __syncthreads();
            if (warp == 0) {
#pragma unroll
              for (int s = 0; s < NS; ++s) {
                double v = 0.0;
                for (int i = lane; i < a_end - c_lo; i += 32) v += sm.ch_part[s][i];
                run[s] += warp_total(v);
              }
            }
          } else if (warp < c1 - c0) {
            body(un, qq, c0 + warp, 0, false);
          }
          if (prof) {
            const unsigned long long t3 = gtimer();
            t_w += t1 - t0;
            t_l += t2 - t1;
            t_b += t3 - t2;
          }
        }
        flush(qq);
      }
      if (prof) {
        unsigned long long* acc = a.prof + 2 * a.prof_cap;
        atomicAdd(acc + 0, t_w);
        atomicAdd(acc + 1, t_l);
        atomicAdd(acc + 2, t_b);
        atomicAdd(acc + 3, gtimer() - t_a);
        atomicMax(acc + 4, gtimer() - t_a);
        atomicAdd(acc + 5, 1ull);
      }
    } else {
      // Warps deal the pass's tiles round robin.
      const int P = sm.q_pos[nq];
#pragma unroll
      for (int s = 0; s < NS1; ++s) run[s] = 0.0;
      int q = 0, cur = -1;
      for (int pos = warp; pos < P; pos += NW) {
        while (pos >= sm.q_pos[q + 1]) ++q;
        if (q != cur) {
          if (cur >= 0) flush(cur);
          cur = q;
#pragma unroll
          for (int s = 0; s < NS1; ++s) run[s] = 0.0;
        }
        const Unit un = a.units[lu[sm.q_list[q]]];
        body(un, q, sm.q_ja[q] + (pos - sm.q_pos[q]), 0, false);
      }
      if (cur >= 0) flush(cur);
    }
    if (NS > 0) {
      if (threadIdx.x == 0) sm.blk_last = -1;
      __syncthreads();
      for (int qq = warp; qq < nq; qq += NW) {
        const int u = lu[sm.q_list[qq]];
        const Unit& un = a.units[u];
        const bool blk = sm.q_kind[qq] != 0;
        const int width = blk ? BW : 1;
        const int nslot = sm.q_ns[qq];
        double tot[NSUM] = {0.0, 0.0, 0.0};
        if (!blk) {
          if (lane == 0)
            for (int w = 0; w < NW; ++w)
#pragma unroll
              for (int s = 0; s < NS; ++s) tot[s] += sm.sums[qq][w][s];
        } else {
          for (int w = 0; w < NW; ++w)
#pragma unroll
            for (int s = 0; s < NS; ++s) tot[s] += bsum[w][s][lane];
        }
        double* pp = a.parts + un.part_off + (long long)(cta - sm.q_cf[qq]) * (NSUM * width);
        if (blk || lane == 0) {
#pragma unroll
          for (int s = 0; s < NS; ++s) __stcg(pp + s * width + (blk ? lane : 0), tot[s]);
          __threadfence();
        }
        __syncwarp();
        int last = 0;
        if (lane == 0) last = atomicAdd(a.tickets + u, 1u) + 1 == unsigned(nslot);
        last = __shfl_sync(0xffffffffu, last, 0);
        if (!last) continue;
        __threadfence();
        if (blk) {
          // The block's partials (one per contributing CTA, up to the grid)
          // are added by the whole CTA below.
          if (lane == 0) sm.blk_last = qq;
          continue;
        }
        double acc[NSUM] = {0.0, 0.0, 0.0};
        if (!blk) {
          for (int sidx = lane; sidx < nslot; sidx += 32) {
            const double* src = a.parts + un.part_off + (long long)sidx * NSUM;
#pragma unroll
            for (int s = 0; s < NS; ++s) acc[s] += __ldcg(src + s);
          }
#pragma unroll
          for (int s = 0; s < NS; ++s) acc[s] = warp_total(acc[s]);
        }
        finish_unit<PH>(x, u, un, blk, acc);
      }
      __syncthreads();
      if (sm.blk_last >= 0) {
        // Block unit completed by this CTA: warp w adds the partials of
        // slots w, w + NW, ... (lane = column), then warp 0 adds the warps'
        // sums in warp order.
        const int qq = sm.blk_last;
        const int u = lu[sm.q_list[qq]];
        const Unit& un = a.units[u];
        const int nslot = sm.q_ns[qq];
        double acc[NSUM] = {0.0, 0.0, 0.0};
        for (int sidx = warp; sidx < nslot; sidx += NW) {
          const double* src = a.parts + un.part_off + (long long)sidx * NSUM * BW;
#pragma unroll
          for (int s = 0; s < NS; ++s) acc[s] += __ldcg(src + s * BW + lane);
        }
#pragma unroll
        for (int s = 0; s < NS; ++s) bsum[warp][s][lane] = acc[s];
        __syncthreads();
        if (warp == 0) {
          double tot[NSUM] = {0.0, 0.0, 0.0};
          for (int w = 0; w < NW; ++w)
#pragma unroll
            for (int s = 0; s < NS; ++s) tot[s] += bsum[w][s][lane];
          finish_unit<PH>(x, u, un, true, tot);
        }
      }
    }
    __syncthreads();
    i0 = sm.next_i;
  }
}

// ---------------------------------------------------------------------------
// The kernel.
// ---------------------------------------------------------------------------
template <typename T, typename CI, int R>
__global__ void __launch_bounds__(NT, 2) lockstep_kernel(const __grid_constant__ Args<T, CI> a) {
  __shared__ Smem sm;
  int* lu = reinterpret_cast<int*>(bat_dyn);
  int* lw = lu + a.nunits;
  unsigned long long epoch = 0;
  Ctx<T, CI> x{a, -1, l2_policy_keep(), l2_policy_stream()};
  if (a.prof && blockIdx.x == 0 && threadIdx.x == 0) {
    a.prof[0] = 0;
    a.prof[1] = gtimer();
  }
  // Units without rows are solved by definition.
  if (blockIdx.x == 0)
    for (int u = int(threadIdx.x); u < a.nunits; u += NT) {
      const Unit& un = a.units[u];
      if (un.n > 0) continue;
      Slot* sl = a.slots + un.slot0;
      sl->rr0 = sl->rr = sl->rr_true = 0.0;
      sl->its = sl->refs = 0;
      sl->status = SPMV_SUCCESS;
      sl->active = 0;
      sl->converged = 1;
      sl->refine_at = -1;
      a.ust[u].active = 0;
      a.ust[u].refine_at = -1;
    }
  auto all_units = [&](int u, int& w) {
    const Unit& un = a.units[u];
    if (un.n <= 0) return false;
    w = unit_tiles(un, a.tile_slices) * tile_weight(a.w, PH_INIT, un.kind, false);
    return true;
  };
  auto active_units_a = [&](int u, int& w) {
    if (__ldcg(&a.ust[u].active) == 0) return false;
    const Unit& un = a.units[u];
    w = unit_tiles(un, a.tile_slices) * tile_weight(a.w, PH_A, un.kind, false);
    return true;
  };
  auto active_units_b = [&](int u, int& w) {
    if (__ldcg(&a.ust[u].active) == 0) return false;
    const Unit& un = a.units[u];
    w = unit_tiles(un, a.tile_slices) * tile_weight(a.w, PH_B, un.kind, false);
    return true;
  };
  int cnt = build_list(a.nunits, lu, lw, sm, all_units);
  run_phase<PH_INIT, T, CI, R>(x, cnt, sm.tot >> 20, lu, lw, sm);
  if (!gbar(a, epoch, sm, 1)) return;
  for (int k = 0; k <= a.kmax; ++k) {
    x.k = k;
    cnt = build_list(a.nunits, lu, lw, sm, active_units_a);
    if (cnt == 0) break;
    run_phase<PH_A, T, CI, R>(x, cnt, sm.tot >> 20, lu, lw, sm);
    if (!gbar(a, epoch, sm, 2)) return;
    // The same units (A's decisions only remove broken-down ones, which B
    // skips anyway) with B's weights.
    cnt = build_list(a.nunits, lu, lw, sm, active_units_b);
    run_phase<PH_B, T, CI, R>(x, cnt, sm.tot >> 20, lu, lw, sm);
    if (!gbar(a, epoch, sm, 3)) return;
    if (threadIdx.x == 0) sm.nref = 0;
    __syncthreads();
    cnt = build_list(a.nunits, lu, lw, sm, [&](int u, int& w) {
      if (__ldcg(&a.ust[u].active) == 0) return false;
      const Unit& un = a.units[u];
      const bool ref = __ldcg(&a.ust[u].refine_at) == k;
      w = unit_tiles(un, a.tile_slices) * tile_weight(a.w, PH_C, un.kind, ref);
      return true;
    });
    // Any unit refining at k?  (the C list holds every active unit)
    int nref_local = 0;
    for (int u = int(threadIdx.x); u < a.nunits; u += NT)
      nref_local += __ldcg(&a.ust[u].refine_at) == k;
    if (nref_local) atomicAdd(&sm.nref, nref_local);
    const long long Wc = sm.tot >> 20;
    __syncthreads();
    const int nref = sm.nref;
    run_phase<PH_C, T, CI, R>(x, cnt, Wc, lu, lw, sm);
    if (!gbar(a, epoch, sm, 4)) return;
    if (nref > 0) {
      cnt = build_list(a.nunits, lu, lw, sm, [&](int u, int& w) {
        if (__ldcg(&a.ust[u].refine_at) != k) return false;
        const Unit& un = a.units[u];
        w = unit_tiles(un, a.tile_slices) * tile_weight(a.w, PH_D, un.kind, false);
        return true;
      });
      run_phase<PH_D, T, CI, R>(x, cnt, sm.tot >> 20, lu, lw, sm);
      if (!gbar(a, epoch, sm, 5)) return;
    }
  }
  cnt = build_list(a.nunits, lu, lw, sm, all_units);
  run_phase<PH_FINAL, T, CI, R>(x, cnt, sm.tot >> 20, lu, lw, sm);
}

// Shared-memory bytes of a launch beyond the static part: the unit list and
// the window region (the window, or the block unit's per-warp sums).
template <typename T, typename CI>
inline size_t dyn_smem(const Args<T, CI>& a) {
  const size_t list = (size_t(2) * sizeof(int) * size_t(a.nunits) + 15) & ~size_t(15);
  const size_t win = std::max(sizeof(T) * size_t(a.win_cap), sizeof(double) * NW * NSUM * BW);
  return list + win;
}

template <typename T, typename CI, int R>
bool launch_one(const Args<T, CI>& a, int cps, int num_sms, cudaStream_t s, bool dry) {
  const void* fn = reinterpret_cast<const void*>(lockstep_kernel<T, CI, R>);
  const size_t smem = dyn_smem(a);
  if (smem > 48 * 1024)
    SPMVB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
  int nb = 0;
  SPMVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, fn, NT, smem));
  if (nb < cps) return false;
  if (dry) return true;
  void* args[] = {const_cast<Args<T, CI>*>(&a)};
  const cudaError_t e =
      cudaLaunchCooperativeKernel(fn, dim3(cps * num_sms), dim3(NT), args, smem, s);
  if (e == cudaErrorCooperativeLaunchTooLarge) {
    (void)cudaGetLastError();
    return false;
  }
  SPMVB_CUDA(e);
  return true;
}

template <typename T, typename CI>
bool launch_ci(const Args<T, CI>& a, const LaunchCfg& c, int num_sms, cudaStream_t s, bool dry) {
  switch (c.rhs_rows) {
    case 2: return launch_one<T, CI, 2>(a, c.cps, num_sms, s, dry);
    default: return launch_one<T, CI, 1>(a, c.cps, num_sms, s, dry);
  }
}

}  // namespace bat
}  // namespace spmvb
