// SELL-32 traversal with the matrix stream staged in shared memory by bulk
// asynchronous copies (cp.async.bulk, completion counted on mbarriers), in a
// warp-specialised pipeline.
//
// The rows of a matrix are cut into tiles of whole slices (a host-built
// table of StagedDesc; at most STAGED_MAX_SLICES slices and
// CFG::max_entries entries per tile).  A
// persistent CTA takes tiles blockIdx.x, blockIdx.x + gridDim.x, ...:
//
//   producer warp (the last warp, one lane): for each tile, waits until the
//     consumers have released the stage buffer and issues three bulk copies
//     that complete on the stage's "full" barrier: the tile's descriptor
//     (rank, slice count, slice offsets) as the stage header, its values and
//     its column indices (or 16-bit offsets), both contiguous in the SELL
//     arrays;
//   consumer warps (STAGED_CONSUMERS): wait for the stage, take their share
//     of its slices (dealt round robin over the CTA's sequence of slices; one
//     lane per row), read the entries from shared memory
//     (consecutive lanes, consecutive words), gather x from global memory
//     (L2), sum each row in storage order, call f, and release the stage.
//
// Consumers never wait on global loads for metadata, and the matrix bytes in
// flight per SM are set by the stage buffers rather than by registers.  Rows
// are summed in the same order as sell_for_rows, so results match that
// traversal bit for bit.
//
// Every wait is bounded (2 s of global time): a barrier that does not
// complete within the limit sets *err and ends that warp's loop; the
// producer then waits (bounded again) for the copies it issued, so no copy
// is left writing to the shared memory of a finished CTA.  Waiting warps
// are suspended between probes, so they take no issue slots from the
// warps that compute.
#pragma once

#include "spmv_kernel.cuh"

namespace spmvb {

constexpr int STAGED_HEADER_BYTES = 128;
constexpr int STAGED_MAX_SLICES = 16;

// Pipeline shape: NC consumer warps (+ one producer warp), STAGES tiles in
// flight per CTA, DATA bytes of values + indices per tile; MINB: CTAs per SM
// a persistent kernel of this shape is compiled to fit (register bound).
template <int NC_, int STAGES_, int DATA_, int MINB_ = 1>
struct StagedCfg {
  static constexpr int NC = NC_;
  static constexpr int STAGES = STAGES_;
  static constexpr int DATA = DATA_;
  static constexpr int MINB = MINB_;
  static constexpr int BS = 32 * (NC + 1);
  // Entries of one stage for `eb` bytes per entry (a multiple of 32).
  __host__ __device__ static constexpr int max_entries(int eb) { return (DATA / eb) / 32 * 32; }
  __host__ __device__ static constexpr int stage_bytes(int eb) {
    return STAGED_HEADER_BYTES + max_entries(eb) * eb;
  }
  // Dynamic shared memory of a launch.
  __host__ __device__ static constexpr int smem_bytes(int eb) { return STAGES * stage_bytes(eb); }
};

// The shape the solvers' products use: 12 consumer warps, 4 stages of 16 KB
// (3 CTAs per SM), measured best of the shapes tried on the 7-point stencil
// in FP64 and FP32.
using SolverStaged = StagedCfg<12, 4, 16384, 3>;

// Descriptor of one tile (host-built, 128 bytes, copied as the stage's
// header): slices [s0, s0 + nslices) of rank `rank`, whose entries start at
// entry e0 of the rank's SELL arrays and number n; off[j] = first entry of
// slice s0 + j relative to e0 (off[nslices] = n).
struct StagedDesc {
  int32_t rank, nslices, s0, e0;
  int32_t n, pad[3];
  int32_t off[24];
};
static_assert(sizeof(StagedDesc) == STAGED_HEADER_BYTES, "staged descriptor is one header");
static_assert(STAGED_MAX_SLICES + 1 <= 24, "staged descriptor too small");

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_addr(bar)) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}

// One probe of the barrier's phase: true once phase `parity` has completed.
// The instruction may suspend the thread until the phase completes, for at
// most `hint_ns` nanoseconds (0: the hardware's own limit).
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity,
                                              uint32_t hint_ns = 0) {
  uint32_t ok;
  if (hint_ns == 0) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
  } else {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
  }
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bound of every pipeline wait (a healthy pipeline waits microseconds).
constexpr uint64_t STAGED_WAIT_LIMIT_NS = 2000000000ull;

// Waits for phase `parity` of `bar`, suspended between probes (so a waiting
// warp takes no issue slots), giving up after STAGED_WAIT_LIMIT_NS of
// global time.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity, 1000000u)) return true;
    if (global_ns() - t0 > STAGED_WAIT_LIMIT_NS) return false;
  }
}

// Bulk copy global -> shared, completion counted on `bar`; the source gets
// an L2 evict-first policy (the matrix is read once per product).
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar, uint64_t policy) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
      " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
      : "memory");
}

// The consumer side of one landed stage (header + values + indices at
// `stage`): warp `warp` sums its share of the tile's slices (dealt round
// robin, continuing from q0 = slices dealt before this tile; q0 is
// advanced), one lane per row, entries in storage order, and calls
// f(P, row, sum) for each row that exists.
template <class CFG, typename T, typename CI, int U, class F, class G>
__device__ __forceinline__ void staged_tile_rows(const SpmvArgs& a,
                                                 const unsigned char* stage, int warp,
                                                 int lane, int& q0, F&& f, const G& gx) {
  constexpr int NC = CFG::NC;
  constexpr int MAXE = CFG::max_entries(int(sizeof(T) + sizeof(CI)));
  // Multi-chunk unmasked slices only where a stencil's rows are several
  // chunks long (U = 9 for 27 entries); the other widths keep their
  // measured code.
  constexpr bool UNMASKED_CHUNKS = U == 9;
  const StagedDesc* h = reinterpret_cast<const StagedDesc*>(stage);
  const T* sv = reinterpret_cast<const T*>(stage + STAGED_HEADER_BYTES);
  const CI* sc = reinterpret_cast<const CI*>(stage + STAGED_HEADER_BYTES + MAXE * int(sizeof(T)));
  const PartArg& P = a.part[h->rank];
  const int ns = h->nslices;
  const int j0 = ((warp - q0) % NC + NC) % NC;
  q0 += ns;
  for (int j = j0; j < ns; j += NC) {
    const int o = h->off[j];
    const int w = (h->off[j + 1] - o) >> 5;
    const int row = (h->s0 + j) * 32 + lane;
    const int g = P.row0 + row;
    T sum = T(0);
    if (!UNMASKED_CHUNKS && w == U) {
      // The slice's rows in one chunk: no slot masks.  A padding entry
      // gathers x[0] (in bounds in every layout; the value is not used).
      T v[U], xv[U];
      bool ok[U];
      int c[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int idx = o + u * 32 + lane;
        const int ci = int(sc[idx]);
        v[u] = sv[idx];
        ok[u] = sizeof(CI) == 2 ? ci != -32768 : ci >= 0;
        c[u] = ok[u] ? (sizeof(CI) == 2 ? g + ci : ci) : 0;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) xv[u] = gx(P, c[u]);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (ok[u]) sum += v[u] * xv[u];
      if (row < P.nrows) f(P, row, sum);
      continue;
    }
    if (UNMASKED_CHUNKS && w % U == 0) {
      // Whole chunks (27 entries at U = 9): the same, chunk by chunk, values
      // read from shared memory when summed (fewer registers held).
      for (int k0 = 0; k0 < w; k0 += U) {
        T xv[U];
        bool ok[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
          const int ci = int(sc[o + (k0 + u) * 32 + lane]);
          ok[u] = sizeof(CI) == 2 ? ci != -32768 : ci >= 0;
          xv[u] = gx(P, ok[u] ? (sizeof(CI) == 2 ? g + ci : ci) : 0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
          if (ok[u]) sum += sv[o + (k0 + u) * 32 + lane] * xv[u];
      }
      if (row < P.nrows) f(P, row, sum);
      continue;
    }
    for (int k0 = 0; k0 < w; k0 += U) {
      T v[U], xv[U];
      bool ok[U];
      int c[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const bool in = k0 + u < w;
        const int idx = o + (k0 + u) * 32 + lane;
        const int ci = in ? int(sc[idx]) : 0;
        v[u] = in ? sv[idx] : T(0);
        if (sizeof(CI) == 2) {
          ok[u] = in && ci != -32768;
          c[u] = g + ci;
        } else {
          ok[u] = in && ci >= 0;
          c[u] = ci;
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u) xv[u] = ok[u] ? gx(P, c[u]) : T(0);
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (ok[u]) sum += v[u] * xv[u];
    }
    if (row < P.nrows) f(P, row, sum);
  }
}

// Issues the bulk copies of one tile (descriptor d, whose rank, first
// entry and entry count the caller has loaded as rk, e0, n) into `stage`,
// completing on `full`.
template <class CFG, typename T, typename CI>
__device__ __forceinline__ void staged_issue(const SpmvArgs& a, const StagedDesc* d, int rk,
                                             int e0, uint32_t n, unsigned char* stage,
                                             uint64_t* full, uint64_t policy) {
  constexpr int EB = int(sizeof(T) + sizeof(CI));
  constexpr int MAXE = CFG::max_entries(EB);
  const PartArg& P = a.part[rk];
  mbar_arrive_expect_tx(full, STAGED_HEADER_BYTES + n * uint32_t(EB));
  bulk_g2s(stage, d, STAGED_HEADER_BYTES, full, policy);
  if (n > 0) {
    bulk_g2s(stage + STAGED_HEADER_BYTES, static_cast<const T*>(P.vals) + e0,
             n * uint32_t(sizeof(T)), full, policy);
    bulk_g2s(stage + STAGED_HEADER_BYTES + MAXE * int(sizeof(T)),
             reinterpret_cast<const CI*>(P.cols) + e0, n * uint32_t(sizeof(CI)), full, policy);
  }
}

// Traversal.  CI: int32_t (columns, -1 = padding) or int16_t (offsets from
// the global row g = row0 + row, -32768 = padding).  U: gathers in flight
// per lane; gx(P, c): the gathered vector (XGather: the PartArg's x).
// f(P, row, sum) is called by the lane owning each row.  All CFG::BS
// threads must call this (block-wide reductions may follow).
template <class CFG, typename T, typename CI, int U, class F, class G>
__device__ __forceinline__ void sell_staged_rows(const SpmvArgs& a,
                                                 const StagedDesc* __restrict__ tiles,
                                                 int ntiles, int* err, F&& f, const G& gx) {
  constexpr int STAGED_STAGES = CFG::STAGES;
  constexpr int STAGED_CONSUMERS = CFG::NC;
  constexpr int STAGE = CFG::stage_bytes(int(sizeof(T) + sizeof(CI)));
  extern __shared__ __align__(128) unsigned char staged_smem[];
  __shared__ __align__(8) uint64_t full[STAGED_STAGES], empty[STAGED_STAGES];

  const int tid = int(threadIdx.x);
  const int warp = tid >> 5, lane = tid & 31;
  const int count = int(blockIdx.x) < ntiles
                        ? (ntiles - int(blockIdx.x) + int(gridDim.x) - 1) / int(gridDim.x)
                        : 0;

  if (tid == 0) {
    for (int s = 0; s < STAGED_STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], STAGED_CONSUMERS);
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // A programmatic launch may start during the previous kernel (usually the
  // ghost gather of L2GMap::update): nothing global is read before it ends.
  pdl_wait();

  if (warp == STAGED_CONSUMERS) {
    // Producer.  The next tile's rank, e0 and n are loaded one tile ahead,
    // so no issue waits on a global load.
    if (lane == 0) {
      const uint64_t stream = l2_policy_stream();
      int issued = 0;
      bool failed = false;
      int4 nxt = make_int4(0, 0, 0, 0);  // rank, e0, n of tile i
      if (count > 0) {
        const StagedDesc* d = tiles + blockIdx.x;
        nxt = make_int4(__ldg(&d->rank), __ldg(&d->e0), __ldg(&d->n), 0);
      }
      for (int i = 0; i < count; ++i) {
        const int st = i % STAGED_STAGES;
        const int4 cur = nxt;
        if (i + 1 < count) {
          const StagedDesc* d = tiles + int(blockIdx.x) + (i + 1) * int(gridDim.x);
          nxt = make_int4(__ldg(&d->rank), __ldg(&d->e0), __ldg(&d->n), 0);
        }
        if (i >= STAGED_STAGES &&
            !mbar_wait_bounded(&empty[st], uint32_t(i / STAGED_STAGES - 1) & 1u)) {
          failed = true;
          break;
        }
        staged_issue<CFG, T, CI>(a, tiles + int(blockIdx.x) + i * int(gridDim.x), cur.x, cur.y,
                                 uint32_t(cur.z), staged_smem + st * STAGE, &full[st], stream);
        issued = i + 1;
      }
      if (failed) {
        if (err) atomicExch(err, 1);
        // Wait (bounded) for the last STAGES tiles issued to land.
        for (int i = issued - STAGED_STAGES < 0 ? 0 : issued - STAGED_STAGES; i < issued; ++i)
          mbar_wait_bounded(&full[i % STAGED_STAGES], uint32_t(i / STAGED_STAGES) & 1u);
      }
    }
    return;
  }

  // Consumers.  Slices are dealt round robin over the CTA's whole sequence
  // of tiles (q0 = slices in the tiles before this one), so a tile with
  // fewer slices than consumer warps leaves no warp idle for long.
  int q0 = 0;
  for (int i = 0; i < count; ++i) {
    const int st = i % STAGED_STAGES;
    if (!mbar_wait_bounded(&full[st], uint32_t(i / STAGED_STAGES) & 1u)) {
      if (err && lane == 0) atomicExch(err, 1);
      break;
    }
    staged_tile_rows<CFG, T, CI, U>(a, staged_smem + st * STAGE, warp, lane, q0, f, gx);
    __syncwarp();
    if (lane == 0) mbar_arrive(&empty[st]);
  }
}

// ---------------------------------------------------------------------------
// Multi-pass form, for a persistent solver kernel that traverses the same
// tiles once per iteration.  The CTA's tiles are tiles[0, count); the
// producer streams them pass after pass (tile sequence number q, tile
// q % count, stage q % STAGES) until the consumers raise `stop`, so the next
// pass's first tiles land while the consumers do other work between passes.
template <class CFG>
struct StagedLoop {
  uint64_t full[CFG::STAGES], empty[CFG::STAGES];
  volatile int stop;
};

// Thread 0; the caller synchronises the CTA before the pipeline starts.
template <class CFG>
__device__ __forceinline__ void staged_loop_init(StagedLoop<CFG>& L) {
  for (int s = 0; s < CFG::STAGES; ++s) {
    mbar_init(&L.full[s], 1);
    mbar_init(&L.empty[s], CFG::NC);
  }
  L.stop = 0;
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// Waits for phase `parity` of `bar` unless `stop` is raised first (looked at
// every 20 us at most).  Returns 0 (phase complete), 1 (stopped) or 2 (gave
// up after STAGED_WAIT_LIMIT_NS).
__device__ __forceinline__ int mbar_wait_or_stop(uint64_t* bar, uint32_t parity,
                                                 const volatile int* stop) {
  if (mbar_try_wait(bar, parity)) return 0;
  const uint64_t t0 = global_ns();
  for (;;) {
    if (mbar_try_wait(bar, parity, 20000u)) return 0;
    if (*stop) return 1;
    if (global_ns() - t0 > STAGED_WAIT_LIMIT_NS) return 2;
  }
}

// Producer: one lane.  On stop (or a wait that gave up, which also sets
// *err) it waits, bounded, for its copies still in flight and returns.
template <class CFG, typename T, typename CI>
__device__ __forceinline__ void staged_loop_produce(const SpmvArgs& a,
                                                    const StagedDesc* __restrict__ tiles,
                                                    int count, StagedLoop<CFG>& L,
                                                    unsigned char* smem, int* err) {
  constexpr int S = CFG::STAGES;
  constexpr int STAGE = CFG::stage_bytes(int(sizeof(T) + sizeof(CI)));
  if (count <= 0) return;
  const uint64_t stream = l2_policy_stream();
  uint64_t issued = 0;
  int4 nxt = make_int4(__ldg(&tiles[0].rank), __ldg(&tiles[0].e0), __ldg(&tiles[0].n), 0);
  int inext = 0;
  for (uint64_t q = 0;; ++q) {
    const int st = int(q % S);
    const int i = inext;
    const int4 cur = nxt;
    inext = i + 1 == count ? 0 : i + 1;
    {
      const StagedDesc* d = tiles + inext;
      nxt = make_int4(__ldg(&d->rank), __ldg(&d->e0), __ldg(&d->n), 0);
    }
    if (q >= uint64_t(S)) {
      const int w = mbar_wait_or_stop(&L.empty[st], uint32_t(q / S - 1) & 1u, &L.stop);
      if (w == 2 && err) atomicExch(err, 1);
      if (w != 0) break;
    }
    if (L.stop) break;
    staged_issue<CFG, T, CI>(a, tiles + i, cur.x, cur.y, uint32_t(cur.z), smem + st * STAGE,
                             &L.full[st], stream);
    issued = q + 1;
  }
  for (uint64_t q = issued > uint64_t(S) ? issued - S : 0; q < issued; ++q)
    mbar_wait_bounded(&L.full[q % S], uint32_t(q / S) & 1u);
}

// Consumers (warps 0 .. NC-1): one pass over the CTA's tiles, whose first
// tile has sequence number q_base.  A stage that does not land within the
// bound sets *err and ends this warp's pass.
template <class CFG, typename T, typename CI, int U, class F, class G>
__device__ __forceinline__ void staged_loop_consume(const SpmvArgs& a, int count, uint64_t q_base,
                                                    StagedLoop<CFG>& L,
                                                    const unsigned char* smem, int* err, F&& f,
                                                    const G& gx) {
  constexpr int S = CFG::STAGES;
  constexpr int STAGE = CFG::stage_bytes(int(sizeof(T) + sizeof(CI)));
  const int warp = int(threadIdx.x) >> 5, lane = int(threadIdx.x) & 31;
  int q0 = 0;
  for (int i = 0; i < count; ++i) {
    const uint64_t q = q_base + uint64_t(i);
    const int st = int(q % S);
    if (!mbar_wait_bounded(&L.full[st], uint32_t(q / S) & 1u)) {
      if (err && lane == 0) atomicExch(err, 1);
      return;
    }
    staged_tile_rows<CFG, T, CI, U>(a, smem + st * STAGE, warp, lane, q0, f, gx);
    __syncwarp();
    if (lane == 0) mbar_arrive(&L.empty[st]);
  }
}

}  // namespace spmvb
