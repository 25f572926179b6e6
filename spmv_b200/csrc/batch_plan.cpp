// Host planning of a batch of SPD systems (no counterpart in the reference).
//
// Each system is renumbered once, at creation, so that its product streams
// well on the GPU:
//  1. reverse Cuthill-McKee (Cuthill & McKee 1969; George & Liu 1981):
//     breadth-first from a pseudo-peripheral vertex, neighbours visited by
//     increasing degree, the order reversed.  For the k-NN graphs of scattered
//     points this turns columns spread over the whole system (bandwidth ~ n)
//     into a band of a few thousand, so the gathers of a warp land on nearby
//     lines and every column fits a 16-bit offset from its row;
//  2. within windows of SIGMA consecutive rows, rows sorted by length
//     (descending, stable), so the 32 rows of a SELL slice have nearly equal
//     lengths and the slice's padding stays small (the SELL-C-sigma layout of
//     Kreutzer et al. 2014);
//  3. the SELL-32 layout: per slice of 32 rows, as many columns as its longest
//     row, entry k of row 32 s + l at soff[s] + 32 k + l.  Padding entries
//     carry value 0 and the row's own column.
// A permutation P A P^T of an SPD matrix is SPD with the same spectrum; the
// solver works on the renumbered system and maps b in and x out.
#include <algorithm>
#include <atomic>
#include <numeric>
#include <thread>

#include "batch.h"

namespace spmvb {
namespace bat {

std::vector<int32_t> rcm_order(int32_t n, const int32_t* rp, const int32_t* ci) {
  std::vector<int32_t> order;
  order.reserve(n);
  if (n == 0) return order;
  std::vector<int32_t> deg(n);
  for (int32_t i = 0; i < n; ++i) deg[i] = rp[i + 1] - rp[i];
  std::vector<int32_t> by_deg(n);
  std::iota(by_deg.begin(), by_deg.end(), 0);
  std::stable_sort(by_deg.begin(), by_deg.end(),
                   [&](int32_t a, int32_t b) { return deg[a] < deg[b]; });
  std::vector<uint8_t> placed(n, 0);
  std::vector<int32_t> stamp(n, -1);  // BFS visit marks for the peripheral search
  std::vector<int32_t> queue(n);
  int32_t bfs_id = 0;
  // Breadth-first levels from `s` over unplaced vertices; returns the depth
  // and leaves the last level in [lo, hi) of `queue`.
  auto levels = [&](int32_t s, int32_t& lo, int32_t& hi) {
    const int32_t id = bfs_id++;
    int32_t head = 0, tail = 0, depth = 0;
    queue[tail++] = s;
    stamp[s] = id;
    lo = 0;
    hi = 1;
    while (head < tail) {
      const int32_t level_end = tail;
      lo = head;
      hi = level_end;
      for (; head < level_end; ++head) {
        const int32_t v = queue[head];
        for (int32_t j = rp[v]; j < rp[v + 1]; ++j) {
          const int32_t w = ci[j];
          if (w < 0 || w >= n || placed[w] || stamp[w] == id) continue;
          stamp[w] = id;
          queue[tail++] = w;
        }
      }
      if (tail > level_end) ++depth;
    }
    return depth;
  };
  std::vector<int32_t> nb;
  for (int32_t seed : by_deg) {
    if (placed[seed]) continue;
    // Pseudo-peripheral start: move to a least-degree vertex of the last
    // level while the eccentricity grows (a few rounds).
    int32_t start = seed, lo = 0, hi = 0;
    int32_t ecc = levels(start, lo, hi);
    for (int round = 0; round < 4; ++round) {
      int32_t cand = queue[lo];
      for (int32_t i = lo; i < hi; ++i)
        if (deg[queue[i]] < deg[cand]) cand = queue[i];
      int32_t lo2 = 0, hi2 = 0;
      const int32_t e2 = levels(cand, lo2, hi2);
      if (e2 <= ecc) break;
      start = cand;
      ecc = e2;
      lo = lo2;
      hi = hi2;
    }
    // Cuthill-McKee from start.
    size_t head = order.size();
    order.push_back(start);
    placed[start] = 1;
    while (head < order.size()) {
      const int32_t v = order[head++];
      nb.clear();
      for (int32_t j = rp[v]; j < rp[v + 1]; ++j) {
        const int32_t w = ci[j];
        if (w < 0 || w >= n || placed[w]) continue;
        placed[w] = 1;
        nb.push_back(w);
      }
      std::sort(nb.begin(), nb.end(), [&](int32_t a, int32_t b) {
        return deg[a] != deg[b] ? deg[a] < deg[b] : a < b;
      });
      order.insert(order.end(), nb.begin(), nb.end());
    }
  }
  std::reverse(order.begin(), order.end());
  return order;
}

namespace {

struct SysLayout {
  std::vector<int32_t> perm;    // new -> old
  std::vector<int64_t> sw;      // slice widths
  int64_t entries = 0;
  bool fits16 = true;
  int max_width = 0;
};

void order_system(int32_t n, const int32_t* rp, const int32_t* ci, SysLayout& L) {
  std::vector<int32_t> ord = rcm_order(n, rp, ci);
  for (int32_t w0 = 0; w0 < n; w0 += SIGMA) {
    const int32_t w1 = std::min(n, w0 + SIGMA);
    std::stable_sort(ord.begin() + w0, ord.begin() + w1, [&](int32_t a, int32_t b) {
      return (rp[a + 1] - rp[a]) > (rp[b + 1] - rp[b]);
    });
  }
  L.perm = std::move(ord);
  const int32_t ns = (n + 31) / 32;
  L.sw.assign(ns, 0);
  std::vector<int32_t> inv(n);
  for (int32_t i = 0; i < n; ++i) inv[L.perm[i]] = i;
  for (int32_t s = 0; s < ns; ++s) {
    int32_t w = 0;
    for (int32_t l = 0; l < 32; ++l) {
      const int32_t row = 32 * s + l;
      if (row >= n) break;
      const int32_t old = L.perm[row];
      w = std::max(w, rp[old + 1] - rp[old]);
      for (int32_t j = rp[old]; j < rp[old + 1]; ++j) {
        const int64_t off = int64_t(inv[ci[j]]) - row;
        if (off < -32767 || off > 32767) L.fits16 = false;
      }
    }
    L.sw[s] = w;
    L.entries += 32 * int64_t(w);
    L.max_width = std::max(L.max_width, w);
  }
}

}  // namespace

void plan_batch(int nsys, const int32_t* n, const int32_t* const* rowptr,
                const int32_t* const* colind, const double* const* values, Plan& P) {
  P.nsys = nsys;
  P.n.assign(n, n + nsys);
  P.nnz.resize(nsys);
  std::vector<SysLayout> lay(nsys);
  // Systems are independent: order them on all host threads.
  std::atomic<int> next{0};
  const int nth = std::max(1, std::min<int>(nsys, int(std::thread::hardware_concurrency())));
  std::vector<std::thread> pool;
  for (int t = 0; t < nth; ++t)
    pool.emplace_back([&] {
      for (int s = next++; s < nsys; s = next++)
        order_system(n[s], rowptr[s], colind[s], lay[s]);
    });
  for (auto& th : pool) th.join();
  P.row0.resize(nsys);
  P.slice0.resize(nsys);
  P.sys_perm.resize(nsys);
  int64_t rows = 0, slices = 0, entries = 0;
  for (int s = 0; s < nsys; ++s) {
    P.nnz[s] = rowptr[s][n[s]];
    P.nnz_total += P.nnz[s];
    P.row0[s] = rows;
    P.slice0[s] = slices;
    rows += 32 * int64_t(lay[s].sw.size());
    slices += int64_t(lay[s].sw.size());
    entries += lay[s].entries;
    P.fits16 = P.fits16 && lay[s].fits16;
    P.max_width = std::max(P.max_width, lay[s].max_width);
  }
  P.rows_pad = rows;
  P.nslices = slices;
  P.entries = entries;
  P.soff.assign(slices + 1, 0);
  {
    int64_t e = 0, k = 0;
    for (int s = 0; s < nsys; ++s)
      for (int64_t w : lay[s].sw) {
        P.soff[k++] = e;
        e += 32 * w;
      }
    P.soff[k] = e;
  }
  P.vals32.assign(entries, 0.0f);
  P.vals64.assign(entries, 0.0);
  if (P.fits16)
    P.off16.assign(entries, 0);
  else
    P.col32.assign(entries, 0);
  P.perm.assign(rows, -1);
  P.sbound.assign(2 * slices, 0);
  // Fill each system's slices (threads over systems again).
  next = 0;
  pool.clear();
  for (int t = 0; t < nth; ++t)
    pool.emplace_back([&] {
      std::vector<int32_t> inv;
      for (int s = next++; s < nsys; s = next++) {
        const SysLayout& L = lay[s];
        const int32_t m = n[s];
        const int32_t* rp = rowptr[s];
        const int32_t* ci = colind[s];
        const double* va = values[s];
        inv.assign(m, 0);
        for (int32_t i = 0; i < m; ++i) inv[L.perm[i]] = i;
        for (int32_t i = 0; i < m; ++i) P.perm[P.row0[s] + i] = L.perm[i];
        for (size_t sl = 0; sl < L.sw.size(); ++sl) {
          const int64_t base = P.soff[P.slice0[s] + int64_t(sl)];
          const int64_t w = L.sw[sl];
          int32_t cmin = int32_t(32 * sl), cmax = int32_t(32 * sl);
          for (int32_t l = 0; l < 32; ++l) {
            const int32_t row = int32_t(32 * sl) + l;
            int32_t len = 0, beg = 0;
            if (row < m) {
              const int32_t old = L.perm[row];
              beg = rp[old];
              len = rp[old + 1] - beg;
            }
            for (int64_t k = 0; k < w; ++k) {
              const int64_t e = base + 32 * k + l;
              int32_t col = row;  // padding: the row itself, value 0
              if (k < len) {
                col = inv[ci[beg + k]];
                P.vals64[e] = va[beg + k];
                P.vals32[e] = float(va[beg + k]);
              }
              if (P.fits16)
                P.off16[e] = int16_t(col - row);
              else
                P.col32[e] = col;
              cmin = std::min(cmin, col);
              cmax = std::max(cmax, col);
            }
          }
          P.sbound[2 * (P.slice0[s] + int64_t(sl))] = cmin;
          P.sbound[2 * (P.slice0[s] + int64_t(sl)) + 1] = cmax;
        }
      }
    });
  for (auto& th : pool) th.join();
  for (int s = 0; s < nsys; ++s) P.sys_perm[s] = std::move(lay[s].perm);
}

}  // namespace bat
}  // namespace spmvb
