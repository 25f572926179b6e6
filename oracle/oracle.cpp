// ORACLE - TEST INFRASTRUCTURE ONLY.
//
// A CPU restatement of libspmv's hot path (chrisrichardson/spmv), used to
// check the CUDA implementation.  Only the tests, the smoke check and the
// CPU-baseline leg of bench.py load this library; the product never does.
//
// Parity is UNPINNED: the reference cannot be built here (it needs Eigen,
// MKL or BLAS, and MPI, none of which are installed) and it ships no tests,
// fixtures or golden outputs.  Each function below restates the reference's
// code at the cited file:line; results are cross-checked against
// scipy.sparse in the tests, which is independent evidence but not a pin.
//
// MPI is replaced by a virtual communicator: all P ranks' data is in this
// process, and each collective is restated by its MPI semantics (who sends
// which block to whom), not by a shortcut, so the arrays it produces are the
// ones each MPI rank would hold.
//
// Floating point: the reference is built with -O3 and no -march (x86-64
// baseline, no FMA); this file is built with -ffp-contract=off so products
// and sums round separately, as they do there.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <fstream>
#include <iterator>
#include <map>
#include <memory>
#include <set>
#include <stdexcept>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

thread_local std::string g_err;

template <class F>
int guard(F&& f) {
  try {
    f();
    return 0;
  } catch (const std::exception& e) {
    g_err = e.what();
    return 1;
  }
}

// ---------------------------------------------------------------------------
// L2GMap restated (L2GMap.cpp:15-122) over a virtual communicator.
// ---------------------------------------------------------------------------
struct Rank {
  int64_t local_size = 0;
  std::vector<int64_t> ghosts;
  std::map<int64_t, int32_t> global_to_local;   // L2GMap.h:76
  std::vector<int> neighbours;
  std::vector<int32_t> ghost_local, send_count, recv_count, send_offset,
      recv_offset, indexbuf;
};

struct Map {
  int P = 0;
  std::vector<int64_t> ranges;
  std::vector<Rank> r;
};

// Position of rank `who` in rank `at`'s neighbour list (the dist-graph
// communicator of L2GMap.cpp:81-84 has sources == destinations ==
// neighbours, in that order).
int position(const Map& m, int at, int who) {
  const auto& nb = m.r[at].neighbours;
  auto it = std::find(nb.begin(), nb.end(), who);
  if (it == nb.end()) throw std::runtime_error("oracle: asymmetric neighbours");
  return int(it - nb.begin());
}

void build_map(Map& m, int P, const int64_t* local_size,
               const int64_t* const* ghosts, const int64_t* nghosts) {
  m.P = P;
  m.r.assign(P, Rank{});
  // MPI_Allgather of local_size, then prefix sum (L2GMap.cpp:23-28).
  m.ranges.assign(P + 1, 0);
  for (int q = 0; q < P; ++q) m.ranges[q + 1] = local_size[q];
  for (int i = 0; i < P; ++i) m.ranges[i + 1] += m.ranges[i];

  std::vector<std::vector<int32_t>> ghost_count(P, std::vector<int32_t>(P, 0));
  for (int rank = 0; rank < P; ++rank) {
    Rank& R = m.r[rank];
    R.local_size = local_size[rank];
    R.ghosts.assign(ghosts[rank], ghosts[rank] + nghosts[rank]);
    const int64_t r0 = m.ranges[rank], r1 = m.ranges[rank + 1];
    if (!std::is_sorted(R.ghosts.begin(), R.ghosts.end()))   // :34-35
      throw std::runtime_error("Ghosts must be sorted");
    for (size_t i = 0; i < R.ghosts.size(); ++i) {            // :40-54
      const int64_t idx = R.ghosts[i];
      if (idx >= r0 and idx < r1)
        throw std::runtime_error("Ghost index in local range");
      R.global_to_local.insert({idx, int32_t(R.local_size + int64_t(i))});
      auto it = std::upper_bound(m.ranges.begin(), m.ranges.end(), idx);
      const int p = int(it - m.ranges.begin()) - 1;
      ++ghost_count[rank][p];
      R.ghost_local.push_back(int32_t(R.ghosts[i] - m.ranges[p]));
    }
  }
  // MPI_Alltoall: remote_count[rank][i] = ghost_count[i][rank] (:59-61);
  // neighbour lists and send counts (:63-78).
  for (int rank = 0; rank < P; ++rank) {
    Rank& R = m.r[rank];
    for (int i = 0; i < P; ++i) {
      const int32_t c = ghost_count[rank][i];
      const int32_t rc = ghost_count[i][rank];
      if (c > 0) {
        R.neighbours.push_back(i);
        R.send_count.push_back(c);
      } else if (rc > 0) {
        R.neighbours.push_back(i);
        R.send_count.push_back(0);
      }
    }
    R.recv_count.assign(R.neighbours.size(), 0);            // :86
    if (R.neighbours.empty()) {                              // :87-92
      R.send_count = {0};
      R.recv_count = {0};
    }
  }
  // MPI_Neighbor_alltoall of send_count (:97-98): block k of rank `rank`
  // comes from neighbour q = neighbours[k], which sends its block for
  // `rank` (at rank's position in q's list).
  for (int rank = 0; rank < P; ++rank) {
    Rank& R = m.r[rank];
    for (size_t k = 0; k < R.neighbours.size(); ++k) {
      const int q = R.neighbours[k];
      R.recv_count[k] = m.r[q].send_count[position(m, q, rank)];
    }
  }
  for (int rank = 0; rank < P; ++rank) {                     // :100-109
    Rank& R = m.r[rank];
    R.send_offset = {0};
    for (int c : R.send_count) R.send_offset.push_back(R.send_offset.back() + c);
    R.recv_offset = {0};
    for (int c : R.recv_count) R.recv_offset.push_back(R.recv_offset.back() + c);
    R.indexbuf.assign(R.recv_offset.back(), 0);
  }
  // MPI_Neighbor_alltoallv of ghost_local (:112-115).
  for (int rank = 0; rank < P; ++rank) {
    Rank& R = m.r[rank];
    for (size_t k = 0; k < R.neighbours.size(); ++k) {
      const int q = R.neighbours[k];
      const int pos = position(m, q, rank);
      const Rank& Q = m.r[q];
      for (int32_t j = 0; j < R.recv_count[k]; ++j)
        R.indexbuf[R.recv_offset[k] + j] = Q.ghost_local[Q.send_offset[pos] + j];
    }
  }
  for (int rank = 0; rank < P; ++rank)                       // :120-121
    for (int32_t& s : m.r[rank].send_offset) s += int32_t(m.r[rank].local_size);
}

// L2GMap::update<T> (L2GMap.cpp:126-150).  Every rank packs databuf from its
// own vector first; then the alltoallv delivers rank q's segment for `rank`
// (recv_count/offset on the sender side, send_count/offset on the receiver
// side: the meanings are reversed, L2GMap.cpp:141-147).
template <typename T>
void update(const Map& m, T* const* vec) {
  std::vector<std::vector<T>> databuf(m.P);
  for (int rank = 0; rank < m.P; ++rank) {
    const Rank& R = m.r[rank];
    databuf[rank].resize(R.indexbuf.size());
    for (size_t i = 0; i < R.indexbuf.size(); ++i)
      databuf[rank][i] = vec[rank][R.indexbuf[i]];
  }
  for (int rank = 0; rank < m.P; ++rank) {
    const Rank& R = m.r[rank];
    for (size_t k = 0; k < R.neighbours.size(); ++k) {
      const int q = R.neighbours[k];
      const int pos = position(m, q, rank);
      const Rank& Q = m.r[q];
      for (int32_t j = 0; j < R.send_count[k]; ++j)
        vec[rank][R.send_offset[k] + j] = databuf[q][Q.recv_offset[pos] + j];
    }
  }
}

// L2GMap::reverse_update<T> (L2GMap.cpp:152-170).
template <typename T>
void reverse_update(const Map& m, T* const* vec) {
  std::vector<std::vector<T>> databuf(m.P);
  for (int rank = 0; rank < m.P; ++rank) {
    const Rank& R = m.r[rank];
    databuf[rank].assign(R.indexbuf.size(), T(0));
    for (size_t k = 0; k < R.neighbours.size(); ++k) {
      const int q = R.neighbours[k];
      const int pos = position(m, q, rank);
      const Rank& Q = m.r[q];
      for (int32_t j = 0; j < R.recv_count[k]; ++j)
        databuf[rank][R.recv_offset[k] + j] = vec[q][Q.send_offset[pos] + j];
    }
  }
  for (int rank = 0; rank < m.P; ++rank) {
    const Rank& R = m.r[rank];
    for (size_t i = 0; i < R.indexbuf.size(); ++i)
      vec[rank][R.indexbuf[i]] += databuf[rank][i];
  }
}

// Matrix::operator* through Eigen's row-major sparse x dense product
// (Matrix.cpp:199-204): per row, tmp = 0; tmp += v * x[c] in storage order.
template <typename T>
void csr_mult(int32_t m, const int32_t* rp, const int32_t* ci, const T* v,
              const T* x, T* y, int nthreads) {
  (void)nthreads;
#pragma omp parallel for schedule(static) num_threads(nthreads) if (nthreads > 1)
  for (int32_t i = 0; i < m; ++i) {
    T tmp = T(0);
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) tmp += v[j] * x[ci[j]];
    y[i] = tmp;
  }
}

// Matrix::transpmult (Matrix.cpp:206-211): Eigen's transposed product
// scatters row by row: y = 0; y[c] += v * x[i].
template <typename T>
void csr_transpmult(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                    const T* v, const T* x, T* y) {
  std::fill(y, y + n, T(0));
  for (int32_t i = 0; i < m; ++i)
    for (int32_t j = rp[i]; j < rp[i + 1]; ++j) y[ci[j]] += v[j] * x[i];
}

double dot(const double* a, const double* b, int64_t n, int nthreads) {
  if (nthreads <= 1) {
    double s = 0.0;
    for (int64_t i = 0; i < n; ++i) s += a[i] * b[i];
    return s;
  }
  // Parallel form (CPU baseline only): fixed chunks summed in chunk order.
  const int64_t chunks = 256;
  std::vector<double> part(chunks, 0.0);
#pragma omp parallel for schedule(static) num_threads(nthreads)
  for (int64_t c = 0; c < chunks; ++c) {
    const int64_t lo = n * c / chunks, hi = n * (c + 1) / chunks;
    double s = 0.0;
    for (int64_t i = lo; i < hi; ++i) s += a[i] * b[i];
    part[c] = s;
  }
  double s = 0.0;
  for (double p : part) s += p;
  return s;
}

struct Mat {
  std::vector<int32_t> nrows, ncols;
  std::vector<const int32_t*> rp, ci;
  std::vector<const double*> v;
};

}  // namespace

extern "C" {

typedef struct OracleMap* oracle_map;
struct OracleMap {
  Map m;
};

const char* oracle_last_error(void) { return g_err.c_str(); }

// owner_ranges (CreateA.cpp:12-29, read_petsc.cpp:13-30): the first N % size
// ranks get one extra row.
void oracle_owner_ranges(int64_t size, int64_t N, int64_t* ranges) {
  const int64_t n = N / size;
  const int64_t r = N % size;
  for (int64_t rank = 0; rank < size + 1; ++rank)
    ranges[rank] = rank < r ? rank * (n + 1) : rank * n + r;
}

int oracle_map_create(int P, const int64_t* local_size,
                      const int64_t* const* ghosts, const int64_t* nghosts,
                      oracle_map* out) {
  return guard([&] {
    auto h = std::make_unique<OracleMap>();
    build_map(h->m, P, local_size, ghosts, nghosts);
    *out = h.release();
  });
}

void oracle_map_free(oracle_map h) { delete h; }

// field: 0 neighbours, 1 send_count, 2 recv_count, 3 send_offset,
// 4 recv_offset, 5 indexbuf (same numbering as spmv_pattern_field).
int oracle_map_field(oracle_map h, int rank, int field, const int32_t** data,
                     int32_t* n) {
  return guard([&] {
    const Rank& R = h->m.r.at(rank);
    static thread_local std::vector<int32_t> nb;
    switch (field) {
      case 0:
        nb.assign(R.neighbours.begin(), R.neighbours.end());
        *data = nb.data();
        *n = int32_t(nb.size());
        return;
      case 1: *data = R.send_count.data(); *n = int32_t(R.send_count.size()); return;
      case 2: *data = R.recv_count.data(); *n = int32_t(R.recv_count.size()); return;
      case 3: *data = R.send_offset.data(); *n = int32_t(R.send_offset.size()); return;
      case 4: *data = R.recv_offset.data(); *n = int32_t(R.recv_offset.size()); return;
      case 5: *data = R.indexbuf.data(); *n = int32_t(R.indexbuf.size()); return;
    }
    throw std::runtime_error("oracle: bad field");
  });
}

// L2GMap::global_to_local (L2GMap.cpp:172-185); -1 where the reference would
// dereference map::end().
int32_t oracle_map_global_to_local(oracle_map h, int rank, int64_t i) {
  const Map& m = h->m;
  const int64_t r0 = m.ranges[rank], r1 = m.ranges[rank + 1];
  if (i >= r0 and i < r1) return int32_t(i - r0);
  auto it = m.r[rank].global_to_local.find(i);
  return it == m.r[rank].global_to_local.end() ? -1 : it->second;
}

void oracle_update_f64(oracle_map h, double* const* vec) { update<double>(h->m, vec); }
void oracle_update_f32(oracle_map h, float* const* vec) { update<float>(h->m, vec); }
void oracle_reverse_update_f64(oracle_map h, double* const* vec) {
  reverse_update<double>(h->m, vec);
}
void oracle_reverse_update_f32(oracle_map h, float* const* vec) {
  reverse_update<float>(h->m, vec);
}

void oracle_csr_mult_f64(int32_t m, const int32_t* rp, const int32_t* ci,
                         const double* v, const double* x, double* y,
                         int nthreads) {
  csr_mult<double>(m, rp, ci, v, x, y, nthreads);
}
void oracle_csr_mult_f32(int32_t m, const int32_t* rp, const int32_t* ci,
                         const float* v, const float* x, float* y) {
  csr_mult<float>(m, rp, ci, v, x, y, 1);
}
void oracle_csr_transpmult_f64(int32_t m, int32_t n, const int32_t* rp,
                               const int32_t* ci, const double* v,
                               const double* x, double* y) {
  csr_transpmult<double>(m, n, rp, ci, v, x, y);
}
void oracle_csr_transpmult_f32(int32_t m, int32_t n, const int32_t* rp,
                               const int32_t* ci, const float* v,
                               const float* x, float* y) {
  csr_transpmult<float>(m, n, rp, ci, v, x, y);
}
// Complex instantiations (Matrix.cpp:441-444; the generic Eigen products of
// Matrix.cpp:199-211, std::complex arithmetic).  Arrays are interleaved
// (re, im) pairs.
void oracle_csr_mult_c128(int32_t m, const int32_t* rp, const int32_t* ci, const void* v,
                          const void* x, void* y) {
  using C = std::complex<double>;
  csr_mult<C>(m, rp, ci, static_cast<const C*>(v), static_cast<const C*>(x),
              static_cast<C*>(y), 1);
}
void oracle_csr_mult_c64(int32_t m, const int32_t* rp, const int32_t* ci, const void* v,
                         const void* x, void* y) {
  using C = std::complex<float>;
  csr_mult<C>(m, rp, ci, static_cast<const C*>(v), static_cast<const C*>(x),
              static_cast<C*>(y), 1);
}
void oracle_csr_transpmult_c128(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                                const void* v, const void* x, void* y) {
  using C = std::complex<double>;
  csr_transpmult<C>(m, n, rp, ci, static_cast<const C*>(v), static_cast<const C*>(x),
                    static_cast<C*>(y));
}
void oracle_csr_transpmult_c64(int32_t m, int32_t n, const int32_t* rp, const int32_t* ci,
                               const void* v, const void* x, void* y) {
  using C = std::complex<float>;
  csr_transpmult<C>(m, n, rp, ci, static_cast<const C*>(v), static_cast<const C*>(x),
                    static_cast<C*>(y));
}

// spmv::cg (cg.cpp:11-83) on all ranks.  The row map is assumed ghost-free
// and b[rank] has local_size entries; x[rank] receives local_size +
// num_ghosts entries (ghost tail zero).  MPI_Allreduce(SUM) is the sum of
// the ranks' values in rank order.  Returns the iteration count k.
// nthreads > 1 parallelises products and dots (CPU baseline timing only).
// max_its_run < max_its stops early after max_its_run iterations (a bounded
// CPU sample); pass max_its_run = max_its for the full algorithm.
int oracle_cg(oracle_map col_map, int P, const int32_t* nrows,
              const int32_t* const* rp, const int32_t* const* ci,
              const double* const* v, const double* const* b, double* const* x,
              int kmax, double rtol, int nthreads, int max_its_run,
              double* rnorm_out) {
  const Map& cm = col_map->m;
  std::vector<std::vector<double>> r(P), y(P), p(P);
  std::vector<double*> pp(P);
  for (int q = 0; q < P; ++q) {
    const int M = nrows[q];
    const int64_t L = cm.r[q].local_size + int64_t(cm.r[q].ghosts.size());
    r[q].assign(b[q], b[q] + M);                        // r = b
    y[q].assign(M, 0.0);
    p[q].assign(L, 0.0);                                // p.setZero()
    std::copy(r[q].begin(), r[q].end(), p[q].begin());  // p.head(M) = r
    std::fill(x[q], x[q] + L, 0.0);                     // x.setZero()
    pp[q] = p[q].data();
  }
  auto allreduce = [&](auto&& f) {
    double s = 0.0;
    for (int q = 0; q < P; ++q) s += f(q);
    return s;
  };
  const double rnorm0 = allreduce([&](int q) {
    return dot(r[q].data(), r[q].data(), nrows[q], nthreads);
  });
  const double rtol2 = rtol * rtol;
  double rnorm_old = rnorm0;
  int k = 0;
  while (k < kmax && k < max_its_run) {
    ++k;
    update<double>(cm, pp.data());                      // col_l2g->update(p)
    for (int q = 0; q < P; ++q)                         // y = A * p
      csr_mult<double>(nrows[q], rp[q], ci[q], v[q], p[q].data(), y[q].data(),
                       nthreads);
    const double pdoty_sum = allreduce([&](int q) {
      return dot(p[q].data(), y[q].data(), nrows[q], nthreads);
    });
    const double alpha = rnorm_old / pdoty_sum;
    for (int q = 0; q < P; ++q) {
      const int M = nrows[q];
      for (int i = 0; i < M; ++i) x[q][i] += alpha * p[q][i];
      for (int i = 0; i < M; ++i) r[q][i] -= alpha * y[q][i];
    }
    const double rnorm_new = allreduce([&](int q) {
      return dot(r[q].data(), r[q].data(), nrows[q], nthreads);
    });
    const double beta = rnorm_new / rnorm_old;
    rnorm_old = rnorm_new;
    for (int q = 0; q < P; ++q)
      for (int i = 0; i < nrows[q]; ++i) p[q][i] = p[q][i] * beta + r[q][i];
    if (rnorm_new / rnorm0 < rtol2) break;
  }
  if (rnorm_out) *rnorm_out = rnorm_old;
  return k;
}

// The matvec demo (matvecmain.cpp:16-121) on P virtual ranks: the operator of
// create_A (CreateA.cpp:31-111) with N rows, psp[i] = exp(-10 (5 (z-0.5))^2),
// z = global index / N, then n_apply times {update(psp); q = A psp;
// psp.head(M) = q}.  Returns sum over ranks of ||psp.head(M)||^2.
double oracle_matvec_demo(int P, int64_t N, int n_apply) {
  std::vector<int64_t> ranges(P + 1);
  oracle_owner_ranges(P, N, ranges.data());
  // create_A: global-column tridiagonal rows, then ghosts and local columns.
  std::vector<std::vector<int32_t>> rp(P), ci(P);
  std::vector<std::vector<double>> va(P);
  std::vector<int64_t> ls(P), ng(P);
  std::vector<std::vector<int64_t>> gh(P);
  const double gamma = 0.1;
  for (int q = 0; q < P; ++q) {
    const int64_t r0 = ranges[q], r1 = ranges[q + 1];
    const int M = int(r1 - r0);
    std::vector<std::vector<std::pair<int64_t, double>>> rows(M);
    for (int i = 0; i < M; ++i) {
      const int64_t c0 = r0 + i;
      if (c0 == 0) {
        rows[i] = {{c0, 1.0 - gamma}, {c0 + 1, gamma}};
      } else if (c0 == N - 1) {
        rows[i] = {{c0 - 1, gamma}, {c0, 1.0 - gamma}};
      } else {
        rows[i] = {{c0 - 1, gamma}, {c0, 1.0 - 2.0 * gamma}, {c0 + 1, gamma}};
      }
    }
    std::vector<int64_t> g;
    for (auto& row : rows)
      for (auto& e : row)
        if (e.first < r0 or e.first >= r1) g.push_back(e.first);
    std::sort(g.begin(), g.end());
    g.erase(std::unique(g.begin(), g.end()), g.end());
    gh[q] = g;
    ls[q] = M;
    ng[q] = int64_t(g.size());
    // Local columns (global_to_local) and setFromTriplets' sorted rows.
    rp[q].assign(M + 1, 0);
    for (int i = 0; i < M; ++i) {
      std::vector<std::pair<int32_t, double>> loc;
      for (auto& e : rows[i]) {
        int32_t c;
        if (e.first >= r0 && e.first < r1)
          c = int32_t(e.first - r0);
        else
          c = int32_t(M + (std::lower_bound(g.begin(), g.end(), e.first) - g.begin()));
        loc.push_back({c, e.second});
      }
      std::sort(loc.begin(), loc.end());
      for (auto& e : loc) {
        ci[q].push_back(e.first);
        va[q].push_back(e.second);
      }
      rp[q][i + 1] = int32_t(ci[q].size());
    }
  }
  std::vector<const int64_t*> gp(P);
  for (int q = 0; q < P; ++q) gp[q] = gh[q].data();
  Map m;
  build_map(m, P, ls.data(), gp.data(), ng.data());
  std::vector<std::vector<double>> psp(P), qv(P);
  std::vector<double*> pp(P);
  for (int q = 0; q < P; ++q) {
    psp[q].assign(ls[q] + ng[q], 0.0);
    for (int64_t i = 0; i < ls[q]; ++i) {
      const double z = double(i + ranges[q]) / double(N);
      psp[q][i] = std::exp(-10 * std::pow(5 * (z - 0.5), 2.0));
    }
    qv[q].assign(ls[q], 0.0);
    pp[q] = psp[q].data();
  }
  for (int it = 0; it < n_apply; ++it) {
    update<double>(m, pp.data());
    for (int q = 0; q < P; ++q)
      csr_mult<double>(int32_t(ls[q]), rp[q].data(), ci[q].data(), va[q].data(),
                       psp[q].data(), qv[q].data(), 1);
    for (int q = 0; q < P; ++q) std::copy(qv[q].begin(), qv[q].end(), psp[q].begin());
  }
  double s = 0.0;
  for (int q = 0; q < P; ++q) {
    double t = 0.0;
    for (int64_t i = 0; i < ls[q]; ++i) t += psp[q][i] * psp[q][i];
    s += t;
  }
  return s;
}

int oracle_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// spmv::read_petsc_binary (read_petsc.cpp:32-191) restated for all P ranks:
// big-endian header and arrays, rows and columns split by owner_ranges, the
// rank's columns numbered through an ordered map (owned first, then the
// other referenced columns in ascending order), entries inserted row by row
// the way Eigen's SparseMatrix::insert places them (ascending inner index; a
// repeated index goes after the ones already there) and then compressed.
// Returns a handle to every rank's CSR and ghosts, or null with an error.
typedef struct OraclePetsc* oracle_petsc;
struct OraclePetsc {
  struct Block {
    std::vector<int32_t> rowptr, colind;
    std::vector<double> vals;
    std::vector<int64_t> ghosts;
    int64_t ncols_local = 0;
  };
  std::vector<Block> blocks;
};

static int32_t swap_i32(const char* p) {
  char b[4] = {p[3], p[2], p[1], p[0]};
  int32_t v;
  std::memcpy(&v, b, 4);
  return v;
}
static double swap_f64(const char* p) {
  char b[8] = {p[7], p[6], p[5], p[4], p[3], p[2], p[1], p[0]};
  double v;
  std::memcpy(&v, b, 8);
  return v;
}

oracle_petsc oracle_petsc_read(const char* filename, int P) {
  oracle_petsc h = nullptr;
  const int st = guard([&] {
    std::ifstream file(filename, std::ios::in | std::ios::binary);
    if (!file.is_open()) throw std::runtime_error("Could not open file");
    std::vector<char> all((std::istreambuf_iterator<char>(file)), std::istreambuf_iterator<char>());
    if (all.size() < 16) throw std::runtime_error("short file");
    if (swap_i32(&all[0]) != 1211216)
      throw std::runtime_error("Bad signature in PETSc Matrix file");
    const int64_t nrows = swap_i32(&all[4]), ncols = swap_i32(&all[8]),
                  nnz_tot = swap_i32(&all[12]);
    const size_t need = 16 + size_t(nrows) * 4 + size_t(nnz_tot) * 12;
    if (all.size() < need) throw std::runtime_error("short file");
    std::vector<int32_t> nnz(nrows);
    for (int64_t i = 0; i < nrows; ++i) nnz[i] = swap_i32(&all[16 + 4 * i]);
    const char* cols = &all[16 + 4 * nrows];
    const char* vals = cols + 4 * nnz_tot;
    std::vector<int64_t> row_ranges(P + 1), col_ranges(P + 1);
    oracle_owner_ranges(P, nrows, row_ranges.data());
    oracle_owner_ranges(P, ncols, col_ranges.data());
    std::unique_ptr<OraclePetsc> out(new OraclePetsc);
    out->blocks.resize(P);
    for (int rank = 0; rank < P; ++rank) {
      OraclePetsc::Block& B = out->blocks[rank];
      int64_t nnz_offset = 0;
      for (int64_t i = 0; i < row_ranges[rank]; ++i) nnz_offset += nnz[i];
      std::map<int32_t, int32_t> col_indices;
      int32_t c = 0;
      for (int64_t col = col_ranges[rank]; col < col_ranges[rank + 1]; ++col)
        col_indices.insert({int32_t(col), c++});
      int64_t j = nnz_offset;
      for (int64_t row = row_ranges[rank]; row < row_ranges[rank + 1]; ++row)
        for (int32_t k = 0; k < nnz[row]; ++k, ++j)
          col_indices.insert({swap_i32(cols + 4 * j), -1});
      for (auto& q : col_indices)
        if (q.second == -1) q.second = c++;
      // Insert row by row into sorted inner vectors.
      const int64_t m = row_ranges[rank + 1] - row_ranges[rank];
      std::vector<std::vector<std::pair<int32_t, double>>> rows(m);
      j = nnz_offset;
      for (int64_t row = row_ranges[rank]; row < row_ranges[rank + 1]; ++row) {
        auto& rv = rows[row - row_ranges[rank]];
        for (int32_t k = 0; k < nnz[row]; ++k, ++j) {
          const int32_t lc = col_indices[swap_i32(cols + 4 * j)];
          const double v = swap_f64(vals + 8 * j);
          // Eigen's insert: shift the larger inner indices up by one.
          auto it = std::upper_bound(rv.begin(), rv.end(), lc,
                                     [](int32_t a, const std::pair<int32_t, double>& e) {
                                       return a < e.first;
                                     });
          rv.insert(it, {lc, v});
        }
      }
      B.rowptr.push_back(0);
      for (const auto& rv : rows) {
        for (const auto& e : rv) {
          B.colind.push_back(e.first);
          B.vals.push_back(e.second);
        }
        B.rowptr.push_back(int32_t(B.colind.size()));
      }
      B.ncols_local = col_ranges[rank + 1] - col_ranges[rank];
      B.ghosts.assign(col_indices.size() - B.ncols_local, 0);
      for (auto& q : col_indices)
        if (q.first < col_ranges[rank] || q.first >= col_ranges[rank + 1])
          B.ghosts[q.second - B.ncols_local] = q.first;
    }
    h = out.release();
  });
  return st == 0 ? h : nullptr;
}

void oracle_petsc_free(oracle_petsc h) { delete h; }

// Rank r's arrays: field 0 rowptr, 1 colind (int32); 2 values (double);
// 3 ghosts (int64).  Returns the element count and the data pointer.
int64_t oracle_petsc_block(oracle_petsc h, int rank, int field, const void** data) {
  const OraclePetsc::Block& B = h->blocks[rank];
  switch (field) {
    case 0: *data = B.rowptr.data(); return int64_t(B.rowptr.size());
    case 1: *data = B.colind.data(); return int64_t(B.colind.size());
    case 2: *data = B.vals.data(); return int64_t(B.vals.size());
    case 3: *data = B.ghosts.data(); return int64_t(B.ghosts.size());
  }
  *data = nullptr;
  return -1;
}

// Matrix::create_matrix (Matrix.cpp:213-438) restated for all P ranks.
// The MPI steps are restated by what they deliver: the Allgathers give the
// prefix ranges; each rank's ghost rows are packed per destination (the
// sorted std::set of owners) as {row, nnz, cols...} / {0, 0, vals...}; the
// neighbourhood alltoallv hands receiver q the segments of its sources in
// ascending rank order.  Eigen's setFromTriplets is restated by its steps: a
// column-major copy filled in triplet order, duplicates collapsed per column
// into the first occurrence (summed in order), then the transposed copy back
// to row-major (rows in ascending column order).
}  // extern "C"

typedef struct OracleAssembled* oracle_assembled;
struct OracleAssembled {
  std::vector<std::vector<int32_t>> rowptr, colind;
  std::vector<std::vector<std::complex<double>>> vals;
  std::vector<std::vector<int64_t>> ghosts;
};

template <typename T>
static void create_matrix_restated(int P, const int64_t* nrows_local, const int64_t* ncols_local,
                                   const int32_t* const* Aouter_all,
                                   const int32_t* const* Ainner_all, const T* const* Aval_all,
                                   const int64_t* const* row_ghosts_all,
                                   const int64_t* n_row_ghosts,
                                   const int64_t* const* col_ghosts_all,
                                   const int64_t* n_col_ghosts, OracleAssembled& out) {
  std::vector<int64_t> row_ranges(P + 1, 0), col_ranges(P + 1, 0);
  for (int i = 0; i < P; ++i) {
    row_ranges[i + 1] = row_ranges[i] + nrows_local[i];
    col_ranges[i + 1] = col_ranges[i] + ncols_local[i];
  }
  // Send side, per rank.
  std::vector<std::vector<int>> dests(P);
  std::vector<std::vector<int64_t>> send_index(P);
  std::vector<std::vector<T>> send_val(P);
  std::vector<std::vector<int>> send_offset(P);
  for (int rank = 0; rank < P; ++rank) {
    const int64_t ng = n_row_ghosts[rank];
    std::vector<int> row_owner(ng);
    for (int64_t i = 0; i < ng; ++i) {
      auto it = std::upper_bound(row_ranges.begin(), row_ranges.end(), row_ghosts_all[rank][i]);
      row_owner[i] = int(it - row_ranges.begin()) - 1;
    }
    std::set<int> neighbour_set(row_owner.begin(), row_owner.end());
    dests[rank].assign(neighbour_set.begin(), neighbour_set.end());
    std::map<int, int> proc_to_dest;
    for (size_t i = 0; i < dests[rank].size(); ++i) proc_to_dest.insert({dests[rank][i], int(i)});
    for (auto& q : row_owner) q = proc_to_dest[q];
    const int32_t* Aouter = Aouter_all[rank];
    const int32_t* Ainner = Ainner_all[rank];
    const T* Aval = Aval_all[rank];
    const int64_t nrl = nrows_local[rank], ncl = ncols_local[rank];
    std::vector<std::vector<int64_t>> p_to_index(dests[rank].size());
    std::vector<std::vector<T>> p_to_val(dests[rank].size());
    for (int64_t i = 0; i < ng; ++i) {
      const int p = row_owner[i];
      p_to_index[p].push_back(row_ghosts_all[rank][i]);
      p_to_val[p].push_back(T(0));
      p_to_index[p].push_back(Aouter[nrl + i + 1] - Aouter[nrl + i]);
      p_to_val[p].push_back(T(0));
      for (int j = Aouter[nrl + i]; j < Aouter[nrl + i + 1]; ++j) {
        const int64_t gi = Ainner[j] < ncl ? Ainner[j] + col_ranges[rank]
                                           : col_ghosts_all[rank][Ainner[j] - ncl];
        p_to_index[p].push_back(gi);
        p_to_val[p].push_back(Aval[j]);
      }
    }
    send_offset[rank] = {0};
    for (size_t p = 0; p < dests[rank].size(); ++p) {
      send_index[rank].insert(send_index[rank].end(), p_to_index[p].begin(), p_to_index[p].end());
      send_val[rank].insert(send_val[rank].end(), p_to_val[p].begin(), p_to_val[p].end());
      send_offset[rank].push_back(int(send_index[rank].size()));
    }
  }
  out.rowptr.assign(P, {});
  out.colind.assign(P, {});
  out.vals.assign(P, {});
  out.ghosts.assign(P, {});
  for (int rank = 0; rank < P; ++rank) {
    // Receive: sources in ascending rank order, each its segment for us.
    std::vector<int64_t> recv_index;
    std::vector<T> recv_val;
    for (int src = 0; src < P; ++src) {
      const auto& d = dests[src];
      auto it = std::find(d.begin(), d.end(), rank);
      if (it == d.end()) continue;
      const int k = int(it - d.begin());
      recv_index.insert(recv_index.end(), send_index[src].begin() + send_offset[src][k],
                        send_index[src].begin() + send_offset[src][k + 1]);
      recv_val.insert(recv_val.end(), send_val[src].begin() + send_offset[src][k],
                      send_val[src].begin() + send_offset[src][k + 1]);
    }
    const int64_t nrl = nrows_local[rank], ncl = ncols_local[rank];
    std::map<int64_t, int> col_ghost_map;
    for (int64_t i = 0; i < n_col_ghosts[rank]; ++i)
      col_ghost_map.insert({col_ghosts_all[rank][i], -1});
    size_t pos = 0;
    while (pos < recv_index.size()) {
      ++pos;
      const int nnz = int(recv_index[pos]);
      ++pos;
      for (int k = 0; k < nnz; ++k) {
        const int64_t recv_col = recv_index[pos++];
        if (recv_col >= col_ranges[rank + 1] || recv_col < col_ranges[rank])
          col_ghost_map.insert({recv_col, -1});
      }
    }
    int c = int(ncl);
    for (auto& q : col_ghost_map) q.second = c++;
    struct Trip {
      int row, col;
      T val;
    };
    std::vector<Trip> mat_data;
    const int32_t* Aouter = Aouter_all[rank];
    const int32_t* Ainner = Ainner_all[rank];
    for (int row = 0; row < nrl; ++row)
      for (int j = Aouter[row]; j < Aouter[row + 1]; ++j) {
        int col = Ainner[j];
        if (col >= ncl) col = col_ghost_map.find(col_ghosts_all[rank][col - ncl])->second;
        mat_data.push_back({row, col, Aval_all[rank][j]});
      }
    pos = 0;
    while (pos < recv_index.size()) {
      const int row = int(recv_index[pos] - row_ranges[rank]);
      ++pos;
      const int nnz = int(recv_index[pos]);
      ++pos;
      for (int k = 0; k < nnz; ++k) {
        const int64_t gc = recv_index[pos];
        const T val = recv_val[pos];
        ++pos;
        const int col = (gc >= col_ranges[rank + 1] || gc < col_ranges[rank])
                            ? col_ghost_map.find(gc)->second
                            : int(gc - col_ranges[rank]);
        mat_data.push_back({row, col, val});
      }
    }
    // setFromTriplets: column-major lists in triplet order.
    const int ncols = c;
    std::vector<std::vector<std::pair<int, T>>> tr(ncols);
    for (const Trip& t : mat_data) tr[t.col].push_back({t.row, t.val});
    // collapseDuplicates per column: first occurrence keeps the running sum.
    std::vector<int> wi(nrl, -1);
    for (int j = 0; j < ncols; ++j) {
      std::vector<std::pair<int, T>> kept;
      for (const auto& e : tr[j]) {
        if (wi[e.first] >= 0 && size_t(wi[e.first]) < kept.size() &&
            kept[wi[e.first]].first == e.first) {
          kept[wi[e.first]].second = kept[wi[e.first]].second + e.second;
        } else {
          wi[e.first] = int(kept.size());
          kept.push_back(e);
        }
      }
      for (const auto& e : kept) wi[e.first] = -1;
      tr[j] = std::move(kept);
    }
    // Transposed copy to row-major: rows in ascending column order.
    std::vector<std::vector<std::pair<int, T>>> rows(nrl);
    for (int j = 0; j < ncols; ++j)
      for (const auto& e : tr[j]) rows[e.first].push_back({j, e.second});
    auto& rp = out.rowptr[rank];
    rp.push_back(0);
    for (const auto& rv : rows) {
      for (const auto& e : rv) {
        out.colind[rank].push_back(e.first);
        out.vals[rank].push_back(std::complex<double>(e.second));
      }
      rp.push_back(int32_t(out.colind[rank].size()));
    }
    for (auto& q : col_ghost_map) out.ghosts[rank].push_back(q.first);
  }
}

extern "C" {

// dtype: 0 float64, 1 complex128 (values interleaved).
oracle_assembled oracle_create_matrix(int P, int dtype, const int64_t* nrows_local,
                                      const int64_t* ncols_local, const int32_t* const* rowptr,
                                      const int32_t* const* colind, const void* const* values,
                                      const int64_t* const* row_ghosts,
                                      const int64_t* n_row_ghosts,
                                      const int64_t* const* col_ghosts,
                                      const int64_t* n_col_ghosts) {
  oracle_assembled h = nullptr;
  const int st = guard([&] {
    std::unique_ptr<OracleAssembled> out(new OracleAssembled);
    if (dtype == 0)
      create_matrix_restated<double>(P, nrows_local, ncols_local, rowptr, colind,
                                     reinterpret_cast<const double* const*>(values), row_ghosts,
                                     n_row_ghosts, col_ghosts, n_col_ghosts, *out);
    else
      create_matrix_restated<std::complex<double>>(
          P, nrows_local, ncols_local, rowptr, colind,
          reinterpret_cast<const std::complex<double>* const*>(values), row_ghosts,
          n_row_ghosts, col_ghosts, n_col_ghosts, *out);
    h = out.release();
  });
  return st == 0 ? h : nullptr;
}

void oracle_assembled_free(oracle_assembled h) { delete h; }

// field: 0 rowptr, 1 colind (int32), 2 values (complex128 pairs), 3 ghosts.
int64_t oracle_assembled_block(oracle_assembled h, int rank, int field, const void** data) {
  switch (field) {
    case 0: *data = h->rowptr[rank].data(); return int64_t(h->rowptr[rank].size());
    case 1: *data = h->colind[rank].data(); return int64_t(h->colind[rank].size());
    case 2: *data = h->vals[rank].data(); return int64_t(h->vals[rank].size());
    case 3: *data = h->ghosts[rank].data(); return int64_t(h->ghosts[rank].size());
  }
  *data = nullptr;
  return -1;
}

}  // extern "C"
