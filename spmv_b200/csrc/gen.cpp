// Seeded synthetic inputs for the benchmarks and tests (libspmv_gen).
//
// The reference ships no input files (its demos read PETSc files that are not
// in the repository, or build a tridiagonal operator in CreateA.cpp:31-111),
// so every workload here is generated.  Generation is host code and
// deterministic: the same seed gives the same matrix on any machine with the
// same libm.
//
// Random numbers are counter based, so each entry can be drawn independently
// (and in parallel):
//   mix(z)       = splitmix64 output function of z + 0x9E3779B97F4A7C15
//   key(s, t)    = mix(mix(s) ^ (t + 0x632BE59BD9B4E019))
//   u64(s, t, i) = mix(key(s, t) + i)
//   uniform      = (u64 >> 11) * 2^-53                     in [0, 1)
//   normal(i)    = Box-Muller on the pair (2*(i/2), 2*(i/2)+1):
//                  sqrt(-2 log(1-u_a)) * (cos|sin)(2 pi u_b), cos for even i
// s is the workload seed, t a stream number naming the quantity drawn.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#include "spmv_gen.h"

namespace {

thread_local std::string g_err;

inline uint64_t mix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
inline uint64_t key(uint64_t s, uint64_t t) {
  return mix(mix(s) ^ (t + 0x632BE59BD9B4E019ull));
}
inline double uni(uint64_t k, uint64_t i) {
  return double(mix(k + i) >> 11) * 0x1.0p-53;
}
inline double nrm(uint64_t k, uint64_t i) {
  const uint64_t a = i & ~uint64_t(1);
  const double ua = uni(k, a), ub = uni(k, a + 1);
  const double rad = std::sqrt(-2.0 * std::log(1.0 - ua));
  const double ang = 2.0 * M_PI * ub;
  return rad * ((i & 1) ? std::sin(ang) : std::cos(ang));
}

}  // namespace

struct spmv_gen_csr_s {
  int64_t nrows = 0, ncols = 0;
  std::vector<int32_t> rowptr, cols;
  std::vector<double> vals;
  // Extra per-matrix outputs (k-NN: bandwidth h; grid: edge list).
  double scalar = 0;
  std::vector<int64_t> aux_i64;
  std::vector<double> aux_f64;
};

namespace {

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

void need(bool ok, const char* msg) {
  if (!ok) throw std::runtime_error(msg);
}

// Builds CSR from per-row entry lists produced by `row(i, cols, vals)`.
template <class RowFn>
std::unique_ptr<spmv_gen_csr_s> build_rows(int64_t n, int64_t ncols, int maxrow,
                                           RowFn row) {
  auto h = std::make_unique<spmv_gen_csr_s>();
  h->nrows = n;
  h->ncols = ncols;
  h->rowptr.assign(n + 1, 0);
  std::vector<int32_t> cnt(n);
#pragma omp parallel
  {
    std::vector<int32_t> c(maxrow);
    std::vector<double> v(maxrow);
#pragma omp for schedule(static)
    for (int64_t i = 0; i < n; ++i) cnt[i] = row(i, c.data(), v.data());
  }
  for (int64_t i = 0; i < n; ++i) h->rowptr[i + 1] = h->rowptr[i] + cnt[i];
  need(h->rowptr[n] >= 0, "generator: too many entries for int32 row pointers");
  h->cols.resize(h->rowptr[n]);
  h->vals.resize(h->rowptr[n]);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    row(i, h->cols.data() + h->rowptr[i], h->vals.data() + h->rowptr[i]);
  return h;
}

}  // namespace

extern "C" {

const char* spmv_gen_last_error(void) { return g_err.c_str(); }

void spmv_gen_uniform(uint64_t seed, uint64_t stream, double lo, double hi,
                      double* out, int64_t n) {
  const uint64_t k = key(seed, stream);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) out[i] = lo + (hi - lo) * uni(k, uint64_t(i));
}

void spmv_gen_normal(uint64_t seed, uint64_t stream, double mean, double std,
                     double* out, int64_t n) {
  const uint64_t k = key(seed, stream);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) out[i] = mean + std * nrm(k, uint64_t(i));
}

void spmv_gen_csr_free(spmv_gen_csr h) { delete h; }

int spmv_gen_csr_info(spmv_gen_csr h, int64_t* nrows, int64_t* ncols,
                      int64_t* nnz) {
  return guard([&] {
    need(h, "generator: NULL handle");
    *nrows = h->nrows;
    *ncols = h->ncols;
    *nnz = h->rowptr.empty() ? 0 : h->rowptr.back();
  });
}

int spmv_gen_csr_arrays(spmv_gen_csr h, const int32_t** rowptr,
                        const int32_t** cols, const double** vals) {
  return guard([&] {
    need(h, "generator: NULL handle");
    *rowptr = h->rowptr.data();
    *cols = h->cols.data();
    *vals = h->vals.data();
  });
}

int spmv_gen_csr_aux(spmv_gen_csr h, double* scalar, const int64_t** i64,
                     int64_t* n_i64, const double** f64, int64_t* n_f64) {
  return guard([&] {
    need(h, "generator: NULL handle");
    if (scalar) *scalar = h->scalar;
    if (i64) *i64 = h->aux_i64.data();
    if (n_i64) *n_i64 = int64_t(h->aux_i64.size());
    if (f64) *f64 = h->aux_f64.data();
    if (n_f64) *n_f64 = int64_t(h->aux_f64.size());
  });
}

// 2D 5-point Laplacian [4, -1 x4] on an nx x ny grid, Dirichlet boundary
// (boundary rows drop their missing neighbours).  Row i = y*nx + x.
int spmv_gen_laplace2d(int64_t nx, int64_t ny, spmv_gen_csr* out) {
  return guard([&] {
    need(nx > 0 && ny > 0 && nx * ny < (int64_t(1) << 31), "laplace2d: bad size");
    *out = build_rows(nx * ny, nx * ny, 5, [=](int64_t i, int32_t* c, double* v) {
             const int64_t x = i % nx, y = i / nx;
             int k = 0;
             auto put = [&](int64_t j, double a) { c[k] = int32_t(j); v[k] = a; ++k; };
             if (y > 0) put(i - nx, -1.0);
             if (x > 0) put(i - 1, -1.0);
             put(i, 4.0);
             if (x + 1 < nx) put(i + 1, -1.0);
             if (y + 1 < ny) put(i + nx, -1.0);
             return k;
           }).release();
  });
}

// 3D 7-point Laplacian [6, -1 x6] on n^3, Dirichlet.  Row i = (z*n + y)*n + x.
int spmv_gen_laplace3d(int64_t n, spmv_gen_csr* out) {
  return guard([&] {
    need(n > 0 && n * n * n < (int64_t(1) << 31), "laplace3d: bad size");
    const int64_t n2 = n * n;
    *out = build_rows(n2 * n, n2 * n, 7, [=](int64_t i, int32_t* c, double* v) {
             const int64_t x = i % n, y = (i / n) % n, z = i / n2;
             int k = 0;
             auto put = [&](int64_t j, double a) { c[k] = int32_t(j); v[k] = a; ++k; };
             if (z > 0) put(i - n2, -1.0);
             if (y > 0) put(i - n, -1.0);
             if (x > 0) put(i - 1, -1.0);
             put(i, 6.0);
             if (x + 1 < n) put(i + 1, -1.0);
             if (y + 1 < n) put(i + n, -1.0);
             if (z + 1 < n) put(i + n2, -1.0);
             return k;
           }).release();
  });
}

// Weighted graph Laplacian of the 27-point stencil on n^3: each undirected
// edge (i, j) carries w ~ lognormal(0, 1) = exp(N(0,1)), drawn from stream 1
// at counter 13*min(i,j) + d, d the index of the direction from min to max
// among the 13 directions with a positive linear offset.  Off-diagonals are
// -w, the diagonal is sum(w) + shift.
int spmv_gen_laplace3d_27pt(int64_t n, uint64_t seed, double shift,
                            spmv_gen_csr* out) {
  return guard([&] {
    need(n > 1 && n * n * n < (int64_t(1) << 31), "laplace3d_27pt: bad size");
    const int64_t n2 = n * n;
    const uint64_t k = key(seed, 1);
    // Direction index of offset (dx,dy,dz) among the 13 "positive" ones.
    auto dir = [](int dx, int dy, int dz) {
      const int lin = (dz * 3 + dy) * 3 + dx;  // in [-13, 13]
      return lin > 0 ? lin - 1 : -lin - 1;     // 0..12 for both signs
    };
    *out = build_rows(n2 * n, n2 * n, 27, [=](int64_t i, int32_t* c, double* v) {
             const int64_t x = i % n, y = (i / n) % n, z = i / n2;
             int kk = 0, diag = -1;
             double wsum = 0.0;
             for (int dz = -1; dz <= 1; ++dz)
               for (int dy = -1; dy <= 1; ++dy)
                 for (int dx = -1; dx <= 1; ++dx) {
                   const int64_t X = x + dx, Y = y + dy, Z = z + dz;
                   if (X < 0 || Y < 0 || Z < 0 || X >= n || Y >= n || Z >= n) continue;
                   const int64_t j = (Z * n + Y) * n + X;
                   c[kk] = int32_t(j);
                   if (j == i) {
                     diag = kk;
                     v[kk++] = 0.0;
                     continue;
                   }
                   const int64_t lo = std::min(i, j);
                   const double w = std::exp(nrm(k, uint64_t(lo) * 13 + dir(dx, dy, dz)));
                   v[kk++] = -w;
                   wsum += w;
                 }
             v[diag] = wsum + shift;
             return kk;
           }).release();
  });
}

// 2D grid graph on nx x ny with 4-neighbour edges and weights softplus(theta):
// edge e joins (i, j), i < j, listed horizontal edges first (row by row),
// then vertical ones; theta_e ~ N(0, sigma) from stream 1.  A = L(w) + shift I.
// aux_i64 holds the edge list (2 per edge) and, for each edge, the CSR
// positions of A_ii, A_jj, A_ij, A_ji (4 per edge, after the edge list);
// aux_f64 holds theta.
int spmv_gen_grid2d_softplus(int64_t nx, int64_t ny, uint64_t seed,
                             double sigma, double shift, spmv_gen_csr* out) {
  return guard([&] {
    need(nx > 1 && ny > 1 && nx * ny < (int64_t(1) << 31), "grid2d: bad size");
    const int64_t n = nx * ny;
    const int64_t ne = (nx - 1) * ny + nx * (ny - 1);
    std::vector<int64_t> ei(ne), ej(ne);
    int64_t e = 0;
    for (int64_t y = 0; y < ny; ++y)
      for (int64_t x = 0; x + 1 < nx; ++x, ++e) {
        ei[e] = y * nx + x;
        ej[e] = y * nx + x + 1;
      }
    for (int64_t y = 0; y + 1 < ny; ++y)
      for (int64_t x = 0; x < nx; ++x, ++e) {
        ei[e] = y * nx + x;
        ej[e] = (y + 1) * nx + x;
      }
    std::vector<double> theta(ne);
    spmv_gen_normal(seed, 1, 0.0, sigma, theta.data(), ne);
    // Edge id of (node, neighbour direction): h-edges index y*(nx-1)+x,
    // v-edges (nx-1)*ny + y*nx + x.
    auto hid = [=](int64_t x, int64_t y) { return y * (nx - 1) + x; };
    auto vid = [=](int64_t x, int64_t y) { return (nx - 1) * ny + y * nx + x; };
    auto sp = [](double t) { return t > 30 ? t : std::log1p(std::exp(t)); };
    auto h = build_rows(n, n, 5, [&](int64_t i, int32_t* c, double* v) {
      const int64_t x = i % nx, y = i / nx;
      int k = 0, diag = -1;
      double ws = 0.0;
      auto put = [&](int64_t j, int64_t eid) {
        const double w = sp(theta[eid]);
        c[k] = int32_t(j);
        v[k++] = -w;
        ws += w;
      };
      if (y > 0) put(i - nx, vid(x, y - 1));
      if (x > 0) put(i - 1, hid(x - 1, y));
      diag = k;
      c[k] = int32_t(i);
      v[k++] = 0.0;
      if (x + 1 < nx) put(i + 1, hid(x, y));
      if (y + 1 < ny) put(i + nx, vid(x, y));
      v[diag] = ws + shift;
      return k;
    });
    auto pos = [&](int64_t r, int64_t col) -> int64_t {
      const int32_t* b = h->cols.data() + h->rowptr[r];
      const int32_t* en = h->cols.data() + h->rowptr[r + 1];
      const int32_t* it = std::lower_bound(b, en, int32_t(col));
      need(it != en && *it == col, "grid2d: missing entry");
      return h->rowptr[r] + (it - b);
    };
    h->aux_i64.resize(size_t(ne) * 6);
    for (int64_t q = 0; q < ne; ++q) {
      h->aux_i64[2 * q] = ei[q];
      h->aux_i64[2 * q + 1] = ej[q];
      int64_t* p4 = h->aux_i64.data() + 2 * ne + 4 * q;
      p4[0] = pos(ei[q], ei[q]);
      p4[1] = pos(ej[q], ej[q]);
      p4[2] = pos(ei[q], ej[q]);
      p4[3] = pos(ej[q], ei[q]);
    }
    h->aux_f64 = std::move(theta);
    *out = h.release();
  });
}

// Symmetrised k-NN graph Laplacian over n points uniform in [0,1]^3 (streams
// 10*sys+1..3 for x, y, z).  Edges join each point to its k nearest others
// (ties by index), united over both directions.  w = exp(-d^2/h^2) with h the
// mean distance over all (point, k-nearest) pairs (returned as the scalar);
// off-diagonals -w, diagonal sum(w) + shift.
int spmv_gen_knn_laplacian(int64_t n, int k, uint64_t seed, uint64_t sys,
                           double shift, spmv_gen_csr* out) {
  return guard([&] {
    need(n > k && k > 0 && n < (int64_t(1) << 31), "knn: bad size");
    std::vector<double> px(n), py(n), pz(n);
    spmv_gen_uniform(seed, 10 * sys + 1, 0.0, 1.0, px.data(), n);
    spmv_gen_uniform(seed, 10 * sys + 2, 0.0, 1.0, py.data(), n);
    spmv_gen_uniform(seed, 10 * sys + 3, 0.0, 1.0, pz.data(), n);
    // Uniform grid with about 2 points per cell.
    const int G = std::max(1, int(std::cbrt(double(n) / 2.0)));
    auto cell = [G](double u) { return std::min(G - 1, int(u * G)); };
    std::vector<int64_t> start(size_t(G) * G * G + 1, 0), order(n);
    std::vector<int> cid(n);
    for (int64_t i = 0; i < n; ++i) {
      cid[i] = (cell(pz[i]) * G + cell(py[i])) * G + cell(px[i]);
      ++start[cid[i] + 1];
    }
    for (size_t c = 0; c + 1 < start.size(); ++c) start[c + 1] += start[c];
    {
      std::vector<int64_t> fill(start.begin(), start.end() - 1);
      for (int64_t i = 0; i < n; ++i) order[fill[cid[i]]++] = i;
    }
    std::vector<int32_t> nb(size_t(n) * k);
    std::vector<double> nd(size_t(n) * k);
#pragma omp parallel
    {
      std::vector<std::pair<double, int64_t>> cand;
#pragma omp for schedule(dynamic, 256)
      for (int64_t i = 0; i < n; ++i) {
        const int cx = cell(px[i]), cy = cell(py[i]), cz = cell(pz[i]);
        for (int rad = 1;; ++rad) {
          cand.clear();
          for (int dz = -rad; dz <= rad; ++dz)
            for (int dy = -rad; dy <= rad; ++dy)
              for (int dx = -rad; dx <= rad; ++dx) {
                const int X = cx + dx, Y = cy + dy, Z = cz + dz;
                if (X < 0 || Y < 0 || Z < 0 || X >= G || Y >= G || Z >= G) continue;
                const int c = (Z * G + Y) * G + X;
                for (int64_t t = start[c]; t < start[c + 1]; ++t) {
                  const int64_t j = order[t];
                  if (j == i) continue;
                  const double ddx = px[j] - px[i], ddy = py[j] - py[i], ddz = pz[j] - pz[i];
                  cand.push_back({ddx * ddx + ddy * ddy + ddz * ddz, j});
                }
              }
          if (int64_t(cand.size()) < k && rad < G) continue;
          std::partial_sort(cand.begin(), cand.begin() + std::min<size_t>(k, cand.size()),
                            cand.end());
          // Every point within distance rad/G of i lies in the searched
          // cells, so the k-th candidate is exact once it is that close.
          const double reach = double(rad) / G;
          if (int64_t(cand.size()) >= k &&
              (cand[k - 1].first <= reach * reach || rad >= G)) {
            for (int q = 0; q < k; ++q) {
              nb[size_t(i) * k + q] = int32_t(cand[q].second);
              nd[size_t(i) * k + q] = std::sqrt(cand[q].first);
            }
            break;
          }
        }
      }
    }
    double hsum = 0.0;
    for (double d : nd) hsum += d;
    const double hh = hsum / double(nd.size());
    // Symmetric adjacency: union of i->nb and nb->i.
    std::vector<int64_t> deg(n + 1, 0);
    for (int64_t i = 0; i < n; ++i)
      for (int q = 0; q < k; ++q) {
        ++deg[i + 1];
        ++deg[nb[size_t(i) * k + q] + 1];
      }
    for (int64_t i = 0; i < n; ++i) deg[i + 1] += deg[i];
    std::vector<int32_t> adj(deg[n]);
    {
      std::vector<int64_t> fill(deg.begin(), deg.end() - 1);
      for (int64_t i = 0; i < n; ++i)
        for (int q = 0; q < k; ++q) {
          const int32_t j = nb[size_t(i) * k + q];
          adj[fill[i]++] = j;
          adj[fill[j]++] = int32_t(i);
        }
    }
    int maxrow = 1;
    for (int64_t i = 0; i < n; ++i) {
      std::sort(adj.begin() + deg[i], adj.begin() + deg[i + 1]);
      const int64_t u = std::unique(adj.begin() + deg[i], adj.begin() + deg[i + 1]) -
                        (adj.begin() + deg[i]);
      maxrow = std::max<int>(maxrow, int(u) + 1);
      // Mark the tail after the unique prefix.
      std::fill(adj.begin() + deg[i] + u, adj.begin() + deg[i + 1], -1);
    }
    const double inv_h2 = 1.0 / (hh * hh);
    auto h = build_rows(n, n, maxrow, [&](int64_t i, int32_t* c, double* v) {
      int kk = 0, diag = -1;
      double ws = 0.0;
      bool placed = false;
      for (int64_t t = deg[i]; t < deg[i + 1] && adj[t] >= 0; ++t) {
        const int32_t j = adj[t];
        if (!placed && j > i) {
          diag = kk;
          c[kk] = int32_t(i);
          v[kk++] = 0.0;
          placed = true;
        }
        const double dx = px[j] - px[i], dy = py[j] - py[i], dz = pz[j] - pz[i];
        const double w = std::exp(-(dx * dx + dy * dy + dz * dz) * inv_h2);
        c[kk] = j;
        v[kk++] = -w;
        ws += w;
      }
      if (!placed) {
        diag = kk;
        c[kk] = int32_t(i);
        v[kk++] = 0.0;
      }
      v[diag] = ws + shift;
      return kk;
    });
    h->scalar = hh;
    *out = h.release();
  });
}

// The operator of the reference's matvec demo (CreateA.cpp:31-75): global
// tridiagonal [g, 1-2g, g] of size N with the first and last rows [1-g, g]
// and [g, 1-g], g = 0.1.
int spmv_gen_create_a(int64_t N, spmv_gen_csr* out) {
  return guard([&] {
    need(N >= 2 && N < (int64_t(1) << 31), "create_a: bad size");
    const double g = 0.1;
    *out = build_rows(N, N, 3, [=](int64_t i, int32_t* c, double* v) {
             int k = 0;
             if (i == 0) {
               c[k] = 0; v[k++] = 1.0 - g;
               c[k] = 1; v[k++] = g;
             } else if (i == N - 1) {
               c[k] = int32_t(i - 1); v[k++] = g;
               c[k] = int32_t(i); v[k++] = 1.0 - g;
             } else {
               c[k] = int32_t(i - 1); v[k++] = g;
               c[k] = int32_t(i); v[k++] = 1.0 - 2.0 * g;
               c[k] = int32_t(i + 1); v[k++] = g;
             }
             return k;
           }).release();
  });
}

}  // extern "C"
