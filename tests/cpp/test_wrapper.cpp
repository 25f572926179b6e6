// Exercises the C++ mirror of the reference API (include/spmv/spmv.hpp).
// argv[1] == "host": host-only checks (maps and errors, no GPU needed).
// argv[1] == "gpu":  also runs update, mult, transpmult and cg on device 0
// for a 1D Laplacian split over 3 ranks and prints the results.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>

#include "spmv/spmv.hpp"

static int fails = 0;
#define EXPECT(c)                                                   \
  do {                                                              \
    if (!(c)) {                                                     \
      std::printf("FAIL %s:%d %s\n", __FILE__, __LINE__, #c);       \
      ++fails;                                                      \
    }                                                               \
  } while (0)

template <class F>
static std::string message_of(F&& f) {
  try {
    f();
  } catch (const std::runtime_error& e) {
    return e.what();
  }
  return "";
}

int main(int argc, char** argv) {
  const bool gpu = argc > 1 && std::strcmp(argv[1], "gpu") == 0;
  {
    spmv::Comm comm(2, -1);
    EXPECT(message_of([&] { spmv::L2GMap m(comm, {4, 4}, {{6, 5}, {}}); }) ==
           "Ghosts must be sorted");
    EXPECT(message_of([&] { spmv::L2GMap m(comm, {4, 4}, {{1}, {}}); }) ==
           "Ghost index in local range");
    spmv::L2GMap m(comm, {4, 4}, {{4}, {3}});
    EXPECT(m.local_size(1) == 4 && m.num_ghosts(0) == 1 && m.global_size() == 8);
    EXPECT(m.global_offset(1) == 4 && m.global_to_local(0, 4) == 4);
    EXPECT(m.ghosts(1).size() == 1 && m.ghosts(1)[0] == 3);
  }
  {
    // create_matrix: two ranks of a 4-point chain, rank 0 owns rows 0-1 and
    // holds a ghost row for node 2 (owned by rank 1) with entries in columns
    // 1 (owned) and 2 (a ghost column); rank 1 adds its own row 2 entry.
    spmv::Comm comm(2, -1);
    std::vector<spmv::CsrBlock<double>> blocks(2);
    blocks[0].rowptr = {0, 1, 2, 4};       // rows 0, 1 and ghost row 2
    blocks[0].colind = {0, 1, 1, 2};       // local col 2 = global 2
    blocks[0].values = {1.0, 2.0, 3.0, 4.0};
    blocks[1].rowptr = {0, 1, 2};          // rows 2, 3
    blocks[1].colind = {0, 1};
    blocks[1].values = {10.0, 20.0};
    auto A = spmv::Matrix<double>::create_matrix(comm, blocks, {2, 2}, {2, 2}, {{2}, {}},
                                                 {{2}, {}});
    // Rank 1, row 0 (global 2): own entry 10 at col 0, plus received 4.0 at
    // global 2 (= local 0, summed: 14) and 3.0 at global 1 (a new ghost).
    const std::int32_t *rp = nullptr, *ci = nullptr;
    const void* va = nullptr;
    spmv::detail::check(spmv_matrix_csr(A.handle(), 1, &rp, &ci, &va));
    const double* v = static_cast<const double*>(va);
    EXPECT(rp[1] == 2 && ci[0] == 0 && v[0] == 14.0 && ci[1] == 2 && v[1] == 3.0);
    EXPECT(A.col_map()->num_ghosts(1) == 1 && A.col_map()->ghosts(1)[0] == 1);
  }
  if (argc > 2) {
    // argv[2]: a PETSc binary file of the 5x5 matrix with A[i][j] = 10 i + j
    // on |i - j| <= 1, rows written with descending columns; argv[3] the
    // vector 0..4.  Two ranks: rows/columns {0,1,2} and {3,4}.
    spmv::Comm comm(2, -1);
    spmv::Matrix<double> A = spmv::read_petsc_binary(comm, argv[2]);
    EXPECT(A.rows(0) == 3 && A.rows(1) == 2);
    EXPECT(A.col_map()->num_ghosts(0) == 1 && A.col_map()->ghosts(0)[0] == 3);
    EXPECT(A.col_map()->num_ghosts(1) == 1 && A.col_map()->ghosts(1)[0] == 2);
    const std::int32_t *rp = nullptr, *ci = nullptr;
    const void* va = nullptr;
    spmv::detail::check(spmv_matrix_csr(A.handle(), 1, &rp, &ci, &va));
    // rank 1 row 0 (global 3): owned columns 3, 4 -> local 0, 1, then the
    // ghost 2 -> local 2, in ascending local order.
    const double* v = static_cast<const double*>(va);
    EXPECT(rp[1] == 3 && ci[0] == 0 && ci[1] == 1 && ci[2] == 2);
    EXPECT(v[0] == 33.0 && v[1] == 34.0 && v[2] == 32.0);
    auto b = spmv::read_petsc_binary_vector(comm, argv[3]);
    EXPECT(b.size() == 2 && b[0].size() == 3 && b[1].size() == 2 && b[1][1] == 4.0);
    EXPECT(message_of([&] { spmv::read_petsc_binary(comm, argv[3]); }) ==
           "Bad signature in PETSc Matrix file");
    EXPECT(message_of([&] { spmv::read_petsc_binary(comm, "/nonexistent/x.dat"); }) ==
           "Could not open file");
  }
  if (gpu) {
    // 1D Laplacian [-1, 2, -1] on 12 points over 3 ranks of 4.
    const int P = 3, M = 4;
    spmv::Comm comm(P, 0);
    std::vector<std::vector<std::int64_t>> gh = {{4}, {3, 8}, {7}};
    auto cm = std::make_shared<spmv::L2GMap>(comm, std::vector<std::int64_t>{M, M, M}, gh);
    auto rm = std::make_shared<spmv::L2GMap>(
        comm, std::vector<std::int64_t>{M, M, M},
        std::vector<std::vector<std::int64_t>>(P));
    std::vector<spmv::CsrBlock<double>> blocks(P);
    for (int r = 0; r < P; ++r) {
      auto& B = blocks[r];
      B.rowptr = {0};
      for (int i = 0; i < M; ++i) {
        const std::int64_t g = r * M + i;
        std::vector<std::pair<int, double>> e;
        for (std::int64_t c : {g - 1, g, g + 1}) {
          if (c < 0 || c >= P * M) continue;
          e.push_back({cm->global_to_local(r, c), c == g ? 2.0 : -1.0});
        }
        std::sort(e.begin(), e.end());
        for (auto& p : e) {
          B.colind.push_back(p.first);
          B.values.push_back(p.second);
        }
        B.rowptr.push_back(std::int32_t(B.colind.size()));
      }
    }
    spmv::Matrix<double> A(comm, blocks, cm, rm);
    std::vector<std::vector<double>> x(P);
    std::vector<double*> xp(P);
    for (int r = 0; r < P; ++r) {
      x[r].assign(M + cm->num_ghosts(r), 0.0);
      for (int i = 0; i < M; ++i) x[r][i] = double(r * M + i);
      xp[r] = x[r].data();
    }
    cm->update(xp);
    EXPECT(x[1][4] == 3.0 && x[1][5] == 8.0 && x[0][4] == 4.0 && x[2][4] == 7.0);
    auto y = A * x;  // A applied to a linear function: zero inside
    EXPECT(y[1][0] == 0.0 && y[1][3] == 0.0 && y[0][0] == -1.0 && y[2][3] == 11.0 * 2 - 10.0);
    std::vector<std::vector<double>> b(P, std::vector<double>(M, 1.0));
    auto [sol, its] = spmv::cg(comm, A, b, 100, 1e-12);
    EXPECT(its <= 12 && its > 0);
    // x_i = i(11 - i)/2 + ... : check the residual instead.
    for (int r = 0; r < P; ++r) sol[r].resize(M + cm->num_ghosts(r));
    std::vector<double*> sp(P);
    for (int r = 0; r < P; ++r) sp[r] = sol[r].data();
    cm->update(sp);
    auto ax = A * sol;
    double res = 0;
    for (int r = 0; r < P; ++r)
      for (int i = 0; i < M; ++i) res = std::max(res, std::fabs(ax[r][i] - 1.0));
    EXPECT(res < 1e-9);
    EXPECT(message_of([&] { spmv::cg(comm, A, {{1, 2}, {1, 2, 3, 4}, {1, 2, 3, 4}}, 10, 1e-8); }) ==
           "spmv::cg - Error: b.rows() != A.rows()");
    std::printf("cg iterations %d residual %g\n", its, res);
  }
  std::printf("%s %d failures\n", fails ? "FAILED" : "OK", fails);
  return fails ? 1 : 0;
}
