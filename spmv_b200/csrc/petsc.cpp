// PETSc binary matrix and vector files (read_petsc.cpp:13-260 of the
// reference), read for all ranks of a communicator at once.
//
// Matrix file (PETSc "-ksp_view_mat binary", 32-bit indices, big endian):
// int32 {1211216, nrows, ncols, nnz}, int32 row lengths[nrows], int32 column
// indices[nnz] (row by row), float64 values[nnz].  Vector file: int32
// {1211214, n}, float64 values[n].
//
// Distribution (read_petsc.cpp:13-30, 66-67): rows and columns are split by
// owner_ranges (the first N % P ranks get one more).  Rank r's local columns
// are its owned columns in order, then every other column its rows reference
// in ascending global order (its ghosts; the reference numbers them through an
// ordered std::map, read_petsc.cpp:114-127).  Within a row, entries are in
// ascending local column order (the order Eigen's insert + makeCompressed
// leaves, read_petsc.cpp:140-156); entries with the same column keep their
// file order.
//
// Where the reference reads out of range or asserts (disabled) - a column
// index outside [0, ncols), row lengths that do not sum to nnz, a short file
// - this reader fails with an error instead.
#include <algorithm>
#include <cstring>
#include <fstream>
#include <numeric>
#include <thread>

#include "internal.h"

namespace spmvb {

std::vector<int64_t> owner_ranges(int P, int64_t N) {
  const int64_t n = N / P, rem = N % P;
  std::vector<int64_t> r(size_t(P) + 1);
  for (int q = 0; q <= P; ++q) r[q] = q < rem ? q * (n + 1) : q * n + rem;
  return r;
}

namespace {

int32_t be32(const unsigned char* p) {
  return int32_t((uint32_t(p[0]) << 24) | (uint32_t(p[1]) << 16) | (uint32_t(p[2]) << 8) |
                 uint32_t(p[3]));
}

double be64(const unsigned char* p) {
  uint64_t u = 0;
  for (int i = 0; i < 8; ++i) u = (u << 8) | uint64_t(p[i]);
  double d;
  std::memcpy(&d, &u, 8);
  return d;
}

// Reads `n` bytes at the current position or fails.
void read_exact(std::ifstream& f, unsigned char* dst, size_t n, const char* what) {
  f.read(reinterpret_cast<char*>(dst), std::streamsize(n));
  if (size_t(f.gcount()) != n)
    fail(SPMV_ERROR_INVALID_ARGUMENT, std::string("PETSc ") + what + " file is truncated");
}

std::ifstream open_file(const char* filename) {
  require(filename != nullptr, "spmv: NULL file name");
  std::ifstream f(filename, std::ios::in | std::ios::binary);
  if (!f.is_open()) fail(SPMV_ERROR_INVALID_ARGUMENT, "Could not open file");
  return f;
}

}  // namespace

// One rank's block of a PETSc matrix: local CSR and sorted ghosts.
struct PetscBlock {
  std::vector<int32_t> rowptr, colind;
  std::vector<double> vals;
  std::vector<int64_t> ghosts;
  int32_t nrows = 0, ncols_local = 0;
};

void read_petsc_matrix(const char* filename, int P, std::vector<PetscBlock>& blocks,
                       int64_t* nrows_out, int64_t* ncols_out) {
  std::ifstream f = open_file(filename);
  unsigned char hdr[16];
  read_exact(f, hdr, 16, "Matrix");
  if (be32(hdr) != 1211216) fail(SPMV_ERROR_INVALID_ARGUMENT, "Bad signature in PETSc Matrix file");
  const int64_t nrows = be32(hdr + 4), ncols = be32(hdr + 8), nnz = be32(hdr + 12);
  require(nrows >= 0 && ncols >= 0 && nnz >= 0, "spmv: negative size in PETSc Matrix file");
  std::vector<unsigned char> buf(size_t(nrows) * 4);
  read_exact(f, buf.data(), buf.size(), "Matrix");
  std::vector<int64_t> rowstart(size_t(nrows) + 1, 0);
  for (int64_t i = 0; i < nrows; ++i) {
    const int32_t len = be32(buf.data() + 4 * i);
    require(len >= 0, "spmv: negative row length in PETSc Matrix file");
    rowstart[i + 1] = rowstart[i] + len;
  }
  require(rowstart[nrows] == nnz, "spmv: PETSc Matrix file row lengths do not sum to nnz");
  std::vector<unsigned char> cbuf(size_t(nnz) * 4), vbuf(size_t(nnz) * 8);
  read_exact(f, cbuf.data(), cbuf.size(), "Matrix");
  read_exact(f, vbuf.data(), vbuf.size(), "Matrix");

  const std::vector<int64_t> rr = owner_ranges(P, nrows), cr = owner_ranges(P, ncols);
  blocks.assign(size_t(P), PetscBlock{});
  // One rank's block.  Rows already in ascending local order (the usual
  // case) are copied straight; others are stably sorted.
  auto build_block = [&](int r) {
    PetscBlock& B = blocks[r];
    const int64_t c0 = cr[r], c1 = cr[r + 1];
    const int64_t e0 = rowstart[rr[r]], e1 = rowstart[rr[r + 1]];
    require(e1 - e0 < (int64_t(1) << 31), "spmv: PETSc rank block too large for int32 indices");
    B.nrows = int32_t(rr[r + 1] - rr[r]);
    B.ncols_local = int32_t(c1 - c0);
    // Global columns of the rank's entries, and its ghosts (sorted, unique).
    std::vector<int64_t> g(size_t(e1 - e0));
    for (int64_t j = e0; j < e1; ++j) {
      const int64_t c = be32(cbuf.data() + 4 * j);
      require(c >= 0 && c < ncols, "spmv: column index out of range in PETSc Matrix file");
      g[size_t(j - e0)] = c;
      if (c < c0 || c >= c1) B.ghosts.push_back(c);
    }
    std::sort(B.ghosts.begin(), B.ghosts.end());
    B.ghosts.erase(std::unique(B.ghosts.begin(), B.ghosts.end()), B.ghosts.end());
    const int64_t nloc = int64_t(B.ncols_local) + int64_t(B.ghosts.size());
    require(nloc < (int64_t(1) << 31), "spmv: PETSc rank block too wide for int32 indices");
    B.rowptr.assign(size_t(B.nrows) + 1, 0);
    B.colind.resize(size_t(e1 - e0));
    B.vals.resize(size_t(e1 - e0));
    std::vector<int32_t> loc, order;
    for (int32_t i = 0; i < B.nrows; ++i) {
      const int64_t s = rowstart[rr[r] + i], e = rowstart[rr[r] + i + 1];
      B.rowptr[i + 1] = int32_t(e - e0);
      loc.resize(size_t(e - s));
      bool sorted = true;
      for (int64_t j = s; j < e; ++j) {
        const int64_t c = g[size_t(j - e0)];
        const int32_t l =
            c >= c0 && c < c1
                ? int32_t(c - c0)
                : int32_t(B.ncols_local +
                          (std::lower_bound(B.ghosts.begin(), B.ghosts.end(), c) - B.ghosts.begin()));
        if (j > s && l < loc[size_t(j - s) - 1]) sorted = false;
        loc[size_t(j - s)] = l;
      }
      int32_t* ci = B.colind.data() + (s - e0);
      double* va = B.vals.data() + (s - e0);
      if (sorted) {
        for (int64_t j = s; j < e; ++j) {
          ci[j - s] = loc[size_t(j - s)];
          va[j - s] = be64(vbuf.data() + 8 * j);
        }
        continue;
      }
      order.resize(loc.size());
      std::iota(order.begin(), order.end(), 0);
      std::stable_sort(order.begin(), order.end(),
                       [&](int32_t a, int32_t b) { return loc[a] < loc[b]; });
      for (size_t k = 0; k < order.size(); ++k) {
        ci[k] = loc[order[k]];
        va[k] = be64(vbuf.data() + 8 * (s + order[k]));
      }
    }
  };
  // Ranks are independent: one host thread each; the first error (in rank
  // order) is reported.
  std::vector<std::string> errs(static_cast<size_t>(P));
  std::vector<std::thread> pool;
  for (int r = 0; r < P; ++r)
    pool.emplace_back([&, r] {
      try {
        build_block(r);
      } catch (const std::exception& e) {
        errs[r] = e.what();
      }
    });
  for (auto& t : pool) t.join();
  for (const std::string& e : errs)
    if (!e.empty()) fail(SPMV_ERROR_INVALID_ARGUMENT, e);
  if (nrows_out) *nrows_out = nrows;
  if (ncols_out) *ncols_out = ncols;
}

int64_t petsc_vector_size(const char* filename) {
  std::ifstream f = open_file(filename);
  unsigned char hdr[8];
  read_exact(f, hdr, 8, "Vector");
  if (be32(hdr) != 1211214) fail(SPMV_ERROR_INVALID_ARGUMENT, "Bad signature in PETSc Vector file");
  const int64_t n = be32(hdr + 4);
  require(n >= 0, "spmv: negative size in PETSc Vector file");
  return n;
}

void read_petsc_vector(const char* filename, int P, double* const* out) {
  const int64_t n = petsc_vector_size(filename);
  std::ifstream f = open_file(filename);
  f.seekg(8, std::ios::beg);
  std::vector<unsigned char> buf(size_t(n) * 8);
  read_exact(f, buf.data(), buf.size(), "Vector");
  const std::vector<int64_t> rr = owner_ranges(P, n);
  for (int r = 0; r < P; ++r) {
    require(out[r] != nullptr || rr[r + 1] == rr[r], "spmv: NULL vector block");
    for (int64_t i = rr[r]; i < rr[r + 1]; ++i) out[r][i - rr[r]] = be64(buf.data() + 8 * i);
  }
}

}  // namespace spmvb

using namespace spmvb;

extern "C" {

int spmv_owner_ranges(int size, int64_t n, int64_t* ranges) {
  return guard([&] {
    require(size >= 1 && n >= 0 && ranges != nullptr, "spmv: invalid owner_ranges arguments");
    const std::vector<int64_t> r = owner_ranges(size, n);
    std::copy(r.begin(), r.end(), ranges);
  });
}

int spmv_petsc_read_matrix(spmv_comm comm, const char* filename, spmv_l2gmap* col_map,
                           spmv_l2gmap* row_map, spmv_matrix* A) {
  spmv_l2gmap cm = nullptr, rm = nullptr;
  const int st = guard([&] {
    require(comm != nullptr, "spmv: communicator is NULL");
    require(col_map && row_map && A, "spmv: NULL output");
    *col_map = nullptr;
    *row_map = nullptr;
    *A = nullptr;
    const int P = comm->size;
    std::vector<PetscBlock> blocks;
    read_petsc_matrix(filename, P, blocks, nullptr, nullptr);
    std::vector<int64_t> ls(P), rs(P), ng(P), zero(P, 0);
    std::vector<const int64_t*> gp(P), none(P, nullptr);
    std::vector<int32_t> nr(P), nc(P);
    std::vector<const int32_t*> rp(P), ci(P);
    std::vector<const void*> va(P);
    for (int r = 0; r < P; ++r) {
      const PetscBlock& B = blocks[r];
      ls[r] = B.ncols_local;
      rs[r] = B.nrows;
      ng[r] = int64_t(B.ghosts.size());
      gp[r] = B.ghosts.data();
      nr[r] = B.nrows;
      nc[r] = int32_t(B.ncols_local + int64_t(B.ghosts.size()));
      rp[r] = B.rowptr.data();
      ci[r] = B.colind.data();
      va[r] = B.vals.data();
    }
    auto check = [](int s) {
      if (s != SPMV_SUCCESS) fail(s, spmv_last_error());
    };
    check(spmv_l2gmap_create(comm, ls.data(), gp.data(), ng.data(), &cm));
    check(spmv_l2gmap_create(comm, rs.data(), none.data(), zero.data(), &rm));
    spmv_matrix m = nullptr;
    check(spmv_matrix_create_csr(comm, SPMV_FLOAT64, cm, rm, nr.data(), nc.data(), rp.data(),
                                 ci.data(), va.data(), &m));
    *col_map = cm;
    *row_map = rm;
    *A = m;
  });
  if (st != SPMV_SUCCESS) {
    // Keep the first error's message while releasing what was built.
    const std::string msg = spmv_last_error();
    if (rm) spmv_l2gmap_destroy(rm);
    if (cm) spmv_l2gmap_destroy(cm);
    spmvb::set_last_error(msg);
  }
  return st;
}

int spmv_petsc_vector_size(const char* filename, int64_t* n) {
  return guard([&] {
    require(n != nullptr, "spmv: NULL output");
    *n = petsc_vector_size(filename);
  });
}

int spmv_petsc_read_vector(spmv_comm comm, const char* filename, double* const* values) {
  return guard([&] {
    require(comm != nullptr, "spmv: communicator is NULL");
    require(values != nullptr, "spmv: vector array is NULL");
    read_petsc_vector(filename, comm->size, values);
  });
}

}  // extern "C"
