// Matrix::create_matrix (Matrix.cpp:213-438 of the reference) for all ranks
// of a communicator at once: each rank's block holds its owned rows followed
// by ghost rows (rows another rank owns, e.g. from element assembly); ghost
// rows go to their owners and are added in, and the owners' column maps grow
// by the new ghost columns those rows bring.
//
// Semantics kept from the reference:
//  * row and column ranges are the prefix sums of the ranks' owned counts
//    (Matrix.cpp:223-235); a ghost row's owner is the rank whose range holds
//    it (:238-246);
//  * each receiving rank sees the ghost rows sent to it in ascending sender
//    order, each sender's rows in that sender's ghost-row order (the
//    neighbourhood alltoallv over the sorted source list, :254-340);
//  * the new ghost columns are the old ones plus every received column
//    outside the owned range, in ascending global order (:342-367);
//  * the matrix is built from triplets - own rows first, in storage order,
//    then the received rows in arrival order - as Eigen's setFromTriplets
//    builds it (:369-428): entries with the same (row, column) are summed in
//    triplet order, and each row ends up in ascending column order.
//
// On a communicator with a GPU the assembly runs there (assemble_dev.cu);
// this file holds the host form, used by communicators without a device.  Where the reference asserts
// (disabled) or reads out of range - a ghost row owned by its own rank or
// outside the global range, a column outside the block - this fails with an
// error.
#include <algorithm>
#include <cstring>
#include <numeric>

#include "internal.h"

namespace spmvb {

namespace {

template <typename T>
struct Assembled {
  std::vector<int32_t> rowptr, colind;
  std::vector<T> vals;
  std::vector<int64_t> ghosts;
};

struct Triplet {
  int32_t row, col;
  int64_t src;  // index into the value source (triplet order)
};

template <typename T>
void assemble(int P, const int64_t* nrows_local, const int64_t* ncols_local,
              const int32_t* const* rowptr, const int32_t* const* colind,
              const void* const* values, const int64_t* const* row_ghosts,
              const int64_t* n_row_ghosts, const int64_t* const* col_ghosts,
              const int64_t* n_col_ghosts, std::vector<Assembled<T>>& out) {
  std::vector<int64_t> rr(size_t(P) + 1, 0), cr(size_t(P) + 1, 0);
  for (int r = 0; r < P; ++r) {
    require(nrows_local[r] >= 0 && ncols_local[r] >= 0 && n_row_ghosts[r] >= 0 &&
                n_col_ghosts[r] >= 0,
            "spmv::Matrix::create_matrix - Error: negative size");
    rr[r + 1] = rr[r] + nrows_local[r];
    cr[r + 1] = cr[r] + ncols_local[r];
  }
  auto val = [&](int r, int64_t j) { return static_cast<const T*>(values[r])[j]; };
  auto global_col = [&](int r, int32_t c) -> int64_t {
    require(c >= 0 && c < ncols_local[r] + n_col_ghosts[r],
            "spmv::Matrix::create_matrix - Error: column index outside the block");
    return c < ncols_local[r] ? cr[r] + c : col_ghosts[r][c - ncols_local[r]];
  };

  // Ghost rows by destination rank, in the order each receiver sees them:
  // inbox[q] lists (sender, ghost row index) by ascending sender, then the
  // sender's ghost-row order.
  std::vector<std::vector<std::pair<int, int64_t>>> inbox(P);
  for (int r = 0; r < P; ++r)
    for (int64_t i = 0; i < n_row_ghosts[r]; ++i) {
      const int64_t g = row_ghosts[r][i];
      require(g >= 0 && g < rr[P], "spmv::Matrix::create_matrix - Error: ghost row out of range");
      const int owner = int(std::upper_bound(rr.begin(), rr.end(), g) - rr.begin()) - 1;
      require(owner != r, "spmv::Matrix::create_matrix - Error: ghost row owned by its own rank");
      inbox[owner].push_back({r, i});
    }
  // (The loop above visits senders in ascending order, so each inbox is
  // already in arrival order.)

  out.assign(size_t(P), Assembled<T>{});
  for (int q = 0; q < P; ++q) {
    Assembled<T>& A = out[q];
    const int64_t nl = nrows_local[q], cl = ncols_local[q];
    // New ghost columns: old ones plus received columns outside the range.
    std::vector<int64_t> ghosts(col_ghosts[q], col_ghosts[q] + n_col_ghosts[q]);
    for (const auto& m : inbox[q]) {
      const int r = m.first;
      const int64_t row = nrows_local[r] + m.second;
      for (int32_t j = rowptr[r][row]; j < rowptr[r][row + 1]; ++j) {
        const int64_t g = global_col(r, colind[r][j]);
        if (g < cr[q] || g >= cr[q + 1]) ghosts.push_back(g);
      }
    }
    std::sort(ghosts.begin(), ghosts.end());
    ghosts.erase(std::unique(ghosts.begin(), ghosts.end()), ghosts.end());
    require(cl + int64_t(ghosts.size()) < (int64_t(1) << 31),
            "spmv::Matrix::create_matrix - Error: block too wide for int32 indices");
    auto local_of = [&](int64_t g) -> int32_t {
      if (g >= cr[q] && g < cr[q + 1]) return int32_t(g - cr[q]);
      return int32_t(cl + (std::lower_bound(ghosts.begin(), ghosts.end(), g) - ghosts.begin()));
    };
    // Triplets in the reference's order, values kept by reference.
    std::vector<Triplet> trip;
    std::vector<T> tval;
    for (int32_t row = 0; row < nl; ++row)
      for (int32_t j = rowptr[q][row]; j < rowptr[q][row + 1]; ++j) {
        const int32_t c = colind[q][j];
        trip.push_back({row, c < cl ? c : local_of(global_col(q, c)), int64_t(tval.size())});
        tval.push_back(val(q, j));
      }
    for (const auto& m : inbox[q]) {
      const int r = m.first;
      const int32_t row = int32_t(row_ghosts[r][m.second] - rr[q]);
      const int64_t lrow = nrows_local[r] + m.second;
      for (int32_t j = rowptr[r][lrow]; j < rowptr[r][lrow + 1]; ++j) {
        trip.push_back({row, local_of(global_col(r, colind[r][j])), int64_t(tval.size())});
        tval.push_back(val(r, j));
      }
    }
    // setFromTriplets: stable order by (row, column), duplicates summed in
    // triplet order.
    std::stable_sort(trip.begin(), trip.end(), [](const Triplet& a, const Triplet& b) {
      return a.row != b.row ? a.row < b.row : a.col < b.col;
    });
    A.rowptr.assign(size_t(nl) + 1, 0);
    for (size_t k = 0; k < trip.size();) {
      T sum = tval[trip[k].src];
      size_t e = k + 1;
      while (e < trip.size() && trip[e].row == trip[k].row && trip[e].col == trip[k].col) {
        sum = sum + tval[trip[e].src];
        ++e;
      }
      A.colind.push_back(trip[k].col);
      A.vals.push_back(sum);
      A.rowptr[trip[k].row + 1] += 1;
      k = e;
    }
    for (int64_t i = 0; i < nl; ++i) A.rowptr[i + 1] += A.rowptr[i];
    A.ghosts = std::move(ghosts);
  }
}

template <typename T>
void create_assembled(spmv_comm comm, spmv_dtype dtype, const int64_t* nrows_local,
                      const int64_t* ncols_local, const int32_t* const* rowptr,
                      const int32_t* const* colind, const void* const* values,
                      const int64_t* const* row_ghosts, const int64_t* n_row_ghosts,
                      const int64_t* const* col_ghosts, const int64_t* n_col_ghosts,
                      spmv_l2gmap* cm, spmv_l2gmap* rm, spmv_matrix* m) {
  const int P = comm->size;
  std::vector<Assembled<T>> blocks;
  assemble<T>(P, nrows_local, ncols_local, rowptr, colind, values, row_ghosts, n_row_ghosts,
              col_ghosts, n_col_ghosts, blocks);
  std::vector<int64_t> ng(P), zero(P, 0);
  std::vector<const int64_t*> gp(P), none(P, nullptr);
  std::vector<int32_t> nr(P), nc(P);
  std::vector<const int32_t*> rp(P), ci(P);
  std::vector<const void*> va(P);
  for (int r = 0; r < P; ++r) {
    ng[r] = int64_t(blocks[r].ghosts.size());
    gp[r] = blocks[r].ghosts.data();
    nr[r] = int32_t(nrows_local[r]);
    nc[r] = int32_t(ncols_local[r] + ng[r]);
    rp[r] = blocks[r].rowptr.data();
    ci[r] = blocks[r].colind.data();
    va[r] = blocks[r].vals.data();
  }
  auto check = [](int s) {
    if (s != SPMV_SUCCESS) fail(s, spmv_last_error());
  };
  check(spmv_l2gmap_create(comm, ncols_local, gp.data(), ng.data(), cm));
  check(spmv_l2gmap_create(comm, nrows_local, none.data(), zero.data(), rm));
  check(spmv_matrix_create_csr(comm, dtype, *cm, *rm, nr.data(), nc.data(), rp.data(),
                               ci.data(), va.data(), m));
}

// Addition of the scalar types (complex values as interleaved pairs).
template <typename F>
struct CplxH {
  F re, im;
  CplxH operator+(const CplxH& o) const { return {re + o.re, im + o.im}; }
};

}  // namespace

// assemble_dev.cu: the same assembly on the communicator's GPU.
void create_assembled_device(spmv_comm comm, spmv_dtype dtype, const int64_t* nrows_local,
                             const int64_t* ncols_local, const int32_t* const* rowptr,
                             const int32_t* const* colind, const void* const* values,
                             const int64_t* const* row_ghosts, const int64_t* n_row_ghosts,
                             const int64_t* const* col_ghosts, const int64_t* n_col_ghosts,
                             spmv_l2gmap* cm, spmv_l2gmap* rm, spmv_matrix* m);

}  // namespace spmvb

using namespace spmvb;

extern "C" {

int spmv_matrix_create_assembled(spmv_comm comm, spmv_dtype dtype, const int64_t* nrows_local,
                                 const int64_t* ncols_local, const int32_t* const* rowptr,
                                 const int32_t* const* colind, const void* const* values,
                                 const int64_t* const* row_ghosts, const int64_t* n_row_ghosts,
                                 const int64_t* const* col_ghosts,
                                 const int64_t* n_col_ghosts, spmv_l2gmap* col_map,
                                 spmv_l2gmap* row_map, spmv_matrix* A) {
  spmv_l2gmap cm = nullptr, rm = nullptr;
  const int st = guard([&] {
    require(comm != nullptr, "spmv: communicator is NULL");
    require(col_map && row_map && A, "spmv: NULL output");
    *col_map = nullptr;
    *row_map = nullptr;
    *A = nullptr;
    require(nrows_local && ncols_local && rowptr && colind && values && row_ghosts &&
                n_row_ghosts && col_ghosts && n_col_ghosts,
            "spmv::Matrix::create_matrix - Error: NULL argument");
    spmv_matrix m = nullptr;
    if (comm->device >= 0) {
      // Routing, triplet sort and duplicate sums on the GPU.
      create_assembled_device(comm, dtype, nrows_local, ncols_local, rowptr, colind, values,
                              row_ghosts, n_row_ghosts, col_ghosts, n_col_ghosts, &cm, &rm, &m);
      *col_map = cm;
      *row_map = rm;
      *A = m;
      return;
    }
    // A communicator without a device (device -1) assembles on the host.
    switch (dtype) {
      case SPMV_FLOAT64:
        create_assembled<double>(comm, dtype, nrows_local, ncols_local, rowptr, colind, values,
                                 row_ghosts, n_row_ghosts, col_ghosts, n_col_ghosts, &cm, &rm,
                                 &m);
        break;
      case SPMV_FLOAT32:
        create_assembled<float>(comm, dtype, nrows_local, ncols_local, rowptr, colind, values,
                                row_ghosts, n_row_ghosts, col_ghosts, n_col_ghosts, &cm, &rm,
                                &m);
        break;
      case SPMV_COMPLEX128:
        create_assembled<CplxH<double>>(comm, dtype, nrows_local, ncols_local, rowptr, colind,
                                        values, row_ghosts, n_row_ghosts, col_ghosts,
                                        n_col_ghosts, &cm, &rm, &m);
        break;
      case SPMV_COMPLEX64:
        create_assembled<CplxH<float>>(comm, dtype, nrows_local, ncols_local, rowptr, colind,
                                       values, row_ghosts, n_row_ghosts, col_ghosts,
                                       n_col_ghosts, &cm, &rm, &m);
        break;
      default:
        fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv::Matrix::create_matrix - Error: unknown dtype");
    }
    *col_map = cm;
    *row_map = rm;
    *A = m;
  });
  if (st != SPMV_SUCCESS) {
    const std::string msg = spmv_last_error();
    if (rm) spmv_l2gmap_destroy(rm);
    if (cm) spmv_l2gmap_destroy(cm);
    spmvb::set_last_error(msg);
  }
  return st;
}

}  // extern "C"
