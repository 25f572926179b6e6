// spmv/spmv.hpp - C++ mirror of libspmv's hot-path API (spmv::L2GMap,
// spmv::Matrix<T>, spmv::cg) over the C ABI of libspmv_b200.
//
// Same class names, method names and error strings as the reference
// (L2GMap.h:14-97, Matrix.h:23-81, cg.h:27-29); errors throw
// std::runtime_error with the reference's message.  Two differences follow
// from running every rank on one GPU:
//  * MPI_Comm becomes spmv::Comm, a virtual communicator of `size` ranks on
//    one device, and the collective calls (the L2GMap constructor, update,
//    reverse_update, cg) take all ranks' data at once, one entry per rank;
//  * Eigen types become std::vector (Eigen is an optional dependency of the
//    reference only); CSR blocks are passed as (rowptr, colind, values).
// Header-only; link with -lspmv_b200.
#pragma once

#include <complex>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <utility>
#include <vector>

#include "../spmv_b200.h"

namespace spmv {

namespace detail {
inline void check(int status) {
  if (status != SPMV_SUCCESS) throw std::runtime_error(spmv_last_error());
}
template <typename T>
constexpr spmv_dtype dtype_of() {
  static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value ||
                    std::is_same<T, std::complex<double>>::value ||
                    std::is_same<T, std::complex<float>>::value,
                "spmv_b200 scalars: float, double, std::complex<float>, std::complex<double>");
  return std::is_same<T, double>::value                 ? SPMV_FLOAT64
         : std::is_same<T, float>::value                ? SPMV_FLOAT32
         : std::is_same<T, std::complex<double>>::value ? SPMV_COMPLEX128
                                                        : SPMV_COMPLEX64;
}
}  // namespace detail

/// Virtual communicator: `size` ranks that live on CUDA device `device`.
class Comm {
 public:
  explicit Comm(int size, int device = 0, void* cuda_stream = nullptr) {
    detail::check(spmv_comm_create(device, cuda_stream, size, &h_));
  }
  ~Comm() { spmv_comm_destroy(h_); }
  Comm(const Comm&) = delete;
  Comm& operator=(const Comm&) = delete;
  int size() const {
    int s = 0;
    detail::check(spmv_comm_size(h_, &s));
    return s;
  }
  void synchronize() const { detail::check(spmv_comm_synchronize(h_)); }
  spmv_comm handle() const { return h_; }

 private:
  spmv_comm h_ = nullptr;
};

/// Local to global map of every rank (L2GMap.h:14-97).
class L2GMap {
 public:
  /// Collective constructor (L2GMap.cpp:15-122): local_size[r] and sorted
  /// ghosts[r] for every rank r.  Throws "Ghosts must be sorted" and "Ghost
  /// index in local range" as the reference does.
  L2GMap(const Comm& comm, const std::vector<std::int64_t>& local_size,
         const std::vector<std::vector<std::int64_t>>& ghosts) {
    std::vector<const std::int64_t*> gp(ghosts.size());
    std::vector<std::int64_t> ng(ghosts.size());
    for (size_t r = 0; r < ghosts.size(); ++r) {
      gp[r] = ghosts[r].data();
      ng[r] = std::int64_t(ghosts[r].size());
    }
    if (int(local_size.size()) != comm.size() || int(ghosts.size()) != comm.size())
      throw std::runtime_error("spmv::L2GMap - Error: need one entry per rank");
    detail::check(spmv_l2gmap_create(comm.handle(), local_size.data(), gp.data(),
                                     ng.data(), &h_));
  }
  /// Takes ownership of a map handle (as returned by spmv_petsc_read_matrix).
  explicit L2GMap(spmv_l2gmap adopted) : h_(adopted) {}
  ~L2GMap() { spmv_l2gmap_destroy(h_); }
  L2GMap(const L2GMap&) = delete;             // as L2GMap.h:36-37
  L2GMap& operator=(const L2GMap&) = delete;

  std::int32_t local_size(int rank) const {
    std::int32_t v = 0;
    detail::check(spmv_l2gmap_local_size(h_, rank, &v));
    return v;
  }
  std::int32_t num_ghosts(int rank) const {
    std::int32_t v = 0;
    detail::check(spmv_l2gmap_num_ghosts(h_, rank, &v));
    return v;
  }
  std::int64_t global_size() const {
    std::int64_t v = 0;
    detail::check(spmv_l2gmap_global_size(h_, &v));
    return v;
  }
  std::int64_t global_offset(int rank) const {
    std::int64_t v = 0;
    detail::check(spmv_l2gmap_global_offset(h_, rank, &v));
    return v;
  }
  std::int32_t global_to_local(int rank, std::int64_t i) const {
    std::int32_t v = 0;
    detail::check(spmv_l2gmap_global_to_local(h_, rank, i, &v));
    return v;
  }
  std::vector<std::int64_t> ghosts(int rank) const {
    const std::int64_t* p = nullptr;
    std::int32_t n = 0;
    detail::check(spmv_l2gmap_ghosts(h_, rank, &p, &n));
    return std::vector<std::int64_t>(p, p + n);
  }

  /// L2GMap::update (L2GMap.cpp:126-150) on every rank's vector (host
  /// pointers, each local_size + num_ghosts long), in place.
  template <typename T>
  void update(const std::vector<T*>& vecs) const {
    halo<T>(vecs, SPMV_MEMORY_HOST, false);
  }
  /// L2GMap::reverse_update (L2GMap.cpp:152-170), in place.
  template <typename T>
  void reverse_update(const std::vector<T*>& vecs) const {
    halo<T>(vecs, SPMV_MEMORY_HOST, true);
  }
  /// Device-pointer forms (ordered on the communicator's stream).
  template <typename T>
  void update_device(const std::vector<T*>& vecs) const {
    halo<T>(vecs, SPMV_MEMORY_DEVICE, false);
  }
  template <typename T>
  void reverse_update_device(const std::vector<T*>& vecs) const {
    halo<T>(vecs, SPMV_MEMORY_DEVICE, true);
  }

  spmv_l2gmap handle() const { return h_; }

 private:
  template <typename T>
  void halo(const std::vector<T*>& vecs, spmv_memory mem, bool rev) const {
    std::vector<void*> v(vecs.begin(), vecs.end());
    const spmv_dtype dt = detail::dtype_of<T>();
    detail::check(rev ? spmv_l2gmap_reverse_update(h_, dt, mem, v.data())
                      : spmv_l2gmap_update(h_, dt, mem, v.data()));
  }
  spmv_l2gmap h_ = nullptr;
};

/// One rank's local CSR block (0-based, int32 indices).
template <typename T>
struct CsrBlock {
  std::vector<std::int32_t> rowptr;
  std::vector<std::int32_t> colind;
  std::vector<T> values;
};

/// Distributed matrix (Matrix.h:23-81): rank r's block has columns numbered
/// by col_map (owned, then ghosts) and rows by row_map.
template <typename T>
class Matrix {
 public:
  Matrix(const Comm& comm, const std::vector<CsrBlock<T>>& blocks,
         std::shared_ptr<L2GMap> col_map, std::shared_ptr<L2GMap> row_map)
      : col_map_(std::move(col_map)), row_map_(std::move(row_map)) {
    const int P = comm.size();
    if (int(blocks.size()) != P)
      throw std::runtime_error("spmv::Matrix - Error: need one block per rank");
    std::vector<std::int32_t> nr(P), nc(P);
    std::vector<const std::int32_t*> rp(P), ci(P);
    std::vector<const void*> va(P);
    for (int r = 0; r < P; ++r) {
      nr[r] = std::int32_t(blocks[r].rowptr.size()) - 1;
      nc[r] = col_map_->local_size(r) + col_map_->num_ghosts(r);
      rp[r] = blocks[r].rowptr.data();
      ci[r] = blocks[r].colind.data();
      va[r] = blocks[r].values.data();
    }
    detail::check(spmv_matrix_create_csr(
        comm.handle(), detail::dtype_of<T>(), col_map_->handle(),
        row_map_ ? row_map_->handle() : nullptr, nr.data(), nc.data(), rp.data(),
        ci.data(), va.data(), &h_));
    nrows_ = nr;
    ncols_ = nc;
  }
  /// Takes ownership of a matrix handle and its maps (as returned by
  /// spmv_petsc_read_matrix) for a communicator of `size` ranks.
  Matrix(spmv_matrix adopted, std::shared_ptr<L2GMap> col_map,
         std::shared_ptr<L2GMap> row_map, int size)
      : h_(adopted), col_map_(std::move(col_map)), row_map_(std::move(row_map)) {
    for (int r = 0; r < size; ++r) {
      nrows_.push_back(row_map_->local_size(r));
      ncols_.push_back(col_map_->local_size(r) + col_map_->num_ghosts(r));
    }
  }
  ~Matrix() { spmv_matrix_destroy(h_); }

  /// Matrix::create_matrix (Matrix.cpp:213-438) for every rank: blocks[r]
  /// holds nrows_local[r] owned rows then one row per row_ghosts[r] entry,
  /// columns owned first then col_ghosts[r]; ghost rows are summed into
  /// their owners and the column maps grow by the columns they bring.
  static Matrix create_matrix(const Comm& comm, const std::vector<CsrBlock<T>>& blocks,
                              const std::vector<std::int64_t>& nrows_local,
                              const std::vector<std::int64_t>& ncols_local,
                              const std::vector<std::vector<std::int64_t>>& row_ghosts,
                              const std::vector<std::vector<std::int64_t>>& col_ghosts) {
    const int P = comm.size();
    if (int(blocks.size()) != P || int(nrows_local.size()) != P ||
        int(ncols_local.size()) != P || int(row_ghosts.size()) != P ||
        int(col_ghosts.size()) != P)
      throw std::runtime_error("spmv::Matrix::create_matrix - Error: need one entry per rank");
    std::vector<const std::int32_t*> rp(P), ci(P);
    std::vector<const void*> va(P);
    std::vector<const std::int64_t*> rg(P), cg(P);
    std::vector<std::int64_t> nrg(P), ncg(P);
    for (int r = 0; r < P; ++r) {
      rp[r] = blocks[r].rowptr.data();
      ci[r] = blocks[r].colind.data();
      va[r] = blocks[r].values.data();
      rg[r] = row_ghosts[r].data();
      cg[r] = col_ghosts[r].data();
      nrg[r] = std::int64_t(row_ghosts[r].size());
      ncg[r] = std::int64_t(col_ghosts[r].size());
    }
    spmv_l2gmap cm = nullptr, rm = nullptr;
    spmv_matrix A = nullptr;
    detail::check(spmv_matrix_create_assembled(
        comm.handle(), detail::dtype_of<T>(), nrows_local.data(), ncols_local.data(), rp.data(),
        ci.data(), va.data(), rg.data(), nrg.data(), cg.data(), ncg.data(), &cm, &rm, &A));
    return Matrix(A, std::make_shared<L2GMap>(cm), std::make_shared<L2GMap>(rm), P);
  }

  // Move-only: the reference's implicit copy duplicates its MKL handle.
  Matrix(const Matrix&) = delete;
  Matrix& operator=(const Matrix&) = delete;
  Matrix(Matrix&& o) noexcept
      : h_(o.h_), col_map_(std::move(o.col_map_)), row_map_(std::move(o.row_map_)),
        nrows_(std::move(o.nrows_)), ncols_(std::move(o.ncols_)) {
    o.h_ = nullptr;
  }

  /// Matrix::operator* (Matrix.cpp:158-166) for every rank; x[r] has
  /// ncols(r) entries (update() its ghosts first), the result nrows(r).
  std::vector<std::vector<T>> operator*(const std::vector<std::vector<T>>& x) const {
    return apply(x, false);
  }
  /// Matrix::transpmult (Matrix.cpp:168-176).
  std::vector<std::vector<T>> transpmult(const std::vector<std::vector<T>>& x) const {
    return apply(x, true);
  }

  std::shared_ptr<const L2GMap> row_map() const { return row_map_; }
  std::shared_ptr<const L2GMap> col_map() const { return col_map_; }
  std::int32_t rows(int rank) const { return nrows_[rank]; }
  std::int32_t cols(int rank) const { return ncols_[rank]; }
  spmv_matrix handle() const { return h_; }

 private:
  std::vector<std::vector<T>> apply(const std::vector<std::vector<T>>& x,
                                    bool trans) const {
    const size_t P = nrows_.size();
    std::vector<std::vector<T>> y(P);
    std::vector<const void*> xp(P);
    std::vector<void*> yp(P);
    for (size_t r = 0; r < P; ++r) {
      const size_t in = trans ? nrows_[r] : ncols_[r];
      if (x[r].size() != in)
        throw std::runtime_error("spmv::Matrix - Error: vector size mismatch");
      y[r].resize(trans ? ncols_[r] : nrows_[r]);
      xp[r] = x[r].data();
      yp[r] = y[r].data();
    }
    detail::check(trans ? spmv_matrix_transpmult(h_, SPMV_MEMORY_HOST, xp.data(), yp.data())
                        : spmv_matrix_mult(h_, SPMV_MEMORY_HOST, xp.data(), yp.data()));
    return y;
  }
  spmv_matrix h_ = nullptr;
  std::shared_ptr<L2GMap> col_map_, row_map_;
  std::vector<std::int32_t> nrows_, ncols_;
};

/// spmv::read_petsc_binary (read_petsc.h:18-24, read_petsc.cpp:32-191) for
/// every rank: a PETSc binary matrix file split by owner_ranges.  Throws
/// "Could not open file" and "Bad signature in PETSc Matrix file" as the
/// reference does.
inline Matrix<double> read_petsc_binary(const Comm& comm, const std::string& filename) {
  spmv_l2gmap cm = nullptr, rm = nullptr;
  spmv_matrix A = nullptr;
  detail::check(spmv_petsc_read_matrix(comm.handle(), filename.c_str(), &cm, &rm, &A));
  return Matrix<double>(A, std::make_shared<L2GMap>(cm), std::make_shared<L2GMap>(rm),
                        comm.size());
}

/// spmv::read_petsc_binary_vector (read_petsc.h:26-32, read_petsc.cpp:193-260):
/// every rank's owner_ranges block of a PETSc binary vector file.
inline std::vector<std::vector<double>> read_petsc_binary_vector(const Comm& comm,
                                                                 const std::string& filename) {
  std::int64_t n = 0;
  detail::check(spmv_petsc_vector_size(filename.c_str(), &n));
  std::vector<std::int64_t> rr(size_t(comm.size()) + 1);
  detail::check(spmv_owner_ranges(comm.size(), n, rr.data()));
  std::vector<std::vector<double>> v(size_t(comm.size()));
  std::vector<double*> vp(size_t(comm.size()));
  for (int r = 0; r < comm.size(); ++r) {
    v[r].resize(size_t(rr[r + 1] - rr[r]));
    vp[r] = v[r].data();
  }
  detail::check(spmv_petsc_read_vector(comm.handle(), filename.c_str(), vp.data()));
  return v;
}

/// spmv::cg (cg.h:27-29, cg.cpp:11-83) on every rank: returns x (each
/// col_map local_size + num_ghosts long, ghost tail zero) and the iteration
/// count.  Throws "spmv::cg - Error: A.row_map() has ghost entries" and
/// "spmv::cg - Error: b.rows() != A.rows()" as the reference does.
inline std::tuple<std::vector<std::vector<double>>, int> cg(
    const Comm& comm, const Matrix<double>& A,
    const std::vector<std::vector<double>>& b, int max_its, double rtol) {
  const int P = comm.size();
  std::vector<const double*> bp(P);
  std::vector<std::int64_t> rows(P);
  std::vector<std::vector<double>> x(P);
  std::vector<double*> xp(P);
  for (int r = 0; r < P; ++r) {
    bp[r] = b[r].data();
    rows[r] = std::int64_t(b[r].size());
    x[r].assign(size_t(A.col_map()->local_size(r) + A.col_map()->num_ghosts(r)), 0.0);
    xp[r] = x[r].data();
  }
  int its = 0;
  detail::check(spmv_cg(A.handle(), SPMV_MEMORY_HOST, bp.data(), rows.data(),
                        xp.data(), max_its, rtol, &its));
  return std::make_tuple(std::move(x), its);
}

}  // namespace spmv
