// Matrix::create_matrix (Matrix.cpp:213-438) on the device: the assembly of
// rank blocks that carry ghost rows, for communicators with a GPU.  The
// semantics are those of assemble.cpp (and of the reference):
//  * a ghost row goes to the rank whose row range holds it; each receiving
//    rank sees the ghost rows in ascending sender order, each sender's rows in
//    its ghost-row order (the reference's neighbourhood alltoallv over its
//    sorted source list, Matrix.cpp:254-340);
//  * the receiver's new ghost columns are its old ones plus every received
//    column outside its range, ascending (Matrix.cpp:342-367);
//  * the block is built from triplets -- own rows in storage order, then the
//    received rows in arrival order -- as Eigen's setFromTriplets does
//    (Matrix.cpp:369-428): entries with the same (row, column) summed in
//    triplet order, each row in ascending column order.
//
// Device steps (one pass over all ranks at once):
//  1. the host computes, per input row (owned or ghost), its destination
//     rank, destination row and the position of its first entry in the
//     destination's triplet list (row-level work: the routing order);
//  2. a kernel writes every entry as a triplet at that position: global
//     column, destination row key, value (the triplet arrays are thus in
//     the reference's triplet order);
//  3. the new ghost columns: (rank, global column) keys of the old ghosts and
//     of every triplet column outside its rank's range, radix-sorted and
//     made unique;
//  4. each triplet's local column (owned: column - range start; else the
//     owned count + its position among the rank's ghosts, by binary search);
//  5. a stable radix sort of the triplets by (global row, local column)
//     (radix sorting is stable, so equal keys keep triplet order);
//  6. one thread per run of equal keys sums the run's values left to right
//     -- the order of setFromTriplets, so the result is bitwise the host
//     assembly's -- and the rows' entry counts give the row pointers.
// The blocks and ghost lists are then read back (Matrix keeps a host copy of
// its CSR, Matrix::mat()) and the maps and matrix are created from them.
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <numeric>
#include <string>

#include "internal.h"

namespace spmvb {

namespace {

template <typename F>
struct DCplx {
  F re, im;
};
template <typename T>
__device__ __forceinline__ T add_in_order(const T& a, const T& b) {
  return a + b;
}
template <typename F>
__device__ __forceinline__ DCplx<F> add_in_order(const DCplx<F>& a, const DCplx<F>& b) {
  return DCplx<F>{a.re + b.re, a.im + b.im};
}

// Per input row (all ranks, owned rows then ghost rows of each rank).
struct RowRoute {
  int64_t first;   // position of the row's first entry in the triplet arrays
  int64_t grow;    // destination global row
  int32_t rank;    // source rank
  int32_t dest;    // destination rank
};

struct RankInfo {
  int64_t cr0, cr1;      // destination column range
  int64_t col_ghost0;    // first old ghost of the source rank in the ghost array
  int64_t ncols_local;   // source rank's owned columns
  int64_t n_col_ghosts;  // source rank's old ghost count
  int64_t src_nz0;       // first input entry of the rank (concatenated)
  int64_t src_row0;      // first input row of the rank (concatenated row pointers)
};

constexpr int MAXP = SPMV_MAX_PARTS;

struct AsmArgs {
  RankInfo rk[MAXP];
};

// 2. Entries -> triplets at their routed positions.
template <typename T>
__global__ void scatter_triplets(const __grid_constant__ AsmArgs A, const RowRoute* routes,
                                 int64_t nrows_in, const int32_t* rowptr_cat,
                                 const int32_t* colind_cat, const T* vals_cat,
                                 const int64_t* old_ghosts, int64_t* tcol, uint64_t* trow,
                                 T* tval, int* err) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nrows_in;
       i += int64_t(gridDim.x) * blockDim.x) {
    const RowRoute R = routes[i];
    const RankInfo& S = A.rk[R.rank];
    const int64_t lrow = i - S.src_row0;  // row within the source rank
    const int32_t* rp = rowptr_cat + S.src_row0 + R.rank;  // rank r's pointers start here
    const int64_t b = rp[lrow], e = rp[lrow + 1];
    for (int64_t j = b; j < e; ++j) {
      const int32_t c = colind_cat[S.src_nz0 + j];
      int64_t g = 0;
      if (c >= 0 && c < S.ncols_local) {
        g = S.cr0 + c;
      } else if (c >= S.ncols_local && c < S.ncols_local + S.n_col_ghosts) {
        g = old_ghosts[S.col_ghost0 + (c - S.ncols_local)];
      } else {
        atomicExch(err, 1);
        g = 0;
      }
      const int64_t t = R.first + (j - b);
      tcol[t] = g;
      trow[t] = uint64_t(R.grow);
      tval[t] = vals_cat[S.src_nz0 + j];
    }
  }
}

// 3. Ghost candidates: (rank, global column) of triplet columns outside the
// destination's range (others get an all-ones key, sorted last and dropped).
__global__ void ghost_candidates(const __grid_constant__ AsmArgs A, const int64_t* tcol,
                                 const uint64_t* trow, const int32_t* tdest, int64_t n,
                                 uint64_t* keys) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int q = tdest[t];
    const int64_t g = tcol[t];
    const bool out = g < A.rk[q].cr0 || g >= A.rk[q].cr1;
    keys[t] = out ? (uint64_t(q) << 56) | uint64_t(g) : ~uint64_t(0);
  }
}

// Destination rank of each triplet (from the row routes).
__global__ void triplet_dest(const RowRoute* routes, int64_t nrows_in, const int32_t* rowptr_cat,
                             const __grid_constant__ AsmArgs A, int32_t* tdest) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < nrows_in;
       i += int64_t(gridDim.x) * blockDim.x) {
    const RowRoute R = routes[i];
    const RankInfo& S = A.rk[R.rank];
    const int32_t* rp = rowptr_cat + S.src_row0 + R.rank;
    const int64_t lrow = i - S.src_row0;
    const int64_t len = rp[lrow + 1] - rp[lrow];
    for (int64_t k = 0; k < len; ++k) tdest[R.first + k] = R.dest;
  }
}

// 4. Local columns and the sort keys (global row, local column).
__global__ void local_columns(const __grid_constant__ AsmArgs A, const int64_t* tcol,
                              const uint64_t* trow, const int32_t* tdest, int64_t n,
                              const uint64_t* ghost_keys, const int64_t* ghost_begin,
                              const int64_t* ncols_local_dest, uint64_t* sort_key,
                              int32_t* idx) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n;
       t += int64_t(gridDim.x) * blockDim.x) {
    const int q = tdest[t];
    const int64_t g = tcol[t];
    int64_t lc;
    if (g >= A.rk[q].cr0 && g < A.rk[q].cr1) {
      lc = g - A.rk[q].cr0;
    } else {
      // lower_bound among rank q's ghost keys
      const uint64_t key = (uint64_t(q) << 56) | uint64_t(g);
      int64_t lo = ghost_begin[q], hi = ghost_begin[q + 1];
      while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (ghost_keys[mid] < key)
          lo = mid + 1;
        else
          hi = mid;
      }
      lc = ncols_local_dest[q] + (lo - ghost_begin[q]);
    }
    sort_key[t] = (trow[t] << 32) | uint64_t(lc);
    idx[t] = int32_t(t);
  }
}

// 6a. Run starts of the sorted keys (flag = 1 where a new (row, col) begins).
__global__ void run_flags(const uint64_t* keys, int64_t n, int32_t* flags) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n;
       t += int64_t(gridDim.x) * blockDim.x)
    flags[t] = (t == 0 || keys[t] != keys[t - 1]) ? 1 : 0;
}

// 6b. One thread per run: the sum of its values in triplet order, its local
// column, and one more entry for its global row.
template <typename T>
__global__ void run_sums(const uint64_t* keys, const int32_t* perm, const T* tval, int64_t n,
                         const int32_t* flags, const int64_t* run_id, T* out_val,
                         int32_t* out_col, int32_t* row_count, int64_t row_base) {
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < n;
       t += int64_t(gridDim.x) * blockDim.x) {
    if (!flags[t]) continue;
    const uint64_t k = keys[t];
    T sum = tval[perm[t]];
    for (int64_t e = t + 1; e < n && keys[e] == k; ++e) sum = add_in_order(sum, tval[perm[e]]);
    const int64_t r = run_id[t];
    out_val[r] = sum;
    out_col[r] = int32_t(k & 0xffffffffull);
    atomicAdd(row_count + (int64_t(k >> 32) - row_base), 1);
  }
}

int grid_of(int64_t n, int num_sms) {
  const int64_t g = (n + 255) / 256;
  return int(std::max<int64_t>(1, std::min<int64_t>(g, int64_t(num_sms) * 16)));
}

template <typename T>
struct DevBlocks {
  std::vector<std::vector<int32_t>> rowptr, colind;
  std::vector<std::vector<T>> vals;
  std::vector<std::vector<int64_t>> ghosts;
};

// Stage times of the assembly, logged under SPMV_B200_DEBUG.
struct StageClock {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  void operator()(const char* what) {
    const auto t = std::chrono::steady_clock::now();
    debug_log(std::string("create_matrix: ") + what + " " +
              std::to_string(std::chrono::duration<double, std::milli>(t - t0).count()) + " ms");
    t0 = t;
  }
};

template <typename T>
void assemble_device(spmv_comm comm, const int64_t* nrows_local, const int64_t* ncols_local,
                     const int32_t* const* rowptr, const int32_t* const* colind,
                     const void* const* values, const int64_t* const* row_ghosts,
                     const int64_t* n_row_ghosts, const int64_t* const* col_ghosts,
                     const int64_t* n_col_ghosts, DevBlocks<T>& out) {
  const int P = comm->size;
  require(P <= MAXP, "spmv::Matrix::create_matrix - Error: too many ranks");
  cudaStream_t s = comm->stream;
  DeviceGuard dg(comm->device);
  StageClock dbg_stage;
  std::vector<int64_t> rr(size_t(P) + 1, 0), cr(size_t(P) + 1, 0);
  for (int r = 0; r < P; ++r) {
    require(nrows_local[r] >= 0 && ncols_local[r] >= 0 && n_row_ghosts[r] >= 0 &&
                n_col_ghosts[r] >= 0,
            "spmv::Matrix::create_matrix - Error: negative size");
    rr[r + 1] = rr[r] + nrows_local[r];
    cr[r + 1] = cr[r] + ncols_local[r];
  }
  require(rr[P] < (int64_t(1) << 32) && cr[P] < (int64_t(1) << 56),
          "spmv::Matrix::create_matrix - Error: global size too large");
  // 1. Row routes, on the host (row-level work): destinations, arrival order.
  AsmArgs A{};
  int64_t nrows_in = 0, nnz_in = 0, nghost_old = 0;
  std::vector<int64_t> rows_in(P), nz_in(P);
  for (int r = 0; r < P; ++r) {
    rows_in[r] = nrows_local[r] + n_row_ghosts[r];
    nz_in[r] = rows_in[r] > 0 ? rowptr[r][rows_in[r]] : 0;
    require(rows_in[r] == 0 || rowptr[r][0] == 0,
            "spmv::Matrix::create_matrix - Error: row pointers must start at 0");
    RankInfo& I = A.rk[r];
    I.cr0 = cr[r];
    I.cr1 = cr[r + 1];
    I.ncols_local = ncols_local[r];
    I.n_col_ghosts = n_col_ghosts[r];
    I.col_ghost0 = nghost_old;
    I.src_nz0 = nnz_in;
    I.src_row0 = nrows_in;
    nrows_in += rows_in[r];
    nnz_in += nz_in[r];
    nghost_old += n_col_ghosts[r];
  }
  for (int r = 0; r < P; ++r)
    for (int64_t i = 0; i < n_col_ghosts[r]; ++i)
      require(col_ghosts[r][i] >= 0 && col_ghosts[r][i] < cr[P],
              "spmv::Matrix::create_matrix - Error: ghost column out of range");
  std::vector<std::vector<std::pair<int, int64_t>>> inbox(P);
  for (int r = 0; r < P; ++r)
    for (int64_t i = 0; i < n_row_ghosts[r]; ++i) {
      const int64_t g = row_ghosts[r][i];
      require(g >= 0 && g < rr[P], "spmv::Matrix::create_matrix - Error: ghost row out of range");
      const int owner = int(std::upper_bound(rr.begin(), rr.end(), g) - rr.begin()) - 1;
      require(owner != r, "spmv::Matrix::create_matrix - Error: ghost row owned by its own rank");
      inbox[owner].push_back({r, i});
    }
  std::vector<RowRoute> routes(size_t(std::max<int64_t>(nrows_in, 1)));
  std::vector<int64_t> tri0(size_t(P) + 1, 0);  // first triplet of each destination
  int64_t pos = 0;
  for (int q = 0; q < P; ++q) {
    tri0[q] = pos;
    const int64_t base = A.rk[q].src_row0;
    for (int64_t row = 0; row < nrows_local[q]; ++row) {
      RowRoute& R = routes[base + row];
      R.first = pos;
      R.grow = rr[q] + row;
      R.rank = q;
      R.dest = q;
      const int64_t len = int64_t(rowptr[q][row + 1]) - rowptr[q][row];
      require(len >= 0, "spmv: row pointers must be non-decreasing");
      pos += len;
    }
    for (const auto& m : inbox[q]) {
      const int r = m.first;
      const int64_t row = nrows_local[r] + m.second;
      RowRoute& R = routes[A.rk[r].src_row0 + row];
      R.first = pos;
      R.grow = row_ghosts[r][m.second];
      R.rank = r;
      R.dest = q;
      const int64_t len = int64_t(rowptr[r][row + 1]) - rowptr[r][row];
      require(len >= 0, "spmv: row pointers must be non-decreasing");
      pos += len;
    }
  }
  tri0[P] = pos;
  const int64_t n = pos;
  require(n == nnz_in, "spmv::Matrix::create_matrix - Error: inconsistent row pointers");
  // Uploads: each rank's arrays straight into their place in the
  // concatenated device arrays (rank r's row pointers start at src_row0 + r:
  // each rank keeps its own n + 1 pointers).
  DevBuf d_routes, d_rp, d_ci, d_va, d_og, d_tcol, d_trow, d_tval, d_tdest, d_gkeys, d_gsorted,
      d_skey, d_skey2, d_idx, d_idx2, d_flags, d_runid, d_oval, d_ocol, d_rcount, d_gbeg, d_ncl,
      d_err, d_tmp;
  auto up = [&](DevBuf& b, const void* src, size_t bytes) {
    b.reserve(std::max<size_t>(bytes, 16));
    if (bytes) SPMVB_CUDA(cudaMemcpyAsync(b.ptr, src, bytes, cudaMemcpyHostToDevice, s));
  };
  up(d_routes, routes.data(), sizeof(RowRoute) * size_t(nrows_in));
  d_rp.reserve(sizeof(int32_t) * size_t(nrows_in + P));
  d_ci.reserve(sizeof(int32_t) * size_t(std::max<int64_t>(nnz_in, 1)));
  d_va.reserve(sizeof(T) * size_t(std::max<int64_t>(nnz_in, 1)));
  d_og.reserve(sizeof(int64_t) * size_t(std::max<int64_t>(nghost_old, 1)));
  const int32_t zero_ptr = 0;
  for (int r = 0; r < P; ++r) {
    const RankInfo& I = A.rk[r];
    int32_t* rpd = d_rp.as<int32_t>() + I.src_row0 + r;
    if (rows_in[r] > 0) {
      SPMVB_CUDA(cudaMemcpyAsync(rpd, rowptr[r], sizeof(int32_t) * size_t(rows_in[r] + 1),
                                 cudaMemcpyHostToDevice, s));
    } else {
      SPMVB_CUDA(cudaMemcpyAsync(rpd, &zero_ptr, sizeof(int32_t), cudaMemcpyHostToDevice, s));
    }
    if (nz_in[r] > 0) {
      require(colind[r] && values[r], "spmv::Matrix::create_matrix - Error: NULL argument");
      SPMVB_CUDA(cudaMemcpyAsync(d_ci.as<int32_t>() + I.src_nz0, colind[r],
                                 sizeof(int32_t) * size_t(nz_in[r]), cudaMemcpyHostToDevice, s));
      SPMVB_CUDA(cudaMemcpyAsync(d_va.as<T>() + I.src_nz0, values[r], sizeof(T) * size_t(nz_in[r]),
                                 cudaMemcpyHostToDevice, s));
    }
    if (n_col_ghosts[r] > 0)
      SPMVB_CUDA(cudaMemcpyAsync(d_og.as<int64_t>() + I.col_ghost0, col_ghosts[r],
                                 sizeof(int64_t) * size_t(n_col_ghosts[r]), cudaMemcpyHostToDevice,
                                 s));
  }
  d_err.reserve(sizeof(int));
  SPMVB_CUDA(cudaMemsetAsync(d_err.ptr, 0, sizeof(int), s));
  const size_t N = size_t(std::max<int64_t>(n, 1));
  d_tcol.reserve(sizeof(int64_t) * N);
  d_trow.reserve(sizeof(uint64_t) * N);
  d_tval.reserve(sizeof(T) * N);
  d_tdest.reserve(sizeof(int32_t) * N);
  const int sms = std::max(1, comm->num_sms);
  // 2. Triplets.
  if (nrows_in > 0) {
    scatter_triplets<T><<<grid_of(nrows_in, sms), 256, 0, s>>>(
        A, d_routes.as<RowRoute>(), nrows_in, d_rp.as<int32_t>(), d_ci.as<int32_t>(),
        d_va.as<T>(), d_og.as<int64_t>(), d_tcol.as<int64_t>(), d_trow.as<uint64_t>(),
        d_tval.as<T>(), d_err.as<int>());
    triplet_dest<<<grid_of(nrows_in, sms), 256, 0, s>>>(d_routes.as<RowRoute>(), nrows_in,
                                                        d_rp.as<int32_t>(), A,
                                                        d_tdest.as<int32_t>());
    SPMVB_CUDA(cudaGetLastError());
  }
  int herr = 0;
  SPMVB_CUDA(cudaMemcpyAsync(&herr, d_err.ptr, sizeof(int), cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
  require(herr == 0, "spmv::Matrix::create_matrix - Error: column index outside the block");
  dbg_stage("routes, uploads, triplets");
  // 3. New ghost columns: old ghosts + outside columns, sorted and unique.
  const int64_t nk = n + nghost_old;
  const size_t NK = size_t(std::max<int64_t>(nk, 1));
  d_gkeys.reserve(sizeof(uint64_t) * NK);
  d_gsorted.reserve(sizeof(uint64_t) * NK);
  if (n > 0)
    ghost_candidates<<<grid_of(n, sms), 256, 0, s>>>(A, d_tcol.as<int64_t>(),
                                                     d_trow.as<uint64_t>(),
                                                     d_tdest.as<int32_t>(), n,
                                                     d_gkeys.as<uint64_t>());
  {
    std::vector<uint64_t> ok;
    ok.reserve(size_t(nghost_old));
    for (int r = 0; r < P; ++r)
      for (int64_t i = 0; i < n_col_ghosts[r]; ++i)
        ok.push_back((uint64_t(r) << 56) | uint64_t(col_ghosts[r][i]));
    if (!ok.empty())
      SPMVB_CUDA(cudaMemcpyAsync(d_gkeys.as<uint64_t>() + n, ok.data(), sizeof(uint64_t) * ok.size(),
                                 cudaMemcpyHostToDevice, s));
    size_t tb = 0;
    SPMVB_CUDA(cub::DeviceRadixSort::SortKeys(nullptr, tb, d_gkeys.as<uint64_t>(),
                                              d_gsorted.as<uint64_t>(), nk, 0, 64, s));
    d_tmp.reserve(std::max<size_t>(tb, 16));
    if (nk > 0)
      SPMVB_CUDA(cub::DeviceRadixSort::SortKeys(d_tmp.ptr, tb, d_gkeys.as<uint64_t>(),
                                                d_gsorted.as<uint64_t>(), nk, 0, 64, s));
    // The rank's ghosts are small next to the entries: unique them on the
    // host from the sorted keys (one read-back), which also gives the lists
    // the column maps are built from.
    std::vector<uint64_t> sorted(NK);
    if (nk > 0)
      SPMVB_CUDA(cudaMemcpyAsync(sorted.data(), d_gsorted.ptr, sizeof(uint64_t) * nk,
                                 cudaMemcpyDeviceToHost, s));
    SPMVB_CUDA(cudaStreamSynchronize(s));
    std::vector<uint64_t> uniq;
    for (int64_t i = 0; i < nk; ++i) {
      if (sorted[i] == ~uint64_t(0)) break;
      if (uniq.empty() || uniq.back() != sorted[i]) uniq.push_back(sorted[i]);
    }
    out.ghosts.assign(P, {});
    std::vector<int64_t> gbeg(size_t(P) + 1, 0), ncl(P);
    for (size_t i = 0; i < uniq.size(); ++i) {
      const int q = int(uniq[i] >> 56);
      out.ghosts[q].push_back(int64_t(uniq[i] & ((uint64_t(1) << 56) - 1)));
      gbeg[q + 1] += 1;
    }
    for (int q = 0; q < P; ++q) {
      gbeg[q + 1] += gbeg[q];
      ncl[q] = ncols_local[q];
      require(ncols_local[q] + int64_t(out.ghosts[q].size()) < (int64_t(1) << 31),
              "spmv::Matrix::create_matrix - Error: block too wide for int32 indices");
    }
    up(d_gsorted, uniq.data(), sizeof(uint64_t) * uniq.size());
    up(d_gbeg, gbeg.data(), sizeof(int64_t) * gbeg.size());
    up(d_ncl, ncl.data(), sizeof(int64_t) * ncl.size());
  }
  dbg_stage("ghost columns");
  // 4-5. Local columns, then the stable sort by (global row, local column).
  d_skey.reserve(sizeof(uint64_t) * N);
  d_skey2.reserve(sizeof(uint64_t) * N);
  d_idx.reserve(sizeof(int32_t) * N);
  d_idx2.reserve(sizeof(int32_t) * N);
  require(n < (int64_t(1) << 31), "spmv::Matrix::create_matrix - Error: too many entries");
  if (n > 0) {
    local_columns<<<grid_of(n, sms), 256, 0, s>>>(
        A, d_tcol.as<int64_t>(), d_trow.as<uint64_t>(), d_tdest.as<int32_t>(), n,
        d_gsorted.as<uint64_t>(), d_gbeg.as<int64_t>(), d_ncl.as<int64_t>(),
        d_skey.as<uint64_t>(), d_idx.as<int32_t>());
    size_t tb = 0;
    SPMVB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, d_skey.as<uint64_t>(),
                                               d_skey2.as<uint64_t>(), d_idx.as<int32_t>(),
                                               d_idx2.as<int32_t>(), n, 0, 64, s));
    d_tmp.reserve(std::max<size_t>(tb, 16));
    SPMVB_CUDA(cub::DeviceRadixSort::SortPairs(d_tmp.ptr, tb, d_skey.as<uint64_t>(),
                                               d_skey2.as<uint64_t>(), d_idx.as<int32_t>(),
                                               d_idx2.as<int32_t>(), n, 0, 64, s));
  }
  // 6. Runs: flags, run ids (exclusive scan), ordered sums, row counts.
  d_flags.reserve(sizeof(int32_t) * N);
  d_runid.reserve(sizeof(int64_t) * N);
  const int64_t nrows_out = rr[P];
  d_rcount.reserve(sizeof(int32_t) * size_t(std::max<int64_t>(nrows_out, 1)));
  SPMVB_CUDA(cudaMemsetAsync(d_rcount.ptr, 0, sizeof(int32_t) * size_t(std::max<int64_t>(nrows_out, 1)), s));
  int64_t nruns = 0;
  if (n > 0) {
    run_flags<<<grid_of(n, sms), 256, 0, s>>>(d_skey2.as<uint64_t>(), n, d_flags.as<int32_t>());
    size_t tb = 0;
    SPMVB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, d_flags.as<int32_t>(),
                                             d_runid.as<int64_t>(), n, s));
    d_tmp.reserve(std::max<size_t>(tb, 16));
    SPMVB_CUDA(cub::DeviceScan::ExclusiveSum(d_tmp.ptr, tb, d_flags.as<int32_t>(),
                                             d_runid.as<int64_t>(), n, s));
    int64_t last_id = 0;
    int32_t last_flag = 0;
    SPMVB_CUDA(cudaMemcpyAsync(&last_id, d_runid.as<int64_t>() + (n - 1), sizeof(int64_t),
                               cudaMemcpyDeviceToHost, s));
    SPMVB_CUDA(cudaMemcpyAsync(&last_flag, d_flags.as<int32_t>() + (n - 1), sizeof(int32_t),
                               cudaMemcpyDeviceToHost, s));
    SPMVB_CUDA(cudaStreamSynchronize(s));
    nruns = last_id + last_flag;
    d_oval.reserve(sizeof(T) * size_t(std::max<int64_t>(nruns, 1)));
    d_ocol.reserve(sizeof(int32_t) * size_t(std::max<int64_t>(nruns, 1)));
    run_sums<T><<<grid_of(n, sms), 256, 0, s>>>(
        d_skey2.as<uint64_t>(), d_idx2.as<int32_t>(), d_tval.as<T>(), n, d_flags.as<int32_t>(),
        d_runid.as<int64_t>(), d_oval.as<T>(), d_ocol.as<int32_t>(), d_rcount.as<int32_t>(), 0);
    SPMVB_CUDA(cudaGetLastError());
  }
  // Read back and split per rank (the runs are in global row order).
  std::vector<int32_t> rc(size_t(std::max<int64_t>(nrows_out, 1)), 0);
  std::vector<int32_t> oc(size_t(std::max<int64_t>(nruns, 1)));
  std::vector<T> ov(size_t(std::max<int64_t>(nruns, 1)));
  if (nrows_out > 0)
    SPMVB_CUDA(cudaMemcpyAsync(rc.data(), d_rcount.ptr, sizeof(int32_t) * size_t(nrows_out),
                               cudaMemcpyDeviceToHost, s));
  if (nruns > 0) {
    SPMVB_CUDA(cudaMemcpyAsync(oc.data(), d_ocol.ptr, sizeof(int32_t) * size_t(nruns),
                               cudaMemcpyDeviceToHost, s));
    SPMVB_CUDA(cudaMemcpyAsync(ov.data(), d_oval.ptr, sizeof(T) * size_t(nruns),
                               cudaMemcpyDeviceToHost, s));
  }
  SPMVB_CUDA(cudaStreamSynchronize(s));
  dbg_stage("sort, sums, read-back");
  out.rowptr.assign(P, {});
  out.colind.assign(P, {});
  out.vals.assign(P, {});
  int64_t e = 0;
  for (int q = 0; q < P; ++q) {
    std::vector<int32_t>& rp = out.rowptr[q];
    rp.assign(size_t(nrows_local[q]) + 1, 0);
    for (int64_t i = 0; i < nrows_local[q]; ++i) rp[i + 1] = rp[i] + rc[rr[q] + i];
    const int64_t m = rp[nrows_local[q]];
    out.colind[q].assign(oc.begin() + e, oc.begin() + e + m);
    out.vals[q].assign(ov.begin() + e, ov.begin() + e + m);
    e += m;
  }
}

template <typename T>
void create_on_device(spmv_comm comm, spmv_dtype dtype, const int64_t* nrows_local,
                      const int64_t* ncols_local, const int32_t* const* rowptr,
                      const int32_t* const* colind, const void* const* values,
                      const int64_t* const* row_ghosts, const int64_t* n_row_ghosts,
                      const int64_t* const* col_ghosts, const int64_t* n_col_ghosts,
                      spmv_l2gmap* cm, spmv_l2gmap* rm, spmv_matrix* m) {
  const int P = comm->size;
  DevBlocks<T> B;
  assemble_device<T>(comm, nrows_local, ncols_local, rowptr, colind, values, row_ghosts,
                     n_row_ghosts, col_ghosts, n_col_ghosts, B);
  std::vector<int64_t> ng(P), zero(P, 0);
  std::vector<const int64_t*> gp(P), none(P, nullptr);
  std::vector<int32_t> nr(P), nc(P);
  std::vector<const int32_t*> rp(P), ci(P);
  std::vector<const void*> va(P);
  for (int r = 0; r < P; ++r) {
    ng[r] = int64_t(B.ghosts[r].size());
    gp[r] = B.ghosts[r].data();
    nr[r] = int32_t(nrows_local[r]);
    nc[r] = int32_t(ncols_local[r] + ng[r]);
    rp[r] = B.rowptr[r].data();
    ci[r] = B.colind[r].data();
    va[r] = B.vals[r].data();
  }
  auto check = [](int st) {
    if (st != SPMV_SUCCESS) fail(st, spmv_last_error());
  };
  StageClock clk;
  check(spmv_l2gmap_create(comm, ncols_local, gp.data(), ng.data(), cm));
  check(spmv_l2gmap_create(comm, nrows_local, none.data(), zero.data(), rm));
  clk("maps");
  check(spmv_matrix_create_csr(comm, dtype, *cm, *rm, nr.data(), nc.data(), rp.data(), ci.data(),
                               va.data(), m));
  clk("matrix");
}

}  // namespace

// Dispatch by value type (complex values as pairs of their real type).
void create_assembled_device(spmv_comm comm, spmv_dtype dtype, const int64_t* nrows_local,
                             const int64_t* ncols_local, const int32_t* const* rowptr,
                             const int32_t* const* colind, const void* const* values,
                             const int64_t* const* row_ghosts, const int64_t* n_row_ghosts,
                             const int64_t* const* col_ghosts, const int64_t* n_col_ghosts,
                             spmv_l2gmap* cm, spmv_l2gmap* rm, spmv_matrix* m) {
  switch (dtype) {
    case SPMV_FLOAT64:
      create_on_device<double>(comm, dtype, nrows_local, ncols_local, rowptr, colind, values,
                               row_ghosts, n_row_ghosts, col_ghosts, n_col_ghosts, cm, rm, m);
      break;
    case SPMV_FLOAT32:
      create_on_device<float>(comm, dtype, nrows_local, ncols_local, rowptr, colind, values,
                              row_ghosts, n_row_ghosts, col_ghosts, n_col_ghosts, cm, rm, m);
      break;
    case SPMV_COMPLEX128:
      create_on_device<DCplx<double>>(comm, dtype, nrows_local, ncols_local, rowptr, colind,
                                      values, row_ghosts, n_row_ghosts, col_ghosts,
                                      n_col_ghosts, cm, rm, m);
      break;
    case SPMV_COMPLEX64:
      create_on_device<DCplx<float>>(comm, dtype, nrows_local, ncols_local, rowptr, colind,
                                     values, row_ghosts, n_row_ghosts, col_ghosts, n_col_ghosts,
                                     cm, rm, m);
      break;
    default:
      fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv::Matrix::create_matrix - Error: unknown dtype");
  }
}

}  // namespace spmvb
