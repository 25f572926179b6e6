// extern "C" entry points of libspmv_b200 (declared in include/spmv_b200.h).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <numeric>

#include "internal.h"

namespace spmvb {

namespace {
thread_local std::string g_last_error;
}

void set_last_error(const std::string& msg) { g_last_error = msg; }

void debug_log(const std::string& msg) {
  static const bool on = std::getenv("SPMV_B200_DEBUG") != nullptr;
  if (on) std::fprintf(stderr, "[spmv_b200] %s\n", msg.c_str());
}

void soft_check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return;
  (void)cudaGetLastError();
  debug_log(std::string(what) + " failed: " + cudaGetErrorString(e));
}

// Entering device work: an error left pending by an earlier call (of this
// library's runtime, in this thread) is cleared and logged here, so that the
// launch checks below only ever report errors of this call.
DeviceGuard::DeviceGuard(int dev) {
  if (dev < 0) return;
  const cudaError_t pending = cudaGetLastError();
  if (pending != cudaSuccess)
    debug_log(std::string("cleared a pending error: ") + cudaGetErrorString(pending));
  SPMVB_CUDA(cudaGetDevice(&prev));
  if (prev != dev) SPMVB_CUDA(cudaSetDevice(dev));
}
DeviceGuard::~DeviceGuard() {
  int cur = -1;
  if (prev < 0) return;
  soft_check(cudaGetDevice(&cur), "cudaGetDevice");
  if (cur >= 0 && cur != prev) soft_check(cudaSetDevice(prev), "cudaSetDevice");
}

namespace {

void check_comm(spmv_comm c) { require(c != nullptr, "spmv: communicator is NULL"); }
void check_map(spmv_l2gmap m) { require(m != nullptr, "spmv: L2GMap is NULL"); }
void check_mat(spmv_matrix A) { require(A != nullptr, "spmv: Matrix is NULL"); }
void check_rank(spmv_comm c, int r) {
  require(r >= 0 && r < c->size, "spmv: rank out of range");
}

inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// Per-rank device views of host vectors: copies host buffers into one staging
// allocation (each rank's slice 256-byte aligned) and back.
struct Staging {
  std::vector<int64_t> off;
  int64_t total = 0;
  void layout(const std::vector<int64_t>& lens, size_t es) {
    off.resize(lens.size());
    total = 0;
    for (size_t r = 0; r < lens.size(); ++r) {
      off[r] = total;
      total += align_up(int64_t(lens[r] * es), 256);
    }
  }
};

}  // namespace

void upload_csr(spmv_matrix A) {
  DevCsr& C = A->fwd;
  const int P = A->comm->size;
  const size_t es = dtype_size(A->dtype);
  C.parts.assign(P, DevPart{});
  int64_t rp = 0, nz = 0, rows = 0, nnz_all = 0;
  int64_t maxr = 0;
  for (int r = 0; r < P; ++r) {
    DevPart& D = C.parts[r];
    D.nrows = A->nrows[r];
    D.ncols = A->ncols[r];
    D.nnz = A->h_rowptr[r][D.nrows];
    D.rp_off = rp;
    D.nz_off = nz;
    rp += D.nrows + 1;
    nz = align_up(nz + D.nnz, 4);
    rows += D.nrows;
    nnz_all += D.nnz;
    for (int32_t i = 0; i < D.nrows; ++i)
      maxr = std::max<int64_t>(maxr, A->h_rowptr[r][i + 1] - A->h_rowptr[r][i]);
  }
  C.rp_total = rp;
  C.nz_total = nz + 4;  // room for the masked tail of the last 16-byte load
  C.mean_row = rows > 0 ? double(nnz_all) / double(rows) : 0.0;
  C.max_row = maxr;
  C.sell_padded = 0;
  for (int r = 0; r < P; ++r)
    C.sell_padded += sell_padded_size(A->h_rowptr[r], A->nrows[r], nullptr);
  if (A->comm->device < 0) return;
  DeviceGuard dg(A->comm->device);
  C.rowptr.reserve(sizeof(int32_t) * std::max<int64_t>(C.rp_total, 1));
  C.cols.reserve(sizeof(int32_t) * C.nz_total);
  C.vals.reserve(es * C.nz_total);
  SPMVB_CUDA(cudaMemset(C.cols.ptr, 0, sizeof(int32_t) * C.nz_total));
  SPMVB_CUDA(cudaMemset(C.vals.ptr, 0, es * C.nz_total));
  for (int r = 0; r < P; ++r) {
    const DevPart& D = C.parts[r];
    SPMVB_CUDA(cudaMemcpy(C.rowptr.as<int32_t>() + D.rp_off, A->h_rowptr[r].data(),
                          sizeof(int32_t) * (D.nrows + 1), cudaMemcpyHostToDevice));
    if (D.nnz == 0) continue;
    SPMVB_CUDA(cudaMemcpy(C.cols.as<int32_t>() + D.nz_off, A->h_colind[r].data(),
                          sizeof(int32_t) * D.nnz, cudaMemcpyHostToDevice));
    SPMVB_CUDA(cudaMemcpy(C.vals.as<char>() + D.nz_off * es, A->h_vals[r].data(),
                          es * D.nnz, cudaMemcpyHostToDevice));
  }
}

// Global column numbering for the fused-halo layout: an owned column c of
// rank r is col_range[r] + c, a ghost column is its global index.
void build_global_cols(spmv_matrix A) {
  DevCsr& C = A->fwd;
  if (C.cols_global.ptr) return;
  spmv_l2gmap cm = A->col_map;
  require(cm != nullptr, "spmv: matrix has no column map");
  require(cm->ranges.back() < (int64_t(1) << 31),
          "spmv: global size too large for 32-bit column indices");
  const int P = A->comm->size;
  std::vector<int32_t> g(C.nz_total, 0);
  // 16-bit offsets from the entry's global row (rows of rank r are numbered
  // from the sum of the earlier ranks' row counts, as in the launch tables).
  std::vector<int16_t> d(C.nz_total, 0);
  bool fits = d16_enabled();
  int64_t row0 = 0;
  for (int r = 0; r < P; ++r) {
    const DevPart& D = C.parts[r];
    const int64_t ls = cm->rank[r].local_size;
    const auto& gh = cm->rank[r].ghosts;
    const auto& rp = A->h_rowptr[r];
    for (int32_t i = 0; i < D.nrows; ++i) {
      for (int32_t j = rp[i]; j < rp[i + 1]; ++j) {
        const int32_t c = A->h_colind[r][j];
        const int64_t cg = c < ls ? cm->ranges[r] + c : gh[size_t(c - ls)];
        g[D.nz_off + j] = int32_t(cg);
        const int64_t off = cg - (row0 + i);
        if (off < -32767 || off > 32767)
          fits = false;
        else
          d[D.nz_off + j] = int16_t(off);
      }
    }
    row0 += D.nrows;
  }
  DeviceGuard dg(A->comm->device);
  C.cols_global.reserve(sizeof(int32_t) * C.nz_total);
  SPMVB_CUDA(cudaMemcpy(C.cols_global.ptr, g.data(), sizeof(int32_t) * C.nz_total,
                        cudaMemcpyHostToDevice));
  C.d16 = fits && row0 < (int64_t(1) << 31) - 65536;
  if (C.d16) {
    C.d16_global.reserve(sizeof(int16_t) * C.nz_total);
    SPMVB_CUDA(cudaMemcpy(C.d16_global.ptr, d.data(), sizeof(int16_t) * C.nz_total,
                          cudaMemcpyHostToDevice));
  }
}

// A^T per rank as its own CSR, built once by a stable counting sort over
// columns: row c of A^T lists the entries of column c in ascending row
// order, the order in which the reference's column-scatter product
// (Matrix.cpp:206-211) accumulates them.
void build_transpose(spmv_matrix A) {
  if (A->trn_built) return;
  DevCsr& T = A->trn;
  const int P = A->comm->size;
  const size_t es = dtype_size(A->dtype);
  T.parts.assign(P, DevPart{});
  std::vector<std::vector<int32_t>> rp(P), ci(P);
  std::vector<std::vector<unsigned char>> va(P);
  int64_t rpo = 0, nzo = 0, rows = 0, nnz_all = 0, maxr = 0;
  for (int r = 0; r < P; ++r) {
    const int32_t m = A->nrows[r], n = A->ncols[r];
    const auto& arp = A->h_rowptr[r];
    const auto& aci = A->h_colind[r];
    const int64_t nnz = arp[m];
    rp[r].assign(size_t(n) + 1, 0);
    for (int64_t j = 0; j < nnz; ++j) ++rp[r][aci[j] + 1];
    for (int32_t c = 0; c < n; ++c) rp[r][c + 1] += rp[r][c];
    ci[r].resize(nnz);
    va[r].resize(nnz * es);
    std::vector<int32_t> fill(rp[r].begin(), rp[r].end() - 1);
    for (int32_t i = 0; i < m; ++i)
      for (int32_t j = arp[i]; j < arp[i + 1]; ++j) {
        const int32_t dst = fill[aci[j]]++;
        ci[r][dst] = i;
        std::memcpy(&va[r][size_t(dst) * es], &A->h_vals[r][size_t(j) * es], es);
      }
    DevPart& D = T.parts[r];
    D.nrows = n;
    D.ncols = m;
    D.nnz = nnz;
    D.rp_off = rpo;
    D.nz_off = nzo;
    rpo += n + 1;
    nzo = align_up(nzo + nnz, 4);
    rows += n;
    nnz_all += nnz;
    for (int32_t c = 0; c < n; ++c)
      maxr = std::max<int64_t>(maxr, rp[r][c + 1] - rp[r][c]);
  }
  T.rp_total = rpo;
  T.nz_total = nzo + 4;
  T.mean_row = rows > 0 ? double(nnz_all) / double(rows) : 0.0;
  T.max_row = maxr;
  T.sell_padded = 0;
  for (int r = 0; r < P; ++r)
    T.sell_padded += sell_padded_size(rp[r], T.parts[r].nrows, nullptr);
  DeviceGuard dg(A->comm->device);
  T.rowptr.reserve(sizeof(int32_t) * std::max<int64_t>(T.rp_total, 1));
  T.cols.reserve(sizeof(int32_t) * T.nz_total);
  T.vals.reserve(es * T.nz_total);
  SPMVB_CUDA(cudaMemset(T.cols.ptr, 0, sizeof(int32_t) * T.nz_total));
  SPMVB_CUDA(cudaMemset(T.vals.ptr, 0, es * T.nz_total));
  for (int r = 0; r < P; ++r) {
    const DevPart& D = T.parts[r];
    SPMVB_CUDA(cudaMemcpy(T.rowptr.as<int32_t>() + D.rp_off, rp[r].data(),
                          sizeof(int32_t) * (D.nrows + 1), cudaMemcpyHostToDevice));
    if (D.nnz == 0) continue;
    SPMVB_CUDA(cudaMemcpy(T.cols.as<int32_t>() + D.nz_off, ci[r].data(),
                          sizeof(int32_t) * D.nnz, cudaMemcpyHostToDevice));
    SPMVB_CUDA(cudaMemcpy(T.vals.as<char>() + D.nz_off * es, va[r].data(),
                          es * D.nnz, cudaMemcpyHostToDevice));
  }
  A->h_trn_rowptr = std::move(rp);
  A->trn_built = true;
}

void release_comm(spmv_comm comm) {
  if (--comm->refs > 0) return;
  if (comm->device >= 0) {
    DeviceGuard dg(comm->device);
    if (comm->own_stream)
      soft_check(cudaStreamDestroy(comm->stream), "cudaStreamDestroy");
    comm->stage_in.release();
    comm->stage_out.release();
  }
  delete comm;
}

void release_map(spmv_l2gmap map) {
  if (--map->refs > 0) return;
  spmv_comm comm = map->comm;
  {
    DeviceGuard dg(comm->device);
    delete map;
  }
  release_comm(comm);
}

namespace {

// y = op(A) x for all ranks, host or device vectors.
void product(spmv_matrix A, bool transpose, spmv_memory memory,
             const void* const* x, void* const* y) {
  check_mat(A);
  spmv_comm comm = A->comm;
  comm->require_device();
  require(x != nullptr && y != nullptr, "spmv: vector array is NULL");
  require(memory == SPMV_MEMORY_HOST || memory == SPMV_MEMORY_DEVICE,
          "spmv: unknown memory kind");
  DeviceGuard dg(comm->device);
  if (transpose) build_transpose(A);
  // The transpose's kernel follows its own row statistics (a kernel set on
  // the matrix is for the forward product); SELL-32 sums each row of A^T in
  // ascending row order of A, the reference's column-scatter order.
  const spmv_kernel requested = transpose ? SPMV_KERNEL_AUTO : A->kernel;
  const spmv_kernel picked = pick_kernel(requested, transpose ? A->trn : A->fwd);
  if (picked == SPMV_KERNEL_SELL || picked == SPMV_KERNEL_STAGED)
    build_sell(A, transpose ? A->trn : A->fwd, comm->stream);
  const DevCsr& C = transpose ? A->trn : A->fwd;
  const int P = comm->size;
  const size_t es = dtype_size(A->dtype);
  std::vector<int64_t> xlen(P), ylen(P);
  for (int r = 0; r < P; ++r) {
    xlen[r] = C.parts[r].ncols;
    ylen[r] = C.parts[r].nrows;
  }
  SpmvLaunch L{};
  L.csr = &C;
  L.cols = C.cols.as<int32_t>();
  L.dtype = A->dtype;
  L.kernel = requested;
  L.width = transpose ? 0 : A->width;
  L.block = transpose ? 0 : A->block;
  L.num_sms = comm->num_sms;
  L.carry = transpose ? &A->trn.merge_carry : &A->fwd.merge_carry;
  L.err = comm->wait_flag();
  cudaStream_t s = comm->stream;
  if (memory == SPMV_MEMORY_DEVICE) {
    L.x = x;
    L.y = y;
    launch_spmv(L, s);
    return;
  }
  Staging si, so;
  si.layout(xlen, es);
  so.layout(ylen, es);
  comm->stage_in.reserve(std::max<int64_t>(si.total, 256));
  comm->stage_out.reserve(std::max<int64_t>(so.total, 256));
  std::vector<const void*> dx(P);
  std::vector<void*> dy(P);
  for (int r = 0; r < P; ++r) {
    dx[r] = comm->stage_in.as<char>() + si.off[r];
    dy[r] = comm->stage_out.as<char>() + so.off[r];
    if (xlen[r] > 0) {
      require(x[r] != nullptr, "spmv: x vector is NULL");
      SPMVB_CUDA(cudaMemcpyAsync(const_cast<void*>(dx[r]), x[r], xlen[r] * es,
                                 cudaMemcpyHostToDevice, s));
    }
  }
  L.x = dx.data();
  L.y = dy.data();
  launch_spmv(L, s);
  for (int r = 0; r < P; ++r)
    if (ylen[r] > 0) {
      require(y[r] != nullptr, "spmv: y vector is NULL");
      SPMVB_CUDA(cudaMemcpyAsync(y[r], dy[r], ylen[r] * es, cudaMemcpyDeviceToHost, s));
    }
  SPMVB_CUDA(cudaStreamSynchronize(s));
}

// update / reverse_update with host or device vectors.
void halo(spmv_l2gmap map, bool reverse, spmv_dtype dtype, spmv_memory memory,
          void* const* vecs) {
  check_map(map);
  spmv_comm comm = map->comm;
  comm->require_device();
  require(vecs != nullptr, "spmv: vector array is NULL");
  const size_t es = dtype_size(dtype);
  DeviceGuard dg(comm->device);
  const int P = comm->size;
  cudaStream_t s = comm->stream;
  if (memory == SPMV_MEMORY_DEVICE) {
    reverse ? launch_reverse_update(map, dtype, vecs, s)
            : launch_update(map, dtype, vecs, s);
    return;
  }
  require(memory == SPMV_MEMORY_HOST, "spmv: unknown memory kind");
  std::vector<int64_t> len(P);
  for (int r = 0; r < P; ++r) len[r] = map->vec_len(r);
  Staging st;
  st.layout(len, es);
  comm->stage_in.reserve(std::max<int64_t>(st.total, 256));
  std::vector<void*> dv(P);
  for (int r = 0; r < P; ++r) {
    dv[r] = comm->stage_in.as<char>() + st.off[r];
    if (len[r] > 0) {
      require(vecs[r] != nullptr, "spmv: vector is NULL");
      SPMVB_CUDA(cudaMemcpyAsync(dv[r], vecs[r], len[r] * es, cudaMemcpyHostToDevice, s));
    }
  }
  reverse ? launch_reverse_update(map, dtype, dv.data(), s)
          : launch_update(map, dtype, dv.data(), s);
  for (int r = 0; r < P; ++r)
    if (len[r] > 0)
      SPMVB_CUDA(cudaMemcpyAsync(vecs[r], dv[r], len[r] * es, cudaMemcpyDeviceToHost, s));
  SPMVB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace
}  // namespace spmvb

namespace spmvb {

// Checks shared by the solvers (cg.cpp:22-28 and the layout the fused-halo
// solve needs).
void check_solve_args(spmv_matrix A, spmv_memory memory, const double* const* b,
                      const int64_t* b_rows, double* const* x) {
  check_mat(A);
  require(A->dtype == SPMV_FLOAT64, "spmv::cg - Error: A must be float64");
  spmv_l2gmap rm = A->row_map, cm = A->col_map;
  require(rm != nullptr && cm != nullptr, "spmv::cg - Error: A needs row and column maps");
  const int P = A->comm->size;
  for (int r = 0; r < P; ++r)
    if (!rm->rank[r].ghosts.empty())
      fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv::cg - Error: A.row_map() has ghost entries");
  if (b_rows)
    for (int r = 0; r < P; ++r)
      if (b_rows[r] != rm->rank[r].local_size)
        fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv::cg - Error: b.rows() != A.rows()");
  // p.head(M) (cg.cpp:41) needs the owned column range to be the row range.
  for (int r = 0; r < P; ++r)
    require(cm->rank[r].local_size == rm->rank[r].local_size,
            "spmv::cg - Error: column map local sizes differ from row map");
  require(b != nullptr && x != nullptr, "spmv::cg - Error: NULL vector array");
  require(memory == SPMV_MEMORY_HOST || memory == SPMV_MEMORY_DEVICE,
          "spmv: unknown memory kind");
  A->comm->require_device();
}

// Rank vectors b[r] into the global-layout device vector.
void copy_rhs_in(spmv_matrix A, spmv_memory memory, const double* const* b, double* db) {
  spmv_l2gmap rm = A->row_map;
  cudaStream_t s = A->comm->stream;
  const cudaMemcpyKind k = memory == SPMV_MEMORY_HOST ? cudaMemcpyHostToDevice
                                                      : cudaMemcpyDeviceToDevice;
  for (int r = 0; r < A->comm->size; ++r) {
    const int64_t M = rm->rank[r].local_size;
    if (M == 0) continue;
    require(b[r] != nullptr, "spmv::cg - Error: b is NULL");
    SPMVB_CUDA(cudaMemcpyAsync(db + rm->ranges[r], b[r], M * sizeof(double), k, s));
  }
}

// Global-layout solution into the rank vectors x[r] (ghost tail zero).
void copy_solution_out(spmv_matrix A, spmv_memory memory, const double* dx,
                       double* const* x) {
  spmv_l2gmap rm = A->row_map, cm = A->col_map;
  cudaStream_t s = A->comm->stream;
  const cudaMemcpyKind k = memory == SPMV_MEMORY_HOST ? cudaMemcpyDeviceToHost
                                                      : cudaMemcpyDeviceToDevice;
  for (int r = 0; r < A->comm->size; ++r) {
    const int64_t M = rm->rank[r].local_size;
    const int64_t G = int64_t(cm->rank[r].ghosts.size());
    if (M + G == 0) continue;
    require(x[r] != nullptr, "spmv::cg - Error: x is NULL");
    if (M > 0)
      SPMVB_CUDA(cudaMemcpyAsync(x[r], dx + rm->ranges[r], M * sizeof(double), k, s));
    if (G > 0) {
      if (memory == SPMV_MEMORY_HOST)
        std::fill(x[r] + M, x[r] + M + G, 0.0);
      else
        SPMVB_CUDA(cudaMemsetAsync(x[r] + M, 0, G * sizeof(double), s));
    }
  }
  SPMVB_CUDA(cudaStreamSynchronize(s));
}

}  // namespace spmvb

using namespace spmvb;

extern "C" {

const char* spmv_last_error(void) { return g_last_error.c_str(); }

int spmv_get_version(int* major, int* minor) {
  return guard([&] {
    require(major && minor, "spmv: NULL output");
    *major = SPMV_B200_VERSION_MAJOR;
    *minor = SPMV_B200_VERSION_MINOR;
  });
}

// ---------------------------------------------------------------- comm ----
int spmv_comm_create(int device, void* stream, int size, spmv_comm* out) {
  return guard([&] {
    require(out != nullptr, "spmv: NULL output");
    *out = nullptr;
    require(size >= 1 && size <= SPMV_MAX_PARTS,
            "spmv: communicator size must be 1.." + std::to_string(SPMV_MAX_PARTS));
    require(device >= -1, "spmv: invalid device");
    std::unique_ptr<spmv_comm_s> c(new spmv_comm_s);
    c->size = size;
    c->device = device;
    if (device >= 0) {
      int count = 0;
      if (cudaGetDeviceCount(&count) != cudaSuccess || count == 0)
        fail(SPMV_ERROR_NO_DEVICE, "spmv: no CUDA device available");
      require(device < count, "spmv: invalid device");
      DeviceGuard dg(device);
      SPMVB_CUDA(cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device));
      if (stream) {
        c->stream = static_cast<cudaStream_t>(stream);
      } else {
        SPMVB_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
      }
    }
    *out = c.release();
  });
}

int spmv_comm_destroy(spmv_comm comm) {
  return guard([&] {
    if (comm) release_comm(comm);
  });
}

int spmv_comm_size(spmv_comm comm, int* size) {
  return guard([&] {
    check_comm(comm);
    require(size, "spmv: NULL output");
    *size = comm->size;
  });
}

int spmv_comm_device(spmv_comm comm, int* device) {
  return guard([&] {
    check_comm(comm);
    require(device, "spmv: NULL output");
    *device = comm->device;
  });
}

int spmv_comm_stream(spmv_comm comm, void** stream) {
  return guard([&] {
    check_comm(comm);
    require(stream, "spmv: NULL output");
    *stream = comm->stream;
  });
}

int spmv_comm_synchronize(spmv_comm comm) {
  return guard([&] {
    check_comm(comm);
    comm->require_device();
    DeviceGuard dg(comm->device);
    SPMVB_CUDA(cudaStreamSynchronize(comm->stream));
    if (comm->wait_err.ptr) {
      int flag = 0;
      SPMVB_CUDA(cudaMemcpy(&flag, comm->wait_err.ptr, sizeof(int), cudaMemcpyDeviceToHost));
      if (flag) {
        SPMVB_CUDA(cudaMemset(comm->wait_err.ptr, 0, sizeof(int)));
        fail(SPMV_ERROR_CUDA, "spmv: a staged product's bounded wait timed out");
      }
    }
  });
}

// -------------------------------------------------------------- L2GMap ----
int spmv_l2gmap_create(spmv_comm comm, const int64_t* local_size,
                       const int64_t* const* ghosts, const int64_t* num_ghosts,
                       spmv_l2gmap* out) {
  return guard([&] {
    check_comm(comm);
    require(out != nullptr, "spmv: NULL output");
    *out = nullptr;
    std::unique_ptr<spmv_l2gmap_s> m(new spmv_l2gmap_s);
    m->comm = comm;
    build_pattern(m.get(), local_size, ghosts, num_ghosts);
    ++comm->refs;
    *out = m.release();
  });
}

int spmv_l2gmap_destroy(spmv_l2gmap map) {
  return guard([&] {
    if (map) release_map(map);
  });
}

int spmv_l2gmap_local_size(spmv_l2gmap map, int rank, int32_t* out) {
  return guard([&] {
    check_map(map);
    check_rank(map->comm, rank);
    require(out, "spmv: NULL output");
    *out = int32_t(map->ranges[rank + 1] - map->ranges[rank]);
  });
}

int spmv_l2gmap_num_ghosts(spmv_l2gmap map, int rank, int32_t* out) {
  return guard([&] {
    check_map(map);
    check_rank(map->comm, rank);
    require(out, "spmv: NULL output");
    *out = int32_t(map->rank[rank].ghosts.size());
  });
}

int spmv_l2gmap_global_size(spmv_l2gmap map, int64_t* out) {
  return guard([&] {
    check_map(map);
    require(out, "spmv: NULL output");
    *out = map->ranges.back();
  });
}

int spmv_l2gmap_global_offset(spmv_l2gmap map, int rank, int64_t* out) {
  return guard([&] {
    check_map(map);
    check_rank(map->comm, rank);
    require(out, "spmv: NULL output");
    *out = map->ranges[rank];
  });
}

int spmv_l2gmap_global_to_local(spmv_l2gmap map, int rank, int64_t i,
                                int32_t* out) {
  return guard([&] {
    check_map(map);
    check_rank(map->comm, rank);
    require(out, "spmv: NULL output");
    const int64_t r0 = map->ranges[rank], r1 = map->ranges[rank + 1];
    if (i >= r0 && i < r1) {
      *out = int32_t(i - r0);
      return;
    }
    const auto& g = map->rank[rank].ghosts;
    auto it = std::lower_bound(g.begin(), g.end(), i);
    require(it != g.end() && *it == i,
            "spmv::L2GMap - Error: global index is neither owned nor a ghost");
    *out = int32_t(map->rank[rank].local_size + (it - g.begin()));
  });
}

int spmv_l2gmap_ghosts(spmv_l2gmap map, int rank, const int64_t** ghosts,
                       int32_t* n) {
  return guard([&] {
    check_map(map);
    check_rank(map->comm, rank);
    require(ghosts && n, "spmv: NULL output");
    *ghosts = map->rank[rank].ghosts.data();
    *n = int32_t(map->rank[rank].ghosts.size());
  });
}

int spmv_l2gmap_pattern(spmv_l2gmap map, int rank, spmv_pattern_field field,
                        const int32_t** data, int32_t* n) {
  return guard([&] {
    check_map(map);
    check_rank(map->comm, rank);
    require(data && n, "spmv: NULL output");
    const RankMap& R = map->rank[rank];
    const std::vector<int32_t>* v = nullptr;
    switch (field) {
      case SPMV_PATTERN_NEIGHBOURS: v = &R.neighbours; break;
      case SPMV_PATTERN_SEND_COUNT: v = &R.send_count; break;
      case SPMV_PATTERN_RECV_COUNT: v = &R.recv_count; break;
      case SPMV_PATTERN_SEND_OFFSET: v = &R.send_offset; break;
      case SPMV_PATTERN_RECV_OFFSET: v = &R.recv_offset; break;
      case SPMV_PATTERN_INDEXBUF: v = &R.indexbuf; break;
      default: fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: unknown pattern field");
    }
    *data = v->data();
    *n = int32_t(v->size());
  });
}

int spmv_l2gmap_update(spmv_l2gmap map, spmv_dtype dtype, spmv_memory memory,
                       void* const* vecs) {
  return guard([&] { halo(map, false, dtype, memory, vecs); });
}

int spmv_l2gmap_reverse_update(spmv_l2gmap map, spmv_dtype dtype,
                               spmv_memory memory, void* const* vecs) {
  return guard([&] { halo(map, true, dtype, memory, vecs); });
}

// -------------------------------------------------------------- Matrix ----
int spmv_matrix_create_csr(spmv_comm comm, spmv_dtype dtype,
                           spmv_l2gmap col_map, spmv_l2gmap row_map,
                           const int32_t* nrows, const int32_t* ncols,
                           const int32_t* const* rowptr,
                           const int32_t* const* colind,
                           const void* const* values, spmv_matrix* out) {
  return guard([&] {
    check_comm(comm);
    require(out != nullptr, "spmv: NULL output");
    *out = nullptr;
    require(dtype == SPMV_FLOAT64 || dtype == SPMV_FLOAT32 || dtype == SPMV_COMPLEX64 ||
                dtype == SPMV_COMPLEX128,
            "spmv::Matrix - Error: unknown dtype");
    require(nrows && ncols && rowptr && colind && values,
            "spmv::Matrix - Error: NULL CSR array");
    require(!col_map || col_map->comm == comm,
            "spmv::Matrix - Error: column map belongs to another communicator");
    require(!row_map || row_map->comm == comm,
            "spmv::Matrix - Error: row map belongs to another communicator");
    const int P = comm->size;
    const size_t es = dtype_size(dtype);
    std::unique_ptr<spmv_matrix_s> A(new spmv_matrix_s);
    A->comm = comm;
    A->dtype = dtype;
    A->col_map = col_map;
    A->row_map = row_map;
    A->nrows.assign(nrows, nrows + P);
    A->ncols.assign(ncols, ncols + P);
    A->h_rowptr.resize(P);
    A->h_colind.resize(P);
    A->h_vals.resize(P);
    for (int r = 0; r < P; ++r) {
      const int32_t m = nrows[r], n = ncols[r];
      require(m >= 0 && n >= 0, "spmv::Matrix - Error: negative dimension");
      require(rowptr[r] != nullptr, "spmv::Matrix - Error: NULL row pointer array");
      require(rowptr[r][0] == 0, "spmv::Matrix - Error: row pointers must start at 0");
      for (int32_t i = 0; i < m; ++i)
        require(rowptr[r][i + 1] >= rowptr[r][i],
                "spmv::Matrix - Error: row pointers must be non-decreasing");
      const int64_t nnz = rowptr[r][m];
      require(nnz == 0 || (colind[r] && values[r]),
              "spmv::Matrix - Error: NULL column or value array");
      if (col_map)
        require(int64_t(n) == col_map->vec_len(r),
                "spmv::Matrix - Error: ncols != col_map local_size + num_ghosts");
      if (row_map)
        require(int64_t(m) == row_map->vec_len(r),
                "spmv::Matrix - Error: nrows != row_map local_size + num_ghosts");
      A->h_rowptr[r].assign(rowptr[r], rowptr[r] + m + 1);
      A->h_colind[r].assign(colind[r], colind[r] + nnz);
      for (int64_t j = 0; j < nnz; ++j)
        require(colind[r][j] >= 0 && colind[r][j] < n,
                "spmv::Matrix - Error: column index out of range");
      const unsigned char* vb = static_cast<const unsigned char*>(values[r]);
      A->h_vals[r].assign(vb, vb + nnz * es);
    }
    upload_csr(A.get());
    ++comm->refs;
    if (col_map) ++col_map->refs;
    if (row_map) ++row_map->refs;
    *out = A.release();
  });
}

int spmv_matrix_destroy(spmv_matrix A) {
  return guard([&] {
    if (!A) return;
    spmv_comm comm = A->comm;
    spmv_l2gmap cm = A->col_map, rm = A->row_map;
    {
      DeviceGuard dg(comm->device);
      delete A;
    }
    if (cm) release_map(cm);
    if (rm) release_map(rm);
    release_comm(comm);
  });
}

int spmv_matrix_mult(spmv_matrix A, spmv_memory memory, const void* const* x,
                     void* const* y) {
  return guard([&] { product(A, false, memory, x, y); });
}

int spmv_matrix_transpmult(spmv_matrix A, spmv_memory memory,
                           const void* const* x, void* const* y) {
  return guard([&] { product(A, true, memory, x, y); });
}

int spmv_matrix_dtype(spmv_matrix A, spmv_dtype* dtype) {
  return guard([&] {
    check_mat(A);
    require(dtype, "spmv: NULL output");
    *dtype = A->dtype;
  });
}

int spmv_matrix_rows(spmv_matrix A, int rank, int32_t* nrows) {
  return guard([&] {
    check_mat(A);
    check_rank(A->comm, rank);
    require(nrows, "spmv: NULL output");
    *nrows = A->nrows[rank];
  });
}

int spmv_matrix_cols(spmv_matrix A, int rank, int32_t* ncols) {
  return guard([&] {
    check_mat(A);
    check_rank(A->comm, rank);
    require(ncols, "spmv: NULL output");
    *ncols = A->ncols[rank];
  });
}

int spmv_matrix_nnz(spmv_matrix A, int rank, int64_t* nnz) {
  return guard([&] {
    check_mat(A);
    check_rank(A->comm, rank);
    require(nnz, "spmv: NULL output");
    *nnz = A->h_rowptr[rank][A->nrows[rank]];
  });
}

int spmv_matrix_csr(spmv_matrix A, int rank, const int32_t** rowptr,
                    const int32_t** colind, const void** values) {
  return guard([&] {
    check_mat(A);
    check_rank(A->comm, rank);
    require(rowptr && colind && values, "spmv: NULL output");
    *rowptr = A->h_rowptr[rank].data();
    *colind = A->h_colind[rank].data();
    *values = A->h_vals[rank].data();
  });
}

int spmv_matrix_col_map(spmv_matrix A, spmv_l2gmap* map) {
  return guard([&] {
    check_mat(A);
    require(map, "spmv: NULL output");
    *map = A->col_map;
  });
}

int spmv_matrix_row_map(spmv_matrix A, spmv_l2gmap* map) {
  return guard([&] {
    check_mat(A);
    require(map, "spmv: NULL output");
    *map = A->row_map;
  });
}

int spmv_matrix_set_values(spmv_matrix A, spmv_memory memory,
                           const void* const* values) {
  return guard([&] {
    check_mat(A);
    require(values, "spmv: NULL value array");
    const int P = A->comm->size;
    const size_t es = dtype_size(A->dtype);
    DeviceGuard dg(A->comm->device);
    for (int r = 0; r < P; ++r) {
      const int64_t nnz = A->h_rowptr[r][A->nrows[r]];
      if (nnz == 0) continue;
      require(values[r] != nullptr, "spmv: NULL value array");
      if (memory == SPMV_MEMORY_HOST) {
        const unsigned char* vb = static_cast<const unsigned char*>(values[r]);
        std::memcpy(A->h_vals[r].data(), vb, nnz * es);
      } else {
        A->comm->require_device();
        SPMVB_CUDA(cudaMemcpy(A->h_vals[r].data(), values[r], nnz * es,
                              cudaMemcpyDeviceToHost));
      }
      if (A->comm->device >= 0)
        SPMVB_CUDA(cudaMemcpy(A->fwd.vals.as<char>() + A->fwd.parts[r].nz_off * es,
                              A->h_vals[r].data(), nnz * es, cudaMemcpyHostToDevice));
    }
    // Derived copies are rebuilt on next use (the mixed solver's graph holds
    // the FP32 copy's address, so it goes too).
    A->trn_built = false;
    A->trn = DevCsr{};
    A->ir.reset();
    A->fwd.vals32.release();
    if (A->comm->device >= 0) refresh_sell_values(A);
  });
}

int spmv_matrix_sample_outer(spmv_matrix A, spmv_memory memory, double scale,
                             const void* const* lambda, const void* const* x,
                             void* const* out) {
  return guard([&] {
    check_mat(A);
    spmv_comm comm = A->comm;
    comm->require_device();
    require(lambda && x && out, "spmv: vector array is NULL");
    require(A->dtype == SPMV_FLOAT64 || A->dtype == SPMV_FLOAT32,
            "spmv: only float64 and float32 matrices are implemented");
    DeviceGuard dg(comm->device);
    cudaStream_t s = comm->stream;
    if (memory == SPMV_MEMORY_DEVICE) {
      launch_sample_outer(A, scale, lambda, x, out, s);
      return;
    }
    require(memory == SPMV_MEMORY_HOST, "spmv: unknown memory kind");
    const int P = comm->size;
    const size_t es = dtype_size(A->dtype);
    std::vector<int64_t> lens;  // lambda[P], x[P], out[P]
    for (int r = 0; r < P; ++r) lens.push_back(A->nrows[r]);
    for (int r = 0; r < P; ++r) lens.push_back(A->ncols[r]);
    for (int r = 0; r < P; ++r) lens.push_back(A->h_rowptr[r][A->nrows[r]]);
    Staging st;
    st.layout(lens, es);
    comm->stage_in.reserve(std::max<int64_t>(st.total, 256));
    std::vector<const void*> dl(P), dx(P);
    std::vector<void*> dout(P);
    char* base = comm->stage_in.as<char>();
    for (int r = 0; r < P; ++r) {
      dl[r] = base + st.off[r];
      dx[r] = base + st.off[P + r];
      dout[r] = base + st.off[2 * P + r];
      if (lens[r] > 0)
        SPMVB_CUDA(cudaMemcpyAsync(const_cast<void*>(dl[r]), lambda[r], lens[r] * es,
                                   cudaMemcpyHostToDevice, s));
      if (lens[P + r] > 0)
        SPMVB_CUDA(cudaMemcpyAsync(const_cast<void*>(dx[r]), x[r], lens[P + r] * es,
                                   cudaMemcpyHostToDevice, s));
    }
    launch_sample_outer(A, scale, dl.data(), dx.data(), dout.data(), s);
    for (int r = 0; r < P; ++r)
      if (lens[2 * P + r] > 0)
        SPMVB_CUDA(cudaMemcpyAsync(out[r], dout[r], lens[2 * P + r] * es,
                                   cudaMemcpyDeviceToHost, s));
    SPMVB_CUDA(cudaStreamSynchronize(s));
  });
}

int spmv_matrix_set_kernel(spmv_matrix A, spmv_kernel kernel, int width,
                           int block) {
  return guard([&] {
    check_mat(A);
    require(kernel == SPMV_KERNEL_AUTO || kernel == SPMV_KERNEL_VECTOR ||
                kernel == SPMV_KERNEL_MERGE || kernel == SPMV_KERNEL_SELL ||
                kernel == SPMV_KERNEL_STAGED,
            "spmv: unknown kernel");
    require(kernel == SPMV_KERNEL_STAGED || width == 0 ||
                (width >= 1 && width <= 32 && (width & (width - 1)) == 0),
            "spmv: width must be 0 or 1..32, a power of two");
    require(kernel != SPMV_KERNEL_SELL || width <= 16,
            "spmv: SELL width (loads in flight per lane) must be 1..16");
    require(kernel != SPMV_KERNEL_STAGED || width == 0 || width == 4 || width == 5 ||
                width == 7 || width == 8 || width == 9,
            "spmv: staged width (gathers in flight per lane) must be 4, 5, 7, 8 or 9");
    require(block == 0 || block == 128 || block == 256 || block == 512,
            "spmv: block must be 0, 128, 256 or 512");
    A->kernel = kernel;
    A->width = width;
    A->block = block;
    A->kernel_set = kernel != SPMV_KERNEL_AUTO;
    A->cg.reset();  // graphs bake the kernel choice in
    A->ir.reset();
  });
}

int spmv_matrix_get_kernel(spmv_matrix A, spmv_kernel* kernel, int* width,
                           int* block) {
  return guard([&] {
    check_mat(A);
    require(kernel && width && block, "spmv: NULL output");
    *kernel = pick_kernel(A->kernel, A->fwd);
    if (*kernel == SPMV_KERNEL_MERGE)
      *width = 0;  // merge-path tiles do not depend on a width
    else if (A->width > 0)
      *width = A->width;
    else
      *width = (*kernel == SPMV_KERNEL_SELL || *kernel == SPMV_KERNEL_STAGED)
                   ? 8
                   : auto_width(A->fwd.mean_row, A->dtype);
    // Threads per CTA the product runs (the staged product has its own shape).
    *block = *kernel == SPMV_KERNEL_STAGED ? kStagedThreads : A->block > 0 ? A->block : 256;
  });
}

// ------------------------------------------------------------------ CG ----
int spmv_cg_ex(spmv_matrix A, spmv_memory memory, const double* const* b,
               const int64_t* b_rows, double* const* x, int max_its,
               double rtol, spmv_cg_info* info) {
  return guard([&] {
    check_solve_args(A, memory, b, b_rows, x);
    DeviceGuard dg(A->comm->device);
    copy_rhs_in(A, memory, b, cg_rhs(A));
    spmv_cg_info local{};
    cg_run(A, max_its, rtol, &local);
    copy_solution_out(A, memory, cg_solution(A), x);
    if (info) *info = local;
    if (local.status == SPMV_ERROR_BREAKDOWN)
      fail(SPMV_ERROR_BREAKDOWN,
           "spmv::cg - Error: breakdown, p.Ap is zero or not finite at iteration " +
               std::to_string(local.iterations));
  });
}

int spmv_cg_mixed(spmv_matrix A, spmv_memory memory, const double* const* b,
                  const int64_t* b_rows, double* const* x, int max_its,
                  double rtol, spmv_ir_info* info) {
  return guard([&] {
    check_solve_args(A, memory, b, b_rows, x);
    DeviceGuard dg(A->comm->device);
    copy_rhs_in(A, memory, b, ir_rhs(A));
    spmv_ir_info local{};
    ir_run(A, max_its, rtol, &local);
    copy_solution_out(A, memory, ir_solution(A), x);
    if (info) *info = local;
    if (local.status == SPMV_ERROR_BREAKDOWN)
      fail(SPMV_ERROR_BREAKDOWN,
           "spmv::cg - Error: breakdown in the mixed-precision solve after " +
               std::to_string(local.iterations) + " iterations");
  });
}

int spmv_cg(spmv_matrix A, spmv_memory memory, const double* const* b,
            const int64_t* b_rows, double* const* x, int max_its, double rtol,
            int* num_its) {
  spmv_cg_info info{};
  const int st = spmv_cg_ex(A, memory, b, b_rows, x, max_its, rtol, &info);
  if (num_its) *num_its = info.iterations;
  return st;
}

int spmv_matrix_solver_product(spmv_matrix A, int solver, spmv_kernel* kernel, int* width,
                               int* index_bits, double* us) {
  return guard([&] {
    check_mat(A);
    require(kernel && width && index_bits && us, "spmv: NULL output");
    require(solver >= 0 && solver <= 2, "spmv: solver must be 0, 1 or 2");
    const SolverProduct p = solver == 0 ? cg_product(A) : ir_product(A, solver == 1);
    *kernel = p.kind == ProductKind::Staged ? SPMV_KERNEL_STAGED
              : p.kind == ProductKind::Sell ? SPMV_KERNEL_SELL
                                            : SPMV_KERNEL_VECTOR;
    *width = p.w;
    *index_bits = p.d16 ? 16 : 32;
    *us = p.us;
  });
}

int spmv_matrix_cg_form(spmv_matrix A, int* fused, int* ctas_per_sm, int* r_shared) {
  return guard([&] {
    check_mat(A);
    require(fused && ctas_per_sm && r_shared, "spmv: NULL output");
    const CgForm f = cg_form(A);
    *fused = f.fused ? (f.merged ? 2 : 1) : 0;
    *ctas_per_sm = f.cps;
    *r_shared = f.rs ? 1 : 0;
  });
}

int spmv_matrix_cg_mixed_form(spmv_matrix A, int* fused, int* ctas_per_sm, int* r_shared) {
  return guard([&] {
    check_mat(A);
    require(fused && ctas_per_sm && r_shared, "spmv: NULL output");
    const CgForm f = ir_form(A);
    *fused = f.fused ? 1 : 0;
    *ctas_per_sm = f.cps;
    *r_shared = f.rs ? 1 : 0;
  });
}

}  // extern "C"
