// Merge-path CSR product: load-balanced for skewed row lengths.
//
// The product is the merge of two lists, the row ends rowptr[1..m] and the
// entry indices 0..nnz-1 (m + nnz items; Merrill & Garland, "Merge-based
// parallel sparse matrix-vector multiplication", SC'16).  Consuming an entry
// adds v[j] * x[c[j]] to the current row's sum; consuming a row end emits the
// row.  Every CTA takes an equal tile of TILE = BS * IPT consecutive items,
// whatever the row lengths, so one long row is spread over many CTAs.
//
// Per CTA: a binary search on the diagonal gives the tile's first and last
// (row, entry) coordinates; the tile's products and row ends are staged in
// shared memory with coalesced loads; each thread searches its own start and
// consumes IPT items.  Partial rows are combined in a fixed order, so results
// are reproducible: a thread whose first emitted row began in earlier threads
// adds their carries (left to right) before storing it; the CTA's last carry
// goes to a per-CTA slot, and merge_fixup adds each run of carries that
// belong to one row, in CTA order, to that row.
#include <algorithm>
#include <mutex>
#include <string>
#include <vector>

#include "internal.h"
#include "kernels.cuh"

namespace spmvb {

namespace {

constexpr int MBS = 256;  // threads per CTA
constexpr int IPT = 8;    // merge items per thread
constexpr int TILE = MBS * IPT;

// Smallest row count i in [lo, hi] (rows consumed) of the split point on
// diagonal d: the first i with rowend(i) > d - i - 1, rowend(i) = rp(i + 1).
template <class RP>
__device__ __forceinline__ int merge_search(int d, int lo, int hi, RP rp) {
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (rp(mid + 1) <= d - mid - 1)
      lo = mid + 1;
    else
      hi = mid;
  }
  return lo;
}

template <typename T>
__global__ void __launch_bounds__(MBS)
    merge_kernel(const __grid_constant__ SpmvArgs a, int* __restrict__ carry_row,
                 T* __restrict__ carry_val) {
  __shared__ int s_rp[TILE + 2];
  __shared__ T s_prod[TILE];
  __shared__ int s_crow[MBS];
  __shared__ T s_cval[MBS];
  __shared__ int s_bounds[4];

  const int p = find_part(a, blockIdx.x);
  const PartArg& P = a.part[p];
  const int m = P.nrows;
  const int32_t* __restrict__ rowptr = P.rowptr;
  const int nnz = rowptr[m];
  const long total = long(m) + nnz;
  const int tile = int(blockIdx.x) - P.block_begin;
  const long d0l = long(tile) * TILE;
  const int d0 = int(d0l);
  const int d1 = int(min(total, d0l + TILE));

  if (threadIdx.x < 2) {
    const int d = threadIdx.x == 0 ? d0 : d1;
    const int i = merge_search(d, max(0, d - nnz), min(d, m),
                               [&](int r) { return __ldg(rowptr + r); });
    s_bounds[2 * threadIdx.x] = i;
    s_bounds[2 * threadIdx.x + 1] = d - i;
  }
  __syncthreads();
  const int i0 = s_bounds[0], j0 = s_bounds[1];
  const int i1 = s_bounds[2], j1 = s_bounds[3];

  // Row pointers rp(i0) .. rp(min(i1 + 1, m)) and products j0 .. j1-1.
  const int nr = min(i1 + 1, m) - i0 + 1;
  for (int k = threadIdx.x; k < nr; k += MBS) s_rp[k] = __ldg(rowptr + i0 + k);
  const T* __restrict__ vals = static_cast<const T*>(P.vals);
  const T* __restrict__ x = static_cast<const T*>(P.x);
  for (int k = threadIdx.x; k < j1 - j0; k += MBS) {
    const int j = j0 + k;
    s_prod[k] = ld_stream(vals + j) * ld_gather(x + ld_stream(P.cols + j));
  }
  __syncthreads();

  auto rp = [&](int r) { return r < m ? s_rp[r - i0] : nnz; };
  // This thread's items: diagonals [dt, dt_end).
  const int dt = min(d0 + int(threadIdx.x) * IPT, d1);
  const int dt_end = min(dt + IPT, d1);
  int i = merge_search(dt, max(i0, dt - j1), min(i1, dt - j0), rp);
  int j = dt - i;
  const int start_i = i;
  const bool mid_row = i < m && j > rp(i);
  T* __restrict__ y = static_cast<T*>(P.y);
  T sum = T(0);
  int first_row = -1;
  T first_val = T(0);
  for (int d = dt; d < dt_end; ++d) {
    if (i < m && j < rp(i + 1)) {
      sum += s_prod[j - j0];
      ++j;
    } else {
      if (i == start_i && mid_row) {
        first_row = i;
        first_val = sum;
      } else if (i < m) {
        y[i] = sum;
      }
      sum = T(0);
      ++i;
    }
  }
  s_crow[threadIdx.x] = i;  // row in progress after this thread's items
  s_cval[threadIdx.x] = sum;
  __syncthreads();

  if (first_row >= 0) {
    // Earlier threads of this CTA that ended inside first_row.
    int t = int(threadIdx.x) - 1;
    while (t >= 0 && s_crow[t] == first_row) --t;
    T acc = T(0);
    for (int u = t + 1; u < int(threadIdx.x); ++u) acc += s_cval[u];
    y[first_row] = acc + first_val;
  }
  if (threadIdx.x == MBS - 1) {
    // The CTA's carry: the run of trailing threads inside the last row.
    const int r = s_crow[MBS - 1];
    int t = MBS - 2;
    while (t >= 0 && s_crow[t] == r) --t;
    T acc = T(0);
    for (int u = t + 1; u < MBS; ++u) acc += s_cval[u];
    carry_row[blockIdx.x] = r < m ? r : -1;
    carry_val[blockIdx.x] = acc;
  }
}

// Adds the carries of CTAs that ended inside a row to that row, one thread
// per run of equal (rank, row) carries, summed in CTA order.
template <typename T>
__global__ void merge_fixup(const __grid_constant__ SpmvArgs a,
                            const int* __restrict__ carry_row,
                            const T* __restrict__ carry_val, int nblocks) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nblocks) return;
  const int r = carry_row[c];
  if (r < 0) return;
  const int p = find_part(a, c);
  if (c > a.part[p].block_begin && carry_row[c - 1] == r) return;  // not a run start
  const int end = a.part[p].block_begin + a.part[p].nblocks;
  T acc = T(0);
  int e = c;
  while (e < end && carry_row[e] == r) acc += carry_val[e++];
  T* y = static_cast<T*>(a.part[p].y);
  y[r] = y[r] + acc;
}

}  // namespace

void launch_merge(const SpmvLaunch& L, cudaStream_t stream, DevBuf& carry) {
  const DevCsr& C = *L.csr;
  const size_t es = dtype_size(L.dtype);
  SpmvArgs a;
  a.nparts = int(C.parts.size());
  int blocks = 0;
  for (int p = 0; p < a.nparts; ++p) {
    const DevPart& D = C.parts[p];
    PartArg& P = a.part[p];
    P.rowptr = C.rowptr.as<int32_t>() + D.rp_off;
    P.cols = L.cols + D.nz_off;
    P.vals = static_cast<const char*>(C.vals.ptr) + D.nz_off * es;
    P.x = L.x[p];
    P.y = L.y[p];
    P.xown = nullptr;
    P.nrows = D.nrows;
    P.block_begin = blocks;
    const int64_t items = int64_t(D.nrows) + D.nnz;
    require(items < (int64_t(1) << 31) - TILE, "spmv: rank too large for merge-path");
    const int64_t nb = (items + TILE - 1) / TILE;
    P.nblocks = int32_t(nb);
    P.ntiles = int32_t(nb);
    require(blocks + nb < (int64_t(1) << 31), "spmv: too many tiles");
    blocks += int(nb);
  }
  a.nblocks = blocks;
  if (blocks == 0) return;
  carry.reserve(size_t(blocks) * (sizeof(int) + 8) + 256);
  int* crow = carry.as<int>();
  void* cval = carry.as<char>() + ((size_t(blocks) * sizeof(int) + 255) / 256) * 256;
  if (L.dtype == SPMV_FLOAT64) {
    merge_kernel<double><<<blocks, MBS, 0, stream>>>(a, crow, static_cast<double*>(cval));
    merge_fixup<double><<<(blocks + 255) / 256, 256, 0, stream>>>(
        a, crow, static_cast<double*>(cval), blocks);
  } else {
    merge_kernel<float><<<blocks, MBS, 0, stream>>>(a, crow, static_cast<float*>(cval));
    merge_fixup<float><<<(blocks + 255) / 256, 256, 0, stream>>>(
        a, crow, static_cast<float*>(cval), blocks);
  }
  SPMVB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Allocation-free product: spmv_matrix_mult_noalloc.
//
// The merge-path product above keeps its per-CTA carries in a buffer that
// spmv_matrix_mult allocates (and grows) on demand.  This variant runs the
// same two kernels with the carries in a fixed file-scope device array, so a
// call allocates no device memory.  The array holds NOALLOC_MAX_TILES tiles of
// TILE (= 2048) merge items, i.e. rows + nonzeros of all ranks together up to
// 16384 * 2048 = 33,554,432; it is 192 KiB and stays resident on every
// device that loads this library until the process exits.
// ---------------------------------------------------------------------------
constexpr int NOALLOC_MAX_TILES = 16384;
constexpr size_t NOALLOC_VAL_OFFSET = size_t(NOALLOC_MAX_TILES) * sizeof(int);
static __device__ __align__(256) unsigned char
    g_noalloc_carry[NOALLOC_VAL_OFFSET + size_t(NOALLOC_MAX_TILES) * sizeof(double)];

namespace {

// Device address of g_noalloc_carry, looked up once per device (with that
// device current).  Host code must not use the symbol's name as an address:
// on the host it names a shadow object, not device memory.  The cached
// address belongs to the device's primary context as it was at the first
// call; a cudaDeviceReset ends that context (and every handle of this
// library made in it), so the cache is not meant to outlive one.
void* noalloc_scratch(int device) {
  static std::mutex mu;
  static std::vector<void*> addr;
  std::lock_guard<std::mutex> lock(mu);
  if (int(addr.size()) <= device) addr.resize(device + 1, nullptr);
  if (!addr[device]) {
    void* p = nullptr;
    SPMVB_CUDA(cudaGetSymbolAddress(&p, g_noalloc_carry));
    addr[device] = p;
  }
  return addr[device];
}

}  // namespace

}  // namespace spmvb

extern "C" int spmv_matrix_mult_noalloc(spmv_matrix A, const void* const* x,
                                        void* const* y) {
  using namespace spmvb;
  return guard([&] {
    require(A != nullptr, "spmv: Matrix is NULL");
    require(x != nullptr && y != nullptr, "spmv: vector array is NULL");
    require(A->dtype == SPMV_FLOAT64 || A->dtype == SPMV_FLOAT32,
            "spmv: only float64 and float32 products are implemented");
    const DevCsr& C = A->fwd;
    const size_t es = dtype_size(A->dtype);
    SpmvArgs a;
    a.nparts = int(C.parts.size());
    int64_t blocks = 0;
    for (int p = 0; p < a.nparts; ++p) {
      const DevPart& D = C.parts[p];
      if (D.ncols > 0) require(x[p] != nullptr, "spmv: x vector is NULL");
      if (D.nrows > 0) require(y[p] != nullptr, "spmv: y vector is NULL");
      const int64_t nb = (int64_t(D.nrows) + D.nnz + TILE - 1) / TILE;
      PartArg& P = a.part[p];
      P.rowptr = C.rowptr.as<int32_t>() + D.rp_off;
      P.cols = C.cols.as<int32_t>() + D.nz_off;
      P.vals = static_cast<const char*>(C.vals.ptr) + D.nz_off * es;
      P.x = x[p];
      P.y = y[p];
      P.xown = nullptr;
      P.nrows = D.nrows;
      P.block_begin = int32_t(std::min<int64_t>(blocks, NOALLOC_MAX_TILES));
      P.nblocks = int32_t(std::min<int64_t>(nb, NOALLOC_MAX_TILES));
      P.ntiles = P.nblocks;
      blocks += nb;
    }
    if (blocks > NOALLOC_MAX_TILES)
      fail(SPMV_ERROR_INVALID_ARGUMENT,
           "spmv_matrix_mult_noalloc: rows + nonzeros over all ranks (" +
               std::to_string(blocks) + " tiles of 2048) exceed the maximum of " +
               std::to_string(NOALLOC_MAX_TILES) + " tiles (33554432 items)");
    a.nblocks = int(blocks);
    A->comm->require_device();
    DeviceGuard dg(A->comm->device);
    if (blocks == 0) return;
    unsigned char* base = static_cast<unsigned char*>(noalloc_scratch(A->comm->device));
    int* crow = reinterpret_cast<int*>(base);
    cudaStream_t s = A->comm->stream;
    // Every CTA writes its carry slot before the fix-up reads it, so the
    // array needs no clearing between calls.
    if (A->dtype == SPMV_FLOAT64) {
      double* cval = reinterpret_cast<double*>(base + NOALLOC_VAL_OFFSET);
      merge_kernel<double><<<int(blocks), MBS, 0, s>>>(a, crow, cval);
      merge_fixup<double><<<int((blocks + 255) / 256), 256, 0, s>>>(a, crow, cval,
                                                                    int(blocks));
    } else {
      float* cval = reinterpret_cast<float*>(base + NOALLOC_VAL_OFFSET);
      merge_kernel<float><<<int(blocks), MBS, 0, s>>>(a, crow, cval);
      merge_fixup<float><<<int((blocks + 255) / 256), 256, 0, s>>>(a, crow, cval,
                                                                   int(blocks));
    }
    SPMVB_CUDA(cudaGetLastError());
  });
}
