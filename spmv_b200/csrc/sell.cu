// SELL-32 (sliced ELLPACK) copy of a matrix, built on the device from its CSR
// (the product kernel itself is sell_for_rows in spmv_kernel.cuh).
//
// Per rank, rows are cut into slices of 32 consecutive rows (no reordering,
// so y is written in row order); slice s is w_s = max row length in the slice
// wide and stored column-major: entry k of row 32s+l at soff[s] + 32k + l,
// padding columns -1 with value 0.  For matrices with even row lengths (the
// stencils) the padding is about 1%, the row pointers are no longer read, and
// each lane's loads are independent of each other.
#include <algorithm>
#include <cstdlib>

#include "internal.h"
#include "spmv_kernel.cuh"
#include "sell_staged.cuh"

static_assert(spmvb::SolverStaged::BS == spmvb::kStagedThreads,
              "the staged product's CTA size as reported to callers");

namespace spmvb {

namespace {

inline int64_t align_up(int64_t v, int64_t a) { return (v + a - 1) / a * a; }

// One thread per (padded) row: copies the row's entries into its SELL
// column and pads the rest of the slice width (column `pad`, value 0).
template <typename T, typename CI>
__global__ void csr_to_sell(const int32_t* __restrict__ rowptr,
                            const CI* __restrict__ cols_in,
                            const T* __restrict__ vals_in,
                            const int32_t* __restrict__ soff, int nrows,
                            int nslices, CI* __restrict__ cols_out,
                            T* __restrict__ vals_out, CI pad) {
  const int64_t total = int64_t(nslices) * 32;
  for (int64_t r = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; r < total;
       r += int64_t(gridDim.x) * blockDim.x) {
    const int s = int(r >> 5), l = int(r & 31);
    const int o = soff[s];
    const int w = (soff[s + 1] - o) >> 5;
    const int base = r < nrows ? rowptr[r] : 0;
    const int len = r < nrows ? rowptr[r + 1] - base : 0;
    for (int k = 0; k < w; ++k) {
      const int idx = o + k * 32 + l;
      if (k < len) {
        cols_out[idx] = cols_in[base + k];
        if (vals_out) vals_out[idx] = vals_in[base + k];
      } else {
        cols_out[idx] = pad;
        if (vals_out) vals_out[idx] = T(0);
      }
    }
  }
}

__global__ void sell_to_float(const double* __restrict__ in, float* __restrict__ out,
                              int64_t n) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = float(in[i]);
}

// Scatters every rank's CSR (cols_in, optional vals_in) into SELL arrays.
template <typename T, typename CI>
void scatter_t(DevCsr& C, const CI* cols_in, CI* cols_out, bool with_vals, CI pad, int grid,
               cudaStream_t s) {
  for (size_t r = 0; r < C.parts.size(); ++r) {
    const DevPart& D = C.parts[r];
    const int nslices = (D.nrows + 31) / 32;
    if (nslices == 0) continue;
    const int32_t* rp = C.rowptr.as<int32_t>() + D.rp_off;
    const int32_t* so = C.sell_off.as<int32_t>() + D.sl_off;
    csr_to_sell<T, CI><<<grid, 256, 0, s>>>(
        rp, cols_in + D.nz_off, C.vals.as<T>() + D.nz_off, so, D.nrows, nslices,
        cols_out + D.sz_off, with_vals ? C.sell_vals.as<T>() + D.sz_off : nullptr, pad);
    SPMVB_CUDA(cudaGetLastError());
  }
}

template <typename CI>
void scatter_all(spmv_matrix A, DevCsr& C, const CI* cols_in, CI* cols_out,
                 bool with_vals, CI pad, cudaStream_t s) {
  const int grid = std::max(1, A->comm->num_sms) * 8;
  switch (A->dtype) {
    case SPMV_FLOAT64: scatter_t<double>(C, cols_in, cols_out, with_vals, pad, grid, s); break;
    case SPMV_FLOAT32: scatter_t<float>(C, cols_in, cols_out, with_vals, pad, grid, s); break;
    case SPMV_COMPLEX128: scatter_t<c128>(C, cols_in, cols_out, with_vals, pad, grid, s); break;
    case SPMV_COMPLEX64: scatter_t<c64>(C, cols_in, cols_out, with_vals, pad, grid, s); break;
  }
}

}  // namespace

// Padded SELL-32 size of a rank's block (host, from its row pointers).
int64_t sell_padded_size(const std::vector<int32_t>& rowptr, int32_t nrows,
                         std::vector<int32_t>* soff) {
  const int nslices = (nrows + 31) / 32;
  if (soff) soff->assign(size_t(nslices) + 1, 0);
  int64_t total = 0;
  for (int s = 0; s < nslices; ++s) {
    int w = 0;
    const int r1 = std::min(nrows, (s + 1) * 32);
    for (int r = s * 32; r < r1; ++r) w = std::max(w, rowptr[r + 1] - rowptr[r]);
    total += int64_t(w) * 32;
    if (soff) (*soff)[s + 1] = int32_t(total);
  }
  return total;
}

void build_sell(spmv_matrix A, DevCsr& C, cudaStream_t stream) {
  if (C.sell_built) return;
  require(&C == &A->fwd || (&C == &A->trn && A->trn_built),
          "spmv: SELL layout of an unknown matrix copy");
  const auto& h_rowptr = &C == &A->fwd ? A->h_rowptr : A->h_trn_rowptr;
  const int P = A->comm->size;
  const size_t es = dtype_size(A->dtype);
  std::vector<int32_t> all_off;
  int64_t sz = 0;
  for (int r = 0; r < P; ++r) {
    DevPart& D = C.parts[r];
    std::vector<int32_t> soff;
    const int64_t padded = sell_padded_size(h_rowptr[r], D.nrows, &soff);
    require(padded < (int64_t(1) << 31), "spmv: rank too large for 32-bit SELL offsets");
    D.sl_off = int64_t(all_off.size());
    D.sz_off = sz;
    D.snnz = padded;
    all_off.insert(all_off.end(), soff.begin(), soff.end());
    sz = align_up(sz + padded, 32);
  }
  C.sl_total = int64_t(all_off.size());
  C.sz_total = std::max<int64_t>(sz, 32);
  C.sell_off.reserve(sizeof(int32_t) * std::max<size_t>(all_off.size(), 1));
  if (!all_off.empty())
    SPMVB_CUDA(cudaMemcpy(C.sell_off.ptr, all_off.data(), sizeof(int32_t) * all_off.size(),
                          cudaMemcpyHostToDevice));
  C.sell_cols.reserve(sizeof(int32_t) * C.sz_total);
  C.sell_vals.reserve(es * C.sz_total);
  scatter_all<int32_t>(A, C, C.cols.as<int32_t>(), C.sell_cols.as<int32_t>(), true, -1,
                       stream);
  SPMVB_CUDA(cudaStreamSynchronize(stream));
  C.h_sell_off = std::move(all_off);
  C.sell_built = true;
}

const DevCsr::StagedTable& staged_table(DevCsr& C, int entry_bytes, int max_entries) {
  require(C.sell_built, "spmv: staged tiles need the SELL layout");
  require(entry_bytes >= 6 && entry_bytes <= 12 && entry_bytes % 2 == 0,
          "spmv: staged entry size must be 6, 8, 10 or 12 bytes");
  DevCsr::StagedTable& t = C.staged[(entry_bytes - 6) / 2];
  if (t.built) return t;
  // Tiles of whole slices: as many consecutive slices of one rank as fit
  // max_entries entries, at most STAGED_MAX_SLICES.
  std::vector<StagedDesc> tiles;
  bool ok = true;
  for (size_t r = 0; r < C.parts.size() && ok; ++r) {
    const DevPart& D = C.parts[r];
    const int nslices = (D.nrows + 31) / 32;
    const int32_t* so = C.h_sell_off.data() + D.sl_off;
    int s = 0;
    while (s < nslices) {
      int e = s;
      while (e < nslices && e - s < STAGED_MAX_SLICES && so[e + 1] - so[s] <= max_entries) ++e;
      if (e == s) {  // one slice wider than a stage
        ok = false;
        break;
      }
      StagedDesc d{};
      d.rank = int32_t(r);
      d.nslices = e - s;
      d.s0 = s;
      d.e0 = so[s];
      d.n = so[e] - so[s];
      for (int j = 0; j <= e - s; ++j) d.off[j] = so[s + j] - so[s];
      tiles.push_back(d);
      s = e;
    }
  }
  t.built = true;
  t.ok = ok && !tiles.empty();
  if (!t.ok) return t;
  t.ntiles = int(tiles.size());
  t.rows.reserve(tiles.size());
  for (const StagedDesc& d : tiles) t.rows.push_back({d.rank, d.s0, d.nslices});
  t.desc.reserve(sizeof(StagedDesc) * tiles.size());
  SPMVB_CUDA(cudaMemcpy(t.desc.ptr, tiles.data(), sizeof(StagedDesc) * tiles.size(),
                        cudaMemcpyHostToDevice));
  return t;
}

void refresh_sell_values(spmv_matrix A) {
  DevCsr& C = A->fwd;
  if (!C.sell_built) return;
  // Same pattern: re-scatter the values (and columns, unchanged) in place.
  scatter_all<int32_t>(A, C, C.cols.as<int32_t>(), C.sell_cols.as<int32_t>(), true, -1,
                       A->comm->stream);
  C.sell_vals32.release();
  SPMVB_CUDA(cudaStreamSynchronize(A->comm->stream));
}

void build_sell_global(spmv_matrix A) {
  DevCsr& C = A->fwd;
  if (C.sell_cols_global.ptr) return;
  build_global_cols(A);
  build_sell(A, C, A->comm->stream);
  C.sell_cols_global.reserve(sizeof(int32_t) * C.sz_total);
  scatter_all<int32_t>(A, C, C.cols_global.as<int32_t>(), C.sell_cols_global.as<int32_t>(),
                       false, -1, A->comm->stream);
  if (C.d16) {
    C.sell_d16_global.reserve(sizeof(int16_t) * C.sz_total);
    scatter_all<int16_t>(A, C, C.d16_global.as<int16_t>(), C.sell_d16_global.as<int16_t>(),
                         false, int16_t(-32768), A->comm->stream);
  }
  SPMVB_CUDA(cudaStreamSynchronize(A->comm->stream));
}

bool d16_enabled() {
  const char* v = std::getenv("SPMV_B200_D16");
  return !(v && v[0] == '0');
}

void use_d16(SpmvArgs& a, const DevCsr& C, bool sell) {
  require(C.d16, "spmv: no 16-bit column offsets for this matrix");
  const int16_t* base = sell ? C.sell_d16_global.as<int16_t>() : C.d16_global.as<int16_t>();
  require(base != nullptr, "spmv: 16-bit offsets not built for this layout");
  for (int p = 0; p < a.nparts; ++p) {
    const DevPart& D = C.parts[p];
    a.part[p].cols = reinterpret_cast<const int32_t*>(base + (sell ? D.sz_off : D.nz_off));
  }
}

void build_sell_vals32(spmv_matrix A) {
  DevCsr& C = A->fwd;
  if (C.sell_vals32.ptr) return;
  require(A->dtype == SPMV_FLOAT64, "spmv: FP32 copy needs an FP64 matrix");
  build_sell(A, C, A->comm->stream);
  C.sell_vals32.reserve(sizeof(float) * C.sz_total);
  sell_to_float<<<std::max(1, A->comm->num_sms) * 8, 256, 0, A->comm->stream>>>(
      C.sell_vals.as<double>(), C.sell_vals32.as<float>(), C.sz_total);
  SPMVB_CUDA(cudaGetLastError());
  SPMVB_CUDA(cudaStreamSynchronize(A->comm->stream));
}

int fill_sell_args(SpmvArgs& a, const DevCsr& C, const int32_t* cols, const void* vals,
                   size_t es, const void* const* x, void* const* y,
                   const void* const* xown, int BS, int max_blocks) {
  a.nparts = int(C.parts.size());
  const int slices_per_tile = BS / 32;
  int64_t tiles_total = 0;
  for (const DevPart& D : C.parts)
    tiles_total += ((D.nrows + 31) / 32 + slices_per_tile - 1) / slices_per_tile;
  int blocks = 0;
  int64_t row0 = 0;
  for (int p = 0; p < a.nparts; ++p) {
    const DevPart& D = C.parts[p];
    PartArg& P = a.part[p];
    P.row0 = int32_t(row0);
    row0 += D.nrows;
    P.rowptr = C.sell_off.as<int32_t>() + D.sl_off;
    P.cols = cols + D.sz_off;
    P.vals = static_cast<const char*>(vals) + D.sz_off * es;
    P.x = x[p];
    P.y = y[p];
    P.xown = xown ? xown[p] : nullptr;
    P.nrows = D.nrows;
    P.block_begin = blocks;
    const int64_t tiles = ((D.nrows + 31) / 32 + slices_per_tile - 1) / slices_per_tile;
    int64_t nb = tiles;
    if (tiles_total > max_blocks)
      nb = std::max<int64_t>(tiles > 0 ? 1 : 0,
                             (tiles * max_blocks + tiles_total - 1) / tiles_total);
    P.ntiles = int32_t(tiles);
    P.nblocks = int32_t(nb);
    blocks += int(nb);
  }
  a.nblocks = blocks;
  return blocks;
}

namespace {

template <typename T, int BS, bool D16 = false, bool KEEP = false>
void launch_sell_u(const SpmvArgs& a, int U, cudaStream_t s) {
  switch (U) {
    case 1: spmv_sell_kernel<T, BS, 1, D16, KEEP><<<a.nblocks, BS, 0, s>>>(a); break;
    case 2: spmv_sell_kernel<T, BS, 2, D16, KEEP><<<a.nblocks, BS, 0, s>>>(a); break;
    case 4: spmv_sell_kernel<T, BS, 4, D16, KEEP><<<a.nblocks, BS, 0, s>>>(a); break;
    case 8: spmv_sell_kernel<T, BS, 8, D16, KEEP><<<a.nblocks, BS, 0, s>>>(a); break;
    case 16: spmv_sell_kernel<T, BS, 16, D16, KEEP><<<a.nblocks, BS, 0, s>>>(a); break;
    default: fail(SPMV_ERROR_INVALID_ARGUMENT, "spmv: SELL width must be 1, 2, 4, 8 or 16");
  }
}

}  // namespace

void launch_sell_args(const SpmvArgs& a, spmv_dtype dtype, int U, int BS,
                      cudaStream_t stream, bool d16, bool keep) {
  if (a.nblocks == 0) return;
  if (d16 || keep) {
    require(BS == 256, "spmv: solver-form products run 256 threads per CTA");
    const bool f64 = dtype == SPMV_FLOAT64;
    if (d16 && keep)
      f64 ? launch_sell_u<double, 256, true, true>(a, U, stream)
          : launch_sell_u<float, 256, true, true>(a, U, stream);
    else if (d16)
      f64 ? launch_sell_u<double, 256, true, false>(a, U, stream)
          : launch_sell_u<float, 256, true, false>(a, U, stream);
    else
      f64 ? launch_sell_u<double, 256, false, true>(a, U, stream)
          : launch_sell_u<float, 256, false, true>(a, U, stream);
  } else if (dtype == SPMV_FLOAT64) {
    switch (BS) {
      case 128: launch_sell_u<double, 128>(a, U, stream); break;
      case 256: launch_sell_u<double, 256>(a, U, stream); break;
      default: launch_sell_u<double, 512>(a, U, stream); break;
    }
  } else {
    switch (BS) {
      case 128: launch_sell_u<float, 128>(a, U, stream); break;
      case 256: launch_sell_u<float, 256>(a, U, stream); break;
      default: launch_sell_u<float, 512>(a, U, stream); break;
    }
  }
  SPMVB_CUDA(cudaGetLastError());
}

void launch_sell(const SpmvLaunch& L, const int32_t* sell_cols, cudaStream_t stream) {
  const DevCsr& C = *L.csr;
  const int U = L.width > 0 ? L.width : 8;
  const int BS = L.block > 0 ? L.block : 256;
  const size_t es = dtype_size(L.dtype);
  SpmvArgs a;
  fill_sell_args(a, C, sell_cols, C.sell_vals.ptr, es, L.x, L.y, nullptr, BS,
                 max_blocks_for(L.num_sms, BS));
  if (a.nblocks == 0) return;
  auto by_bs = [&](auto tag) {
    using T = decltype(tag);
    switch (BS) {
      case 128: launch_sell_u<T, 128>(a, U, stream); break;
      case 256: launch_sell_u<T, 256>(a, U, stream); break;
      case 512: launch_sell_u<T, 512>(a, U, stream); break;
    }
  };
  switch (L.dtype) {
    case SPMV_FLOAT64: by_bs(double{}); break;
    case SPMV_FLOAT32: by_bs(float{}); break;
    case SPMV_COMPLEX128: by_bs(c128{}); break;
    case SPMV_COMPLEX64: by_bs(c64{}); break;
  }
  SPMVB_CUDA(cudaGetLastError());
}

StagedShape staged_shape(const void* fn, int entry_bytes, int ntiles, int num_sms) {
  StagedShape sh;
  sh.smem = SolverStaged::smem_bytes(entry_bytes);
  SPMVB_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, sh.smem));
  int occ = 0;
  SPMVB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, SolverStaged::BS, sh.smem));
  require(occ > 0, "spmv: staged product does not fit on an SM");
  sh.grid = std::max(1, std::min(ntiles, std::max(1, num_sms) * occ));
  return sh;
}

namespace {

template <typename T, typename CI, int U>
__global__ void __launch_bounds__(SolverStaged::BS, SolverStaged::MINB)
    spmv_staged_kernel(const __grid_constant__ SpmvArgs a, const StagedDesc* tiles, int ntiles,
                       int* err) {
  sell_staged_rows<SolverStaged, T, CI, U>(
      a, tiles, ntiles, err,
      [](const PartArg& P, int row, T sum) { static_cast<T*>(P.y)[row] = sum; }, XGather<T>());
}

template <typename T>
void launch_staged_t(const SpmvLaunch& L, const SpmvArgs& a, const DevCsr::StagedTable& t,
                     int U, cudaStream_t s) {
  const int u = staged_width(U);
  const void* fn = u == 9   ? (const void*)spmv_staged_kernel<T, int32_t, 9>
                   : u == 8 ? (const void*)spmv_staged_kernel<T, int32_t, 8>
                   : u == 7 ? (const void*)spmv_staged_kernel<T, int32_t, 7>
                   : u == 5 ? (const void*)spmv_staged_kernel<T, int32_t, 5>
                            : (const void*)spmv_staged_kernel<T, int32_t, 4>;
  const StagedShape sh = staged_shape(fn, int(sizeof(T)) + 4, t.ntiles, L.num_sms);
  const StagedDesc* tiles = t.desc.as<StagedDesc>();
  int ntiles = t.ntiles;
  int* err = L.err;
  void* args[] = {const_cast<SpmvArgs*>(&a), &tiles, &ntiles, &err};
  launch_pdl(fn, dim3(sh.grid), dim3(SolverStaged::BS), size_t(sh.smem), s, args);
}

}  // namespace

void launch_staged(const SpmvLaunch& L, cudaStream_t stream) {
  DevCsr& C = const_cast<DevCsr&>(*L.csr);
  require(C.sell_built, "spmv: staged product needs the SELL layout");
  const size_t es = dtype_size(L.dtype);
  const int eb = int(es) + 4;
  const DevCsr::StagedTable& t = staged_table(C, eb, SolverStaged::max_entries(eb));
  if (!t.ok) {
    SpmvLaunch Ls = L;
    Ls.width = 0;  // the staged width means gathers in flight, not SELL loads
    launch_sell(Ls, C.sell_cols.as<int32_t>(), stream);
    return;
  }
  SpmvArgs a;
  fill_sell_args(a, C, C.sell_cols.as<int32_t>(), C.sell_vals.ptr, es, L.x, L.y, nullptr, 256,
                 max_blocks_for(L.num_sms, 256));
  const int U = L.width > 0 ? L.width : 8;
  if (L.dtype == SPMV_FLOAT64)
    launch_staged_t<double>(L, a, t, U, stream);
  else
    launch_staged_t<float>(L, a, t, U, stream);
}

}  // namespace spmvb
