// Batched solver internals shared by the planner (batch_plan.cpp), the API
// and autotuner (batch.cu) and the kernel instantiations (batch_f32.cu,
// batch_f64.cu).  No counterpart in the reference: the batch builds on
// spmv::cg (cg.cpp:11-83) and Matrix::operator* (Matrix.cpp:199-204).
#pragma once

#include <cstdint>
#include <vector>

#include "internal.h"

namespace spmvb {
namespace bat {

constexpr int NT = 512;        // threads per CTA
constexpr int NW = NT / 32;    // warps per CTA
constexpr int BW = 32;         // columns of the block of right-hand sides (padded)
constexpr int MAXQ = 32;       // units of one CTA range handled per pass
constexpr int NSUM = 3;        // sums one reduction carries at most
constexpr int SIGMA = 1024;    // rows per length-sorting window
constexpr int MAX_UNITS = 8192;

// A scheduling unit: one system with its single right-hand side (kind 0), or
// the block of up to BW right-hand sides of one system (kind 1).
struct Unit {
  int64_t row0;      // first row in the unit's vectors (kind 0: the concatenated
                     // single vectors; kind 1: row 0 of the block vectors)
  int64_t slice0;    // kind 0: first slice in the slice table
  int64_t part_off;  // first partial-sum slot (doubles)
  int32_t n;         // rows
  int32_t nslices;   // kind 0: padded rows / 32; kind 1: padded rows
  int32_t kind;
  int32_t slot0;     // first recurrence slot
  int32_t sys;       // user's system index
  int32_t pad;
};

// One CG recurrence (a system's right-hand side, or one block column).
struct Slot {
  double rr0, rr, rr_max, rr_true, rr_prev, alpha, beta, c;
  int its, refs, status, active, converged, refine_at, pad0, pad1;
};

// Unit-level flags, kept by the CTA that completes each reduction.
struct UnitState {
  int active;     // some slot still iterating
  int refine_at;  // lockstep iteration of the unit's latest refinement
};

// Tile weights per phase, in eighths of a single unit's tile (which weighs
// 8): the block unit's per phase (c2: its refinement) and a single unit's
// refinement tile.
struct Weights {
  int blk_a, blk_b, blk_c, blk_c2, one_c2;
};

// Kernel arguments (T: inner precision; CI: int16_t row offsets or int32_t
// unit-local columns).
template <typename T, typename CI>
struct Args {
  const Unit* units;
  int nunits;
  int kmax;
  double rtol2, delta2;
  int tile_slices;                 // slices per single-unit tile (= block rows per tile)
  Weights w;                       // the block's tile weights
  int nrhs;                        // block right-hand sides (0: no block in this solve)
  // Single units (SELL-32 slices, rows in the planned order).
  const int64_t* soff;             // entry offset of each slice (+1 at the end)
  const int2* sbound;              // per slice: smallest and largest unit-local column
  int win_cap;                     // rows of p a shared-memory window holds
  const T* vals;                   // inner-precision values
  const double* vals64;            // FP64 values
  const CI* idx;
  const int32_t* perm;             // internal row -> user row (-1: padding)
  T *r, *p, *y, *d;
  double *x, *b;
  // Block (CSR, rows in the planned order; vectors n x BW row-major).
  const int32_t* brp;
  const int32_t* bcol;
  const T* bval;
  const double* bval64;
  const int32_t* bperm;
  T *rB, *pB, *yB, *dB;
  double *xB, *bB;
  // The caller's vectors.
  const double* const* b_user;
  double* const* x_user;
  const double* B_user;
  double* X_user;
  // Solve state.
  Slot* slots;
  UnitState* ust;
  unsigned int* tickets;
  double* parts;
  unsigned long long* bar;
  int* err;
  unsigned long long limit_ns;
  unsigned long long* prof;  // phase timeline (NULL: not recorded)
  int prof_cap;
};

// The batch's device layout, built once by the planner.
struct Plan {
  int nsys = 0;
  std::vector<int32_t> n;            // rows per system
  std::vector<int64_t> nnz;          // entries per system
  int64_t rows_pad = 0;              // rows of the single vectors (all units, padded)
  int64_t nslices = 0;
  int64_t entries = 0;               // stored SELL entries (with padding)
  int64_t nnz_total = 0;
  int max_width = 0;
  bool fits16 = true;                // every row offset fits int16
  std::vector<int64_t> row0, slice0; // per system
  // Host copies (uploaded, then freed).
  std::vector<int64_t> soff;
  std::vector<int32_t> sbound;       // 2 per slice: min and max unit-local column
  std::vector<float> vals32;
  std::vector<double> vals64;
  std::vector<int16_t> off16;
  std::vector<int32_t> col32;
  std::vector<int32_t> perm;
  std::vector<std::vector<int32_t>> sys_perm;  // per system: new -> old row
};

// Host planning of one batch: per system a reverse Cuthill-McKee order,
// rows sorted by length (descending, stable) within windows of SIGMA rows,
// and the SELL-32 layout of the reordered matrix.
void plan_batch(int nsys, const int32_t* n, const int32_t* const* rowptr,
                const int32_t* const* colind, const double* const* values, Plan& P);

// Reverse Cuthill-McKee order of one symmetric pattern (new -> old).
std::vector<int32_t> rcm_order(int32_t n, const int32_t* rowptr, const int32_t* colind);

struct LaunchCfg {
  int cps = 2;           // CTAs per SM
  int tile_slices = 8;   // rows per warp tile: 32 x tile_slices (single units)
  int rhs_rows = 1;      // block rows per warp step (lanes per row 32 / rhs_rows)
  int window = 1;        // products stage the gathered vector in shared memory
};

// Launch of the lockstep kernel (cooperative; the grid must be resident):
// args points to Args<float|double, int16_t|int32_t> per d16.  Returns false
// when the configuration cannot be made resident; dry: only that check.
bool launch_f32(const void* args, bool d16, const LaunchCfg& c, int num_sms, cudaStream_t s,
                bool dry);
bool launch_f64(const void* args, bool d16, const LaunchCfg& c, int num_sms, cudaStream_t s,
                bool dry);

}  // namespace bat
}  // namespace spmvb
