// xi_kernels.cuh — device code of the XiEstimator pair count.
//
// Work decomposition (replaces XiEstimator::run's one-task-per-sky-cell
// ThreadPool loop, XiEstimator.cc:31-44 and 121-159):
//   1. a work item is one accepted sightline pair (i, j), i < j,
//      cos(theta_ij) > cos(max_ang), attributed to the cell of i;
//   2. persistent warps pull work items from a global counter; a warp sweeps
//      the N_i x N_j pixel-pair matrix of its item in chunks of 32 rows
//      (lane = row p1 of sightline i) along skewed diagonals: at step t lane L
//      looks at column p2 = t + L of sightline j, so all lanes see the same
//      line-of-sight separation at the same step and change bins together;
//   3. every pair is binned in FP32 (well-conditioned forms of the reference's
//      expressions); pairs within 2^-K bins of an edge are re-binned with the
//      reference's exact FP64 expression order;
//   4. each lane keeps a run of consecutive columns with the same bin; when the
//      bin changes, the run's contribution to all eight XiBin fields comes
//      from FP64 prefix sums of sightline j and is quantised to fixed point
//      (two u32 words per field); the lanes that close a run in the same slot
//      are summed with warp reductions (redux.sync) and one lane adds the sums
//      into the warp's private window in shared memory (u32 adds are native,
//      and aligned lanes would otherwise serialise on one address);
//   5. at the end of every 32-row chunk the window is added into per-cell
//      128-bit fixed-point accumulators in global memory, so every sum is
//      exact, deterministic and independent of scheduling.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "tos_common.h"

namespace tos {

constexpr uint32_t kInvalidKey = 0xFFFFFFFFu;
constexpr uint32_t kNoGrid = 0xFFFFFFFFu;  // sightline not contiguous on the common grid
constexpr int kPairWarps = 16;  // warps per CTA of the pair kernel
// u32 words per window slot: the three signed sums (didj, di, dj) as 22+22+rest
// bit words of a 62-bit fixed-point value, the four positive sums (wgt, wi,
// wj, z) as 22+rest bit words of a 42-bit value, the pair count and the
// number of contributions.
constexpr int kWinWords = 19;
constexpr int kSplit = 22;      // bits in each low word of the fixed-point split
constexpr int kSigned = 3;      // fields 0..2 are signed (3 words), 3..6 positive (2 words)
constexpr uint32_t kSlotCap = 1024u - 64u;  // contributions per slot before the window is emptied
// u64 words per (row, bin): field f's sum is hi[f] * 2^32 + lo[f], where
// lo[f] (word f) is the unsigned sum of the low 32 bits of every value added
// and hi[f] (word 7 + f) the signed sum of the values shifted right by 32.
// The format carries nothing between words, so an add is two fire-and-forget
// atomics; lo wraps after 2^32 adds to one (row, bin), which the host rules
// out before a run (kMaxAddsPerItemBin).  Word 14: the pair count.
constexpr int kAccWords = 16;
// Adds one sightline pair can make to one (row, bin, field), per pixel of its
// primary: at most two codes of a run-sweep lane per row and side, or three
// runs of one key per row (monotone segments) plus window flushes.
constexpr int kMaxAddsPerItemBin = 8;
constexpr double kMagic52 = 6755399441055744.0;  // 1.5 * 2^52
constexpr long long kMagic52Bits = 0x4338000000000000LL;

struct PairArgs {
  // catalogue
  const uint64_t* off;       // compact pixel offset of each sightline
  const uint32_t* npix;      // pixels per sightline
  const float* dist_pad;     // padded distances
  const float* loglam_pad;   // padded log10 wavelengths
  const PixPack* pack;       // padded (distance, weight, w*delta)
  const double* wd;          // w * delta (exact double) per pixel
  const float* w;            // weight per pixel
  const double4* prefix;     // per sightline, N+1 exclusive prefix sums of (wd, w, loglam)
  const float4* range;       // per sightline (dmin, dmax, lmin, lmax)
  const uint32_t* cell_idx;  // cell index of each sightline
  // accumulation row of a pair: the primary sightline's cell, or, when
  // row_key is set, the slot of the unordered pair of the two sightlines' keys
  const uint32_t* row_key;   // per sightline key, or null
  const uint32_t* slot_start;// per key a: slots [slot_start[a], slot_start[a+1]) of pairs (a, b >= a)
  const uint32_t* slot_key;  // per slot: its partner key b
  uint32_t spill_row;        // row of a pair whose keys have no slot (checked empty by the host)
  // work items
  const uint32_t* item_i;
  const uint32_t* item_j;
  const double* item_c;
  const uint32_t* item_sep;  // theta index (observing coordinates)
  unsigned long long n_items;
  unsigned long long* next_item;
  // grid (reference constants and FP32 fast-path maps t = x * inv + off)
  RefGrid g;
  float inv0f, off0f, inv1f, off1f;
  float n0f, n1f, n0p1f, n1p1f;
  float inv1sqf;             // Cartesian: u = X * inv1^2
  float mag0, mag1;          // 1.5 * 2^(23-K) for the two axes
  int k0, k1;                // fractional bits kept (edge half-width 2^-K)
  int bits0, bits1;          // bit patterns of mag0/mag1
  float r2_small;            // Polar: squared separations below this are re-binned in FP64
  float win_lim;             // |x1 - x2| >= win_lim (float) is always rejected
  double polar_r2;           // Polar: R^2 of the largest accepted r (with margin), or 0
  double polar_e2;           // Polar: bound on the float rounding of d1^2, plus margin
  int prune;                 // sightlines sorted: restrict columns to the r_par window
  // accumulation
  double scale[7];           // 2^F per field
  double scale_hi[7];        // 2^(F-44): wide (62-bit) conversion of a field
  int wide_all;              // every field uses the wide conversion (direct adds only)
  int run_split;             // the run-sweep kernel takes the items run_item() accepts; the
                             // pixel-pair kernel skips those and evaluates the rest exactly
  double run_amin;           // Cartesian: smallest 2(1 - cos theta) the run sweep accepts
  const float* thr;          // run sweep: first-axis thresholds T[0..n0]
  // boundary table of the catalogue's common first-axis grid (grid sweep)
  const uint16_t* gq;        // [ng][2 n0 + 2]: a grid row's run boundaries in column order
                             // (k_grid_table, engine.cu)
  const uint32_t* gfirst;    // per sightline: grid index of pixel 0, or kNoGrid
  int ng;                    // grid values
  int grid_split;            // the grid kernel takes the run items whose sightlines are on the grid
  int diag_split;            // Polar: the diagonal-sweep kernel takes the items whose z index is
                             // constant; the pixel-pair kernel evaluates the rest exactly
  int win_w1;                // window width along axis 1 (Cartesian)
  int win_slots;             // slots per warp window
  unsigned long long* acc;   // [n_rows][ntotal][kAccWords] 128-bit fixed point
  unsigned long long* counters;  // [0] evaluated pairs [1] rechecks [2] overflow pairs
                                 // [3] direct runs [6] window flushes
  int force_exact;           // evaluate every pixel pair with the FP64 reference
};

// Accumulation row of sightline pair (i, j).
__device__ __forceinline__ uint32_t dest_row(const PairArgs& A, uint32_t i, uint32_t j) {
  if (A.row_key == nullptr) return A.cell_idx[i];
  uint32_t a = A.row_key[i], b = A.row_key[j];
  if (a > b) {
    const uint32_t t = a;
    a = b;
    b = t;
  }
  const uint32_t e = A.slot_start[a + 1];
  for (uint32_t q = A.slot_start[a]; q < e; ++q)
    if (A.slot_key[q] == b) return q;
  return A.spill_row;
}

// Launch the persistent pixel-pair kernel (coordinate type from a.g/a.* fields).
cudaError_t launch_pair_kernel(const PairArgs& a, int coord, bool exact0, bool minpos, int grid,
                               cudaStream_t stream);
size_t pair_kernel_smem(int win_slots);

// Launch the persistent grid-sweep kernel (xi_grid.cu) over the items that
// run_item() accepts and whose two sightlines lie on the common grid.
// ctas_per_sm: CTAs per SM (0: as many as fit); with max_out set, only
// report that limit.
cudaError_t launch_grid_kernel(const PairArgs& a, int coord, bool minpos, int num_sms, int ctas_per_sm,
                               cudaStream_t stream, int* max_out = nullptr);

// Launch the persistent diagonal-sweep kernel (xi_diag.cu) over the Polar
// items that diag_item() accepts (every field on the wide scale).
cudaError_t launch_diag_kernel(const PairArgs& a, bool minpos, int num_sms, int ctas_per_sm, cudaStream_t stream,
                               int* max_out = nullptr);

// Launch the persistent run-sweep kernel (xi_runs.cu) over the items that
// run_item() accepts: Cartesian and observing coordinates, catalogue sorted
// by distance and loglam, a.thr set and every field on the wide scale.
cudaError_t launch_run_kernel(const PairArgs& a, int coord, bool minpos, int num_sms,
                              cudaStream_t stream);

}  // namespace tos
