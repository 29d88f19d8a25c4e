// engine_internal.h — engine/catalogue objects and helpers shared by the
// translation units of the pair-counting engine.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "tos_common.h"

namespace tos {

// ---- error plumbing -------------------------------------------------------
void set_error(const std::string& msg);
tos_status fail(tos_status s, const std::string& msg);

#define TOS_CUDA_TRY(expr)                                                                   \
  do {                                                                                       \
    cudaError_t e_ = (expr);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return ::tos::fail(e_ == cudaErrorMemoryAllocation ? TOS_ERR_OOM : TOS_ERR_CUDA,        \
                         std::string(#expr) + ": " + cudaGetErrorString(e_));               \
  } while (0)

#define TOS_TRY(expr)                 \
  do {                                \
    tos_status s_ = (expr);           \
    if (s_ != TOS_OK) return s_;      \
  } while (0)

// Device buffer owned by the engine (freed on destruction / resize).
template <class T>
struct DevBuf {
  T* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { release(); }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    n = 0;
  }
  tos_status alloc(size_t count) {
    if (count <= n && p) return TOS_OK;
    release();
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc((void**)&p, count * sizeof(T));
    if (e != cudaSuccess) {
      p = nullptr;
      return fail(TOS_ERR_OOM, std::string("cudaMalloc failed: ") + cudaGetErrorString(e));
    }
    n = count;
    return TOS_OK;
  }
  size_t bytes() const { return p ? n * sizeof(T) : 0; }
};

}  // namespace tos

namespace tos {

// Device scratch of one pair count, kept between runs so that a caller that
// runs again (a server slot, the catalogue's own runs) allocates only when a
// run needs more than before.
struct Workspace {
  DevBuf<uint32_t> d_nb_count, d_nb_start, d_nb;  // cell neighbour CSR (per sightline for plate cells)
  DevBuf<unsigned long long> d_plate_edge;        // plate-ring tests within the margin (plate cells)
  DevBuf<uint32_t> d_cnt;                         // per primary: accepted pairs
  DevBuf<unsigned long long> d_cand;              // per primary candidates (for stats)
  DevBuf<uint32_t> d_item_off;
  DevBuf<uint32_t> d_item_i, d_item_j, d_item_sep;
  DevBuf<double> d_item_c;
  DevBuf<unsigned long long> d_cell_pairs;        // per cell sum N_i N_j
  DevBuf<unsigned long long> d_acc;               // [n_rows][n_bins][16] 128-bit fixed point
  DevBuf<tos_xibin> d_out;                        // combined / per row output
  DevBuf<unsigned long long> d_counters;          // misc counters
  DevBuf<float> d_thr;                            // first-axis thresholds of the run sweep
  DevBuf<uint16_t> d_gq;                          // boundary table of the current call
  DevBuf<unsigned char> d_cub_tmp;
  // the last completed per-cell run in d_acc
  bool last_valid = false;
  uint32_t last_nb = 0;
  double last_inv_scale[7] = {};                  // fixed point -> value, per field
  // bytes held by the buffers above
  size_t bytes() const;
};

}  // namespace tos

struct tos_engine {
  int device = 0;
  int num_sms = 0;
  size_t smem_optin = 0;  // opt-in shared memory per block (bytes)
  cudaStream_t stream = nullptr;
  cudaEvent_t ev[8] = {};
  std::mutex mu;
  // launch shapes picked by the autotuner (tos_brute_tune), by bin count:
  // (kernel variant, warps per CTA)
  std::mutex tune_mu;
  std::map<int, std::pair<int, int>> brute_tuned;
  // CTAs per SM of the dominant pair-count kernel picked by TOS_XI_TUNE, by
  // (coordinate type, total bins)
  std::map<std::pair<int, int>, int> xi_tuned;
};

struct tos_catalog {
  tos_engine* eng = nullptr;
  int device = 0;
  size_t n_los = 0, n_pix = 0;
  int order = 0;                    // HEALPix order (-1: plate cells)
  int64_t nside = 0;
  double cell_sr = 0;               // solid angle of a cell (work estimates)
  // plate cells (tos_catalog_create_plates): the platelist's plates in
  // ascending id (a repeated id: its last row) and their centres
  bool plates = false;
  std::vector<int32_t> plate_ids;
  std::vector<double4> plate_trig;  // sin_dec, cos_dec, sin_ra, cos_ra of the centre
  tos::DevBuf<int32_t> d_plate_ids;
  tos::DevBuf<double4> d_plate_trig;
  tos::DevBuf<int64_t> d_cells;     // `cells` on the device (plate-cell lookup)
  // host-side index
  std::vector<int64_t> cell_of;     // cell id of each sightline: group << 32 | HEALPix pixel (or plate)
  std::vector<int64_t> cells;       // occupied cells, ascending
  std::vector<double4> caps;        // per cell: unit centre xyz and angular radius of its members
  std::vector<uint32_t> groups;     // distinct sightline groups, ascending
  std::vector<uint32_t> group_cell_start;  // CSR (n_groups+1) into cells
  std::vector<uint32_t> cell_idx;   // per sightline: index into `cells`
  std::vector<uint32_t> cell_start; // CSR (n_cells+1) into members
  std::vector<uint32_t> members;    // sightlines grouped by cell, ascending index within a cell
  std::vector<uint32_t> npix;       // pixels per sightline
  std::vector<uint64_t> off;        // compact pixel offset per sightline
  // device data
  tos::DevBuf<double4> d_trig;      // sin_dec, cos_dec, sin_ra, cos_ra
  tos::DevBuf<double4> d_cap;       // cell cap: unit centre xyz, angular radius
  tos::DevBuf<uint2> d_cell_grange; // per cell: [first, end) cells of its group
  tos::DevBuf<uint32_t> d_group_cell_start;  // group_cell_start on the device
  tos::DevBuf<uint32_t> d_cell_idx, d_cell_start, d_members, d_npix;
  tos::DevBuf<uint64_t> d_off;      // compact offset (per-pixel double/float arrays)
  tos::DevBuf<tos_pixel> d_raw;     // uploaded pixels, compact order
  tos::DevBuf<float> d_dist_pad, d_loglam_pad;
  tos::DevBuf<tos::PixPack> d_pack;  // padded like d_dist_pad
  tos::DevBuf<double> d_wd;         // w*delta per pixel, exact in double
  tos::DevBuf<float> d_w;           // weight per pixel
  tos::DevBuf<double4> d_prefix;    // per sightline N+1 exclusive prefix sums of (w*delta, w, loglam)
  tos::DevBuf<float4> d_range;      // per sightline (dmin, dmax, lmin, lmax)
  tos::DevBuf<unsigned int> d_flags;// [0]: bit 0 some sightline is not sorted by distance and
                                    // loglam, bit 1 a non-finite value; [1] order key of the
                                    // smallest distance; [2] smallest positive gap between
                                    // consecutive distances of a sightline (float bits)
  tos::DevBuf<double> d_maxes;      // [0] max|wd|, [1] max w, [2] max |loglam|, [3] max distance
  bool sorted = true;
  double max_abs_wd = 0, max_w = 0, max_l = 0, max_d = 0;
  double min_d = 0;                 // smallest distance
  double min_gap = 0;               // smallest positive distance step within a sightline (lower bound)
  uint32_t max_np = 0;
  // common first-axis grids (0: distance, 1: loglam), built on first use
  std::mutex grid_mu;                                  // guards the grid build
  bool grid_built[2] = {false, false};
  int grid_n[2] = {0, 0};                              // distinct values (0: no usable grid)
  uint64_t grid_los[2] = {0, 0};                       // sightlines contiguous on the grid
  tos::DevBuf<float> d_grid[2];                        // sorted distinct values
  tos::DevBuf<uint32_t> d_gfirst[2];                   // per sightline grid index of pixel 0 or kNoGrid
  // the workspace of tos_xi_run on this catalogue; its per-cell sums stay
  // there after the run for the covariance calls
  tos::Workspace run;
  std::mutex run_mu;                                   // one tos_xi_run at a time on `run`
};

namespace tos {

// Accumulation rows of a run other than one per cell: the slots of unordered
// pairs of sightline keys (rows 0..n_rows-2; row n_rows-1 catches a pair
// without a slot), and the combine that turns them into the run's results.
struct RowPlan {
  uint32_t n_rows = 0;
  const uint32_t* row_key = nullptr;
  const uint32_t* slot_start = nullptr;
  const uint32_t* slot_key = nullptr;
  // enqueues the combine on the stream: writes the nb run totals to
  // d_out[0..nb) and any further outputs; inv_scale converts fixed point
  std::function<tos_status(cudaStream_t, uint32_t nb, const double* inv_scale,
                           const unsigned long long* d_acc, tos_xibin* d_out)>
      combine;
  // the most sightline pairs one row can receive, given the pairs whose
  // primary lies in each cell
  std::function<uint64_t(const std::vector<uint64_t>& cell_items)> max_row_items;
};

// Catalogue creation behind tos_catalog_create, tos_catalog_create_dc and
// tos_catalog_create_plates; omega_matter > 0: each pixel's distance is
// computed on the device from its loglam (the pixels' own distances are
// ignored).  platelist != null: cells are the sightlines' plates (order is
// not used).
tos_status catalog_create_impl(tos_engine* e, const tos_sightline* los, size_t n_los, const tos_pixel* pixels,
                               size_t n_pixels, int order, double omega_matter, const tos_plate* platelist,
                               size_t n_plates, tos_catalog** out);

// How a run shares the GPU with runs on other streams (the request
// server): the dominant kernel (grid or diagonal sweep) is launched in
// chunks of sightline pairs.  Before each chunk the run calls acquire with
// its remaining pixel pairs (this chunk's included); acquire blocks until the
// chunk may launch and returns its CTAs per SM (0: as many as fit).  When a
// chunk's kernel has completed, release is called from a host callback on the
// run's stream (it must not call CUDA).  The server's scheduler so decides,
// chunk by chunk, which running request uses the SMs next, while other
// requests' expansion and result phases run beside it.
struct SweepShare {
  std::function<int(uint64_t remaining_pairs)> acquire;
  std::function<void()> release;
  int chunks = 16;  // chunks per run (fewer when a run has few sightline pairs)
};

// The pair count behind tos_xi_run, with its scratch in `ws` (the caller
// owns ws exclusively for the call): plan = null accumulates per cell (and
// honours TOS_XI_SUBSAMPLES / TOS_XI_PER_GROUP), otherwise into the plan's
// slots, combined by plan->combine.  Takes the engine lock; the catalogue is
// only read, so runs with different workspaces may share it.
tos_status xi_run_impl(tos_engine* e, tos_catalog* cat, Workspace* ws, const tos_grid* grid,
                       double scale, uint32_t flags, const RowPlan* plan, tos_xibin* out_bins,
                       tos_xibin* out_cells, tos_xi_stats* stats, const SweepShare* share = nullptr);

// out[b] = rows[0][b] + rows[1][b] + ... (n_rows x nb XiBins, ascending row order).
void launch_sum_rows(const tos_xibin* rows, uint32_t n_rows, uint32_t nb, tos_xibin* out,
                     int blocks, cudaStream_t st);

// Device bytes of a catalogue's own data (not its workspace).
uint64_t catalog_data_bytes(const tos_catalog* c);

// Maximum angular scale of a grid (the grid classes' maxAngularScale).
double max_angular_scale(const tos_grid& g, double scale);

}  // namespace tos

// Build (once) the catalogue's common first-axis grid w (0: distance,
// 1: loglam) for the grid sweep; thread-safe.
tos_status ensure_grid(tos_engine* e, tos_catalog* cat, int w, cudaStream_t st);
