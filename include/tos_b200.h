/*
 * tos_b200.h — C ABI of the B200 pair-counting engine for the Lyman-alpha
 * forest two-point correlation function
 *     xi = sum w_i w_j delta_i delta_j / sum w_i w_j.
 *
 * This is the drop-in boundary for the pair-counting step of
 * turbooctospice::XiEstimator (turbooctospice/XiEstimator.h:17-86,
 * turbooctospice/XiEstimator.cc:19-305) and for the brute-force cubic-grid
 * estimator bruteGPU (gpu/brute.h:20, gpu/brute.cu:63-225).  Paths are
 * relative to the dmargala/turbo-octo-spice source tree.
 *
 * Conventions
 *  - Every function returns tos_status; nothing throws and nothing calls exit().
 *    tos_last_error() returns a thread-local message for the last failure.
 *  - Plain C types only: pointers, sizes, fixed-width integers.  Host buffers
 *    are owned by the caller; device copies are owned by the engine.
 *  - All compute runs on the engine's CUDA device (sm_100a).  There is no CPU
 *    fallback: on a host without that device every compute entry point fails
 *    with TOS_ERR_NO_DEVICE.
 *  - The library keeps no global state apart from the engines it creates and
 *    the thread-local error string, so engines on different devices (or one
 *    engine per host thread) are independent.
 */
#ifndef TOS_B200_H
#define TOS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TOS_ABI_VERSION 1

typedef enum {
  TOS_OK = 0,
  TOS_ERR_INVALID_ARG = 1,  /* bad pointer, size, grid or option */
  TOS_ERR_OOM = 2,          /* device or pinned host allocation failed */
  TOS_ERR_CUDA = 3,         /* a CUDA runtime call failed */
  TOS_ERR_TIMEOUT = 4,      /* a bounded device wait gave up */
  TOS_ERR_UNSUPPORTED = 5,  /* valid request this build cannot serve */
  TOS_ERR_NO_DEVICE = 6,    /* no sm_100 device, or the device id is out of range */
  TOS_ERR_INTERNAL = 7      /* consistency check failed inside the engine */
} tos_status;

/* Binning coordinate type.  Same values and meaning as
 * XiEstimator::BinningCoordinateType (XiEstimator.h:19-21):
 *  POLAR      (r, mu, log10(lya(1+z)))         PolarGrid   (PolarGrid.h:21-23)
 *  CARTESIAN  (r_par, r_perp, log10(lya(1+z))) CartesianGrid (CartesianGrid.h:21-23)
 *  OBSERVING  (dloglam, theta, log10(lya(1+z))) QuasarGrid (QuasarGrid.h:21-23) */
typedef enum { TOS_POLAR = 0, TOS_CARTESIAN = 1, TOS_OBSERVING = 2 } tos_coord_type;

/* One forest pixel.  Same fields, order and types as ForestPixel
 * (types.h:44-53): delta value, log10 wavelength, weight, comoving distance. */
typedef struct {
  float value, loglam, weight, distance;
} tos_pixel;

/* One sightline.  Position in radians (ra in [0, 2pi), dec in [-pi/2, pi/2]),
 * identifiers as in Forest (types.h:56-67), and its pixels as a range of a
 * flat pixel array.  Pixels are expected in increasing loglam order, as
 * HDF5Delta::loadForests produces them (HDF5Delta.cc:62-73).
 * `group` names the catalogue (mock realisation) the sightline belongs to:
 * sightlines of different groups never pair, so one resident catalogue can
 * hold many independent catalogues (0 for a single one, the reference's
 * case: one XiEstimator per catalogue). */
typedef struct {
  double ra, dec;
  int32_t forest_id, plate;
  uint64_t pixel_offset;
  uint32_t num_pixels, group;
} tos_sightline;

/* A linear axis "[min:max]*nbins" with bin width (max-min)/nbins, the binning
 * AbsTwoPointGrid reads through getAxisMin/getAxisBinWidth/getAxisNBins
 * (AbsTwoPointGrid.h:74-85). */
typedef struct {
  double min, max;
  int32_t nbins, reserved;
} tos_axis;

/* A three-axis grid: AbsTwoPointGrid plus the coordinate type that selects
 * CartesianGrid / PolarGrid / QuasarGrid.  Axis order is the reference's
 * (axis1, axis2, axis3) of h5healxi (h5healxi.cc:81-86, 138-153). */
typedef struct {
  int32_t type; /* tos_coord_type */
  int32_t reserved;
  tos_axis axis[3];
} tos_grid;

/* Per-bin accumulator.  Same fields and meaning as XiBin (types.h:69-121);
 * raw sums until tos_xibin_finalize() divides them as XiBin::finalize does. */
typedef struct {
  double didj, di, dj, wgt, wi, wj, z;
  int64_t num_pairs;
} tos_xibin;

/* Counters of XiEstimator::print_stats (XiEstimator.cc:389-408) plus the
 * engine's own work counters and device timings. */
typedef struct {
  uint64_t num_sightlines;
  uint64_t num_sightline_pairs;      /* candidates j > i from neighbouring cells (depends on the cell search) */
  uint64_t num_sightline_pairs_used; /* pairs passing cos(theta) > cos(max_ang) */
  uint64_t num_pixels;               /* pixels of all sightlines in occupied cells */
  uint64_t num_pixel_pairs;          /* sum of N_i*N_j over used sightline pairs */
  uint64_t num_pixel_pairs_used;     /* pixel pairs accumulated into a bin */
  uint64_t num_pixel_pairs_evaluated;/* pixel pairs the kernel evaluated (the rest were pruned by r_par window) */
  uint64_t num_edge_rechecks;        /* pixel pairs re-evaluated in FP64 near a bin edge */
  uint64_t num_index_overflow;       /* pairs whose unchecked z or theta index ran past the grid (dropped) */
  uint64_t num_cells;                /* occupied sky cells */
  uint64_t num_direct_runs;          /* runs added straight to global memory (outside the shared window) */
  uint64_t num_window_flushes;       /* shared-window flushes into the per-cell sums */
  double max_ang, cos_max_ang;       /* angular cut actually used (radians) */
  double ms_expand;                  /* device time: sightline-pair expansion */
  double ms_pairs;                   /* device time: run-sweep and pixel-pair kernels */
  double ms_total;                   /* wall time of the call */
  double ms_device;                  /* device time of the whole call (expansion to results) */
  uint64_t num_run_items;            /* sightline pairs counted by the boundary-sweep kernels */
  double ms_runs;                    /* device time: grid- and run-sweep kernels (part of ms_pairs) */
  uint64_t num_grid_items;           /* of num_run_items: sightline pairs counted by the grid-sweep kernel */
  double ms_grid;                    /* device time: grid-sweep kernel (part of ms_runs) */
  uint64_t num_diag_items;           /* sightline pairs counted by the diagonal-sweep kernel (Polar) */
  double ms_diag;                    /* device time: diagonal-sweep kernel (part of ms_pairs) */
} tos_xi_stats;

/* Opaque handles. */
typedef struct tos_engine tos_engine;
typedef struct tos_catalog tos_catalog;

/* ---- library / errors ---------------------------------------------------- */

/* Thread-local message describing the last non-OK status on this thread. */
const char* tos_last_error(void);
int tos_abi_version(void);

/* ---- engine -------------------------------------------------------------- */

/* Create an engine on CUDA device `device`.  Replaces nothing in the reference
 * one to one: it owns the device, streams and scratch that XiEstimator::run's
 * ThreadPool owned on the CPU (XiEstimator.cc:31-44, ThreadPool.cc:19-25). */
tos_status tos_engine_create(int device, tos_engine** out);
void tos_engine_destroy(tos_engine* engine);

/* ---- catalogue (sightlines + pixels resident on the device) --------------- */

/* Upload sightlines and pixels, and bin sightlines into HEALPix RING cells of
 * the given order (nside = 2^order), as HealpixBins::addItem does for every
 * sightline in h5healxi (HealpixBins.h:31-43, h5healxi.cc:196-205).
 * Sightline index = position in `los`; pairs are ordered by that index
 * (XiEstimator.cc:142). Host buffers may be freed after return. */
tos_status tos_catalog_create(tos_engine* engine, const tos_sightline* los, size_t n_los,
                              const tos_pixel* pixels, size_t n_pixels, int healpix_order,
                              tos_catalog** out);

/* tos_catalog_create with every pixel's comoving distance computed on the
 * device from its loglam for a flat universe of matter density omega_matter
 * (the pixels' own distance fields are ignored): the redshift and distance of
 * h5healxi.cc:38-40, 196-203, with the same bits as tos_fill_distances on the
 * host.  TOS_ERR_INVALID_ARG for a loglam that is not finite or below
 * log10(1216). */
tos_status tos_catalog_create_dc(tos_engine* engine, const tos_sightline* los, size_t n_los,
                                 const tos_pixel* pixels, size_t n_pixels, int order, double omega_matter,
                                 tos_catalog** out);

/* One forest as HDF5Delta::loadForests reads it from a group of the delta
 * file's `lines_of_sight` group (HDF5Delta.cc:52-66): the group's name, its
 * ra, dec, z and plate attributes, and its delta, weight, r_comov and loglam
 * datasets of n floats each (z is read by the reference and not used). */
typedef struct {
  const char* name;
  double ra, dec, z;
  int32_t plate, reserved;
  uint64_t n;
  const float *delta, *weight, *r_comov, *loglam;
} tos_forest;

/* The sightlines and pixels HDF5Delta::loadForests (HDF5Delta.cc:40-93)
 * builds from those forests, ready for tos_catalog_create: forests in
 * increasing byte-wise name order (its H5Literate over H5_INDEX_NAME,
 * increasing); a pixel kept when delta and weight are finite and the weight
 * is positive, in stored order, as {delta, loglam, weight, r_comov}; forests
 * left without pixels dropped; forest_id = 0, 1, ... over the kept forests;
 * ra, dec and plate as given; group 0; pixel ranges contiguous.  Host only
 * (no device needed).  With los or pixels NULL only *n_los and *n_pixels are
 * set (size query); otherwise the capacities must hold them. */
tos_status tos_forests_assemble(const tos_forest* forests, size_t n_forests, tos_sightline* los,
                                size_t los_capacity, size_t* n_los, tos_pixel* pixels, size_t pixel_capacity,
                                size_t* n_pixels);

/* One platelist row: the PLATE, RACEN and DECCEN columns (centre in degrees)
 * that PlateBins reads from the platelist FITS file (PlateBins.h:38-45). */
typedef struct {
  int32_t plate;
  float ra_center, dec_center;
} tos_plate;

/* tos_catalog_create with the sightlines binned by BOSS plate instead of
 * HEALPix: PlateBins (PlateBins.h:18-92), what h5healxi builds when its
 * HEALPix order is 0 (h5healxi.cc:166-174).  A sightline's cell is its
 * `plate` (cell id group * 2^32 + plate; plate ids must be >= 0).  The
 * sightlines a primary pairs with are those on the platelist plates whose
 * centre lies at an angle theta from it with |theta - 1.5 deg| < max_ang
 * (PlateBins::getBinIndicesWithinRadius, PlateBins.h:73-84; theta = acos of
 * SkyObject::angularSeparation, as the reference computes it), then the
 * cos(theta_ij) cut as for HEALPix cells.  That test is a ring, not a disc:
 * when max_ang < 1.5 deg, plates whose centre is nearer than 1.5 deg -
 * max_ang are skipped, and their pairs with it are not counted, exactly as
 * in the reference.  A plate id listed twice keeps its last row (the map
 * assignment of PlateBins.h:44); sightlines on a plate absent from the
 * platelist are primaries but nobody's neighbours.  omega_matter: 0 to keep
 * the pixels' distances, else as tos_catalog_create_dc.  tos_xi_run_jackknife
 * and tos_xi_jackknife (HEALPix regions) return TOS_ERR_UNSUPPORTED on such
 * a catalogue. */
tos_status tos_catalog_create_plates(tos_engine* engine, const tos_sightline* los, size_t n_los,
                                     const tos_pixel* pixels, size_t n_pixels, const tos_plate* platelist,
                                     size_t n_plates, double omega_matter, tos_catalog** out);

/* The catalogue's per-pixel comoving distances (float, in the compact order
 * of the catalogue: the pixels of sightline 0, then of sightline 1, ...). */
tos_status tos_catalog_distances(const tos_catalog* catalog, float* out, size_t capacity);
void tos_catalog_destroy(tos_catalog* catalog);

/* Number of occupied sky cells (SkyBins::getNBins, SkyBins.h:53). */
tos_status tos_catalog_num_cells(const tos_catalog* catalog, size_t* n_cells);
/* Occupied cell ids in ascending order — the key order of
 * XiEstimator::skybin_xis_ (XiEstimator.h:78) and of the subsample files.
 * A cell id is group * 2^32 + HEALPix pixel (the pixel alone in group 0),
 * or group * 2^32 + plate in a catalogue of tos_catalog_create_plates. */
tos_status tos_catalog_cells(const tos_catalog* catalog, int64_t* cell_ids, size_t capacity);
/* Cell id of each sightline (HealpixBins::ang2pix, HealpixBins.h:58-66, or
 * its plate, PlateBins.h:59). */
tos_status tos_catalog_sightline_cells(const tos_catalog* catalog, int64_t* cells, size_t capacity);
/* Number of distinct sightline groups, and their ids in ascending order (the
 * row order of a TOS_XI_PER_GROUP result). */
tos_status tos_catalog_num_groups(const tos_catalog* catalog, size_t* n_groups);
tos_status tos_catalog_groups(const tos_catalog* catalog, uint32_t* group_ids, size_t capacity);

/* ---- the hot path: XiEstimator pair counting ----------------------------- */

#define TOS_XI_SUBSAMPLES 0x1u   /* also return per-cell sums (skybin_xis_) */
#define TOS_XI_EXACT      0x2u   /* evaluate every pixel pair in FP64 (validation path, slow) */
#define TOS_XI_PER_GROUP  0x4u   /* return per-group sums: one xi per catalogue of a batch */
#define TOS_XI_TUNE       0x8u   /* autotune first: time the dominant kernel (grid or diagonal
                                  * sweep) with 1 .. max CTAs per SM on the first 65,536
                                  * sightline pairs, keep the fastest on the engine for this
                                  * coordinate type and bin count (later calls use it); the
                                  * results do not depend on the pick */

/* Maximum angular scale of a grid for a transverse comoving scale:
 * CartesianGrid::maxAngularScale (CartesianGrid.h:45-46),
 * PolarGrid::maxAngularScale (PolarGrid.h:45-46),
 * QuasarGrid::maxAngularScale (QuasarGrid.h:44-45). */
tos_status tos_grid_max_angular_scale(const tos_grid* grid, double scale, double* max_ang);
size_t tos_grid_num_bins(const tos_grid* grid);

/* Run the pair count of XiEstimator::run (XiEstimator.cc:31-58) over a
 * resident catalogue: sightline-pair search with the cut
 * cos(theta_ij) > cos(grid.maxAngularScale(scale)) (XiEstimator.cc:121-159),
 * then every pixel pair of every accepted sightline pair is binned and
 * accumulated (XiEstimator.cc:161-296, types.h:77-87).
 *   out_bins  : n_bins raw (unfinalized) sums over all cells, merged in
 *               ascending cell order as xi_finalize_task does (XiEstimator.cc:298-305).
 *   out_cells : NULL, or n_cells*n_bins raw per-cell sums (cell-major, cells
 *               ascending) when flags has TOS_XI_SUBSAMPLES.
 * With TOS_XI_PER_GROUP (not combined with TOS_XI_SUBSAMPLES) out_cells
 * receives n_groups*n_bins sums instead, group-major in ascending group id:
 * group g's row is its cells merged in ascending order, with the pair counts
 * of running that group alone and the sums to within the fixed-point
 * rounding (about 1e-12 relative), and out_bins is the sum of the groups'
 * rows in ascending group order.  This is the batched form of running
 * XiEstimator once per mock catalogue: every group's pairs go through one
 * set of launches.
 *   stats     : optional counters and timings. */
tos_status tos_xi_run(tos_engine* engine, tos_catalog* catalog, const tos_grid* grid, double scale,
                      uint32_t flags, tos_xibin* out_bins, tos_xibin* out_cells, tos_xi_stats* stats);

/* Covariance of the per-cell correlation functions of the last tos_xi_run on
 * `catalog` (XiEstimator::run with do_cov, XiEstimator.cc:60-97).  Every
 * occupied cell c is a sample x_c[b] = didj/wgt (0 where wgt = 0) of weight
 * W_c = sum of wgt over its bins with wgt > 0; mean = sum_c W_c x_c / W and
 * cov = sum_c W_c (x_c - mean)(x_c - mean)^T / W with W = sum_c W_c
 * (n_bins x n_bins, row-major; n_bins of that run).  The reference hands the
 * samples to likely::CovarianceAccumulator, whose source is not part of it;
 * this is the weighted covariance.  mean and total_weight may be NULL. */
tos_status tos_xi_cell_covariance(tos_engine* engine, tos_catalog* catalog, double* mean, double* cov,
                                  double* total_weight);
/* Jackknife of the last tos_xi_run on `catalog` over the HEALPix pixels of
 * order region_order (<= the catalogue's order) that hold occupied cells:
 * region k's estimate xi_jk[k][b] = (D - D_k) / (G - G_k), where D and G are
 * the run's didj and wgt sums of bin b and D_k, G_k those of the cells inside
 * region k (subtracted exactly; 0 where G - G_k <= 0), and
 * cov = (N - 1)/N sum_k (xi_k - mean)(xi_k - mean)^T over the N regions.
 * With region_ids, xi_jk or cov NULL only *n_regions is set (size query);
 * otherwise cap must be >= N; region_ids ascending, xi_jk [N][n_bins]. */
tos_status tos_xi_jackknife(tos_engine* engine, tos_catalog* catalog, int region_order, size_t cap,
                            size_t* n_regions, int64_t* region_ids, double* xi_jk, double* cov);

/* Exact delete-one-region jackknife in one pass over the pairs: the
 * jackknife subsamples of a batched run.  Region k is a HEALPix RING pixel of
 * order region_order (<= the catalogue's order) within one sightline group;
 * a sightline belongs to the region that holds its cell.  Subsample k is the
 * catalogue without region k's sightlines.  The reference forms it by running
 * XiEstimator again on the reduced catalogue; here every pair is added to the
 * slot of its two regions and out_drop[k] = (total of k's group) - (slots
 * that name k), subtracted exactly in 128-bit fixed point, so each subsample
 * has the pair counts of that separate run and its sums to within the
 * fixed-point rounding (about 1e-12 relative).
 *   flags      : 0 or TOS_XI_EXACT.
 *   n_regions  : set to the number of (group, region) subsamples N.  With
 *                region_ids, out_bins or out_drop NULL nothing else happens
 *                (size query); otherwise capacity must be >= N.
 *   region_ids : N ids group * 2^32 + region pixel, ascending.
 *   out_bins   : n_bins sums of the whole catalogue (groups added in order).
 *   out_groups : NULL or n_groups*n_bins per-group sums (ascending group id).
 *   out_drop   : N*n_bins raw sums of the subsamples, region-major.
 * The per-cell sums of this run are not kept: tos_xi_cell_covariance and
 * tos_xi_jackknife need a tos_xi_run after it. */
tos_status tos_xi_run_jackknife(tos_engine* engine, tos_catalog* catalog, const tos_grid* grid,
                                double scale, uint32_t flags, int region_order, size_t capacity,
                                size_t* n_regions, int64_t* region_ids, tos_xibin* out_bins,
                                tos_xibin* out_groups, tos_xibin* out_drop, tos_xi_stats* stats);

/* Jackknife covariance of n_rows delete-one subsamples, such as the out_drop
 * rows of one group from tos_xi_run_jackknife: xi_k[b] = didj/wgt (0 where
 * wgt <= 0), mean = sum_k xi_k / N and cov = (N - 1)/N sum_k (xi_k - mean)
 * (xi_k - mean)^T (n_bins x n_bins, row-major; N = n_rows >= 2), the
 * estimator tos_xi_jackknife applies to its region estimates.  xi (n_rows x
 * n_bins) and mean may be NULL.  No counterpart in the reference, which
 * leaves subsample covariances to likely (XiEstimator.cc:60-97). */
tos_status tos_xi_subsample_covariance(tos_engine* engine, const tos_xibin* rows, size_t n_rows,
                                       size_t n_bins, double* xi, double* mean, double* cov);

/* XiBin::finalize (types.h:96-101) applied to n bins in place. */
void tos_xibin_finalize(tos_xibin* bins, size_t n);

/* ---- serving: continuous admission of xi requests ------------------------ */

/* A request server on one device.  No counterpart in the reference (which
 * runs one XiEstimator per process): it serves pair counts of resident
 * catalogues to many callers.  `slots` worker slots each own a stream and a
 * workspace and run one request at a time, so requests on different slots
 * overlap on the device.  A submitted request waits in arrival order until a
 * slot is free and its workspace fits in memory_budget_bytes beside the
 * attached catalogues and the other slots' workspaces; idle slots give their
 * workspaces back when the next request needs the room.  Results equal
 * tos_xi_run's on the same catalogue, bit for bit (the fixed-point sums do
 * not depend on the order of the pairs).  The workspace of a request is an
 * estimate made at submission (exact sizes, sightline pairs estimated for a
 * uniform sky density with a 1.5 margin). */
typedef struct tos_server tos_server;

typedef struct {
  double submit_s, start_s, end_s; /* seconds since the server was created */
  int32_t slot;                    /* slot that ran the request */
  int32_t reserved;
  uint64_t workspace_bytes;        /* workspace estimate used for admission */
} tos_request_info;

typedef struct {
  uint64_t budget_bytes, resident_bytes, in_use_bytes, peak_bytes;
  uint64_t queued, running, completed;
  uint32_t slots, reserved;
} tos_server_status;

tos_status tos_server_create(int device, int slots, uint64_t memory_budget_bytes, tos_server** out);
/* Finishes running requests; queued ones end with TOS_ERR_INVALID_ARG. */
void tos_server_destroy(tos_server* server);
/* Count a resident catalogue (created on the server's device with
 * tos_catalog_create) against the budget; TOS_ERR_OOM when it does not fit.
 * The catalogue must outlive its requests; detach it before destroying it. */
tos_status tos_server_attach(tos_server* server, tos_catalog* catalog);
tos_status tos_server_detach(tos_server* server, tos_catalog* catalog);
/* Queue tos_xi_run(catalog, grid, scale, flags) without blocking.  flags as
 * tos_xi_run; TOS_ERR_OOM when the request can never fit in the budget. */
tos_status tos_server_submit(tos_server* server, tos_catalog* catalog, const tos_grid* grid,
                             double scale, uint32_t flags, uint64_t* request_id);
/* Block until the request is done and take its results (then the id is
 * released): out_bins n_bins sums, out_rows the per-cell or per-group rows
 * its flags ask for (NULL to drop them), stats and info optional. */
tos_status tos_server_wait(tos_server* server, uint64_t request_id, tos_xibin* out_bins,
                           tos_xibin* out_rows, tos_xi_stats* stats, tos_request_info* info);
/* Admission order of queued requests: TOS_SERVER_FIFO (arrival order, the
 * default) or TOS_SERVER_SHORTEST (least estimated pixel pairs first; a
 * request that has waited more than max_wait_s seconds goes first and is not
 * overtaken, so none waits forever behind smaller ones). */
#define TOS_SERVER_FIFO 0
#define TOS_SERVER_SHORTEST 1
tos_status tos_server_set_policy(tos_server* server, int policy, double max_wait_s);
/* Non-blocking: *done = 1 when the request has finished (tos_server_wait then
 * returns at once), 0 while it is queued or running. */
tos_status tos_server_poll(tos_server* server, uint64_t request_id, int* done);
tos_status tos_server_status_get(tos_server* server, tos_server_status* out);

/* Device bytes held by a catalogue (its data and the workspace of its own
 * tos_xi_run calls). */
tos_status tos_catalog_device_bytes(const tos_catalog* catalog, uint64_t* bytes);

/* ---- brute-force cubic-grid estimator ------------------------------------ */

/* All-pairs isotropic xi(r) of bruteGPU (gpu/brute.cu:63-225) without its
 * chunked host loop: points are (x, y, z, delta, w) rows (DataStruct,
 * gpu/brute.cu:3-5), r = |x_i - x_j| over all i < j, bins of width
 * (max-min)/nbins with bin 0 = underflow and nbins+1 = overflow
 * (gpu/brute.cu:40-48).  Outputs have nbins+2 entries:
 *   dsum[k] = sum w_i w_j d_i d_j, wsum[k] = sum w_i w_j, counts[k] = pairs.
 * Binning is exact against the FP64 separation (FP32 fast path with an FP64
 * recheck near bin edges); the sums are exact fixed-point sums of FP64
 * products, the same for every launch shape.  2 <= n_points <= 2^24 and
 * nbins in [1, 4096]: each warp keeps a shared-memory window of the nbins + 2
 * bins, and a block holds as many warps (up to 16) as the device's shared
 * memory has windows for. */
tos_status tos_brute_run(tos_engine* engine, const float* points, size_t n_points, double min,
                         double max, int nbins, double* dsum, double* wsum, uint64_t* counts,
                         double* ms_kernel);

/* Autotuner of tos_brute_run's launch shape for one bin count (the
 * reference fixes its shape from device properties, gpu/brute.cu:99-131):
 * times every kernel variant (1, 2 or 4 diagonals per lane) with 4, 8 and 16
 * warps per CTA on the first min(n_points, 131072) points and keeps the
 * fastest on the engine.  Later tos_brute_run and tos_brute_run_noalloc calls
 * with that bin count use it; results do not depend on the shape (exact
 * integer sums).  The pick is written to *diagonals_per_lane and
 * *warps_per_cta (either may be null). */
tos_status tos_brute_tune(tos_engine* engine, const float* points, size_t n_points, double min,
                          double max, int nbins, int* diagonals_per_lane, int* warps_per_cta);

/* tos_brute_run without any device allocation.  No counterpart in the
 * reference: it is for callers that cannot allocate GPU memory while they
 * count pairs (memory managed entirely by their own pool, code where a
 * cudaMalloc would synchronise the device or is not allowed, loops that must
 * not touch the allocator).  points (n_points x 5 floats: x, y, z, delta, w),
 * dsum, wsum and counts (nbins + 2 each) are DEVICE pointers on the engine's
 * device; results equal tos_brute_run's.  The call reads the points and
 * writes the results on the engine's own stream, with no ordering against
 * the caller's streams: the writes that produced the points must be complete
 * (for example the caller's stream synchronised) before the call.  All
 * scratch lives in one static device array of about 6.5 MB that the
 * library reserves on every GPU that loads it, until the process exits,
 * which limits a call to n_points <= 262144 and nbins <= 4096 (larger
 * requests fail with TOS_ERR_INVALID_ARG).  The first call on a device looks
 * up that array (and may load the module on the device): make it before any
 * stream capture.  Every call shares the array, so calls that overlap on the
 * GPU (other engines or threads on the same device) race; the call
 * synchronises the engine's stream before it returns. */
tos_status tos_brute_run_noalloc(tos_engine* engine, const float* points, size_t n_points,
                                 double min, double max, int nbins, double* dsum, double* wsum,
                                 uint64_t* counts, double* ms_kernel);

/* ---- flat LCDM comoving distance (h5healxi.cc:123-131, 196-203) ---------- */

/* Line-of-sight comoving distance in Mpc/h of a flat universe with the given
 * Omega_matter (Omega_lambda = 1 - Omega_matter):
 *   D_C(z) = (c / 100 km/s/Mpc) * int_0^z dz' / sqrt(Om (1+z')^3 + OL),
 * evaluated in FP64.  Replaces cosmo::LambdaCdmUniverse::
 * getLineOfSightComovingDistance as called at h5healxi.cc:201. */
tos_status tos_comoving_distance(double omega_matter, const double* z, size_t n, double* out);
/* Fill pixels[k].distance = D_C(10^(loglam - log10(1216)) - 1) on the host
 * (h5healxi.cc:38-40, 196-203), stored as float like ForestPixel::distance. */
tos_status tos_fill_distances(double omega_matter, tos_pixel* pixels, size_t n);

#ifdef __cplusplus
}
#endif

#endif /* TOS_B200_H */
