/*
 * xi_oracle.c — CPU oracle for the pair-counting hot path of the
 * turbo-octo-spice XiEstimator.  TEST INFRASTRUCTURE ONLY: tests, the smoke
 * check and the CPU-baseline leg of bench.py call it to check (and time
 * beside) the GPU engine; the engine never calls it.
 *
 * What it restates (paths relative to the dmargala/turbo-octo-spice tree):
 *  - XiEstimator::run / skybin_xi_task (XiEstimator.cc:31-58, 121-159):
 *    one task per occupied sky cell, in a pool of threads; for every primary
 *    sightline i of the cell and every sightline j > i within the angular cut
 *    cos(theta_ij) > cos(max_ang), all pixel pairs are binned and accumulated
 *    into the cell's bins; cells are merged in ascending cell-id order
 *    (xi_finalize_task, XiEstimator.cc:298-305);
 *  - accumulate_pixel_pairs (XiEstimator.cc:161-296), the three coordinate
 *    branches with their exact float/double expression order and quirks
 *    (float product p1.distance*p1.distance, 1/nbins z scaling, unchecked z
 *    and theta indices, truncating unsigned casts, r == 0 skip in Polar);
 *  - SkyObject::angularSeparation (types.h:37-39) and XiBin::accumulate_pair
 *    (types.h:77-87): in mode 0 exactly as written (float products
 *    w*delta and wdi*wdj); in mode 1 ("FP64 oracle") every product and sum in
 *    double from the float inputs; mode 2 is mode 1 with the absolute value
 *    of every signed term (didj, di, dj), the scale against which a bin whose
 *    signed sum cancels is judged;
 *  - HealpixBins::ang2pix (HealpixBins.h:58-72) with RING numbering
 *    (Gorski et al. 2005) for the cell of each sightline, or, in
 *    orc_xi_plates, PlateBins (PlateBins.h:18-92): cells keyed by plate and
 *    the neighbour plates of its ring test |theta - 1.5 deg| < max_ang;
 *  - the brute-force estimator's histogram (gpu/brute.cu:40-52) with the FP64
 *    separation of bucketxi (src/bucketxi.cc:79-98).
 * The neighbour search is a declination band scan instead of HEALPix
 * query_disc_inclusive: both return every sightline within max_ang, and the
 * exact cos cut decides, so the accepted pairs are the same.
 *
 * Parity pinned: the reference ships no expected outputs for this path, so
 * its own XiEstimator.cc, grid classes, ThreadPool.cc and PlateBins.h are
 * compiled unchanged against stand-in headers (oracle/ref_harness.cc,
 * oracle/refshim, `make -C oracle ref`), and the tests compare this
 * restatement with that build: the golden fixtures of tests/golden hold its
 * outputs (tests/golden/make_golden.py), and the live build is compared
 * wherever it is present.  Mode 0 reproduces it bit for bit.  Also checked
 * against a literal transcription of the reference's loop
 * (tests/ref_loop.py), hand-built known answers at bin edges, and HEALPix
 * known pixels.
 *
 * static_cast<unsigned>(double) is reproduced as the x86-64 code of the
 * reference build computes it (cvttsd2si into 64 bits, low 32 bits kept).
 * Build strictly (-fno-fast-math -ffp-contract=off) for parity.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { float value, loglam, weight, distance; } orc_pixel;
typedef struct { double didj, di, dj, wgt, wi, wj, z; int64_t num_pairs; } orc_xibin;
typedef struct {
  uint64_t num_sightline_pairs_used, num_pixels, num_pixel_pairs, num_pixel_pairs_used,
      num_index_overflow;
  double max_ang, cos_max_ang;
  uint64_t num_sightline_pairs; /* candidates j > i in neighbour cells: plate cells only (0 otherwise) */
} orc_stats;

enum { ORC_POLAR = 0, ORC_CARTESIAN = 1, ORC_OBSERVING = 2 };

static uint32_t ref_u32(double x) {
  if (!(x > -9223372036854775808.0 && x < 9223372036854775808.0)) return 0u;
  return (uint32_t)(int64_t)x;
}

/* ---------------- HEALPix RING ang2pix (Gorski et al. 2005) -------------- */
static int64_t orc_ang2pix(int64_t nside, double theta, double phi) {
  const double pi = 3.141592653589793238462643383279502884197;
  const double z = cos(theta), za = fabs(z);
  double tt = phi * 0.6366197723675813430755350534900574;  /* phi / (pi/2) */
  if (tt >= 0) {
    if (tt >= 4.0) tt = fmod(tt, 4.0);
  } else {
    tt = fmod(tt, 4.0) + 4.0;
    if (tt == 4.0) tt = 0.0;
  }
  const int64_t npix = 12 * nside * nside, ncap = 2 * nside * (nside - 1);
  if (za <= 2.0 / 3.0) {
    const int64_t nl4 = 4 * nside;
    const double a = nside * (0.5 + tt), b = nside * z * 0.75;
    const int64_t jp = (int64_t)(a - b), jm = (int64_t)(a + b);
    const int64_t ir = nside + 1 + jp - jm;
    const int64_t kshift = 1 - (ir & 1);
    const int64_t ip = ((jp + jm - nside + kshift + 1 + 2 * nl4) / 2) % nl4;
    return ncap + (ir - 1) * nl4 + ip;
  } else {
    const int near_pole = (theta < 0.01) || (theta > pi - 0.01);
    const double tp = tt - (double)(int64_t)tt;
    const double tmp = (za < 0.99 || !near_pole) ? nside * sqrt(3.0 * (1.0 - za))
                                                 : nside * sin(theta) / sqrt((1.0 + za) / 3.0);
    const int64_t jp = (int64_t)(tp * tmp), jm = (int64_t)((1.0 - tp) * tmp);
    const int64_t ir = jp + jm + 1;
    int64_t ip = (int64_t)(tt * (double)ir);
    if (ip >= 4 * ir) ip -= 4 * ir;
    return (z > 0) ? 2 * ir * (ir - 1) + ip : npix - 2 * ir * (ir + 1) + ip;
  }
}

int64_t orc_radec2pix(int order, double ra, double dec) {
  const double pi = atan(1.0) * 4;
  return orc_ang2pix((int64_t)1 << order, 0.5 * pi - dec, ra);
}

/* ---------------- grid ---------------------------------------------------- */
typedef struct {
  int coord;
  double min0, inv0, min1, inv1, min2, invn2;
  uint32_t n0, n1, n2, ntotal;
  double max_ang;
} orc_grid;

static void make_grid(orc_grid* g, int coord, const double* ax, double scale) {
  /* ax = {min0, max0, n0, min1, max1, n1, min2, max2, n2} */
  double w[3], hi[3];
  for (int k = 0; k < 3; ++k) {
    w[k] = (ax[3 * k + 1] - ax[3 * k]) / ax[3 * k + 2];
    hi[k] = ax[3 * k] + ax[3 * k + 2] * w[k];
  }
  g->coord = coord;
  g->min0 = ax[0];
  g->inv0 = 1.0 / w[0];
  g->min1 = ax[3];
  g->inv1 = 1.0 / w[1];
  g->min2 = ax[6];
  g->invn2 = 1.0 / ax[8];
  g->n0 = (uint32_t)ax[2];
  g->n1 = (uint32_t)ax[5];
  g->n2 = (uint32_t)ax[8];
  g->ntotal = g->n0 * g->n1 * g->n2;
  if (coord == ORC_CARTESIAN)
    g->max_ang = hi[1] / scale; /* CartesianGrid.h:46 */
  else if (coord == ORC_POLAR)
    g->max_ang = hi[0] * sqrt(1.0 - ax[3] * ax[3]) / scale; /* PolarGrid.h:46 */
  else
    g->max_ang = hi[1]; /* QuasarGrid.h:45 */
}

/* ---------------- per-cell accumulation ------------------------------------ */
typedef struct {
  /* catalogue */
  const double *sd, *cd, *sr, *cr; /* sin/cos of dec and ra */
  const double* dec;
  const uint64_t* off;
  const uint32_t* npix;
  const orc_pixel* px;
  size_t n_los;
  const uint32_t* by_dec; /* sightline indices sorted by dec */
  const double* dec_sorted;
  /* cells */
  const uint32_t* cell_start; /* CSR over members */
  const uint32_t* members;
  /* plate cells (orc_xi_plates): the platelist, one entry per plate id in
   * ascending id order, its centres' sines and cosines, and the cell of each
   * entry (-1: no sightline on that plate) */
  size_t n_plates;
  const double *psd, *pcd, *psr, *pcr;
  const int64_t* plate_cell;
  /* run */
  orc_grid g;
  double cos_max;
  int mode;
  orc_xibin* cell_bins; /* [n_cells][ntotal] */
  uint64_t* cell_ctr;   /* [n_cells][5]: used pairs, pixel pairs, pixel pairs used, overflow, candidates */
  const uint32_t* todo; /* cells to process */
  size_t n_todo;
  size_t next;
  pthread_mutex_t mu;
} orc_job;

static void acc_pair(orc_xibin* b, const orc_pixel* i, const orc_pixel* j, int mode) {
  if (mode == 0) { /* XiBin::accumulate_pair as written (types.h:77-87) */
    float wdi = i->weight * i->value, wdj = j->weight * j->value;
    b->didj += wdi * wdj;
    b->di += wdi;
    b->dj += wdj;
    b->wgt += i->weight * j->weight;
    b->wi += i->weight;
    b->wj += j->weight;
    b->z += 0.5 * (i->loglam + j->loglam);
  } else { /* FP64; mode 2 sums absolute values (the scale of each signed sum) */
    const double wdi = (double)i->weight * (double)i->value;
    const double wdj = (double)j->weight * (double)j->value;
    b->didj += (mode == 2) ? fabs(wdi * wdj) : wdi * wdj;
    b->di += (mode == 2) ? fabs(wdi) : wdi;
    b->dj += (mode == 2) ? fabs(wdj) : wdj;
    b->wgt += (double)i->weight * (double)j->weight;
    b->wi += (double)i->weight;
    b->wj += (double)j->weight;
    b->z += 0.5 * ((double)i->loglam + (double)j->loglam);
  }
  ++b->num_pairs;
}

/* accumulate_pixel_pairs; returns pixel pairs used, adds index overflows to *ovf */
static uint64_t pixel_pairs(const orc_job* J, uint32_t a, uint32_t b, double c, orc_xibin* xi,
                            uint64_t* ovf) {
  const orc_grid* g = &J->g;
  const orc_pixel* P1 = J->px + J->off[a];
  const orc_pixel* P2 = J->px + J->off[b];
  const uint32_t n1 = J->npix[a], n2 = J->npix[b];
  uint64_t used = 0;
  const double separation = acos(c);
  if (g->coord == ORC_POLAR) {
    for (uint32_t k = 0; k < n1; ++k) {
      const orc_pixel* p1 = P1 + k;
      const double r1_sq = p1->distance * p1->distance;  /* float product */
      const double two_r1_cos12 = 2 * p1->distance * c;
      for (uint32_t m = 0; m < n2; ++m) {
        const orc_pixel* p2 = P2 + m;
        const double r_sq = r1_sq + (p2->distance - two_r1_cos12) * p2->distance;
        const double r = sqrt(r_sq);
        uint32_t idx = ref_u32((r - g->min0) * g->inv0);
        if (idx >= g->n0) continue;
        if (r == 0) continue;
        const double mu = fabsf(p1->distance - p2->distance) / r;
        const uint32_t mb = ref_u32((mu - g->min1) * g->inv1);
        if (mb >= g->n1) continue;
        idx = mb + idx * g->n1;
        const double lz = 0.5 * (p1->loglam + p2->loglam);
        const uint32_t zb = ref_u32((lz - g->min2) * g->invn2);
        idx = zb + idx * g->n2;
        ++used;
        if (idx >= g->ntotal) {
          ++*ovf;
          continue;
        }
        acc_pair(xi + idx, p1, p2, J->mode);
      }
    }
  } else if (g->coord == ORC_CARTESIAN) {
    for (uint32_t k = 0; k < n1; ++k) {
      const orc_pixel* p1 = P1 + k;
      const double r1_sq = p1->distance * p1->distance;  /* float product */
      const double two_r1_cos12 = 2 * p1->distance * c;
      for (uint32_t m = 0; m < n2; ++m) {
        const orc_pixel* p2 = P2 + m;
        const double r_para = fabsf(p1->distance - p2->distance);
        uint32_t idx = ref_u32((r_para - g->min0) * g->inv0);
        if (idx >= g->n0) continue;
        const double r_sq = r1_sq + (p2->distance - two_r1_cos12) * p2->distance;
        const uint32_t pb = ref_u32((sqrt(fabs(r_sq - r_para * r_para)) - g->min1) * g->inv1);
        if (pb >= g->n1) continue;
        idx = pb + idx * g->n1;
        const double lz = 0.5 * (p1->loglam + p2->loglam);
        const uint32_t zb = ref_u32((lz - g->min2) * g->invn2);
        idx = zb + idx * g->n2;
        ++used;
        if (idx >= g->ntotal) {
          ++*ovf;
          continue;
        }
        acc_pair(xi + idx, p1, p2, J->mode);
      }
    }
  } else {
    const uint32_t sep = ref_u32((separation - g->min1) * g->inv1);
    for (uint32_t k = 0; k < n1; ++k) {
      const orc_pixel* p1 = P1 + k;
      for (uint32_t m = 0; m < n2; ++m) {
        const orc_pixel* p2 = P2 + m;
        uint32_t idx = ref_u32((fabsf(p1->loglam - p2->loglam) - g->min0) * g->inv0);
        if (idx >= g->n0) continue;
        idx = sep + idx * g->n1;
        const double lz = 0.5 * (p1->loglam + p2->loglam);
        const uint32_t zb = ref_u32((lz - g->min2) * g->invn2);
        idx = zb + idx * g->n2;
        ++used;
        if (idx >= g->ntotal) {
          ++*ovf;
          continue;
        }
        acc_pair(xi + idx, p1, p2, J->mode);
      }
    }
  }
  return used;
}

/* One accepted-or-not candidate pair (i, j), j > i (XiEstimator.cc:141-151). */
static void candidate(orc_job* J, uint32_t i, uint32_t j, orc_xibin* xi, uint64_t* ctr) {
  const double c = J->sd[i] * J->sd[j] + J->cd[i] * J->cd[j] * (J->sr[i] * J->sr[j] + J->cr[i] * J->cr[j]);
  ctr[4] += 1;
  if (c <= J->cos_max) return;
  ctr[0] += 1;
  ctr[1] += (uint64_t)J->npix[i] * J->npix[j];
  ctr[2] += pixel_pairs(J, i, j, c, xi, &ctr[3]);
}

/* Plate cells: PlateBins::getBinIndicesWithinRadius (PlateBins.h:73-84)
 * takes every platelist plate, in ascending plate id, whose centre's angular
 * separation from the primary is within max_ang of 1.5 degrees:
 * |acos(cos_sep) - 1.5 deg| < max_ang; plates without sightlines are skipped
 * (XiEstimator.cc:136-137), every sightline j > i of the others is a
 * candidate. */
static void plate_task(orc_job* J, uint32_t cell, orc_xibin* xi, uint64_t* ctr) {
  const double deg2rad = (atan(1.0) * 4) / 180.0; /* constants.h:12-13 */
  const double ring = 1.5 * deg2rad;
  for (uint32_t q = J->cell_start[cell]; q < J->cell_start[cell + 1]; ++q) {
    const uint32_t i = J->members[q];
    for (size_t k = 0; k < J->n_plates; ++k) {
      const double cs = J->sd[i] * J->psd[k] + J->cd[i] * J->pcd[k] * (J->sr[i] * J->psr[k] + J->cr[i] * J->pcr[k]);
      if (!(fabs(acos(cs) - ring) < J->g.max_ang)) continue;
      if (J->plate_cell[k] < 0) continue;
      const uint32_t nc = (uint32_t)J->plate_cell[k];
      for (uint32_t m = J->cell_start[nc]; m < J->cell_start[nc + 1]; ++m) {
        const uint32_t j = J->members[m];
        if (j <= i) continue;
        candidate(J, i, j, xi, ctr);
      }
    }
  }
}

static void skybin_task(orc_job* J, uint32_t cell) {
  orc_xibin* xi = J->cell_bins + (size_t)cell * J->g.ntotal;
  uint64_t* ctr = J->cell_ctr + 5 * (size_t)cell;
  if (J->plate_cell) {
    plate_task(J, cell, xi, ctr);
    return;
  }
  const double lim = J->g.max_ang + 1e-9;
  for (uint32_t q = J->cell_start[cell]; q < J->cell_start[cell + 1]; ++q) {
    const uint32_t i = J->members[q];
    /* candidates: declination band [dec_i - lim, dec_i + lim] */
    const double lo = J->dec[i] - lim, hi = J->dec[i] + lim;
    size_t a = 0, b = J->n_los;
    while (a < b) {
      size_t m = (a + b) / 2;
      if (J->dec_sorted[m] < lo) a = m + 1; else b = m;
    }
    for (size_t k = a; k < J->n_los && J->dec_sorted[k] <= hi; ++k) {
      const uint32_t j = J->by_dec[k];
      if (j <= i) continue;
      const double c = J->sd[i] * J->sd[j] + J->cd[i] * J->cd[j] * (J->sr[i] * J->sr[j] + J->cr[i] * J->cr[j]);
      if (c <= J->cos_max) continue;
      ctr[0] += 1;
      ctr[1] += (uint64_t)J->npix[i] * J->npix[j];
      ctr[2] += pixel_pairs(J, i, j, c, xi, &ctr[3]);
    }
  }
}

static void* worker(void* arg) {
  orc_job* J = (orc_job*)arg;
  for (;;) {
    pthread_mutex_lock(&J->mu);
    const size_t t = J->next++;
    pthread_mutex_unlock(&J->mu);
    if (t >= J->n_todo) break;
    skybin_task(J, J->todo[t]);
  }
  return NULL;
}

typedef struct { double key; uint32_t idx; } kv;
static int cmp_kv(const void* x, const void* y) {
  const kv *a = (const kv*)x, *b = (const kv*)y;
  if (a->key < b->key) return -1;
  if (a->key > b->key) return 1;
  return (a->idx > b->idx) - (a->idx < b->idx);
}
typedef struct { int64_t key; uint32_t idx; } kvi;
static int cmp_kvi(const void* x, const void* y) {
  const kvi *a = (const kvi*)x, *b = (const kvi*)y;
  if (a->key != b->key) return (a->key > b->key) - (a->key < b->key);
  return (a->idx > b->idx) - (a->idx < b->idx);
}

/* Runs the tasks of the chosen cells (every cell when cell_subset is NULL)
 * in nthreads threads, merges the cells in ascending order
 * (xi_finalize_task, XiEstimator.cc:298-305) and fills the outputs.
 * Returns the number of occupied cells. */
static long run_cells(orc_job* J, size_t nc, const int64_t* cell_ids, const uint32_t* cell_subset,
                      size_t n_subset, int nthreads, orc_xibin* out_bins, orc_xibin* out_cells,
                      int64_t* out_cell_ids, orc_stats* stats) {
  J->cell_bins = (orc_xibin*)calloc((size_t)nc * J->g.ntotal, sizeof(orc_xibin));
  J->cell_ctr = (uint64_t*)calloc(5 * nc, sizeof(uint64_t));
  uint32_t* todo = (uint32_t*)malloc(4 * (nc ? nc : 1) + 4 * n_subset);
  if (cell_subset) {
    for (size_t k = 0; k < n_subset; ++k) todo[k] = cell_subset[k];
    J->n_todo = n_subset;
  } else {
    for (size_t k = 0; k < nc; ++k) todo[k] = (uint32_t)k;
    J->n_todo = nc;
  }
  J->todo = todo;
  J->next = 0;
  pthread_mutex_init(&J->mu, NULL);
  if (nthreads < 1) nthreads = 1;
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
  for (int t = 0; t < nthreads; ++t) pthread_create(&th[t], NULL, worker, J);
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&J->mu);
  memset(out_bins, 0, sizeof(orc_xibin) * J->g.ntotal);
  orc_stats st;
  memset(&st, 0, sizeof st);
  for (size_t c = 0; c < nc; ++c) {
    const orc_xibin* x = J->cell_bins + c * J->g.ntotal;
    for (uint32_t b = 0; b < J->g.ntotal; ++b) {
      out_bins[b].didj += x[b].didj; out_bins[b].di += x[b].di; out_bins[b].dj += x[b].dj;
      out_bins[b].wgt += x[b].wgt; out_bins[b].wi += x[b].wi; out_bins[b].wj += x[b].wj;
      out_bins[b].z += x[b].z; out_bins[b].num_pairs += x[b].num_pairs;
    }
    st.num_sightline_pairs_used += J->cell_ctr[5 * c];
    st.num_pixel_pairs += J->cell_ctr[5 * c + 1];
    st.num_pixel_pairs_used += J->cell_ctr[5 * c + 2];
    st.num_index_overflow += J->cell_ctr[5 * c + 3];
    st.num_sightline_pairs += J->cell_ctr[5 * c + 4];
  }
  for (size_t k = 0; k < J->n_todo; ++k)
    for (uint32_t q = J->cell_start[todo[k]]; q < J->cell_start[todo[k] + 1]; ++q)
      st.num_pixels += J->npix[J->members[q]];
  st.max_ang = J->g.max_ang;
  st.cos_max_ang = J->cos_max;
  if (out_cells) memcpy(out_cells, J->cell_bins, sizeof(orc_xibin) * nc * J->g.ntotal);
  if (out_cell_ids) memcpy(out_cell_ids, cell_ids, 8 * nc);
  if (stats) *stats = st;
  free(J->cell_bins); free(J->cell_ctr); free(todo);
  return (long)nc;
}

/*
 * Pair count over a catalogue.  axes = 9 doubles {min,max,nbins} x 3.
 * cell_subset: NULL for all occupied cells, else the occupied-cell positions
 * (0-based, ascending cell-id order) whose primaries are processed.
 * out_cells (optional): n_cells*ntotal raw per-cell sums; out_cell_ids
 * (optional): the n_cells occupied cell ids ascending.  Returns the number of
 * occupied cells, or -1 on bad input.
 */
long orc_xi(const double* ra, const double* dec, const uint64_t* off, const uint32_t* npix,
            size_t n_los, const orc_pixel* px, int order, int coord, const double* axes,
            double scale, int mode, int nthreads, const uint32_t* cell_subset, size_t n_subset,
            orc_xibin* out_bins, orc_xibin* out_cells, int64_t* out_cell_ids, orc_stats* stats) {
  if (n_los == 0 || coord < 0 || coord > 2) return -1;
  orc_job J;
  memset(&J, 0, sizeof J);
  make_grid(&J.g, coord, axes, scale);
  J.cos_max = cos(J.g.max_ang);
  J.mode = mode;
  J.off = off;
  J.npix = npix;
  J.px = px;
  J.n_los = n_los;
  J.dec = dec;
  double* trig = (double*)malloc(sizeof(double) * 4 * n_los);
  double* sd = trig; double* cd = trig + n_los; double* sr = trig + 2 * n_los; double* cr = trig + 3 * n_los;
  for (size_t s = 0; s < n_los; ++s) {
    sd[s] = sin(dec[s]); cd[s] = cos(dec[s]); sr[s] = sin(ra[s]); cr[s] = cos(ra[s]);
  }
  J.sd = sd; J.cd = cd; J.sr = sr; J.cr = cr;
  kv* bd = (kv*)malloc(sizeof(kv) * n_los);
  for (size_t s = 0; s < n_los; ++s) { bd[s].key = dec[s]; bd[s].idx = (uint32_t)s; }
  qsort(bd, n_los, sizeof(kv), cmp_kv);
  uint32_t* by_dec = (uint32_t*)malloc(4 * n_los);
  double* dec_sorted = (double*)malloc(8 * n_los);
  for (size_t s = 0; s < n_los; ++s) { by_dec[s] = bd[s].idx; dec_sorted[s] = bd[s].key; }
  free(bd);
  J.by_dec = by_dec; J.dec_sorted = dec_sorted;
  /* cells */
  kvi* cs = (kvi*)malloc(sizeof(kvi) * n_los);
  for (size_t s = 0; s < n_los; ++s) { cs[s].key = orc_radec2pix(order, ra[s], dec[s]); cs[s].idx = (uint32_t)s; }
  qsort(cs, n_los, sizeof(kvi), cmp_kvi);
  uint32_t* members = (uint32_t*)malloc(4 * n_los);
  uint32_t* cell_start = (uint32_t*)malloc(4 * (n_los + 1));
  int64_t* cell_ids = (int64_t*)malloc(8 * n_los);
  size_t nc = 0;
  for (size_t s = 0; s < n_los; ++s) {
    if (s == 0 || cs[s].key != cs[s - 1].key) { cell_start[nc] = (uint32_t)s; cell_ids[nc] = cs[s].key; ++nc; }
    members[s] = cs[s].idx;
  }
  cell_start[nc] = (uint32_t)n_los;
  free(cs);
  J.cell_start = cell_start; J.members = members;
  const long r = run_cells(&J, nc, cell_ids, cell_subset, n_subset, nthreads, out_bins, out_cells, out_cell_ids,
                           stats);
  free(trig); free(by_dec); free(dec_sorted); free(members); free(cell_start); free(cell_ids);
  return r;
}

/*
 * orc_xi with the sightlines binned by BOSS plate (PlateBins, PlateBins.h:18-92):
 * plate[s] is sightline s's cell, cells ascending by plate id (the key order
 * of skybin_xis_); the platelist gives n_list rows of plate id and centre
 * (RACEN, DECCEN in degrees, as read from the platelist FITS file,
 * PlateBins.h:38-45).  A plate id listed twice keeps its last row (the
 * std::map assignment of PlateBins.h:44).  Cell ids are plate ids.
 */
long orc_xi_plates(const double* ra, const double* dec, const int32_t* plate, const uint64_t* off,
                   const uint32_t* npix, size_t n_los, const orc_pixel* px, const int32_t* list_plate,
                   const float* list_racen, const float* list_deccen, size_t n_list, int coord, const double* axes,
                   double scale, int mode, int nthreads, const uint32_t* cell_subset, size_t n_subset,
                   orc_xibin* out_bins, orc_xibin* out_cells, int64_t* out_cell_ids, orc_stats* stats) {
  if (n_los == 0 || coord < 0 || coord > 2) return -1;
  orc_job J;
  memset(&J, 0, sizeof J);
  make_grid(&J.g, coord, axes, scale);
  J.cos_max = cos(J.g.max_ang);
  J.mode = mode;
  J.off = off;
  J.npix = npix;
  J.px = px;
  J.n_los = n_los;
  J.dec = dec;
  double* trig = (double*)malloc(sizeof(double) * 4 * n_los);
  double* sd = trig; double* cd = trig + n_los; double* sr = trig + 2 * n_los; double* cr = trig + 3 * n_los;
  for (size_t s = 0; s < n_los; ++s) {
    sd[s] = sin(dec[s]); cd[s] = cos(dec[s]); sr[s] = sin(ra[s]); cr[s] = cos(ra[s]);
  }
  J.sd = sd; J.cd = cd; J.sr = sr; J.cr = cr;
  /* cells: sightlines by (plate, index) */
  kvi* cs = (kvi*)malloc(sizeof(kvi) * n_los);
  for (size_t s = 0; s < n_los; ++s) { cs[s].key = plate[s]; cs[s].idx = (uint32_t)s; }
  qsort(cs, n_los, sizeof(kvi), cmp_kvi);
  uint32_t* members = (uint32_t*)malloc(4 * n_los);
  uint32_t* cell_start = (uint32_t*)malloc(4 * (n_los + 1));
  int64_t* cell_ids = (int64_t*)malloc(8 * n_los);
  size_t nc = 0;
  for (size_t s = 0; s < n_los; ++s) {
    if (s == 0 || cs[s].key != cs[s - 1].key) { cell_start[nc] = (uint32_t)s; cell_ids[nc] = cs[s].key; ++nc; }
    members[s] = cs[s].idx;
  }
  cell_start[nc] = (uint32_t)n_los;
  free(cs);
  J.cell_start = cell_start; J.members = members;
  /* the platelist: ascending plate id, the last row of a repeated id */
  kvi* pl = (kvi*)malloc(sizeof(kvi) * (n_list ? n_list : 1));
  for (size_t k = 0; k < n_list; ++k) { pl[k].key = list_plate[k]; pl[k].idx = (uint32_t)k; }
  qsort(pl, n_list, sizeof(kvi), cmp_kvi);
  double* ptrig = (double*)malloc(sizeof(double) * 4 * (n_list ? n_list : 1));
  int64_t* pcell = (int64_t*)malloc(8 * (n_list ? n_list : 1));
  const double deg2rad = (atan(1.0) * 4) / 180.0;
  size_t np = 0;
  for (size_t k = 0; k < n_list; ++k) {
    if (k + 1 < n_list && pl[k + 1].key == pl[k].key) continue; /* a later row of the same plate wins */
    const uint32_t r = pl[k].idx;
    const double pra = list_racen[r] * deg2rad, pdec = list_deccen[r] * deg2rad;
    ptrig[np] = sin(pdec); ptrig[n_list + np] = cos(pdec);
    ptrig[2 * n_list + np] = sin(pra); ptrig[3 * n_list + np] = cos(pra);
    pcell[np] = -1;
    for (size_t c = 0; c < nc; ++c)
      if (cell_ids[c] == pl[k].key) pcell[np] = (int64_t)c;
    ++np;
  }
  free(pl);
  J.n_plates = np;
  J.psd = ptrig; J.pcd = ptrig + n_list; J.psr = ptrig + 2 * n_list; J.pcr = ptrig + 3 * n_list;
  J.plate_cell = pcell;
  const long r = run_cells(&J, nc, cell_ids, cell_subset, n_subset, nthreads, out_bins, out_cells, out_cell_ids,
                           stats);
  free(trig); free(ptrig); free(pcell); free(members); free(cell_start); free(cell_ids);
  return r;
}

/* Number of occupied cells and, per occupied cell (ascending id), the pixel
 * pairs its primaries would accumulate in sum N_i N_j over accepted pairs
 * (used to size a bounded baseline sample). */
long orc_cell_costs(const double* ra, const double* dec, const uint32_t* npix, size_t n_los,
                    int order, int coord, const double* axes, double scale, uint64_t* cost) {
  orc_grid g;
  make_grid(&g, coord, axes, scale);
  const double cmax = cos(g.max_ang);
  kvi* cs = (kvi*)malloc(sizeof(kvi) * n_los);
  for (size_t s = 0; s < n_los; ++s) { cs[s].key = orc_radec2pix(order, ra[s], dec[s]); cs[s].idx = (uint32_t)s; }
  qsort(cs, n_los, sizeof(kvi), cmp_kvi);
  kv* bd = (kv*)malloc(sizeof(kv) * n_los);
  for (size_t s = 0; s < n_los; ++s) { bd[s].key = dec[s]; bd[s].idx = (uint32_t)s; }
  qsort(bd, n_los, sizeof(kv), cmp_kv);
  long nc = 0;
  for (size_t s = 0; s < n_los; ++s) {
    if (s == 0 || cs[s].key != cs[s - 1].key) { if (cost) cost[nc] = 0; ++nc; }
    if (!cost) continue;
    const uint32_t i = cs[s].idx;
    const double sdi = sin(dec[i]), cdi = cos(dec[i]), sri = sin(ra[i]), cri = cos(ra[i]);
    const double lo = dec[i] - g.max_ang - 1e-9, hi = dec[i] + g.max_ang + 1e-9;
    size_t a = 0, b = n_los;
    while (a < b) { size_t m = (a + b) / 2; if (bd[m].key < lo) a = m + 1; else b = m; }
    for (size_t k = a; k < n_los && bd[k].key <= hi; ++k) {
      const uint32_t j = bd[k].idx;
      if (j <= i) continue;
      const double c = sdi * sin(dec[j]) + cdi * cos(dec[j]) * (sri * sin(ra[j]) + cri * cos(ra[j]));
      if (c <= cmax) continue;
      cost[nc - 1] += (uint64_t)npix[i] * npix[j];
    }
  }
  free(cs); free(bd);
  return nc;
}

/* ---------------- brute-force estimator ------------------------------------ */
typedef struct {
  const float* p;
  size_t n, rows; /* pairs (i, j) with i < rows and i < j < n */
  double min, max, spacing;
  int nbins;
  double* dsum; double* wsum; uint64_t* cnt; /* per thread [nbins+2] */
  int nthreads;
} orc_brute_job;
typedef struct { orc_brute_job* J; int t; } orc_brute_arg;

static void* brute_worker(void* arg) {
  orc_brute_arg* A = (orc_brute_arg*)arg;
  orc_brute_job* J = A->J;
  const int nb = J->nbins + 2;
  double* ds = J->dsum + (size_t)A->t * nb;
  double* ws = J->wsum + (size_t)A->t * nb;
  uint64_t* ct = J->cnt + (size_t)A->t * nb;
  for (size_t i = (size_t)A->t; i < J->rows; i += (size_t)J->nthreads) {
    const float* a = J->p + 5 * i;
    const double wdi = (double)a[4] * (double)a[3], wi = a[4];
    for (size_t j = i + 1; j < J->n; ++j) {
      const float* b = J->p + 5 * j;
      const double dx = (double)a[0] - (double)b[0], dy = (double)a[1] - (double)b[1],
                   dz = (double)a[2] - (double)b[2];
      const double r = sqrt(dx * dx + dy * dy + dz * dz);
      int idx;
      if (r < J->min) idx = 0;
      else if (r >= J->max) idx = J->nbins + 1;
      else {
        double k = floor((r - J->min) / J->spacing);
        if (k > J->nbins - 1) k = J->nbins - 1;
        idx = (int)k + 1;
      }
      ds[idx] += wdi * ((double)b[4] * (double)b[3]);
      ws[idx] += wi * (double)b[4];
      ct[idx] += 1;
    }
  }
  return NULL;
}

/* Pairs (i, j), i < rows and i < j < n, of n points (x,y,z,delta,w rows);
 * outputs nbins+2 entries.  rows = n gives all pairs. */
int orc_brute_rows(const float* points, size_t n, size_t rows, double min, double max, int nbins, int nthreads,
                   double* dsum, double* wsum, uint64_t* counts) {
  if (nthreads < 1) nthreads = 1;
  const int nb = nbins + 2;
  orc_brute_job J;
  J.p = points; J.n = n; J.rows = rows < n ? rows : n; J.min = min; J.max = max; J.spacing = (max - min) / nbins; J.nbins = nbins;
  J.nthreads = nthreads;
  J.dsum = (double*)calloc((size_t)nthreads * nb, 8);
  J.wsum = (double*)calloc((size_t)nthreads * nb, 8);
  J.cnt = (uint64_t*)calloc((size_t)nthreads * nb, 8);
  pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * nthreads);
  orc_brute_arg* args = (orc_brute_arg*)malloc(sizeof(orc_brute_arg) * nthreads);
  for (int t = 0; t < nthreads; ++t) { args[t].J = &J; args[t].t = t; pthread_create(&th[t], NULL, brute_worker, &args[t]); }
  for (int t = 0; t < nthreads; ++t) pthread_join(th[t], NULL);
  for (int b = 0; b < nb; ++b) { dsum[b] = 0; wsum[b] = 0; counts[b] = 0; }
  for (int t = 0; t < nthreads; ++t)
    for (int b = 0; b < nb; ++b) {
      dsum[b] += J.dsum[(size_t)t * nb + b];
      wsum[b] += J.wsum[(size_t)t * nb + b];
      counts[b] += J.cnt[(size_t)t * nb + b];
    }
  free(J.dsum); free(J.wsum); free(J.cnt); free(th); free(args);
  return 0;
}

/* All pairs i < j of n points. */
int orc_brute(const float* points, size_t n, double min, double max, int nbins, int nthreads,
              double* dsum, double* wsum, uint64_t* counts) {
  return orc_brute_rows(points, n, n, min, max, nbins, nthreads, dsum, wsum, counts);
}

/* Exact single-pair binning, for tests of the expression order. Returns 1
 * and the flat index when the pair is accumulated, 0 when skipped. */
int orc_bin_pair(int coord, const double* axes, double scale, float d1, float l1, float d2,
                 float l2, double c, uint32_t* idx) {
  orc_job J;
  memset(&J, 0, sizeof J);
  make_grid(&J.g, coord, axes, scale);
  orc_pixel p1 = {1.0f, l1, 1.0f, d1}, p2 = {1.0f, l2, 1.0f, d2};
  uint64_t off[2] = {0, 1};
  uint32_t np[2] = {1, 1};
  orc_pixel px[2] = {p1, p2};
  J.off = off; J.npix = np; J.px = px; J.mode = 1;
  orc_xibin* xi = (orc_xibin*)calloc(J.g.ntotal, sizeof(orc_xibin));
  uint64_t ovf = 0;
  const uint64_t used = pixel_pairs(&J, 0, 1, c, xi, &ovf);
  int found = 0;
  for (uint32_t b = 0; b < J.g.ntotal; ++b) if (xi[b].num_pairs) { *idx = b; found = 1; }
  if (!found && ovf) { *idx = 0xFFFFFFFFu; found = 1; }
  free(xi);
  return used ? found : 0;
}
