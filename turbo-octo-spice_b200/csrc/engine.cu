// engine.cu — engine, catalogue upload, sightline-pair expansion and the
// XiEstimator run entry point of the C ABI (include/tos_b200.h).
#include <cub/cub.cuh>

#include <memory>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <string>
#include <vector>

#include "cosmology.h"
#include "engine_internal.h"
#include "healpix.h"
#include "fixed128.cuh"
#include "xi_kernels.cuh"

namespace tos {

namespace {
thread_local std::string g_error;
}  // namespace

void set_error(const std::string& msg) { g_error = msg; }
tos_status fail(tos_status s, const std::string& msg) {
  g_error = msg;
  return s;
}

namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;

// ---- catalogue preparation -------------------------------------------------

__global__ void k_fill_pack(PixPack* p, size_t n) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    PixPack q;
    q.d = kSentinel;
    q.w = 0.f;
    q.wd = 0.0;
    p[k] = q;
  }
}

__global__ void k_fill(float* p, size_t n, float v) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n;
       k += (size_t)gridDim.x * blockDim.x)
    p[k] = v;
}

// One warp per sightline: scatter pixels into the padded coordinate arrays,
// w*delta (exact product of two floats in double), weights; exclusive prefix
// sums of (w*delta, w, loglam); coordinate ranges; sortedness.
__global__ void k_prep(const tos_pixel* raw, const uint64_t* off, const uint32_t* npix,
                       size_t n_los, float* dist_pad, float* loglam_pad, PixPack* pack, double* wd, float* w,
                       double4* prefix, float4* range, unsigned int* flags,
                       unsigned long long* maxbits) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t s = warp; s < n_los; s += nwarps) {
    const uint64_t o = off[s];
    const uint32_t n = npix[s];
    const uint64_t po = o + (uint64_t)kPad * (s + 1);
    double4* pre = prefix + o + s;
    double c0 = 0, c1 = 0, c2 = 0;
    float dmin = INFINITY, dmax = -INFINITY, lmin = INFINITY, lmax = -INFINITY;
    double mwd = 0, mw = 0, ml = 0, md = 0;
    float gap = INFINITY;  // smallest positive step between consecutive distances
    bool unsorted = false;
    if (lane == 0) pre[0] = make_double4(0, 0, 0, 0);
    for (uint32_t b = 0; b < n; b += 32) {
      const uint32_t k = b + lane;
      double v0 = 0, v1 = 0, v2 = 0;
      if (k < n) {
        const tos_pixel px = raw[o + k];
        dist_pad[po + k] = px.distance;
        loglam_pad[po + k] = px.loglam;
        v0 = (double)px.weight * (double)px.value;
        v1 = (double)px.weight;
        v2 = (double)px.loglam;
        wd[o + k] = v0;
        w[o + k] = px.weight;
        PixPack q;
        q.d = px.distance;
        q.w = px.weight;
        q.wd = v0;
        pack[po + k] = q;
        dmin = fminf(dmin, px.distance);
        dmax = fmaxf(dmax, px.distance);
        lmin = fminf(lmin, px.loglam);
        lmax = fmaxf(lmax, px.loglam);
        mwd = fmax(mwd, fabs(v0));
        mw = fmax(mw, fabs(v1));
        ml = fmax(ml, fabs(v2));
        md = fmax(md, fabs((double)px.distance));
        if (!isfinite(px.value) || !isfinite(px.weight) || !isfinite(px.loglam) ||
            !isfinite(px.distance))
          atomicOr(flags, 2u);
        if (k + 1 < n) {
          const tos_pixel nx = raw[o + k + 1];
          if (!(nx.distance >= px.distance) || !(nx.loglam >= px.loglam)) unsorted = true;
          if (nx.distance > px.distance) gap = fminf(gap, __fsub_rd(nx.distance, px.distance));
        }
      }
      // inclusive warp scan, in order, of the three sums
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
        const double u0 = __shfl_up_sync(kFull, v0, d), u1 = __shfl_up_sync(kFull, v1, d),
                     u2 = __shfl_up_sync(kFull, v2, d);
        if (lane >= d) {
          v0 += u0;
          v1 += u1;
          v2 += u2;
        }
      }
      if (k < n) pre[k + 1] = make_double4(c0 + v0, c1 + v1, c2 + v2, 0);
      c0 += __shfl_sync(kFull, v0, 31);
      c1 += __shfl_sync(kFull, v1, 31);
      c2 += __shfl_sync(kFull, v2, 31);
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      dmin = fminf(dmin, __shfl_xor_sync(kFull, dmin, d));
      dmax = fmaxf(dmax, __shfl_xor_sync(kFull, dmax, d));
      lmin = fminf(lmin, __shfl_xor_sync(kFull, lmin, d));
      lmax = fmaxf(lmax, __shfl_xor_sync(kFull, lmax, d));
      mwd = fmax(mwd, __shfl_xor_sync(kFull, mwd, d));
      mw = fmax(mw, __shfl_xor_sync(kFull, mw, d));
      ml = fmax(ml, __shfl_xor_sync(kFull, ml, d));
      md = fmax(md, __shfl_xor_sync(kFull, md, d));
      gap = fminf(gap, __shfl_xor_sync(kFull, gap, d));
    }
    unsorted = __any_sync(kFull, unsorted);
    if (lane == 0) {
      range[s] = make_float4(dmin, dmax, lmin, lmax);
      if (unsorted) atomicOr(flags, 1u);
      if (n > 0) {
        // order key of a float: unsigned comparison of keys = float comparison
        const unsigned u = __float_as_uint(dmin);
        atomicMin(&flags[1], (u & 0x80000000u) ? ~u : (u | 0x80000000u));
      }
      atomicMin(&flags[2], __float_as_uint(gap));  // non-negative: bits order like values
      // non-negative doubles order like their bit patterns
      atomicMax(&maxbits[0], (unsigned long long)__double_as_longlong(mwd));
      atomicMax(&maxbits[1], (unsigned long long)__double_as_longlong(mw));
      atomicMax(&maxbits[2], (unsigned long long)__double_as_longlong(ml));
      atomicMax(&maxbits[3], (unsigned long long)__double_as_longlong(md));
    }
  }
}

// ---- sightline-pair expansion ----------------------------------------------

// Conservative cell neighbours: cells A, B can hold a sightline pair within
// max_ang only if the angle between their caps' centres is at most
// max_ang + r_A + r_B (caps bound every member).  Only cells of A's own
// sightline group are searched.
__global__ void k_cell_neighbours(const double4* cap, const uint2* grange, uint32_t n_cells,
                                  double max_ang, const uint32_t* start, uint32_t* count,
                                  uint32_t* out) {
  for (uint32_t a = blockIdx.x * blockDim.x + threadIdx.x; a < n_cells;
       a += gridDim.x * blockDim.x) {
    const double4 ca = cap[a];
    const uint2 gr = grange[a];
    uint32_t n = 0;
    uint32_t o = out ? start[a] : 0;
    for (uint32_t b = gr.x; b < gr.y; ++b) {
      const double4 cb = cap[b];
      const double lim = max_ang + ca.w + cb.w + 1e-9;
      bool near;
      if (lim >= 3.14159) {
        near = true;
      } else {
        const double dot = ca.x * cb.x + ca.y * cb.y + ca.z * cb.z;
        near = dot >= cos(lim) - 1e-12;
      }
      if (near) {
        if (out) out[o + n] = b;
        ++n;
      }
    }
    if (!out) count[a] = n;
  }
}

// Plate cells: PlateBins::getBinIndicesWithinRadius (PlateBins.h:73-84) for
// every sightline i, as a per-sightline neighbour list of cell indices:
// the platelist plates k (ascending id) whose centre passes
//   |acos(cos_sep(i, k)) - ring| < max_ang,   ring = 1.5 deg,
// and that hold sightlines of i's group.  cos_sep has the reference's bits
// (ref_cos_sep, the host trig of both); the device acos may differ from the
// host libm's in the last bits, so a test within kPlateEdgeMargin of its
// threshold is settled on the host: pass 0 records it (key i << 32 | k and
// the cosine), passes 1 and 2 look up the host's decision.
constexpr double kPlateEdgeMargin = 1e-12;
constexpr uint32_t kPlateEdgeCap = 65536;
// edge buffer: [0] count, [1, 1 + cap) sorted keys, [1 + cap, 1 + 2 cap)
// pass 0: the cosines' bits, passes 1-2: the host's decisions (0 or 1)

// 1 pass, 0 fail, 2 within the margin
__device__ __forceinline__ int plate_ring(const SkyTrig& si, const double4 pt, double ring, double max_ang,
                                          double* c_out) {
  const double c = ref_cos_sep(si, SkyTrig{pt.x, pt.y, pt.z, pt.w});
  *c_out = c;
  const double v = fabs(acos(c) - ring) - max_ang;
  if (isnan(v)) return 0;  // |c| > 1: acos is NaN on the host too, and NaN < max_ang fails
  if (v < -kPlateEdgeMargin) return 1;
  if (v > kPlateEdgeMargin) return 0;
  return 2;
}

__device__ bool plate_edge_decision(const unsigned long long* edge, unsigned long long key) {
  const uint32_t n = (uint32_t)min(edge[0], (unsigned long long)kPlateEdgeCap);
  uint32_t a = 0, b = n;
  while (a < b) {
    const uint32_t m = (a + b) >> 1;
    if (edge[1 + m] < key) a = m + 1; else b = m;
  }
  return a < n && edge[1 + a] == key && edge[1 + kPlateEdgeCap + a] != 0;
}

// One warp per sightline, lanes over the platelist.  pass 0: record the
// tests within the margin; pass 1: count[i] = neighbour cells; pass 2: write
// them at out[start[i] ...] in ascending plate order.
__global__ void k_plate_neighbours(int pass, const double4* trig, const uint32_t* cell_idx, const uint2* grange,
                                   const int64_t* cells, size_t n_los, const int32_t* plate_ids,
                                   const double4* plate_trig, uint32_t n_plates, double ring, double max_ang,
                                   unsigned long long* edge, uint32_t* count, const uint32_t* start,
                                   uint32_t* out) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t i = warp; i < n_los; i += nwarps) {
    const double4 ti = trig[i];
    const SkyTrig si{ti.x, ti.y, ti.z, ti.w};
    const uint32_t ca = cell_idx[i];
    const uint2 gr = grange[ca];
    const int64_t gkey = cells[ca] & ~0xFFFFFFFFll;
    uint32_t n = 0;
    const uint32_t o = (pass == 2) ? start[i] : 0;
    for (uint32_t base = 0; base < n_plates; base += 32) {
      const uint32_t k = base + lane;
      bool hit = false;
      uint32_t cell = 0;
      if (k < n_plates) {
        double c;
        int r = plate_ring(si, plate_trig[k], ring, max_ang, &c);
        const unsigned long long key = ((unsigned long long)i << 32) | k;
        if (r == 2) {
          if (pass == 0) {
            const unsigned long long slot = atomicAdd(&edge[0], 1ull);
            if (slot < kPlateEdgeCap) {
              edge[1 + slot] = key;
              edge[1 + kPlateEdgeCap + slot] = (unsigned long long)__double_as_longlong(c);
            }
          }
          r = (pass != 0 && plate_edge_decision(edge, key)) ? 1 : 0;
        }
        if (r == 1 && pass != 0) {
          // the cell (group of i, plate k), if occupied: binary search in the group's cells
          const int64_t want = gkey | (int64_t)plate_ids[k];
          uint32_t a = gr.x, b = gr.y;
          while (a < b) {
            const uint32_t m = (a + b) >> 1;
            if (cells[m] < want) a = m + 1; else b = m;
          }
          if (a < gr.y && cells[a] == want) {
            hit = true;
            cell = a;
          }
        }
      }
      const unsigned m = __ballot_sync(kFull, hit);
      if (pass == 2 && hit) out[o + n + __popc(m & ((1u << lane) - 1u))] = cell;
      n += __popc(m);
    }
    if (pass == 1 && lane == 0) count[i] = n;
  }
}

// One warp per primary sightline (in cell order).  Pass 1 (items == null)
// counts accepted pairs and candidates; pass 2 writes the accepted pairs at
// their offsets in a fixed order (neighbour cells ascending, j ascending).
// The neighbour cells are the CSR nb_start/nb of the primary's cell, or of
// the primary itself (nb_by_sightline: plate cells).
// Mirrors skybin_xi_task's loop (XiEstimator.cc:130-152): skip j <= i, cut
// cos(theta) <= cos_max.
__global__ void k_expand(const uint32_t* members, uint32_t n_members, const uint32_t* cell_idx,
                         const uint32_t* cell_start, const uint32_t* nb_start, const uint32_t* nb,
                         int nb_by_sightline, const double4* trig, const uint32_t* npix, double cos_max,
                         uint32_t* cnt, unsigned long long* cand, unsigned long long* cell_pairs,
                         const uint32_t* item_off, uint32_t* item_i, uint32_t* item_j,
                         double* item_c, uint32_t* item_sep, int coord, double theta_min,
                         double theta_inv, unsigned long long* sep_flagged) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t p = warp; p < n_members; p += nwarps) {
    const uint32_t i = members[p];
    const uint32_t ca = cell_idx[i];
    const double4 ti = trig[i];
    const SkyTrig si{ti.x, ti.y, ti.z, ti.w};
    uint32_t n_acc = 0;
    unsigned long long n_cand = 0, n_pairs = 0;
    uint32_t o = item_i ? item_off[p] : 0;
    const uint32_t nbk = nb_by_sightline ? i : ca;  // plate cells: sightline i's own list
    for (uint32_t q = nb_start[nbk]; q < nb_start[nbk + 1]; ++q) {
      const uint32_t cb = nb[q];
      const uint32_t b0 = cell_start[cb], b1 = cell_start[cb + 1];
      for (uint32_t base = b0; base < b1; base += 32) {
        const uint32_t k = base + lane;
        bool cnd = false, acc = false;
        double c = 0;
        uint32_t j = 0;
        if (k < b1) {
          j = members[k];
          if (j > i) {
            cnd = true;
            const double4 tj = trig[j];
            c = ref_cos_sep(si, SkyTrig{tj.x, tj.y, tj.z, tj.w});
            acc = !(c <= cos_max);
          }
        }
        const unsigned mc = __ballot_sync(kFull, cnd), ma = __ballot_sync(kFull, acc);
        n_cand += __popc(mc);
        if (acc) n_pairs += npix[j];
        if (item_i && acc) {
          const uint32_t at = o + n_acc + __popc(ma & ((1u << lane) - 1u));
          item_i[at] = i;
          item_j[at] = j;
          item_c[at] = c;
          if (coord == TOS_OBSERVING) {
            // theta index of XiEstimator.cc:166, 273 (acos, unchecked)
            const double th = acos(c);
            const double t = dmul(dsub(th, theta_min), theta_inv);
            item_sep[at] = ref_u32(t);
            const double fr = t - floor(t);
            if (fr < 1e-9 || fr > 1.0 - 1e-9) {
              const unsigned long long slot = atomicAdd(&sep_flagged[0], 1ull);
              if (slot < 4096) sep_flagged[1 + slot] = at;
            }
          }
        }
        n_acc += __popc(ma);
      }
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) n_pairs += __shfl_xor_sync(kFull, n_pairs, d);
    if (!item_i && lane == 0) {
      cnt[p] = n_acc;
      cand[p] = n_cand;
      atomicAdd(&cell_pairs[ca], n_pairs * (unsigned long long)npix[i]);
    }
  }
}

// ---- results ----------------------------------------------------------------

// Per bin: convert every cell's 128-bit fixed-point sums to double and add
// them in ascending cell order (the order of xi_finalize_task,
// XiEstimator.cc:298-305).
__global__ void k_combine(const unsigned long long* acc, uint32_t n_cells, uint32_t nb,
                          double4 inv_a, double4 inv_b, tos_xibin* out, tos_xibin* cells_out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    const double inv[7] = {inv_a.x, inv_a.y, inv_a.z, inv_a.w, inv_b.x, inv_b.y, inv_b.z};
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    long long n = 0;
    for (uint32_t c = 0; c < n_cells; ++c) {
      const unsigned long long* a = acc + ((size_t)c * nb + b) * kAccWords;
      // a bin without pairs has zero sums: the telescoped dipoles of its
      // neighbours cancel in it only up to the rounding of their FP64 sums
      const long long cnt = (long long)a[14];
      double v[7];
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        v[k] = (cnt != 0) ? i128_double(acc128(a, k)) * inv[k] : 0.0;
        s[k] += v[k];
      }
      n += cnt;
      if (cells_out) {
        tos_xibin x;
        x.didj = v[0];
        x.di = v[1];
        x.dj = v[2];
        x.wgt = v[3];
        x.wi = v[4];
        x.wj = v[5];
        x.z = v[6];
        x.num_pairs = cnt;
        cells_out[(size_t)c * nb + b] = x;
      }
    }
    tos_xibin x;
    x.didj = s[0];
    x.di = s[1];
    x.dj = s[2];
    x.wgt = s[3];
    x.wi = s[4];
    x.wj = s[5];
    x.z = s[6];
    x.num_pairs = n;
    out[b] = x;
  }
}

// Per (group, bin): the group's cells merged in ascending cell order, the
// merge k_combine makes over all cells of a one-group catalogue.
__global__ void k_combine_groups(const unsigned long long* acc, const uint32_t* gstart,
                                 uint32_t n_groups, uint32_t nb, double4 inv_a, double4 inv_b,
                                 tos_xibin* groups_out) {
  const size_t n = (size_t)n_groups * nb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const uint32_t g = (uint32_t)(t / nb), b = (uint32_t)(t % nb);
    const double inv[7] = {inv_a.x, inv_a.y, inv_a.z, inv_a.w, inv_b.x, inv_b.y, inv_b.z};
    double s[7] = {0, 0, 0, 0, 0, 0, 0};
    long long cnt_sum = 0;
    for (uint32_t c = gstart[g]; c < gstart[g + 1]; ++c) {
      const unsigned long long* a = acc + ((size_t)c * nb + b) * kAccWords;
      const long long cnt = (long long)a[14];
      if (cnt == 0) continue;  // no pairs: zero sums (as k_combine)
#pragma unroll
      for (int k = 0; k < 7; ++k) s[k] += i128_double(acc128(a, k)) * inv[k];
      cnt_sum += cnt;
    }
    tos_xibin x;
    x.didj = s[0];
    x.di = s[1];
    x.dj = s[2];
    x.wgt = s[3];
    x.wi = s[4];
    x.wj = s[5];
    x.z = s[6];
    x.num_pairs = cnt_sum;
    groups_out[t] = x;
  }
}

// Per bin: the groups' rows added in ascending group order.
__global__ void k_sum_groups(const tos_xibin* groups, uint32_t n_groups, uint32_t nb,
                             tos_xibin* out) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    tos_xibin x{};
    for (uint32_t g = 0; g < n_groups; ++g) {
      const tos_xibin y = groups[(size_t)g * nb + b];
      x.didj += y.didj;
      x.di += y.di;
      x.dj += y.dj;
      x.wgt += y.wgt;
      x.wi += y.wi;
      x.wj += y.wj;
      x.z += y.z;
      x.num_pairs += y.num_pairs;
    }
    out[b] = x;
  }
}

}  // namespace

void launch_sum_rows(const tos_xibin* rows, uint32_t n_rows, uint32_t nb, tos_xibin* out,
                     int blocks, cudaStream_t st) {
  k_sum_groups<<<blocks, 128, 0, st>>>(rows, n_rows, nb, out);
}

namespace {

int grid_for(const tos_engine* e, size_t work, int block) {
  size_t g = (work + block - 1) / block;
  size_t cap = (size_t)e->num_sms * 16;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// First-axis bin of a float separation r >= 0 as the reference decides it
// (XiEstimator.cc:243, 280): -1 below the axis (t <= -1, where ref_u32 wraps),
// the bin, or n above the axis.  Non-decreasing in r.
int first_axis_code(float r, double min, double inv, uint32_t n) {
  const double t = dmul(dsub((double)r, min), inv);
  if (!(t > -1.0)) return -1;
  if (t >= (double)n) return (int)n;
  return (int)ref_u32(t);
}

// Smallest float r >= 0 whose first-axis code is >= k (k = 0..n); +inf when
// there is none.  T[0] is the first accepted separation, T[k] <= r < T[k+1]
// is bin k, and every |fl32(x1 - x2)| >= T[n] is rejected.
float first_axis_threshold(double min, double inv, uint32_t n, int k) {
  auto reached = [&](float r) { return first_axis_code(r, min, inv, n) >= k; };
  if (reached(0.0f)) return 0.0f;
  float hi = (float)std::max(1.0, min + (double)k / inv);
  int guard = 0;
  while (!reached(hi) && guard++ < 200) hi = hi * 2.0f + 1.0f;
  if (!reached(hi)) return INFINITY;
  // bisection over the ordered bit patterns of non-negative floats
  uint32_t a = 0, b;
  std::memcpy(&b, &hi, 4);
  while (b - a > 1) {
    const uint32_t m = a + (b - a) / 2;
    float fm;
    std::memcpy(&fm, &m, 4);
    if (reached(fm))
      b = m;
    else
      a = m;
  }
  float r;
  std::memcpy(&r, &b, 4);
  return r;
}

int bitlen(uint32_t v) {
  int b = 0;
  while (v) {
    ++b;
    v >>= 1;
  }
  return b;
}

bool is_pow2(double v) {
  if (!(v > 0) || !std::isfinite(v)) return false;
  int e;
  const double m = std::frexp(v, &e);
  return m == 0.5;
}

}  // namespace

// ---- grid helpers -----------------------------------------------------------

tos_status check_grid(const tos_grid* g) {
  if (!g) return fail(TOS_ERR_INVALID_ARG, "grid is null");
  if (g->type != TOS_POLAR && g->type != TOS_CARTESIAN && g->type != TOS_OBSERVING)
    return fail(TOS_ERR_INVALID_ARG, "unknown coordinate type");
  for (int k = 0; k < 3; ++k) {
    const tos_axis& a = g->axis[k];
    if (a.nbins <= 0 || a.nbins > 32767)
      return fail(TOS_ERR_INVALID_ARG, "axis bins must be in [1, 32767]");
    if (!std::isfinite(a.min) || !std::isfinite(a.max) || !(a.max > a.min))
      return fail(TOS_ERR_INVALID_ARG, "axis needs finite min < max");
  }
  const double total = (double)g->axis[0].nbins * g->axis[1].nbins * g->axis[2].nbins;
  if (total > 1.0e7) return fail(TOS_ERR_UNSUPPORTED, "grid has more than 1e7 bins");
  return TOS_OK;
}

double max_angular_scale(const tos_grid& g, double scale) {
  switch (g.type) {
    case TOS_CARTESIAN: return axis_high(g.axis[1]) / scale;  // CartesianGrid.h:46
    case TOS_POLAR:  // PolarGrid.h:46
      return axis_high(g.axis[0]) * std::sqrt(1.0 - g.axis[1].min * g.axis[1].min) / scale;
    default: return axis_high(g.axis[1]);  // QuasarGrid.h:45 (no scaling)
  }
}

}  // namespace tos

using namespace tos;

// ---------------------------------------------------------------------------
// Common first-axis grid of a catalogue (grid sweep, xi_grid.cu)
// ---------------------------------------------------------------------------

// One warp per sightline: grid index of pixel 0 when the sightline's values
// are consecutive entries of the sorted distinct values U, else kNoGrid.
__global__ void k_grid_first(const float* xpad, const uint64_t* off, const uint32_t* npix,
                             size_t n_los, const float* U, int ng, uint32_t* gfirst,
                             unsigned long long* n_ok) {
  const int lane = threadIdx.x & 31;
  const size_t warp = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
  const size_t nwarps = ((size_t)gridDim.x * blockDim.x) >> 5;
  for (size_t s = warp; s < n_los; s += nwarps) {
    const uint32_t n = npix[s];
    const float* x = xpad + off[s] + (uint64_t)kPad * (s + 1);
    uint32_t f = kNoGrid;
    if (n > 0) {
      int lo = 0, hi = ng;  // first U >= x[0]
      const float x0 = x[0];
      while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (U[mid] < x0)
          lo = mid + 1;
        else
          hi = mid;
      }
      bool ok = (uint64_t)lo + n <= (uint64_t)ng;
      for (uint32_t p = lane; ok && p < n; p += 32) ok = U[lo + p] == x[p];
      ok = __all_sync(kFull, ok);
      if (ok) f = (uint32_t)lo;
    }
    if (lane == 0) {
      gfirst[s] = f;
      if (f != kNoGrid) atomicAdd(n_ok, 1ull);
    }
  }
}

// Boundary table B[g][t], t = 0 .. 2 nk - 1 (nk = n0 + 1 thresholds): the
// first grid index g2 whose value x2 = U[g2] passes the boundary predicate of
// threshold T[k] against x1 = U[g],
//   side 1, t <= n0 (k = n0 - t):      x2 >= x1 or  fl(x1 - x2) <  T[k];
//   side 0, t = n0 + 1 + k:            x2 >= x1 and fl(x2 - x1) >= T[k].
// Along t the entries are non-decreasing, so the row's columns split into the
// consecutive runs [B[t], B[t+1]): first-axis bin n0 - 1 - t below x1
// (t < n0), the |x1 - x2| < T[0] gap (t = n0), bin t - n0 - 1 above x1.
__global__ void k_grid_table(const float* U, int ng, const float* thr, int nk, uint16_t* Q) {
  const int nb = 2 * nk;
  const size_t total = (size_t)ng * nb;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const int tb = (int)(e % nb);
    const int g = (int)(e / nb);
    const int side = tb < nk ? 1 : 0;
    const int k = side ? nk - 1 - tb : tb - nk;
    const float x1 = U[g], t = thr[k];
    int lo = 0, hi = ng;
    while (lo < hi) {
      const int mid = (lo + hi) >> 1;
      const float x2 = U[mid];
      const bool ge = x2 >= x1;
      const bool pass = side ? (ge || !(__fsub_rn(x1, x2) >= t)) : (ge && __fsub_rn(x2, x1) >= t);
      if (pass)
        hi = mid;
      else
        lo = mid + 1;
    }
    Q[e] = (uint16_t)lo;
  }
}

// Build (once per catalogue and coordinate) the sorted distinct values of the
// padded coordinate array and the per-sightline grid offsets.  Grids of more
// than 65535 values are not used.
tos_status ensure_grid(tos_engine* e, tos_catalog* cat, int w, cudaStream_t st) {
  std::lock_guard<std::mutex> lock(cat->grid_mu);
  if (cat->grid_built[w]) return TOS_OK;
  const float* x = (w == 0) ? cat->d_dist_pad.p : cat->d_loglam_pad.p;
  const size_t n = (w == 0) ? cat->d_dist_pad.n : cat->d_loglam_pad.n;
  if (n > (size_t)0x7FFFFFFF) {  // beyond the 32-bit item counts of the sort
    cat->grid_built[w] = true;
    cat->grid_n[w] = 0;
    return TOS_OK;
  }
  DevBuf<float> sorted, uniq;
  DevBuf<int> nsel;
  TOS_TRY(sorted.alloc(n));
  TOS_TRY(uniq.alloc(n));
  TOS_TRY(nsel.alloc(1));
  size_t tb1 = 0, tb2 = 0;
  cub::DeviceRadixSort::SortKeys(nullptr, tb1, x, sorted.p, (int)n, 0, 32, st);
  cub::DeviceSelect::Unique(nullptr, tb2, sorted.p, uniq.p, nsel.p, (int)n, st);
  DevBuf<unsigned char> tmp;
  TOS_TRY(tmp.alloc(std::max(tb1, tb2) + 16));
  TOS_CUDA_TRY(cub::DeviceRadixSort::SortKeys(tmp.p, tb1, x, sorted.p, (int)n, 0, 32, st));
  TOS_CUDA_TRY(cub::DeviceSelect::Unique(tmp.p, tb2, sorted.p, uniq.p, nsel.p, (int)n, st));
  int ng = 0;
  TOS_CUDA_TRY(cudaMemcpyAsync(&ng, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  // the padding sentinel is the largest value: not part of the grid
  if (ng > 0) {
    float last = 0;
    TOS_CUDA_TRY(cudaMemcpy(&last, uniq.p + ng - 1, sizeof(float), cudaMemcpyDeviceToHost));
    if (last == kSentinel) --ng;
  }
  cat->grid_built[w] = true;
  cat->grid_n[w] = 0;
  if (ng <= 0 || ng > 65535) return TOS_OK;
  TOS_TRY(cat->d_grid[w].alloc(ng));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_grid[w].p, uniq.p, ng * sizeof(float), cudaMemcpyDeviceToDevice, st));
  TOS_TRY(cat->d_gfirst[w].alloc(cat->n_los));
  TOS_CUDA_TRY(cudaMemsetAsync(nsel.p, 0, sizeof(int), st));
  DevBuf<unsigned long long> nok;
  TOS_TRY(nok.alloc(1));
  TOS_CUDA_TRY(cudaMemsetAsync(nok.p, 0, 8, st));
  k_grid_first<<<grid_for(e, cat->n_los * 32, 256), 256, 0, st>>>(
      x, cat->d_off.p, cat->d_npix.p, cat->n_los, cat->d_grid[w].p, ng, cat->d_gfirst[w].p, nok.p);
  TOS_CUDA_TRY(cudaGetLastError());
  unsigned long long h = 0;
  TOS_CUDA_TRY(cudaMemcpyAsync(&h, nok.p, 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  cat->grid_n[w] = ng;
  cat->grid_los[w] = h;
  return TOS_OK;
}

// Smallest and largest loglam of the pixels as ordered float bits
// (mm[0] = min, mm[1] = max), and whether one is not finite (mm[2]).
__device__ __forceinline__ unsigned int float_order(float f) {
  const unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

__global__ void k_loglam_range(const tos_pixel* px, size_t n, unsigned int* mm) {
  unsigned int lo = 0xFFFFFFFFu, hi = 0u, bad = 0u;
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x) {
    const float l = px[k].loglam;
    if (!isfinite(l)) bad = 1u;
    const unsigned int o = float_order(l);
    lo = min(lo, o);
    hi = max(hi, o);
  }
  for (int o = 16; o > 0; o >>= 1) {
    lo = min(lo, __shfl_xor_sync(0xFFFFFFFFu, lo, o));
    hi = max(hi, __shfl_xor_sync(0xFFFFFFFFu, hi, o));
    bad |= __shfl_xor_sync(0xFFFFFFFFu, bad, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&mm[0], lo);
    atomicMax(&mm[1], hi);
    if (bad) atomicOr(&mm[2], 1u);
  }
}

// Every pixel's distance from its loglam (cosmology.h: the same bits as the
// host's tos_fill_distances).
__global__ void k_fill_distances(tos_pixel* px, size_t n, double log_lya, const double* table, size_t nt,
                                 double om, double dz) {
  for (size_t k = blockIdx.x * (size_t)blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    px[k].distance = pixel_distance_hd(px[k].loglam, log_lya, table, nt, om, dz);
}

// Fill the distances of the catalogue's device pixels (d_raw, n of them)
// for a flat universe of matter density `om` (stream st).  Fails like
// tos_fill_distances on a loglam that is not finite or gives z < 0.
tos_status fill_distances_device(tos_engine* e, tos_pixel* d_px, size_t n, double om, cudaStream_t st) {
  if (!(om > 0 && om <= 1)) return fail(TOS_ERR_INVALID_ARG, "omega_matter must be in (0, 1]");
  if (n == 0) return TOS_OK;
  DevBuf<unsigned int> mm;
  TOS_TRY(mm.alloc(3));
  const unsigned int init[3] = {0xFFFFFFFFu, 0u, 0u};
  TOS_CUDA_TRY(cudaMemcpyAsync(mm.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_loglam_range<<<grid_for(e, n, 256), 256, 0, st>>>(d_px, n, mm.p);
  TOS_CUDA_TRY(cudaGetLastError());
  unsigned int h[3];
  TOS_CUDA_TRY(cudaMemcpyAsync(h, mm.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  auto unorder = [](unsigned int o) {
    const unsigned int u = (o & 0x80000000u) ? (o & 0x7FFFFFFFu) : ~o;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
  };
  const double lya = log_lya();
  const float lmin = unorder(h[0]), lmax = unorder(h[1]);
  if (h[2] || !(pixel_z_hd(lmin, lya) >= 0))
    return fail(TOS_ERR_INVALID_ARG, "pixel loglam must be finite and at least log10(1216)");
  // one table step of margin above the largest z covers rounding
  std::vector<double> table;
  double dz = 0;
  dc_table(om, pixel_z_hd(lmax, lya) + 2e-3, &table, &dz);
  DevBuf<double> d_table;
  TOS_TRY(d_table.alloc(table.size()));
  TOS_CUDA_TRY(cudaMemcpyAsync(d_table.p, table.data(), table.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  k_fill_distances<<<grid_for(e, n, 256), 256, 0, st>>>(d_px, n, lya, d_table.p, table.size(), om, dz);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaStreamSynchronize(st));  // the table buffer is freed on return
  return TOS_OK;
}

// ============================================================================
// C ABI
// ============================================================================

extern "C" {

const char* tos_last_error(void) { return tos::g_error.c_str(); }
int tos_abi_version(void) { return TOS_ABI_VERSION; }

tos_status tos_engine_create(int device, tos_engine** out) {
  if (!out) return fail(TOS_ERR_INVALID_ARG, "out is null");
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return fail(TOS_ERR_NO_DEVICE, "no CUDA device");
  }
  if (device < 0 || device >= n) return fail(TOS_ERR_NO_DEVICE, "device id out of range");
  cudaDeviceProp prop;
  TOS_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
  if (prop.major < 10)
    return fail(TOS_ERR_NO_DEVICE, "device is not sm_100 (Blackwell): " + std::string(prop.name));
  auto* e = new tos_engine();
  e->device = device;
  e->num_sms = prop.multiProcessorCount;
  e->smem_optin = prop.sharedMemPerBlockOptin;
  DeviceGuard g(device);
  if (cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete e;
    return fail(TOS_ERR_CUDA, "stream creation failed");
  }
  for (auto& ev : e->ev) cudaEventCreate(&ev);
  *out = e;
  return TOS_OK;
}

void tos_engine_destroy(tos_engine* e) {
  if (!e) return;
  {
    DeviceGuard g(e->device);
    cudaStreamSynchronize(e->stream);
    for (auto& ev : e->ev) cudaEventDestroy(ev);
    cudaStreamDestroy(e->stream);
  }
  delete e;
}

tos_status tos_catalog_create(tos_engine* e, const tos_sightline* los, size_t n_los,
                              const tos_pixel* pixels, size_t n_pixels, int order,
                              tos_catalog** out) {
  return tos::catalog_create_impl(e, los, n_los, pixels, n_pixels, order, 0.0, nullptr, 0, out);
}

tos_status tos_catalog_create_dc(tos_engine* e, const tos_sightline* los, size_t n_los,
                                 const tos_pixel* pixels, size_t n_pixels, int order, double omega_matter,
                                 tos_catalog** out) {
  if (!(omega_matter > 0 && omega_matter <= 1))
    return fail(TOS_ERR_INVALID_ARG, "omega_matter must be in (0, 1]");
  return tos::catalog_create_impl(e, los, n_los, pixels, n_pixels, order, omega_matter, nullptr, 0, out);
}

tos_status tos_catalog_create_plates(tos_engine* e, const tos_sightline* los, size_t n_los,
                                     const tos_pixel* pixels, size_t n_pixels, const tos_plate* platelist,
                                     size_t n_plates, double omega_matter, tos_catalog** out) {
  if (!(omega_matter == 0 || (omega_matter > 0 && omega_matter <= 1)))
    return fail(TOS_ERR_INVALID_ARG, "omega_matter must be 0 (keep the pixels' distances) or in (0, 1]");
  if (n_plates > 0 && !platelist) return fail(TOS_ERR_INVALID_ARG, "platelist is null");
  static const tos_plate kNone{};
  return tos::catalog_create_impl(e, los, n_los, pixels, n_pixels, 0, omega_matter,
                                  n_plates ? platelist : &kNone, n_plates, out);
}

}  // extern "C"

// Catalogue creation; omega_matter > 0: each pixel's distance is computed on
// the device from its loglam (the pixels' own distances are ignored);
// platelist != null: the cells are the sightlines' plates.
tos_status tos::catalog_create_impl(tos_engine* e, const tos_sightline* los, size_t n_los,
                                    const tos_pixel* pixels, size_t n_pixels, int order, double omega_matter,
                                    const tos_plate* platelist, size_t n_plates, tos_catalog** out) {
  if (!e || !out) return fail(TOS_ERR_INVALID_ARG, "engine/out is null");
  *out = nullptr;
  if (n_los == 0 || !los) return fail(TOS_ERR_INVALID_ARG, "no sightlines");
  if (n_los >= 0xFFFFFFF0ull) return fail(TOS_ERR_UNSUPPORTED, "too many sightlines");
  const bool plates = platelist != nullptr;
  if (!plates && (order < 0 || order > 13)) return fail(TOS_ERR_INVALID_ARG, "healpix order must be in [0, 13]");
  if (n_pixels > 0 && !pixels) return fail(TOS_ERR_INVALID_ARG, "pixels is null");
  std::lock_guard<std::mutex> lock(e->mu);
  DeviceGuard g(e->device);
  std::unique_ptr<tos_catalog> cat(new tos_catalog());
  cat->eng = e;
  cat->device = e->device;
  cat->n_los = n_los;
  cat->plates = plates;
  cat->order = plates ? -1 : order;
  cat->nside = plates ? 0 : (int64_t)1 << order;
  // a HEALPix cell's solid angle, or a plate's (radius 1.5 degrees)
  {
    const double pi = 3.14159265358979323846, rp = 1.5 * pi / 180.0;
    cat->cell_sr = plates ? pi * rp * rp : 4.0 * pi / (12.0 * (double)cat->nside * (double)cat->nside);
  }
  // --- host index: pixel ranges, trig, cells
  cat->npix.resize(n_los);
  cat->off.resize(n_los);
  bool contiguous = true;
  uint64_t total = 0;
  for (size_t s = 0; s < n_los; ++s) {
    const tos_sightline& l = los[s];
    if (l.pixel_offset > n_pixels || (uint64_t)l.num_pixels > n_pixels - l.pixel_offset)
      return fail(TOS_ERR_INVALID_ARG, "sightline " + std::to_string(s) + " pixel range out of bounds");
    if (!std::isfinite(l.ra) || !std::isfinite(l.dec))
      return fail(TOS_ERR_INVALID_ARG, "sightline " + std::to_string(s) + " has non-finite position");
    if (plates && l.plate < 0)
      return fail(TOS_ERR_INVALID_ARG, "sightline " + std::to_string(s) + " has a negative plate id");
    cat->npix[s] = l.num_pixels;
    cat->off[s] = total;
    if (l.pixel_offset != total) contiguous = false;
    total += l.num_pixels;
    cat->max_np = std::max(cat->max_np, l.num_pixels);
  }
  cat->n_pix = total;
  std::vector<double4> trig(n_los);
  cat->cell_of.resize(n_los);
  for (size_t s = 0; s < n_los; ++s) {
    // SkyObject's cached sines and cosines (types.h:20-26)
    trig[s] = make_double4(std::sin(los[s].dec), std::cos(los[s].dec), std::sin(los[s].ra),
                           std::cos(los[s].ra));
    // cells of different groups never meet: the group is the key's high word
    cat->cell_of[s] = ((int64_t)los[s].group << 32) |
                      (plates ? (int64_t)los[s].plate : healpix_radec2pix(cat->nside, los[s].ra, los[s].dec));
  }
  if (plates) {
    // PlateBins' platelist (PlateBins.h:38-45): a std::map from plate id to
    // the centre, ra/dec in degrees times deg2rad (constants.h:12-13)
    const double deg2rad = (std::atan(1.0) * 4) / 180.0;
    std::map<int32_t, std::pair<double, double>> list;
    for (size_t k = 0; k < n_plates; ++k) {
      if (!std::isfinite(platelist[k].ra_center) || !std::isfinite(platelist[k].dec_center))
        return fail(TOS_ERR_INVALID_ARG, "platelist row " + std::to_string(k) + " has a non-finite centre");
      list[platelist[k].plate] = {platelist[k].ra_center * deg2rad, platelist[k].dec_center * deg2rad};
    }
    for (const auto& p : list) {
      cat->plate_ids.push_back(p.first);
      // SkyObject's cached sines and cosines (types.h:20-26)
      cat->plate_trig.push_back(make_double4(std::sin(p.second.second), std::cos(p.second.second),
                                             std::sin(p.second.first), std::cos(p.second.first)));
    }
  }
  cat->cells = cat->cell_of;
  std::sort(cat->cells.begin(), cat->cells.end());
  cat->cells.erase(std::unique(cat->cells.begin(), cat->cells.end()), cat->cells.end());
  const size_t nc = cat->cells.size();
  // groups: contiguous ranges of the sorted cells
  cat->groups.clear();
  cat->group_cell_start.clear();
  for (size_t c = 0; c < nc; ++c) {
    const uint32_t gid = (uint32_t)((uint64_t)cat->cells[c] >> 32);
    if (cat->groups.empty() || cat->groups.back() != gid) {
      cat->groups.push_back(gid);
      cat->group_cell_start.push_back((uint32_t)c);
    }
  }
  cat->group_cell_start.push_back((uint32_t)nc);
  std::vector<uint2> grange(nc);
  for (size_t g = 0; g + 1 < cat->group_cell_start.size(); ++g)
    for (uint32_t c = cat->group_cell_start[g]; c < cat->group_cell_start[g + 1]; ++c)
      grange[c] = make_uint2(cat->group_cell_start[g], cat->group_cell_start[g + 1]);
  cat->cell_idx.resize(n_los);
  std::vector<uint32_t> ccount(nc + 1, 0);
  for (size_t s = 0; s < n_los; ++s) {
    const uint32_t ci = (uint32_t)(std::lower_bound(cat->cells.begin(), cat->cells.end(),
                                                    cat->cell_of[s]) - cat->cells.begin());
    cat->cell_idx[s] = ci;
    ccount[ci + 1]++;
  }
  cat->cell_start.assign(nc + 1, 0);
  for (size_t c = 0; c < nc; ++c) cat->cell_start[c + 1] = cat->cell_start[c] + ccount[c + 1];
  cat->members.resize(n_los);
  {
    std::vector<uint32_t> fill(cat->cell_start.begin(), cat->cell_start.end() - 1);
    for (size_t s = 0; s < n_los; ++s) cat->members[fill[cat->cell_idx[s]]++] = (uint32_t)s;
  }
  // cell caps: unit centre and angular radius bounding every member
  std::vector<double4> caps(nc);
  for (size_t c = 0; c < nc; ++c) {
    double x = 0, y = 0, z = 0;
    for (uint32_t k = cat->cell_start[c]; k < cat->cell_start[c + 1]; ++k) {
      const double4 t = trig[cat->members[k]];
      x += t.y * t.w;
      y += t.y * t.z;
      z += t.x;
    }
    double nrm = std::sqrt(x * x + y * y + z * z);
    if (!(nrm > 0)) {
      const double4 t = trig[cat->members[cat->cell_start[c]]];
      x = t.y * t.w, y = t.y * t.z, z = t.x, nrm = 1.0;
    }
    x /= nrm, y /= nrm, z /= nrm;
    double rad = 0;
    for (uint32_t k = cat->cell_start[c]; k < cat->cell_start[c + 1]; ++k) {
      const double4 t = trig[cat->members[k]];
      double d = x * t.y * t.w + y * t.y * t.z + z * t.x;
      d = std::max(-1.0, std::min(1.0, d));
      rad = std::max(rad, std::acos(d));
    }
    caps[c] = make_double4(x, y, z, rad * (1 + 1e-9) + 1e-12);
  }
  cat->caps = caps;
  // --- device buffers
  TOS_TRY(cat->d_trig.alloc(n_los));
  TOS_TRY(cat->d_cap.alloc(nc));
  TOS_TRY(cat->d_cells.alloc(nc));
  if (plates && !cat->plate_ids.empty()) {
    TOS_TRY(cat->d_plate_ids.alloc(cat->plate_ids.size()));
    TOS_TRY(cat->d_plate_trig.alloc(cat->plate_ids.size()));
  }
  TOS_TRY(cat->d_cell_grange.alloc(nc));
  TOS_TRY(cat->d_group_cell_start.alloc(cat->group_cell_start.size()));
  TOS_TRY(cat->d_cell_idx.alloc(n_los));
  TOS_TRY(cat->d_cell_start.alloc(nc + 1));
  TOS_TRY(cat->d_members.alloc(n_los));
  TOS_TRY(cat->d_npix.alloc(n_los));
  TOS_TRY(cat->d_off.alloc(n_los));
  TOS_TRY(cat->d_raw.alloc(total));
  const size_t padded = total + (size_t)kPad * (n_los + 1);
  TOS_TRY(cat->d_dist_pad.alloc(padded));
  TOS_TRY(cat->d_loglam_pad.alloc(padded));
  TOS_TRY(cat->d_pack.alloc(padded));
  TOS_TRY(cat->d_wd.alloc(total));
  TOS_TRY(cat->d_w.alloc(total));
  TOS_TRY(cat->d_prefix.alloc(total + n_los));
  TOS_TRY(cat->d_range.alloc(n_los));
  TOS_TRY(cat->d_flags.alloc(3));
  TOS_TRY(cat->d_maxes.alloc(4));
  cudaStream_t st = e->stream;
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_trig.p, trig.data(), n_los * sizeof(double4),
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_cap.p, caps.data(), nc * sizeof(double4),
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_cells.p, cat->cells.data(), nc * sizeof(int64_t),
                               cudaMemcpyHostToDevice, st));
  if (!cat->plate_ids.empty()) {
    TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_plate_ids.p, cat->plate_ids.data(), cat->plate_ids.size() * 4,
                                 cudaMemcpyHostToDevice, st));
    TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_plate_trig.p, cat->plate_trig.data(),
                                 cat->plate_trig.size() * sizeof(double4), cudaMemcpyHostToDevice, st));
  }
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_cell_grange.p, grange.data(), nc * sizeof(uint2),
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_group_cell_start.p, cat->group_cell_start.data(),
                               cat->group_cell_start.size() * 4, cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_cell_idx.p, cat->cell_idx.data(), n_los * 4,
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_cell_start.p, cat->cell_start.data(), (nc + 1) * 4,
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_members.p, cat->members.data(), n_los * 4,
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_npix.p, cat->npix.data(), n_los * 4,
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_off.p, cat->off.data(), n_los * 8,
                               cudaMemcpyHostToDevice, st));
  if (total > 0) {
    if (contiguous) {
      TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_raw.p, pixels + los[0].pixel_offset,
                                   total * sizeof(tos_pixel), cudaMemcpyHostToDevice, st));
    } else {
      for (size_t s = 0; s < n_los; ++s)
        if (los[s].num_pixels)
          TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_raw.p + cat->off[s], pixels + los[s].pixel_offset,
                                       (size_t)los[s].num_pixels * sizeof(tos_pixel),
                                       cudaMemcpyHostToDevice, st));
    }
  }
  {
    const unsigned int init[3] = {0u, 0xFFFFFFFFu, 0x7F800000u /* +inf */};
    TOS_CUDA_TRY(cudaMemcpyAsync(cat->d_flags.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  }
  TOS_CUDA_TRY(cudaMemsetAsync(cat->d_maxes.p, 0, 4 * sizeof(double), st));
  if (omega_matter > 0) TOS_TRY(fill_distances_device(e, cat->d_raw.p, total, omega_matter, st));
  k_fill<<<grid_for(e, padded, 256), 256, 0, st>>>(cat->d_dist_pad.p, padded, kSentinel);
  k_fill<<<grid_for(e, padded, 256), 256, 0, st>>>(cat->d_loglam_pad.p, padded, kSentinel);
  k_fill_pack<<<grid_for(e, padded, 256), 256, 0, st>>>(cat->d_pack.p, padded);
  k_prep<<<grid_for(e, n_los * 32, 256), 256, 0, st>>>(
      cat->d_raw.p, cat->d_off.p, cat->d_npix.p, n_los, cat->d_dist_pad.p, cat->d_loglam_pad.p, cat->d_pack.p,
      cat->d_wd.p, cat->d_w.p, cat->d_prefix.p, cat->d_range.p, cat->d_flags.p,
      (unsigned long long*)cat->d_maxes.p);
  TOS_CUDA_TRY(cudaGetLastError());
  unsigned int fl[3] = {0u, 0u, 0u};
  double maxes[4];
  TOS_CUDA_TRY(cudaMemcpyAsync(fl, cat->d_flags.p, sizeof(fl), cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(maxes, cat->d_maxes.p, 32, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  const unsigned int flags = fl[0];
  cat->sorted = (flags & 1u) == 0;
  {
    const unsigned int key = fl[1];
    const unsigned int u = (key & 0x80000000u) ? (key & 0x7FFFFFFFu) : ~key;
    float f;
    std::memcpy(&f, &u, 4);
    cat->min_d = (total > 0) ? (double)f : 0.0;
    std::memcpy(&f, &fl[2], 4);
    cat->min_gap = (double)f;
  }
  cat->max_abs_wd = maxes[0];
  cat->max_w = maxes[1];
  cat->max_l = maxes[2];
  cat->max_d = maxes[3];
  if ((flags & 2u) || !std::isfinite(cat->max_abs_wd) || !std::isfinite(cat->max_w) ||
      !std::isfinite(cat->max_l) || !std::isfinite(cat->max_d))
    return fail(TOS_ERR_INVALID_ARG,
                "pixels must have finite value, weight, loglam and distance (filter them as "
                "HDF5Delta::loadForests does)");
  // the raw copy is no longer needed
  cat->d_raw.release();
  *out = cat.release();
  return TOS_OK;
}

namespace tos {
namespace {
// Compact copy of the padded per-pixel distances (pixel p of sightline s at
// off[s] + p).
__global__ void k_gather_distances(const float* dist_pad, const uint64_t* off, const uint32_t* npix, size_t n_los,
                                   float* out) {
  const int lane = threadIdx.x & 31;
  for (size_t s = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) / 32; s < n_los;
       s += (size_t)gridDim.x * blockDim.x / 32) {
    const float* src = dist_pad + off[s] + (uint64_t)kPad * (s + 1);
    for (uint32_t p = lane; p < npix[s]; p += 32) out[off[s] + p] = src[p];
  }
}
}  // namespace
}  // namespace tos

extern "C" {

tos_status tos_catalog_distances(const tos_catalog* c, float* out, size_t cap) {
  if (!c || (!out && c->n_pix)) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cap < c->n_pix) return fail(TOS_ERR_INVALID_ARG, "capacity too small");
  if (c->n_pix == 0) return TOS_OK;
  tos_engine* e = c->eng;
  std::lock_guard<std::mutex> lock(e->mu);
  DeviceGuard g(e->device);
  DevBuf<float> tmp;
  TOS_TRY(tmp.alloc(c->n_pix));
  k_gather_distances<<<grid_for(e, c->n_los * 32, 256), 256, 0, e->stream>>>(c->d_dist_pad.p, c->d_off.p,
                                                                           c->d_npix.p, c->n_los, tmp.p);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaMemcpyAsync(out, tmp.p, c->n_pix * sizeof(float), cudaMemcpyDeviceToHost, e->stream));
  TOS_CUDA_TRY(cudaStreamSynchronize(e->stream));
  return TOS_OK;
}

void tos_catalog_destroy(tos_catalog* c) {
  if (!c) return;
  DeviceGuard g(c->device);
  delete c;  // cudaFree synchronises with pending work on the device
}

tos_status tos_catalog_num_cells(const tos_catalog* c, size_t* n) {
  if (!c || !n) return fail(TOS_ERR_INVALID_ARG, "null argument");
  *n = c->cells.size();
  return TOS_OK;
}

tos_status tos_catalog_cells(const tos_catalog* c, int64_t* ids, size_t cap) {
  if (!c || !ids) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cap < c->cells.size()) return fail(TOS_ERR_INVALID_ARG, "capacity too small");
  std::copy(c->cells.begin(), c->cells.end(), ids);
  return TOS_OK;
}

tos_status tos_catalog_device_bytes(const tos_catalog* c, uint64_t* bytes) {
  if (!c || !bytes) return fail(TOS_ERR_INVALID_ARG, "null argument");
  *bytes = catalog_data_bytes(c) + c->run.bytes();
  return TOS_OK;
}

tos_status tos_catalog_num_groups(const tos_catalog* c, size_t* n) {
  if (!c || !n) return fail(TOS_ERR_INVALID_ARG, "null argument");
  *n = c->groups.size();
  return TOS_OK;
}

tos_status tos_catalog_groups(const tos_catalog* c, uint32_t* ids, size_t cap) {
  if (!c || !ids) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cap < c->groups.size()) return fail(TOS_ERR_INVALID_ARG, "capacity too small");
  std::copy(c->groups.begin(), c->groups.end(), ids);
  return TOS_OK;
}

tos_status tos_catalog_sightline_cells(const tos_catalog* c, int64_t* cells, size_t cap) {
  if (!c || !cells) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cap < c->cell_of.size()) return fail(TOS_ERR_INVALID_ARG, "capacity too small");
  std::copy(c->cell_of.begin(), c->cell_of.end(), cells);
  return TOS_OK;
}

tos_status tos_grid_max_angular_scale(const tos_grid* g, double scale, double* max_ang) {
  TOS_TRY(check_grid(g));
  if (!max_ang) return fail(TOS_ERR_INVALID_ARG, "max_ang is null");
  if (g->type != TOS_OBSERVING && !(scale > 0)) return fail(TOS_ERR_INVALID_ARG, "scale must be > 0");
  *max_ang = max_angular_scale(*g, scale);
  return TOS_OK;
}

size_t tos_grid_num_bins(const tos_grid* g) {
  if (!g || check_grid(g) != TOS_OK) return 0;
  return (size_t)g->axis[0].nbins * g->axis[1].nbins * g->axis[2].nbins;
}

void tos_xibin_finalize(tos_xibin* b, size_t n) {
  // XiBin::finalize (types.h:96-101)
  for (size_t k = 0; k < n; ++k) {
    tos_xibin& x = b[k];
    (x.wgt > 0) ? x.didj /= x.wgt : x.didj = 0;
    (x.wi > 0) ? x.di /= x.wi : x.di = 0;
    (x.wj > 0) ? x.dj /= x.wj : x.dj = 0;
    (x.num_pairs > 0) ? x.z /= (double)x.num_pairs : x.z = 0;
  }
}

}  // extern "C"

namespace tos {

uint64_t catalog_data_bytes(const tos_catalog* c) {
  uint64_t b = c->d_trig.bytes() + c->d_cap.bytes() + c->d_cells.bytes() + c->d_plate_ids.bytes() +
               c->d_plate_trig.bytes() + c->d_cell_grange.bytes() +
               c->d_group_cell_start.bytes() + c->d_cell_idx.bytes() + c->d_cell_start.bytes() +
               c->d_members.bytes() + c->d_npix.bytes() + c->d_off.bytes() + c->d_raw.bytes() +
               c->d_dist_pad.bytes() + c->d_loglam_pad.bytes() + c->d_pack.bytes() + c->d_wd.bytes() +
               c->d_w.bytes() +
               c->d_prefix.bytes() + c->d_range.bytes() + c->d_flags.bytes() + c->d_maxes.bytes();
  for (int w = 0; w < 2; ++w) b += c->d_grid[w].bytes() + c->d_gfirst[w].bytes();
  return b;
}

size_t Workspace::bytes() const {
  return d_nb_count.bytes() + d_nb_start.bytes() + d_nb.bytes() + d_plate_edge.bytes() + d_cnt.bytes() +
         d_cand.bytes() +
         d_item_off.bytes() + d_item_i.bytes() + d_item_j.bytes() + d_item_sep.bytes() +
         d_item_c.bytes() + d_cell_pairs.bytes() + d_acc.bytes() + d_out.bytes() +
         d_counters.bytes() + d_thr.bytes() + d_gq.bytes() + d_cub_tmp.bytes();
}

// Counter words of a run: kernel counters [0, 16), the theta-edge flags of
// observing grids from 16 (at most 1 + 4096), then one item counter per
// chunk of a shared-GPU sweep.
constexpr int kChunkCounters = 4128;
constexpr int kMaxChunks = 64;
constexpr uint64_t kChunkItemsMin = 131072;  // tens of ms per chunk: the launch tail stays small
constexpr size_t kCounterWords = kChunkCounters + kMaxChunks;

// Host callback after a shared-GPU sweep chunk: hands the SMs back.
static void CUDART_CB sweep_chunk_done(void* share) { static_cast<SweepShare*>(share)->release(); }

// Fixed-point scales for kernels whose FP64 register sums can hold a whole
// item's pairs of a bin (at most max_np^2 pairs): every field takes the wide
// 62-bit conversion (the run, grid and diagonal sweeps).
static void set_wide_scales(PairArgs& A, const tos_catalog* cat) {
  const double m = std::max<double>(1.0, cat->max_np);
  const double wdm = std::max(cat->max_abs_wd, 1e-300), wm = std::max(cat->max_w, 1e-300),
               lm = std::max(cat->max_l, 1e-300);
  const double bound[7] = {wdm * m * wdm, wdm * m, m * wdm, wm * m * wm, wm * m, m * wm, lm * m};
  for (int k = 0; k < 7; ++k) {
    int f = (int)std::floor(62.0 - std::log2(bound[k] * m));
    f = std::max(-60, std::min(f, 200));
    A.scale[k] = std::ldexp(1.0, f);
    A.scale_hi[k] = std::ldexp(1.0, f - 44);
  }
  A.wide_all = 1;
}

tos_status xi_run_impl(tos_engine* e, tos_catalog* cat, Workspace* ws, const tos_grid* grid,
                       double scale, uint32_t flags, const RowPlan* plan, tos_xibin* out_bins,
                       tos_xibin* out_cells, tos_xi_stats* stats, const SweepShare* share) {
  const auto t_start = std::chrono::steady_clock::now();
  if (!e || !cat || !ws || !out_bins) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cat->device != e->device) return fail(TOS_ERR_INVALID_ARG, "catalogue is on another device");
  TOS_TRY(check_grid(grid));
  if ((flags & TOS_XI_SUBSAMPLES) && !out_cells)
    return fail(TOS_ERR_INVALID_ARG, "TOS_XI_SUBSAMPLES needs out_cells");
  if ((flags & TOS_XI_PER_GROUP) && !out_cells)
    return fail(TOS_ERR_INVALID_ARG, "TOS_XI_PER_GROUP needs out_cells");
  if ((flags & TOS_XI_PER_GROUP) && (flags & TOS_XI_SUBSAMPLES))
    return fail(TOS_ERR_INVALID_ARG, "TOS_XI_PER_GROUP and TOS_XI_SUBSAMPLES are exclusive");
  if (grid->type != TOS_OBSERVING && !(scale > 0 && std::isfinite(scale)))
    return fail(TOS_ERR_INVALID_ARG, "scale must be a positive finite number");
  std::lock_guard<std::mutex> lock(e->mu);
  DeviceGuard dg(e->device);
  cudaStream_t st = e->stream;
  ws->last_valid = false;
  const tos_grid& G = *grid;
  const RefGrid rg = make_ref_grid(G);
  {
    // separations are at most twice the largest |coordinate|; a bin index
    // computed from one must stay below 2^31, where the reference's 32-bit
    // cast would wrap it back into the grid
    const double xr = (G.type == TOS_OBSERVING) ? 2.0 * cat->max_l : 2.0 * cat->max_d;
    const double span0 = (xr * (1.0 + 1e-6) + 1.0 + std::fabs(rg.min0)) * rg.inv0;
    const double span1 = (G.type == TOS_CARTESIAN)
                             ? (xr * (1.0 + 1e-6) + 1.0 + std::fabs(rg.min1)) * rg.inv1
                             : 0.0;
    if (!(span0 < 2147483648.0) || !(span1 < 2147483648.0))
      return fail(TOS_ERR_UNSUPPORTED,
                  "grid bins too fine for the catalogue's coordinates: a separation's bin index "
                  "would pass 2^31 and wrap the reference's 32-bit index");
  }
  const uint32_t nb = rg.ntotal;
  const uint32_t nc = (uint32_t)cat->cells.size();
  const double max_ang = max_angular_scale(G, scale);
  const double cos_max = std::cos(max_ang);  // XiEstimator.cc:25

  // --- cell neighbours
  TOS_CUDA_TRY(cudaEventRecord(e->ev[0], st));
  if (cat->plates) {
    // per sightline: the occupied plates of PlateBins' ring test
    const size_t nl = cat->n_los;
    const uint32_t np = (uint32_t)cat->plate_ids.size();
    const double ring = 1.5 * ((std::atan(1.0) * 4) / 180.0);  // 1.5*deg2rad, PlateBins.h:80
    TOS_TRY(ws->d_nb_count.alloc(nl));
    TOS_TRY(ws->d_nb_start.alloc(nl + 1));
    TOS_TRY(ws->d_plate_edge.alloc(1 + 2 * (size_t)kPlateEdgeCap));
    unsigned long long* edge = ws->d_plate_edge.p;
    TOS_CUDA_TRY(cudaMemsetAsync(edge, 0, sizeof(unsigned long long), st));
    TOS_CUDA_TRY(cudaMemsetAsync(ws->d_nb_count.p, 0, nl * 4, st));
    const int gp = grid_for(e, nl * 32, 256);
    if (np > 0) {
      k_plate_neighbours<<<gp, 256, 0, st>>>(0, cat->d_trig.p, cat->d_cell_idx.p, cat->d_cell_grange.p,
                                             cat->d_cells.p, nl, cat->d_plate_ids.p, cat->d_plate_trig.p, np,
                                             ring, max_ang, edge, nullptr, nullptr, nullptr);
      TOS_CUDA_TRY(cudaGetLastError());
      unsigned long long ne = 0;
      TOS_CUDA_TRY(cudaMemcpyAsync(&ne, edge, 8, cudaMemcpyDeviceToHost, st));
      TOS_CUDA_TRY(cudaStreamSynchronize(st));
      if (ne > kPlateEdgeCap)
        return fail(TOS_ERR_UNSUPPORTED, std::to_string(ne) + " sightline-plate angles lie within 1e-12 rad of "
                                         "the plate ring's edge (at most 65536 are settled on the host)");
      if (ne) {
        // settled with the host libm's acos, the function PlateBins calls
        std::vector<unsigned long long> keys(ne), cbits(ne), sk(ne), dec(ne);
        TOS_CUDA_TRY(cudaMemcpy(keys.data(), edge + 1, ne * 8, cudaMemcpyDeviceToHost));
        TOS_CUDA_TRY(cudaMemcpy(cbits.data(), edge + 1 + kPlateEdgeCap, ne * 8, cudaMemcpyDeviceToHost));
        std::vector<size_t> ord(ne);
        std::iota(ord.begin(), ord.end(), 0);
        std::sort(ord.begin(), ord.end(), [&](size_t a, size_t b) { return keys[a] < keys[b]; });
        for (size_t t = 0; t < ne; ++t) {
          double c;
          std::memcpy(&c, &cbits[ord[t]], 8);
          sk[t] = keys[ord[t]];
          dec[t] = (std::fabs(std::acos(c) - ring) < max_ang) ? 1ull : 0ull;
        }
        TOS_CUDA_TRY(cudaMemcpy(edge + 1, sk.data(), ne * 8, cudaMemcpyHostToDevice));
        TOS_CUDA_TRY(cudaMemcpy(edge + 1 + kPlateEdgeCap, dec.data(), ne * 8, cudaMemcpyHostToDevice));
      }
      k_plate_neighbours<<<gp, 256, 0, st>>>(1, cat->d_trig.p, cat->d_cell_idx.p, cat->d_cell_grange.p,
                                             cat->d_cells.p, nl, cat->d_plate_ids.p, cat->d_plate_trig.p, np,
                                             ring, max_ang, edge, ws->d_nb_count.p, nullptr, nullptr);
      TOS_CUDA_TRY(cudaGetLastError());
    }
    std::vector<uint32_t> nbc(nl), nbs(nl + 1, 0);
    TOS_CUDA_TRY(cudaMemcpyAsync(nbc.data(), ws->d_nb_count.p, nl * 4, cudaMemcpyDeviceToHost, st));
    TOS_CUDA_TRY(cudaStreamSynchronize(st));
    for (size_t i = 0; i < nl; ++i) nbs[i + 1] = nbs[i] + nbc[i];
    TOS_TRY(ws->d_nb.alloc(nbs[nl]));
    TOS_CUDA_TRY(cudaMemcpyAsync(ws->d_nb_start.p, nbs.data(), (nl + 1) * 4, cudaMemcpyHostToDevice, st));
    if (np > 0 && nbs[nl] > 0) {
      k_plate_neighbours<<<gp, 256, 0, st>>>(2, cat->d_trig.p, cat->d_cell_idx.p, cat->d_cell_grange.p,
                                             cat->d_cells.p, nl, cat->d_plate_ids.p, cat->d_plate_trig.p, np,
                                             ring, max_ang, edge, nullptr, ws->d_nb_start.p, ws->d_nb.p);
      TOS_CUDA_TRY(cudaGetLastError());
    }
  } else {
    TOS_TRY(ws->d_nb_count.alloc(nc));
    TOS_TRY(ws->d_nb_start.alloc(nc + 1));
    const int gb = grid_for(e, nc, 128);
    k_cell_neighbours<<<gb, 128, 0, st>>>(cat->d_cap.p, cat->d_cell_grange.p, nc, max_ang,
                                          nullptr, ws->d_nb_count.p, nullptr);
    TOS_CUDA_TRY(cudaGetLastError());
    std::vector<uint32_t> nbc(nc), nbs(nc + 1, 0);
    TOS_CUDA_TRY(cudaMemcpyAsync(nbc.data(), ws->d_nb_count.p, nc * 4, cudaMemcpyDeviceToHost, st));
    TOS_CUDA_TRY(cudaStreamSynchronize(st));
    for (uint32_t c = 0; c < nc; ++c) nbs[c + 1] = nbs[c] + nbc[c];
    TOS_TRY(ws->d_nb.alloc(nbs[nc]));
    TOS_CUDA_TRY(cudaMemcpyAsync(ws->d_nb_start.p, nbs.data(), (nc + 1) * 4,
                                 cudaMemcpyHostToDevice, st));
    k_cell_neighbours<<<gb, 128, 0, st>>>(cat->d_cap.p, cat->d_cell_grange.p, nc, max_ang,
                                          ws->d_nb_start.p, nullptr, ws->d_nb.p);
    TOS_CUDA_TRY(cudaGetLastError());
  }
  // --- expansion pass 1: counts
  const uint32_t nm = (uint32_t)cat->n_los;
  TOS_TRY(ws->d_cnt.alloc(nm));
  TOS_TRY(ws->d_cand.alloc(nm));
  TOS_TRY(ws->d_item_off.alloc(nm));
  TOS_TRY(ws->d_cell_pairs.alloc(nc));
  TOS_TRY(ws->d_counters.alloc(kCounterWords));
  TOS_CUDA_TRY(cudaMemsetAsync(ws->d_cell_pairs.p, 0, nc * 8, st));
  TOS_CUDA_TRY(cudaMemsetAsync(ws->d_counters.p, 0, kCounterWords * 8, st));
  // [0..3] kernel counters, [4] pair-kernel item counter, [5] candidates,
  // [6] window flushes, [7] run-kernel item counter, [8] run items, [9] grid
  // items, [10] grid-kernel item counter,
  // [16] theta indices on an edge, [17..] their item numbers (4096 at most)
  unsigned long long* ctr = ws->d_counters.p;
  const double theta_min = G.axis[1].min, theta_inv = 1.0 / axis_width(G.axis[1]);
  const int ge = grid_for(e, (size_t)nm * 32, 256);
  k_expand<<<ge, 256, 0, st>>>(cat->d_members.p, nm, cat->d_cell_idx.p, cat->d_cell_start.p,
                               ws->d_nb_start.p, ws->d_nb.p, cat->plates ? 1 : 0, cat->d_trig.p, cat->d_npix.p, cos_max,
                               ws->d_cnt.p, ws->d_cand.p, ws->d_cell_pairs.p, nullptr, nullptr,
                               nullptr, nullptr, nullptr, G.type, theta_min, theta_inv, ctr + 16);
  TOS_CUDA_TRY(cudaGetLastError());
  // exclusive scan of counts -> item offsets
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, ws->d_cnt.p, ws->d_item_off.p, nm, st);
  TOS_TRY(ws->d_cub_tmp.alloc(tmp_bytes + 16));
  TOS_CUDA_TRY(cub::DeviceScan::ExclusiveSum(ws->d_cub_tmp.p, tmp_bytes, ws->d_cnt.p,
                                             ws->d_item_off.p, nm, st));
  uint32_t last_off = 0, last_cnt = 0;
  TOS_CUDA_TRY(cudaMemcpyAsync(&last_off, ws->d_item_off.p + nm - 1, 4, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(&last_cnt, ws->d_cnt.p + nm - 1, 4, cudaMemcpyDeviceToHost, st));
  std::vector<unsigned long long> cell_pairs(nc);
  TOS_CUDA_TRY(cudaMemcpyAsync(cell_pairs.data(), ws->d_cell_pairs.p, nc * 8,
                               cudaMemcpyDeviceToHost, st));
  unsigned long long n_cand_total = 0;
  {
    // candidates: reduce on the device
    size_t tb = 0;
    cub::DeviceReduce::Sum(nullptr, tb, ws->d_cand.p, ctr + 5, nm, st);
    if (tb > ws->d_cub_tmp.n) {
      TOS_CUDA_TRY(cudaStreamSynchronize(st));
      TOS_TRY(ws->d_cub_tmp.alloc(tb + 16));
    }
    TOS_CUDA_TRY(cub::DeviceReduce::Sum(ws->d_cub_tmp.p, tb, ws->d_cand.p, ctr + 5, nm, st));
    TOS_CUDA_TRY(cudaMemcpyAsync(&n_cand_total, ctr + 5, 8, cudaMemcpyDeviceToHost, st));
  }
  std::vector<uint32_t> prim_items(nm);  // accepted pairs per primary sightline
  TOS_CUDA_TRY(cudaMemcpyAsync(prim_items.data(), ws->d_cnt.p, (size_t)nm * 4,
                               cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  const uint64_t n_items = (uint64_t)last_off + last_cnt;
  unsigned long long n_pixel_pairs = 0, max_cell_pairs = 0;
  for (auto v : cell_pairs) {
    n_pixel_pairs += v;
    max_cell_pairs = std::max(max_cell_pairs, v);
  }
  {
    // the carry-free accumulators take fewer than 2^32 adds per (row, bin):
    // a sightline pair makes at most kMaxAddsPerItemBin * max_np of them
    std::vector<uint64_t> cell_items(nc, 0);
    for (uint32_t s = 0; s < nm; ++s) cell_items[cat->cell_idx[s]] += prim_items[s];
    uint64_t max_row_items = 0;
    if (plan)
      max_row_items = plan->max_row_items(cell_items);
    else
      for (uint64_t v : cell_items) max_row_items = std::max(max_row_items, v);
    const double adds = (double)max_row_items * kMaxAddsPerItemBin * std::max<double>(1, cat->max_np);
    if (!(adds < 4294967296.0))
      return fail(TOS_ERR_UNSUPPORTED,
                  "up to " + std::to_string(max_row_items) +
                      " sightline pairs share one accumulator row, which could pass 2^32 adds "
                      "to one bin: use a finer HEALPix order");
  }
  // --- expansion pass 2: items
  TOS_TRY(ws->d_item_i.alloc(n_items));
  TOS_TRY(ws->d_item_j.alloc(n_items));
  TOS_TRY(ws->d_item_c.alloc(n_items));
  TOS_TRY(ws->d_item_sep.alloc(G.type == TOS_OBSERVING ? n_items : 1));
  k_expand<<<ge, 256, 0, st>>>(cat->d_members.p, nm, cat->d_cell_idx.p, cat->d_cell_start.p,
                               ws->d_nb_start.p, ws->d_nb.p, cat->plates ? 1 : 0, cat->d_trig.p, cat->d_npix.p, cos_max,
                               ws->d_cnt.p, ws->d_cand.p, ws->d_cell_pairs.p, ws->d_item_off.p,
                               ws->d_item_i.p, ws->d_item_j.p, ws->d_item_c.p,
                               ws->d_item_sep.p, G.type, theta_min, theta_inv, ctr + 16);
  TOS_CUDA_TRY(cudaGetLastError());
  if (G.type == TOS_OBSERVING) {
    // theta indices within 1e-9 of an edge: recompute with the host libm acos,
    // the function the reference calls (XiEstimator.cc:166).
    unsigned long long nflag = 0;
    TOS_CUDA_TRY(cudaMemcpyAsync(&nflag, ctr + 16, 8, cudaMemcpyDeviceToHost, st));
    TOS_CUDA_TRY(cudaStreamSynchronize(st));
    if (nflag > 4096) return fail(TOS_ERR_UNSUPPORTED, "too many theta indices on a bin edge");
    if (nflag) {
      std::vector<unsigned long long> at(nflag);
      TOS_CUDA_TRY(cudaMemcpy(at.data(), ctr + 17, nflag * 8, cudaMemcpyDeviceToHost));
      for (auto a : at) {
        double c;
        TOS_CUDA_TRY(cudaMemcpy(&c, ws->d_item_c.p + a, 8, cudaMemcpyDeviceToHost));
        const uint32_t sep = tos::ref_u32(tos::dmul(tos::dsub(std::acos(c), theta_min), theta_inv));
        TOS_CUDA_TRY(cudaMemcpy(ws->d_item_sep.p + a, &sep, 4, cudaMemcpyHostToDevice));
      }
    }
  }
  TOS_CUDA_TRY(cudaEventRecord(e->ev[1], st));

  // --- accumulation layout and fixed-point scales
  const size_t n_acc_rows = plan ? (size_t)plan->n_rows : (size_t)nc;
  const size_t acc_words = n_acc_rows * nb * kAccWords;
  TOS_TRY(ws->d_acc.alloc(acc_words));
  TOS_CUDA_TRY(cudaMemsetAsync(ws->d_acc.p, 0, acc_words * 8, st));
  PairArgs A{};
  A.off = cat->d_off.p;
  A.npix = cat->d_npix.p;
  A.dist_pad = cat->d_dist_pad.p;
  A.loglam_pad = cat->d_loglam_pad.p;
  A.pack = cat->d_pack.p;
  A.wd = cat->d_wd.p;
  A.w = cat->d_w.p;
  A.prefix = cat->d_prefix.p;
  A.range = cat->d_range.p;
  A.cell_idx = cat->d_cell_idx.p;
  if (plan) {
    A.row_key = plan->row_key;
    A.slot_start = plan->slot_start;
    A.slot_key = plan->slot_key;
    A.spill_row = plan->n_rows - 1;
  }
  A.item_i = ws->d_item_i.p;
  A.item_j = ws->d_item_j.p;
  A.item_c = ws->d_item_c.p;
  A.item_sep = ws->d_item_sep.p;
  A.n_items = n_items;
  A.next_item = ctr + 4;
  A.g = rg;
  A.acc = ws->d_acc.p;
  A.counters = ctr;
  A.force_exact = (flags & TOS_XI_EXACT) ? 1 : 0;
  // fixed point: 2^F per field.  A run contributes c with |c| <= bound
  // (a run has at most max_np pixels).  Signed sums (didj, di, dj) use
  // |round(c 2^F)| < 2^62 split into 22+22+18-bit words, positive sums
  // |round(c 2^F)| < 2^42 split into 22+20-bit words; a window slot takes at
  // most 1024 contributions, and the per-cell accumulators are 128-bit.
  {
    const double m = std::max<double>(1.0, cat->max_np);
    const double wdm = std::max(cat->max_abs_wd, 1e-300), wm = std::max(cat->max_w, 1e-300),
                 lm = std::max(cat->max_l, 1e-300);
    const double bound[7] = {wdm * m * wdm, wdm * m, m * wdm, wm * m * wm, wm * m, m * wm, lm * m};
    for (int k = 0; k < 7; ++k) {
      const double top = (k < kSigned) ? 62.0 : 42.0;
      int f = (int)std::floor(top - std::log2(bound[k]));
      f = std::max(-60, std::min(f, 200));
      A.scale[k] = std::ldexp(1.0, f);
      if (k < kSigned) A.scale_hi[k] = std::ldexp(1.0, f - 44);
    }
  }
  // FP32 fast-path constants
  const uint32_t n0 = rg.n0, n1 = (G.type == TOS_OBSERVING) ? 1u : rg.n1;
  A.inv0f = (float)rg.inv0;
  A.off0f = (float)(-rg.min0 * rg.inv0);
  if (G.type == TOS_CARTESIAN) {
    A.inv1f = 1.0f;
    A.off1f = (float)(-rg.min1 * rg.inv1);
    A.inv1sqf = (float)(rg.inv1 * rg.inv1);
  } else {
    A.inv1f = (float)rg.inv1;
    A.off1f = (float)(-rg.min1 * rg.inv1);
    A.inv1sqf = 1.0f;
  }
  A.n0f = (float)n0;
  A.n1f = (float)n1;
  A.n0p1f = (float)n0 + 1.0f;
  A.n1p1f = (float)n1 + 1.0f;
  A.k0 = std::max(0, std::min(13, 21 - bitlen(n0 + 2)));
  A.k1 = std::max(0, std::min(13, 21 - bitlen(n1 + 2)));
  A.mag0 = std::ldexp(1.5f, 23 - A.k0);
  A.mag1 = std::ldexp(1.5f, 23 - A.k1);
  std::memcpy(&A.bits0, &A.mag0, 4);
  std::memcpy(&A.bits1, &A.mag1, 4);
  A.r2_small = 1e-4f;
  const bool exact0 = (G.type != TOS_POLAR) && rg.min0 == 0.0 && is_pow2(rg.inv0);
  const bool minpos = (rg.min0 > 0.0) || (G.type != TOS_OBSERVING && rg.min1 > 0.0) ||
                      (rg.min0 < 0.0) || (G.type != TOS_OBSERVING && rg.min1 < 0.0);
  // column pruning window
  A.prune = cat->sorted ? 1 : 0;
  {
    float lim;
    if (G.type == TOS_POLAR) {
      // r >= R rejected; r_sq >= s^2 - |float rounding of d1^2| - tiny
      double R = rg.min0 + (double)n0 / rg.inv0;
      R = std::max(R, 0.0) * (1.0 + 1e-6) + 1e-6;
      const double dm = cat->max_d;
      A.polar_r2 = R * R;
      A.polar_e2 = std::ldexp(dm * dm, -23) + 1e-3;
      lim = (float)(std::sqrt(R * R + std::ldexp(dm * dm, -23) + 1e-3) * (1.0 + 1e-6) + 1e-3);
    } else {
      lim = first_axis_threshold(rg.min0, rg.inv0, n0, (int)n0);
    }
    A.win_lim = lim;
    if (!std::isfinite(lim)) A.prune = 0;
  }
  // window layout: per warp, slots of kWinWords u32 words within ~200 KB per CTA
  {
    const int budget = (int)(200 * 1024 / ((size_t)kWinWords * 4 * kPairWarps));
    if (G.type == TOS_CARTESIAN) {
      A.win_w1 = (int)std::min<uint32_t>(4u, rg.n1);
      if ((int)n0 * A.win_w1 > budget) A.win_w1 = std::max(0, budget / (int)n0);
      A.win_slots = std::max(1, (int)n0 * A.win_w1);
    } else if (G.type == TOS_POLAR) {
      A.win_w1 = 0;
      A.win_slots = (int)std::min<uint32_t>(n0 * rg.n1, (uint32_t)budget);
    } else {
      A.win_w1 = 0;
      A.win_slots = (int)std::min<uint32_t>(n0, (uint32_t)budget);
    }
  }
  // --- run sweep (Cartesian and observing coordinates, sorted sightlines).
  // The first-axis bin of |fl32(x1 - x2)| is decided by the exact float
  // thresholds T[k]; for Cartesian coordinates r_perp must also be a
  // non-decreasing function of the column distance along every row, as the
  // reference computes it (XiEstimator.cc:244-248):
  //   Y(d2) = fl(fl(r1_sq + fl(fl(d2 - tc) * d2)) - r_para^2)
  //         = S * d2 - err + N,  S = 2 d1 - tc >= d1 (a - 2^-52), a = 2(1 - c),
  // where err = d1^2 - fl32(d1^2) (|err| <= 2^-24 D^2) and the FP64 rounding
  // |N| <= 11 * 2^-53 D^2 < 2^-49 D^2 (D the largest distance), provided
  // fl32(d1 - d2) is exact (Sterbenz: |d1 - d2| < T[n0] <= d_min).  Then
  //   (1) two columns at least `gap` apart differ in Y by S * gap - 2 |N| > 0
  //       when a > 2^-52 + 2^-48 D^2 / (d_min * gap)   (per item: run_amin);
  //   (2) Y >= -E with E = (2^-24 + 2^-49) D^2, and every |Y| <= E falls into
  //       the r_perp code of 0 when the grid puts 0 and E in the same code,
  // so the code of |Y| is non-decreasing along the row.
  bool use_runs = false;
  // (per-lane pair counts are 32-bit: at most max_np^2 < 2^32 pairs per item)
  if (G.type != TOS_POLAR && cat->sorted && !A.force_exact && n_items > 0 && cat->max_np < 65536) {
    std::vector<float> thr(n0 + 1);
    for (uint32_t k = 0; k <= n0; ++k)
      thr[k] = first_axis_threshold(rg.min0, rg.inv0, n0, (int)k);
    use_runs = true;
    A.run_amin = -1.0;
    if (G.type == TOS_CARTESIAN) {
      const double D = cat->max_d, dmin = cat->min_d, gap = cat->min_gap;
      auto perp_code = [&](double x) {
        const double t = tos::dmul(tos::dsub(std::sqrt(x), rg.min1), rg.inv1);
        if (!(t > -1.0)) return -1;
        return t >= (double)rg.n1 ? (int)rg.n1 : (int)ref_u32(t);
      };
      const double E = (std::ldexp(1.0, -24) + std::ldexp(1.0, -49)) * D * D * (1.0 + 1e-6);
      if (!(dmin > 0) || !std::isfinite(thr[n0]) || !((double)thr[n0] * (1.0 + 1e-6) <= dmin) ||
          !(D * rg.inv1 < 1e6) ||
          perp_code(0.0) != perp_code(E) || !(gap > 0)) {
        use_runs = false;
      } else {
        A.run_amin = std::isfinite(gap)
                         ? (std::ldexp(1.0, -52) + std::ldexp(D * D, -48) / (dmin * gap)) * (1.0 + 1e-3)
                         : std::ldexp(1.0, -51);
      }
    }
    if (use_runs) {
      TOS_TRY(ws->d_thr.alloc(n0 + 1));
      TOS_CUDA_TRY(cudaMemcpyAsync(ws->d_thr.p, thr.data(), (n0 + 1) * sizeof(float),
                                   cudaMemcpyHostToDevice, st));
      A.thr = ws->d_thr.p;
      set_wide_scales(A, cat);
      A.run_split = 1;
    }
  }
  // --- grid sweep: catalogues whose first-axis values lie on a small common grid
  bool use_grid = false;
  if (use_runs) {
    const int w = (G.type == TOS_OBSERVING) ? 1 : 0;
    TOS_TRY(ensure_grid(e, cat, w, st));
    const int ng = cat->grid_n[w];
    if (ng > 0 && cat->grid_los[w] > 0) {
      const size_t nq = (size_t)2 * ng * (n0 + 1);
      TOS_TRY(ws->d_gq.alloc(nq));
      k_grid_table<<<grid_for(e, nq, 256), 256, 0, st>>>(cat->d_grid[w].p, ng, ws->d_thr.p,
                                                         (int)n0 + 1, ws->d_gq.p);
      TOS_CUDA_TRY(cudaGetLastError());
      A.gq = ws->d_gq.p;
      A.gfirst = cat->d_gfirst[w].p;
      A.ng = ng;
      A.grid_split = 1;
      use_grid = true;
    }
  }
  // --- diagonal sweep (Polar, sorted sightlines): every item whose z index is
  // constant.  Its lanes add one run of pairs at a time, so the adds to one
  // (row, bin) are at most the row's pixel pairs, which must stay below the
  // 2^32 adds the carry-free sums take.
  bool use_diag = false;
  if (G.type == TOS_POLAR && cat->sorted && !A.force_exact && n_items > 0) {
    const uint64_t max_row_pairs =
        plan ? plan->max_row_items(std::vector<uint64_t>(cell_pairs.begin(), cell_pairs.end())) : max_cell_pairs;
    if (max_row_pairs < (1ull << 32)) {
      set_wide_scales(A, cat);
      A.diag_split = 1;
      use_diag = true;
    }
  }
  // --- launch shape of the dominant kernel: the tuned CTAs per SM for this
  // coordinate type and bin count (0: as many as fit).  With TOS_XI_TUNE,
  // first time every count from 1 to the occupancy limit on the first
  // kTuneItems sightline pairs (after a warm-up launch), keep the fastest,
  // and clear what the trials added.  The sums do not depend on the shape: a
  // warp sweeps an item on its own and every add is an integer add.
  int ctas_per_sm = 0;
  const std::pair<int, int> tune_key(G.type, (int)nb);
  {
    std::lock_guard<std::mutex> lk(e->tune_mu);
    auto it = e->xi_tuned.find(tune_key);
    if (it != e->xi_tuned.end()) ctas_per_sm = it->second;
  }
  if ((flags & TOS_XI_TUNE) && (use_grid || use_diag) && n_items > 0) {
    constexpr uint64_t kTuneItems = 65536;
    auto trial = [&](int per_sm, int* max_out) -> cudaError_t {
      PairArgs R = A;
      R.n_items = std::min<uint64_t>(n_items, kTuneItems);
      R.next_item = ctr + (use_diag ? 11 : 10);
      return use_diag ? launch_diag_kernel(R, minpos, e->num_sms, per_sm, st, max_out)
                      : launch_grid_kernel(R, G.type, minpos, e->num_sms, per_sm, st, max_out);
    };
    int max_per_sm = 1;
    const cudaError_t qe = trial(0, &max_per_sm);
    if (qe != cudaSuccess) return fail(TOS_ERR_CUDA, std::string("tuning: ") + cudaGetErrorString(qe));
    float best = 0.f;
    int pick = max_per_sm;
    for (int p = 0; p <= max_per_sm; ++p) {  // p = 0: warm-up at the occupancy limit
      TOS_CUDA_TRY(cudaMemsetAsync(ctr + (use_diag ? 11 : 10), 0, 8, st));
      TOS_CUDA_TRY(cudaEventRecord(e->ev[4], st));
      const cudaError_t te = trial(p == 0 ? max_per_sm : p, nullptr);
      if (te != cudaSuccess) return fail(TOS_ERR_CUDA, std::string("tuning: ") + cudaGetErrorString(te));
      TOS_CUDA_TRY(cudaEventRecord(e->ev[5], st));
      TOS_CUDA_TRY(cudaEventSynchronize(e->ev[5]));
      float ms = 0.f;
      TOS_CUDA_TRY(cudaEventElapsedTime(&ms, e->ev[4], e->ev[5]));
      if (p > 0 && (best == 0.f || ms < best)) {
        best = ms;
        pick = p;
      }
    }
    ctas_per_sm = pick;
    {
      std::lock_guard<std::mutex> lk(e->tune_mu);
      e->xi_tuned[tune_key] = pick;
    }
    TOS_CUDA_TRY(cudaMemsetAsync(ws->d_acc.p, 0, acc_words * 8, st));
    TOS_CUDA_TRY(cudaMemsetAsync(ctr, 0, 4 * 8, st));          // evaluated, rechecks, overflow, direct
    TOS_CUDA_TRY(cudaMemsetAsync(ctr + 6, 0, 7 * 8, st));      // flushes, item counters, taken
  }
  // Dominant kernel (grid or diagonal sweep): one persistent launch, or for
  // a shared GPU (SweepShare) a chain of chunk launches, each with its own
  // item counter (ctr[kChunkCounters + k], after the theta-edge flags of
  // observing grids at ctr[16 ..]) and its CTA count asked just before launch.
  auto sweep = [&](bool diag, unsigned long long* counter) -> tos_status {
    auto launch = [&](const PairArgs& R, int per_sm) -> cudaError_t {
      return diag ? launch_diag_kernel(R, minpos, e->num_sms, per_sm, st)
                  : launch_grid_kernel(R, G.type, minpos, e->num_sms, per_sm, st);
    };
    if (!share) {
      PairArgs R = A;
      R.next_item = counter;
      const cudaError_t ke = launch(R, ctas_per_sm);
      if (ke != cudaSuccess)
        return fail(TOS_ERR_CUDA, std::string(diag ? "diagonal" : "grid") + " kernel: " + cudaGetErrorString(ke));
      return TOS_OK;
    }
    const uint64_t chunks = std::max<uint64_t>(
        1, std::min<uint64_t>((uint64_t)std::min(std::max(1, share->chunks), kMaxChunks), n_items / kChunkItemsMin));
    const uint64_t per = (n_items + chunks - 1) / chunks;
    for (uint64_t c = 0; c < chunks; ++c) {
      const uint64_t a = c * per, b = std::min<uint64_t>(n_items, a + per);
      if (a >= b) break;
      PairArgs R = A;
      R.item_i = A.item_i + a;
      R.item_j = A.item_j + a;
      R.item_c = A.item_c + a;
      R.item_sep = (G.type == TOS_OBSERVING) ? A.item_sep + a : A.item_sep;
      R.n_items = b - a;
      R.next_item = ctr + kChunkCounters + c;
      const uint64_t remaining = (uint64_t)((double)n_pixel_pairs * (double)(n_items - a) / (double)n_items);
      const int per_sm = share->acquire(remaining);
      const cudaError_t ke = launch(R, per_sm);
      if (ke != cudaSuccess) {
        share->release();
        return fail(TOS_ERR_CUDA, std::string(diag ? "diagonal" : "grid") + " kernel: " + cudaGetErrorString(ke));
      }
      const cudaError_t he = cudaLaunchHostFunc(st, sweep_chunk_done, const_cast<SweepShare*>(share));
      if (he != cudaSuccess) {
        cudaStreamSynchronize(st);
        share->release();
        return fail(TOS_ERR_CUDA, std::string("chunk callback: ") + cudaGetErrorString(he));
      }
    }
    return TOS_OK;
  };
  if (n_items > 0) {
    TOS_CUDA_TRY(cudaEventRecord(e->ev[2], st));
    if (use_diag) TOS_TRY(sweep(true, ctr + 11));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[7], st));
    if (use_grid) TOS_TRY(sweep(false, ctr + 10));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[6], st));
    if (use_runs) {
      PairArgs R = A;
      R.next_item = ctr + 7;
      const cudaError_t re = launch_run_kernel(R, G.type, minpos, e->num_sms, st);
      if (re != cudaSuccess)
        return fail(TOS_ERR_CUDA, std::string("run kernel: ") + cudaGetErrorString(re));
    }
    TOS_CUDA_TRY(cudaEventRecord(e->ev[5], st));
    const cudaError_t le =
        launch_pair_kernel(A, G.type, exact0, minpos, e->num_sms, st);
    if (le != cudaSuccess) return fail(TOS_ERR_CUDA, std::string("pair kernel: ") + cudaGetErrorString(le));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[3], st));
  } else {
    TOS_CUDA_TRY(cudaEventRecord(e->ev[2], st));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[7], st));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[6], st));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[5], st));
    TOS_CUDA_TRY(cudaEventRecord(e->ev[3], st));
  }
  // --- combine cells
  const bool want_cells = (flags & TOS_XI_SUBSAMPLES) != 0;
  const bool per_group = (flags & TOS_XI_PER_GROUP) != 0;
  const uint32_t ngr = (uint32_t)cat->groups.size();
  const size_t n_rows = want_cells ? (size_t)nc : per_group ? (size_t)ngr : 0;
  TOS_TRY(ws->d_out.alloc((size_t)nb * (n_rows + 1)));
  double4 ia, ib;
  ia.x = 1.0 / A.scale[0], ia.y = 1.0 / A.scale[1], ia.z = 1.0 / A.scale[2], ia.w = 1.0 / A.scale[3];
  ib.x = 1.0 / A.scale[4], ib.y = 1.0 / A.scale[5], ib.z = 1.0 / A.scale[6], ib.w = 0;
  if (plan) {
    double inv[7];
    for (int k = 0; k < 7; ++k) inv[k] = 1.0 / A.scale[k];
    TOS_TRY(plan->combine(st, nb, inv, ws->d_acc.p, ws->d_out.p));
  } else if (per_group) {
    k_combine_groups<<<grid_for(e, (size_t)ngr * nb, 128), 128, 0, st>>>(
        ws->d_acc.p, cat->d_group_cell_start.p, ngr, nb, ia, ib, ws->d_out.p + nb);
    TOS_CUDA_TRY(cudaGetLastError());
    launch_sum_rows(ws->d_out.p + nb, ngr, nb, ws->d_out.p, grid_for(e, nb, 128), st);
  } else {
    k_combine<<<grid_for(e, nb, 128), 128, 0, st>>>(ws->d_acc.p, nc, nb, ia, ib, ws->d_out.p,
                                                     want_cells ? ws->d_out.p + nb : nullptr);
  }
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaMemcpyAsync(out_bins, ws->d_out.p, (size_t)nb * sizeof(tos_xibin),
                               cudaMemcpyDeviceToHost, st));
  if (n_rows)
    TOS_CUDA_TRY(cudaMemcpyAsync(out_cells, ws->d_out.p + nb, n_rows * nb * sizeof(tos_xibin),
                                 cudaMemcpyDeviceToHost, st));
  unsigned long long hc[13];
  TOS_CUDA_TRY(cudaMemcpyAsync(hc, ctr, sizeof(hc), cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaEventRecord(e->ev[4], st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  ws->last_valid = (plan == nullptr);  // slot rows are not per-cell sums
  ws->last_nb = nb;
  for (int k = 0; k < 7; ++k) ws->last_inv_scale[k] = 1.0 / A.scale[k];
  if (stats) {
    std::memset(stats, 0, sizeof(*stats));
    stats->num_sightlines = cat->n_los;
    stats->num_sightline_pairs = n_cand_total;
    stats->num_sightline_pairs_used = n_items;
    stats->num_pixels = cat->n_pix;
    stats->num_pixel_pairs = n_pixel_pairs;
    unsigned long long used = 0;
    for (uint32_t b = 0; b < nb; ++b) used += (unsigned long long)out_bins[b].num_pairs;
    stats->num_pixel_pairs_used = used + hc[2];
    stats->num_pixel_pairs_evaluated = hc[0];
    stats->num_edge_rechecks = hc[1];
    stats->num_index_overflow = hc[2];
    stats->num_direct_runs = hc[3];
    stats->num_window_flushes = hc[6];
    stats->num_cells = nc;
    stats->max_ang = max_ang;
    stats->cos_max_ang = cos_max;
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[0], e->ev[1]);
    stats->ms_expand = ms;
    cudaEventElapsedTime(&ms, e->ev[2], e->ev[3]);
    stats->ms_pairs = ms;
    cudaEventElapsedTime(&ms, e->ev[0], e->ev[4]);
    stats->ms_device = ms;
    cudaEventElapsedTime(&ms, e->ev[7], e->ev[5]);
    stats->ms_runs = ms;
    cudaEventElapsedTime(&ms, e->ev[7], e->ev[6]);
    stats->ms_grid = ms;
    stats->num_run_items = hc[8] + hc[9];
    stats->num_grid_items = hc[9];
    cudaEventElapsedTime(&ms, e->ev[2], e->ev[7]);
    stats->ms_diag = ms;
    stats->num_diag_items = hc[12];
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
  }
  return TOS_OK;
}

}  // namespace tos

extern "C" {

tos_status tos_xi_run(tos_engine* e, tos_catalog* cat, const tos_grid* grid, double scale,
                      uint32_t flags, tos_xibin* out_bins, tos_xibin* out_cells,
                      tos_xi_stats* stats) {
  if (!cat) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> lock(cat->run_mu);
  return xi_run_impl(e, cat, &cat->run, grid, scale, flags, nullptr, out_bins, out_cells, stats);
}

}  // extern "C"
