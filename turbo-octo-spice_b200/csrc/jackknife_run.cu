// jackknife_run.cu — the exact delete-one-region jackknife of the pair count
// in one pass over the pairs: the jackknife subsamples of a batched run.
//
// A region is a HEALPix pixel of a coarser order than the catalogue's cells,
// taken within one sightline group; a sightline belongs to the region that
// holds its cell (the orders nest, so the region holds the whole cell).
// Instead of the primary's cell, every pair's sums go to the slot of the
// unordered pair {a, b} of its two sightlines' regions.  Every pair that
// touches region k sits in a slot that names k and no other pair does, so
//     drop_k = total of k's group - sum over b of slot {k, b}
// is the count of the catalogue without region k's sightlines, computed
// exactly in the 128-bit fixed point of the slots.  The reference forms a
// subsample by re-running XiEstimator on the reduced catalogue; here one pass
// serves every subsample.
//
// Slots exist only for region pairs that can hold a pair within the grid's
// maximum angle (the cap test of the cell-neighbour search); a pair without
// a slot would land in a spill row, which the host checks is empty.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "fixed128.cuh"
#include "healpix.h"
#include "xi_kernels.cuh"

namespace tos {
namespace {

struct Inv7 {
  double v[7];
};

__device__ __forceinline__ tos_xibin to_bin(const __int128* s, long long n, const Inv7& inv) {
  tos_xibin x{};
  if (n != 0) {  // a bin without pairs has zero sums (as the per-cell merge)
    x.didj = i128_double(s[0]) * inv.v[0];
    x.di = i128_double(s[1]) * inv.v[1];
    x.dj = i128_double(s[2]) * inv.v[2];
    x.wgt = i128_double(s[3]) * inv.v[3];
    x.wi = i128_double(s[4]) * inv.v[4];
    x.wj = i128_double(s[5]) * inv.v[5];
    x.z = i128_double(s[6]) * inv.v[6];
  }
  x.num_pairs = n;
  return x;
}

// Per (group g, bin b): the 128-bit sums of the group's slots
// [gslot[g], gslot[g+1]) that hold pairs in b, kept in the accumulator
// layout, and converted to a XiBin.
__global__ void k_group_totals(const unsigned long long* acc, uint32_t nb, const uint32_t* gslot,
                               uint32_t ngr, Inv7 inv, unsigned long long* gtot, tos_xibin* gout) {
  const size_t n = (size_t)ngr * nb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const uint32_t g = (uint32_t)(t / nb), b = (uint32_t)(t % nb);
    __int128 s[7] = {0, 0, 0, 0, 0, 0, 0};
    long long cnt = 0;
    for (uint32_t q = gslot[g]; q < gslot[g + 1]; ++q) {
      const unsigned long long* base = acc + ((size_t)q * nb + b) * kAccWords;
      const long long c = (long long)base[14];
      if (c == 0) continue;
#pragma unroll
      for (int f = 0; f < 7; ++f) s[f] += acc128(base, f);
      cnt += c;
    }
    unsigned long long* o = gtot + t * kAccWords;
#pragma unroll
    for (int f = 0; f < 7; ++f) store128(o, f, s[f]);
    o[14] = (unsigned long long)cnt;
    o[15] = 0;
    gout[t] = to_bin(s, cnt, inv);
  }
}

// Per (region k, bin b): its group's total minus every slot that names k.
__global__ void k_drop(const unsigned long long* acc, const unsigned long long* gtot, uint32_t nb,
                       const uint32_t* kslot_start, const uint32_t* kslot, const uint32_t* kgroup,
                       uint32_t nk, Inv7 inv, tos_xibin* out) {
  const size_t n = (size_t)nk * nb;
  for (size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x; t < n;
       t += (size_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)(t / nb), b = (uint32_t)(t % nb);
    const unsigned long long* tot = gtot + ((size_t)kgroup[k] * nb + b) * kAccWords;
    __int128 s[7];
#pragma unroll
    for (int f = 0; f < 7; ++f) s[f] = acc128(tot, f);
    long long cnt = (long long)tot[14];
    for (uint32_t m = kslot_start[k]; m < kslot_start[k + 1]; ++m) {
      const unsigned long long* base = acc + ((size_t)kslot[m] * nb + b) * kAccWords;
      const long long c = (long long)base[14];
      if (c == 0) continue;
#pragma unroll
      for (int f = 0; f < 7; ++f) s[f] -= acc128(base, f);
      cnt -= c;
    }
    out[t] = to_bin(s, cnt, inv);
  }
}

// Pairs that found no slot: the count words of the spill row.
__global__ void k_row_count(const unsigned long long* row, uint32_t nb, unsigned long long* out) {
  unsigned long long s = 0;
  for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) s += row[(size_t)b * kAccWords + 14];
  if (s) atomicAdd(out, s);
}

int blocks(const tos_engine* e, size_t work) {
  const size_t g = (work + 127) / 128, cap = (size_t)e->num_sms * 16;
  return (int)std::max<size_t>(1, std::min(g, cap));
}

struct DevGuard {
  int prev = -1;
  explicit DevGuard(int dev) {
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
  }
  ~DevGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace
}  // namespace tos

using namespace tos;

extern "C" tos_status tos_xi_run_jackknife(tos_engine* e, tos_catalog* cat, const tos_grid* grid,
                                           double scale, uint32_t flags, int region_order,
                                           size_t capacity, size_t* n_regions, int64_t* region_ids,
                                           tos_xibin* out_bins, tos_xibin* out_groups,
                                           tos_xibin* out_drop, tos_xi_stats* stats) {
  if (!e || !cat || !grid || !n_regions) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cat->device != e->device) return fail(TOS_ERR_INVALID_ARG, "catalogue is on another device");
  if (flags & ~TOS_XI_EXACT)
    return fail(TOS_ERR_INVALID_ARG, "a jackknife run takes no flag but TOS_XI_EXACT");
  if (cat->plates)
    return fail(TOS_ERR_UNSUPPORTED, "jackknife regions are HEALPix pixels: a plate catalogue has none");
  if (region_order < 0 || region_order > cat->order)
    return fail(TOS_ERR_INVALID_ARG, "region order must be in [0, catalogue order]");
  double max_ang = 0;
  TOS_TRY(tos_grid_max_angular_scale(grid, scale, &max_ang));
  // --- regions of the cells: group << 32 | pixel of order region_order
  const int64_t nside_r = (int64_t)1 << region_order;
  const size_t nc = cat->cells.size();
  std::vector<int64_t> creg(nc);
  for (size_t c = 0; c < nc; ++c) {
    double th, ph;
    healpix_pix2ang_ring(cat->nside, cat->cells[c] & 0xFFFFFFFFll, &th, &ph);
    creg[c] = (cat->cells[c] & ~0xFFFFFFFFll) | healpix_ang2pix_ring(nside_r, th, ph);
  }
  std::vector<int64_t> ids(creg);
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  const uint32_t nk = (uint32_t)ids.size();
  *n_regions = nk;
  if (!region_ids || !out_bins || !out_drop) return TOS_OK;  // size query
  if (capacity < nk) return fail(TOS_ERR_INVALID_ARG, "capacity below the number of regions");
  std::copy(ids.begin(), ids.end(), region_ids);
  // --- keys (dense region index) of cells and sightlines; key caps
  std::vector<uint32_t> ckey(nc), skey(cat->n_los), kgroup(nk);
  for (size_t c = 0; c < nc; ++c)
    ckey[c] = (uint32_t)(std::lower_bound(ids.begin(), ids.end(), creg[c]) - ids.begin());
  for (size_t s = 0; s < cat->n_los; ++s) skey[s] = ckey[cat->cell_idx[s]];
  std::vector<double4> kcap(nk, make_double4(0, 0, 0, 0));
  for (size_t c = 0; c < nc; ++c) {
    double4& k = kcap[ckey[c]];
    k.x += cat->caps[c].x, k.y += cat->caps[c].y, k.z += cat->caps[c].z;
  }
  for (uint32_t k = 0; k < nk; ++k) {
    double4& q = kcap[k];
    const double nrm = std::sqrt(q.x * q.x + q.y * q.y + q.z * q.z);
    if (nrm > 0) q.x /= nrm, q.y /= nrm, q.z /= nrm;
    else q.x = 0, q.y = 0, q.z = 1;
    q.w = 0;
  }
  for (size_t c = 0; c < nc; ++c) {  // radius: bounds every member cell's cap
    double4& q = kcap[ckey[c]];
    const double4& p = cat->caps[c];
    const double d = std::max(-1.0, std::min(1.0, q.x * p.x + q.y * p.y + q.z * p.z));
    q.w = std::max(q.w, (std::acos(d) + p.w) * (1 + 1e-9) + 1e-12);
  }
  // group of each key (keys are group-major, as the groups)
  for (uint32_t k = 0, g = 0; k < nk; ++k) {
    const uint32_t gid = (uint32_t)((uint64_t)ids[k] >> 32);
    while (cat->groups[g] != gid) ++g;
    kgroup[k] = g;
  }
  // --- slots of region pairs (a, b >= a) of one group that can hold a pair
  std::vector<uint32_t> slot_start(nk + 1, 0), slot_key;
  for (uint32_t a = 0; a < nk; ++a) {
    for (uint32_t b = a; b < nk && kgroup[b] == kgroup[a]; ++b) {
      const double lim = max_ang + kcap[a].w + kcap[b].w + 1e-9;
      bool near = true;
      if (lim < 3.14159) {
        const double dot = kcap[a].x * kcap[b].x + kcap[a].y * kcap[b].y + kcap[a].z * kcap[b].z;
        near = dot >= std::cos(lim) - 1e-12;
      }
      if (near) slot_key.push_back(b);
    }
    slot_start[a + 1] = (uint32_t)slot_key.size();
  }
  const uint32_t ns = (uint32_t)slot_key.size();
  // slots that name each key, and each group's slot range
  std::vector<uint32_t> kcount(nk + 1, 0), kslot_start(nk + 1, 0), kslot;
  for (uint32_t a = 0; a < nk; ++a)
    for (uint32_t q = slot_start[a]; q < slot_start[a + 1]; ++q) {
      kcount[a]++;
      if (slot_key[q] != a) kcount[slot_key[q]]++;
    }
  for (uint32_t k = 0; k < nk; ++k) kslot_start[k + 1] = kslot_start[k] + kcount[k];
  kslot.resize(kslot_start[nk]);
  {
    std::vector<uint32_t> fill(kslot_start.begin(), kslot_start.end() - 1);
    for (uint32_t a = 0; a < nk; ++a)
      for (uint32_t q = slot_start[a]; q < slot_start[a + 1]; ++q) {
        kslot[fill[a]++] = q;
        if (slot_key[q] != a) kslot[fill[slot_key[q]]++] = q;
      }
  }
  const uint32_t ngr = (uint32_t)cat->groups.size();
  std::vector<uint32_t> gslot(ngr + 1, ns);
  for (uint32_t k = nk; k-- > 0;) gslot[kgroup[k]] = slot_start[k];
  // --- device copies (local: released, on the engine's device, when the call returns)
  DevGuard dg(e->device);
  DevBuf<uint32_t> d_skey, d_slot_start, d_slot_key, d_kslot_start, d_kslot, d_kgroup, d_gslot;
  DevBuf<unsigned long long> d_gtot, d_spill;
  DevBuf<tos_xibin> d_gout, d_drop;
  {
    std::lock_guard<std::mutex> lock(e->mu);
    TOS_TRY(d_skey.alloc(cat->n_los));
    TOS_TRY(d_slot_start.alloc(nk + 1));
    TOS_TRY(d_slot_key.alloc(ns));
    TOS_TRY(d_kslot_start.alloc(nk + 1));
    TOS_TRY(d_kslot.alloc(kslot.size()));
    TOS_TRY(d_kgroup.alloc(nk));
    TOS_TRY(d_gslot.alloc(ngr + 1));
    TOS_TRY(d_spill.alloc(1));
    TOS_CUDA_TRY(cudaMemcpy(d_skey.p, skey.data(), skey.size() * 4, cudaMemcpyHostToDevice));
    TOS_CUDA_TRY(cudaMemcpy(d_slot_start.p, slot_start.data(), (nk + 1) * 4, cudaMemcpyHostToDevice));
    TOS_CUDA_TRY(cudaMemcpy(d_slot_key.p, slot_key.data(), (size_t)ns * 4, cudaMemcpyHostToDevice));
    TOS_CUDA_TRY(cudaMemcpy(d_kslot_start.p, kslot_start.data(), (nk + 1) * 4, cudaMemcpyHostToDevice));
    TOS_CUDA_TRY(cudaMemcpy(d_kslot.p, kslot.data(), kslot.size() * 4, cudaMemcpyHostToDevice));
    TOS_CUDA_TRY(cudaMemcpy(d_kgroup.p, kgroup.data(), (size_t)nk * 4, cudaMemcpyHostToDevice));
    TOS_CUDA_TRY(cudaMemcpy(d_gslot.p, gslot.data(), (ngr + 1) * 4, cudaMemcpyHostToDevice));
  }
  unsigned long long spill = 0;
  RowPlan plan;
  plan.n_rows = ns + 1;
  plan.row_key = d_skey.p;
  plan.slot_start = d_slot_start.p;
  plan.slot_key = d_slot_key.p;
  plan.max_row_items = [&](const std::vector<uint64_t>& cell_items) -> uint64_t {
    // a pair of slot {a, b} has its primary in region a or b
    std::vector<uint64_t> kitems(nk, 0);
    for (size_t c = 0; c < nc; ++c) kitems[ckey[c]] += cell_items[c];
    uint64_t m = 0;
    for (uint32_t a = 0; a < nk; ++a)
      for (uint32_t q = slot_start[a]; q < slot_start[a + 1]; ++q)
        m = std::max(m, kitems[a] + (slot_key[q] != a ? kitems[slot_key[q]] : 0));
    return m;
  };
  plan.combine = [&](cudaStream_t st, uint32_t nb, const double* inv_scale,
                     const unsigned long long* d_acc, tos_xibin* d_out) -> tos_status {
    Inv7 inv;
    for (int k = 0; k < 7; ++k) inv.v[k] = inv_scale[k];
    TOS_TRY(d_gtot.alloc((size_t)ngr * nb * kAccWords));
    TOS_TRY(d_gout.alloc((size_t)ngr * nb));
    TOS_TRY(d_drop.alloc((size_t)nk * nb));
    TOS_CUDA_TRY(cudaMemsetAsync(d_spill.p, 0, 8, st));
    k_group_totals<<<blocks(e, (size_t)ngr * nb), 128, 0, st>>>(d_acc, nb, d_gslot.p, ngr, inv,
                                                                d_gtot.p, d_gout.p);
    TOS_CUDA_TRY(cudaGetLastError());
    launch_sum_rows(d_gout.p, ngr, nb, d_out, blocks(e, nb), st);
    TOS_CUDA_TRY(cudaGetLastError());
    k_drop<<<blocks(e, (size_t)nk * nb), 128, 0, st>>>(d_acc, d_gtot.p, nb, d_kslot_start.p,
                                                       d_kslot.p, d_kgroup.p, nk, inv, d_drop.p);
    TOS_CUDA_TRY(cudaGetLastError());
    k_row_count<<<1, 256, 0, st>>>(d_acc + (size_t)ns * nb * kAccWords, nb, d_spill.p);
    TOS_CUDA_TRY(cudaGetLastError());
    if (out_groups)
      TOS_CUDA_TRY(cudaMemcpyAsync(out_groups, d_gout.p, (size_t)ngr * nb * sizeof(tos_xibin),
                                   cudaMemcpyDeviceToHost, st));
    TOS_CUDA_TRY(cudaMemcpyAsync(out_drop, d_drop.p, (size_t)nk * nb * sizeof(tos_xibin),
                                 cudaMemcpyDeviceToHost, st));
    TOS_CUDA_TRY(cudaMemcpyAsync(&spill, d_spill.p, 8, cudaMemcpyDeviceToHost, st));
    return TOS_OK;
  };
  {
    std::lock_guard<std::mutex> lock(cat->run_mu);
    TOS_TRY(xi_run_impl(e, cat, &cat->run, grid, scale, flags, &plan, out_bins, nullptr, stats));
  }
  if (spill != 0)
    return fail(TOS_ERR_INTERNAL, std::to_string(spill) + " pixel pairs found no region slot");
  return TOS_OK;
}
