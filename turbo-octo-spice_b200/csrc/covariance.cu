// covariance.cu — sample covariances of the XiEstimator pair count from the
// per-cell sums that tos_xi_run leaves on the device:
//  - the reference's covariance of per-cell correlation functions
//    (XiEstimator::run with do_cov, XiEstimator.cc:60-97): each occupied sky
//    cell is a sample x_c[b] = didj/wgt (0 where wgt = 0) of weight W_c, the
//    sum of wgt over its bins with wgt > 0;
//  - a leave-one-region-out jackknife over HEALPix regions of a coarser order
//    (the jackknife subsamples of the batched configuration): region k's
//    estimate is the full count minus the cells inside region k, subtracted
//    exactly in the 128-bit fixed point of the per-cell sums.
// Both end in C = s * X^T X for a centred sample matrix X (k_gram), an FP64
// product whose summation order is fixed, so results are deterministic.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "engine_internal.h"
#include "healpix.h"
#include "fixed128.cuh"
#include "xi_kernels.cuh"

namespace tos {
namespace {

constexpr unsigned kFullMask = 0xFFFFFFFFu;

// One block per cell: x[c][b] = didj/wgt (wgt > 0) else 0, w[c] = sum of wgt > 0.
__global__ void k_cell_samples(const unsigned long long* acc, uint32_t nb, double inv_didj,
                               double inv_wgt, double* X, double* w) {
  const uint32_t c = blockIdx.x;
  double ws = 0;
  for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
    const unsigned long long* base = acc + ((size_t)c * nb + b) * kAccWords;
    const double didj = (base[14] != 0) ? i128_double(acc128(base, 0)) * inv_didj : 0.0;
    const double wgt = (base[14] != 0) ? i128_double(acc128(base, 3)) * inv_wgt : 0.0;
    const bool ok = wgt > 0;
    X[(size_t)c * nb + b] = ok ? didj / wgt : 0.0;
    ws += ok ? wgt : 0.0;
  }
  // block sum in a fixed order: warp trees, then warp 0
  __shared__ double part[32];
  for (int o = 16; o > 0; o >>= 1) ws += __shfl_down_sync(kFullMask, ws, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = ws;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = (threadIdx.x < (blockDim.x >> 5)) ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(kFullMask, v, o);
    if (threadIdx.x == 0) w[c] = v;
  }
}

// Weighted column means over n samples, summed in sample order (w = null:
// unit weights).  mean[b] = sum_s w_s X[s][b] / W.
__global__ void k_col_mean(const double* X, const double* w, uint32_t n, uint32_t nb, double inv_W,
                           double* mean) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    double s = 0;
    for (uint32_t r = 0; r < n; ++r) s = __fma_rn(w ? w[r] : 1.0, X[(size_t)r * nb + b], s);
    mean[b] = s * inv_W;
  }
}

// X[s][b] = sqrt(w_s) (X[s][b] - mean[b])  (w = null: unit weights)
__global__ void k_center(double* X, const double* w, const double* mean, uint32_t n, uint32_t nb) {
  const size_t total = (size_t)n * nb;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint32_t r = (uint32_t)(e / nb), b = (uint32_t)(e % nb);
    const double sw = w ? sqrt(w[r]) : 1.0;
    X[e] = sw * (X[e] - mean[b]);
  }
}

// C = s * X^T X (nb x nb, row-major) for X of n rows: 64 x 64 output tiles of
// 16 x 16 threads (4 x 4 outputs each); rows of X staged 16 at a time in
// shared memory.  Each output sums its products in row order.
constexpr int kT = 64, kK = 16;
__global__ void __launch_bounds__(256) k_gram(const double* X, uint32_t n, uint32_t nb, double s,
                                              double* C) {
  __shared__ double A[kK][kT], B[kK][kT];
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  const uint32_t i0 = blockIdx.y * kT, j0 = blockIdx.x * kT;
  double acc[4][4] = {};
  for (uint32_t r0 = 0; r0 < n; r0 += kK) {
    for (int e = threadIdx.x; e < kK * kT; e += 256) {
      const int rr = e / kT, cc = e % kT;
      const uint32_t r = r0 + rr;
      A[rr][cc] = (r < n && i0 + cc < nb) ? X[(size_t)r * nb + i0 + cc] : 0.0;
      B[rr][cc] = (r < n && j0 + cc < nb) ? X[(size_t)r * nb + j0 + cc] : 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int rr = 0; rr < kK; ++rr) {
      double a[4], b[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        a[q] = A[rr][ty + 16 * q];
        b[q] = B[rr][tx + 16 * q];
      }
#pragma unroll
      for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = 0; q < 4; ++q) acc[p][q] = __fma_rn(a[p], b[q], acc[p][q]);
    }
    __syncthreads();
  }
#pragma unroll
  for (int p = 0; p < 4; ++p)
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const uint32_t i = i0 + ty + 16 * p, j = j0 + tx + 16 * q;
      if (i < nb && j < nb) C[(size_t)i * nb + j] = s * acc[p][q];
    }
}

// Exact totals over all cells of the didj and wgt sums of each bin.
__global__ void k_total(const unsigned long long* acc, uint32_t nc, uint32_t nb, __int128* tot) {
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    __int128 d = 0, g = 0;
    for (uint32_t c = 0; c < nc; ++c) {
      const unsigned long long* base = acc + ((size_t)c * nb + b) * kAccWords;
      d += acc128(base, 0);
      g += acc128(base, 3);
    }
    tot[2 * b] = d;
    tot[2 * b + 1] = g;
  }
}

// Leave-one-region-out estimates: xi[k][b] = (D - D_k) / (G - G_k) with the
// region's cells cells[start[k] .. start[k+1]) subtracted exactly (0 where
// the remaining wgt is not positive).
__global__ void k_region_xi(const unsigned long long* acc, uint32_t nb, const __int128* tot,
                            const uint32_t* start, const uint32_t* cells, uint32_t nreg,
                            double inv_didj, double inv_wgt, double* xi) {
  const size_t total = (size_t)nreg * nb;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total;
       e += (size_t)gridDim.x * blockDim.x) {
    const uint32_t k = (uint32_t)(e / nb), b = (uint32_t)(e % nb);
    __int128 d = tot[2 * b], g = tot[2 * b + 1];
    for (uint32_t m = start[k]; m < start[k + 1]; ++m) {
      const unsigned long long* base = acc + ((size_t)cells[m] * nb + b) * kAccWords;
      d -= acc128(base, 0);
      g -= acc128(base, 3);
    }
    const double gw = i128_double(g) * inv_wgt;
    xi[e] = gw > 0 ? i128_double(d) * inv_didj / gw : 0.0;
  }
}

int blocks_for(size_t work, int block, int nsm) {
  size_t g = (work + block - 1) / block;
  const size_t cap = (size_t)nsm * 32;
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

// mean and C = scale * sum_r w_r (X_r - mean)(X_r - mean)^T of X (n x nb) on
// the device; w = null for unit weights.
tos_status sample_covariance(tos_engine* e, double* dX, const double* dw, uint32_t n, uint32_t nb,
                             double W, double scale, double* mean_out, double* cov_out) {
  cudaStream_t st = e->stream;
  DevBuf<double> dmean, dC;
  TOS_TRY(dmean.alloc(nb));
  TOS_TRY(dC.alloc((size_t)nb * nb));
  k_col_mean<<<blocks_for(nb, 128, e->num_sms), 128, 0, st>>>(dX, dw, n, nb, 1.0 / W, dmean.p);
  k_center<<<blocks_for((size_t)n * nb, 256, e->num_sms), 256, 0, st>>>(dX, dw, dmean.p, n, nb);
  const dim3 grid((nb + kT - 1) / kT, (nb + kT - 1) / kT);
  k_gram<<<grid, 256, 0, st>>>(dX, n, nb, scale, dC.p);
  TOS_CUDA_TRY(cudaGetLastError());
  if (mean_out)
    TOS_CUDA_TRY(cudaMemcpyAsync(mean_out, dmean.p, (size_t)nb * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cov_out, dC.p, (size_t)nb * nb * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  return TOS_OK;
}

tos_status check_last_run(tos_engine* e, tos_catalog* cat) {
  if (!e || !cat) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (cat->device != e->device) return fail(TOS_ERR_INVALID_ARG, "catalogue is on another device");
  if (!cat->run.last_valid || !cat->run.d_acc.p)
    return fail(TOS_ERR_INVALID_ARG, "no completed tos_xi_run on this catalogue");
  return TOS_OK;
}

}  // namespace
}  // namespace tos

using namespace tos;

extern "C" tos_status tos_xi_cell_covariance(tos_engine* e, tos_catalog* cat, double* mean,
                                             double* cov, double* total_weight) {
  if (!cat) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> run_lock(cat->run_mu);  // the sums of cat->run stay put
  TOS_TRY(check_last_run(e, cat));
  if (!cov) return fail(TOS_ERR_INVALID_ARG, "cov is null");
  std::lock_guard<std::mutex> lock(e->mu);
  DevGuard g(e->device);
  const uint32_t nb = cat->run.last_nb, nc = (uint32_t)cat->cells.size();
  cudaStream_t st = e->stream;
  DevBuf<double> dX, dw;
  TOS_TRY(dX.alloc((size_t)nc * nb));
  TOS_TRY(dw.alloc(nc));
  k_cell_samples<<<nc, 256, 0, st>>>(cat->run.d_acc.p, nb, cat->run.last_inv_scale[0], cat->run.last_inv_scale[3],
                                     dX.p, dw.p);
  TOS_CUDA_TRY(cudaGetLastError());
  std::vector<double> w(nc);
  TOS_CUDA_TRY(cudaMemcpyAsync(w.data(), dw.p, (size_t)nc * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  double W = 0;
  for (double v : w) W += v;  // cell order
  if (total_weight) *total_weight = W;
  if (!(W > 0)) return fail(TOS_ERR_INVALID_ARG, "no cell has a bin with positive weight");
  return sample_covariance(e, dX.p, dw.p, nc, nb, W, 1.0 / W, mean, cov);
}

extern "C" tos_status tos_xi_jackknife(tos_engine* e, tos_catalog* cat, int region_order, size_t cap,
                                       size_t* n_regions, int64_t* region_ids, double* xi_jk,
                                       double* cov) {
  if (!cat) return fail(TOS_ERR_INVALID_ARG, "null argument");
  std::lock_guard<std::mutex> run_lock(cat->run_mu);  // the sums of cat->run stay put
  TOS_TRY(check_last_run(e, cat));
  if (!n_regions) return fail(TOS_ERR_INVALID_ARG, "n_regions is null");
  if (cat->plates)
    return fail(TOS_ERR_UNSUPPORTED, "jackknife regions are HEALPix pixels: a plate catalogue has none");
  if (region_order < 0 || region_order > cat->order)
    return fail(TOS_ERR_INVALID_ARG, "region order must be in [0, catalogue order]");
  if (cat->groups.size() != 1)
    return fail(TOS_ERR_INVALID_ARG, "jackknife regions need a catalogue of one sightline group");
  // regions of the occupied cells (a cell lies inside the coarser pixel that
  // holds its centre: both orders tile the same HEALPix hierarchy)
  const int64_t nside_r = (int64_t)1 << region_order;
  const size_t nc = cat->cells.size();
  std::vector<int64_t> reg(nc);
  for (size_t c = 0; c < nc; ++c) {
    double th, ph;
    healpix_pix2ang_ring(cat->nside, cat->cells[c] & 0xFFFFFFFFll, &th, &ph);
    reg[c] = healpix_ang2pix_ring(nside_r, th, ph);
  }
  std::vector<int64_t> ids(reg);
  std::sort(ids.begin(), ids.end());
  ids.erase(std::unique(ids.begin(), ids.end()), ids.end());
  const size_t nr = ids.size();
  *n_regions = nr;
  if (!region_ids || !xi_jk || !cov) return TOS_OK;  // size query
  if (cap < nr) return fail(TOS_ERR_INVALID_ARG, "capacity below the number of regions");
  if (nr < 2) return fail(TOS_ERR_INVALID_ARG, "a jackknife needs at least two regions");
  std::vector<uint32_t> start(nr + 1, 0), members(nc);
  for (size_t c = 0; c < nc; ++c)
    ++start[std::lower_bound(ids.begin(), ids.end(), reg[c]) - ids.begin() + 1];
  for (size_t k = 0; k < nr; ++k) start[k + 1] += start[k];
  {
    std::vector<uint32_t> fill(start.begin(), start.end() - 1);
    for (size_t c = 0; c < nc; ++c)
      members[fill[std::lower_bound(ids.begin(), ids.end(), reg[c]) - ids.begin()]++] = (uint32_t)c;
  }
  std::copy(ids.begin(), ids.end(), region_ids);
  std::lock_guard<std::mutex> lock(e->mu);
  DevGuard g(e->device);
  const uint32_t nb = cat->run.last_nb;
  cudaStream_t st = e->stream;
  DevBuf<__int128> dtot;
  DevBuf<uint32_t> dstart, dmem;
  DevBuf<double> dX;
  TOS_TRY(dtot.alloc((size_t)2 * nb));
  TOS_TRY(dstart.alloc(nr + 1));
  TOS_TRY(dmem.alloc(nc));
  TOS_TRY(dX.alloc((size_t)nr * nb));
  TOS_CUDA_TRY(cudaMemcpyAsync(dstart.p, start.data(), (nr + 1) * 4, cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(dmem.p, members.data(), nc * 4, cudaMemcpyHostToDevice, st));
  k_total<<<blocks_for(nb, 128, e->num_sms), 128, 0, st>>>(cat->run.d_acc.p, (uint32_t)nc, nb, dtot.p);
  k_region_xi<<<blocks_for((size_t)nr * nb, 128, e->num_sms), 128, 0, st>>>(
      cat->run.d_acc.p, nb, dtot.p, dstart.p, dmem.p, (uint32_t)nr, cat->run.last_inv_scale[0],
      cat->run.last_inv_scale[3], dX.p);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaMemcpyAsync(xi_jk, dX.p, (size_t)nr * nb * 8, cudaMemcpyDeviceToHost, st));
  // C = (N - 1)/N sum_k (xi_k - mean)(xi_k - mean)^T
  return sample_covariance(e, dX.p, nullptr, (uint32_t)nr, nb, (double)nr, (double)(nr - 1) / (double)nr,
                           nullptr, cov);
}

extern "C" tos_status tos_xi_subsample_covariance(tos_engine* e, const tos_xibin* rows,
                                                  size_t n_rows, size_t n_bins, double* xi,
                                                  double* mean, double* cov) {
  if (!e || !rows || !cov) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (n_rows < 2) return fail(TOS_ERR_INVALID_ARG, "need at least two subsamples");
  if (n_bins < 1 || n_bins > 65536 || n_rows > 0xFFFFFFFFull)
    return fail(TOS_ERR_INVALID_ARG, "n_bins must be in [1, 65536]");
  // xi_k[b] = didj / wgt, 0 where wgt <= 0 (as the per-cell samples)
  std::vector<double> X(n_rows * n_bins);
  for (size_t k = 0; k < n_rows * n_bins; ++k)
    X[k] = rows[k].wgt > 0 ? rows[k].didj / rows[k].wgt : 0.0;
  if (xi) std::copy(X.begin(), X.end(), xi);
  std::lock_guard<std::mutex> lock(e->mu);
  DevGuard g(e->device);
  DevBuf<double> dX;
  TOS_TRY(dX.alloc(X.size()));
  TOS_CUDA_TRY(cudaMemcpyAsync(dX.p, X.data(), X.size() * 8, cudaMemcpyHostToDevice, e->stream));
  const double n = (double)n_rows;
  // C = (N - 1)/N sum_k (xi_k - mean)(xi_k - mean)^T
  return sample_covariance(e, dX.p, nullptr, (uint32_t)n_rows, (uint32_t)n_bins, n, (n - 1.0) / n,
                           mean, cov);
}
