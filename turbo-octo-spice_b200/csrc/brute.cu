// brute.cu — all-pairs isotropic xi(r) of points (x, y, z, delta, w): the
// computation of bruteGPU / histo_kernel (gpu/brute.cu:7-61, 63-225), redone
// for sm_100a.
//
// Differences from the reference design, all in service of exactness and
// throughput:
//  - points stay resident in HBM (no per-chunk host copies, brute.cu:155-193);
//  - every unordered pair i < j is visited once by a persistent sweep: a warp
//    owns 32 consecutive points i (lane = i) and walks j = t + lane, so on a
//    regular grid every lane has the same separation vector at the same step;
//  - separations are binned in FP32 with an FP64 re-binning of pairs within
//    2^-K bins of an edge, so bins equal those of the FP64 separation
//    sqrt(dx^2+dy^2+dz^2) (the double-precision estimator of bucketxi.cc:79-98);
//  - sums are exact: runs of equal bins are summed from FP64 prefix sums,
//    quantised to fixed point and added with u32 shared atomics into a
//    per-warp window, which is added to FP64 global sums when a slot fills.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "engine_internal.h"

namespace tos {
namespace {

constexpr unsigned kFull = 0xFFFFFFFFu;
constexpr int kBruteWarps = 16;
constexpr int kBWords = 6;          // dsum lo/hi, wsum lo/hi, count, contributions
constexpr int kBSplit = 20;
constexpr uint32_t kSlotLimit = 3800;  // contributions per slot before the window is emptied
constexpr int kRunCap = 64;            // longest run summed as one contribution
constexpr double kMagic = 6755399441055744.0;
constexpr long long kMagicBits = 0x4338000000000000LL;

struct BruteArgs {
  const float4* pos;      // (x, y, z, 0), n entries
  const double2* prefix;  // n+1 exclusive prefix sums of (w*delta, w)
  const double* wd;       // w*delta per point
  const double* w;        // w per point
  int n;
  int nbins;
  double min, max, spacing;
  float invf, offf, nbf, nbp1f;
  int k;
  float mag;
  int bits;
  double scale[2];
  double inv_scale[2];
  double* out;            // [nbins+2][2] FP64 sums
  unsigned long long* counts;  // [nbins+2]
  unsigned long long* next;    // chunk counter
  unsigned long long* counters;  // [0] rechecks
};

__device__ __forceinline__ float sqrt_approx(float x) {
  float r;
  asm("sqrt.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ long long to_fixed(double c, double scale) {
  return __double_as_longlong(__fma_rn(c, scale, kMagic)) - kMagicBits;
}

// Histogram index of the FP64 separation: 0 below min, nbins+1 at or above
// max, else floor((r - min) / spacing) + 1 (gpu/brute.cu:40-48 in FP64).
__device__ __forceinline__ uint32_t exact_index(const BruteArgs& A, float4 a, float4 b) {
  const double dx = dsub((double)a.x, (double)b.x), dy = dsub((double)a.y, (double)b.y),
               dz = dsub((double)a.z, (double)b.z);
  const double r = dsqrt(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
  if (r < A.min) return 0u;
  if (r >= A.max) return (uint32_t)A.nbins + 1u;
  double k = floor(ddiv(dsub(r, A.min), A.spacing));
  if (k > (double)(A.nbins - 1)) k = (double)(A.nbins - 1);
  return (uint32_t)k + 1u;
}

__device__ void flush(const BruteArgs& A, uint32_t* win, int lane) {
  const int S = A.nbins + 2;
  for (int s = lane; s < S; s += 32) {
    const uint32_t cnt = win[4 * S + s];
    if (cnt == 0) continue;
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const uint32_t lo = win[(2 * f) * S + s];
      const int hi = (int)win[(2 * f + 1) * S + s];
      const long long q = ((long long)hi << kBSplit) + (long long)lo;
      atomicAdd(&A.out[2 * s + f], (double)q * A.inv_scale[f]);
    }
    atomicAdd(&A.counts[s], (unsigned long long)cnt);
#pragma unroll
    for (int w = 0; w < kBWords; ++w) win[w * S + s] = 0u;
  }
  __syncwarp();
}

__global__ void __launch_bounds__(kBruteWarps * 32, 1) brute_kernel(BruteArgs A) {
  extern __shared__ uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int S = A.nbins + 2;
  uint32_t* win = smem + (size_t)warp * kBWords * S;
  for (int k = lane; k < kBWords * S; k += 32) win[k] = 0u;
  __syncwarp();
  unsigned long long n_recheck = 0;
  const int nchunks = (A.n + 31) / 32;
  bool full = false;
  for (;;) {
    unsigned long long c = 0;
    if (lane == 0) c = atomicAdd(A.next, 1ull);
    c = __shfl_sync(kFull, c, 0);
    if (c >= (unsigned long long)nchunks) break;
    // big chunks (long sweeps) first: chunk c covers rows i0 = 32*c'
    const int i0 = 32 * (int)c;
    const int i = i0 + lane;
    const bool active = i < A.n;
    const float4 pi = active ? A.pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
    const double wdi = active ? A.wd[i] : 0.0, wi = active ? A.w[i] : 0.0;
    uint32_t cur = 0xFFFFFFFFu;
    int run_start = 0;
    double ps0 = 0, ps1 = 0;
    // Add the runs that lanes with `emit` close (bin `slot`, its words):
    // lanes closing a run in the same bin, which on a regular grid is most
    // of the warp (one separation vector per step), sum their words with
    // redux.sync and one of them adds the sums to the window.
    auto emit_runs = [&](bool emit, uint32_t slot, const uint32_t (&wv)[5]) {
      unsigned pending = __ballot_sync(kFull, emit);
      while (pending) {
        const int leader = __ffs(pending) - 1;
        const uint32_t ls = __shfl_sync(kFull, slot, leader);
        const unsigned peers = __ballot_sync(kFull, ((pending >> lane) & 1u) && slot == ls);
        if ((peers >> lane) & 1u) {
          uint32_t sw[5];
#pragma unroll
          for (int w = 0; w < 5; ++w) sw[w] = __reduce_add_sync(peers, wv[w]);
          if (lane == leader) {
#pragma unroll
            for (int w = 0; w < 5; ++w) atomicAdd(&win[w * S + ls], sw[w]);
            const uint32_t n = (uint32_t)__popc(peers);
            const uint32_t old = atomicAdd(&win[5 * S + ls], n);
            if (old + n > kSlotLimit) full = true;
          }
        }
        pending &= ~peers;
      }
    };
    auto run_words = [&](int p_end, double2 pn, uint32_t (&wv)[5]) {
      const double c0 = wdi * (pn.x - ps0), c1 = wi * (pn.y - ps1);
      const long long q0 = to_fixed(c0, A.scale[0]), q1 = to_fixed(c1, A.scale[1]);
      wv[0] = (uint32_t)q0 & ((1u << kBSplit) - 1u);
      wv[1] = (uint32_t)(int)(q0 >> kBSplit);
      wv[2] = (uint32_t)q1 & ((1u << kBSplit) - 1u);
      wv[3] = (uint32_t)(int)(q1 >> kBSplit);
      wv[4] = (uint32_t)(p_end - run_start);
    };
    for (int t = i0 + 1; t < A.n; ++t) {
      const int j = t + lane;
      uint32_t key = 0xFFFFFFFFu;
      bool recheck = false;
      float4 pj = make_float4(0.f, 0.f, 0.f, 0.f);
      if (active && j < A.n) {
        pj = A.pos[j];
        const float dx = __fsub_rn(pi.x, pj.x), dy = __fsub_rn(pi.y, pj.y),
                    dz = __fsub_rn(pi.z, pj.z);
        const float r2 = __fmaf_rn(dx, dx, __fmaf_rn(dy, dy, __fmul_rn(dz, dz)));
        const float tt = __fmaf_rn(sqrt_approx(r2), A.invf, A.offf);
        const int q = __float_as_int(__fadd_rz(tt, A.mag)) - A.bits;
        int b = (q >> A.k) + 1;
        b = (tt < 0.f) ? 0 : ((tt >= A.nbf) ? A.nbins + 1 : b);
        key = (uint32_t)b;
        recheck = (((q + 1) & ((1 << A.k) - 1)) < 2) && (tt < A.nbp1f) && (tt > -1.f);
      }
      if (__any_sync(kFull, recheck)) {
        if (recheck) {
          key = exact_index(A, pi, pj);
          ++n_recheck;
        }
      }
      const bool change = (key != cur) || (cur != 0xFFFFFFFFu && j - run_start >= kRunCap);
      if (__any_sync(kFull, change)) {
        uint32_t wv[5] = {0u, 0u, 0u, 0u, 0u};
        const bool emit = change && cur != 0xFFFFFFFFu;
        const uint32_t slot = cur;
        if (change) {
          const int pc = min(j, A.n);
          const double2 pn = A.prefix[pc];
          if (emit) run_words(j, pn, wv);
          cur = key;
          run_start = j;
          ps0 = pn.x;
          ps1 = pn.y;
        }
        emit_runs(emit, slot, wv);
        if (__any_sync(kFull, full)) {
          flush(A, win, lane);
          full = false;
        }
      }
    }
    {
      // the sweep ended at t = n-1, so lane's last j = n-1+lane; runs only
      // cover real points, hence every open run ends at n
      uint32_t wv[5] = {0u, 0u, 0u, 0u, 0u};
      const bool emit = cur != 0xFFFFFFFFu;
      if (emit) run_words(A.n, A.prefix[A.n], wv);
      emit_runs(emit, cur, wv);
    }
    if (__any_sync(kFull, full)) {
      flush(A, win, lane);
      full = false;
    }
  }
  flush(A, win, lane);
  for (int o = 16; o > 0; o >>= 1) n_recheck += __shfl_xor_sync(kFull, n_recheck, o);
  if (lane == 0) atomicAdd(&A.counters[0], n_recheck);
}

// Launch shape: a warp's window holds kBWords words for each of the
// nbins + 2 bins, so as many warps (up to kBruteWarps) as the block's opt-in
// shared memory holds windows for.  The kernel takes its warp count from the
// block size.  Fails only if not even one window fits.
tos_status brute_shape(const tos_engine* e, int nbins, int* warps, size_t* smem) {
  const size_t per_warp = (size_t)kBWords * (nbins + 2) * sizeof(uint32_t);
  const size_t fit = e->smem_optin / per_warp;
  if (fit < 1)
    return fail(TOS_ERR_UNSUPPORTED, "nbins too large for one warp's shared-memory window on this device");
  *warps = (int)std::min<size_t>(kBruteWarps, fit);
  *smem = (size_t)*warps * per_warp;
  return TOS_OK;
}

__global__ void k_brute_prep(const float* pts, int n, float4* pos, double* wd, double* w) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float* p = pts + 5 * (size_t)k;
    pos[k] = make_float4(p[0], p[1], p[2], 0.f);
    wd[k] = (double)p[4] * (double)p[3];
    w[k] = (double)p[4];
  }
}

// single-block exclusive scan of (wd, w) (n up to a few million: fine for a prep step)
__global__ void k_brute_scan(const double* wd, const double* w, int n, double2* prefix) {
  __shared__ double s0[1024], s1[1024];
  double c0 = 0, c1 = 0;
  if (threadIdx.x == 0) prefix[0] = make_double2(0, 0);
  for (int base = 0; base < n; base += 1024) {
    const int k = base + threadIdx.x;
    s0[threadIdx.x] = k < n ? wd[k] : 0.0;
    s1[threadIdx.x] = k < n ? w[k] : 0.0;
    __syncthreads();
    for (int d = 1; d < 1024; d <<= 1) {
      double a0 = 0, a1 = 0;
      if (threadIdx.x >= (unsigned)d) {
        a0 = s0[threadIdx.x - d];
        a1 = s1[threadIdx.x - d];
      }
      __syncthreads();
      s0[threadIdx.x] += a0;
      s1[threadIdx.x] += a1;
      __syncthreads();
    }
    if (k < n) prefix[k + 1] = make_double2(c0 + s0[threadIdx.x], c1 + s1[threadIdx.x]);
    c0 += s0[1023];
    c1 += s1[1023];
    __syncthreads();
  }
}

}  // namespace
}  // namespace tos

using namespace tos;

extern "C" tos_status tos_brute_run(tos_engine* e, const float* points, size_t n_points, double min,
                                    double max, int nbins, double* dsum, double* wsum,
                                    uint64_t* counts, double* ms_kernel) {
  if (!e || !points || !dsum || !wsum || !counts) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (n_points < 2 || n_points > (1u << 28)) return fail(TOS_ERR_INVALID_ARG, "need 2 <= n < 2^28 points");
  if (nbins <= 0 || nbins > 4096) return fail(TOS_ERR_INVALID_ARG, "nbins must be in [1, 4096]");
  if (!(max > min) || !std::isfinite(min) || !std::isfinite(max))
    return fail(TOS_ERR_INVALID_ARG, "need finite min < max");
  std::lock_guard<std::mutex> lock(e->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  const int n = (int)n_points;
  cudaStream_t st = e->stream;
  DevBuf<float> d_pts;
  DevBuf<float4> d_pos;
  DevBuf<double> d_wd, d_w, d_out;
  DevBuf<double2> d_prefix;
  DevBuf<unsigned long long> d_counts, d_misc;
  TOS_TRY(d_pts.alloc((size_t)n * 5));
  TOS_TRY(d_pos.alloc(n));
  TOS_TRY(d_wd.alloc(n));
  TOS_TRY(d_w.alloc(n));
  TOS_TRY(d_prefix.alloc((size_t)n + 1));
  TOS_TRY(d_out.alloc((size_t)(nbins + 2) * 2));
  TOS_TRY(d_counts.alloc(nbins + 2));
  TOS_TRY(d_misc.alloc(4));
  TOS_CUDA_TRY(cudaMemcpyAsync(d_pts.p, points, (size_t)n * 5 * sizeof(float),
                               cudaMemcpyHostToDevice, st));
  TOS_CUDA_TRY(cudaMemsetAsync(d_out.p, 0, (size_t)(nbins + 2) * 2 * 8, st));
  TOS_CUDA_TRY(cudaMemsetAsync(d_counts.p, 0, (size_t)(nbins + 2) * 8, st));
  TOS_CUDA_TRY(cudaMemsetAsync(d_misc.p, 0, 32, st));
  k_brute_prep<<<std::min(4096, (n + 255) / 256), 256, 0, st>>>(d_pts.p, n, d_pos.p, d_wd.p, d_w.p);
  k_brute_scan<<<1, 1024, 0, st>>>(d_wd.p, d_w.p, n, d_prefix.p);
  TOS_CUDA_TRY(cudaGetLastError());
  // bounds of |w*delta| and |w| for the fixed-point scale
  std::vector<float> hp((size_t)n * 5);
  std::memcpy(hp.data(), points, hp.size() * sizeof(float));
  double mwd = 1e-300, mw = 1e-300;
  for (int k = 0; k < n; ++k) {
    const double wv = hp[5 * (size_t)k + 4], dv = hp[5 * (size_t)k + 3];
    if (!std::isfinite(wv) || !std::isfinite(dv) || !std::isfinite(hp[5 * (size_t)k]) ||
        !std::isfinite(hp[5 * (size_t)k + 1]) || !std::isfinite(hp[5 * (size_t)k + 2]))
      return fail(TOS_ERR_INVALID_ARG, "points must be finite");
    mwd = std::max(mwd, std::fabs(wv * dv));
    mw = std::max(mw, std::fabs(wv));
  }
  BruteArgs A{};
  A.pos = d_pos.p;
  A.prefix = d_prefix.p;
  A.wd = d_wd.p;
  A.w = d_w.p;
  A.n = n;
  A.nbins = nbins;
  A.min = min;
  A.max = max;
  A.spacing = (max - min) / nbins;
  A.invf = (float)(1.0 / A.spacing);
  A.offf = (float)(-min / A.spacing);
  A.nbf = (float)nbins;
  A.nbp1f = (float)nbins + 1.0f;
  int bl = 0;
  for (uint32_t v = (uint32_t)nbins + 2; v; v >>= 1) ++bl;
  A.k = std::max(0, std::min(13, 21 - bl));
  A.mag = std::ldexp(1.5f, 23 - A.k);
  std::memcpy(&A.bits, &A.mag, 4);
  const double per[2] = {mwd * kRunCap * mwd, mw * kRunCap * mw};
  for (int f = 0; f < 2; ++f) {
    const int F = (int)std::floor(38.0 - std::log2(per[f]));
    A.scale[f] = std::ldexp(1.0, F);
    A.inv_scale[f] = std::ldexp(1.0, -F);
  }
  A.out = d_out.p;
  A.counts = d_counts.p;
  A.next = d_misc.p;
  A.counters = d_misc.p + 1;
  int warps = 0;
  size_t smem = 0;
  TOS_TRY(brute_shape(e, nbins, &warps, &smem));
  TOS_CUDA_TRY(cudaFuncSetAttribute(brute_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  TOS_CUDA_TRY(cudaEventRecord(e->ev[4], st));
  brute_kernel<<<e->num_sms, warps * 32, smem, st>>>(A);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaEventRecord(e->ev[5], st));
  std::vector<double> out((size_t)(nbins + 2) * 2);
  std::vector<unsigned long long> cnt(nbins + 2);
  TOS_CUDA_TRY(cudaMemcpyAsync(out.data(), d_out.p, out.size() * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaMemcpyAsync(cnt.data(), d_counts.p, cnt.size() * 8, cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  for (int b = 0; b < nbins + 2; ++b) {
    dsum[b] = out[2 * b];
    wsum[b] = out[2 * b + 1];
    counts[b] = cnt[b];
  }
  if (ms_kernel) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[4], e->ev[5]);
    *ms_kernel = ms;
  }
  return TOS_OK;
}

// ============================================================================
// Allocation-free variant of tos_brute_run.
//
// Some callers cannot allocate device memory while they count pairs: code
// that manages every byte of the GPU through its own pool, code that runs
// where a cudaMalloc would synchronise the device or is not allowed, or
// service loops that must not touch the allocator at all.  tos_brute_run allocates its
// scratch on every call; tos_brute_run_noalloc takes its inputs and outputs
// in device memory and keeps all scratch in one statically sized device
// array that the library reserves on every GPU that loads it, until exit.
// ============================================================================

namespace tos {
namespace {

constexpr size_t kNoAllocMaxPoints = size_t(1) << 18;  // 262,144 points (a 64^3 grid)
constexpr int kNoAllocMaxBins = 4096;

constexpr size_t round256(size_t b) { return (b + 255) & ~size_t(255); }
// scratch layout (byte offsets, each 256-byte aligned)
constexpr size_t kNaPos = 0;                                                  // float4[n]
constexpr size_t kNaWd = kNaPos + round256(16 * kNoAllocMaxPoints);           // double[n]
constexpr size_t kNaW = kNaWd + round256(8 * kNoAllocMaxPoints);              // double[n]
constexpr size_t kNaPrefix = kNaW + round256(8 * kNoAllocMaxPoints);          // double2[n + 1]
constexpr size_t kNaOut = kNaPrefix + round256(16 * (kNoAllocMaxPoints + 1));  // double[2 (nbins + 2)]
constexpr size_t kNaCounts = kNaOut + round256(16 * (kNoAllocMaxBins + 2));   // u64[nbins + 2]
constexpr size_t kNaMisc = kNaCounts + round256(8 * (kNoAllocMaxBins + 2));   // u64[8]
constexpr size_t kNoAllocBytes = kNaMisc + 256;                               // ~12.7 MB

// The scratch.  Host code must not pass this name to a kernel: on the host
// it stands for a host-side shadow, not for the device memory; the device
// address comes from cudaGetSymbolAddress (noalloc_scratch below).
static __device__ __align__(256) unsigned char g_brute_scratch[kNoAllocBytes];

// max |w * delta| and max |w| (as ordered bit patterns of non-negative
// doubles) and a flag for non-finite coordinates, weights or deltas
__global__ void k_brute_bounds(const float* pts, int n, unsigned long long* maxbits,
                               unsigned long long* bad) {
  double mwd = 0, mw = 0;
  bool nonfinite = false;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    const float* p = pts + 5 * (size_t)k;
    if (!isfinite(p[0]) || !isfinite(p[1]) || !isfinite(p[2]) || !isfinite(p[3]) || !isfinite(p[4]))
      nonfinite = true;
    mwd = fmax(mwd, fabs((double)p[4] * (double)p[3]));
    mw = fmax(mw, fabs((double)p[4]));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mwd = fmax(mwd, __shfl_xor_sync(kFull, mwd, o));
    mw = fmax(mw, __shfl_xor_sync(kFull, mw, o));
  }
  nonfinite = __any_sync(kFull, nonfinite);
  if ((threadIdx.x & 31) == 0) {
    atomicMax(&maxbits[0], (unsigned long long)__double_as_longlong(mwd));
    atomicMax(&maxbits[1], (unsigned long long)__double_as_longlong(mw));
    if (nonfinite) atomicOr(bad, 1ull);
  }
}

// interleaved (dsum, wsum) sums and counts -> the caller's three arrays
__global__ void k_brute_unpack(const double* out, const unsigned long long* cnt, int nb2, double* dsum,
                               double* wsum, uint64_t* counts) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < nb2; b += gridDim.x * blockDim.x) {
    dsum[b] = out[2 * b];
    wsum[b] = out[2 * b + 1];
    counts[b] = cnt[b];
  }
}

// Device address of g_brute_scratch on `device` (current): looked up once per
// device; the lookup may load the module on that device.
tos_status noalloc_scratch(int device, unsigned char** out) {
  static std::mutex mu;
  static std::vector<unsigned char*> addr;
  std::lock_guard<std::mutex> lock(mu);
  if ((size_t)device >= addr.size()) addr.resize(device + 1, nullptr);
  if (!addr[device]) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_brute_scratch);
    if (err != cudaSuccess || !p)
      return fail(TOS_ERR_CUDA, std::string("cudaGetSymbolAddress of the brute scratch: ") +
                                    cudaGetErrorString(err));
    addr[device] = (unsigned char*)p;
  }
  *out = addr[device];
  return TOS_OK;
}

}  // namespace
}  // namespace tos

extern "C" tos_status tos_brute_run_noalloc(tos_engine* e, const float* d_points, size_t n_points,
                                            double min, double max, int nbins, double* d_dsum,
                                            double* d_wsum, uint64_t* d_counts, double* ms_kernel) {
  if (!e || !d_points || !d_dsum || !d_wsum || !d_counts) return fail(TOS_ERR_INVALID_ARG, "null argument");
  if (n_points < 2) return fail(TOS_ERR_INVALID_ARG, "need at least 2 points");
  if (n_points > kNoAllocMaxPoints)
    return fail(TOS_ERR_INVALID_ARG, "tos_brute_run_noalloc takes at most " +
                                         std::to_string(kNoAllocMaxPoints) + " points (got " +
                                         std::to_string(n_points) + "); use tos_brute_run");
  if (nbins <= 0 || nbins > kNoAllocMaxBins)
    return fail(TOS_ERR_INVALID_ARG, "nbins must be in [1, " + std::to_string(kNoAllocMaxBins) + "]");
  if (!(max > min) || !std::isfinite(min) || !std::isfinite(max))
    return fail(TOS_ERR_INVALID_ARG, "need finite min < max");
  std::lock_guard<std::mutex> lock(e->mu);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(e->device);
  struct Restore {
    int d;
    ~Restore() { cudaSetDevice(d); }
  } restore{prev};
  unsigned char* S = nullptr;
  TOS_TRY(noalloc_scratch(e->device, &S));
  const int n = (int)n_points;
  const int nb2 = nbins + 2;
  cudaStream_t st = e->stream;
  float4* pos = (float4*)(S + kNaPos);
  double* wd = (double*)(S + kNaWd);
  double* w = (double*)(S + kNaW);
  double2* prefix = (double2*)(S + kNaPrefix);
  double* out = (double*)(S + kNaOut);
  unsigned long long* cnt = (unsigned long long*)(S + kNaCounts);
  unsigned long long* misc = (unsigned long long*)(S + kNaMisc);  // [0] chunk counter [1] rechecks
                                                                   // [2,3] bounds [4] non-finite
  // the scratch keeps the previous call's contents: clear what accumulates
  TOS_CUDA_TRY(cudaMemsetAsync(out, 0, (size_t)nb2 * 2 * sizeof(double), st));
  TOS_CUDA_TRY(cudaMemsetAsync(cnt, 0, (size_t)nb2 * sizeof(unsigned long long), st));
  TOS_CUDA_TRY(cudaMemsetAsync(misc, 0, 8 * sizeof(unsigned long long), st));
  k_brute_bounds<<<std::min(1024, (n + 255) / 256), 256, 0, st>>>(d_points, n, misc + 2, misc + 4);
  k_brute_prep<<<std::min(4096, (n + 255) / 256), 256, 0, st>>>(d_points, n, pos, wd, w);
  k_brute_scan<<<1, 1024, 0, st>>>(wd, w, n, prefix);
  TOS_CUDA_TRY(cudaGetLastError());
  unsigned long long hb[3] = {0, 0, 0};
  TOS_CUDA_TRY(cudaMemcpyAsync(hb, misc + 2, sizeof(hb), cudaMemcpyDeviceToHost, st));
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  if (hb[2]) return fail(TOS_ERR_INVALID_ARG, "points must be finite");
  double mwd, mw;
  std::memcpy(&mwd, &hb[0], 8);
  std::memcpy(&mw, &hb[1], 8);
  mwd = std::max(mwd, 1e-300);
  mw = std::max(mw, 1e-300);
  // the same kernel arguments as tos_brute_run, pointing into the scratch
  BruteArgs A{};
  A.pos = pos;
  A.prefix = prefix;
  A.wd = wd;
  A.w = w;
  A.n = n;
  A.nbins = nbins;
  A.min = min;
  A.max = max;
  A.spacing = (max - min) / nbins;
  A.invf = (float)(1.0 / A.spacing);
  A.offf = (float)(-min / A.spacing);
  A.nbf = (float)nbins;
  A.nbp1f = (float)nbins + 1.0f;
  int bl = 0;
  for (uint32_t v = (uint32_t)nbins + 2; v; v >>= 1) ++bl;
  A.k = std::max(0, std::min(13, 21 - bl));
  A.mag = std::ldexp(1.5f, 23 - A.k);
  std::memcpy(&A.bits, &A.mag, 4);
  const double per[2] = {mwd * kRunCap * mwd, mw * kRunCap * mw};
  for (int f = 0; f < 2; ++f) {
    const int F = (int)std::floor(38.0 - std::log2(per[f]));
    A.scale[f] = std::ldexp(1.0, F);
    A.inv_scale[f] = std::ldexp(1.0, -F);
  }
  A.out = out;
  A.counts = cnt;
  A.next = misc;
  A.counters = misc + 1;
  int warps = 0;
  size_t smem = 0;
  TOS_TRY(brute_shape(e, nbins, &warps, &smem));
  TOS_CUDA_TRY(cudaFuncSetAttribute(brute_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
  TOS_CUDA_TRY(cudaEventRecord(e->ev[4], st));
  brute_kernel<<<e->num_sms, warps * 32, smem, st>>>(A);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaEventRecord(e->ev[5], st));
  k_brute_unpack<<<(nb2 + 255) / 256, 256, 0, st>>>(out, cnt, nb2, d_dsum, d_wsum, d_counts);
  TOS_CUDA_TRY(cudaGetLastError());
  TOS_CUDA_TRY(cudaStreamSynchronize(st));
  if (ms_kernel) {
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev[4], e->ev[5]);
    *ms_kernel = ms;
  }
  return TOS_OK;
}
