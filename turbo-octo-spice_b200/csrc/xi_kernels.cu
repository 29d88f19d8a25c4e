// xi_kernels.cu — the persistent pixel-pair kernel (see xi_kernels.cuh).
#include "xi_kernels.cuh"
#include "xi_device.cuh"

namespace tos {

namespace {

// Per-row (lane) state of a chunk.
struct Row {
  float x1;     // distance (or loglam for observing coordinates)
  float d1, l1; // raw distance and loglam for the exact path
  float A1;     // Cartesian: d1 * a * inv1^2; Polar: d1 * a
  float dl1;    // float rounding of d1*d1 (scaled like A1), exact residual
  double wd1, w1, hl1;  // w*delta, w, 0.5*loglam
};

// Per-item constants shared by the warp.
struct Item {
  uint32_t i, j, ni, nj, cell;
  double c;
  float ap;          // 2(1-c) [* inv1^2 for Cartesian]
  uint32_t zb;       // constant z index of the item
  uint32_t sep;      // observing: theta index
  int zconst;        // z index constant over the item
  int lo1;           // Cartesian window: first axis-1 bin of the current chunk
  const float* colx; // padded column coordinate (distance or loglam) of sightline j
  const float* coll; // padded column loglam
  const float* cold; // padded column distance
  const double4* pre;// prefix sums of sightline j
};

// Window slot of a packed key (b0 << 16 | b1), or -1 when outside the window.
template <int COORD>
__device__ __forceinline__ int window_slot(const PairArgs& A, const Item& it, uint32_t key) {
  const int b0 = (int)(key >> 16), b1 = (int)(key & 0xFFFFu);
  if (COORD == kCart) {
    const int d = b1 - it.lo1;
    return (d >= 0 && d < A.win_w1) ? b0 * A.win_w1 + d : -1;
  } else if (COORD == kPolar) {
    return (A.g.n0 * A.g.n1 <= (uint32_t)A.win_slots) ? b0 * (int)A.g.n1 + b1 : -1;
  } else {
    return (b0 < A.win_slots) ? b0 : -1;
  }
}

// Flat reference index of a packed key with the item's z index (unsigned
// arithmetic as in XiEstimator.cc:196-201, 249-254, 283-288).
template <int COORD>
__device__ __forceinline__ uint32_t flat_index(const PairArgs& A, const Item& it, uint32_t key) {
  const uint32_t b0 = key >> 16, b1 = key & 0xFFFFu;
  uint32_t b = (COORD == kObs) ? it.sep + b0 * A.g.n1 : b1 + b0 * A.g.n1;
  return it.zb + b * A.g.n2;
}

__device__ __forceinline__ unsigned long long* acc_base(const PairArgs& A, uint32_t cell,
                                                        uint32_t idx) {
  return A.acc + ((size_t)cell * A.g.ntotal + idx) * kAccWords;
}

// Add one run's contribution directly to the global per-cell accumulator
// (keys outside the window, and the all-FP64 validation path).
__device__ void add_direct(const PairArgs& A, uint32_t cell, uint32_t idx, const double* c,
                           uint32_t m) {
  if (idx >= A.g.ntotal) {
    atomicAdd(&A.counters[2], (unsigned long long)m);
    return;
  }
  unsigned long long* base = acc_base(A, cell, idx);
#pragma unroll
  for (int k = 0; k < 7; ++k)
    add128(base + k, base + 7 + k,
           (k < kSigned || A.wide_all) ? to_fixed_wide(c[k], A.scale_hi[k])
                                       : to_fixed(c[k], A.scale[k]));
  red_add(base + 14, (unsigned long long)m);
  atomicAdd(&A.counters[3], 1ull);
}

// Add field k's split fixed-point words (sums over at most a window slot's
// contributions) to the global sums at base: signed fields carry
// lo + mid * 2^22 + hi * 2^44 (hi signed), positive fields lo + mid * 2^22.
__device__ __forceinline__ void add_words(unsigned long long* base, int k, uint32_t lo,
                                          uint32_t mid, uint32_t hi_bits) {
  __int128 v;
  if (k < kSigned)
    v = (__int128)(int)hi_bits * 17592186044416ll /* 2^44 */ + (__int128)((long long)mid << kSplit) +
        (__int128)lo;
  else
    v = (__int128)(((long long)(int)mid << kSplit) + (long long)lo);
  add_wide(base + k, base + 7 + k, v);
}

// Move the warp window into the global accumulators and clear it.
template <int COORD>
__device__ void flush_window(const PairArgs& A, const Item& it, uint32_t* win, int lane) {
  const int S = A.win_slots;
  int nslots = (COORD == kCart) ? (int)A.g.n0 * A.win_w1
               : (COORD == kPolar) ? (int)(A.g.n0 * A.g.n1)
                                   : (int)A.g.n0;
  if (nslots > S) nslots = S;
  for (int s = lane; s < nslots; s += 32) {
    const uint32_t contrib = win[kWordContrib * S + s];
    if (contrib == 0) continue;
    const uint32_t cnt = win[kWordCount * S + s];
    uint32_t key;
    if (COORD == kCart)
      key = ((uint32_t)(s / A.win_w1) << 16) | (uint32_t)(it.lo1 + s % A.win_w1);
    else if (COORD == kPolar)
      key = ((uint32_t)(s / (int)A.g.n1) << 16) | (uint32_t)(s % (int)A.g.n1);
    else
      key = (uint32_t)s << 16;
    const uint32_t idx = flat_index<COORD>(A, it, key);
    if (idx < A.g.ntotal) {
      unsigned long long* base = acc_base(A, it.cell, idx);
#pragma unroll
      for (int k = 0; k < 7; ++k)
        add_words(base, k, win[wword(k, 0) * S + s], win[wword(k, 1) * S + s],
                  k < kSigned ? win[wword(k, 2) * S + s] : 0u);
      red_add(base + 14, (unsigned long long)cnt);
    } else {
      atomicAdd(&A.counters[2], (unsigned long long)cnt);
    }
#pragma unroll
    for (int w = 0; w < kWinWords; ++w) win[w * S + s] = 0u;
  }
  if (lane == 0) atomicAdd(&A.counters[6], 1ull);
  __syncwarp();
}

// FP32 binning of one pixel pair.  key = packed (b0, b1) or kInvalidKey;
// recheck = the pair lies within 2^-K bins of a decision edge (or in a
// degenerate corner) and must be re-binned in FP64.
template <int COORD, bool EXACT0, bool MINPOS>
__device__ __forceinline__ void fast_bin(const PairArgs& A, const Row& R, float x2, uint32_t& key,
                                         bool& recheck) {
  float t0, t1;
  bool small = false;
  if (COORD == kCart) {
    const float s = __fsub_rn(x2, R.x1);
    t0 = __fmaf_rn(fabsf(s), A.inv0f, A.off0f);
    const float u = fabsf(__fmaf_rn(R.A1, x2, R.dl1));
    t1 = __fadd_rn(sqrt_approx(u), A.off1f);
  } else if (COORD == kPolar) {
    const float s = __fsub_rn(x2, R.x1);
    const float r2 = __fmaf_rn(s, s, __fmaf_rn(R.A1, x2, R.dl1));
    const float rs = rsqrt_approx(r2);
    t0 = __fmaf_rn(__fmul_rn(r2, rs), A.inv0f, A.off0f);
    t1 = __fmaf_rn(__fmul_rn(fabsf(s), rs), A.inv1f, A.off1f);
    small = !(r2 >= A.r2_small);
  } else {
    const float dl = fabsf(__fsub_rn(x2, R.x1));
    t0 = __fmaf_rn(dl, A.inv0f, A.off0f);
    t1 = 0.5f;
  }
  const int q0 = __float_as_int(__fadd_rz(t0, A.mag0)) - A.bits0;
  const int q1 = __float_as_int(__fadd_rz(t1, A.mag1)) - A.bits1;
  bool valid = (t0 < A.n0f) && (t1 < A.n1f);
  bool coarse = (t0 < A.n0p1f) && (t1 < A.n1p1f);
  if (MINPOS) {
    valid = valid && (t0 > -1.0f) && (t1 > -1.0f);
    coarse = coarse && (t0 > -2.0f) && (t1 > -2.0f);
  }
  int b0 = q0 >> A.k0, b1 = q1 >> A.k1;
  if (MINPOS) {
    b0 = max(b0, 0);
    b1 = max(b1, 0);
  }
  key = valid ? (((uint32_t)b0 << 16) | (uint32_t)b1) : kInvalidKey;
  bool edge = (((q1 + 1) & ((1 << A.k1) - 1)) < 2);
  if (COORD == kObs) edge = false;
  if (!EXACT0) edge = edge || (((q0 + 1) & ((1 << A.k0) - 1)) < 2);
  recheck = (coarse && edge) || small;
}

// Exact (FP64 reference) key of one pair.
template <int COORD>
__device__ __forceinline__ uint32_t exact_key(const PairArgs& A, const Row& R, const Item& it,
                                              float x2) {
  uint32_t b0 = 0, b1 = 0;
  bool ok;
  if (COORD == kCart)
    ok = exact_cart(R.d1, x2, it.c, A.g, &b0, &b1);
  else if (COORD == kPolar)
    ok = exact_polar(R.d1, x2, it.c, A.g, &b0, &b1);
  else
    ok = exact_obs(R.x1, x2, A.g, &b0);
  return ok ? ((b0 << 16) | b1) : kInvalidKey;
}

// Exact flat key including a per-pair z index (items whose z index varies).
template <int COORD>
__device__ __forceinline__ uint32_t exact_flat_key(const PairArgs& A, const Row& R, const Item& it,
                                                   float d2, float l2) {
  uint32_t idx = 0;
  bool ok;
  if (COORD == kCart)
    ok = ref_bin_cartesian(R.d1, R.l1, d2, l2, it.c, A.g, &idx);
  else if (COORD == kPolar)
    ok = ref_bin_polar(R.d1, R.l1, d2, l2, it.c, A.g, &idx);
  else
    ok = ref_bin_observing(R.l1, l2, it.sep, A.g, &idx);
  // kInvalidKey is reserved; an index equal to it can only be an overflow.
  return ok ? (idx == kInvalidKey ? kInvalidKey - 1u : idx) : kInvalidKey;
}

// Contribution of one closed run to the seven XiBin sums and the count.
struct Contrib {
  double c[7];
  uint32_t m;
};

__device__ __forceinline__ void make_contrib(const Row& R, uint32_t m, double dwd, double dw,
                                             double dl, Contrib& o) {
  const double md = (double)m;
  o.m = m;
  o.c[0] = R.wd1 * dwd;
  o.c[1] = R.wd1 * md;
  o.c[2] = dwd;
  o.c[3] = R.w1 * dw;
  o.c[4] = R.w1 * md;
  o.c[5] = dw;
  o.c[6] = __fma_rn(R.hl1, md, 0.5 * dl);
}

// Add the runs closed by lanes with `emit`: lanes that close a run with the
// same key are summed with redux.sync on the split fixed-point words and one
// of them adds the sums, to the warp window, or straight to the global
// accumulators for keys outside the window.  The fixed-point values are the
// same either way, so the integer totals do not depend on the grouping.
// Returns (warp-uniform) whether some slot reached its capacity.
template <int COORD>
__device__ __forceinline__ bool emit_runs(const PairArgs& A, const Item& it, uint32_t* win,
                                          int lane, bool emit, uint32_t key, const Contrib& ct) {
  int slot = -1;
  if (emit) slot = window_slot<COORD>(A, it, key);
  unsigned pending = __ballot_sync(kFull, emit);
  bool full = false;
  if (pending) {
    uint32_t wv[kWordCount];
    if (emit) {
#pragma unroll
      for (int k = 0; k < 7; ++k) {
        if (k < kSigned) {
          const long long q = to_fixed_wide(ct.c[k], A.scale_hi[k]);
          wv[wword(k, 0)] = (uint32_t)q & ((1u << kSplit) - 1u);
          wv[wword(k, 1)] = (uint32_t)(q >> kSplit) & ((1u << kSplit) - 1u);
          wv[wword(k, 2)] = (uint32_t)(int)(q >> (2 * kSplit));
        } else {
          const long long q = to_fixed(ct.c[k], A.scale[k]);
          wv[wword(k, 0)] = (uint32_t)q & ((1u << kSplit) - 1u);
          wv[wword(k, 1)] = (uint32_t)(int)(q >> kSplit);
        }
      }
    }
    const int S = A.win_slots;
    while (pending) {
      const int leader = __ffs(pending) - 1;
      const uint32_t lkey = __shfl_sync(kFull, key, leader);
      const unsigned peers = __ballot_sync(kFull, ((pending >> lane) & 1u) && key == lkey);
      if ((peers >> lane) & 1u) {
        const bool lead = lane == leader;
        if (slot >= 0) {  // the same for every peer: the slot is a function of the key
#pragma unroll
          for (int w = 0; w < kWordCount; ++w) {
            const uint32_t sw = __reduce_add_sync(peers, wv[w]);
            if (lead) atomicAdd(&win[w * S + slot], sw);
          }
          const uint32_t sm = __reduce_add_sync(peers, ct.m);
          if (lead) {
            atomicAdd(&win[kWordCount * S + slot], sm);
            const uint32_t n = (uint32_t)__popc(peers);
            const uint32_t old = atomicAdd(&win[kWordContrib * S + slot], n);
            full = old + n > kSlotCap;
          }
        } else {
          uint32_t sw[kWordCount];
#pragma unroll
          for (int w = 0; w < kWordCount; ++w) sw[w] = __reduce_add_sync(peers, wv[w]);
          const uint32_t sm = __reduce_add_sync(peers, ct.m);
          if (lead) {
            const uint32_t idx = flat_index<COORD>(A, it, lkey);
            if (idx < A.g.ntotal) {
              unsigned long long* base = acc_base(A, it.cell, idx);
#pragma unroll
              for (int k = 0; k < 7; ++k)
                add_words(base, k, sw[wword(k, 0)], sw[wword(k, 1)], k < kSigned ? sw[wword(k, 2)] : 0u);
              red_add(base + 14, (unsigned long long)sm);
              atomicAdd(&A.counters[3], 1ull);
            } else {
              atomicAdd(&A.counters[2], (unsigned long long)sm);
            }
          }
        }
      }
      pending &= ~peers;
    }
  }
  return __any_sync(kFull, full);
}

// Sweep one 32-row chunk.  MODE 0: fast path with packed keys and the warp
// window; MODE 1: every pair exact, flat keys, direct global adds.
template <int COORD, bool EXACT0, bool MINPOS, int MODE>
__device__ void sweep_chunk(const PairArgs& A, const Item& it, const Row& R, bool active,
                            int t_begin, int t_end, uint32_t* win, int lane,
                            unsigned long long& n_recheck) {
  uint32_t cur = kInvalidKey;
  int run_start = 0;
  double ps0 = 0, ps1 = 0, ps2 = 0;
  float x2n = it.colx[t_begin + lane];
  for (int t = t_begin; t < t_end; ++t) {
    const int p2 = t + lane;
    const float x2 = x2n;
    x2n = it.colx[p2 + 1];  // next step (p2 + 1 <= nj + 31: inside the padding)
    uint32_t key;
    if (MODE == 0) {
      bool recheck;
      fast_bin<COORD, EXACT0, MINPOS>(A, R, x2, key, recheck);
      if (__any_sync(kFull, recheck)) {
        if (recheck) {
          key = exact_key<COORD>(A, R, it, x2);
          ++n_recheck;
        }
      }
    } else {
      key = kInvalidKey;
      if (active && p2 >= 0 && p2 < (int)it.nj)
        key = exact_flat_key<COORD>(A, R, it, it.cold[p2], it.coll[p2]);
    }
    const bool changed = key != cur;
    if (__any_sync(kFull, changed)) {
      Contrib ct;
      bool emit = false;
      if (changed) {
        const int pc = min(max(p2, 0), (int)it.nj);
        const double4 pn = it.pre[pc];
        if (cur != kInvalidKey) {
          emit = true;
          make_contrib(R, (uint32_t)(p2 - run_start), pn.x - ps0, pn.y - ps1, pn.z - ps2, ct);
        }
        ps0 = pn.x;
        ps1 = pn.y;
        ps2 = pn.z;
      }
      if (MODE == 0) {
        if (emit_runs<COORD>(A, it, win, lane, emit, cur, ct)) flush_window<COORD>(A, it, win, lane);
      } else if (emit) {
        add_direct(A, it.cell, cur, ct.c, ct.m);
      }
      if (changed) {
        cur = key;
        run_start = p2;
      }
    }
  }
  // close runs still open at the end of the sweep
  Contrib ct;
  const bool emit = cur != kInvalidKey;
  if (emit) {
    const int p_end = t_end + lane;
    const double4 pn = it.pre[min(max(p_end, 0), (int)it.nj)];
    make_contrib(R, (uint32_t)(p_end - run_start), pn.x - ps0, pn.y - ps1, pn.z - ps2, ct);
  }
  if (MODE == 0) {
    emit_runs<COORD>(A, it, win, lane, emit, cur, ct);
    flush_window<COORD>(A, it, win, lane);
  } else if (emit) {
    add_direct(A, it.cell, cur, ct.c, ct.m);
  }
}

// Lower bound on the sorted padded column array: first p in [0, n) with
// pred(x[p]) true, pred monotone (false ... false true ... true).
template <class Pred>
__device__ __forceinline__ int lower_bound_pred(const float* x, int n, Pred pred) {
  int lo = 0, hi = n;
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (pred(x[mid]))
      hi = mid;
    else
      lo = mid + 1;
  }
  return lo;
}

template <int COORD, bool EXACT0, bool MINPOS, int MODE>
__device__ void process_item(const PairArgs& A, Item& it, uint32_t* win, int lane,
                             unsigned long long& n_eval, unsigned long long& n_recheck) {
  const uint64_t oi = A.off[it.i];
  const float* rowd = A.dist_pad + oi + (uint64_t)kPad * (it.i + 1);
  const float* rowl = A.loglam_pad + oi + (uint64_t)kPad * (it.i + 1);
  const double* rowwd = A.wd + oi;
  const float* roww = A.w + oi;
  const float4 rj = A.range[it.j];
  // Column window |x1 - x2| < lim.  For Polar binning a pair is accepted only
  // if r^2 = (d2 - d1)^2 + 2(1 - c) d1 d2 - err < R^2 (err: float rounding of
  // d1^2, XiEstimator.cc:179-184), and d1 d2 >= dmin_i dmin_j when both
  // sightlines' distances are positive, so the item's window narrows to
  // |d2 - d1| < sqrt(R^2 - 2(1 - c) dmin_i dmin_j + err bound).
  float lim = A.win_lim;
  if (COORD == kPolar && A.prune) {
    const float4 ri = A.range[it.i];
    if (ri.x > 0.f && rj.x > 0.f) {
      const double a = fmax(2.0 * (1.0 - it.c), 0.0);
      const double q = A.polar_r2 - a * (double)ri.x * (double)rj.x * (1.0 - 1e-6) + A.polar_e2;
      lim = fminf(lim, (float)(sqrt(fmax(q, 0.0)) * (1.0 + 1e-6) + 1e-3));
    }
  }
  for (uint32_t r0 = 0; r0 < it.ni; r0 += 32) {
    const uint32_t row = r0 + lane;
    const bool active = row < it.ni;
    Row R;
    if (active) {
      R.d1 = rowd[row];
      R.l1 = rowl[row];
      R.wd1 = rowwd[row];
      R.w1 = (double)roww[row];
      R.hl1 = 0.5 * (double)R.l1;
      R.x1 = (COORD == kObs) ? R.l1 : R.d1;
      const float p = __fmul_rn(R.d1, R.d1);
      const float e = __fmaf_rn(R.d1, R.d1, -p);  // d1*d1 = p + e exactly
      if (COORD == kCart) {
        R.A1 = __fmul_rn(R.d1, it.ap);
        R.dl1 = __fmul_rn(-e, A.inv1sqf);
      } else if (COORD == kPolar) {
        R.A1 = __fmul_rn(R.d1, it.ap);
        R.dl1 = -e;
      } else {
        R.A1 = 0.f;
        R.dl1 = 0.f;
      }
    } else {
      R.d1 = R.l1 = 0.f;
      R.wd1 = R.w1 = R.hl1 = 0.0;
      R.x1 = -kSentinel;
      R.A1 = 0.f;
      R.dl1 = 0.f;
    }
    // column window of this chunk
    int t_begin, t_end;
    if (A.prune) {
      int lo = (int)it.nj, hi = 0;
      if (active) {
        const float x1 = R.x1;
        lo = lower_bound_pred(it.colx, (int)it.nj, [&](float x2) { return __fsub_rn(x1, x2) < lim; });
        hi = lower_bound_pred(it.colx, (int)it.nj,
                              [&](float x2) { return x2 >= x1 && __fsub_rn(x2, x1) >= lim; });
      }
      int tb = active ? lo - lane : 0x7FFFFFFF;
      int te = active ? hi - lane : -0x7FFFFFFF;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        tb = min(tb, __shfl_xor_sync(kFull, tb, o));
        te = max(te, __shfl_xor_sync(kFull, te, o));
      }
      t_begin = tb;
      t_end = te;
    } else {
      t_begin = -31;
      t_end = (int)it.nj;
    }
    if (t_end <= t_begin) continue;
    if (active) {
      const int a = max(t_begin + (int)lane, 0), b = min(t_end + (int)lane, (int)it.nj);
      if (b > a) n_eval += (unsigned long long)(b - a);
    }
    if (COORD == kCart && MODE == 0) {
      // window along axis 1: lowest r_perp bin of the chunk, from its smallest
      // row distance (lane 0 when sorted) and the smallest column distance,
      // less the float rounding of d1*d1; keys below it go direct
      const float d1min = __shfl_sync(kFull, R.d1, 0);
      const float u = it.ap * d1min * rj.x * (1.f - 1e-5f) -
                      ldexpf(d1min * d1min * A.inv1sqf, -22);
      const int lo1 = (int)floorf(sqrtf(fmaxf(u, 0.f)) + A.off1f - 1e-2f);
      it.lo1 = max(0, min(lo1, (int)A.g.n1 - 1));
    }
    sweep_chunk<COORD, EXACT0, MINPOS, MODE>(A, it, R, active, t_begin, t_end, win, lane, n_recheck);
  }
}

template <int COORD, bool EXACT0, bool MINPOS>
__global__ void __launch_bounds__(kPairWarps * 32, 1) pair_kernel(PairArgs A) {
  extern __shared__ uint32_t smem[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* win = smem + (size_t)warp * kWinWords * A.win_slots;
  for (int k = lane; k < kWinWords * A.win_slots; k += 32) win[k] = 0u;
  __syncwarp();
  unsigned long long n_eval = 0, n_recheck = 0;
  for (;;) {
    unsigned long long base = 0;
    if (lane == 0) base = atomicAdd(A.next_item, (unsigned long long)kClaimItems);
    base = __shfl_sync(kFull, base, 0);
    if (base >= A.n_items) break;
    const unsigned long long mine = base + lane;
    unsigned todo = __ballot_sync(kFull, mine < A.n_items && item_owner(A, mine) == kOwnerPair);
    while (todo) {
      const unsigned long long idx = base + (__ffs(todo) - 1);
      todo &= todo - 1;
      Item it;
      it.i = A.item_i[idx];
      it.j = A.item_j[idx];
      it.c = A.item_c[idx];
      it.ni = A.npix[it.i];
      it.nj = A.npix[it.j];
      if (it.ni == 0 || it.nj == 0) continue;
      it.cell = dest_row(A, it.i, it.j);
      it.sep = (COORD == kObs) ? A.item_sep[idx] : 0u;
      const uint64_t oj = A.off[it.j] + (uint64_t)kPad * (it.j + 1);
      it.cold = A.dist_pad + oj;
      it.coll = A.loglam_pad + oj;
      it.colx = (COORD == kObs) ? it.coll : it.cold;
      it.pre = A.prefix + A.off[it.j] + it.j;
      const double a = 2.0 * dsub(1.0, it.c);
      it.ap = (COORD == kCart) ? (float)(a * A.g.inv1 * A.g.inv1) : (float)a;
      // z index: constant over the item when both ends of the loglam-sum range agree
      const float4 ri = A.range[it.i], rj = A.range[it.j];
      const float lsum_lo = __fadd_rn(ri.z, rj.z), lsum_hi = __fadd_rn(ri.w, rj.w);
      const double zlo = dmul(dsub(dmul(0.5, (double)lsum_lo), A.g.min2), A.g.invn2);
      const double zhi = dmul(dsub(dmul(0.5, (double)lsum_hi), A.g.min2), A.g.invn2);
      it.zb = zbin_of_sum(lsum_lo, A.g);
      const uint32_t zb_hi = zbin_of_sum(lsum_hi, A.g);
      it.zconst = (zlo > -1.0 && zhi < 2147483648.0 && it.zb == zb_hi) ? 1 : 0;
      it.lo1 = 0;
      if (A.run_split && run_item(A, it.c, it.zconst)) continue;  // run-sweep kernel's item
      if (diag_item(A, zlo, zhi, it.zb, zb_hi)) continue;          // diagonal-sweep kernel's item
      // with run_split or diag_split every field uses the wide fixed-point
      // scale, which only the direct (exact) path supports
      const bool exact_item = A.force_exact || !it.zconst || A.run_split || A.diag_split;
      if (exact_item)
        process_item<COORD, EXACT0, MINPOS, 1>(A, it, win, lane, n_eval, n_recheck);
      else
        process_item<COORD, EXACT0, MINPOS, 0>(A, it, win, lane, n_eval, n_recheck);
    }
  }
  // counters
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    n_eval += __shfl_xor_sync(kFull, n_eval, o);
    n_recheck += __shfl_xor_sync(kFull, n_recheck, o);
  }
  if (lane == 0) {
    atomicAdd(&A.counters[0], n_eval);
    atomicAdd(&A.counters[1], n_recheck);
  }
}

template <int COORD, bool EXACT0, bool MINPOS>
cudaError_t launch3(const PairArgs& a, int grid, cudaStream_t stream) {
  const size_t smem = pair_kernel_smem(a.win_slots);
  auto k = pair_kernel<COORD, EXACT0, MINPOS>;
  cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  k<<<grid, kPairWarps * 32, smem, stream>>>(a);
  return cudaGetLastError();
}

template <int COORD>
cudaError_t launch2(const PairArgs& a, bool exact0, bool minpos, int grid, cudaStream_t stream) {
  if (exact0)
    return minpos ? launch3<COORD, true, true>(a, grid, stream)
                  : launch3<COORD, true, false>(a, grid, stream);
  return minpos ? launch3<COORD, false, true>(a, grid, stream)
                : launch3<COORD, false, false>(a, grid, stream);
}

}  // namespace

size_t pair_kernel_smem(int win_slots) {
  return (size_t)kPairWarps * kWinWords * (size_t)win_slots * sizeof(uint32_t);
}

cudaError_t launch_pair_kernel(const PairArgs& a, int coord, bool exact0, bool minpos, int grid,
                               cudaStream_t stream) {
  switch (coord) {
    case TOS_CARTESIAN: return launch2<kCart>(a, exact0, minpos, grid, stream);
    case TOS_POLAR: return launch2<kPolar>(a, exact0, minpos, grid, stream);
    default: return launch2<kObs>(a, exact0, minpos, grid, stream);
  }
}

}  // namespace tos
