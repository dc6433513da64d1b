// TLS period search kernels for sm_100a.
//
// Per trial period the reference (src/gputls/core.py:770-875 with the kernels
// of src/gputls/GPUFun.py) folds the light curve, sorts it by phase, pads the
// sorted flux with its first maxD samples, and evaluates for every duration d
// and phase start k the template chi2
//
//   chi2(d,k) = sum_{i<w} (y_{k+i} - 1 + s_i c)^2 w_{k+i}          (in transit)
//             + sum over the other samples of (1 - y)^2 w            (out of transit)
//             - edge correction (the wrapped tail)                  (GPUFun.py:425-434)
//
// with c = 2 * overshoot_d * mean depth of the window.  Written in terms of
// v = y - 1, u = v w and the baseline E = sum_{i<n} v_i^2 w_i (a constant of
// the light curve: the reference's E[M-1] - edge), this is exactly
//
//   chi2(d,k) = E + c (2 B_k + c C_k),  B_k = sum_i s_i u_{k+i},  C_k = sum_i s_i^2 w_{k+i}
//
// which is what these kernels evaluate.  B and C are sliding correlations of
// the template with the folded (u, w) records; the work is FMA-bound and runs
// on the FP64 or FP32 pipes (nothing here is a dense contraction, so no tensor
// cores).  The mean depth comes from prefix sums of v (FP64; stored as
// float-float pairs in the FP32 form).  Only starts k that are multiples of
// skip(d) = w / skip_point (for w > skip_point) are evaluated in the main pass
// (GPUFun.py:402,409); every other (d,k) carries the value n
// (GPUFun.py:407,437), which takes part in the minimum like any value.
//
// Kernels:
//   curve_setup_kernel   (v, w) records per original sample and E.
//   prepare_kernel       one CTA per period: FP64 fold (GPUFun.py:30-41),
//                        stable bucket ranking of the phases (cupy argsort),
//                        each ranked sample written straight to its place in
//                        the padded sorted record array (patchData
//                        GPUFun.py:110-129), then the prefix of v.
//   chi2_kernel          one CTA per (period, tile of starts): the tile of
//                        records is staged in shared memory, warps pull
//                        (duration, start-group) tasks from a CTA-local queue,
//                        register-blocked correlations produce B, C for R
//                        starts at a time, each CTA keeps its (min, argmin).
//   finish_kernel        per-period minimum over tiles (first occurrence).
#include <cuda_runtime.h>

#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include "chi2_core.cuh"
#include "common.cuh"
#include "tma.cuh"

namespace gtls {

constexpr int kPrepThreads = 1024;
constexpr int kPrepThreadsSmall = 512;   // curves of at most kPrepSmallMaxN samples: two CTAs per SM
constexpr int kPrepSmallMaxN = 1 << 15;
constexpr int kSmallBucket = 8;     // entries of buckets up to this size are ranked by their own thread
constexpr int kSmallBucketSm = 32;  // the same, for buckets in shared memory
constexpr int kBigBuckets = 512;    // capacity of the list of larger buckets (warp-ranked)
constexpr int kMaxRounds = 32;      // rounds of the shared-memory prepare path
constexpr int kRoundShift = 20;     // hist entries of that path: position | round << kRoundShift
constexpr int kPosMask = (1 << kRoundShift) - 1;
constexpr int kPrepStaticSmem = 4096;  // static shared memory of prepare_kernel, rounded up
constexpr int kChiThreads = 512;
constexpr int kSplitMinSkip = 32;  // skip >= this: lanes split the block offset rho
// Split-path task: a window of kWin consecutive starts of one duration.  Its
// starts are first put through the depth test; the starts that pass are then
// covered by groups of kR consecutive starts (each beginning at the first
// uncovered start that passes), and only those groups are correlated.
constexpr int kWin = 6 * kR;
// All-starts pass, lane-path task of a width of at least kLaneGateMinW: a
// window of 32 * kLaneG groups of kR consecutive starts; the groups whose
// starts all fail the depth test are dropped and the others are dealt out to
// the lanes round by round.  (For shorter widths, and for the main pass's
// lane-path widths, measured: a group's sums cost about what its depth tests
// do, and the task is the plain 32 groups.)
constexpr int kLaneG = 6;            // (2 and 4 measured slower)
constexpr int kLaneGateMinW = 64;
// Zeroed records after each shared-memory tile: a skip-1 group whose kR
// starts all lie in the tile reads at most kR - 2 records past it (only ever
// against zero template entries), so those groups need no clamping.
constexpr int kTilePad = 16;

// float-float helpers (Knuth two-sum; no multiplications, so no contraction)
__device__ __forceinline__ float2 ff_add(float2 a, float2 b) {
  float s = a.x + b.x;
  float bb = s - a.x;
  float e = (a.x - (s - bb)) + (b.x - bb);
  e += a.y + b.y;
  float hi = s + e;
  return make_float2(hi, e - (hi - s));
}
__device__ __forceinline__ float2 ff_from_double(double v) {
  float hi = (float)v;
  return make_float2(hi, (float)(v - (double)hi));
}
// Store prefix value v at pre[r] through the FP64 view of the prefix array:
// as a double (FP64 form) or as the float-float pair (hi, lo) occupying the
// same 8 bytes (FP32 form; hi at the lower address).  Streaming stores: the
// chi2 kernel reads them back only after the whole chunk is prepared.
template <typename Real>
__device__ __forceinline__ void store_prefix(double* pre, int r, double v) {
  if constexpr (sizeof(Real) == 8) {
    __stcs(pre + r, v);
  } else {
    const float2 f = ff_from_double(v);
    const unsigned long long bits = ((unsigned long long)__float_as_uint(f.y) << 32) | __float_as_uint(f.x);
    __stcs(pre + r, __longlong_as_double((long long)bits));
  }
}

// ------------------------------------------------------------ descriptors
// Per-light-curve parameters and buffers on the device.  A search covers one
// or many light curves; every kernel finds its curve through these.
template <typename Real>
struct CurveDev {
  const double* t;              // [n] times
  const double* y;              // [n] flux
  const double* dy;             // [n] uncertainties
  const double* periods;        // [np] this curve's trial periods
  double* chi2_out;             // [np]
  int64_t* loc_out;             // [np] or NULL
  double2* vw;                  // [n] (v, w) per original sample (scratch)
  double* ebase;                // sum v^2 w (scratch)
  int* wmin;                    // [np] duration range (scratch)
  int* wmax;
  const int* widths;            // [D]
  const double* overshoot;      // [D]
  const double* templates;      // [D * max_width]
  const int* skips;             // [D]
  const int* trow_off;          // [D] offsets into trows
  const int* trow_len;          // [D]
  typename Tr<Real>::R2* trows; // template rows (s, s^2), zero-padded
  int* union_cnt;               // [nbatch]
  int* union_list;              // [nbatch * D] ascending duration indices
  short* cost_order;            // [nbatch * D] positions in union_list, longest task first
  long long np;
  int n, maxd, M, Mrec, D, max_width, batch, nbatch;
  int tile, ntiles, nb_log2;
  int rnb_log2, rcap;           // shared-memory prepare path: bucket bits and round capacity (0: off)
  int global_rec;               // 1: chi2 reads the records from global memory (no shared tile)
  int maxd_l;                   // > 0 (global records, main pass): the lane path's records, the tile
                                // plus this halo (its longest width), are staged in shared memory
  float span;
};

// A run: consecutive periods of one curve inside a chunk of the period list,
// with the offsets of their scratch rows.  Chunk items and chi2 CTAs are
// numbered run after run.
struct Run {
  int curve;
  int item0;          // first item (period) of the run in its chunk
  int count;          // periods in the run
  int tile0;          // first chi2 CTA of the run in its chunk
  long long pidx0;    // index of the run's first period within its curve
  long long slot_off; // element offsets of the run's first row in each scratch array
  long long rec_off;
  long long pv_off;
  long long part_off;
};

// Largest i in [lo, hi) with key(i) <= x (keys ascending, key(lo) <= x).
template <typename F>
__device__ __forceinline__ int upper_find(int lo, int hi, long long x, F key) {
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (key(mid) <= x) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ------------------------------------------------------------ curve set-up
// (v, w) per original sample: v = y - 1 (exact), w = 1/(dy*dy)
// (calcInverseSquaredPatchedDy GPUFun.py:134-142), and E = sum v^2 w
// (calculate_base_error GPUFun.py:293-312 summed over the n samples).
template <typename Real>
__global__ void __launch_bounds__(1024) curve_setup_kernel(const CurveDev<Real>* __restrict__ cds) {
  __shared__ double red[1024];
  const CurveDev<Real>& C = cds[blockIdx.x];
  const double* __restrict__ y = C.y;
  const double* __restrict__ dy = C.dy;
  double2* __restrict__ vw = C.vw;
  const int n = C.n;
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    double v = y[i] - 1.0;
    double d = dy[i];
    double w = 1.0 / (d * d);
    vw[i] = make_double2(v, w);
    double diff = 1.0 - y[i];
    acc += diff * diff * w;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) *C.ebase = red[0];
}

// ------------------------------------------------------------ block scans
// Exclusive scan of an int array in shared memory, in place; returns the
// total.  Warp w owns the contiguous range [w*per, (w+1)*per) and walks it 32
// consecutive entries at a time, so that lanes never share a bank.
__device__ int block_exclusive_scan_smem(int* a, int len, int* warp_tmp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int per = ((len + nw - 1) / nw + 31) & ~31;
  const int beg = min(len, wid * per), end = min(len, beg + per);
  int sum = 0;
  for (int i = beg + lane; i < end; i += 32) sum += a[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if (lane == 0) warp_tmp[wid] = sum;
  __syncthreads();
  int carry = lane < wid ? warp_tmp[lane] : 0;
  int total = lane < nw ? warp_tmp[lane] : 0;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    carry += __shfl_xor_sync(0xffffffffu, carry, o);
    total += __shfl_xor_sync(0xffffffffu, total, o);
  }
  for (int i0 = beg; i0 < end; i0 += 32) {
    const int i = i0 + lane;
    const int x = i < end ? a[i] : 0;
    int inc = x;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int yv = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += yv;
    }
    if (i < end) a[i] = carry + inc - x;
    carry += __shfl_sync(0xffffffffu, inc, 31);
  }
  __syncthreads();
  return total;
}

// ---------------------------------------------------------------- prepare
// Phase of sample t for period P: t/P minus its truncation, as foldFast
// (GPUFun.py:38-39) computes it (IEEE division, int truncation).
__device__ __forceinline__ double fold_phase(double t, double P) {
  double x = __ddiv_rn(t, P);
  return x - (double)(int)x;
}

// Bucket of a phase from x = phase * NB (exact: NB = scale is a power of
// two, and |phase| < 1): floor(x), clamped so that out-of-range phases land
// in the first or last bucket.
__device__ __forceinline__ int phase_bin(double x, int nb) {
  int b = (int)x;
  b = b < 0 ? 0 : b;
  return b >= nb ? nb - 1 : b;
}

// Strict order of two slots of the same bucket: by phase, then by original
// index (the order of a stable argsort).  The 32-bit keys are the in-bucket
// fractions rounded to float, which preserves every strict inequality; equal
// keys are decided on the exact FP64 phases, recomputed.
// Slot index words hold the sample index, and for curves of at most
// kPackedMaxN samples also the bucket in the bits above it (the same for two
// slots of one bucket, so comparing whole words compares the indices).
constexpr int kPackedShift = 17;
constexpr int kPackedMaxN = 1 << kPackedShift;
__device__ __forceinline__ bool slot_less(uint2 a, uint2 b, const double* __restrict__ t, double P, unsigned imask) {
  const float fa = __uint_as_float(a.x), fb = __uint_as_float(b.x);
  if (fa != fb) return fa < fb;
  const double pa = fold_phase(t[a.y & imask], P), pb = fold_phase(t[b.y & imask], P);
  if (pa != pb) return pa < pb;
  return a.y < b.y;
}

// Rank of every entry of bucket slots [s, e) among the bucket (emit(s + rank,
// original index)), by a whole warp: each lane ranks one entry of a group of
// 32 against the bucket, streamed 32 entries at a time and broadcast by
// shuffles.  Used for large buckets, whose O(k^2) comparisons would
// otherwise fall on single threads.
template <typename Emit>
__device__ __forceinline__ void rank_bucket_warp(const uint2* __restrict__ slot, int s, int e,
                                                 const double* __restrict__ t, double P, unsigned imask, Emit emit) {
  const int lane = threadIdx.x & 31;
  for (int j0 = s; j0 < e; j0 += 32) {
    const int j = j0 + lane;
    const uint2 mine = slot[min(j, e - 1)];
    int r = 0;
    for (int m0 = s; m0 < e; m0 += 32) {
      const uint2 oth = slot[min(m0 + lane, e - 1)];
      const int cnt = min(32, e - m0);
      for (int q = 0; q < cnt; ++q) {
        uint2 o;
        o.x = __shfl_sync(0xffffffffu, oth.x, q);
        o.y = __shfl_sync(0xffffffffu, oth.y, q);
        if (o.y != mine.y && slot_less(o, mine, t, P, imask)) ++r;
      }
    }
    if (j < e) emit(s + r, (int)(mine.y & imask));
  }
}

// Prefix of v in place over pre[1..M], accumulated in FP64 for both forms
// (the FP32 form then stores each prefix as a float-float pair (hi, lo) in
// the same 8 bytes): each warp scans a contiguous range (coalesced), then
// adds the sum of the ranges before it.  pre[0] = 0.  wsum: 32 doubles.
template <typename Real>
__device__ void prefix_of_v(double* pre_d, int M, double* wsum) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int per = (M + nwarp - 1) / nwarp;
  const int beg = 1 + min(M, wid * per);
  const int end = 1 + min(M, (wid + 1) * per);
  double acc = 0.0;
  for (int r = beg + lane; r < end; r += 32) acc += pre_d[r];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) wsum[wid] = acc;
  __syncthreads();
  double carry = 0.0;
  for (int w = 0; w < wid; ++w) carry += wsum[w];
  if (wid == 0 && lane == 0) store_prefix<Real>(pre_d, 0, 0.0);
  for (int r0 = beg; r0 < end; r0 += 32) {
    const int r = r0 + lane;
    double x = r < end ? pre_d[r] : 0.0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const double yv = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += yv;
    }
    if (r < end) store_prefix<Real>(pre_d, r, carry + x);
    carry += __shfl_sync(0xffffffffu, x, 31);
  }
}

// Prefix value at pre[r] as a double (the inverse of store_prefix; in the
// FP32 form the float-float pair is summed back in FP64).
template <typename Real>
__device__ __forceinline__ double load_prefix(const double* pre, int r) {
  if constexpr (sizeof(Real) == 8) {
    return pre[r];
  } else {
    const unsigned long long bits = (unsigned long long)__double_as_longlong(pre[r]);
    return (double)__uint_as_float((unsigned)bits) + (double)__uint_as_float((unsigned)(bits >> 32));
  }
}

// Inclusive prefix of src[0, cnt) (shared memory, FP64) plus carry0, stored
// at pre[dst0 + q] for q < cnt; returns, in every thread, the last stored
// value (carry0 when cnt == 0).  Thread i sums its own chunk of K
// consecutive entries (K odd, so that the lanes' strided reads fall in
// distinct banks), the chunk sums are scanned across the block (shuffles,
// then the warp totals), each thread rewrites its chunk in place as the
// running prefix, and the block stores the result coalesced.  wsum: 32
// doubles.  Ends with a barrier, after which src may be overwritten.
template <typename Real>
__device__ double scan_store(double* src, int cnt, double carry0, double* pre_d, int dst0, double* wsum) {
  if (cnt <= 0) return carry0;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int K = ((cnt + blockDim.x - 1) / blockDim.x) | 1;
  const int beg = min(cnt, (int)threadIdx.x * K), end = min(cnt, beg + K);
  double acc = 0.0;
  for (int r = beg; r < end; ++r) acc += src[r];
  // exclusive prefix of the chunk sums: within the warp, then over the warps
  double inc = acc;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const double yv = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += yv;
  }
  if (lane == 31) wsum[wid] = inc;
  __syncthreads();
  double exc = __shfl_up_sync(0xffffffffu, inc, 1);
  double run = carry0;
  for (int w = 0; w < wid; ++w) run += wsum[w];
  if (lane > 0) run += exc;
  for (int r = beg; r < end; ++r) {
    run += src[r];
    src[r] = run;
  }
  __syncthreads();
  for (int q = threadIdx.x; q < cnt; q += blockDim.x) store_prefix<Real>(pre_d, dst0 + q, src[q]);
  const double last = src[cnt - 1];
  __syncthreads();
  return last;
}

// Round tables of the shared-memory prepare path.
struct RoundTables {
  int nrounds;               // rounds; -1: the period takes the global-scatter path
  int rb[kMaxRounds + 1];    // first bucket of each round (rb[nrounds] = NB)
  int rpos[kMaxRounds + 1];  // first sorted position of each round (rpos[nrounds] = n)
  int cursor[kMaxRounds];    // append cursors of the round-partitioned sample words
};

// Shared-memory prepare of one period (curves of at most kPackedMaxN
// samples).  The samples are folded (GPUFun.py:30-41) and counted into NB
// phase buckets; the buckets are cut greedily into rounds of whole buckets
// holding at most `cap` samples each; a second fold appends each sample's
// word (in-bucket key, index | bucket << kPackedShift) to its round's range
// of the scratch row `stage` (warp-aggregated, so the stores stay nearly
// coalesced).  Each round then
//   (a) reads its words (coalesced) into shared-memory slots by bucket,
//   (b) ranks every slot within its bucket (the stable argsort order of
//       the fold, as slot_less defines it) and writes the record of the
//       resulting sorted position (close to the slot's, so nearly
//       coalesced), with its v into shared memory, and
//   (c) stores the FP64 prefix of v over its positions,
// so that nothing is scattered through global memory.  Afterwards the
// wrapped copy of the first maxd positions (patchData, GPUFun.py:110-129)
// gets its prefix from pre[n] + pre[q + 1].  Returns false, having written
// nothing, when a single bucket holds more than `cap` samples or more than
// kMaxRounds rounds would be needed; the caller then takes the global path.
// Dynamic shared memory: hist [NB] ints, slots [cap] words, vbuf [cap]
// doubles.
template <typename Real, bool kOrder>
__device__ __noinline__ bool prepare_rounds(int* dyn, int* wtmp_i, double* wsum, int* big, int* nbig, RoundTables& rt,
                               const double* __restrict__ t, const double2* __restrict__ vw, int n, int maxd,
                               double P, int nb_log2, int cap, uint2* __restrict__ stage,
                               typename Tr<Real>::R2* __restrict__ out, double* __restrict__ pre_d,
                               int* __restrict__ ord) {
  using R2 = typename Tr<Real>::R2;
  const int nb = 1 << nb_log2;
  const double scale = (double)nb;
  constexpr unsigned imask = (unsigned)(kPackedMaxN - 1);
  int* hist = dyn;
  uint2* slots = reinterpret_cast<uint2*>(dyn + nb);
  double* vbuf = reinterpret_cast<double*>(slots + cap);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  constexpr int kB = 2;   // elements per thread in flight in each pass (4 and 8 measured slower)
  const int stride = blockDim.x * kB;

  for (int b = threadIdx.x; b < nb; b += blockDim.x) hist[b] = 0;
  __syncthreads();
  // (1) fold and histogram of buckets
  for (int i0 = threadIdx.x; i0 < n; i0 += stride) {
    double tv[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      tv[u] = i < n ? t[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) atomicAdd(&hist[phase_bin(fold_phase(tv[u], P) * scale, nb)], 1);
    }
  }
  __syncthreads();
  block_exclusive_scan_smem(hist, nb, wtmp_i);   // hist[b]: first position of bucket b
  // (2) rounds, by warp 0: from bucket b0, the largest b1 with
  //     start(b1) <= start(b0) + cap (a 32-way search of the bucket starts)
  if (wid == 0) {
    auto S = [&](int x) { return x < nb ? hist[x] : n; };
    int r = 0, b0 = 0;
    bool ok = true;
    if (lane == 0) {
      rt.rb[0] = 0;
      rt.rpos[0] = 0;
    }
    while (b0 < nb) {
      const int lim = S(b0) + cap;
      int lo = b0, hi = nb;   // S(lo) <= lim; the answer lies in [lo, hi]
      while (lo < hi) {
        const int step = (hi - lo + 31) >> 5;
        const int x = min(hi, lo + (lane + 1) * step);
        const int c = __popc(__ballot_sync(0xffffffffu, S(x) <= lim));   // a prefix of the lanes
        const int nlo = min(hi, lo + c * step);
        const int nhi = c == 32 ? hi : min(hi, lo + (c + 1) * step) - 1;
        lo = nlo;
        hi = nhi;
      }
      if (lo == b0 || r == kMaxRounds) {   // bucket b0 alone exceeds cap, or too many rounds
        ok = false;
        break;
      }
      if (lane == 0) {
        rt.cursor[r] = S(b0);
        rt.rb[r + 1] = lo;
        rt.rpos[r + 1] = S(lo);
      }
      ++r;
      b0 = lo;
    }
    if (lane == 0) rt.nrounds = ok ? r : -1;
  }
  __syncthreads();
  const int nr = rt.nrounds;
  if (nr < 0) return false;
  // each bucket's round in the bits of hist above the positions
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    hist[b] |= upper_find(0, nr, b, [&](int q) { return (long long)rt.rb[q]; }) << kRoundShift;
  auto H = [&](int b) { return hist[b] & kPosMask; };
  __syncthreads();
  // (3) fold again; each sample's word to its round's range of the scratch
  //     row (the loop runs over whole warps for the warp-wide match)
  for (int i0 = threadIdx.x - lane; i0 < n; i0 += stride) {
    double tv[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + lane + u * blockDim.x;
      tv[u] = i < n ? t[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + lane + u * blockDim.x;
      int r = -1;
      uint2 wd = make_uint2(0u, 0u);
      if (i < n) {
        const double x = fold_phase(tv[u], P) * scale;
        const int b = phase_bin(x, nb);
        wd = make_uint2(__float_as_uint((float)(x - (double)b)), (unsigned)i | ((unsigned)b << kPackedShift));
        r = hist[b] >> kRoundShift;
      }
      const unsigned peers = __match_any_sync(0xffffffffu, r);
      const int leader = __ffs(peers) - 1;
      int pos = 0;
      if (lane == leader && r >= 0) pos = atomicAdd(&rt.cursor[r], __popc(peers));
      pos = __shfl_sync(0xffffffffu, pos, leader) + __popc(peers & ((1u << lane) - 1u));
      if (r >= 0 && pos < rt.rpos[r + 1]) stage[pos] = wd;   // always true: the counts of pass (1)
    }
  }
  __syncthreads();
  double carry = 0.0;   // prefix of v up to the current round (FP64)
  for (int r = 0; r < nr; ++r) {
    const int rs = rt.rpos[r], cnt = rt.rpos[r + 1] - rs;
    const int b0 = rt.rb[r], b1 = rt.rb[r + 1];
    // (a) the round's words into slots by bucket; afterwards the position
    //     H(b) is the end of bucket b and H(b - 1) its start (for the round's
    //     first bucket that is the end of the previous round's last one, rs)
    for (int q0 = threadIdx.x; q0 < cnt; q0 += stride) {
      uint2 wd[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int q = q0 + u * blockDim.x;
        wd[u] = q < cnt ? stage[rs + q] : make_uint2(0u, 0u);
      }
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int q = q0 + u * blockDim.x;
        if (q < cnt) {
          const int b = (int)(wd[u].y >> kPackedShift);
          const int sl = (atomicAdd(&hist[b], 1) & kPosMask) - rs;
          if ((unsigned)sl < (unsigned)cnt) slots[sl] = wd[u];   // always true: the counts of pass (1)
        }
      }
    }
    if (threadIdx.x == 0) *nbig = 0;
    __syncthreads();
    // the scratch lines read so far, whole 128-byte lines inside this
    // period's row, are dropped from L2 without being written back
    {
      const uintptr_t row0 = ((uintptr_t)stage + 127) & ~(uintptr_t)127;
      const uintptr_t lo = max(row0, (uintptr_t)(stage + rs) & ~(uintptr_t)127);
      const uintptr_t hi = (uintptr_t)(stage + rs + cnt) & ~(uintptr_t)127;
      for (uintptr_t a = lo + (uintptr_t)threadIdx.x * 128; a < hi; a += (uintptr_t)blockDim.x * 128)
        asm volatile("discard.global.L2 [%0], 128;" ::"l"(a) : "memory");
    }
    // (b) ranks, and the records at once: the entry of sorted position p
    //     (round-local q = p - rs) and original sample i gets its record
    //     (u, w) at p (and at p + n when p < maxd: the wrap of patchData,
    //     GPUFun.py:110-129) and its v at vbuf[q]; i is clamped so that a
    //     malformed input can never address outside the curve.  Buckets of
    //     more than kSmallBucketSm entries are listed and ranked by whole warps
    //     (unless the list overflows); every other slot by its own thread.
    for (int b = b0 + (int)threadIdx.x; b < b1; b += blockDim.x) {
      const int k = H(b) - (b == 0 ? 0 : H(b - 1));
      if (k > kSmallBucketSm) {
        const int q = atomicAdd(nbig, 1);
        if (q < kBigBuckets) big[q] = b;
      }
    }
    __syncthreads();
    const int nbg = *nbig;
    const bool warp_ranked = nbg <= kBigBuckets;
    auto emit = [&](int q, int i) {
      i = min(max(i, 0), n - 1);
      const int p = rs + q;
      if constexpr (kOrder) {
        ord[p] = i;
        return;
      }
      const double2 g = vw[i];
      R2 o;
      o.x = (Real)(g.x * g.y);
      o.y = (Real)g.y;
      __stcs(out + p, o);
      if (p < maxd) __stcs(out + p + n, o);
      vbuf[q] = g.x;
    };
    if (warp_ranked)
      for (int q = wid; q < nbg; q += nwarp) {
        const int b = big[q];
        rank_bucket_warp(slots, (b == 0 ? 0 : H(b - 1)) - rs, H(b) - rs, t, P, imask, emit);
      }
    for (int j0 = threadIdx.x; j0 < cnt; j0 += stride) {
      int pos[kB], idx[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) {
        const int j = j0 + u * blockDim.x;
        pos[u] = -1;
        idx[u] = 0;
        if (j < cnt) {
          const uint2 sj = slots[j];
          const int b = (int)(sj.y >> kPackedShift);
          const int s = (b == 0 ? 0 : H(b - 1)) - rs;
          const int e = H(b) - rs;
          idx[u] = (int)(sj.y & imask);
          if (e - s == 1) {
            pos[u] = j;
          } else if (e - s <= kSmallBucketSm || !warp_ranked) {
            // entries of smaller key, and of equal key (itself included);
            // equal keys, rare, are then ordered on the exact phases
            const float kj = __uint_as_float(sj.x);
            int lt = 0, eq = 0;
#pragma unroll 4
            for (int m = s; m < e; ++m) {
              const float km = __uint_as_float(slots[m].x);
              lt += km < kj;
              eq += km == kj;
            }
            if (eq > 1)
              for (int m = s; m < e; ++m)
                if (m != j && __uint_as_float(slots[m].x) == kj) lt += slot_less(slots[m], sj, t, P, imask);
            pos[u] = s + lt;
          }
        }
      }
      // the gathers of the kB entries in flight together
      if constexpr (kOrder) {
#pragma unroll
        for (int u = 0; u < kB; ++u)
          if (pos[u] >= 0) emit(pos[u], idx[u]);
      } else {
        double2 g[kB];
#pragma unroll
        for (int u = 0; u < kB; ++u) g[u] = pos[u] >= 0 ? vw[min(max(idx[u], 0), n - 1)] : make_double2(0.0, 0.0);
#pragma unroll
        for (int u = 0; u < kB; ++u) {
          if (pos[u] >= 0) {
            const int p = rs + pos[u];
            R2 o;
            o.x = (Real)(g[u].x * g[u].y);
            o.y = (Real)g[u].y;
            __stcs(out + p, o);
            if (p < maxd) __stcs(out + p + n, o);
            vbuf[pos[u]] = g[u].x;
          }
        }
      }
    }
    __syncthreads();
    // (c) pre[rs + q + 1] = carry + v[0..q] (ends with a barrier)
    if constexpr (!kOrder) carry = scan_store<Real>(vbuf, cnt, carry, pre_d, rs + 1, wsum);
  }
  if constexpr (!kOrder) {
    // pre[0] = 0, and the wrapped copy: pre[n + 1 + q] = pre[n] + pre[q + 1]
    if (threadIdx.x == 0) store_prefix<Real>(pre_d, 0, 0.0);
    const int nw = min(maxd, n);
    for (int q = threadIdx.x; q < nw; q += blockDim.x)
      store_prefix<Real>(pre_d, n + 1 + q, carry + load_prefix<Real>(pre_d, q + 1));
  }
  return true;
}

// kOrder: write only the stable fold order of each period (order_out[rec_off
// + local * n + p] = original index of sorted position p) instead of the
// records and prefix (gtls_fold_order).  kThreads: kPrepThreads (one CTA per
// SM), or kPrepThreadsSmall for curves of at most kPrepSmallMaxN samples
// (two CTAs per SM, each with half the shared memory: the barriers of one
// overlap the other's work, which pays on short curves).
template <typename Real, bool kOrder = false, int kThreads = kPrepThreads>
__global__ void __launch_bounds__(kThreads, kPrepThreads / kThreads)
prepare_kernel(const CurveDev<Real>* __restrict__ cds, const Run* __restrict__ runs, int nruns,
               uint2* __restrict__ scr_slot, typename Tr<Real>::R2* __restrict__ rec,
               typename Tr<Real>::Pv* __restrict__ pv, int* __restrict__ order_out = nullptr) {
  using R2 = typename Tr<Real>::R2;
  using Pv = typename Tr<Real>::Pv;
  extern __shared__ int hist[];
  __shared__ int wtmp_i[32];
  __shared__ double wsum[32];
  __shared__ int big[kBigBuckets];
  __shared__ int nbig;
  const int item = blockIdx.x;
  const int ri = upper_find(0, nruns, item, [&](int i) { return (long long)runs[i].item0; });
  const Run& R = runs[ri];
  const CurveDev<Real>& C = cds[R.curve];
  const int local = item - R.item0;
  const double* __restrict__ t = C.t;
  const double2* __restrict__ vw = C.vw;
  const int n = C.n;
  const int maxd = C.maxd;
  const int nb_log2 = C.nb_log2;
  const int nb = 1 << nb_log2;
  const double scale = (double)nb;
  const bool packed = n <= kPackedMaxN && nb_log2 <= 32 - kPackedShift;
  const unsigned imask = packed ? (unsigned)(kPackedMaxN - 1) : 0xffffffffu;
  const double P = C.periods[R.pidx0 + local];
  const int M = C.M;
  const int Mrec = C.Mrec;
  uint2* slot = scr_slot + R.slot_off + (size_t)local * n;
  R2* out = kOrder ? nullptr : rec + R.rec_off + (size_t)local * Mrec;
  Pv* pre = kOrder ? nullptr : pv + R.pv_off + (size_t)local * (M + 1);
  double* pre_d = reinterpret_cast<double*>(pre);   // FP64 view during the scan (Pv is 8 bytes)
  int* ord = kOrder ? order_out + R.rec_off + (size_t)local * n : nullptr;
  constexpr int kB = 4;   // elements per thread in flight in each pass
  const int stride = blockDim.x * kB;
  __shared__ RoundTables rt;
  if (C.rnb_log2 > 0 && prepare_rounds<Real, kOrder>(hist, wtmp_i, wsum, big, &nbig, rt, t, vw, n, maxd, P,
                                                     C.rnb_log2, C.rcap, slot, out, pre_d, ord))
    return;
  // global path: buckets scattered through the scratch row

  for (int b = threadIdx.x; b < nb; b += blockDim.x) hist[b] = 0;
  if (threadIdx.x == 0) nbig = 0;
  __syncthreads();
  // (1) fold and histogram of buckets
  for (int i0 = threadIdx.x; i0 < n; i0 += stride) {
    double tv[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      tv[u] = i < n ? t[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) atomicAdd(&hist[phase_bin(fold_phase(tv[u], P) * scale, nb)], 1);
    }
  }
  __syncthreads();
  block_exclusive_scan_smem(hist, nb, wtmp_i);
  // (2) scatter (in-bucket key, index) into bucket slots; afterwards hist[b]
  //     is the end of bucket b and hist[b-1] its start
  for (int i0 = threadIdx.x; i0 < n; i0 += stride) {
    double tv[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      tv[u] = i < n ? t[i] : 0.0;
    }
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) {
        const double x = fold_phase(tv[u], P) * scale;
        const int b = phase_bin(x, nb);
        const int s = atomicAdd(&hist[b], 1);
        const float f = (float)(x - (double)b);
        slot[s] = make_uint2(__float_as_uint(f), (unsigned)i | (packed ? (unsigned)b << kPackedShift : 0u));
      }
    }
  }
  __syncthreads();
  // (3) ranking within buckets.  The entry of final sorted position p and
  //     original sample i is emitted at once: its record (u, w) at p, v at
  //     pre[p + 1] for the scan, and the same at n + p when p < maxd (the
  //     wrap of patchData, GPUFun.py:110-129); i is clamped so that a
  //     malformed input can never address outside the curve.
  auto emit = [&](int p, int i) {
    i = min(max(i, 0), n - 1);
    if constexpr (kOrder) {
      ord[p] = i;
      return;
    }
    const double2 g = vw[i];
    R2 o;
    o.x = (Real)(g.x * g.y);
    o.y = (Real)g.y;
    out[p] = o;
    pre_d[p + 1] = g.x;
    if (p < maxd) {
      out[p + n] = o;
      pre_d[p + n + 1] = g.x;
    }
  };
  //     (a) buckets of more than kSmallBucket entries (clustered phases, as
  //         when the period is close to a multiple of a regular cadence) are
  //         listed, from the shared-memory counts alone;
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int k = hist[b] - (b == 0 ? 0 : hist[b - 1]);
    if (k > kSmallBucket) {
      const int q = atomicAdd(&nbig, 1);
      if (q < kBigBuckets) big[q] = b;
    }
  }
  __syncthreads();
  //     (b) whole warps rank the listed buckets (unless the list overflowed);
  const bool warp_ranked = nbig <= kBigBuckets;
  if (warp_ranked)
    for (int q = (int)(threadIdx.x >> 5); q < nbig; q += (int)(blockDim.x >> 5)) {
      const int b = big[q];
      rank_bucket_warp(slot, b == 0 ? 0 : hist[b - 1], hist[b], t, P, imask, emit);
    }
  //     (c) every other entry is ranked by its own thread: coalesced over the
  //         slots, its bucket read from the slot word (packed) or found by
  //         binary search of the bucket ends (the emitted positions are then
  //         close to the slot index, so the record writes stay nearly
  //         coalesced).
  for (int i0 = threadIdx.x; i0 < n; i0 += stride) {
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int j = i0 + u * blockDim.x;
      if (j < n) {
        const uint2 sj = slot[j];
        int lo;
        if (packed) {
          lo = (int)(sj.y >> kPackedShift);
        } else {
          lo = 0;
          int hi = nb - 1;
          while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (hist[mid] > j) hi = mid;
            else lo = mid + 1;
          }
        }
        const int s = lo == 0 ? 0 : hist[lo - 1];
        const int e = hist[lo];
        if (e - s == 1) {
          emit(j, (int)(sj.y & imask));
        } else if (e - s <= kSmallBucket || !warp_ranked) {
          int r = 0;
          for (int m = s; m < e; ++m)
            if (m != j) r += slot_less(slot[m], sj, t, P, imask);
          emit(s + r, (int)(sj.y & imask));
        }
      }
    }
  }
  __syncthreads();
  if constexpr (kOrder) return;
  // (5) prefix of v in place over pre[1..M] (accumulated in FP64; the FP32
  //     form stores float-float pairs)
  prefix_of_v<Real>(pre_d, M, wsum);
}

// ------------------------------------------------------------------ chi2
struct Best {
  double v;
  long long loc;
};
__device__ __forceinline__ void best_update(Best& b, double v, long long loc) {
  if (v < b.v || (v == b.v && loc < b.loc)) {
    b.v = v;
    b.loc = loc;
  }
}

struct Chi2Args {
  int pass;                 // GTLS_PASS_MAIN / GTLS_PASS_ALL
  int nruns;
  double depth_min;
  int* status;              // device status word (bit 0: tile copy did not complete)
  double* part_v;           // [chunk tiles]
  long long* part_loc;      // [chunk tiles]
  unsigned long long* work; // NULL, or [2]: multiply-adds of the starts passing the depth test, and issued
};

// Mean depth of the window [k, k+w): -(sum v)/w  (calcAverageFromCumsum, GPUFun.py:366-375),
// with 1/w computed once per duration.
// From the two prefix values a = pre[k + w] and b = pre[k]:
__device__ __forceinline__ double window_mean_of(double a, double b, double inv_w) { return -(a - b) * inv_w; }
__device__ __forceinline__ float window_mean_of(float2 a, float2 b, float inv_w) {
  // two-diff of the high parts, then the low parts
  float s = a.x - b.x;
  float bb = s - a.x;
  float e = (a.x - (s - bb)) - (b.x + bb);
  e += a.y - b.y;
  return -(s + e) * inv_w;
}
template <typename Pv, typename Real>
__device__ __forceinline__ Real window_mean(const Pv* pre, int k, int w, Real inv_w) {
  return window_mean_of(pre[k + w], pre[k], inv_w);
}

// Value of start k for duration d from its sums (B, C).
template <typename Real>
__device__ __forceinline__ void eval_mean(Best& best, Real mean, Real os, Real B, Real C, double depth_min,
                                          double ebase, double sentinel, long long loc) {
  if ((double)mean > depth_min) {
    Real c = mean * os * (Real)2;
    Real delta = c * ((Real)2 * B + c * C);
    best_update(best, ebase + (double)delta, loc);
  } else {
    best_update(best, sentinel, loc);
  }
}
template <typename Real>
__device__ __forceinline__ void eval_start(Best& best, const typename Tr<Real>::Pv* pre, int k, int w, Real inv_w,
                                           Real os, Real B, Real C, double depth_min, double ebase,
                                           double sentinel, long long loc) {
  eval_mean<Real>(best, window_mean(pre, k, w, inv_w), os, B, C, depth_min, ebase, sentinel, loc);
}

// Butterfly reduce-scatter of 2*kR = 18 per-lane values over the warp
// (9 + 5 + 3 + 2 + 1 shuffles): value i ends, summed over all lanes, in lane
// kLaneOf[i].  Returns this lane's value (meaningful only in those lanes).
__constant__ int kLaneOf[2 * kR] = {0, 1, 2, 4, 5, 8, 9, 10, 12, 16, 17, 18, 20, 21, 24, 25, 26, 28};

template <typename Real>
__device__ __forceinline__ Real warp_reduce_scatter18(const typename Tr<Real>::R2 (&acc)[kR]) {
  const int lane = threadIdx.x & 31;
  Real v[18];
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    v[r] = acc[r].x;
    v[kR + r] = acc[r].y;
  }
  // level xor 16: keep 9 of 18
  {
    const bool hi = lane & 16;
    Real nv[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      Real send = hi ? v[i] : v[9 + i];
      Real recv = __shfl_xor_sync(0xffffffffu, send, 16);
      nv[i] = (hi ? v[9 + i] : v[i]) + recv;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) v[i] = nv[i];
  }
  // level xor 8: keep 5 of 9 (v[9] = 0 pad)
  {
    const bool hi = lane & 8;
    v[9] = (Real)0;
    Real nv[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      Real send = hi ? v[i] : v[5 + i];
      Real recv = __shfl_xor_sync(0xffffffffu, send, 8);
      nv[i] = (hi ? v[5 + i] : v[i]) + recv;
    }
#pragma unroll
    for (int i = 0; i < 5; ++i) v[i] = nv[i];
  }
  // level xor 4: keep 3 of 5 (v[5] = 0 pad)
  {
    const bool hi = lane & 4;
    v[5] = (Real)0;
    Real nv[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      Real send = hi ? v[i] : v[3 + i];
      Real recv = __shfl_xor_sync(0xffffffffu, send, 4);
      nv[i] = (hi ? v[3 + i] : v[i]) + recv;
    }
#pragma unroll
    for (int i = 0; i < 3; ++i) v[i] = nv[i];
  }
  // level xor 2: keep 2 of 3 (v[3] = 0 pad)
  {
    const bool hi = lane & 2;
    v[3] = (Real)0;
    Real nv[2];
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      Real send = hi ? v[i] : v[2 + i];
      Real recv = __shfl_xor_sync(0xffffffffu, send, 2);
      nv[i] = (hi ? v[2 + i] : v[i]) + recv;
    }
    v[0] = nv[0];
    v[1] = nv[1];
  }
  // level xor 1: keep 1 of 2
  {
    const bool hi = lane & 1;
    Real send = hi ? v[0] : v[1];
    Real recv = __shfl_xor_sync(0xffffffffu, send, 1);
    v[0] = (hi ? v[1] : v[0]) + recv;
  }
  return v[0];
}

// correlate() with the template entries of the offset rho taken from the
// lanes instead of memory: lane q (q < Q) holds T[q*s + rho] in tl, and step
// q reads it by shuffle.  The products and their order are those of
// correlate(); only where the template value comes from differs.  All 32
// lanes must call it (lanes without starts read clamped records and discard
// the sums).
template <typename Real, bool kTwoLevel>
__device__ __forceinline__ void correlate_bc(const typename Tr<Real>::R2* __restrict__ tile, int L, int base, int s,
                                             typename Tr<Real>::R2 tl, int Q, typename Tr<Real>::R2 (&acc)[kR]) {
  using R2 = typename Tr<Real>::R2;
  R2 xs[kR];
  const int last = L - 1;
#pragma unroll
  for (int i = 0; i < kR - 1; ++i) xs[i] = tile[min(base + i * s, last)];
  R2 pr[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) pr[r] = kTwoLevel ? zero_pair<R2>() : acc[r];
  int pos = base + (kR - 1) * s;
  for (int q0 = 0; q0 < Q; q0 += kR) {
#pragma unroll
    for (int qq = 0; qq < kR; ++qq) {
      if (q0 + qq >= Q) break;
      xs[(qq + kR - 1) % kR] = tile[min(pos, last)];
      R2 tq;
      tq.x = __shfl_sync(0xffffffffu, tl.x, q0 + qq);
      tq.y = __shfl_sync(0xffffffffu, tl.y, q0 + qq);
      pos += s;
#pragma unroll
      for (int r = 0; r < kR; ++r) fma_pair(tq, xs[(qq + r) % kR], pr[r]);
    }
  }
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    if (kTwoLevel)
      add_pair(acc[r], pr[r]);
    else
      acc[r] = pr[r];
  }
}

// Dynamic shared memory of one chi2 CTA: the record tile (rounded up to 16
// bytes) followed by the per-duration table (overshoot, width | skip << 16,
// template row offset).
template <typename Real>
__host__ __device__ __forceinline__ size_t chi2_tile_bytes(int tile, int maxd) {
  return ((size_t)(tile + maxd + kTilePad) * sizeof(typename Tr<Real>::R2) + 15) & ~(size_t)15;
}
template <typename Real>
__host__ __device__ __forceinline__ size_t chi2_smem_bytes(int tile, int maxd, int D) {
  return chi2_tile_bytes<Real>(tile, maxd) + (size_t)D * (sizeof(Real) + 2 * sizeof(int));
}

// kAllStarts: the instance for the all-starts pass (every skip is 1), which
// alone carries the unclamped skip-1 path, so that the main-pass instance
// keeps its register allocation.  kGlobal: the records are read from global
// memory (through L1/L2) instead of a shared-memory tile, for curves whose
// longest duration leaves no room for a tile in shared memory (or when the
// caller asks for it); results are the same either way.
template <typename Real, bool kAllStarts, bool kGlobal>
__global__ void __launch_bounds__(kChiThreads, 1)
chi2_kernel(const CurveDev<Real>* __restrict__ cds, const Run* __restrict__ runs,
            const typename Tr<Real>::R2* __restrict__ rec, const typename Tr<Real>::Pv* __restrict__ pv,
            Chi2Args a) {
  using R2 = typename Tr<Real>::R2;
  using Pv = typename Tr<Real>::Pv;
  constexpr bool kTwoLevel = sizeof(Real) == 4;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R2* tile = reinterpret_cast<R2*>(smem_raw);
  __shared__ int task_pre[GTLS_MAX_DURATIONS + 1];
  __shared__ short task_dur[GTLS_MAX_DURATIONS];
  __shared__ int task_next;
  __shared__ Best red[kChiThreads / 32];
  __shared__ __align__(8) uint64_t tile_bar;
  __shared__ int tile_ok;
  __shared__ unsigned long long work_sm[2];

  const int cta = blockIdx.x;
  const int ri = upper_find(0, a.nruns, cta, [&](int i) { return (long long)runs[i].tile0; });
  const Run& R = runs[ri];
  const CurveDev<Real>& C = cds[R.curve];
  const int local = (cta - R.tile0) / C.ntiles;
  const int tix = (cta - R.tile0) - local * C.ntiles;
  const long long pg = R.pidx0 + local;       // period index within the curve
  const int bidx = (int)(pg / C.batch);
  const int D = C.D;
  const int n = C.n;
  const int ucnt = C.union_cnt[bidx];
  const int* ulist = C.union_list + (size_t)bidx * D;
  const int k0 = tix * C.tile;
  const int k1 = min(n, k0 + C.tile);
  const int L = (k1 - k0) + C.maxd - 1;
  const R2* src = rec + R.rec_off + (size_t)local * C.Mrec + k0;
  const Pv* pre = pv + R.pv_off + (size_t)local * (C.M + 1);
  const double ebase = *C.ebase;
  const double sentinel = (double)n;
  const int* __restrict__ skips = C.skips;
  const int lane = threadIdx.x & 31;
  // per-duration table after the tile: overshoot, (width | skip << 16), template row offset
  // staged records: the whole tile and halo, or (global records) only what
  // the lane path reads, when the host made room for it
  const bool stage = !kGlobal || C.maxd_l > 0;
  const int Lt = kGlobal ? (k1 - k0) + C.maxd_l - 1 : L;
  Real* dtab_os = reinterpret_cast<Real*>(
      smem_raw + (kGlobal ? (C.maxd_l > 0 ? chi2_tile_bytes<Real>(C.tile, C.maxd_l) : 0)
                          : chi2_tile_bytes<Real>(C.tile, C.maxd)));
  int* dtab_ws = reinterpret_cast<int*>(dtab_os + D);
  int* dtab_row = dtab_ws + D;
  const R2* __restrict__ trows = C.trows;
  if (threadIdx.x >= 32)
    for (int d = (int)threadIdx.x - 32; d < D; d += (int)blockDim.x - 32) {
      dtab_os[d] = (Real)C.overshoot[d];
      dtab_ws[d] = C.widths[d] | (skips[d] << 16);
      dtab_row[d] = C.trow_off[d];
    }

  // stage the records [k0, k0 + L) in shared memory with one bulk (TMA) copy;
  // the byte count is rounded up to 16 (the record rows are padded for it)
  const uint32_t tile_bytes = (uint32_t)(((size_t)Lt * sizeof(R2) + 15) & ~(size_t)15);
  if (stage && threadIdx.x == 0) {
    mbar_init(&tile_bar, 1);
    mbar_arrive_expect_tx(&tile_bar, tile_bytes);
    bulk_g2s(tile, src, tile_bytes, &tile_bar);
  }
  // task table (warp 0, overlapping the copy): the batch's durations in the
  // precomputed cost order (longest task first, so the CTA's last tasks are short)
  const short* corder = C.cost_order + (size_t)bidx * D;
  if (threadIdx.x < 32) {
    int carry = 0;
    for (int u0 = 0; u0 < ucnt; u0 += 32) {
      const int u = u0 + lane;
      int nt = 0;
      if (u < ucnt) {
        task_dur[u] = corder[u];
        const int d = ulist[corder[u]];
        const int sk = skips[d];
        const int jlo = (k0 + sk - 1) / sk, jhi = (k1 + sk - 1) / sk;
        const int nj = max(0, jhi - jlo);
        const int wd = C.widths[d];
        nt = (sk >= kSplitMinSkip) ? (nj + kWin - 1) / kWin
             : (kAllStarts && wd >= kLaneGateMinW ? (nj + 32 * kR * kLaneG - 1) / (32 * kR * kLaneG)
                                    : (nj + 32 * kR - 1) / (32 * kR));
      }
      int inc = nt;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        int yv = __shfl_up_sync(0xffffffffu, inc, o);
        if (lane >= o) inc += yv;
      }
      if (u < ucnt) task_pre[u] = carry + inc - nt;
      carry += __shfl_sync(0xffffffffu, inc, 31);
    }
    if (lane == 0) {
      task_pre[ucnt] = carry;
      task_next = 0;
      work_sm[0] = work_sm[1] = 0;
      if (!stage || kGlobal) {
        tile_ok = 1;   // global records: the warps that need the lane path's tile wait for it
      } else {
        tile_ok = mbar_wait_bounded(&tile_bar, 0, 1LL << 22) ? 1 : 0;
        if (!tile_ok) {
          // The copy into this CTA's shared memory may still be in flight:
          // record the failure, then wait for it again (bounded, 16x longer)
          // before the CTA goes on to evaluate nothing and exit, so that the
          // copy does not land in shared memory that a later CTA owns.
          atomicOr(a.status, 1);
          mbar_wait_bounded(&tile_bar, 0, 1LL << 26);
        }
      }
    }
  }
  __syncthreads();
  if (stage && !kGlobal) {
    // zero the pad after the tile's Lt records (the copy's rounding to 16 bytes
    // may have brought in one record past them, possibly an unwritten one)
    for (int i = Lt + (int)threadIdx.x; i < Lt + kTilePad; i += blockDim.x) {
      R2 zr;
      zr.x = (Real)0;
      zr.y = (Real)0;
      tile[i] = zr;
    }
  }
  __syncthreads();
  const R2* recs = kGlobal ? src : tile;   // the records [k0, k0 + L)
  const R2* recl = stage ? tile : src;     // the lane path's: [k0, k0 + Ll)
  const int Ll = stage ? Lt : L;

  Best best{INFINITY, 0x7fffffffffffffffLL};
  // the first start skipped by k % skip != 0 carries the value n (GPUFun.py:407,409)
  if (a.pass == GTLS_PASS_MAIN && k0 == 0 && threadIdx.x == 0 && n > 1) {
    for (int u = 0; u < ucnt; ++u)
      if (skips[ulist[u]] > 1) {
        best_update(best, sentinel, (long long)u * n + 1);
        break;
      }
  }
  const int ntask = tile_ok ? task_pre[ucnt] : 0;
  const bool count_work = a.work != nullptr;
  // global records with a staged lane-path tile: the split path starts at
  // once; a warp waits for the tile (bounded) before its first lane-path task
  bool lane_tile = !(kGlobal && stage);
  bool lane_skip = false;
  while (true) {
    int tk = 0;
    if (lane == 0) tk = atomicAdd(&task_next, 1);
    tk = __shfl_sync(0xffffffffu, tk, 0);
    if (tk >= ntask) break;
    // binary search: the entry u with task_pre[u] <= tk < task_pre[u + 1]
    int lo = 0, hi = ucnt - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (task_pre[mid] <= tk) lo = mid;
      else hi = mid - 1;
    }
    const int u = lo;
    const int sub = tk - task_pre[u];
    const int upos = task_dur[u];        // position in ascending union order
    const int d = ulist[upos];
    const int ws = dtab_ws[d];
    const int w = ws & 0xffff;
    const int s = ws >> 16;
    const int Q = (w + s - 1) / s;
    const int jlo = (k0 + s - 1) / s;
    const int jhi = (k1 + s - 1) / s;
    const R2* trow = trows + dtab_row[d];
    const Real os = dtab_os[d];
    const Real inv_w = (Real)1 / (Real)w;
    const long long locb = (long long)upos * n;
    const int Qr = (Q + kR - 1) / kR * kR;
    R2 acc[kR];
    if (s >= kSplitMinSkip) {
      // lanes split the offset rho inside a skip block.  (1) the depth test
      // of the window's starts (one start per lane); a start that fails it
      // takes the value n here and needs no sums (GPUFun.py:407,437)
      const int jw = jlo + sub * kWin;
      const int jend = min(jhi, jw + kWin);
      unsigned long long act = 0;
#pragma unroll
      for (int i0 = 0; i0 < kWin; i0 += 32) {
        const int j = jw + i0 + lane;
        bool on = false;
        if (i0 + lane < kWin && j < jend) {
          const int k = j * s;
          on = (double)window_mean(pre, k, w, inv_w) > a.depth_min;
          if (!on) best_update(best, sentinel, locb + k);
        }
        act |= (unsigned long long)__ballot_sync(0xffffffffu, on) << i0;
      }
      if (count_work && lane == 0) atomicAdd(&work_sm[0], (unsigned long long)__popcll(act) * 2ULL * (unsigned)w);
      // (2) groups of kR consecutive starts, each from the first start of the
      //     window that passes and is not yet covered (moved back so that it
      //     ends inside the window: the starts it then re-covers are either
      //     covered already or fail the test)
      while (act) {
        const int off = min(__ffsll((long long)act) - 1, kWin - kR);
        act &= ~(((1ULL << kR) - 1ULL) << off);
        const int jb = jw + off;
#pragma unroll
        for (int r = 0; r < kR; ++r) acc[r] = zero_pair<R2>();
        // every load of the group inside the tile: no clamping needed
        if ((jb + Qr + kR - 1) * s - k0 <= L) {
          if (!kTwoLevel && Qr == kR) {
            correlate_rounds<Real>(recs, jb * s - k0, s, trow, lane, acc);
          } else {
            for (int rho = lane; rho < s; rho += 32)
              correlate_pre<Real, kTwoLevel, false>(recs, L, jb * s + rho - k0, s, trow, rho, Q, acc);
          }
        } else {
          for (int rho = lane; rho < s; rho += 32)
            correlate_pre<Real, kTwoLevel, true>(recs, L, jb * s + rho - k0, s, trow, rho, Q, acc);
        }
        if (count_work && lane == 0) atomicAdd(&work_sm[1], (unsigned long long)kR * 2ULL * (unsigned)(Qr * s));
        const Real mine = warp_reduce_scatter18<Real>(acc);
        // lane kLaneOf[r] holds B_r, lane kLaneOf[kR + r] holds C_r
        int r = -1;
#pragma unroll
        for (int i = 0; i < kR; ++i)
          if (lane == kLaneOf[i]) r = i;
        const int srcl = r >= 0 ? kLaneOf[kR + r] : lane;
        const Real C = __shfl_sync(0xffffffffu, mine, srcl);
        if (r >= 0) {
          const int j = jb + r;
          if (j < jend) {
            const int k = j * s;
            eval_start<Real>(best, pre, k, w, inv_w, os, mine, C, a.depth_min, ebase, sentinel, locb + k);
          }
        }
      }
    } else if (kAllStarts && w >= kLaneGateMinW) {
      // lanes own groups of kR consecutive starts.  (1) the depth test of the
      // window's groups, kLaneG per lane (a start that fails it takes the value
      // n here); (2) the groups with a passing start, dealt out 32 at a time
      const int g0 = sub * 32 * kLaneG;
      unsigned masks[kLaneG];
      int total = 0;
#pragma unroll
      for (int i = 0; i < kLaneG; ++i) {
        const int jb = jlo + (g0 + 32 * i + lane) * kR;
        bool any = false;
        if (jb < jhi) {
          Pv p0[kR], pw[kR];
#pragma unroll
          for (int r = 0; r < kR; ++r) {
            const int k = min(jb + r, jhi - 1) * s;
            p0[r] = pre[k];
            pw[r] = pre[k + w];
          }
#pragma unroll
          for (int r = 0; r < kR; ++r) {
            if (jb + r < jhi) {
              const bool on = (double)window_mean_of(pw[r], p0[r], inv_w) > a.depth_min;
              any |= on;
              if (!on) best_update(best, sentinel, locb + (long long)(jb + r) * s);
            }
          }
        }
        masks[i] = __ballot_sync(0xffffffffu, any);
        total += __popc(masks[i]);
      }
      for (int q0 = 0; q0 < total; q0 += 32) {
        const int q = q0 + lane;
        int jb = jhi;   // no group for lanes past the last one
        if (q < total) {
          int before = 0;
#pragma unroll
          for (int i = 0; i < kLaneG; ++i) {
            const int c = __popc(masks[i]);
            if (q >= before && q < before + c) jb = jlo + (g0 + 32 * i + (int)__fns(masks[i], 0, q - before + 1)) * kR;
            before += c;
          }
        }
#pragma unroll
        for (int r = 0; r < kR; ++r) acc[r] = zero_pair<R2>();
        if (jb < jhi) {
          if (kAllStarts && !kGlobal && s == 1 && jb + kR <= jhi) {
            correlate_s1<Real, kTwoLevel>(recl, jb - k0, trow, Qr, acc);
          } else {
            for (int rho = 0; rho < s; ++rho)
              correlate<Real, kTwoLevel>(recl, Ll, jb * s + rho - k0, s, trow, rho, Q, acc);
          }
          Pv p0[kR], pw[kR];
#pragma unroll
          for (int r = 0; r < kR; ++r) {
            const int k = min(jb + r, jhi - 1) * s;
            p0[r] = pre[k];
            pw[r] = pre[k + w];
          }
#pragma unroll
          for (int r = 0; r < kR; ++r) {
            const int j = jb + r;
            if (j < jhi) {
              const int k = j * s;
              eval_mean<Real>(best, window_mean_of(pw[r], p0[r], inv_w), os, acc[r].x, acc[r].y, a.depth_min, ebase,
                              sentinel, locb + k);
            }
          }
        }
        if (count_work) {
          const unsigned ng = __popc(__ballot_sync(0xffffffffu, jb < jhi));
          if (lane == 0) atomicAdd(&work_sm[1], (unsigned long long)ng * kR * 2ULL * (unsigned)(Qr * s));
        }
      }
      if (count_work) {
        // starts passing the depth test, counted from the prefix values again
        unsigned nact = 0;
        for (int i = 0; i < kLaneG; ++i) {
          const int jb = jlo + (g0 + 32 * i + lane) * kR;
          for (int r = 0; r < kR && jb + r < jhi; ++r)
            nact += (double)window_mean(pre, (jb + r) * s, w, inv_w) > a.depth_min;
        }
        nact = __reduce_add_sync(0xffffffffu, nact);
        if (lane == 0) atomicAdd(&work_sm[0], (unsigned long long)nact * 2ULL * (unsigned)w);
      }
    } else {
      if constexpr (kGlobal) {
        if (!lane_tile) {
          int ok = 1;
          if (lane == 0) {
            ok = mbar_wait_bounded(&tile_bar, 0, 1LL << 22) ? 1 : 0;
            if (!ok) atomicOr(a.status, 1);
          }
          ok = __shfl_sync(0xffffffffu, ok, 0);
          lane_skip = !ok;
          if (ok)
            for (int i = Lt + lane; i < Lt + kTilePad; i += 32) tile[i] = zero_pair<R2>();
          __syncwarp();
          lane_tile = true;
        }
        if (lane_skip) continue;   // the status word reports it
      }
#pragma unroll
      for (int r = 0; r < kR; ++r) acc[r] = zero_pair<R2>();
      // each lane takes kR consecutive start blocks and every rho
      const int jb = jlo + (sub * 32 + lane) * kR;
      if (!kAllStarts && Q <= 32) {
        // the main pass (Q <= 16 here): every lane, the template entries of each
        // offset held across the lanes, the next offset's loaded ahead
        R2 tcur = lane < Q ? trow[lane * s] : zero_pair<R2>();
        for (int rho = 0; rho < s; ++rho) {
          const R2 tnx = (lane < Q && rho + 1 < s) ? trow[rho + 1 + lane * s] : zero_pair<R2>();
          correlate_bc<Real, kTwoLevel>(recl, Ll, min(jb, jhi) * s + rho - k0, s, tcur, Q, acc);
          tcur = tnx;
        }
      }
      if (jb < jhi) {
        if (kAllStarts && !kGlobal && s == 1 && jb + kR <= jhi) {
          correlate_s1<Real, kTwoLevel>(recl, jb - k0, trow, Qr, acc);
        } else if (kAllStarts || Q > 32) {
          for (int rho = 0; rho < s; ++rho)
            correlate<Real, kTwoLevel>(recl, Ll, jb * s + rho - k0, s, trow, rho, Q, acc);
        }
        // the prefix values of the lane's kR starts, all loads in flight
        // together (indices clamped to the last start of the tile; values of
        // starts past it are discarded)
        Pv p0[kR], pw[kR];
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          const int k = min(jb + r, jhi - 1) * s;
          p0[r] = pre[k];
          pw[r] = pre[k + w];
        }
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          const int j = jb + r;
          if (j < jhi) {
            const int k = j * s;
            eval_mean<Real>(best, window_mean_of(pw[r], p0[r], inv_w), os, acc[r].x, acc[r].y, a.depth_min, ebase,
                            sentinel, locb + k);
          }
        }
      }
      if (count_work) {
        // work counters: the lanes' starts, and those passing the depth test
        unsigned nst = 0, nact = 0;
        if (jb < jhi)
          for (int r = 0; r < kR && jb + r < jhi; ++r) {
            ++nst;
            nact += (double)window_mean(pre, (jb + r) * s, w, inv_w) > a.depth_min;
          }
        nst = __reduce_add_sync(0xffffffffu, nst);
        nact = __reduce_add_sync(0xffffffffu, nact);
        if (lane == 0) {
          atomicAdd(&work_sm[0], (unsigned long long)nact * 2ULL * (unsigned)w);
          atomicAdd(&work_sm[1], (unsigned long long)((nst + kR - 1) / kR * kR) * 2ULL * (unsigned)(Qr * s));
        }
      }
    }
  }
  // a staged copy that no warp waited for must land before the CTA exits
  if (kGlobal && stage && threadIdx.x == 0) mbar_wait_bounded(&tile_bar, 0, 1LL << 26);
  // CTA minimum (value, then location)
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    double v = __shfl_xor_sync(0xffffffffu, best.v, o);
    long long l = __shfl_xor_sync(0xffffffffu, best.loc, o);
    best_update(best, v, l);
  }
  if (lane == 0) red[threadIdx.x >> 5] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    Best b = red[0];
    for (int i = 1; i < kChiThreads / 32; ++i) best_update(b, red[i].v, red[i].loc);
    a.part_v[cta] = b.v;
    a.part_loc[cta] = b.loc;
    if (a.work) {
      atomicAdd(a.work, work_sm[0]);
      atomicAdd(a.work + 1, work_sm[1]);
    }
  }
}

template <typename Real>
__global__ void finish_kernel(const CurveDev<Real>* __restrict__ cds, const Run* __restrict__ runs, int nruns,
                              int count, const double* __restrict__ part_v, const long long* __restrict__ part_loc) {
  const int item = blockIdx.x * blockDim.x + threadIdx.x;
  if (item >= count) return;
  const int ri = upper_find(0, nruns, item, [&](int i) { return (long long)runs[i].item0; });
  const Run& R = runs[ri];
  const CurveDev<Real>& C = cds[R.curve];
  const int local = item - R.item0;
  const long long pg = R.pidx0 + local;
  Best b{INFINITY, 0x7fffffffffffffffLL};
  if (C.union_cnt[pg / C.batch] == 0) {
    b.v = NAN;
    b.loc = -1;
  } else {
    const long long c0 = (long long)R.tile0 + (long long)local * C.ntiles;
    for (int i = 0; i < C.ntiles; ++i) best_update(b, part_v[c0 + i], part_loc[c0 + i]);
  }
  C.chi2_out[pg] = b.v;
  if (C.loc_out) C.loc_out[pg] = b.loc;
}

// ------------------------------------------------- durations, unions, rows
// durationsGrid (GPUFun.py:47-86) with the same operation order.
__device__ __forceinline__ void duration_range(double period_days, float span, int n, int* wmin, int* wmax) {
  const double kSecondsPerDay = 86400;
  const double kRsMin = 695508000 * 0.05, kRsMax = 695508000 * 4.0;
  const double kRjup = 69911000;
  float length = span;
  double nt = length / period_days;
  double corr = (nt + 1.0) / nt;
  double ps = period_days * kSecondsPerDay;
  double fmin = (4.0 * ps) / (20848 * 1000000000000000.0);
  double fmax = (4.0 * ps) / (416970 * 1000000000000000.0);
  double t14min = kRsMin * pow(fmin, 1.0 / 3.0);
  double t14max = (kRsMax + kRjup * 2.0) * pow(fmax, 1.0 / 3.0);
  double dmin = t14min / ps;
  double dmax = t14max / ps;
  dmin = dmin > 0.15 ? 0.15 : dmin;
  dmax = dmax > 0.15 ? 0.15 : dmax;
  *wmin = (int)floor(dmin * n);
  *wmax = (int)ceil(dmax * n * corr);
}

__global__ void duration_range_kernel(const double* __restrict__ periods, long long np, float span, int n,
                                      int* __restrict__ wmin, int* __restrict__ wmax) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= np) return;
  duration_range(periods[i], span, n, &wmin[i], &wmax[i]);
}

// Duration ranges of every period of every curve (period offsets p_off).
template <typename Real>
__global__ void duration_range_batch_kernel(const CurveDev<Real>* __restrict__ cds,
                                            const long long* __restrict__ p_off, int n_curves) {
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= p_off[n_curves]) return;
  const int c = upper_find(0, n_curves, g, [&](int i) { return p_off[i]; });
  const CurveDev<Real>& C = cds[c];
  const long long i = g - p_off[c];
  duration_range(C.periods[i], C.span, C.n, &C.wmin[i], &C.wmax[i]);
}

// One CTA per union batch (batch offsets b_off): the ascending list of
// durations valid for at least one period of the batch (durationBool
// GPUFun.py:91-105 OR-ed as core.py:704-716), and the same entries ordered by
// the cost of one chi2 task, longest first (cost_order holds positions in
// the ascending list).
template <typename Real>
__global__ void union_kernel(const CurveDev<Real>* __restrict__ cds, const long long* __restrict__ b_off,
                             int n_curves, int all_durations) {
  __shared__ int flags[GTLS_MAX_DURATIONS];
  __shared__ int cost[GTLS_MAX_DURATIONS];
  __shared__ short pos[GTLS_MAX_DURATIONS];
  const long long gb = blockIdx.x;
  const int c = upper_find(0, n_curves, gb, [&](int i) { return b_off[i]; });
  const CurveDev<Real>& C = cds[c];
  const long long b = gb - b_off[c];
  const int D = C.D;
  const long long p0 = b * C.batch;
  const long long p1 = min(C.np, p0 + C.batch);
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    int w = C.widths[d];
    int any = 0;
    for (long long p = p0; p < p1 && !any; ++p) any = (w >= C.wmin[p]) && (w <= C.wmax[p]);
    flags[d] = any || (all_durations && p1 > p0);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int cnt = 0;
    int* ulist = C.union_list + b * D;
    for (int d = 0; d < D; ++d)
      if (flags[d]) {
        ulist[cnt] = d;
        const int sk = C.skips[d];
        const int Qb = ((C.widths[d] + sk - 1) / sk + kR - 1) / kR;
        // per-lane work of one task: every rho (thread-group path) or rho / 32 (split path)
        cost[cnt] = (sk >= kSplitMinSkip ? (sk + 31) / 32 * 5 / 4 : sk) * Qb;
        pos[cnt] = (short)cnt;
        ++cnt;
      }
    C.union_cnt[b] = cnt;
    // insertion sort by cost, descending (ties: wider first)
    for (int i = 1; i < cnt; ++i) {
      int cv = cost[i];
      short pv = pos[i];
      int j = i - 1;
      while (j >= 0 && (cost[j] < cv || (cost[j] == cv && pos[j] < pv))) {
        cost[j + 1] = cost[j];
        pos[j + 1] = pos[j];
        --j;
      }
      cost[j + 1] = cv;
      pos[j + 1] = pv;
    }
    for (int i = 0; i < cnt; ++i) C.cost_order[b * D + i] = pos[i];
  }
}

// Template rows in the layout the chi2 kernel reads: row d holds (s_i, s_i^2)
// for i < w_d and zeros up to its length.  One CTA per (curve, duration).
template <typename Real>
__global__ void template_rows_kernel(const CurveDev<Real>* __restrict__ cds, const long long* __restrict__ d_off,
                                     int n_curves) {
  const long long gd = blockIdx.x;
  const int c = upper_find(0, n_curves, gd, [&](int i) { return d_off[i]; });
  const CurveDev<Real>& C = cds[c];
  const int d = (int)(gd - d_off[c]);
  const int w = C.widths[d];
  const int len = C.trow_len[d];
  typename Tr<Real>::R2* row = C.trows + C.trow_off[d];
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    double sv = i < w ? C.templates[(size_t)d * C.max_width + i] : 0.0;
    typename Tr<Real>::R2 o;
    o.x = (Real)sv;
    o.y = (Real)(sv * sv);
    row[i] = o;
  }
}

// ------------------------------------------------------------------ host
static int nb_log2_for(int n, int shift) {
  int k = 1;
  while ((1 << k) < n) ++k;
  // at most 32768 buckets (128 KB of counters), 16384 in the two-per-SM shape
  k = std::min(n <= kPrepSmallMaxN ? 14 : 15, k + shift);
  return std::max(1, k);
}

// Shared-memory prepare path of a curve of n samples: NB = 2^(ceil(log2 n) -
// 2) buckets (at most 2^14, about four samples a bucket), and the largest
// round capacity that fits the CTA's shared memory next to them (16 bytes a
// sample: slot word and v).  Off (0) for curves beyond the packed slot
// words or when fewer than 1,024 samples fit a round.  The rounds fix the
// summation order of the prefix, so they depend on n and the device alone
// (not on the tuning, which must not change a result).
template <typename Real>
static void rounds_params(CurveDev<Real>& C, int smem_optin) {
  C.rnb_log2 = 0;
  C.rcap = 0;
  const int n = C.n;
  if (n < 1 || n > kPackedMaxN) return;
  int k = 1;
  while ((1 << k) < n) ++k;
  const int nbl = std::max(1, std::min(14, k - 2));
  // two CTAs per SM for short curves: each gets half the shared memory
  const long long budget = (n <= kPrepSmallMaxN ? smem_optin / 2 : smem_optin) - kPrepStaticSmem;
  const long long c = std::min<long long>((budget - (4LL << nbl)) / 16, n);
  if (c < 1024 && c < n) return;
  C.rnb_log2 = nbl;
  C.rcap = (int)c;
}
// Dynamic shared memory of prepare_kernel for a curve: the larger of the
// two paths' needs (a period falls back to the global path when its
// buckets do not fit the rounds).
template <typename Real>
static size_t prep_smem_bytes(const CurveDev<Real>& C) {
  size_t b = sizeof(int) << C.nb_log2;
  if (C.rnb_log2 > 0) b = std::max(b, (sizeof(int) << C.rnb_log2) + 16 * (size_t)C.rcap);
  return b;
}

// One light curve of a search, as the host sees it.
struct CurveHost {
  const double *t, *y, *dy, *periods;
  double* chi2_out;
  int64_t* loc_out;
  const int* widths;
  const double* overshoot;
  const double* templates;
  long long np;
  int n, D, max_width, batch;
  float span;
};

template <typename Real>
static int run_search(gtls_ctx* ctx, const CurveHost* ch, int n_curves, int precision_pass, int skip_point,
                      double depth_min, int flags, gtls_timing* tm, cudaStream_t st) {
  using R2 = typename Tr<Real>::R2;
  using Pv = typename Tr<Real>::Pv;
  const bool all = precision_pass == GTLS_PASS_ALL;
  const size_t smem_budget = (size_t)ctx->smem_optin - 12 * 1024;   // static shared memory ~10.5 KB

  // ---- per-curve layout on the host
  std::vector<CurveDev<Real>> cd(n_curves);
  std::vector<std::vector<int>> hw(n_curves), hskip(n_curves), hoff(n_curves), hlen(n_curves);
  std::vector<long long> p_off(n_curves + 1, 0), b_off(n_curves + 1, 0), d_off(n_curves + 1, 0);
  size_t fixed = 0, rows_total = 0;
  for (int c = 0; c < n_curves; ++c) {
    const CurveHost& h = ch[c];
    const int D = h.D;
    hw[c].resize(D);
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(hw[c].data(), h.widths, sizeof(int) * D, cudaMemcpyDeviceToHost, st));
  }
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  for (int c = 0; c < n_curves; ++c) {
    const CurveHost& h = ch[c];
    const int n = h.n, D = h.D, maxd = h.max_width;
    CurveDev<Real>& C = cd[c];
    std::memset(&C, 0, sizeof(C));
    hskip[c].resize(D);
    hoff[c].resize(D);
    hlen[c].resize(D);
    int rows = 0;
    for (int i = 0; i < D; ++i) {
      const int w = hw[c][i];
      if (w < 1 || w > maxd || (i > 0 && w <= hw[c][i - 1]))
        return fail(ctx, GTLS_E_INVALID, "widths must be ascending, >= 1 and <= max_width");
      const int sk = (!all && w > skip_point) ? w / skip_point : 1;
      const int Q = (w + sk - 1) / sk;
      const int Qr = (Q + kR - 1) / kR * kR;
      hskip[c][i] = sk;
      hoff[c][i] = rows;
      hlen[c][i] = (Qr + 1) * sk;   // one extra zero block: the one-step template prefetch reads it
      rows += hlen[c][i];
    }
    if (maxd > 0xffff) return fail(ctx, GTLS_E_RANGE, "max_width above 65535");
    const size_t table = (size_t)D * (sizeof(Real) + 2 * sizeof(int)) + 16;
    const long long cap = sizeof(Real) == 4 ? ctx->tile_cap_fp32 : ctx->tile_cap_fp64;
    long long tile = ((long long)((smem_budget - table) / sizeof(R2)) - maxd - kTilePad) / 256 * 256;
    // records in global memory when the longest duration leaves no room for a
    // shared-memory tile of at least 256 starts (or when the caller asks for it)
    // (the all-starts pass keeps the tile: its dense skip-1 sums reuse each
    // record many times, and it measured faster on the tile)
    const bool global_rec = (ctx->records_global && !all) || tile < 256;
    if (global_rec) tile = cap;
    tile = std::min<long long>(tile, cap);
    if (tile > n) tile = (n + 255) / 256 * 256;
    C.t = h.t;
    C.y = h.y;
    C.dy = h.dy;
    C.periods = h.periods;
    C.chi2_out = h.chi2_out;
    C.loc_out = h.loc_out;
    C.widths = h.widths;
    C.overshoot = h.overshoot;
    C.templates = h.templates;
    C.np = h.np;
    C.n = n;
    C.maxd = maxd;
    C.M = n + maxd;
    C.Mrec = (C.M + 1) & ~1;
    C.D = D;
    C.max_width = maxd;
    C.batch = h.batch;
    C.nbatch = (int)((h.np + h.batch - 1) / h.batch);
    C.tile = (int)tile;
    C.ntiles = (int)((n + tile - 1) / tile);
    C.nb_log2 = nb_log2_for(n, ctx->bucket_shift);
    rounds_params(C, ctx->smem_optin);
    C.global_rec = global_rec ? 1 : 0;
    C.maxd_l = 0;
    if (global_rec && !all) {
      int mx = 0;
      for (int i = 0; i < D; ++i)
        if (hskip[c][i] < kSplitMinSkip) mx = std::max(mx, hw[c][i]);
      if (mx > 0 && chi2_smem_bytes<Real>((int)tile, mx, D) <= smem_budget) C.maxd_l = mx;
    }
    C.span = h.span;
    p_off[c + 1] = p_off[c] + h.np;
    b_off[c + 1] = b_off[c] + C.nbatch;
    d_off[c + 1] = d_off[c] + D;
    carve_size<double2>(fixed, n);
    carve_size<double>(fixed, 1);
    carve_size<int>(fixed, h.np);
    carve_size<int>(fixed, h.np);
    carve_size<int>(fixed, (size_t)C.nbatch);
    carve_size<int>(fixed, (size_t)C.nbatch * D);
    carve_size<short>(fixed, (size_t)C.nbatch * D);
    carve_size<int>(fixed, 3 * (size_t)D);
    carve_size<R2>(fixed, (size_t)rows);
    rows_total += rows;
  }

  // ---- small searches (a few periods: the harmonics, the best period):
  // narrower tiles, so that the chi2 launch still has about two CTAs per SM
  // (a start's value does not depend on the width of its tile)
  {
    long long ctas = 0, np_total = 0;
    for (int c = 0; c < n_curves; ++c) {
      ctas += cd[c].np * cd[c].ntiles;
      np_total += cd[c].np;
    }
    const long long want = 2LL * ctx->num_sms;
    if (np_total > 0 && ctas < want) {
      const long long per = (want + np_total - 1) / np_total;   // tiles wanted per period
      for (int c = 0; c < n_curves; ++c) {
        CurveDev<Real>& C = cd[c];
        const long long narrow = std::max<long long>(256, ((C.n + per - 1) / per + 255) / 256 * 256);
        if (narrow < C.tile) {
          C.tile = (int)narrow;
          C.ntiles = (int)((C.n + narrow - 1) / narrow);
        }
      }
    }
  }

  // ---- chunks of the period list (curve after curve) and their runs
  const size_t budget = ctx->chunk_budget;
  std::vector<Run> runs;
  std::vector<int> chunk_r0, chunk_items, chunk_tiles;
  std::vector<size_t> chunk_smem_prep, chunk_smem_chi;
  std::vector<int> chunk_global;   // per chunk: records of all its curves in global memory (1) or tiles (0)
  std::vector<int> chunk_small;    // per chunk: all its curves take the two-per-SM prepare shape
  size_t max_slot = 0, max_rec = 0, max_pv = 0, max_part = 0;
  {
    size_t slot = 0, rec = 0, pvs = 0, bytes = 0;
    int items = 0, tiles = 0;
    size_t sm_prep = 0, sm_chi = 0;
    int mode = -1;
    chunk_r0.push_back(0);
    auto close_chunk = [&]() {
      if (items == 0) return;
      chunk_global.push_back(mode & 1);
      chunk_small.push_back(mode >> 1);
      chunk_items.push_back(items);
      chunk_tiles.push_back(tiles);
      chunk_smem_prep.push_back(sm_prep);
      chunk_smem_chi.push_back(sm_chi);
      max_slot = std::max(max_slot, slot);
      max_rec = std::max(max_rec, rec);
      max_pv = std::max(max_pv, pvs);
      max_part = std::max(max_part, (size_t)tiles);
      chunk_r0.push_back((int)runs.size());
      slot = rec = pvs = bytes = 0;
      items = tiles = 0;
      sm_prep = sm_chi = 0;
      mode = -1;
    };
    for (int c = 0; c < n_curves; ++c) {
      const CurveDev<Real>& C = cd[c];
      const size_t per = (size_t)C.n * 8 + (size_t)C.Mrec * sizeof(R2) + (size_t)(C.M + 1) * sizeof(Pv) +
                         (size_t)C.ntiles * 16;
      long long p = 0;
      // one records mode and one prepare shape per chunk
      const int cmode = C.global_rec | (C.n <= kPrepSmallMaxN ? 2 : 0);
      if (C.np > 0 && mode != -1 && mode != cmode) close_chunk();
      while (p < C.np) {
        long long fit = (long long)((budget > bytes ? budget - bytes : 0) / per);
        fit = std::min<long long>(fit, (long long)INT32_MAX - items);
        fit = std::min<long long>(fit, ((1LL << 31) - 1 - tiles) / C.ntiles);
        if (fit <= 0) {
          if (items == 0) return fail(ctx, GTLS_E_RANGE, "one period does not fit the scratch budget");
          close_chunk();
          continue;
        }
        const long long take = std::min<long long>(fit, C.np - p);
        Run r;
        r.curve = c;
        r.item0 = items;
        r.count = (int)take;
        r.tile0 = tiles;
        r.pidx0 = p;
        r.slot_off = (long long)slot;
        r.rec_off = (long long)rec;
        r.pv_off = (long long)pvs;
        r.part_off = tiles;
        runs.push_back(r);
        slot += (size_t)take * C.n;
        rec += (size_t)take * C.Mrec;
        pvs += (size_t)take * (C.M + 1);
        bytes += (size_t)take * per;
        items += (int)take;
        tiles += (int)(take * C.ntiles);
        sm_prep = std::max(sm_prep, prep_smem_bytes(C));
        sm_chi = std::max(sm_chi, C.global_rec ? (C.maxd_l > 0 ? chi2_smem_bytes<Real>(C.tile, C.maxd_l, C.D)
                                                                : (size_t)C.D * (sizeof(Real) + 2 * sizeof(int)))
                                               : chi2_smem_bytes<Real>(C.tile, C.maxd, C.D));
        mode = cmode;
        p += take;
      }
    }
    close_chunk();
  }
  const int nchunks = (int)chunk_items.size();
  const int nruns_total = (int)runs.size();

  // ---- arena: fixed per-curve buffers, descriptors, and one chunk of scratch
  size_t total = fixed;
  carve_size<CurveDev<Real>>(total, n_curves);
  carve_size<Run>(total, std::max(1, nruns_total));
  carve_size<long long>(total, 3 * (size_t)(n_curves + 1));
  carve_size<uint2>(total, max_slot);
  carve_size<R2>(total, max_rec);
  carve_size<Pv>(total, max_pv);
  carve_size<double>(total, max_part);
  carve_size<long long>(total, max_part);
  carve_size<unsigned long long>(total, 2);
  total += 32 * 256;
  void* mem = arena(ctx, total);
  if (!mem) return fail(ctx, GTLS_E_NOMEM, "scratch allocation failed");
  Carver cv(mem);
  for (int c = 0; c < n_curves; ++c) {
    CurveDev<Real>& C = cd[c];
    C.vw = cv.take<double2>(C.n);
    C.ebase = cv.take<double>(1);
    C.wmin = cv.take<int>(C.np);
    C.wmax = cv.take<int>(C.np);
    C.union_cnt = cv.take<int>(C.nbatch);
    C.union_list = cv.take<int>((size_t)C.nbatch * C.D);
    C.cost_order = cv.take<short>((size_t)C.nbatch * C.D);
    int* dint = cv.take<int>(3 * (size_t)C.D);
    C.skips = dint;
    C.trow_off = dint + C.D;
    C.trow_len = dint + 2 * C.D;
    int rows = 0;
    for (int i = 0; i < C.D; ++i) rows += hlen[c][i];
    C.trows = cv.take<R2>(rows);
    std::vector<int> tmp(3 * (size_t)C.D);
    std::copy(hskip[c].begin(), hskip[c].end(), tmp.begin());
    std::copy(hoff[c].begin(), hoff[c].end(), tmp.begin() + C.D);
    std::copy(hlen[c].begin(), hlen[c].end(), tmp.begin() + 2 * C.D);
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(dint, tmp.data(), sizeof(int) * tmp.size(), cudaMemcpyHostToDevice, st));
  }
  CurveDev<Real>* d_cd = cv.take<CurveDev<Real>>(n_curves);
  Run* d_runs = cv.take<Run>(std::max(1, nruns_total));
  long long* d_offs = cv.take<long long>(3 * (size_t)(n_curves + 1));
  uint2* scr_slot = cv.take<uint2>(max_slot);
  R2* rec = cv.take<R2>(max_rec);
  Pv* pv = cv.take<Pv>(max_pv);
  double* part_v = cv.take<double>(max_part);
  long long* part_loc = cv.take<long long>(max_part);
  unsigned long long* work = cv.take<unsigned long long>(2);
  {
    std::vector<long long> offs(3 * (size_t)(n_curves + 1));
    std::copy(p_off.begin(), p_off.end(), offs.begin());
    std::copy(b_off.begin(), b_off.end(), offs.begin() + (n_curves + 1));
    std::copy(d_off.begin(), d_off.end(), offs.begin() + 2 * (n_curves + 1));
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_cd, cd.data(), sizeof(CurveDev<Real>) * n_curves, cudaMemcpyHostToDevice,
                                       st));
    if (nruns_total)
      GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_runs, runs.data(), sizeof(Run) * nruns_total, cudaMemcpyHostToDevice,
                                         st));
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_offs, offs.data(), sizeof(long long) * offs.size(), cudaMemcpyHostToDevice,
                                       st));
  }
  const long long* d_poff = d_offs;
  const long long* d_boff = d_offs + (n_curves + 1);
  const long long* d_doff = d_offs + 2 * (n_curves + 1);

  // ---- optional stage timing with CUDA events on the call's stream
  cudaEvent_t ev[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> evc;
  if (tm) {
    std::memset(tm, 0, sizeof(*tm));
    for (auto& e : ev) GTLS_TRY_CUDA(ctx, cudaEventCreate(&e));
    GTLS_TRY_CUDA(ctx, cudaEventRecord(ev[0], st));
  }
  GTLS_TRY_CUDA(ctx, cudaMemsetAsync(ctx->status, 0, sizeof(int), st));
  if (tm) GTLS_TRY_CUDA(ctx, cudaMemsetAsync(work, 0, 2 * sizeof(unsigned long long), st));
  curve_setup_kernel<Real><<<n_curves, 1024, 0, st>>>(d_cd);
  if (p_off[n_curves] > 0)
    duration_range_batch_kernel<Real><<<(unsigned)((p_off[n_curves] + 255) / 256), 256, 0, st>>>(d_cd, d_poff,
                                                                                                 n_curves);
  if (b_off[n_curves] > 0)
    union_kernel<Real><<<(unsigned)b_off[n_curves], 256, 0, st>>>(d_cd, d_boff, n_curves,
                                                                   (flags & GTLS_SEARCH_ALL_DURATIONS) ? 1 : 0);
  template_rows_kernel<Real><<<(unsigned)d_off[n_curves], 256, 0, st>>>(d_cd, d_doff, n_curves);
  ctx->launches += 4;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  if (tm) GTLS_TRY_CUDA(ctx, cudaEventRecord(ev[1], st));

  size_t max_prep = 0, max_chi = 0;
  for (int k = 0; k < nchunks; ++k) {
    max_prep = std::max(max_prep, chunk_smem_prep[k]);
    max_chi = std::max(max_chi, chunk_smem_chi[k]);
  }
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(prepare_kernel<Real, false, kPrepThreadsSmall>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(max_prep, 1)));
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(prepare_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)std::max<size_t>(max_prep, 1)));
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(chi2_kernel<Real, false, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(max_chi, 1)));
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(chi2_kernel<Real, true, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(max_chi, 1)));
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(chi2_kernel<Real, false, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(max_chi, 1)));
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(chi2_kernel<Real, true, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(max_chi, 1)));
  Chi2Args ca;
  ca.pass = precision_pass;
  ca.depth_min = depth_min;
  ca.status = ctx->status;
  ca.part_v = part_v;
  ca.part_loc = part_loc;
  ca.work = tm ? work : nullptr;
  for (int k = 0; k < nchunks; ++k) {
    const int r0 = chunk_r0[k], nr = chunk_r0[k + 1] - r0;
    const int items = chunk_items[k], tiles = chunk_tiles[k];
    cudaEvent_t e3[4];
    if (tm) {
      for (auto& e : e3) GTLS_TRY_CUDA(ctx, cudaEventCreate(&e));
      GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[0], st));
    }
    if (chunk_small[k])
      prepare_kernel<Real, false, kPrepThreadsSmall><<<items, kPrepThreadsSmall, chunk_smem_prep[k], st>>>(
          d_cd, d_runs + r0, nr, scr_slot, rec, pv);
    else
      prepare_kernel<Real><<<items, kPrepThreads, chunk_smem_prep[k], st>>>(d_cd, d_runs + r0, nr, scr_slot, rec, pv);
    if (tm) GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[1], st));
    ca.nruns = nr;
    using ChiKernel = void (*)(const CurveDev<Real>*, const Run*, const R2*, const Pv*, Chi2Args);
    const ChiKernel kern = all ? (chunk_global[k] ? &chi2_kernel<Real, true, true> : &chi2_kernel<Real, true, false>)
                               : (chunk_global[k] ? &chi2_kernel<Real, false, true>
                                                  : &chi2_kernel<Real, false, false>);
    kern<<<tiles, kChiThreads, chunk_smem_chi[k], st>>>(d_cd, d_runs + r0, rec, pv, ca);
    if (tm) GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[2], st));
    finish_kernel<Real><<<(items + 127) / 128, 128, 0, st>>>(d_cd, d_runs + r0, nr, items, part_v, part_loc);
    if (tm) {
      GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[3], st));
      for (auto& e : e3) evc.push_back(e);
    }
    ctx->launches += 3;
    GTLS_TRY_CUDA(ctx, cudaGetLastError());
  }
  if (tm) {
    GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    float ms = 0;
    GTLS_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, ev[0], ev[1]));
    tm->setup_ms = ms;
    for (size_t i = 0; i < evc.size(); i += 4) {
      GTLS_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, evc[i], evc[i + 1]));
      tm->prepare_ms += ms;
      GTLS_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, evc[i + 1], evc[i + 2]));
      tm->chi2_ms += ms;
      GTLS_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, evc[i + 2], evc[i + 3]));
      tm->finish_ms += ms;
    }
    tm->chunks = (int)(evc.size() / 4);
    for (auto e : evc) cudaEventDestroy(e);
    for (auto e : ev) cudaEventDestroy(e);
    // work counters of the chi2 kernel, from the unions the kernel used
    long long starts = 0, fma = 0;
    for (int c = 0; c < n_curves; ++c) {
      const CurveDev<Real>& C = cd[c];
      std::vector<int> hc(C.nbatch), hl((size_t)C.nbatch * C.D);
      GTLS_TRY_CUDA(ctx, cudaMemcpy(hc.data(), C.union_cnt, sizeof(int) * C.nbatch, cudaMemcpyDeviceToHost));
      GTLS_TRY_CUDA(ctx, cudaMemcpy(hl.data(), C.union_list, sizeof(int) * hl.size(), cudaMemcpyDeviceToHost));
      for (long long b = 0; b < C.nbatch; ++b) {
        long long np_b = std::min<long long>(C.batch, C.np - b * C.batch);
        for (int u = 0; u < hc[b]; ++u) {
          int dd = hl[(size_t)b * C.D + u];
          long long sk = hskip[c][dd];
          long long js = (C.n + sk - 1) / sk;
          starts += np_b * js;
          fma += np_b * js * 2LL * hw[c][dd];
        }
      }
    }
    tm->chi2_starts = starts;
    tm->chi2_fma = fma;
    unsigned long long hwk[2] = {0, 0};
    GTLS_TRY_CUDA(ctx, cudaMemcpy(hwk, work, sizeof(hwk), cudaMemcpyDeviceToHost));
    tm->chi2_active_fma = (long long)hwk[0];
    tm->chi2_issued_fma = (long long)hwk[1];
  }
  // device status word: a tile copy that did not complete within its bound
  int hst = 0;
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(&hst, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  if (hst != 0) {
    char msg[200];
    return fail(ctx, gtls_decode_status(hst, msg, sizeof(msg)), msg);
  }
  return GTLS_OK;
}

static int check_curve(gtls_ctx* ctx, const CurveHost& h) {
  if (h.n < 2 || !h.t || !h.y || !h.dy || (h.np > 0 && !h.periods) || !h.widths || !h.overshoot || !h.templates ||
      (h.np > 0 && !h.chi2_out))
    return fail(ctx, GTLS_E_INVALID, "null pointer or fewer than 2 samples");
  if (h.np < 0 || h.D < 1 || h.D > GTLS_MAX_DURATIONS)
    return fail(ctx, GTLS_E_INVALID, "n_periods >= 0 and 1 <= n_durations <= GTLS_MAX_DURATIONS required");
  if (h.max_width < 1 || h.max_width > h.n) return fail(ctx, GTLS_E_INVALID, "max_width must be in [1, n]");
  if (h.batch < 1) return fail(ctx, GTLS_E_INVALID, "batch must be >= 1");
  return GTLS_OK;
}

}  // namespace gtls

using namespace gtls;

extern "C" int gtls_search(gtls_ctx* ctx, const gtls_search_desc* d, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!d || d->abi_version != GTLS_ABI_VERSION) return fail(ctx, GTLS_E_INVALID, "bad descriptor or ABI version");
  if (d->n_periods < 1) return fail(ctx, GTLS_E_INVALID, "n_periods >= 1 required");
  if (d->skip_point < 1) return fail(ctx, GTLS_E_INVALID, "skip_point must be >= 1");
  if (d->pass != GTLS_PASS_MAIN && d->pass != GTLS_PASS_ALL) return fail(ctx, GTLS_E_INVALID, "unknown pass");
  if (d->flags & ~GTLS_SEARCH_ALL_DURATIONS) return fail(ctx, GTLS_E_INVALID, "unknown flags");
  CurveHost h;
  h.t = d->t;
  h.y = d->y;
  h.dy = d->dy;
  h.periods = d->periods;
  h.chi2_out = d->chi2_out;
  h.loc_out = d->loc_out;
  h.widths = d->widths;
  h.overshoot = d->overshoot;
  h.templates = d->templates;
  h.np = d->n_periods;
  h.n = d->n;
  h.D = d->n_durations;
  h.max_width = d->max_width;
  h.batch = d->batch;
  h.span = d->span;
  int rc = check_curve(ctx, h);
  if (rc) return rc;
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (d->precision == GTLS_FP64)
    return run_search<double>(ctx, &h, 1, d->pass, d->skip_point, d->depth_min, d->flags, d->timing, st);
  if (d->precision == GTLS_FP32)
    return run_search<float>(ctx, &h, 1, d->pass, d->skip_point, d->depth_min, d->flags, d->timing, st);
  return fail(ctx, GTLS_E_INVALID, "unknown precision");
}

extern "C" int gtls_search_batch(gtls_ctx* ctx, const gtls_batch_desc* d, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!d || d->abi_version != GTLS_ABI_VERSION) return fail(ctx, GTLS_E_INVALID, "bad descriptor or ABI version");
  if (d->n_curves < 1 || !d->sample_off || !d->period_off || !d->dur_off || !d->tmpl_off || !d->max_width ||
      !d->batch || !d->span)
    return fail(ctx, GTLS_E_INVALID, "null host array or no curves");
  // device bases first: a NULL base plus a curve's offset would not be NULL
  const bool any_period = d->period_off[d->n_curves] != d->period_off[0];
  if (!d->t || !d->y || !d->dy || !d->widths || !d->overshoot || !d->templates ||
      (any_period && (!d->periods || !d->chi2_out)))
    return fail(ctx, GTLS_E_INVALID, "null device array");
  if (d->skip_point < 1) return fail(ctx, GTLS_E_INVALID, "skip_point must be >= 1");
  if (d->pass != GTLS_PASS_MAIN && d->pass != GTLS_PASS_ALL) return fail(ctx, GTLS_E_INVALID, "unknown pass");
  if (d->flags & ~GTLS_SEARCH_ALL_DURATIONS) return fail(ctx, GTLS_E_INVALID, "unknown flags");
  std::vector<CurveHost> hs(d->n_curves);
  for (int c = 0; c < d->n_curves; ++c) {
    CurveHost& h = hs[c];
    const long long s0 = d->sample_off[c], s1 = d->sample_off[c + 1];
    const long long p0 = d->period_off[c], p1 = d->period_off[c + 1];
    const long long q0 = d->dur_off[c], q1 = d->dur_off[c + 1];
    if (s1 - s0 > (1LL << 30) || s1 < s0 || p1 < p0 || q1 <= q0)
      return fail(ctx, GTLS_E_INVALID, "offsets must be non-decreasing (every curve needs a duration)");
    h.t = d->t + s0;
    h.y = d->y + s0;
    h.dy = d->dy + s0;
    h.periods = d->periods + p0;
    h.chi2_out = d->chi2_out + p0;
    h.loc_out = d->loc_out ? d->loc_out + p0 : nullptr;
    h.widths = d->widths + q0;
    h.overshoot = d->overshoot + q0;
    h.templates = d->templates + d->tmpl_off[c];
    h.np = p1 - p0;
    h.n = (int)(s1 - s0);
    h.D = (int)(q1 - q0);
    h.max_width = d->max_width[c];
    h.batch = d->batch[c];
    h.span = d->span[c];
    int rc = check_curve(ctx, h);
    if (rc) return rc;
  }
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (d->precision == GTLS_FP64)
    return run_search<double>(ctx, hs.data(), d->n_curves, d->pass, d->skip_point, d->depth_min, d->flags,
                              d->timing, st);
  if (d->precision == GTLS_FP32)
    return run_search<float>(ctx, hs.data(), d->n_curves, d->pass, d->skip_point, d->depth_min, d->flags,
                             d->timing, st);
  return fail(ctx, GTLS_E_INVALID, "unknown precision");
}

extern "C" int gtls_fold_order(gtls_ctx* ctx, const double* t, int32_t n, const double* periods, int64_t n_periods,
                               int32_t* order_out, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!t || n < 1 || n_periods < 0 || (n_periods > 0 && (!periods || !order_out)))
    return fail(ctx, GTLS_E_INVALID, "bad arguments to gtls_fold_order");
  if (n_periods == 0) return GTLS_OK;
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  CurveDev<double> C;
  std::memset(&C, 0, sizeof(C));
  C.t = t;
  C.periods = periods;
  C.np = n_periods;
  C.n = n;
  C.M = n;
  C.Mrec = (n + 1) & ~1;
  C.nb_log2 = nb_log2_for(n, ctx->bucket_shift);
  rounds_params(C, ctx->smem_optin);
  // chunks of periods sized to the scratch budget (8 bytes of slots per sample and period)
  const long long per_chunk = std::max<long long>(
      1, std::min<long long>((long long)(ctx->chunk_budget / (8 * (size_t)n)), (long long)INT32_MAX));
  std::vector<Run> runs;
  for (long long p0 = 0; p0 < n_periods; p0 += per_chunk) {
    Run r;
    std::memset(&r, 0, sizeof(r));
    r.count = (int)std::min<long long>(per_chunk, n_periods - p0);
    r.pidx0 = p0;
    r.rec_off = p0 * n;   // offset of the run's rows in order_out
    runs.push_back(r);
  }
  size_t total = 0;
  carve_size<CurveDev<double>>(total, 1);
  carve_size<Run>(total, runs.size());
  carve_size<uint2>(total, (size_t)std::min<long long>(per_chunk, n_periods) * n);
  void* mem = arena(ctx, total);
  if (!mem) return fail(ctx, GTLS_E_NOMEM, "scratch allocation failed");
  Carver cv(mem);
  CurveDev<double>* d_cd = cv.take<CurveDev<double>>(1);
  Run* d_runs = cv.take<Run>(runs.size());
  uint2* slots = cv.take<uint2>((size_t)std::min<long long>(per_chunk, n_periods) * n);
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_cd, &C, sizeof(C), cudaMemcpyHostToDevice, st));
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_runs, runs.data(), sizeof(Run) * runs.size(), cudaMemcpyHostToDevice, st));
  const size_t smem = prep_smem_bytes(C);
  const bool small = n <= kPrepSmallMaxN;
  GTLS_TRY_CUDA(ctx, small ? cudaFuncSetAttribute(prepare_kernel<double, true, kPrepThreadsSmall>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                           : cudaFuncSetAttribute(prepare_kernel<double, true>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  for (size_t k = 0; k < runs.size(); ++k) {
    if (small)
      prepare_kernel<double, true, kPrepThreadsSmall><<<runs[k].count, kPrepThreadsSmall, smem, st>>>(
          d_cd, d_runs + k, 1, slots, nullptr, nullptr, order_out);
    else
      prepare_kernel<double, true><<<runs[k].count, kPrepThreads, smem, st>>>(d_cd, d_runs + k, 1, slots, nullptr,
                                                                               nullptr, order_out);
    ctx->launches += 1;
    GTLS_TRY_CUDA(ctx, cudaGetLastError());
  }
  // the host copies above read C and runs: wait for them before they go out of scope
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  return GTLS_OK;
}

extern "C" int gtls_duration_ranges(gtls_ctx* ctx, const double* periods, int64_t n_periods, float span,
                                    int32_t n_samples, int32_t* wmin, int32_t* wmax, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!periods || !wmin || !wmax || n_periods < 0 || n_samples < 1)
    return fail(ctx, GTLS_E_INVALID, "bad arguments to gtls_duration_ranges");
  if (n_periods == 0) return GTLS_OK;
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  duration_range_kernel<<<(unsigned)((n_periods + 255) / 256), 256, 0, st>>>(periods, n_periods, span, n_samples,
                                                                             wmin, wmax);
  ctx->launches += 1;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  return GTLS_OK;
}
