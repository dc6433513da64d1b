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
// cores).  The mean depth comes from prefix sums of v (FP64, or compensated
// float-float in the FP32 form).  Only starts k that are multiples of
// skip(d) = w / skip_point (for w > skip_point) are evaluated in the main pass
// (GPUFun.py:402,409); every other (d,k) carries the value n
// (GPUFun.py:407,437), which takes part in the minimum like any value.
//
// Kernels:
//   curve_setup_kernel   (v, w) records per original sample and E.
//   prepare_kernel       one CTA per period: FP64 fold (GPUFun.py:30-41),
//                        stable bucket ranking of the phases (cupy argsort),
//                        gather into the padded sorted record array
//                        (patchData GPUFun.py:110-129) and the prefix of v.
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

#include "common.cuh"
#include "tma.cuh"

namespace gtls {

constexpr int kPrepThreads = 1024;
constexpr int kChiThreads = 512;
constexpr int kR = 9;            // starts per register block (odd: conflict-free strides)
constexpr int kSplitMinSkip = 32;  // skip >= this: lanes split the block offset rho

// ---------------------------------------------------------------- precision
template <typename Real> struct Tr;
template <> struct Tr<double> {
  using R2 = double2;   // (u, w) record / (s, s^2) template pair
  using Pv = double;    // prefix of v
};
template <> struct Tr<float> {
  using R2 = float2;
  using Pv = float2;    // (hi, lo) float-float prefix of v
};

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

// ------------------------------------------------------------ curve set-up
// (v, w) per original sample: v = y - 1 (exact), w = 1/(dy*dy)
// (calcInverseSquaredPatchedDy GPUFun.py:134-142), and E = sum v^2 w
// (calculate_base_error GPUFun.py:293-312 summed over the n samples).
__global__ void __launch_bounds__(1024) curve_setup_kernel(const double* __restrict__ y,
                                                           const double* __restrict__ dy, int n,
                                                           double2* __restrict__ vw,
                                                           double* __restrict__ ebase) {
  __shared__ double red[1024];
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
  if (threadIdx.x == 0) *ebase = red[0];
}

// ------------------------------------------------------------ block scans
// Exclusive scan of an int array in shared memory, in place; returns total.
__device__ int block_exclusive_scan_smem(int* a, int len, int* warp_tmp) {
  const int per = (len + blockDim.x - 1) / blockDim.x;
  const int beg = min(len, (int)threadIdx.x * per);
  const int end = min(len, beg + per);
  int local = 0;
  for (int i = beg; i < end; ++i) local += a[i];
  // block exclusive scan of `local`
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int x = local;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int yv = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += yv;
  }
  if (lane == 31) warp_tmp[wid] = x;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    int z = lane < nw ? warp_tmp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int yv = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += yv;
    }
    if (lane < nw) warp_tmp[lane] = z;  // inclusive warp totals
  }
  __syncthreads();
  int total = warp_tmp[(blockDim.x >> 5) - 1];
  int run = x - local + (wid > 0 ? warp_tmp[wid - 1] : 0);
  for (int i = beg; i < end; ++i) {
    int c = a[i];
    a[i] = run;
    run += c;
  }
  __syncthreads();
  return total;
}

// Exclusive block scan of one double per thread (fixed order, deterministic).
__device__ double block_exclusive_scan_double(double x, double* warp_tmp, double* total) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    double yv = __shfl_up_sync(0xffffffffu, inc, o);
    if (lane >= o) inc += yv;
  }
  if (lane == 31) warp_tmp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    double z = lane < nw ? warp_tmp[lane] : 0.0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      double yv = __shfl_up_sync(0xffffffffu, z, o);
      if (lane >= o) z += yv;
    }
    if (lane < nw) warp_tmp[lane] = z;
  }
  __syncthreads();
  *total = warp_tmp[(blockDim.x >> 5) - 1];
  double r = inc - x + (wid > 0 ? warp_tmp[wid - 1] : 0.0);
  __syncthreads();
  return r;
}

__device__ float2 block_exclusive_scan_ff(float2 x, float2* warp_tmp) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float2 inc = x;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    float2 yv;
    yv.x = __shfl_up_sync(0xffffffffu, inc.x, o);
    yv.y = __shfl_up_sync(0xffffffffu, inc.y, o);
    if (lane >= o) inc = ff_add(yv, inc);
  }
  if (lane == 31) warp_tmp[wid] = inc;
  __syncthreads();
  if (wid == 0) {
    int nw = blockDim.x >> 5;
    float2 z = lane < nw ? warp_tmp[lane] : make_float2(0.f, 0.f);
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      float2 yv;
      yv.x = __shfl_up_sync(0xffffffffu, z.x, o);
      yv.y = __shfl_up_sync(0xffffffffu, z.y, o);
      if (lane >= o) z = ff_add(yv, z);
    }
    if (lane < nw) warp_tmp[lane] = z;
  }
  __syncthreads();
  // exclusive = (warp prefix before this warp) + (inclusive - x) recomputed as a scan shift
  float2 prev = (wid > 0) ? warp_tmp[wid - 1] : make_float2(0.f, 0.f);
  float2 lanex;
  lanex.x = __shfl_up_sync(0xffffffffu, inc.x, 1);
  lanex.y = __shfl_up_sync(0xffffffffu, inc.y, 1);
  float2 r = (lane == 0) ? prev : ff_add(prev, lanex);
  __syncthreads();
  return r;
}

// ---------------------------------------------------------------- prepare
// Phase of sample t for period P: t/P minus its truncation, as foldFast
// (GPUFun.py:38-39) computes it (IEEE division, int truncation).
__device__ __forceinline__ double fold_phase(double t, double P) {
  double x = __ddiv_rn(t, P);
  return x - (double)(int)x;
}

// Bucket of a phase: floor(phase * NB) (exact: NB is a power of two),
// clamped so that out-of-range phases land in the first or last bucket.
__device__ __forceinline__ int phase_bin(double ph, int nb_log2) {
  double x = ldexp(ph, nb_log2);
  int b = (int)x;
  b = b < 0 ? 0 : b;
  int nb = 1 << nb_log2;
  return b >= nb ? nb - 1 : b;
}

// Strict order of two slots of the same bucket: by phase, then by original
// index (the order of a stable argsort).  The 32-bit keys are the in-bucket
// fractions rounded to float, which preserves every strict inequality; equal
// keys are decided on the exact FP64 phases, recomputed.
__device__ __forceinline__ bool slot_less(uint2 a, uint2 b, const double* __restrict__ t, double P) {
  const float fa = __uint_as_float(a.x), fb = __uint_as_float(b.x);
  if (fa != fb) return fa < fb;
  const double pa = fold_phase(t[a.y], P), pb = fold_phase(t[b.y], P);
  if (pa != pb) return pa < pb;
  return a.y < b.y;
}

template <typename Real>
__global__ void __launch_bounds__(kPrepThreads)
prepare_kernel(const double* __restrict__ t, const double2* __restrict__ vw, int n, int maxd,
               const double* __restrict__ periods, int nb_log2, uint2* __restrict__ scr_slot,
               int* __restrict__ scr_ord, typename Tr<Real>::R2* __restrict__ rec,
               typename Tr<Real>::Pv* __restrict__ pv) {
  using R2 = typename Tr<Real>::R2;
  using Pv = typename Tr<Real>::Pv;
  extern __shared__ int hist[];
  __shared__ int wtmp_i[32];
  __shared__ Pv wsum[32];
  const int nb = 1 << nb_log2;
  const int pl = blockIdx.x;
  const double P = periods[pl];
  const int M = n + maxd;
  const int Mrec = (M + 1) & ~1;   // record row stride, even
  uint2* slot = scr_slot + (size_t)pl * n;
  int* ord = scr_ord + (size_t)pl * n;
  R2* out = rec + (size_t)pl * Mrec;
  Pv* pre = pv + (size_t)pl * (M + 1);
  constexpr int kB = 4;   // elements per thread in flight in each pass
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
      if (i < n) atomicAdd(&hist[phase_bin(fold_phase(tv[u], P), nb_log2)], 1);
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
        const double ph = fold_phase(tv[u], P);
        const int b = phase_bin(ph, nb_log2);
        const int s = atomicAdd(&hist[b], 1);
        const float f = (float)(ldexp(ph, nb_log2) - (double)b);
        slot[s] = make_uint2(__float_as_uint(f), (unsigned)i);
      }
    }
  }
  __syncthreads();
  // (3) each thread ranks whole buckets: ord[start + rank] = original index
  for (int b = threadIdx.x; b < nb; b += blockDim.x) {
    const int s = b == 0 ? 0 : hist[b - 1];
    const int e = hist[b];
    if (e - s == 1) {
      ord[s] = (int)slot[s].y;
    } else if (e - s > 1) {
      for (int j = s; j < e; ++j) {
        const uint2 sj = slot[j];
        int r = 0;
        for (int m = s; m < e; ++m)
          if (m != j) r += slot_less(slot[m], sj, t, P);
        ord[s + r] = (int)sj.y;
      }
    }
  }
  __syncthreads();
  // (4) gather (u, w) into the padded sorted order (patchData) and keep v in
  //     pre[r + 1] for the scan; indices are clamped so that a malformed
  //     input can never address outside the curve
  for (int r0 = threadIdx.x; r0 < M; r0 += stride) {
    int ii[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int r = r0 + u * blockDim.x;
      ii[u] = r < M ? ord[r < n ? r : r - n] : 0;
      ii[u] = min(max(ii[u], 0), n - 1);
    }
    double2 g[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) g[u] = vw[ii[u]];
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      const int r = r0 + u * blockDim.x;
      if (r < M) {
        R2 o;
        o.x = (Real)(g[u].x * g[u].y);
        o.y = (Real)g[u].y;
        out[r] = o;
        if constexpr (sizeof(Real) == 8) pre[r + 1] = g[u].x;
        else pre[r + 1] = ff_from_double(g[u].x);
      }
    }
  }
  __syncthreads();
  // (5) prefix of v in place over pre[1..M]: each warp scans a contiguous
  //     range (coalesced), then adds the sum of the ranges before it
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int per = (M + nwarp - 1) / nwarp;
  const int beg = 1 + min(M, wid * per);
  const int end = 1 + min(M, (wid + 1) * per);
  if constexpr (sizeof(Real) == 8) {
    double acc = 0.0;
    for (int r = beg + lane; r < end; r += 32) acc += pre[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) wsum[wid] = acc;
    __syncthreads();
    double carry = 0.0;
    for (int w = 0; w < wid; ++w) carry += wsum[w];
    if (wid == 0 && lane == 0) pre[0] = 0.0;
    for (int r0 = beg; r0 < end; r0 += 32) {
      const int r = r0 + lane;
      double x = r < end ? pre[r] : 0.0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        double yv = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += yv;
      }
      if (r < end) pre[r] = carry + x;
      carry += __shfl_sync(0xffffffffu, x, 31);
    }
  } else {
    float2 acc = make_float2(0.f, 0.f);
    for (int r = beg + lane; r < end; r += 32) acc = ff_add(acc, pre[r]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      float2 yv;
      yv.x = __shfl_xor_sync(0xffffffffu, acc.x, o);
      yv.y = __shfl_xor_sync(0xffffffffu, acc.y, o);
      acc = ff_add(acc, yv);
    }
    if (lane == 0) wsum[wid] = acc;
    __syncthreads();
    float2 carry = make_float2(0.f, 0.f);
    for (int w = 0; w < wid; ++w) carry = ff_add(carry, wsum[w]);
    if (wid == 0 && lane == 0) pre[0] = make_float2(0.f, 0.f);
    for (int r0 = beg; r0 < end; r0 += 32) {
      const int r = r0 + lane;
      float2 x = r < end ? pre[r] : make_float2(0.f, 0.f);
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        float2 yv;
        yv.x = __shfl_up_sync(0xffffffffu, x.x, o);
        yv.y = __shfl_up_sync(0xffffffffu, x.y, o);
        if (lane >= o) x = ff_add(yv, x);
      }
      if (r < end) pre[r] = ff_add(carry, x);
      float2 tot;
      tot.x = __shfl_sync(0xffffffffu, x.x, 31);
      tot.y = __shfl_sync(0xffffffffu, x.y, 31);
      carry = ff_add(carry, tot);
    }
  }
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
  int n, maxd, M;
  int Mrec;                 // record row stride (M rounded up to even)
  int* status;              // device status word (bit 0: tile copy did not complete)
  int tile;                 // starts per CTA tile
  int ntiles;
  int pass;                 // GTLS_PASS_MAIN / GTLS_PASS_ALL
  int batch;                // periods per union batch
  long long p_global0;      // global index of the chunk's first period
  int D;
  const int* widths;        // [D]
  const int* skips;         // [D]  (1 for every d in the all-starts pass)
  const int* trow_off;      // [D]  offset of duration d's template row (in pairs)
  const double* overshoot;  // [D]
  const int* union_cnt;     // [nbatch]
  const int* union_list;    // [nbatch * D] ascending duration indices
  const short* cost_order;  // [nbatch * D] positions in union_list, longest task first
  double depth_min;
  const double* ebase;      // device scalar
  double* part_v;           // [chunk * ntiles]
  long long* part_loc;      // [chunk * ntiles]
};

// Mean depth of the window [k, k+w): -(sum v)/w  (calcAverageFromCumsum, GPUFun.py:366-375),
// with 1/w computed once per duration.
__device__ __forceinline__ double window_mean(const double* pre, int k, int w, double inv_w) {
  return -(pre[k + w] - pre[k]) * inv_w;
}
__device__ __forceinline__ float window_mean(const float2* pre, int k, int w, float inv_w) {
  float2 a = pre[k + w], b = pre[k];
  // two-diff of the high parts, then the low parts
  float s = a.x - b.x;
  float bb = s - a.x;
  float e = (a.x - (s - bb)) - (b.x + bb);
  e += a.y - b.y;
  return -(s + e) * inv_w;
}

// Value of start k for duration d from its sums (B, C).
template <typename Real>
__device__ __forceinline__ void eval_start(Best& best, const typename Tr<Real>::Pv* pre, int k, int w, Real inv_w,
                                           Real os, Real B, Real C, double depth_min, double ebase,
                                           double sentinel, long long loc) {
  Real mean = window_mean(pre, k, w, inv_w);
  if ((double)mean > depth_min) {
    Real c = mean * os * (Real)2;
    Real delta = c * ((Real)2 * B + c * C);
    best_update(best, ebase + (double)delta, loc);
  } else {
    best_update(best, sentinel, loc);
  }
}

// Correlate template offset rho of kR consecutive starts with the tile:
//   aB[r] += sum_{q<Q} T[q*s + rho] * u[base + (r+q)*s],  aC[r] likewise with (T^2, w)
// where base = jb*s + rho - k0 addresses start block jb.  A sliding window of
// kR records in registers gives one shared-memory load and one template load
// per kR multiply-add pairs (slot of record q+r is (q+r) % kR; the q loop is
// unrolled by kR so every slot index is a constant).  Template rows are zero
// at and beyond w.  Loads past the tile are clamped to its last record: for a
// start inside the tile they only meet those zero template entries, and the
// sums of starts past the tile are discarded.
template <typename Real, bool kTwoLevel>
__device__ __forceinline__ void correlate(const typename Tr<Real>::R2* __restrict__ tile, int L, int base, int s,
                                          const typename Tr<Real>::R2* __restrict__ trow, int rho, int Q,
                                          Real (&aB)[kR], Real (&aC)[kR]) {
  using R2 = typename Tr<Real>::R2;
  R2 xs[kR];
  const int last = L - 1;
#pragma unroll
  for (int i = 0; i < kR - 1; ++i) xs[i] = tile[min(base + i * s, last)];
  Real pB[kR], pC[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    pB[r] = kTwoLevel ? (Real)0 : aB[r];
    pC[r] = kTwoLevel ? (Real)0 : aC[r];
  }
  int pos = base + (kR - 1) * s;
  int toff = rho;
  R2 tnext = trow[toff];
  for (int q0 = 0; q0 < Q; q0 += kR) {
#pragma unroll
    for (int qq = 0; qq < kR; ++qq) {
      if (q0 + qq >= Q) break;
      xs[(qq + kR - 1) % kR] = tile[min(pos, last)];
      const R2 tq = tnext;
      pos += s;
      toff += s;
      tnext = trow[toff];   // next template entry (rows carry one zero block past Q)
#pragma unroll
      for (int r = 0; r < kR; ++r) {
        const R2 x = xs[(qq + r) % kR];
        pB[r] = fma(tq.x, x.x, pB[r]);
        pC[r] = fma(tq.y, x.y, pC[r]);
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    if (kTwoLevel) {
      aB[r] += pB[r];
      aC[r] += pC[r];
    } else {
      aB[r] = pB[r];
      aC[r] = pC[r];
    }
  }
}

// Same sums for the lanes-split path: the kR template entries of one block of
// kR template offsets are loaded together first (kR loads in flight), then the
// 2*kR-1 records they touch stream through once.
template <typename Real, bool kTwoLevel>
__device__ __forceinline__ void correlate_pre(const typename Tr<Real>::R2* __restrict__ tile, int L, int base,
                                              int s, const typename Tr<Real>::R2* __restrict__ trow, int rho,
                                              int Q, Real (&aB)[kR], Real (&aC)[kR]) {
  using R2 = typename Tr<Real>::R2;
  Real pB[kR], pC[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    pB[r] = kTwoLevel ? (Real)0 : aB[r];
    pC[r] = kTwoLevel ? (Real)0 : aC[r];
  }
  const int last = L - 1;
  int toff = rho;
  for (int q0 = 0; q0 < Q; q0 += kR) {
    R2 tq[kR];
#pragma unroll
    for (int qq = 0; qq < kR; ++qq) tq[qq] = trow[toff + qq * s];
    toff += kR * s;
    int pos = base + q0 * s;
#pragma unroll
    for (int m = 0; m < 2 * kR - 1; ++m) {
      const R2 x = tile[min(pos, last)];
      pos += s;
#pragma unroll
      for (int qq = 0; qq < kR; ++qq) {
        const int r = m - qq;
        if (r >= 0 && r < kR) {
          pB[r] = fma(tq[qq].x, x.x, pB[r]);
          pC[r] = fma(tq[qq].y, x.y, pC[r]);
        }
      }
    }
  }
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    if (kTwoLevel) {
      aB[r] += pB[r];
      aC[r] += pC[r];
    } else {
      aB[r] = pB[r];
      aC[r] = pC[r];
    }
  }
}

// Butterfly reduce-scatter of 2*kR = 18 per-lane values over the warp
// (9 + 5 + 3 + 2 + 1 shuffles): value i ends, summed over all lanes, in lane
// kLaneOf[i].  Returns this lane's value (meaningful only in those lanes).
__constant__ int kLaneOf[2 * kR] = {0, 1, 2, 4, 5, 8, 9, 10, 12, 16, 17, 18, 20, 21, 24, 25, 26, 28};

template <typename Real>
__device__ __forceinline__ Real warp_reduce_scatter18(const Real (&aB)[kR], const Real (&aC)[kR]) {
  const int lane = threadIdx.x & 31;
  Real v[18];
#pragma unroll
  for (int r = 0; r < kR; ++r) {
    v[r] = aB[r];
    v[kR + r] = aC[r];
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

template <typename Real>
__global__ void __launch_bounds__(kChiThreads, 1)
chi2_kernel(const typename Tr<Real>::R2* __restrict__ rec, const typename Tr<Real>::Pv* __restrict__ pv,
            const typename Tr<Real>::R2* __restrict__ trows, Chi2Args a) {
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

  const int tix = blockIdx.x;
  const int pl = blockIdx.y;
  const long long pg = a.p_global0 + pl;
  const int bidx = (int)(pg / a.batch);
  const int ucnt = a.union_cnt[bidx];
  const int* ulist = a.union_list + (size_t)bidx * a.D;
  const int k0 = tix * a.tile;
  const int k1 = min(a.n, k0 + a.tile);
  const int L = (k1 - k0) + a.maxd - 1;
  const R2* src = rec + (size_t)pl * a.Mrec + k0;
  const Pv* pre = pv + (size_t)pl * (a.M + 1);
  const double ebase = *a.ebase;
  const double sentinel = (double)a.n;
  const int lane = threadIdx.x & 31;

  // stage the records [k0, k0 + L) in shared memory with one bulk (TMA) copy;
  // the byte count is rounded up to 16 (the record rows are padded for it)
  const uint32_t tile_bytes = (uint32_t)(((size_t)L * sizeof(R2) + 15) & ~(size_t)15);
  if (threadIdx.x == 0) {
    mbar_init(&tile_bar, 1);
    mbar_arrive_expect_tx(&tile_bar, tile_bytes);
    bulk_g2s(tile, src, tile_bytes, &tile_bar);
  }
  // task table (warp 0, overlapping the copy): the batch's durations in the
  // precomputed cost order (longest task first, so the CTA's last tasks are short)
  const short* corder = a.cost_order + (size_t)bidx * a.D;
  if (threadIdx.x < 32) {
    int carry = 0;
    for (int u0 = 0; u0 < ucnt; u0 += 32) {
      const int u = u0 + lane;
      int nt = 0;
      if (u < ucnt) {
        task_dur[u] = corder[u];
        const int d = ulist[corder[u]];
        const int sk = a.skips[d];
        const int jlo = (k0 + sk - 1) / sk, jhi = (k1 + sk - 1) / sk;
        const int nj = max(0, jhi - jlo);
        nt = (sk >= kSplitMinSkip) ? (nj + kR - 1) / kR : (nj + 32 * kR - 1) / (32 * kR);
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
      tile_ok = mbar_wait_bounded(&tile_bar, 0, 1LL << 22) ? 1 : 0;
      if (!tile_ok) atomicOr(a.status, 1);
    }
  }
  __syncthreads();

  Best best{INFINITY, 0x7fffffffffffffffLL};
  // the first start skipped by k % skip != 0 carries the value n (GPUFun.py:407,409)
  if (a.pass == GTLS_PASS_MAIN && k0 == 0 && threadIdx.x == 0 && a.n > 1) {
    for (int u = 0; u < ucnt; ++u)
      if (a.skips[ulist[u]] > 1) {
        best_update(best, sentinel, (long long)u * a.n + 1);
        break;
      }
  }
  const int ntask = tile_ok ? task_pre[ucnt] : 0;
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
    const int w = a.widths[d];
    const int s = a.skips[d];
    const int Q = (w + s - 1) / s;
    const int jlo = (k0 + s - 1) / s;
    const int jhi = (k1 + s - 1) / s;
    const R2* trow = trows + a.trow_off[d];
    const Real os = (Real)a.overshoot[d];
    const Real inv_w = (Real)1 / (Real)w;
    const long long locb = (long long)upos * a.n;
    Real aB[kR], aC[kR];
#pragma unroll
    for (int r = 0; r < kR; ++r) {
      aB[r] = (Real)0;
      aC[r] = (Real)0;
    }
    if (s >= kSplitMinSkip) {
      // lanes split the offset rho inside a skip block; one task = kR starts
      const int jb = jlo + sub * kR;
      for (int rho = lane; rho < s; rho += 32)
        correlate_pre<Real, kTwoLevel>(tile, L, jb * s + rho - k0, s, trow, rho, Q, aB, aC);
      const Real mine = warp_reduce_scatter18<Real>(aB, aC);
      // lane kLaneOf[r] holds B_r, lane kLaneOf[kR + r] holds C_r
      int r = -1;
#pragma unroll
      for (int i = 0; i < kR; ++i)
        if (lane == kLaneOf[i]) r = i;
      const int srcl = r >= 0 ? kLaneOf[kR + r] : lane;
      const Real C = __shfl_sync(0xffffffffu, mine, srcl);
      if (r >= 0) {
        const int j = jb + r;
        if (j < jhi) {
          const int k = j * s;
          eval_start<Real>(best, pre, k, w, inv_w, os, mine, C, a.depth_min, ebase, sentinel, locb + k);
        }
      }
    } else {
      // each lane takes kR consecutive start blocks and every rho
      const int jb = jlo + (sub * 32 + lane) * kR;
      if (jb < jhi) {
        for (int rho = 0; rho < s; ++rho)
          correlate<Real, kTwoLevel>(tile, L, jb * s + rho - k0, s, trow, rho, Q, aB, aC);
#pragma unroll
        for (int r = 0; r < kR; ++r) {
          const int j = jb + r;
          if (j < jhi) {
            const int k = j * s;
            eval_start<Real>(best, pre, k, w, inv_w, os, aB[r], aC[r], a.depth_min, ebase, sentinel, locb + k);
          }
        }
      }
    }
  }
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
    a.part_v[(size_t)pl * a.ntiles + tix] = b.v;
    a.part_loc[(size_t)pl * a.ntiles + tix] = b.loc;
  }
}

__global__ void finish_kernel(const double* __restrict__ part_v, const long long* __restrict__ part_loc,
                              int ntiles, int count, long long p_global0, int batch,
                              const int* __restrict__ union_cnt, double* __restrict__ chi2,
                              int64_t* __restrict__ loc) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= count) return;
  long long pg = p_global0 + p;
  Best b{INFINITY, 0x7fffffffffffffffLL};
  if (union_cnt[pg / batch] == 0) {
    b.v = NAN;
    b.loc = -1;
  } else {
    for (int i = 0; i < ntiles; ++i) best_update(b, part_v[(size_t)p * ntiles + i], part_loc[(size_t)p * ntiles + i]);
  }
  chi2[pg] = b.v;
  if (loc) loc[pg] = b.loc;
}

// ------------------------------------------------- durations, unions, rows
// durationsGrid (GPUFun.py:47-86) with the same operation order.
__global__ void duration_range_kernel(const double* __restrict__ periods, long long np, float span, int n,
                                      int* __restrict__ wmin, int* __restrict__ wmax) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= np) return;
  const double kSecondsPerDay = 86400;
  const double kRsMin = 695508000 * 0.05, kRsMax = 695508000 * 4.0;
  const double kRjup = 69911000;
  float length = span;
  double period_days = periods[i];
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
  wmin[i] = (int)floor(dmin * n);
  wmax[i] = (int)ceil(dmax * n * corr);
}

// One CTA per batch: the ascending list of durations valid for at least one
// period of the batch (durationBool GPUFun.py:91-105 OR-ed as core.py:704-716),
// and the same entries ordered by the cost of one chi2 task, longest first
// (cost_order holds positions in the ascending list).
__global__ void union_kernel(const int* __restrict__ wmin, const int* __restrict__ wmax, long long np,
                             int batch, const int* __restrict__ widths, const int* __restrict__ skips, int D,
                             int* __restrict__ union_cnt, int* __restrict__ union_list,
                             short* __restrict__ cost_order) {
  __shared__ int flags[GTLS_MAX_DURATIONS];
  __shared__ int cost[GTLS_MAX_DURATIONS];
  __shared__ short pos[GTLS_MAX_DURATIONS];
  const long long b = blockIdx.x;
  const long long p0 = b * batch;
  const long long p1 = min(np, p0 + batch);
  for (int d = threadIdx.x; d < D; d += blockDim.x) {
    int w = widths[d];
    int any = 0;
    for (long long p = p0; p < p1 && !any; ++p) any = (w >= wmin[p]) && (w <= wmax[p]);
    flags[d] = any;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int c = 0;
    for (int d = 0; d < D; ++d)
      if (flags[d]) {
        union_list[b * D + c] = d;
        const int sk = skips[d];
        const int Qb = ((widths[d] + sk - 1) / sk + kR - 1) / kR;
        // per-lane work of one task: every rho (thread-group path) or rho / 32 (split path)
        cost[c] = (sk >= kSplitMinSkip ? (sk + 31) / 32 * 5 / 4 : sk) * Qb;
        pos[c] = (short)c;
        ++c;
      }
    union_cnt[b] = c;
    // insertion sort by cost, descending (ties: wider first)
    for (int i = 1; i < c; ++i) {
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
    for (int i = 0; i < c; ++i) cost_order[b * D + i] = pos[i];
  }
}

// Template rows in the layout the chi2 kernel reads: row d holds (s_i, s_i^2)
// for i < w_d and zeros up to `len` (a multiple of kR skip blocks).
template <typename Real>
__global__ void template_rows_kernel(const double* __restrict__ templates, int max_width,
                                     const int* __restrict__ widths, const int* __restrict__ row_off,
                                     const int* __restrict__ row_len, int D,
                                     typename Tr<Real>::R2* __restrict__ rows) {
  const int d = blockIdx.x;
  if (d >= D) return;
  const int w = widths[d];
  const int len = row_len[d];
  typename Tr<Real>::R2* row = rows + row_off[d];
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    double s = i < w ? templates[(size_t)d * max_width + i] : 0.0;
    typename Tr<Real>::R2 o;
    o.x = (Real)s;
    o.y = (Real)(s * s);
    row[i] = o;
  }
}

// ------------------------------------------------------------------ host
static int nb_log2_for(int n) {
  int k = 1;
  while ((1 << k) < n && k < 15) ++k;  // at most 32768 buckets (128 KB of counters)
  return k;
}

template <typename Real>
static int run_search(gtls_ctx* ctx, const gtls_search_desc* d, cudaStream_t st) {
  using R2 = typename Tr<Real>::R2;
  using Pv = typename Tr<Real>::Pv;
  const int n = d->n;
  const int maxd = d->max_width;
  const int M = n + maxd;
  const int Mrec = (M + 1) & ~1;
  const int D = d->n_durations;
  const long long np = d->n_periods;
  const int batch = d->batch;
  const long long nbatch = (np + batch - 1) / batch;
  const bool all = d->pass == GTLS_PASS_ALL;

  // host-side per-duration layout (skip, template row offsets)
  std::vector<int> hw(D), hskip(D), hoff(D), hlen(D);
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(hw.data(), d->widths, sizeof(int) * D, cudaMemcpyDeviceToHost, st));
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  size_t rows_total = 0;
  for (int i = 0; i < D; ++i) {
    int w = hw[i];
    if (w < 1 || w > maxd || (i > 0 && w <= hw[i - 1]))
      return fail(ctx, GTLS_E_INVALID, "widths must be ascending, >= 1 and <= max_width");
    int s = (!all && w > d->skip_point) ? w / d->skip_point : 1;
    int Q = (w + s - 1) / s;
    int Qr = (Q + kR - 1) / kR * kR;
    hskip[i] = s;
    hoff[i] = (int)rows_total;
    hlen[i] = (Qr + 1) * s;   // one extra zero block: the one-step template prefetch reads it
    rows_total += (size_t)hlen[i];
  }

  // tile size: as many starts as fit next to the maxd halo in shared memory
  const size_t smem_budget = (size_t)ctx->smem_optin - 12 * 1024;   // static shared memory ~10.5 KB
  long long tile = ((long long)(smem_budget / sizeof(R2)) - maxd) / 256 * 256;
  if (tile < 256) return fail(ctx, GTLS_E_RANGE, "light curve too long for the shared-memory tile");
  tile = std::min<long long>(tile, 8192);
  if (tile > n) tile = (n + 255) / 256 * 256;
  const int ntiles = (int)((n + tile - 1) / tile);
  const size_t smem_chi = (size_t)(tile + maxd) * sizeof(R2);
  const int nb_log2 = nb_log2_for(n);
  const size_t smem_prep = sizeof(int) << nb_log2;

  // period chunk sized to the scratch budget
  size_t per_period = 0;
  carve_size<uint2>(per_period, n);
  carve_size<int>(per_period, n);
  carve_size<R2>(per_period, Mrec);
  carve_size<Pv>(per_period, M + 1);
  carve_size<double>(per_period, ntiles);
  carve_size<long long>(per_period, ntiles);
  per_period += 6 * 256;
  const size_t budget = (size_t)8 << 30;
  long long chunk = std::max<long long>(1, std::min<long long>(np, (long long)(budget / per_period)));
  chunk = std::min<long long>(chunk, 65535);

  size_t fixed = 0;
  carve_size<double2>(fixed, n);
  carve_size<double>(fixed, 1);
  carve_size<int>(fixed, np);
  carve_size<int>(fixed, np);
  carve_size<int>(fixed, nbatch);
  carve_size<int>(fixed, nbatch * D);
  carve_size<short>(fixed, nbatch * D);
  carve_size<int>(fixed, D);
  carve_size<int>(fixed, D);
  carve_size<int>(fixed, D);
  carve_size<int>(fixed, D);
  carve_size<R2>(fixed, rows_total);
  fixed += 16 * 256;
  size_t chunk_bytes = 0;
  carve_size<uint2>(chunk_bytes, (size_t)chunk * n);
  carve_size<int>(chunk_bytes, (size_t)chunk * n);
  carve_size<R2>(chunk_bytes, (size_t)chunk * Mrec);
  carve_size<Pv>(chunk_bytes, (size_t)chunk * (M + 1));
  carve_size<double>(chunk_bytes, (size_t)chunk * ntiles);
  carve_size<long long>(chunk_bytes, (size_t)chunk * ntiles);
  chunk_bytes += 8 * 256;
  void* mem = arena(ctx, fixed + chunk_bytes);
  if (!mem) return fail(ctx, GTLS_E_NOMEM, "scratch allocation failed");
  Carver cv(mem);
  double2* vw = cv.take<double2>(n);
  double* ebase = cv.take<double>(1);
  int* wmin = cv.take<int>(np);
  int* wmax = cv.take<int>(np);
  int* ucnt = cv.take<int>(nbatch);
  int* ulist = cv.take<int>(nbatch * D);
  short* corder = cv.take<short>(nbatch * D);
  int* dskip = cv.take<int>(D);
  int* doff = cv.take<int>(D);
  int* dlen = cv.take<int>(D);
  int* dwid = cv.take<int>(D);
  R2* trows = cv.take<R2>(rows_total);
  uint2* scr_slot = cv.take<uint2>((size_t)chunk * n);
  int* scr_ord = cv.take<int>((size_t)chunk * n);
  R2* rec = cv.take<R2>((size_t)chunk * Mrec);
  Pv* pv = cv.take<Pv>((size_t)chunk * (M + 1));
  double* part_v = cv.take<double>((size_t)chunk * ntiles);
  long long* part_loc = cv.take<long long>((size_t)chunk * ntiles);

  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(dskip, hskip.data(), sizeof(int) * D, cudaMemcpyHostToDevice, st));
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(doff, hoff.data(), sizeof(int) * D, cudaMemcpyHostToDevice, st));
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(dlen, hlen.data(), sizeof(int) * D, cudaMemcpyHostToDevice, st));
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(dwid, hw.data(), sizeof(int) * D, cudaMemcpyHostToDevice, st));
  // the caller's pageable vectors must stay alive until the copies ran
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));

  // optional stage timing with CUDA events on the call's stream
  gtls_timing* tm = d->timing;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> evc;
  if (tm) {
    std::memset(tm, 0, sizeof(*tm));
    for (auto& e : ev) GTLS_TRY_CUDA(ctx, cudaEventCreate(&e));
    GTLS_TRY_CUDA(ctx, cudaEventRecord(ev[0], st));
  }
  GTLS_TRY_CUDA(ctx, cudaMemsetAsync(ctx->status, 0, sizeof(int), st));
  curve_setup_kernel<<<1, 1024, 0, st>>>(d->y, d->dy, n, vw, ebase);
  duration_range_kernel<<<(unsigned)((np + 255) / 256), 256, 0, st>>>(d->periods, np, d->span, n, wmin, wmax);
  union_kernel<<<(unsigned)nbatch, 256, 0, st>>>(wmin, wmax, np, batch, dwid, dskip, D, ucnt, ulist, corder);
  template_rows_kernel<Real><<<D, 256, 0, st>>>(d->templates, maxd, dwid, doff, dlen, D, trows);
  ctx->launches += 4;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  if (tm) GTLS_TRY_CUDA(ctx, cudaEventRecord(ev[1], st));

  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(prepare_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_prep));
  GTLS_TRY_CUDA(ctx, cudaFuncSetAttribute(chi2_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)smem_chi));
  Chi2Args ca;
  ca.n = n;
  ca.maxd = maxd;
  ca.M = M;
  ca.Mrec = Mrec;
  ca.status = ctx->status;
  ca.tile = (int)tile;
  ca.ntiles = ntiles;
  ca.pass = d->pass;
  ca.batch = batch;
  ca.D = D;
  ca.widths = dwid;
  ca.skips = dskip;
  ca.trow_off = doff;
  ca.overshoot = d->overshoot;
  ca.union_cnt = ucnt;
  ca.union_list = ulist;
  ca.cost_order = corder;
  ca.depth_min = d->depth_min;
  ca.ebase = ebase;
  ca.part_v = part_v;
  ca.part_loc = part_loc;
  for (long long p0 = 0; p0 < np; p0 += chunk) {
    const int cnt = (int)std::min<long long>(chunk, np - p0);
    cudaEvent_t e3[4];
    if (tm) {
      for (auto& e : e3) GTLS_TRY_CUDA(ctx, cudaEventCreate(&e));
      GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[0], st));
    }
    prepare_kernel<Real><<<cnt, kPrepThreads, smem_prep, st>>>(d->t, vw, n, maxd, d->periods + p0, nb_log2,
                                                               scr_slot, scr_ord, rec, pv);
    if (tm) GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[1], st));
    ca.p_global0 = p0;
    dim3 grid(ntiles, cnt);
    chi2_kernel<Real><<<grid, kChiThreads, smem_chi, st>>>(rec, pv, trows, ca);
    if (tm) GTLS_TRY_CUDA(ctx, cudaEventRecord(e3[2], st));
    finish_kernel<<<(cnt + 127) / 128, 128, 0, st>>>(part_v, part_loc, ntiles, cnt, p0, batch, ucnt, d->chi2_out,
                                                     d->loc_out);
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
    // work counters of the chi2 kernel, from the same layout the kernel uses
    std::vector<int> hc(nbatch), hl((size_t)nbatch * D);
    GTLS_TRY_CUDA(ctx, cudaMemcpy(hc.data(), ucnt, sizeof(int) * nbatch, cudaMemcpyDeviceToHost));
    GTLS_TRY_CUDA(ctx, cudaMemcpy(hl.data(), ulist, sizeof(int) * nbatch * D, cudaMemcpyDeviceToHost));
    long long starts = 0, fma = 0;
    for (long long b = 0; b < nbatch; ++b) {
      long long np_b = std::min<long long>(batch, np - b * batch);
      for (int u = 0; u < hc[b]; ++u) {
        int dd = hl[(size_t)b * D + u];
        long long s = hskip[dd];
        long long js = (n + s - 1) / s;
        starts += np_b * js;
        fma += np_b * js * 2LL * hw[dd];
      }
    }
    tm->chi2_starts = starts;
    tm->chi2_fma = fma;
  }
  // device status word: a tile copy that did not complete within its bound
  int hst = 0;
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(&hst, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, st));
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  if (hst != 0) return fail(ctx, GTLS_E_DEVICE, "chi2 kernel: shared-memory tile copy timed out");
  return GTLS_OK;
}

}  // namespace gtls

using namespace gtls;

extern "C" int gtls_search(gtls_ctx* ctx, const gtls_search_desc* d, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!d || d->abi_version != GTLS_ABI_VERSION) return fail(ctx, GTLS_E_INVALID, "bad descriptor or ABI version");
  if (d->n < 2 || !d->t || !d->y || !d->dy || !d->periods || !d->widths || !d->overshoot || !d->templates ||
      !d->chi2_out)
    return fail(ctx, GTLS_E_INVALID, "null pointer or fewer than 2 samples");
  if (d->n_periods < 1 || d->n_durations < 1 || d->n_durations > GTLS_MAX_DURATIONS)
    return fail(ctx, GTLS_E_INVALID, "n_periods >= 1 and 1 <= n_durations <= GTLS_MAX_DURATIONS required");
  if (d->max_width < 1 || d->max_width > d->n)
    return fail(ctx, GTLS_E_INVALID, "max_width must be in [1, n]");
  if (d->batch < 1 || d->skip_point < 1) return fail(ctx, GTLS_E_INVALID, "batch and skip_point must be >= 1");
  if (d->pass != GTLS_PASS_MAIN && d->pass != GTLS_PASS_ALL) return fail(ctx, GTLS_E_INVALID, "unknown pass");
  if ((long long)d->n * d->n_durations >= (1LL << 62)) return fail(ctx, GTLS_E_RANGE, "index overflow");
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (d->precision == GTLS_FP64) return run_search<double>(ctx, d, st);
  if (d->precision == GTLS_FP32) return run_search<float>(ctx, d, st);
  return fail(ctx, GTLS_E_INVALID, "unknown precision");
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
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  return GTLS_OK;
}
