// The arithmetic core of the chi2 kernel: record/template pair types and the
// register-blocked correlations of a template row with the folded records
// (B and C sums of kR consecutive starts).  Host-callable as well, so that
// the summation orders can be checked on the CPU (the device build uses the
// packed two-lane FP32 instructions, the host build two scalar FMAs with the
// same IEEE rounding).
#pragma once
#include <cuda_runtime.h>

#include <cmath>

namespace gtls {

constexpr int kR = 9;            // starts per register block (odd: conflict-free strides)

// ---------------------------------------------------------------- precision
template <typename Real> struct Tr;
template <> struct Tr<double> {
  using R2 = double2;   // (u, w) record / (s, s^2) template pair
  using Pv = double;    // prefix of v
};
static_assert(sizeof(float2) == sizeof(double), "float-float prefix shares the FP64 slot");
template <> struct Tr<float> {
  using R2 = float2;
  using Pv = float2;    // (hi, lo) float-float prefix of v
};

// (b, c) += (t.x * x.x, t.y * x.y) for an accumulator pair (B, C): one
// packed two-lane FMA in FP32 (sm_100), two FMAs in FP64.  Same IEEE
// rounding either way.
__host__ __device__ __forceinline__ void fma_pair(const double2& t, const double2& x, double2& a) {
  a.x = fma(t.x, x.x, a.x);
  a.y = fma(t.y, x.y, a.y);
}
__host__ __device__ __forceinline__ void fma_pair(const float2& t, const float2& x, float2& a) {
#ifdef __CUDA_ARCH__
  a = __ffma2_rn(t, x, a);
#else
  a.x = fmaf(t.x, x.x, a.x);
  a.y = fmaf(t.y, x.y, a.y);
#endif
}
__host__ __device__ __forceinline__ void add_pair(double2& a, const double2& b) {
  a.x += b.x;
  a.y += b.y;
}
__host__ __device__ __forceinline__ void add_pair(float2& a, const float2& b) {
#ifdef __CUDA_ARCH__
  a = __fadd2_rn(a, b);
#else
  a.x = a.x + b.x;
  a.y = a.y + b.y;
#endif
}
template <typename R2>
__host__ __device__ __forceinline__ R2 zero_pair() {
  R2 z;
  z.x = 0;
  z.y = 0;
  return z;
}

// Correlate template offset rho of kR consecutive starts with the tile:
//   acc[r].x (B) += sum_{q<Q} T[q*s + rho] * u[base + (r+q)*s],  acc[r].y (C) likewise with (T^2, w)
// where base = jb*s + rho - k0 addresses start block jb.  A sliding window of
// kR records in registers gives one shared-memory load and one template load
// per kR multiply-add pairs (slot of record q+r is (q+r) % kR; the q loop is
// unrolled by kR so every slot index is a constant).  Template rows are zero
// at and beyond w.  Loads past the tile are clamped to its last record: for a
// start inside the tile they only meet those zero template entries, and the
// sums of starts past the tile are discarded.
template <typename Real, bool kTwoLevel>
__host__ __device__ __forceinline__ void correlate(const typename Tr<Real>::R2* __restrict__ tile, int L, int base, int s,
                                          const typename Tr<Real>::R2* __restrict__ trow, int rho, int Q,
                                          typename Tr<Real>::R2 (&acc)[kR]) {
  using R2 = typename Tr<Real>::R2;
  R2 xs[kR];
  const int last = L - 1;
#pragma unroll
  for (int i = 0; i < kR - 1; ++i) xs[i] = tile[min(base + i * s, last)];
  R2 pr[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) pr[r] = kTwoLevel ? zero_pair<R2>() : acc[r];
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
        fma_pair(tq, x, pr[r]);
      }
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

// correlate() for skip 1 (every start: the all-starts pass and widths up to
// the skip point) and a group whose kR starts all lie in the tile: no
// clamping (the reads stay inside the tile and its zeroed pad), whole blocks
// of kR template entries (entries past Q are zero), consecutive records and
// template entries addressed with constant offsets from block pointers.  The
// sums are formed in exactly the order of correlate() with skip 1 (entries
// past Q add exact zeros), so a start's value does not depend on which of
// the two paths the tile boundaries send it through.
template <typename Real, bool kTwoLevel>
__host__ __device__ __forceinline__ void correlate_s1(const typename Tr<Real>::R2* __restrict__ tile, int base,
                                             const typename Tr<Real>::R2* __restrict__ trow, int Qr,
                                             typename Tr<Real>::R2 (&acc)[kR]) {
  using R2 = typename Tr<Real>::R2;
  R2 xs[kR];
  const R2* xp = tile + base;
#pragma unroll
  for (int i = 0; i < kR - 1; ++i) xs[i] = xp[i];
  R2 pr[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) pr[r] = kTwoLevel ? zero_pair<R2>() : acc[r];
  for (int q0 = 0; q0 < Qr; q0 += kR) {
    const R2* xb = xp + q0 + kR - 1;
    const R2* tb = trow + q0;
#pragma unroll
    for (int qq = 0; qq < kR; ++qq) {
      xs[(qq + kR - 1) % kR] = xb[qq];
      const R2 tq = tb[qq];
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

// Same sums for the lanes-split path: the kR template entries of one block of
// kR template offsets are loaded together first (kR loads in flight), then the
// 2*kR-1 records they touch stream through once.  kClamp: clamp record reads
// to the tile (needed only for tasks whose reads may pass its end).
template <typename Real, bool kTwoLevel, bool kClamp>
__host__ __device__ __forceinline__ void correlate_pre(const typename Tr<Real>::R2* __restrict__ tile, int L, int base,
                                              int s, const typename Tr<Real>::R2* __restrict__ trow, int rho,
                                              int Q, typename Tr<Real>::R2 (&acc)[kR]) {
  using R2 = typename Tr<Real>::R2;
  R2 pr[kR];
#pragma unroll
  for (int r = 0; r < kR; ++r) pr[r] = kTwoLevel ? zero_pair<R2>() : acc[r];
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
      const R2 x = tile[kClamp ? min(pos, last) : pos];
      pos += s;
#pragma unroll
      for (int qq = 0; qq < kR; ++qq) {
        const int r = m - qq;
        if (r >= 0 && r < kR) {
          fma_pair(tq[qq], x, pr[r]);
        }
      }
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

// correlate_pre() over all of a lane's offsets rho = lane, lane + 32, ... < s
// for a task whose template rows fit one block (Q <= kR) and whose reads stay
// in the tile, with the accumulators carried from one rho to the next (the
// single-level form).  One rho's 2*kR-1 record steps update 1, 2, ..., kR,
// ..., 2, 1 accumulators; here the last kR-1 steps of one rho run together
// with the first kR-1 of the next, so that every step updates each of the kR
// accumulators exactly once (no short dependency chains at the ends of a
// rho).  Each accumulator still receives its products in the same order
// (rho by rho, and within a rho by record), so the sums are bitwise those of
// correlate_pre().  Template slot q switches to the next rho at step q: its
// last use for the previous rho is at step q - 1.
template <typename Real>
__host__ __device__ __forceinline__ void correlate_rounds(const typename Tr<Real>::R2* __restrict__ tile, int base, int s,
                                                 const typename Tr<Real>::R2* __restrict__ trow, int lane,
                                                 typename Tr<Real>::R2 (&acc)[kR]) {
  using R2 = typename Tr<Real>::R2;
  const int nr = (s - lane + 31) >> 5;   // offsets of this lane (s >= 32, so at least one)
  const R2* xh = tile + base + lane;     // records of the current rho: x[m] = xh[m * s]
  const R2* th = trow + lane;            // its template entries: t[q] = th[q * s]
  R2 tq[kR];
#pragma unroll
  for (int q = 0; q < kR; ++q) tq[q] = th[q * s];
  // first rho: its first kR steps (step m updates r = 0..m)
#pragma unroll
  for (int m = 0; m < kR; ++m) {
    const R2 x = xh[m * s];
#pragma unroll
    for (int r = m; r >= 0; --r) fma_pair(tq[m - r], x, acc[r]);
  }
  for (int i = 1; i < nr; ++i) {
    const R2* xt = xh;
    xh += 32;
    th += 32;
    // step m: the previous rho's step kR + m (r = m+1..kR-1, template slots
    // m+1..kR-1 still hold its entries), then this rho's step m (r = m..0)
#pragma unroll
    for (int m = 0; m < kR; ++m) {
      tq[m] = th[m * s];
      if (m < kR - 1) {
        const R2 xa = xt[(kR + m) * s];
#pragma unroll
        for (int r = kR - 1; r > m; --r) fma_pair(tq[kR + m - r], xa, acc[r]);
      }
      const R2 xb = xh[m * s];
#pragma unroll
      for (int r = m; r >= 0; --r) fma_pair(tq[m - r], xb, acc[r]);
    }
  }
  // last rho: its remaining kR-1 steps
#pragma unroll
  for (int m = 0; m < kR - 1; ++m) {
    const R2 xa = xh[(kR + m) * s];
#pragma unroll
    for (int r = kR - 1; r > m; --r) fma_pair(tq[kR + m - r], xa, acc[r]);
  }
}

}  // namespace gtls
