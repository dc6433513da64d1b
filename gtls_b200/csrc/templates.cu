// Transit template cache on the GPU: the tables the search kernels read
// (per duration: the template row and its overshoot) for many light curves,
// built the way the reference's src/gputls/transit.py does on the host:
//   reference_transit (:8-42)   the template planet's light curve on the
//                               10,000-point supersample grid over one day
//                               (batman there, the limb-darkened occultation
//                               of occultation.cuh here), trimmed to its
//                               in-transit part, linearly interpolated to the
//                               curve's maximum width in samples and rescaled
//                               to [0, 1];
//   fractional_transit (:45-95) squeezed to each duration's width and scaled
//                               to SIGNAL_DEPTH = 0.5;
//   get_cache (:98-160)         trimmed to the samples below 1 - 1e-8, with
//                               overshoot = 1 / (2 - mean / min);
// and the row layout the search reads (core.py:753-754): 1 - template,
// padded with 1.  Every grid point (numpy.linspace), interpolation weight and
// value is formed with the same IEEE operations in the same order as the
// host code (non-contracted intrinsics: no fused multiply-adds), so the only
// differences from the host tables come from the occultation's own
// transcendental functions and sums (about 1e-16 relative).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"
#include "occultation.cuh"

namespace gtls {

constexpr int kSupersample = 10000;     // constants.py SUPERSAMPLE_SIZE
constexpr double kSignalDepth = 0.5;    // constants.py SIGNAL_DEPTH
constexpr double kCutoff = 1.0 - 0.01e-6;   // 1 - NUMERICAL_STABILITY_CUTOFF (constants.py)
constexpr int kTmplThreads = 256;

// numpy.linspace(start, stop, num)[i]: i * ((stop - start) / (num - 1)) + start,
// the last point stop itself, a single point start.
__device__ __forceinline__ double linspace_at(double start, double stop, int num, int i) {
  const double delta = __dsub_rn(stop, start);
  if (num <= 1) return __dadd_rn(__dmul_rn(0.0, delta), start);
  if (i == num - 1) return stop;
  return __dadd_rn(__dmul_rn((double)i, __ddiv_rn(delta, (double)(num - 1))), start);
}

// Linear interpolation at xn of the n knots (x(j), y(j)) (interpolation.py:8-58):
// the last knot not above xn, clamped to [0, n-2], then
// (1 - theta) y[i] + theta y[i+1], theta = (xn - x[i]) / (x[i+1] - x[i]).
template <typename X, typename Y>
__device__ __forceinline__ double interp_at(double xn, int n, X x, Y y) {
  int lo = 0, hi = n;   // first knot with x > xn, by binary search
  while (lo < hi) {
    const int mid = (lo + hi) >> 1;
    if (x(mid) > xn) hi = mid;
    else lo = mid + 1;
  }
  const int i = min(max(lo - 1, 0), n - 2);
  const double xi = x(i), xj = x(i + 1);
  const double theta = __ddiv_rn(__dsub_rn(xn, xi), __dsub_rn(xj, xi));
  return __dadd_rn(__dmul_rn(__dsub_rn(1.0, theta), y(i)), __dmul_rn(theta, y(i + 1)));
}

struct TemplatePlanet {
  double per, rp, a, ci, u1, u2;   // ci = cos(inclination)
};

// ldmodel.light_curve on the supersample grid: phase = 2 pi t / per,
// z = a sqrt(sin^2 + (ci cos)^2), no occultation on the far side (cos < 0).
__global__ void template_base_kernel(TemplatePlanet tp, double* __restrict__ flux, const GLTable g) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= kSupersample) return;
  const double t = linspace_at(-0.5, 0.5, kSupersample, i);
  const double phase = __ddiv_rn(__dmul_rn(2.0 * kPi, t), tp.per);
  double s, c;
  sincos(phase, &s, &c);
  const double cc = __dmul_rn(tp.ci, c);
  double z = __dmul_rn(tp.a, sqrt(__dadd_rn(__dmul_rn(s, s), __dmul_rn(cc, cc))));
  if (c < 0.0) z = __dadd_rn(1e3, tp.a);
  flux[i] = __dsub_rn(1.0, occulted_fraction(z, tp.rp, tp.u1, tp.u2, g));
}

// Block minimum of v (all threads get it); sh: 32 doubles.
__device__ __forceinline__ double block_min(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double m = sh[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmin(m, sh[w]);
  return m;
}
__device__ __forceinline__ int block_min_int(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v = min(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  int m = sh[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = min(m, sh[w]);
  return m;
}
__device__ __forceinline__ int block_max_int(int v, int* sh) {
  for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
  __syncthreads();
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  int m = sh[0];
  for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = max(m, sh[w]);
  return m;
}

// One CTA per curve: reference_transit(samples) (transit.py:8-42) into ref.
__global__ void template_ref_kernel(const double* __restrict__ flux, const int* __restrict__ samples,
                                    const long long* __restrict__ ref_off, double* __restrict__ ref) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  const int c = blockIdx.x;
  const int S = samples[c];
  double* out = ref + ref_off[c];
  // first supersample point in transit (numpy.argmax(flux < 1); 0 if none)
  int f = kSupersample;
  for (int i = threadIdx.x; i < kSupersample; i += blockDim.x)
    if (flux[i] < 1.0) f = min(f, i);
  f = block_min_int(f, shi);
  if (f == kSupersample) f = 0;
  // flux[f : -f + 1] and t[f : -f + 1] (Python slice bounds), knots of the interpolation
  const int k0 = f;
  const int k1 = (f == 0) ? 1 : kSupersample - f + 1;
  const int nk = k1 - k0;
  const double x0 = linspace_at(-0.5, 0.5, kSupersample, f);
  const double x1 = linspace_at(-0.5, 0.5, kSupersample, kSupersample - f - 1);
  auto kx = [&](int j) { return linspace_at(-0.5, 0.5, kSupersample, k0 + j); };
  auto ky = [&](int j) { return flux[k0 + j]; };
  double mn = INFINITY;
  for (int i = threadIdx.x; i < S; i += blockDim.x) {
    const double d = nk >= 2 ? interp_at(linspace_at(x0, x1, S, i), nk, kx, ky) : flux[k0];
    out[i] = d;
    mn = fmin(mn, d);
  }
  mn = block_min(mn, shd);
  __syncthreads();
  for (int i = threadIdx.x; i < S; i += blockDim.x) out[i] = __ddiv_rn(__dsub_rn(mn, out[i]), __dsub_rn(mn, 1.0));
}

// One CTA per template row: the squeezed, scaled template of width w
// (fractional_transit's in-transit part, transit.py:65-95), trimmed to the
// samples below the cutoff (get_cache, transit.py:128-158); writes
// overshoot[row] and the row (1 - template, padded with 1); bad[0] += 1 for a
// row with no sample below the cutoff.
__global__ void template_rows_kernel(const double* __restrict__ ref, const long long* __restrict__ ref_off,
                                     const int* __restrict__ samples, const long long* __restrict__ row_off,
                                     int n_curves, const int* __restrict__ widths,
                                     const long long* __restrict__ tmpl_off, const int* __restrict__ row_len,
                                     double* __restrict__ overshoot, double* __restrict__ templates,
                                     int* __restrict__ bad) {
  __shared__ double shd[32];
  __shared__ int shi[32];
  const long long row = blockIdx.x;
  int c = 0, hi = n_curves;   // the curve of this row: row_off[c] <= row < row_off[c + 1]
  while (hi - c > 1) {
    const int mid = (c + hi) >> 1;
    if (row_off[mid] <= row) c = mid;
    else hi = mid;
  }
  const int S = samples[c];
  const double* rf = ref + ref_off[c];
  const int w = widths[row];
  const int len = row_len[c];
  double* out = templates + tmpl_off[c] + (row - row_off[c]) * (long long)len;
  auto scaled_at = [&](int i) {
    const double xn = linspace_at(-0.5, 0.5, w, i);
    auto kx = [&](int j) { return linspace_at(-0.5, 0.5, S, j); };
    auto ky = [&](int j) { return rf[j]; };
    const double y = interp_at(xn, S, kx, ky);
    return __dsub_rn(1.0, __dmul_rn(__dsub_rn(1.0, y), kSignalDepth));
  };
  int first = w, last = -1;
  for (int i = threadIdx.x; i < w; i += blockDim.x)
    if (scaled_at(i) < kCutoff) {
      first = min(first, i);
      last = max(last, i);
    }
  first = block_min_int(first, shi);
  last = block_max_int(last, shi);
  if (last < 0) {
    if (threadIdx.x == 0) atomicAdd(bad, 1);
    return;
  }
  const int m = last - first + 1;
  double mn = INFINITY, sum = 0.0;
  for (int i = threadIdx.x; i < len; i += blockDim.x) {
    double v = 1.0;
    if (i < m) {
      const double sv = scaled_at(first + i);
      mn = fmin(mn, sv);
      sum += sv;
      v = __dsub_rn(1.0, sv);
    }
    out[i] = v;
  }
  mn = block_min(mn, shd);
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
  if ((threadIdx.x & 31) == 0) shd[threadIdx.x >> 5] = sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += shd[k];
    overshoot[row] = 1.0 / (2.0 - (s / m) / mn);
  }
}

}  // namespace gtls

using namespace gtls;

extern "C" int gtls_template_cache(gtls_ctx* ctx, const gtls_template_desc* d, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!d || d->abi_version != GTLS_ABI_VERSION) return fail(ctx, GTLS_E_INVALID, "bad descriptor or ABI version");
  const int C = d->n_curves;
  if (C < 1 || !d->samples || !d->row_off || !d->widths || !d->tmpl_off || !d->row_len || !d->overshoot ||
      !d->templates)
    return fail(ctx, GTLS_E_INVALID, "null array or no curves in gtls_template_cache");
  if (!(d->per > 0) || !(d->a > 0) || !(d->rp >= 0))
    return fail(ctx, GTLS_E_INVALID, "template planet needs per > 0, a > 0, rp >= 0");
  long long rows = d->row_off[C] - d->row_off[0];
  if (d->row_off[0] != 0 || rows < 1) return fail(ctx, GTLS_E_INVALID, "row_off must start at 0 and hold rows");
  std::vector<long long> ref_off(C + 1, 0);
  for (int c = 0; c < C; ++c) {
    const int S = d->samples[c];
    if (S < 2 || d->row_len[c] < S || d->row_off[c + 1] < d->row_off[c])
      return fail(ctx, GTLS_E_INVALID, "samples >= 2, row_len >= samples and non-decreasing row_off required");
    for (long long r = d->row_off[c]; r < d->row_off[c + 1]; ++r)
      if (d->widths[r] < 1 || d->widths[r] > S) return fail(ctx, GTLS_E_INVALID, "widths must lie in [1, samples]");
    ref_off[c + 1] = ref_off[c] + S;
  }
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  size_t total = 0;
  carve_size<double>(total, kSupersample);
  carve_size<double>(total, (size_t)ref_off[C]);
  carve_size<long long>(total, 2 * (size_t)(C + 1) + C);
  carve_size<int>(total, 2 * (size_t)C + (size_t)rows + 1);
  void* mem = arena(ctx, total);
  if (!mem) return fail(ctx, GTLS_E_NOMEM, "scratch allocation failed");
  Carver cv(mem);
  double* flux = cv.take<double>(kSupersample);
  double* ref = cv.take<double>((size_t)ref_off[C]);
  long long* d_ll = cv.take<long long>(2 * (size_t)(C + 1) + C);
  int* d_int = cv.take<int>(2 * (size_t)C + (size_t)rows + 1);
  std::vector<long long> ll(2 * (size_t)(C + 1) + C);
  std::copy(ref_off.begin(), ref_off.end(), ll.begin());
  std::copy(d->row_off, d->row_off + C + 1, ll.begin() + (C + 1));
  std::copy(d->tmpl_off, d->tmpl_off + C, ll.begin() + 2 * (C + 1));
  std::vector<int> ii(2 * (size_t)C + (size_t)rows + 1, 0);
  std::copy(d->samples, d->samples + C, ii.begin());
  std::copy(d->row_len, d->row_len + C, ii.begin() + C);
  std::copy(d->widths, d->widths + rows, ii.begin() + 2 * C);
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_ll, ll.data(), sizeof(long long) * ll.size(), cudaMemcpyHostToDevice, st));
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(d_int, ii.data(), sizeof(int) * ii.size(), cudaMemcpyHostToDevice, st));
  int* bad = d_int + 2 * C + rows;
  // the inclination enters as cos(radians(inc)), formed on the host as numpy does
  TemplatePlanet tp{d->per, d->rp, d->a, std::cos(d->inc * (kPi / 180.0)), d->u1, d->u2};
  template_base_kernel<<<(kSupersample + 255) / 256, 256, 0, st>>>(tp, flux, gl_table());
  template_ref_kernel<<<C, kTmplThreads, 0, st>>>(flux, d_int, d_ll, ref);
  template_rows_kernel<<<(unsigned)rows, kTmplThreads, 0, st>>>(ref, d_ll, d_int, d_ll + (C + 1), C, d_int + 2 * C,
                                                                 d_ll + 2 * (C + 1), d_int + C, d->overshoot,
                                                                 d->templates, bad);
  ctx->launches += 3;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  int hbad = 0;
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(&hbad, bad, sizeof(int), cudaMemcpyDeviceToHost, st));
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  if (hbad)
    return fail(ctx, GTLS_E_INVALID, std::to_string(hbad) + " template row(s) have no in-transit samples "
                                     "(light curve too short for the duration grid)");
  return GTLS_OK;
}
