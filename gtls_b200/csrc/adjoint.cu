// Chi2 of an unfolded limb-darkened transit model and its adjoint (gradient
// with respect to the six shape parameters), for many light curves at once.
// An addition with no counterpart in the reference: it refines a search
// peak below the period/duration grid resolution.
//
// The model is the search's own template model (gtls_b200/ldmodel.py, which
// stands in for the batman light curve of src/gputls/transit.py:8-42): a
// central (impact parameter 0) transit on a circular orbit of an opaque disk
// of radius p (stellar radii) across a star with quadratic limb darkening
// I(r) = 1 - u1 (1 - mu) - u2 (1 - mu)^2, mu = sqrt(1 - r^2).  For one light
// curve with parameters (P, T0, D, depth, u1, u2):
//   K   = 1 - u1/3 - u2/6,  p = sqrt(depth K)     (depth = central depth)
//   a   = (1 + p) / sin(pi D / P)                 (D = first-to-fourth contact)
//   phi = 2 pi ((t - T0)/P - n),  n = round((t - T0)/P)
//   z   = a |sin phi|            (no occultation when cos phi < 0)
//   m   = 1 - lambda(z, p, u1, u2),
// lambda = [int_0^{p-z} 2 pi r I dr + int_{|z-p|}^{min(1,z+p)} 2 r acos(c) I dr] / (pi K),
// c = (r^2 + z^2 - p^2) / (2 r z), both integrals by 96-node Gauss-Legendre
// quadrature after r = m + h sin(theta), exactly as ldmodel does.  Written as
// lambda = (M0 - u1 M1 - u2 M2) / (pi K) with the moments Mk of (1 - mu)^k,
// the u-derivatives are closed-form; the (z, p)-derivatives are those of the
// discrete quadrature itself (dual numbers through the nodes, the limits and
// c), so the gradient is exact for the model the forward pass evaluates.
// chi2 = sum_i w_i (y_i - m(t_i))^2, w_i = 1/dy_i^2.  n is locally constant,
// so dphi/dP = -2 pi (t - T0) / P^2.  The backward pass recomputes the model
// per sample instead of storing it.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "occultation.cuh"

namespace gtls {

constexpr int kAdjThreads = 256;
struct ModelGrad {
  double m;
  double d[6];   // dm / d(P, T0, D, depth, u1, u2)
};

// Model flux at time t for parameters th, and with kGrad its six derivatives.
template <bool kGrad>
__device__ __forceinline__ ModelGrad transit_model(double t, const double* th, const GLTable& g) {
  const double P = th[0], T0 = th[1], D = th[2], depth = th[3], u1 = th[4], u2 = th[5];
  ModelGrad r;
  r.m = 1.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) r.d[k] = 0.0;
  const double K = 1.0 - u1 / 3.0 - u2 / 6.0;
  const double dk = depth * K;
  if (!(dk > 0.0)) return r;
  const double p = sqrt(dk);
  const double ang = kPi * D / P;
  const double sD = sin(ang);
  const double a = (1.0 + p) / sD;
  const double x = t - T0;
  const double q = x / P;
  const double phi = 2.0 * kPi * (q - rint(q));
  double sphi, cphi;
  sincos(phi, &sphi, &cphi);
  if (cphi < 0.0) return r;                 // the far side of the orbit never occults
  const double S = fabs(sphi);
  const double z = a * S;
  if (!(z < 1.0 + p)) return r;
  const double norm = kPi * K;
  if (!kGrad) {
    double M[3];
    occultation_moments<double>(z, p, g, M);
    r.m = 1.0 - (M[0] - u1 * M[1] - u2 * M[2]) / norm;
    return r;
  }
  D2 M[3];
  occultation_moments<D2>(D2{z, 1.0, 0.0}, D2{p, 0.0, 1.0}, g, M);
  const D2 N = M[0] - M[1] * u1 - M[2] * u2;
  r.m = 1.0 - N.v / norm;
  const double lz = N.z / norm, lp = N.p / norm;
  const double lu1 = (-M[1].v + N.v / (3.0 * K)) / norm;
  const double lu2 = (-M[2].v + N.v / (6.0 * K)) / norm;
  // chain rule to the parameters
  const double cD = cos(ang);
  const double dp_depth = K / (2.0 * p), dp_u1 = -depth / (6.0 * p), dp_u2 = -depth / (12.0 * p);
  const double da_p = 1.0 / sD;
  const double da_D = -(1.0 + p) * cD * (kPi / P) / (sD * sD);
  const double da_P = (1.0 + p) * cD * (kPi * D / (P * P)) / (sD * sD);
  const double dS_phi = (sphi > 0.0 ? 1.0 : (sphi < 0.0 ? -1.0 : 0.0)) * cphi;
  const double dphi_P = -2.0 * kPi * x / (P * P), dphi_T0 = -2.0 * kPi / P;
  const double dz_P = S * da_P + a * dS_phi * dphi_P;
  const double dz_T0 = a * dS_phi * dphi_T0;
  const double dz_D = S * da_D;
  const double dz_p = S * da_p;
  r.d[0] = -(lz * dz_P);
  r.d[1] = -(lz * dz_T0);
  r.d[2] = -(lz * dz_D);
  r.d[3] = -((lz * dz_p + lp) * dp_depth);
  r.d[4] = -((lz * dz_p + lp) * dp_u1 + lu1);
  r.d[5] = -((lz * dz_p + lp) * dp_u2 + lu2);
  return r;
}

// Deterministic block sum of K values per thread.
template <int K>
__device__ void block_sum(double (&v)[K], double* sh) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int k = 0; k < K; ++k) {
    double x = v[k];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if (lane == 0) sh[k * 32 + wid] = x;
  }
  __syncthreads();
  if (threadIdx.x < K) {
    double x = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) x += sh[threadIdx.x * 32 + w];
    sh[K * 32 + threadIdx.x] = x;
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < K; ++k) v[k] = sh[K * 32 + k];
}

__global__ void __launch_bounds__(kAdjThreads) model_fwd_kernel(const double* __restrict__ t,
                                                                const double* __restrict__ y,
                                                                const double* __restrict__ w,
                                                                const int64_t* __restrict__ off,
                                                                const double* __restrict__ params,
                                                                double* __restrict__ chi2, const GLTable g) {
  __shared__ double sh[2 * 32 + 2];
  const int c = blockIdx.x;
  double th[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) th[k] = params[6 * c + k];
  double acc[1] = {0.0};
  for (long long i = off[c] + threadIdx.x; i < off[c + 1]; i += blockDim.x) {
    const ModelGrad r = transit_model<false>(t[i], th, g);
    const double res = y[i] - r.m;
    acc[0] += w[i] * res * res;
  }
  block_sum<1>(acc, sh);
  if (threadIdx.x == 0) chi2[c] = acc[0];
}

__global__ void __launch_bounds__(kAdjThreads) model_bwd_kernel(const double* __restrict__ t,
                                                                const double* __restrict__ y,
                                                                const double* __restrict__ w,
                                                                const int64_t* __restrict__ off,
                                                                const double* __restrict__ params,
                                                                const double* __restrict__ grad_out,
                                                                double* __restrict__ grad, const GLTable g) {
  __shared__ double sh[7 * 32 + 7];
  const int c = blockIdx.x;
  double th[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) th[k] = params[6 * c + k];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = off[c] + threadIdx.x; i < off[c + 1]; i += blockDim.x) {
    const ModelGrad r = transit_model<true>(t[i], th, g);
    const double f = -2.0 * w[i] * (y[i] - r.m);
#pragma unroll
    for (int k = 0; k < 6; ++k) acc[k] += f * r.d[k];
  }
  block_sum<6>(acc, sh);
  if (threadIdx.x < 6) grad[6 * c + threadIdx.x] = grad_out[c] * acc[threadIdx.x];
}

}  // namespace gtls

using namespace gtls;

extern "C" int gtls_model_chi2(gtls_ctx* ctx, const double* t, const double* y, const double* w,
                               const int64_t* curve_off, int32_t n_curves, const double* params, double* chi2_out,
                               void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!t || !y || !w || !curve_off || !params || !chi2_out || n_curves < 1)
    return fail(ctx, GTLS_E_INVALID, "bad arguments to gtls_model_chi2");
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  model_fwd_kernel<<<n_curves, kAdjThreads, 0, static_cast<cudaStream_t>(stream)>>>(t, y, w, curve_off, params,
                                                                                    chi2_out, gl_table());
  ctx->launches += 1;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  return GTLS_OK;
}

extern "C" int gtls_model_chi2_grad(gtls_ctx* ctx, const double* t, const double* y, const double* w,
                                    const int64_t* curve_off, int32_t n_curves, const double* params,
                                    const double* grad_chi2, double* grad_params, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!t || !y || !w || !curve_off || !params || !grad_chi2 || !grad_params || n_curves < 1)
    return fail(ctx, GTLS_E_INVALID, "bad arguments to gtls_model_chi2_grad");
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  model_bwd_kernel<<<n_curves, kAdjThreads, 0, static_cast<cudaStream_t>(stream)>>>(t, y, w, curve_off, params,
                                                                                    grad_chi2, grad_params,
                                                                                    gl_table());
  ctx->launches += 1;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  return GTLS_OK;
}
