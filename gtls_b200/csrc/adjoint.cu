// Chi2 of an unfolded limb-darkened transit model and its adjoint (gradient
// with respect to the six shape parameters), for many light curves at once.
// An addition with no counterpart in the reference: it refines a search
// peak below the period/duration grid resolution.
//
// Model, for one light curve with parameters (P, T0, D, depth, u1, u2):
//   n    = round((t - T0) / P)                 nearest transit epoch
//   tau  = (t - T0) - n P                      time from mid-transit
//   s    = 2 tau / D                           chord coordinate (|s| < 1 in transit)
//   B(s) = sigmoid((1 - s^2) / kEdge)          smooth ingress/egress
//   mu   = sqrt(softplus_k(1 - s^2))           cosine of the emission angle on the chord,
//                                              softplus_k(x) = log(1 + exp(k x)) / k
//   I(s) = 1 - u1 (1 - mu) - u2 (1 - mu)^2    quadratic limb darkening
//   m(t) = 1 - depth * B(s) * I(s) / I(0)
// chi2 = sum_i w_i (y_i - m(t_i))^2, w_i = 1/dy_i^2.  Every factor is smooth,
// so the gradient is exact everywhere (n is locally constant: dtau/dP = -n).
// The backward pass recomputes m and dm/dtheta per sample instead of storing them.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"

namespace gtls {

constexpr double kEdge = 0.05;       // ingress/egress softness in chord units
constexpr double kSoftK = 200.0;     // softplus sharpness of the limb
constexpr int kAdjThreads = 256;

struct ModelGrad {
  double m;
  double d[6];   // dm / d(P, T0, D, depth, u1, u2)
};

__device__ __forceinline__ double sigmoid(double x) { return 1.0 / (1.0 + exp(-x)); }

// softplus_k(x) and its derivative
__device__ __forceinline__ void softplus_k(double x, double* v, double* dv) {
  const double kx = kSoftK * x;
  if (kx > 30.0) {
    *v = x + log1p(exp(-kx)) / kSoftK;
  } else {
    *v = log1p(exp(kx)) / kSoftK;
  }
  *dv = sigmoid(kx);
}

template <bool kGrad>
__device__ __forceinline__ ModelGrad transit_model(double t, const double* th) {
  const double P = th[0], T0 = th[1], D = th[2], depth = th[3], u1 = th[4], u2 = th[5];
  const double x = t - T0;
  const double ep = rint(x / P);
  const double tau = x - ep * P;
  const double s = 2.0 * tau / D;
  const double q = 1.0 - s * s;
  const double B = sigmoid(q / kEdge);
  double g, dg;
  softplus_k(q, &g, &dg);
  // far outside the transit softplus underflows; the floor keeps d(sqrt g) = 0 there
  const double mu = sqrt(fmax(g, 1e-300));
  const double om = 1.0 - mu;
  const double I = 1.0 - u1 * om - u2 * om * om;
  double g0, dg0;
  softplus_k(1.0, &g0, &dg0);
  const double mu0 = sqrt(g0);
  const double om0 = 1.0 - mu0;
  const double I0 = 1.0 - u1 * om0 - u2 * om0 * om0;
  const double shape = B * I / I0;
  ModelGrad r;
  r.m = 1.0 - depth * shape;
  if (kGrad) {
    // d/ds of B*I
    const double dq = -2.0 * s;
    const double dB = B * (1.0 - B) * dq / kEdge;
    const double dmu = dg * dq / (2.0 * mu);
    const double dI = (u1 + 2.0 * u2 * om) * dmu;
    const double dm_ds = -depth * (dB * I + B * dI) / I0;
    const double ds_dtau = 2.0 / D;
    r.d[0] = dm_ds * ds_dtau * (-ep);           // P
    r.d[1] = dm_ds * ds_dtau * (-1.0);          // T0
    r.d[2] = dm_ds * (-s / D);                  // D
    r.d[3] = -shape;                            // depth
    // u1, u2 through I and I0
    const double dI_u1 = -om, dI0_u1 = -om0;
    const double dI_u2 = -om * om, dI0_u2 = -om0 * om0;
    r.d[4] = -depth * B * (dI_u1 * I0 - I * dI0_u1) / (I0 * I0);
    r.d[5] = -depth * B * (dI_u2 * I0 - I * dI0_u2) / (I0 * I0);
  }
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
                                                                double* __restrict__ chi2) {
  __shared__ double sh[2 * 32 + 2];
  const int c = blockIdx.x;
  double th[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) th[k] = params[6 * c + k];
  double acc[1] = {0.0};
  for (long long i = off[c] + threadIdx.x; i < off[c + 1]; i += blockDim.x) {
    const ModelGrad r = transit_model<false>(t[i], th);
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
                                                                double* __restrict__ grad) {
  __shared__ double sh[7 * 32 + 7];
  const int c = blockIdx.x;
  double th[6];
#pragma unroll
  for (int k = 0; k < 6; ++k) th[k] = params[6 * c + k];
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (long long i = off[c] + threadIdx.x; i < off[c + 1]; i += blockDim.x) {
    const ModelGrad r = transit_model<true>(t[i], th);
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
                                                                                    chi2_out);
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
                                                                                    grad_chi2, grad_params);
  ctx->launches += 1;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  return GTLS_OK;
}
