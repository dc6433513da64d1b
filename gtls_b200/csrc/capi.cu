// C-ABI entry points of gtls_b200: context, period grid, spectra.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>

#include "common.cuh"
#include "spectra.cuh"

namespace gtls {

static thread_local std::string g_create_error;

int fail(gtls_ctx* ctx, int code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  else g_create_error = msg;
  return code;
}

void* arena(gtls_ctx* ctx, size_t bytes) {
  if (bytes <= ctx->arena_bytes) return ctx->arena;
  if (ctx->arena) {
    cudaDeviceSynchronize();
    cudaFree(ctx->arena);
    ctx->arena = nullptr;
    ctx->arena_bytes = 0;
  }
  size_t want = align_up(bytes + bytes / 8, (size_t)1 << 21);
  if (cudaMalloc(&ctx->arena, want) != cudaSuccess) {
    cudaGetLastError();
    ctx->arena = nullptr;
    return nullptr;
  }
  ctx->arena_bytes = want;
  return ctx->arena;
}

// ------------------------------------------------------------ period grid
// x^3 correctly rounded: x*x = h + l and h*x = p + e exactly (FMA), then one
// rounding of p + (e + l*x).
__device__ __forceinline__ double cube_rn(double x) {
  double h = x * x;
  double l = fma(x, x, -h);
  double p = h * x;
  double e = fma(h, x, -p);
  return p + fma(l, x, e);
}

// P(X) = 1 / (a3 * X + c)^3 / 86400 with numpy's operation order
// (grid.py:128-132): no contraction of a3*X + c.
__global__ void period_eval_kernel(double a3, double c, long long npts, double pmin, double pmax,
                                   double* __restrict__ tmp, int* __restrict__ bounds) {
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= npts) return;
  double X = (double)(i + 1);
  double f = __dadd_rn(__dmul_rn(a3, X), c);
  double fx = cube_rn(f);
  double P = __ddiv_rn(__ddiv_rn(1.0, fx), 86400.0);
  tmp[i] = P;
  if (P > pmin && P <= pmax) {
    atomicMin(&bounds[0], (int)i);
    atomicMax(&bounds[1], (int)i);
  }
}

__global__ void period_reverse_kernel(const double* __restrict__ tmp, const int* __restrict__ bounds,
                                      double* __restrict__ out) {
  int lo = bounds[0], hi = bounds[1];
  long long cnt = hi >= lo ? (long long)(hi - lo + 1) : 0;
  long long j = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (j < cnt) out[j] = tmp[hi - j];
}

// ---------------------------------------------------------------- spectra
// stats.spectra (stats.py:95-122) with numpy.ma semantics for masked entries
// (SpecState and the kernel declarations are in spectra.cuh).

__device__ __forceinline__ bool unmasked(const uint8_t* mask, long long i) { return !mask || !mask[i]; }

// Deterministic single-CTA reductions (fixed tree).
template <typename Op>
__device__ double block_reduce(double v, Op op, double* sh) {
  sh[threadIdx.x] = v;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] = op(sh[threadIdx.x], sh[threadIdx.x + s]);
    __syncthreads();
  }
  double r = sh[0];
  __syncthreads();
  return r;
}
struct OpAdd { __device__ double operator()(double a, double b) const { return a + b; } };
// NaN-propagating like numpy's min/max
struct OpMin {
  __device__ double operator()(double a, double b) const { return (a != a) ? a : ((b != b) ? b : fmin(a, b)); }
};
struct OpMax {
  __device__ double operator()(double a, double b) const { return (a != a) ? a : ((b != b) ? b : fmax(a, b)); }
};

__global__ void __launch_bounds__(1024) spectra_raw_kernel(const double* __restrict__ chi2,
                                                           const uint8_t* __restrict__ mask, long long n,
                                                           double* __restrict__ sr, double* __restrict__ praw,
                                                           SpecState* st) {
  __shared__ double sh[1024];
  double mn = INFINITY, cnt = 0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    if (unmasked(mask, i)) {
      mn = OpMin()(mn, chi2[i]);
      cnt += 1;
    }
  mn = block_reduce(mn, OpMin(), sh);
  cnt = block_reduce(cnt, OpAdd(), sh);
  double s = 0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    double v = mn / chi2[i];
    sr[i] = v;
    if (unmasked(mask, i)) s += v;
  }
  double mean = block_reduce(s, OpAdd(), sh) / cnt;
  double q = 0, mx = -INFINITY;
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    if (unmasked(mask, i)) {
      double dv = sr[i] - mean;
      q += dv * dv;
      mx = OpMax()(mx, dv);
    }
  double sd = sqrt(block_reduce(q, OpAdd(), sh) / cnt);
  mx = block_reduce(mx, OpMax(), sh);
  double sde_raw = (1 - mean) / sd;
  double scale = sde_raw / mx;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) praw[i] = (sr[i] - mean) * scale;
  if (threadIdx.x == 0) {
    st->mean_sr = mean;
    st->std_sr = sd;
    st->sde_raw = sde_raw;
    st->scale_raw = scale;
    st->count = (int)cnt;
  }
}

// Running median (helpers.py:91-106): window rows i = 0..n-k, median of the
// unmasked values of praw[i, i+k) as numpy.ma.median takes it ((lo+hi)/2 of
// the middle pair), then edge rows repeated to length n.
__global__ void running_median_kernel(const double* __restrict__ praw, const uint8_t* __restrict__ mask,
                                      long long n, int k, double* __restrict__ med) {
  long long rows = n - k + 1;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= rows) return;
  int cnt = 0;
  for (int j = 0; j < k; ++j) cnt += unmasked(mask, i + j);
  double out = NAN;
  if (cnt > 0) {
    int h = cnt / 2;
    int lo_r = (cnt & 1) ? h : h - 1;
    int hi_r = h;
    double lo = NAN, hi = NAN;
    // rank of element j among the unmasked window values, ties broken by position
    for (int j = 0; j < k; ++j) {
      if (!unmasked(mask, i + j)) continue;
      double v = praw[i + j];
      int r = 0;
      for (int m = 0; m < k; ++m) {
        if (!unmasked(mask, i + m)) continue;
        double x = praw[i + m];
        r += (x < v) || (x == v && m < j);
      }
      if (r == lo_r) lo = v;
      if (r == hi_r) hi = v;
    }
    out = (lo + hi) / 2.0;
  }
  long long front = (n - rows) / 2;
  med[front + i] = out;
}

__global__ void median_pad_kernel(double* med, long long n, long long rows) {
  long long front = (n - rows) / 2;
  long long back = n - rows - front;
  long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i < front) med[i] = med[front];
  if (i < back) med[front + rows + i] = med[front + rows - 1];
}

__global__ void __launch_bounds__(1024) spectra_final_kernel(const double* __restrict__ praw,
                                                             const uint8_t* __restrict__ mask,
                                                             const double* __restrict__ med, long long n,
                                                             double* __restrict__ power, SpecState* st) {
  __shared__ double sh[1024];
  const double cnt = st->count;
  double s = 0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    double p = praw[i] - med[i];
    power[i] = p;
    if (unmasked(mask, i)) s += p;
  }
  double mean = block_reduce(s, OpAdd(), sh) / cnt;
  double q = 0;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) {
    double p = power[i] - mean;
    power[i] = p;
    if (unmasked(mask, i)) q += p * p;
  }
  double sd = sqrt(block_reduce(q, OpAdd(), sh) / cnt);
  double mx = -INFINITY, mxp = -INFINITY;
  for (long long i = threadIdx.x; i < n; i += blockDim.x)
    if (unmasked(mask, i)) {
      mx = OpMax()(mx, power[i] / sd);
      mxp = OpMax()(mxp, power[i]);
    }
  double sde = block_reduce(mx, OpMax(), sh);
  mxp = block_reduce(mxp, OpMax(), sh);
  double scale = sde / mxp;
  for (long long i = threadIdx.x; i < n; i += blockDim.x) power[i] = power[i] * scale;
  if (threadIdx.x == 0) st->sde = sde;
}

}  // namespace gtls

using namespace gtls;

extern "C" {

int gtls_abi_version(void) { return GTLS_ABI_VERSION; }

int64_t gtls_launch_count(const gtls_ctx* ctx) { return ctx ? ctx->launches : 0; }

int gtls_set_tuning(gtls_ctx* ctx, const gtls_tuning* t) {
  if (!ctx) return GTLS_E_INVALID;
  if (!t) return fail(ctx, GTLS_E_INVALID, "null tuning");
  auto cap_ok = [](int c) { return c == 0 || (c >= 256 && c <= 65536 && c % 256 == 0); };
  if (!cap_ok(t->tile_cap_fp32) || !cap_ok(t->tile_cap_fp64))
    return fail(ctx, GTLS_E_INVALID, "tile caps must be 0 or multiples of 256 in [256, 65536]");
  if (t->bucket_shift < -3 || t->bucket_shift > 0) return fail(ctx, GTLS_E_INVALID, "bucket_shift must be in [-3, 0]");
  if (t->records_global != 0 && t->records_global != 1) return fail(ctx, GTLS_E_INVALID, "records_global must be 0 or 1");
  ctx->tile_cap_fp32 = t->tile_cap_fp32 ? t->tile_cap_fp32 : 16384;
  ctx->tile_cap_fp64 = t->tile_cap_fp64 ? t->tile_cap_fp64 : 8192;
  ctx->bucket_shift = t->bucket_shift;
  ctx->records_global = t->records_global;
  return GTLS_OK;
}

int gtls_get_tuning(const gtls_ctx* ctx, gtls_tuning* t) {
  if (!ctx || !t) return GTLS_E_INVALID;
  t->tile_cap_fp32 = ctx->tile_cap_fp32;
  t->tile_cap_fp64 = ctx->tile_cap_fp64;
  t->bucket_shift = ctx->bucket_shift;
  t->records_global = ctx->records_global;
  return GTLS_OK;
}

int gtls_set_chunk_budget(gtls_ctx* ctx, uint64_t bytes) {
  if (!ctx) return GTLS_E_INVALID;
  if (bytes < ((uint64_t)1 << 20)) return fail(ctx, GTLS_E_INVALID, "chunk budget must be >= 1 MiB");
  ctx->chunk_budget = (size_t)bytes;
  return GTLS_OK;
}

int gtls_decode_status(int32_t word, char* msg, size_t cap) {
  std::string m;
  if (word == 0) m = "ok";
  if (word & 1) m += "chi2 kernel: shared-memory tile copy did not complete within its bounded wait";
  if (word & ~1) m += (m.empty() ? "" : "; ") + std::string("unknown device status bits ") + std::to_string(word & ~1);
  if (msg && cap > 0) {
    const size_t k = std::min(cap - 1, m.size());
    std::memcpy(msg, m.data(), k);
    msg[k] = 0;
  }
  return word == 0 ? GTLS_OK : GTLS_E_DEVICE;
}

const char* gtls_last_error(const gtls_ctx* ctx) {
  return ctx ? ctx->err.c_str() : g_create_error.c_str();
}

int gtls_ctx_create(int device, gtls_ctx** out) {
  if (!out) return fail(nullptr, GTLS_E_INVALID, "out is NULL");
  *out = nullptr;
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return fail(nullptr, GTLS_E_CUDA, std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
  if (device < 0 || device >= ndev) return fail(nullptr, GTLS_E_INVALID, "no such CUDA device");
  e = cudaSetDevice(device);
  if (e != cudaSuccess) return fail(nullptr, GTLS_E_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
  cudaDeviceProp prop;
  e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) return fail(nullptr, GTLS_E_CUDA, cudaGetErrorString(e));
  if (prop.major < 10) return fail(nullptr, GTLS_E_DEVICE, "gtls_b200 is built for sm_100a (B200)");
  gtls_ctx* c = new gtls_ctx();
  c->device = device;
  c->num_sms = prop.multiProcessorCount;
  c->smem_optin = (int)prop.sharedMemPerBlockOptin;
  if (cudaMalloc(&c->status, 64) != cudaSuccess) {
    delete c;
    return fail(nullptr, GTLS_E_NOMEM, "status word allocation failed");
  }
  cudaMemset(c->status, 0, 64);
  *out = c;
  return GTLS_OK;
}

int gtls_ctx_destroy(gtls_ctx* ctx) {
  if (!ctx) return GTLS_OK;
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  if (ctx->arena) cudaFree(ctx->arena);
  if (ctx->status) cudaFree(ctx->status);
  delete ctx;
  return GTLS_OK;
}

int gtls_period_grid(gtls_ctx* ctx, double a_over_3, double c, int64_t n_points, double period_min,
                     double period_max, double* periods_out, int64_t* count_out, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!periods_out || !count_out || n_points < 0 || n_points >= (1LL << 31))
    return fail(ctx, GTLS_E_INVALID, "bad arguments to gtls_period_grid");
  *count_out = 0;
  if (n_points == 0) return GTLS_OK;
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  size_t bytes = align_up(sizeof(double) * n_points, 256) + 256;
  void* mem = arena(ctx, bytes);
  if (!mem) return fail(ctx, GTLS_E_NOMEM, "scratch allocation failed");
  Carver cv(mem);
  double* tmp = cv.take<double>(n_points);
  int* bounds = cv.take<int>(2);
  int init[2] = {0x7fffffff, -1};
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(bounds, init, sizeof(init), cudaMemcpyHostToDevice, st));
  unsigned g = (unsigned)((n_points + 255) / 256);
  period_eval_kernel<<<g, 256, 0, st>>>(a_over_3, c, n_points, period_min, period_max, tmp, bounds);
  period_reverse_kernel<<<g, 256, 0, st>>>(tmp, bounds, periods_out);
  ctx->launches += 2;
  GTLS_TRY_CUDA(ctx, cudaGetLastError());
  int hb[2];
  GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(hb, bounds, sizeof(hb), cudaMemcpyDeviceToHost, st));
  GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
  *count_out = hb[1] >= hb[0] ? (int64_t)(hb[1] - hb[0] + 1) : 0;
  return GTLS_OK;
}

int gtls_spectra(gtls_ctx* ctx, const double* chi2, const uint8_t* mask, int64_t n, double oversampling_factor,
                 double* sr, double* power_raw, double* power, double* sde_raw, double* sde, void* stream) {
  if (!ctx) return GTLS_E_INVALID;
  if (!chi2 || !sr || !power_raw || !power || !sde_raw || !sde || n < 1)
    return fail(ctx, GTLS_E_INVALID, "bad arguments to gtls_spectra");
  double kd = oversampling_factor * 30;
  if (kd != std::floor(kd) || kd < 1) return fail(ctx, GTLS_E_INVALID, "oversampling_factor * 30 must be an integer");
  long long k = (long long)kd;
  if (k % 2 == 0) k += 1;
  GTLS_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  size_t bytes = align_up(sizeof(double) * n, 256) + align_up(sizeof(SpecState), 256) + 256;
  void* mem = arena(ctx, bytes);
  if (!mem) return fail(ctx, GTLS_E_NOMEM, "scratch allocation failed");
  Carver cv(mem);
  double* med = cv.take<double>(n);
  SpecState* dst = cv.take<SpecState>(1);
  spectra_raw_kernel<<<1, 1024, 0, st>>>(chi2, mask, n, sr, power_raw, dst);
  ctx->launches += 1;
  SpecState hs;
  if (n > 2 * k) {
    long long rows = n - k + 1;
    running_median_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(power_raw, mask, n, (int)k, med);
    median_pad_kernel<<<(unsigned)((n - rows + 255) / 256 + 1), 256, 0, st>>>(med, n, rows);
    spectra_final_kernel<<<1, 1024, 0, st>>>(power_raw, mask, med, n, power, dst);
    ctx->launches += 3;
    GTLS_TRY_CUDA(ctx, cudaGetLastError());
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(&hs, dst, sizeof(hs), cudaMemcpyDeviceToHost, st));
    GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    *sde = hs.sde;
  } else {
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(power, power_raw, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    GTLS_TRY_CUDA(ctx, cudaGetLastError());
    GTLS_TRY_CUDA(ctx, cudaMemcpyAsync(&hs, dst, sizeof(hs), cudaMemcpyDeviceToHost, st));
    GTLS_TRY_CUDA(ctx, cudaStreamSynchronize(st));
    *sde = hs.sde_raw;
  }
  *sde_raw = hs.sde_raw;
  return GTLS_OK;
}

}  // extern "C"
