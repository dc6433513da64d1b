// gtls_spectra_noalloc: the spectra/SDE computation with no device allocation.
//
// Who needs it: code that must not call cudaMalloc at the point where it
// computes a periodogram's SDE -- for example a host application that runs
// inside a strict memory budget handed out by another framework's pool, a
// real-time pipeline that forbids allocator calls (and the device-wide
// synchronisation cudaFree implies) after start-up, or a caller that cannot
// create a gtls context (context creation itself allocates).  Such callers
// pass their own input and output buffers; the one scratch array the
// computation needs (the running median, plus a small state record) lives in
// the file-scope device array below instead of being allocated.
//
// Costs and limits of that choice:
//  * the array is part of this library's device image, so every GPU that
//    loads the library holds GTLS_NOALLOC_SCRATCH_BYTES until the process exits;
//  * at most GTLS_NOALLOC_MAX_PERIODS periods per call; larger inputs are
//    rejected with GTLS_E_RANGE before anything is launched;
//  * all calls on one device share the array: calls that overlap on the GPU
//    (different streams, or different host threads) race on it.  Every value
//    read from it is written first by the same call, so nothing needs zeroing
//    between calls;
//  * the first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, which also loads the module on that device); make
//    that first call before any stream capture on the device.  The address is
//    kept for the life of the process, so the entry point must not be used on
//    a device after a cudaDeviceReset of it (the module, and the array with
//    it, may then be loaded at another address).
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <string>

#include "common.cuh"
#include "spectra.cuh"

namespace gtls {
namespace {

constexpr size_t kMedBytes = sizeof(double) * (size_t)GTLS_NOALLOC_MAX_PERIODS;
constexpr size_t kStateOff = (kMedBytes + 255) / 256 * 256;
static_assert(kStateOff + sizeof(SpecState) <= GTLS_NOALLOC_SCRATCH_BYTES, "scratch too small");

__device__ __align__(256) unsigned char g_noalloc_scratch[GTLS_NOALLOC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;
std::atomic<void*> g_scratch_ptr[kMaxDevices];
std::mutex g_setup_mutex;
thread_local std::string g_noalloc_error;

int noalloc_fail(int code, const std::string& msg) {
  g_noalloc_error = msg;
  return code;
}

// Device address of the scratch array on the current device (set up once per device).
int scratch_on_current_device(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(GTLS_E_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return noalloc_fail(GTLS_E_RANGE, "device index too large");
  void* p = g_scratch_ptr[dev].load(std::memory_order_acquire);
  if (!p) {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    p = g_scratch_ptr[dev].load(std::memory_order_acquire);
    if (!p) {
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess || !p)
        return noalloc_fail(GTLS_E_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_ptr[dev].store(p, std::memory_order_release);
    }
  }
  *out = p;
  return GTLS_OK;
}

}  // namespace
}  // namespace gtls

using namespace gtls;

extern "C" const char* gtls_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

extern "C" int gtls_spectra_noalloc(const double* chi2, const uint8_t* mask, int64_t n, double oversampling_factor,
                                    double* sr, double* power_raw, double* power, double* sde_raw, double* sde,
                                    void* stream) {
  if (!chi2 || !sr || !power_raw || !power || !sde_raw || !sde || n < 1)
    return noalloc_fail(GTLS_E_INVALID, "bad arguments to gtls_spectra_noalloc");
  if (n > GTLS_NOALLOC_MAX_PERIODS)
    return noalloc_fail(GTLS_E_RANGE, "gtls_spectra_noalloc: n = " + std::to_string(n) +
                                          " exceeds GTLS_NOALLOC_MAX_PERIODS = " +
                                          std::to_string((long long)GTLS_NOALLOC_MAX_PERIODS));
  const double kd = oversampling_factor * 30;
  if (kd != std::floor(kd) || kd < 1)
    return noalloc_fail(GTLS_E_INVALID, "oversampling_factor * 30 must be an integer");
  long long k = (long long)kd;
  if (k % 2 == 0) k += 1;
  void* base = nullptr;
  int rc = scratch_on_current_device(&base);
  if (rc != GTLS_OK) return rc;
  double* med = static_cast<double*>(base);
  SpecState* dst = reinterpret_cast<SpecState*>(static_cast<unsigned char*>(base) + kStateOff);
  cudaStream_t st = static_cast<cudaStream_t>(stream);

  spectra_raw_kernel<<<1, 1024, 0, st>>>(chi2, mask, n, sr, power_raw, dst);
  SpecState hs;
  cudaError_t e;
  if (n > 2 * k) {
    long long rows = n - k + 1;
    running_median_kernel<<<(unsigned)((rows + 127) / 128), 128, 0, st>>>(power_raw, mask, n, (int)k, med);
    median_pad_kernel<<<(unsigned)((n - rows + 255) / 256 + 1), 256, 0, st>>>(med, n, rows);
    spectra_final_kernel<<<1, 1024, 0, st>>>(power_raw, mask, med, n, power, dst);
  } else {
    e = cudaMemcpyAsync(power, power_raw, sizeof(double) * n, cudaMemcpyDeviceToDevice, st);
    if (e != cudaSuccess) return noalloc_fail(GTLS_E_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(GTLS_E_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  e = cudaMemcpyAsync(&hs, dst, sizeof(hs), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return noalloc_fail(GTLS_E_CUDA, std::string("readback: ") + cudaGetErrorString(e));
  *sde_raw = hs.sde_raw;
  *sde = n > 2 * k ? hs.sde : hs.sde_raw;
  return GTLS_OK;
}
