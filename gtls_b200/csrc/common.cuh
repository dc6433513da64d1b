// Shared definitions of the gtls_b200 CUDA sources (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "gtls_b200.h"

struct gtls_ctx {
  int device = 0;
  int num_sms = 0;
  int smem_optin = 0;
  std::string err;
  void* arena = nullptr;       // scratch arena (grows on demand)
  size_t arena_bytes = 0;
  int* status = nullptr;       // device status word(s) written by kernels
  long long launches = 0;      // kernels launched through this context
  size_t chunk_budget = (size_t)8 << 30;   // per-chunk scratch of a search, bytes
  int tile_cap_fp32 = 16384;   // launch-shape tuning (gtls_set_tuning); results do not depend on it
  int tile_cap_fp64 = 8192;
  int bucket_shift = 0;
  int records_global = 0;      // 1: chi2 reads records from global memory for every curve
};

namespace gtls {

int fail(gtls_ctx* ctx, int code, const std::string& msg);
// Returns a device buffer of at least `bytes` from the context's arena
// (contents undefined, previous contents of the arena are not kept), or NULL.
void* arena(gtls_ctx* ctx, size_t bytes);

inline size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Carve consecutive 256-byte aligned sub-buffers out of one allocation.
struct Carver {
  char* base;
  size_t off = 0;
  explicit Carver(void* b) : base(static_cast<char*>(b)) {}
  template <typename T>
  T* take(size_t count) {
    off = align_up(off, 256);
    T* p = reinterpret_cast<T*>(base + off);
    off += count * sizeof(T);
    return p;
  }
};
template <typename T>
inline size_t carve_size(size_t& acc, size_t count) {
  acc = align_up(acc, 256) + count * sizeof(T);
  return acc;
}

}  // namespace gtls

#define GTLS_TRY_CUDA(ctx, call)                                                         \
  do {                                                                                   \
    cudaError_t e_ = (call);                                                             \
    if (e_ != cudaSuccess)                                                               \
      return gtls::fail((ctx), GTLS_E_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)
