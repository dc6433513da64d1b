/* Host (CPU) stand-ins for the few CUDA built-ins that the reference's kernel
 * source uses, so that the unmodified kernel file compiles with g++ and every
 * launch can be replayed on the CPU block by block, thread by thread.
 *
 * TEST INFRASTRUCTURE ONLY: it builds the checker (oracle/_ref), never the
 * product.  The kernels replayed through it use neither shared memory nor
 * barriers, so a sequential replay of each thread computes exactly what each
 * GPU thread computes (minus the FMA contraction nvcc applies on the GPU).
 *
 * With GTLS_REF_R64 defined, `float` is redefined to `double` for the kernel
 * source that follows: the "R64" variant (every float promoted to double,
 * which is what the reference's float64 host buffers intend).
 */
#pragma once
#include <cmath>
#include <cstdint>
#include <cstring>

struct gtls_ref_dim3 { int x, y, z; };
extern thread_local gtls_ref_dim3 threadIdx, blockIdx, blockDim, gridDim;

#define __global__
#define __device__
#define __host__
#define __shared__
#define __restrict__
#define __syncthreads() ((void)0)
template <class T> static inline T __ldg(const T* p) { return *p; }

#ifdef GTLS_REF_R64
extern "C" { extern double s_signal[]; }
#define float double
#else
extern "C" { extern float s_signal[]; }
#endif
using std::pow; using std::floor; using std::ceil; using std::fmaf;
