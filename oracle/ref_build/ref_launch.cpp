/* CPU launcher for the reference's kernel source (src/gputls/GPUFun.cu).
 *
 * TEST INFRASTRUCTURE ONLY.  The kernel file is included from the reference
 * tree (after the SKIP_POINT substitution that core.py:597-601 applies at run
 * time), and each kernel the reference's host code launches gets an
 * `extern "C" ref_<name>(grid, block, args...)` entry that replays the launch
 * over every (block, thread) index, blocks spread over OpenMP threads.
 */
/* Compiled as: (reference kernel text; this file) | g++ -include cuda_host_shim.h -x c++ -
 * so the kernels are already declared when this part is read. */
thread_local gtls_ref_dim3 threadIdx, blockIdx, blockDim, gridDim;
#ifdef GTLS_REF_R64
extern "C" { double s_signal[1]; }
#else
extern "C" { float s_signal[1]; }
#endif

template <class F, class... A>
static void replay(int gx, int gy, int gz, int bx, int by, int bz, F f, A... a) {
  long nblk = (long)gx * gy * gz;
#pragma omp parallel for schedule(dynamic, 16)
  for (long b = 0; b < nblk; ++b) {
    gridDim = {gx, gy, gz};
    blockDim = {bx, by, bz};
    blockIdx = {(int)(b % gx), (int)((b / gx) % gy), (int)(b / ((long)gx * gy))};
    for (int tz = 0; tz < bz; ++tz)
      for (int ty = 0; ty < by; ++ty)
        for (int tx = 0; tx < bx; ++tx) {
          threadIdx = {tx, ty, tz};
          f(a...);
        }
  }
}

#define GRID int gx, int gy, int gz, int bx, int by, int bz
#define DIMS gx, gy, gz, bx, by, bz
extern "C" {
void ref_foldFast(GRID, const double* t, const double* p, double* ph, int* ps, int* ts) {
  replay(DIMS, foldFast, t, p, ph, ps, ts);
}
void ref_durationsGrid(GRID, const double* p, int* dmax, int* dmin, const float* len, const int* n, const int* np_) {
  replay(DIMS, durationsGrid, p, dmax, dmin, len, n, np_);
}
void ref_durationBool(GRID, int* dmax, int* dmin, const int* ds, const int* ps, const int* d, bool* out) {
  replay(DIMS, durationBool, dmax, dmin, ds, ps, d, out);
}
void ref_patchData(GRID, float* pd, float* pdy, int* m, int* si, int* maxd, float* fl, float* dy, int* n) {
  replay(DIMS, patchData, pd, pdy, m, si, maxd, fl, dy, n);
}
void ref_calcInverseSquaredPatchedDy(GRID, float* out, float* pdy, int* m) {
  replay(DIMS, calcInverseSquaredPatchedDy, out, pdy, m);
}
void ref_calcEdgeEffectCorrections(GRID, float* out, float* pd, float* inv, int* m, int* maxd, int* ps) {
  replay(DIMS, calcEdgeEffectCorrections, out, pd, inv, m, maxd, ps);
}
void ref_calcAllFullSum(GRID, float* fs, float* pd, float* inv, int* m, int* d, int* ds, int* ps) {
  replay(DIMS, calcAllFullSum, fs, pd, inv, m, d, ds, ps);
}
void ref_calcAllFullSum_v2(GRID, float* fs, float* eps, int m, int* d, int ds, int ps) {
  replay(DIMS, calcAllFullSum_v2, fs, eps, m, d, ds, ps);
}
void ref_step1(GRID, float* tmp, float* pd, int* d, int* ds, float* inv, int* m, int* rx) {
  replay(DIMS, calcAllOutOfTransitResiduals_step1_2GPU, tmp, pd, d, ds, inv, m, rx);
}
void ref_step2(GRID, float* ootr, int* ds, int* m, int* d, int* rx, float* fs) {
  replay(DIMS, calcAllOutOfTransitResiduals_step2_2GPU, ootr, ds, m, d, rx, fs);
}
void ref_calculate_base_error(GRID, float* out, const float* pd, const float* inv, int m, int np_) {
  replay(DIMS, calculate_base_error, out, pd, inv, m, np_);
}
void ref_calculate_final_ootr_v3(GRID, float* out, const float* eps, const float* fs, const int* d,
                                 int n, int m, int ds, int np_) {
  replay(DIMS, calculate_final_ootr_v3, out, eps, fs, d, n, m, ds, np_);
}
void ref_lowest_v2(GRID, float* out, int* rx, float* pd, int* m, int* d, int* ds, float* sig, int* msx,
                   float* inv, float* os, float* ootr, float* fs, float* edge, int* dp, float* cs, float* dmin) {
  replay(DIMS, calcAllLowestResidualsGPUB_SignalTiled_v2, out, rx, pd, m, d, ds, sig, msx, inv, os, ootr,
         fs, edge, dp, cs, dmin);
}
void ref_lowest_noskip(GRID, float* out, int* rx, float* pd, int* m, int* d, int* ds, float* sig, int* msx,
                       float* inv, float* os, float* ootr, float* fs, float* edge, int* dp, float* cs,
                       int* dmx, int* dmn, float* dmin) {
  replay(DIMS, calcAllLowestResidualsGPUBNoSkip, out, rx, pd, m, d, ds, sig, msx, inv, os, ootr, fs, edge,
         dp, cs, dmx, dmn, dmin);
}
void ref_lowest_noskip_temp(GRID, float* out, int* rx, float* pd, int* m, int* d, int* ds, float* sig,
                            int* msx, float* inv, float* os, float* ootr, float* fs, float* edge, int* dp,
                            float* cs, float* dmin) {
  replay(DIMS, calcAllLowestResidualsGPUBNoSkipTemp, out, rx, pd, m, d, ds, sig, msx, inv, os, ootr, fs,
         edge, dp, cs, dmin);
}
}
