/* Launchers for the reference's kernel source (src/gputls/GPUFun.cu) compiled
 * for sm_100a -- BASELINE INFRASTRUCTURE ONLY (the "reference kernels on the
 * same GPU" leg of bench.py; nothing in gtls_b200 loads it).
 *
 * The reference file is included from the reference tree (REF_GPUFUN, set by
 * oracle/Makefile); its kernels keep their own text and SKIP_POINT 8, the
 * value core.py:597-601 substitutes for the default T0_fit_margin of 0.125.
 * Each launcher takes the grid and block the reference's host code uses
 * (_worker.py:100-300, the type-consistent caller) and a CUDA stream, and
 * returns the launch's cudaError_t.
 */
#include <cuda_runtime.h>

#include REF_GPUFUN

#define REF_GRID int gx, int gy, int gz, int bx, void *stream
#define REF_LAUNCH(k) k<<<dim3(gx, gy, gz), dim3(bx, 1, 1), 0, (cudaStream_t)stream>>>

extern "C" {
int refgpu_foldFast(REF_GRID, const double *t, const double *p, double *ph, int *ps, int *ts) {
  REF_LAUNCH(foldFast)(t, p, ph, ps, ts);
  return (int)cudaGetLastError();
}
int refgpu_durationsGrid(REF_GRID, const double *p, int *dmax, int *dmin, float *len, int *n, int *np_) {
  REF_LAUNCH(durationsGrid)(p, dmax, dmin, len, n, np_);
  return (int)cudaGetLastError();
}
int refgpu_durationBool(REF_GRID, int *dmax, int *dmin, int *ds, int *ps, int *d, bool *out) {
  REF_LAUNCH(durationBool)(dmax, dmin, ds, ps, d, out);
  return (int)cudaGetLastError();
}
int refgpu_patchData(REF_GRID, float *pd, float *pdy, int *m, int *si, int *maxd, float *fl, float *dy, int *n) {
  REF_LAUNCH(patchData)(pd, pdy, m, si, maxd, fl, dy, n);
  return (int)cudaGetLastError();
}
int refgpu_calcInverseSquaredPatchedDy(REF_GRID, float *out, float *pdy, int *m) {
  REF_LAUNCH(calcInverseSquaredPatchedDy)(out, pdy, m);
  return (int)cudaGetLastError();
}
int refgpu_calcEdgeEffectCorrections(REF_GRID, float *out, float *pd, float *inv, int *m, int *maxd, int *ps) {
  REF_LAUNCH(calcEdgeEffectCorrections)(out, pd, inv, m, maxd, ps);
  return (int)cudaGetLastError();
}
int refgpu_calculate_base_error(REF_GRID, float *out, const float *pd, const float *inv, int m, int np_) {
  REF_LAUNCH(calculate_base_error)(out, pd, inv, m, np_);
  return (int)cudaGetLastError();
}
int refgpu_calcAllFullSum_v2(REF_GRID, float *fs, float *eps, int m, int *d, int ds, int ps) {
  REF_LAUNCH(calcAllFullSum_v2)(fs, eps, m, d, ds, ps);
  return (int)cudaGetLastError();
}
int refgpu_calculate_final_ootr_v3(REF_GRID, float *out, const float *eps, const float *fs, const int *d, int n,
                                   int m, int ds, int np_) {
  REF_LAUNCH(calculate_final_ootr_v3)(out, eps, fs, d, n, m, ds, np_);
  return (int)cudaGetLastError();
}
int refgpu_lowest_v2(REF_GRID, float *out, int *rx, float *pd, int *m, int *d, int *ds, float *sig, int *msx,
                     float *inv, float *os, float *ootr, float *fs, float *edge, int *dp, float *cs, float *dmin) {
  REF_LAUNCH(calcAllLowestResidualsGPUB_SignalTiled_v2)(out, rx, pd, m, d, ds, sig, msx, inv, os, ootr, fs, edge,
                                                        dp, cs, dmin);
  return (int)cudaGetLastError();
}
}
