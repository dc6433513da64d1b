// Spectra kernels (defined in capi.cu), shared with the allocation-free entry point.
#pragma once
#include <cstdint>

namespace gtls {

struct SpecState {
  double mean_sr, std_sr, sde_raw, scale_raw;
  double sde;
  int count;
  int has_median;
};

__global__ void spectra_raw_kernel(const double* __restrict__ chi2, const uint8_t* __restrict__ mask, long long n,
                                   double* __restrict__ sr, double* __restrict__ praw, SpecState* st);
__global__ void running_median_kernel(const double* __restrict__ praw, const uint8_t* __restrict__ mask,
                                      long long n, int k, double* __restrict__ med);
__global__ void median_pad_kernel(double* med, long long n, long long rows);
__global__ void spectra_final_kernel(const double* __restrict__ praw, const uint8_t* __restrict__ mask,
                                     const double* __restrict__ med, long long n, double* __restrict__ power,
                                     SpecState* st);

}  // namespace gtls
