/*
 * gtls_b200 -- C-ABI of the B200-native Transit Least Squares search.
 *
 * Every buffer argument is a DEVICE pointer owned by the caller unless the
 * comment says "host".  Every call is asynchronous on the given stream
 * (cudaStream_t passed as void*; NULL = the legacy default stream) except
 * where it says it synchronises.  Every call returns 0 on success and a
 * GTLS_E_* code otherwise; gtls_last_error() gives the message.  No C++
 * exception crosses this interface.  A context belongs to one device and
 * must not be used from two host threads at once.  Its calls share one
 * scratch arena: calls on one context that go to different streams must be
 * ordered by the caller (an event or a synchronisation between them); calls
 * on one stream are ordered by the stream.  Use one context per concurrent
 * stream for overlapping searches.
 *
 * These entry points replace the reference's cupy RawModule kernel launches
 * and their host glue (reference file:line given per function).
 */
#ifndef GTLS_B200_H
#define GTLS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GTLS_ABI_VERSION 2

enum gtls_status {
  GTLS_OK = 0,
  GTLS_E_INVALID = 1,   /* bad argument (size, pointer, mode)            */
  GTLS_E_CUDA = 2,      /* a CUDA runtime call failed                    */
  GTLS_E_NOMEM = 3,     /* scratch allocation failed                     */
  GTLS_E_RANGE = 4,     /* input outside the supported range             */
  GTLS_E_DEVICE = 5     /* a kernel reported an error through its status word */
};

enum gtls_precision {
  GTLS_FP64 = 0,        /* plain FP64 chi2                                */
  GTLS_FP32 = 1         /* FP32 chi2, compensated FP32 prefix sums, FP64 baseline */
};

enum gtls_pass {
  GTLS_PASS_MAIN = 0,   /* starts k with k % skip == 0 (GPUFun.py:402,409) */
  GTLS_PASS_ALL = 1     /* every start (GPUFun.py:646-695, 819-873)         */
};

typedef struct gtls_ctx gtls_ctx;

/* Create / destroy a context on CUDA device `device`.  The context owns the
 * scratch arena the searches use. */
int gtls_ctx_create(int device, gtls_ctx** out);
int gtls_ctx_destroy(gtls_ctx* ctx);

/* Message of the last failed call on this context (or of the last failed
 * gtls_ctx_create when ctx is NULL).  Never NULL. */
const char* gtls_last_error(const gtls_ctx* ctx);

/* ABI version compiled into the library (GTLS_ABI_VERSION). */
int gtls_abi_version(void);

/* Meaning of a search's device status word (no counterpart in the
 * reference, whose kernels have no error path).  The search kernels set bits
 * of a per-context word instead of hanging: bit 0 = a chi2 CTA's
 * shared-memory tile copy did not complete within its bounded wait (the CTA
 * then waited, bounded again, for the copy in flight, evaluated nothing and
 * left its period's minimum at +inf).  Returns GTLS_OK for 0 and
 * GTLS_E_DEVICE otherwise, and writes a NUL-terminated message of at most
 * `cap` bytes to `msg` (host; msg may be NULL). */
int gtls_decode_status(int32_t word, char* msg, size_t cap);

/* Number of kernels this context has launched since it was created
 * (no counterpart in the reference; used to account for device work). */
int64_t gtls_launch_count(const gtls_ctx* ctx);

/* Bytes of per-chunk scratch a search may use (fold records, prefix sums,
 * sort slots; default 8 GiB).  Periods are processed in chunks that fit it;
 * results do not depend on it.  No counterpart in the reference, whose
 * batch size comes from the free-memory formula of core.py:620-628.
 * bytes must be >= 1 MiB. */
int gtls_set_chunk_budget(gtls_ctx* ctx, uint64_t bytes);

/* Launch-shape parameters of the searches on a context (no counterpart in
 * the reference).  None changes a result: chi2 values and argmin locations
 * are the same for every setting; only the time differs, so a caller (or
 * gtls_b200.tune) may time a few settings on its own data and keep the
 * fastest.  A zero field means the default. */
typedef struct gtls_tuning {
  int32_t tile_cap_fp32;      /* max starts per chi2 tile (CTA), FP32 form: a multiple of 256 in
                                 [256, 65536], or 0 = 16384.  The shared-memory size caps it too. */
  int32_t tile_cap_fp64;      /* the same for the FP64 form, 0 = 8192                        */
  int32_t bucket_shift;       /* phase buckets of the global-scatter fold ordering (curves above
                                 2^17 samples, and periods whose phases cluster beyond what the
                                 shared-memory ordering holds) = 2^min(15, ceil(log2 N) + shift),
                                 shift in [-3, 0] (0 = default)                               */
  int32_t records_global;     /* 1: the main pass's chi2 kernel reads the folded records from
                                 global memory (L1/L2) for every curve; 0: from a shared-memory
                                 tile when the curve's longest duration leaves room for one
                                 (default).  The all-starts pass always uses the tile when it fits */
} gtls_tuning;

int gtls_set_tuning(gtls_ctx* ctx, const gtls_tuning* tuning);
int gtls_get_tuning(const gtls_ctx* ctx, gtls_tuning* tuning);

/*
 * Ofir-optimal period grid, evaluated on the device.
 * Replaces the per-point part of grid.period_grid (grid.py:126-137):
 * P(X) = 1 / (a_over_3 * X + c)^3 / 86400 for X = 1..n_points, keeping
 * period_min < P <= period_max.  Writes the kept periods in ASCENDING order
 * (main.py:75 sorts them) to periods_out (capacity n_points) and their count
 * to *count_out (host).  Synchronises the stream.
 */
int gtls_period_grid(gtls_ctx* ctx, double a_over_3, double c, int64_t n_points,
                     double period_min, double period_max, double* periods_out,
                     int64_t* count_out, void* stream);

/*
 * Per-period duration range in samples.  Replaces the durationsGrid kernel
 * (GPUFun.py:47-86): wmin = floor(min(T14min/P, 0.15) * n_samples),
 * wmax = ceil(min(T14max/P, 0.15) * n_samples * (span/P + 1)/(span/P)),
 * with the time span given as float (as _worker.py:107 passes it).
 */
int gtls_duration_ranges(gtls_ctx* ctx, const double* periods, int64_t n_periods, float span,
                         int32_t n_samples, int32_t* wmin, int32_t* wmax, void* stream);

/*
 * The stable fold ordering of a light curve for each of n_periods trial
 * periods: order_out[p * n + j] = index of the sample at sorted position j
 * of period p, sorting by phase = t/P - (int)(t/P) (foldFast,
 * GPUFun.py:30-41) with ties kept in index order.  Replaces the cupy
 * argsort of the folded phases (core.py:775-777); gtls_search computes the
 * same ordering internally.  order_out: device, n_periods * n int32.
 * Requires t >= 0 and max(t) / min(period) < 2^31 (the fold's int
 * truncation, as in the reference).  Synchronises the stream.
 */
int gtls_fold_order(gtls_ctx* ctx, const double* t, int32_t n, const double* periods, int64_t n_periods,
                    int32_t* order_out, void* stream);

/* Stage times of one gtls_search call, measured with CUDA events on the
 * call's stream (filled only when gtls_search_desc.timing is non-NULL; the
 * call then synchronises the stream before returning). */
typedef struct gtls_timing {
  int32_t chunks;             /* period chunks (one prepare + chi2 launch each) */
  int32_t reserved;
  double setup_ms;            /* curve set-up, duration ranges, unions, template rows */
  double prepare_ms;          /* fold + ranking + gather + prefix, all chunks   */
  double chi2_ms;             /* chi2 kernel, all chunks                        */
  double finish_ms;           /* per-period minimum, all chunks                 */
  int64_t chi2_starts;        /* (duration, start) evaluations done by the chi2 kernel */
  int64_t chi2_fma;           /* multiply-adds of B and C over every evaluated start
                                 (2 * width per start, whether or not its window
                                 passes the depth test)                          */
  int64_t chi2_active_fma;    /* the same over the starts whose window mean passes
                                 the depth test: the only starts whose sums enter
                                 the result (the reference's in-transit loop runs
                                 for these alone, GPUFun.py:409-424)            */
  int64_t chi2_issued_fma;    /* multiply-adds the kernel performed (register
                                 groups of consecutive starts, padded template
                                 blocks included)                                */
} gtls_timing;

/*
 * One light curve's search over a list of trial periods.  Replaces the batch
 * loop of core.search_multi_periods (core.py:691-875), of
 * core.search_multi_periods_again (core.py:1081-1237) and the chi2 part of
 * core.search_single_periods (core.py:1292-1418).
 *
 * For every period p the durations searched are those d with
 * wmin(q) <= widths[d] <= wmax(q) for at least one period q of p's batch
 * (consecutive groups of `batch` periods; the reference's per-batch union,
 * core.py:693-716).  chi2_out[p] is the minimum over (duration, start) of
 *   - the template chi2 of the window of `widths[d]` folded samples starting
 *     at k, when the window's mean depth exceeds depth_min and (pass MAIN)
 *     k % skip(d) == 0 with skip(d) = widths[d] / skip_point if
 *     widths[d] > skip_point else 1;
 *   - n (the sample count) otherwise (GPUFun.py:407,437).
 * loc_out[p] = d_pos * n + k of the first minimum, d_pos counting the
 * batch's durations in ascending width.  A batch with no duration gets NaN
 * and loc -1 (core.py:722-729).
 */
typedef struct gtls_search_desc {
  int32_t abi_version;        /* GTLS_ABI_VERSION                               */
  int32_t precision;          /* gtls_precision                                 */
  int32_t pass;               /* gtls_pass                                      */
  int32_t n;                  /* samples                                        */
  const double* t;            /* [n] times, days, finite and > 0                */
  const double* y;            /* [n] flux                                       */
  const double* dy;           /* [n] flux uncertainty, > 0                      */
  int64_t n_periods;
  const double* periods;      /* [n_periods] days, > 0                          */
  int32_t n_durations;        /* D, <= GTLS_MAX_DURATIONS                       */
  int32_t max_width;          /* maxDuration (core.py:608-612): max width, made even */
  const int32_t* widths;      /* [D] ascending, >= 1, <= max_width              */
  const double* overshoot;    /* [D]                                            */
  const double* templates;    /* [D * max_width] row d: 1 - template (core.py:753-754) */
  double depth_min;           /* transit_depth_min                              */
  int32_t skip_point;         /* int(1/T0_fit_margin) or 0x7f800000             */
  int32_t batch;              /* periods per duration-union batch, >= 1         */
  float span;                 /* max(t) - min(t) as float                       */
  int32_t flags;              /* 0, or GTLS_SEARCH_ALL_DURATIONS                */
  double* chi2_out;           /* [n_periods]                                    */
  int64_t* loc_out;           /* [n_periods] or NULL                            */
  gtls_timing* timing;        /* host, or NULL                                  */
} gtls_search_desc;

#define GTLS_MAX_DURATIONS 1024

/* flags: search every given duration for every period, instead of the
 * durations valid for at least one period of its batch.  With it a caller
 * re-searches a few periods of a batch with that batch's own duration union
 * (computed from all its periods), e.g. to re-check candidates in another
 * precision.  No counterpart in the reference. */
#define GTLS_SEARCH_ALL_DURATIONS 1

int gtls_search(gtls_ctx* ctx, const gtls_search_desc* desc, void* stream);

/*
 * Many light curves searched in one call (the batched survey case: one
 * independent search per curve, as a loop of gtls_search calls would do, with
 * the prepare/chi2/finish launches shared by all curves).  No counterpart in
 * the reference, which searches one curve per gtls() object.  Curve c owns
 *   samples   [sample_off[c], sample_off[c+1])  of t, y, dy
 *   periods   [period_off[c], period_off[c+1])  of periods, chi2_out, loc_out
 *   durations [dur_off[c], dur_off[c+1])        of widths, overshoot
 *   templates starting at tmpl_off[c], (dur_off[c+1]-dur_off[c]) * max_width[c] values
 * and its own max_width, batch and span (host arrays of n_curves values);
 * offsets are host arrays of n_curves + 1 values.  Results per curve are the
 * ones gtls_search gives for that curve alone.  timing, when non-NULL, sums
 * over all curves.
 */
typedef struct gtls_batch_desc {
  int32_t abi_version;        /* GTLS_ABI_VERSION                               */
  int32_t precision;          /* gtls_precision                                 */
  int32_t pass;               /* gtls_pass                                      */
  int32_t n_curves;
  const int64_t* sample_off;  /* host [n_curves + 1]                            */
  const int64_t* period_off;  /* host [n_curves + 1]                            */
  const int64_t* dur_off;     /* host [n_curves + 1]                            */
  const int64_t* tmpl_off;    /* host [n_curves]                                */
  const int32_t* max_width;   /* host [n_curves]                                */
  const int32_t* batch;       /* host [n_curves]                                */
  const float* span;          /* host [n_curves]                                */
  const double* t;            /* device, all curves' samples                    */
  const double* y;
  const double* dy;
  const double* periods;      /* device, all curves' periods                    */
  const int32_t* widths;      /* device, all curves' durations                  */
  const double* overshoot;
  const double* templates;    /* device, all curves' template rows              */
  double depth_min;
  int32_t skip_point;
  int32_t flags;              /* 0, or GTLS_SEARCH_ALL_DURATIONS                */
  double* chi2_out;           /* device, all curves' periods                    */
  int64_t* loc_out;           /* device or NULL                                 */
  gtls_timing* timing;        /* host, or NULL                                  */
} gtls_batch_desc;

int gtls_search_batch(gtls_ctx* ctx, const gtls_batch_desc* desc, void* stream);

/*
 * Spectra of a chi2 array (stats.spectra, stats.py:95-122, with the
 * running median of helpers.py:91-106).  mask may be NULL (nothing masked);
 * masked entries are left out of every min/mean/std/max/median as numpy.ma
 * does.  Outputs sr, power_raw, power: [n]; sde_raw and sde: host scalars.
 * kernel = oversampling_factor * 30, made odd.  Synchronises the stream.
 */
int gtls_spectra(gtls_ctx* ctx, const double* chi2, const uint8_t* mask, int64_t n,
                 double oversampling_factor, double* sr, double* power_raw, double* power,
                 double* sde_raw, double* sde, void* stream);

/*
 * Transit template tables for many light curves, built on the device the
 * way the reference builds its template cache on the host
 * (transit.py:8-160: reference_transit, fractional_transit, get_cache,
 * through core.py:753-754's 1 - pad(template)).  The template planet (a
 * circular orbit of period `per` days, radius rp and semi-major axis a in
 * stellar radii, inclination `inc` degrees, quadratic limb darkening u1, u2;
 * the reference's "default", "grazing" and "box" templates are parameter
 * sets of it) is sampled on 10,000 points over one day with the limb-darkened
 * occultation integral (batman in the reference), trimmed to its in-transit
 * part, interpolated to each curve's `samples` (its maximum template width)
 * and rescaled; for every row r of curve c (widths[r], ascending unique
 * widths in [1, samples[c]]) it is squeezed to widths[r] samples, scaled to
 * depth 0.5 and trimmed to the samples below 1 - 1e-8.  Outputs (device):
 * overshoot[r] = 1 / (2 - mean / min) of the trimmed template, and the row
 * 1 - template padded with 1 to row_len[c] values at
 * templates[tmpl_off[c] + (r - row_off[c]) * row_len[c]].  Fails with
 * GTLS_E_INVALID if a row has no sample below 1 - 1e-8.  Synchronises the
 * stream.
 */
typedef struct gtls_template_desc {
  int32_t abi_version;        /* GTLS_ABI_VERSION                               */
  int32_t n_curves;
  double per, rp, a, inc;     /* template planet (days, stellar radii, degrees) */
  double u1, u2;              /* quadratic limb darkening (linear: u2 = 0)      */
  const int32_t* samples;     /* host [n_curves]: max template width, >= 2      */
  const int64_t* row_off;     /* host [n_curves + 1]: rows of curve c           */
  const int32_t* widths;      /* host [rows]: template width of each row        */
  const int64_t* tmpl_off;    /* host [n_curves]: offset of curve c's rows      */
  const int32_t* row_len;     /* host [n_curves]: row length, >= samples[c]     */
  double* overshoot;          /* device [rows] out                              */
  double* templates;          /* device out                                     */
} gtls_template_desc;

int gtls_template_cache(gtls_ctx* ctx, const gtls_template_desc* desc, void* stream);

/*
 * Chi2 of the unfolded limb-darkened transit model and its gradient, for
 * n_curves light curves concatenated in t/y/w (curve c owns samples
 * curve_off[c] .. curve_off[c+1]-1, w = 1/dy^2).  params[6c..6c+5] =
 * (P, T0, D, depth, u1, u2) of curve c.  An addition with no counterpart in
 * the reference, used to refine a search peak below grid resolution.
 * Model: the search's template model, a central (impact parameter 0)
 * circular-orbit transit of an opaque disk across a star with quadratic limb
 * darkening I = 1 - u1 (1-mu) - u2 (1-mu)^2: K = 1 - u1/3 - u2/6,
 * p = sqrt(depth K), a = (1 + p) / sin(pi D / P),
 * phi = 2 pi ((t-T0)/P - round((t-T0)/P)), z = a |sin phi| (no occultation
 * when cos phi < 0), m = 1 - (occulted flux at separation z) / (pi K), the
 * occulted flux integrated over annuli with 96-node Gauss-Legendre
 * quadrature after r = m + h sin(theta) (the template generator's own
 * quadrature).  D is the first-to-fourth-contact duration, depth the central
 * depth.  gtls_model_chi2_grad writes grad_params[6c+k] =
 * grad_chi2[c] * dchi2_c/dparam_k, the exact derivative of that discrete
 * formula, recomputing the model instead of storing it.
 */
int gtls_model_chi2(gtls_ctx* ctx, const double* t, const double* y, const double* w,
                    const int64_t* curve_off, int32_t n_curves, const double* params,
                    double* chi2_out, void* stream);
int gtls_model_chi2_grad(gtls_ctx* ctx, const double* t, const double* y, const double* w,
                         const int64_t* curve_off, int32_t n_curves, const double* params,
                         const double* grad_chi2, double* grad_params, void* stream);

/*
 * Allocation-free spectra (no counterpart in the reference: the reference
 * always allocates through cupy's memory pool).
 *
 * For callers that cannot call cudaMalloc when they compute the SDE: code
 * running under a fixed memory budget owned by another framework, real-time
 * loops that forbid allocator calls after start-up, or callers without a
 * gtls context (creating one allocates).  Same inputs, outputs and results as
 * gtls_spectra; runs on the current device, needs no context, and calls no
 * allocator: its scratch is a static device array of
 * GTLS_NOALLOC_SCRATCH_BYTES that every GPU loading the library holds until
 * exit.  Limits and rules:
 *   - n <= GTLS_NOALLOC_MAX_PERIODS, else GTLS_E_RANGE (nothing launched);
 *   - all calls on a device share the scratch array, so calls that overlap
 *     on the GPU race; each call writes every scratch value it reads;
 *   - the first call on a device looks up the array's address (and loads the
 *     library's device code there): make it before any stream capture;
 *   - that address is kept for the life of the process: do not call it on a
 *     device after a cudaDeviceReset of that device (the array may then sit
 *     at another address);
 *   - synchronises the stream; errors are described by
 *     gtls_noalloc_last_error() (thread-local).
 */
#define GTLS_NOALLOC_MAX_PERIODS (1 << 20)
#define GTLS_NOALLOC_SCRATCH_BYTES ((size_t)8 * 1024 * 1024 + 256)

int gtls_spectra_noalloc(const double* chi2, const uint8_t* mask, int64_t n, double oversampling_factor,
                         double* sr, double* power_raw, double* power, double* sde_raw, double* sde,
                         void* stream);
const char* gtls_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* GTLS_B200_H */
