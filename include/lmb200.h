/*
 * lmb200 -- B200 (sm_100a) Lorenz-Mie holography kernels behind a C ABI.
 *
 * Plain C entry points: device pointers, sizes and a cudaStream_t passed
 * as void*.  Every function returns an int status (LMB_OK = 0) and never
 * throws, traps or spin-waits.  All arrays are device memory unless a
 * parameter says "host".  Calls on one stream are ordered; the library
 * keeps no hidden state between calls except what is named here.
 *
 * Units follow the reference: pixel coordinates and particle positions in
 * pixels, radii and wavelength in micrometres, magnification in
 * micrometres per pixel, the wave number k in radians per pixel.
 */
#ifndef LMB200_H
#define LMB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define LMB_OK 0
#define LMB_ERR_ARG 1          /* invalid argument (null pointer, bad size) */
#define LMB_ERR_CUDA 2         /* a CUDA runtime call failed */
#define LMB_ERR_NMAX 3         /* a sphere needs more orders than nmax_cap */
#define LMB_ERR_WORKSPACE 4    /* workspace too small */
#define LMB_ERR_UNSUPPORTED 5  /* flag combination not supported */
#define LMB_ERR_TIMEOUT 6      /* streamed fit: data did not arrive in time */

/* flags */
#define LMB_CARTESIAN 1   /* project the field on x, y, z (else r, theta, phi) */
#define LMB_BOHREN 2      /* Bohren & Huffman sign convention */
#define LMB_FP64 4        /* compute the field sum in FP64 (else FP32) */

/* Largest number of partial-wave orders any entry point accepts. */
#define LMB_NMAX_LIMIT 1024

/*
 * A homogeneous sphere: position (pixels), radius a_p (um), refractive
 * index n_p and absorption k_p.  Same six properties, same order, as
 * Sphere.properties (theory/Sphere.py:63-68, theory/Particle.py:91-95).
 */
typedef struct lmb_sphere {
  double x_p, y_p, z_p, a_p, n_p, k_p;
} lmb_sphere;

/* Library version as major*10000 + minor*100 + patch. */
int lmb_version(void);

/* Human-readable text of a status code (static storage). */
const char *lmb_status_string(int status);

/*
 * Mie coefficients of nspheres homogeneous spheres, FP64.
 * Replaces Sphere.ab / Sphere.mie_coefficients (theory/Sphere.py:70-89,
 * 147-226) and Sphere.wiscombe_yang (:91-123).
 *   ab    [nspheres][nmax_cap+1][2] complex128 (interleaved re, im):
 *         ab[s][n][0] = a_n, ab[s][n][1] = b_n, row 0 and rows above
 *         nmax[s] are zero.
 *   dab   optional (may be NULL): [nspheres][nmax_cap+1][4] complex128,
 *         d a_n/d a_p, d b_n/d a_p, d a_n/d n_p, d b_n/d n_p.
 *   nmax  [nspheres] int: number of orders (the reference's nmax;
 *         norders = nmax + 1).
 *   status [nspheres] int: LMB_OK or LMB_ERR_NMAX.
 */
int lmb_sphere_ab(const lmb_sphere *spheres, int nspheres, double n_m,
                  double wavelength, int nmax_cap, double *ab, double *dab,
                  int *nmax, int *status, void *stream);

/*
 * Multilayer (core-shell) spheres, FP64, Yang (2003) recurrences.
 * Replaces lib/obsolete/sphere_coefficients.py:65-220 (with its list-input
 * handling repaired).  Each sphere has nlayers radii and complex indices,
 * ordered from the core outwards:
 *   radii    [nspheres][nlayers] um
 *   indices  [nspheres][nlayers][2] (re, im)
 * Outputs as lmb_sphere_ab; dab (optional) holds the derivatives with
 * respect to the outer radius (all radii scaled together, i.e. at fixed
 * radius fractions) and to the real part of the outer layer's index.
 */
int lmb_layered_ab(const double *radii, const double *indices, int nlayers,
                   int nspheres, double n_m, double wavelength, int nmax_cap,
                   double *ab, double *dab, int *nmax, int *status,
                   void *stream);

/*
 * Scattered field of nitems independent particle lists at npts shared
 * coordinates.  Replaces LorenzMie.field / scattered_field / lorenzmie
 * (theory/LorenzMie.py:135-342) and TorchLorenzMieBatch.batch_field
 * (theory/torchLorenzMieBatch.py:285-373).
 *   coords      [3][npts] FP64 (x row, y row, z row)
 *   spheres     [nparticles] positions; ab/nmax as from lmb_sphere_ab
 *               (or lmb_layered_ab) for the same particles
 *   item_start  [nitems+1] int: particles of item i are
 *               item_start[i] .. item_start[i+1]-1 (CSR)
 *   k           wave number in the medium, rad/pixel (Instrument.wavenumber)
 *   out         [nitems][3][npts] complex64 (FP32) or complex128 (LMB_FP64)
 */
int lmb_field(const double *coords, long long npts, const lmb_sphere *spheres,
              const int *item_start, int nitems, const double *ab,
              const int *nmax, int nmax_cap, double k, int flags, void *out,
              void *stream);

/*
 * Holograms |E + x|^2 of nitems particle lists; same inputs as lmb_field.
 * Replaces LorenzMie.hologram (theory/LorenzMie.py:113-133) and
 * TorchLorenzMieBatch.batch_hologram (theory/torchLorenzMieBatch.py:258-283).
 *   out [nitems][npts] float32 (FP32) or float64 (LMB_FP64)
 */
int lmb_hologram(const double *coords, long long npts,
                 const lmb_sphere *spheres, const int *item_start, int nitems,
                 const double *ab, const int *nmax, int nmax_cap, double k,
                 int flags, void *out, void *stream);

/*
 * lmb_field / lmb_hologram of an instrument with spherical aberration:
 * each particle's scattered field is multiplied by exp(i Phi) with
 *   Phi = aberration * r^4 / (r^2 + z_p^2)^2,
 *   aberration = 4 n_m^3 spherical / k  (k in rad/pixel),
 * r the in-plane distance from the particle and z_p its axial position
 * (pixels).  Replaces AberratedLorenzMie._aberration / scattered_field
 * (theory/Aberrated.py:62-85); aberration = 0 is lmb_field / lmb_hologram.
 */
int lmb_field_aberrated(const double *coords, long long npts,
                        const lmb_sphere *spheres, const int *item_start,
                        int nitems, const double *ab, const int *nmax,
                        int nmax_cap, double k, int flags, double aberration,
                        void *out, void *stream);
int lmb_hologram_aberrated(const double *coords, long long npts,
                           const lmb_sphere *spheres, const int *item_start,
                           int nitems, const double *ab, const int *nmax,
                           int nmax_cap, double k, int flags,
                           double aberration, void *out, void *stream);

/*
 * chi^2 = sum over pixels of ((hologram - data) / noise)^2 for each of
 * nitems particle lists at shared coordinates: the objective of one
 * differential-evolution generation in one launch.  Replaces the
 * per-candidate _DEObjective calls of DEEstimator
 * (analysis/DEEstimator.py:32-37, driven by scipy's differential_evolution
 * at :158-166) and of RadialEstimator (analysis/RadialEstimator.py:32-37).
 * NaN residuals are skipped (numpy.nansum).  Inputs as lmb_hologram, plus
 *   data       [npts] FP64 normalized intensities
 *   chi2       [nitems] FP64 out
 *   nonfinite  [nitems] int out, or NULL: pixels whose hologram came out
 *              NaN or infinite.  With FP32 sums these mark candidates whose
 *              focal plane cuts the sphere, where the partial waves outgrow
 *              FP32's range; the caller re-evaluates them with LMB_FP64 so
 *              that NaN pixels are skipped only where the FP64 model (the
 *              reference's) gives NaN.
 *   workspace  of lmb_chi2_workspace_bytes(npts, nitems) bytes
 * FP32 field sums unless LMB_FP64; the residuals and sums are FP64.
 */
size_t lmb_chi2_workspace_bytes(long long npts, int nitems);
int lmb_chi2_batch(const double *coords, long long npts, const double *data,
                   double noise, const lmb_sphere *spheres,
                   const int *item_start, int nitems, const double *ab,
                   const int *nmax, int nmax_cap, double k, int flags,
                   double *chi2, int *nonfinite, void *workspace,
                   size_t workspace_bytes, void *stream);

/*
 * lmb_chi2_batch for the searches of many features at once: item i is
 * compared with the pixels of its own crop item_crop[i].  Replaces the
 * serial Frame.estimate loop (analysis/Frame.py:158-161), whose features
 * each run DEEstimator.estimate (analysis/DEEstimator.py:132-173) one
 * candidate at a time; here one generation of every feature's search is
 * one launch.
 *   coords     [3][npts] FP64: the crops' pixels, concatenated
 *   data       [npts] FP64
 *   crop_start [ncrops + 1] int64 on the device: crop c is pixels
 *              [crop_start[c], crop_start[c + 1])
 *   item_crop  [nitems] int on the device, each in [0, ncrops)
 *   max_crop_npts  the largest crop (sets the grid; a crop larger than it,
 *              or a range outside [0, npts), gives that item NaN)
 *   workspace  of lmb_chi2_workspace_bytes(max_crop_npts, nitems) bytes
 *   aberration the spherical-aberration coefficient c of
 *              lmb_field_aberrated (0: ideal optics), for the searches of
 *              AberratedLorenzMie models
 * Every other argument as lmb_chi2_batch; with aberration 0 each item's
 * chi2 is bit-identical to lmb_chi2_batch over its crop alone.
 */
int lmb_chi2_crops(const double *coords, long long npts, const double *data,
                   double noise, const long long *crop_start, int ncrops,
                   const int *item_crop, long long max_crop_npts,
                   const lmb_sphere *spheres, const int *item_start, int nitems,
                   const double *ab, const int *nmax, int nmax_cap, double k,
                   int flags, double *chi2, int *nonfinite, void *workspace,
                   size_t workspace_bytes, void *stream, double aberration);

/*
 * Differential evolution on the device, for the global estimates of many
 * features at once.  The reference's DEEstimator and RadialEstimator run
 * scipy's differential_evolution on the host (analysis/DEEstimator.py:
 * 158-166, analysis/RadialEstimator.py:150-158), one feature at a time;
 * these two kernels step the searches of many features together on the
 * GPU, the caller evaluating each trial population in between
 * (lmb_sphere_ab, then lmb_chi2_crops with item i = s * npop + c compared
 * with search s's crop).  The step is scipy's best1bin with deferred
 * updating, dithered mutation and binomial crossover; the random numbers
 * are a counter-based hash (SplitMix64) of (keys[s], generation,
 * candidate, draw): reproducible for given keys, not scipy's stream.
 *
 * Both step the searches live[0..nlive) of the nsearch (indices in
 * [0, nsearch); others are skipped), so that finished searches cost
 * nothing: their candidates are laid out by position k in live.
 *
 * lmb_de_trial: for searches of npop candidates (>= 3) of nparam (1..6)
 * parameters, from pop [nsearch][npop][nparam] (unit cube) write the trial
 * population trial [same shape] and the sphere records of the live
 * searches spheres [nlive * npop] (search live[k] at k * npop): parameter
 * j is mid[s][j] + (v - 0.5) span[s][j] in
 * slot slots[j] of the six, the rest from base [nsearch][6].  Mutation F
 * uniform in [mutation_lo, mutation_hi] per search and generation (equal
 * bounds: constant), recombination [nsearch].  With copy_only, or for a
 * search with done[s] != 0, the trial is the population itself (for the
 * first evaluation).
 *
 * lmb_de_select: with the trial energies [nlive * npop], keep each
 * trial whose energy does not exceed its candidate's (first: take all, the
 * initial population's energies), move each search's best to index 0, and
 * count the generation in nit [nsearch]; done[s] becomes 1 when
 * std(E) <= atol[s] + tol[s] |mean(E)| with no infinite energy, 2 when
 * nit reaches maxiter[s].  Finished searches are left as they are.
 */
int lmb_de_trial(int nsearch, int nlive, const int *live, int npop,
                 int nparam, const double *pop, double *trial,
                 const unsigned long long *keys, int generation,
                 double mutation_lo, double mutation_hi,
                 const double *recombination, const double *mid,
                 const double *span, const double *base, const int *slots,
                 const int *done, int copy_only, lmb_sphere *spheres,
                 void *stream);
int lmb_de_select(int nsearch, int nlive, const int *live, int npop,
                  int nparam, double *pop, double *energies,
                  const double *trial, const double *trial_energies,
                  const double *tol, const double *atol, const int *maxiter,
                  int *nit, int *done, int first, void *stream);

/*
 * Hologram and its Jacobian for nitems single-sphere items, FP32 sums,
 * Cartesian field (LMB_BOHREN honoured).  Fills the analytic-Jacobian
 * slot of the reference: jaxLorenzMie.jac / jac_params
 * (theory/jaxLorenzMie.py:321, 354-395) used by Optimizer._analytical_jac
 * (analysis/Optimizer.py:218-220, 251-255); covers k_p as well.
 *   spheres [nitems]; ab/dab/nmax from lmb_sphere_ab with dab != NULL
 *   holo    [nitems][npts] float64 (may be NULL)
 *   jac     [nitems][6][npts] float64: dH/d(x_p, y_p, z_p, a_p, n_p, k_p)
 */
int lmb_jacobian(const double *coords, long long npts,
                 const lmb_sphere *spheres, int nitems, const double *ab,
                 const double *dab, const int *nmax, int nmax_cap, double k,
                 int flags, double *holo, double *jac, void *stream);

/*
 * lmb_jacobian for an instrument with spherical aberration: the hologram
 * |E e^{i Phi} + x|^2 and its derivatives, with the phase and coefficient
 * of lmb_fit_batch_aberrated (aberration = c = 4 n_m^3 s / k).  Fills the
 * analytic-Jacobian slot for AberratedLorenzMie models (the reference's
 * JAX backend differentiates the aberrated model, theory/Aberrated.py:
 * 62-85 on theory/jaxLorenzMie.py:354-395); the spherical coefficient
 * itself is not a column.  aberration 0 gives lmb_jacobian's output.
 */
int lmb_jacobian_aberrated(const double *coords, long long npts,
                           const lmb_sphere *spheres, int nitems,
                           const double *ab, const double *dab,
                           const int *nmax, int nmax_cap, double k, int flags,
                           double aberration, double *holo, double *jac,
                           void *stream);

/*
 * Vector-Jacobian product of the hologram: grad[i][j] =
 * sum_p gout[i][p] dH_i[p]/d param_j for single-sphere items, without
 * forming the Jacobian (the backward pass of an autograd function).
 * Uses caller-provided scratch of lmb_vjp_workspace_bytes(...) bytes.
 *   gout [nitems][npts] float32; grad [nitems][6] float64
 */
size_t lmb_vjp_workspace_bytes(long long npts, int nitems);
int lmb_hologram_vjp(const double *coords, long long npts,
                     const lmb_sphere *spheres, int nitems, const double *ab,
                     const double *dab, const int *nmax, int nmax_cap,
                     double k, int flags, const float *gout, double *grad,
                     void *workspace, size_t workspace_bytes, void *stream);

/*
 * A feature to fit: a crop of a normalized hologram.  Pixels are either a
 * regular grid (nx > 0: pixel i sits at x = x0 + i % nx, y = y0 + i / nx,
 * npix = nx*ny, as Hologram.flat_coordinates, analysis/Hologram.py:69-77)
 * or an explicit list (nx == 0: npix pixels with coordinates in coords).
 * data_offset indexes the packed data (and coords) arrays.
 */
typedef struct lmb_feature {
  double x0, y0;
  int nx, ny;
  long long npix;
  long long data_offset;
} lmb_feature;

/* Fit settings; defaults of Optimizer.settings (analysis/Optimizer.py:102-113). */
typedef struct lmb_fit_settings {
  double ftol, xtol, gtol, factor;
  int max_nfev;
  int variables;   /* bit j set = parameter j of (x_p,y_p,z_p,a_p,n_p,k_p) free */
  int flags;       /* LMB_BOHREN */
  int max_iterations; /* hard cap on evaluations per call, >= 1 */
  int tile_config;    /* launch shape of the evaluation kernel, 0 = default;
                         see lmb_fit_tile_config */
  int reserved;
} lmb_fit_settings;

/*
 * Launch shapes of the fit's evaluation kernel (threads per CTA, pixels per
 * thread, minimum resident CTAs per SM), for lmb_fit_settings.tile_config.
 * Returns LMB_ERR_ARG past the last index.  The autotuner of the Python
 * package times them per problem class.
 */
int lmb_fit_tile_config(int index, int *threads, int *pixels_per_thread,
                        int *min_blocks);

/* Per-feature fit result (Optimizer.result, analysis/Optimizer.py:166-186). */
typedef struct lmb_fit_result {
  double dparams[6];  /* uncertainty of each free parameter (0 when fixed) */
  double redchi;
  double cost;        /* 0.5 * sum of squared residuals */
  int status;         /* scipy least_squares status: 1..4 success, 0 max_nfev,
                         <0 failure (-1 improper input, -2 non-finite
                         residuals, -3 nmax above cap, -4 withdrawn before
                         its data arrived: lmb_fit_batch_streamed) */
  int success;
  int nfev, njev;
} lmb_fit_result;

/*
 * Optional measurements of one lmb_fit_batch call (host struct).  When
 * requested, the call records CUDA events around each evaluation launch on
 * its stream and counts the work done on the device.  Evaluation launches
 * queued after the last productive round (they find no work) are not
 * counted in eval_launches and eval_ms.
 */
typedef struct lmb_fit_stats {
  double eval_ms;        /* summed device time of the evaluation launches */
  double total_ms;       /* device time from the first launch to the end of
                            the last evaluation that found work (to the last
                            launch with streamed admission) */
  double pixels;         /* pixels evaluated, summed over launches */
  double pixel_orders;   /* pixels x partial-wave orders evaluated */
  int eval_launches;     /* evaluation kernel launches */
  int kernel_launches;   /* all kernels the call launched */
  int iterations;        /* evaluation/step rounds */
  int pad;
} lmb_fit_stats;

/* Scratch bytes lmb_fit_batch needs for these sizes. */
size_t lmb_fit_workspace_bytes(int nfeatures, long long total_pixels,
                               int nmax_cap);

/*
 * Batched Levenberg-Marquardt fit of one sphere per feature, entirely on
 * the device.  Replaces Optimizer.optimize (analysis/Optimizer.py:196-222)
 * with its scipy least_squares(method='lm') loop, residuals
 * (H - data)/noise (:257-260) and _statistics (:262-278); one call fits
 * every feature (the reference loops over features in Frame.optimize,
 * analysis/Frame.py:163-174).
 *   features [nfeatures]
 *   data     packed float32 normalized intensities
 *   coords   packed float32 (x, y) pairs for explicit-pixel features, or NULL
 *   params   [nfeatures] in: start values, out: fitted values
 *   results  [nfeatures]
 *   settings host pointer
 *   workspace / workspace_bytes: scratch of lmb_fit_workspace_bytes(...)
 *   stats    optional host pointer (NULL: no measurement)
 * The call returns once every feature has terminated (or
 * max_iterations evaluations have run).  The last kernel it queues, which
 * writes params and results, may still be running on the stream then:
 * read them in stream order (a copy on the same stream, or after
 * cudaStreamSynchronize).  With stats the call waits for that kernel too.
 * Features whose pixels fall outside [0, total_pixels) end with status -1.
 * Host resources: a calling thread's first fit on a device makes a ring of
 * 32 pinned 64-byte slots with an event each (plus timing events with
 * stats); they are kept for that thread's later fits and released when
 * the thread exits.
 */
int lmb_fit_batch(const lmb_feature *features, int nfeatures,
                  long long total_pixels, const float *data,
                  const float *coords, lmb_sphere *params, double n_m,
                  double wavelength, double magnification, double noise,
                  int nmax_cap, const lmb_fit_settings *settings,
                  lmb_fit_result *results, void *workspace,
                  size_t workspace_bytes, lmb_fit_stats *stats, void *stream);

/*
 * lmb_fit_batch for an instrument with spherical aberration: the model
 * hologram of each feature is |E e^{i Phi} + x|^2 with the phase of
 * AberratedLorenzMie._aberration (theory/Aberrated.py:62-79),
 * Phi = c r^4 / (r^2 + z_p^2)^2, r the in-plane distance of the pixel from
 * the particle and c = aberration = 4 n_m^3 s / k (k = Instrument.wavenumber,
 * s = spherical, the same coefficient lmb_field_aberrated takes); its
 * derivatives enter the x_p, y_p, z_p columns of the Jacobian.  Replaces
 * the reference's Optimizer.optimize of an AberratedLorenzMie model
 * (analysis/Optimizer.py:196-278 with a forward-difference Jacobian).
 * Multilayer spheres as lmb_fit_batch_layered (nlayers 1: homogeneous).
 * aberration 0 gives lmb_fit_batch's (or lmb_fit_batch_layered's) results
 * exactly; a non-finite value returns LMB_ERR_ARG.
 */
int lmb_fit_batch_aberrated(const lmb_feature *features, int nfeatures,
                            long long total_pixels, const float *data,
                            const float *coords, lmb_sphere *params,
                            int nlayers, const double *layer_fractions,
                            const double *layer_indices, double n_m,
                            double wavelength, double magnification,
                            double noise, int nmax_cap, double aberration,
                            const lmb_fit_settings *settings,
                            lmb_fit_result *results, void *workspace,
                            size_t workspace_bytes, lmb_fit_stats *stats,
                            void *stream);

/*
 * lmb_fit_batch for multilayer (core-shell) spheres: the free parameters
 * are the outer radius a_p and the outer layer's index n_p + i k_p (with
 * the position); every inner radius keeps its fraction of a_p.  Layered
 * particles have no live fitting path in the reference (their coefficients
 * are lib/obsolete/sphere_coefficients.py:65-220).
 *   nlayers          layers per sphere (1..8; 1 = lmb_fit_batch)
 *   layer_fractions  [nfeatures][nlayers-1] inner radii / a_p, ascending
 *   layer_indices    [nfeatures][nlayers-1][2] inner layer indices (re, im)
 * Workspace: lmb_fit_workspace_bytes as for lmb_fit_batch.
 */
int lmb_fit_batch_layered(const lmb_feature *features, int nfeatures,
                          long long total_pixels, const float *data,
                          const float *coords, lmb_sphere *params, int nlayers,
                          const double *layer_fractions,
                          const double *layer_indices, double n_m,
                          double wavelength, double magnification,
                          double noise, int nmax_cap,
                          const lmb_fit_settings *settings,
                          lmb_fit_result *results, void *workspace,
                          size_t workspace_bytes, lmb_fit_stats *stats,
                          void *stream);

/*
 * Host-side packing: concatenate nsources crops (sources[i]: counts[i]
 * contiguous values, LMB_PACK_F64 doubles or LMB_PACK_F32 floats) as
 * float32 into dst, on up to nthreads native threads (a persistent pool;
 * the calling thread takes a share).  For the pinned staging buffer of a
 * batched or streamed fit.  No counterpart in the reference, whose fits
 * subtract float64 data on the host (analysis/Optimizer.py:257-260).
 */
#define LMB_PACK_F64 0
#define LMB_PACK_F32 1
int lmb_pack_crops(const void *const *sources, const long long *counts,
                   int nsources, int src_type, float *dst, int nthreads);

/*
 * Host-side draws of a differential-evolution generation: count times,
 * shuffle index[0..n) in place exactly as numpy's Generator.shuffle and
 * RandomState.shuffle do (Fisher-Yates, partners by numpy's masked
 * rejection on the generator's 32-bit draws), and copy the first keep
 * entries to out[c * keep ..].  bitgen is numpy's bitgen_t of the
 * generator (BitGenerator.ctypes.bit_generator); the caller holds the bit
 * generator's lock.  Replaces the per-candidate shuffle of scipy's
 * DifferentialEvolutionSolver._select_samples, which the reference's
 * estimators reach through differential_evolution
 * (analysis/DEEstimator.py:158-166, analysis/RadialEstimator.py:150-158):
 * the same draws in the same order, so a seeded search is unchanged.
 */
int lmb_de_shuffles(void *bitgen, long long *index, long long n,
                    long long count, int keep, long long *out);

/*
 * All draws of one search's generation, in scipy's order, on numpy's bit
 * generator (its lock held by the caller): with dither, *scale =
 * rng.uniform(dlo, dhi); then n shuffles of index as lmb_de_shuffles
 * (count = n, the first keep entries of each to first[c * keep ..]); then
 * fill[0..n) = rng.integers(nparam, size=n) (masked != 0: the masked
 * rejection of RandomState.randint; 0: Generator.integers, Lemire's
 * method); then cross[0..n*nparam) = rng.uniform(size=(n, nparam)) < cr.
 * The same draws as DifferentialEvolutionSolver's best1bin trial
 * construction with binomial crossover and dithered mutation, which the
 * reference's estimators reach (analysis/DEEstimator.py:158-166).
 */
int lmb_de_draws(void *bitgen, int masked, int dither, double dlo,
                 double dhi, double *scale, long long *index, long long n,
                 int keep, long long *first, int nparam, double cr,
                 long long *fill, unsigned char *cross);

/*
 * lmb_de_draws for nsearch searches in turn (each search's draws complete
 * before the next, so searches that share a generator draw in the order of
 * separate calls): per search s its bit generator, flags, dither bounds,
 * crossover probability and index row; outputs packed by search (scale[s],
 * first + s*n*keep, fill + s*n, cross + s*n*nparam).  The caller holds
 * every generator's lock.
 */
int lmb_de_draws_many(int nsearch, void *const *bitgens, const int *masked,
                      const int *dither, const double *dlo, const double *dhi,
                      double *scale, long long *const *index, long long n,
                      int keep, long long *first, int nparam, const double *cr,
                      long long *fill, unsigned char *cross);

/*
 * The random pixel subset that Mask draws for a fit (analysis/Mask.py:64-72,
 * 82-105: np.random.rand(*shape) < fraction, excluded pixels removed), on
 * the global RandomState's own bit generator (BitGenerator.ctypes
 * .bit_generator): one uniform per pixel in pixel order, as
 * RandomState.random_sample draws them, so the generator ends where numpy
 * leaves it and the subset is numpy's.  Pixel i is kept when its draw is
 * below fraction and exclude[i] (exclude may be NULL) is zero; index
 * (room for n) receives the kept pixels in increasing order, *count their
 * number.  layout 0 draws through the generator's next_double; layout 1
 * advances numpy's MT19937 state (624 words and a position) itself, a
 * block at a time -- for an MT19937 only, after checking that both
 * layouts give the same subsets and states.  Host only; the caller holds
 * the generator's lock.
 */
int lmb_mask_select(void *bitgen, long long n, double fraction,
                    const unsigned char *exclude, int layout,
                    long long *index, long long *count);

/*
 * lmb_fit_batch (any layer count) that starts before all of its pixel data
 * is on the device.  No counterpart in the reference, whose fits run one
 * feature at a time on the host.
 *
 * The feature records, params (start values) and, for layered spheres,
 * the layer arrays must be on the device when the call is made (they are
 * read by its first kernel).  The pixel data (and explicit coordinates)
 * may still be arriving: features are admitted in order as the caller
 * advances the device int *ready -- features [0, *ready) have their data
 * in place -- which the caller writes on another stream (or from another
 * thread) after each portion of the data has been copied, for example with
 * cudaMemcpyAsync of the new count on the copy's stream.  Admitted features
 * start their Levenberg-Marquardt iterations at the next round while the
 * others wait, so the host's conversion and transfer of later features
 * overlaps the fitting of earlier ones.  A negative *ready withdraws the
 * batch: features not yet admitted end with status -4.  The call returns
 * LMB_ERR_TIMEOUT if no feature is running and no new feature has been
 * admitted for wait_seconds.  nlayers = 1 with null layer arrays fits
 * homogeneous spheres; a nonzero aberration fits the aberrated model of
 * lmb_fit_batch_aberrated (0: ideal optics).
 */
int lmb_fit_batch_streamed(const lmb_feature *features, int nfeatures,
                           long long total_pixels, const float *data,
                           const float *coords, lmb_sphere *params,
                           int nlayers, const double *layer_fractions,
                           const double *layer_indices, double n_m,
                           double wavelength, double magnification,
                           double noise, int nmax_cap,
                           const lmb_fit_settings *settings, const int *ready,
                           double wait_seconds, lmb_fit_result *results,
                           void *workspace, size_t workspace_bytes,
                           lmb_fit_stats *stats, void *stream,
                           double aberration);

/*
 * lmb_fit_batch for callers that cannot allocate device memory.  No
 * counterpart in the reference (its fits run on the host).
 *
 * Who needs it: cudaMalloc and cudaFree synchronize the device and can
 * fail under memory pressure, so a caller that runs inside a real-time
 * acquisition loop, or that owns all of its device memory through another
 * allocator (a framework's caching allocator, an instrument vendor's SDK)
 * and may not allocate outside it, cannot obtain a workspace for each call.
 * This entry point takes the same inputs and outputs as lmb_fit_batch but
 * no workspace: its scratch is a file-scope device array of
 * LMB_FIT_NOALLOC_SCRATCH_BYTES (16 MiB) that every GPU which loads the
 * library holds until the process exits.  It calls no cudaMalloc, cudaFree
 * or other allocating routine and takes no stats.
 *
 * The first call on a device looks up the array's device address
 * (cudaGetSymbolAddress, with that device current).  The fit runs the
 * synchronous round loop: it reads the round counters back and waits for
 * the stream every round, and returns only when the stream has drained,
 * errors included.  So no call, the first or any later one, may be made
 * while the stream (or, in global capture mode, any stream) is being
 * captured into a graph.  Requests
 * whose lmb_fit_workspace_bytes exceed LMB_FIT_NOALLOC_SCRATCH_BYTES are
 * rejected with LMB_ERR_WORKSPACE before anything is launched; check
 * lmb_fit_workspace_bytes(n, pixels, nmax_cap) against it.  For 201x201
 * crops that is at most 568 features at nmax_cap 26, 487 at 40 and 404 at
 * 60.  All calls share the one array, which keeps the last call's contents;
 * the fit re-initializes every counter, state and table it reads, and the
 * counters are zeroed again at each call.  Calls from this process are
 * serialized by a lock, but calls whose work could overlap on the GPU (for
 * example from another thread that bypasses this entry point's return)
 * would race on the array.
 */
#define LMB_FIT_NOALLOC_SCRATCH_BYTES (16u * 1024u * 1024u)
int lmb_fit_batch_noalloc(const lmb_feature *features, int nfeatures,
                          long long total_pixels, const float *data,
                          const float *coords, lmb_sphere *params,
                          double n_m, double wavelength, double magnification,
                          double noise, int nmax_cap,
                          const lmb_fit_settings *settings,
                          lmb_fit_result *results, void *stream);

/*
 * Measured FP32 fused-multiply-add throughput of the current device in
 * FLOP/s (2 per FMA), for roofline reporting.  Runs a short kernel.
 */
int lmb_measure_fp32_peak(double *flops, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* LMB200_H */
