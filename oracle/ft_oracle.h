/* Test infrastructure only: a CPU restatement of the FaintTrail 0.9.1 search hot
 * path (static-sky median, noise, scatter mask, normalise/CR/clip, matched
 * filter, shift-and-stack, peaks, null calibration). The parity tests compare the
 * CUDA library against it; nothing in the product links or loads it.
 *
 * Images are row-major float32, frames stacked as n x h x w. Every function cites
 * the reference file:line (paths relative to the FaintTrail source tree) whose
 * arithmetic it restates. Build: make -C oracle (compiled with -ffp-contract=off,
 * like the reference, so no multiply-add is ever fused). */
#ifndef FT_ORACLE_H
#define FT_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct fto_stage_params {
    double fwhm_px;        /* PSF FWHM (fixed; the null-run form of build_stage)     */
    int static_exclude;    /* -1 = max(1, lround(n/8))                              */
    double clip_sigma;     /* 8                                                      */
    double cr_sigma;       /* 5                                                      */
    double mask_scatter;   /* 2.5                                                    */
    double weight_scatter; /* 1.5                                                    */
} fto_stage_params;

/* ---- numeric helpers (common.hpp) ---- */
double fto_median(float* v, size_t n);
double fto_robust_sigma(float* v, size_t n);
size_t fto_sample_pixels(const float* img, int w, int h, size_t max_samples, const float* mask, int border,
                         float* out);

/* ---- preprocessing (preprocess.cpp) ---- */
void fto_time_rank(const double* t_h, int n, int* rank);
int fto_static_exclude(int requested, int n);
void fto_static_sky(const float* sub, int w, int h, int n, const int* rank, int exclude, float* sky,
                    float* residual);
double fto_frame_sigma(const float* residual, int w, int h);
void fto_scatter(const float* residual, int w, int h, int n, const double* sigma, float* scatter);
void fto_mask(const float* scatter, int w, int h, double fwhm_px, double mask_scatter, float* mask);
int fto_normalise_frame(const float* residual, const float* mask, const float* scatter, int w, int h, double sigma,
                        double fwhm_px, const fto_stage_params* sp, float* z);
void fto_matched_filter(const float* z, int w, int h, double psf_sigma, float* out);
double fto_filter_sigma(const float* g, const float* mask, int w, int h, double psf_sigma);
void fto_build_stage(const float* sub, int w, int h, int n, const double* t_h, const fto_stage_params* sp,
                     float* filtered, float* static_sky, float* mask, double* sigma, int* cr, float* scatter_out);
double fto_background(const float* raw, int w, int h);
void fto_subtract_and_grow(const float* raw, int w, int h, double bg, float* sub);

/* ---- motions and shifts (search.cpp, backend.cpp) ---- */
int fto_velocity_grid(double span_h, double vmin, double vmax, double grid_tol, double* out, int cap, double* dv);
void fto_shift_table(const double* t_h, int n, const double* vel, int m, int* dx, int* dy);
int fto_min_count(double min_coverage, int n);

/* ---- the stack contract (backend.hpp:10-40) ---- */
void fto_stack(const float* frames, int w, int h, int n, const int* dx, const int* dy, int m, int min_count,
               float* max_snr, int* best_v);

/* ---- null calibration (search.cpp, random.hpp) ---- */
void fto_null_orders(const double* t_h, int n, int runs, unsigned long long seed, double* out);
int fto_find_peaks(const float* max_snr, const int* best_v, int w, int h, float floor, int radius, int edge,
                   int max_peaks, int* px, int* py, float* psnr, int* pv);
int fto_is_artefact_peak(const float* filtered, const float* sub, const float* static_sky, const double* t_h, int n,
                         int w, int h, double fwhm_px, int x, int y, double vx, double vy, double max_frame_fraction,
                         const double* reg_dx, const double* reg_dy);
double fto_set_threshold(const float* pooled, int count, int runs, double target_false_per_run,
                         double min_snr_floor, int gauss, int* method, double* a, double* k, double* inv_s2);

#ifdef __cplusplus
}
#endif
#endif
