// The preprocessing stage (FaintTrail build_stage) on the device.
#pragma once

#include <vector>

#include "engine.h"

namespace ftb {

struct StageParams {
    double fwhm_px = 0.0;         // PSF FWHM (fixed)
    int static_exclude = -1;      // -1: max(1, lround(n / 8))
    double clip_sigma = 8.0;
    double cr_sigma = 5.0;
    double mask_scatter = 2.5;
    double weight_scatter = 1.5;
};

// Device scratch of one stage: residuals, scatter map, sample buffers, tables.
struct StageScratch {
    StageScratch(Context& c, int w, int h, int n, double fwhm_px);
    bool fits(int w, int h, int n, double fwhm_px) const;
    bool holds(int w, int h, int n) const;  // a band of at most h rows
    DevBuf residual, scatter, samples, small;
    int cap = 0;  // samples per frame
    int w_ = 0, h_ = 0, n_ = 0;
};

// Maximum sample-grid points of sample_pixels(…, 200000, …, border) on w x h.
int sample_grid_points(int w, int h, int border);

void stage_time_ranks(const double* t_h, int n, std::vector<int>& rank);

// The two halves of build_stage, so that a PSF estimate can sit between them as
// in the reference (preprocess.cpp:368): static sky, residuals and per-frame
// noise; then scatter, mask, matched filter and its normalisation.
void stage_noise(Context& c, StageScratch& sc, const float* d_sub, int w, int h, int n, const double* t_h,
                 int static_exclude, float* d_sky);
void stage_filter(Context& c, StageScratch& sc, int w, int h, int n, const StageParams& sp, float* d_filtered,
                  float* d_mask, double* h_sigma, int* h_cr);
void stage_sigma_to_host(Context& c, StageScratch& sc, int n, double* h_sigma);

// build_stage on device frames d_sub (n x h x pitch, pitch = frame_pitch(w)):
// d_filtered (same layout), d_sky and d_mask (h x pitch); h_sigma / h_cr (host,
// may be null) receive the per-frame noise and cosmic-ray counts after the
// stream is synchronised by the caller.
void stage_run(Context& c, StageScratch& sc, const float* d_sub, int w, int h, int n, const double* t_h,
               const StageParams& sp, float* d_filtered, float* d_sky, float* d_mask, double* h_sigma, int* h_cr);

// Median and robust sigma (common.hpp:64-82) of the regular sample of each of k
// device frames (sample_pixels(frame, 200000), common.hpp:85-100; w x h, rows
// `pitch` floats apart): d_stats[i] the median, d_stats[k + i] the robust sigma
// (0 for fewer than 3 samples), d_counts[i] the number of samples. d_samples
// holds k * cap floats, cap >= sample_grid_points(w, h, 0).
void frame_sample_stats(Context& c, const float* const* d_frames, int k, int w, int h, int pitch, float* d_samples,
                        int cap, int* d_counts, double* d_stats);

// ---- bands of a larger image (the tiled search): frames of `rows` rows, the
// per-frame quantities of the whole image given or sampled at its grid.
int filter_border(double fwhm_px);  // ceil(3 sigma_psf) + 1
// static sky and residuals (into sc.residual) only
void stage_sky(Context& c, StageScratch& sc, const float* d_sub, int w, int rows, int n, const double* t_h,
               int static_exclude, float* d_sky);
// the samples sample_pixels(…, 200000, mask, border) takes from the w x h image
// in its rows [core_y0, core_y1), read from a band holding rows [oy, oy + band
// rows); appended to d_samples (n x cap) and d_counts
void sample_band(Context& c, const float* d_img, size_t plane, int pitch, int n, int w, int h, int border, int oy,
                 int core_y0, int core_y1, const float* d_mask, float* d_samples, int cap, int* d_counts);
// the same for whole frames (n x h x pitch, plane apart)
void sample_frames(Context& c, const float* d_frames, size_t plane, int pitch, int n, int w, int h, int border,
                   float* d_samples, int cap, int* d_counts);
// per-frame robust sigma (unit_if_zero: 1.0 where not > 0, the noise rule) and
// median of accumulated samples, into device doubles
void select_sigma(Context& c, const float* d_samples, int cap, const int* d_counts, int n, double* d_out,
                  int unit_if_zero);
void select_median(Context& c, const float* d_samples, int cap, const int* d_counts, int n, double* d_out);
// background subtraction with per-frame backgrounds (device) and blank growth by 3
void subtract_grow(Context& c, float* d_raw, float* d_sub, int w, int rows, int n, const double* d_bg);
// scatter, mask and matched filter of sc.residual with the noise given (device);
// with d_sg, normalised by it, else left unnormalised
void stage_filter_given(Context& c, StageScratch& sc, int w, int rows, int n, const StageParams& sp,
                        const double* d_sigma, const double* d_sg, float* d_filtered, float* d_mask);

}  // namespace ftb
