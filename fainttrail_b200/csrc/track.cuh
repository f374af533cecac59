// Sub-pixel track sampling shared by the artefact screen and the candidate
// refinement: the reference's bilinear() (common.hpp:125-138) with its border
// rule and double arithmetic, every operation rounded to nearest (no
// contraction), and track_pos() for straight tracks (internal.hpp:107-116).
#pragma once

#include <math_constants.h>

namespace ftb {

// A band of an image: rows [oy, oy + rows) of an image of h rows, row y held at
// img + (y - oy) * pitch (the whole image: oy 0, rows h). Coordinates and the
// border rule are the whole image's, so a band gives the whole image's values;
// a sample whose rows the band does not hold is NaN.
__device__ __forceinline__ float track_bilinear_band(const float* img, int w, int h, int pitch, int oy, int rows,
                                                     double x, double y) {
    const int x0 = static_cast<int>(floor(x)), y0 = static_cast<int>(floor(y));
    if (x0 < 0 || y0 < 0 || x0 + 1 >= w || y0 + 1 >= h) {
        const int xr = static_cast<int>(lround(x)), yr = static_cast<int>(lround(y));
        if (xr >= 0 && yr >= 0 && xr < w && yr < h && fabs(x - xr) < 1e-9 && fabs(y - yr) < 1e-9) {
            if (yr - oy < 0 || yr - oy >= rows) return CUDART_NAN_F;
            return img[static_cast<size_t>(yr - oy) * pitch + xr];
        }
        return CUDART_NAN_F;
    }
    if (y0 - oy < 0 || y0 + 1 - oy >= rows) return CUDART_NAN_F;
    const double fx = __dsub_rn(x, static_cast<double>(x0)), fy = __dsub_rn(y, static_cast<double>(y0));
    const float* r0 = img + static_cast<size_t>(y0 - oy) * pitch + x0;
    const float* r1 = r0 + pitch;
    const double gx = __dsub_rn(1.0, fx), gy = __dsub_rn(1.0, fy);
    const double top = __dadd_rn(__dmul_rn(gx, r0[0]), __dmul_rn(fx, r0[1]));
    const double bot = __dadd_rn(__dmul_rn(gx, r1[0]), __dmul_rn(fx, r1[1]));
    return __double2float_rn(__dadd_rn(__dmul_rn(gy, top), __dmul_rn(fy, bot)));
}

__device__ __forceinline__ float track_bilinear(const float* img, int w, int h, int pitch, double x, double y) {
    return track_bilinear_band(img, w, h, pitch, 0, h, x, y);
}

// x + v t, rounded as the reference's track_pos
__device__ __forceinline__ double track_coord(double x0, double v, double t) { return __dadd_rn(x0, __dmul_rn(v, t)); }

// detector_flag (search.cpp:196-225) for one straight track, by a warp: the
// largest S/N of a source fixed on the detector near the track's mean detector
// position. Lane 0 forms the mean of (track position + registration offset) in
// frame order; the lanes share the grid of offsets (steps x steps, dy outer),
// each summing its frames' bilinear values in frame order; the maximum is
// order-independent. Returns the maximum (0 if no position has 3 frames) to
// every lane. The frames may be a band of the image (oy, rows).
__device__ __forceinline__ double detector_best_fixed(const float* filtered, size_t plane, int w, int h, int pitch,
                                                      int oy, int rows, int n, const double* t_h,
                                                      const double* reg_dx, const double* reg_dy, const double* steps,
                                                      int nsteps, double bx, double by, double bvx, double bvy) {
    const int lane = static_cast<int>(threadIdx.x & 31);
    double mx = 0.0, my = 0.0;
    if (lane == 0) {
        for (int i = 0; i < n; ++i) {
            mx = __dadd_rn(mx, __dadd_rn(track_coord(bx, bvx, t_h[i]), reg_dx[i]));
            my = __dadd_rn(my, __dadd_rn(track_coord(by, bvy, t_h[i]), reg_dy[i]));
        }
        mx = __ddiv_rn(mx, static_cast<double>(n));
        my = __ddiv_rn(my, static_cast<double>(n));
    }
    mx = __shfl_sync(0xffffffffu, mx, 0);
    my = __shfl_sync(0xffffffffu, my, 0);
    double best = 0.0;
    for (int q = lane; q < nsteps * nsteps; q += 32) {
        const double X = __dadd_rn(mx, steps[q % nsteps]), Y = __dadd_rn(my, steps[q / nsteps]);
        double sum = 0.0;
        int count = 0;
        for (int i = 0; i < n; ++i) {
            const float v = track_bilinear_band(filtered + i * plane, w, h, pitch, oy, rows, __dsub_rn(X, reg_dx[i]),
                                                __dsub_rn(Y, reg_dy[i]));
            if (!isfinite(v)) continue;
            sum = __dadd_rn(sum, static_cast<double>(v));
            ++count;
        }
        const double snr = count >= 3 ? __ddiv_rn(sum, __dsqrt_rn(static_cast<double>(count))) : 0.0;
        best = best < snr ? snr : best;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double other = __shfl_xor_sync(0xffffffffu, best, o);
        best = best < other ? other : best;
    }
    return best;
}

}  // namespace ftb
