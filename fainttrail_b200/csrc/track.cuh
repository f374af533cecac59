// Sub-pixel track sampling shared by the artefact screen and the candidate
// refinement: the reference's bilinear() (common.hpp:125-138) with its border
// rule and double arithmetic, every operation rounded to nearest (no
// contraction), and track_pos() for straight tracks (internal.hpp:107-116).
#pragma once

#include <math_constants.h>

namespace ftb {

__device__ __forceinline__ float track_bilinear(const float* img, int w, int h, int pitch, double x, double y) {
    const int x0 = static_cast<int>(floor(x)), y0 = static_cast<int>(floor(y));
    if (x0 < 0 || y0 < 0 || x0 + 1 >= w || y0 + 1 >= h) {
        const int xr = static_cast<int>(lround(x)), yr = static_cast<int>(lround(y));
        if (xr >= 0 && yr >= 0 && xr < w && yr < h && fabs(x - xr) < 1e-9 && fabs(y - yr) < 1e-9)
            return img[static_cast<size_t>(yr) * pitch + xr];
        return CUDART_NAN_F;
    }
    const double fx = __dsub_rn(x, static_cast<double>(x0)), fy = __dsub_rn(y, static_cast<double>(y0));
    const float* r0 = img + static_cast<size_t>(y0) * pitch + x0;
    const float* r1 = r0 + pitch;
    const double gx = __dsub_rn(1.0, fx), gy = __dsub_rn(1.0, fy);
    const double top = __dadd_rn(__dmul_rn(gx, r0[0]), __dmul_rn(fx, r0[1]));
    const double bot = __dadd_rn(__dmul_rn(gx, r1[0]), __dmul_rn(fx, r1[1]));
    return __double2float_rn(__dadd_rn(__dmul_rn(gy, top), __dmul_rn(fy, bot)));
}

// x + v t, rounded as the reference's track_pos
__device__ __forceinline__ double track_coord(double x0, double v, double t) { return __dadd_rn(x0, __dmul_rn(v, t)); }

}  // namespace ftb
