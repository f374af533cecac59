// The star test of the registration check (FaintTrail registration.cpp:36-89),
// one pixel at a time, for the device scan (registration.cu) and, compiled as
// plain C++, for host-side checks of the same source.
//
// A star is a pixel above bg + 5 sigma that is the strict maximum of its 5 x 5
// neighbourhood (ties go to the earlier pixel in raster order; a non-finite
// neighbour rejects it) with at least 5 of its 8 neighbours above
// bg + 2.5 sigma. Its position is the centroid of the 7 x 7 window around it,
// weighted by max(0, u - bg - 2 sigma), computed twice (the second time around
// the rounded first centroid). Every operation is the reference's, in double and
// in the same order, so that with no contraction of multiply-adds the centroid
// is bit-identical.
#pragma once

#include <cmath>

#ifdef __CUDACC__
#define FTB_HD __host__ __device__ __forceinline__
#else
#define FTB_HD inline
#endif

namespace ftb {

// One star as the scan reports it: pixel, centroid and peak above background.
struct StarRec {
    double cx, cy, peak;
    int x, y;
};

FTB_HD bool star_finite(float u) {
#ifdef __CUDA_ARCH__
    return isfinite(u);
#else
    return std::isfinite(u);
#endif
}

FTB_HD int star_round(double v) {
#ifdef __CUDA_ARCH__
    return static_cast<int>(lround(v));
#else
    return static_cast<int>(std::lround(v));
#endif
}

// Pixel (x, y) of a w x h frame with row pitch `pitch`, for 4 <= x < w - 4 and
// 4 <= y < h - 4 (all reads stay inside the frame). thr = float(bg + 5 sigma),
// nthr = float(bg + 2.5 sigma). Returns true and fills *s for a star.
FTB_HD bool star_at(const float* im, int pitch, int w, int h, int x, int y, float thr, float nthr, double bg,
                    double sig, StarRec* s) {
    const float v = im[static_cast<long long>(y) * pitch + x];
    if (!(v > thr)) return false;
    int lit = 0;
    for (int dy = -2; dy <= 2; ++dy)
        for (int dx = -2; dx <= 2; ++dx) {
            if (dx == 0 && dy == 0) continue;
            const float u = im[static_cast<long long>(y + dy) * pitch + (x + dx)];
            // a later pixel of equal value loses to this one; an earlier one wins
            const bool earlier = dy < 0 || (dy == 0 && dx < 0);
            if (!star_finite(u) || u > v || (u == v && earlier)) return false;
            if (dx >= -1 && dx <= 1 && dy >= -1 && dy <= 1 && u > nthr) ++lit;
        }
    if (lit < 5) return false;
    double cx = x, cy = y;
    const double floor_w = 2.0 * sig;
    for (int pass = 0; pass < 2; ++pass) {
        const int ix = star_round(cx), iy = star_round(cy);
        if (ix < 3 || iy < 3 || ix >= w - 3 || iy >= h - 3) break;
        double sw = 0.0, sx = 0.0, sy = 0.0;
        for (int dy = -3; dy <= 3; ++dy)
            for (int dx = -3; dx <= 3; ++dx) {
                const float u = im[static_cast<long long>(iy + dy) * pitch + (ix + dx)];
                if (!star_finite(u)) continue;
                const double e = (static_cast<double>(u) - bg) - floor_w;
                const double wgt = (0.0 < e) ? e : 0.0;
                sw += wgt;
                sx += wgt * static_cast<double>(ix + dx);
                sy += wgt * static_cast<double>(iy + dy);
            }
        if (sw <= 0.0) break;
        cx = sx / sw;
        cy = sy / sw;
    }
    s->cx = cx;
    s->cy = cy;
    s->peak = static_cast<double>(v) - bg;
    s->x = x;
    s->y = y;
    return true;
}

}  // namespace ftb
