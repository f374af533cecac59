// Host half of the registration check (FaintTrail check_registration,
// registration.cpp:260-312): plain C++ with no CUDA dependency, so that the
// check's host logic and the star test (registration.cuh) also build for
// host-only tests.
#pragma once

#include <string>
#include <vector>

#include "registration.cuh"

namespace ftb {

// DriftCheck (registration.hpp:22-30)
struct DriftCheck {
    bool measured = false;    // enough stars matched to tell
    bool registered = true;   // true when not measured
    double dx = 0.0, dy = 0.0, mid_dx = 0.0, mid_dy = 0.0, rate_pxh = 0.0;
    int stars = 0, matched = 0;
    std::string message;      // why the frames are not registered
};

struct Star {
    double x, y, peak;
};

// find_stars' list from the scan's records (any order): raster order, then the
// reference's sort by peak (registration.cpp:85-87), at most `keep`.
std::vector<Star> order_stars(std::vector<StarRec> recs, int keep);

// The check from the three frames' star lists (first frame: at most 60 stars,
// middle and last: at most 120), the frame size and the time from the first to
// the last frame in hours (registration.cpp:268-311).
DriftCheck drift_from_stars(const std::vector<Star>& first, const std::vector<Star>& mid,
                            const std::vector<Star>& last, int w, int h, double dt_h);

// The three frames the check uses (registration.cpp:264-267): indices of the
// first, middle and last frame by t_h.
void registration_frames(const double* t_h, int n, int* first, int* mid, int* last);

}  // namespace ftb
