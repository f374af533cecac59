// Test infrastructure only: the registration check's host half
// (fainttrail_b200/csrc/registration_host.cpp) and its per-pixel star test
// (registration.cuh) built for the host, with the frame statistics of
// find_stars (sample grid, median, robust sigma; FaintTrail common.hpp:64-100)
// restated here, so that the CPU tests can compare the check's logic with the
// reference's golden verdicts on a machine without a GPU. The product runs the
// star test on the device (registration.cu).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "registration_host.h"

namespace {

double median_of(std::vector<float>& v) {
    if (v.empty()) return 0.0;
    const size_t mid = v.size() / 2;
    std::nth_element(v.begin(), v.begin() + static_cast<long>(mid), v.end());
    double m = v[mid];
    if (v.size() % 2 == 0) m = 0.5 * (m + *std::max_element(v.begin(), v.begin() + static_cast<long>(mid)));
    return m;
}

std::vector<ftb::Star> stars_of(const float* im, int w, int h, int keep) {
    const size_t usable = static_cast<size_t>(w) * h;
    const int step = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(usable) / 200000)));
    std::vector<float> s;
    for (int y = 0; y < h; y += step)
        for (int x = 0; x < w; x += step)
            if (std::isfinite(im[static_cast<size_t>(y) * w + x])) s.push_back(im[static_cast<size_t>(y) * w + x]);
    if (s.size() < 100) return {};
    const double bg = median_of(s);
    for (float& x : s) x = static_cast<float>(std::fabs(x - bg));
    const double sig = 1.4826 * median_of(s);
    if (!(sig > 0)) return {};
    const float thr = static_cast<float>(bg + 5.0 * sig), nthr = static_cast<float>(bg + 2.5 * sig);
    std::vector<ftb::StarRec> recs;
    for (int y = h - 5; y >= 4; --y)  // any order: the records are put in raster order
        for (int x = w - 5; x >= 4; --x) {
            ftb::StarRec r;
            if (ftb::star_at(im, w, w, h, x, y, thr, nthr, bg, sig, &r)) recs.push_back(r);
        }
    return ftb::order_stars(recs, keep);
}

}  // namespace

// The check of n frames (n x h x w) at t_h hours: out[0..8] = measured,
// registered, dx, dy, mid_dx, mid_dy, rate_pxh, stars, matched; the message
// into msg (NUL-terminated).
extern "C" int ftb_host_check_registration(const float* frames, int n, int w, int h, const double* t_h, double* out,
                                           char* msg, int msg_len) {
    ftb::DriftCheck d;
    if (n >= 3) {
        int fi[3];
        ftb::registration_frames(t_h, n, &fi[0], &fi[1], &fi[2]);
        const size_t plane = static_cast<size_t>(w) * h;
        d = ftb::drift_from_stars(stars_of(frames + fi[0] * plane, w, h, 60), stars_of(frames + fi[1] * plane, w, h, 120),
                                  stars_of(frames + fi[2] * plane, w, h, 120), w, h, t_h[fi[2]] - t_h[fi[0]]);
    }
    const double v[9] = {d.measured ? 1.0 : 0.0, d.registered ? 1.0 : 0.0, d.dx, d.dy, d.mid_dx, d.mid_dy,
                         d.rate_pxh, static_cast<double>(d.stars), static_cast<double>(d.matched)};
    std::memcpy(out, v, sizeof v);
    std::strncpy(msg, d.message.c_str(), static_cast<size_t>(msg_len) - 1);
    msg[msg_len - 1] = 0;
    return 0;
}
