// Host half of the registration check: the order of the star lists, the coarse
// offset vote, the similarity fit with clipping and the verdict
// (FaintTrail registration.cpp:36-312). At most 120 stars per frame take part,
// so this stays on the host; the per-pixel star scan runs on the device
// (registration.cu).
//
// The arithmetic follows the reference step for step (sums in pair order, the
// same expression trees, std::hypot and std::sqrt of the host library), so the
// check's offsets, rate and message are bit-identical to it.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <numeric>
#include <utility>

#include "registration_host.h"

namespace ftb {

namespace {

// frame pixel = (a, -b; b, a) * reference pixel + (tx, ty)  (registration.cpp:92-101)
struct Similarity {
    double a = 1.0, b = 0.0, tx = 0.0, ty = 0.0;
    void map(double x, double y, double& u, double& v) const {
        u = a * x - b * y + tx;
        v = b * x + a * y + ty;
    }
    double rotation_deg() const { return std::atan2(b, a) * 180.0 / 3.14159265358979323846; }
};

// The coarse offset (registration.cpp:103-131): every pair of one of the 30
// brightest reference stars (rotated by 180 degrees about the centre for a
// meridian flip) and one of the 80 brightest frame stars within max_shift votes
// for its offset's 2-px bin; the best 2 x 2 block of bins wins, the first in
// bin order on a tie. Returns the block's votes; (ox, oy) its far corner.
int vote_offset(const std::vector<Star>& ref, const std::vector<Star>& fr, bool flip, double cx, double cy,
                double max_shift, double& ox, double& oy) {
    const size_t nr = std::min<size_t>(ref.size(), 30), nf = std::min<size_t>(fr.size(), 80);
    std::vector<std::pair<int, int>> keys;
    for (size_t i = 0; i < nr; ++i) {
        const double px = flip ? 2 * cx - ref[i].x : ref[i].x;
        const double py = flip ? 2 * cy - ref[i].y : ref[i].y;
        for (size_t k = 0; k < nf; ++k) {
            const double dx = fr[k].x - px, dy = fr[k].y - py;
            if (std::fabs(dx) > max_shift || std::fabs(dy) > max_shift) continue;
            keys.emplace_back(static_cast<int>(std::floor(dx / 2.0)), static_cast<int>(std::floor(dy / 2.0)));
        }
    }
    // bins in ascending key order with their counts
    std::sort(keys.begin(), keys.end());
    std::vector<std::pair<std::pair<int, int>, int>> bins;
    for (const auto& k : keys) {
        if (!bins.empty() && bins.back().first == k)
            ++bins.back().second;
        else
            bins.push_back({k, 1});
    }
    auto count = [&](int bx, int by) {
        const std::pair<int, int> k{bx, by};
        const auto it = std::lower_bound(bins.begin(), bins.end(), k,
                                         [](const std::pair<std::pair<int, int>, int>& e,
                                            const std::pair<int, int>& q) { return e.first < q; });
        return (it != bins.end() && it->first == k) ? it->second : 0;
    };
    int best = 0;
    std::pair<int, int> at{0, 0};
    for (const auto& e : bins) {
        const int bx = e.first.first, by = e.first.second;
        const int sum = count(bx, by) + count(bx, by + 1) + count(bx + 1, by) + count(bx + 1, by + 1);
        if (sum > best) {
            best = sum;
            at = e.first;
        }
    }
    ox = 2.0 * at.first + 2.0;
    oy = 2.0 * at.second + 2.0;
    return best;
}

using Pair = std::pair<const Star*, const Star*>;

// One least-squares pass on centred coordinates with 3-sigma clipping
// (registration.cpp:167-209). False when the pairs are degenerate or fewer
// than 5 survive.
bool fit_pass(std::vector<Pair>& pairs, Similarity& T, double& rms) {
    double mpx = 0, mpy = 0, mqx = 0, mqy = 0;
    for (const Pair& p : pairs) {
        mpx += p.first->x;
        mpy += p.first->y;
        mqx += p.second->x;
        mqy += p.second->y;
    }
    const double m = static_cast<double>(pairs.size());
    mpx /= m;
    mpy /= m;
    mqx /= m;
    mqy /= m;
    double sab = 0, sbb = 0, spp = 0;
    for (const Pair& p : pairs) {
        const double px = p.first->x - mpx, py = p.first->y - mpy;
        const double qx = p.second->x - mqx, qy = p.second->y - mqy;
        sab += px * qx + py * qy;
        sbb += px * qy - py * qx;
        spp += px * px + py * py;
    }
    if (spp <= 0) return false;
    if (pairs.size() >= 12) {
        T.a = sab / spp;
        T.b = sbb / spp;
    } else {  // too few pairs for rotation and scale: the shift alone (and the flip)
        T.a = T.a < 0 ? -1.0 : 1.0;
        T.b = 0.0;
    }
    T.tx = mqx - (T.a * mpx - T.b * mpy);
    T.ty = mqy - (T.b * mpx + T.a * mpy);
    std::vector<double> res(pairs.size());
    double ss = 0;
    for (size_t k = 0; k < pairs.size(); ++k) {
        double u, v;
        T.map(pairs[k].first->x, pairs[k].first->y, u, v);
        res[k] = std::hypot(pairs[k].second->x - u, pairs[k].second->y - v);
        ss += res[k] * res[k];
    }
    rms = std::sqrt(ss / m);
    const double cut = std::max(0.5, 3.0 * rms);
    std::vector<Pair> kept;
    for (size_t k = 0; k < pairs.size(); ++k)
        if (res[k] <= cut) kept.push_back(pairs[k]);
    if (kept.size() < 5) return false;
    pairs.swap(kept);
    return true;
}

// The transform taking reference stars onto frame stars (registration.cpp:133-213):
// the vote (and the flipped vote) seeds it, then nearest-neighbour matching
// within 4, 2.5, 1.5 and 1.5 px, each followed by two clipped fits.
bool fit_similarity(const std::vector<Star>& ref, const std::vector<Star>& fr, double cx, double cy,
                    double max_shift, Similarity& T, int& used) {
    const size_t nr = std::min<size_t>(ref.size(), 30);
    if (nr < 6 || fr.size() < 6) return false;
    double ox = 0, oy = 0, fx = 0, fy = 0;
    const int v_plain = vote_offset(ref, fr, false, cx, cy, max_shift, ox, oy);
    const int v_flip = vote_offset(ref, fr, true, cx, cy, max_shift, fx, fy);
    const bool flip = v_flip > v_plain;
    if (std::max(v_plain, v_flip) < std::max<int>(5, static_cast<int>(nr) / 3)) return false;
    T = flip ? Similarity{-1, 0, 2 * cx + fx, 2 * cy + fy} : Similarity{1, 0, ox, oy};
    static const double radii[] = {4.0, 2.5, 1.5, 1.5};
    std::vector<Pair> pairs;
    double rms = 0;
    for (const double r0 : radii) {
        pairs.clear();
        for (const Star& s : ref) {
            double u, v;
            T.map(s.x, s.y, u, v);
            const Star* near = nullptr;
            double nd = r0;
            for (const Star& f : fr) {
                const double d = std::hypot(f.x - u, f.y - v);
                if (d < nd) {
                    nd = d;
                    near = &f;
                }
            }
            if (near) pairs.emplace_back(&s, near);
        }
        if (pairs.size() < 5) return false;
        for (int pass = 0; pass < 2; ++pass)
            if (!fit_pass(pairs, T, rms)) return false;
    }
    used = static_cast<int>(pairs.size());
    return used >= 5;
}

// Displacement of the field centre (dx, dy) and the largest displacement of the
// centre and the four corners (registration.cpp:279-291).
double displacement(const Similarity& T, double cx, double cy, double& dx, double& dy) {
    T.map(cx, cy, dx, dy);
    dx -= cx;
    dy -= cy;
    double worst = 0;
    for (const double x : {0.0, 2 * cx})
        for (const double y : {0.0, 2 * cy}) {
            double u, v;
            T.map(x, y, u, v);
            worst = std::max(worst, std::hypot(u - x, v - y));
        }
    return worst;
}

}  // namespace

std::vector<Star> order_stars(std::vector<StarRec> recs, int keep) {
    std::sort(recs.begin(), recs.end(),
              [](const StarRec& a, const StarRec& b) { return a.y != b.y ? a.y < b.y : a.x < b.x; });
    std::vector<Star> out;
    out.reserve(recs.size());
    for (const StarRec& r : recs) out.push_back({r.cx, r.cy, r.peak});
    std::sort(out.begin(), out.end(), [](const Star& a, const Star& b) { return a.peak > b.peak; });
    if (static_cast<int>(out.size()) > keep) out.resize(static_cast<size_t>(keep));
    return out;
}

void registration_frames(const double* t_h, int n, int* first, int* mid, int* last) {
    std::vector<size_t> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), size_t{0});
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return t_h[a] < t_h[b]; });
    *first = static_cast<int>(order.front());
    *last = static_cast<int>(order.back());
    *mid = static_cast<int>(order[static_cast<size_t>(n) / 2]);
}

DriftCheck drift_from_stars(const std::vector<Star>& first, const std::vector<Star>& mid,
                            const std::vector<Star>& last, int w, int h, double dt_h) {
    DriftCheck r;
    const double cx = 0.5 * (w - 1), cy = 0.5 * (h - 1);
    const double max_shift = std::min(w, h) / 3.0;
    r.stars = static_cast<int>(first.size());
    Similarity tl, tm;
    int nl = 0, nm = 0;
    if (!fit_similarity(first, last, cx, cy, max_shift, tl, nl)) return r;
    r.measured = true;
    r.matched = nl;
    const double ml = displacement(tl, cx, cy, r.dx, r.dy);
    double mm = 0;
    if (fit_similarity(first, mid, cx, cy, max_shift, tm, nm)) mm = displacement(tm, cx, cy, r.mid_dx, r.mid_dy);
    if (dt_h > 0) r.rate_pxh = std::hypot(r.dx, r.dy) / dt_h;
    r.registered = ml <= 1.5 && mm <= 1.5;
    if (!r.registered) {
        char buf[800];  // room for two doubles of any size in %.1f
        std::snprintf(buf, sizeof buf, "the frames are not registered: the stars move by (%.1f, %.1f) px", r.dx, r.dy);
        r.message = buf;
        std::snprintf(buf, sizeof buf, " from the first to the last frame (%.1f px/h, %d stars matched", r.rate_pxh, nl);
        r.message += buf;
        const double rot = tl.rotation_deg();
        if (std::fabs(rot) > 0.05) {
            std::snprintf(buf, sizeof buf, ", rotation %.1f deg", rot);
            r.message += buf;
        }
        r.message += "). Without registration every star is detected as a moving object.";
    }
    return r;
}

}  // namespace ftb
