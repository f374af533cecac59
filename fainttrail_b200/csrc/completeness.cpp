// The injection-recovery test on the device's batched search: FaintTrail's
// completeness() (validate.cpp:62-165) with the same placements, injections,
// searches and matching, so its report equals the reference's.
#include <algorithm>
#include <cmath>
#include <limits>

#include "search.h"

namespace ftb {

namespace {

constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;  // psf.hpp:16
constexpr double kPi = 3.14159265358979323846;

struct Truth {
    double x_ref, y_ref, vx_pxh, vy_pxh;
};

struct MatchResult {
    int truth, candidate;
    double dpos, dv;
};

// flux_for_snr (validate.cpp:31-34)
double flux_for_snr(double stack_snr, double sigma, double fwhm_px, int nframes) {
    const double s = fwhm_px * kFwhmToSigma;
    return stack_snr / std::sqrt(static_cast<double>(std::max(1, nframes))) * sigma * std::sqrt(4.0 * kPi) * s;
}

// match (validate.cpp:36-60): each injected track takes the nearest unused
// candidate within max_dpos and max_dv, in truth order
std::vector<MatchResult> match(const std::vector<Candidate>& cands, const std::vector<Truth>& truth, double max_dpos,
                               double max_dv, bool ok_only) {
    std::vector<MatchResult> out;
    std::vector<bool> used(cands.size(), false);
    for (size_t t = 0; t < truth.size(); ++t) {
        double best = std::numeric_limits<double>::infinity(), bdv = 0;
        int bi = -1;
        for (size_t k = 0; k < cands.size(); ++k) {
            if (used[k] || (ok_only && !cands[k].ok)) continue;
            const double dp = std::hypot(cands[k].x - truth[t].x_ref, cands[k].y - truth[t].y_ref);
            const double dv = std::hypot(cands[k].vx_pxh - truth[t].vx_pxh, cands[k].vy_pxh - truth[t].vy_pxh);
            if (dp <= max_dpos && dv <= max_dv && dp < best) {
                best = dp;
                bi = static_cast<int>(k);
                bdv = dv;
            }
        }
        if (bi >= 0) {
            used[static_cast<size_t>(bi)] = true;
            out.push_back({static_cast<int>(t), bi, best, bdv});
        }
    }
    return out;
}

}  // namespace

CompletenessOut completeness_host(Context& c, const float* frames, int w, int h, int n, const double* mjd,
                                  const double* exptime, const SearchParams& p, const std::vector<double>& levels,
                                  int per_level, double min_separation, uint64_t seed) {
    CompletenessOut rep;
    // the baseline: the threshold calibrated on the untouched data
    std::vector<SearchOut> none;
    const SearchOut base = search_batch_host(c, frames, w, h, n, mjd, exptime, p, {}, none, {});
    rep.threshold_snr = base.thr.snr;
    rep.threshold_method = base.thr.method;
    for (const Candidate& cd : base.candidates)
        if (cd.ok) ++rep.baseline_ok;
    std::vector<double> sg(base.sigma);
    std::nth_element(sg.begin(), sg.begin() + static_cast<std::ptrdiff_t>(sg.size() / 2), sg.end());
    const double sigma = sg[sg.size() / 2];
    const double fwhm = base.fwhm_px;
    const double margin = std::max(12.0, 3.0 * fwhm);

    SearchParams fixed = p;
    fixed.threshold_snr = rep.threshold_snr;
    fixed.fwhm_px = fwhm;
    fixed.null_runs = 0;

    // placements, level by level, from one seeded stream
    Xoshiro rng(seed);
    std::vector<std::vector<Injection>> copies;
    std::vector<std::vector<Truth>> truths;
    for (double level : levels) {
        std::vector<Injection> inj;
        std::vector<Truth> truth;
        for (int k = 0; k < per_level; ++k) {
            Injection o;
            bool placed = false;
            for (int attempt = 0; attempt < 500 && !placed; ++attempt) {
                o.x_ref = rng.uniform(margin, w - margin);
                o.y_ref = rng.uniform(margin, h - margin);
                placed = true;
                for (const Injection& q : inj)
                    if (std::hypot(q.x_ref - o.x_ref, q.y_ref - o.y_ref) < min_separation) placed = false;
                for (const Candidate& cd : base.candidates)  // clear of objects already in the data
                    if (cd.ok && std::hypot(cd.x - o.x_ref, cd.y - o.y_ref) < min_separation) placed = false;
            }
            if (!placed) continue;
            const double vlo = std::max(p.vmin_pxh, 0.0) * 1.05, vhi = p.vmax_pxh * 0.95;
            const double v = rng.uniform(vlo, std::max(vlo, vhi));
            const double ang = rng.uniform(0.0, 2.0 * kPi);
            o.vx_pxh = v * std::cos(ang);
            o.vy_pxh = v * std::sin(ang);
            o.flux = flux_for_snr(level, sigma, fwhm, n);
            inj.push_back(o);
            truth.push_back({o.x_ref, o.y_ref, o.vx_pxh, o.vy_pxh});
        }
        copies.push_back(std::move(inj));
        truths.push_back(std::move(truth));
    }
    // every level's copy searched with the fixed threshold, in one batch
    std::vector<SearchOut> outs;
    search_batch_host(c, frames, w, h, n, mjd, exptime, fixed, copies, outs, {});
    for (size_t li = 0; li < levels.size(); ++li) {
        const SearchOut& r = outs[li];
        const double max_dv = std::max(3.0, 2.0 * r.dv);
        const std::vector<MatchResult> ok_m = match(r.candidates, truths[li], 2.0, max_dv, true);
        const std::vector<MatchResult> any_m = match(r.candidates, truths[li], 2.0, max_dv, false);
        CompletenessRow row;
        row.target_snr = levels[li];
        row.injected = static_cast<int>(copies[li].size());
        row.recovered = static_cast<int>(ok_m.size());
        row.detected = static_cast<int>(any_m.size());
        for (const MatchResult& m : ok_m) {
            row.mean_snr += r.candidates[static_cast<size_t>(m.candidate)].snr;
            row.mean_dpos += m.dpos;
            row.mean_dv += m.dv;
        }
        if (!ok_m.empty()) {
            row.mean_snr /= ok_m.size();
            row.mean_dpos /= ok_m.size();
            row.mean_dv /= ok_m.size();
        }
        rep.rows.push_back(row);
    }
    // S/N at 50 % completeness by linear interpolation
    for (size_t i = 1; i < rep.rows.size(); ++i) {
        const CompletenessRow& a = rep.rows[i - 1];
        const CompletenessRow& b = rep.rows[i];
        if (a.injected == 0 || b.injected == 0) continue;
        const double fa = static_cast<double>(a.recovered) / a.injected;
        const double fb = static_cast<double>(b.recovered) / b.injected;
        if (fa < 0.5 && fb >= 0.5) {
            rep.snr50 = a.target_snr + (0.5 - fa) / (fb - fa) * (b.target_snr - a.target_snr);
            break;
        }
    }
    if (rep.snr50 == 0.0 && !rep.rows.empty() && rep.rows.front().injected > 0 &&
        static_cast<double>(rep.rows.front().recovered) / rep.rows.front().injected >= 0.5)
        rep.snr50 = rep.rows.front().target_snr;
    return rep;
}

}  // namespace ftb
