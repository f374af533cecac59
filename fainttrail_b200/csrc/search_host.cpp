// Host steps of the search: the motion grid, the null-run time orders, the peak
// order, the null-tail fit and threshold, and the PSF estimate. These are small
// sequential computations; each follows the reference's arithmetic exactly so
// that grids, orders and thresholds are bit-identical.
#include <algorithm>
#include <cmath>
#include <functional>
#include <numeric>
#include <stdexcept>

#include "search.h"

namespace ftb {

namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;
}  // namespace

// search.cpp:39-58: square lattice of step dv = 4 max(0.05, tol) / span over
// the annulus [vmin - dv/2, vmax + dv/2], vy-major
std::vector<std::pair<double, double>> velocity_grid(double span_h, const SearchParams& p, double* dv_out) {
    if (span_h <= 0.0) throw std::runtime_error("invalid time span");
    if (p.vmax_pxh <= 0.0 || p.vmax_pxh < p.vmin_pxh) throw std::runtime_error("invalid velocity range");
    const double dv = 4.0 * std::max(0.05, p.grid_tol_px) / span_h;
    if (dv_out) *dv_out = dv;
    const int K = static_cast<int>(std::ceil(p.vmax_pxh / dv));
    const double lo = std::max(0.0, p.vmin_pxh - 0.5 * dv), hi = p.vmax_pxh + 0.5 * dv;
    std::vector<std::pair<double, double>> g;
    for (int j = -K; j <= K; ++j)
        for (int i = -K; i <= K; ++i) {
            const double vx = i * dv, vy = j * dv, v = std::hypot(vx, vy);
            if (v >= lo && v <= hi) g.emplace_back(vx, vy);
        }
    if (g.size() > 5000000) throw std::runtime_error("velocity grid too large; narrow the range");
    return g;
}

// search.cpp:559-571: K Fisher-Yates shuffles of the frame times
std::vector<std::vector<double>> null_time_orders(const std::vector<double>& t_h, int runs, uint64_t seed) {
    Xoshiro rng(seed);
    std::vector<std::vector<double>> out;
    for (int k = 0; k < runs; ++k) {
        std::vector<double> t = t_h;
        for (size_t i = t.size() - 1; i > 0; --i) std::swap(t[i], t[static_cast<size_t>(rng.uniform() * (i + 1))]);
        out.push_back(std::move(t));
    }
    return out;
}

// backend.cpp:114-123: round(v t) half away from zero, in double
void shift_table(const std::vector<double>& t_h, const std::vector<std::pair<double, double>>& grid,
                 std::vector<int>& dx, std::vector<int>& dy) {
    const size_t n = t_h.size();
    dx.resize(grid.size() * n);
    dy.resize(grid.size() * n);
    for (size_t j = 0; j < grid.size(); ++j)
        for (size_t i = 0; i < n; ++i) {
            dx[j * n + i] = static_cast<int>(std::lround(grid[j].first * t_h[i]));
            dy[j * n + i] = static_cast<int>(std::lround(grid[j].second * t_h[i]));
        }
}

int pass_min_count(double min_coverage, int n) { return std::max(3, static_cast<int>(std::ceil(min_coverage * n))); }

void order_peaks(std::vector<Peak>& peaks, size_t max_peaks) {
    // the same (unstable) std::sort on the same raster-ordered sequence as
    // search.cpp:132, so equal-S/N peaks keep the reference's order
    std::sort(peaks.begin(), peaks.end(), [](const Peak& a, const Peak& b) { return a.snr > b.snr; });
    if (peaks.size() > max_peaks) peaks.resize(max_peaks);
}

double median_of(std::vector<float> v) {
    if (v.empty()) return 0.0;
    const size_t n = v.size(), mid = n / 2;
    std::nth_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(mid), v.end());
    double m = v[mid];
    if (n % 2 == 0) m = 0.5 * (m + *std::max_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(mid)));
    return m;
}

namespace {

// search.cpp:471-510
bool fit_gauss(std::vector<float> pooled, double runs, double& a, double& k, double& inv_s2, double max_per_run) {
    std::sort(pooled.begin(), pooled.end(), std::greater<float>());
    const size_t m = std::min(pooled.size(), static_cast<size_t>(max_per_run * runs));
    if (m < 8) return false;
    double S[3][3] = {{0}}, R[3] = {0};
    for (size_t j = 0; j < m; ++j) {
        const double u = pooled[j];
        if (!(u > 0.0)) return false;
        const double f[3] = {1.0, std::log(u), -0.5 * u * u};
        const double y = std::log(static_cast<double>(j + 1) / runs);
        for (int r = 0; r < 3; ++r) {
            R[r] += f[r] * y;
            for (int c = 0; c < 3; ++c) S[r][c] += f[r] * f[c];
        }
    }
    double A[3][4];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) A[r][c] = S[r][c];
        A[r][3] = R[r];
    }
    for (int c = 0; c < 3; ++c) {
        int piv = c;
        for (int r = c + 1; r < 3; ++r)
            if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
        if (std::fabs(A[piv][c]) < 1e-300) return false;
        for (int q = 0; q < 4; ++q) std::swap(A[c][q], A[piv][q]);
        for (int r = 0; r < 3; ++r) {
            if (r == c) continue;
            const double f = A[r][c] / A[c][c];
            for (int q = c; q < 4; ++q) A[r][q] -= f * A[c][q];
        }
    }
    a = A[0][3] / A[0][0];
    k = A[1][3] / A[1][1];
    inv_s2 = A[2][3] / A[2][2];
    return std::isfinite(a) && std::isfinite(k) && inv_s2 > 0.0 && std::isfinite(inv_s2);
}

double log_rate(double a, double k, double inv_s2, double u) { return a + k * std::log(u) - 0.5 * inv_s2 * u * u; }

// search.cpp:517-527
double tail_level(double a, double k, double inv_s2, double rate) {
    const double lt = std::log(rate);
    double lo = std::max(1.0, k > 0.0 ? std::sqrt(k / inv_s2) : 1.0), hi = 100.0;
    if (log_rate(a, k, inv_s2, lo) <= lt) return lo;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (log_rate(a, k, inv_s2, mid) > lt) lo = mid;
        else hi = mid;
    }
    return hi;
}

// search.cpp:529-553
bool fit_linear(std::vector<float> pooled, double runs, double& a, double& b) {
    std::sort(pooled.begin(), pooled.end(), std::greater<float>());
    std::vector<double> xs, ys;
    for (size_t j = 0; j < pooled.size(); ++j) {
        const double npr = static_cast<double>(j + 1) / runs;
        if (npr < 0.67) continue;
        if (npr > 30.0) break;
        xs.push_back(pooled[j]);
        ys.push_back(std::log(npr));
    }
    if (xs.size() < 8) return false;
    const double mx = std::accumulate(xs.begin(), xs.end(), 0.0) / xs.size();
    const double my = std::accumulate(ys.begin(), ys.end(), 0.0) / ys.size();
    double sxy = 0, sxx = 0;
    for (size_t i = 0; i < xs.size(); ++i) {
        sxy += (xs[i] - mx) * (ys[i] - my);
        sxx += (xs[i] - mx) * (xs[i] - mx);
    }
    if (sxx <= 0.0) return false;
    const double slope = sxy / sxx;
    if (slope >= 0.0) return false;
    b = -slope;
    a = my + b * mx;
    return true;
}

}  // namespace

double expected_null_peaks(const Threshold& t, double snr) {
    if (t.inv_s2 > 0.0 && snr > 0.0) return std::exp(log_rate(t.a, t.k, t.inv_s2, snr));
    if (t.b > 0.0) return std::exp(t.a - t.b * snr);
    return 0.0;
}

Threshold set_threshold(const SearchParams& p, const std::vector<float>& pooled, int runs, double fwhm_px, int w,
                        int h, size_t n_motions) {
    Threshold t;
    if (p.threshold_snr > 0.0) {
        t.snr = p.threshold_snr;
        t.method = "fixed";
    } else if (runs > 0) {
        const double target = std::max(1e-6, p.target_false_per_run);
        if (p.gauss_model && fit_gauss(pooled, runs, t.a, t.k, t.inv_s2, 3000.0)) {
            t.snr = tail_level(t.a, t.k, t.inv_s2, target);
            t.method = "null-fit gauss";
        } else if (fit_linear(pooled, runs, t.a, t.b)) {
            t.k = t.inv_s2 = 0.0;
            t.snr = (t.a - std::log(target)) / t.b;
            t.method = "null-fit linear";
        } else {
            t.a = t.b = t.k = t.inv_s2 = 0.0;
            const float mx = pooled.empty() ? 0.0f : *std::max_element(pooled.begin(), pooled.end());
            t.snr = mx + 0.5;
            t.method = "null-quantile";
        }
        t.snr = std::max(t.snr, p.min_snr_floor);
    } else {
        const double resel = 4.0 * kPi * std::pow(fwhm_px * kFwhmToSigma, 2);
        const double trials = std::max(1.0, w * h / resel * n_motions * 0.5);
        double lo = 3.0, hi = 12.0;
        for (int it = 0; it < 60; ++it) {
            const double mid = 0.5 * (lo + hi);
            if (trials * (0.5 * std::erfc(mid / std::sqrt(2.0))) > p.target_false_per_run) lo = mid;
            else hi = mid;
        }
        t.snr = std::max(hi, p.min_snr_floor);
        t.method = "gaussian";
    }
    return t;
}

// The stellar FWHM from the static sky (preprocess.cpp:24-110): isolated local
// maxima between 25 sigma and 0.6 x the brightest pixel, background from an
// annulus, Gaussian-weighted adaptive second moments.
double estimate_fwhm(const std::vector<float>& img, int w, int h, double noise_sigma) {
    if (img.empty() || noise_sigma <= 0.0) return 0.0;
    auto at = [&](int x, int y) { return img[static_cast<size_t>(y) * w + x]; };
    float vmax = -1e30f;
    for (float v : img)
        if (std::isfinite(v)) vmax = std::max(vmax, v);
    const double lo = 25.0 * noise_sigma, hi = 0.6 * vmax;
    const int R = 5, B = 9;
    std::vector<double> fwhms;
    for (int y = B; y < h - B && fwhms.size() < 400; ++y) {
        for (int x = B; x < w - B && fwhms.size() < 400; ++x) {
            const float p = at(x, y);
            if (!(p > lo && p < hi)) continue;
            bool is_max = true;
            for (int dy = -1; dy <= 1 && is_max; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                    if ((dx || dy) && at(x + dx, y + dy) >= p) {
                        is_max = false;
                        break;
                    }
            if (!is_max) continue;
            bool fin = true;
            for (int dy = -R; dy <= R && fin; ++dy)
                for (int dx = -R; dx <= R; ++dx)
                    if (!std::isfinite(at(x + dx, y + dy))) {
                        fin = false;
                        break;
                    }
            if (!fin) continue;
            std::vector<float> ann;
            bool isolated = true;
            for (int dy = -B; dy <= B; ++dy)
                for (int dx = -B; dx <= B; ++dx) {
                    const double r = std::hypot(dx, dy);
                    const float v = at(x + dx, y + dy);
                    if (r > R + 1 && r <= B && std::isfinite(v)) ann.push_back(v);
                    if (r > 0 && v > p) isolated = false;
                    if (r > 2 && r <= B && v > 0.3f * p && x + dx > 0 && y + dy > 0 && x + dx < w - 1 && y + dy < h - 1) {
                        bool local = true;
                        for (int ey = -1; ey <= 1 && local; ++ey)
                            for (int ex = -1; ex <= 1; ++ex)
                                if ((ex || ey) && at(x + dx + ex, y + dy + ey) > v) {
                                    local = false;
                                    break;
                                }
                        if (local) isolated = false;
                    }
                }
            if (!isolated || ann.size() < 20) continue;
            const double bg = median_of(ann);
            const double peak = p - bg;
            const double n4 = 0.25 * (at(x - 1, y) + at(x + 1, y) + at(x, y - 1) + at(x, y + 1)) - bg;
            if (n4 < 0.2 * peak) continue;
            double sw2 = 1.5 * 1.5;
            bool good = true;
            for (int it = 0; it < 12 && good; ++it) {
                double s = 0, sxx = 0;
                for (int dy = -B; dy <= B; ++dy)
                    for (int dx = -B; dx <= B; ++dx) {
                        const float pv = at(x + dx, y + dy);
                        if (!std::isfinite(pv)) continue;
                        const double r2 = dx * dx + dy * dy;
                        const double wgt = std::exp(-0.5 * r2 / sw2);
                        const double v = (pv - bg) * wgt;
                        s += v;
                        sxx += v * r2;
                    }
                if (s <= 0) {
                    good = false;
                    break;
                }
                const double m = 0.5 * sxx / s;
                const double next = std::clamp(2.0 * m, 0.25, 49.0);
                if (std::fabs(next - sw2) < 1e-4) {
                    sw2 = next;
                    break;
                }
                sw2 = next;
            }
            if (!good) continue;
            const double var = sw2 - 1.0 / 12.0;
            if (var <= 0.1) continue;
            fwhms.push_back(2.354820045 * std::sqrt(var));
        }
    }
    if (fwhms.size() < 5) return 0.0;
    std::vector<float> f(fwhms.begin(), fwhms.end());
    return std::clamp(median_of(f), 1.0, 20.0);
}

// preprocess.cpp:256-263
double estimate_psf_fwhm(const std::vector<float>& static_sky, int w, int h, std::vector<double> sg,
                         const SearchParams& p) {
    const int n = static_cast<int>(sg.size());
    std::nth_element(sg.begin(), sg.begin() + n / 2, sg.end());
    const double static_noise = sg[static_cast<size_t>(n / 2)] / std::sqrt(static_cast<double>(n));
    double f = p.fwhm_px > 0.0 ? p.fwhm_px : estimate_fwhm(static_sky, w, h, static_noise);
    if (!(f > 0.0)) f = 3.0;
    return f;
}

// add_gaussian (psf.hpp:20-44) as a patch of float increments
static void gaussian_patch(InjectionPatches& ip, int frame, int w, int h, double x0, double y0, double flux,
                           double sigma) {
    const int max_radius = 30;
    if (flux <= 0.0 || sigma <= 0.0) return;
    const double peak = flux / (2.0 * kPi * sigma * sigma);
    int r = static_cast<int>(std::ceil(sigma * std::sqrt(2.0 * std::log(std::max(peak / 0.05, 2.0)))));
    r = std::clamp(r, 2, max_radius);
    const int xc = static_cast<int>(std::floor(x0 + 0.5));
    const int yc = static_cast<int>(std::floor(y0 + 0.5));
    const int x_lo = std::max(0, xc - r), x_hi = std::min(w - 1, xc + r);
    const int y_lo = std::max(0, yc - r), y_hi = std::min(h - 1, yc + r);
    if (x_lo > x_hi || y_lo > y_hi) return;
    const double inv = 1.0 / (sigma * std::sqrt(2.0));
    std::vector<double> wx(static_cast<size_t>(x_hi - x_lo + 1)), wy(static_cast<size_t>(y_hi - y_lo + 1));
    for (int x = x_lo; x <= x_hi; ++x)
        wx[static_cast<size_t>(x - x_lo)] = 0.5 * (std::erf((x + 0.5 - x0) * inv) - std::erf((x - 0.5 - x0) * inv));
    for (int y = y_lo; y <= y_hi; ++y)
        wy[static_cast<size_t>(y - y_lo)] = 0.5 * (std::erf((y + 0.5 - y0) * inv) - std::erf((y - 0.5 - y0) * inv));
    ip.frame.push_back(frame);
    ip.x0.push_back(x_lo);
    ip.y0.push_back(y_lo);
    ip.pw.push_back(x_hi - x_lo + 1);
    ip.ph.push_back(y_hi - y_lo + 1);
    ip.off.push_back(ip.values.size());
    for (int y = y_lo; y <= y_hi; ++y) {
        const double fy = flux * wy[static_cast<size_t>(y - y_lo)];
        for (int x = x_lo; x <= x_hi; ++x) ip.values.push_back(static_cast<float>(fy * wx[static_cast<size_t>(x - x_lo)]));
    }
}

InjectionPatches injection_patches(const std::vector<Injection>& objects, const std::vector<double>& t_mid_h,
                                   const std::vector<double>& exptime_s, double fwhm_px, int w, int h) {
    InjectionPatches ip;
    const double s = fwhm_px * kFwhmToSigma;
    for (size_t f = 0; f < t_mid_h.size(); ++f) {
        const double t_mid = t_mid_h[f];
        const double half = 0.5 * exptime_s[f] / 3600.0;
        for (const Injection& o : objects) {
            // add_trailed (psf.hpp:47-57)
            const double x0 = o.x_ref + o.vx_pxh * (t_mid - half), y0 = o.y_ref + o.vy_pxh * (t_mid - half);
            const double x1 = o.x_ref + o.vx_pxh * (t_mid + half), y1 = o.y_ref + o.vy_pxh * (t_mid + half);
            const double len = std::hypot(x1 - x0, y1 - y0);
            const int steps = std::max(1, static_cast<int>(std::ceil(len / 0.25)));
            const double fl = o.flux / steps;
            for (int k = 0; k < steps; ++k) {
                const double u = (k + 0.5) / steps;
                gaussian_patch(ip, static_cast<int>(f), w, h, x0 + u * (x1 - x0), y0 + u * (y1 - y0), fl, s);
            }
        }
    }
    return ip;
}

}  // namespace ftb
