// Test infrastructure only (see ft_oracle.h): the CPU restatement the parity
// tests check the CUDA path against. Written from the reference's algorithm
// description and arithmetic; each function cites the reference lines it
// follows. Must be compiled with -ffp-contract=off (oracle/Makefile does).
#include "ft_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <numeric>
#include <utility>
#include <vector>

namespace {

constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;  // psf.hpp:16
constexpr int kBlankGrow = 3;                              // internal.hpp:62

inline bool finite(float v) { return std::isfinite(v); }

// bilinear sample with the reference's border rule (common.hpp:125-138)
float bilinear(const float* img, int w, int h, double x, double y) {
    const int x0 = static_cast<int>(std::floor(x)), y0 = static_cast<int>(std::floor(y));
    if (x0 < 0 || y0 < 0 || x0 + 1 >= w || y0 + 1 >= h) {
        const int xr = static_cast<int>(std::lround(x)), yr = static_cast<int>(std::lround(y));
        const bool in = xr >= 0 && yr >= 0 && xr < w && yr < h;
        if (in && std::fabs(x - xr) < 1e-9 && std::fabs(y - yr) < 1e-9) return img[static_cast<size_t>(yr) * w + xr];
        return NAN;
    }
    const double fx = x - x0, fy = y - y0;
    const float* r0 = img + static_cast<size_t>(y0) * w + x0;
    const float* r1 = r0 + w;
    const double top = (1 - fx) * r0[0] + fx * r0[1];
    const double bot = (1 - fx) * r1[0] + fx * r1[1];
    return static_cast<float>((1 - fy) * top + fy * bot);
}

// xoshiro256** seeded by splitmix64 (random.hpp:14-42, 75-82)
struct Xoshiro {
    uint64_t s[4];
    explicit Xoshiro(uint64_t seed) {
        uint64_t z = seed;
        for (auto& v : s) {
            uint64_t r = (z += 0x9e3779b97f4a7c15ULL);
            r = (r ^ (r >> 30)) * 0xbf58476d1ce4e5b9ULL;
            r = (r ^ (r >> 27)) * 0x94d049bb133111ebULL;
            v = r ^ (r >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t out = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return out;
    }
    double uniform() { return static_cast<double>(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct PeakRec {
    int x, y;
    float snr;
    int vidx;
};

}  // namespace

extern "C" {

// median of finite values, mean of the middle two for even n (common.hpp:64-74)
double fto_median(float* v, size_t n) {
    if (n == 0) return 0.0;
    const size_t mid = n / 2;
    std::nth_element(v, v + mid, v + n);
    double m = v[mid];
    if (n % 2 == 0) {
        const float lower = *std::max_element(v, v + mid);
        m = 0.5 * (m + lower);
    }
    return m;
}

// 1.4826 * MAD (common.hpp:77-82); overwrites v
double fto_robust_sigma(float* v, size_t n) {
    if (n < 3) return 0.0;
    const double med = fto_median(v, n);
    for (size_t k = 0; k < n; ++k) v[k] = static_cast<float>(std::fabs(v[k] - med));
    return 1.4826 * fto_median(v, n);
}

// regular grid of finite samples, optional mask and border (common.hpp:85-100)
size_t fto_sample_pixels(const float* img, int w, int h, size_t max_samples, const float* mask, int border,
                         float* out) {
    const size_t usable = static_cast<size_t>(std::max(0, w - 2 * border)) * static_cast<size_t>(std::max(0, h - 2 * border));
    if (usable == 0) return 0;
    const int step = std::max(1, static_cast<int>(std::sqrt(static_cast<double>(usable) / max_samples)));
    size_t c = 0;
    for (int y = border; y < h - border; y += step)
        for (int x = border; x < w - border; x += step) {
            const size_t k = static_cast<size_t>(y) * w + x;
            if (mask && mask[k] == 0.0f) continue;
            if (finite(img[k])) out[c++] = img[k];
        }
    return c;
}

// rank of each frame in time, ties by index (preprocess.cpp:323-331)
void fto_time_rank(const double* t_h, int n, int* rank) {
    std::vector<int> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return t_h[a] < t_h[b]; });
    for (int r = 0; r < n; ++r) rank[order[static_cast<size_t>(r)]] = r;
}

// preprocess.cpp:332-333
int fto_static_exclude(int requested, int n) {
    return requested >= 0 ? requested : std::max(1, static_cast<int>(std::lround(n / 8.0)));
}

// per-pixel static sky and leave-out residuals (preprocess.cpp:154-204, 336-349).
// The global median adds the two middle floats in float; the leave-out median
// adds them in double -- exactly as the reference does.
void fto_static_sky(const float* sub, int w, int h, int n, const int* rank, int exclude, float* sky,
                    float* residual) {
    const size_t plane = static_cast<size_t>(w) * h;
    const size_t need = std::max<size_t>(5, static_cast<size_t>(0.6 * n));
#pragma omp parallel
    {
        std::vector<std::pair<float, int>> s;
        s.reserve(static_cast<size_t>(n));
#pragma omp for schedule(static)
        for (long long q = 0; q < static_cast<long long>(plane); ++q) {
            s.clear();
            for (int i = 0; i < n; ++i) {
                const float v = sub[i * plane + q];
                if (finite(v)) s.emplace_back(v, rank[i]);
            }
            if (s.size() < need) {
                sky[q] = NAN;
                for (int i = 0; i < n; ++i) residual[i * plane + q] = NAN;
                continue;
            }
            std::sort(s.begin(), s.end());
            const size_t m_all = s.size();
            const float mid_sum = s[(m_all - 1) / 2].first + s[m_all / 2].first;  // float add
            const double global = 0.5 * mid_sum;
            sky[q] = static_cast<float>(global);
            for (int i = 0; i < n; ++i) {
                const float v = sub[i * plane + q];
                if (!finite(v)) {
                    residual[i * plane + q] = NAN;
                    continue;
                }
                double st = global;
                if (exclude > 0) {
                    const int ri = rank[i];
                    size_t m = 0;
                    for (const auto& e : s) m += std::abs(e.second - ri) > exclude;
                    if (m >= 5) {
                        const size_t lo = (m - 1) / 2, hi = m / 2;
                        double a = 0.0, b = 0.0;
                        size_t k = 0;
                        for (const auto& e : s) {
                            if (std::abs(e.second - ri) <= exclude) continue;
                            if (k == lo) a = e.first;
                            if (k == hi) {
                                b = e.first;
                                break;
                            }
                            ++k;
                        }
                        st = 0.5 * (a + b);  // double add
                    }
                }
                residual[i * plane + q] = static_cast<float>(v - st);
            }
        }
    }
}

// per-frame residual noise from <= 200000 samples, border 2 (preprocess.cpp:356-365, 265-268)
double fto_frame_sigma(const float* residual, int w, int h) {
    std::vector<float> s(static_cast<size_t>(w) * h);
    const size_t c = fto_sample_pixels(residual, w, h, 200000, nullptr, 2, s.data());
    const double sg = fto_robust_sigma(s.data(), c);
    return sg > 0.0 ? sg : 1.0;
}

// temporal scatter map (preprocess.cpp:373-391)
void fto_scatter(const float* residual, int w, int h, int n, const double* sigma, float* scatter) {
    const size_t plane = static_cast<size_t>(w) * h;
#pragma omp parallel
    {
        std::vector<float> col(static_cast<size_t>(n));
#pragma omp for schedule(static)
        for (long long q = 0; q < static_cast<long long>(plane); ++q) {
            size_t c = 0;
            for (int i = 0; i < n; ++i) {
                const float v = residual[i * plane + q];
                if (finite(v)) col[c++] = static_cast<float>(std::fabs(v) / sigma[i]);
            }
            scatter[q] = c < static_cast<size_t>(n) / 2 ? 1e9f : static_cast<float>(1.4826 * fto_median(col.data(), c));
        }
    }
}

// mask: zero within +-dil of any pixel whose scatter exceeds mask_scatter (preprocess.cpp:392-400)
void fto_mask(const float* scatter, int w, int h, double fwhm_px, double mask_scatter, float* mask) {
    const int dil = std::max(1, static_cast<int>(std::lround(0.5 * fwhm_px)));
    std::fill(mask, mask + static_cast<size_t>(w) * h, 1.0f);
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            if (scatter[static_cast<size_t>(y) * w + x] <= mask_scatter) continue;
            for (int yy = std::max(0, y - dil); yy <= std::min(h - 1, y + dil); ++yy)
                for (int xx = std::max(0, x - dil); xx <= std::min(w - 1, x + dil); ++xx)
                    mask[static_cast<size_t>(yy) * w + xx] = 0.0f;
        }
}

// normalise + weight, cosmic-ray rejection, clip (preprocess.cpp:414-451).
// Returns the number of cosmic-ray hits.
int fto_normalise_frame(const float* r, const float* mask, const float* scatter, int w, int h, double sigma,
                        double fwhm_px, const fto_stage_params* sp, float* z) {
    const size_t plane = static_cast<size_t>(w) * h;
    const float inv = static_cast<float>(1.0 / sigma);
    const float wscat = static_cast<float>(sp->weight_scatter);
    for (size_t k = 0; k < plane; ++k) {
        z[k] = 0.0f;
        const float v = r[k];
        if (mask[k] == 0.0f || !finite(v)) continue;
        const float e = scatter[k] > wscat ? scatter[k] : 1.0f;
        const float vi = v * inv;
        z[k] = vi / e;
    }
    const double psf_sigma = fwhm_px * kFwhmToSigma;
    const float ratio = static_cast<float>(0.5 * std::exp(-0.5 / (psf_sigma * psf_sigma)));
    const float hit = static_cast<float>(sp->cr_sigma);
    std::vector<size_t> kill;
    int cr = 0;
    for (int y = 1; y < h - 1; ++y)
        for (int x = 1; x < w - 1; ++x) {
            const size_t k = static_cast<size_t>(y) * w + x;
            const float v = z[k];
            if (v < hit) continue;
            const float s4 = ((z[k - 1] + z[k + 1]) + z[k - w]) + z[k + w];
            const float n4 = 0.25f * s4;
            if (n4 >= ratio * v) continue;
            ++cr;
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const size_t q = static_cast<size_t>(y + dy) * w + (x + dx);
                    if ((dx == 0 && dy == 0) || z[q] > 2.5f) kill.push_back(q);
                }
        }
    for (size_t q : kill) z[q] = 0.0f;
    const float clip = static_cast<float>(sp->clip_sigma);
    for (size_t k = 0; k < plane; ++k) z[k] = z[k] < -clip ? -clip : (clip < z[k] ? clip : z[k]);
    return cr;
}

// separable Gaussian matched filter normalised by sum k^2 (preprocess.cpp:116-148)
void fto_matched_filter(const float* in, int w, int h, double sigma, float* out) {
    const int R = std::max(1, static_cast<int>(std::ceil(3.0 * sigma)));
    std::vector<float> k(static_cast<size_t>(2 * R + 1));
    double k2 = 0.0;
    for (int i = -R; i <= R; ++i) {
        const double v = std::exp(-0.5 * i * i / (sigma * sigma));
        k[static_cast<size_t>(i + R)] = static_cast<float>(v);
        k2 += v * v;
    }
    const float norm = static_cast<float>(1.0 / k2);
    std::vector<float> tmp(static_cast<size_t>(w) * h);
    for (int y = 0; y < h; ++y) {
        const float* row = in + static_cast<size_t>(y) * w;
        for (int x = 0; x < w; ++x) {
            const int a = std::max(0, x - R), b = std::min(w - 1, x + R);
            float acc = 0.0f;
            for (int j = a; j <= b; ++j) {
                const float prod = row[j] * k[static_cast<size_t>(j - x + R)];
                acc += prod;
            }
            tmp[static_cast<size_t>(y) * w + x] = acc;
        }
    }
    for (int y = 0; y < h; ++y) {
        const int a = std::max(0, y - R), b = std::min(h - 1, y + R);
        float* o = out + static_cast<size_t>(y) * w;
        for (int x = 0; x < w; ++x) o[x] = 0.0f;
        for (int j = a; j <= b; ++j) {
            const float kj = k[static_cast<size_t>(j - y + R)] * norm;
            const float* t = tmp.data() + static_cast<size_t>(j) * w;
            for (int x = 0; x < w; ++x) {
                const float prod = kj * t[x];
                o[x] += prod;
            }
        }
    }
}

// robust sigma of the unnormalised filter output over masked samples (preprocess.cpp:454-467)
double fto_filter_sigma(const float* g, const float* mask, int w, int h, double psf_sigma) {
    const int fborder = static_cast<int>(std::ceil(3 * psf_sigma)) + 1;
    std::vector<float> s(static_cast<size_t>(w) * h);
    const size_t c = fto_sample_pixels(g, w, h, 200000, mask, fborder, s.data());
    return fto_robust_sigma(s.data(), c);
}

// build_stage, whole image, fixed PSF width (preprocess.cpp:286-486)
void fto_build_stage(const float* sub, int w, int h, int n, const double* t_h, const fto_stage_params* sp,
                     float* filtered, float* static_sky, float* mask, double* sigma, int* cr, float* scatter_out) {
    const size_t plane = static_cast<size_t>(w) * h;
    std::vector<int> rank(static_cast<size_t>(n));
    fto_time_rank(t_h, n, rank.data());
    const int exclude = fto_static_exclude(sp->static_exclude, n);
    std::vector<float> residual(plane * n);
    fto_static_sky(sub, w, h, n, rank.data(), exclude, static_sky, residual.data());
    for (int i = 0; i < n; ++i) sigma[i] = fto_frame_sigma(residual.data() + i * plane, w, h);
    std::vector<float> scatter(plane);
    fto_scatter(residual.data(), w, h, n, sigma, scatter.data());
    fto_mask(scatter.data(), w, h, sp->fwhm_px, sp->mask_scatter, mask);
    if (scatter_out) std::memcpy(scatter_out, scatter.data(), plane * sizeof(float));
    const double psf_sigma = sp->fwhm_px * kFwhmToSigma;
#pragma omp parallel for schedule(dynamic)
    for (int i = 0; i < n; ++i) {
        std::vector<float> z(plane);
        cr[i] = fto_normalise_frame(residual.data() + i * plane, mask, scatter.data(), w, h, sigma[i], sp->fwhm_px, sp,
                                    z.data());
        float* g = filtered + i * plane;
        fto_matched_filter(z.data(), w, h, psf_sigma, g);
        const double sg = fto_filter_sigma(g, mask, w, h, psf_sigma);
        if (sg > 0.0) {
            const float ig = static_cast<float>(1.0 / sg);
            for (size_t k = 0; k < plane; ++k) g[k] *= ig;
        }
    }
}

// per-frame background: median of <= 200000 samples (preprocess.cpp:572-576)
double fto_background(const float* raw, int w, int h) {
    std::vector<float> s(static_cast<size_t>(w) * h);
    const size_t c = fto_sample_pixels(raw, w, h, 200000, nullptr, 0, s.data());
    return fto_median(s.data(), c);
}

// background subtraction and growth of blank areas by 3 px (preprocess.cpp:233-254)
void fto_subtract_and_grow(const float* raw, int w, int h, double bg, float* sub) {
    const size_t plane = static_cast<size_t>(w) * h;
    std::vector<unsigned char> bad(plane, 0);
    bool any = false;
    for (size_t k = 0; k < plane; ++k) {
        sub[k] = finite(raw[k]) ? static_cast<float>(raw[k] - bg) : NAN;
        if (!finite(sub[k])) {
            bad[k] = 1;
            any = true;
        }
    }
    if (!any) return;
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            if (!bad[static_cast<size_t>(y) * w + x]) continue;
            for (int yy = std::max(0, y - kBlankGrow); yy <= std::min(h - 1, y + kBlankGrow); ++yy)
                for (int xx = std::max(0, x - kBlankGrow); xx <= std::min(w - 1, x + kBlankGrow); ++xx)
                    sub[static_cast<size_t>(yy) * w + xx] = NAN;
        }
}

// the motion grid: square lattice of step dv inside the annulus, vy-major (search.cpp:39-58)
int fto_velocity_grid(double span_h, double vmin, double vmax, double grid_tol, double* out, int cap, double* dv_out) {
    if (span_h <= 0.0 || vmax <= 0.0 || vmax < vmin) return -1;
    const double dv = 4.0 * std::max(0.05, grid_tol) / span_h;
    if (dv_out) *dv_out = dv;
    const int K = static_cast<int>(std::ceil(vmax / dv));
    const double vlo = std::max(0.0, vmin - 0.5 * dv), vhi = vmax + 0.5 * dv;
    int c = 0;
    for (int j = -K; j <= K; ++j)
        for (int i = -K; i <= K; ++i) {
            const double vx = i * dv, vy = j * dv;
            const double v = std::hypot(vx, vy);
            if (v >= vlo && v <= vhi) {
                if (c < cap) {
                    out[2 * c] = vx;
                    out[2 * c + 1] = vy;
                }
                ++c;
            }
        }
    return c;
}

// round(v t) half away from zero, in double (backend.cpp:114-123)
void fto_shift_table(const double* t_h, int n, const double* vel, int m, int* dx, int* dy) {
    for (int j = 0; j < m; ++j)
        for (int i = 0; i < n; ++i) {
            dx[static_cast<size_t>(j) * n + i] = static_cast<int>(std::lround(vel[2 * j] * t_h[i]));
            dy[static_cast<size_t>(j) * n + i] = static_cast<int>(std::lround(vel[2 * j + 1] * t_h[i]));
        }
}

// search.cpp:98
int fto_min_count(double min_coverage, int n) {
    return std::max(3, static_cast<int>(std::ceil(min_coverage * n)));
}

// The stacking contract (backend.hpp:10-40; the plain form backend.cpp:128-172):
// per motion and pixel, covered frames summed in ascending order from +0.0f, times
// float(1/sqrt(c)); strict max over ascending motions; non-finite -> 0
// (backend_cpu.cpp:191-192). Motions run in parallel, one full-image accumulator
// each; per-thread maxima merge with the (value, lowest index) rule, which is the
// same order-independent result as the ascending strict scan.
void fto_stack(const float* frames, int w, int h, int n, const int* dx, const int* dy, int m, int min_count,
               float* max_snr, int* best_v) {
    const size_t plane = static_cast<size_t>(w) * h;
    std::vector<float> inv_sqrt(static_cast<size_t>(n) + 1, 0.0f);
    for (int c = 1; c <= n; ++c) inv_sqrt[static_cast<size_t>(c)] = static_cast<float>(1.0 / std::sqrt(static_cast<double>(c)));
    const float neg = -std::numeric_limits<float>::infinity();
    std::fill(max_snr, max_snr + plane, neg);
    std::fill(best_v, best_v + plane, -1);
#pragma omp parallel
    {
        std::vector<float> best(plane, neg), acc(plane);
        std::vector<int> arg(plane, -1), cnt(plane);
#pragma omp for schedule(dynamic, 1)
        for (int j = 0; j < m; ++j) {
            std::fill(acc.begin(), acc.end(), 0.0f);
            std::fill(cnt.begin(), cnt.end(), 0);
            for (int i = 0; i < n; ++i) {
                const int sx = dx[static_cast<size_t>(j) * n + i], sy = dy[static_cast<size_t>(j) * n + i];
                const long long x0 = std::max<long long>(0, -static_cast<long long>(sx));
                const long long x1 = std::min<long long>(w, static_cast<long long>(w) - sx);
                const long long y0 = std::max<long long>(0, -static_cast<long long>(sy));
                const long long y1 = std::min<long long>(h, static_cast<long long>(h) - sy);
                const float* g = frames + i * plane;
                for (long long y = y0; y < y1; ++y)
                    for (long long x = x0; x < x1; ++x) {
                        const size_t o = static_cast<size_t>(y) * w + static_cast<size_t>(x);
                        acc[o] += g[static_cast<size_t>(y + sy) * w + static_cast<size_t>(x + sx)];
                        ++cnt[o];
                    }
            }
            for (size_t o = 0; o < plane; ++o) {
                if (cnt[o] < min_count) continue;
                const float s = acc[o] * inv_sqrt[static_cast<size_t>(cnt[o])];
                if (s > best[o] || (s == best[o] && arg[o] >= 0 && j < arg[o])) {
                    best[o] = s;
                    arg[o] = j;
                }
            }
        }
#pragma omp critical
        for (size_t o = 0; o < plane; ++o) {
            if (arg[o] < 0) continue;
            if (best[o] > max_snr[o] || (best[o] == max_snr[o] && (best_v[o] < 0 || arg[o] < best_v[o]))) {
                max_snr[o] = best[o];
                best_v[o] = arg[o];
            }
        }
    }
    for (size_t o = 0; o < plane; ++o)
        if (!std::isfinite(max_snr[o])) max_snr[o] = 0.0f;
}

// K Fisher-Yates permutations of the frame times (search.cpp:559-571)
void fto_null_orders(const double* t_h, int n, int runs, unsigned long long seed, double* out) {
    Xoshiro rng(seed);
    for (int k = 0; k < runs; ++k) {
        double* t = out + static_cast<size_t>(k) * n;
        std::copy(t_h, t_h + n, t);
        for (size_t i = static_cast<size_t>(n) - 1; i > 0; --i) {
            const size_t j = static_cast<size_t>(rng.uniform() * (i + 1));
            std::swap(t[i], t[j]);
        }
    }
}

// local maxima with the plateau rule, then std::sort by S/N descending
// (search.cpp:105-135). The sort is the same (unstable) std::sort on the same
// raster-ordered sequence, so equal-S/N peaks come out in the same order.
int fto_find_peaks(const float* M, const int* best_v, int w, int h, float floor, int radius, int edge, int max_peaks,
                   int* px, int* py, float* psnr, int* pv) {
    std::vector<PeakRec> peaks;
    for (int y = edge; y < h - edge; ++y)
        for (int x = edge; x < w - edge; ++x) {
            const float v = M[static_cast<size_t>(y) * w + x];
            if (v < floor) continue;
            bool is_max = true;
            for (int dy = -radius; dy <= radius && is_max; ++dy) {
                const int yy = y + dy;
                if (yy < 0 || yy >= h) continue;
                for (int dx = -radius; dx <= radius; ++dx) {
                    const int xx = x + dx;
                    if ((!dx && !dy) || xx < 0 || xx >= w) continue;
                    const float u = M[static_cast<size_t>(yy) * w + xx];
                    if (u > v || (u == v && (dy < 0 || (dy == 0 && dx < 0)))) {
                        is_max = false;
                        break;
                    }
                }
            }
            if (is_max) peaks.push_back({x, y, v, best_v[static_cast<size_t>(y) * w + x]});
        }
    std::sort(peaks.begin(), peaks.end(), [](const PeakRec& a, const PeakRec& b) { return a.snr > b.snr; });
    if (static_cast<int>(peaks.size()) > max_peaks) peaks.resize(static_cast<size_t>(max_peaks));
    for (size_t k = 0; k < peaks.size(); ++k) {
        px[k] = peaks[k].x;
        py[k] = peaks[k].y;
        psnr[k] = peaks[k].snr;
        pv[k] = peaks[k].vidx;
    }
    return static_cast<int>(peaks.size());
}

// artefact tests at a peak's grid position and motion: single-frame share, field
// edge, detector-fixed (search.cpp:142-163, 167-190, 196-225, 229-243)
int fto_is_artefact_peak(const float* filtered, const float* sub, const float* static_sky, const double* t_h, int n,
                         int w, int h, double fwhm_px, int x, int y, double vx, double vy, double max_frame_fraction,
                         const double* reg_dx, const double* reg_dy) {
    const size_t plane = static_cast<size_t>(w) * h;
    double sum = 0.0;
    int count = 0;
    std::vector<double> per(static_cast<size_t>(n), NAN);
    for (int i = 0; i < n; ++i) {
        const double t = t_h[i];
        const double pxp = x + vx * t, pyp = y + vy * t;
        const float v = bilinear(filtered + i * plane, w, h, pxp, pyp);
        if (!finite(v)) continue;
        sum += v;
        ++count;
        per[static_cast<size_t>(i)] = v;
    }
    const double track_all = count >= 3 ? sum / std::sqrt(static_cast<double>(count)) : 0.0;
    double pos_sum = 0.0, maxc = 0.0;
    for (double v : per) {
        if (!std::isfinite(v)) continue;
        pos_sum += std::max(0.0, v);
        maxc = std::max(maxc, v);
    }
    const double frac = pos_sum > 0.0 ? maxc / pos_sum : 1.0;
    if (n >= 8 && frac > max_frame_fraction) return 1;
    // edge
    {
        const int r = static_cast<int>(std::ceil(2.0 * fwhm_px)) + 1;
        int near_blank = 0, total = 0;
        for (int i = 0; i < n; ++i) {
            const double t = t_h[i];
            const int xi = static_cast<int>(std::lround(x + vx * t)), yi = static_cast<int>(std::lround(y + vy * t));
            ++total;
            bool blank = false;
            for (int dy = -r; dy <= r && !blank; ++dy)
                for (int dx = -r; dx <= r; ++dx) {
                    const int xx = xi + dx, yy = yi + dy;
                    if (xx < 0 || yy < 0 || xx >= w || yy >= h || !finite(sub[i * plane + static_cast<size_t>(yy) * w + xx]) ||
                        !finite(static_sky[static_cast<size_t>(yy) * w + xx])) {
                        blank = true;
                        break;
                    }
                }
            near_blank += blank;
        }
        if (total > 0 && near_blank > std::max(1, total / 10)) return 1;
    }
    // detector
    if (!reg_dx || !reg_dy) return 0;
    double mx = 0, my = 0;
    for (int i = 0; i < n; ++i) {
        mx += x + vx * t_h[i] + reg_dx[i];
        my += y + vy * t_h[i] + reg_dy[i];
    }
    mx /= n;
    my /= n;
    double best_fixed = 0.0;
    const double span = std::max(2.0, 2.0 * fwhm_px);
    for (double dy = -span; dy <= span; dy += 0.5)
        for (double dx = -span; dx <= span; dx += 0.5) {
            double s = 0.0;
            int c = 0;
            for (int i = 0; i < n; ++i) {
                const float v = bilinear(filtered + i * plane, w, h, mx + dx - reg_dx[i], my + dy - reg_dy[i]);
                if (!finite(v)) continue;
                s += v;
                ++c;
            }
            best_fixed = std::max(best_fixed, c >= 3 ? s / std::sqrt(static_cast<double>(c)) : 0.0);
        }
    return best_fixed >= 0.8 * track_all ? 1 : 0;
}

}  // extern "C"

namespace {

// least-squares fit of log N(>u) = a + k log u - inv_s2 u^2 / 2 (search.cpp:471-510)
bool fit_gauss(std::vector<float> pooled, double runs, double& a, double& k, double& inv_s2, double max_per_run) {
    std::sort(pooled.begin(), pooled.end(), std::greater<float>());
    const size_t m = std::min(pooled.size(), static_cast<size_t>(max_per_run * runs));
    if (m < 8) return false;
    double S[3][3] = {{0}}, R[3] = {0};
    for (size_t j = 0; j < m; ++j) {
        const double u = pooled[j];
        if (!(u > 0.0)) return false;
        const double f[3] = {1.0, std::log(u), -0.5 * u * u};
        const double yv = std::log(static_cast<double>(j + 1) / runs);
        for (int r = 0; r < 3; ++r) {
            R[r] += f[r] * yv;
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

double tail_log_rate(double a, double k, double inv_s2, double u) { return a + k * std::log(u) - 0.5 * inv_s2 * u * u; }

// bisection for the level of `rate` peaks per run (search.cpp:517-527)
double tail_level(double a, double k, double inv_s2, double rate) {
    const double lt = std::log(rate);
    double lo = std::max(1.0, k > 0.0 ? std::sqrt(k / inv_s2) : 1.0), hi = 100.0;
    if (tail_log_rate(a, k, inv_s2, lo) <= lt) return lo;
    for (int it = 0; it < 200; ++it) {
        const double mid = 0.5 * (lo + hi);
        if (tail_log_rate(a, k, inv_s2, mid) > lt) lo = mid;
        else hi = mid;
    }
    return hi;
}

// log N(>s) = a - b s between 0.67 and 30 peaks per run (search.cpp:529-553)
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

extern "C" {

// threshold from the pooled null peaks (search.cpp:573-598). method: 1 gauss fit,
// 2 linear fit, 3 quantile. *k receives b for the linear model.
double fto_set_threshold(const float* pooled, int count, int runs, double target_false_per_run, double min_snr_floor,
                         int gauss, int* method, double* a, double* k, double* inv_s2) {
    const std::vector<float> p(pooled, pooled + count);
    const double target = std::max(1e-6, target_false_per_run);
    double thr;
    *a = *k = *inv_s2 = 0.0;
    if (gauss && fit_gauss(p, runs, *a, *k, *inv_s2, 3000.0)) {
        thr = tail_level(*a, *k, *inv_s2, target);
        *method = 1;
    } else if (fit_linear(p, runs, *a, *k)) {
        thr = (*a - std::log(target)) / *k;
        *method = 2;
    } else {
        const float mx = p.empty() ? 0.0f : *std::max_element(p.begin(), p.end());
        thr = mx + 0.5;
        *method = 3;
    }
    return std::max(thr, min_snr_floor);
}

}  // extern "C"
