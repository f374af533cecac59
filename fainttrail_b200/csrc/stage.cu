// The time-order-dependent preprocessing stage on the B200: FaintTrail's
// build_stage (preprocess.cpp:286-486) for a whole image with a fixed PSF width,
// bit-identical to the reference CPU code.
//
//  sky_kernel      static sky + leave-out residuals (preprocess.cpp:154-204)
//  sample + select per-frame residual noise: regular sample grid, exact medians
//                  by radix select (common.hpp:64-100, preprocess.cpp:356-365)
//  scatter_kernel  temporal scatter (preprocess.cpp:373-391)
//  mask_kernel     dilated scatter mask (preprocess.cpp:392-400)
//  filter_kernel   normalise + weight, cosmic-ray rejection, clip, separable
//                  matched filter, fused per tile (preprocess.cpp:414-451, 116-148)
//  sample + select robust sigma of the filter output, then rescale
//                  (preprocess.cpp:454-471)
//
// Arithmetic follows the reference operation by operation: float adds and
// multiplies with round-to-nearest and no contraction, double where the
// reference promotes to double, the same summation orders, NaN rules and casts.
#include <cooperative_groups.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#include "engine.h"
#include "search.h"
#include "stage.h"

namespace ftb {

namespace {

constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;  // psf.hpp:16

__device__ __forceinline__ bool finitef(float v) { return isfinite(v); }

// ------------------------------------------------------------------ static sky

struct SkyArgs {
    const float* sub;
    float* residual;
    float* sky;
    const unsigned char* rank;         // time rank of each frame
    const unsigned char* frame_of;     // frame of each time rank
    int w, h, pitch, n, exclude, need;
};

// One thread per pixel. The pixel's values are held in time-rank order, so the
// reference's sort of (value, time rank) pairs orders equal values by index.
// Each finite value's sorted position is counted against all others, eight
// values per pass over the column (the non-finite ones are held as +inf and
// never counted). The leave-out median of the frame of rank r is then the lo-th /
// hi-th sorted value outside the exclusion window [r - exclude, r + exclude]; the
// window's sorted positions are a bitmask of W words that slides one rank per
// frame (one position leaves, one enters), and the kept positions are picked
// with popc / fns.
// flips sorted position p (255: a non-finite value, no position) in the window
// mask; returns 1 if a position was flipped
template <int W>
__device__ __forceinline__ int sky_toggle(uint32_t (&ex)[W], int p) {
    if (p == 255) return 0;
#pragma unroll
    for (int wd = 0; wd < W; ++wd) ex[wd] ^= (p >> 5) == wd ? 1u << (p & 31) : 0u;
    return 1;
}

// Position of the k-th (0-based) set bit of x, k < popc(x): a binary search on
// the population counts of halves.
__device__ __forceinline__ int nth_set_bit(uint32_t x, int k) {
    int pos = 0;
    int c = __popc(x & 0xffffu);
    if (k >= c) { k -= c; pos += 16; x >>= 16; }
    c = __popc(x & 0xffu);
    if (k >= c) { k -= c; pos += 8; x >>= 8; }
    c = __popc(x & 0xfu);
    if (k >= c) { k -= c; pos += 4; x >>= 4; }
    c = __popc(x & 0x3u);
    if (k >= c) { k -= c; pos += 2; x >>= 2; }
    if (k >= static_cast<int>(x & 1u)) pos += 1;
    return pos;
}

// Position of the k-th (0-based) set bit of a 64-bit x, k < popc(x): the
// half that holds it by one population count, then nth_set_bit.
__device__ __forceinline__ int nth_set_bit64(uint64_t x, int k) {
    const uint32_t lo = static_cast<uint32_t>(x);
    const int c = __popc(lo);
    const bool up = k >= c;
    return (up ? 32 : 0) + nth_set_bit(up ? static_cast<uint32_t>(x >> 32) : lo, up ? k - c : k);
}

// sky_finish for at most 64 W64 frames: the kept sorted positions (set:
// outside the exclusion window) in W64 64-bit words (1 or 2), the lo-th by
// population counts (nth_set_bit64 within its word) and the hi-th, when it
// differs, as the next set bit above it.
template <int W64>
__device__ __forceinline__ void sky_finish_words(const SkyArgs& a, const float* V, const float* S,
                                                 const unsigned char* PF, int T, int t, int m_all, size_t pix,
                                                 size_t plane) {
    static_assert(W64 == 1 || W64 == 2, "one or two words");
    const int n = a.n, e = a.exclude;
    // global median: the two middle floats are added in float (preprocess.cpp:171)
    const float mid_sum = __fadd_rn(S[((m_all - 1) / 2) * T + t], S[(m_all / 2) * T + t]);
    const double global = 0.5 * static_cast<double>(mid_sum);
    a.sky[pix] = __double2float_rn(global);
    uint64_t k0 = m_all >= 64 ? ~0ull : (1ull << m_all) - 1ull;
    uint64_t k1 = W64 == 1 || m_all <= 64 ? 0ull : (m_all >= 128 ? ~0ull : (1ull << (m_all - 64)) - 1ull);
    int m = m_all;
    // flips position p (255: a non-finite value, none); d: the change in m
    auto flip = [&](int p, int d) {
        if (p == 255) return;
        const uint64_t b = 1ull << (p & 63);
        if (W64 == 1 || p < 64)
            k0 ^= b;
        else
            k1 ^= b;
        m += d;
    };
    if (e > 0)
        for (int r = 0; r <= min(e, n - 1); ++r) flip(PF[r * T + t], -1);  // rank 0's window
    for (int r = 0; r < n; ++r) {
        if (e > 0 && r > 0) {
            if (r - 1 - e >= 0) flip(PF[(r - 1 - e) * T + t], 1);  // leaves the window: kept again
            if (r + e < n) flip(PF[(r + e) * T + t], -1);          // enters: excluded
        }
        const float v = V[r * T + t];
        float* out = a.residual + a.frame_of[r] * plane + pix;
        if (v == CUDART_INF_F) {
            *out = CUDART_NAN_F;
            continue;
        }
        double st = global;
        if (e > 0 && m >= 5) {
            const int lo = (m - 1) / 2, hi = m / 2;
            int plo, phi;
            if (W64 == 1) {
                plo = nth_set_bit64(k0, lo);
                phi = hi == lo ? plo : plo + __ffsll(static_cast<long long>(k0 >> (plo + 1)));
            } else {
                const int c0 = __popcll(k0);
                plo = lo < c0 ? nth_set_bit64(k0, lo) : 64 + nth_set_bit64(k1, lo - c0);
                if (hi == lo) {
                    phi = plo;
                } else if (hi < c0) {  // the next kept position is in the first word
                    phi = plo + __ffsll(static_cast<long long>(k0 >> (plo + 1)));
                } else if (lo < c0) {  // plo is the first word's last: the second word's first
                    phi = 63 + __ffsll(static_cast<long long>(k1));
                } else {
                    phi = plo + __ffsll(static_cast<long long>(k1 >> (plo - 63)));
                }
            }
            // double add of the two middle values (preprocess.cpp:198)
            st = 0.5 * (static_cast<double>(S[plo * T + t]) + static_cast<double>(S[phi * T + t]));
        }
        *out = __double2float_rn(static_cast<double>(v) - st);
    }
}

// The static sky and the leave-out residuals of one pixel from its values by
// time rank (V, +inf where not finite), its m_all finite values in sorted order
// (S) and each rank's sorted position (PF, 255 where not finite).
template <int W>
__device__ __forceinline__ void sky_finish(const SkyArgs& a, const float* V, const float* S, const unsigned char* PF,
                                           int T, int t, int m_all, size_t pix, size_t plane) {
    const int n = a.n;
    // global median: the two middle floats are added in float (preprocess.cpp:171)
    const float mid_sum = __fadd_rn(S[((m_all - 1) / 2) * T + t], S[(m_all / 2) * T + t]);
    const double global = 0.5 * static_cast<double>(mid_sum);
    a.sky[pix] = __double2float_rn(global);
    uint32_t ex[W];
#pragma unroll
    for (int wd = 0; wd < W; ++wd) ex[wd] = 0;
    int excluded = 0;
    if (a.exclude > 0)
        for (int r = 0; r <= min(a.exclude, n - 1); ++r) excluded += sky_toggle<W>(ex, PF[r * T + t]);  // rank 0's window
    for (int r = 0; r < n; ++r) {
        if (a.exclude > 0 && r > 0) {
            if (r - 1 - a.exclude >= 0) excluded -= sky_toggle<W>(ex, PF[(r - 1 - a.exclude) * T + t]);
            if (r + a.exclude < n) excluded += sky_toggle<W>(ex, PF[(r + a.exclude) * T + t]);
        }
        const float v = V[r * T + t];
        float* out = a.residual + a.frame_of[r] * plane + pix;
        if (v == CUDART_INF_F) {
            *out = CUDART_NAN_F;
            continue;
        }
        double st = global;
        const int m = m_all - excluded;
        if (a.exclude > 0 && m >= 5) {
            const int lo = (m - 1) / 2, hi = m / 2;
            int plo = -1, phi = -1, seen = 0;
#pragma unroll
            for (int wd = 0; wd < W; ++wd) {
                const int nb = min(32, max(0, m_all - wd * 32));
                const uint32_t valid = nb >= 32 ? 0xffffffffu : ((1u << nb) - 1u);
                const uint32_t keep = ~ex[wd] & valid;
                const int c = __popc(keep);
                if (plo < 0 && lo < seen + c) plo = wd * 32 + nth_set_bit(keep, lo - seen);
                if (phi < 0 && hi < seen + c) phi = wd * 32 + nth_set_bit(keep, hi - seen);
                seen += c;
            }
            // double add of the two middle values (preprocess.cpp:198)
            st = 0.5 * (static_cast<double>(S[plo * T + t]) + static_cast<double>(S[phi * T + t]));
        }
        *out = __double2float_rn(static_cast<double>(v) - st);
    }
}

template <int W>
__global__ void __launch_bounds__(64) sky_kernel(const SkyArgs a) {
    extern __shared__ unsigned char sm[];
    const int T = blockDim.x, t = threadIdx.x;
    const int n = a.n;
    float* V = reinterpret_cast<float*>(sm);                            // [n][T] values by time rank, +inf if not finite
    float* S = V + n * T;                                               // [n][T] finite values in sorted order
    unsigned char* PF = reinterpret_cast<unsigned char*>(S + n * T);    // [n][T] sorted position by rank, 255: none
    const long long q = static_cast<long long>(blockIdx.x) * T + t;
    const int x = static_cast<int>(q % a.w), y = static_cast<int>(q / a.w);
    if (y >= a.h) return;
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    const size_t pix = static_cast<size_t>(y) * a.pitch + x;
    int m_all = 0;
    for (int r = 0; r < n; ++r) {
        const float v = a.sub[a.frame_of[r] * plane + pix];
        const bool fin = finitef(v);
        V[r * T + t] = fin ? v : CUDART_INF_F;
        m_all += fin;
    }
    if (m_all < a.need) {
        a.sky[pix] = CUDART_NAN_F;
        for (int i = 0; i < n; ++i) a.residual[i * plane + pix] = CUDART_NAN_F;
        return;
    }
    constexpr int B = 8;
    for (int e0 = 0; e0 < n; e0 += B) {
        float ve[B];
        int pos[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            ve[b] = e0 + b < n ? V[(e0 + b) * T + t] : CUDART_INF_F;
            pos[b] = 0;
        }
        for (int f = 0; f < e0; ++f) {  // lower ranks: equal values sort first
            const float vf = V[f * T + t];
#pragma unroll
            for (int b = 0; b < B; ++b) pos[b] += vf <= ve[b];
        }
        const int e1 = min(e0 + B, n);
        if (e1 - e0 == B) {
            // a full block against itself: rank e0 + c before rank e0 + b sorts an
            // equal value first, so the comparison is fixed per (c, b) pair
#pragma unroll
            for (int c = 0; c < B; ++c) {
                const float vf = V[(e0 + c) * T + t];
#pragma unroll
                for (int b = 0; b < B; ++b) pos[b] += c < b ? vf <= ve[b] : vf < ve[b];
            }
        } else {
            for (int f = e0; f < e1; ++f) {
                const float vf = V[f * T + t];
#pragma unroll
                for (int b = 0; b < B; ++b) pos[b] += vf < ve[b] || (vf == ve[b] && f < e0 + b);
            }
        }
        for (int f = e1; f < n; ++f) {  // higher ranks: only smaller values
            const float vf = V[f * T + t];
#pragma unroll
            for (int b = 0; b < B; ++b) pos[b] += vf < ve[b];
        }
#pragma unroll
        for (int b = 0; b < B; ++b) {
            if (e0 + b >= n) break;
            const bool fin = ve[b] != CUDART_INF_F;
            if (fin) S[pos[b] * T + t] = ve[b];
            PF[(e0 + b) * T + t] = fin ? static_cast<unsigned char>(pos[b]) : 255;
        }
    }
    if constexpr (W <= 2)
        sky_finish_words<1>(a, V, S, PF, T, t, m_all, pix, plane);
    else
        sky_finish<W>(a, V, S, PF, T, t, m_all, pix, plane);
}

// The same for n <= N <= 128 with the sorted order from a bitonic network in
// registers instead of counting ranks: the pixel's values (non-finite ones as
// +inf) are sorted with float min / max, which orders everything but the two
// zeros; where a -0.0 is present the zero run is rewritten with the zeros in
// time-rank order, which is the reference's order of equal (value, rank) pairs.
// Each rank's sorted position is then the lower bound of its value in the
// sorted values plus the number of equal values of lower rank.
template <int N>
__global__ void __launch_bounds__(64) sky_net_kernel(const SkyArgs a) {
    constexpr int W = (N + 31) / 32;
    extern __shared__ unsigned char sm[];
    const int T = blockDim.x, t = threadIdx.x;
    const int n = a.n;
    float* V = reinterpret_cast<float*>(sm);                            // [n][T] values by time rank, +inf if not finite
    float* S = V + n * T;                                               // [n][T] finite values in sorted order
    unsigned char* PF = reinterpret_cast<unsigned char*>(S + n * T);    // [n][T] sorted position by rank, 255: none
    const long long q = static_cast<long long>(blockIdx.x) * T + t;
    const int x = static_cast<int>(q % a.w), y = static_cast<int>(q / a.w);
    if (y >= a.h) return;
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    const size_t pix = static_cast<size_t>(y) * a.pitch + x;
    float sv[N];
    int m_all = 0;
    bool negzero = false;
#pragma unroll
    for (int r = 0; r < N; ++r) {
        float v = CUDART_INF_F;
        if (r < n) {
            const float u = a.sub[a.frame_of[r] * plane + pix];
            const bool fin = finitef(u);
            v = fin ? u : CUDART_INF_F;
            m_all += fin;
            negzero |= __float_as_uint(u) == 0x80000000u;
            V[r * T + t] = v;
        }
        sv[r] = v;
    }
    if (m_all < a.need) {
        a.sky[pix] = CUDART_NAN_F;
        for (int i = 0; i < n; ++i) a.residual[i * plane + pix] = CUDART_NAN_F;
        return;
    }
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const float lo = fminf(sv[i], sv[l]), hi = fmaxf(sv[i], sv[l]);
                    if ((i & k) == 0) {
                        sv[i] = lo;
                        sv[l] = hi;
                    } else {
                        sv[i] = hi;
                        sv[l] = lo;
                    }
                }
            }
#pragma unroll
    for (int p = 0; p < N; ++p)
        if (p < m_all) S[p * T + t] = sv[p];
    if (negzero) {
        int p = 0;
        while (p < m_all && S[p * T + t] < 0.0f) ++p;
        for (int r = 0; r < n; ++r) {
            const float v = V[r * T + t];
            if (v == 0.0f) S[(p++) * T + t] = v;
        }
    }
    for (int r = 0; r < n; ++r) {
        const float v = V[r * T + t];
        if (v == CUDART_INF_F) {
            PF[r * T + t] = 255;
            continue;
        }
        int lo = 0, len = m_all;
        while (len > 0) {
            const int half = len >> 1;
            if (S[(lo + half) * T + t] < v) {
                lo += half + 1;
                len -= half + 1;
            } else {
                len = half;
            }
        }
        int p = lo;
        if (lo + 1 < m_all && S[(lo + 1) * T + t] == v)
            for (int f = 0; f < r; ++f) p += V[f * T + t] == v;
        PF[r * T + t] = static_cast<unsigned char>(p);
    }
    if constexpr (N <= 128)
        sky_finish_words<(N + 63) / 64>(a, V, S, PF, T, t, m_all, pix, plane);
    else
        sky_finish<W>(a, V, S, PF, T, t, m_all, pix, plane);
}

// ------------------------------------------------------------------ samples + exact medians

// The regular sample grid of sample_pixels (common.hpp:85-100): every step-th
// column and row from `border`, finite values only, optionally masked. Order is
// irrelevant (only order statistics are taken); the count is exact.
__global__ void sample_kernel(const float* img, size_t plane, int w, int h, int pitch, int n, int border, int step,
                              int gw, int gh, const float* mask, float* out, int cap, int* counts) {
    const int f = blockIdx.y;
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= static_cast<long long>(gw) * gh) return;
    const int x = border + static_cast<int>(g % gw) * step, y = border + static_cast<int>(g / gw) * step;
    const size_t pix = static_cast<size_t>(y) * pitch + x;
    if (mask && mask[pix] == 0.0f) return;
    const float v = img[f * plane + pix];
    if (!finitef(v)) return;
    const int k = atomicAdd(&counts[f], 1);
    if (k < cap) out[static_cast<size_t>(f) * cap + k] = v;
}

// sample_kernel for a band of a larger image: the band holds image rows
// [oy, oy + rows) (row y at img + (y - oy) * pitch); the grid is the whole
// image's (columns border + i step, rows border + (j0 + j) step for the gh grid
// rows inside the band's core), so the samples are those the whole image gives
// in those rows.
__global__ void sample_band_kernel(const float* img, size_t plane, int pitch, int n, int border, int step, int gw,
                                   int j0, int gh, int oy, const float* mask, float* out, int cap, int* counts) {
    const int f = blockIdx.y;
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= static_cast<long long>(gw) * gh) return;
    const int x = border + static_cast<int>(g % gw) * step;
    const int y = border + (j0 + static_cast<int>(g / gw)) * step - oy;
    const size_t pix = static_cast<size_t>(y) * pitch + x;
    if (mask && mask[pix] == 0.0f) return;
    const float v = img[f * plane + pix];
    if (!finitef(v)) return;
    const int k = atomicAdd(&counts[f], 1);
    if (k < cap) out[static_cast<size_t>(f) * cap + k] = v;
}

__device__ __forceinline__ uint32_t order_key(float v) {
    const uint32_t b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key_value(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// k-th smallest key (0-based) of the CTA's values, by four 8-bit radix passes.
// MODE 0: keys of x; MODE 1: keys of float(|x - med|) (the MAD deviations,
// common.hpp:80). Needs >= 256 threads.
// ---- exact order statistics of a frame's samples by a cluster of CTAs: four
// 8-bit radix passes over order-preserving keys; each CTA counts its share of
// the samples into its own histogram, CTA 0 merges the cluster's histograms
// through distributed shared memory and picks the digit, and a cluster barrier
// separates the passes (eight SMs per frame).

namespace cg = cooperative_groups;
constexpr int kSelCluster = 8;

template <int MODE>
__device__ uint32_t cluster_select(const float* x, int cnt, int k, double med, uint32_t* hist, uint32_t* merged,
                                   uint32_t* res) {
    cg::cluster_group cl = cg::this_cluster();
    const unsigned rank = cl.block_rank();
    const int stride = static_cast<int>(blockDim.x) * kSelCluster;
    uint32_t prefix = 0, pmask = 0;
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
        cl.sync();  // no CTA still reads a histogram of the previous pass
        for (int e = static_cast<int>(rank * blockDim.x + threadIdx.x); e < cnt; e += stride) {
            float v = x[e];
            if (MODE == 1) v = __double2float_rn(fabs(static_cast<double>(v) - med));
            const uint32_t key = order_key(v);
            if ((key & pmask) == prefix) atomicAdd(&hist[(key >> shift) & 255u], 1u);
        }
        cl.sync();
        if (rank == 0) {
            for (int b = threadIdx.x; b < 256; b += blockDim.x) {
                uint32_t sum = 0;
                for (int r = 0; r < kSelCluster; ++r) sum += cl.map_shared_rank(hist, r)[b];
                merged[b] = sum;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                uint32_t acc = 0;
                int d = 0;
                for (; d < 255; ++d) {
                    if (acc + merged[d] > static_cast<uint32_t>(k)) break;
                    acc += merged[d];
                }
                res[0] = static_cast<uint32_t>(d);
                res[1] = acc;
            }
        }
        cl.sync();
        const uint32_t* r0 = cl.map_shared_rank(res, 0);
        const uint32_t d = r0[0];
        k -= static_cast<int>(r0[1]);
        prefix |= d << shift;
        pmask |= 255u << shift;
    }
    cl.sync();  // CTA 0's result is read before it is overwritten
    return prefix;
}

template <int MODE>
__device__ double cluster_median(const float* x, int cnt, double med, uint32_t* hist, uint32_t* merged, uint32_t* res) {
    if (cnt == 0) return 0.0;
    const int mid = cnt / 2;
    double m = key_value(cluster_select<MODE>(x, cnt, mid, med, hist, merged, res));
    if (cnt % 2 == 0) {
        const float lower = key_value(cluster_select<MODE>(x, cnt, mid - 1, med, hist, merged, res));
        m = 0.5 * (m + lower);
    }
    return m;
}

// robust_sigma_kernel with a cluster of kSelCluster CTAs per frame
__global__ void __cluster_dims__(kSelCluster, 1, 1) __launch_bounds__(256)
    robust_sigma_cluster_kernel(const float* samples, int cap, const int* counts, double* out, int unit_if_zero) {
    __shared__ uint32_t hist[256], merged[256], res[2];
    const int f = blockIdx.x / kSelCluster;
    const int cnt = min(counts[f], cap);
    const float* x = samples + static_cast<size_t>(f) * cap;
    double sg = 0.0;
    if (cnt >= 3) {
        const double med = cluster_median<0>(x, cnt, 0.0, hist, merged, res);
        sg = 1.4826 * cluster_median<1>(x, cnt, med, hist, merged, res);
    }
    if (cg::this_cluster().block_rank() == 0 && threadIdx.x == 0) out[f] = (unit_if_zero && !(sg > 0.0)) ? 1.0 : sg;
}

// median_kernel with a cluster per frame
__global__ void __cluster_dims__(kSelCluster, 1, 1) __launch_bounds__(256)
    median_cluster_kernel(const float* samples, int cap, const int* counts, double* out) {
    __shared__ uint32_t hist[256], merged[256], res[2];
    const int f = blockIdx.x / kSelCluster;
    const int cnt = min(counts[f], cap);
    const double m = cluster_median<0>(samples + static_cast<size_t>(f) * cap, cnt, 0.0, hist, merged, res);
    if (cg::this_cluster().block_rank() == 0 && threadIdx.x == 0) out[f] = m;
}

// ------------------------------------------------------------------ scatter + mask

struct ScatterArgs {
    const float* residual;
    const double* sigma;
    float* scatter;
    int w, h, pitch, n;
};

// scatter = 1.4826 * median_i float(|r_i| / sigma_i) over finite residuals, or
// 1e9 with fewer than n/2 of them (preprocess.cpp:380-389). The median's order
// statistics are found by counting (the values are >= 0, so their bit patterns
// order like the values).
__global__ void __launch_bounds__(128) scatter_kernel(const ScatterArgs a) {
    extern __shared__ unsigned char sm[];
    const int T = blockDim.x, t = threadIdx.x;
    uint32_t* C = reinterpret_cast<uint32_t*>(sm);
    const long long q = static_cast<long long>(blockIdx.x) * T + t;
    const int x = static_cast<int>(q % a.w), y = static_cast<int>(q / a.w);
    if (y >= a.h) return;
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    const size_t pix = static_cast<size_t>(y) * a.pitch + x;
    int c = 0;
    for (int i = 0; i < a.n; ++i) {
        const float v = a.residual[i * plane + pix];
        if (!finitef(v)) continue;
        const float d = __double2float_rn(__ddiv_rn(static_cast<double>(fabsf(v)), a.sigma[i]));
        C[c * T + t] = __float_as_uint(d);
        ++c;
    }
    if (c < a.n / 2) {
        a.scatter[pix] = 1e9f;
        return;
    }
    const int mid = c / 2;
    uint32_t vmid = 0, vlow = 0;
    for (int e = 0; e < c; ++e) {
        const uint32_t ve = C[e * T + t];
        int less = 0, leq = 0;
        for (int f = 0; f < c; ++f) {
            const uint32_t vf = C[f * T + t];
            less += vf < ve;
            leq += vf <= ve;
        }
        if (less <= mid && mid < leq) vmid = ve;
        if (less <= mid - 1 && mid - 1 < leq) vlow = ve;
    }
    double m = __uint_as_float(vmid);
    if (c % 2 == 0) m = 0.5 * (m + __uint_as_float(vlow));
    a.scatter[pix] = __double2float_rn(1.4826 * m);
}

// The same for n <= N <= 128 by a bitonic network in registers over the values'
// bit patterns (the values are >= +0.0 or +inf, so their patterns order like the
// values; absent frames are padded with 0xffffffff, above every pattern): the
// middle pair is then read from the sorted registers.
template <int N>
__global__ void __launch_bounds__(N <= 64 ? 128 : 64) scatter_net_kernel(const ScatterArgs a) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int x = static_cast<int>(q % a.w), y = static_cast<int>(q / a.w);
    if (y >= a.h) return;
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    const size_t pix = static_cast<size_t>(y) * a.pitch + x;
    uint32_t sv[N];
    int c = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        uint32_t key = 0xffffffffu;
        if (i < a.n) {
            const float v = a.residual[i * plane + pix];
            if (finitef(v)) {
                key = __float_as_uint(__double2float_rn(__ddiv_rn(static_cast<double>(fabsf(v)), a.sigma[i])));
                ++c;
            }
        }
        sv[i] = key;
    }
    if (c < a.n / 2) {
        a.scatter[pix] = 1e9f;
        return;
    }
#pragma unroll
    for (int k = 2; k <= N; k <<= 1)
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1)
#pragma unroll
            for (int i = 0; i < N; ++i) {
                const int l = i ^ j;
                if (l > i) {
                    const uint32_t lo = min(sv[i], sv[l]), hi = max(sv[i], sv[l]);
                    if ((i & k) == 0) {
                        sv[i] = lo;
                        sv[l] = hi;
                    } else {
                        sv[i] = hi;
                        sv[l] = lo;
                    }
                }
            }
    const int mid = c / 2;
    uint32_t vmid = 0, vlow = 0;
#pragma unroll
    for (int i = 0; i < N; ++i) {
        vmid = i == mid ? sv[i] : vmid;
        vlow = i == mid - 1 ? sv[i] : vlow;
    }
    double m = __uint_as_float(vmid);
    if (c % 2 == 0) m = 0.5 * (m + __uint_as_float(vlow));
    a.scatter[pix] = __double2float_rn(1.4826 * m);
}

__global__ void mask_kernel(const float* scatter, float* mask, int w, int h, int pitch, int dil, double limit) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int x = static_cast<int>(q % w), y = static_cast<int>(q / w);
    if (y >= h) return;
    float out = 1.0f;
    for (int yy = max(0, y - dil); yy <= min(h - 1, y + dil) && out != 0.0f; ++yy)
        for (int xx = max(0, x - dil); xx <= min(w - 1, x + dil); ++xx)
            if (static_cast<double>(scatter[static_cast<size_t>(yy) * pitch + xx]) > limit) {
                out = 0.0f;
                break;
            }
    mask[static_cast<size_t>(y) * pitch + x] = out;
}

// ------------------------------------------------------------------ matched filter


struct FilterArgs {
    const float* residual;
    const float* mask;
    const float* scatter;
    const double* sigma;   // per-frame residual noise
    float* out;            // unnormalised filter output
    int* cr;               // cosmic-ray hits per frame
    const float* k;        // 2R+1 taps, float(exp(-i^2 / 2 s^2))
    float norm;            // float(1 / sum k^2)
    float wscat, hit, ratio, clip;
    int w, h, pitch, R;
};

// One CTA per (frame, 32 x 16 tile). z (normalised, weighted) over the tile plus
// a halo of R + 2; cosmic-ray centres over the tile plus R + 1; cleaned and
// clipped z over the tile plus R; then the horizontal pass over the tile's
// columns and the vertical pass. Pixels outside the image hold 0: a product with
// 0 adds +0.0f to a sum that starts at +0.0f, which equals the reference's
// truncated sums at the borders (preprocess.cpp:133-135, 140-145).
// RT > 0: the filter radius fixed at compile time (the tile loops' index
// arithmetic by constants, the taps in registers); RT = 0: any radius (a.R).
// TWc x THc: the output tile.
template <int RT, int TWc, int THc>
__global__ void __launch_bounds__(256) filter_kernel(const FilterArgs a) {
    extern __shared__ float fs[];
    const int R = RT > 0 ? RT : a.R, H = R + 2;
    const int ZW = TWc + 2 * H, ZH = THc + 2 * H;
    float* Z = fs;                                    // ZH x ZW  z, then cleaned z
    unsigned char* F = reinterpret_cast<unsigned char*>(Z + ZW * ZH);  // ZH x ZW cosmic-ray centre flags
    float* Tt = reinterpret_cast<float*>(F + ((ZW * ZH + 15) / 16) * 16);  // (THc + 2R) x TWc horizontal pass
    __shared__ int cr_tile;
    constexpr int KN = RT > 0 ? 2 * RT + 1 : 1;
    float kr[KN], kn[KN];  // taps and taps x norm (the reference's float product) when RT > 0
    if constexpr (RT > 0) {
#pragma unroll
        for (int j = 0; j < KN; ++j) {
            kr[j] = a.k[j];
            kn[j] = __fmul_rn(kr[j], a.norm);
        }
    }
    const int f = blockIdx.z;
    const int x0 = blockIdx.x * TWc, y0 = blockIdx.y * THc;
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    const float inv = __double2float_rn(__ddiv_rn(1.0, a.sigma[f]));
    if (threadIdx.x == 0) cr_tile = 0;
    for (int e = threadIdx.x; e < ZW * ZH; e += blockDim.x) {
        const int gx = x0 - H + e % ZW, gy = y0 - H + e / ZW;
        float z = 0.0f;
        if (gx >= 0 && gy >= 0 && gx < a.w && gy < a.h) {
            // the three loads are independent, so they are in flight together
            const size_t pix = static_cast<size_t>(gy) * a.pitch + gx;
            const float v = __ldg(a.residual + f * plane + pix);
            const float mk = __ldg(a.mask + pix);
            const float s = __ldg(a.scatter + pix);
            if (mk != 0.0f && finitef(v)) {
                const float vm = __fmul_rn(v, inv);
                // (v / sigma) / e with e = scatter above weight_scatter, else 1 (an exact division)
                z = s > a.wscat ? __fdiv_rn(vm, s) : vm;
            }
        }
        Z[e] = z;
    }
    __syncthreads();
    // cosmic-ray centres (preprocess.cpp:433-447): inside [1, w-2] x [1, h-2]
    for (int e = threadIdx.x; e < ZW * ZH; e += blockDim.x) {
        const int lx = e % ZW, ly = e / ZW;
        const int gx = x0 - H + lx, gy = y0 - H + ly;
        unsigned char flag = 0;
        if (lx >= 1 && ly >= 1 && lx < ZW - 1 && ly < ZH - 1 && gx >= 1 && gy >= 1 && gx < a.w - 1 && gy < a.h - 1) {
            const float v = Z[e];
            if (v >= a.hit) {
                const float s4 = __fadd_rn(__fadd_rn(__fadd_rn(Z[e - 1], Z[e + 1]), Z[e - ZW]), Z[e + ZW]);
                const float n4 = __fmul_rn(0.25f, s4);
                if (!(n4 >= __fmul_rn(a.ratio, v))) {
                    flag = 1;
                    if (gx >= x0 && gx < x0 + TWc && gy >= y0 && gy < y0 + THc) atomicAdd(&cr_tile, 1);
                }
            }
        }
        F[e] = flag;
    }
    __syncthreads();
    // cleaned, clipped z over the tile plus R (kills applied after the scan)
    float* Zc = Z;  // in place: the kill test reads the original z of the same pixel only
    for (int e = threadIdx.x; e < ZW * ZH; e += blockDim.x) {
        const int lx = e % ZW, ly = e / ZW;
        if (lx < 2 || ly < 2 || lx >= ZW - 2 || ly >= ZH - 2) continue;
        const float v = Z[e];
        bool kill = F[e] != 0;
        if (!kill && v > 2.5f)
            for (int dy = -1; dy <= 1 && !kill; ++dy)
                for (int dx = -1; dx <= 1; ++dx)
                    if (F[e + dy * ZW + dx]) {
                        kill = true;
                        break;
                    }
        const float zc = kill ? 0.0f : v;
        Zc[e] = zc < -a.clip ? -a.clip : (a.clip < zc ? a.clip : zc);
    }
    __syncthreads();
    // horizontal pass over rows y0-R .. y0+THc+R-1, the tile's columns
    const int TR = THc + 2 * R;
    for (int e = threadIdx.x; e < TR * TWc; e += blockDim.x) {
        const int c = e % TWc, r = e / TWc;
        const float* row = Zc + (r + 2) * ZW + (c + 2);  // centre column at H + c, row at 2 + r (= H - R + r)
        float acc = 0.0f;
        if constexpr (RT > 0) {
#pragma unroll
            for (int j = 0; j < KN; ++j) acc = __fadd_rn(acc, __fmul_rn(row[j], kr[j]));
        } else {
            for (int j = 0; j <= 2 * R; ++j) acc = __fadd_rn(acc, __fmul_rn(row[j], a.k[j]));
        }
        const int gy = y0 - R + r;
        Tt[e] = (gy >= 0 && gy < a.h) ? acc : 0.0f;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < TWc * THc; e += blockDim.x) {
        const int c = e % TWc, r = e / TWc;
        const int gx = x0 + c, gy = y0 + r;
        if (gx >= a.w || gy >= a.h) continue;
        float acc = 0.0f;
        if constexpr (RT > 0) {
#pragma unroll
            for (int j = 0; j < KN; ++j) acc = __fadd_rn(acc, __fmul_rn(kn[j], Tt[(r + j) * TWc + c]));
        } else {
            for (int j = 0; j <= 2 * R; ++j)
                acc = __fadd_rn(acc, __fmul_rn(__fmul_rn(a.k[j], a.norm), Tt[(r + j) * TWc + c]));
        }
        a.out[f * plane + static_cast<size_t>(gy) * a.pitch + gx] = acc;
    }
    __syncthreads();
    if (threadIdx.x == 0 && cr_tile) atomicAdd(&a.cr[f], cr_tile);
}

// the static sky: counted ranks up to 64 frames (measured faster there: 554
// against 375 GB/s at 40 frames), the sorting network up to 128 (where the
// counting grows with n^2), counted ranks beyond
void launch_sky(const SkyArgs& a, int n, long long npix, cudaStream_t s) {
    const int T = 64;
    const size_t smem = static_cast<size_t>(T) * n * 9;
    auto kern = n <= 64 ? sky_kernel<2> : n <= 128 ? sky_net_kernel<128> : sky_kernel<8>;
    allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    kern<<<static_cast<unsigned>((npix + T - 1) / T), T, smem, s>>>(a);
    FTB_CHECK(cudaGetLastError());
}

// the temporal scatter: the sorting network up to 128 frames, counting beyond
void launch_scatter(const ScatterArgs& a, int n, long long npix, cudaStream_t s) {
    if (n <= 128) {
        const int T = n <= 64 ? 128 : 64;
        auto kern = n <= 32 ? scatter_net_kernel<32> : n <= 64 ? scatter_net_kernel<64> : scatter_net_kernel<128>;
        kern<<<static_cast<unsigned>((npix + T - 1) / T), T, 0, s>>>(a);
    } else {
        const int T = 128;
        const size_t smem = static_cast<size_t>(T) * n * 4;
        allow_dynamic_smem(reinterpret_cast<const void*>(scatter_kernel), smem);
        scatter_kernel<<<static_cast<unsigned>((npix + T - 1) / T), T, smem, s>>>(a);
    }
    FTB_CHECK(cudaGetLastError());
}

// 4-byte asynchronous copy global -> shared; a source outside the image copies
// nothing and fills zero (src-size 0).
__device__ __forceinline__ void cp_async4(float* dst, const float* src, bool valid) {
    const unsigned d = static_cast<unsigned>(__cvta_generic_to_shared(dst));
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(d), "l"(src), "r"(valid ? 4 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// The filter of filter_kernel for a run of frames per CTA (fixed radius RT):
// the tile's mask and scatter weight are read once for all its frames (one
// float per pixel: NaN where masked or outside the image, else the divisor,
// 1 for none), and the next frame's residual tile plus halo is copied
// asynchronously into a second buffer while the current one is filtered, so
// the loads of frame f + 1 overlap the arithmetic of frame f. Per frame the
// steps, their arithmetic and their order are filter_kernel's.
template <int RT, int TWc, int THc>
__global__ void __launch_bounds__(256) filter_frames_kernel(const FilterArgs a, int n, int fpc) {
    extern __shared__ float fs[];
    constexpr int R = RT, H = R + 2, ZW = TWc + 2 * H, ZH = THc + 2 * H, ZN = ZW * ZH, KN = 2 * RT + 1;
    constexpr int TR = THc + 2 * R;
    float* const Rb0 = fs;                  // residual tile + halo, double-buffered
    float* const Rb1 = fs + ZN;
    float* E = fs + 2 * ZN;                 // weight divisor, NaN: masked or outside
    float* Z = fs + 3 * ZN;                 // z, then cleaned and clipped z
    float* Tt = fs + 4 * ZN;                // TR x TWc horizontal pass
    unsigned char* F = reinterpret_cast<unsigned char*>(Tt + TR * TWc);  // ZN cosmic-ray centre flags
    __shared__ int cr_tile;
    static_assert(TWc % 4 == 0 && THc % 4 == 0, "tile in column quads and row quads");
    float kk[KN], kp[KN];  // the taps, and the taps times the norm (the reference's float product)
#pragma unroll
    for (int j = 0; j < KN; ++j) {
        kk[j] = a.k[j];
        kp[j] = __fmul_rn(kk[j], a.norm);
    }
    const int x0 = blockIdx.x * TWc, y0 = blockIdx.y * THc;
    const int fa = blockIdx.z * fpc, fb = min(n, fa + fpc);
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    const int tid = threadIdx.x;
    auto issue = [&](float* dst, int f) {
        const float* base = a.residual + f * plane;
        for (int e = tid; e < ZN; e += blockDim.x) {
            const int gx = x0 - H + e % ZW, gy = y0 - H + e / ZW;
            const bool in = gx >= 0 && gy >= 0 && gx < a.w && gy < a.h;
            cp_async4(dst + e, in ? base + static_cast<size_t>(gy) * a.pitch + gx : base, in);
        }
        cp_async_commit();
    };
    if (fa < fb) issue(Rb0, fa);
    for (int e = tid; e < ZN; e += blockDim.x) {
        const int gx = x0 - H + e % ZW, gy = y0 - H + e / ZW;
        float ev = CUDART_NAN_F;
        if (gx >= 0 && gy >= 0 && gx < a.w && gy < a.h) {
            const size_t pix = static_cast<size_t>(gy) * a.pitch + gx;
            const float mk = __ldg(a.mask + pix), sc = __ldg(a.scatter + pix);
            if (mk != 0.0f) ev = sc > a.wscat ? sc : 1.0f;
        }
        E[e] = ev;
    }
    for (int f = fa; f < fb; ++f) {
        const float* cur = ((f - fa) & 1) ? Rb1 : Rb0;
        cp_async_wait_all();
        __syncthreads();  // cur is complete; every thread is past its last read of the other buffer
        if (f + 1 < fb) issue(((f - fa) & 1) ? Rb0 : Rb1, f + 1);
        if (tid == 0) cr_tile = 0;
        const float inv = __double2float_rn(__ddiv_rn(1.0, a.sigma[f]));
        // z of element e: (v / sigma) / weight, 0 where masked, outside or not finite
        auto zval = [&](int e) {
            const float v = cur[e], ev = E[e];
            float z = 0.0f;
            if (ev == ev && finitef(v)) {
                const float vm = __fmul_rn(v, inv);
                // (v / sigma) / e, e = scatter above weight_scatter, else 1 (an exact division)
                z = ev != 1.0f ? __fdiv_rn(vm, ev) : vm;
            }
            return z;
        };
        // z over the tile + R + 2, and in the same pass the cosmic-ray centres
        // (preprocess.cpp:433-447, inside [1, w-2] x [1, h-2]): a z at or above
        // the hit level takes its four neighbours' z from the residual tile
        // (the same arithmetic as their own entries)
        for (int e = tid; e < ZN; e += blockDim.x) {
            const float v = zval(e);
            Z[e] = v;
            const int lx = e % ZW, ly = e / ZW;
            const int gx = x0 - H + lx, gy = y0 - H + ly;
            unsigned char flag = 0;
            if (v >= a.hit && lx >= 1 && ly >= 1 && lx < ZW - 1 && ly < ZH - 1 && gx >= 1 && gy >= 1 &&
                gx < a.w - 1 && gy < a.h - 1) {
                const float s4 = __fadd_rn(__fadd_rn(__fadd_rn(zval(e - 1), zval(e + 1)), zval(e - ZW)), zval(e + ZW));
                const float n4 = __fmul_rn(0.25f, s4);
                if (!(n4 >= __fmul_rn(a.ratio, v))) {
                    flag = 1;
                    if (gx >= x0 && gx < x0 + TWc && gy >= y0 && gy < y0 + THc) atomicAdd(&cr_tile, 1);
                }
            }
            F[e] = flag;
        }
        __syncthreads();
        // cleaned, clipped z over the tile plus R (kills applied after the scan)
        for (int e = tid; e < ZN; e += blockDim.x) {
            const int lx = e % ZW, ly = e / ZW;
            if (lx < 2 || ly < 2 || lx >= ZW - 2 || ly >= ZH - 2) continue;
            const float v = Z[e];
            bool kill = F[e] != 0;
            if (!kill && v > 2.5f)
                for (int dy = -1; dy <= 1 && !kill; ++dy)
                    for (int dx = -1; dx <= 1; ++dx)
                        if (F[e + dy * ZW + dx]) {
                            kill = true;
                            break;
                        }
            const float zc = kill ? 0.0f : v;
            Z[e] = zc < -a.clip ? -a.clip : (a.clip < zc ? a.clip : zc);
        }
        __syncthreads();
        // horizontal pass over rows y0-R .. y0+THc+R-1, the tile's columns: rows
        // in pairs (r, r + 1) and CQ adjacent columns per item; the pair's two
        // products of a tap are scalar round-to-nearest multiplies and their adds
        // into the pair's sums one __fadd2_rn (each output the reference's row[j]
        // * k[j] added in tap order), and the CQ columns share the loaded row
        // segments. The products stay scalar: a paired multiply followed by a
        // paired add was contracted into a fused multiply-add by the compiler
        // (even from inline PTX mul.rn.f32x2, and with --fmad=false), which rounds
        // once and differs from the reference in the last bits.
        {
            constexpr int CQ = 4, NV = CQ + KN - 1, ITEMS = (TR / 2) * (TWc / CQ);
            for (int it = tid; it < ITEMS; it += blockDim.x) {
                const int c = (it % (TWc / CQ)) * CQ, r = 2 * (it / (TWc / CQ));
                const float* r0 = Z + (r + 2) * ZW + (c + 2);
                float2 v[NV];
#pragma unroll
                for (int x = 0; x < NV; ++x) v[x] = make_float2(r0[x], r0[x + ZW]);
                const bool in0 = y0 - R + r >= 0 && y0 - R + r < a.h, in1 = y0 - R + r + 1 >= 0 && y0 - R + r + 1 < a.h;
#pragma unroll
                for (int q = 0; q < CQ; ++q) {
                    float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                    for (int j = 0; j < KN; ++j)
                        acc = __fadd2_rn(acc, make_float2(__fmul_rn(v[q + j].x, kk[j]), __fmul_rn(v[q + j].y, kk[j])));
                    Tt[r * TWc + c + q] = in0 ? acc.x : 0.0f;
                    Tt[(r + 1) * TWc + c + q] = in1 ? acc.y : 0.0f;
                }
            }
        }
        __syncthreads();
        // vertical pass: two adjacent columns (one 8-byte load of the horizontal
        // pass) and RQ rows per item, the loaded column pairs shared by the rows
        {
            constexpr int RQ = 4, NV = RQ + KN - 1, ITEMS = (THc / RQ) * (TWc / 2);
            float* out = a.out + f * plane;
            for (int it = tid; it < ITEMS; it += blockDim.x) {
                const int c = 2 * (it % (TWc / 2)), r = (it / (TWc / 2)) * RQ;
                const int gx = x0 + c;
                if (gx >= a.w) continue;
                float2 tv[NV];
#pragma unroll
                for (int x = 0; x < NV; ++x) tv[x] = *reinterpret_cast<const float2*>(Tt + (r + x) * TWc + c);
#pragma unroll
                for (int q = 0; q < RQ; ++q) {
                    const int gy = y0 + r + q;
                    if (gy >= a.h) break;
                    float2 acc = make_float2(0.0f, 0.0f);
#pragma unroll
                    for (int j = 0; j < KN; ++j)
                        acc = __fadd2_rn(acc, make_float2(__fmul_rn(kp[j], tv[q + j].x), __fmul_rn(kp[j], tv[q + j].y)));
                    float* o = out + static_cast<size_t>(gy) * a.pitch + gx;
                    if (gx + 1 < a.w) {
                        *reinterpret_cast<float2*>(o) = acc;
                    } else {
                        o[0] = acc.x;
                    }
                }
            }
        }
        if (tid == 0 && cr_tile) atomicAdd(&a.cr[f], cr_tile);
    }
}

template <int RT, int TWc, int THc>
void launch_filter_frames(const FilterArgs& a, int n, int sms, cudaStream_t s) {
    constexpr int H = RT + 2, ZW = TWc + 2 * H, ZH = THc + 2 * H, ZN = ZW * ZH;
    const size_t smem = sizeof(float) * (4 * ZN + (THc + 2 * RT) * TWc) + ((ZN + 15) / 16) * 16;
    const int tx = (a.w + TWc - 1) / TWc, ty = (a.h + THc - 1) / THc;
    // frames split over CTAs only when the tiles alone leave SMs idle
    const long long tiles = static_cast<long long>(tx) * ty;
    const int groups = static_cast<int>(std::min<long long>(n, std::max<long long>(1, (4LL * sms + tiles - 1) / tiles)));
    const int fpc = (n + groups - 1) / groups;
    auto kern = filter_frames_kernel<RT, TWc, THc>;
    allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    kern<<<dim3(tx, ty, (n + fpc - 1) / fpc), 256, smem, s>>>(a, n, fpc);
    FTB_CHECK(cudaGetLastError());
}

// one launch of the filter kernel for radius R (compile-time radius up to 8)
template <int RT, int TWc, int THc>
void launch_filter(const FilterArgs& a, int n, cudaStream_t s) {
    const int R = RT > 0 ? RT : a.R, H = R + 2, ZW = TWc + 2 * H, ZH = THc + 2 * H;
    const size_t smem = sizeof(float) * ZW * ZH + ((ZW * ZH + 15) / 16) * 16 + sizeof(float) * (THc + 2 * R) * TWc;
    auto kern = filter_kernel<RT, TWc, THc>;
    allow_dynamic_smem(reinterpret_cast<const void*>(kern), smem);
    kern<<<dim3((a.w + TWc - 1) / TWc, (a.h + THc - 1) / THc, n), 256, smem, s>>>(a);
    FTB_CHECK(cudaGetLastError());
}

void launch_filter_any(const FilterArgs& a, int n, int sms, cudaStream_t s) {
    switch (a.R) {
        case 1: launch_filter_frames<1, 64, 32>(a, n, sms, s); break;
        case 2: launch_filter_frames<2, 64, 32>(a, n, sms, s); break;
        case 3: launch_filter_frames<3, 64, 32>(a, n, sms, s); break;
        case 4: launch_filter_frames<4, 64, 32>(a, n, sms, s); break;
        case 5: launch_filter_frames<5, 64, 32>(a, n, sms, s); break;
        case 6: launch_filter_frames<6, 64, 32>(a, n, sms, s); break;
        case 7: launch_filter_frames<7, 64, 32>(a, n, sms, s); break;
        case 8: launch_filter_frames<8, 64, 32>(a, n, sms, s); break;
        default: launch_filter<0, 32, 16>(a, n, s); break;
    }
}

__global__ void rescale_kernel(float* g, size_t plane, int w, int h, int pitch, const double* sg) {
    const int f = blockIdx.y;
    const double s = sg[f];
    if (!(s > 0.0)) return;
    const float ig = __double2float_rn(__ddiv_rn(1.0, s));
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int x = static_cast<int>(q % w), y = static_cast<int>(q / w);
    if (y >= h) return;
    float* p = g + f * plane + static_cast<size_t>(y) * pitch + x;
    *p = __fmul_rn(*p, ig);
}

// v -> float(v - bg), NaN stays NaN (preprocess.cpp:235), in place
__global__ void subtract_kernel(float* img, size_t plane, int w, int h, int pitch, const double* bg) {
    const int f = blockIdx.y;
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int x = static_cast<int>(q % w), y = static_cast<int>(q / w);
    if (y >= h) return;
    float* p = img + f * plane + static_cast<size_t>(y) * pitch + x;
    const float v = *p;
    *p = finitef(v) ? __double2float_rn(static_cast<double>(v) - bg[f]) : CUDART_NAN_F;
}

// blank areas grown by `grow` pixels: NaN wherever a non-finite pixel lies within
// +-grow in x and y (preprocess.cpp:240-253)
__global__ void grow_kernel(const float* in, float* out, size_t plane, int w, int h, int pitch, int grow) {
    const int f = blockIdx.y;
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int x = static_cast<int>(q % w), y = static_cast<int>(q / w);
    if (y >= h) return;
    const float* src = in + f * plane;
    bool bad = false;
    for (int yy = max(0, y - grow); yy <= min(h - 1, y + grow) && !bad; ++yy)
        for (int xx = max(0, x - grow); xx <= min(w - 1, x + grow); ++xx)
            if (!finitef(src[static_cast<size_t>(yy) * pitch + xx])) {
                bad = true;
                break;
            }
    out[f * plane + static_cast<size_t>(y) * pitch + x] = bad ? CUDART_NAN_F : src[static_cast<size_t>(y) * pitch + x];
}

inline int grid_step(int w, int h, int border, size_t max_samples) {
    const size_t usable = static_cast<size_t>(std::max(0, w - 2 * border)) * static_cast<size_t>(std::max(0, h - 2 * border));
    if (usable == 0) return 0;
    return std::max(1, static_cast<int>(std::sqrt(static_cast<double>(usable) / static_cast<double>(max_samples))));
}

inline int grid_count(int lo, int hi, int step) { return hi <= lo ? 0 : (hi - lo + step - 1) / step; }

}  // namespace

// ------------------------------------------------------------------ host driver

void stage_time_ranks(const double* t_h, int n, std::vector<int>& rank) {
    // stable sort of the frame indices by time (preprocess.cpp:323-331)
    std::vector<int> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return t_h[a] < t_h[b]; });
    rank.assign(static_cast<size_t>(n), 0);
    for (int r = 0; r < n; ++r) rank[static_cast<size_t>(order[static_cast<size_t>(r)])] = r;
}

int sample_grid_points(int w, int h, int border) {
    const int st = grid_step(w, h, border, 200000);
    return st > 0 ? grid_count(border, w - border, st) * grid_count(border, h - border, st) : 0;
}

namespace {
}  // namespace

int filter_border(double fwhm_px) { return static_cast<int>(std::ceil(3 * fwhm_px * kFwhmToSigma)) + 1; }

StageScratch::StageScratch(Context& c, int w, int h, int n, double fwhm_px) : w_(w), h_(h), n_(n) {
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * h;
    residual = DevBuf(&c, sizeof(float) * plane * n, "residuals");
    scatter = DevBuf(&c, sizeof(float) * plane, "scatter map");
    // room for any sample grid this stage can use (borders 0 .. 64, and the PSF's)
    cap = std::max(1, sample_grid_points(w, h, filter_border(fwhm_px)));
    for (int b = 0; b <= 64; ++b) cap = std::max(cap, sample_grid_points(w, h, b));
    samples = DevBuf(&c, sizeof(float) * static_cast<size_t>(cap) * n, "noise samples");
    small = DevBuf(&c, 4096 + sizeof(double) * 2 * n + sizeof(int) * 2 * n + 2 * static_cast<size_t>(n), "stage tables");
}

bool StageScratch::fits(int w, int h, int n, double fwhm_px) const {
    return w == w_ && h == h_ && n == n_ && sample_grid_points(w, h, filter_border(fwhm_px)) <= cap;
}

bool StageScratch::holds(int w, int h, int n) const { return w == w_ && h <= h_ && n == n_; }

// The device tables of a stage in StageScratch::small: filter taps, per-frame
// sigma, filter sigma, sample counts, cosmic-ray tallies, rank tables.
struct StageTables {
    float* taps;
    double* sigma;
    double* sg;
    int* counts;
    int* cr;
    unsigned char* tab;
};

static StageTables stage_tables(StageScratch& sc, int n) {
    unsigned char* base = sc.small.as<unsigned char>();
    StageTables t;
    t.taps = reinterpret_cast<float*>(base);  // up to 512 floats
    t.sigma = reinterpret_cast<double*>(base + 2048);
    t.sg = t.sigma + n;
    t.counts = reinterpret_cast<int*>(t.sg + n);
    t.cr = t.counts + n;
    t.tab = reinterpret_cast<unsigned char*>(t.cr + n);
    return t;
}

void stage_noise(Context& c, StageScratch& sc, const float* d_sub, int w, int h, int n, const double* t_h,
                 int static_exclude, float* d_sky) {
    if (n < 1 || n > 255) throw std::runtime_error("stage: between 1 and 255 frames are supported");
    if (w != sc.w_ || h != sc.h_ || n != sc.n_) throw std::runtime_error("stage: scratch sized for another shape");
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * h;
    const long long npix = static_cast<long long>(w) * h;
    cudaStream_t s = c.stream();
    const StageTables tb = stage_tables(sc, n);

    // host tables: time ranks and the frame of each rank
    std::vector<int> rank;
    stage_time_ranks(t_h, n, rank);
    const int exclude = static_exclude >= 0 ? static_exclude : std::max(1, static_cast<int>(std::lround(n / 8.0)));
    std::vector<unsigned char> tab(2 * static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        tab[static_cast<size_t>(i)] = static_cast<unsigned char>(rank[static_cast<size_t>(i)]);
        tab[static_cast<size_t>(n + rank[static_cast<size_t>(i)])] = static_cast<unsigned char>(i);
    }
    FTB_CHECK(cudaMemcpyAsync(tb.tab, tab.data(), tab.size(), cudaMemcpyHostToDevice, s));
    FTB_CHECK(cudaMemsetAsync(tb.counts, 0, sizeof(int) * 2 * n, s));  // counts and cosmic-ray tallies
    // 1. static sky + residuals
    {
        const int span = c.span_begin("static sky + residuals");
        SkyArgs a{d_sub, sc.residual.as<float>(), d_sky, tb.tab, tb.tab + n, w, h, pitch, n, exclude,
                  std::max(5, static_cast<int>(0.6 * n))};
        launch_sky(a, n, npix, s);
        ++c.launches;
        c.span_end(span);
    }
    // 2. per-frame noise from the residual samples (border 2)
    {
        const int span = c.span_begin("noise");
        const int st = grid_step(w, h, 2, 200000);
        if (st > 0) {
            const int gw = grid_count(2, w - 2, st), gh = grid_count(2, h - 2, st);
            const long long g = static_cast<long long>(gw) * gh;
            sample_kernel<<<dim3(static_cast<unsigned>((g + 255) / 256), n), 256, 0, s>>>(
                sc.residual.as<float>(), plane, w, h, pitch, n, 2, st, gw, gh, nullptr, sc.samples.as<float>(), sc.cap,
                tb.counts);
            FTB_CHECK(cudaGetLastError());
        ++c.launches;
        }
        robust_sigma_cluster_kernel<<<n * kSelCluster, 256, 0, s>>>(sc.samples.as<float>(), sc.cap, tb.counts,
                                                                     tb.sigma, 1);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        c.span_end(span);
    }
}

void stage_filter(Context& c, StageScratch& sc, int w, int h, int n, const StageParams& sp, float* d_filtered,
                  float* d_mask, double* h_sigma, int* h_cr) {
    if (!sc.fits(w, h, n, sp.fwhm_px)) throw std::runtime_error("stage: scratch sized for another shape");
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * h;
    const long long npix = static_cast<long long>(w) * h;
    cudaStream_t s = c.stream();
    const StageTables tb = stage_tables(sc, n);
    // the separable filter taps (preprocess.cpp:118-126)
    const double psf_sigma = sp.fwhm_px * kFwhmToSigma;
    const int R = std::max(1, static_cast<int>(std::ceil(3.0 * psf_sigma)));
    std::vector<float> taps(static_cast<size_t>(2 * R + 1));
    double k2 = 0.0;
    for (int i = -R; i <= R; ++i) {
        const double v = std::exp(-0.5 * i * i / (psf_sigma * psf_sigma));
        taps[static_cast<size_t>(i + R)] = static_cast<float>(v);
        k2 += v * v;
    }
    if (taps.size() > 512) throw std::runtime_error("stage: PSF too wide");
    FTB_CHECK(cudaMemcpyAsync(tb.taps, taps.data(), sizeof(float) * taps.size(), cudaMemcpyHostToDevice, s));
    float* d_taps = tb.taps;
    double* d_sigma = tb.sigma;
    double* d_sg = tb.sg;
    int* d_counts = tb.counts;
    int* d_cr = tb.cr;
    // 3. scatter map and mask
    {
        const int span = c.span_begin("scatter mask");
        ScatterArgs a{sc.residual.as<float>(), d_sigma, sc.scatter.as<float>(), w, h, pitch, n};
        launch_scatter(a, n, npix, s);
        ++c.launches;
        const int dil = std::max(1, static_cast<int>(std::lround(0.5 * sp.fwhm_px)));
        mask_kernel<<<static_cast<unsigned>((npix + 255) / 256), 256, 0, s>>>(sc.scatter.as<float>(), d_mask, w, h,
                                                                              pitch, dil, sp.mask_scatter);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        c.span_end(span);
    }
    // 4. normalise, cosmic rays, clip, matched filter
    {
        const int span = c.span_begin("matched filter");
        FilterArgs a;
        a.residual = sc.residual.as<float>();
        a.mask = d_mask;
        a.scatter = sc.scatter.as<float>();
        a.sigma = d_sigma;
        a.out = d_filtered;
        a.cr = d_cr;
        a.k = d_taps;
        a.norm = static_cast<float>(1.0 / k2);
        a.wscat = static_cast<float>(sp.weight_scatter);
        a.hit = static_cast<float>(sp.cr_sigma);
        a.ratio = static_cast<float>(0.5 * std::exp(-0.5 / (psf_sigma * psf_sigma)));
        a.clip = static_cast<float>(sp.clip_sigma);
        a.w = w;
        a.h = h;
        a.pitch = pitch;
        a.R = R;
        launch_filter_any(a, n, c.sms(), s);
        ++c.launches;
        c.span_end(span);
    }
    // 5. robust sigma of the masked filter output (border ceil(3 s) + 1), rescale
    {
        const int span = c.span_begin("filter normalisation");
        const int fb = static_cast<int>(std::ceil(3 * psf_sigma)) + 1;
        FTB_CHECK(cudaMemsetAsync(d_counts, 0, sizeof(int) * n, s));
        const int st = grid_step(w, h, fb, 200000);
        if (st > 0) {
            const int gw = grid_count(fb, w - fb, st), gh = grid_count(fb, h - fb, st);
            const long long g = static_cast<long long>(gw) * gh;
            if (static_cast<long long>(gw) * gh > sc.cap) throw std::runtime_error("stage: sample buffer too small");
            sample_kernel<<<dim3(static_cast<unsigned>((g + 255) / 256), n), 256, 0, s>>>(
                d_filtered, plane, w, h, pitch, n, fb, st, gw, gh, d_mask, sc.samples.as<float>(), sc.cap, d_counts);
            FTB_CHECK(cudaGetLastError());
        ++c.launches;
        }
        robust_sigma_cluster_kernel<<<n * kSelCluster, 256, 0, s>>>(sc.samples.as<float>(), sc.cap, d_counts, d_sg,
                                                                     0);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        rescale_kernel<<<dim3(static_cast<unsigned>((npix + 255) / 256), n), 256, 0, s>>>(d_filtered, plane, w, h, pitch,
                                                                                       d_sg);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        c.span_end(span);
    }
    if (h_sigma) FTB_CHECK(cudaMemcpyAsync(h_sigma, d_sigma, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
    if (h_cr) FTB_CHECK(cudaMemcpyAsync(h_cr, d_cr, sizeof(int) * n, cudaMemcpyDeviceToHost, s));
}

void stage_run(Context& c, StageScratch& sc, const float* d_sub, int w, int h, int n, const double* t_h,
               const StageParams& sp, float* d_filtered, float* d_sky, float* d_mask, double* h_sigma, int* h_cr) {
    stage_noise(c, sc, d_sub, w, h, n, t_h, sp.static_exclude, d_sky);
    stage_filter(c, sc, w, h, n, sp, d_filtered, d_mask, h_sigma, h_cr);
}

void stage_sigma_to_host(Context& c, StageScratch& sc, int n, double* h_sigma) {
    FTB_CHECK(cudaMemcpyAsync(h_sigma, stage_tables(sc, n).sigma, sizeof(double) * n, cudaMemcpyDeviceToHost,
                              c.stream()));
}

void prepare_sub(Context& c, StageScratch& sc, float* d_raw, float* d_sub, int w, int h, int n, double* h_bg) {
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * h;
    const long long npix = static_cast<long long>(w) * h;
    cudaStream_t s = c.stream();
    const StageTables tb = stage_tables(sc, n);
    const int span = c.span_begin("background + borders");
    FTB_CHECK(cudaMemsetAsync(tb.counts, 0, sizeof(int) * n, s));
    const int st = grid_step(w, h, 0, 200000);
    if (st > 0) {
        const int gw = grid_count(0, w, st), gh = grid_count(0, h, st);
        const long long g = static_cast<long long>(gw) * gh;
        sample_kernel<<<dim3(static_cast<unsigned>((g + 255) / 256), n), 256, 0, s>>>(
            d_raw, plane, w, h, pitch, n, 0, st, gw, gh, nullptr, sc.samples.as<float>(), sc.cap, tb.counts);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
    }
    median_cluster_kernel<<<n * kSelCluster, 256, 0, s>>>(sc.samples.as<float>(), sc.cap, tb.counts, tb.sg);
    FTB_CHECK(cudaGetLastError());
        ++c.launches;
    const dim3 grid(static_cast<unsigned>((npix + 255) / 256), n);
    subtract_kernel<<<grid, 256, 0, s>>>(d_raw, plane, w, h, pitch, tb.sg);
    FTB_CHECK(cudaGetLastError());
        ++c.launches;
    grow_kernel<<<grid, 256, 0, s>>>(d_raw, d_sub, plane, w, h, pitch, 3);
    FTB_CHECK(cudaGetLastError());
        ++c.launches;
    c.span_end(span);
    if (h_bg) FTB_CHECK(cudaMemcpyAsync(h_bg, tb.sg, sizeof(double) * n, cudaMemcpyDeviceToHost, s));
}

// ------------------------------------------------------------------ bands (the tiled search)

void stage_sky(Context& c, StageScratch& sc, const float* d_sub, int w, int rows, int n, const double* t_h,
               int static_exclude, float* d_sky) {
    if (!sc.holds(w, rows, n)) throw std::runtime_error("stage: scratch sized for another shape");
    const int pitch = frame_pitch(w);
    const long long npix = static_cast<long long>(w) * rows;
    cudaStream_t s = c.stream();
    const StageTables tb = stage_tables(sc, n);
    std::vector<int> rank;
    stage_time_ranks(t_h, n, rank);
    const int exclude = static_exclude >= 0 ? static_exclude : std::max(1, static_cast<int>(std::lround(n / 8.0)));
    std::vector<unsigned char> tab(2 * static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) {
        tab[static_cast<size_t>(i)] = static_cast<unsigned char>(rank[static_cast<size_t>(i)]);
        tab[static_cast<size_t>(n + rank[static_cast<size_t>(i)])] = static_cast<unsigned char>(i);
    }
    FTB_CHECK(cudaMemcpyAsync(tb.tab, tab.data(), tab.size(), cudaMemcpyHostToDevice, s));
    const int span = c.span_begin("static sky + residuals");
    SkyArgs a{d_sub, sc.residual.as<float>(), d_sky, tb.tab, tb.tab + n, w, rows, pitch, n, exclude,
              std::max(5, static_cast<int>(0.6 * n))};
    launch_sky(a, n, npix, s);
    ++c.launches;
    c.span_end(span);
}

void sample_band(Context& c, const float* d_img, size_t plane, int pitch, int n, int w, int h, int border, int oy,
                 int core_y0, int core_y1, const float* d_mask, float* d_samples, int cap, int* d_counts) {
    const int st = grid_step(w, h, border, 200000);
    if (st <= 0) return;
    const int gw = grid_count(border, w - border, st);
    // the whole image's grid rows border + j st (< h - border) inside the core
    const int lo = std::max(core_y0, border), hi = std::min(core_y1, h - border);
    if (hi <= lo) return;
    const int j0 = (lo - border + st - 1) / st;
    const int j1 = (hi - border + st - 1) / st;
    const int gh = j1 - j0;
    if (gh <= 0 || gw <= 0) return;
    const long long g = static_cast<long long>(gw) * gh;
    sample_band_kernel<<<dim3(static_cast<unsigned>((g + 255) / 256), n), 256, 0, c.stream()>>>(
        d_img, plane, pitch, n, border, st, gw, j0, gh, oy, d_mask, d_samples, cap, d_counts);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
}

void select_sigma(Context& c, const float* d_samples, int cap, const int* d_counts, int n, double* d_out,
                  int unit_if_zero) {
    robust_sigma_cluster_kernel<<<n * kSelCluster, 256, 0, c.stream()>>>(d_samples, cap, d_counts, d_out,
                                                                          unit_if_zero);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
}

void select_median(Context& c, const float* d_samples, int cap, const int* d_counts, int n, double* d_out) {
    median_cluster_kernel<<<n * kSelCluster, 256, 0, c.stream()>>>(d_samples, cap, d_counts, d_out);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
}

void sample_frames(Context& c, const float* d_frames, size_t plane, int pitch, int n, int w, int h, int border,
                   float* d_samples, int cap, int* d_counts) {
    const int st = grid_step(w, h, border, 200000);
    if (st <= 0) return;
    const int gw = grid_count(border, w - border, st), gh = grid_count(border, h - border, st);
    const long long g = static_cast<long long>(gw) * gh;
    if (g > cap) throw std::runtime_error("sample_frames: sample buffer too small");
    sample_kernel<<<dim3(static_cast<unsigned>((g + 255) / 256), n), 256, 0, c.stream()>>>(
        d_frames, plane, w, h, pitch, n, border, st, gw, gh, nullptr, d_samples, cap, d_counts);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
}

void subtract_grow(Context& c, float* d_raw, float* d_sub, int w, int rows, int n, const double* d_bg) {
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * rows;
    const long long npix = static_cast<long long>(w) * rows;
    const dim3 grid(static_cast<unsigned>((npix + 255) / 256), n);
    subtract_kernel<<<grid, 256, 0, c.stream()>>>(d_raw, plane, w, rows, pitch, d_bg);
    FTB_CHECK(cudaGetLastError());
    grow_kernel<<<grid, 256, 0, c.stream()>>>(d_raw, d_sub, plane, w, rows, pitch, 3);
    FTB_CHECK(cudaGetLastError());
    c.launches += 2;
}

void stage_filter_given(Context& c, StageScratch& sc, int w, int rows, int n, const StageParams& sp,
                        const double* d_sigma, const double* d_sg, float* d_filtered, float* d_mask) {
    if (!sc.holds(w, rows, n)) throw std::runtime_error("stage: scratch sized for another shape");
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * rows;
    const long long npix = static_cast<long long>(w) * rows;
    cudaStream_t s = c.stream();
    const StageTables tb = stage_tables(sc, n);
    const double psf_sigma = sp.fwhm_px * kFwhmToSigma;
    const int R = std::max(1, static_cast<int>(std::ceil(3.0 * psf_sigma)));
    std::vector<float> taps(static_cast<size_t>(2 * R + 1));
    double k2 = 0.0;
    for (int i = -R; i <= R; ++i) {
        const double v = std::exp(-0.5 * i * i / (psf_sigma * psf_sigma));
        taps[static_cast<size_t>(i + R)] = static_cast<float>(v);
        k2 += v * v;
    }
    if (taps.size() > 512) throw std::runtime_error("stage: PSF too wide");
    FTB_CHECK(cudaMemcpyAsync(tb.taps, taps.data(), sizeof(float) * taps.size(), cudaMemcpyHostToDevice, s));
    {
        const int span = c.span_begin("scatter mask");
        ScatterArgs a{sc.residual.as<float>(), d_sigma, sc.scatter.as<float>(), w, rows, pitch, n};
        launch_scatter(a, n, npix, s);
        const int dil = std::max(1, static_cast<int>(std::lround(0.5 * sp.fwhm_px)));
        mask_kernel<<<static_cast<unsigned>((npix + 255) / 256), 256, 0, s>>>(sc.scatter.as<float>(), d_mask, w, rows,
                                                                              pitch, dil, sp.mask_scatter);
        FTB_CHECK(cudaGetLastError());
        c.launches += 2;
        c.span_end(span);
    }
    {
        const int span = c.span_begin("matched filter");
        FTB_CHECK(cudaMemsetAsync(tb.cr, 0, sizeof(int) * n, s));
        FilterArgs a;
        a.residual = sc.residual.as<float>();
        a.mask = d_mask;
        a.scatter = sc.scatter.as<float>();
        a.sigma = d_sigma;
        a.out = d_filtered;
        a.cr = tb.cr;
        a.k = tb.taps;
        a.norm = static_cast<float>(1.0 / k2);
        a.wscat = static_cast<float>(sp.weight_scatter);
        a.hit = static_cast<float>(sp.cr_sigma);
        a.ratio = static_cast<float>(0.5 * std::exp(-0.5 / (psf_sigma * psf_sigma)));
        a.clip = static_cast<float>(sp.clip_sigma);
        a.w = w;
        a.h = rows;
        a.pitch = pitch;
        a.R = R;
        launch_filter_any(a, n, c.sms(), s);
        ++c.launches;
        c.span_end(span);
    }
    if (d_sg) {
        rescale_kernel<<<dim3(static_cast<unsigned>((npix + 255) / 256), n), 256, 0, s>>>(d_filtered, plane, w, rows,
                                                                                       pitch, d_sg);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
    }
}

void frame_sample_stats(Context& c, const float* const* d_frames, int k, int w, int h, int pitch, float* d_samples,
                        int cap, int* d_counts, double* d_stats) {
    cudaStream_t s = c.stream();
    FTB_CHECK(cudaMemsetAsync(d_counts, 0, sizeof(int) * k, s));
    const int st = grid_step(w, h, 0, 200000);
    if (st > 0) {
        const int gw = grid_count(0, w, st), gh = grid_count(0, h, st);
        const long long g = static_cast<long long>(gw) * gh;
        if (g > cap) throw std::runtime_error("frame_sample_stats: sample buffer too small");
        for (int i = 0; i < k; ++i) {
            sample_kernel<<<dim3(static_cast<unsigned>((g + 255) / 256), 1), 256, 0, s>>>(
                d_frames[i], 0, w, h, pitch, 1, 0, st, gw, gh, nullptr, d_samples + static_cast<size_t>(i) * cap, cap,
                d_counts + i);
            FTB_CHECK(cudaGetLastError());
            ++c.launches;
        }
    }
    median_cluster_kernel<<<k * kSelCluster, 256, 0, s>>>(d_samples, cap, d_counts, d_stats);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
    robust_sigma_cluster_kernel<<<k * kSelCluster, 256, 0, s>>>(d_samples, cap, d_counts, d_stats + k, 0);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
}

}  // namespace ftb
