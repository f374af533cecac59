// The registration check on the device (FaintTrail check_registration,
// registration.cpp:260-312, with find_stars, :36-89): the first, middle and last
// frame by time are sampled for their background and noise (the exact-median
// kernels of the stage) and scanned for stars in one launch, one thread per
// pixel; the star lists (at most 120 per frame after the cut) go to the host for
// the vote and the fit (registration_host.cpp).
//
// The scan reads each of the three frames once (4 bytes per pixel) and writes a
// 32-byte record per star: an HBM-bound pass of ~0.2 ms for three 4096^2 frames.
#include <algorithm>
#include <stdexcept>

#include "ft_internal.h"
#include "registration.h"
#include "stage.h"

namespace ftb {

namespace {

struct StarScan {
    const float* frame[3];
    float thr[3], nthr[3];
    double bg[3], sig[3];
    int active[3];
};

// one of the three frames' values, read from the kernel parameters (a dynamic
// index into a by-value argument would copy it to local memory)
template <class T>
__device__ __forceinline__ T pick(const T (&v)[3], int f) {
    return f == 0 ? v[0] : (f == 1 ? v[1] : v[2]);
}

// blockIdx.y: the frame (0 first, 1 middle, 2 last); one thread per pixel of
// the interior [4, w - 4) x [4, h - 4), in raster order. Stars are appended in
// any order (the host restores raster order); at most `cap` per frame are
// stored, the count is exact.
__global__ void __launch_bounds__(256) star_kernel(const StarScan a, int w, int h, int pitch, StarRec* out, int cap,
                                                   int* count) {
    const int f = blockIdx.y;
    if (!pick(a.active, f)) return;
    const int iw = w - 8, ih = h - 8;
    const long long g = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= static_cast<long long>(iw) * ih) return;
    const int x = 4 + static_cast<int>(g % iw), y = 4 + static_cast<int>(g / iw);
    StarRec s;
    if (!star_at(pick(a.frame, f), pitch, w, h, x, y, pick(a.thr, f), pick(a.nthr, f), pick(a.bg, f), pick(a.sig, f),
                 &s))
        return;
    const int k = atomicAdd(&count[f], 1);
    if (k < cap) out[static_cast<size_t>(f) * cap + k] = s;
}

}  // namespace

DriftCheck check_registration_three(Context& c, const float* const frames[3], int pitch, int w, int h, double dt_h) {
    if (w < 1 || h < 1 || pitch < w) throw std::runtime_error("registration check: bad frame geometry");
    const int span = c.span_begin("registration check");
    cudaStream_t s = c.stream();

    // background and noise of each frame's sample (find_stars, registration.cpp:37-41)
    const int cap = std::max(1, sample_grid_points(w, h, 0));
    DevBuf samples(&c, sizeof(float) * static_cast<size_t>(cap) * 3, "registration samples");
    DevBuf tab(&c, 256, "registration tables");
    double* d_stats = tab.as<double>();
    int* d_counts = reinterpret_cast<int*>(d_stats + 6);
    int* d_nstar = d_counts + 3;
    frame_sample_stats(c, frames, 3, w, h, pitch, samples.as<float>(), cap, d_counts, d_stats);
    double stats[6];
    int counts[3];
    FTB_CHECK(cudaMemcpyAsync(stats, d_stats, sizeof stats, cudaMemcpyDeviceToHost, s));
    FTB_CHECK(cudaMemcpyAsync(counts, d_counts, sizeof counts, cudaMemcpyDeviceToHost, s));
    FTB_CHECK(cudaStreamSynchronize(s));

    StarScan a{};
    bool any = false;
    for (int k = 0; k < 3; ++k) {
        a.frame[k] = frames[k];
        a.bg[k] = stats[k];
        a.sig[k] = stats[3 + k];
        a.thr[k] = static_cast<float>(a.bg[k] + 5.0 * a.sig[k]);
        a.nthr[k] = static_cast<float>(a.bg[k] + 2.5 * a.sig[k]);
        // fewer than 100 samples or no noise: no stars (registration.cpp:38, 41)
        a.active[k] = counts[k] >= 100 && a.sig[k] > 0 ? 1 : 0;
        any = any || a.active[k];
    }
    std::vector<StarRec> recs[3];
    if (any && w > 8 && h > 8) {
        const long long interior = static_cast<long long>(w - 8) * (h - 8);
        int scap = 1 << 14;
        for (;;) {
            DevBuf out(&c, sizeof(StarRec) * static_cast<size_t>(scap) * 3, "registration stars");
            FTB_CHECK(cudaMemsetAsync(d_nstar, 0, sizeof(int) * 3, s));
            star_kernel<<<dim3(static_cast<unsigned>((interior + 255) / 256), 3), 256, 0, s>>>(
                a, w, h, pitch, out.as<StarRec>(), scap, d_nstar);
            FTB_CHECK(cudaGetLastError());
            ++c.launches;
            int found[3];
            FTB_CHECK(cudaMemcpyAsync(found, d_nstar, sizeof found, cudaMemcpyDeviceToHost, s));
            FTB_CHECK(cudaStreamSynchronize(s));
            const int most = std::max(found[0], std::max(found[1], found[2]));
            if (most > scap) {  // more stars than room: rescan with room for all
                scap = most;
                continue;
            }
            for (int k = 0; k < 3; ++k) {
                recs[k].resize(static_cast<size_t>(found[k]));
                if (found[k] > 0)
                    FTB_CHECK(cudaMemcpyAsync(recs[k].data(), out.as<StarRec>() + static_cast<size_t>(k) * scap,
                                              sizeof(StarRec) * static_cast<size_t>(found[k]), cudaMemcpyDeviceToHost,
                                              s));
            }
            FTB_CHECK(cudaStreamSynchronize(s));
            break;
        }
    }
    c.span_end(span);
    FTB_CHECK(cudaStreamSynchronize(s));  // the span's end event is complete before timings are read
    const std::vector<Star> sa = order_stars(std::move(recs[0]), 60);
    const std::vector<Star> sm = order_stars(std::move(recs[1]), 120);
    const std::vector<Star> sl = order_stars(std::move(recs[2]), 120);
    return drift_from_stars(sa, sm, sl, w, h, dt_h);
}

DriftCheck check_registration_device(Context& c, const float* d_frames, size_t plane, int pitch, int w, int h, int n,
                                     const double* t_h) {
    if (n < 3) return DriftCheck{};
    int fi[3];
    registration_frames(t_h, n, &fi[0], &fi[1], &fi[2]);
    const float* frames[3];
    for (int k = 0; k < 3; ++k) frames[k] = d_frames + static_cast<size_t>(fi[k]) * plane;
    return check_registration_three(c, frames, pitch, w, h, t_h[fi[2]] - t_h[fi[0]]);
}

}  // namespace ftb
