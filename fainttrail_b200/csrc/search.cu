// The search on the B200 (FaintTrail search.cpp:716-809 without the candidate
// refinement): prepare, the real pass and its peaks, the time-shuffled null
// runs (preprocessing rebuilt with permuted times, stack, peaks, artefact
// screen of the strongest null peaks), the null-tail fit and threshold, and the
// selected peaks. Pixel work runs on the device; the grid, the time orders, the
// peak order (std::sort, as the reference) and the fit run on the host.
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <numeric>
#include <thread>

#include "search.h"
#include "track.cuh"

namespace ftb {

namespace {

struct PeakRec {
    int x, y;
    float snr;
    int vidx;
};

// local maxima above `floor` inside the edge margin, strict for later pixels and
// non-strict for earlier ones, so a plateau yields one peak (search.cpp:110-129)
__device__ __forceinline__ bool is_peak(const float* M, int w, int h, float floor, int radius, int edge, int x, int y,
                                        float& v) {
    if (y >= h || x < edge || y < edge || x >= w - edge || y >= h - edge) return false;
    v = M[static_cast<size_t>(y) * w + x];
    if (v < floor) return false;
    for (int dy = -radius; dy <= radius; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -radius; dx <= radius; ++dx) {
            const int xx = x + dx;
            if ((!dx && !dy) || xx < 0 || xx >= w) continue;
            const float u = M[static_cast<size_t>(yy) * w + xx];
            if (u > v || (u == v && (dy < 0 || (dy == 0 && dx < 0)))) return false;
        }
    }
    return true;
}

// The peaks in raster order (the reference's visit order) without a sort: the
// peaks of each block of kPeakBlock consecutive pixels are counted, the counts
// scanned, and each block writes its peaks at its offset in pixel order.
constexpr int kPeakBlock = 256;

__global__ void __launch_bounds__(kPeakBlock) peak_count_kernel(const float* M, int w, int h, float floor, int radius,
                                                                int edge, int* block_count) {
    const long long q = static_cast<long long>(blockIdx.x) * kPeakBlock + threadIdx.x;
    float v;
    const bool pk = is_peak(M, w, h, floor, radius, edge, static_cast<int>(q % w), static_cast<int>(q / w), v);
    const int c = __syncthreads_count(pk);
    if (threadIdx.x == 0) block_count[blockIdx.x] = c;
}

// exclusive scan of the block counts in place (one CTA of 1024 threads, a
// contiguous chunk per thread); the sum into *total
__global__ void __launch_bounds__(1024) peak_scan_kernel(int* cnt, int nblocks, int* total) {
    __shared__ int part[1024];
    const int t = threadIdx.x;
    const int chunk = (nblocks + 1023) / 1024;
    const int b0 = min(nblocks, t * chunk), b1 = min(nblocks, b0 + chunk);
    int s = 0;
    for (int b = b0; b < b1; ++b) s += cnt[b];
    part[t] = s;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {  // inclusive scan of the chunk sums
        const int add = t >= off ? part[t - off] : 0;
        __syncthreads();
        part[t] += add;
        __syncthreads();
    }
    int run = part[t] - s;
    for (int b = b0; b < b1; ++b) {
        const int c = cnt[b];
        cnt[b] = run;
        run += c;
    }
    if (t == 1023) *total = part[1023];
}

__global__ void __launch_bounds__(kPeakBlock) peak_write_kernel(const float* M, const int* best_v, int w, int h,
                                                                float floor, int radius, int edge,
                                                                const int* block_offset, PeakRec* out, int cap) {
    __shared__ int warp_base[kPeakBlock / 32];
    const long long q = static_cast<long long>(blockIdx.x) * kPeakBlock + threadIdx.x;
    const int x = static_cast<int>(q % w), y = static_cast<int>(q / w);
    float v = 0.0f;
    const bool pk = is_peak(M, w, h, floor, radius, edge, x, y, v);
    const unsigned lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const unsigned bal = __ballot_sync(0xffffffffu, pk);
    if (lane == 0) warp_base[warp] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        int run = 0;
        for (int k = 0; k < kPeakBlock / 32; ++k) {
            const int c = warp_base[k];
            warp_base[k] = run;
            run += c;
        }
    }
    __syncthreads();
    if (pk) {
        const int pos = block_offset[blockIdx.x] + warp_base[warp] + __popc(bal & ((1u << lane) - 1u));
        if (pos < cap) out[pos] = {x, y, v, best_v[static_cast<size_t>(y) * w + x]};
    }
}

// the three launches for one map; the count of its peaks lands in *d_total
void launch_peaks(Context& c, const float* d_max, const int* d_bv, int w, int h, float floor, int radius, int edge,
                  int* d_blocks, int* d_total, PeakRec* d_out, int cap) {
    cudaStream_t s = c.stream();
    const long long npix = static_cast<long long>(w) * h;
    const int nb = static_cast<int>((npix + kPeakBlock - 1) / kPeakBlock);
    peak_count_kernel<<<nb, kPeakBlock, 0, s>>>(d_max, w, h, floor, radius, edge, d_blocks);
    peak_scan_kernel<<<1, 1024, 0, s>>>(d_blocks, nb, d_total);
    peak_write_kernel<<<nb, kPeakBlock, 0, s>>>(d_max, d_bv, w, h, floor, radius, edge, d_blocks, d_out, cap);
    FTB_CHECK(cudaGetLastError());
    c.launches += 3;
}

__device__ __forceinline__ float bilinear(const float* img, int w, int h, int pitch, double x, double y) {
    return track_bilinear(img, w, h, pitch, x, y);
}

struct ArtArgs {
    const PeakRec* peaks;
    int count;
    const double* vel;      // (vx, vy) per motion
    const float* filtered;  // n frames
    const float* sub;       // n frames
    const float* sky;
    const double* t_h;
    int w, h, pitch, n, r;
    double max_frame_fraction;
    char* out;
    const double* reg_dx;   // registration offsets by frame (null: no detector test)
    const double* reg_dy;
    const double* steps;    // detector_flag's grid of offsets
    int nsteps;
    int oy, rows;           // the frames are rows [oy, oy + rows) of the image (h rows)
};

// is_artefact_peak (search.cpp:229-243): the single-frame share of the track's
// positive signal, then the field-edge test (blank sub-frame or static-sky
// pixels within r of the track in more than max(1, n/10) frames), then, with
// registration offsets, the detector test (a source fixed on the sensor
// explains at least 0.8 of the track's S/N). One warp per peak: the lanes
// sample the frames, scan the edge boxes and share the detector grid; lane 0
// adds the signal in frame order, as the reference does.
constexpr int kArtWarps = 4;

__global__ void __launch_bounds__(32 * kArtWarps) artefact_kernel(const ArtArgs a) {
    __shared__ double vals[kArtWarps][256];  // a warp's track values, n <= 255 frames
    const int warp = static_cast<int>(threadIdx.x >> 5), lane = static_cast<int>(threadIdx.x & 31);
    const int k = blockIdx.x * kArtWarps + warp;
    if (k >= a.count) return;  // the whole warp
    const PeakRec pk = a.peaks[k];
    const double vx = a.vel[2 * pk.vidx], vy = a.vel[2 * pk.vidx + 1];
    const size_t plane = static_cast<size_t>(a.pitch) * a.rows;
    for (int i = lane; i < a.n; i += 32) {
        const double t = a.t_h[i];
        const double px = __dadd_rn(static_cast<double>(pk.x), __dmul_rn(vx, t));
        const double py = __dadd_rn(static_cast<double>(pk.y), __dmul_rn(vy, t));
        const float v = track_bilinear_band(a.filtered + i * plane, a.w, a.h, a.pitch, a.oy, a.rows, px, py);
        vals[warp][i] = isfinite(v) ? static_cast<double>(v) : CUDART_NAN;
    }
    __syncwarp();
    int single = 0;
    if (lane == 0) {
        double pos_sum = 0.0, maxc = 0.0;
        for (int i = 0; i < a.n; ++i) {
            const double d = vals[warp][i];
            if (!isfinite(d)) continue;
            pos_sum = __dadd_rn(pos_sum, d > 0.0 ? d : 0.0);
            maxc = maxc < d ? d : maxc;
        }
        const double frac = pos_sum > 0.0 ? maxc / pos_sum : 1.0;
        single = a.n >= 8 && frac > a.max_frame_fraction;
    }
    if (__shfl_sync(0xffffffffu, single, 0)) {
        if (lane == 0) a.out[k] = 1;
        return;
    }
    const int side = 2 * a.r + 1, box = side * side;
    int near_blank = 0;
    for (int i = 0; i < a.n; ++i) {
        const double t = a.t_h[i];
        const int xi = static_cast<int>(lround(__dadd_rn(static_cast<double>(pk.x), __dmul_rn(vx, t))));
        const int yi = static_cast<int>(lround(__dadd_rn(static_cast<double>(pk.y), __dmul_rn(vy, t))));
        bool blank = false;
        for (int e = lane; e < box && !blank; e += 32) {
            const int xx = xi + e % side - a.r, yy = yi + e / side - a.r;
            blank = xx < 0 || yy < 0 || xx >= a.w || yy >= a.h || yy - a.oy < 0 || yy - a.oy >= a.rows ||
                    !isfinite(a.sub[i * plane + static_cast<size_t>(yy - a.oy) * a.pitch + xx]) ||
                    !isfinite(a.sky[static_cast<size_t>(yy - a.oy) * a.pitch + xx]);
        }
        near_blank += __any_sync(0xffffffffu, blank) ? 1 : 0;
    }
    const bool edge = near_blank > max(1, a.n / 10);
    if (edge || !a.reg_dx) {
        if (lane == 0) a.out[k] = edge ? 1 : 0;
        return;
    }
    // the track's S/N over all frames (track_snr, search.cpp:142-163)
    double all = 0.0;
    if (lane == 0) {
        double sum = 0.0;
        int count = 0;
        for (int i = 0; i < a.n; ++i) {
            const double d = vals[warp][i];
            if (!isfinite(d)) continue;
            sum = __dadd_rn(sum, d);
            ++count;
        }
        all = count >= 3 ? __ddiv_rn(sum, __dsqrt_rn(static_cast<double>(count))) : 0.0;
    }
    all = __shfl_sync(0xffffffffu, all, 0);
    const double best = detector_best_fixed(a.filtered, plane, a.w, a.h, a.pitch, a.oy, a.rows, a.n, a.t_h,
                                            a.reg_dx, a.reg_dy, a.steps, a.nsteps, static_cast<double>(pk.x),
                                            static_cast<double>(pk.y), vx, vy);
    if (lane == 0) a.out[k] = best >= __dmul_rn(0.8, all) ? 1 : 0;
}

// Injection increments added in order: one CTA per frame walks its patches in
// sequence (patches may overlap; every pixel of one patch is touched once), so
// each pixel receives its float additions in the reference's order.
__global__ void patch_kernel(float* frames, size_t plane, int pitch, const int* pstart, const int* pframe_x0_y0_w_h,
                             const unsigned long long* poff, const float* values) {
    const int f = blockIdx.x;
    float* img = frames + f * plane;
    for (int q = pstart[f]; q < pstart[f + 1]; ++q) {
        const int x0 = pframe_x0_y0_w_h[4 * q], y0 = pframe_x0_y0_w_h[4 * q + 1];
        const int pw = pframe_x0_y0_w_h[4 * q + 2], ph = pframe_x0_y0_w_h[4 * q + 3];
        const float* v = values + poff[q];
        for (int e = threadIdx.x; e < pw * ph; e += blockDim.x) {
            float* px = img + static_cast<size_t>(y0 + e / pw) * pitch + x0 + e % pw;
            *px = __fadd_rn(*px, v[e]);
        }
        __syncthreads();
    }
}

}  // namespace

void apply_patches(Context& c, const InjectionPatches& ip, float* d_frames, int w, int h, int n) {
    const size_t np = ip.frame.size();
    if (np == 0) return;
    const int pitch = frame_pitch(w);
    std::vector<int> start(static_cast<size_t>(n) + 1, 0), geo(4 * np);
    std::vector<unsigned long long> off(np);
    for (size_t q = 0; q < np; ++q) {
        if (q > 0 && ip.frame[q] < ip.frame[q - 1]) throw std::runtime_error("injection patches out of frame order");
        ++start[static_cast<size_t>(ip.frame[q]) + 1];
        geo[4 * q] = ip.x0[q];
        geo[4 * q + 1] = ip.y0[q];
        geo[4 * q + 2] = ip.pw[q];
        geo[4 * q + 3] = ip.ph[q];
        off[q] = ip.off[q];
    }
    for (int f = 0; f < n; ++f) start[static_cast<size_t>(f) + 1] += start[static_cast<size_t>(f)];
    const size_t bytes = sizeof(int) * (start.size() + geo.size()) + sizeof(unsigned long long) * np +
                         sizeof(float) * ip.values.size() + 1024;
    DevBuf buf(&c, bytes, "injection patches");
    unsigned char* b = buf.as<unsigned char>();
    int* d_start = reinterpret_cast<int*>(b);
    int* d_geo = d_start + start.size();
    unsigned long long* d_off =
        reinterpret_cast<unsigned long long*>(b + ((sizeof(int) * (start.size() + geo.size()) + 15) / 16) * 16);
    float* d_val = reinterpret_cast<float*>(d_off + np);
    cudaStream_t s = c.stream();
    FTB_CHECK(cudaMemcpyAsync(d_start, start.data(), sizeof(int) * start.size(), cudaMemcpyHostToDevice, s));
    FTB_CHECK(cudaMemcpyAsync(d_geo, geo.data(), sizeof(int) * geo.size(), cudaMemcpyHostToDevice, s));
    FTB_CHECK(cudaMemcpyAsync(d_off, off.data(), sizeof(unsigned long long) * np, cudaMemcpyHostToDevice, s));
    FTB_CHECK(cudaMemcpyAsync(d_val, ip.values.data(), sizeof(float) * ip.values.size(), cudaMemcpyHostToDevice, s));
    patch_kernel<<<n, 256, 0, s>>>(d_frames, static_cast<size_t>(pitch) * h, pitch, d_start, d_geo, d_off, d_val);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
}  // buf is released in stream order after the kernel

namespace {
// f(k) for k < count on up to 16 host threads
template <class F>
void for_each_map(size_t count, const F& f) {
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t workers = std::min<size_t>(hw, count);
    if (workers <= 1) {
        for (size_t k = 0; k < count; ++k) f(k);
        return;
    }
    std::vector<std::thread> pool;
    for (size_t wk = 0; wk < workers; ++wk)
        pool.emplace_back([&, wk] {
            for (size_t k = wk; k < count; k += workers) f(k);
        });
    for (auto& t : pool) t.join();
}
}  // namespace

std::vector<Peak> device_peaks(Context& c, const float* d_max, const int* d_best_v, int w, int h, float floor,
                               int radius, int edge) {
    return device_peaks_many(c, {{d_max, d_best_v}}, w, h, floor, radius, edge, 0)[0];
}

std::vector<std::vector<Peak>> device_peaks_many(Context& c, const std::vector<PeakMap>& maps, int w, int h,
                                                 float floor, int radius, int edge, size_t keep) {
    const size_t k_maps = maps.size();
    std::vector<std::vector<Peak>> out(k_maps);
    if (k_maps == 0) return out;
    cudaStream_t s = c.stream();
    const long long npix = static_cast<long long>(w) * h;
    const size_t nb = static_cast<size_t>((npix + kPeakBlock - 1) / kPeakBlock);
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    int cap = std::max(1 << 16, static_cast<int>(std::min<long long>(1LL << 22, npix / 16)));
    std::vector<int> count(k_maps);
    for (;;) {
        // per map: block counts (scanned in place), then its peaks; the totals first
        const size_t per = al(sizeof(int) * nb) + al(sizeof(PeakRec) * static_cast<size_t>(cap));
        DevBuf& buf = c.scratch(22, al(sizeof(int) * k_maps) + per * k_maps, "peaks (batch)");
        unsigned char* base = buf.as<unsigned char>();
        int* d_total = reinterpret_cast<int*>(base);
        auto blocks = [&](size_t k) { return reinterpret_cast<int*>(base + al(sizeof(int) * k_maps) + per * k); };
        auto recs = [&](size_t k) {
            return reinterpret_cast<PeakRec*>(base + al(sizeof(int) * k_maps) + per * k + al(sizeof(int) * nb));
        };
        for (size_t k = 0; k < k_maps; ++k)
            launch_peaks(c, maps[k].d_max, maps[k].d_best_v, w, h, floor, radius, edge, blocks(k), d_total + k, recs(k),
                         cap);
        FTB_CHECK(cudaMemcpyAsync(count.data(), d_total, sizeof(int) * k_maps, cudaMemcpyDeviceToHost, s));
        FTB_CHECK(cudaStreamSynchronize(s));
        const int most = *std::max_element(count.begin(), count.end());
        if (most > cap) {  // more peaks than room: again with room for all
            cap = most;
            continue;
        }
        std::vector<std::vector<PeakRec>> rec(k_maps);
        for (size_t k = 0; k < k_maps; ++k) {
            rec[k].resize(static_cast<size_t>(count[k]));
            if (count[k])
                FTB_CHECK(cudaMemcpyAsync(rec[k].data(), recs(k), sizeof(PeakRec) * count[k], cudaMemcpyDeviceToHost, s));
        }
        FTB_CHECK(cudaStreamSynchronize(s));
        // already in raster order; order_peaks' std::sort by S/N (ties as the
        // reference's) and the truncation, one map per host thread
        for (size_t k = 0; k < k_maps; ++k) {
            const std::vector<PeakRec>& r = rec[k];
            out[k].resize(r.size());
            for (size_t q = 0; q < r.size(); ++q) out[k][q] = {r[q].x, r[q].y, r[q].snr, r[q].vidx};
        }
        if (keep) for_each_map(k_maps, [&](size_t k) { order_peaks(out[k], keep); });
        return out;
    }
}

NullPeaks split_null_peaks(std::vector<Peak> raster, size_t keep, size_t tested) {
    NullPeaks out;
    const size_t N = raster.size(), nk = std::min(N, keep), t = std::min(nk, tested);
    if (N == 0) return out;
    std::vector<float> v(N);
    for (size_t q = 0; q < N; ++q) v[q] = raster[q].snr;
    if (t > 0 && t < N) {
        // the t-th and (t+1)-th largest S/N: the screened set is unique unless they tie
        std::nth_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(t), v.end(), std::greater<float>());
        const float after = v[t];
        const float last = *std::min_element(v.begin(), v.begin() + static_cast<std::ptrdiff_t>(t));
        if (!(last > after)) {  // a tie at the boundary: the reference's sort decides
            order_peaks(raster, keep);
            out.tested.assign(raster.begin(), raster.begin() + static_cast<std::ptrdiff_t>(t));
            for (size_t q = t; q < raster.size(); ++q) out.rest.push_back(raster[q].snr);
            return out;
        }
        for (const Peak& p : raster)
            if (p.snr >= last) out.tested.push_back(p);
        out.rest.assign(v.begin() + static_cast<std::ptrdiff_t>(t), v.end());
    } else if (t == 0) {
        out.rest = v;
    } else {  // t == N: every peak is screened
        out.tested = std::move(raster);
        return out;
    }
    // the untested values down to the truncation, descending (equal values are
    // interchangeable in the pooled list)
    if (out.rest.size() > nk - t) {
        std::nth_element(out.rest.begin(), out.rest.begin() + static_cast<std::ptrdiff_t>(nk - t), out.rest.end(),
                         std::greater<float>());
        out.rest.resize(nk - t);
    }
    std::sort(out.rest.begin(), out.rest.end(), std::greater<float>());
    return out;
}

std::vector<double> detector_steps(double fwhm_px) {
    std::vector<double> v;
    const double span = std::max(2.0, 2.0 * fwhm_px);
    for (double d = -span; d <= span; d += 0.5) v.push_back(d);
    return v;
}

std::vector<std::vector<char>> device_artefacts_many(Context& c, const std::vector<ArtefactJob>& jobs,
                                                     const std::vector<std::pair<double, double>>& grid,
                                                     const float* d_sub, int w, int h, int n, double fwhm_px,
                                                     double max_frame_fraction, const std::vector<double>& reg_dx,
                                                     const std::vector<double>& reg_dy, Band band) {
    std::vector<std::vector<char>> out(jobs.size());
    size_t total = 0;
    for (size_t k = 0; k < jobs.size(); ++k) {
        out[k].assign(jobs[k].count, 0);
        total += jobs[k].count;
    }
    if (total == 0) return out;
    cudaStream_t s = c.stream();
    // per job: its peaks and times, then one flag per peak; the grid once
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    std::vector<size_t> off(jobs.size());
    // the grid, then the registration offsets and the detector steps (if any), then the jobs
    const bool reg = static_cast<int>(reg_dx.size()) == n && static_cast<int>(reg_dy.size()) == n;
    const std::vector<double> steps = reg ? detector_steps(fwhm_px) : std::vector<double>();
    const size_t reg_off = al(sizeof(double) * 2 * grid.size());
    size_t bytes = reg_off + (reg ? al(sizeof(double) * (2 * static_cast<size_t>(n) + steps.size())) : 0);
    for (size_t k = 0; k < jobs.size(); ++k) {
        off[k] = bytes;
        bytes += al(sizeof(PeakRec) * jobs[k].count) + al(sizeof(double) * n) + al(jobs[k].count);
    }
    DevBuf& buf = c.scratch(23, bytes, "artefact screen (batch)");
    unsigned char* base = buf.as<unsigned char>();
    std::vector<unsigned char> host(bytes);
    std::memcpy(host.data(), grid.data(), sizeof(double) * 2 * grid.size());
    if (reg) {
        double* r = reinterpret_cast<double*>(host.data() + reg_off);
        std::memcpy(r, reg_dx.data(), sizeof(double) * n);
        std::memcpy(r + n, reg_dy.data(), sizeof(double) * n);
        std::memcpy(r + 2 * n, steps.data(), sizeof(double) * steps.size());
    }
    for (size_t k = 0; k < jobs.size(); ++k) {
        PeakRec* r = reinterpret_cast<PeakRec*>(host.data() + off[k]);
        for (size_t q = 0; q < jobs[k].count; ++q) {
            const Peak& p = (*jobs[k].peaks)[q];
            r[q] = {p.x, p.y, p.snr, p.vidx};
        }
        std::memcpy(host.data() + off[k] + al(sizeof(PeakRec) * jobs[k].count), jobs[k].t_h->data(), sizeof(double) * n);
    }
    FTB_CHECK(cudaMemcpyAsync(base, host.data(), bytes, cudaMemcpyHostToDevice, s));
    const int r = static_cast<int>(std::ceil(2.0 * fwhm_px)) + 1;
    for (size_t k = 0; k < jobs.size(); ++k) {
        if (jobs[k].count == 0) continue;
        unsigned char* b = base + off[k];
        const double* d_t = reinterpret_cast<const double*>(b + al(sizeof(PeakRec) * jobs[k].count));
        char* d_out = reinterpret_cast<char*>(b + al(sizeof(PeakRec) * jobs[k].count) + al(sizeof(double) * n));
        ArtArgs a{reinterpret_cast<const PeakRec*>(b), static_cast<int>(jobs[k].count),
                  reinterpret_cast<const double*>(base), jobs[k].d_filtered, d_sub, jobs[k].d_sky, d_t, w, h,
                  frame_pitch(w), n, r, max_frame_fraction, d_out, nullptr, nullptr, nullptr, 0, band.oy,
                  band.rows > 0 ? band.rows : h};
        if (reg) {
            const double* d_reg = reinterpret_cast<const double*>(base + reg_off);
            a.reg_dx = d_reg;
            a.reg_dy = d_reg + n;
            a.steps = d_reg + 2 * n;
            a.nsteps = static_cast<int>(steps.size());
        }
        artefact_kernel<<<static_cast<unsigned>((jobs[k].count + kArtWarps - 1) / kArtWarps), 32 * kArtWarps, 0, s>>>(a);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
    }
    FTB_CHECK(cudaMemcpyAsync(host.data(), base, bytes, cudaMemcpyDeviceToHost, s));
    FTB_CHECK(cudaStreamSynchronize(s));
    for (size_t k = 0; k < jobs.size(); ++k)
        if (jobs[k].count)
            std::memcpy(out[k].data(),
                        host.data() + off[k] + al(sizeof(PeakRec) * jobs[k].count) + al(sizeof(double) * n),
                        jobs[k].count);
    return out;
}

// ------------------------------------------------------------------ a search request in phases

SearchRequest::SearchRequest(Context& c, const SearchParams& p, int w, int h, int n) : c_(c), p_(p) {
    if (n < 5) throw std::runtime_error("synthetic tracking needs at least 5 frames");
    if (w < 16 || h < 16) throw std::runtime_error("frames are too small");
    if (n > 255) throw std::runtime_error("at most 255 frames per search");
    o_.w = w;
    o_.h = h;
    o_.n = n;
    pitch_ = frame_pitch(w);
    plane_ = static_cast<size_t>(pitch_) * h;
    map_bytes_ = sizeof(float) * static_cast<size_t>(w) * h;
}

size_t SearchRequest::base_bytes(int w, int h, int n) {
    const size_t plane = static_cast<size_t>(frame_pitch(w)) * h;
    // raw, sub, filtered, residuals (stage scratch), the real residuals + sky, mask, scatter + maps + samples
    return sizeof(float) * (5 * plane * n + 3 * plane) + 2 * sizeof(float) * static_cast<size_t>(w) * h +
           (size_t{64} << 20);
}

size_t SearchRequest::item_bytes() const {
    // a null run: filtered frames, sky, mask, maps; an injection copy also keeps
    // its sub frames and residuals until it is refined
    return sizeof(float) * ((copies_ ? 3 : 1) * plane_ * o_.n + 2 * plane_) + 2 * map_bytes_;
}

void SearchRequest::prepare(const float* frames, const double* mjd, const double* exptime, bool on_device,
                            int in_pitch, bool keep_raw, const std::function<void(double, const char*)>& report) {
    const int w = o_.w, h = o_.h, n = o_.n;
    Context& c = c_;
    const double t_setup = wall_seconds();
    // frames in time order (the C API stable-sorts by mid-exposure, c_api.cpp:177-179)
    std::vector<int> order(static_cast<size_t>(n));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return mjd[a] < mjd[b]; });
    double tmin = mjd[order[0]], tmax = tmin;
    for (int i = 0; i < n; ++i) {
        tmin = std::min(tmin, mjd[i]);
        tmax = std::max(tmax, mjd[i]);
    }
    o_.t_ref_mjd = 0.5 * (tmin + tmax);
    o_.span_h = (tmax - tmin) * 24.0;
    if (o_.span_h <= 0.0) throw std::runtime_error("frames must span a non-zero time interval");
    for (int i = 0; i < n; ++i) o_.t_h.push_back((mjd[order[static_cast<size_t>(i)]] - o_.t_ref_mjd) * 24.0);
    if (exptime)
        for (int i = 0; i < n; ++i) exp_sorted_.push_back(exptime[order[static_cast<size_t>(i)]]);
    if (!p_.reg_dx.empty() || !p_.reg_dy.empty()) {
        if (static_cast<int>(p_.reg_dx.size()) != n || static_cast<int>(p_.reg_dy.size()) != n)
            throw std::runtime_error("search: registration offsets need one (dx, dy) per frame");
        for (int i = 0; i < n; ++i) {
            o_.reg_dx.push_back(p_.reg_dx[static_cast<size_t>(order[static_cast<size_t>(i)])]);
            o_.reg_dy.push_back(p_.reg_dy[static_cast<size_t>(order[static_cast<size_t>(i)])]);
        }
    }

    raw_ = DevBuf(&c, sizeof(float) * plane_ * n, "raw frames");
    sub_ = DevBuf(&c, sizeof(float) * plane_ * n, "background-subtracted frames");
    filt_ = DevBuf(&c, sizeof(float) * plane_ * n, "filtered frames");
    sky_ = DevBuf(&c, sizeof(float) * plane_, "static sky");
    mask_ = DevBuf(&c, sizeof(float) * plane_, "mask");
    max_ = DevBuf(&c, map_bytes_, "max_snr");
    bv_ = DevBuf(&c, map_bytes_, "best_v");
    c.host_time("setup", wall_seconds() - t_setup);

    const int up = c.span_begin(on_device ? "copy in" : "upload");
    const size_t in_plane = on_device ? static_cast<size_t>(in_pitch) * h : static_cast<size_t>(w) * h;
    for (int i = 0; i < n; ++i)
        FTB_CHECK(cudaMemcpy2DAsync(raw_.as<float>() + static_cast<size_t>(i) * plane_, sizeof(float) * pitch_,
                                    frames + static_cast<size_t>(order[static_cast<size_t>(i)]) * in_plane,
                                    sizeof(float) * (on_device ? in_pitch : w), sizeof(float) * w,
                                    static_cast<size_t>(h), on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c.stream()));
    c.span_end(up);
    if (p_.align != 0) {
        // the registration check of the raw frames (preprocess.cpp:605-630), with
        // the times from the first frame that prepare_frames gives it
        std::vector<double> t0(static_cast<size_t>(n));
        for (int i = 0; i < n; ++i)
            t0[static_cast<size_t>(i)] = (mjd[order[static_cast<size_t>(i)]] - mjd[order[0]]) * 24.0;
        o_.registration = check_registration_device(c, raw_.as<float>(), plane_, pitch_, w, h, n, t0.data());
        if (!o_.registration.registered)
            throw std::runtime_error(p_.align == 1 ? o_.registration.message
                                                   : o_.registration.message +
                                                         " This backend does not align frames: register them first.");
    }
    if (report) report(0.0, "background");
    if (keep_raw) {
        raw0_ = DevBuf(&c, sizeof(float) * plane_ * n, "raw frames (copies)");
        FTB_CHECK(cudaMemcpyAsync(raw0_.as<float>(), raw_.as<float>(), sizeof(float) * plane_ * n,
                                  cudaMemcpyDeviceToDevice, c.stream()));
    }
    // prepare (preprocess.cpp:528-585)
    sc_ = std::make_unique<StageScratch>(c, w, h, n, std::max(p_.fwhm_px > 0.0 ? p_.fwhm_px : 20.0, 20.0));
    o_.background.resize(static_cast<size_t>(n));
    prepare_sub(c, *sc_, raw_.as<float>(), sub_.as<float>(), w, h, n, o_.background.data());
    sp_.static_exclude = p_.static_exclude;
    sp_.clip_sigma = p_.clip_sigma;
    sp_.cr_sigma = p_.cr_sigma;
    sp_.mask_scatter = p_.mask_scatter;
    sp_.weight_scatter = p_.weight_scatter;
    stage_noise(c, *sc_, sub_.as<float>(), w, h, n, o_.t_h.data(), p_.static_exclude, sky_.as<float>());
    o_.sigma.resize(static_cast<size_t>(n));
    stage_sigma_to_host(c, *sc_, n, o_.sigma.data());
    if (p_.fwhm_px > 0.0) {
        o_.fwhm_px = p_.fwhm_px;
    } else {
        std::vector<float> sky(static_cast<size_t>(w) * h);
        FTB_CHECK(cudaMemcpy2DAsync(sky.data(), sizeof(float) * w, sky_.as<float>(), sizeof(float) * pitch_,
                                    sizeof(float) * w, h, cudaMemcpyDeviceToHost, c.stream()));
        FTB_CHECK(cudaStreamSynchronize(c.stream()));
        o_.fwhm_px = estimate_psf_fwhm(sky, w, h, o_.sigma, p_);
    }
    sp_.fwhm_px = o_.fwhm_px;
    if (!sc_->fits(w, h, n, sp_.fwhm_px)) throw std::runtime_error("PSF too wide for the sample buffers");
    stage_filter(c, *sc_, w, h, n, sp_, filt_.as<float>(), mask_.as<float>(), nullptr, nullptr);
    // the real residuals stay for the candidates' photometry (null runs reuse the stage scratch)
    if (p_.shard_count <= 1) {
        res_ = DevBuf(&c, sizeof(float) * plane_ * n, "real residuals");
        FTB_CHECK(cudaMemcpyAsync(res_.as<float>(), sc_->residual.as<float>(), sizeof(float) * plane_ * n,
                                  cudaMemcpyDeviceToDevice, c.stream()));
    }
    if (report) report(0.1, "prepared");
    // search setup (search.cpp:716-746)
    o_.grid = velocity_grid(o_.span_h, p_, &o_.dv);
    m_ = o_.grid.size();
    auto_thr_ = p_.threshold_snr <= 0.0;
    calibrated_ = auto_thr_ && p_.calibrated_threshold > 0.0;  // the null runs ran elsewhere
    runs_ = auto_thr_ && !calibrated_ ? std::max(0, p_.null_runs) : 0;
    nms_ = std::max(2, static_cast<int>(std::lround(o_.fwhm_px)));
    edge_ = std::max(p_.edge_px, 1);
    min_count_ = pass_min_count(p_.min_coverage, n);
    floor_ = static_cast<float>(auto_thr_ ? p_.min_snr_floor : p_.threshold_snr);
    runs_total_ = runs_;
    orders_ = null_time_orders(o_.t_h, runs_total_, p_.seed);
    sharded_ = p_.shard_count > 1;
    if (sharded_) {
        // this shard's block of the null runs: the same permutations (one seeded
        // stream for all runs) and, pooled in shard order, the same null peaks
        if (!auto_thr_ || calibrated_)
            throw std::runtime_error("search: sharding splits the null runs; a fixed threshold has none");
        if (keep_raw) throw std::runtime_error("search: injection copies need the whole null calibration on one GPU");
        const long long k0 = static_cast<long long>(runs_total_) * p_.shard_index / p_.shard_count;
        const long long k1 = static_cast<long long>(runs_total_) * (p_.shard_index + 1) / p_.shard_count;
        orders_ = std::vector<std::vector<double>>(orders_.begin() + k0, orders_.begin() + k1);
        runs_ = static_cast<int>(k1 - k0);
        real_ = false;  // the real pass runs once the pooled threshold is known
        real_queued_ = real_done_ = true;
    }
    raw_needed_ = keep_raw;
    if (!keep_raw) raw_.reset();
}

PassJob SearchRequest::job(const float* frames, const std::vector<double>& t, float* d_max, int* d_bv) const {
    PassJob j;
    j.d_frames = frames;
    j.pitch = pitch_;
    j.w = o_.w;
    j.h = o_.h;
    j.n = o_.n;
    shift_table(t, o_.grid, j.dx, j.dy);
    j.m = static_cast<int>(m_);
    j.min_count = min_count_;
    j.d_max = d_max;
    j.d_bv = d_bv;
    return j;
}

std::vector<PassJob> SearchRequest::pass_tables(int k0, int k1) const {
    std::vector<PassJob> jobs;
    if (!real_queued_) jobs.push_back(job(nullptr, o_.t_h, nullptr, nullptr));
    for (int k = k0; k < k1; ++k)
        jobs.push_back(job(nullptr, k < runs_ ? orders_[static_cast<size_t>(k)] : o_.t_h, nullptr, nullptr));
    return jobs;
}

void SearchRequest::stage_items(int k0, int k1, const std::vector<std::vector<Injection>>& copies,
                                std::vector<PassJob>& jobs, size_t at) {
    Context& c = c_;
    const int w = o_.w, h = o_.h, n = o_.n;
    const bool add_real = !real_queued_;
    // jobs[at ..] holds pass_tables(k0, k1) (the shift tables, made ahead), or
    // at is kAppend and the jobs are appended with their tables
    const bool tabled = at != kAppend;
    if (tabled && jobs.size() < at + static_cast<size_t>(k1 - k0 + (add_real ? 1 : 0)))
        throw std::runtime_error("search: pass tables do not match the batch");
    size_t next = at;
    auto put = [&](float* filt, const std::vector<double>& t, float* d_max, int* d_bv) {
        if (tabled) {
            PassJob& j = jobs[next++];
            j.d_frames = filt;
            j.d_max = d_max;
            j.d_bv = d_bv;
        } else {
            jobs.push_back(job(filt, t, d_max, d_bv));
        }
    };
    if (add_real) {
        put(filt_.as<float>(), o_.t_h, max_.as<float>(), bv_.as<int>());
        real_queued_ = true;
    }
    for (int k = k0; k < k1; ++k) {
        Item it;
        it.filt = DevBuf(&c, sizeof(float) * plane_ * n, "null filtered frames");
        it.max = DevBuf(&c, map_bytes_, "null max_snr");
        it.bv = DevBuf(&c, map_bytes_, "null best_v");
        if (k < runs_) {
            // preprocessing rebuilt with permuted times on the same sub frames (with_times, preprocess.cpp:488-521)
            it.sky = DevBuf(&c, sizeof(float) * plane_, "null static sky");
            it.mask = DevBuf(&c, sizeof(float) * plane_, "null mask");
            stage_run(c, *sc_, sub_.as<float>(), w, h, n, orders_[static_cast<size_t>(k)].data(), sp_,
                      it.filt.as<float>(), it.sky.as<float>(), it.mask.as<float>(), nullptr, nullptr);
            put(it.filt.as<float>(), orders_[static_cast<size_t>(k)], it.max.as<float>(), it.bv.as<int>());
        } else {
            // an injection copy: raw frames + objects, prepared again with the same PSF width
            const int j = k - runs_;
            if (!raw_) raw_ = DevBuf(&c, sizeof(float) * plane_ * n, "raw frames");
            it.sub = DevBuf(&c, sizeof(float) * plane_ * n, "copy sub frames");
            it.res = DevBuf(&c, sizeof(float) * plane_ * n, "copy residuals");
            it.sky = DevBuf(&c, sizeof(float) * plane_, "copy static sky");
            it.mask = DevBuf(&c, sizeof(float) * plane_, "copy mask");
            FTB_CHECK(cudaMemcpyAsync(raw_.as<float>(), raw0_.as<float>(), sizeof(float) * plane_ * n,
                                      cudaMemcpyDeviceToDevice, c.stream()));
            apply_patches(c, injection_patches(copies[static_cast<size_t>(j)], o_.t_h, exp_sorted_, o_.fwhm_px, w, h),
                          raw_.as<float>(), w, h, n);
            it.background.resize(static_cast<size_t>(n));
            it.sigma.resize(static_cast<size_t>(n));
            prepare_sub(c, *sc_, raw_.as<float>(), it.sub.as<float>(), w, h, n, it.background.data());
            stage_run(c, *sc_, it.sub.as<float>(), w, h, n, o_.t_h.data(), sp_, it.filt.as<float>(),
                      it.sky.as<float>(), it.mask.as<float>(), it.sigma.data(), nullptr);
            FTB_CHECK(cudaMemcpyAsync(it.res.as<float>(), sc_->residual.as<float>(), sizeof(float) * plane_ * n,
                                      cudaMemcpyDeviceToDevice, c.stream()));
            put(it.filt.as<float>(), o_.t_h, it.max.as<float>(), it.bv.as<int>());
        }
        items_.emplace(k, std::move(it));
    }
    o_.adds += static_cast<double>(m_) * n * w * h * static_cast<double>(std::max(0, k1 - k0) + (add_real ? 1 : 0));
}

void SearchRequest::finish_items(int k0, int k1) {
    Context& c = c_;
    const int w = o_.w, h = o_.h, n = o_.n;
    if (!real_done_) {
        o_.peaks = device_peaks(c, max_.as<float>(), bv_.as<int>(), w, h, floor_, nms_, edge_);
        order_peaks(o_.peaks, 100000);
        real_done_ = true;
    }
    // the null runs of this batch together: peaks of every map, then the
    // artefact screen of every run's strongest peaks, then pooling in run order
    const int kn1 = std::min(k1, runs_);
    if (k0 < kn1) {
        std::vector<PeakMap> maps;
        for (int k = k0; k < kn1; ++k) {
            Item& it = items_.at(k);
            maps.push_back({it.max.as<float>(), it.bv.as<int>()});
        }
        // raster-ordered peaks of every map, then per map the screened set and
        // the rest of the pooled values (no full sort unless a tie needs one)
        std::vector<std::vector<Peak>> raster = device_peaks_many(c, maps, w, h, 3.0f, nms_, edge_, 0);
        const size_t tested = (p_.gauss_model && p_.null_tested > 0) ? static_cast<size_t>(p_.null_tested) : 0;
        std::vector<NullPeaks> np(raster.size());
        for_each_map(raster.size(), [&](size_t k) { np[k] = split_null_peaks(std::move(raster[k]), 20000, tested); });
        std::vector<ArtefactJob> jobs;
        for (int k = k0; k < kn1; ++k) {
            Item& it = items_.at(k);
            const NullPeaks& q = np[static_cast<size_t>(k - k0)];
            jobs.push_back({&q.tested, q.tested.size(), it.filt.as<float>(), it.sky.as<float>(),
                            &orders_[static_cast<size_t>(k)]});
        }
        const std::vector<std::vector<char>> art = device_artefacts_many(
            c, jobs, o_.grid, sub_.as<float>(), w, h, n, o_.fwhm_px, p_.max_frame_fraction, o_.reg_dx, o_.reg_dy);
        // pool_null_peaks (search.cpp:690-693): the screened peaks that are not
        // artefacts, then the rest, in descending S/N as the reference's list
        for (int k = k0; k < kn1; ++k) {
            const NullPeaks& q = np[static_cast<size_t>(k - k0)];
            const std::vector<char>& a = art[static_cast<size_t>(k - k0)];
            std::vector<float> kept;
            for (size_t e = 0; e < q.tested.size(); ++e)
                if (!a[e]) kept.push_back(q.tested[e].snr);
            std::sort(kept.begin(), kept.end(), std::greater<float>());
            pooled_.insert(pooled_.end(), kept.begin(), kept.end());
            pooled_.insert(pooled_.end(), q.rest.begin(), q.rest.end());
            items_.erase(k);  // the null run's buffers are released in stream order
        }
    }
    // the copies keep their frames: they are refined with the calibrated threshold
}

SearchOut SearchRequest::finalize(std::vector<SearchOut>* copies_out) {
    Context& c = c_;
    const int w = o_.w, h = o_.h, n = o_.n;
    if (sharded_) {
        // the threshold needs every shard's null peaks: the caller pools them
        // (ft_b200_null_threshold) and selects from shard 0's peaks
        o_.thr.method = "shard";
        o_.null_peaks.assign(pooled_.begin(), pooled_.end());
    } else {
        if (calibrated_) {
            o_.thr.snr = p_.calibrated_threshold;
            o_.thr.method = "calibrated";
            o_.thr.a = p_.cal_a;
            o_.thr.b = p_.cal_b;
            o_.thr.k = p_.cal_k;
            o_.thr.inv_s2 = p_.cal_inv_s2;
        } else {
            o_.thr = set_threshold(p_, pooled_, runs_, o_.fwhm_px, w, h, m_);
        }
        if (runs_ > 0 && auto_thr_) o_.null_peaks.assign(pooled_.begin(), pooled_.end());
        for (const Peak& pk : o_.peaks)
            if (pk.snr >= o_.thr.snr && pk.vidx >= 0) o_.selected.push_back(pk);
        if (static_cast<int>(o_.selected.size()) > p_.max_candidates)
            o_.selected.resize(static_cast<size_t>(p_.max_candidates));
        if (!o_.selected.empty()) {
            const int rf = c.span_begin("refine");
            o_.candidates = refine_candidates(c, o_, p_,
                                              {filt_.as<float>(), res_.as<float>(), sub_.as<float>(), sky_.as<float>(),
                                               mask_.as<float>(), w, h, pitch_, n});
            c.span_end(rf);
        }
    }
    res_.reset();
    if (real_) {
        o_.max_snr.resize(static_cast<size_t>(w) * h);
        o_.best_v.resize(static_cast<size_t>(w) * h);
        FTB_CHECK(cudaMemcpyAsync(o_.max_snr.data(), max_.as<float>(), map_bytes_, cudaMemcpyDeviceToHost, c.stream()));
        FTB_CHECK(cudaMemcpyAsync(o_.best_v.data(), bv_.as<int>(), map_bytes_, cudaMemcpyDeviceToHost, c.stream()));
    }
    if (copies_out) {
        // the copies: peaks above the calibrated threshold, which they were searched with
        copies_out->clear();
        for (auto& kv : items_) {
            if (kv.first < runs_) continue;
            Item& it = kv.second;
            SearchOut co;
            co.w = w;
            co.h = h;
            co.n = n;
            co.fwhm_px = o_.fwhm_px;
            co.span_h = o_.span_h;
            co.t_ref_mjd = o_.t_ref_mjd;
            co.dv = o_.dv;
            co.t_h = o_.t_h;
            co.grid = o_.grid;
            co.background = it.background;
            co.sigma = it.sigma;
            co.thr.snr = o_.thr.snr;
            co.thr.method = "fixed";
            co.adds = static_cast<double>(m_) * n * w * h;
            co.peaks = device_peaks(c, it.max.as<float>(), it.bv.as<int>(), w, h, static_cast<float>(o_.thr.snr), nms_,
                                    edge_);
            order_peaks(co.peaks, 100000);
            for (const Peak& pk : co.peaks)
                if (pk.snr >= co.thr.snr && pk.vidx >= 0) co.selected.push_back(pk);
            if (static_cast<int>(co.selected.size()) > p_.max_candidates)
                co.selected.resize(static_cast<size_t>(p_.max_candidates));
            // the copy's candidates, as completeness() reads them (validate.cpp:126-130)
            if (!co.selected.empty())
                co.candidates = refine_candidates(c, co, p_,
                                                  {it.filt.as<float>(), it.res.as<float>(), it.sub.as<float>(),
                                                   it.sky.as<float>(), it.mask.as<float>(), w, h, pitch_, n});
            co.max_snr.resize(static_cast<size_t>(w) * h);
            co.best_v.resize(static_cast<size_t>(w) * h);
            FTB_CHECK(cudaMemcpyAsync(co.max_snr.data(), it.max.as<float>(), map_bytes_, cudaMemcpyDeviceToHost,
                                      c.stream()));
            FTB_CHECK(cudaMemcpyAsync(co.best_v.data(), it.bv.as<int>(), map_bytes_, cudaMemcpyDeviceToHost,
                                      c.stream()));
            copies_out->push_back(std::move(co));
        }
    }
    FTB_CHECK(cudaStreamSynchronize(c.stream()));
    items_.clear();
    return std::move(o_);
}

SearchOut search_host(Context& c, const float* frames, int w, int h, int n, const double* mjd, const double* exptime,
                      const SearchParams& p, const Progress& progress, bool frames_on_device, int in_pitch) {
    std::vector<SearchOut> none;
    return search_batch_host(c, frames, w, h, n, mjd, exptime, p, {}, none, progress, frames_on_device, in_pitch);
}

SearchOut search_batch_host(Context& c, const float* frames, int w, int h, int n, const double* mjd,
                            const double* exptime, const SearchParams& p,
                            const std::vector<std::vector<Injection>>& copies, std::vector<SearchOut>& copies_out,
                            const Progress& progress, bool frames_on_device, int in_pitch) {
    c.bind();
    if (!copies.empty() && !exptime) throw std::runtime_error("injection copies need the exposure times");
    auto report = [&](double f, const char* stage) {
        if (progress && !progress(f, stage)) throw Cancelled();
    };
    c.timing_reset();
    const int total = c.span_begin("total");
    SearchRequest r(c, p, w, h, n);
    r.expect_copies(!copies.empty());
    r.prepare(frames, mjd, exptime, frames_on_device, in_pitch, !copies.empty(), report);
    // the real pass, the null runs and the copies as batches, each batch stacked
    // in persistent launches; a batch holds as many items as the HBM budget allows
    const int items = r.runs() + static_cast<int>(copies.size());
    const size_t reserve = size_t{256} << 20;  // plans, peaks, descriptors
    const size_t avail = c.budget() > c.used() + reserve ? c.budget() - c.used() - reserve : 0;
    int per_batch =
        static_cast<int>(std::max<size_t>(1, std::min<size_t>(std::max(items, 1), avail / r.item_bytes())));
    // a launch cap: the real pass goes alone first, then at most k items per launch
    const bool capped = p.passes_per_launch > 0 && items > 0;
    if (capped) per_batch = std::min(per_batch, p.passes_per_launch);
    std::vector<std::pair<int, int>> batches;
    if (capped) batches.emplace_back(0, 0);
    for (int k0 = 0; k0 < std::max(items, 1); k0 += per_batch) batches.emplace_back(k0, std::min(items, k0 + per_batch));
    const double share = 0.9 / (1 + items);
    for (const auto& [k0, k1] : batches) {
        report(0.1 + 0.9 * share * (k0 + 1), "null");
        // the passes' plans are made on host threads while the GPU runs the
        // batch's preprocessing
        std::vector<PassJob> jobs = r.pass_tables(k0, k1);
        PlanAhead ahead = plan_ahead(c, jobs);
        r.stage_items(k0, k1, copies, jobs, 0);
        stack_passes_device(c, jobs, &ahead);
        const int pk = c.span_begin("peaks");
        r.finish_items(k0, k1);
        c.span_end(pk);
    }
    SearchOut o = r.finalize(&copies_out);
    c.span_end(total);
    FTB_CHECK(cudaStreamSynchronize(c.stream()));
    c.timing_resolve();
    report(1.0, "done");
    return o;
}

}  // namespace ftb
