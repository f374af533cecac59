// The search on the B200 (FaintTrail search.cpp:716-809 without the candidate
// refinement): prepare, the real pass and its peaks, the time-shuffled null
// runs (preprocessing rebuilt with permuted times, stack, peaks, artefact
// screen of the strongest null peaks), the null-tail fit and threshold, and the
// selected peaks. Pixel work runs on the device; the grid, the time orders, the
// peak order (std::sort, as the reference) and the fit run on the host.
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <numeric>

#include "search.h"

namespace ftb {

namespace {

struct PeakRec {
    int x, y;
    float snr;
    int vidx;
};

// local maxima above `floor` inside the edge margin, strict for later pixels and
// non-strict for earlier ones, so a plateau yields one peak (search.cpp:110-129)
__global__ void peak_kernel(const float* M, const int* best_v, int w, int h, float floor, int radius, int edge,
                            int* count, PeakRec* out, int cap) {
    const long long q = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int x = static_cast<int>(q % w), y = static_cast<int>(q / w);
    if (y >= h || x < edge || y < edge || x >= w - edge || y >= h - edge) return;
    const float v = M[static_cast<size_t>(y) * w + x];
    if (v < floor) return;
    for (int dy = -radius; dy <= radius; ++dy) {
        const int yy = y + dy;
        if (yy < 0 || yy >= h) continue;
        for (int dx = -radius; dx <= radius; ++dx) {
            const int xx = x + dx;
            if ((!dx && !dy) || xx < 0 || xx >= w) continue;
            const float u = M[static_cast<size_t>(yy) * w + xx];
            if (u > v || (u == v && (dy < 0 || (dy == 0 && dx < 0)))) return;
        }
    }
    const int k = atomicAdd(count, 1);
    if (k < cap) out[k] = {x, y, v, best_v[static_cast<size_t>(y) * w + x]};
}

// bilinear sample with the reference's border rule, double arithmetic, no
// contraction (common.hpp:125-138)
__device__ float bilinear(const float* img, int w, int h, int pitch, double x, double y) {
    const int x0 = static_cast<int>(floor(x)), y0 = static_cast<int>(floor(y));
    if (x0 < 0 || y0 < 0 || x0 + 1 >= w || y0 + 1 >= h) {
        const int xr = static_cast<int>(lround(x)), yr = static_cast<int>(lround(y));
        if (xr >= 0 && yr >= 0 && xr < w && yr < h && fabs(x - xr) < 1e-9 && fabs(y - yr) < 1e-9)
            return img[static_cast<size_t>(yr) * pitch + xr];
        return CUDART_NAN_F;
    }
    const double fx = __dsub_rn(x, static_cast<double>(x0)), fy = __dsub_rn(y, static_cast<double>(y0));
    const float* r0 = img + static_cast<size_t>(y0) * pitch + x0;
    const float* r1 = r0 + pitch;
    const double gx = __dsub_rn(1.0, fx), gy = __dsub_rn(1.0, fy);
    const double top = __dadd_rn(__dmul_rn(gx, r0[0]), __dmul_rn(fx, r0[1]));
    const double bot = __dadd_rn(__dmul_rn(gx, r1[0]), __dmul_rn(fx, r1[1]));
    return __double2float_rn(__dadd_rn(__dmul_rn(gy, top), __dmul_rn(fy, bot)));
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
};

// is_artefact_peak without registration offsets (search.cpp:229-243): the
// single-frame share of the track's positive signal, then the field-edge test
// (blank sub-frame or static-sky pixels within r of the track in more than
// max(1, n/10) frames). One thread per peak.
__global__ void artefact_kernel(const ArtArgs a) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= a.count) return;
    const PeakRec pk = a.peaks[k];
    const double vx = a.vel[2 * pk.vidx], vy = a.vel[2 * pk.vidx + 1];
    const size_t plane = static_cast<size_t>(a.pitch) * a.h;
    double pos_sum = 0.0, maxc = 0.0;
    for (int i = 0; i < a.n; ++i) {
        const double t = a.t_h[i];
        const double px = __dadd_rn(static_cast<double>(pk.x), __dmul_rn(vx, t));
        const double py = __dadd_rn(static_cast<double>(pk.y), __dmul_rn(vy, t));
        const float v = bilinear(a.filtered + i * plane, a.w, a.h, a.pitch, px, py);
        if (!isfinite(v)) continue;
        const double d = v;
        pos_sum = __dadd_rn(pos_sum, d > 0.0 ? d : 0.0);
        maxc = maxc < d ? d : maxc;
    }
    const double frac = pos_sum > 0.0 ? maxc / pos_sum : 1.0;
    if (a.n >= 8 && frac > a.max_frame_fraction) {
        a.out[k] = 1;
        return;
    }
    int near_blank = 0;
    for (int i = 0; i < a.n; ++i) {
        const double t = a.t_h[i];
        const int xi = static_cast<int>(lround(__dadd_rn(static_cast<double>(pk.x), __dmul_rn(vx, t))));
        const int yi = static_cast<int>(lround(__dadd_rn(static_cast<double>(pk.y), __dmul_rn(vy, t))));
        bool blank = false;
        for (int dy = -a.r; dy <= a.r && !blank; ++dy)
            for (int dx = -a.r; dx <= a.r; ++dx) {
                const int xx = xi + dx, yy = yi + dy;
                if (xx < 0 || yy < 0 || xx >= a.w || yy >= a.h ||
                    !isfinite(a.sub[i * plane + static_cast<size_t>(yy) * a.pitch + xx]) ||
                    !isfinite(a.sky[static_cast<size_t>(yy) * a.pitch + xx])) {
                    blank = true;
                    break;
                }
            }
        near_blank += blank;
    }
    a.out[k] = (near_blank > max(1, a.n / 10)) ? 1 : 0;
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

std::vector<Peak> device_peaks(Context& c, const float* d_max, const int* d_best_v, int w, int h, float floor,
                               int radius, int edge) {
    cudaStream_t s = c.stream();
    int cap = std::max(1 << 16, static_cast<int>(std::min<long long>(1LL << 22, static_cast<long long>(w) * h / 16)));
    for (;;) {
        DevBuf& buf = c.scratch(20, sizeof(PeakRec) * static_cast<size_t>(cap) + 256, "peaks");
        int* d_count = reinterpret_cast<int*>(buf.as<unsigned char>());
        PeakRec* d_out = reinterpret_cast<PeakRec*>(buf.as<unsigned char>() + 256);
        FTB_CHECK(cudaMemsetAsync(d_count, 0, sizeof(int), s));
        const long long npix = static_cast<long long>(w) * h;
        peak_kernel<<<static_cast<unsigned>((npix + 255) / 256), 256, 0, s>>>(d_max, d_best_v, w, h, floor, radius,
                                                                             edge, d_count, d_out, cap);
        FTB_CHECK(cudaGetLastError());
        ++c.launches;
        int count = 0;
        FTB_CHECK(cudaMemcpyAsync(&count, d_count, sizeof(int), cudaMemcpyDeviceToHost, s));
        FTB_CHECK(cudaStreamSynchronize(s));
        if (count > cap) {
            cap = count;
            continue;
        }
        std::vector<PeakRec> rec(static_cast<size_t>(count));
        if (count) FTB_CHECK(cudaMemcpy(rec.data(), d_out, sizeof(PeakRec) * count, cudaMemcpyDeviceToHost));
        // the reference visits pixels in raster order; restore it
        std::sort(rec.begin(), rec.end(), [](const PeakRec& a, const PeakRec& b) {
            return a.y != b.y ? a.y < b.y : a.x < b.x;
        });
        std::vector<Peak> out(rec.size());
        for (size_t k = 0; k < rec.size(); ++k) out[k] = {rec[k].x, rec[k].y, rec[k].snr, rec[k].vidx};
        return out;
    }
}

std::vector<char> device_artefacts(Context& c, const std::vector<Peak>& peaks, size_t count,
                                   const std::vector<std::pair<double, double>>& grid, const float* d_filtered,
                                   const float* d_sub, const float* d_sky, const std::vector<double>& t_h, int w,
                                   int h, int n, double fwhm_px, double max_frame_fraction) {
    std::vector<char> art(count, 0);
    if (count == 0) return art;
    cudaStream_t s = c.stream();
    std::vector<PeakRec> rec(count);
    for (size_t k = 0; k < count; ++k) rec[k] = {peaks[k].x, peaks[k].y, peaks[k].snr, peaks[k].vidx};
    const size_t bytes = sizeof(PeakRec) * count + sizeof(double) * (2 * grid.size() + t_h.size()) + count + 1024;
    DevBuf& buf = c.scratch(21, bytes, "artefact screen");
    unsigned char* base = buf.as<unsigned char>();
    PeakRec* d_peaks = reinterpret_cast<PeakRec*>(base);
    double* d_vel = reinterpret_cast<double*>(base + ((sizeof(PeakRec) * count + 255) / 256) * 256);
    double* d_t = d_vel + 2 * grid.size();
    char* d_out = reinterpret_cast<char*>(d_t + t_h.size());
    FTB_CHECK(cudaMemcpyAsync(d_peaks, rec.data(), sizeof(PeakRec) * count, cudaMemcpyHostToDevice, s));
    FTB_CHECK(cudaMemcpyAsync(d_vel, grid.data(), sizeof(double) * 2 * grid.size(), cudaMemcpyHostToDevice, s));
    FTB_CHECK(cudaMemcpyAsync(d_t, t_h.data(), sizeof(double) * t_h.size(), cudaMemcpyHostToDevice, s));
    ArtArgs a{d_peaks, static_cast<int>(count), d_vel, d_filtered, d_sub, d_sky, d_t, w, h, frame_pitch(w), n,
              static_cast<int>(std::ceil(2.0 * fwhm_px)) + 1, max_frame_fraction, d_out};
    artefact_kernel<<<static_cast<unsigned>((count + 127) / 128), 128, 0, s>>>(a);
    FTB_CHECK(cudaGetLastError());
    ++c.launches;
    FTB_CHECK(cudaMemcpyAsync(art.data(), d_out, count, cudaMemcpyDeviceToHost, s));
    FTB_CHECK(cudaStreamSynchronize(s));
    return art;
}

namespace {

enum SearchSlot { kRaw = 30, kSub, kFiltReal, kFiltNull, kSkyReal, kSkyNull, kMaskReal, kMaskNull, kMaxMap, kBestMap };

}  // namespace

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
    if (n < 5) throw std::runtime_error("synthetic tracking needs at least 5 frames");
    if (w < 16 || h < 16) throw std::runtime_error("frames are too small");
    auto report = [&](double f, const char* stage) {
        if (progress && !progress(f, stage)) throw Cancelled();
    };
    SearchOut o;
    o.w = w;
    o.h = h;
    o.n = n;
    c.timing_reset();
    const int total = c.span_begin("total");
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
    o.t_ref_mjd = 0.5 * (tmin + tmax);
    o.span_h = (tmax - tmin) * 24.0;
    if (o.span_h <= 0.0) throw std::runtime_error("frames must span a non-zero time interval");
    for (int i = 0; i < n; ++i) o.t_h.push_back((mjd[order[static_cast<size_t>(i)]] - o.t_ref_mjd) * 24.0);

    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * h;
    float* d_raw = c.scratch(kRaw, sizeof(float) * plane * n, "raw frames").as<float>();
    float* d_sub = c.scratch(kSub, sizeof(float) * plane * n, "background-subtracted frames").as<float>();
    float* d_filt = c.scratch(kFiltReal, sizeof(float) * plane * n, "filtered frames").as<float>();
    float* d_sky = c.scratch(kSkyReal, sizeof(float) * plane, "static sky").as<float>();
    float* d_mask = c.scratch(kMaskReal, sizeof(float) * plane, "mask").as<float>();
    float* d_max = c.scratch(kMaxMap, sizeof(float) * static_cast<size_t>(w) * h, "max_snr").as<float>();
    int* d_bv = c.scratch(kBestMap, sizeof(int) * static_cast<size_t>(w) * h, "best_v").as<int>();
    c.host_time("setup", wall_seconds() - t_setup);

    const int up = c.span_begin(frames_on_device ? "copy in" : "upload");
    const size_t in_plane = frames_on_device ? static_cast<size_t>(in_pitch) * h : static_cast<size_t>(w) * h;
    for (int i = 0; i < n; ++i)
        FTB_CHECK(cudaMemcpy2DAsync(d_raw + static_cast<size_t>(i) * plane, sizeof(float) * pitch,
                                    frames + static_cast<size_t>(order[static_cast<size_t>(i)]) * in_plane,
                                    sizeof(float) * (frames_on_device ? in_pitch : w), sizeof(float) * w,
                                    static_cast<size_t>(h),
                                    frames_on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                                    c.stream()));
    c.span_end(up);
    report(0.0, "background");
    // the raw frames stay available for the injection copies
    const int ncopies = static_cast<int>(copies.size());
    DevBuf raw0, sub2, copy_sky, copy_mask;
    std::vector<double> exp_sorted;
    if (ncopies > 0) {
        raw0 = DevBuf(&c, sizeof(float) * plane * n, "raw frames (copies)");
        sub2 = DevBuf(&c, sizeof(float) * plane * n, "copy sub frames");
        copy_sky = DevBuf(&c, sizeof(float) * plane, "copy static sky");
        copy_mask = DevBuf(&c, sizeof(float) * plane, "copy mask");
        FTB_CHECK(cudaMemcpyAsync(raw0.as<float>(), d_raw, sizeof(float) * plane * n, cudaMemcpyDeviceToDevice,
                                  c.stream()));
        for (int i = 0; i < n; ++i) exp_sorted.push_back(exptime[order[static_cast<size_t>(i)]]);
    }

    // prepare (preprocess.cpp:528-585)
    const double fwhm_guess = p.fwhm_px > 0.0 ? p.fwhm_px : 20.0;  // sizes the sample buffers
    StageScratch sc(c, w, h, n, std::max(fwhm_guess, 20.0));
    o.background.resize(static_cast<size_t>(n));
    prepare_sub(c, sc, d_raw, d_sub, w, h, n, o.background.data());
    StageParams sp;
    sp.static_exclude = p.static_exclude;
    sp.clip_sigma = p.clip_sigma;
    sp.cr_sigma = p.cr_sigma;
    sp.mask_scatter = p.mask_scatter;
    sp.weight_scatter = p.weight_scatter;
    stage_noise(c, sc, d_sub, w, h, n, o.t_h.data(), p.static_exclude, d_sky);
    o.sigma.resize(static_cast<size_t>(n));
    stage_sigma_to_host(c, sc, n, o.sigma.data());
    if (p.fwhm_px > 0.0) {
        o.fwhm_px = p.fwhm_px;
    } else {
        std::vector<float> sky(static_cast<size_t>(w) * h);
        FTB_CHECK(cudaMemcpy2DAsync(sky.data(), sizeof(float) * w, d_sky, sizeof(float) * pitch, sizeof(float) * w, h,
                                    cudaMemcpyDeviceToHost, c.stream()));
        FTB_CHECK(cudaStreamSynchronize(c.stream()));
        o.fwhm_px = estimate_psf_fwhm(sky, w, h, o.sigma, p);
    }
    sp.fwhm_px = o.fwhm_px;
    if (!sc.fits(w, h, n, sp.fwhm_px)) throw std::runtime_error("PSF too wide for the sample buffers");
    stage_filter(c, sc, w, h, n, sp, d_filt, d_mask, nullptr, nullptr);
    report(0.1, "prepared");

    // search (search.cpp:716-785)
    o.grid = velocity_grid(o.span_h, p, &o.dv);
    const size_t m = o.grid.size();
    const bool auto_thr = p.threshold_snr <= 0.0;
    const int runs = auto_thr ? std::max(0, p.null_runs) : 0;
    const double share = 0.9 / (1 + runs);
    const int nms = std::max(2, static_cast<int>(std::lround(o.fwhm_px)));
    const int edge = std::max(p.edge_px, 1);
    const int min_count = pass_min_count(p.min_coverage, n);

    // the real pass and the null runs (preprocessing rebuilt with permuted times
    // on the same sub frames) as batches of passes, each batch stacked in one
    // persistent launch; a batch holds as many null runs as the HBM budget allows
    const std::vector<std::vector<double>> orders = null_time_orders(o.t_h, runs, p.seed);
    const size_t map_bytes = sizeof(float) * static_cast<size_t>(w) * h;
    const size_t per_null = sizeof(float) * (plane * n + 2 * plane) + 2 * map_bytes;
    const size_t reserve = size_t{256} << 20;  // plans, peaks, descriptors
    const size_t avail = c.budget() > c.used() + reserve ? c.budget() - c.used() - reserve : 0;
    const int per_batch = static_cast<int>(
        std::max<size_t>(1, std::min<size_t>(std::max(runs + static_cast<int>(copies.size()), 1), avail / per_null)));
    std::vector<float> pooled;
    const float floor = static_cast<float>(auto_thr ? p.min_snr_floor : p.threshold_snr);
    bool real_done = false;
    // copies keep their maps to the end (their peaks need the calibrated threshold)
    std::vector<DevBuf> copy_max(static_cast<size_t>(ncopies)), copy_bv(static_cast<size_t>(ncopies));
    copies_out.assign(static_cast<size_t>(ncopies), SearchOut());
    const int total_items = runs + ncopies;
    for (int k0 = 0; k0 < std::max(total_items, 1); k0 += per_batch) {
        const int k1 = std::min(runs, k0 + per_batch);
        const int c0 = std::max(0, k0 - runs), c1 = std::max(0, std::min(total_items, k0 + per_batch) - runs);
        struct NullBufs {
            DevBuf filt, sky, mask, max, bv;
        };
        std::vector<NullBufs> nb(static_cast<size_t>(std::max(0, k1 - k0)));
        std::vector<DevBuf> copy_filt(static_cast<size_t>(std::max(0, c1 - c0)));
        std::vector<PassJob> jobs;
        if (!real_done) {
            PassJob j;
            j.d_frames = d_filt;
            j.pitch = pitch;
            j.w = w;
            j.h = h;
            j.n = n;
            shift_table(o.t_h, o.grid, j.dx, j.dy);
            j.m = static_cast<int>(m);
            j.min_count = min_count;
            j.d_max = d_max;
            j.d_bv = d_bv;
            jobs.push_back(std::move(j));
        }
        for (int k = k0; k < k1; ++k) {
            NullBufs& b = nb[static_cast<size_t>(k - k0)];
            b.filt = DevBuf(&c, sizeof(float) * plane * n, "null filtered frames");
            b.sky = DevBuf(&c, sizeof(float) * plane, "null static sky");
            b.mask = DevBuf(&c, sizeof(float) * plane, "null mask");
            b.max = DevBuf(&c, map_bytes, "null max_snr");
            b.bv = DevBuf(&c, map_bytes, "null best_v");
            report(0.1 + 0.9 * share * (k + 1), "null");
            stage_run(c, sc, d_sub, w, h, n, orders[static_cast<size_t>(k)].data(), sp, b.filt.as<float>(),
                      b.sky.as<float>(), b.mask.as<float>(), nullptr, nullptr);
            PassJob j;
            j.d_frames = b.filt.as<float>();
            j.pitch = pitch;
            j.w = w;
            j.h = h;
            j.n = n;
            shift_table(orders[static_cast<size_t>(k)], o.grid, j.dx, j.dy);
            j.m = static_cast<int>(m);
            j.min_count = min_count;
            j.d_max = b.max.as<float>();
            j.d_bv = b.bv.as<int>();
            jobs.push_back(std::move(j));
        }
        for (int j = c0; j < c1; ++j) {
            // the raw frames plus this copy's objects, prepared again (fixed PSF width)
            DevBuf& f = copy_filt[static_cast<size_t>(j - c0)];
            f = DevBuf(&c, sizeof(float) * plane * n, "copy filtered frames");
            copy_max[static_cast<size_t>(j)] = DevBuf(&c, map_bytes, "copy max_snr");
            copy_bv[static_cast<size_t>(j)] = DevBuf(&c, map_bytes, "copy best_v");
            FTB_CHECK(cudaMemcpyAsync(d_raw, raw0.as<float>(), sizeof(float) * plane * n, cudaMemcpyDeviceToDevice,
                                      c.stream()));
            apply_patches(c, injection_patches(copies[static_cast<size_t>(j)], o.t_h, exp_sorted, o.fwhm_px, w, h),
                          d_raw, w, h, n);
            SearchOut& co = copies_out[static_cast<size_t>(j)];
            co.background.resize(static_cast<size_t>(n));
            prepare_sub(c, sc, d_raw, sub2.as<float>(), w, h, n, co.background.data());
            co.sigma.resize(static_cast<size_t>(n));
            stage_run(c, sc, sub2.as<float>(), w, h, n, o.t_h.data(), sp, f.as<float>(), copy_sky.as<float>(),
                      copy_mask.as<float>(), co.sigma.data(), nullptr);
            PassJob jb;
            jb.d_frames = f.as<float>();
            jb.pitch = pitch;
            jb.w = w;
            jb.h = h;
            jb.n = n;
            shift_table(o.t_h, o.grid, jb.dx, jb.dy);
            jb.m = static_cast<int>(m);
            jb.min_count = min_count;
            jb.d_max = copy_max[static_cast<size_t>(j)].as<float>();
            jb.d_bv = copy_bv[static_cast<size_t>(j)].as<int>();
            jobs.push_back(std::move(jb));
        }
        stack_passes_device(c, jobs);
        o.adds += static_cast<double>(m) * n * w * h * static_cast<double>(jobs.size());
        report(0.1 + 0.9 * share * (k1 + 1), "null");
        const int pk_span = c.span_begin("peaks");
        if (!real_done) {
            o.peaks = device_peaks(c, d_max, d_bv, w, h, floor, nms, edge);
            order_peaks(o.peaks, 100000);
            real_done = true;
        }
        for (int k = k0; k < k1; ++k) {
            NullBufs& b = nb[static_cast<size_t>(k - k0)];
            std::vector<Peak> npk = device_peaks(c, b.max.as<float>(), b.bv.as<int>(), w, h, 3.0f, nms, edge);
            order_peaks(npk, 20000);
            const size_t tested = (p.gauss_model && p.null_tested > 0)
                                      ? std::min(npk.size(), static_cast<size_t>(p.null_tested))
                                      : 0;
            const std::vector<char> art =
                device_artefacts(c, npk, tested, o.grid, b.filt.as<float>(), d_sub, b.sky.as<float>(),
                                 orders[static_cast<size_t>(k)], w, h, n, o.fwhm_px, p.max_frame_fraction);
            for (size_t q = 0; q < npk.size(); ++q)
                if (q >= art.size() || !art[q]) pooled.push_back(npk[q].snr);
        }
        c.span_end(pk_span);
    }
    o.max_snr.resize(static_cast<size_t>(w) * h);
    o.best_v.resize(static_cast<size_t>(w) * h);
    FTB_CHECK(cudaMemcpyAsync(o.max_snr.data(), d_max, sizeof(float) * o.max_snr.size(), cudaMemcpyDeviceToHost,
                              c.stream()));
    FTB_CHECK(cudaMemcpyAsync(o.best_v.data(), d_bv, sizeof(int) * o.best_v.size(), cudaMemcpyDeviceToHost,
                              c.stream()));
    o.thr = set_threshold(p, pooled, runs, o.fwhm_px, w, h, m);
    // the copies: peaks above the calibrated threshold, searched with it fixed
    for (int j = 0; j < ncopies; ++j) {
        SearchOut& co = copies_out[static_cast<size_t>(j)];
        co.w = w;
        co.h = h;
        co.n = n;
        co.fwhm_px = o.fwhm_px;
        co.span_h = o.span_h;
        co.t_ref_mjd = o.t_ref_mjd;
        co.dv = o.dv;
        co.t_h = o.t_h;
        co.grid = o.grid;
        co.thr.snr = o.thr.snr;
        co.thr.method = "fixed";
        co.adds = static_cast<double>(m) * n * w * h;
        const float* dm = copy_max[static_cast<size_t>(j)].as<float>();
        const int* db = copy_bv[static_cast<size_t>(j)].as<int>();
        co.peaks = device_peaks(c, dm, db, w, h, static_cast<float>(o.thr.snr), nms, edge);
        order_peaks(co.peaks, 100000);
        for (const Peak& pk : co.peaks)
            if (pk.snr >= co.thr.snr && pk.vidx >= 0) co.selected.push_back(pk);
        if (static_cast<int>(co.selected.size()) > p.max_candidates)
            co.selected.resize(static_cast<size_t>(p.max_candidates));
        co.max_snr.resize(static_cast<size_t>(w) * h);
        co.best_v.resize(static_cast<size_t>(w) * h);
        FTB_CHECK(cudaMemcpyAsync(co.max_snr.data(), dm, map_bytes, cudaMemcpyDeviceToHost, c.stream()));
        FTB_CHECK(cudaMemcpyAsync(co.best_v.data(), db, map_bytes, cudaMemcpyDeviceToHost, c.stream()));
    }
    if (runs > 0 && auto_thr) o.null_peaks.assign(pooled.begin(), pooled.end());
    for (const Peak& pk : o.peaks)
        if (pk.snr >= o.thr.snr && pk.vidx >= 0) o.selected.push_back(pk);
    if (static_cast<int>(o.selected.size()) > p.max_candidates) o.selected.resize(static_cast<size_t>(p.max_candidates));
    c.span_end(total);
    FTB_CHECK(cudaStreamSynchronize(c.stream()));
    c.timing_resolve();
    report(1.0, "done");
    return o;
}

}  // namespace ftb
