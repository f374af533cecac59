// The tiled search for sequences larger than HBM: FaintTrail's search_tiled
// (tiled.cpp:157-647), built on the device in full-width bands of rows. The
// frames stay in host memory; for every band only its rows, grown by a halo,
// are uploaded and preprocessed. The halos follow the reference's geometry
// (tiled.cpp:157-186): the longest shift of any trial motion (stack), the reach
// of the matched filter, cosmic-ray test and mask dilation (filter), and the
// refinement's track, photometry, edge and detector reach (refine).
//
// Quantities that belong to a whole frame are measured on the whole frame, from
// the samples the untiled search takes: the background (the median of the
// regular grid of each raw frame), the residual noise (the grid of the
// residuals, sampled band by band in each band's core rows, one exact selection
// over all of them) and the matched filter's normalisation (likewise, with the
// filter halo). With both given, every band is preprocessed and stacked with the
// stack halo, and the core rows of its maps are assembled into the whole
// image's maps before any peak is found. The null runs' artefact screen and the
// candidates' refinement run on bands with the refinement halo, in the whole
// image's coordinates (the band kernels index rows from the band's origin), so
// every value equals the untiled search's: the same maps, null peaks,
// threshold and candidates, bit for bit.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

#include "search.h"
#include "stage.h"

namespace ftb {

namespace {

constexpr double kFwhmToSigma = 1.0 / 2.354820045030949;  // psf.hpp:16
constexpr int kBlankGrow = 3;                              // subtract_and_grow's growth (tiled.cpp:321)

struct Halos {
    int stack = 0, filter = 0, refine = 0;
};

// geometry (tiled.cpp:157-186); times and registration offsets in time order
Halos halos(const std::vector<double>& t_h, const std::vector<std::pair<double, double>>& grid, double dv,
            double fwhm, const std::vector<double>& reg_dx, const std::vector<double>& reg_dy) {
    Halos g;
    double tmax = 0.0;
    for (double t : t_h) tmax = std::max(tmax, std::fabs(t));
    int s = 0;
    for (const auto& v : grid)
        for (double t : t_h)
            s = std::max({s, std::abs(static_cast<int>(std::lround(v.first * t))),
                          std::abs(static_cast<int>(std::lround(v.second * t)))});
    g.stack = s;
    const double psf_sigma = fwhm * kFwhmToSigma;
    const int R = std::max(1, static_cast<int>(std::ceil(3.0 * psf_sigma)));
    const int dil = std::max(1, static_cast<int>(std::lround(0.5 * fwhm)));
    g.filter = R + 2 + dil + 1;
    double reg_range = 0.0;
    if (!reg_dx.empty()) {
        const auto [ax, bx] = std::minmax_element(reg_dx.begin(), reg_dx.end());
        const auto [ay, by] = std::minmax_element(reg_dy.begin(), reg_dy.end());
        reg_range = std::max(*bx - *ax, *by - *ay);
    }
    const int track = s + static_cast<int>(std::ceil(1.25 * dv * tmax)) + 2;
    g.refine = 2 * track + static_cast<int>(std::ceil(reg_range)) + R + 2 + static_cast<int>(std::ceil(2.0 * fwhm)) +
               1 + static_cast<int>(std::ceil(std::max(2.0, 2.0 * fwhm))) + 4 + g.filter;
    return g;
}

// The device side of the tiled search: band buffers sized for the largest
// region, and the frames' host copy with its time order.
class Bands {
public:
    Bands(Context& c, const float* frames, int w, int h, int n, const std::vector<int>& order, int max_rows)
        : c_(c), frames_(frames), w_(w), h_(h), n_(n), order_(order), pitch_(frame_pitch(w)), max_rows_(max_rows) {
        const size_t grown = static_cast<size_t>(pitch_) * (max_rows + 2 * kBlankGrow) * n;
        raw_ = DevBuf(&c, sizeof(float) * grown, "band raw frames");
        tmp_ = DevBuf(&c, sizeof(float) * grown, "band background-subtracted frames");
        sub_ = DevBuf(&c, sizeof(float) * static_cast<size_t>(pitch_) * max_rows * n, "band sub frames");
        filt_ = DevBuf(&c, sizeof(float) * static_cast<size_t>(pitch_) * max_rows * n, "band filtered frames");
        sky_ = DevBuf(&c, sizeof(float) * static_cast<size_t>(pitch_) * max_rows, "band static sky");
        mask_ = DevBuf(&c, sizeof(float) * static_cast<size_t>(pitch_) * max_rows, "band mask");
        bmax_ = DevBuf(&c, sizeof(float) * static_cast<size_t>(w) * max_rows, "band max_snr");
        bbv_ = DevBuf(&c, sizeof(int) * static_cast<size_t>(w) * max_rows, "band best_v");
        bg_ = DevBuf(&c, sizeof(double) * 3 * n, "per-frame values");
    }
    int pitch() const { return pitch_; }
    float* sub() const { return sub_.as<float>(); }
    float* filt() const { return filt_.as<float>(); }
    float* sky() const { return sky_.as<float>(); }
    float* mask() const { return mask_.as<float>(); }
    float* bmax() const { return bmax_.as<float>(); }
    int* bbv() const { return bbv_.as<int>(); }
    double* bg() const { return bg_.as<double>(); }          // per-frame background
    double* sigma() const { return bg_.as<double>() + n_; }  // per-frame residual noise
    double* sg() const { return bg_.as<double>() + 2 * n_; } // per-frame filter normalisation

    // background-subtracted frames (blank areas grown) of image rows [r0, r1),
    // in time order, into sub(): the rows grown by kBlankGrow are uploaded, so
    // the growth inside [r0, r1) sees every neighbour the whole frame has
    void load_sub(int r0, int r1) {
        const int g0 = std::max(0, r0 - kBlankGrow), g1 = std::min(h_, r1 + kBlankGrow);
        const int grows = g1 - g0, rows = r1 - r0;
        const size_t gplane = static_cast<size_t>(pitch_) * grows, plane = static_cast<size_t>(pitch_) * rows;
        const int up = c_.span_begin("upload");
        for (int i = 0; i < n_; ++i)
            FTB_CHECK(cudaMemcpy2DAsync(raw_.as<float>() + i * gplane, sizeof(float) * pitch_,
                                        frames_ + (static_cast<size_t>(order_[static_cast<size_t>(i)]) * h_ + g0) * w_,
                                        sizeof(float) * w_, sizeof(float) * w_, grows, cudaMemcpyHostToDevice,
                                        c_.stream()));
        c_.span_end(up);
        subtract_grow(c_, raw_.as<float>(), tmp_.as<float>(), w_, grows, n_, bg());
        FTB_CHECK(cudaMemcpy2DAsync(sub_.as<float>(), sizeof(float) * plane,
                                    tmp_.as<float>() + static_cast<size_t>(r0 - g0) * pitch_, sizeof(float) * gplane,
                                    sizeof(float) * plane, n_, cudaMemcpyDeviceToDevice, c_.stream()));
    }

    // the per-frame backgrounds: the median of each raw frame's regular sample
    // grid (prepare_core, preprocess.cpp:572-580), whole frames uploaded in chunks
    void backgrounds() {
        const size_t plane = static_cast<size_t>(pitch_) * h_;
        size_t room = raw_.bytes() / (sizeof(float) * plane);
        DevBuf one;  // a frame's room, when the band buffers hold less
        float* chunk = raw_.as<float>();
        if (room < 1) {
            one = DevBuf(&c_, sizeof(float) * plane, "background frame");
            chunk = one.as<float>();
            room = 1;
        }
        const int cap = std::max(1, sample_grid_points(w_, h_, 0));
        DevBuf samples(&c_, sizeof(float) * static_cast<size_t>(cap) * n_, "background samples");
        DevBuf counts(&c_, sizeof(int) * n_, "background sample counts");
        FTB_CHECK(cudaMemsetAsync(counts.as<int>(), 0, sizeof(int) * n_, c_.stream()));
        for (int i0 = 0; i0 < n_; i0 += static_cast<int>(room)) {
            const int k = std::min(n_ - i0, static_cast<int>(room));
            for (int i = 0; i < k; ++i)
                FTB_CHECK(cudaMemcpy2DAsync(chunk + i * plane, sizeof(float) * pitch_,
                                            frames_ + static_cast<size_t>(order_[static_cast<size_t>(i0 + i)]) * h_ * w_,
                                            sizeof(float) * w_, sizeof(float) * w_, h_, cudaMemcpyHostToDevice,
                                            c_.stream()));
            sample_frames(c_, chunk, plane, pitch_, k, w_, h_, 0,
                          samples.as<float>() + static_cast<size_t>(i0) * cap, cap, counts.as<int>() + i0);
        }
        select_median(c_, samples.as<float>(), cap, counts.as<int>(), n_, bg());
        FTB_CHECK(cudaStreamSynchronize(c_.stream()));
    }

private:
    Context& c_;
    const float* frames_;
    int w_, h_, n_;
    std::vector<int> order_;
    int pitch_, max_rows_;
    DevBuf raw_, tmp_, sub_, filt_, sky_, mask_, bmax_, bbv_, bg_;
};

}  // namespace

SearchOut search_tiled_host(Context& c, const float* frames, int w, int h, int n, const double* mjd,
                            const double* exptime, const SearchParams& p, int band_rows, const Progress& progress) {
    c.bind();
    auto report = [&](double f, const char* stage) {
        if (progress && !progress(f, stage)) throw Cancelled();
    };
    if (!frames || !mjd) throw std::runtime_error("tiled search: missing frames or times");
    if (n < 5) throw std::runtime_error("synthetic tracking needs at least 5 frames");
    if (w < 16 || h < 16) throw std::runtime_error("frames are too small");
    if (n > 255) throw std::runtime_error("at most 255 frames per search");
    if (p.shard_count > 1 || p.calibrated_threshold > 0.0)
        throw std::runtime_error("tiled search: null-run shards are searched untiled");
    c.timing_reset();
    const int total = c.span_begin("total");
    SearchOut o;
    o.w = w;
    o.h = h;
    o.n = n;
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
    if (!p.reg_dx.empty()) {
        if (static_cast<int>(p.reg_dx.size()) != n || static_cast<int>(p.reg_dy.size()) != n)
            throw std::runtime_error("search: registration offsets need one (dx, dy) per frame");
        for (int i = 0; i < n; ++i) {
            o.reg_dx.push_back(p.reg_dx[static_cast<size_t>(order[static_cast<size_t>(i)])]);
            o.reg_dy.push_back(p.reg_dy[static_cast<size_t>(order[static_cast<size_t>(i)])]);
        }
    }
    (void)exptime;
    o.grid = velocity_grid(o.span_h, p, &o.dv);
    const size_t m = o.grid.size();
    const bool auto_thr = p.threshold_snr <= 0.0;
    const int runs = auto_thr ? std::max(0, p.null_runs) : 0;
    std::vector<std::vector<double>> orders{o.t_h};
    for (auto& t : null_time_orders(o.t_h, runs, p.seed)) orders.push_back(std::move(t));
    const int edge = std::max(p.edge_px, 1);
    const float floor = static_cast<float>(auto_thr ? p.min_snr_floor : p.threshold_snr);
    const int min_count = pass_min_count(p.min_coverage, n);
    const size_t tested = (p.gauss_model && p.null_tested > 0) ? static_cast<size_t>(p.null_tested) : 0;

    // bands: core rows, plus the largest halo any phase needs (the PSF width is
    // known only after the real run's noise phase: until then 3 px, as the
    // reference plans, tiled.cpp:422; the buffers take the wider of the two)
    const int T = std::max(16, std::min(h, band_rows > 0 ? band_rows : 1024));
    const double fwhm_plan = p.fwhm_px > 0.0 ? p.fwhm_px : 3.0;
    Halos g = halos(o.t_h, o.grid, o.dv, fwhm_plan, o.reg_dx, o.reg_dy);
    const int halo_cap = std::max(g.stack + g.filter, g.refine) + 64;  // room for a PSF wider than planned
    const int max_rows = std::min(h, T + 2 * halo_cap);
    Bands B(c, frames, w, h, n, order, max_rows);
    StageScratch sc(c, w, max_rows, n, std::max(fwhm_plan, 20.0));
    const int pitch = B.pitch();
    std::vector<std::pair<int, int>> cores;
    for (int y0 = 0; y0 < h; y0 += T) cores.emplace_back(y0, std::min(h, y0 + T));
    auto region = [&](std::pair<int, int> core, int halo) {
        return std::make_pair(std::max(0, core.first - halo), std::min(h, core.second + halo));
    };
    auto check_rows = [&](std::pair<int, int> r) {
        if (r.second - r.first > max_rows) throw std::runtime_error("tiled search: a band exceeds its buffers");
    };

    report(0.0, "background");
    B.backgrounds();
    o.background.resize(static_cast<size_t>(n));
    FTB_CHECK(cudaMemcpy(o.background.data(), B.bg(), sizeof(double) * n, cudaMemcpyDeviceToHost));

    StageParams sp;
    sp.static_exclude = p.static_exclude;
    sp.clip_sigma = p.clip_sigma;
    sp.cr_sigma = p.cr_sigma;
    sp.mask_scatter = p.mask_scatter;
    sp.weight_scatter = p.weight_scatter;
    const int capA = std::max(1, sample_grid_points(w, h, 2));
    DevBuf sampA(&c, sizeof(float) * static_cast<size_t>(capA) * n, "noise samples (whole image)");
    DevBuf sampB;
    DevBuf counts(&c, sizeof(int) * 2 * n, "sample counts");
    DevBuf fmax(&c, sizeof(float) * static_cast<size_t>(w) * h, "max_snr");
    DevBuf fbv(&c, sizeof(int) * static_cast<size_t>(w) * h, "best_v");
    std::vector<double> sigma_real, sg_real;
    std::vector<float> pooled;
    std::vector<int> dx, dy;
    const double units = static_cast<double>(orders.size()) + 1.0;

    for (size_t oi = 0; oi < orders.size(); ++oi) {
        const std::vector<double>& t = orders[oi];
        const bool real = oi == 0;
        report(static_cast<double>(oi) / units, real ? "real" : "null");
        // ---- A: residual noise per frame from the whole image's sample grid
        // (and, for the real run, the static sky of the whole image for the PSF)
        std::vector<float> sky_full;
        if (real) sky_full.assign(static_cast<size_t>(w) * h, 0.0f);
        FTB_CHECK(cudaMemsetAsync(counts.as<int>(), 0, sizeof(int) * 2 * n, c.stream()));
        for (const auto& core : cores) {
            const int rows = core.second - core.first;
            B.load_sub(core.first, core.second);
            stage_sky(c, sc, B.sub(), w, rows, n, t.data(), p.static_exclude, B.sky());
            sample_band(c, sc.residual.as<float>(), static_cast<size_t>(pitch) * rows, pitch, n, w, h, 2, core.first,
                        core.first, core.second, nullptr, sampA.as<float>(), capA, counts.as<int>());
            if (real)
                FTB_CHECK(cudaMemcpy2DAsync(sky_full.data() + static_cast<size_t>(core.first) * w, sizeof(float) * w,
                                            B.sky(), sizeof(float) * pitch, sizeof(float) * w, rows,
                                            cudaMemcpyDeviceToHost, c.stream()));
        }
        select_sigma(c, sampA.as<float>(), capA, counts.as<int>(), n, B.sigma(), 1);
        std::vector<double> sigma(static_cast<size_t>(n));
        FTB_CHECK(cudaMemcpyAsync(sigma.data(), B.sigma(), sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream()));
        FTB_CHECK(cudaStreamSynchronize(c.stream()));
        if (real) {
            o.sigma = sigma;
            o.fwhm_px = p.fwhm_px > 0.0 ? p.fwhm_px : estimate_psf_fwhm(sky_full, w, h, sigma, p);
            sp.fwhm_px = o.fwhm_px;
            g = halos(o.t_h, o.grid, o.dv, o.fwhm_px, o.reg_dx, o.reg_dy);
            if (std::max(g.stack + g.filter, g.refine) > halo_cap && max_rows < h)
                throw std::runtime_error("tiled search: the PSF is too wide for the planned halos");
            const int capB = std::max(1, sample_grid_points(w, h, filter_border(o.fwhm_px)));
            sampB = DevBuf(&c, sizeof(float) * static_cast<size_t>(capB) * n, "filter samples (whole image)");
        }
        const int fb = filter_border(o.fwhm_px);
        const int capB = static_cast<int>(sampB.bytes() / (sizeof(float) * n));
        // ---- B: the matched filter's normalisation per frame, from the whole
        // image's masked sample grid, each band with the filter halo
        for (const auto& core : cores) {
            const auto r = region(core, g.filter);
            check_rows(r);
            const int rows = r.second - r.first;
            B.load_sub(r.first, r.second);
            stage_sky(c, sc, B.sub(), w, rows, n, t.data(), p.static_exclude, B.sky());
            stage_filter_given(c, sc, w, rows, n, sp, B.sigma(), nullptr, B.filt(), B.mask());
            sample_band(c, B.filt(), static_cast<size_t>(pitch) * rows, pitch, n, w, h, fb, r.first, core.first,
                        core.second, B.mask(), sampB.as<float>(), capB, counts.as<int>() + n);
        }
        select_sigma(c, sampB.as<float>(), capB, counts.as<int>() + n, n, B.sg(), 0);
        if (real) {
            sigma_real = sigma;
            sg_real.resize(static_cast<size_t>(n));
            FTB_CHECK(cudaMemcpyAsync(sg_real.data(), B.sg(), sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream()));
        }
        // ---- C: every band preprocessed and stacked with the stack halo; the
        // core rows of its maps go into the whole image's maps
        shift_table(t, o.grid, dx, dy);
        for (const auto& core : cores) {
            const auto r = region(core, g.stack + g.filter);
            check_rows(r);
            const int rows = r.second - r.first;
            B.load_sub(r.first, r.second);
            stage_sky(c, sc, B.sub(), w, rows, n, t.data(), p.static_exclude, B.sky());
            stage_filter_given(c, sc, w, rows, n, sp, B.sigma(), B.sg(), B.filt(), B.mask());
            std::vector<PassJob> jobs(1);
            PassJob& j = jobs[0];
            j.d_frames = B.filt();
            j.pitch = pitch;
            j.w = w;
            j.h = rows;
            j.n = n;
            j.dx = dx;
            j.dy = dy;
            j.m = static_cast<int>(m);
            j.min_count = min_count;
            j.d_max = B.bmax();
            j.d_bv = B.bbv();
            stack_passes_device(c, jobs);
            const size_t off = static_cast<size_t>(core.first - r.first) * w;
            const size_t cnt = static_cast<size_t>(core.second - core.first) * w;
            FTB_CHECK(cudaMemcpyAsync(fmax.as<float>() + static_cast<size_t>(core.first) * w, B.bmax() + off,
                                      sizeof(float) * cnt, cudaMemcpyDeviceToDevice, c.stream()));
            FTB_CHECK(cudaMemcpyAsync(fbv.as<int>() + static_cast<size_t>(core.first) * w, B.bbv() + off,
                                      sizeof(int) * cnt, cudaMemcpyDeviceToDevice, c.stream()));
        }
        o.adds += static_cast<double>(m) * n * w * h;
        const int nms = std::max(2, static_cast<int>(std::lround(o.fwhm_px)));
        if (real) {
            o.peaks = device_peaks(c, fmax.as<float>(), fbv.as<int>(), w, h, floor, nms, edge);
            order_peaks(o.peaks, 100000);
            o.max_snr.resize(static_cast<size_t>(w) * h);
            o.best_v.resize(static_cast<size_t>(w) * h);
            FTB_CHECK(cudaMemcpyAsync(o.max_snr.data(), fmax.as<float>(), sizeof(float) * w * h,
                                      cudaMemcpyDeviceToHost, c.stream()));
            FTB_CHECK(cudaMemcpyAsync(o.best_v.data(), fbv.as<int>(), sizeof(int) * w * h, cudaMemcpyDeviceToHost,
                                      c.stream()));
            continue;
        }
        // ---- null run: its peaks, the artefact screen of the strongest on
        // bands with the refinement halo, pooled (search.cpp:766-781, 690-693)
        NullPeaks q = split_null_peaks(device_peaks(c, fmax.as<float>(), fbv.as<int>(), w, h, 3.0f, nms, edge), 20000,
                                       tested);
        std::vector<char> art(q.tested.size(), 0);
        for (const auto& core : cores) {
            std::vector<Peak> mine;
            std::vector<size_t> idx;
            for (size_t e = 0; e < q.tested.size(); ++e)
                if (q.tested[e].y >= core.first && q.tested[e].y < core.second) {
                    mine.push_back(q.tested[e]);
                    idx.push_back(e);
                }
            if (mine.empty()) continue;
            const auto r = region(core, g.refine);
            check_rows(r);
            const int rows = r.second - r.first;
            B.load_sub(r.first, r.second);
            stage_sky(c, sc, B.sub(), w, rows, n, t.data(), p.static_exclude, B.sky());
            stage_filter_given(c, sc, w, rows, n, sp, B.sigma(), B.sg(), B.filt(), B.mask());
            const std::vector<std::vector<char>> a = device_artefacts_many(
                c, {{&mine, mine.size(), B.filt(), B.sky(), &t}}, o.grid, B.sub(), w, h, n, o.fwhm_px,
                p.max_frame_fraction, o.reg_dx, o.reg_dy, Band{r.first, rows});
            for (size_t e = 0; e < idx.size(); ++e) art[idx[e]] = a[0][e];
        }
        std::vector<float> kept;
        for (size_t e = 0; e < q.tested.size(); ++e)
            if (!art[e]) kept.push_back(q.tested[e].snr);
        std::sort(kept.begin(), kept.end(), std::greater<float>());
        pooled.insert(pooled.end(), kept.begin(), kept.end());
        pooled.insert(pooled.end(), q.rest.begin(), q.rest.end());
    }

    // ---- threshold, selection, refinement on bands with the refinement halo
    o.thr = set_threshold(p, pooled, runs, o.fwhm_px, w, h, m);
    if (runs > 0 && auto_thr) o.null_peaks.assign(pooled.begin(), pooled.end());
    for (const Peak& pk : o.peaks)
        if (pk.snr >= o.thr.snr && pk.vidx >= 0) o.selected.push_back(pk);
    if (static_cast<int>(o.selected.size()) > p.max_candidates) o.selected.resize(static_cast<size_t>(p.max_candidates));
    if (!o.selected.empty()) {
        report(1.0 - 1.0 / units, "refine");
        const int rf = c.span_begin("refine");
        FTB_CHECK(cudaMemcpyAsync(B.sigma(), sigma_real.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c.stream()));
        FTB_CHECK(cudaMemcpyAsync(B.sg(), sg_real.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c.stream()));
        std::vector<RefinedCandidate> rc(o.selected.size());
        for (const auto& core : cores) {
            std::vector<Peak> mine;
            std::vector<size_t> idx;
            for (size_t e = 0; e < o.selected.size(); ++e)
                if (o.selected[e].y >= core.first && o.selected[e].y < core.second) {
                    mine.push_back(o.selected[e]);
                    idx.push_back(e);
                }
            if (mine.empty()) continue;
            const auto r = region(core, g.refine);
            check_rows(r);
            const int rows = r.second - r.first;
            B.load_sub(r.first, r.second);
            stage_sky(c, sc, B.sub(), w, rows, n, o.t_h.data(), p.static_exclude, B.sky());
            stage_filter_given(c, sc, w, rows, n, sp, B.sigma(), B.sg(), B.filt(), B.mask());
            std::vector<RefinedCandidate> part =
                refine_tracks(c, o, p,
                              {B.filt(), sc.residual.as<float>(), B.sub(), B.sky(), B.mask(), w, h, pitch, n,
                               Band{r.first, rows}},
                              mine);
            for (size_t e = 0; e < idx.size(); ++e) rc[idx[e]] = std::move(part[e]);
        }
        o.candidates = finish_candidates(o, std::move(rc));
        c.span_end(rf);
    }
    c.span_end(total);
    FTB_CHECK(cudaStreamSynchronize(c.stream()));
    c.timing_resolve();
    report(1.0, "done");
    return o;
}

}  // namespace ftb
