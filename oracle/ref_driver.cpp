// Test infrastructure only: a plain-C driver over the reference library
// (FaintTrail 0.9.1, built from its own sources by oracle/Makefile), so that the
// Python tests can run the reference's own preprocessing, stacking backends and
// search on the same inputs as the CUDA path and compare the results bit for bit.
// Nothing in the product library links or loads this file.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "fainttrail/backend.hpp"
#include "fainttrail/fainttrail.h"
#include "fainttrail/fits.hpp"
#include "fainttrail/io.hpp"
#include "fainttrail/search.hpp"
#include "fainttrail/simulate.hpp"
#include "fainttrail/validate.hpp"
#include "internal.hpp"
#include "cuda_plan.hpp"

using namespace fainttrail;

namespace {

thread_local std::string g_err;

SearchParams to_search_params(const ft_params* p) {
    SearchParams s;
    if (!p) return s;
    s.vmin_pxh = p->vmin_pxh;
    s.vmax_pxh = p->vmax_pxh;
    s.grid_tol_px = p->grid_tol_px;
    s.fwhm_px = p->fwhm_px;
    s.clip_sigma = p->clip_sigma;
    s.cr_sigma = p->cr_sigma;
    s.mask_scatter = p->mask_scatter;
    s.weight_scatter = p->weight_scatter;
    s.static_exclude = p->static_exclude;
    s.min_coverage = p->min_coverage;
    s.threshold_snr = p->threshold_snr;
    s.min_snr_floor = p->min_snr_floor;
    s.target_false_per_run = p->target_false_per_run;
    s.max_frame_fraction = p->max_frame_fraction;
    s.half_tolerance = p->half_tolerance;
    s.null_runs = p->null_runs;
    s.max_candidates = p->max_candidates;
    s.edge_px = p->edge_px;
    s.threads = p->threads;
    s.seed = p->seed;
    s.backend = std::string(p->backend, strnlen(p->backend, sizeof p->backend));
    if (s.backend.empty()) s.backend = "auto";
    s.align = "off";  // synthetic frames are registered by construction
    return s;
}

std::vector<Image> images_from(const float* px, int n, int w, int h) {
    std::vector<Image> v(static_cast<std::size_t>(n), Image(w, h));
    const std::size_t plane = static_cast<std::size_t>(w) * h;
    for (int i = 0; i < n; ++i) std::memcpy(v[static_cast<std::size_t>(i)].data.data(), px + i * plane, plane * sizeof(float));
    return v;
}

void copy_images(const std::vector<Image>& v, float* out) {
    std::size_t o = 0;
    for (const auto& im : v) {
        std::memcpy(out + o, im.data.data(), im.data.size() * sizeof(float));
        o += im.data.size();
    }
}

struct Result {
    SearchResult r;
};

}  // namespace

extern "C" {

const char* ftref_last_error(void) { return g_err.c_str(); }

void ftref_params_default(ft_params* p) { ft_params_default(p); }

// Synthetic sequence from the reference simulator. Fields follow SimParams.
typedef struct ftref_sim {
    int width, height, nframes, nstars, nmovers, hot_pixels;
    double exptime_s, cadence_s, fwhm_px, sky_e_per_s, read_noise_e, gain_e_per_adu, bias_adu;
    double rate_min_arcsec_min, rate_max_arcsec_min, pixscale_arcsec, cosmic_rays_per_frame;
    double fwhm_jitter, transparency_jitter, star_mag_bright, star_mag_faint;
    unsigned long long seed;
} ftref_sim;

void ftref_sim_default(ftref_sim* s) {
    const SimParams d;
    s->width = d.width;
    s->height = d.height;
    s->nframes = d.nframes;
    s->nstars = d.nstars;
    s->nmovers = d.nmovers;
    s->hot_pixels = d.hot_pixels;
    s->exptime_s = d.exptime_s;
    s->cadence_s = d.cadence_s;
    s->fwhm_px = d.fwhm_px;
    s->sky_e_per_s = d.sky_e_per_s;
    s->read_noise_e = d.read_noise_e;
    s->gain_e_per_adu = d.gain_e_per_adu;
    s->bias_adu = d.bias_adu;
    s->rate_min_arcsec_min = d.rate_min_arcsec_min;
    s->rate_max_arcsec_min = d.rate_max_arcsec_min;
    s->pixscale_arcsec = d.pixscale_arcsec;
    s->cosmic_rays_per_frame = d.cosmic_rays_per_frame;
    s->fwhm_jitter = d.fwhm_jitter;
    s->transparency_jitter = d.transparency_jitter;
    s->star_mag_bright = d.star_mag_bright;
    s->star_mag_faint = d.star_mag_faint;
    s->seed = d.seed;
}

// simulate() with the given movers (movers[5 k ..] = x_ref, y_ref, vx_pxh, vy_pxh,
// mag; none: the simulation draws its own).
int ftref_simulate_movers(const ftref_sim* s, const double* movers, int nmovers, float* frames, double* mjd,
                          double* exptime) {
    try {
        SimParams p;
        p.width = s->width;
        p.height = s->height;
        p.nframes = s->nframes;
        p.nstars = s->nstars;
        p.nmovers = s->nmovers;
        p.hot_pixels = s->hot_pixels;
        p.exptime_s = s->exptime_s;
        p.cadence_s = s->cadence_s;
        p.fwhm_px = s->fwhm_px;
        p.sky_e_per_s = s->sky_e_per_s;
        p.read_noise_e = s->read_noise_e;
        p.gain_e_per_adu = s->gain_e_per_adu;
        p.bias_adu = s->bias_adu;
        p.rate_min_arcsec_min = s->rate_min_arcsec_min;
        p.rate_max_arcsec_min = s->rate_max_arcsec_min;
        p.pixscale_arcsec = s->pixscale_arcsec;
        p.cosmic_rays_per_frame = s->cosmic_rays_per_frame;
        p.fwhm_jitter = s->fwhm_jitter;
        p.transparency_jitter = s->transparency_jitter;
        p.star_mag_bright = s->star_mag_bright;
        p.star_mag_faint = s->star_mag_faint;
        p.seed = s->seed;
        std::vector<SimMover> given(static_cast<std::size_t>(std::max(0, nmovers)));
        for (int k = 0; k < nmovers; ++k) {
            SimMover& m = given[static_cast<std::size_t>(k)];
            m.id = "M" + std::to_string(k + 1);
            m.x_ref = movers[5 * k];
            m.y_ref = movers[5 * k + 1];
            m.vx_pxh = movers[5 * k + 2];
            m.vy_pxh = movers[5 * k + 3];
            m.mag = movers[5 * k + 4];
        }
        const SimResult r = simulate(p, given);
        std::size_t o = 0;
        for (std::size_t i = 0; i < r.frames.size(); ++i) {
            const auto& f = r.frames[i];
            std::memcpy(frames + o, f.image.data.data(), f.image.data.size() * sizeof(float));
            o += f.image.data.size();
            mjd[i] = f.mjd_mid;
            exptime[i] = f.exptime_s;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

int ftref_simulate(const ftref_sim* s, float* frames, double* mjd, double* exptime) {
    return ftref_simulate_movers(s, nullptr, 0, frames, mjd, exptime);
}

// prepare(): returns an opaque Prepared*.
// prepare() of frames given as arrays; reg_dx / reg_dy (or NULL): per-frame
// registration offsets, as load_frames() reads them from REGDX / REGDY.
void* ftref_prepare_reg(int n, int w, int h, const float* frames, const double* mjd, const double* exptime,
                        const double* reg_dx, const double* reg_dy, const ft_params* params) {
    try {
        std::vector<Frame> fr(static_cast<std::size_t>(n));
        const std::size_t plane = static_cast<std::size_t>(w) * h;
        for (int i = 0; i < n; ++i) {
            fr[static_cast<std::size_t>(i)].image = Image(w, h);
            std::memcpy(fr[static_cast<std::size_t>(i)].image.data.data(), frames + i * plane, plane * sizeof(float));
            fr[static_cast<std::size_t>(i)].mjd_mid = mjd[i];
            fr[static_cast<std::size_t>(i)].exptime_s = exptime[i];
            if (reg_dx && reg_dy) {
                fr[static_cast<std::size_t>(i)].has_reg_offset = true;
                fr[static_cast<std::size_t>(i)].reg_dx = reg_dx[i];
                fr[static_cast<std::size_t>(i)].reg_dy = reg_dy[i];
            }
        }
        SearchParams sp = to_search_params(params);
        return new Prepared(prepare(std::move(fr), sp));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void* ftref_prepare(int n, int w, int h, const float* frames, const double* mjd, const double* exptime,
                    const ft_params* params) {
    return ftref_prepare_reg(n, w, h, frames, mjd, exptime, nullptr, nullptr, params);
}

// load_frames() of FITS files (newline-separated paths): with pixels NULL only
// the sizes; else the pixels (n x h x w), mid-exposure MJD, exposure time and
// registration offsets (has_reg = 1 when every frame carries REGDX / REGDY).
int ftref_load_frames(const char* paths_nl, float* pixels, double* mjd, double* exptime, double* reg_dx,
                      double* reg_dy, int* has_reg, int* w, int* h, int* n) {
    try {
        std::vector<std::string> paths;
        std::string cur;
        for (const char* c = paths_nl; *c; ++c) {
            if (*c == '\n') {
                if (!cur.empty()) paths.push_back(cur);
                cur.clear();
            } else {
                cur += *c;
            }
        }
        if (!cur.empty()) paths.push_back(cur);
        const std::vector<Frame> fr = load_frames(paths);
        *n = static_cast<int>(fr.size());
        *w = fr.empty() ? 0 : fr[0].image.width;
        *h = fr.empty() ? 0 : fr[0].image.height;
        if (!pixels) return 0;
        bool all = true;
        const std::size_t plane = static_cast<std::size_t>(*w) * *h;
        for (std::size_t i = 0; i < fr.size(); ++i) {
            std::memcpy(pixels + i * plane, fr[i].image.data.data(), plane * sizeof(float));
            mjd[i] = fr[i].mjd_mid;
            exptime[i] = fr[i].exptime_s;
            reg_dx[i] = fr[i].reg_dx;
            reg_dy[i] = fr[i].reg_dy;
            all = all && fr[i].has_reg_offset;
        }
        *has_reg = all ? 1 : 0;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

void ftref_prep_free(void* h) { delete static_cast<Prepared*>(h); }

void ftref_prep_info(void* hp, int* w, int* h, int* n, double* fwhm, double* span_h, double* t_ref) {
    const Prepared& p = *static_cast<Prepared*>(hp);
    *w = p.width;
    *h = p.height;
    *n = p.nframes;
    *fwhm = p.fwhm_px;
    *span_h = p.span_h;
    *t_ref = p.t_ref_mjd;
}

void ftref_prep_vectors(void* hp, double* t_h, double* sigma, double* background, int* cr, int* rank) {
    const Prepared& p = *static_cast<Prepared*>(hp);
    for (int i = 0; i < p.nframes; ++i) {
        if (t_h) t_h[i] = p.t_h[static_cast<std::size_t>(i)];
        if (sigma) sigma[i] = p.sigma[static_cast<std::size_t>(i)];
        if (background) background[i] = p.background[static_cast<std::size_t>(i)];
        if (cr) cr[i] = p.cr_pixels[static_cast<std::size_t>(i)];
        if (rank) rank[i] = p.time_rank[static_cast<std::size_t>(i)];
    }
}

void ftref_prep_images(void* hp, float* sub, float* filtered, float* static_sky, float* mask) {
    const Prepared& p = *static_cast<Prepared*>(hp);
    if (sub) copy_images(p.sub, sub);
    if (filtered) copy_images(p.filtered, filtered);
    if (static_sky) std::memcpy(static_sky, p.static_sky.data.data(), p.static_sky.data.size() * sizeof(float));
    if (mask) std::memcpy(mask, p.mask.data.data(), p.mask.data.size() * sizeof(float));
}

// detail::build_stage on background-subtracted frames with the given times and a
// fixed PSF width (the null-run form: no PSF estimate).
int ftref_build_stage(const float* sub, int n, int w, int h, const double* t_h, double fwhm_px, const ft_params* params,
                      float* filtered, float* static_sky, float* mask, double* sigma, int* cr, float* residual) {
    try {
        const std::vector<Image> subs = images_from(sub, n, w, h);
        Prepared p;
        p.width = w;
        p.height = h;
        p.nframes = n;
        p.t_h.assign(t_h, t_h + n);
        p.fwhm_px = fwhm_px;
        SearchParams sp = to_search_params(params);
        sp.keep_residuals = residual != nullptr;
        detail::build_stage(subs, p, sp, {}, false);
        if (filtered) copy_images(p.filtered, filtered);
        if (static_sky) std::memcpy(static_sky, p.static_sky.data.data(), p.static_sky.data.size() * sizeof(float));
        if (mask) std::memcpy(mask, p.mask.data.data(), p.mask.data.size() * sizeof(float));
        for (int i = 0; i < n; ++i) {
            if (sigma) sigma[i] = p.sigma[static_cast<std::size_t>(i)];
            if (cr) cr[i] = p.cr_pixels[static_cast<std::size_t>(i)];
        }
        if (residual) copy_images(p.residual, residual);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// One stacking pass. which: 0 CPU backend, 1 run_pass_naive, 2 run_pass_simple,
// 3 the reference CUDA backend ("cuda"). dx/dy: motion-major tables, or NULL with
// t_h + vel (vx, vy pairs) for straight-line shifts.
int ftref_stack(const float* frames, int w, int h, int n, const int* dx, const int* dy, const double* t_h,
                const double* vel, int m, int min_count, int threads, int which, float* max_snr, int* best_v) {
    try {
        const std::vector<Image> fr = images_from(frames, n, w, h);
        std::vector<double> t;
        std::vector<std::pair<double, double>> v;
        ShiftTable table;
        StackPass pass;
        pass.frames = &fr;
        if (dx) {
            table.resize(m, n);
            std::memcpy(table.dx.data(), dx, sizeof(int) * static_cast<std::size_t>(m) * n);
            std::memcpy(table.dy.data(), dy, sizeof(int) * static_cast<std::size_t>(m) * n);
            pass.shifts = &table;
        } else {
            t.assign(t_h, t_h + n);
            for (int j = 0; j < m; ++j) v.emplace_back(vel[2 * j], vel[2 * j + 1]);
            pass.t_h = &t;
            pass.velocities = &v;
        }
        pass.min_count = min_count;
        pass.threads = threads;
        StackResult r;
        if (which == 0) r = make_backend("cpu")->run(pass);
        else if (which == 1) r = run_pass_naive(pass);
        else if (which == 2) r = run_pass_simple(pass);
        else r = make_backend("cuda")->run(pass);
        std::memcpy(max_snr, r.max_snr.data.data(), r.max_snr.data.size() * sizeof(float));
        std::memcpy(best_v, r.best_v.data(), r.best_v.size() * sizeof(int));
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// The reference CUDA backend's pass (CudaBackend::run, backend_cuda.cu:99-195)
// with straight-line shifts, and its own timing breakdown: timings[0..3] =
// upload, kernel, download, setup seconds (the StageTime entries it reports).
int ftref_stack_cuda_timed(const float* frames, int w, int h, int n, const double* t_h, const double* vel, int m,
                           int min_count, float* max_snr, int* best_v, double* timings) {
    try {
        const std::vector<Image> fr = images_from(frames, n, w, h);
        std::vector<double> t(t_h, t_h + n);
        std::vector<std::pair<double, double>> v;
        for (int j = 0; j < m; ++j) v.emplace_back(vel[2 * j], vel[2 * j + 1]);
        StackPass pass;
        pass.frames = &fr;
        pass.t_h = &t;
        pass.velocities = &v;
        pass.min_count = min_count;
        const StackResult r = make_backend("cuda")->run(pass);
        std::memcpy(max_snr, r.max_snr.data.data(), r.max_snr.data.size() * sizeof(float));
        std::memcpy(best_v, r.best_v.data(), r.best_v.size() * sizeof(int));
        const char* names[4] = {"upload", "kernel", "download", "setup"};
        for (int k = 0; k < 4; ++k) {
            timings[k] = 0.0;
            for (const auto& st : r.timings)
                if (st.name == names[k]) timings[k] = st.seconds;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// The reference's backend conformance procedure (the CLI's check-backend,
// cli/main.cpp:697-741) for a registered backend `name`: a simulated 72 x 52 x 12
// sequence against run_pass_naive, the same frames with a curved shift table,
// and a 384 x 320 x 40 sequence against run_pass_simple, each judged by
// check_backend (backend.cpp:281-314). Writes one line per check into `report`;
// returns the number of checks that conform; *identical counts those whose maps
// are also bit-identical; -1 on error.
int ftref_check_backend(const char* name, char* report, int cap, int* checks, int* identical) {
    try {
        const std::unique_ptr<SearchBackend> cand = make_backend(name);
        std::string text;
        int ok = 0, same = 0, total = 0;
        auto judge = [&](const char* what, const StackPass& pass, const StackResult& ref, const StackResult& got) {
            const BackendCheck c = check_backend(pass, ref, got);
            const bool bits = ref.best_v == got.best_v && ref.max_snr.data.size() == got.max_snr.data.size() &&
                              std::memcmp(ref.max_snr.data.data(), got.max_snr.data.data(),
                                          ref.max_snr.data.size() * sizeof(float)) == 0;
            ++total;
            ok += c.ok;
            same += c.ok && bits;
            text += std::string(what) + ": " + c.message + (bits ? ", bit-identical" : "") + "\n";
        };
        for (int round = 0; round < 2; ++round) {
            SimParams sp;
            sp.width = round == 0 ? 72 : 384;
            sp.height = round == 0 ? 52 : 320;
            sp.nframes = round == 0 ? 12 : 40;
            sp.nstars = round == 0 ? 20 : 400;
            sp.seed = 77 + static_cast<std::uint64_t>(round);
            const SimResult sim = simulate(sp);
            SearchParams p;
            p.vmin_pxh = 2;
            p.vmax_pxh = round == 0 ? 20 : 45;
            const Prepared prep = prepare(sim.frames, p);
            const auto grid = velocity_grid(prep, p);
            StackPass pass;
            pass.frames = &prep.filtered;
            pass.t_h = &prep.t_h;
            pass.velocities = &grid;
            pass.min_count = std::max(3, static_cast<int>(std::ceil(p.min_coverage * prep.nframes)));
            const StackResult got = cand->run(pass);
            if (round == 0) {
                judge("vs naive contract (72x52, 12 fr)", pass, run_pass_naive(pass), got);
                ShiftTable curved = linear_shift_table(prep.t_h, grid);
                for (int j = 0; j < curved.motions; ++j)
                    for (int i = 0; i < curved.frames; ++i) {
                        const double ti = prep.t_h[static_cast<std::size_t>(i)];
                        curved.x(j, i) += static_cast<int>(std::lround(((j % 9) - 4) * 2.0 * ti * ti));
                        curved.y(j, i) += static_cast<int>(std::lround(((j % 7) - 3) * 2.0 * ti * ti));
                    }
                StackPass cp = pass;
                cp.shifts = &curved;
                judge("curved shift table vs naive", cp, run_pass_naive(cp), cand->run(cp));
            } else {
                judge("vs simple reference (384x320, 40 fr)", pass, run_pass_simple(pass), got);
            }
        }
        if (report && cap > 0) {
            std::strncpy(report, text.c_str(), static_cast<std::size_t>(cap) - 1);
            report[cap - 1] = 0;
        }
        if (checks) *checks = total;
        if (identical) *identical = same;
        return ok;
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

int ftref_cuda_available(void) { return cuda_backend_available(nullptr) ? 1 : 0; }

// velocity_grid for a sequence of the given span. Returns the count (or -1);
// writes at most `cap` (vx, vy) pairs.
int ftref_velocity_grid(double span_h, const ft_params* params, double* out, int cap, double* dv) {
    try {
        Prepared p;
        p.span_h = span_h;
        const auto g = velocity_grid(p, to_search_params(params), dv);
        for (std::size_t j = 0; j < g.size() && static_cast<int>(j) < cap; ++j) {
            out[2 * j] = g[j].first;
            out[2 * j + 1] = g[j].second;
        }
        return static_cast<int>(g.size());
    } catch (const std::exception& e) {
        g_err = e.what();
        return -1;
    }
}

void ftref_null_orders(const double* t_h, int n, int runs, unsigned long long seed, double* out) {
    const auto o = detail::null_time_orders(std::vector<double>(t_h, t_h + n), runs, seed);
    for (int k = 0; k < runs; ++k)
        for (int i = 0; i < n; ++i) out[k * n + i] = o[static_cast<std::size_t>(k)][static_cast<std::size_t>(i)];
}

int ftref_find_peaks(const float* max_snr, const int* best_v, int w, int h, float floor, int radius, int edge,
                     int max_peaks, int* px, int* py, float* psnr, int* pv) {
    StackResult r;
    r.max_snr = Image(w, h);
    std::memcpy(r.max_snr.data.data(), max_snr, sizeof(float) * static_cast<std::size_t>(w) * h);
    r.best_v.assign(best_v, best_v + static_cast<std::size_t>(w) * h);
    const auto pk = detail::find_peaks(r, floor, radius, edge, static_cast<std::size_t>(max_peaks));
    for (std::size_t k = 0; k < pk.size(); ++k) {
        px[k] = pk[k].x;
        py[k] = pk[k].y;
        psnr[k] = pk[k].snr;
        pv[k] = pk[k].vidx;
    }
    return static_cast<int>(pk.size());
}

// set_threshold from pooled null peaks. method_out: at least 32 bytes.
double ftref_set_threshold(const float* pooled, int count, int runs, const ft_params* params, char* method_out,
                           double* a, double* k, double* inv_s2) {
    Prepared p;
    SearchResult res;
    detail::set_threshold(p, to_search_params(params), 1, runs, std::vector<float>(pooled, pooled + count), res);
    std::strncpy(method_out, res.threshold_method.c_str(), 31);
    method_out[31] = 0;
    *a = res.null_a;
    *k = res.null_k;
    *inv_s2 = res.null_inv_s2;
    return res.threshold_snr;
}

// is_artefact_peak on a Prepared (its filtered frames, sub frames, static sky).
int ftref_is_artefact_peak(void* hp, int x, int y, float snr, int vidx, double vx, double vy, const ft_params* params) {
    const Prepared& p = *static_cast<Prepared*>(hp);
    detail::Peak pk;
    pk.x = x;
    pk.y = y;
    pk.snr = snr;
    pk.vidx = vidx;
    return detail::is_artefact_peak(p, pk, {vx, vy}, to_search_params(params)) ? 1 : 0;
}

// A Prepared for the null run with the given times (detail::with_times).
void* ftref_with_times(void* hp, const double* t_h, const ft_params* params) {
    try {
        const Prepared& p = *static_cast<Prepared*>(hp);
        return new Prepared(detail::with_times(p, std::vector<double>(t_h, t_h + p.nframes), to_search_params(params)));
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

// search() on a Prepared; returns an opaque result.
void* ftref_search(void* hp, const ft_params* params) {
    try {
        return new Result{search(*static_cast<Prepared*>(hp), to_search_params(params))};
    } catch (const std::exception& e) {
        g_err = e.what();
        return nullptr;
    }
}

void ftref_result_free(void* r) { delete static_cast<Result*>(r); }

double ftref_result_scalars(void* rp, char* method_out, double* dv, int* n_velocities, int* n_candidates,
                            int* n_null_peaks, double* null_a, double* null_k, double* null_inv_s2) {
    const SearchResult& r = static_cast<Result*>(rp)->r;
    std::strncpy(method_out, r.threshold_method.c_str(), 31);
    method_out[31] = 0;
    *dv = r.dv_pxh;
    *n_velocities = static_cast<int>(r.n_velocities);
    *n_candidates = static_cast<int>(r.candidates.size());
    *n_null_peaks = static_cast<int>(r.null_peaks.size());
    *null_a = r.null_a;
    *null_k = r.null_k;
    *null_inv_s2 = r.null_inv_s2;
    return r.threshold_snr;
}

void ftref_result_arrays(void* rp, float* max_snr, double* null_peaks) {
    const SearchResult& r = static_cast<Result*>(rp)->r;
    if (max_snr) std::memcpy(max_snr, r.max_snr.data.data(), r.max_snr.data.size() * sizeof(float));
    if (null_peaks) std::copy(r.null_peaks.begin(), r.null_peaks.end(), null_peaks);
}

// Candidate k as 17 doubles: x, y, vx, vy, pos_err, vel_err, snr, snr_coarse,
// snr_half1, snr_half2, max_frame_fraction, false_alarms_per_run, flux, mag_inst,
// ok, id, inv_dist; flags into flags_out (64 bytes).
void ftref_result_candidate(void* rp, int k, double* out, char* flags_out) {
    const Candidate& c = static_cast<Result*>(rp)->r.candidates[static_cast<std::size_t>(k)];
    const double v[17] = {c.x, c.y, c.vx_pxh, c.vy_pxh, c.pos_err_px, c.vel_err_pxh, c.snr, c.snr_coarse, c.snr_half1,
                          c.snr_half2, c.max_frame_fraction, c.false_alarms_per_run, c.flux, c.mag_inst,
                          c.ok ? 1.0 : 0.0, static_cast<double>(c.id), c.inv_dist_au};
    std::memcpy(out, v, sizeof v);
    std::strncpy(flags_out, c.flags.c_str(), 63);
    flags_out[63] = 0;
}

// The reference epoch and PSF width of a result, and its candidate file
// (write_candidates_csv, io.cpp:82-115) written to path (NULL: not written).
int ftref_result_csv(void* rp, const char* path, double* t_ref_mjd, double* fwhm_px) {
    const SearchResult& r = static_cast<Result*>(rp)->r;
    *t_ref_mjd = r.t_ref_mjd;
    *fwhm_px = r.fwhm_px;
    if (!path) return 0;
    try {
        write_candidates_csv(path, r);
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// ft_get_track_point (c_api.cpp:248-261) of candidate k in frame i of a result
// of the prepared sequence hp: out = mjd, x, y (FITS 1-based), ra, dec.
int ftref_track_point(void* hp, void* rp, int k, int frame, double* out) {
    const Prepared& p = *static_cast<Prepared*>(hp);
    const SearchResult& r = static_cast<Result*>(rp)->r;
    if (k < 0 || k >= static_cast<int>(r.candidates.size()) || frame < 0 || frame >= p.nframes) return 1;
    const auto pts = track_points(p, r.candidates[static_cast<std::size_t>(k)]);
    const TrackPoint& q = pts[static_cast<std::size_t>(frame)];
    const double v[5] = {q.mjd, q.x + 1.0, q.y + 1.0, q.ra_deg, q.dec_deg};
    std::memcpy(out, v, sizeof v);
    return 0;
}

// iso_from_mjd (fits.cpp:474-504) into out (cap bytes, NUL-terminated).
void ftref_iso_from_mjd(double mjd, int decimals, char* out, int cap) {
    const std::string s = iso_from_mjd(mjd, decimals);
    std::strncpy(out, s.c_str(), static_cast<std::size_t>(cap) - 1);
    out[cap - 1] = 0;
}

// completeness() on raw frames: rows of 7 doubles per level (target_snr,
// injected, recovered, detected, mean_snr, mean_dpos, mean_dv).
int ftref_completeness(int n, int w, int h, const float* frames, const double* mjd, const double* exptime,
                       const ft_params* params, const double* levels, int nlevels, int per_level, double min_sep,
                       unsigned long long seed, double* rows, double* thr, char* method_out, int* baseline_ok,
                       double* snr50) {
    try {
        std::vector<Frame> fr(static_cast<std::size_t>(n));
        const std::size_t plane = static_cast<std::size_t>(w) * h;
        for (int i = 0; i < n; ++i) {
            fr[static_cast<std::size_t>(i)].image = Image(w, h);
            std::memcpy(fr[static_cast<std::size_t>(i)].image.data.data(), frames + i * plane, plane * sizeof(float));
            fr[static_cast<std::size_t>(i)].mjd_mid = mjd[i];
            fr[static_cast<std::size_t>(i)].exptime_s = exptime[i];
        }
        CompletenessParams cp;
        cp.snr_levels.assign(levels, levels + nlevels);
        cp.per_level = per_level;
        cp.min_separation = min_sep;
        cp.seed = seed;
        const CompletenessReport r = completeness(fr, to_search_params(params), cp);
        for (std::size_t k = 0; k < r.rows.size(); ++k) {
            const CompletenessRow& q = r.rows[k];
            const double v[7] = {q.target_snr, static_cast<double>(q.injected), static_cast<double>(q.recovered),
                                 static_cast<double>(q.detected), q.mean_snr, q.mean_dpos, q.mean_dv};
            std::memcpy(rows + 7 * k, v, sizeof v);
        }
        *thr = r.threshold_snr;
        std::strncpy(method_out, r.threshold_method.c_str(), 31);
        method_out[31] = 0;
        *baseline_ok = r.baseline_ok;
        *snr50 = r.snr50;
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

// Injection of trailed movers (validate.cpp inject) into raw frames, in place.
void ftref_inject(float* frames, int n, int w, int h, const double* mjd, const double* exptime, const double* obj,
                  int nobj, double t_ref_mjd, double fwhm_px) {
    std::vector<Frame> fr(static_cast<std::size_t>(n));
    const std::size_t plane = static_cast<std::size_t>(w) * h;
    for (int i = 0; i < n; ++i) {
        fr[static_cast<std::size_t>(i)].image = Image(w, h);
        std::memcpy(fr[static_cast<std::size_t>(i)].image.data.data(), frames + i * plane, plane * sizeof(float));
        fr[static_cast<std::size_t>(i)].mjd_mid = mjd[i];
        fr[static_cast<std::size_t>(i)].exptime_s = exptime[i];
    }
    std::vector<Injection> inj(static_cast<std::size_t>(nobj));
    for (int k = 0; k < nobj; ++k) {
        inj[static_cast<std::size_t>(k)].x_ref = obj[5 * k];
        inj[static_cast<std::size_t>(k)].y_ref = obj[5 * k + 1];
        inj[static_cast<std::size_t>(k)].vx_pxh = obj[5 * k + 2];
        inj[static_cast<std::size_t>(k)].vy_pxh = obj[5 * k + 3];
        inj[static_cast<std::size_t>(k)].flux = obj[5 * k + 4];
    }
    inject(fr, inj, t_ref_mjd, fwhm_px);
    for (int i = 0; i < n; ++i) std::memcpy(frames + i * plane, fr[static_cast<std::size_t>(i)].image.data.data(), plane * sizeof(float));
}

// check_registration (registration.cpp:260-312) of n frames (n x h x w) observed
// at t_h hours: out[0..8] = measured, registered, dx, dy, mid_dx, mid_dy,
// rate_pxh, stars, matched; the message into msg (NUL-terminated).
int ftref_check_registration(const float* frames, int n, int w, int h, const double* t_h, double* out, char* msg,
                             int msg_len) {
    try {
        const std::vector<Image> ims = images_from(frames, n, w, h);
        std::vector<const Image*> ptrs;
        for (const auto& im : ims) ptrs.push_back(&im);
        const DriftCheck r = check_registration(ptrs, std::vector<double>(t_h, t_h + n));
        const double v[9] = {r.measured ? 1.0 : 0.0, r.registered ? 1.0 : 0.0, r.dx, r.dy, r.mid_dx, r.mid_dy,
                             r.rate_pxh, static_cast<double>(r.stars), static_cast<double>(r.matched)};
        std::memcpy(out, v, sizeof v);
        if (msg && msg_len > 0) {
            std::strncpy(msg, r.message.c_str(), static_cast<std::size_t>(msg_len) - 1);
            msg[msg_len - 1] = 0;
        }
        return 0;
    } catch (const std::exception& e) {
        g_err = e.what();
        return 1;
    }
}

}  // extern "C"
