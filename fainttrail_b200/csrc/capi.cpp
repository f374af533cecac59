// The C ABI of the B200 backend (include/ft_b200.h): argument checks, error
// capture and status codes around the C++ engine.
#include "ft_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <string>
#include <vector>

#include "candidate.h"
#include "engine.h"
#include "ft_internal.h"
#include "registration.h"
#include "search.h"
#include "serve.h"
#include "stage.h"

struct ft_b200_ctx {
    std::unique_ptr<ftb::Context> c;
};

struct ft_b200_result {
    ftb::SearchOut o;
};

struct ft_b200_server {
    std::unique_ptr<ftb::Server> s;
    std::string error;
};

namespace {

thread_local std::string g_open_error;

ftb::Progress wrap(ft_b200_progress_fn fn, void* user) {
    if (!fn) return {};
    return [fn, user](double f, const char* stage) { return fn(f, stage, user) != 0; };
}

template <class F>
int guarded(ft_b200_ctx* ctx, F&& f) {
    if (!ctx || !ctx->c) return FT_B200_ERROR;
    try {
        ctx->c->bind();
        f(*ctx->c);
        return FT_B200_OK;
    } catch (const ftb::Cancelled&) {
        ctx->c->error = "cancelled";
        return FT_B200_CANCELLED;
    } catch (const std::exception& e) {
        ctx->c->error = e.what();
        return FT_B200_ERROR;
    }
}

// validate_pass (backend.cpp:89-108) for the C form of a pass
void check_pass(const float* frames, int w, int h, int n, int m, int min_count) {
    if (!frames) throw std::runtime_error("stack pass: missing frames");
    if (n < 1) throw std::runtime_error("stack pass: no frames");
    if (w < 1 || h < 1) throw std::runtime_error("stack pass: frames differ in size");
    if (m < 1) throw std::runtime_error("stack pass: malformed shift table");
    if (min_count < 1) throw std::runtime_error("stack pass: min_count must be at least 1");
}

double max_abs(const double* t, int n) {
    double m = 0;
    for (int i = 0; i < n; ++i) m = std::max(m, std::fabs(t[i]));
    return m;
}

}  // namespace

namespace ftb {
void set_thread_error(const std::string& msg) { g_open_error = msg; }
}  // namespace ftb

extern "C" {

const char* ft_b200_version(void) { return "0.9.1-b200.1"; }

int ft_b200_open(int device, double hbm_budget_bytes, ft_b200_ctx** out) {
    if (!out) return FT_B200_ERROR;
    *out = nullptr;
    try {
        auto h = std::make_unique<ft_b200_ctx>();
        h->c = std::make_unique<ftb::Context>(device, hbm_budget_bytes);
        *out = h.release();
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

void ft_b200_close(ft_b200_ctx* ctx) { delete ctx; }

const char* ft_b200_last_error(const ft_b200_ctx* ctx) {
    if (!ctx || !ctx->c) return g_open_error.c_str();
    return ctx->c->error.c_str();
}

int ft_b200_device_info(ft_b200_ctx* ctx, char* name, int name_len, int* sms, double* hbm_bytes) {
    return guarded(ctx, [&](ftb::Context& c) {
        if (name && name_len > 0) {
            std::strncpy(name, c.name().c_str(), static_cast<size_t>(name_len) - 1);
            name[name_len - 1] = 0;
        }
        if (sms) *sms = c.sms();
        if (hbm_bytes) *hbm_bytes = c.total_bytes();
    });
}

int ft_b200_stack(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const int* dx,
                  const int* dy, int motions, int min_count, float* max_snr, int* best_v,
                  ft_b200_progress_fn progress, void* user) {
    return guarded(ctx, [&](ftb::Context& c) {
        check_pass(frames, width, height, nframes, motions, min_count);
        if (!dx || !dy) throw std::runtime_error("stack pass: malformed shift table");
        if (!max_snr || !best_v) throw std::runtime_error("stack pass: missing outputs");
        ftb::stack_pass_host(c, frames, width, height, nframes, dx, dy, motions, min_count, nullptr, 0.0, max_snr,
                             best_v, wrap(progress, user));
    });
}

int ft_b200_stack_linear(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes,
                         const double* t_h, const double* velocities, int motions, int min_count, float* max_snr,
                         int* best_v, ft_b200_progress_fn progress, void* user) {
    return guarded(ctx, [&](ftb::Context& c) {
        check_pass(frames, width, height, nframes, motions, min_count);
        if (!t_h || !velocities) throw std::runtime_error("stack pass: missing times or velocities");
        if (!max_snr || !best_v) throw std::runtime_error("stack pass: missing outputs");
        // round(v t), half away from zero, in double (pass_shift, backend.hpp:87-97)
        std::vector<int> dx(static_cast<size_t>(motions) * nframes), dy(dx.size());
        for (int j = 0; j < motions; ++j)
            for (int i = 0; i < nframes; ++i) {
                dx[static_cast<size_t>(j) * nframes + i] = static_cast<int>(std::lround(velocities[2 * j] * t_h[i]));
                dy[static_cast<size_t>(j) * nframes + i] = static_cast<int>(std::lround(velocities[2 * j + 1] * t_h[i]));
            }
        ftb::stack_pass_host(c, frames, width, height, nframes, dx.data(), dy.data(), motions, min_count, velocities,
                             max_abs(t_h, nframes), max_snr, best_v, wrap(progress, user));
    });
}

int ft_b200_stack_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch, int nframes,
                      const int* dx, const int* dy, int motions, int min_count, float* d_max_snr, int* d_best_v) {
    return guarded(ctx, [&](ftb::Context& c) {
        check_pass(d_frames, width, height, nframes, motions, min_count);
        if (!dx || !dy) throw std::runtime_error("stack pass: malformed shift table");
        if (!d_max_snr || !d_best_v) throw std::runtime_error("stack pass: missing outputs");
        if (pitch < width || (pitch * 4) % 16 != 0 || reinterpret_cast<uintptr_t>(d_frames) % 16 != 0)
            throw std::runtime_error("stack pass: device frames need a 16-byte aligned base and row pitch");
        c.timing_reset();
        ftb::stack_pass_device(c, d_frames, pitch, width, height, nframes, dx, dy, motions, min_count, nullptr, 0.0,
                               d_max_snr, d_best_v, {});
        c.timing_resolve();
    });
}

namespace {
static void put_drift(const ftb::DriftCheck& d, ft_b200_drift_check* out) {
    std::memset(out, 0, sizeof *out);
    out->measured = d.measured ? 1 : 0;
    out->registered = d.registered ? 1 : 0;
    out->stars = d.stars;
    out->matched = d.matched;
    out->dx = d.dx;
    out->dy = d.dy;
    out->mid_dx = d.mid_dx;
    out->mid_dy = d.mid_dy;
    out->rate_pxh = d.rate_pxh;
    std::strncpy(out->message, d.message.c_str(), sizeof out->message - 1);
}
}  // namespace

int ft_b200_check_registration(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes,
                               const double* t_h, ft_b200_drift_check* out) {
    return guarded(ctx, [&](ftb::Context& c) {
        if (!frames || !t_h || !out) throw std::runtime_error("registration check: missing frames, times or output");
        if (nframes < 0 || width < 1 || height < 1) throw std::runtime_error("registration check: empty frames");
        c.timing_reset();
        ftb::DriftCheck d;
        if (nframes >= 3) {  // only the first, middle and last frame by time are read
            int fi[3];
            ftb::registration_frames(t_h, nframes, &fi[0], &fi[1], &fi[2]);
            const int pitch = ftb::frame_pitch(width);
            const size_t plane = static_cast<size_t>(pitch) * height;
            ftb::DevBuf buf(&c, sizeof(float) * plane * 3, "registration frames");
            const float* three[3];
            for (int k = 0; k < 3; ++k) {
                float* dst = buf.as<float>() + static_cast<size_t>(k) * plane;
                FTB_CHECK(cudaMemcpy2DAsync(dst, sizeof(float) * pitch,
                                            frames + static_cast<size_t>(fi[k]) * width * height, sizeof(float) * width,
                                            sizeof(float) * width, static_cast<size_t>(height), cudaMemcpyHostToDevice,
                                            c.stream()));
                three[k] = dst;
            }
            d = ftb::check_registration_three(c, three, pitch, width, height, t_h[fi[2]] - t_h[fi[0]]);
        }
        c.timing_resolve();
        put_drift(d, out);
    });
}

int ft_b200_check_registration_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch,
                                   int nframes, const double* t_h, ft_b200_drift_check* out) {
    return guarded(ctx, [&](ftb::Context& c) {
        if (!d_frames || !t_h || !out) throw std::runtime_error("registration check: missing frames, times or output");
        if (nframes < 0 || width < 1 || height < 1) throw std::runtime_error("registration check: empty frames");
        if (pitch < width) throw std::runtime_error("registration check: pitch must be >= width");
        c.timing_reset();
        const ftb::DriftCheck d = ftb::check_registration_device(c, d_frames, static_cast<size_t>(pitch) * height,
                                                                 pitch, width, height, nframes, t_h);
        c.timing_resolve();
        put_drift(d, out);
    });
}

int ft_b200_result_registration(const ft_b200_result* r, ft_b200_drift_check* out) {
    if (!r || !out) return FT_B200_ERROR;
    put_drift(r->o.registration, out);
    return FT_B200_OK;
}

int ft_b200_stage_dev(ft_b200_ctx* ctx, const float* d_sub, int width, int height, int pitch, int nframes,
                      const double* t_h, const ft_b200_stage_params* params, float* d_filtered,
                      float* d_static_sky, float* d_mask, double* sigma, int* cr_pixels) {
    return guarded(ctx, [&](ftb::Context& c) {
        if (!d_sub || !t_h || !params) throw std::runtime_error("stage: missing frames, times or parameters");
        if (nframes < 1 || width < 1 || height < 1) throw std::runtime_error("stage: empty frames");
        if (pitch < width) throw std::runtime_error("stage: pitch must be >= width");
        if (!(params->fwhm_px > 0.0)) throw std::runtime_error("stage: the PSF FWHM must be positive");
        ftb::StageParams sp;
        sp.fwhm_px = params->fwhm_px;
        sp.static_exclude = params->static_exclude;
        sp.clip_sigma = params->clip_sigma;
        sp.cr_sigma = params->cr_sigma;
        sp.mask_scatter = params->mask_scatter;
        sp.weight_scatter = params->weight_scatter;
        ftb::stage_device(c, d_sub, pitch, width, height, nframes, t_h, sp, d_filtered, d_static_sky, d_mask, sigma,
                          cr_pixels);
    });
}

int ft_b200_emulate_stack(const float* frames, int width, int height, int nframes, const int* dx, const int* dy,
                          int motions, int min_count, int shape, float* max_snr, int* best_v) {
    try {
        check_pass(frames, width, height, nframes, motions, min_count);
        if (!dx || !dy) throw std::runtime_error("stack pass: malformed shift table");
        if (!max_snr || !best_v) throw std::runtime_error("stack pass: missing outputs");
        if (shape < 0 || shape > ftb::kStackShapes) throw std::runtime_error("emulate: unknown tile shape");
        const size_t pixels = static_cast<size_t>(width) * height;
        if (min_count > nframes) {  // as the device entries: no S/N is defined anywhere
            std::fill(max_snr, max_snr + pixels, 0.0f);
            std::fill(best_v, best_v + pixels, -1);
            return FT_B200_OK;
        }
        constexpr int kB200SmemOptin = 232448;  // 227 KB of shared memory per block
        // a fixed shape whose windows do not fit falls back to the automatic
        // choice, as ft_b200_set_tile_shape does for the device
        ftb::StackConfig cfg = ftb::choose_stack_config(width, height, nframes, kB200SmemOptin);
        if (shape > 0 && ftb::stack_shape_fits(ftb::stack_shape_config(shape, kB200SmemOptin), nframes))
            cfg = ftb::stack_shape_config(shape, kB200SmemOptin);
        const ftb::StackPlan plan =
            ftb::make_stack_plan(width, height, nframes, dx, dy, motions, min_count,
                                 ftb::motion_order(dx, dy, motions, nframes, 4.0, 4.0), cfg);
        ftb::emulate_stack_pass(plan, frames, max_snr, best_v);
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

int ft_b200_set_wait_test(int extra_bytes, long long wait_cycles) {
    try {
        ftb::set_wait_test(extra_bytes, wait_cycles);
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

int ft_b200_plan_stats(int width, int height, int nframes, const int* dx, const int* dy, int motions, int shape,
                       long long* stats) {
    try {
        if (!dx || !dy || !stats || width < 1 || height < 1 || nframes < 1 || motions < 1)
            throw std::runtime_error("plan_stats: malformed pass");
        if (shape < 0 || shape > ftb::kStackShapes) throw std::runtime_error("plan_stats: unknown tile shape");
        constexpr int kB200SmemOptin = 232448;
        ftb::StackConfig cfg = ftb::choose_stack_config(width, height, nframes, kB200SmemOptin);
        if (shape > 0 && ftb::stack_shape_fits(ftb::stack_shape_config(shape, kB200SmemOptin), nframes))
            cfg = ftb::stack_shape_config(shape, kB200SmemOptin);
        const ftb::StackPlan plan = ftb::make_stack_plan(width, height, nframes, dx, dy, motions, 1,
                                                         ftb::motion_order(dx, dy, motions, nframes, 4.0, 4.0), cfg);
        long long fast = 0, pads = 0, fast_slots = 0;
        for (const auto& g : plan.groups) {
            fast += g.rows_fast;
            fast_slots += g.rows_fast ? g.nslots : 0;
        }
        for (int j : plan.slot_motion) pads += j < 0;
        stats[0] = static_cast<long long>(plan.groups.size());
        stats[1] = fast;
        stats[2] = static_cast<long long>(plan.slot_motion.size());
        stats[3] = pads;
        stats[4] = fast_slots;
        stats[5] = plan.max_group_bytes;
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

void ft_b200_stage_params_default(ft_b200_stage_params* p) {
    if (!p) return;
    const ftb::StageParams d;
    p->fwhm_px = 0.0;
    p->static_exclude = d.static_exclude;
    p->clip_sigma = d.clip_sigma;
    p->cr_sigma = d.cr_sigma;
    p->mask_scatter = d.mask_scatter;
    p->weight_scatter = d.weight_scatter;
}

int ft_b200_stage(ft_b200_ctx* ctx, const float* sub, int width, int height, int nframes, const double* t_h,
                  const ft_b200_stage_params* params, float* filtered, float* static_sky, float* mask, double* sigma,
                  int* cr_pixels) {
    return guarded(ctx, [&](ftb::Context& c) {
        if (!sub || !t_h || !params) throw std::runtime_error("stage: missing frames, times or parameters");
        if (nframes < 1 || width < 1 || height < 1) throw std::runtime_error("stage: empty frames");
        if (!(params->fwhm_px > 0.0)) throw std::runtime_error("stage: the PSF FWHM must be positive");
        ftb::StageParams sp;
        sp.fwhm_px = params->fwhm_px;
        sp.static_exclude = params->static_exclude;
        sp.clip_sigma = params->clip_sigma;
        sp.cr_sigma = params->cr_sigma;
        sp.mask_scatter = params->mask_scatter;
        sp.weight_scatter = params->weight_scatter;
        ftb::stage_host(c, sub, width, height, nframes, t_h, sp, filtered, static_sky, mask, sigma, cr_pixels);
    });
}

void ft_b200_search_params_default(ft_b200_search_params* p) {
    if (!p) return;
    const ftb::SearchParams d;
    std::memset(p, 0, sizeof *p);
    p->vmin_pxh = d.vmin_pxh;
    p->vmax_pxh = d.vmax_pxh;
    p->grid_tol_px = d.grid_tol_px;
    p->fwhm_px = d.fwhm_px;
    p->clip_sigma = d.clip_sigma;
    p->cr_sigma = d.cr_sigma;
    p->mask_scatter = d.mask_scatter;
    p->weight_scatter = d.weight_scatter;
    p->min_coverage = d.min_coverage;
    p->threshold_snr = d.threshold_snr;
    p->min_snr_floor = d.min_snr_floor;
    p->target_false_per_run = d.target_false_per_run;
    p->max_frame_fraction = d.max_frame_fraction;
    p->half_tolerance = d.half_tolerance;
    p->static_exclude = d.static_exclude;
    p->null_runs = d.null_runs;
    p->max_candidates = d.max_candidates;
    p->edge_px = d.edge_px;
    p->threads = 0;
    p->seed = d.seed;
    p->null_tested = d.null_tested;
    p->null_model_gauss = d.gauss_model ? 1 : 0;
    p->passes_per_launch = d.passes_per_launch;
    p->shard_index = d.shard_index;
    p->shard_count = d.shard_count;
    p->align = d.align;
}

namespace {
// nframes: the frames of the search (for the per-frame registration offsets;
// 0 where a call has no frames)
static ftb::SearchParams to_search_params(const ft_b200_search_params* params, int nframes) {
    ft_b200_search_params d;
    ft_b200_search_params_default(&d);
    const ft_b200_search_params& q = params ? *params : d;
    ftb::SearchParams p;
    p.vmin_pxh = q.vmin_pxh;
    p.vmax_pxh = q.vmax_pxh;
    p.grid_tol_px = q.grid_tol_px;
    p.fwhm_px = q.fwhm_px;
    p.clip_sigma = q.clip_sigma;
    p.cr_sigma = q.cr_sigma;
    p.mask_scatter = q.mask_scatter;
    p.weight_scatter = q.weight_scatter;
    p.min_coverage = q.min_coverage;
    p.threshold_snr = q.threshold_snr;
    p.min_snr_floor = q.min_snr_floor;
    p.target_false_per_run = q.target_false_per_run;
    p.max_frame_fraction = q.max_frame_fraction;
    p.static_exclude = q.static_exclude;
    p.null_runs = q.null_runs;
    p.null_tested = q.null_tested;
    p.max_candidates = q.max_candidates;
    p.edge_px = q.edge_px;
    p.gauss_model = q.null_model_gauss != 0;
    p.passes_per_launch = std::max(0, q.passes_per_launch);
    p.half_tolerance = q.half_tolerance;
    p.calibrated_threshold = q.calibrated_threshold;
    p.cal_a = q.calibrated_tail[0];
    p.cal_b = q.calibrated_tail[1];
    p.cal_k = q.calibrated_tail[2];
    p.cal_inv_s2 = q.calibrated_tail[3];
    p.shard_count = std::max(1, q.shard_count);
    p.shard_index = q.shard_index;
    if (p.shard_index < 0 || p.shard_index >= p.shard_count)
        throw std::runtime_error("search: shard_index must lie in [0, shard_count)");
    p.seed = q.seed;
    p.align = q.align;
    if (p.align < 0 || p.align > 2) throw std::runtime_error("search: align must be 0 (off), 1 (check) or 2 (auto)");
    if ((q.reg_dx != nullptr) != (q.reg_dy != nullptr))
        throw std::runtime_error("search: registration offsets need both reg_dx and reg_dy");
    if (q.reg_dx && nframes > 0) {
        p.reg_dx.assign(q.reg_dx, q.reg_dx + nframes);
        p.reg_dy.assign(q.reg_dy, q.reg_dy + nframes);
    }
    return p;
}
}  // namespace

int ft_b200_search(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const double* mjd,
                   const double* exptime, const ft_b200_search_params* params, ft_b200_progress_fn progress,
                   void* user, ft_b200_result** out) {
    if (out) *out = nullptr;
    return guarded(ctx, [&](ftb::Context& c) {
        if (!frames || !mjd || !out) throw std::runtime_error("search: missing frames, times or result pointer");
        auto r = std::make_unique<ft_b200_result>();
        r->o = ftb::search_host(c, frames, width, height, nframes, mjd, exptime, to_search_params(params, nframes),
                                wrap(progress, user));
        *out = r.release();
    });
}

int ft_b200_search_tiled(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const double* mjd,
                         const double* exptime, const ft_b200_search_params* params, int band_rows,
                         ft_b200_progress_fn progress, void* user, ft_b200_result** out) {
    if (out) *out = nullptr;
    return guarded(ctx, [&](ftb::Context& c) {
        if (!frames || !mjd || !out) throw std::runtime_error("search: missing frames, times or result pointer");
        if (band_rows < 0) throw std::runtime_error("tiled search: band_rows must be 0 (automatic) or positive");
        auto r = std::make_unique<ft_b200_result>();
        r->o = ftb::search_tiled_host(c, frames, width, height, nframes, mjd, exptime,
                                      to_search_params(params, nframes), band_rows, wrap(progress, user));
        *out = r.release();
    });
}

namespace {
static int search_batch_common(ft_b200_ctx* ctx, const float* frames, bool on_device, int pitch, int width, int height,
                               int nframes, const double* mjd, const double* exptime, const ft_b200_search_params* params,
                               int copies, const int* objects_per_copy, const ft_b200_injection* objects,
                               ft_b200_progress_fn progress, void* user, ft_b200_result** base,
                               ft_b200_result** copy_results) {
    if (base) *base = nullptr;
    for (int k = 0; copy_results && k < copies; ++k) copy_results[k] = nullptr;
    return guarded(ctx, [&](ftb::Context& c) {
        if (!frames || !mjd || !exptime || !base) throw std::runtime_error("search: missing frames, times or result");
        if (copies < 0 || (copies > 0 && (!objects_per_copy || !objects || !copy_results)))
            throw std::runtime_error("search: malformed injection copies");
        if (on_device && pitch < width) throw std::runtime_error("search: row pitch below the width");
        std::vector<std::vector<ftb::Injection>> sets(static_cast<size_t>(copies));
        size_t at = 0;
        for (int k = 0; k < copies; ++k) {
            if (objects_per_copy[k] < 0) throw std::runtime_error("search: negative object count");
            for (int q = 0; q < objects_per_copy[k]; ++q, ++at)
                sets[static_cast<size_t>(k)].push_back(
                    {objects[at].x_ref, objects[at].y_ref, objects[at].vx_pxh, objects[at].vy_pxh, objects[at].flux});
        }
        std::vector<ftb::SearchOut> outs;
        auto r = std::make_unique<ft_b200_result>();
        r->o = ftb::search_batch_host(c, frames, width, height, nframes, mjd, exptime, to_search_params(params, nframes), sets,
                                      outs, wrap(progress, user), on_device, on_device ? pitch : width);
        std::vector<std::unique_ptr<ft_b200_result>> rs;
        for (auto& o : outs) {
            rs.push_back(std::make_unique<ft_b200_result>());
            rs.back()->o = std::move(o);
        }
        *base = r.release();
        for (int k = 0; k < copies; ++k) copy_results[k] = rs[static_cast<size_t>(k)].release();
    });
}
}  // namespace

int ft_b200_search_batch(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes,
                         const double* mjd, const double* exptime, const ft_b200_search_params* params, int copies,
                         const int* objects_per_copy, const ft_b200_injection* objects, ft_b200_progress_fn progress,
                         void* user, ft_b200_result** base, ft_b200_result** copy_results) {
    return search_batch_common(ctx, frames, false, width, width, height, nframes, mjd, exptime, params, copies,
                               objects_per_copy, objects, progress, user, base, copy_results);
}

int ft_b200_search_batch_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch, int nframes,
                             const double* mjd, const double* exptime, const ft_b200_search_params* params,
                             int copies, const int* objects_per_copy, const ft_b200_injection* objects,
                             ft_b200_result** base, ft_b200_result** copy_results) {
    return search_batch_common(ctx, d_frames, true, pitch, width, height, nframes, mjd, exptime, params, copies,
                               objects_per_copy, objects, nullptr, nullptr, base, copy_results);
}

int ft_b200_search_dev(ft_b200_ctx* ctx, const float* d_frames, int width, int height, int pitch, int nframes,
                       const double* mjd, const double* exptime, const ft_b200_search_params* params,
                       ft_b200_result** out) {
    if (out) *out = nullptr;
    return guarded(ctx, [&](ftb::Context& c) {
        if (!d_frames || !mjd || !out) throw std::runtime_error("search: missing frames, times or result pointer");
        if (pitch < width) throw std::runtime_error("search: row pitch below the width");
        auto r = std::make_unique<ft_b200_result>();
        r->o = ftb::search_host(c, d_frames, width, height, nframes, mjd, exptime, to_search_params(params, nframes), {}, true,
                                pitch);
        *out = r.release();
    });
}

int ft_b200_set_tile_shape(int shape) {
    try {
        ftb::set_stack_shape(shape);
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

int ft_b200_tile_shape(void) { return ftb::stack_shape(); }

int ft_b200_tuned_shapes(int* keys, int* shapes, int cap) {
    const auto v = ftb::tuned_shapes();
    for (size_t k = 0; k < v.size() && static_cast<int>(k) < cap; ++k) {
        if (keys)
            for (int q = 0; q < 4; ++q) keys[4 * k + q] = v[k].first[static_cast<size_t>(q)];
        if (shapes) shapes[k] = v[k].second;
    }
    return static_cast<int>(v.size());
}

void ft_b200_clear_tuned_shapes(void) { ftb::clear_tuned_shapes(); }

int ft_b200_server_open(int device, double hbm_budget_bytes, int max_batch, int workers, ft_b200_server** out) {
    if (!out) return FT_B200_ERROR;
    *out = nullptr;
    try {
        auto h = std::make_unique<ft_b200_server>();
        h->s = std::make_unique<ftb::Server>(device, hbm_budget_bytes, max_batch, workers > 0 ? workers : 2);
        *out = h.release();
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

void ft_b200_server_close(ft_b200_server* s) { delete s; }

int ft_b200_server_submit(ft_b200_server* s, const float* frames, int width, int height, int nframes,
                          const double* mjd, const double* exptime, const ft_b200_search_params* params,
                          long long* request_id) {
    if (!s || !request_id) return FT_B200_ERROR;
    try {
        *request_id = s->s->submit(frames, width, height, nframes, mjd, exptime, to_search_params(params, nframes));
        return FT_B200_OK;
    } catch (const std::exception& e) {
        s->error = e.what();
        return FT_B200_ERROR;
    }
}

int ft_b200_server_poll(ft_b200_server* s, long long request_id, int wait_ms, ft_b200_result** out) {
    if (!s) return FT_B200_ERROR;
    if (out) *out = nullptr;
    auto r = std::make_unique<ft_b200_result>();
    std::string err;
    const int rc = s->s->poll(request_id, wait_ms, &r->o, &err);
    if (rc == 3) return FT_B200_PENDING;
    if (rc != 0) {
        s->error = err;
        return FT_B200_ERROR;
    }
    if (out) *out = r.release();
    return FT_B200_OK;
}

const char* ft_b200_server_error(const ft_b200_server* s) { return s ? s->error.c_str() : g_open_error.c_str(); }

int ft_b200_server_pause(ft_b200_server* s, int paused) {
    if (!s) return FT_B200_ERROR;
    s->s->pause(paused != 0);
    return FT_B200_OK;
}

int ft_b200_server_stats(ft_b200_server* s, long long* completed, double* p50_s, double* p99_s,
                         double* searches_per_s, long long* rounds, double* mean_batch, long long* launches) {
    if (!s) return FT_B200_ERROR;
    const ftb::ServerStats st = s->s->stats();
    if (completed) *completed = st.completed;
    if (p50_s) *p50_s = st.p50_s;
    if (p99_s) *p99_s = st.p99_s;
    if (searches_per_s) *searches_per_s = st.searches_per_s;
    if (rounds) *rounds = st.rounds;
    if (mean_batch) *mean_batch = st.mean_batch;
    if (launches) *launches = st.launches;
    return FT_B200_OK;
}

int ft_b200_stats(const ft_b200_ctx* ctx, long long* kernel_launches, double* pixel_adds) {
    if (!ctx || !ctx->c) return FT_B200_ERROR;
    if (kernel_launches) *kernel_launches = ctx->c->launches;
    (void)pixel_adds;
    return FT_B200_OK;
}

void ft_b200_result_free(ft_b200_result* r) { delete r; }

double ft_b200_result_threshold(const ft_b200_result* r, char* method, int method_len, double* null_a,
                                double* null_b, double* null_k, double* null_inv_s2) {
    if (!r) return 0.0;
    const ftb::Threshold& t = r->o.thr;
    if (method && method_len > 0) {
        std::strncpy(method, t.method.c_str(), static_cast<size_t>(method_len) - 1);
        method[method_len - 1] = 0;
    }
    if (null_a) *null_a = t.a;
    if (null_b) *null_b = t.b;
    if (null_k) *null_k = t.k;
    if (null_inv_s2) *null_inv_s2 = t.inv_s2;
    return t.snr;
}

int ft_b200_result_info(const ft_b200_result* r, double* fwhm_px, double* dv_pxh, double* t_ref_mjd,
                        int* n_velocities) {
    if (!r) return FT_B200_ERROR;
    if (fwhm_px) *fwhm_px = r->o.fwhm_px;
    if (dv_pxh) *dv_pxh = r->o.dv;
    if (t_ref_mjd) *t_ref_mjd = r->o.t_ref_mjd;
    if (n_velocities) *n_velocities = static_cast<int>(r->o.grid.size());
    return FT_B200_OK;
}

int ft_b200_result_peaks(const ft_b200_result* r, int which, ft_b200_peak* out, int cap) {
    if (!r) return 0;
    const auto& v = which == 1 ? r->o.selected : r->o.peaks;
    for (size_t k = 0; out && k < v.size() && static_cast<int>(k) < cap; ++k)
        out[k] = {v[k].x, v[k].y, v[k].snr, v[k].vidx};
    return static_cast<int>(v.size());
}

int ft_b200_completeness(ft_b200_ctx* ctx, const float* frames, int width, int height, int nframes, const double* mjd,
                         const double* exptime, const ft_b200_search_params* params, const double* snr_levels,
                         int nlevels, int per_level, double min_separation, unsigned long long seed,
                         ft_b200_completeness_row* rows, double* threshold_snr, char* method, int method_cap,
                         int* baseline_ok, double* snr50) {
    return guarded(ctx, [&](ftb::Context& c) {
        if (!frames || !mjd || !exptime || !rows || nlevels < 0 || (nlevels > 0 && !snr_levels) || per_level < 0)
            throw std::runtime_error("completeness: missing or malformed arguments");
        const std::vector<double> levels(snr_levels, snr_levels + nlevels);
        const ftb::CompletenessOut r = ftb::completeness_host(c, frames, width, height, nframes, mjd, exptime,
                                                               to_search_params(params, nframes), levels, per_level,
                                                               min_separation, seed);
        for (int k = 0; k < nlevels; ++k) {
            const ftb::CompletenessRow& q = r.rows[static_cast<size_t>(k)];
            rows[k] = {q.target_snr, q.injected, q.recovered, q.detected, q.mean_snr, q.mean_dpos, q.mean_dv};
        }
        if (threshold_snr) *threshold_snr = r.threshold_snr;
        if (method && method_cap > 0) {
            std::strncpy(method, r.threshold_method.c_str(), static_cast<size_t>(method_cap) - 1);
            method[method_cap - 1] = 0;
        }
        if (baseline_ok) *baseline_ok = r.baseline_ok;
        if (snr50) *snr50 = r.snr50;
    });
}

int ft_b200_pool_null_peaks(const ft_b200_peak* raster, int count, const unsigned char* artefact, int keep,
                            int tested, int mode, float* pooled, int cap) {
    try {
        if (count < 0 || (count > 0 && (!raster || !artefact)) || keep < 0 || tested < 0)
            throw std::runtime_error("pool null peaks: bad arguments");
        // the flags travel with the peaks (x, y identify a raster peak)
        std::vector<ftb::Peak> pk(static_cast<size_t>(count));
        std::map<std::pair<int, int>, unsigned char> flag;
        for (int q = 0; q < count; ++q) {
            pk[static_cast<size_t>(q)] = {raster[q].x, raster[q].y, raster[q].snr, raster[q].vidx};
            flag[{raster[q].x, raster[q].y}] = artefact[q];
        }
        std::vector<float> out;
        if (mode == 0) {
            ftb::order_peaks(pk, static_cast<size_t>(keep));
            for (size_t q = 0; q < pk.size(); ++q)
                if (q >= static_cast<size_t>(tested) || !flag[{pk[q].x, pk[q].y}]) out.push_back(pk[q].snr);
        } else {
            const ftb::NullPeaks np = ftb::split_null_peaks(pk, static_cast<size_t>(keep), static_cast<size_t>(tested));
            std::vector<float> kept;
            for (const ftb::Peak& p : np.tested)
                if (!flag[{p.x, p.y}]) kept.push_back(p.snr);
            std::sort(kept.begin(), kept.end(), std::greater<float>());
            out = kept;
            out.insert(out.end(), np.rest.begin(), np.rest.end());
        }
        for (size_t q = 0; q < out.size() && static_cast<int>(q) < cap; ++q) pooled[q] = out[q];
        return static_cast<int>(out.size());
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return -1;
    }
}

int ft_b200_null_threshold(const double* pooled, long long count, int runs, double fwhm_px, int width, int height,
                           int motions, const ft_b200_search_params* params, double* threshold, char* method,
                           int method_cap, double* a, double* b, double* k, double* inv_s2) {
    try {
        if (count < 0 || (count > 0 && !pooled)) throw std::runtime_error("null threshold: missing pooled peaks");
        if (runs < 0 || width < 1 || height < 1 || motions < 0) throw std::runtime_error("null threshold: bad sizes");
        ftb::SearchParams p = to_search_params(params, 0);
        p.shard_index = 0;
        p.shard_count = 1;
        // the engine pools the S/N values as float; doubles that came from a result convert back exactly
        std::vector<float> v(static_cast<size_t>(count));
        for (long long q = 0; q < count; ++q) v[static_cast<size_t>(q)] = static_cast<float>(pooled[q]);
        const ftb::Threshold t = ftb::set_threshold(p, v, runs, fwhm_px, width, height, static_cast<size_t>(motions));
        if (threshold) *threshold = t.snr;
        if (method && method_cap > 0) {
            std::strncpy(method, t.method.c_str(), static_cast<size_t>(method_cap) - 1);
            method[method_cap - 1] = 0;
        }
        if (a) *a = t.a;
        if (b) *b = t.b;
        if (k) *k = t.k;
        if (inv_s2) *inv_s2 = t.inv_s2;
        return FT_B200_OK;
    } catch (const std::exception& e) {
        g_open_error = e.what();
        return FT_B200_ERROR;
    }
}

int ft_b200_result_null_peaks(const ft_b200_result* r, double* out, int cap) {
    if (!r) return 0;
    const auto& v = r->o.null_peaks;
    for (size_t k = 0; out && k < v.size() && static_cast<int>(k) < cap; ++k) out[k] = v[k];
    return static_cast<int>(v.size());
}

int ft_b200_result_candidates(const ft_b200_result* r, double* rows, char* flags, int cap) {
    if (!r) return 0;
    const auto& v = r->o.candidates;
    for (size_t k = 0; k < v.size() && static_cast<int>(k) < cap; ++k) {
        const ftb::Candidate& c = v[k];
        if (rows) {
            const double row[17] = {c.x, c.y, c.vx_pxh, c.vy_pxh, c.pos_err_px, c.vel_err_pxh, c.snr, c.snr_coarse,
                                    c.snr_half1, c.snr_half2, c.max_frame_fraction, c.false_alarms_per_run, c.flux,
                                    c.mag_inst, c.ok ? 1.0 : 0.0, static_cast<double>(c.id), c.inv_dist_au};
            std::memcpy(rows + 17 * k, row, sizeof row);
        }
        if (flags) {
            std::strncpy(flags + 64 * k, c.flags.c_str(), 63);
            flags[64 * k + 63] = 0;
        }
    }
    return static_cast<int>(v.size());
}

namespace {
static std::string result_csv(const ft_b200_result* r) {
    ftb::CandidateListInfo info;
    info.t_ref_mjd = r->o.t_ref_mjd;
    info.threshold_snr = r->o.thr.snr;
    info.method = r->o.thr.method;
    info.dv_pxh = r->o.dv;
    info.fwhm_px = r->o.fwhm_px;
    info.n_velocities = static_cast<long long>(r->o.grid.size());
    return ftb::candidates_csv(info, r->o.candidates);
}
}  // namespace

int ft_b200_result_candidate(const ft_b200_result* r, int index, ft_b200_candidate* out) {
    if (!r || !out || index < 0 || index >= static_cast<int>(r->o.candidates.size())) return FT_B200_ERROR;
    const ftb::Candidate& c = r->o.candidates[static_cast<size_t>(index)];
    std::memset(out, 0, sizeof *out);
    out->id = c.id;
    out->ok = c.ok ? 1 : 0;
    out->x = c.x + 1.0;
    out->y = c.y + 1.0;
    out->vx_pxh = c.vx_pxh;
    out->vy_pxh = c.vy_pxh;
    out->pos_err_px = c.pos_err_px;
    out->vel_err_pxh = c.vel_err_pxh;
    out->snr = c.snr;
    out->snr_coarse = c.snr_coarse;
    out->snr_half1 = c.snr_half1;
    out->snr_half2 = c.snr_half2;
    out->max_frame_fraction = c.max_frame_fraction;
    out->false_alarms_per_run = c.false_alarms_per_run;
    out->flux = c.flux;
    out->mag_inst = c.mag_inst;
    std::strncpy(out->flags, c.flags.c_str(), sizeof out->flags - 1);
    return FT_B200_OK;
}

int ft_b200_result_track_point(const ft_b200_result* r, int index, int frame, double* mjd, double* x, double* y,
                               double* ra_deg, double* dec_deg) {
    if (!r || index < 0 || index >= static_cast<int>(r->o.candidates.size()) || frame < 0 ||
        frame >= static_cast<int>(r->o.t_h.size()))
        return FT_B200_ERROR;
    const ftb::TrackPoint p = ftb::track_point(r->o.t_ref_mjd, r->o.t_h[static_cast<size_t>(frame)],
                                               r->o.candidates[static_cast<size_t>(index)]);
    if (mjd) *mjd = p.mjd;
    if (x) *x = p.x;
    if (y) *y = p.y;
    if (ra_deg) *ra_deg = 0.0;
    if (dec_deg) *dec_deg = 0.0;
    return FT_B200_OK;
}

long long ft_b200_result_candidates_csv(const ft_b200_result* r, char* buf, long long cap) {
    if (!r) return -1;
    const std::string text = result_csv(r);
    if (buf && cap > 0) {
        const size_t k = std::min(text.size(), static_cast<size_t>(cap - 1));
        std::memcpy(buf, text.data(), k);
        buf[k] = 0;
    }
    return static_cast<long long>(text.size());
}

int ft_b200_write_candidates_csv(const ft_b200_result* r, const char* path) {
    if (!r || !path) {
        g_open_error = "write_candidates_csv: missing result or path";
        return FT_B200_ERROR;
    }
    const std::string text = result_csv(r);
    std::FILE* f = std::fopen(path, "wb");
    if (!f) {
        g_open_error = std::string("cannot write ") + path;
        return FT_B200_ERROR;
    }
    const bool written = std::fwrite(text.data(), 1, text.size(), f) == text.size();
    if (std::fclose(f) != 0 || !written) {
        g_open_error = std::string("cannot write ") + path;
        return FT_B200_ERROR;
    }
    return FT_B200_OK;
}

int ft_b200_result_maps(const ft_b200_result* r, float* max_snr, int* best_v) {
    if (!r || r->o.max_snr.empty()) return FT_B200_ERROR;  // a null-run shard other than 0 has no maps
    if (max_snr) std::memcpy(max_snr, r->o.max_snr.data(), sizeof(float) * r->o.max_snr.size());
    if (best_v) std::memcpy(best_v, r->o.best_v.data(), sizeof(int) * r->o.best_v.size());
    return FT_B200_OK;
}

int ft_b200_result_velocity(const ft_b200_result* r, int vidx, double* vx_pxh, double* vy_pxh) {
    if (!r || vidx < 0 || vidx >= static_cast<int>(r->o.grid.size())) return FT_B200_ERROR;
    if (vx_pxh) *vx_pxh = r->o.grid[static_cast<size_t>(vidx)].first;
    if (vy_pxh) *vy_pxh = r->o.grid[static_cast<size_t>(vidx)].second;
    return FT_B200_OK;
}

int ft_b200_timings(const ft_b200_ctx* ctx, char* names, int names_len, double* seconds, int cap) {
    if (!ctx || !ctx->c) return 0;
    const auto& t = ctx->c->timings;
    std::string joined;
    for (size_t k = 0; k < t.size(); ++k) {
        if (seconds && static_cast<int>(k) < cap) seconds[k] = t[k].second;
        joined += (k ? ";" : "") + t[k].first;
    }
    if (names && names_len > 0) {
        std::strncpy(names, joined.c_str(), static_cast<size_t>(names_len) - 1);
        names[names_len - 1] = 0;
    }
    return static_cast<int>(t.size());
}

}  // extern "C"
