// Device context and the stacking-pass driver of the B200 backend.
#include "engine.h"

#include "stage.h"

#include <algorithm>
#include <chrono>
#include <map>
#include <mutex>
#include <thread>
#include <tuple>
#include <cmath>
#include <cstdlib>

namespace ftb {

// ------------------------------------------------------------------ memory

DevBuf::DevBuf(Context* c, size_t bytes, const char* what) : ctx_(c), bytes_(bytes) {
    c->charge(bytes, what);
    p_ = c->take_cached(bytes);
    if (p_) return;
    cudaError_t e = cudaMallocAsync(&p_, std::max<size_t>(bytes, 1), c->stream());
    if (e != cudaSuccess) {
        // the cached blocks back to the device, then once more
        cudaGetLastError();
        c->drop_cache();
        cudaStreamSynchronize(c->stream());
        e = cudaMallocAsync(&p_, std::max<size_t>(bytes, 1), c->stream());
    }
    if (e != cudaSuccess) {
        c->release(bytes);
        p_ = nullptr;
        cudaGetLastError();
        throw CudaError(std::string("allocate ") + what + " (" + std::to_string(bytes) + " bytes): " +
                        cudaGetErrorString(e));
    }
}

void DevBuf::reset() {
    if (p_) {
        if (!ctx_->put_cached(p_, bytes_)) cudaFreeAsync(p_, ctx_->stream());
        ctx_->release(bytes_);
    }
    p_ = nullptr;
    bytes_ = 0;
    ctx_ = nullptr;
}

void* Context::take_cached(size_t bytes) {
    std::lock_guard<std::mutex> lk(cache_mu_);
    auto it = cache_.find(bytes);
    if (it == cache_.end()) return nullptr;
    void* p = it->second;
    cache_.erase(it);
    cached_ -= bytes;
    return p;
}

bool Context::put_cached(void* p, size_t bytes) {
    std::lock_guard<std::mutex> lk(cache_mu_);
    if (bytes < (size_t{1} << 20) || acct_.use_count() > 1) return false;  // small blocks: the pool
    if (cached_ + bytes > kCacheBytes || acct_->used.load() + cached_ + bytes > acct_->budget) return false;
    cache_.emplace(bytes, p);
    cached_ += bytes;
    return true;
}

void Context::drop_cache() {
    std::lock_guard<std::mutex> lk(cache_mu_);
    for (auto& kv : cache_) cudaFreeAsync(kv.second, stream_);
    cache_.clear();
    cached_ = 0;
}

Context::Context(int device, double budget_bytes) {
    init(device);
    size_t free_b = 0, total_b = 0;
    FTB_CHECK(cudaMemGetInfo(&free_b, &total_b));
    acct_ = std::make_shared<BudgetAccount>();
    acct_->budget = budget_bytes > 0 ? static_cast<size_t>(budget_bytes) : static_cast<size_t>(0.9 * free_b);
}

Context::Context(int device, std::shared_ptr<BudgetAccount> account) {
    if (!account) throw std::runtime_error("context: no budget account");
    init(device);
    acct_ = std::move(account);
}

void Context::init(int device) {
    if (device < 0) {
        const char* e = std::getenv("FAINTTRAIL_CUDA_DEVICE");
        device = e ? std::atoi(e) : 0;
    }
    int count = 0;
    FTB_CHECK(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count)
        throw std::runtime_error("CUDA device " + std::to_string(device) + " not present (" + std::to_string(count) +
                                 " found)");
    device_ = device;
    FTB_CHECK(cudaSetDevice(device_));
    cudaDeviceProp prop{};
    FTB_CHECK(cudaGetDeviceProperties(&prop, device_));
    if (prop.major != 10) throw std::runtime_error(std::string("this backend is built for sm_100a (B200); device is ") + prop.name);
    name_ = prop.name;
    sms_ = prop.multiProcessorCount;
    smem_optin_ = static_cast<int>(prop.sharedMemPerBlockOptin);
    total_ = static_cast<double>(prop.totalGlobalMem);
    FTB_CHECK(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
    FTB_CHECK(cudaMalloc(&d_err_, sizeof(int)));
    FTB_CHECK(cudaMemset(d_err_, 0, sizeof(int)));
    // keep freed pool memory for reuse instead of returning it at every sync
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, device_) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
}

double wall_seconds() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

int Context::event() {
    if (next_event_ >= static_cast<int>(events_.size())) {
        cudaEvent_t e;
        FTB_CHECK(cudaEventCreate(&e));
        events_.push_back(e);
    }
    return next_event_++;
}

void Context::timing_reset() {
    spans_.clear();
    timings.clear();
    next_event_ = 0;
    launches = 0;
}

int Context::span_begin(const std::string& name) {
    Span s;
    s.name = name;
    s.a = event();
    FTB_CHECK(cudaEventRecord(events_[static_cast<size_t>(s.a)], stream_));
    spans_.push_back(s);
    return static_cast<int>(spans_.size()) - 1;
}

void Context::span_end(int span) {
    Span& s = spans_[static_cast<size_t>(span)];
    s.b = event();
    FTB_CHECK(cudaEventRecord(events_[static_cast<size_t>(s.b)], stream_));
}

void Context::host_time(const std::string& name, double seconds) {
    Span s;
    s.name = name;
    s.host = seconds;
    spans_.push_back(s);
}

void Context::timing_resolve() {
    timings.clear();
    for (const Span& s : spans_) {
        double sec = s.host;
        if (s.a >= 0 && s.b >= 0) {
            float ms = 0;
            FTB_CHECK(cudaEventElapsedTime(&ms, events_[static_cast<size_t>(s.a)], events_[static_cast<size_t>(s.b)]));
            sec = ms * 1e-3;
        }
        bool merged = false;
        for (auto& t : timings)
            if (t.first == s.name) {
                t.second += sec;
                merged = true;
            }
        if (!merged) timings.emplace_back(s.name, sec);
    }
}

Context::~Context() {
    cudaSetDevice(device_);
    scratch_.clear();
    drop_cache();
    for (cudaEvent_t e : events_) cudaEventDestroy(e);
    if (stream_) cudaStreamSynchronize(stream_);
    if (d_err_) cudaFree(d_err_);
    if (stream_) cudaStreamDestroy(stream_);
}

void Context::bind() const { FTB_CHECK(cudaSetDevice(device_)); }

void Context::charge(size_t bytes, const char* what) {
    size_t cur = acct_->used.load();
    do {
        if (cur + bytes > acct_->budget)
            throw std::runtime_error(std::string("HBM budget exceeded allocating ") + what + ": " +
                                     std::to_string((cur + bytes) / 1048576) + " MiB needed, budget " +
                                     std::to_string(acct_->budget / 1048576) + " MiB");
    } while (!acct_->used.compare_exchange_weak(cur, cur + bytes));
}

void Context::check_kernel_error(const char* what) {
    FTB_CHECK(cudaStreamSynchronize(stream_));
    int e = 0;
    FTB_CHECK(cudaMemcpy(&e, d_err_, sizeof(int), cudaMemcpyDeviceToHost));
    if (e != 0) {
        FTB_CHECK(cudaMemset(d_err_, 0, sizeof(int)));
        throw std::runtime_error(std::string(what) + ": a device wait timed out (error " + std::to_string(e) + ")");
    }
}

DevBuf& Context::scratch(int slot, size_t bytes, const char* what) {
    if (static_cast<int>(scratch_.size()) <= slot) scratch_.resize(static_cast<size_t>(slot) + 1);
    DevBuf& b = scratch_[static_cast<size_t>(slot)];
    if (b.bytes() < bytes) {
        b.reset();
        b = DevBuf(this, bytes, what);
    }
    return b;
}

// ------------------------------------------------------------------ stacking

enum Slot { kFrames = 0, kBest, kArg, kMax, kBestV, kStageOut, kSky, kMask, kDesc };

namespace {

// Launch a planned pass in group ranges; between ranges the progress callback
// is asked (fraction of groups done), as the reference CUDA backend does between
// its launches (backend_cuda.cu:167-173).
void run_plan(Context& c, const StackPlan& plan, const float* d_frames, float* d_max, int* d_bv,
              const Progress& progress) {
    StackPlanDev dev;
    dev.upload(plan, c.stream());
    const int ng = static_cast<int>(plan.groups.size());
    const int chunks = progress ? std::min(ng, 16) : 1;
    float* d_best = nullptr;
    int* d_arg = nullptr;
    if (chunks > 1) {
        d_best = c.scratch(kBest, sizeof(float) * static_cast<size_t>(plan.w) * plan.h, "stack maxima").as<float>();
        d_arg = c.scratch(kArg, sizeof(int) * static_cast<size_t>(plan.w) * plan.h, "stack argmax").as<int>();
    }
    try {
        const int span = c.span_begin("kernel");
        for (int q = 0; q < chunks; ++q) {
            const int g0 = static_cast<int>(static_cast<long long>(ng) * q / chunks);
            const int g1 = static_cast<int>(static_cast<long long>(ng) * (q + 1) / chunks);
            BatchPass bp;
            bp.plan = &plan;
            bp.dev = &dev;
            bp.frames = d_frames;
            bp.g0 = g0;
            bp.g1 = g1;
            bp.first = q == 0;
            bp.last = q == chunks - 1;
            bp.best = d_best;
            bp.arg = d_arg;
            bp.max_snr = d_max;
            bp.best_v = d_bv;
            DevBuf& desc = c.scratch(kDesc, batch_desc_bytes(1), "stack descriptors");
            stack_launch_batch({bp}, desc.as<unsigned char>(), desc.bytes(), c.err_flag(), c.sms(), c.stream());
            ++c.launches;
            if (progress) {
                c.check_kernel_error("stack kernel");
                if (!progress(static_cast<double>(q + 1) / chunks, "stack")) throw Cancelled();
            }
        }
        c.span_end(span);
        c.check_kernel_error("stack kernel");
    } catch (...) {
        cudaStreamSynchronize(c.stream());
        dev.release();
        throw;
    }
    dev.release();
}

}  // namespace

void stack_pass_device(Context& c, const float* d_frames, int pitch, int w, int h, int n, const int* dx,
                       const int* dy, int m, int min_count, const double* vel, double tmax, float* d_max_snr,
                       int* d_best_v, const Progress& progress) {
    if (min_count > n) {
        // no pixel is covered by min_count frames for any motion: every S/N is
        // undefined, so max_snr is 0 and best_v -1 everywhere (the kernel's
        // interior tiles take c = n without testing min_count)
        fill_undefined_maps(d_max_snr, d_best_v, static_cast<size_t>(w) * h, c.stream());
        FTB_CHECK(cudaStreamSynchronize(c.stream()));
        return;
    }
    const double t0 = wall_seconds();
    const StackConfig cfg = choose_stack_config(w, h, n, c.smem_optin());
    const std::vector<int> order = motion_order(dx, dy, m, n, 4.0, 4.0);
    (void)vel;
    (void)tmax;
    StackPlan plan = make_stack_plan(w, h, n, dx, dy, m, min_count, order, cfg);
    plan.pitch = pitch;
    c.host_time("setup", wall_seconds() - t0);
    run_plan(c, plan, d_frames, d_max_snr, d_best_v, progress);
}

void stack_pass_host(Context& c, const float* frames, int w, int h, int n, const int* dx, const int* dy, int m,
                     int min_count, const double* vel, double tmax, float* max_snr, int* best_v,
                     const Progress& progress) {
    c.bind();
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(w) * h;
    float* d_frames =
        c.scratch(kFrames, sizeof(float) * static_cast<size_t>(pitch) * h * n, "frames").as<float>();
    float* d_max = c.scratch(kMax, sizeof(float) * plane, "max_snr").as<float>();
    int* d_bv = c.scratch(kBestV, sizeof(int) * plane, "best_v").as<int>();
    c.timing_reset();
    const int up = c.span_begin("upload");
    FTB_CHECK(cudaMemcpy2DAsync(d_frames, sizeof(float) * pitch, frames, sizeof(float) * w, sizeof(float) * w,
                                static_cast<size_t>(h) * n, cudaMemcpyHostToDevice, c.stream()));
    c.span_end(up);
    stack_pass_device(c, d_frames, pitch, w, h, n, dx, dy, m, min_count, vel, tmax, d_max, d_bv, progress);
    const int down = c.span_begin("download");
    FTB_CHECK(cudaMemcpyAsync(max_snr, d_max, sizeof(float) * plane, cudaMemcpyDeviceToHost, c.stream()));
    FTB_CHECK(cudaMemcpyAsync(best_v, d_bv, sizeof(int) * plane, cudaMemcpyDeviceToHost, c.stream()));
    c.span_end(down);
    FTB_CHECK(cudaStreamSynchronize(c.stream()));
    c.timing_resolve();
}

// ------------------------------------------------------------------ stage

namespace {

// build_stage with the caller's frames and outputs in host memory (io_pitch =
// w) or device memory (rows io_pitch floats apart), copied to and from the
// stage's own layout around the device stage.
void stage_io(Context& c, const float* sub, bool on_device, int io_pitch, int w, int h, int n, const double* t_h,
              const StageParams& sp, float* filtered, float* static_sky, float* mask, double* sigma, int* cr) {
    c.bind();
    const int pitch = frame_pitch(w);
    const size_t plane = static_cast<size_t>(pitch) * h;
    const cudaMemcpyKind in_kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const cudaMemcpyKind out_kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const size_t io_row = sizeof(float) * static_cast<size_t>(io_pitch);
    c.timing_reset();
    float* d_sub = c.scratch(kFrames, sizeof(float) * plane * n, "frames").as<float>();
    float* d_filt = c.scratch(kStageOut, sizeof(float) * plane * n, "filtered frames").as<float>();
    float* d_sky = c.scratch(kSky, sizeof(float) * plane, "static sky").as<float>();
    float* d_mask = c.scratch(kMask, sizeof(float) * plane, "mask").as<float>();
    StageScratch sc(c, w, h, n, sp.fwhm_px);
    const int up = c.span_begin("upload");
    FTB_CHECK(cudaMemcpy2DAsync(d_sub, sizeof(float) * pitch, sub, io_row, sizeof(float) * w,
                                static_cast<size_t>(h) * n, in_kind, c.stream()));
    c.span_end(up);
    std::vector<double> sg(static_cast<size_t>(n));
    std::vector<int> crv(static_cast<size_t>(n));
    stage_run(c, sc, d_sub, w, h, n, t_h, sp, d_filt, d_sky, d_mask, sg.data(), crv.data());
    const int down = c.span_begin("download");
    if (filtered)
        FTB_CHECK(cudaMemcpy2DAsync(filtered, io_row, d_filt, sizeof(float) * pitch, sizeof(float) * w,
                                    static_cast<size_t>(h) * n, out_kind, c.stream()));
    if (static_sky)
        FTB_CHECK(cudaMemcpy2DAsync(static_sky, io_row, d_sky, sizeof(float) * pitch, sizeof(float) * w,
                                    static_cast<size_t>(h), out_kind, c.stream()));
    if (mask)
        FTB_CHECK(cudaMemcpy2DAsync(mask, io_row, d_mask, sizeof(float) * pitch, sizeof(float) * w,
                                    static_cast<size_t>(h), out_kind, c.stream()));
    c.span_end(down);
    FTB_CHECK(cudaStreamSynchronize(c.stream()));
    c.timing_resolve();
    if (sigma) std::copy(sg.begin(), sg.end(), sigma);
    if (cr) std::copy(crv.begin(), crv.end(), cr);
}

}  // namespace

void stage_host(Context& c, const float* sub, int w, int h, int n, const double* t_h, const StageParams& sp,
                float* filtered, float* static_sky, float* mask, double* sigma, int* cr) {
    stage_io(c, sub, false, w, w, h, n, t_h, sp, filtered, static_sky, mask, sigma, cr);
}

void stage_device(Context& c, const float* d_sub, int pitch, int w, int h, int n, const double* t_h,
                  const StageParams& sp, float* d_filtered, float* d_static_sky, float* d_mask, double* sigma,
                  int* cr) {
    stage_io(c, d_sub, true, pitch, w, h, n, t_h, sp, d_filtered, d_static_sky, d_mask, sigma, cr);
}

// ------------------------------------------------------------------ tile-shape autotuner

namespace {

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int>, int> g_tuned;  // (frames, motions, width, height) -> shape

// Passes below this many adds keep the frame-count rule: a probe would cost
// more than a better shape can save.
constexpr double kTuneMinAdds = 5e11;

// The tile shape for a pass: the cached choice for its (frames, motions, size),
// else, for a large pass, every shape whose windows fit is planned and timed on a
// band of tile rows in the middle of the image (about 8 tiles per SM, so each
// probe is a few per cent of the pass), and the fastest per output pixel wins.
// The probes write the pass's own output maps, which its real launch rewrites.
// Returns 0 for "use the frame-count rule".
int autotune_shape(Context& c, const PassJob& j) {
    if (stack_shape() != 0) return 0;  // a fixed shape was asked for
    if (static_cast<double>(j.m) * j.n * j.w * j.h < kTuneMinAdds) return 0;
    const auto key = std::make_tuple(j.n, j.m, j.w, j.h);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(key);
        if (it != g_tuned.end()) return it->second;
    }
    std::vector<int> cands;
    for (int s = 1; s <= kStackShapes; ++s)
        if (stack_shape_fits(stack_shape_config(s, c.smem_optin()), j.n)) cands.push_back(s);
    int best = cands.empty() ? 0 : cands[0];
    if (cands.size() > 1) {
        const double t0 = wall_seconds();
        double best_t = 1e300;
        cudaEvent_t e0, e1;
        FTB_CHECK(cudaEventCreate(&e0));
        FTB_CHECK(cudaEventCreate(&e1));
        try {
            const std::vector<int> order = motion_order(j.dx.data(), j.dy.data(), j.m, j.n, 4.0, 4.0);
            for (int s : cands) {
                const StackConfig cfg = stack_shape_config(s, c.smem_optin());
                StackPlan plan = make_stack_plan(j.w, j.h, j.n, j.dx.data(), j.dy.data(), j.m, j.min_count, order, cfg);
                plan.pitch = j.pitch;
                StackPlanDev dev;
                dev.upload(plan, c.stream());
                const int tiles_x = (j.w + cfg.tile_w - 1) / cfg.tile_w, tiles_y = (j.h + cfg.p - 1) / cfg.p;
                const int band = std::min(tiles_y, std::max(1, (8 * c.sms() + tiles_x - 1) / tiles_x));
                BatchPass bp;
                bp.plan = &plan;
                bp.dev = &dev;
                bp.frames = j.d_frames;
                bp.g0 = 0;
                bp.g1 = static_cast<int>(plan.groups.size());
                bp.max_snr = j.d_max;
                bp.best_v = j.d_bv;
                bp.tile_rows0 = (tiles_y - band) / 2;
                bp.tile_rows = band;
                DevBuf& desc = c.scratch(kDesc, batch_desc_bytes(1), "stack descriptors");
                FTB_CHECK(cudaEventRecord(e0, c.stream()));
                stack_launch_batch({bp}, desc.as<unsigned char>(), desc.bytes(), c.err_flag(), c.sms(), c.stream());
                FTB_CHECK(cudaEventRecord(e1, c.stream()));
                ++c.launches;
                c.check_kernel_error("stack kernel (autotune probe)");
                float ms = 0.0f;
                FTB_CHECK(cudaEventElapsedTime(&ms, e0, e1));
                dev.release();
                const double per_px = ms / (static_cast<double>(band) * cfg.p * j.w);
                if (per_px < best_t) {
                    best_t = per_px;
                    best = s;
                }
            }
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        c.host_time("autotune", wall_seconds() - t0);
    }
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned[key] = best;
    return best;
}

}  // namespace

std::vector<std::pair<std::array<int, 4>, int>> tuned_shapes() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    std::vector<std::pair<std::array<int, 4>, int>> out;
    for (const auto& kv : g_tuned)
        out.push_back({{std::get<0>(kv.first), std::get<1>(kv.first), std::get<2>(kv.first), std::get<3>(kv.first)},
                       kv.second});
    return out;
}

void clear_tuned_shapes() {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    g_tuned.clear();
}

// ------------------------------------------------------------------ batched passes

namespace {

// The configuration a pass takes when no probe has to run first: a fixed
// shape, the autotuner's cached choice, or the frame-count rule for a pass too
// small to tune. False when the autotuner still has to time the pass's kind.
bool known_config(const Context& c, const PassJob& j, StackConfig& cfg) {
    int shape = 0;
    if (stack_shape() == 0 && static_cast<double>(j.m) * j.n * j.w * j.h >= kTuneMinAdds) {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tuned.find(std::make_tuple(j.n, j.m, j.w, j.h));
        if (it == g_tuned.end()) return false;
        shape = it->second;
    }
    cfg = shape > 0 ? stack_shape_config(shape, c.smem_optin()) : choose_stack_config(j.w, j.h, j.n, c.smem_optin());
    return true;
}

bool same_config(const StackConfig& a, const StackConfig& b) {
    return a.ty == b.ty && a.p == b.p && a.tile_w == b.tile_w && a.wp == b.wp && a.merge == b.merge &&
           a.rows == b.rows && a.smem_bytes == b.smem_bytes;
}

}  // namespace

PlanAhead plan_ahead(Context& c, std::vector<PassJob> tables) {
    PlanAhead out;
    out.plans.resize(tables.size());
    auto jobs = std::make_shared<std::vector<PassJob>>(std::move(tables));
    auto cfgs = std::make_shared<std::vector<StackConfig>>(jobs->size());
    auto promises = std::make_shared<std::vector<std::promise<StackPlan>>>();
    std::vector<size_t> todo;
    for (size_t k = 0; k < jobs->size(); ++k)
        if ((*jobs)[k].min_count <= (*jobs)[k].n && known_config(c, (*jobs)[k], (*cfgs)[k])) todo.push_back(k);
    promises->resize(todo.size());
    for (size_t q = 0; q < todo.size(); ++q) out.plans[todo[q]] = (*promises)[q].get_future().share();
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t workers = std::min<size_t>(hw, todo.size());
    for (size_t wkr = 0; wkr < workers; ++wkr)
        std::thread([jobs, cfgs, promises, todo, wkr, workers] {
            for (size_t q = wkr; q < todo.size(); q += workers) {
                const PassJob& j = (*jobs)[todo[q]];
                try {
                    StackPlan plan = make_stack_plan(j.w, j.h, j.n, j.dx.data(), j.dy.data(), j.m, j.min_count,
                                                     motion_order(j.dx.data(), j.dy.data(), j.m, j.n, 4.0, 4.0),
                                                     (*cfgs)[todo[q]]);
                    plan.pitch = j.pitch;
                    (*promises)[q].set_value(std::move(plan));
                } catch (...) {
                    (*promises)[q].set_exception(std::current_exception());
                }
            }
        }).detach();
    out.cfgs = *cfgs;
    return out;
}

void stack_passes_device(Context& c, std::vector<PassJob>& jobs, PlanAhead* ahead) {
    if (jobs.empty()) return;
    // a pass whose min_count exceeds its frame count (a search's min_coverage
    // above 1) defines no S/N anywhere: its maps are filled, not stacked
    if (std::any_of(jobs.begin(), jobs.end(), [](const PassJob& j) { return j.min_count > j.n; })) {
        std::vector<PassJob> rest;
        for (const PassJob& j : jobs) {
            if (j.min_count > j.n)
                fill_undefined_maps(j.d_max, j.d_bv, static_cast<size_t>(j.w) * j.h, c.stream());
            else
                rest.push_back(j);
        }
        stack_passes_device(c, rest);
        FTB_CHECK(cudaStreamSynchronize(c.stream()));
        return;
    }
    // tile shapes first (probes run on the stream, before this batch's launches)
    std::vector<int> shapes_for(jobs.size(), 0);
    for (size_t k = 0; k < jobs.size(); ++k) shapes_for[k] = autotune_shape(c, jobs[k]);
    const double t0 = wall_seconds();
    // plans on host threads (the GPU keeps running whatever was queued before)
    std::vector<StackPlan> plans(jobs.size());
    const unsigned hw = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
    const size_t workers = std::min<size_t>(hw, jobs.size());
    std::vector<std::thread> pool;
    std::vector<std::exception_ptr> errs(workers);
    for (size_t wkr = 0; wkr < workers; ++wkr)
        pool.emplace_back([&, wkr] {
            try {
                for (size_t k = wkr; k < jobs.size(); k += workers) {
                    const PassJob& j = jobs[k];
                    const StackConfig cfg = shapes_for[k] > 0 ? stack_shape_config(shapes_for[k], c.smem_optin())
                                                              : choose_stack_config(j.w, j.h, j.n, c.smem_optin());
                    // a plan made ahead for the same configuration (the tables are the job's)
                    if (ahead && k < ahead->plans.size() && ahead->plans[k].valid() &&
                        same_config(ahead->cfgs[k], cfg)) {
                        plans[k] = ahead->plans[k].get();
                        plans[k].pitch = j.pitch;
                        continue;
                    }
                    plans[k] = make_stack_plan(j.w, j.h, j.n, j.dx.data(), j.dy.data(), j.m, j.min_count,
                                               motion_order(j.dx.data(), j.dy.data(), j.m, j.n, 4.0, 4.0), cfg);
                    plans[k].pitch = j.pitch;
                }
            } catch (...) {
                errs[wkr] = std::current_exception();
            }
        });
    for (auto& t : pool) t.join();
    for (auto& e : errs)
        if (e) std::rethrow_exception(e);
    c.host_time("plans", wall_seconds() - t0);
    std::vector<StackPlanDev> devs(jobs.size());
    try {
        for (size_t k = 0; k < jobs.size(); ++k) devs[k].upload(plans[k], c.stream());
        // one persistent launch per kernel shape
        auto key = [](const StackConfig& q) { return std::make_pair((q.ty * 1000 + q.p) * 2 + q.merge, q.tile_w); };
        std::vector<std::pair<int, int>> shapes;
        for (const auto& p : plans)
            if (std::find(shapes.begin(), shapes.end(), key(p.cfg)) == shapes.end()) shapes.push_back(key(p.cfg));
        const int span = c.span_begin("kernel");
        for (const auto& sh : shapes) {
            std::vector<BatchPass> batch;
            for (size_t k = 0; k < jobs.size(); ++k) {
                if (key(plans[k].cfg) != sh) continue;
                BatchPass bp;
                bp.plan = &plans[k];
                bp.dev = &devs[k];
                bp.frames = jobs[k].d_frames;
                bp.g0 = 0;
                bp.g1 = static_cast<int>(plans[k].groups.size());
                bp.max_snr = jobs[k].d_max;
                bp.best_v = jobs[k].d_bv;
                batch.push_back(bp);
            }
            DevBuf& desc = c.scratch(kDesc, batch_desc_bytes(static_cast<int>(batch.size())), "stack descriptors");
            stack_launch_batch(batch, desc.as<unsigned char>(), desc.bytes(), c.err_flag(), c.sms(), c.stream());
            ++c.launches;
        }
        c.span_end(span);
        c.check_kernel_error("stack kernel");
    } catch (...) {
        cudaStreamSynchronize(c.stream());
        for (auto& d : devs) d.release();
        throw;
    }
    for (auto& d : devs) d.release();
}

}  // namespace ftb
