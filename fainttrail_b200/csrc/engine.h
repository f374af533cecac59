// Host engine of the B200 backend: device context, memory budget, and the
// search orchestration behind the C ABI (capi.cpp).
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <atomic>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <future>
#include <vector>

#include "ft_internal.h"

namespace ftb {

struct Cancelled : std::runtime_error {
    Cancelled() : std::runtime_error("cancelled") {}
};

// Progress callback in the reference's form: fraction, stage; false cancels.
using Progress = std::function<bool(double, const char*)>;

class Context;

// Device allocation charged against the context's HBM budget.
class DevBuf {
public:
    DevBuf() = default;
    DevBuf(Context* c, size_t bytes, const char* what);
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept { swap(o); }
    DevBuf& operator=(DevBuf&& o) noexcept {
        DevBuf t(std::move(o));
        swap(t);
        return *this;
    }
    ~DevBuf() { reset(); }
    void reset();
    void swap(DevBuf& o) noexcept {
        std::swap(ctx_, o.ctx_);
        std::swap(p_, o.p_);
        std::swap(bytes_, o.bytes_);
    }
    template <class T>
    T* as() const { return static_cast<T*>(p_); }
    size_t bytes() const { return bytes_; }
    explicit operator bool() const { return p_ != nullptr; }

private:
    Context* ctx_ = nullptr;
    void* p_ = nullptr;
    size_t bytes_ = 0;
};

// An HBM budget and what is charged against it; contexts on one device can
// share one (the server's workers), so each sees the others' allocations.
struct BudgetAccount {
    size_t budget = 0;
    std::atomic<size_t> used{0};
};

class Context {
public:
    Context(int device, double budget_bytes);
    // a context charging a shared account (its budget is the account's)
    Context(int device, std::shared_ptr<BudgetAccount> account);
    ~Context();
    int device() const { return device_; }
    cudaStream_t stream() const { return stream_; }
    int sms() const { return sms_; }
    int smem_optin() const { return smem_optin_; }
    const std::string& name() const { return name_; }
    double total_bytes() const { return total_; }
    size_t budget() const { return acct_->budget; }
    size_t used() const { return acct_->used.load(); }
    const std::shared_ptr<BudgetAccount>& account() const { return acct_; }
    void charge(size_t bytes, const char* what);
    void release(size_t bytes) { acct_->used -= bytes; }
    int* err_flag() const { return d_err_; }
    void check_kernel_error(const char* what);  // syncs the stream, reads the error flag
    void bind() const;                          // make the device current on this thread

    // reusable device buffers, grown on demand
    DevBuf& scratch(int slot, size_t bytes, const char* what);

    // Blocks freed by this context's DevBufs, kept by size for the next
    // allocation of the same size (in order on the context's stream), so that
    // repeated searches of one shape allocate nothing; at most kCacheBytes, and
    // no more than the budget leaves beside what is charged, are kept, all of
    // them are returned when an allocation fails, and a context whose budget
    // account is shared with others (the server's workers) keeps none.
    void* take_cached(size_t bytes);
    bool put_cached(void* p, size_t bytes);  // false: not kept (the caller frees it)
    void drop_cache();
    static constexpr size_t kCacheBytes = size_t{48} << 30;

    // stage timings of the last call: CUDA-event spans on the stream, or host time
    void timing_reset();
    int span_begin(const std::string& name);   // records a start event
    void span_end(int span);                    // records its end event
    void host_time(const std::string& name, double seconds);
    void timing_resolve();                      // after a stream sync: event spans -> seconds
    std::vector<std::pair<std::string, double>> timings;
    long long launches = 0;  // kernels launched by the last call (reset with the timings)

    std::string error;

private:
    int device_ = 0;
    cudaStream_t stream_ = nullptr;
    int sms_ = 0, smem_optin_ = 0;
    std::string name_;
    double total_ = 0;
    std::shared_ptr<BudgetAccount> acct_;
    void init(int device);
    int* d_err_ = nullptr;
    std::vector<DevBuf> scratch_;
    std::mutex cache_mu_;
    std::multimap<size_t, void*> cache_;
    size_t cached_ = 0;
    struct Span {
        std::string name;
        int a = -1, b = -1;
        double host = -1;
    };
    std::vector<Span> spans_;
    std::vector<cudaEvent_t> events_;
    int next_event_ = 0;
    int event();
};

// Wall-clock seconds since an arbitrary epoch (host stages).
double wall_seconds();

// One stacking pass over host frames (nframes x h x w) with a motion-major shift
// table; vel (2 m doubles) only guides the planner's motion order (may be null).
void stack_pass_host(Context& c, const float* frames, int w, int h, int n, const int* dx, const int* dy, int m,
                     int min_count, const double* vel, double tmax, float* max_snr, int* best_v,
                     const Progress& progress);

// The same over frames already on the device (n x h x pitch), results on the
// device; the split into launches follows the progress granularity.
void stack_pass_device(Context& c, const float* d_frames, int pitch, int w, int h, int n, const int* dx,
                       const int* dy, int m, int min_count, const double* vel, double tmax, float* d_max_snr,
                       int* d_best_v, const Progress& progress);

// One stacking pass of a batch: device frames (n x h x pitch), a motion-major
// shift table, device outputs (h x w).
struct PassJob {
    const float* d_frames = nullptr;
    int pitch = 0, w = 0, h = 0, n = 0;
    std::vector<int> dx, dy;
    int m = 0, min_count = 3;
    float* d_max = nullptr;
    int* d_bv = nullptr;
};

// Plans built ahead on host threads: a pass's plan depends only on its shift
// table, sizes and tile shape, so it can be made while the GPU still runs the
// work queued before the stacking (the null runs' preprocessing). A pass whose
// shape is not yet known (the autotuner has not timed its kind) gets none.
struct PlanAhead {
    std::vector<std::shared_future<StackPlan>> plans;  // per job; invalid: none
    std::vector<StackConfig> cfgs;                     // the configuration each plan is made for
};
PlanAhead plan_ahead(Context& c, std::vector<PassJob> tables);

// Several passes, possibly of different shapes: plans built on host threads (or
// taken from `ahead`, in the same job order), then one persistent launch per
// kernel shape; returns when all are complete.
void stack_passes_device(Context& c, std::vector<PassJob>& jobs, PlanAhead* ahead = nullptr);

// The tile-shape autotuner's cache: ((frames, motions, width, height), shape).
std::vector<std::pair<std::array<int, 4>, int>> tuned_shapes();
void clear_tuned_shapes();

struct StageParams;

// build_stage over host buffers (the C ABI's ft_b200_stage).
void stage_host(Context& c, const float* sub, int w, int h, int n, const double* t_h, const StageParams& sp,
                float* filtered, float* static_sky, float* mask, double* sigma, int* cr);
// The same over device buffers whose rows are `pitch` floats apart
// (ft_b200_stage_dev); sigma and cr are host arrays.
void stage_device(Context& c, const float* d_sub, int pitch, int w, int h, int n, const double* t_h,
                  const StageParams& sp, float* d_filtered, float* d_static_sky, float* d_mask, double* sigma,
                  int* cr);

}  // namespace ftb
