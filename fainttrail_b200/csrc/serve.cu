// The serving loop: search requests of any frame count, image size and motion
// range arrive at any time. At submit a request's frames are copied into HBM
// and stay resident there while it waits (as long as the resident stacks take
// at most half of the HBM budget; beyond that a request waits in host memory).
// Worker threads, each with its own context and stream, run steps: at every
// step a worker first admits queued requests whose estimated device memory fits
// what the admitted ones leave of the budget and prepares them (background,
// preprocessing, grid), then takes up to max_batch passes -- real passes, null
// runs with their rebuilt preprocessing -- from all its admitted requests in
// turn and stacks them together in persistent launches, and finally publishes
// every request whose passes are all done (peaks, artefact screen, threshold,
// candidates) and frees its memory. A request that arrives while others are on
// the GPU is admitted at the next step boundary, as memory frees up, and its
// passes share launches with theirs. Every result is bit-identical to the same
// search run alone.
#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>

#include "search.h"
#include "serve.h"

namespace ftb {

namespace {
double now_s() { return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count(); }
}  // namespace

struct Server::Req {
    long long id = 0;
    int w = 0, h = 0, n = 0;
    std::vector<float> frames;  // host copy, when the frames are not resident
    DevBuf resident;            // the frames in HBM (n x h x w), from submit until prepared
    std::vector<double> mjd, exptime;
    SearchParams p;
    double t_submit = 0, t_admit = 0, t_done = 0;
    bool done = false, failed = false;
    std::string error;
    SearchOut out;
    int runs() const { return p.threshold_snr <= 0.0 ? std::max(0, p.null_runs) : 0; }
    size_t item_bytes() const {
        const size_t plane = static_cast<size_t>(frame_pitch(w)) * h;
        return sizeof(float) * (plane * n + 2 * plane) + 8 * static_cast<size_t>(w) * h;
    }
    // device bytes while admitted: the prepared request and up to `items` passes in flight
    size_t bytes(int items) const {
        return SearchRequest::base_bytes(w, h, n) + static_cast<size_t>(std::min(runs(), items)) * item_bytes();
    }
};

// An admitted request on a worker: its search state and the next pass to stack.
struct Server::Active {
    std::shared_ptr<Req> r;
    std::unique_ptr<SearchRequest> s;
    int next = 0;
    bool real_staged = false;
    size_t reserved = 0;
};

Server::Server(int device, double budget_bytes, int max_batch, int workers) : max_batch_(std::max(1, max_batch)) {
    workers = std::max(1, std::min(workers, 8));
    // the first context resolves the device and the budget (default 90 % of free);
    // the others charge the same account, so every worker sees all allocations
    ctx_.push_back(std::make_unique<Context>(device, budget_bytes));
    for (int k = 1; k < workers; ++k)
        ctx_.push_back(std::make_unique<Context>(ctx_[0]->device(), ctx_[0]->account()));
    // the context of the uploads at submit (its own stream), charging the same account
    upload_ = std::make_unique<Context>(ctx_[0]->device(), ctx_[0]->account());
    for (auto& c : ctx_) {
        Context* cp = c.get();
        workers_.emplace_back([this, cp] { loop(*cp); });
    }
}

Server::~Server() {
    {
        std::lock_guard<std::mutex> lk(mu_);
        stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : workers_)
        if (t.joinable()) t.join();
}

long long Server::submit(const float* frames, int w, int h, int n, const double* mjd, const double* exptime,
                         const SearchParams& p) {
    if (!frames || !mjd || w < 1 || h < 1 || n < 1) throw std::runtime_error("submit: empty request");
    auto r = std::make_shared<Req>();
    r->w = w;
    r->h = h;
    r->n = n;
    const size_t bytes = sizeof(float) * static_cast<size_t>(w) * h * n;
    bool keep = false;
    {
        std::lock_guard<std::mutex> lk(mu_);
        if (resident_ + bytes <= upload_->budget() / 2) {
            resident_ += bytes;
            keep = true;
        }
    }
    if (keep) {
        // resident in HBM from now on; host memory if the device has no room after all
        try {
            std::lock_guard<std::mutex> ul(upload_mu_);
            upload_->bind();
            r->resident = DevBuf(upload_.get(), bytes, "resident frames");
            FTB_CHECK(cudaMemcpyAsync(r->resident.as<float>(), frames, bytes, cudaMemcpyHostToDevice,
                                      upload_->stream()));
            FTB_CHECK(cudaStreamSynchronize(upload_->stream()));
        } catch (const std::exception&) {
            r->resident.reset();
            std::lock_guard<std::mutex> lk(mu_);
            resident_ -= bytes;
            keep = false;
        }
    }
    if (!keep) r->frames.assign(frames, frames + static_cast<size_t>(w) * h * n);
    r->mjd.assign(mjd, mjd + n);
    if (exptime) r->exptime.assign(exptime, exptime + n);
    r->p = p;
    {
        std::lock_guard<std::mutex> lk(mu_);
        r->id = ++next_id_;
        r->t_submit = now_s();
        if (first_submit_ == 0) first_submit_ = r->t_submit;
        queue_.push_back(r);
        reqs_[r->id] = r;
    }
    cv_.notify_all();
    return r->id;
}

int Server::poll(long long id, int wait_ms, SearchOut* out, std::string* err) {
    std::unique_lock<std::mutex> lk(mu_);
    auto it = reqs_.find(id);
    if (it == reqs_.end()) {
        if (err) *err = "unknown request id " + std::to_string(id);
        return 1;
    }
    std::shared_ptr<Req> r = it->second;
    if (!r->done && wait_ms != 0) {
        auto pred = [&] { return r->done; };
        if (wait_ms < 0) done_cv_.wait(lk, pred);
        else done_cv_.wait_for(lk, std::chrono::milliseconds(wait_ms), pred);
    }
    if (!r->done) return 3;
    reqs_.erase(id);
    if (!r->error.empty()) {
        if (err) *err = r->error;
        return 1;
    }
    if (out) *out = std::move(r->out);
    return 0;
}

void Server::pause(bool paused) {
    {
        std::lock_guard<std::mutex> lk(mu_);
        paused_ = paused;
    }
    cv_.notify_all();
}

ServerStats Server::stats() {
    std::lock_guard<std::mutex> lk(mu_);
    ServerStats s;
    s.completed = static_cast<long long>(latencies_.size());
    if (!latencies_.empty()) {
        std::vector<double> v = latencies_;
        std::sort(v.begin(), v.end());
        // nearest-rank percentiles
        auto pct = [&](double q) {
            const size_t k = static_cast<size_t>(std::ceil(q * v.size()));
            return v[std::min(v.size(), std::max<size_t>(1, k)) - 1];
        };
        s.p50_s = pct(0.50);
        s.p99_s = pct(0.99);
        s.searches_per_s = last_done_ > first_submit_ ? s.completed / (last_done_ - first_submit_) : 0.0;
    }
    s.rounds = rounds_;
    s.launches = launches_;
    s.mean_batch = rounds_ ? static_cast<double>(batched_) / rounds_ : 0.0;
    return s;
}

void Server::loop(Context& c) {
    try {
        c.bind();
    } catch (...) {
    }
    std::vector<Active> active;
    for (;;) {
        std::vector<std::shared_ptr<Req>> admitted;
        {
            std::unique_lock<std::mutex> lk(mu_);
            ++idle_;
            cv_.wait(lk, [&] { return stop_ || !active.empty() || (!paused_ && !queue_.empty()); });
            --idle_;
            if (stop_ && active.empty() && (queue_.empty() || paused_)) break;
            // admission at every step: the oldest requests whose memory (prepared
            // request plus a step's passes) fits what the admitted ones leave of
            // the budget; a request is admitted alone when nothing else is
            // the queue is shared out among this worker and the idle ones (at least one each)
            const int share = static_cast<int>((queue_.size() + idle_) / (idle_ + 1));
            int taken = 0;
            while (!paused_ && !queue_.empty() && static_cast<int>(active.size() + admitted.size()) < max_batch_ &&
                   taken < share) {
                ++taken;
                const size_t need = queue_.front()->bytes(max_batch_);
                const size_t held = reserved_ + resident_;
                const bool alone = reserved_ == 0 && active.empty() && admitted.empty();
                if (held + need > c.budget() && !alone) break;
                reserved_ += need;
                admitted.push_back(queue_.front());
                admitted.back()->t_admit = now_s();
                queue_.pop_front();
            }
            if (active.empty() && admitted.empty()) {
                cv_.wait(lk);  // memory held by other workers: wait for a step to end
                continue;
            }
        }
        c.timing_reset();
        // prepare the admitted requests (frames from HBM where resident)
        for (auto& r : admitted) {
            Active a;
            a.r = r;
            a.reserved = r->bytes(max_batch_);
            try {
                a.s = std::make_unique<SearchRequest>(c, r->p, r->w, r->h, r->n);
                if (r->resident)
                    a.s->prepare(r->resident.as<float>(), r->mjd.data(), r->exptime.empty() ? nullptr : r->exptime.data(),
                                 true, r->w, false, {});
                else
                    a.s->prepare(r->frames.data(), r->mjd.data(), r->exptime.empty() ? nullptr : r->exptime.data(),
                                 false, 0, false, {});
                FTB_CHECK(cudaStreamSynchronize(c.stream()));
            } catch (const std::exception& e) {
                r->error = e.what();
                a.s.reset();
                cudaStreamSynchronize(c.stream());
            }
            release_frames(*r);
            active.push_back(std::move(a));
        }
        // one step: up to max_batch passes from the admitted requests in turn,
        // stacked together; each request's real pass goes with its first passes
        std::vector<PassJob> jobs;
        std::vector<std::array<int, 3>> ranges;  // (active index, k0, k1)
        int quota = max_batch_;
        const size_t margin = size_t{256} << 20;
        bool progress = true;
        std::vector<int> take(active.size(), 0);
        while (quota > 0 && progress) {  // round-robin, one pass per request per turn
            progress = false;
            for (size_t k = 0; k < active.size() && quota > 0; ++k) {
                Active& a = active[k];
                if (!a.s || a.next + take[k] >= a.s->runs()) continue;
                const size_t avail = c.budget() > c.used() + margin ? c.budget() - c.used() - margin : 0;
                if (take[k] + 1 > 1 && (static_cast<size_t>(take[k]) + 1) * a.s->item_bytes() > avail) continue;
                ++take[k];
                --quota;
                progress = true;
            }
        }
        int requests_in_step = 0;
        try {
            // every request's shift tables first, their plans made on host
            // threads while the GPU runs the step's preprocessing
            std::vector<size_t> at(active.size(), SearchRequest::kAppend);
            for (size_t k = 0; k < active.size(); ++k) {
                Active& a = active[k];
                if (!a.s || a.r->failed) continue;
                if (take[k] == 0 && a.real_staged) continue;
                at[k] = jobs.size();
                std::vector<PassJob> t = a.s->pass_tables(a.next, a.next + take[k]);
                for (auto& j : t) jobs.push_back(std::move(j));
            }
            PlanAhead ahead = plan_ahead(c, jobs);
            for (size_t k = 0; k < active.size(); ++k) {
                if (at[k] == SearchRequest::kAppend) continue;
                Active& a = active[k];
                a.s->stage_items(a.next, a.next + take[k], {}, jobs, at[k]);
                ranges.push_back({static_cast<int>(k), a.next, a.next + take[k]});
                a.real_staged = true;
                ++requests_in_step;
            }
            if (!jobs.empty()) stack_passes_device(c, jobs, &ahead);
            for (const auto& rg : ranges) {
                Active& a = active[static_cast<size_t>(rg[0])];
                a.s->finish_items(rg[1], rg[2]);
                a.next = rg[2];
            }
        } catch (const std::exception& e) {
            cudaStreamSynchronize(c.stream());
            for (const auto& rg : ranges) {
                Active& a = active[static_cast<size_t>(rg[0])];
                if (a.r->error.empty()) a.r->error = e.what();
                a.r->failed = true;
            }
        }
        // publish every request whose passes are all done (or that failed)
        std::vector<Active> keep;
        std::vector<std::shared_ptr<Req>> done;
        size_t freed = 0;
        for (auto& a : active) {
            const bool finished = !a.s || a.r->failed || (a.real_staged && a.next >= a.s->runs());
            if (!finished) {
                keep.push_back(std::move(a));
                continue;
            }
            if (a.s && !a.r->failed) {
                try {
                    a.r->out = a.s->finalize(nullptr);
                } catch (const std::exception& e) {
                    a.r->error = e.what();
                }
            }
            a.s.reset();
            cudaStreamSynchronize(c.stream());
            freed += a.reserved;
            done.push_back(a.r);
        }
        active.swap(keep);
        {
            std::lock_guard<std::mutex> lk(mu_);
            const double t = now_s();
            for (auto& r : done) {
                r->t_done = t;
                r->done = true;
                if (r->error.empty()) latencies_.push_back(r->t_done - r->t_submit);
            }
            if (!done.empty()) last_done_ = t;
            launches_ += c.launches;
            reserved_ -= freed;
            ++rounds_;
            batched_ += requests_in_step;
        }
        if (!done.empty()) done_cv_.notify_all();
        cv_.notify_all();  // memory freed or a step ended: a waiting worker may admit now
    }
}

void Server::release_frames(Req& r) {
    if (r.resident) {
        const size_t b = r.resident.bytes();
        {
            std::lock_guard<std::mutex> ul(upload_mu_);
            r.resident.reset();
        }
        std::lock_guard<std::mutex> lk(mu_);
        resident_ -= b;
    }
    r.frames.clear();
    r.frames.shrink_to_fit();
}

}  // namespace ftb
