// The serving loop: search requests of any frame count, image size and motion
// range arrive at any time; a worker thread admits them by the HBM budget and
// runs them in rounds. A round prepares every admitted request (upload,
// background, preprocessing, grid), rebuilds all their null runs, and stacks the
// real and null passes of all of them together in persistent launches (one per
// kernel shape), so their work shares the device; then each request's peaks,
// artefact screen and threshold are finished and its result published. Requests
// that arrive during a round are admitted at the next one, as memory frees up.
// Every result is bit-identical to the same search run alone.
#include <algorithm>
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
    std::vector<float> frames;
    std::vector<double> mjd, exptime;
    SearchParams p;
    double t_submit = 0, t_done = 0;
    bool done = false;
    std::string error;
    SearchOut out;
    size_t bytes() const {
        const int runs = p.threshold_snr <= 0.0 ? std::max(0, p.null_runs) : 0;
        const size_t plane = static_cast<size_t>(frame_pitch(w)) * h;
        return SearchRequest::base_bytes(w, h, n) +
               static_cast<size_t>(runs) * (sizeof(float) * (plane * n + 2 * plane) + 8 * static_cast<size_t>(w) * h);
    }
};

Server::Server(int device, double budget_bytes, int max_batch, int workers) : max_batch_(std::max(1, max_batch)) {
    workers = std::max(1, std::min(workers, 8));
    // the first context resolves the device and the budget (default 90 % of free);
    // the others charge the same account, so every worker sees all allocations
    ctx_.push_back(std::make_unique<Context>(device, budget_bytes));
    for (int k = 1; k < workers; ++k)
        ctx_.push_back(std::make_unique<Context>(ctx_[0]->device(), ctx_[0]->account()));
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
    r->frames.assign(frames, frames + static_cast<size_t>(w) * h * n);
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
    for (;;) {
        std::vector<std::shared_ptr<Req>> round;
        size_t round_bytes = 0;
        {
            std::unique_lock<std::mutex> lk(mu_);
            ++idle_;
            cv_.wait(lk, [&] { return stop_ || (!paused_ && !queue_.empty()); });
            if (stop_ && (queue_.empty() || paused_)) {
                --idle_;
                break;
            }
            // admission: the oldest requests whose device memory fits what the
            // rounds in flight leave of the budget, the queue shared out among the
            // idle workers; a request is admitted alone when nothing else runs
            const int share = static_cast<int>((queue_.size() + idle_ - 1) / std::max(1, idle_));
            const int cap = std::max(1, std::min(max_batch_, share));
            const size_t budget = c.budget() > reserved_ ? c.budget() - reserved_ : 0;
            size_t need = 0;
            while (!queue_.empty() && static_cast<int>(round.size()) < cap) {
                const size_t b = queue_.front()->bytes();
                if (need + b > budget && !(round.empty() && reserved_ == 0)) break;
                need += b;
                round.push_back(queue_.front());
                queue_.pop_front();
            }
            if (round.empty()) {  // waits for a round in flight to end
                cv_.wait(lk);
                --idle_;
                continue;
            }
            --idle_;
            reserved_ += need;
            round_bytes = need;
        }
        run_round(c, round);
        {
            std::lock_guard<std::mutex> lk(mu_);
            const double t = now_s();
            for (auto& r : round) {
                r->t_done = t;
                r->done = true;
                if (r->error.empty()) latencies_.push_back(r->t_done - r->t_submit);
            }
            last_done_ = t;
            launches_ += c.launches;
            reserved_ -= round_bytes;
            ++rounds_;
            batched_ += static_cast<long long>(round.size());
        }
        done_cv_.notify_all();
        cv_.notify_all();  // memory freed: a waiting worker may admit now
    }
}

void Server::run_round(Context& c, std::vector<std::shared_ptr<Req>>& round) {
    c.timing_reset();
    std::vector<std::unique_ptr<SearchRequest>> rs(round.size());
    for (size_t k = 0; k < round.size(); ++k) {
        Req& r = *round[k];
        try {
            rs[k] = std::make_unique<SearchRequest>(c, r.p, r.w, r.h, r.n);
            rs[k]->prepare(r.frames.data(), r.mjd.data(), r.exptime.empty() ? nullptr : r.exptime.data(), false, 0,
                           false, {});
        } catch (const std::exception& e) {
            r.error = e.what();
            rs[k].reset();
            cudaStreamSynchronize(c.stream());
        }
    }
    try {
        if (round.size() == 1 && rs[0]) {
            // one request alone: its null runs in as many batches as the budget needs
            SearchRequest& s = *rs[0];
            const int items = s.runs();
            const size_t avail = c.budget() > c.used() + (size_t{256} << 20) ? c.budget() - c.used() - (size_t{256} << 20) : 0;
            const int per = static_cast<int>(std::max<size_t>(1, std::min<size_t>(std::max(items, 1), avail / s.item_bytes())));
            for (int k0 = 0; k0 < std::max(items, 1); k0 += per) {
                const int k1 = std::min(items, k0 + per);
                std::vector<PassJob> jobs;
                s.stage_items(k0, k1, {}, jobs);
                stack_passes_device(c, jobs);
                s.finish_items(k0, k1);
            }
        } else {
            std::vector<PassJob> jobs;
            for (auto& s : rs)
                if (s) s->stage_items(0, s->runs(), {}, jobs);
            stack_passes_device(c, jobs);  // every request's passes in shared launches
            for (auto& s : rs)
                if (s) s->finish_items(0, s->runs());
        }
        for (size_t k = 0; k < round.size(); ++k)
            if (rs[k]) round[k]->out = rs[k]->finalize(nullptr);
    } catch (const std::exception& e) {
        cudaStreamSynchronize(c.stream());
        for (size_t k = 0; k < round.size(); ++k)
            if (rs[k] && round[k]->error.empty()) round[k]->error = e.what();
    }
    rs.clear();
    for (auto& r : round) {
        r->frames.clear();
        r->frames.shrink_to_fit();
    }
}

}  // namespace ftb
