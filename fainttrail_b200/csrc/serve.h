// The serving loop (serve.cu): frames resident in HBM from submit, admission by
// the HBM budget at every step, and steps in which the passes of all admitted
// requests share persistent launches.
#pragma once

#include <condition_variable>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"
#include "search.h"

namespace ftb {

struct ServerStats {
    long long completed = 0, rounds = 0, launches = 0;
    double p50_s = 0, p99_s = 0, searches_per_s = 0, mean_batch = 0;
};

class Server {
public:
    // workers: steps in flight at once, each worker on its own stream charging
    // the one budget, so one step's host phases (plans, peak sorting, the
    // threshold fit) overlap another's kernels; max_batch: passes per step (and
    // requests admitted per worker)
    Server(int device, double budget_bytes, int max_batch, int workers = 2);
    ~Server();
    // copies the request's frames into HBM (host memory when the resident stacks
    // would take more than half the budget); returns its id
    long long submit(const float* frames, int w, int h, int n, const double* mjd, const double* exptime,
                     const SearchParams& p);
    // 0: done (out filled), 3: not done yet, 1: failed or unknown id (err filled).
    // wait_ms: 0 = do not wait, < 0 = wait until done.
    int poll(long long id, int wait_ms, SearchOut* out, std::string* err);
    void pause(bool paused);  // hold admission (requests queue up) or resume
    ServerStats stats();

private:
    struct Req;
    struct Active;
    void loop(Context& c);
    void release_frames(Req& r);
    std::vector<std::unique_ptr<Context>> ctx_;
    std::unique_ptr<Context> upload_;  // uploads at submit, on their own stream
    std::mutex upload_mu_;
    size_t resident_ = 0;  // bytes of frames held in HBM for requests not yet prepared
    int max_batch_ = 16, idle_ = 0;
    size_t reserved_ = 0;  // estimated device bytes of the admitted requests
    std::vector<std::thread> workers_;
    std::mutex mu_;
    std::condition_variable cv_, done_cv_;
    bool stop_ = false, paused_ = false;
    long long next_id_ = 0, rounds_ = 0, batched_ = 0, launches_ = 0;
    std::deque<std::shared_ptr<Req>> queue_;
    std::unordered_map<long long, std::shared_ptr<Req>> reqs_;
    std::vector<double> latencies_;
    double first_submit_ = 0, last_done_ = 0;
};

}  // namespace ftb
