// Served form: a request loop with continuous batching over device-resident workspaces.
//
// Requests (a stereo pair with its quality mode and disparity range) are queued in arrival order.
// A fixed number of worker threads -- the slots -- each take the next request, borrow an idle
// engine of the request's (mode, size, range) from the pool or create one, run the pair on that
// engine's own stream, and hand the engine back.  Requests that arrive while others are on the
// GPU are admitted as slots and memory free up, and their kernels overlap on the device.
//
// Admission is budgeted in HBM bytes: an engine's footprint is its workspace (cost volume, path
// buffers, 2-D planes; the exact arena the engine allocates).  Creating an engine reserves its
// footprint against the budget (min of the configured budget and the device's free memory at
// start); when the budget is full, idle engines of other buckets are released first, and only
// then does the request wait for running ones to return theirs.  Engines stay resident between
// requests (no per-request allocation in steady state).  A request larger than the whole budget
// fails with RESOURCE_LIMIT_EXCEEDED.
//
// Latency is the time from submission to completion (outputs on the host), measured with the
// host's steady clock.  Each result equals the single-pair engine's output for that pair.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/apg_sgm_cuda.h"
#include "engine.h"

namespace apgcu {
namespace {

using Clock = std::chrono::steady_clock;

struct PoolKey {
    int mode, w, h, ch, dmin, dmax;
    bool operator<(const PoolKey& o) const {
        const int a[6] = {mode, w, h, ch, dmin, dmax};
        const int b[6] = {o.mode, o.w, o.h, o.ch, o.dmin, o.dmax};
        return std::lexicographical_compare(a, a + 6, b, b + 6);
    }
};

struct Req {
    apgcu_request_t r{};
    Clock::time_point t_submit, t_done;
    int status = 0;
    bool done = false;
    std::string err;
};

struct Held {
    std::unique_ptr<Engine> eng;
    size_t bytes = 0;
};

}  // namespace

class Server {
public:
    Server(int device, size_t budget, int slots) : device_(device), slots_(std::max(1, slots)) {
        cudaSetDevice(device_);
        size_t free_b = 0, total_b = 0;
        if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
            cudaGetLastError();
            free_b = budget;
        }
        // leave room for the runtime and other users of the device
        const size_t margin = (size_t)2 << 30;
        const size_t avail = free_b > margin ? free_b - margin : 0;
        budget_ = std::min(budget, avail);
        for (int i = 0; i < slots_; ++i) workers_.emplace_back([this] { worker(); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
            // requests still queued never run: they complete now with an error, so that a thread
            // waiting for one returns
            for (const unsigned long long id : queue_) {
                Req& q = *reqs_.at(id);
                q.status = kInternalError;
                q.err = "server stopped before the request ran";
                q.t_done = Clock::now();
                q.done = true;
                ++failed_;
            }
            queue_.clear();
        }
        cv_done_.notify_all();
        cv_work_.notify_all();
        cv_mem_.notify_all();
        for (auto& t : workers_) t.join();
        {
            // threads inside wait() leave before the members they read go away
            std::unique_lock<std::mutex> lk(mu_);
            cv_done_.wait(lk, [&] { return waiters_ == 0; });
        }
        cudaSetDevice(device_);
        idle_.clear();
    }

    int submit(const apgcu_request_t& r, unsigned long long* ticket) {
        if (!r.left || !r.right || r.width <= 0 || r.height <= 0) return kEmptyInput;
        if (r.channels != 1 && r.channels != 3 && r.channels != 4) return kSizeMismatch;
        if (r.stride < r.width * r.channels) return kSizeMismatch;
        auto q = std::make_unique<Req>();
        q->r = r;
        q->t_submit = Clock::now();
        std::lock_guard<std::mutex> lk(mu_);
        const unsigned long long id = ++next_id_;
        queue_.push_back(id);
        reqs_[id] = std::move(q);
        *ticket = id;
        cv_work_.notify_one();
        return kOk;
    }

    int wait(unsigned long long id, double* latency_ms) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) return fail_locked(kInternalError, "unknown ticket");
        ++waiters_;
        cv_done_.wait(lk, [&] { return it->second->done; });
        Req& q = *it->second;
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(q.t_done - q.t_submit).count();
        const int st = q.status;
        if (st) err_ = q.err;
        reqs_.erase(it);
        --waiters_;
        cv_done_.notify_all();
        return st;
    }

    void stats(unsigned long long* c4, size_t* b2) {
        std::lock_guard<std::mutex> lk(mu_);
        if (c4) {
            c4[0] = completed_;
            c4[1] = failed_;
            c4[2] = evictions_;
            c4[3] = peak_in_flight_;
        }
        if (b2) {
            b2[0] = reserved_;
            b2[1] = peak_reserved_;
        }
    }

    // Creates `count` idle engines for requests like `r` (its mode, size and range), each warmed by
    // one blank pair (workspace, staging and tables allocated, kernels loaded), so that the first
    // requests of a bucket do not pay for them.  Fails when the budget cannot hold them.
    int reserve(const apgcu_request_t& r, int count) {
        if (r.width <= 0 || r.height <= 0 || (r.channels != 1 && r.channels != 3 && r.channels != 4)) return kEmptyInput;
        const apg_pipeline_config_t c = config_of(r);
        std::string msg;
        int rc = Engine::validate_config(c, msg);
        if (rc) return rc;
        const PoolKey k{r.mode, r.width, r.height, r.channels, c.min_disparity, c.max_disparity};
        const size_t need = Engine::workspace_bytes(c, k.w, k.h, k.ch, 0);
        std::vector<uint8_t> blank((size_t)r.width * r.height * r.channels, 0);
        for (int i = 0; i < count; ++i) {
            {
                std::lock_guard<std::mutex> lk(mu_);
                if (reserved_ + need > budget_) return kResourceLimitExceeded;
                reserved_ += need;
                peak_reserved_ = std::max(peak_reserved_, reserved_);
            }
            Held h;
            h.bytes = need;
            cudaSetDevice(device_);
            try {
                h.eng = std::make_unique<Engine>(c, device_, nullptr);
                rc = h.eng->process_host(blank.data(), blank.data(), r.width, r.height, r.width * r.channels,
                                         r.channels, nullptr, nullptr, nullptr, nullptr);
            } catch (...) {
                rc = kAllocationFailure;
            }
            std::lock_guard<std::mutex> lk(mu_);
            if (rc) {
                reserved_ -= need;
                return rc;
            }
            idle_[k].push_back(std::move(h));
        }
        cv_mem_.notify_all();
        return kOk;
    }

    size_t budget() const { return budget_; }
    std::string last_error() {
        std::lock_guard<std::mutex> lk(mu_);
        return err_;
    }

private:
    int fail_locked(int code, const std::string& m) {
        err_ = m;
        return code;
    }

    static apg_pipeline_config_t config_of(const apgcu_request_t& r) {
        apg_pipeline_config_t c = apg_config_from_mode(r.mode, r.max_disparity > 0 ? r.max_disparity : 128);
        c.min_disparity = r.min_disparity;
        return c;
    }

    // Under the lock: an engine for key k (idle one, or a new reservation), or nullptr with
    // *wait_mem set when the budget is full and nothing can be evicted yet.
    Held acquire_locked(const PoolKey& k, const apg_pipeline_config_t& c, int* code, bool* wait_mem) {
        *wait_mem = false;
        *code = kOk;
        auto it = idle_.find(k);
        if (it != idle_.end() && !it->second.empty()) {
            Held h = std::move(it->second.back());
            it->second.pop_back();
            return h;
        }
        const size_t need = Engine::workspace_bytes(c, k.w, k.h, k.ch, 0);
        if (need > budget_) {
            *code = kResourceLimitExceeded;
            return Held();
        }
        // evict idle engines of other buckets until the reservation fits
        while (reserved_ + need > budget_) {
            bool evicted = false;
            for (auto& kv : idle_) {
                if (kv.second.empty()) continue;
                reserved_ -= kv.second.back().bytes;
                kv.second.pop_back();  // releases its device workspace
                ++evictions_;
                evicted = true;
                break;
            }
            if (!evicted) {
                *wait_mem = true;
                return Held();
            }
        }
        reserved_ += need;
        peak_reserved_ = std::max(peak_reserved_, reserved_);
        Held h;
        h.bytes = need;
        return h;  // engine created by the caller, outside the lock
    }

    void worker() {
        cudaSetDevice(device_);
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            cv_work_.wait(lk, [&] { return stop_ || !queue_.empty(); });
            if (stop_) return;
            const unsigned long long id = queue_.front();
            queue_.pop_front();
            Req* q = reqs_.at(id).get();
            const apgcu_request_t r = q->r;
            const apg_pipeline_config_t c = config_of(r);
            std::string msg;
            int rc = Engine::validate_config(c, msg);
            Held h;
            if (rc == kOk) {
                const PoolKey k{r.mode, r.width, r.height, r.channels, c.min_disparity, c.max_disparity};
                bool stopped = false;
                for (;;) {
                    bool wait_mem = false;
                    h = acquire_locked(k, c, &rc, &wait_mem);
                    if (!wait_mem) break;
                    if (stop_) {
                        stopped = true;  // no reservation was made: the request fails
                        break;
                    }
                    cv_mem_.wait(lk);
                }
                if (stopped) {
                    rc = kInternalError;
                    msg = "server stopped while the request waited for device memory";
                } else if (rc == kResourceLimitExceeded) {
                    msg = "request workspace exceeds the HBM admission budget";
                }
            }
            ++in_flight_;
            peak_in_flight_ = std::max(peak_in_flight_, (unsigned long long)in_flight_);
            lk.unlock();
            if (rc == kOk && !h.eng) {
                try {
                    h.eng = std::make_unique<Engine>(c, device_, nullptr);
                } catch (...) {
                    rc = kAllocationFailure;
                    msg = "engine creation failed";
                }
            }
            if (rc == kOk) {
                rc = h.eng->process_host(r.left, r.right, r.width, r.height, r.stride, r.channels, r.disparity,
                                         r.confidence, r.invalid_reason, r.reliable_mask);
                if (rc) msg = h.eng->last_error();
            }
            const PoolKey k{r.mode, r.width, r.height, r.channels, c.min_disparity, c.max_disparity};
            lk.lock();
            --in_flight_;
            if (h.eng) {
                if (rc == kOk) idle_[k].push_back(std::move(h));
                else reserved_ -= h.bytes;  // a failed engine is dropped
            } else if (h.bytes) {
                reserved_ -= h.bytes;
            }
            q->status = rc;
            q->err = msg;
            q->t_done = Clock::now();
            q->done = true;
            if (rc == kOk) ++completed_;
            else ++failed_;
            cv_done_.notify_all();
            cv_mem_.notify_all();
        }
    }

    int device_;
    int slots_;
    size_t budget_ = 0;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_, cv_mem_;
    std::deque<unsigned long long> queue_;
    std::map<unsigned long long, std::unique_ptr<Req>> reqs_;
    std::map<PoolKey, std::vector<Held>> idle_;
    std::vector<std::thread> workers_;
    unsigned long long next_id_ = 0, completed_ = 0, failed_ = 0, evictions_ = 0, peak_in_flight_ = 0;
    int in_flight_ = 0;
    int waiters_ = 0;  // threads inside wait()
    size_t reserved_ = 0, peak_reserved_ = 0;
    bool stop_ = false;
    std::string err_;
};

}  // namespace apgcu

struct apgcu_server_s {
    apgcu::Server* s;
};

extern "C" {

APGCU_API apgcu_server_t apgcu_server_create(int device, size_t hbm_budget_bytes, int slots) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
        cudaGetLastError();
        return nullptr;
    }
    try {
        auto* h = new apgcu_server_s;
        h->s = new apgcu::Server(device, hbm_budget_bytes, slots);
        return h;
    } catch (...) {
        return nullptr;
    }
}

APGCU_API void apgcu_server_destroy(apgcu_server_t s) {
    if (!s) return;
    delete s->s;
    delete s;
}

APGCU_API int apgcu_server_submit(apgcu_server_t s, const apgcu_request_t* r, unsigned long long* ticket) {
    if (!s || !r || !ticket) return APG_STATUS_INTERNAL_ERROR;
    try {
        return s->s->submit(*r, ticket);
    } catch (...) {
        return APG_STATUS_INTERNAL_ERROR;
    }
}

APGCU_API int apgcu_server_wait(apgcu_server_t s, unsigned long long ticket, double* latency_ms) {
    if (!s) return APG_STATUS_INTERNAL_ERROR;
    return s->s->wait(ticket, latency_ms);
}

APGCU_API int apgcu_server_stats(apgcu_server_t s, unsigned long long* counts4, size_t* bytes2) {
    if (!s) return APG_STATUS_INTERNAL_ERROR;
    s->s->stats(counts4, bytes2);
    return APG_STATUS_OK;
}

APGCU_API size_t apgcu_server_budget(apgcu_server_t s) { return s ? s->s->budget() : 0; }

APGCU_API int apgcu_server_reserve(apgcu_server_t s, const apgcu_request_t* like, int count) {
    if (!s || !like) return APG_STATUS_INTERNAL_ERROR;
    try {
        return s->s->reserve(*like, count);
    } catch (...) {
        return APG_STATUS_INTERNAL_ERROR;
    }
}

APGCU_API const char* apgcu_server_last_error(apgcu_server_t s) {
    static thread_local std::string tl;
    tl = s ? s->s->last_error() : std::string("Invalid server handle");
    return tl.c_str();
}

}  // extern "C"
