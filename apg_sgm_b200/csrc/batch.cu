// Batched form: many stereo pairs, of uneven sizes, per call.
//
// Pairs are grouped into buckets of equal (width, height, channels, max_disparity).  A bucket owns
// one engine (device workspace + stream) per pair slot.  A call runs, per bucket:
//   * every pair's phases before the SGM (aux, range, cost + cross-H + right argmin, cross-V) on
//     its own stream, so the pairs' kernels overlap on the device;
//   * ONE persistent SGM launch per phase for all the bucket's pairs (sgm_batch_kernel: warps pull
//     (pair, direction, scanline) units from a work queue), so the latency-bound sweeps of small
//     pairs fill the GPU together;
//   * every pair's phases after the SGM (confidence, LR, fill, median, frame counters) on its
//     stream again.
// The whole per-bucket sequence is captured once into a CUDA graph per (bucket, pair count) and
// replayed; inputs are copied into the slots' fixed input buffers before the replay and the
// outputs copied out after it.  Buckets run on their own streams, concurrently.
//
// Tuning (tile width of the cost kernel, lanes per SGM scanline, persistent-grid cap) is chosen
// per (W, D) bucket by an autotuner that times the candidates on the bucket's first pair and
// caches the winner (in memory, and in a text file when APGCU_TUNE_CACHE names one).
//
// Results are identical to processing each pair alone: every kernel of a pair reads and writes
// only that pair's workspace, and the batched SGM runs the same per-chain code.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <vector>

#include "../../include/apg_sgm_cuda.h"
#include "engine.h"
#include "kernels.h"

namespace apgcu {
namespace {

struct BucketKey {
    int w, h, ch, dmax;
    bool operator<(const BucketKey& o) const {
        if (w != o.w) return w < o.w;
        if (h != o.h) return h < o.h;
        if (ch != o.ch) return ch < o.ch;
        return dmax < o.dmax;
    }
};

struct Tuning {
    int sgm_lanes = 32;         // lanes per scanline chain (32 = one warp per scanline, 16 = half a warp)
    int max_blocks_per_sm = 0;  // cap of the persistent SGM grid (0 = occupancy limit)
    int cost_tile = 0;          // columns per block of the cost kernel (0 = the default for Dp)
};

struct Bucket {
    BucketKey key{};
    apg_pipeline_config_t cfg{};
    std::vector<std::unique_ptr<Engine>> slots;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr, sgm_done = nullptr;
    std::vector<cudaEvent_t> joined;
    std::map<int, SgmBatchPlan> plans;        // by pair count (graphs hold their device tables)
    std::map<int, cudaGraphExec_t> graphs;    // by pair count
    std::map<int, unsigned long long> graph_launches;  // kernels per replay
    cudaEvent_t done = nullptr;               // end of the bucket's last call (timing)
    Tuning tune;
    bool tuned = false;
    ExperimentalScope scope;  // the experimental scopes the bucket's plans and graphs were built under
};

// process-wide tuning cache, keyed "mode W H D"
std::mutex g_tune_mu;
std::map<std::string, Tuning> g_tune;
bool g_tune_loaded = false;

std::string tune_key(const apg_pipeline_config_t& c, const BucketKey& k) {
    std::ostringstream o;
    o << c.mode << " " << k.w << " " << k.h << " " << (c.max_disparity - c.min_disparity);
    return o.str();
}

void tune_load_locked() {
    if (g_tune_loaded) return;
    g_tune_loaded = true;
    const char* path = std::getenv("APGCU_TUNE_CACHE");
    if (!path) return;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        std::istringstream in(line);
        int mode, w, h, D;
        Tuning t;
        if (in >> mode >> w >> h >> D >> t.sgm_lanes >> t.max_blocks_per_sm >> t.cost_tile) {
            std::ostringstream k;
            k << mode << " " << w << " " << h << " " << D;
            g_tune[k.str()] = t;
        }
    }
}

void tune_store_locked(const std::string& key, const Tuning& t) {
    g_tune[key] = t;
    const char* path = std::getenv("APGCU_TUNE_CACHE");
    if (!path) return;
    std::ofstream f(path, std::ios::app);
    f << key << " " << t.sgm_lanes << " " << t.max_blocks_per_sm << " " << t.cost_tile << "\n";
}

}  // namespace

class Batch {
public:
    Batch(const apg_pipeline_config_t& cfg, int device) : cfg_(cfg), device_(device) {}
    ~Batch() { release(); }

    int process(int n, const apgcu_pair_t* pairs, bool device_buffers);
    int set_option(const char* key, int value);
    size_t allocated_bytes() const;
    float last_time_ms() const { return last_ms_; }
    void release();
    const std::string& last_error() const { return err_; }

private:
    int fail(int code, const std::string& m) {
        err_ = m;
        return code;
    }
    Bucket& bucket_for(const BucketKey& k);
    int ensure_slots(Bucket& b, int m);
    int ensure_plan(Bucket& b, int m);
    int enqueue(Bucket& b, int m, bool batched_sgm);
    int run_bucket(Bucket& b, int m, bool batched_sgm);
    int autotune(Bucket& b, const apgcu_pair_t& sample, bool device_buffers);

    apg_pipeline_config_t cfg_;
    int device_ = 0;
    bool use_graphs_ = true;
    bool use_batched_sgm_ = true;
    bool autotune_ = true;
    bool graph_capture_ = false;  // inside a capture: launches are counted at replay
    int forced_lanes_ = 0;
    int forced_max_blocks_ = -1;
    int forced_tile_ = -1;
    std::map<BucketKey, std::unique_ptr<Bucket>> buckets_;
    cudaStream_t start_stream_ = nullptr;
    cudaEvent_t start_ = nullptr;
    float last_ms_ = 0.f;
    std::string err_;
};

Bucket& Batch::bucket_for(const BucketKey& k) {
    auto it = buckets_.find(k);
    if (it != buckets_.end()) return *it->second;
    auto b = std::make_unique<Bucket>();
    b->key = k;
    b->cfg = cfg_;
    b->cfg.max_disparity = k.dmax;
    Bucket& ref = *b;
    buckets_[k] = std::move(b);
    return ref;
}

int Batch::ensure_slots(Bucket& b, int m) {
    if (!b.stream) {
        if (cudaStreamCreateWithFlags(&b.stream, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&b.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&b.sgm_done, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreate(&b.done) != cudaSuccess) {
            cudaGetLastError();
            return fail(kInternalError, "batch stream creation failed");
        }
    }
    while ((int)b.slots.size() < m) {
        std::unique_ptr<Engine> e;
        try {
            e = std::make_unique<Engine>(b.cfg, device_, nullptr);
        } catch (...) {
            return fail(kAllocationFailure, "engine creation failed");
        }
        e->set_sgm_lanes(b.tune.sgm_lanes);
        e->set_cost_tile(b.tune.cost_tile);
        b.slots.push_back(std::move(e));
        cudaEvent_t ev;
        if (cudaEventCreateWithFlags(&ev, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return fail(kInternalError, "batch event creation failed");
        }
        b.joined.push_back(ev);
    }
    return kOk;
}

// Forget the bucket's graphs and plans (after a tuning or option change).
void drop_plans(Bucket& b) {
    if (b.stream) cudaStreamSynchronize(b.stream);
    for (auto& g : b.graphs) cudaGraphExecDestroy(g.second);
    b.graphs.clear();
    for (auto& p : b.plans) sgm_batch_plan_destroy(&p.second);
    b.plans.clear();
}

int Batch::ensure_plan(Bucket& b, int m) {
    if (b.plans.count(m)) return kOk;
    std::vector<SgmLaunch> pl(m);
    std::vector<uint32_t*> sb;
    int nsbuf = 0;
    for (int k = 0; k < m; ++k) {
        uint32_t* s7[7];
        nsbuf = b.slots[k]->sgm_launch(&pl[k], s7);
        sb.insert(sb.end(), s7, s7 + nsbuf);
    }
    SgmBatchPlan plan;
    cudaError_t e = sgm_batch_plan_create(pl.data(), sb.data(), m, nsbuf, b.tune.sgm_lanes, &plan);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(kInternalError, std::string("batch plan: ") + cudaGetErrorString(e));
    }
    b.plans[m] = plan;
    return kOk;
}

// The bucket's work for its first m slots, enqueued on the slot streams joined to b.stream.
int Batch::enqueue(Bucket& b, int m, bool batched_sgm) {
    int rc = kOk;
    cudaEventRecord(b.fork, b.stream);
    for (int k = 0; k < m; ++k) {
        Engine& e = *b.slots[k];
        cudaStreamWaitEvent(e.stream(), b.fork, 0);
        rc = e.enqueue_pre();
        if (rc == kOk && !batched_sgm) rc = e.enqueue_sgm();
        if (rc == kOk && !batched_sgm) rc = e.enqueue_post();
        if (rc) return fail(rc, e.last_error());
        cudaEventRecord(b.joined[k], e.stream());
        cudaStreamWaitEvent(b.stream, b.joined[k], 0);
    }
    if (!batched_sgm) return kOk;
    cudaError_t ce = launch_sgm_batch(b.plans.at(m), b.tune.max_blocks_per_sm, b.stream);
    if (!graph_capture_) count_launches(2);
    if (ce != cudaSuccess) return fail(kInternalError, std::string("batched SGM: ") + cudaGetErrorString(ce));
    cudaEventRecord(b.sgm_done, b.stream);
    for (int k = 0; k < m; ++k) {
        Engine& e = *b.slots[k];
        cudaStreamWaitEvent(e.stream(), b.sgm_done, 0);
        rc = e.enqueue_post();
        if (rc) return fail(rc, e.last_error());
        cudaEventRecord(b.joined[k], e.stream());
        cudaStreamWaitEvent(b.stream, b.joined[k], 0);
    }
    return kOk;
}

int Batch::run_bucket(Bucket& b, int m, bool batched_sgm) {
    // HighQuality refinement reads a counter back to the host between its passes: not capturable
    const bool graph = use_graphs_ && !b.slots[0]->refine_enabled();
    if (!graph) return enqueue(b, m, batched_sgm);
    auto it = b.graphs.find(m);
    if (it == b.graphs.end()) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(b.stream, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return enqueue(b, m, batched_sgm);
        }
        graph_capture_ = true;
        const unsigned long long before = launch_count();
        const int rc = enqueue(b, m, batched_sgm);
        const unsigned long long captured = launch_count() - before;
        const cudaError_t ce = cudaStreamEndCapture(b.stream, &g);
        graph_capture_ = false;
        if (rc != kOk || ce != cudaSuccess) {
            cudaGetLastError();
            if (g) cudaGraphDestroy(g);
            if (rc != kOk) return rc;
            return fail(kInternalError, std::string("batch graph capture: ") + cudaGetErrorString(ce));
        }
        cudaGraphExec_t ex = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (ie != cudaSuccess) {
            cudaGetLastError();
            return fail(kInternalError, std::string("batch graph instantiate: ") + cudaGetErrorString(ie));
        }
        it = b.graphs.emplace(m, ex).first;
        b.graph_launches[m] = captured + (batched_sgm ? 2 : 0);
        count_launches(0);
    } else {
        count_launches((unsigned)b.graph_launches[m]);
    }
    const cudaError_t le = cudaGraphLaunch(it->second, b.stream);
    if (le != cudaSuccess) return fail(kInternalError, std::string("batch graph launch: ") + cudaGetErrorString(le));
    return kOk;
}

// Times the candidate tunings on one pair of the bucket (a single-pair batch through the batched
// SGM) and keeps the fastest; the caches make this happen once per (mode, W, H, D).
int Batch::autotune(Bucket& b, const apgcu_pair_t& sample, bool device_buffers) {
    const std::string key = tune_key(b.cfg, b.key);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        tune_load_locked();
        auto it = g_tune.find(key);
        if (it != g_tune.end()) {
            b.tune = it->second;
            b.tuned = true;
            return kOk;
        }
    }
    const int Dp = round_up(b.key.dmax - b.cfg.min_disparity, 64);
    std::vector<Tuning> cand;
    const int alt_tile = Dp <= 128 ? 256 : 128;
    for (int tile : {0, alt_tile})
        for (int lanes : {32, 16})
            for (int mb : {0, 2}) {
                if (lanes == 16 && Dp > 256) continue;
                Tuning t;
                t.sgm_lanes = lanes;
                t.max_blocks_per_sm = mb;
                t.cost_tile = tile;
                cand.push_back(t);
            }
    int rc = ensure_slots(b, 1);
    if (rc) return rc;
    Engine& e = *b.slots[0];
    rc = e.upload(sample.left, sample.right, sample.width, sample.height, sample.stride, sample.channels,
                  device_buffers, b.stream);
    if (rc) return fail(rc, e.last_error());
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    float best_ms = 1e30f;
    Tuning best = cand[0];
    for (const Tuning& t : cand) {
        b.tune = t;
        e.set_sgm_lanes(t.sgm_lanes);
        e.set_cost_tile(t.cost_tile);
        drop_plans(b);
        rc = ensure_plan(b, 1);
        if (rc) break;
        rc = enqueue(b, 1, true);  // warm-up
        if (rc) break;
        cudaStreamSynchronize(b.stream);
        cudaEventRecord(t0, b.stream);
        for (int rep = 0; rep < 2 && rc == kOk; ++rep) rc = enqueue(b, 1, true);
        cudaEventRecord(t1, b.stream);
        cudaEventSynchronize(t1);
        float total = 0.f;
        if (cudaEventElapsedTime(&total, t0, t1) != cudaSuccess) {
            cudaGetLastError();
            total = 1e30f;
        }
        if (rc) break;
        if (std::getenv("APGCU_TUNE_LOG"))
            std::fprintf(stderr, "apgcu tune %s lanes %d max_blocks %d cost_tile %d: %.3f ms (2 runs, rc %d)\n",
                         key.c_str(), t.sgm_lanes, t.max_blocks_per_sm, t.cost_tile, total, rc);
        if (total < best_ms) {
            best_ms = total;
            best = t;
        }
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaStreamSynchronize(b.stream);
    if (rc) return rc;
    b.tune = best;
    b.tuned = true;
    for (auto& s : b.slots) {
        s->set_sgm_lanes(best.sgm_lanes);
        s->set_cost_tile(best.cost_tile);
    }
    drop_plans(b);
    std::lock_guard<std::mutex> lk(g_tune_mu);
    tune_store_locked(key, best);
    return kOk;
}

int Batch::process(int n, const apgcu_pair_t* pairs, bool device_buffers) {
    if (n < 0 || (n > 0 && !pairs)) return fail(kEmptyInput, "no pairs");
    cudaSetDevice(device_);
    err_.clear();
    // validation and bucketing
    std::map<BucketKey, std::vector<int>> groups;
    for (int i = 0; i < n; ++i) {
        const apgcu_pair_t& p = pairs[i];
        if (!p.left || !p.right || p.width <= 0 || p.height <= 0)
            return fail(kEmptyInput, "pair " + std::to_string(i) + ": empty input image(left or right)");
        if (p.channels != 1 && p.channels != 3 && p.channels != 4)
            return fail(kSizeMismatch, "pair " + std::to_string(i) + ": unsupported channel count (1, 3 or 4)");
        if (p.stride < p.width * p.channels)
            return fail(kSizeMismatch, "pair " + std::to_string(i) + ": invalid row stride (stride less than row byte length)");
        apg_pipeline_config_t c = cfg_;
        if (p.max_disparity > 0) c.max_disparity = p.max_disparity;
        std::string msg;
        const int rc = Engine::validate_config(c, msg);
        if (rc) return fail(rc, "pair " + std::to_string(i) + ": " + msg);
        groups[BucketKey{p.width, p.height, p.channels, c.max_disparity}].push_back(i);
    }
    // per bucket: tune (first time), upload, run (graph), download; every bucket stream starts
    // after one start event, so the call's device time is the latest bucket end minus it
    if (!start_stream_) {
        if (cudaStreamCreateWithFlags(&start_stream_, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreate(&start_) != cudaSuccess) {
            cudaGetLastError();
            return fail(kInternalError, "batch timing stream creation failed");
        }
    }
    for (auto& g : groups) {
        Bucket& b = bucket_for(g.first);
        if (b.tuned) continue;
        if (autotune_ && use_batched_sgm_) {
            const int rc = autotune(b, pairs[g.second[0]], device_buffers);
            if (rc) return rc;
        }
        b.tuned = true;
        if (forced_lanes_) b.tune.sgm_lanes = forced_lanes_;
        if (forced_max_blocks_ >= 0) b.tune.max_blocks_per_sm = forced_max_blocks_;
        if (forced_tile_ >= 0) b.tune.cost_tile = forced_tile_;
        for (auto& sl : b.slots) {
            sl->set_sgm_lanes(b.tune.sgm_lanes);
            sl->set_cost_tile(b.tune.cost_tile);
        }
        drop_plans(b);
    }
    cudaEventRecord(start_, start_stream_);
    std::vector<std::pair<Bucket*, const std::vector<int>*>> order;
    for (auto& g : groups) {
        Bucket& b = bucket_for(g.first);
        const std::vector<int>& idx = g.second;
        const int m = (int)idx.size();
        int rc = ensure_slots(b, m);
        if (rc) return rc;
        cudaStreamWaitEvent(b.stream, start_, 0);
        for (int k = 0; k < m; ++k) {
            const apgcu_pair_t& p = pairs[idx[k]];
            rc = b.slots[k]->upload(p.left, p.right, p.width, p.height, p.stride, p.channels, device_buffers, b.stream);
            if (rc) return fail(rc, b.slots[k]->last_error());
        }
        // plans and graphs hold the kernels' arguments, the experimental scopes among them: a call
        // under other scopes than the cached ones rebuilds them
        const ExperimentalScope cur = experimental_scope();
        if (!same_scope(cur, b.scope)) {
            drop_plans(b);
            b.scope = cur;
        }
        for (int k = 0; k < m; ++k) b.slots[k]->capture_scope();
        const int Dp = round_up(b.key.dmax - b.cfg.min_disparity, 64);
        SgmLaunch probe;
        uint32_t* s7[7];
        b.slots[0]->sgm_launch(&probe, s7);
        const bool batched = use_batched_sgm_ && sgm_batch_supported(Dp) && probe.cvol != nullptr;
        if (batched) {
            rc = ensure_plan(b, m);
            if (rc) return rc;
        }
        rc = run_bucket(b, m, batched);
        if (rc) return rc;
        for (int k = 0; k < m; ++k) {
            const apgcu_pair_t& p = pairs[idx[k]];
            rc = b.slots[k]->download(p.disparity, p.confidence, p.invalid_reason, p.reliable_mask, device_buffers,
                                      b.stream);
            if (rc) return fail(rc, b.slots[k]->last_error());
        }
        cudaEventRecord(b.done, b.stream);
        order.emplace_back(&b, &idx);
    }
    for (auto& o : order) {
        const cudaError_t e = cudaStreamSynchronize(o.first->stream);
        if (e != cudaSuccess) return fail(kInternalError, std::string("batch: ") + cudaGetErrorString(e));
        // the experimental scopes' telemetry of the bucket's pairs, into this thread's totals
        for (size_t k = 0; k < o.second->size(); ++k) {
            const int rc = o.first->slots[k]->collect_telemetry();
            if (rc) return fail(rc, o.first->slots[k]->last_error());
        }
    }
    last_ms_ = 0.f;
    for (auto& o : order) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, start_, o.first->done) == cudaSuccess) last_ms_ = std::max(last_ms_, ms);
        else cudaGetLastError();
    }
    if (!device_buffers) {
        for (auto& o : order) {
            for (size_t k = 0; k < o.second->size(); ++k) {
                const apgcu_pair_t& p = pairs[(*o.second)[k]];
                o.first->slots[k]->finish_download(p.disparity, p.confidence, p.invalid_reason, p.reliable_mask);
            }
        }
    }
    return kOk;
}

int Batch::set_option(const char* key, int value) {
    if (!key) return kInvalidConfig;
    const std::string k(key);
    if (k == "graphs") use_graphs_ = value != 0;
    else if (k == "batched_sgm") use_batched_sgm_ = value != 0;
    else if (k == "autotune") autotune_ = value != 0;
    else if (k == "sgm_lanes") {
        if (value != 0 && value != 16 && value != 32) return kInvalidConfig;
        forced_lanes_ = value;
    } else if (k == "cost_tile") {
        if (value != 0 && value != 64 && value != 128 && value != 256) return kInvalidConfig;
        forced_tile_ = value;
    } else if (k == "max_blocks_per_sm") {
        if (value < -1 || value > 64) return kInvalidConfig;
        forced_max_blocks_ = value;
    } else {
        return kInvalidConfig;
    }
    // a changed option invalidates plans, graphs and tunings
    for (auto& kv : buckets_) {
        drop_plans(*kv.second);
        kv.second->tuned = false;
    }
    return kOk;
}

size_t Batch::allocated_bytes() const {
    size_t t = 0;
    for (auto& kv : buckets_)
        for (auto& s : kv.second->slots) t += s->allocated_bytes();
    return t;
}

void Batch::release() {
    cudaSetDevice(device_);
    for (auto& kv : buckets_) {
        Bucket& b = *kv.second;
        drop_plans(b);
        b.slots.clear();
        for (auto ev : b.joined) cudaEventDestroy(ev);
        if (b.fork) cudaEventDestroy(b.fork);
        if (b.sgm_done) cudaEventDestroy(b.sgm_done);
        if (b.done) cudaEventDestroy(b.done);
        if (b.stream) cudaStreamDestroy(b.stream);
    }
    buckets_.clear();
    if (start_) cudaEventDestroy(start_);
    if (start_stream_) cudaStreamDestroy(start_stream_);
    start_ = nullptr;
    start_stream_ = nullptr;
}

}  // namespace apgcu

struct apgcu_batch_s {
    apgcu::Batch* b;
};

extern "C" {

APGCU_API apgcu_batch_t apgcu_batch_create(const apg_pipeline_config_t* cfg, int device) {
    if (!cfg) return nullptr;
    std::string msg;
    if (apgcu::Engine::validate_config(*cfg, msg) != 0) return nullptr;
    try {
        auto* h = new apgcu_batch_s;
        h->b = new apgcu::Batch(*cfg, device);
        return h;
    } catch (...) {
        return nullptr;
    }
}

APGCU_API void apgcu_batch_destroy(apgcu_batch_t b) {
    if (!b) return;
    delete b->b;
    delete b;
}

APGCU_API const char* apgcu_batch_last_error(apgcu_batch_t b) {
    return b ? b->b->last_error().c_str() : "Invalid batch handle";
}

APGCU_API int apgcu_batch_process(apgcu_batch_t b, int npairs, const apgcu_pair_t* pairs, int device_buffers) {
    if (!b) return APG_STATUS_INTERNAL_ERROR;
    try {
        return b->b->process(npairs, pairs, device_buffers != 0);
    } catch (...) {
        return APG_STATUS_INTERNAL_ERROR;
    }
}

APGCU_API int apgcu_batch_set_option(apgcu_batch_t b, const char* key, int value) {
    if (!b) return APG_STATUS_INTERNAL_ERROR;
    return b->b->set_option(key, value);
}

APGCU_API size_t apgcu_batch_allocated_bytes(apgcu_batch_t b) { return b ? b->b->allocated_bytes() : 0; }

APGCU_API float apgcu_batch_last_time_ms(apgcu_batch_t b) { return b ? b->b->last_time_ms() : 0.f; }

APGCU_API void apgcu_batch_release(apgcu_batch_t b) {
    if (b) b->b->release();
}

}  // extern "C"
