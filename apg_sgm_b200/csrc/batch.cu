// Batched form: many stereo pairs, of uneven sizes, per call.
//
// Pairs are grouped into buckets of equal (width, height, channels, max_disparity).  A bucket owns
// one engine (device workspace + stream) per pair slot.  A call runs:
//   * every pair's phases before the SGM (aux, range, cost + cross-H + right argmin, cross-V) on
//     its own stream, so the pairs' kernels overlap on the device;
//   * ONE persistent SGM launch per phase for the pairs of ALL buckets, whatever their sizes and
//     disparity ranges (sgm_batch_mixed_kernel: warps pull (pair, direction, scanline) units,
//     longest chains first, from one work queue, each unit running with its own pair's words per
//     lane), so the latency-bound sweeps of every pair fill the GPU together;
//   * every pair's phases after the SGM (confidence, LR, fill, median, frame counters) on its
//     stream again.
// The whole sequence is captured once into a CUDA graph per batch composition (the buckets and
// their pair counts) and replayed; inputs are copied into the slots' fixed input buffers before
// the replay and the outputs copied out after it.  The option "unified_sgm" 0 (or 16 lanes per
// chain from the tuner) runs each bucket on its own stream instead, with one SGM launch per phase
// per bucket, captured per (bucket, pair count).
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
    using Composition = std::vector<std::pair<BucketKey, int>>;  // buckets of a call and their pair counts
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
    // one SGM launch per phase over every bucket of the call
    struct Unified {
        SgmBatchPlan plan;
        cudaGraphExec_t graph = nullptr;
        unsigned long long launches = 0;  // kernels per replay
    };
    int ensure_unified_streams();
    int enqueue_unified(const Composition& comp, Unified& u);
    int run_unified(const Composition& comp);
    void drop_unified();

    apg_pipeline_config_t cfg_;
    int device_ = 0;
    bool use_graphs_ = true;
    bool use_batched_sgm_ = true;
    bool use_unified_ = true;
    bool autotune_ = true;
    bool graph_capture_ = false;  // inside a capture: launches are counted at replay
    int forced_lanes_ = 0;
    int forced_max_blocks_ = -1;
    int forced_tile_ = -1;
    std::map<BucketKey, std::unique_ptr<Bucket>> buckets_;
    std::map<Composition, Unified> unified_;
    cudaStream_t ustream_ = nullptr;  // the unified sequence's stream
    cudaEvent_t ufork_ = nullptr, usgm_done_ = nullptr, udone_ = nullptr;
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
        e->set_cost8(1);  // the batched SGM kernels read two-byte volumes
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

int Batch::ensure_unified_streams() {
    if (ustream_) return kOk;
    if (cudaStreamCreateWithFlags(&ustream_, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&ufork_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&usgm_done_, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&udone_, cudaEventDisableTiming) != cudaSuccess) {
        cudaGetLastError();
        return fail(kInternalError, "batch stream creation failed");
    }
    return kOk;
}

void Batch::drop_unified() {
    if (ustream_) cudaStreamSynchronize(ustream_);
    for (auto& kv : unified_) {
        if (kv.second.graph) cudaGraphExecDestroy(kv.second.graph);
        sgm_batch_plan_destroy(&kv.second.plan);
    }
    unified_.clear();
}

// Every bucket's pairs: pre-SGM phases on the slot streams, the two SGM launches on ustream_ over
// all pairs, post-SGM phases on the slot streams, everything joined back to ustream_.
int Batch::enqueue_unified(const Composition& comp, Unified& u) {
    cudaEventRecord(ufork_, ustream_);
    for (const auto& bm : comp) {
        Bucket& b = bucket_for(bm.first);
        for (int k = 0; k < bm.second; ++k) {
            Engine& e = *b.slots[k];
            cudaStreamWaitEvent(e.stream(), ufork_, 0);
            const int rc = e.enqueue_pre();
            if (rc) return fail(rc, e.last_error());
            cudaEventRecord(b.joined[k], e.stream());
            cudaStreamWaitEvent(ustream_, b.joined[k], 0);
        }
    }
    int max_blocks = forced_max_blocks_ >= 0 ? forced_max_blocks_ : 0;
    const cudaError_t ce = launch_sgm_batch(u.plan, max_blocks, ustream_);
    if (!graph_capture_) count_launches(2);
    if (ce != cudaSuccess) return fail(kInternalError, std::string("batched SGM: ") + cudaGetErrorString(ce));
    cudaEventRecord(usgm_done_, ustream_);
    for (const auto& bm : comp) {
        Bucket& b = bucket_for(bm.first);
        for (int k = 0; k < bm.second; ++k) {
            Engine& e = *b.slots[k];
            cudaStreamWaitEvent(e.stream(), usgm_done_, 0);
            const int rc = e.enqueue_post();
            if (rc) return fail(rc, e.last_error());
            cudaEventRecord(b.joined[k], e.stream());
            cudaStreamWaitEvent(ustream_, b.joined[k], 0);
        }
    }
    return kOk;
}

int Batch::run_unified(const Composition& comp) {
    auto it = unified_.find(comp);
    if (it == unified_.end()) {
        std::vector<SgmLaunch> pl;
        std::vector<uint32_t*> sb;
        int nsbuf = 0;
        for (const auto& bm : comp) {
            Bucket& b = bucket_for(bm.first);
            for (int k = 0; k < bm.second; ++k) {
                SgmLaunch l;
                uint32_t* s7[7];
                nsbuf = b.slots[k]->sgm_launch(&l, s7);
                pl.push_back(l);
                sb.insert(sb.end(), s7, s7 + nsbuf);
            }
        }
        Unified u;
        const cudaError_t e = sgm_batch_plan_create(pl.data(), sb.data(), (int)pl.size(), nsbuf, 32, &u.plan);
        if (e != cudaSuccess) {
            cudaGetLastError();
            return fail(kInternalError, std::string("batch plan: ") + cudaGetErrorString(e));
        }
        it = unified_.emplace(comp, u).first;
    }
    Unified& u = it->second;
    // HighQuality refinement is not captured (as in run_bucket)
    bool graph = use_graphs_;
    for (const auto& bm : comp)
        if (bucket_for(bm.first).slots[0]->refine_enabled()) graph = false;
    if (!graph) return enqueue_unified(comp, u);
    if (!u.graph) {
        cudaGraph_t g = nullptr;
        if (cudaStreamBeginCapture(ustream_, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            cudaGetLastError();
            return enqueue_unified(comp, u);
        }
        graph_capture_ = true;
        const unsigned long long before = launch_count();
        const int rc = enqueue_unified(comp, u);
        const unsigned long long captured = launch_count() - before;
        const cudaError_t ce = cudaStreamEndCapture(ustream_, &g);
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
        u.graph = ex;
        u.launches = captured + 2;
        count_launches(0);
    } else {
        count_launches((unsigned)u.launches);
    }
    const cudaError_t le = cudaGraphLaunch(u.graph, ustream_);
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
                // one launch serves every bucket: 32 lanes per chain, the occupancy-limited grid
                if (use_unified_ && (lanes != 32 || mb != 0)) continue;
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
        drop_unified();  // graphs of compositions with this bucket hold its old tuning
    }
    cudaEventRecord(start_, start_stream_);
    std::vector<std::pair<Bucket*, const std::vector<int>*>> order;
    std::vector<bool> batched_of;
    Composition comp;
    bool unified = use_unified_ && use_batched_sgm_;
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
            drop_unified();
            b.scope = cur;
        }
        for (int k = 0; k < m; ++k) b.slots[k]->capture_scope();
        const int Dp = round_up(b.key.dmax - b.cfg.min_disparity, 64);
        SgmLaunch probe;
        uint32_t* s7[7];
        b.slots[0]->sgm_launch(&probe, s7);
        const bool batched = use_batched_sgm_ && sgm_batch_supported(Dp) && probe.cvol != nullptr;
        if (!batched || b.tune.sgm_lanes != 32) unified = false;
        batched_of.push_back(batched);
        comp.emplace_back(g.first, m);
        order.emplace_back(&b, &idx);
    }
    if (unified) {
        int rc = ensure_unified_streams();
        if (rc) return rc;
        for (auto& o : order) {
            cudaEventRecord(o.first->fork, o.first->stream);  // the bucket's uploads are enqueued
            cudaStreamWaitEvent(ustream_, o.first->fork, 0);
        }
        rc = run_unified(comp);
        if (rc) return rc;
        cudaEventRecord(udone_, ustream_);
    }
    for (size_t bi = 0; bi < order.size(); ++bi) {
        Bucket& b = *order[bi].first;
        const std::vector<int>& idx = *order[bi].second;
        const int m = (int)idx.size();
        int rc = kOk;
        if (unified) {
            cudaStreamWaitEvent(b.stream, udone_, 0);
        } else {
            if (batched_of[bi]) {
                rc = ensure_plan(b, m);
                if (rc) return rc;
            }
            rc = run_bucket(b, m, batched_of[bi]);
            if (rc) return rc;
        }
        for (int k = 0; k < m; ++k) {
            const apgcu_pair_t& p = pairs[idx[k]];
            rc = b.slots[k]->download(p.disparity, p.confidence, p.invalid_reason, p.reliable_mask, device_buffers,
                                      b.stream);
            if (rc) return fail(rc, b.slots[k]->last_error());
        }
        cudaEventRecord(b.done, b.stream);
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
    else if (k == "unified_sgm") use_unified_ = value != 0;
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
    drop_unified();
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
    drop_unified();
    if (ufork_) cudaEventDestroy(ufork_);
    if (usgm_done_) cudaEventDestroy(usgm_done_);
    if (udone_) cudaEventDestroy(udone_);
    if (ustream_) cudaStreamDestroy(ustream_);
    ufork_ = usgm_done_ = udone_ = nullptr;
    ustream_ = nullptr;
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
