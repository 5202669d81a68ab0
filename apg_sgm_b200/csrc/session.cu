// Reference-compatible session layer: the C API of include/apg_sgm/c_api.h on the CUDA engine.
//
// Follows src/c_api.cpp:10-204, StereoSession (include/apg_sgm/session.hpp:17-110) and
// StereoMatcher::compute_status (src/pipeline.cpp:337-397):
//   * validation order and messages of validate_inputs / validate_config (:171-232);
//   * the pre-compute budget gate: a frame whose workspace estimate exceeds max_retained_bytes
//     is rejected with RESOURCE_LIMIT_EXCEEDED before anything is allocated;
//   * ReleasePerFrame frees the device workspace after every frame (0 retained bytes);
//     BoundedReuse keeps it (capacity is retained when a smaller frame follows a larger one) and
//     re-checks the budget after the frame;
//   * frame_count / total_time_ms advance only on success; results are owned host copies.
#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/apg_sgm/c_api.h"
#include "../../include/apg_sgm_cuda.h"
#include "engine.h"

namespace {

struct Options {
    int memory_policy = APG_MEMORY_RELEASE_PER_FRAME;
    size_t max_retained_bytes = 0;
    int num_threads = 0;
    int backend = 0;
};

}  // namespace

struct apg_session_s {
    apg_pipeline_config_t cfg;
    Options opt;
    apgcu::Engine* eng = nullptr;
    std::string last_error;
    size_t frame_count = 0;
    double total_ms = 0.0;
    // workspace accounting (StereoWorkspace, include/apg_sgm/workspace.hpp:10-75)
    int last_w = 0, last_h = 0, last_dmax = 0;
    size_t frame_alloc = 0, frame_reuse = 0;
    double stage_ms[11] = {};
    unsigned long long counts[6] = {};  // Engine::frame_counts of the last frame
    double hier[6] = {};                 // Engine::hier_telemetry of the last frame
    int frame_w = 0, frame_h = 0;        // its size
    size_t peak_bytes = 0;
    std::vector<std::pair<std::string, int>> tuning;  // apgcu_session_set_tuning, applied every frame
    std::mutex mu;
    ~apg_session_s() { delete eng; }
};

// Result maps live in one page-locked host buffer owned by the result object and reused across
// frames, so the engine's device-to-host copies land in them directly.
struct apg_result_s {
    int w = 0, h = 0;
    bool has = false;
    float* disparity = nullptr;
    float* confidence = nullptr;
    uint8_t* invalid_reason = nullptr;
    uint8_t* reliable_mask = nullptr;
    unsigned char* buf = nullptr;
    size_t cap = 0;
    bool pinned = false;
    bool ensure(size_t n) {
        const size_t need = n * 10;
        if (cap < need) {
            release();
            void* p = nullptr;
            if (cudaMallocHost(&p, need) == cudaSuccess) {
                pinned = true;
            } else {
                cudaGetLastError();
                p = std::malloc(need);
                pinned = false;
                if (!p) return false;
            }
            buf = static_cast<unsigned char*>(p);
            cap = need;
        }
        disparity = reinterpret_cast<float*>(buf);
        confidence = disparity + n;
        invalid_reason = reinterpret_cast<uint8_t*>(confidence + n);
        reliable_mask = invalid_reason + n;
        return true;
    }
    void release() {
        if (buf) {
            if (pinned) cudaFreeHost(buf);
            else std::free(buf);
        }
        buf = nullptr;
        cap = 0;
    }
    void clear() {
        w = h = 0;
        has = false;
    }
    ~apg_result_s() { release(); }
};

namespace {

int validate_views(const apg_image_view_t* l, const apg_image_view_t* r, std::string& msg) {
    // validate_inputs, src/pipeline.cpp:215-232
    if (!l->data || !r->data || l->width <= 0 || l->height <= 0 || r->width <= 0 || r->height <= 0) {
        msg = (!l->data || !r->data) ? "empty input image(left or right)" : "image dimensions must be positive non-zero";
        return APG_STATUS_EMPTY_INPUT;
    }
    if (l->width != r->width || l->height != r->height) {
        msg = "left/right size mismatch (images must be rectified and aligned)";
        return APG_STATUS_SIZE_MISMATCH;
    }
    if (l->channels != r->channels) {
        msg = "left/right channel count mismatch";
        return APG_STATUS_SIZE_MISMATCH;
    }
    if (l->stride < l->width * l->channels || r->stride < r->width * r->channels) {
        msg = "invalid row stride (stride less than row byte length)";
        return APG_STATUS_SIZE_MISMATCH;
    }
    if (l->channels != 1 && l->channels != 3 && l->channels != 4) {
        msg = "unsupported channel count (1, 3 or 4)";
        return APG_STATUS_SIZE_MISMATCH;
    }
    if ((long long)l->width * l->height * l->channels >= (1ll << 31)) {
        msg = "image too large for the CUDA backend's 32-bit pixel indexing";
        return APG_STATUS_UNSUPPORTED_BACKEND;
    }
    return APG_STATUS_OK;
}

// Device workspace estimate used by the budget gate: the exact arena the engine would allocate
// plus the pinned staging buffers of the host copies.
size_t estimate_bytes(const apg_pipeline_config_t& cfg, int w, int h, int ch) {
    if (w <= 0 || h <= 0) return 0;
    const size_t n = (size_t)w * h;
    return apgcu::Engine::workspace_bytes(cfg, w, h, ch, 0) + 2 * n * ch + n * 10;
}

}  // namespace

extern "C" {

apg_session_t apg_session_create(int quality_mode, int memory_policy) {
    apg_session_options_t o = {};
    o.struct_size = (uint32_t)sizeof(apg_session_options_t);
    o.quality_mode = quality_mode;
    o.memory_policy = memory_policy;
    o.max_disparity = 128;
    return apg_session_create_ex(&o);
}

apg_session_t apg_session_create_ex(const apg_session_options_t* o) {
    if (!o) return nullptr;
    if (o->struct_size != 0 && o->struct_size != sizeof(apg_session_options_t)) return nullptr;
    try {
        int mode = APG_QUALITY_BALANCED;
        if (o->quality_mode == APG_QUALITY_FAST) mode = APG_QUALITY_FAST;
        else if (o->quality_mode == APG_QUALITY_HIGH_QUALITY) mode = APG_QUALITY_HIGH_QUALITY;
        const int max_disp = o->max_disparity > o->min_disparity ? o->max_disparity : 128;
        auto* s = new apg_session_s;
        s->cfg = apg_config_from_mode(mode, max_disp);
        s->cfg.min_disparity = o->min_disparity;
        s->cfg.max_disparity = max_disp;
        s->cfg.num_threads = o->num_threads;
        s->cfg.volume_backend = APG_BACKEND_CUDA;
        s->opt.memory_policy = o->memory_policy == APG_MEMORY_BOUNDED_REUSE ? APG_MEMORY_BOUNDED_REUSE
                                                                            : APG_MEMORY_RELEASE_PER_FRAME;
        s->opt.max_retained_bytes = o->max_retained_bytes;
        s->opt.num_threads = o->num_threads;
        s->opt.backend = o->backend;
        return s;
    } catch (...) {
        return nullptr;
    }
}

void apg_session_destroy(apg_session_t s) { delete s; }

void apg_session_reset(apg_session_t s) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->eng) s->eng->release();
    s->last_w = s->last_h = s->last_dmax = 0;
    s->frame_count = 0;
    s->total_ms = 0.0;
    s->last_error.clear();
}

apg_result_t apg_result_create(void) {
    try {
        return new apg_result_s;
    } catch (...) {
        return nullptr;
    }
}

void apg_result_destroy(apg_result_t r) { delete r; }

int apg_session_process(apg_session_t s, const apg_image_view_t* left, const apg_image_view_t* right,
                        apg_result_t result) {
    if (!s || !result) return APG_STATUS_INTERNAL_ERROR;
    if (!left || !right || !left->data || !right->data) {
        s->last_error = "Null input pointer";
        return APG_STATUS_EMPTY_INPUT;
    }
    std::lock_guard<std::mutex> lk(s->mu);
    try {
        const auto t0 = std::chrono::steady_clock::now();
        std::string msg;
        int rc = validate_views(left, right, msg);
        if (rc == APG_STATUS_OK) rc = apgcu::Engine::validate_config(s->cfg, msg);
        if (rc != APG_STATUS_OK) {
            result->clear();
            s->last_error = msg;
            return rc;
        }
        const int w = left->width, h = left->height, ch = left->channels;
        if (s->opt.max_retained_bytes > 0 && estimate_bytes(s->cfg, w, h, ch) > s->opt.max_retained_bytes) {
            result->clear();
            s->last_error = "workspace memory budget exceeded before compute";
            return APG_STATUS_RESOURCE_LIMIT_EXCEEDED;
        }
        int ndev = 0;
        if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
            cudaGetLastError();
            result->clear();
            s->last_error = "no CUDA device available for the CUDA backend";
            return APG_STATUS_UNSUPPORTED_BACKEND;
        }
        if (!s->eng) s->eng = new apgcu::Engine(s->cfg, 0, nullptr);
        for (const auto& kv : s->tuning) apgcu::set_tuning(s->eng, kv.first.c_str(), kv.second);
        const bool was_reuse = s->opt.memory_policy == APG_MEMORY_BOUNDED_REUSE && w == s->last_w && h == s->last_h &&
                               s->cfg.max_disparity == s->last_dmax && s->eng->allocated_bytes() > 0;
        const size_t n = (size_t)w * h;
        if (!result->ensure(n)) {
            result->clear();
            s->last_error = "Memory allocation failure";
            return APG_STATUS_ALLOCATION_FAILURE;
        }
        // the engine reads the two views with one common stride: repack only if they differ
        const uint8_t* lp = left->data;
        const uint8_t* rp = right->data;
        int stride = left->stride;
        std::vector<uint8_t> repack;
        if (left->stride != right->stride) {
            const size_t row = (size_t)w * ch;
            repack.resize(2 * row * h);
            for (int y = 0; y < h; ++y) {
                std::memcpy(repack.data() + y * row, left->data + (size_t)y * left->stride, row);
                std::memcpy(repack.data() + (h + y) * row, right->data + (size_t)y * right->stride, row);
            }
            lp = repack.data();
            rp = repack.data() + row * h;
            stride = (int)row;
        }
        rc = s->eng->process_host(lp, rp, w, h, stride, ch, result->disparity, result->confidence,
                                  result->invalid_reason, result->reliable_mask, result->pinned);
        if (rc == APG_STATUS_OK) rc = s->eng->frame_counts(s->counts);
        if (rc == APG_STATUS_OK) rc = s->eng->hier_telemetry(s->hier);
        if (rc != APG_STATUS_OK) {
            s->last_error = s->eng->last_error();
            result->clear();
            if (s->opt.memory_policy == APG_MEMORY_RELEASE_PER_FRAME) s->eng->release();
            return rc;
        }
        result->w = w;
        result->h = h;
        result->has = true;
        s->frame_w = w;
        s->frame_h = h;
        s->eng->stage_times(s->stage_ms);
        s->peak_bytes = std::max(s->peak_bytes, s->eng->allocated_bytes());
        if (was_reuse) ++s->frame_reuse;
        else ++s->frame_alloc;
        s->last_w = w;
        s->last_h = h;
        s->last_dmax = s->cfg.max_disparity;
        if (s->opt.memory_policy == APG_MEMORY_RELEASE_PER_FRAME) {
            s->eng->release();
            s->last_w = s->last_h = s->last_dmax = 0;
        } else if (s->opt.max_retained_bytes > 0 && s->eng->allocated_bytes() > s->opt.max_retained_bytes) {
            s->eng->release();
            result->clear();
            s->last_error = "workspace memory budget exceeded after compute";
            return APG_STATUS_RESOURCE_LIMIT_EXCEEDED;
        }
        const auto t1 = std::chrono::steady_clock::now();
        ++s->frame_count;
        s->total_ms += std::chrono::duration<double, std::milli>(t1 - t0).count();
        s->last_error.clear();
        return APG_STATUS_OK;
    } catch (const std::bad_alloc&) {
        s->last_error = "Memory allocation failure";
        return APG_STATUS_ALLOCATION_FAILURE;
    } catch (const std::exception& e) {
        s->last_error = e.what();
        return APG_STATUS_INTERNAL_ERROR;
    } catch (...) {
        s->last_error = "Unknown error";
        return APG_STATUS_INTERNAL_ERROR;
    }
}

#define APG_RESULT_GETTER(name, field, T)                                  \
    const T* name(apg_result_t r, int* width, int* height) {               \
        if (!r || !r->has) {                                               \
            if (width) *width = 0;                                         \
            if (height) *height = 0;                                       \
            return nullptr;                                                \
        }                                                                  \
        if (width) *width = r->w;                                          \
        if (height) *height = r->h;                                        \
        return r->field;                                                   \
    }
APG_RESULT_GETTER(apg_result_get_disparity, disparity, float)
APG_RESULT_GETTER(apg_result_get_confidence, confidence, float)
APG_RESULT_GETTER(apg_result_get_invalid_reason, invalid_reason, uint8_t)
APG_RESULT_GETTER(apg_result_get_reliable_mask, reliable_mask, uint8_t)
#undef APG_RESULT_GETTER

const char* apg_session_get_last_error(apg_session_t s) { return s ? s->last_error.c_str() : "Invalid session handle"; }

size_t apg_session_get_allocated_bytes(apg_session_t s) {
    if (!s) return 0;
    return s->eng ? s->eng->allocated_bytes() : 0;
}

size_t apg_session_get_frame_count(apg_session_t s) { return s ? s->frame_count : 0; }

double apg_session_get_total_time_ms(apg_session_t s) { return s ? s->total_ms : 0.0; }

const char* apg_status_string(int code) {
    // status_code_string, include/apg_sgm/status.hpp:56-69
    switch (code) {
        case 0: return "Ok";
        case 1: return "EmptyInput";
        case 2: return "SizeMismatch";
        case 3: return "InvalidDisparityRange";
        case 4: return "InvalidConfig";
        case 5: return "UnsupportedBackend";
        case 6: return "ResourceLimitExceeded";
        case 7: return "AllocationFailure";
        case 8: return "InternalError";
        default: return "Unknown";
    }
}

const char* apg_version_string(void) { return "1.0.0"; }

// ---- extensions (include/apg_sgm_cuda.h) ----

APGCU_API apg_session_t apgcu_session_create_config(const apg_pipeline_config_t* cfg, int memory_policy,
                                                    size_t max_retained_bytes) {
    if (!cfg) return nullptr;
    try {
        auto* s = new apg_session_s;
        s->cfg = *cfg;
        s->opt.memory_policy = memory_policy == APG_MEMORY_BOUNDED_REUSE ? APG_MEMORY_BOUNDED_REUSE
                                                                         : APG_MEMORY_RELEASE_PER_FRAME;
        s->opt.max_retained_bytes = max_retained_bytes;
        return s;
    } catch (...) {
        return nullptr;
    }
}

APGCU_API int apgcu_session_get_stats(apg_session_t s, double* stage_ms11, size_t* counters4) {
    if (!s) return APG_STATUS_INTERNAL_ERROR;
    if (stage_ms11) std::memcpy(stage_ms11, s->stage_ms, sizeof(s->stage_ms));
    if (counters4) {
        counters4[0] = s->frame_alloc;
        counters4[1] = s->frame_reuse;
        counters4[2] = s->peak_bytes;
        counters4[3] = s->eng ? s->eng->allocated_bytes() : 0;
    }
    return APG_STATUS_OK;
}

APGCU_API int apgcu_session_set_tuning(apg_session_t s, const char* key, int value) {
    if (!s || !key) return APG_STATUS_INTERNAL_ERROR;
    std::lock_guard<std::mutex> lk(s->mu);
    const int rc = apgcu::set_tuning(nullptr, key, value);
    if (rc != APG_STATUS_OK) return rc;
    for (auto& kv : s->tuning) {
        if (kv.first == key) {
            kv.second = value;
            return APG_STATUS_OK;
        }
    }
    s->tuning.emplace_back(key, value);
    return APG_STATUS_OK;
}

APGCU_API int apgcu_session_hier_telemetry(apg_session_t s, double* out6) {
    if (!s || !out6) return APG_STATUS_INTERNAL_ERROR;
    std::memcpy(out6, s->hier, sizeof(s->hier));
    return APG_STATUS_OK;
}

APGCU_API int apgcu_session_get_frame_counts(apg_session_t s, unsigned long long* counts8) {
    if (!s || !counts8) return APG_STATUS_INTERNAL_ERROR;
    const unsigned long long* c = s->counts;
    const unsigned long long n = (unsigned long long)s->frame_w * (unsigned long long)s->frame_h;
    counts8[0] = c[0];                     // valid_pixels
    counts8[1] = c[1];                     // reliable_pixels
    counts8[2] = n >= c[1] ? n - c[1] : 0; // unreliable_pixels
    counts8[3] = c[3];                     // refine_changed_pixels
    counts8[4] = c[2];                     // lr_fail_pixels
    counts8[5] = c[5];                     // prior_support_count
    counts8[6] = c[4];                     // sum over pixels of the search range width
    // sum over pixels of the geometric width max(min(dmax, x+1) - dmin, 0) (src/pipeline.cpp:659-661)
    unsigned long long g = 0;
    for (int x = 0; x < s->frame_w; ++x) {
        const int hi = std::min(s->cfg.max_disparity, x + 1);
        g += hi > s->cfg.min_disparity ? (unsigned long long)(hi - s->cfg.min_disparity) : 0ull;
    }
    counts8[7] = g * (unsigned long long)s->frame_h;
    return APG_STATUS_OK;
}

APGCU_API size_t apgcu_session_estimate_bytes(apg_session_t s, int width, int height, int channels) {
    return s ? estimate_bytes(s->cfg, width, height, channels) : 0;
}

}  // extern "C"
