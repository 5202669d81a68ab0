// On-disk image formats (src/image.cpp:62-206) and a page-locked pair loader.
//
// Readers and writers follow the reference's formats byte for byte:
//   * load_image: binary PGM (P5, 1 channel) / PPM (P6, 3 channels), maxval 1..255; header tokens
//     are whitespace-separated, a token starting with '#' discards the rest of its line, and
//     exactly one byte follows the maxval before the samples;
//   * save_pgm (P5, maxval 255), save_pgm16 (P5, maxval 65535, big-endian, negatives as 0),
//     save_disparity_preview (d * 255 / dmax + 0.5 truncated, clamped; invalid -> 0);
//   * load_pfm / save_pfm: "Pf" (1 channel) or "PF" (3, channel 0 kept), rows bottom-up, a
//     positive scale means big-endian samples; '#' starts a comment anywhere in the header and
//     exactly one whitespace byte ends each header token.
// The loader reads pairs on worker threads into page-locked buffers that it recycles, so a
// server or engine takes them by DMA with no staging copy.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/apg_sgm_cuda.h"

namespace {

// Whole-file read (the formats are small and read once).
bool read_file(const char* path, std::vector<unsigned char>& buf) {
    FILE* f = std::fopen(path, "rb");
    if (!f) return false;
    buf.clear();
    unsigned char tmp[1 << 16];
    size_t n;
    while ((n = std::fread(tmp, 1, sizeof(tmp), f)) > 0) buf.insert(buf.end(), tmp, tmp + n);
    const bool ok = !std::ferror(f);
    std::fclose(f);
    return ok;
}

bool write_file(const char* path, const std::string& head, const void* data, size_t bytes) {
    FILE* f = std::fopen(path, "wb");
    if (!f) return false;
    bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
    if (ok && bytes) ok = std::fwrite(data, 1, bytes, f) == bytes;
    ok = (std::fclose(f) == 0) && ok;
    return ok;
}

// Decimal integer token as std::stoi reads it (leading whitespace, sign, digits; the rest ignored);
// false where stoi would throw.
bool parse_int(const std::string& t, int* out) {
    errno = 0;
    char* end = nullptr;
    const long v = std::strtol(t.c_str(), &end, 10);
    if (end == t.c_str() || errno == ERANGE || v < INT32_MIN || v > INT32_MAX) return false;
    *out = (int)v;
    return true;
}

bool parse_float(const std::string& t, float* out) {
    errno = 0;
    char* end = nullptr;
    const float v = std::strtof(t.c_str(), &end);
    if (end == t.c_str() || errno == ERANGE) return false;
    *out = v;
    return true;
}

// PNM header (load_image's read_token: ">>" tokens, '#' tokens discard their line).
struct PnmHeader {
    int w = 0, h = 0, ch = 0;
    size_t data = 0;  // offset of the first sample
};

bool pnm_header(const std::vector<unsigned char>& b, PnmHeader* hd) {
    size_t p = 0;
    auto token = [&](std::string& tok) -> bool {
        for (;;) {
            while (p < b.size() && std::isspace(b[p])) ++p;
            if (p >= b.size()) return false;
            tok.clear();
            while (p < b.size() && !std::isspace(b[p])) tok.push_back((char)b[p++]);
            if (tok[0] == '#') {  // getline: the rest of the line, its newline included
                while (p < b.size() && b[p] != '\n') ++p;
                if (p < b.size()) ++p;
                continue;
            }
            return true;
        }
    };
    std::string magic, ws, hs, ms;
    if (!token(magic) || !token(ws) || !token(hs) || !token(ms)) return false;
    int w, h, mx;
    if (!parse_int(ws, &w) || !parse_int(hs, &h) || !parse_int(ms, &mx)) return false;
    if (w <= 0 || h <= 0 || mx <= 0 || mx > 255) return false;
    if (magic == "P5") hd->ch = 1;
    else if (magic == "P6") hd->ch = 3;
    else return false;
    if (p < b.size()) ++p;  // ifs.get(): one byte after the maxval
    hd->w = w;
    hd->h = h;
    hd->data = p;
    return true;
}

// PFM header (load_pfm's read_token: '#' comments anywhere, one whitespace byte after a token).
struct PfmHeader {
    int w = 0, h = 0, ch = 0;
    bool big_endian = false;
    size_t data = 0;
};

bool pfm_header(const std::vector<unsigned char>& b, PfmHeader* hd) {
    size_t p = 0;
    auto token = [&](std::string& tok) -> bool {
        tok.clear();
        while (p < b.size()) {
            const int c = b[p++];
            if (c == '#') {
                while (p < b.size() && b[p++] != '\n') {
                }
                continue;
            }
            if (!std::isspace(c)) {
                tok.push_back((char)c);
                break;
            }
        }
        if (tok.empty()) return false;
        while (p < b.size()) {
            const int c = b[p++];
            if (std::isspace(c)) break;
            tok.push_back((char)c);
        }
        return true;
    };
    std::string tag, ws, hs, ss;
    if (!token(tag) || !token(ws) || !token(hs) || !token(ss)) return false;
    if (tag != "Pf" && tag != "PF") return false;
    int w, h;
    float scale;
    if (!parse_int(ws, &w) || !parse_int(hs, &h) || !parse_float(ss, &scale)) return false;
    if (w <= 0 || h <= 0) return false;
    hd->w = w;
    hd->h = h;
    hd->ch = tag == "PF" ? 3 : 1;
    hd->big_endian = scale > 0.0f;
    hd->data = p;
    return true;
}

int status_of(bool ok) { return ok ? APG_STATUS_OK : APG_STATUS_INVALID_CONFIG; }

}  // namespace

extern "C" {

APGCU_API int apgcu_image_info(const char* path, int* width, int* height, int* channels) {
    std::vector<unsigned char> b;
    if (!path || !read_file(path, b)) return APG_STATUS_EMPTY_INPUT;
    PnmHeader hd;
    if (!pnm_header(b, &hd)) return APG_STATUS_INVALID_CONFIG;
    if (width) *width = hd.w;
    if (height) *height = hd.h;
    if (channels) *channels = hd.ch;
    return APG_STATUS_OK;
}

APGCU_API int apgcu_load_image(const char* path, uint8_t* dst, size_t dst_bytes, int* width, int* height,
                               int* channels) {
    std::vector<unsigned char> b;
    if (!path || !read_file(path, b)) return APG_STATUS_EMPTY_INPUT;
    PnmHeader hd;
    if (!pnm_header(b, &hd)) return APG_STATUS_INVALID_CONFIG;
    if (width) *width = hd.w;
    if (height) *height = hd.h;
    if (channels) *channels = hd.ch;
    const size_t need = (size_t)hd.w * hd.h * hd.ch;
    if (!dst || dst_bytes < need) return APG_STATUS_SIZE_MISMATCH;
    if (b.size() - std::min(b.size(), hd.data) < need) return APG_STATUS_INVALID_CONFIG;  // short file
    std::memcpy(dst, b.data() + hd.data, need);
    return APG_STATUS_OK;
}

APGCU_API int apgcu_save_pgm(const char* path, const uint8_t* img, int width, int height) {
    if (!path || !img || width <= 0 || height <= 0) return APG_STATUS_EMPTY_INPUT;
    const std::string head = "P5\n" + std::to_string(width) + " " + std::to_string(height) + "\n255\n";
    return status_of(write_file(path, head, img, (size_t)width * height));
}

APGCU_API int apgcu_save_pgm16(const char* path, const int16_t* disp, int width, int height) {
    if (!path || !disp || width < 0 || height < 0) return APG_STATUS_EMPTY_INPUT;
    const std::string head = "P5\n" + std::to_string(width) + " " + std::to_string(height) + "\n65535\n";
    const size_t n = (size_t)width * height;
    std::vector<uint8_t> raw(n * 2);
    for (size_t i = 0; i < n; ++i) {
        const int v = std::max(0, (int)disp[i]);
        raw[2 * i] = (uint8_t)(v >> 8);
        raw[2 * i + 1] = (uint8_t)(v & 0xff);
    }
    return status_of(write_file(path, head, raw.data(), raw.size()));
}

APGCU_API int apgcu_save_disparity_preview(const char* path, const float* disp, int width, int height, float dmax) {
    if (!path || !disp || width <= 0 || height <= 0) return APG_STATUS_EMPTY_INPUT;
    const size_t n = (size_t)width * height;
    std::vector<uint8_t> p(n);
    const float inv = dmax > 1.f ? 255.f / dmax : 1.f;
    for (size_t i = 0; i < n; ++i) {
        const float d = disp[i];
        if (d < 0.f) {
            p[i] = 0;
        } else {
            const int q = (int)(d * inv + 0.5f);
            p[i] = (uint8_t)std::min(std::max(q, 0), 255);
        }
    }
    return apgcu_save_pgm(path, p.data(), width, height);
}

APGCU_API int apgcu_pfm_info(const char* path, int* width, int* height, int* channels) {
    std::vector<unsigned char> b;
    if (!path || !read_file(path, b)) return APG_STATUS_EMPTY_INPUT;
    PfmHeader hd;
    if (!pfm_header(b, &hd)) return APG_STATUS_INVALID_CONFIG;
    if (width) *width = hd.w;
    if (height) *height = hd.h;
    if (channels) *channels = hd.ch;
    return APG_STATUS_OK;
}

APGCU_API int apgcu_load_pfm(const char* path, float* dst, size_t dst_floats, int* width, int* height) {
    std::vector<unsigned char> b;
    if (!path || !read_file(path, b)) return APG_STATUS_EMPTY_INPUT;
    PfmHeader hd;
    if (!pfm_header(b, &hd)) return APG_STATUS_INVALID_CONFIG;
    if (width) *width = hd.w;
    if (height) *height = hd.h;
    const size_t n = (size_t)hd.w * hd.h;
    if (!dst || dst_floats < n) return APG_STATUS_SIZE_MISMATCH;
    const size_t row = (size_t)hd.w * hd.ch * 4;
    if (b.size() - std::min(b.size(), hd.data) < row * hd.h) return APG_STATUS_INVALID_CONFIG;  // short file
    for (int r = 0; r < hd.h; ++r) {
        const unsigned char* src = b.data() + hd.data + (size_t)r * row;
        float* out = dst + (size_t)(hd.h - 1 - r) * hd.w;  // the first stored row is the bottom one
        for (int x = 0; x < hd.w; ++x) {
            uint32_t u;
            std::memcpy(&u, src + (size_t)x * hd.ch * 4, 4);
            if (hd.big_endian) u = __builtin_bswap32(u);
            std::memcpy(out + x, &u, 4);
        }
    }
    return APG_STATUS_OK;
}

APGCU_API int apgcu_save_pfm(const char* path, const float* img, int width, int height) {
    if (!path || !img || width <= 0 || height <= 0) return APG_STATUS_EMPTY_INPUT;
    const std::string head = "Pf\n" + std::to_string(width) + " " + std::to_string(height) + "\n-1.0\n";
    std::vector<float> rows((size_t)width * height);
    for (int y = height - 1, r = 0; y >= 0; --y, ++r)
        std::memcpy(rows.data() + (size_t)r * width, img + (size_t)y * width, (size_t)width * 4);
    return status_of(write_file(path, head, rows.data(), rows.size() * 4));
}

}  // extern "C"

// ------------------------------------------------------------------------------------------------
// Pair loader: worker threads read (left, right) files into recycled page-locked buffers.
// ------------------------------------------------------------------------------------------------
struct apgcu_loader_s {
    struct Job {
        unsigned long long id;
        std::string left, right;
    };
    struct Done {
        int status = 0;
        int w = 0, h = 0, ch = 0;
        uint8_t* buf = nullptr;  // left then right, page-locked
        size_t cap = 0;
    };
    std::mutex mu;
    std::condition_variable cv_job, cv_done;
    std::deque<Job> jobs;
    std::map<unsigned long long, Done> done;
    std::multimap<size_t, uint8_t*> free_bufs;  // capacity -> page-locked buffer
    std::vector<std::thread> workers;
    unsigned long long next_id = 1;
    size_t pinned_bytes = 0;
    bool stop = false;

    uint8_t* take_buffer(size_t need, size_t* cap) {
        std::lock_guard<std::mutex> lk(mu);
        auto it = free_bufs.lower_bound(need);
        if (it != free_bufs.end()) {
            uint8_t* p = it->second;
            *cap = it->first;
            free_bufs.erase(it);
            return p;
        }
        void* p = nullptr;
        if (cudaHostAlloc(&p, need, cudaHostAllocPortable) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        pinned_bytes += need;
        *cap = need;
        return static_cast<uint8_t*>(p);
    }

    void work() {
        for (;;) {
            Job j;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_job.wait(lk, [&] { return stop || !jobs.empty(); });
                if (stop && jobs.empty()) return;
                j = std::move(jobs.front());
                jobs.pop_front();
            }
            Done d;
            int lw = 0, lh = 0, lc = 0, rw = 0, rh = 0, rc = 0;
            d.status = apgcu_image_info(j.left.c_str(), &lw, &lh, &lc);
            if (d.status == 0) d.status = apgcu_image_info(j.right.c_str(), &rw, &rh, &rc);
            if (d.status == 0 && (lw != rw || lh != rh || lc != rc)) d.status = APG_STATUS_SIZE_MISMATCH;
            if (d.status == 0) {
                const size_t one = (size_t)lw * lh * lc;
                d.buf = take_buffer(2 * one, &d.cap);
                if (!d.buf) d.status = APG_STATUS_ALLOCATION_FAILURE;
                if (d.status == 0) d.status = apgcu_load_image(j.left.c_str(), d.buf, one, nullptr, nullptr, nullptr);
                if (d.status == 0)
                    d.status = apgcu_load_image(j.right.c_str(), d.buf + one, one, nullptr, nullptr, nullptr);
                d.w = lw;
                d.h = lh;
                d.ch = lc;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                done[j.id] = d;
            }
            cv_done.notify_all();
        }
    }
};

extern "C" {

APGCU_API apgcu_loader_t apgcu_loader_create(int threads) {
    try {
        auto* L = new apgcu_loader_s;
        const int n = std::max(1, threads);
        for (int i = 0; i < n; ++i) L->workers.emplace_back([L] { L->work(); });
        return L;
    } catch (...) {
        return nullptr;
    }
}

APGCU_API void apgcu_loader_destroy(apgcu_loader_t L) {
    if (!L) return;
    {
        std::lock_guard<std::mutex> lk(L->mu);
        L->stop = true;
    }
    L->cv_job.notify_all();
    for (auto& t : L->workers) t.join();
    for (auto& kv : L->free_bufs) cudaFreeHost(kv.second);
    for (auto& kv : L->done)
        if (kv.second.buf) cudaFreeHost(kv.second.buf);
    delete L;
}

APGCU_API int apgcu_loader_submit(apgcu_loader_t L, const char* left_path, const char* right_path,
                                  unsigned long long* ticket) {
    if (!L || !left_path || !right_path || !ticket) return APG_STATUS_INTERNAL_ERROR;
    {
        std::lock_guard<std::mutex> lk(L->mu);
        *ticket = L->next_id++;
        L->jobs.push_back({*ticket, left_path, right_path});
    }
    L->cv_job.notify_one();
    return APG_STATUS_OK;
}

APGCU_API int apgcu_loader_wait(apgcu_loader_t L, unsigned long long ticket, apgcu_loaded_pair_t* out) {
    if (!L || !out) return APG_STATUS_INTERNAL_ERROR;
    std::unique_lock<std::mutex> lk(L->mu);
    if (ticket == 0 || ticket >= L->next_id) return APG_STATUS_INTERNAL_ERROR;
    L->cv_done.wait(lk, [&] { return L->done.count(ticket) != 0; });
    const auto& d = L->done[ticket];
    out->status = d.status;
    out->width = d.w;
    out->height = d.h;
    out->channels = d.ch;
    const size_t one = (size_t)d.w * d.h * d.ch;
    out->left = d.status == 0 ? d.buf : nullptr;
    out->right = d.status == 0 ? d.buf + one : nullptr;
    return d.status;
}

APGCU_API int apgcu_loader_release(apgcu_loader_t L, unsigned long long ticket) {
    if (!L) return APG_STATUS_INTERNAL_ERROR;
    std::lock_guard<std::mutex> lk(L->mu);
    auto it = L->done.find(ticket);
    if (it == L->done.end()) return APG_STATUS_INTERNAL_ERROR;
    if (it->second.buf) L->free_bufs.emplace(it->second.cap, it->second.buf);
    L->done.erase(it);
    return APG_STATUS_OK;
}

APGCU_API size_t apgcu_loader_pinned_bytes(apgcu_loader_t L) {
    if (!L) return 0;
    std::lock_guard<std::mutex> lk(L->mu);
    return L->pinned_bytes;
}

}  // extern "C"
