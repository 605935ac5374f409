// Device memory cache behind DevBuf.
//
// cudaMalloc / cudaFree of a problem's ~100-200 buffers costs tens to hundreds
// of milliseconds on a B200 (measured 27-580 ms for 0.3 GB, varying from call
// to call), more than solving the problem.  Freed blocks are therefore kept,
// keyed by device and rounded size (512 B granules up to 1 MiB, 2 MiB above),
// and handed out again to the next request of that size on that device.
//
// * A block is cached only after cudaDeviceSynchronize, the same implicit
//   synchronisation cudaFree performs, so no kernel still reading it can see
//   it reused.
// * At most GANIT_B200_POOL_BYTES (default 4 GiB) are kept; beyond that a
//   freed block goes back to the driver.  gb_release_cached_memory() returns
//   every cached block; a failed cudaMalloc does so too and retries once.
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <unordered_map>
#include <utility>
#include <vector>

#include "../../include/ganit_b200.h"
#include "gb_common.cuh"

namespace gb {

bool trace_enabled() {
    static const bool on = [] {
        const char* v = std::getenv("GANIT_B200_TRACE");
        return v != nullptr && std::strcmp(v, "1") == 0;
    }();
    return on;
}

double StageTrace::now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

namespace {

struct Block {
    int device;
    size_t bytes;
};

struct PairHash {
    size_t operator()(const std::pair<int, size_t>& k) const { return std::hash<size_t>()(k.second * 131 + k.first); }
};

struct Pool {
    std::mutex mu;
    std::unordered_map<void*, Block> live;
    std::unordered_map<std::pair<int, size_t>, std::vector<void*>, PairHash> cached;
    size_t cached_bytes = 0;
    std::unordered_map<void*, size_t> host_live;               // pinned host blocks
    std::unordered_map<size_t, std::vector<void*>> host_cached;
    size_t host_cached_bytes = 0;
    size_t cap = size_t(4) << 30;
    Pool() {
        if (const char* e = std::getenv("GANIT_B200_POOL_BYTES")) cap = static_cast<size_t>(std::strtoull(e, nullptr, 10));
    }
};

constexpr size_t kHostCacheCap = size_t(256) << 20;

// Free batch of this thread: depth, device, and whether its one
// synchronisation succeeded.
thread_local int tl_batch = 0;
thread_local int tl_batch_device = -1;
thread_local bool tl_batch_ok = false;

// True when nothing still running on `device` can use a block freed now.
bool quiesced(int device) {
    if (tl_batch > 0 && tl_batch_device == device) return tl_batch_ok;
    return cudaDeviceSynchronize() == cudaSuccess;
}

Pool& pool() {
    static Pool* p = new Pool();  // never destroyed: blocks may be freed during process teardown
    return *p;
}

size_t rounded(size_t b) {
    if (b == 0) b = 1;
    if (b <= (size_t(1) << 20)) return (b + 511) & ~size_t(511);
    const size_t g = size_t(2) << 20;
    return (b + g - 1) & ~(g - 1);
}

// Returns every cached block of `device` (all devices when < 0) to the driver.
void drain(int device) {
    Pool& P = pool();
    std::vector<std::pair<int, void*>> out;
    {
        std::lock_guard<std::mutex> g(P.mu);
        for (auto it = P.cached.begin(); it != P.cached.end();) {
            if (device < 0 || it->first.first == device) {
                for (void* q : it->second) {
                    out.emplace_back(it->first.first, q);
                    P.cached_bytes -= it->first.second;
                }
                it = P.cached.erase(it);
            } else {
                ++it;
            }
        }
    }
    int cur = 0;
    cudaGetDevice(&cur);
    for (auto& [dev, q] : out) {
        cudaSetDevice(dev);
        cudaFree(q);
    }
    cudaSetDevice(cur);
    if (device < 0) {  // and the pinned host blocks
        std::vector<void*> hout;
        {
            std::lock_guard<std::mutex> g(P.mu);
            for (auto& [b, v] : P.host_cached) hout.insert(hout.end(), v.begin(), v.end());
            P.host_cached.clear();
            P.host_cached_bytes = 0;
        }
        for (void* q : hout) cudaFreeHost(q);
    }
}

}  // namespace

void* dev_alloc(size_t bytes) {
    const size_t b = rounded(bytes);
    int dev = 0;
    GB_CUDA(cudaGetDevice(&dev));
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.cached.find({dev, b});
        if (it != P.cached.end() && !it->second.empty()) {
            void* q = it->second.back();
            it->second.pop_back();
            P.cached_bytes -= b;
            P.live[q] = Block{dev, b};
            return q;
        }
    }
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, b);
    if (e == cudaErrorMemoryAllocation) {
        cudaGetLastError();
        drain(dev);
        e = cudaMalloc(&q, b);
    }
    GB_CUDA(e);
    std::lock_guard<std::mutex> g(P.mu);
    P.live[q] = Block{dev, b};
    return q;
}

void dev_free(void* q) {
    if (!q) return;
    Pool& P = pool();
    Block blk{};
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.live.find(q);
        if (it == P.live.end()) return;
        blk = it->second;
        P.live.erase(it);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != blk.device) cudaSetDevice(blk.device);
    const bool ok = quiesced(blk.device);
    bool keep = false;
    if (ok) {
        std::lock_guard<std::mutex> g(P.mu);
        if (P.cached_bytes + blk.bytes <= P.cap) {
            P.cached[{blk.device, blk.bytes}].push_back(q);
            P.cached_bytes += blk.bytes;
            keep = true;
        }
    }
    if (!keep) cudaFree(q);
    if (cur != blk.device) cudaSetDevice(cur);
}

void* host_alloc(size_t bytes) {
    const size_t b = rounded(bytes);
    Pool& P = pool();
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.host_cached.find(b);
        if (it != P.host_cached.end() && !it->second.empty()) {
            void* q = it->second.back();
            it->second.pop_back();
            P.host_cached_bytes -= b;
            P.host_live[q] = b;
            return q;
        }
    }
    void* q = nullptr;
    GB_CUDA(cudaMallocHost(&q, b));  // portable: unified addressing makes pinned memory visible to every device
    std::lock_guard<std::mutex> g(P.mu);
    P.host_live[q] = b;
    return q;
}

void host_free(void* q) {
    if (!q) return;
    Pool& P = pool();
    size_t b = 0;
    {
        std::lock_guard<std::mutex> g(P.mu);
        auto it = P.host_live.find(q);
        if (it == P.host_live.end()) return;
        b = it->second;
        P.host_live.erase(it);
    }
    int cur = 0;
    cudaGetDevice(&cur);
    // a copy into or out of the block may still run on any device; the
    // current one is the problem's (the owners set it before tearing down)
    bool keep = false;
    if (quiesced(cur)) {
        std::lock_guard<std::mutex> g(P.mu);
        if (P.host_cached_bytes + b <= kHostCacheCap) {
            P.host_cached[b].push_back(q);
            P.host_cached_bytes += b;
            keep = true;
        }
    }
    if (!keep) cudaFreeHost(q);
}

void begin_free_batch() {
    int cur = 0;
    cudaGetDevice(&cur);
    if (tl_batch == 0 || tl_batch_device != cur) {
        tl_batch_device = cur;
        tl_batch_ok = cudaDeviceSynchronize() == cudaSuccess;
    }
    ++tl_batch;
}

void end_free_batch() {
    if (tl_batch > 0) --tl_batch;
}

}  // namespace gb

extern "C" {

void gb_release_cached_memory(void) { gb::drain(-1); }

int64_t gb_cached_memory_bytes(void) {
    gb::Pool& P = gb::pool();
    std::lock_guard<std::mutex> g(P.mu);
    return static_cast<int64_t>(P.cached_bytes);
}

}  // extern "C"
