// cvl_pinned.h -- page-locked host memory for results and requests.
//
// A few large page-locked chunks, sub-allocated first-fit with coalescing.
// Pinning memory (cudaMallocHost) costs about as much as copying it several
// times, and while it runs it holds up other CUDA calls of the process. So
// chunks grow geometrically: each new chunk is at least as large as all
// previous chunks together, and a steady stream of mixed sizes stops
// allocating after a few chunks. Blocks are 256-byte aligned.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstddef>
#include <cstdint>
#include <iterator>
#include <map>
#include <mutex>
#include <unordered_map>
#include <vector>

// The library's allocation-failure injector (cvl_debug_fail_allocations): true when
// this allocation is to fail as if the memory were exhausted.
bool cvl_alloc_fault_injected();

namespace cvl {

class PinnedArena {
  public:
    explicit PinnedArena(size_t first_chunk = (size_t)64 << 20) : first_(first_chunk) {}
    PinnedArena(const PinnedArena &) = delete;
    PinnedArena &operator=(const PinnedArena &) = delete;
    ~PinnedArena() {
        for (Chunk &c : chunks_) cudaFreeHost(c.base);
    }

    // a block of at least `bytes`, or nullptr if no page-locked memory could be had
    void *get(size_t bytes) {
        bytes = round(bytes ? bytes : 1);
        std::lock_guard<std::mutex> lk(mu_);
        for (size_t ci = 0; ci < chunks_.size(); ++ci) {
            void *p = take(ci, bytes);
            if (p) return p;
        }
        size_t total = 0;
        for (const Chunk &c : chunks_) total += c.size;
        const size_t want = round(std::max({bytes, first_, total}));
        void *base = nullptr;
        if (cvl_alloc_fault_injected()) return nullptr;
        const auto t0 = std::chrono::steady_clock::now();
        const cudaError_t ce = cudaMallocHost(&base, want);
        grow_ns_ += (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
                        std::chrono::steady_clock::now() - t0).count();
        ++grows_;
        if (ce != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        Chunk c;
        c.base = (char *)base;
        c.size = want;
        c.free[0] = want;
        chunks_.push_back(c);
        return take(chunks_.size() - 1, bytes);
    }

    void put(void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> lk(mu_);
        auto it = live_.find(p);
        if (it == live_.end()) return;
        const size_t ci = it->second.first, sz = it->second.second;
        live_.erase(it);
        Chunk &c = chunks_[ci];
        size_t off = (size_t)((char *)p - c.base), len = sz;
        auto next = c.free.lower_bound(off);
        if (next != c.free.end() && off + len == next->first) {  // merge with the following range
            len += next->second;
            next = c.free.erase(next);
        }
        if (next != c.free.begin()) {  // merge with the preceding range
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += len;
                return;
            }
        }
        c.free[off] = len;
    }

    // chunks pinned so far (cudaMallocHost calls) and the host time they took
    uint64_t grows() const { return grows_.load(); }
    double grow_ms() const { return (double)grow_ns_.load() * 1e-6; }

    // ensures one free range of at least `bytes` (a chunk made ahead of time)
    bool reserve(size_t bytes) {
        void *p = get(bytes);
        put(p);
        return p != nullptr;
    }

  private:
    struct Chunk {
        char *base = nullptr;
        size_t size = 0;
        std::map<size_t, size_t> free;  // offset -> length
    };

    static size_t round(size_t b) { return (b + 255) & ~(size_t)255; }

    void *take(size_t ci, size_t bytes) {  // first fit in chunk ci (mu_ held)
        Chunk &c = chunks_[ci];
        for (auto it = c.free.begin(); it != c.free.end(); ++it) {
            if (it->second < bytes) continue;
            const size_t off = it->first, len = it->second;
            c.free.erase(it);
            if (len > bytes) c.free[off + bytes] = len - bytes;
            void *p = c.base + off;
            live_[p] = {ci, bytes};
            return p;
        }
        return nullptr;
    }

    std::mutex mu_;
    std::atomic<uint64_t> grows_{0}, grow_ns_{0};
    size_t first_;
    std::vector<Chunk> chunks_;
    std::unordered_map<void *, std::pair<size_t, size_t>> live_;
};

}  // namespace cvl
