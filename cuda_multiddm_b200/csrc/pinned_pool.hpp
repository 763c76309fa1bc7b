// Process-wide pool of page-locked host buffers. cudaMallocHost is slow and cudaFreeHost
// synchronises the device, so buffers that engines and servers create and drop while other
// work runs (pair tables, norms, chunk and result buffers of served streams) are kept and
// reused: blocks are rounded up to a power of two and returned to a free list of that size.
// A block no free list holds is carved from an arena page-locked up front (reserve_arena, which
// a server calls at open): pinning tens of MB while streams run was measured to take 0.1-0.3 s
// and to hold up other threads' launches for as long. Only when the arena is used up does a
// miss call cudaMallocHost.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <map>
#include <mutex>
#include <vector>

namespace ddm {

class PinnedPool {
  public:
    static PinnedPool &get() {
        static PinnedPool pool;  // lives until exit; the driver frees page-locked memory then
        return pool;
    }
    void *alloc(size_t bytes) {
        const size_t cls = round_up(bytes);
        std::lock_guard<std::mutex> g(lock_);
        auto &fl = free_[cls];
        if (!fl.empty()) {
            void *p = fl.back();
            fl.pop_back();
            size_of_[p] = cls;
            return p;
        }
        void *p = nullptr;
        if (arena_used_ + cls <= arena_bytes_) {
            p = arena_ + arena_used_;
            arena_used_ += cls;
        } else if (cudaMallocHost(&p, cls) != cudaSuccess) {
            return nullptr;
        }
        size_of_[p] = cls;
        return p;
    }
    // Page-locks an arena of at least `bytes` for later misses (once: a larger request later
    // adds nothing). False if the memory could not be page-locked.
    bool reserve_arena(size_t bytes) {
        std::lock_guard<std::mutex> g(lock_);
        if (arena_bytes_ >= bytes) return true;
        if (arena_bytes_ > 0) return true;  // one arena per process
        void *p = nullptr;
        if (cudaMallocHost(&p, bytes) != cudaSuccess) return false;
        arena_ = static_cast<char *>(p);
        arena_bytes_ = bytes;
        arena_used_ = 0;
        return true;
    }
    void release(void *p) {
        if (!p) return;
        std::lock_guard<std::mutex> g(lock_);
        auto it = size_of_.find(p);
        if (it == size_of_.end()) return;
        free_[it->second].push_back(p);
        size_of_.erase(it);
    }

  private:
    static size_t round_up(size_t b) {
        size_t c = 4096;
        while (c < b) c <<= 1;
        return c;
    }
    std::mutex lock_;
    std::map<size_t, std::vector<void *>> free_;
    std::map<void *, size_t> size_of_;
    char *arena_ = nullptr;
    size_t arena_bytes_ = 0, arena_used_ = 0;
};

inline void *pinned_alloc(size_t bytes) { return PinnedPool::get().alloc(bytes); }
inline void pinned_release(void *p) { PinnedPool::get().release(p); }

}  // namespace ddm
