// Process-wide pool of page-locked host buffers. cudaMallocHost is slow and cudaFreeHost
// synchronises the device, so buffers that engines and servers create and drop while other
// work runs (pair tables, norms, chunk and result buffers of served streams) are kept and
// reused: blocks are rounded up to a power of two and returned to a free list of that size.
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
        if (cudaMallocHost(&p, cls) != cudaSuccess) return nullptr;
        size_of_[p] = cls;
        return p;
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
};

inline void *pinned_alloc(size_t bytes) { return PinnedPool::get().alloc(bytes); }
inline void pinned_release(void *p) { PinnedPool::get().release(p); }

}  // namespace ddm
