// Process-wide pool of non-blocking CUDA streams, per device. Creating a stream while the
// device is busy was measured to take tens of milliseconds and to hold up other threads'
// launches meanwhile (a server admitting a stream stalled the steps of the admitted ones by
// up to 0.2 s), so engines take their private streams from this pool and hand them back at
// close; a server creates the streams of all its slots up front, while the device is idle.
// A returned stream may still have work queued: the next owner's work simply runs after it.
#pragma once

#include <cuda_runtime.h>

#include <map>
#include <mutex>
#include <vector>

namespace ddm {

class StreamPool {
  public:
    static StreamPool &get() {
        static StreamPool pool;  // lives until exit; the driver releases the streams then
        return pool;
    }
    // A non-blocking stream of `device` (the calling thread's current device), or nullptr.
    cudaStream_t acquire(int device) {
        {
            std::lock_guard<std::mutex> g(lock_);
            auto &fl = free_[device];
            if (!fl.empty()) {
                cudaStream_t s = fl.back();
                fl.pop_back();
                return s;
            }
        }
        cudaStream_t s = nullptr;
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
        return s;
    }
    void release(int device, cudaStream_t s) {
        if (!s) return;
        std::lock_guard<std::mutex> g(lock_);
        free_[device].push_back(s);
    }
    // Makes at least n streams of `device` (the current device) idle in the pool.
    void reserve(int device, int n) {
        std::vector<cudaStream_t> made;
        {
            std::lock_guard<std::mutex> g(lock_);
            n -= static_cast<int>(free_[device].size());
        }
        for (int i = 0; i < n; i++) {
            cudaStream_t s = nullptr;
            if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) break;
            made.push_back(s);
        }
        std::lock_guard<std::mutex> g(lock_);
        for (cudaStream_t s : made) free_[device].push_back(s);
    }

  private:
    std::mutex lock_;
    std::map<int, std::vector<cudaStream_t>> free_;
};

inline cudaStream_t stream_acquire(int device) { return StreamPool::get().acquire(device); }
inline void stream_release(int device, cudaStream_t s) { StreamPool::get().release(device, s); }

}  // namespace ddm
