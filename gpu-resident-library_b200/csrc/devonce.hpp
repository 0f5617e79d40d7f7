// Per-device one-time set-up for host code: kernel attributes such as the
// dynamic shared-memory limit are properties of a kernel on one device, so a
// limit set while device 0 was current does not hold on device 1. DeviceOnce
// runs its function once for every device it is reached on (with that device
// current), and several host threads reaching it together run it once and
// wait for it to finish.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>

namespace gfx {

class DeviceOnce {
public:
    static constexpr int MAX_DEVICES = 64;

    template <class F>
    void operator()(F&& f) {
        int dev = 0;
        if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= MAX_DEVICES) {
            f();   // no usable device number: set up every time rather than never
            return;
        }
        if (done_[dev].load(std::memory_order_acquire)) return;
        std::lock_guard<std::mutex> g(mu_);
        if (done_[dev].load(std::memory_order_relaxed)) return;
        f();
        done_[dev].store(true, std::memory_order_release);
    }

private:
    std::mutex mu_;
    std::atomic<bool> done_[MAX_DEVICES] = {};
};

// Multiprocessor count of the current device, queried once per device.
inline int current_sm_count() {
    static std::atomic<int> count[DeviceOnce::MAX_DEVICES] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= DeviceOnce::MAX_DEVICES) return 148;
    int n = count[dev].load(std::memory_order_relaxed);
    if (n > 0) return n;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) n = 148;
    count[dev].store(n, std::memory_order_relaxed);
    return n;
}

}  // namespace gfx
