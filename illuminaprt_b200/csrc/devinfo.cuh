// Per-device launch facts cached on the host: the SM count that sizes
// persistent grids, and the dynamic shared-memory opt-in of kernels that use
// more than 48 KB. cudaFuncSetAttribute acts on the current device only, so
// the opt-in is made once per (device, kernel, size); both caches are
// thread-safe, so contexts on several devices may be used from several host
// threads.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <set>
#include <tuple>

namespace ilg {

// SM count of the current device (148 if the query fails).
inline int current_sm_count()
{
    constexpr int kDevices = 64;
    static std::mutex mu;
    static int cache[kDevices] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return 148;
    auto query = [dev] {
        int s = 0;
        if (cudaDeviceGetAttribute(&s, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || s <= 0) s = 148;
        return s;
    };
    if (dev >= kDevices) return query();
    std::lock_guard<std::mutex> g(mu);
    if (!cache[dev]) cache[dev] = query();
    return cache[dev];
}

// Lets `func` launch with `bytes` of dynamic shared memory on the current device.
inline cudaError_t ensure_dynamic_smem(const void *func, int bytes)
{
    static std::mutex mu;
    static std::set<std::tuple<int, const void *, int>> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const auto key = std::make_tuple(dev, func, bytes);
    std::lock_guard<std::mutex> g(mu);
    if (done.count(key)) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.insert(key);
    return e;
}

}  // namespace ilg
