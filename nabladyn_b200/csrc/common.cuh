// Shared types, status bits, launch helpers and the error channel of the C-ABI.
//
// Every entry point of libnabladyn_b200.so returns an int status (ND_OK on success) and keeps
// a per-thread message for nd_last_error(). Argument errors never reach a kernel; data errors
// (a bad cell, a non-finite coordinate, an overflowing list) become device status bits, as in
// the reference's neighbor operator (src/nabladyn/neighbors/csrc/common/common.cuh:13-16).

#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstddef>
#include <cstdint>
#include <cstdio>
#include <mutex>
#include <string>

#include "nabladyn_b200.h"

namespace nd {

using index_t = std::int32_t;

// Status bits of status[0]. They latch until the list is allocated again.
constexpr index_t kInvalidCell = 1;  // a cell length is not finite or at most twice the cutoff
constexpr index_t kNonFinite = 2;    // a coordinate is not finite
constexpr index_t kOverflow = 8;     // the pairs (or one atom's neighbors) exceed the capacity

constexpr int kWarp = 32;
constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kThreads = 256;

inline unsigned int blocks_for(std::int64_t items, int threads = kThreads)
{
    return static_cast<unsigned int>((items + threads - 1) / threads);
}

// The per-thread message behind nd_last_error().
void set_error(const std::string& message);
const char* last_error();

// Returns from the calling entry point with ND_EINVAL unless `condition` holds.
#define ND_REQUIRE(condition, message)      \
    do                                      \
    {                                       \
        if (!(condition))                   \
        {                                   \
            ::nd::set_error(message);       \
            return ND_EINVAL;               \
        }                                   \
    } while (0)

// Returns ND_ECUDA, with the CUDA error text, when a runtime call or a launch failed.
#define ND_CUDA_TRY(expression)                                                            \
    do                                                                                     \
    {                                                                                      \
        const cudaError_t nd_error_ = (expression);                                        \
        if (nd_error_ != cudaSuccess)                                                      \
        {                                                                                  \
            ::nd::set_error(std::string("CUDA error: ") + cudaGetErrorString(nd_error_) + \
                            " at " __FILE__ ":" + std::to_string(__LINE__));               \
            return ND_ECUDA;                                                               \
        }                                                                                  \
    } while (0)

#define ND_LAUNCH_CHECK() ND_CUDA_TRY(cudaGetLastError())

// Kernel attributes (dynamic shared-memory limits, carveouts) and device properties belong to
// one device: a library used from several GPUs in one process sets and reads them per device.
constexpr int kMaxDevices = 64;

// Runs a setup once per device (the current one), under a lock; a setup that failed is run
// again by the next call instead of being remembered.
class DeviceOnce
{
public:
    template <typename Setup>
    cudaError_t run(Setup setup)
    {
        int device = 0;
        cudaError_t rc = cudaGetDevice(&device);
        if (rc != cudaSuccess)
        {
            return rc;
        }
        if (device < 0 || device >= kMaxDevices)
        {
            return cudaErrorInvalidDevice;
        }
        if (done_[device].load(std::memory_order_acquire))
        {
            return cudaSuccess;
        }
        std::lock_guard<std::mutex> lock(mutex_);
        if (done_[device].load(std::memory_order_relaxed))
        {
            return cudaSuccess;
        }
        rc = setup();
        if (rc == cudaSuccess)
        {
            done_[device].store(true, std::memory_order_release);
        }
        return rc;
    }

private:
    std::mutex mutex_;
    std::atomic<bool> done_[kMaxDevices] = {};
};

// The dynamic shared memory one kernel may use on each device: raised when a launch needs more
// than any launch before it on that device. A kernel gets 48 KB of static and dynamic shared
// memory together without the raise, so the kernel's static bytes (read once per device)
// count against that limit.
class DeviceGrant
{
public:
    template <typename Kernel>
    cudaError_t allow(Kernel kernel, std::size_t bytes)
    {
        if (bytes == 0)
        {
            return cudaSuccess;
        }
        int device = 0;
        cudaError_t rc = cudaGetDevice(&device);
        if (rc != cudaSuccess)
        {
            return rc;
        }
        if (device < 0 || device >= kMaxDevices)
        {
            return cudaErrorInvalidDevice;
        }
        std::lock_guard<std::mutex> lock(mutex_);
        if (bytes <= granted_[device])
        {
            return cudaSuccess;
        }
        if (!static_known_[device])
        {
            cudaFuncAttributes attributes{};
            rc = cudaFuncGetAttributes(&attributes, kernel);
            if (rc != cudaSuccess)
            {
                return rc;
            }
            static_bytes_[device] = attributes.sharedSizeBytes;
            static_known_[device] = true;
        }
        if (bytes + static_bytes_[device] > 48 * 1024)
        {
            rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      static_cast<int>(bytes));
            if (rc != cudaSuccess)
            {
                return rc;
            }
        }
        granted_[device] = bytes;
        return cudaSuccess;
    }

private:
    std::mutex mutex_;
    std::size_t granted_[kMaxDevices] = {};
    std::size_t static_bytes_[kMaxDevices] = {};
    bool static_known_[kMaxDevices] = {};
};

// The current device's multiprocessor count, looked up once per device.
inline cudaError_t multiprocessors(int* count)
{
    static std::atomic<int> known[kMaxDevices] = {};
    int device = 0;
    cudaError_t rc = cudaGetDevice(&device);
    if (rc != cudaSuccess)
    {
        return rc;
    }
    if (device < 0 || device >= kMaxDevices)
    {
        return cudaErrorInvalidDevice;
    }
    int value = known[device].load(std::memory_order_relaxed);
    if (value == 0)
    {
        rc = cudaDeviceGetAttribute(&value, cudaDevAttrMultiProcessorCount, device);
        if (rc != cudaSuccess)
        {
            return rc;
        }
        known[device].store(value, std::memory_order_relaxed);
    }
    *count = value;
    return cudaSuccess;
}

// Whether a gated rebuild kernel does work: a build from allocate passes no flag and always
// runs; an update runs only when the reuse check asked for a rebuild and no error latched.
__device__ __forceinline__ bool rebuilding(const index_t* rebuild, const index_t* status)
{
    return rebuild == nullptr || (rebuild[0] != 0 && status[0] == 0);
}

template <typename T>
__device__ __forceinline__ T warp_sum(T value)
{
#pragma unroll
    for (int offset = kWarp / 2; offset > 0; offset /= 2)
    {
        value += __shfl_xor_sync(kFullMask, value, offset);
    }
    return value;
}

}  // namespace nd
