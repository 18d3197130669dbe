// Shared types, status bits, launch helpers and the error channel of the C-ABI.
//
// Every entry point of libnabladyn_b200.so returns an int status (ND_OK on success) and keeps
// a per-thread message for nd_last_error(). Argument errors never reach a kernel; data errors
// (a bad cell, a non-finite coordinate, an overflowing list) become device status bits, as in
// the reference's neighbor operator (src/nabladyn/neighbors/csrc/common/common.cuh:13-16).

#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
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
