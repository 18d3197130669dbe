// Device-wide exclusive prefix sum of int32 counts, gated like the rebuild kernels.
//
// The reference calls CUB's DeviceScan::ExclusiveSum (src/nabladyn/neighbors/csrc/runtime/
// entry_points.cu:106-122), which cannot be gated and so runs on every update. This scan is
// our own: one launch for inputs that fit one tile of kTileItems, otherwise reduce -> scan of
// the tile sums in one block -> scan of each tile with its carry. No spin-waits, deterministic.

#pragma once

#include "common.cuh"

namespace nd {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;  // per thread
constexpr std::int64_t kTileItems = static_cast<std::int64_t>(kScanThreads) * kScanItems;

inline std::int64_t scan_tiles(std::int64_t items)
{
    return (items + kTileItems - 1) / kTileItems;
}

// Scratch bytes of scan_exclusive over `items` values: one int per tile beyond the first.
inline std::int64_t scan_scratch_bytes(std::int64_t items)
{
    const std::int64_t tiles = scan_tiles(items);
    return tiles > 1 ? tiles * static_cast<std::int64_t>(sizeof(index_t)) : 16;
}

// Exclusive scan of one value per thread across the block; returns the block total too.
template <int THREADS>
__device__ __forceinline__ index_t block_exclusive(index_t value, index_t& total)
{
    __shared__ index_t warp_totals[THREADS / kWarp];
    const int lane = threadIdx.x % kWarp;
    const int warp = threadIdx.x / kWarp;
    index_t inclusive = value;
#pragma unroll
    for (int offset = 1; offset < kWarp; offset *= 2)
    {
        const index_t up = __shfl_up_sync(kFullMask, inclusive, offset);
        if (lane >= offset)
        {
            inclusive += up;
        }
    }
    if (lane == kWarp - 1)
    {
        warp_totals[warp] = inclusive;
    }
    __syncthreads();
    if (warp == 0)
    {
        index_t t = lane < THREADS / kWarp ? warp_totals[lane] : 0;
        index_t scanned = t;
#pragma unroll
        for (int offset = 1; offset < kWarp; offset *= 2)
        {
            const index_t up = __shfl_up_sync(kFullMask, scanned, offset);
            if (lane >= offset)
            {
                scanned += up;
            }
        }
        if (lane < THREADS / kWarp)
        {
            warp_totals[lane] = scanned - t;  // exclusive warp offsets
        }
    }
    __syncthreads();
    const index_t warp_offset = warp_totals[warp];
    // The total is the last warp's offset plus that warp's inclusive sum.
    __shared__ index_t block_total;
    if (threadIdx.x == THREADS - 1)
    {
        block_total = warp_offset + inclusive;
    }
    __syncthreads();
    total = block_total;
    const index_t result = warp_offset + inclusive - value;
    __syncthreads();  // the shared words are reused by the next call
    return result;
}

// The kernels have internal linkage: every translation unit that scans owns a copy.
namespace {

// Sums each tile of the input into tile_sums[tile].
__global__ void scan_reduce_kernel(
    const index_t* __restrict__ input,
    std::int64_t items,
    index_t* __restrict__ tile_sums,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    if (!rebuilding(rebuild, status))
    {
        return;
    }
    const std::int64_t begin = static_cast<std::int64_t>(blockIdx.x) * kTileItems;
    index_t sum = 0;
    for (int k = 0; k < kScanItems; ++k)
    {
        const std::int64_t i = begin + static_cast<std::int64_t>(k) * kScanThreads + threadIdx.x;
        if (i < items)
        {
            sum += input[i];
        }
    }
    index_t total;
    block_exclusive<kScanThreads>(sum, total);
    if (threadIdx.x == 0)
    {
        tile_sums[blockIdx.x] = total;
    }
}

// One block: the exclusive scan of the tile sums, in place.
__global__ void scan_tile_sums_kernel(
    index_t* __restrict__ tile_sums,
    std::int64_t tiles,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    if (!rebuilding(rebuild, status))
    {
        return;
    }
    index_t carry = 0;
    for (std::int64_t base = 0; base < tiles; base += kScanThreads)
    {
        const std::int64_t i = base + threadIdx.x;
        const index_t value = i < tiles ? tile_sums[i] : 0;
        index_t total;
        const index_t prefix = block_exclusive<kScanThreads>(value, total);
        if (i < tiles)
        {
            tile_sums[i] = carry + prefix;
        }
        carry += total;
    }
}

// Scans each tile from its carry (tile_sums[tile], or 0 with a single tile). Each thread
// owns kScanItems consecutive values, staged through shared memory so that global reads
// and writes stay coalesced.
__global__ void scan_tiles_kernel(
    const index_t* __restrict__ input,
    std::int64_t items,
    const index_t* __restrict__ tile_sums,
    index_t* __restrict__ output,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    if (!rebuilding(rebuild, status))
    {
        return;
    }
    __shared__ index_t staged[kTileItems + kTileItems / kWarp];  // padded against bank conflicts
    const std::int64_t begin = static_cast<std::int64_t>(blockIdx.x) * kTileItems;
    auto slot = [](int k) { return k + k / kWarp; };
    for (int k = 0; k < kScanItems; ++k)
    {
        const int local = k * kScanThreads + threadIdx.x;
        const std::int64_t i = begin + local;
        staged[slot(local)] = i < items ? input[i] : 0;
    }
    __syncthreads();
    index_t values[kScanItems];
    index_t sum = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        values[k] = staged[slot(threadIdx.x * kScanItems + k)];
        sum += values[k];
    }
    index_t total;
    index_t running = block_exclusive<kScanThreads>(sum, total);
    if (tile_sums != nullptr)
    {
        running += tile_sums[blockIdx.x];
    }
#pragma unroll
    for (int k = 0; k < kScanItems; ++k)
    {
        staged[slot(threadIdx.x * kScanItems + k)] = running;
        running += values[k];
    }
    __syncthreads();
    for (int k = 0; k < kScanItems; ++k)
    {
        const int local = k * kScanThreads + threadIdx.x;
        const std::int64_t i = begin + local;
        if (i < items)
        {
            output[i] = staged[slot(local)];
        }
    }
}

}  // namespace

// Launches the exclusive scan of `items` values. `scratch` holds scan_scratch_bytes(items).
inline cudaError_t scan_exclusive(
    const index_t* input,
    index_t* output,
    std::int64_t items,
    void* scratch,
    const index_t* rebuild,
    const index_t* status,
    cudaStream_t stream
)
{
    const std::int64_t tiles = scan_tiles(items);
    if (tiles <= 1)
    {
        scan_tiles_kernel<<<1, kScanThreads, 0, stream>>>(
            input, items, nullptr, output, rebuild, status);
        return cudaGetLastError();
    }
    auto* sums = static_cast<index_t*>(scratch);
    scan_reduce_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(
        input, items, sums, rebuild, status);
    scan_tile_sums_kernel<<<1, kScanThreads, 0, stream>>>(sums, tiles, rebuild, status);
    scan_tiles_kernel<<<static_cast<unsigned>(tiles), kScanThreads, 0, stream>>>(
        input, items, sums, output, rebuild, status);
    return cudaGetLastError();
}

}  // namespace nd
