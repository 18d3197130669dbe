// Pieces shared by the SchNet kernels (schnet.cu: E, F and W; schnet_tangent.cu: the
// parameter gradient of a force and virial loss): sizes, the packed parameter block and the
// workspace layouts, the activations, BF16 feature rows, the per-CTA tensor-core context,
// the Gaussian basis and the run sums of first-atom rows.

#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "umma.cuh"

namespace nd {
namespace {

constexpr int kFeatures = 64;
constexpr int kHidden = 32;      // the readout's hidden layer, features / 2
constexpr int kTile = 128;       // rows per tensor-core tile = threads per CTA
constexpr int kImagesPerBlock = 10;
constexpr float kLn2 = 0.693147180559945309f;
constexpr int kGatherBatch = 2;  // feature words (8 features) a pair kernel gathers before use

// Status bits of the SchNet status word.
constexpr int kBadPair = 1;       // a pair index outside [0, N)
constexpr int kProductLost = 16;  // a tensor-core product did not complete in time

// Weight images of one block, in this order.
enum Image : int
{
    kB1 = 0,   // filter1.weight [64 out][K in, zero-padded to 64]
    kB2 = 1,   // filter2.weight [out][in]
    kB2T = 2,  // its transpose
    kB1T = 3,  // filter1.weight^T [K, zero-padded to 64][64]
    kA = 4,    // atoms.weight
    kAT = 5,
    kD1 = 6,   // update1.weight
    kD1T = 7,
    kD2 = 8,   // update2.weight
    kD2T = 9,
};

// Byte layout of the packed parameter block (nd_schnet_weight_bytes).
struct WeightLayout
{
    std::int64_t vectors;  // per block: b1, b2, d1, d2 (64 floats each)
    std::int64_t readout;  // R1 [32][64], e1 [32], R2 [32], e2 (padded to 32)
    std::int64_t tables;   // embedding [T][64], v0 = embedding A0^T [T][64]
    std::int64_t total;

    __host__ __device__ WeightLayout(int blocks, int types)
    {
        vectors = static_cast<std::int64_t>(blocks) * kImagesPerBlock * umma::kImageBytes;
        readout = vectors + static_cast<std::int64_t>(blocks) * 4 * kFeatures * 4;
        tables = readout + (kHidden * kFeatures + 3 * kHidden) * 4;
        total = tables + 2 * static_cast<std::int64_t>(types) * kFeatures * 4;
    }
};

__host__ __device__ inline std::int64_t align256(std::int64_t bytes)
{
    return (bytes + 255) / 256 * 256;
}

constexpr int kVirialSlots = 1024;  // per-CTA virial partials of the last reverse pass

// Byte layout of the workspace (nd_schnet_workspace_bytes).
struct Workspace
{
    std::int64_t counters, block_counts, block_offsets, pairs, geometry, x, v, h, m, grad,
        grad_m, grad_v, dedr, energy, virial, total;

    Workspace(std::int64_t atoms, std::int64_t columns, int blocks)
    {
        const std::int64_t row = atoms * kFeatures * 4;
        const std::int64_t tiles = (atoms + kTile - 1) / kTile;
        const std::int64_t column_blocks = (columns + kThreads - 1) / kThreads;
        counters = 0;
        block_counts = 256;
        block_offsets = block_counts + align256(column_blocks * 4);
        pairs = block_offsets + align256(column_blocks * 4);
        geometry = pairs + align256(columns * 8);
        x = geometry + align256(columns * 16);
        v = x + align256(row);
        h = v + blocks * align256(row);
        m = h + blocks * align256(row);  // one message buffer per block (the tangent pass reuses them)
        grad = m + blocks * align256(row);
        grad_m = grad + align256(row);
        grad_v = grad_m + align256(row);
        dedr = grad_v + align256(row);
        energy = dedr + align256(columns * 4);
        virial = energy + align256(tiles * 8);
        total = virial + align256(kVirialSlots * 9 * 8);
    }
};

__device__ __forceinline__ float approx_reciprocal(float x)
{
    float y;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ln(1 + e^x) - ln 2 and its derivative, in FP32 with the hardware exp and log; the results
// feed BF16 operands.
__device__ __forceinline__ float softplus_shifted(float x)
{
    return fmaxf(x, 0.0f) + __logf(1.0f + __expf(-fabsf(x))) - kLn2;
}

// 1 / (1 + e^-x) = (1 + tanh(x / 2)) / 2, with the hardware tanh (one special-function op).
__device__ __forceinline__ float sigmoid(float x)
{
    float t;
    asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(0.5f * x));
    return fmaf(0.5f, t, 0.5f);
}

// Feature rows that the pair kernels gather (v = x A^T and Gm) are kept in BF16: 128 B per
// row, read 16 bytes at a time. Eight consecutive features (the word at group = 8 row +
// feature / 8), widened to floats.
__device__ __forceinline__ void widen8(const uint4& word, float (&out)[8])
{
    const std::uint32_t w[4] = {word.x, word.y, word.z, word.w};
#pragma unroll
    for (int i = 0; i < 4; ++i)
    {
        out[2 * i] = __uint_as_float(w[i] << 16);
        out[2 * i + 1] = __uint_as_float(w[i] & 0xFFFF0000u);
    }
}

__device__ __forceinline__ void load8(const uint4* __restrict__ rows, std::int64_t group,
                                      float (&out)[8])
{
    widen8(__ldg(rows + group), out);
}

__device__ __forceinline__ std::uint32_t pack2(float lo, float hi)
{
    __nv_bfloat162 pair = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<std::uint32_t*>(&pair);
}

// Shared-memory staging of weight images and bias vectors, by all 128 threads.
__device__ __forceinline__ void copy_bytes(unsigned char* to, const unsigned char* from, int bytes)
{
    for (int i = threadIdx.x * 16; i < bytes; i += kTile * 16)
    {
        *reinterpret_cast<uint4*>(to + i) = __ldg(reinterpret_cast<const uint4*>(from + i));
    }
}

// The per-CTA tensor-core context: tensor memory, the completion barrier and its phase.
struct Cores
{
    std::uint64_t* barrier;
    std::uint32_t* slot;
    std::uint32_t tmem;  // this warp's lanes, column 0
    unsigned phase;

    __device__ void open(std::uint64_t* barrier_, std::uint32_t* slot_, std::uint32_t columns,
                         int* counters_, int stage_)
    {
        barrier = barrier_;
        slot = slot_;
        phase = 0;
        counters = counters_;
        stage = stage_;
        tile_index = -1;
        if (threadIdx.x == 0)
        {
            umma::barrier_init(barrier);
        }
        if (threadIdx.x < 32)
        {
            umma::allocate(slot, columns);
        }
        umma::fence_before_sync();
        __syncthreads();
        umma::fence_after_sync();
        tmem = *slot + ((32u * (threadIdx.x / 32)) << 16);
    }

    int* counters;  // [4]: pairs, status bits, first stage that gave up, its tile
    int stage;      // the kernel's stage code, for the diagnostics
    int tile_index; // the tile in work, for the diagnostics

    // D[column offset] = tile * image^T, after every thread wrote its row of the tile; waits
    // for the product. False (on every thread) when it did not complete in time; then the
    // status bit is set and the first stage and tile that gave up are recorded.
    __device__ bool run(std::uint32_t column, const unsigned char* tile, const unsigned char* image,
                        int step)
    {
        return run2(column, tile, image, 0, nullptr, nullptr, step);
    }

    // As run, with a second product D[column2] = tile2 * image2^T (when tile2 is not null)
    // issued behind the first and completing on the same commit.
    __device__ bool run2(std::uint32_t column, const unsigned char* tile, const unsigned char* image,
                         std::uint32_t column2, const unsigned char* tile2,
                         const unsigned char* image2, int step)
    {
        umma::fence_operands();
        umma::fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0)
        {
            umma::fence_after_sync();
            umma::product(*slot + column, umma::smem_address(tile), umma::smem_address(image));
            if (tile2 != nullptr)
            {
                umma::product(*slot + column2, umma::smem_address(tile2),
                              umma::smem_address(image2));
            }
            umma::commit(barrier);
        }
        const bool done = umma::barrier_wait(barrier, phase);
        phase ^= 1u;
        const bool lost = __syncthreads_or(!done);
        umma::fence_after_sync();
        if (lost && threadIdx.x == 0)
        {
            atomicOr(counters + 1, kProductLost);
            if (atomicCAS(counters + 2, 0, 16 * stage + step) == 0)
            {
                counters[3] = tile_index;
            }
        }
        return !lost;
    }

    __device__ void close(std::uint32_t columns)
    {
        umma::fence_before_sync();
        __syncthreads();
        if (threadIdx.x < 32)
        {
            umma::fence_after_sync();
            umma::deallocate(*slot, columns);
        }
    }
};

// Gaussians g_k(r) = exp(-(r / D - k)^2 / 2), k < K, zero above, into this thread's row.
__device__ __forceinline__ void store_basis(unsigned char* tile, float r_over_width, int gaussians,
                                            bool live)
{
#pragma unroll
    for (int c = 0; c < 8; ++c)
    {
        float values[8];
#pragma unroll
        for (int e = 0; e < 8; ++e)
        {
            const int k = 8 * c + e;
            const float u = r_over_width - static_cast<float>(k);
            values[e] = (live && k < gaussians) ? __expf(-0.5f * u * u) : 0.0f;
        }
        umma::store8(tile, threadIdx.x, c, values);
    }
}

// Run sums of first-atom rows. Every pair's first-atom vector (32 columns, [32 half,
// 32 half + 32) of a [N][64] target) is staged in shared memory (16 KB: float4 chunks
// swizzled by row against bank conflicts; thread t stages row t); the tile's pairs keep the
// list's order, so a first atom's pairs are runs of rows: each warp sums its 32 rows column
// by column and adds one atomic per run and column instead of one per pair. Dead rows carry
// first = -1.

// Stages chunk q (columns 4q .. 4q + 3 of the half) of this thread's row.
__device__ __forceinline__ void put_run_part(float* stage, int q, float4 value)
{
    reinterpret_cast<float4*>(stage)[threadIdx.x * 8 + (q ^ (threadIdx.x & 7))] = value;
}

// Sums the staged rows over runs into `target`. Each warp sums the 32 rows its own threads
// staged, so a warp barrier orders the staging; `block_barrier` ends with a block barrier,
// for callers whose next writes to the stage's bytes come from other warps.
__device__ __forceinline__ void sum_runs(const float* stage, const int* first, float* target,
                                         int half, bool block_barrier)
{
    __syncwarp();
    const int column = threadIdx.x & 31;
    const int begin = (threadIdx.x >> 5) * 32;
    float sum = 0.0f;
    for (int r = begin; r < begin + 32; ++r)
    {
        sum += stage[(r * 8 + ((column >> 2) ^ (r & 7))) * 4 + (column & 3)];
        const int atom = first[r];
        if (r == begin + 31 || first[r + 1] != atom)
        {
            if (atom >= 0)
            {
                atomicAdd(target + static_cast<std::int64_t>(atom) * kFeatures + 32 * half + column,
                          sum);
            }
            sum = 0.0f;
        }
    }
    if (block_barrier)
    {
        __syncthreads();
    }
    else
    {
        __syncwarp();
    }
}

// Resident CTAs per SM times the SM count, for a persistent grid: the least of the register
// file, shared memory (227 KB a CTA can use, 1 KB reserved per CTA) and tensor memory (512
// columns) over one CTA's needs.
int pair_grid(const void* kernel, int shared_bytes, int tmem_columns)
{
    int sms = 148;
    multiprocessors(&sms);
    int per_sm = 1;
    cudaFuncAttributes attributes{};
    if (cudaFuncGetAttributes(&attributes, kernel) == cudaSuccess)
    {
        const int registers = ((attributes.numRegs * 32 + 255) / 256) * 256 * (kTile / 32);
        const int by_registers = 65536 / std::max(1, registers);
        const int by_shared =
            (228 * 1024) / (shared_bytes + static_cast<int>(attributes.sharedSizeBytes) + 1024);
        per_sm = std::max(1, std::min({by_registers, by_shared, 512 / tmem_columns}));
    }
    cudaGetLastError();
    return per_sm * std::max(1, sms);
}

}  // namespace
}  // namespace nd
