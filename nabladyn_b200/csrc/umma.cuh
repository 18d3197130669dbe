// Fifth-generation tensor cores (tcgen05) for 128 x 64 x 64 BF16 tiles: shared-memory
// operand images, the matrix and instruction descriptors, tensor-memory allocation, the MMA
// issue, its completion on an mbarrier, and tensor-memory loads. sm_100a only.
//
// Operand images. An operand is a [rows x 64] BF16 matrix, K (the reduction index) contiguous,
// stored without swizzle as 8 x 8 "core matrices" of 128 bytes (8 rows of 16 bytes): element
// (row, k) sits at byte (row / 8) * 1024 + (k / 8) * 128 + (row % 8) * 16 + (k % 8) * 2. For
// such a K-major, no-swizzle operand the descriptor's leading-dimension offset is the step
// between the two 16-byte K chunks of one instruction (128 bytes) and its stride-dimension
// offset the step between 8-row groups (1024 bytes); one instruction takes K = 16 (32 bytes),
// so the k-th of the four instructions of a K = 64 product starts 256 * k bytes in.
//
// A is the 128-row tile (one row per thread of a 128-thread CTA), B the 64-row weight image
// (row n = output feature), and D = A B^T lands in tensor memory: lane m = row m, one 32-bit
// column per output feature. Warp w may only read lanes 32 (w % 4) .. 32 (w % 4) + 31.

#pragma once

#include <cuda_bf16.h>

#include <cstdint>

namespace nd::umma {

constexpr int kRows = 128;          // M of every product
constexpr int kCols = 64;           // N and K of every product
constexpr int kImageBytes = 64 * 64 * 2;   // one 64 x 64 BF16 weight image
constexpr int kTileBytes = 128 * 64 * 2;   // one 128 x 64 BF16 row tile
constexpr int kWaitLimit = 1 << 22;        // mbarrier polls before a product counts as lost
constexpr std::uint64_t kWaitNanoseconds = 500000000;  // and at most 0.5 s of waiting

// Byte offset of element (row, k) in an operand image.
__host__ __device__ constexpr std::uint32_t image_offset(int row, int k)
{
    return static_cast<std::uint32_t>((row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 +
                                      (k & 7) * 2);
}

__device__ __forceinline__ std::uint32_t smem_address(const void* pointer)
{
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(pointer));
}

// Shared-memory matrix descriptor: start address, leading and stride byte offsets (all in
// 16-byte units), the sm_100 descriptor version (bit 46) and no swizzle (bits 61-63 = 0).
__device__ __forceinline__ std::uint64_t matrix_descriptor(std::uint32_t address)
{
    std::uint64_t descriptor = (address >> 4) & 0x3FFFu;
    descriptor |= static_cast<std::uint64_t>(128 >> 4) << 16;
    descriptor |= static_cast<std::uint64_t>(1024 >> 4) << 32;
    descriptor |= static_cast<std::uint64_t>(1) << 46;
    return descriptor;
}

// Instruction descriptor of kind::f16: D F32 (bits 4-5 = 1), A and B BF16 (bits 7-9 and
// 10-12 = 1), both K-major (bits 15, 16 = 0), N / 8 at bits 17-22, M / 16 at bits 24-28.
constexpr std::uint32_t kInstruction = (1u << 4) | (1u << 7) | (1u << 10) |
                                       ((64u >> 3) << 17) | ((128u >> 4) << 24);

// D (+)= A B^T for one K = 16 step; issued by one thread.
__device__ __forceinline__ void mma(std::uint32_t tmem, std::uint64_t a, std::uint64_t b,
                                    std::uint32_t accumulate)
{
    asm volatile(
        "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
        " tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem),
        "l"(a), "l"(b), "r"(kInstruction), "r"(accumulate));
}

// D = A B^T over K = 64: four instructions; `a` and `b` are shared-memory byte addresses.
__device__ __forceinline__ void product(std::uint32_t tmem, std::uint32_t a, std::uint32_t b)
{
#pragma unroll
    for (int step = 0; step < 4; ++step)
    {
        mma(tmem, matrix_descriptor(a + 256 * step), matrix_descriptor(b + 256 * step),
            step > 0 ? 1u : 0u);
    }
}

// Arrive on `barrier` once every product this thread issued has completed.
__device__ __forceinline__ void commit(std::uint64_t* barrier)
{
    asm volatile(
        "tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
            smem_address(barrier))
        : "memory");
}

__device__ __forceinline__ void fence_before_sync()
{
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}

__device__ __forceinline__ void fence_after_sync()
{
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}

// Makes this thread's generic-proxy shared-memory writes visible to the tensor cores.
__device__ __forceinline__ void fence_operands()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Tensor-memory allocation of `columns` (a power of two, at least 32), by one whole warp;
// the base address lands in `*slot`. Like every .sync.aligned instruction here it needs the
// warp converged, which __syncwarp() guarantees after data-dependent branches.
__device__ __forceinline__ void allocate(std::uint32_t* slot, std::uint32_t columns)
{
    __syncwarp();
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                     smem_address(slot)),
                 "r"(columns)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void deallocate(std::uint32_t tmem, std::uint32_t columns)
{
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                 "r"(columns)
                 : "memory");
}

// 32 consecutive 32-bit columns of this thread's lane, starting at `tmem` (lane in bits
// 16-31, column in bits 0-15). Follow with wait_loads() before using the values.
__device__ __forceinline__ void load32(std::uint32_t tmem, float (&out)[32])
{
    std::uint32_t r[32];
    __syncwarp();
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
        "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
        "%28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
          "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
          "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
          "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
          "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
          "=r"(r[31])
        : "r"(tmem));
#pragma unroll
    for (int i = 0; i < 32; ++i)
    {
        out[i] = __uint_as_float(r[i]);
    }
}

// 8 consecutive 32-bit columns of this thread's lane (follow with wait_loads()).
__device__ __forceinline__ void load8(std::uint32_t tmem, float (&out)[8])
{
    std::uint32_t r[8];
    __syncwarp();
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7])
                 : "r"(tmem));
#pragma unroll
    for (int i = 0; i < 8; ++i)
    {
        out[i] = __uint_as_float(r[i]);
    }
}

__device__ __forceinline__ void wait_loads()
{
    __syncwarp();
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// mbarrier with one arrival per phase (the commit).
__device__ __forceinline__ void barrier_init(std::uint64_t* barrier)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_address(barrier)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ bool barrier_test(std::uint64_t* barrier, unsigned phase)
{
    std::uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_address(barrier)), "r"(phase)
        : "memory");
    return done != 0;
}

__device__ __forceinline__ std::uint64_t nanoseconds()
{
    std::uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for `phase` of the barrier, at most kWaitLimit polls and kWaitNanoseconds (a poll
// may suspend the thread for a while); false when it gave up.
__device__ __forceinline__ bool barrier_wait(std::uint64_t* barrier, unsigned phase)
{
    const std::uint64_t start = nanoseconds();
    for (int poll = 0; poll < kWaitLimit; ++poll)
    {
        if (barrier_test(barrier, phase))
        {
            return true;
        }
        if (nanoseconds() - start > kWaitNanoseconds)
        {
            return false;
        }
    }
    return false;
}

// Eight floats as eight BF16 (round to nearest even) in one 16-byte word.
__device__ __forceinline__ uint4 pack8(const float* v)
{
    uint4 word;
    __nv_bfloat162 p0 = __floats2bfloat162_rn(v[0], v[1]);
    __nv_bfloat162 p1 = __floats2bfloat162_rn(v[2], v[3]);
    __nv_bfloat162 p2 = __floats2bfloat162_rn(v[4], v[5]);
    __nv_bfloat162 p3 = __floats2bfloat162_rn(v[6], v[7]);
    word.x = *reinterpret_cast<std::uint32_t*>(&p0);
    word.y = *reinterpret_cast<std::uint32_t*>(&p1);
    word.z = *reinterpret_cast<std::uint32_t*>(&p2);
    word.w = *reinterpret_cast<std::uint32_t*>(&p3);
    return word;
}

// Stores 8 values as columns 8c .. 8c + 7 of `row` of a row tile.
__device__ __forceinline__ void store8(unsigned char* tile, int row, int c, const float* v)
{
    *reinterpret_cast<uint4*>(tile + image_offset(row, 8 * c)) = pack8(v);
}

}  // namespace nd::umma
