// SchNet energy, forces and virial with the dense layers on BF16 tcgen05 tensor cores.
//
// The model is src/nabladyn/potential/_schnet/_potential.py:45-208 (64 features, K <= 64
// Gaussians, any number of blocks). The reference differentiates it with autograd
// (src/nabladyn/quantity.py:93-117); here the reverse pass is written out:
//
//   forward, per block b:  v = x A^T;  per pair p = (a, b) within the cutoff
//       z1 = g(r) B1^T + b1,  f_raw = ssp(z1) B2^T + b2,  f = f_raw C(r),
//       m_a += f * v_b,  m_b += f * v_a;
//     h = m D1^T + d1,  x += ssp(h) D2^T + d2;  E = sum_i ssp(x R1^T + e1) R2^T + e2
//   reverse:  G = dE/dx = (sigmoid(y) * R2) R1;  per block, last first:
//     Gh = (G D2) * sigmoid(h),  Gm = Gh D1;  per pair  Gf = Gm_a * v_b + Gm_b * v_a,
//       Gv_b += f * Gm_a,  Gv_a += f * Gm_b,
//       dE/dr += C'(r) (Gf . f_raw) + [((Gf C) B2 * sigmoid(z1)) B1] . g'(r);
//     G += Gv A
//   F_a -= dE/dr d / r,  F_b += dE/dr d / r,  W -= dE/dr d d^T / r.
//
// Every 64 x 64 product runs as a 128-row tile on the tensor cores: a [128 x 64] BF16 row
// tile (one pair or one atom per thread of a 128-thread CTA) times a BF16 weight image,
// FP32 accumulation in tensor memory (umma.cuh). The per-pair products (filter network
// forward, and its reverse) run in persistent CTAs that keep their weight images in shared
// memory; the atom-wise products in one CTA per 128 atoms. Everything else is FP32, the
// energy and virial sums FP64 in a fixed order. The feature rows the pair kernels gather
// (v and Gm) are stored in BF16; messages, their reverse and forces are summed in FP32.

#include "schnet.cuh"

namespace nd {
namespace {

// ---------------------------------------------------------------------------------------
// Pairs within the cutoff, compacted: (a, b) and (d, r), d = r_a - r_b of the minimum image
// as src/nabladyn/space.py:11-19 rounds it.

// Whether column c is a pair within the cutoff, with its atoms and geometry.
__device__ __forceinline__ bool column_pair(const float* __restrict__ positions,
                                            const float* __restrict__ cell,
                                            const std::int32_t* __restrict__ pairs,
                                            std::int64_t columns, std::int64_t c,
                                            std::int64_t atoms, float cutoff_squared, int2& ab,
                                            float4& g, int* counters)
{
    if (c >= columns)
    {
        return false;
    }
    ab = make_int2(pairs[c], pairs[columns + c]);
    if (ab.x == ab.y)
    {
        return false;
    }
    if (ab.x < 0 || ab.y < 0 || ab.x >= atoms || ab.y >= atoms)
    {
        atomicOr(counters + 1, kBadPair);
        return false;
    }
    float d[3];
#pragma unroll
    for (int axis = 0; axis < 3; ++axis)
    {
        const float length = cell[axis];
        const float left = positions[3 * ab.x + axis];
        const float right = positions[3 * ab.y + axis];
        const float raw = left - right;
        const float half = 0.5f * length;
        d[axis] = (left - (raw > half ? length : 0.0f)) - (right - (raw < -half ? length : 0.0f));
    }
    const float squared = __fadd_rn(__fadd_rn(__fmul_rn(d[0], d[0]), __fmul_rn(d[1], d[1])),
                                    __fmul_rn(d[2], d[2]));
    g = make_float4(d[0], d[1], d[2], sqrtf(squared));
    return squared < cutoff_squared;
}

// The compaction keeps the list's column order (count per block, scan, write), so the pairs
// of one first atom stay contiguous, as the list stores them.
__global__ void __launch_bounds__(kThreads) compact_count_kernel(
    const float* __restrict__ positions, const float* __restrict__ cell,
    const std::int32_t* __restrict__ pairs, std::int64_t columns, std::int64_t atoms,
    float cutoff_squared, int* __restrict__ block_counts, int* __restrict__ counters)
{
    int2 ab;
    float4 g;
    const std::int64_t c = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool keep = column_pair(positions, cell, pairs, columns, c, atoms, cutoff_squared, ab,
                                  g, counters);
    const int count = __syncthreads_count(keep);
    if (threadIdx.x == 0)
    {
        block_counts[blockIdx.x] = count;
    }
}

constexpr int kScanThreads = 1024;

__global__ void __launch_bounds__(kScanThreads) compact_scan_kernel(
    const int* __restrict__ block_counts, int blocks, int* __restrict__ block_offsets,
    int* __restrict__ counters)
{
    __shared__ int warp_totals[kScanThreads / kWarp];
    __shared__ int carry;
    if (threadIdx.x == 0)
    {
        carry = 0;
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x / 32;
    for (int base = 0; base < blocks; base += kScanThreads)
    {
        const int i = base + threadIdx.x;
        const int value = i < blocks ? block_counts[i] : 0;
        int inclusive = value;
#pragma unroll
        for (int offset = 1; offset < 32; offset *= 2)
        {
            const int other = __shfl_up_sync(kFullMask, inclusive, offset);
            inclusive += lane >= offset ? other : 0;
        }
        if (lane == 31)
        {
            warp_totals[warp] = inclusive;
        }
        __syncthreads();
        if (warp == 0)
        {
            int total = warp_totals[lane];
#pragma unroll
            for (int offset = 1; offset < 32; offset *= 2)
            {
                const int other = __shfl_up_sync(kFullMask, total, offset);
                total += lane >= offset ? other : 0;
            }
            warp_totals[lane] = total;  // inclusive over warps
        }
        __syncthreads();
        const int before = (warp > 0 ? warp_totals[warp - 1] : 0) + inclusive - value;
        if (i < blocks)
        {
            block_offsets[i] = carry + before;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            carry += warp_totals[kScanThreads / kWarp - 1];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0)
    {
        counters[0] = carry;
    }
}

__global__ void __launch_bounds__(kThreads) compact_write_kernel(
    const float* __restrict__ positions, const float* __restrict__ cell,
    const std::int32_t* __restrict__ pairs, std::int64_t columns, std::int64_t atoms,
    float cutoff_squared, const int* __restrict__ block_offsets, int2* __restrict__ kept,
    float4* __restrict__ geometry, int* __restrict__ counters)
{
    __shared__ int warp_base[kThreads / kWarp];
    int2 ab = make_int2(0, 0);
    float4 g = make_float4(0.f, 0.f, 0.f, 0.f);
    const std::int64_t c = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool keep = column_pair(positions, cell, pairs, columns, c, atoms, cutoff_squared, ab,
                                  g, counters);
    const unsigned ballot = __ballot_sync(kFullMask, keep);
    const int lane = threadIdx.x & 31, warp = threadIdx.x / 32;
    if (lane == 0)
    {
        warp_base[warp] = __popc(ballot);
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        int running = block_offsets[blockIdx.x];
        for (int w = 0; w < kThreads / kWarp; ++w)
        {
            const int count = warp_base[w];
            warp_base[w] = running;
            running += count;
        }
    }
    __syncthreads();
    if (keep)
    {
        const int slot = warp_base[warp] + __popc(ballot & ((1u << lane) - 1u));
        kept[slot] = ab;
        geometry[slot] = g;
    }
}

// x = embedding[type], v0 = (embedding A0^T)[type].
__global__ void embed_kernel(const std::int64_t* __restrict__ types, std::int64_t atoms,
                             const float* __restrict__ table, const float* __restrict__ table_v,
                             float* __restrict__ x, float* __restrict__ v)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= atoms * 16)
    {
        return;
    }
    const std::int64_t atom = i / 16;
    const int q = static_cast<int>(i % 16);
    const std::int64_t type = types[atom];
    reinterpret_cast<float4*>(x)[i] = reinterpret_cast<const float4*>(table)[type * 16 + q];
    const float4 value = reinterpret_cast<const float4*>(table_v)[type * 16 + q];
    reinterpret_cast<uint2*>(v)[i] = make_uint2(pack2(value.x, value.y), pack2(value.z, value.w));
}

struct PairPass
{
    const int2* pairs;
    const float4* geometry;
    int* counters;
    const unsigned char* images;  // this block's ten images
    const float* b1;
    const float* b2;
    const float* v;           // [N][64] BF16: this block's x A^T
    float* m;                 // forward: messages
    const float* grad_m;      // reverse: Gm, [N][64] BF16
    float* grad_v;            // reverse: Gv (null for the first block)
    float* dedr;              // reverse: per-pair dE/dr over the blocks so far
    float* forces;            // reverse, last pass: F (null when not wanted)
    double* virial;           // reverse, last pass: per-CTA partials [gridDim.x][9]
    float width;              // Gaussian spacing D
    float phase;              // pi / r_c
    int gaussians;
    int first;                // reverse: the first pass (last block) starts dE/dr
    int last;                 // reverse: the last pass (block 0) applies forces and virial
};

// Shared memory of the pair passes: weight images, one row tile (each product's operand
// replaces the last once that product completed), biases, barrier and tensor-memory slot. The
// reverse pass's 16 KB run stage overlays its B1 and B1^T images, which only the first and
// the last product of a tile read; they are copied in again (from L2) after the stage was used,
// so four CTAs fit an SM.
constexpr int kPairForwardShared = 2 * umma::kImageBytes + umma::kTileBytes + 2 * 256 + 64;
constexpr int kPairReverseShared = 4 * umma::kImageBytes + umma::kTileBytes + 2 * 256 + 64;

__global__ void __launch_bounds__(kTile, 6) pair_forward_kernel(PairPass a)
{
    extern __shared__ __align__(1024) unsigned char shared[];
    unsigned char* image_b1 = shared;
    unsigned char* image_b2 = image_b1 + umma::kImageBytes;
    unsigned char* basis = image_b2 + umma::kImageBytes;
    unsigned char* work = basis;  // the basis is dead once the first product completed
    float* bias1 = reinterpret_cast<float*>(work + umma::kTileBytes);
    float* bias2 = bias1 + kFeatures;
    auto* barrier = reinterpret_cast<std::uint64_t*>(bias2 + kFeatures);
    auto* slot = reinterpret_cast<std::uint32_t*>(barrier + 1);

    copy_bytes(image_b1, a.images + kB1 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b2, a.images + kB2 * umma::kImageBytes, umma::kImageBytes);
    if (threadIdx.x < kFeatures)
    {
        bias1[threadIdx.x] = a.b1[threadIdx.x];
        bias2[threadIdx.x] = a.b2[threadIdx.x];
    }
    Cores cores;
    cores.open(barrier, slot, 64, a.counters, 1);
    const int count = *reinterpret_cast<volatile int*>(a.counters);
    const uint4* v8 = reinterpret_cast<const uint4*>(a.v);
    float4* m4 = reinterpret_cast<float4*>(a.m);
    __shared__ int tile_first[kTile];

    // Each tile's pair records are loaded one tile ahead, so their latency hides behind the
    // previous tile's products.
    int2 next_ab = make_int2(0, 0);
    float4 next_g = make_float4(0.f, 0.f, 0.f, 1.f);
    if (blockIdx.x * kTile + static_cast<int>(threadIdx.x) < count)
    {
        next_ab = a.pairs[blockIdx.x * kTile + threadIdx.x];
        next_g = a.geometry[blockIdx.x * kTile + threadIdx.x];
    }
    for (int tile = blockIdx.x; tile * kTile < count; tile += gridDim.x)
    {
        const int p = tile * kTile + threadIdx.x;
        const bool live = p < count;
        const int2 ab = next_ab;
        const float4 g = next_g;
        const int ahead = p + gridDim.x * kTile;
        next_ab = ahead < count ? a.pairs[ahead] : make_int2(0, 0);
        next_g = ahead < count ? a.geometry[ahead] : make_float4(0.f, 0.f, 0.f, 1.f);
        const float envelope = live ? 0.5f * (__cosf(g.w * a.phase) + 1.0f) : 0.0f;
        tile_first[threadIdx.x] = live ? ab.x : -1;
        cores.tile_index = tile;
        store_basis(basis, g.w / a.width, a.gaussians, live);
        if (!cores.run(0, basis, image_b1, 1))
        {
            break;
        }
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            float z[32];
            umma::load32(cores.tmem + 32 * half, z);
            umma::wait_loads();
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                float s[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                {
                    s[e] = softplus_shifted(z[8 * c + e] + bias1[32 * half + 8 * c + e]);
                }
                umma::store8(work, threadIdx.x, 4 * half + c, s);
            }
        }
        if (!cores.run(0, work, image_b2, 2))
        {
            break;
        }
        float* stage = reinterpret_cast<float*>(work);  // free once the second product is done
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
#pragma unroll
            for (int batch = 0; batch < 4; batch += kGatherBatch)
            {
                // The batch's gathers first, so their latencies overlap; dead rows read atom 0
                // and contribute zeros (their envelope is zero).
                uint4 raw[kGatherBatch][2];
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int k = 32 * half + 8 * (batch + i);
                    raw[i][0] = __ldg(v8 + 8 * static_cast<std::int64_t>(ab.x) + k / 8);
                    raw[i][1] = __ldg(v8 + 8 * static_cast<std::int64_t>(ab.y) + k / 8);
                }
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int c = batch + i;
                    const int k = 32 * half + 8 * c;
                    float f[8];
                    umma::load8(cores.tmem + k, f);
                    umma::wait_loads();
                    float va[8], vb[8], filter[8];
                    widen8(raw[i][0], va);
                    widen8(raw[i][1], vb);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                    {
                        filter[j] = (f[j] + bias2[k + j]) * envelope;
                    }
                    if (live)
                    {
                        const std::int64_t gb = 8 * static_cast<std::int64_t>(ab.y) + k / 8;
                        atomicAdd(m4 + 2 * gb, make_float4(filter[0] * va[0], filter[1] * va[1],
                                                           filter[2] * va[2], filter[3] * va[3]));
                        atomicAdd(m4 + 2 * gb + 1,
                                  make_float4(filter[4] * va[4], filter[5] * va[5],
                                              filter[6] * va[6], filter[7] * va[7]));
                    }
                    put_run_part(stage, 2 * c, make_float4(filter[0] * vb[0], filter[1] * vb[1],
                                                           filter[2] * vb[2], filter[3] * vb[3]));
                    put_run_part(stage, 2 * c + 1,
                                 make_float4(filter[4] * vb[4], filter[5] * vb[5],
                                             filter[6] * vb[6], filter[7] * vb[7]));
                }
            }
            sum_runs(stage, tile_first, a.m, half, half == 1);  // the next basis overwrites it
        }
    }
    cores.close(64);
}

__global__ void __launch_bounds__(kTile, 4) pair_reverse_kernel(PairPass a)
{
    extern __shared__ __align__(1024) unsigned char shared[];
    unsigned char* image_b1 = shared;
    unsigned char* image_b1t = image_b1 + umma::kImageBytes;
    unsigned char* image_b2 = image_b1t + umma::kImageBytes;
    unsigned char* image_b2t = image_b2 + umma::kImageBytes;
    unsigned char* basis = image_b2t + umma::kImageBytes;
    unsigned char* work = basis;  // each operand replaces the last once its product completed
    float* stage = reinterpret_cast<float*>(image_b1);  // Gv runs, 16 KB over B1 and B1^T
    float* bias1 = reinterpret_cast<float*>(work + umma::kTileBytes);
    float* bias2 = bias1 + kFeatures;
    auto* barrier = reinterpret_cast<std::uint64_t*>(bias2 + kFeatures);
    auto* slot = reinterpret_cast<std::uint32_t*>(barrier + 1);

    copy_bytes(image_b1, a.images + kB1 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b2, a.images + kB2 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b2t, a.images + kB2T * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b1t, a.images + kB1T * umma::kImageBytes, umma::kImageBytes);
    if (threadIdx.x < kFeatures)
    {
        bias1[threadIdx.x] = a.b1[threadIdx.x];
        bias2[threadIdx.x] = a.b2[threadIdx.x];
    }
    // Columns 0-63 keep z1 - b1 for the whole tile; 64-127 take the other products in turn.
    Cores cores;
    cores.open(barrier, slot, 128, a.counters, 2);
    const int count = *reinterpret_cast<volatile int*>(a.counters);
    const uint4* v8 = reinterpret_cast<const uint4*>(a.v);
    const uint4* gm8 = reinterpret_cast<const uint4*>(a.grad_m);
    float4* gv4 = reinterpret_cast<float4*>(a.grad_v);
    __shared__ int tile_first[kTile];
    double w[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // xx yy zz xy xz yz

    // Each tile's pair records are loaded one tile ahead (see pair_forward_kernel).
    int2 next_ab = make_int2(0, 0);
    float4 next_g = make_float4(0.f, 0.f, 0.f, 1.f);
    if (blockIdx.x * kTile + static_cast<int>(threadIdx.x) < count)
    {
        next_ab = a.pairs[blockIdx.x * kTile + threadIdx.x];
        next_g = a.geometry[blockIdx.x * kTile + threadIdx.x];
    }
    for (int tile = blockIdx.x; tile * kTile < count; tile += gridDim.x)
    {
        const int p = tile * kTile + threadIdx.x;
        const bool live = p < count;
        const int2 ab = next_ab;
        const float4 g = next_g;
        const int ahead = p + gridDim.x * kTile;
        next_ab = ahead < count ? a.pairs[ahead] : make_int2(0, 0);
        next_g = ahead < count ? a.geometry[ahead] : make_float4(0.f, 0.f, 0.f, 1.f);
        float sine, cosine;
        __sincosf(g.w * a.phase, &sine, &cosine);
        const float envelope = live ? 0.5f * (cosine + 1.0f) : 0.0f;
        const float slope = live ? -0.5f * a.phase * sine : 0.0f;
        const float t = g.w / a.width;
        tile_first[threadIdx.x] = live ? ab.x : -1;
        cores.tile_index = tile;
        if (gv4 != nullptr && tile != blockIdx.x)
        {
            // the previous tile's run stage overwrote B1
            copy_bytes(image_b1, a.images + kB1 * umma::kImageBytes, umma::kImageBytes);
        }
        store_basis(basis, t, a.gaussians, live);
        if (!cores.run(0, basis, image_b1, 1))
        {
            break;
        }
        // ssp(z1) into the work tile; z1 - b1 stays in columns 0-63.
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            float z[32];
            umma::load32(cores.tmem + 32 * half, z);
            umma::wait_loads();
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                float s[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                {
                    s[e] = softplus_shifted(z[8 * c + e] + bias1[32 * half + 8 * c + e]);
                }
                umma::store8(work, threadIdx.x, 4 * half + c, s);
            }
        }
        if (!cores.run(64, work, image_b2, 2))
        {
            break;
        }
        // f_raw, Gf = Gm_a v_b + Gm_b v_a, C' Gf . f_raw, Gv, and Gf C into the work tile.
        float along = 0.0f;
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
#pragma unroll
            for (int batch = 0; batch < 4; batch += kGatherBatch)
            {
                // The batch's gathers first; dead rows read atom 0 and contribute zeros.
                uint4 raw[kGatherBatch][4];
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int k = 32 * half + 8 * (batch + i);
                    const std::int64_t ga = 8 * static_cast<std::int64_t>(ab.x) + k / 8;
                    const std::int64_t gb = 8 * static_cast<std::int64_t>(ab.y) + k / 8;
                    raw[i][0] = __ldg(v8 + ga);
                    raw[i][1] = __ldg(v8 + gb);
                    raw[i][2] = __ldg(gm8 + ga);
                    raw[i][3] = __ldg(gm8 + gb);
                }
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int c = batch + i;
                    const int k = 32 * half + 8 * c;
                    float f[8];
                    umma::load8(cores.tmem + 64 + k, f);
                    umma::wait_loads();
                    float va[8], vb[8], ma[8], mb[8];
                    widen8(raw[i][0], va);
                    widen8(raw[i][1], vb);
                    widen8(raw[i][2], ma);
                    widen8(raw[i][3], mb);
                    float scaled[8], to_first[8], to_second[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                    {
                        const float gf = ma[j] * vb[j] + mb[j] * va[j];
                        const float raw_filter = f[j] + bias2[k + j];
                        along += gf * raw_filter;
                        to_second[j] = raw_filter * envelope * ma[j];
                        to_first[j] = raw_filter * envelope * mb[j];
                        scaled[j] = gf * envelope;
                    }
                    if (gv4 != nullptr)
                    {
                        if (live)
                        {
                            const std::int64_t gb = 8 * static_cast<std::int64_t>(ab.y) + k / 8;
                            atomicAdd(gv4 + 2 * gb, make_float4(to_second[0], to_second[1],
                                                                to_second[2], to_second[3]));
                            atomicAdd(gv4 + 2 * gb + 1, make_float4(to_second[4], to_second[5],
                                                                    to_second[6], to_second[7]));
                        }
                        put_run_part(stage, 2 * c, make_float4(to_first[0], to_first[1],
                                                               to_first[2], to_first[3]));
                        put_run_part(stage, 2 * c + 1, make_float4(to_first[4], to_first[5],
                                                                   to_first[6], to_first[7]));
                    }
                    umma::store8(work, threadIdx.x, 4 * half + c, scaled);
                }
            }
            if (gv4 != nullptr)
            {
                sum_runs(stage, tile_first, a.grad_v, half, half == 1);  // B1^T is copied over it
            }
        }
        if (!cores.run(64, work, image_b2t, 3))
        {
            break;
        }
        // ((Gf C) B2) * sigmoid(z1) into the work tile.
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            float q[32];
            float z[32];
            umma::load32(cores.tmem + 64 + 32 * half, q);
            umma::load32(cores.tmem + 32 * half, z);
            umma::wait_loads();
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                float s[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                {
                    s[e] = q[8 * c + e] * sigmoid(z[8 * c + e] + bias1[32 * half + 8 * c + e]);
                }
                umma::store8(work, threadIdx.x, 4 * half + c, s);
            }
        }
        if (gv4 != nullptr)
        {
            // this tile's run stage overwrote B1^T
            copy_bytes(image_b1t, a.images + kB1T * umma::kImageBytes, umma::kImageBytes);
        }
        if (!cores.run(64, work, image_b1t, 4))
        {
            break;
        }
        // dE/dr = C' Gf . f_raw + sum_k [..]_k g_k', g_k' = -g_k (r / D - k) / D, with the
        // Gaussians evaluated again in FP32 (columns k >= K hold zeros).
        float through = 0.0f;
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            float u[32];
            umma::load32(cores.tmem + 64 + 32 * half, u);
            umma::wait_loads();
#pragma unroll
            for (int e = 0; e < 32; ++e)
            {
                const int k = 32 * half + e;
                const float offset = t - static_cast<float>(k);
                const float g = k < a.gaussians ? __expf(-0.5f * offset * offset) : 0.0f;
                through -= u[e] * g * offset;
            }
        }
        if (live)
        {
            float total = slope * along + through / a.width;
            if (!a.first)
            {
                total += a.dedr[p];
            }
            if (!a.last)
            {
                a.dedr[p] = total;
            }
            else
            {
                const float scale = total / g.w;
                const float ux = scale * g.x, uy = scale * g.y, uz = scale * g.z;
                if (a.forces != nullptr)
                {
                    atomicAdd(a.forces + 3 * static_cast<std::int64_t>(ab.x), -ux);
                    atomicAdd(a.forces + 3 * static_cast<std::int64_t>(ab.x) + 1, -uy);
                    atomicAdd(a.forces + 3 * static_cast<std::int64_t>(ab.x) + 2, -uz);
                    atomicAdd(a.forces + 3 * static_cast<std::int64_t>(ab.y), ux);
                    atomicAdd(a.forces + 3 * static_cast<std::int64_t>(ab.y) + 1, uy);
                    atomicAdd(a.forces + 3 * static_cast<std::int64_t>(ab.y) + 2, uz);
                }
                w[0] -= static_cast<double>(ux) * g.x;
                w[1] -= static_cast<double>(uy) * g.y;
                w[2] -= static_cast<double>(uz) * g.z;
                w[3] -= static_cast<double>(ux) * g.y;
                w[4] -= static_cast<double>(ux) * g.z;
                w[5] -= static_cast<double>(uy) * g.z;
            }
        }
    }
    if (a.last && a.virial != nullptr)
    {
        __shared__ double sums[4][6];
#pragma unroll
        for (int k = 0; k < 6; ++k)
        {
            const double s = warp_sum(w[k]);
            if ((threadIdx.x & 31) == 0)
            {
                sums[threadIdx.x / 32][k] = s;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double t6[6];
            for (int k = 0; k < 6; ++k)
            {
                t6[k] = ((sums[0][k] + sums[1][k]) + sums[2][k]) + sums[3][k];
            }
            double* out = a.virial + 9 * static_cast<std::int64_t>(blockIdx.x);
            out[0] = t6[0];
            out[4] = t6[1];
            out[8] = t6[2];
            out[1] = out[3] = t6[3];
            out[2] = out[6] = t6[4];
            out[5] = out[7] = t6[5];
        }
    }
    cores.close(128);
}

struct AtomPass
{
    std::int64_t atoms;
    const unsigned char* images;       // this block's images
    const unsigned char* next_images;  // forward: the next block's (for v); reverse: its (for Gv A)
    const float* d1;
    const float* d2;
    const float* m;        // forward
    float* h;              // forward: writes; reverse: reads
    float* x;              // forward: updated in place
    float* v_next;         // forward: the next block's v in BF16 (null for the last block)
    const float* readout;  // forward, last block: R1, e1, R2, e2
    float* grad;           // forward, last block: writes dE/dx; reverse: reads, updates
    const float* grad_v;   // reverse: Gv of the next block (null for the last block)
    float* grad_m;         // reverse: writes Gm in BF16
    double* energy;        // forward, last block: per-CTA partials
    int* counters;
};

constexpr int kAtomShared = 3 * umma::kImageBytes + umma::kTileBytes +
                            (kHidden * kFeatures + 3 * kHidden) * 4 + 2 * 256 + 64;

__device__ __forceinline__ void load_row(const float* source, std::int64_t row, bool live, float* out)
{
    const float4* s4 = reinterpret_cast<const float4*>(source) + 16 * row;
#pragma unroll
    for (int q = 0; q < 16; ++q)
    {
        const float4 value = live ? s4[q] : make_float4(0.f, 0.f, 0.f, 0.f);
        out[4 * q] = value.x;
        out[4 * q + 1] = value.y;
        out[4 * q + 2] = value.z;
        out[4 * q + 3] = value.w;
    }
}

__device__ __forceinline__ void store_tile_row(unsigned char* tile, const float* values)
{
#pragma unroll
    for (int c = 0; c < 8; ++c)
    {
        umma::store8(tile, threadIdx.x, c, values + 8 * c);
    }
}

// The 64 accumulator columns of this thread's row.
__device__ __forceinline__ void load_row_tmem(std::uint32_t tmem, float* out)
{
    float part[32];
    umma::load32(tmem, part);
    umma::wait_loads();
#pragma unroll
    for (int i = 0; i < 32; ++i)
    {
        out[i] = part[i];
    }
    umma::load32(tmem + 32, part);
    umma::wait_loads();
#pragma unroll
    for (int i = 0; i < 32; ++i)
    {
        out[32 + i] = part[i];
    }
}

__device__ __forceinline__ void store_row(float* target, std::int64_t row, const float* values)
{
    float4* t4 = reinterpret_cast<float4*>(target) + 16 * row;
#pragma unroll
    for (int q = 0; q < 16; ++q)
    {
        t4[q] = make_float4(values[4 * q], values[4 * q + 1], values[4 * q + 2], values[4 * q + 3]);
    }
}

__device__ __forceinline__ void store_row_bf16(float* target, std::int64_t row, const float* values)
{
    uint4* t4 = reinterpret_cast<uint4*>(target) + 8 * row;
#pragma unroll
    for (int q = 0; q < 8; ++q)
    {
        t4[q] = make_uint4(pack2(values[8 * q], values[8 * q + 1]),
                           pack2(values[8 * q + 2], values[8 * q + 3]),
                           pack2(values[8 * q + 4], values[8 * q + 5]),
                           pack2(values[8 * q + 6], values[8 * q + 7]));
    }
}

// h = m D1^T + d1, x += ssp(h) D2^T + d2, then v' = x A'^T, or on the last block the readout:
// e = ssp(x R1^T + e1) R2^T + e2 and dE/dx.
template <bool kLast>
__global__ void __launch_bounds__(kTile) atom_forward_kernel(AtomPass a)
{
    extern __shared__ __align__(1024) unsigned char shared[];
    unsigned char* image_d1 = shared;
    unsigned char* image_d2 = image_d1 + umma::kImageBytes;
    unsigned char* image_a = image_d2 + umma::kImageBytes;
    unsigned char* tile = image_a + umma::kImageBytes;
    float* readout = reinterpret_cast<float*>(tile + umma::kTileBytes);
    float* bias1 = readout + kHidden * kFeatures + 3 * kHidden;
    float* bias2 = bias1 + kFeatures;
    auto* barrier = reinterpret_cast<std::uint64_t*>(bias2 + kFeatures);
    auto* slot = reinterpret_cast<std::uint32_t*>(barrier + 1);

    copy_bytes(image_d1, a.images + kD1 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_d2, a.images + kD2 * umma::kImageBytes, umma::kImageBytes);
    if (!kLast)
    {
        copy_bytes(image_a, a.next_images + kA * umma::kImageBytes, umma::kImageBytes);
    }
    else
    {
        for (int i = threadIdx.x; i < kHidden * kFeatures + 3 * kHidden; i += kTile)
        {
            readout[i] = a.readout[i];
        }
    }
    if (threadIdx.x < kFeatures)
    {
        bias1[threadIdx.x] = a.d1[threadIdx.x];
        bias2[threadIdx.x] = a.d2[threadIdx.x];
    }
    Cores cores;
    cores.open(barrier, slot, 64, a.counters, 3);
    cores.tile_index = blockIdx.x;
    const std::int64_t row = static_cast<std::int64_t>(blockIdx.x) * kTile + threadIdx.x;
    const bool live = row < a.atoms;
    double energy = 0.0;
    bool ok = true;
    {
        float values[kFeatures];
        load_row(a.m, row, live, values);
        store_tile_row(tile, values);
        ok = cores.run(0, tile, image_d1, 1);
        if (ok)
        {
            load_row_tmem(cores.tmem, values);
#pragma unroll
            for (int k = 0; k < kFeatures; ++k)
            {
                values[k] += bias1[k];
            }
            if (live)
            {
                store_row(a.h, row, values);
            }
#pragma unroll
            for (int k = 0; k < kFeatures; ++k)
            {
                values[k] = softplus_shifted(values[k]);
            }
            store_tile_row(tile, values);
            ok = cores.run(0, tile, image_d2, 2);
        }
        if (ok)
        {
            float x[kFeatures];
            load_row(a.x, row, live, x);
            load_row_tmem(cores.tmem, values);
#pragma unroll
            for (int k = 0; k < kFeatures; ++k)
            {
                x[k] += values[k] + bias2[k];
            }
            if (!kLast)
            {
                if (live)
                {
                    store_row(a.x, row, x);
                }
                store_tile_row(tile, x);
                ok = cores.run(0, tile, image_a, 3);
                if (ok)
                {
                    load_row_tmem(cores.tmem, values);
                    if (live)
                    {
                        store_row_bf16(a.v_next, row, values);
                    }
                }
            }
            else
            {
                const float* r1 = readout;
                const float* e1 = readout + kHidden * kFeatures;
                const float* r2 = e1 + kHidden;
                const float e2 = r2[kHidden];
                float grad[kFeatures];
#pragma unroll
                for (int k = 0; k < kFeatures; ++k)
                {
                    grad[k] = 0.0f;
                }
                float e = e2;
                for (int j = 0; j < kHidden; ++j)
                {
                    float y = e1[j];
#pragma unroll
                    for (int k = 0; k < kFeatures; ++k)
                    {
                        y = fmaf(x[k], r1[j * kFeatures + k], y);
                    }
                    e += softplus_shifted(y) * r2[j];
                    const float s = sigmoid(y) * r2[j];
#pragma unroll
                    for (int k = 0; k < kFeatures; ++k)
                    {
                        grad[k] = fmaf(s, r1[j * kFeatures + k], grad[k]);
                    }
                }
                if (live)
                {
                    store_row(a.grad, row, grad);
                    energy = e;
                }
            }
        }
    }
    if (kLast)
    {
        __shared__ double sums[4];
        const double s = warp_sum(energy);
        if ((threadIdx.x & 31) == 0)
        {
            sums[threadIdx.x / 32] = s;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            a.energy[blockIdx.x] = ((sums[0] + sums[1]) + sums[2]) + sums[3];
        }
    }
    cores.close(64);
}

// Reverse of one block's atom-wise layers: G += Gv' A' (the next block's messages), then
// Gh = (G D2) * sigmoid(h) and Gm = Gh D1.
__global__ void __launch_bounds__(kTile) atom_reverse_kernel(AtomPass a)
{
    extern __shared__ __align__(1024) unsigned char shared[];
    unsigned char* image_d2t = shared;
    unsigned char* image_d1t = image_d2t + umma::kImageBytes;
    unsigned char* image_at = image_d1t + umma::kImageBytes;
    unsigned char* tile = image_at + umma::kImageBytes;
    auto* barrier = reinterpret_cast<std::uint64_t*>(tile + umma::kTileBytes);
    auto* slot = reinterpret_cast<std::uint32_t*>(barrier + 1);

    copy_bytes(image_d2t, a.images + kD2T * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_d1t, a.images + kD1T * umma::kImageBytes, umma::kImageBytes);
    const bool chained = a.grad_v != nullptr;
    if (chained)
    {
        copy_bytes(image_at, a.next_images + kAT * umma::kImageBytes, umma::kImageBytes);
    }
    Cores cores;
    cores.open(barrier, slot, 64, a.counters, 4);
    cores.tile_index = blockIdx.x;
    const std::int64_t row = static_cast<std::int64_t>(blockIdx.x) * kTile + threadIdx.x;
    const bool live = row < a.atoms;
    bool ok = true;
    float grad[kFeatures];
    float values[kFeatures];
    load_row(a.grad, row, live, grad);
    if (chained)
    {
        load_row(a.grad_v, row, live, values);
        store_tile_row(tile, values);
        ok = cores.run(0, tile, image_at, 1);
        if (ok)
        {
            load_row_tmem(cores.tmem, values);
#pragma unroll
            for (int k = 0; k < kFeatures; ++k)
            {
                grad[k] += values[k];
            }
            if (live)
            {
                store_row(a.grad, row, grad);
            }
        }
    }
    if (ok)
    {
        store_tile_row(tile, grad);
        ok = cores.run(0, tile, image_d2t, 2);
    }
    if (ok)
    {
        float h[kFeatures];
        load_row(a.h, row, live, h);
        load_row_tmem(cores.tmem, values);
#pragma unroll
        for (int k = 0; k < kFeatures; ++k)
        {
            values[k] *= sigmoid(h[k]);
        }
        store_tile_row(tile, values);
        ok = cores.run(0, tile, image_d1t, 3);
    }
    if (ok)
    {
        load_row_tmem(cores.tmem, values);
        if (live)
        {
            store_row_bf16(a.grad_m, row, values);
        }
    }
    cores.close(64);
}

// E and W from the per-CTA partials in a fixed order; the status word out.
__global__ void finalize_kernel(const double* __restrict__ energy_partials, int energy_count,
                                const double* __restrict__ virial_partials, int virial_count,
                                double* energy, double* virial)
{
    __shared__ double sums[10][8];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x / 32;
    double e = 0.0;
    for (int i = threadIdx.x; i < energy_count; i += blockDim.x)
    {
        e += energy_partials[i];
    }
    e = warp_sum(e);
    if (lane == 0)
    {
        sums[0][warp] = e;
    }
    for (int c = 0; c < 9; ++c)
    {
        double s = 0.0;
        for (int i = threadIdx.x; i < virial_count; i += blockDim.x)
        {
            s += virial_partials[9 * i + c];
        }
        s = warp_sum(s);
        if (lane == 0)
        {
            sums[1 + c][warp] = s;
        }
    }
    __syncthreads();
    if (threadIdx.x < 10)
    {
        double total = 0.0;
        for (int w = 0; w < 8; ++w)
        {
            total += sums[threadIdx.x][w];
        }
        if (threadIdx.x == 0)
        {
            if (energy != nullptr)
            {
                energy[0] = total;
            }
        }
        else if (virial != nullptr)
        {
            virial[threadIdx.x - 1] = total;
        }
    }
}

}  // namespace
}  // namespace nd

extern "C" {

int64_t nd_schnet_weight_bytes(int32_t interactions, int32_t num_types)
{
    if (interactions < 1 || num_types < 1)
    {
        return -1;
    }
    return nd::WeightLayout(interactions, num_types).total;
}

int64_t nd_schnet_workspace_bytes(int64_t num_atoms, int64_t num_columns, int32_t interactions)
{
    if (num_atoms < 1 || num_columns < 0 || interactions < 1)
    {
        return -1;
    }
    return nd::Workspace(num_atoms, num_columns, interactions).total;
}

int nd_schnet_energy_force_virial(const nd_schnet_args* args, nd_stream_t stream_handle)
{
    using namespace nd;
    ND_REQUIRE(args != nullptr, "args is null");
    const nd_schnet_args& s = *args;
    ND_REQUIRE(s.num_atoms >= 1 && s.num_atoms <= (int64_t{1} << 30), "num_atoms out of range");
    ND_REQUIRE(s.num_columns >= 0 && s.num_columns < (int64_t{1} << 31), "num_columns out of range");
    ND_REQUIRE(s.interactions >= 1 && s.interactions <= 64, "interactions out of range");
    ND_REQUIRE(s.num_types >= 1, "num_types must be positive");
    ND_REQUIRE(s.gaussians >= 2 && s.gaussians <= 64, "gaussians must lie in [2, 64]");
    ND_REQUIRE(s.cutoff > 0.0, "cutoff must be positive");
    ND_REQUIRE(s.positions && s.cell && s.atom_types && s.weights && s.workspace && s.status,
               "a required buffer is null");
    ND_REQUIRE(s.num_columns == 0 || s.pairs != nullptr, "pairs is null");
    ND_REQUIRE(reinterpret_cast<std::uintptr_t>(s.workspace) % 256 == 0 &&
                   reinterpret_cast<std::uintptr_t>(s.weights) % 256 == 0,
               "weights and workspace must be 256-byte aligned");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    const WeightLayout wl(s.interactions, s.num_types);
    const Workspace ws(s.num_atoms, s.num_columns, s.interactions);
    auto* weights = static_cast<const unsigned char*>(s.weights);
    auto* base = static_cast<unsigned char*>(s.workspace);
    auto at = [&](std::int64_t offset) { return base + offset; };
    const std::int64_t row_bytes = align256(s.num_atoms * kFeatures * 4);
    auto block_images = [&](int b) { return weights + static_cast<std::int64_t>(b) * kImagesPerBlock * umma::kImageBytes; };
    auto block_vector = [&](int b, int j) {
        return reinterpret_cast<const float*>(weights + wl.vectors + (static_cast<std::int64_t>(b) * 4 + j) * kFeatures * 4);
    };
    int* counters = reinterpret_cast<int*>(at(ws.counters));
    auto* pairs = reinterpret_cast<int2*>(at(ws.pairs));
    auto* geometry = reinterpret_cast<float4*>(at(ws.geometry));
    auto* x = reinterpret_cast<float*>(at(ws.x));
    auto v = [&](int b) { return reinterpret_cast<float*>(at(ws.v + b * row_bytes)); };
    auto h = [&](int b) { return reinterpret_cast<float*>(at(ws.h + b * row_bytes)); };
    auto m = [&](int b) { return reinterpret_cast<float*>(at(ws.m + b * row_bytes)); };
    auto* grad = reinterpret_cast<float*>(at(ws.grad));
    auto* grad_m = reinterpret_cast<float*>(at(ws.grad_m));
    auto* grad_v = reinterpret_cast<float*>(at(ws.grad_v));
    auto* dedr = reinterpret_cast<float*>(at(ws.dedr));
    auto* energy_partials = reinterpret_cast<double*>(at(ws.energy));
    auto* virial_partials = reinterpret_cast<double*>(at(ws.virial));
    const int atom_tiles = static_cast<int>((s.num_atoms + kTile - 1) / kTile);
    const bool reverse = s.forces != nullptr || s.virial != nullptr;

    // The kernels' attributes, set once per device (they belong to its instance of a kernel).
    static DeviceOnce configured;  // per device, retried after a failure
    ND_CUDA_TRY(configured.run([] {
        cudaError_t rc = cudaFuncSetAttribute(pair_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairForwardShared);
        auto then = [&rc](cudaError_t next) { rc = rc != cudaSuccess ? rc : next; };
        then(cudaFuncSetAttribute(pair_reverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kPairReverseShared));
        then(cudaFuncSetAttribute(atom_forward_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAtomShared));
        then(cudaFuncSetAttribute(atom_forward_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, kAtomShared));
        then(cudaFuncSetAttribute(atom_reverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kAtomShared));
        then(cudaFuncSetAttribute(pair_forward_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
        then(cudaFuncSetAttribute(pair_reverse_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
        return rc;
    }));
    const int forward_grid = pair_grid(reinterpret_cast<const void*>(pair_forward_kernel), kPairForwardShared, 64);
    const int reverse_grid = std::min(kVirialSlots, pair_grid(reinterpret_cast<const void*>(pair_reverse_kernel), kPairReverseShared, 128));

    ND_CUDA_TRY(cudaMemsetAsync(counters, 0, 256, stream));
    if (s.forces != nullptr)
    {
        ND_CUDA_TRY(cudaMemsetAsync(s.forces, 0, s.num_atoms * 3 * sizeof(float), stream));
    }
    if (s.num_columns > 0)
    {
        const unsigned column_blocks = blocks_for(s.num_columns);
        auto* block_counts = reinterpret_cast<int*>(at(ws.block_counts));
        auto* block_offsets = reinterpret_cast<int*>(at(ws.block_offsets));
        const float cutoff_squared = static_cast<float>(s.cutoff * s.cutoff);
        compact_count_kernel<<<column_blocks, kThreads, 0, stream>>>(
            s.positions, s.cell, s.pairs, s.num_columns, s.num_atoms, cutoff_squared,
            block_counts, counters);
        ND_LAUNCH_CHECK();
        compact_scan_kernel<<<1, kScanThreads, 0, stream>>>(
            block_counts, static_cast<int>(column_blocks), block_offsets, counters);
        ND_LAUNCH_CHECK();
        compact_write_kernel<<<column_blocks, kThreads, 0, stream>>>(
            s.positions, s.cell, s.pairs, s.num_columns, s.num_atoms, cutoff_squared,
            block_offsets, pairs, geometry, counters);
        ND_LAUNCH_CHECK();
    }
    embed_kernel<<<blocks_for(s.num_atoms * 16), kThreads, 0, stream>>>(
        s.atom_types, s.num_atoms, reinterpret_cast<const float*>(weights + wl.tables),
        reinterpret_cast<const float*>(weights + wl.tables + s.num_types * kFeatures * 4), x, v(0));
    ND_LAUNCH_CHECK();

    PairPass pass{};
    pass.pairs = pairs;
    pass.geometry = geometry;
    pass.counters = counters;
    pass.width = static_cast<float>(s.cutoff / (s.gaussians - 1));
    pass.phase = static_cast<float>(3.14159265358979323846 / s.cutoff);
    pass.gaussians = s.gaussians;
    const float* readout = reinterpret_cast<const float*>(weights + wl.readout);
    for (int b = 0; b < s.interactions; ++b)
    {
        const bool last = b == s.interactions - 1;
        ND_CUDA_TRY(cudaMemsetAsync(m(b), 0, s.num_atoms * kFeatures * 4, stream));
        pass.images = block_images(b);
        pass.b1 = block_vector(b, 0);
        pass.b2 = block_vector(b, 1);
        pass.v = v(b);
        pass.m = m(b);
        pair_forward_kernel<<<forward_grid, kTile, kPairForwardShared, stream>>>(pass);
        ND_LAUNCH_CHECK();
        AtomPass atoms{};
        atoms.atoms = s.num_atoms;
        atoms.images = block_images(b);
        atoms.next_images = last ? nullptr : block_images(b + 1);
        atoms.d1 = block_vector(b, 2);
        atoms.d2 = block_vector(b, 3);
        atoms.m = m(b);
        atoms.h = h(b);
        atoms.x = x;
        atoms.v_next = last ? nullptr : v(b + 1);
        atoms.readout = readout;
        atoms.grad = grad;
        atoms.energy = energy_partials;
        atoms.counters = counters;
        if (last)
        {
            atom_forward_kernel<true><<<atom_tiles, kTile, kAtomShared, stream>>>(atoms);
        }
        else
        {
            atom_forward_kernel<false><<<atom_tiles, kTile, kAtomShared, stream>>>(atoms);
        }
        ND_LAUNCH_CHECK();
    }
    if (reverse)
    {
        ND_CUDA_TRY(cudaMemsetAsync(virial_partials, 0, kVirialSlots * 9 * sizeof(double), stream));
        for (int b = s.interactions - 1; b >= 0; --b)
        {
            const bool last = b == s.interactions - 1;
            AtomPass atoms{};
            atoms.atoms = s.num_atoms;
            atoms.images = block_images(b);
            atoms.next_images = last ? nullptr : block_images(b + 1);
            atoms.h = h(b);
            atoms.grad = grad;
            atoms.grad_v = last ? nullptr : grad_v;
            atoms.grad_m = grad_m;
            atoms.counters = counters;
            atom_reverse_kernel<<<atom_tiles, kTile, kAtomShared, stream>>>(atoms);
            ND_LAUNCH_CHECK();
            if (b > 0)
            {
                ND_CUDA_TRY(cudaMemsetAsync(grad_v, 0, s.num_atoms * kFeatures * 4, stream));
            }
            pass.images = block_images(b);
            pass.b1 = block_vector(b, 0);
            pass.b2 = block_vector(b, 1);
            pass.v = v(b);
            pass.grad_m = grad_m;
            pass.grad_v = b > 0 ? grad_v : nullptr;
            pass.dedr = dedr;
            pass.first = last ? 1 : 0;
            pass.last = b == 0 ? 1 : 0;
            pass.forces = s.forces;
            pass.virial = virial_partials;
            pair_reverse_kernel<<<reverse_grid, kTile, kPairReverseShared, stream>>>(pass);
            ND_LAUNCH_CHECK();
        }
    }
    finalize_kernel<<<1, 256, 0, stream>>>(energy_partials, atom_tiles, virial_partials,
                                           reverse ? reverse_grid : 0, s.energy,
                                           reverse ? s.virial : nullptr);
    ND_LAUNCH_CHECK();
    ND_CUDA_TRY(cudaMemcpyAsync(s.status, counters, 4 * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    return ND_OK;
}

}  // extern "C"
