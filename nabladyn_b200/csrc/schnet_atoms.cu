// The atom-wise layers of the SchNet parameter gradient, with their tangents and reverse.
//
// The per-pair passes (schnet_tangent.cu) give each block's messages m and m_dot and, in
// reverse, v_bar and v_dot_bar. Between them sit the atom-wise layers of
// src/nabladyn/potential/_schnet/_potential.py:76-88 and :190-208, here carried with their
// derivative along the loss's direction (forward) and then reversed over both streams:
//
//   start:    x_0 = embedding[type], x_dot_0 = 0, v_0 = x_0 A_0^T, v_dot_0 = 0;
//   forward:  h = m D1^T + d1, h_dot = m_dot D1^T;  x' = x + ssp(h) D2^T + d2,
//             x_dot' = x_dot + (sigmoid(h) h_dot) D2^T;  v' = x' A'^T, v_dot' = x_dot' A'^T;
//   readout:  y = x R1^T + e1, y_dot = x_dot R1^T;  for Phi = e_bar E - Edot:
//             y_bar = (e_bar sigmoid(y) - sigmoid'(y) y_dot) R2, y_dot_bar = -sigmoid(y) R2,
//             x_bar = y_bar R1, x_dot_bar = y_dot_bar R1;
//   reverse:  ssp_bar = x_bar D2, q_bar = x_dot_bar D2;
//             h_bar = ssp_bar sigmoid(h) + q_bar h_dot sigmoid'(h), h_dot_bar = q_bar sigmoid(h);
//             m_bar = h_bar D1, m_dot_bar = h_dot_bar D1;   (the pair reverse runs here)
//             x_bar += v_bar A, x_dot_bar += v_dot_bar A;
//
// and the weights' gradients, sums over atoms (D2: x_bar^T ssp(h) + x_dot_bar^T q, D1:
// h_bar^T m + h_dot_bar^T m_dot, A: v_bar^T x + v_dot_bar^T x_dot, R1: y_bar^T x +
// y_dot_bar^T x_dot, the biases and R2 column sums). One CTA of 256 threads takes 64 atoms:
// rows and weights are staged in shared memory (FP32, rows of 68 floats), each thread
// computes a 4 x 4 block of every 64 x 64 product, and every sum over atoms is written as the
// tile's partial, then summed over 16 ranges of tiles in parallel and added to the gradient
// (FP32 atomics: the order of those 16 additions varies).

#include "common.cuh"

#include <cuda_bf16.h>

namespace nd {
namespace {

constexpr int kAtoms = 64;          // atoms per tile
constexpr int kAtomThreads = 256;   // threads per CTA: a 16 x 16 grid of 4 x 4 blocks
constexpr int kRow = 68;            // floats per shared-memory row (16-byte aligned)
constexpr int kMatrix = 64 * kRow;  // floats per shared-memory matrix
constexpr int kBlockFloats = 3 * 4096 + 2 * 64;  // A, D1, d1, D2, d2 of one block
constexpr int kReadoutFloats = 2048 + 3 * 32;    // R1 [32][64], e1 [32], R2 [32], e2 (pad 32)
constexpr int kPartialFloats = 2 * (4096 + 64);  // one tile's partial sums, the largest stage
constexpr float kLn2 = 0.693147180559945309f;

// Offsets inside one block's parameters (floats).
constexpr int kOffA = 0, kOffD1 = 4096, kOffd1 = 8192, kOffD2 = 8256, kOffd2 = 12352;
// Offsets inside the readout's parameters.
constexpr int kOffR1 = 0, kOffe1 = 2048, kOffR2 = 2080, kOffe2 = 2112;

// Per-atom arrays of the workspace: FP32 [N][64] per block, then FP32 globals, then BF16.
enum Kind : int
{
    kX = 0, kXDot = 1, kH = 2, kHDot = 3, kM = 4, kMDot = 5, kVBar = 6, kVDotBar = 7,  // per block
    kXLast = 8, kXDotLast = 9, kXBar = 10, kXDotBar = 11,                             // FP32
    kV = 12, kVDot = 13,                                                               // BF16, per block
    kMBar = 14, kMDotBar = 15,                                                         // BF16
    kPartials = 16,
};

inline std::int64_t align256(std::int64_t bytes)
{
    return (bytes + 255) / 256 * 256;
}

struct AtomLayout
{
    std::int64_t f32_row, bf16_row, f32_base, bf16_base, partials, total, tiles;

    AtomLayout(std::int64_t atoms, int blocks)
    {
        f32_row = align256(atoms * 64 * 4);
        bf16_row = align256(atoms * 64 * 2);
        tiles = (atoms + kAtoms - 1) / kAtoms;
        f32_base = 0;
        bf16_base = (static_cast<std::int64_t>(blocks) * 8 + 4) * f32_row;
        partials = bf16_base + (static_cast<std::int64_t>(blocks) * 2 + 2) * bf16_row;
        total = partials + align256(tiles * kPartialFloats * 4);
    }

    // Byte offset of array `kind` (of `block` for the per-block kinds); -1 if out of range.
    std::int64_t offset(int kind, int block, int blocks) const
    {
        if (kind >= kX && kind <= kVDotBar)
        {
            return (static_cast<std::int64_t>(block) * 8 + kind) * f32_row;
        }
        if (kind >= kXLast && kind <= kXDotBar)
        {
            return (static_cast<std::int64_t>(blocks) * 8 + (kind - kXLast)) * f32_row;
        }
        if (kind == kV || kind == kVDot)
        {
            return bf16_base + (static_cast<std::int64_t>(block) * 2 + (kind - kV)) * bf16_row;
        }
        if (kind == kMBar || kind == kMDotBar)
        {
            return bf16_base + (static_cast<std::int64_t>(blocks) * 2 + (kind - kMBar)) * bf16_row;
        }
        if (kind == kPartials)
        {
            return partials;
        }
        return -1;
    }
};

struct AtomPassArgs
{
    std::int64_t atoms;
    const std::int64_t* types;
    const float* block;     // this block's parameters (start: block 0)
    const float* next;      // forward: the next block's parameters, or null on the last
    const float* readout;
    const float* embedding;
    const double* energy_adjoint;
    const float* x;         // this block's x and x_dot
    const float* x_dot;
    float* x_out;           // forward: x' and x_dot'; start: x_0
    float* x_dot_out;
    const float* m;         // forward and reverse: this block's m, m_dot
    const float* m_dot;
    float* h;               // forward: written; reverse: read
    float* h_dot;
    __nv_bfloat16* v_out;   // start and forward: the next v and v_dot (BF16)
    __nv_bfloat16* v_dot_out;
    float* x_bar;           // readout: written; reverse: read, after the pair pass: added to
    float* x_dot_bar;
    __nv_bfloat16* m_bar;   // reverse: written (BF16)
    __nv_bfloat16* m_dot_bar;
    const float* v_bar;     // after the pair reverse
    const float* v_dot_bar;
    float* partials;        // [tiles][kPartialFloats]
};

struct Quad
{
    int a0;  // first of this thread's 4 rows (atoms, or a Gram's row features)
    int c0;  // first of its 4 columns
};

__device__ __forceinline__ Quad quad()
{
    return Quad{static_cast<int>(threadIdx.x >> 4) * 4, static_cast<int>(threadIdx.x & 15) * 4};
}

__device__ __forceinline__ float ssp(float x)
{
    return fmaxf(x, 0.0f) + log1pf(expf(-fabsf(x))) - kLn2;
}

__device__ __forceinline__ float sigmoid(float x)
{
    return 1.0f / (1.0f + expf(-x));
}

// S[a][c] = src[atom0 + a][c] (zero past N).
__device__ void load_rows(float* S, const float* __restrict__ src, std::int64_t atom0,
                          std::int64_t atoms)
{
    for (int e = threadIdx.x; e < kAtoms * 16; e += kAtomThreads)
    {
        const int a = e >> 4, q = e & 15;
        const std::int64_t atom = atom0 + a;
        const float4 value = atom < atoms
                                 ? reinterpret_cast<const float4*>(src + atom * 64)[q]
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
        *reinterpret_cast<float4*>(S + a * kRow + 4 * q) = value;
    }
}

// M[k][c] = W[c][k] for c < rows (W [rows][64] row-major), zero above: x W^T is x times M.
__device__ void load_transposed(float* M, const float* __restrict__ W, int rows)
{
    for (int e = threadIdx.x; e < 64 * 64; e += kAtomThreads)
    {
        const int c = e >> 6, k = e & 63;
        M[k * kRow + c] = c < rows ? W[c * 64 + k] : 0.0f;
    }
}

// M[k][c] = W[k][c] for k < rows (W [rows][64]), zero above: x W is x times M.
__device__ void load_direct(float* M, const float* __restrict__ W, int rows)
{
    for (int e = threadIdx.x; e < 64 * 16; e += kAtomThreads)
    {
        const int k = e >> 4, q = e & 15;
        const float4 value = k < rows ? reinterpret_cast<const float4*>(W + k * 64)[q]
                                      : make_float4(0.f, 0.f, 0.f, 0.f);
        *reinterpret_cast<float4*>(M + k * kRow + 4 * q) = value;
    }
}

// acc[r][j] = sum_k A[a0 + r][k] M[k][c0 + j]
__device__ __forceinline__ void product(const float* A, const float* M, float (&acc)[4][4], Quad q)
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            acc[r][j] = 0.0f;
        }
    }
#pragma unroll 2
    for (int k = 0; k < 64; k += 4)
    {
        float a[4][4];
#pragma unroll
        for (int r = 0; r < 4; ++r)
        {
            const float4 row = *reinterpret_cast<const float4*>(A + (q.a0 + r) * kRow + k);
            a[r][0] = row.x;
            a[r][1] = row.y;
            a[r][2] = row.z;
            a[r][3] = row.w;
        }
#pragma unroll
        for (int kk = 0; kk < 4; ++kk)
        {
            const float4 m = *reinterpret_cast<const float4*>(M + (k + kk) * kRow + q.c0);
#pragma unroll
            for (int r = 0; r < 4; ++r)
            {
                acc[r][0] = fmaf(a[r][kk], m.x, acc[r][0]);
                acc[r][1] = fmaf(a[r][kk], m.y, acc[r][1]);
                acc[r][2] = fmaf(a[r][kk], m.z, acc[r][2]);
                acc[r][3] = fmaf(a[r][kk], m.w, acc[r][3]);
            }
        }
    }
}

// acc[r][j] += sum_a P[a][a0 + r] Q[a][c0 + j] over the tile's atoms (a Gram block).
__device__ __forceinline__ void gram(const float* P, const float* Q, float (&acc)[4][4], Quad q)
{
#pragma unroll 8
    for (int a = 0; a < kAtoms; ++a)
    {
        const float4 p = *reinterpret_cast<const float4*>(P + a * kRow + q.a0);
        const float4 m = *reinterpret_cast<const float4*>(Q + a * kRow + q.c0);
        const float pr[4] = {p.x, p.y, p.z, p.w};
#pragma unroll
        for (int r = 0; r < 4; ++r)
        {
            acc[r][0] = fmaf(pr[r], m.x, acc[r][0]);
            acc[r][1] = fmaf(pr[r], m.y, acc[r][1]);
            acc[r][2] = fmaf(pr[r], m.z, acc[r][2]);
            acc[r][3] = fmaf(pr[r], m.w, acc[r][3]);
        }
    }
}

__device__ __forceinline__ void zero(float (&v)[4][4])
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            v[r][j] = 0.0f;
        }
    }
}

// S[a0 + r][c0 + j] = v[r][j]
__device__ __forceinline__ void put(float* S, const float (&v)[4][4], Quad q)
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        *reinterpret_cast<float4*>(S + (q.a0 + r) * kRow + q.c0) =
            make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
    }
}

// v[r][j] = src[atom0 + a0 + r][c0 + j] (zero past N)
__device__ __forceinline__ void get(const float* __restrict__ src, float (&v)[4][4],
                                    std::int64_t atom0, std::int64_t atoms, Quad q)
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        const std::int64_t atom = atom0 + q.a0 + r;
        const float4 value = atom < atoms
                                 ? *reinterpret_cast<const float4*>(src + atom * 64 + q.c0)
                                 : make_float4(0.f, 0.f, 0.f, 0.f);
        v[r][0] = value.x;
        v[r][1] = value.y;
        v[r][2] = value.z;
        v[r][3] = value.w;
    }
}

__device__ __forceinline__ void store(float* dst, const float (&v)[4][4], std::int64_t atom0,
                                      std::int64_t atoms, Quad q)
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        const std::int64_t atom = atom0 + q.a0 + r;
        if (atom < atoms)
        {
            *reinterpret_cast<float4*>(dst + atom * 64 + q.c0) =
                make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
        }
    }
}

__device__ __forceinline__ void store_bf16(__nv_bfloat16* dst, const float (&v)[4][4],
                                           std::int64_t atom0, std::int64_t atoms, Quad q)
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        const std::int64_t atom = atom0 + q.a0 + r;
        if (atom < atoms)
        {
            const __nv_bfloat162 lo = __floats2bfloat162_rn(v[r][0], v[r][1]);
            const __nv_bfloat162 hi = __floats2bfloat162_rn(v[r][2], v[r][3]);
            uint2 word;
            word.x = *reinterpret_cast<const std::uint32_t*>(&lo);
            word.y = *reinterpret_cast<const std::uint32_t*>(&hi);
            *reinterpret_cast<uint2*>(dst + atom * 64 + q.c0) = word;
        }
    }
}

// The tile's partial of a Gram block (rows < `rows`), at `offset` of its partial row.
__device__ __forceinline__ void put_partial(float* partial, int offset, const float (&v)[4][4],
                                            int rows, Quad q)
{
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        if (q.a0 + r < rows)
        {
            *reinterpret_cast<float4*>(partial + offset + (q.a0 + r) * 64 + q.c0) =
                make_float4(v[r][0], v[r][1], v[r][2], v[r][3]);
        }
    }
}

// partial[offset + c] = sum over the tile's atoms of S[a][c], c < columns.
__device__ __forceinline__ void put_column_sums(float* partial, int offset, const float* S,
                                                int columns)
{
    if (threadIdx.x < columns)
    {
        float sum = 0.0f;
        for (int a = 0; a < kAtoms; ++a)
        {
            sum += S[a * kRow + threadIdx.x];
        }
        partial[offset + threadIdx.x] = sum;
    }
}

// ---------------------------------------------------------------------------------------
// Stages, one CTA per 64 atoms.

// x_0 = embedding[type]; v_0 = x_0 A_0^T (BF16).
__global__ void __launch_bounds__(kAtomThreads) start_kernel(AtomPassArgs p)
{
    extern __shared__ __align__(16) float smem[];
    float* X = smem;
    float* W = X + kMatrix;
    const std::int64_t atom0 = static_cast<std::int64_t>(blockIdx.x) * kAtoms;
    const Quad q = quad();
    for (int e = threadIdx.x; e < kAtoms * 16; e += kAtomThreads)
    {
        const int a = e >> 4, c4 = e & 15;
        const std::int64_t atom = atom0 + a;
        const float4 value =
            atom < p.atoms ? reinterpret_cast<const float4*>(p.embedding + p.types[atom] * 64)[c4]
                           : make_float4(0.f, 0.f, 0.f, 0.f);
        *reinterpret_cast<float4*>(X + a * kRow + 4 * c4) = value;
    }
    load_transposed(W, p.block + kOffA, 64);
    __syncthreads();
    float x[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            x[r][j] = X[(q.a0 + r) * kRow + q.c0 + j];
        }
    }
    store(p.x_out, x, atom0, p.atoms, q);
    float v[4][4];
    product(X, W, v, q);
    store_bf16(p.v_out, v, atom0, p.atoms, q);
}

// h, h_dot from m, m_dot; x', x_dot'; and v', v_dot' for the next block.
__global__ void __launch_bounds__(kAtomThreads) forward_kernel(AtomPassArgs p)
{
    extern __shared__ __align__(16) float smem[];
    float* A = smem;             // m, then ssp(h), then x'
    float* B = A + kMatrix;      // m_dot, then q, then x_dot'
    float* W = B + kMatrix;      // D1^T, then D2^T, then A'^T
    const std::int64_t atom0 = static_cast<std::int64_t>(blockIdx.x) * kAtoms;
    const Quad q = quad();
    load_rows(A, p.m, atom0, p.atoms);
    load_rows(B, p.m_dot, atom0, p.atoms);
    load_transposed(W, p.block + kOffD1, 64);
    __syncthreads();
    float h[4][4], hd[4][4];
    product(A, W, h, q);
    product(B, W, hd, q);
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            h[r][j] += p.block[kOffd1 + q.c0 + j];
        }
    }
    store(p.h, h, atom0, p.atoms, q);
    store(p.h_dot, hd, atom0, p.atoms, q);
    float s[4][4], qd[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            s[r][j] = ssp(h[r][j]);
            qd[r][j] = sigmoid(h[r][j]) * hd[r][j];
        }
    }
    __syncthreads();
    put(A, s, q);
    put(B, qd, q);
    load_transposed(W, p.block + kOffD2, 64);
    __syncthreads();
    float x[4][4], xd[4][4], t[4][4];
    get(p.x, x, atom0, p.atoms, q);
    get(p.x_dot, xd, atom0, p.atoms, q);
    product(A, W, t, q);
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            x[r][j] += t[r][j] + p.block[kOffd2 + q.c0 + j];
        }
    }
    product(B, W, t, q);
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            xd[r][j] += t[r][j];
        }
    }
    store(p.x_out, x, atom0, p.atoms, q);
    store(p.x_dot_out, xd, atom0, p.atoms, q);
    if (p.next == nullptr)
    {
        return;
    }
    __syncthreads();
    put(A, x, q);
    put(B, xd, q);
    load_transposed(W, p.next + kOffA, 64);
    __syncthreads();
    product(A, W, t, q);
    store_bf16(p.v_out, t, atom0, p.atoms, q);
    product(B, W, t, q);
    store_bf16(p.v_dot_out, t, atom0, p.atoms, q);
}

// The readout of Phi = e_bar E - Edot: x_bar, x_dot_bar and the readout's partials.
__global__ void __launch_bounds__(kAtomThreads) readout_kernel(AtomPassArgs p)
{
    extern __shared__ __align__(16) float smem[];
    float* X = smem;
    float* XD = X + kMatrix;
    float* W = XD + kMatrix;     // R1^T, then R1
    float* YB = W + kMatrix;     // y_bar
    float* YDB = YB + kMatrix;   // y_dot_bar
    float* T2 = YDB + kMatrix;   // e_bar ssp(y) - sigmoid(y) y_dot
    const std::int64_t atom0 = static_cast<std::int64_t>(blockIdx.x) * kAtoms;
    const Quad q = quad();
    float* partial = p.partials + static_cast<std::int64_t>(blockIdx.x) * kPartialFloats;
    load_rows(X, p.x, atom0, p.atoms);
    load_rows(XD, p.x_dot, atom0, p.atoms);
    load_transposed(W, p.readout + kOffR1, 32);
    __syncthreads();
    float y[4][4], yd[4][4];
    product(X, W, y, q);
    product(XD, W, yd, q);
    const float e = static_cast<float>(p.energy_adjoint[0]);
    float yb[4][4], ydb[4][4], t2[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
        const bool live = atom0 + q.a0 + r < p.atoms;
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            const int c = q.c0 + j;
            const float r2 = (c < 32 && live) ? p.readout[kOffR2 + c] : 0.0f;
            const float value = y[r][j] + (c < 32 ? p.readout[kOffe1 + c] : 0.0f);
            const float sy = sigmoid(value);
            yb[r][j] = (e * sy - sy * (1.0f - sy) * yd[r][j]) * r2;
            ydb[r][j] = -sy * r2;
            t2[r][j] = (c < 32 && live) ? e * ssp(value) - sy * yd[r][j] : 0.0f;
        }
    }
    put(YB, yb, q);
    put(YDB, ydb, q);
    put(T2, t2, q);
    __syncthreads();
    float g[4][4];
    zero(g);
    gram(YB, X, g, q);
    gram(YDB, XD, g, q);
    put_partial(partial, kOffR1, g, 32, q);
    put_column_sums(partial, kOffe1, YB, 32);
    put_column_sums(partial, kOffR2, T2, 32);
    if (threadIdx.x == 0)
    {
        const std::int64_t live = min(static_cast<std::int64_t>(kAtoms), p.atoms - atom0);
        partial[kOffe2] = e * static_cast<float>(live);
    }
    __syncthreads();
    load_direct(W, p.readout + kOffR1, 32);
    __syncthreads();
    float xb[4][4];
    product(YB, W, xb, q);
    store(p.x_bar, xb, atom0, p.atoms, q);
    product(YDB, W, xb, q);
    store(p.x_dot_bar, xb, atom0, p.atoms, q);
}

// Reverse of one block's atom-wise layers up to the messages: m_bar, m_dot_bar and the
// partials of D2, d2, D1, d1.
__global__ void __launch_bounds__(kAtomThreads) reverse_kernel(AtomPassArgs p)
{
    extern __shared__ __align__(16) float smem[];
    float* XB = smem;            // x_bar, then m
    float* XDB = XB + kMatrix;   // x_dot_bar, then m_dot
    float* W = XDB + kMatrix;    // D2, then D1
    float* S = W + kMatrix;      // ssp(h), then h_bar
    float* Q = S + kMatrix;      // sigmoid(h) h_dot, then h_dot_bar
    const std::int64_t atom0 = static_cast<std::int64_t>(blockIdx.x) * kAtoms;
    const Quad q = quad();
    float* partial = p.partials + static_cast<std::int64_t>(blockIdx.x) * kPartialFloats;
    load_rows(XB, p.x_bar, atom0, p.atoms);
    load_rows(XDB, p.x_dot_bar, atom0, p.atoms);
    load_direct(W, p.block + kOffD2, 64);
    float h[4][4], hd[4][4];
    get(p.h, h, atom0, p.atoms, q);
    get(p.h_dot, hd, atom0, p.atoms, q);
    float sg[4][4], s[4][4], qd[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            sg[r][j] = sigmoid(h[r][j]);
            const bool live = atom0 + q.a0 + r < p.atoms;
            s[r][j] = live ? ssp(h[r][j]) : 0.0f;
            qd[r][j] = sg[r][j] * hd[r][j];
        }
    }
    put(S, s, q);
    put(Q, qd, q);
    __syncthreads();
    float sb[4][4], qb[4][4];
    product(XB, W, sb, q);
    product(XDB, W, qb, q);
    float g[4][4];
    zero(g);
    gram(XB, S, g, q);
    gram(XDB, Q, g, q);
    put_partial(partial, 0, g, 64, q);
    put_column_sums(partial, 4096, XB, 64);
    float hb[4][4], hdb[4][4];
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            hb[r][j] = sb[r][j] * sg[r][j] + qb[r][j] * hd[r][j] * sg[r][j] * (1.0f - sg[r][j]);
            hdb[r][j] = qb[r][j] * sg[r][j];
        }
    }
    __syncthreads();
    put(S, hb, q);
    put(Q, hdb, q);
    load_rows(XB, p.m, atom0, p.atoms);
    load_rows(XDB, p.m_dot, atom0, p.atoms);
    load_direct(W, p.block + kOffD1, 64);
    __syncthreads();
    float mb[4][4];
    product(S, W, mb, q);
    store_bf16(p.m_bar, mb, atom0, p.atoms, q);
    product(Q, W, mb, q);
    store_bf16(p.m_dot_bar, mb, atom0, p.atoms, q);
    zero(g);
    gram(S, XB, g, q);
    gram(Q, XDB, g, q);
    put_partial(partial, 4160, g, 64, q);
    put_column_sums(partial, 4160 + 4096, S, 64);
}

// After the pair reverse: x_bar += v_bar A, x_dot_bar += v_dot_bar A, and A's partial.
__global__ void __launch_bounds__(kAtomThreads) scatter_kernel(AtomPassArgs p)
{
    extern __shared__ __align__(16) float smem[];
    float* VB = smem;
    float* VDB = VB + kMatrix;
    float* W = VDB + kMatrix;    // A
    float* X = W + kMatrix;
    float* XD = X + kMatrix;
    const std::int64_t atom0 = static_cast<std::int64_t>(blockIdx.x) * kAtoms;
    const Quad q = quad();
    float* partial = p.partials + static_cast<std::int64_t>(blockIdx.x) * kPartialFloats;
    load_rows(VB, p.v_bar, atom0, p.atoms);
    load_rows(VDB, p.v_dot_bar, atom0, p.atoms);
    load_direct(W, p.block + kOffA, 64);
    load_rows(X, p.x, atom0, p.atoms);
    load_rows(XD, p.x_dot, atom0, p.atoms);
    __syncthreads();
    float t[4][4], xb[4][4];
    product(VB, W, t, q);
    get(p.x_bar, xb, atom0, p.atoms, q);
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            xb[r][j] += t[r][j];
        }
    }
    store(p.x_bar, xb, atom0, p.atoms, q);
    product(VDB, W, t, q);
    get(p.x_dot_bar, xb, atom0, p.atoms, q);
#pragma unroll
    for (int r = 0; r < 4; ++r)
    {
#pragma unroll
        for (int j = 0; j < 4; ++j)
        {
            xb[r][j] += t[r][j];
        }
    }
    store(p.x_dot_bar, xb, atom0, p.atoms, q);
    float g[4][4];
    zero(g);
    gram(VB, X, g, q);
    gram(VDB, XD, g, q);
    put_partial(partial, 0, g, 64, q);
}

// Segments of the tiles' partials to reduce: gradient[dst + j] += sum_t partial[t][src + j].
struct Segments
{
    int count;
    int src[4];
    int length[4];
    float* dst[4];
};

constexpr int kReduceSlices = 16;  // tile ranges summed in parallel, then added atomically

__global__ void reduce_kernel(const float* __restrict__ partials, std::int64_t tiles, Segments s)
{
    int j = blockIdx.x * blockDim.x + threadIdx.x;
    const std::int64_t per_slice = (tiles + kReduceSlices - 1) / kReduceSlices;
    const std::int64_t begin = blockIdx.y * per_slice;
    const std::int64_t end = min(tiles, begin + per_slice);
    for (int k = 0; k < s.count; ++k)
    {
        if (j < s.length[k])
        {
            float sums[4] = {0.0f, 0.0f, 0.0f, 0.0f};
            std::int64_t t = begin;
            for (; t + 4 <= end; t += 4)
            {
#pragma unroll
                for (int u = 0; u < 4; ++u)
                {
                    sums[u] += partials[(t + u) * kPartialFloats + s.src[k] + j];
                }
            }
            for (; t < end; ++t)
            {
                sums[0] += partials[t * kPartialFloats + s.src[k] + j];
            }
            if (begin < end)
            {
                atomicAdd(s.dst[k] + j, (sums[0] + sums[1]) + (sums[2] + sums[3]));
            }
            return;
        }
        j -= s.length[k];
    }
}

constexpr int kStartShared = 2 * kMatrix * 4;
constexpr int kForwardShared = 3 * kMatrix * 4;
constexpr int kReadoutShared = 6 * kMatrix * 4;
constexpr int kReverseShared = 5 * kMatrix * 4;
constexpr int kScatterShared = 5 * kMatrix * 4;

}  // namespace
}  // namespace nd

extern "C" {

int64_t nd_schnet_atom_parameter_floats(int32_t interactions, int32_t num_types)
{
    if (interactions < 1 || num_types < 1)
    {
        return -1;
    }
    return static_cast<int64_t>(interactions) * nd::kBlockFloats + nd::kReadoutFloats +
           static_cast<int64_t>(num_types) * 64;
}

int64_t nd_schnet_atom_workspace_bytes(int64_t num_atoms, int32_t interactions)
{
    if (num_atoms < 1 || interactions < 1)
    {
        return -1;
    }
    return nd::AtomLayout(num_atoms, interactions).total;
}

int64_t nd_schnet_atom_offset(int64_t num_atoms, int32_t interactions, int32_t kind,
                              int32_t block)
{
    if (num_atoms < 1 || interactions < 1 || block < 0 || block >= interactions)
    {
        return -1;
    }
    return nd::AtomLayout(num_atoms, interactions).offset(kind, block, interactions);
}

int nd_schnet_atoms(const nd_schnet_atom_args* args, int32_t stage, int32_t block,
                    nd_stream_t stream_handle)
{
    using namespace nd;
    ND_REQUIRE(args != nullptr, "args is null");
    const nd_schnet_atom_args& s = *args;
    ND_REQUIRE(s.num_atoms >= 1 && s.num_atoms <= (int64_t{1} << 30), "num_atoms out of range");
    ND_REQUIRE(s.interactions >= 1 && s.interactions <= 64, "interactions out of range");
    ND_REQUIRE(s.num_types >= 1, "num_types must be positive");
    ND_REQUIRE(stage >= 0 && stage <= 4, "stage must lie in [0, 4]");
    ND_REQUIRE(block >= 0 && block < s.interactions, "block out of range");
    ND_REQUIRE(s.atom_types && s.parameters && s.gradient && s.energy_adjoint && s.workspace,
               "a required buffer is null");
    ND_REQUIRE(reinterpret_cast<std::uintptr_t>(s.workspace) % 256 == 0 &&
                   reinterpret_cast<std::uintptr_t>(s.parameters) % 16 == 0 &&
                   reinterpret_cast<std::uintptr_t>(s.gradient) % 16 == 0,
               "workspace must be 256-byte and parameters and gradient 16-byte aligned");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    const AtomLayout layout(s.num_atoms, s.interactions);
    auto* base = static_cast<unsigned char*>(s.workspace);
    const int blocks = s.interactions;
    auto f32 = [&](int kind, int b) {
        return reinterpret_cast<float*>(base + layout.offset(kind, b, blocks));
    };
    auto bf16 = [&](int kind, int b) {
        return reinterpret_cast<__nv_bfloat16*>(base + layout.offset(kind, b, blocks));
    };
    const float* parameters = s.parameters;
    float* gradient = s.gradient;
    const std::int64_t readout = static_cast<std::int64_t>(blocks) * kBlockFloats;
    AtomPassArgs p{};
    p.atoms = s.num_atoms;
    p.types = s.atom_types;
    p.block = parameters + static_cast<std::int64_t>(block) * kBlockFloats;
    p.readout = parameters + readout;
    p.embedding = parameters + readout + kReadoutFloats;
    p.energy_adjoint = s.energy_adjoint;
    p.partials = reinterpret_cast<float*>(base + layout.partials);
    p.x_bar = f32(kXBar, 0);
    p.x_dot_bar = f32(kXDotBar, 0);
    const unsigned tiles = static_cast<unsigned>(layout.tiles);

    // The kernels' attributes, set once per device (they belong to its instance of a kernel).
    static DeviceOnce configured;  // per device, retried after a failure
    ND_CUDA_TRY(configured.run([] {
        cudaError_t rc = cudaFuncSetAttribute(start_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kStartShared);
        auto then = [&rc](cudaError_t next) { rc = rc != cudaSuccess ? rc : next; };
        then(cudaFuncSetAttribute(forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kForwardShared));
        then(cudaFuncSetAttribute(readout_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kReadoutShared));
        then(cudaFuncSetAttribute(reverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kReverseShared));
        then(cudaFuncSetAttribute(scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kScatterShared));
        return rc;
    }));
    auto reduce = [&](const Segments& segments) -> int {
        int total = 0;
        for (int k = 0; k < segments.count; ++k)
        {
            total += segments.length[k];
        }
        const dim3 grid(blocks_for(total), kReduceSlices);
        reduce_kernel<<<grid, kThreads, 0, stream>>>(p.partials, layout.tiles, segments);
        ND_LAUNCH_CHECK();
        return ND_OK;
    };
    float* block_gradient = gradient + static_cast<std::int64_t>(block) * kBlockFloats;

    switch (stage)
    {
    case 0:  // start: x_0, v_0; zero x_dot_0, v_dot_0 and every block's m, m_dot, v_bar, v_dot_bar
        for (int b = 0; b < blocks; ++b)
        {
            ND_CUDA_TRY(cudaMemsetAsync(f32(kM, b), 0, 4 * layout.f32_row, stream));
        }
        ND_CUDA_TRY(cudaMemsetAsync(f32(kXDot, 0), 0, layout.f32_row, stream));
        ND_CUDA_TRY(cudaMemsetAsync(bf16(kVDot, 0), 0, layout.bf16_row, stream));
        p.block = parameters;
        p.x_out = f32(kX, 0);
        p.v_out = bf16(kV, 0);
        start_kernel<<<tiles, kAtomThreads, kStartShared, stream>>>(p);
        ND_LAUNCH_CHECK();
        return ND_OK;
    case 1:  // block forward, after its tangent forward pass filled m, m_dot
    {
        const bool last = block == blocks - 1;
        p.next = last ? nullptr : parameters + static_cast<std::int64_t>(block + 1) * kBlockFloats;
        p.x = f32(kX, block);
        p.x_dot = f32(kXDot, block);
        p.m = f32(kM, block);
        p.m_dot = f32(kMDot, block);
        p.h = f32(kH, block);
        p.h_dot = f32(kHDot, block);
        p.x_out = last ? f32(kXLast, 0) : f32(kX, block + 1);
        p.x_dot_out = last ? f32(kXDotLast, 0) : f32(kXDot, block + 1);
        p.v_out = last ? nullptr : bf16(kV, block + 1);
        p.v_dot_out = last ? nullptr : bf16(kVDot, block + 1);
        forward_kernel<<<tiles, kAtomThreads, kForwardShared, stream>>>(p);
        ND_LAUNCH_CHECK();
        return ND_OK;
    }
    case 2:  // readout
    {
        p.x = f32(kXLast, 0);
        p.x_dot = f32(kXDotLast, 0);
        readout_kernel<<<tiles, kAtomThreads, kReadoutShared, stream>>>(p);
        ND_LAUNCH_CHECK();
        float* g = gradient + readout;
        Segments segments{};
        segments.count = 4;
        segments.src[0] = kOffR1;
        segments.length[0] = 2048;
        segments.dst[0] = g + kOffR1;
        segments.src[1] = kOffe1;
        segments.length[1] = 32;
        segments.dst[1] = g + kOffe1;
        segments.src[2] = kOffR2;
        segments.length[2] = 32;
        segments.dst[2] = g + kOffR2;
        segments.src[3] = kOffe2;
        segments.length[3] = 1;
        segments.dst[3] = g + kOffe2;
        return reduce(segments);
    }
    case 3:  // block reverse, before its tangent reverse pass
    {
        p.m = f32(kM, block);
        p.m_dot = f32(kMDot, block);
        p.h = f32(kH, block);
        p.h_dot = f32(kHDot, block);
        p.m_bar = bf16(kMBar, 0);
        p.m_dot_bar = bf16(kMDotBar, 0);
        reverse_kernel<<<tiles, kAtomThreads, kReverseShared, stream>>>(p);
        ND_LAUNCH_CHECK();
        Segments segments{};
        segments.count = 4;
        segments.src[0] = 0;
        segments.length[0] = 4096;
        segments.dst[0] = block_gradient + kOffD2;
        segments.src[1] = 4096;
        segments.length[1] = 64;
        segments.dst[1] = block_gradient + kOffd2;
        segments.src[2] = 4160;
        segments.length[2] = 4096;
        segments.dst[2] = block_gradient + kOffD1;
        segments.src[3] = 4160 + 4096;
        segments.length[3] = 64;
        segments.dst[3] = block_gradient + kOffd1;
        return reduce(segments);
    }
    default:  // 4: block reverse, after its tangent reverse pass filled v_bar, v_dot_bar
    {
        p.x = f32(kX, block);
        p.x_dot = f32(kXDot, block);
        p.v_bar = f32(kVBar, block);
        p.v_dot_bar = f32(kVDotBar, block);
        scatter_kernel<<<tiles, kAtomThreads, kScatterShared, stream>>>(p);
        ND_LAUNCH_CHECK();
        Segments segments{};
        segments.count = 1;
        segments.src[0] = 0;
        segments.length[0] = 4096;
        segments.dst[0] = block_gradient + kOffA;
        return reduce(segments);
    }
    }
}

}  // extern "C"
