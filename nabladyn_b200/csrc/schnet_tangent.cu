// The per-pair passes of the SchNet parameter gradient of a training loss over E, F and W.
//
// The reference differentiates its loss with torch.func through a double backward
// (src/nabladyn/training/_fit.py:245-271, _loss.py:49-102). Written out: with the loss's
// adjoints e_bar = dL/dE, f_bar = dL/dF [N, 3] and w_bar = dL/dW [3, 3], F = -dE/dr and
// W = -dE/d(strain) make f_bar . F + w_bar : W the derivative of -E along a direction in which
// each pair's distance moves at
//     rdot = (d . (f_bar_a - f_bar_b) + d^T w_bar d) / r,
// so dL/dtheta = d/dtheta (e_bar E - Edot): a forward pass carrying beside each value its
// derivative along rdot, then one reverse pass over both streams. Per block, the pair work:
//
//   forward:  g, g_dot = g * (-(r / D - k) / D) rdot;  z, z_dot = (g, g_dot) B1^T (+ b1 on z);
//             s = ssp(z), s_dot = sigmoid(z) z_dot;  u, u_dot = (s, s_dot) B2^T (+ b2 on u);
//             f = u C, f_dot = u_dot C + u C' rdot;
//             m_dot_a += f_dot v_b + f v_dot_b, m_dot_b likewise (m itself, f v of the other
//             atom, is the E/F/W call's, copied from its workspace);
//   reverse, given m_bar and m_dot_bar from the atom-wise layers:
//             fb = m_bar_a v_b + m_bar_b v_a + m_dot_bar_a v_dot_b + m_dot_bar_b v_dot_a,
//             fdb = m_dot_bar_a v_b + m_dot_bar_b v_a;
//             v_bar_b += f m_bar_a + f_dot m_dot_bar_a, v_dot_bar_b += f m_dot_bar_a, and for a;
//             u_bar = fb C + fdb C' rdot, u_dot_bar = fdb C;
//             (s_bar, s_dot_bar) = (u_bar, u_dot_bar) B2;
//             z_bar = s_bar sigmoid(z) + s_dot_bar z_dot sigmoid'(z), z_dot_bar = s_dot_bar sigmoid(z).
//
// The reverse pass writes every pair's BF16 rows g, g_dot, s, s_dot, z_bar, z_dot_bar, u_bar,
// u_dot_bar, so the filter weights' gradients, sums over pairs (B1: z_bar^T g + z_dot_bar^T
// g_dot, B2: u_bar^T s + u_dot_bar^T s_dot, the biases the column sums of z_bar and u_bar), are
// plain GEMMs for the caller, as are the atom-wise 64 x 64 layers. With fewer than 64
// Gaussians the g row's last column holds 1, so column 63 of z_bar^T g is the sum of z_bar.
// Each product runs with its tangent as two 128 x 64 x 64 BF16 tcgen05 products on one commit;
// the tiles' rows are pairs in the compacted order of the preceding
// nd_schnet_energy_force_virial call, whose workspace this pass reads.

#include "schnet.cuh"

namespace nd {
namespace {

// Per-pair rows of the reverse pass, in this order, [8][capacity][64] BF16.
enum Row : int
{
    kRowG = 0,
    kRowGDot = 1,
    kRowS = 2,
    kRowSDot = 3,
    kRowZBar = 4,
    kRowZDotBar = 5,
    kRowUBar = 6,
    kRowUDotBar = 7,
};

struct TangentPass
{
    const int2* pairs;
    const float4* geometry;
    int* counters;
    const unsigned char* images;  // this block's ten images
    const float* b1;
    const float* b2;
    const float* force_adjoint;    // [N][3]
    const double* virial_adjoint;  // [9]
    const uint4* v;                // [N][64] BF16, 8 features a word
    const uint4* v_dot;
    float* m;                      // forward: [N][64], added to
    float* m_dot;
    const uint4* m_bar;            // reverse: [N][64] BF16
    const uint4* m_dot_bar;
    float* v_bar;                  // reverse: [N][64], added to
    float* v_dot_bar;
    uint4* rows;                   // reverse: [8][capacity][64] BF16 as 16-byte words
    std::int64_t capacity;
    float width;  // Gaussian spacing D
    float phase;  // pi / r_c
    int gaussians;
};

// The pair's geometry and the rate rdot at which the loss's direction moves its distance.
struct PairTerms
{
    int2 ab;
    float4 g;        // d, r
    bool live;
    float envelope;  // C(r)
    float moving;    // C'(r) rdot
    float rate;      // rdot
};

__device__ __forceinline__ PairTerms pair_terms(const TangentPass& a, const float* wbar, int p,
                                                int count)
{
    PairTerms t;
    t.live = p < count;
    t.ab = make_int2(0, 0);
    t.g = make_float4(0.f, 0.f, 0.f, 1.f);
    t.rate = 0.0f;
    if (t.live)
    {
        t.ab = a.pairs[p];
        t.g = a.geometry[p];
        const float* fa = a.force_adjoint + 3 * static_cast<std::int64_t>(t.ab.x);
        const float* fb = a.force_adjoint + 3 * static_cast<std::int64_t>(t.ab.y);
        const float d[3] = {t.g.x, t.g.y, t.g.z};
        float along = 0.0f;
#pragma unroll
        for (int i = 0; i < 3; ++i)
        {
            along += d[i] * (__ldg(fa + i) - __ldg(fb + i));
#pragma unroll
            for (int j = 0; j < 3; ++j)
            {
                along += d[i] * wbar[3 * i + j] * d[j];
            }
        }
        t.rate = along / t.g.w;
    }
    float sine, cosine;
    __sincosf(t.g.w * a.phase, &sine, &cosine);
    t.envelope = t.live ? 0.5f * (cosine + 1.0f) : 0.0f;
    t.moving = t.live ? -0.5f * a.phase * sine * t.rate : 0.0f;
    return t;
}

// Row p of per-pair array `kind`, or null for a dead row.
__device__ __forceinline__ uint4* pair_row(const TangentPass& a, int kind, int p, bool live)
{
    return live ? a.rows + (static_cast<std::int64_t>(kind) * a.capacity + p) * 8 : nullptr;
}

// g_k = exp(-(t - k)^2 / 2) (zero for k >= K) and g_dot_k = g_k (t - k) scale, scale = -rdot / D,
// into this thread's row of two tiles, and into HBM rows when given (there with g_63 = 1 when
// K < 64).
__device__ __forceinline__ void store_basis_tangent(unsigned char* tile, unsigned char* tile_dot,
                                                    float t, float scale, int gaussians, bool live,
                                                    uint4* row, uint4* row_dot)
{
#pragma unroll
    for (int c = 0; c < 8; ++c)
    {
        float g[8];
        float gd[8];
#pragma unroll
        for (int e = 0; e < 8; ++e)
        {
            const int k = 8 * c + e;
            const float u = t - static_cast<float>(k);
            g[e] = (live && k < gaussians) ? __expf(-0.5f * u * u) : 0.0f;
            gd[e] = g[e] * u * scale;
        }
        const uint4 word = umma::pack8(g);
        const uint4 word_dot = umma::pack8(gd);
        *reinterpret_cast<uint4*>(tile + umma::image_offset(threadIdx.x, 8 * c)) = word;
        *reinterpret_cast<uint4*>(tile_dot + umma::image_offset(threadIdx.x, 8 * c)) = word_dot;
        if (row != nullptr)
        {
            // With K < 64 the HBM row's column 63 (a zero the products never use) holds 1, so
            // the sum over pairs of z_bar^T g carries the bias gradient sum(z_bar) there.
            if (c == 7 && gaussians < 64)
            {
                g[7] = 1.0f;
                row[c] = umma::pack8(g);
            }
            else
            {
                row[c] = word;
            }
            row_dot[c] = word_dot;
        }
    }
}

// s = ssp(z + b1) and s_dot = sigmoid(z + b1) z_dot from tensor-memory columns 0-63 (z - b1) and
// 64-127 (z_dot) into this thread's row of two tiles, and into HBM rows when given.
__device__ __forceinline__ void store_activations(std::uint32_t tmem, const float* bias1,
                                                  unsigned char* tile, unsigned char* tile_dot,
                                                  uint4* row, uint4* row_dot)
{
#pragma unroll
    for (int half = 0; half < 2; ++half)
    {
        float z[32];
        float zd[32];
        umma::load32(tmem + 32 * half, z);
        umma::load32(tmem + 64 + 32 * half, zd);
        umma::wait_loads();
#pragma unroll
        for (int c = 0; c < 4; ++c)
        {
            float s[8];
            float sd[8];
#pragma unroll
            for (int e = 0; e < 8; ++e)
            {
                const float x = z[8 * c + e] + bias1[32 * half + 8 * c + e];
                s[e] = softplus_shifted(x);
                sd[e] = sigmoid(x) * zd[8 * c + e];
            }
            const int column = 4 * half + c;
            const uint4 word = umma::pack8(s);
            const uint4 word_dot = umma::pack8(sd);
            *reinterpret_cast<uint4*>(tile + umma::image_offset(threadIdx.x, 8 * column)) = word;
            *reinterpret_cast<uint4*>(tile_dot + umma::image_offset(threadIdx.x, 8 * column)) =
                word_dot;
            if (row != nullptr)
            {
                row[column] = word;
                row_dot[column] = word_dot;
            }
        }
    }
}

// Shared memory: weight images, two row tiles, (reverse) two 16 KB run stages, biases,
// barrier and tensor-memory slot.
constexpr int kTangentForwardShared = 2 * umma::kImageBytes + 2 * umma::kTileBytes + 2 * 256 + 64;
constexpr int kTangentReverseShared = 3 * umma::kImageBytes + 4 * umma::kTileBytes + 2 * 256 + 64;

__global__ void __launch_bounds__(kTile, 3) tangent_forward_kernel(TangentPass a)
{
    extern __shared__ __align__(1024) unsigned char shared[];
    unsigned char* image_b1 = shared;
    unsigned char* image_b2 = image_b1 + umma::kImageBytes;
    unsigned char* tile = image_b2 + umma::kImageBytes;
    unsigned char* tile_dot = tile + umma::kTileBytes;
    // first-atom runs of m_dot, in a row tile once the products are done
    float* stage_dot = reinterpret_cast<float*>(tile);
    float* bias1 = reinterpret_cast<float*>(tile_dot + umma::kTileBytes);
    float* bias2 = bias1 + kFeatures;
    auto* barrier = reinterpret_cast<std::uint64_t*>(bias2 + kFeatures);
    auto* slot = reinterpret_cast<std::uint32_t*>(barrier + 1);
    __shared__ int tile_first[kTile];
    __shared__ float wbar[9];

    copy_bytes(image_b1, a.images + kB1 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b2, a.images + kB2 * umma::kImageBytes, umma::kImageBytes);
    if (threadIdx.x < kFeatures)
    {
        bias1[threadIdx.x] = a.b1[threadIdx.x];
        bias2[threadIdx.x] = a.b2[threadIdx.x];
    }
    if (threadIdx.x < 9)
    {
        wbar[threadIdx.x] = static_cast<float>(a.virial_adjoint[threadIdx.x]);
    }
    // Columns 0-63: z, then u; 64-127: z_dot, then u_dot.
    Cores cores;
    cores.open(barrier, slot, 128, a.counters, 5);
    const int count = *reinterpret_cast<volatile int*>(a.counters);
    float4* md4 = reinterpret_cast<float4*>(a.m_dot);

    for (int index = blockIdx.x; index * kTile < count; index += gridDim.x)
    {
        const int p = index * kTile + threadIdx.x;
        const PairTerms t = pair_terms(a, wbar, p, count);
        tile_first[threadIdx.x] = t.live ? t.ab.x : -1;
        cores.tile_index = index;
        store_basis_tangent(tile, tile_dot, t.g.w / a.width, -t.rate / a.width, a.gaussians,
                            t.live, nullptr, nullptr);
        if (!cores.run2(0, tile, image_b1, 64, tile_dot, image_b1, 1))
        {
            break;
        }
        store_activations(cores.tmem, bias1, tile, tile_dot, nullptr, nullptr);
        if (!cores.run2(0, tile, image_b2, 64, tile_dot, image_b2, 2))
        {
            break;
        }
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
                    const std::int64_t ga = 8 * static_cast<std::int64_t>(t.ab.x) + k / 8;
                    const std::int64_t gb = 8 * static_cast<std::int64_t>(t.ab.y) + k / 8;
                    raw[i][0] = __ldg(a.v + ga);
                    raw[i][1] = __ldg(a.v + gb);
                    raw[i][2] = __ldg(a.v_dot + ga);
                    raw[i][3] = __ldg(a.v_dot + gb);
                }
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int c = batch + i;
                    const int k = 32 * half + 8 * c;
                    float u[8];
                    float ud[8];
                    umma::load8(cores.tmem + k, u);
                    umma::load8(cores.tmem + 64 + k, ud);
                    umma::wait_loads();
                    float va[8], vb[8], vda[8], vdb[8], f[8], fd[8];
                    widen8(raw[i][0], va);
                    widen8(raw[i][1], vb);
                    widen8(raw[i][2], vda);
                    widen8(raw[i][3], vdb);
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                    {
                        const float raw_filter = u[j] + bias2[k + j];
                        f[j] = raw_filter * t.envelope;
                        fd[j] = ud[j] * t.envelope + raw_filter * t.moving;
                    }
                    if (t.live)
                    {
                        const std::int64_t gb = 8 * static_cast<std::int64_t>(t.ab.y) + k / 8;
#pragma unroll
                        for (int h4 = 0; h4 < 2; ++h4)
                        {
                            const int o = 4 * h4;
                            atomicAdd(md4 + 2 * gb + h4,
                                      make_float4(fd[o] * va[o] + f[o] * vda[o],
                                                  fd[o + 1] * va[o + 1] + f[o + 1] * vda[o + 1],
                                                  fd[o + 2] * va[o + 2] + f[o + 2] * vda[o + 2],
                                                  fd[o + 3] * va[o + 3] + f[o + 3] * vda[o + 3]));
                        }
                    }
#pragma unroll
                    for (int h4 = 0; h4 < 2; ++h4)
                    {
                        const int o = 4 * h4;
                        put_run_part(stage_dot, 2 * c + h4,
                                     make_float4(fd[o] * vb[o] + f[o] * vdb[o],
                                                 fd[o + 1] * vb[o + 1] + f[o + 1] * vdb[o + 1],
                                                 fd[o + 2] * vb[o + 2] + f[o + 2] * vdb[o + 2],
                                                 fd[o + 3] * vb[o + 3] + f[o + 3] * vdb[o + 3]));
                    }
                }
            }
            sum_runs(stage_dot, tile_first, a.m_dot, half, half == 1);  // the next basis overwrites it
        }
    }
    cores.close(128);
}

__global__ void __launch_bounds__(kTile, 2) tangent_reverse_kernel(TangentPass a)
{
    extern __shared__ __align__(1024) unsigned char shared[];
    unsigned char* image_b1 = shared;
    unsigned char* image_b2 = image_b1 + umma::kImageBytes;
    unsigned char* image_b2t = image_b2 + umma::kImageBytes;
    unsigned char* tile = image_b2t + umma::kImageBytes;
    unsigned char* tile_dot = tile + umma::kTileBytes;
    float* stage = reinterpret_cast<float*>(tile_dot + umma::kTileBytes);  // v_bar runs, 16 KB
    float* stage_dot = stage + kTile * 32;                                  // v_dot_bar runs
    float* bias1 = stage_dot + kTile * 32;
    float* bias2 = bias1 + kFeatures;
    auto* barrier = reinterpret_cast<std::uint64_t*>(bias2 + kFeatures);
    auto* slot = reinterpret_cast<std::uint32_t*>(barrier + 1);
    __shared__ int tile_first[kTile];
    __shared__ float wbar[9];

    copy_bytes(image_b1, a.images + kB1 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b2, a.images + kB2 * umma::kImageBytes, umma::kImageBytes);
    copy_bytes(image_b2t, a.images + kB2T * umma::kImageBytes, umma::kImageBytes);
    if (threadIdx.x < kFeatures)
    {
        bias1[threadIdx.x] = a.b1[threadIdx.x];
        bias2[threadIdx.x] = a.b2[threadIdx.x];
    }
    if (threadIdx.x < 9)
    {
        wbar[threadIdx.x] = static_cast<float>(a.virial_adjoint[threadIdx.x]);
    }
    // Columns 0-63 keep z - b1 and 64-127 z_dot for the whole tile; 128-191 take u, then s_bar;
    // 192-255 u_dot, then s_dot_bar.
    Cores cores;
    cores.open(barrier, slot, 256, a.counters, 6);
    const int count = *reinterpret_cast<volatile int*>(a.counters);
    float4* vbar4 = reinterpret_cast<float4*>(a.v_bar);
    float4* vdbar4 = reinterpret_cast<float4*>(a.v_dot_bar);

    for (int index = blockIdx.x; index * kTile < count; index += gridDim.x)
    {
        const int p = index * kTile + threadIdx.x;
        const PairTerms t = pair_terms(a, wbar, p, count);
        tile_first[threadIdx.x] = t.live ? t.ab.x : -1;
        cores.tile_index = index;
        store_basis_tangent(tile, tile_dot, t.g.w / a.width, -t.rate / a.width, a.gaussians,
                            t.live, pair_row(a, kRowG, p, t.live), pair_row(a, kRowGDot, p, t.live));
        if (!cores.run2(0, tile, image_b1, 64, tile_dot, image_b1, 1))
        {
            break;
        }
        store_activations(cores.tmem, bias1, tile, tile_dot, pair_row(a, kRowS, p, t.live),
                          pair_row(a, kRowSDot, p, t.live));
        if (!cores.run2(128, tile, image_b2, 192, tile_dot, image_b2, 2))
        {
            break;
        }
        uint4* row_ub = pair_row(a, kRowUBar, p, t.live);
        uint4* row_udb = pair_row(a, kRowUDotBar, p, t.live);
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
#pragma unroll
            for (int batch = 0; batch < 4; batch += kGatherBatch)
            {
                // The batch's gathers first (eight rows, kGatherBatch words each), so their
                // latencies overlap; dead rows read atom 0 and contribute zeros.
                uint4 raw[kGatherBatch][8];
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int k = 32 * half + 8 * (batch + i);
                    const std::int64_t ga = 8 * static_cast<std::int64_t>(t.ab.x) + k / 8;
                    const std::int64_t gb = 8 * static_cast<std::int64_t>(t.ab.y) + k / 8;
                    raw[i][0] = __ldg(a.v + ga);
                    raw[i][1] = __ldg(a.v + gb);
                    raw[i][2] = __ldg(a.v_dot + ga);
                    raw[i][3] = __ldg(a.v_dot + gb);
                    raw[i][4] = __ldg(a.m_bar + ga);
                    raw[i][5] = __ldg(a.m_bar + gb);
                    raw[i][6] = __ldg(a.m_dot_bar + ga);
                    raw[i][7] = __ldg(a.m_dot_bar + gb);
                }
#pragma unroll
                for (int i = 0; i < kGatherBatch; ++i)
                {
                    const int c = batch + i;
                    const int k = 32 * half + 8 * c;
                    float u[8];
                    float ud[8];
                    umma::load8(cores.tmem + 128 + k, u);
                    umma::load8(cores.tmem + 192 + k, ud);
                    umma::wait_loads();
                    float va[8], vb[8], vda[8], vdb[8], ma[8], mb[8], mda[8], mdb[8];
                    widen8(raw[i][0], va);
                    widen8(raw[i][1], vb);
                    widen8(raw[i][2], vda);
                    widen8(raw[i][3], vdb);
                    widen8(raw[i][4], ma);
                    widen8(raw[i][5], mb);
                    widen8(raw[i][6], mda);
                    widen8(raw[i][7], mdb);
                    float ub[8], udb[8], first[8], first_dot[8], to_second[8], to_second_dot[8];
#pragma unroll
                    for (int j = 0; j < 8; ++j)
                    {
                        const float raw_filter = u[j] + bias2[k + j];
                        const float f = raw_filter * t.envelope;
                        const float fd = ud[j] * t.envelope + raw_filter * t.moving;
                        const float fb = ma[j] * vb[j] + mb[j] * va[j] + mda[j] * vdb[j] +
                                         mdb[j] * vda[j];
                        const float fdb = mda[j] * vb[j] + mdb[j] * va[j];
                        to_second[j] = f * ma[j] + fd * mda[j];
                        to_second_dot[j] = f * mda[j];
                        first[j] = f * mb[j] + fd * mdb[j];
                        first_dot[j] = f * mdb[j];
                        ub[j] = fb * t.envelope + fdb * t.moving;
                        udb[j] = fdb * t.envelope;
                    }
                    if (t.live)
                    {
                        const std::int64_t gb = 8 * static_cast<std::int64_t>(t.ab.y) + k / 8;
#pragma unroll
                        for (int h4 = 0; h4 < 2; ++h4)
                        {
                            const int o = 4 * h4;
                            atomicAdd(vbar4 + 2 * gb + h4,
                                      make_float4(to_second[o], to_second[o + 1],
                                                  to_second[o + 2], to_second[o + 3]));
                            atomicAdd(vdbar4 + 2 * gb + h4,
                                      make_float4(to_second_dot[o], to_second_dot[o + 1],
                                                  to_second_dot[o + 2], to_second_dot[o + 3]));
                        }
                    }
                    put_run_part(stage, 2 * c, make_float4(first[0], first[1], first[2], first[3]));
                    put_run_part(stage, 2 * c + 1,
                                 make_float4(first[4], first[5], first[6], first[7]));
                    put_run_part(stage_dot, 2 * c,
                                 make_float4(first_dot[0], first_dot[1], first_dot[2], first_dot[3]));
                    put_run_part(stage_dot, 2 * c + 1,
                                 make_float4(first_dot[4], first_dot[5], first_dot[6], first_dot[7]));
                    const int column = 4 * half + c;
                    const uint4 word = umma::pack8(ub);
                    const uint4 word_dot = umma::pack8(udb);
                    *reinterpret_cast<uint4*>(tile + umma::image_offset(threadIdx.x, 8 * column)) =
                        word;
                    *reinterpret_cast<uint4*>(tile_dot +
                                              umma::image_offset(threadIdx.x, 8 * column)) =
                        word_dot;
                    if (row_ub != nullptr)
                    {
                        row_ub[column] = word;
                        row_udb[column] = word_dot;
                    }
                }
            }
            // the stages are this kernel's own: only this warp writes their rows again
            sum_runs(stage, tile_first, a.v_bar, half, false);
            sum_runs(stage_dot, tile_first, a.v_dot_bar, half, false);
        }
        if (!cores.run2(128, tile, image_b2t, 192, tile_dot, image_b2t, 3))
        {
            break;
        }
        uint4* row_zb = pair_row(a, kRowZBar, p, t.live);
        uint4* row_zdb = pair_row(a, kRowZDotBar, p, t.live);
#pragma unroll
        for (int half = 0; half < 2; ++half)
        {
            float sb[32];
            float sdb[32];
            float z[32];
            float zd[32];
            umma::load32(cores.tmem + 128 + 32 * half, sb);
            umma::load32(cores.tmem + 192 + 32 * half, sdb);
            umma::load32(cores.tmem + 32 * half, z);
            umma::load32(cores.tmem + 64 + 32 * half, zd);
            umma::wait_loads();
#pragma unroll
            for (int c = 0; c < 4; ++c)
            {
                float zb[8];
                float zdb[8];
#pragma unroll
                for (int e = 0; e < 8; ++e)
                {
                    const int i = 8 * c + e;
                    const float sg = sigmoid(z[i] + bias1[32 * half + i]);
                    zb[e] = sb[i] * sg + sdb[i] * zd[i] * sg * (1.0f - sg);
                    zdb[e] = sdb[i] * sg;
                }
                if (row_zb != nullptr)
                {
                    row_zb[4 * half + c] = umma::pack8(zb);
                    row_zdb[4 * half + c] = umma::pack8(zdb);
                }
            }
        }
    }
    cores.close(256);
}

// Rows [count, capacity) of the eight per-pair arrays set to zero, the pair count read from the
// workspace's counters, so sums over every row of an array equal sums over the pairs.
__global__ void zero_tail_kernel(uint4* rows, std::int64_t capacity, const int* counters)
{
    const std::int64_t count = *reinterpret_cast<const volatile int*>(counters);
    const std::int64_t words = (capacity - count) * 8;  // 16-byte words past the count, per array
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t i = blockIdx.x * static_cast<std::int64_t>(blockDim.x) + threadIdx.x;
         i < 8 * words; i += stride)
    {
        const std::int64_t array = i / words;
        rows[(array * capacity + count) * 8 + i % words] = make_uint4(0u, 0u, 0u, 0u);
    }
}

}  // namespace
}  // namespace nd

extern "C" {

int nd_schnet_tangent(const nd_schnet_tangent_args* args, int32_t direction,
                      nd_stream_t stream_handle)
{
    using namespace nd;
    ND_REQUIRE(args != nullptr, "args is null");
    ND_REQUIRE(direction == 0 || direction == 1, "direction must be 0 (forward) or 1 (reverse)");
    const nd_schnet_tangent_args& s = *args;
    ND_REQUIRE(s.num_atoms >= 1 && s.num_atoms <= (int64_t{1} << 30), "num_atoms out of range");
    ND_REQUIRE(s.num_columns >= 0 && s.num_columns < (int64_t{1} << 31), "num_columns out of range");
    ND_REQUIRE(s.interactions >= 1 && s.interactions <= 64, "interactions out of range");
    ND_REQUIRE(s.block >= 0 && s.block < s.interactions, "block out of range");
    ND_REQUIRE(s.num_types >= 1, "num_types must be positive");
    ND_REQUIRE(s.gaussians >= 2 && s.gaussians <= 64, "gaussians must lie in [2, 64]");
    ND_REQUIRE(s.cutoff > 0.0, "cutoff must be positive");
    ND_REQUIRE(s.weights && s.workspace && s.force_adjoint && s.virial_adjoint && s.v && s.v_dot &&
                   s.status,
               "a required buffer is null");
    ND_REQUIRE(reinterpret_cast<std::uintptr_t>(s.workspace) % 256 == 0 &&
                   reinterpret_cast<std::uintptr_t>(s.weights) % 256 == 0,
               "weights and workspace must be 256-byte aligned");
    auto aligned16 = [](const void* pointer) {
        return reinterpret_cast<std::uintptr_t>(pointer) % 16 == 0;
    };
    ND_REQUIRE(aligned16(s.v) && aligned16(s.v_dot) && aligned16(s.m) && aligned16(s.m_dot) &&
                   aligned16(s.m_bar) && aligned16(s.m_dot_bar) && aligned16(s.v_bar) &&
                   aligned16(s.v_dot_bar),
               "feature rows must be 16-byte aligned");
    if (direction == 0)
    {
        ND_REQUIRE(s.m && s.m_dot, "the forward pass needs m and m_dot");
    }
    else
    {
        ND_REQUIRE(s.m_bar && s.m_dot_bar && s.v_bar && s.v_dot_bar && s.pair_rows,
                   "the reverse pass needs m_bar, m_dot_bar, v_bar, v_dot_bar and pair_rows");
        ND_REQUIRE(s.capacity >= s.num_columns, "capacity must be at least num_columns");
        ND_REQUIRE(reinterpret_cast<std::uintptr_t>(s.pair_rows) % 16 == 0,
                   "pair_rows must be 16-byte aligned");
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_handle);
    const WeightLayout wl(s.interactions, s.num_types);
    const Workspace ws(s.num_atoms, s.num_columns, s.interactions);
    auto* weights = static_cast<const unsigned char*>(s.weights);
    auto* base = static_cast<unsigned char*>(s.workspace);

    TangentPass pass{};
    pass.pairs = reinterpret_cast<const int2*>(base + ws.pairs);
    pass.geometry = reinterpret_cast<const float4*>(base + ws.geometry);
    pass.counters = reinterpret_cast<int*>(base + ws.counters);
    pass.images = weights + static_cast<std::int64_t>(s.block) * kImagesPerBlock * umma::kImageBytes;
    pass.b1 = reinterpret_cast<const float*>(weights + wl.vectors + (static_cast<std::int64_t>(s.block) * 4) * kFeatures * 4);
    pass.b2 = reinterpret_cast<const float*>(weights + wl.vectors + (static_cast<std::int64_t>(s.block) * 4 + 1) * kFeatures * 4);
    pass.force_adjoint = s.force_adjoint;
    pass.virial_adjoint = s.virial_adjoint;
    pass.v = static_cast<const uint4*>(s.v);
    pass.v_dot = static_cast<const uint4*>(s.v_dot);
    pass.m = s.m;
    pass.m_dot = s.m_dot;
    pass.m_bar = static_cast<const uint4*>(s.m_bar);
    pass.m_dot_bar = static_cast<const uint4*>(s.m_dot_bar);
    pass.v_bar = s.v_bar;
    pass.v_dot_bar = s.v_dot_bar;
    pass.rows = static_cast<uint4*>(s.pair_rows);
    pass.capacity = s.capacity;
    pass.width = static_cast<float>(s.cutoff / (s.gaussians - 1));
    pass.phase = static_cast<float>(3.14159265358979323846 / s.cutoff);
    pass.gaussians = s.gaussians;

    // The kernels' attributes, set once per device (they belong to its instance of a kernel).
    static DeviceOnce configured;  // per device, retried after a failure
    ND_CUDA_TRY(configured.run([] {
        cudaError_t rc = cudaFuncSetAttribute(tangent_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTangentForwardShared);
        auto then = [&rc](cudaError_t next) { rc = rc != cudaSuccess ? rc : next; };
        then(cudaFuncSetAttribute(tangent_reverse_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTangentReverseShared));
        then(cudaFuncSetAttribute(tangent_forward_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
        then(cudaFuncSetAttribute(tangent_reverse_kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared));
        return rc;
    }));
    if (direction == 0)
    {
        // The messages m are the E/F/W call's for this block; only their tangent is computed.
        const std::int64_t row_bytes = align256(s.num_atoms * kFeatures * 4);
        ND_CUDA_TRY(cudaMemcpyAsync(s.m, base + ws.m + s.block * row_bytes,
                                    s.num_atoms * kFeatures * sizeof(float),
                                    cudaMemcpyDeviceToDevice, stream));
        const int grid = pair_grid(reinterpret_cast<const void*>(tangent_forward_kernel), kTangentForwardShared, 128);
        tangent_forward_kernel<<<grid, kTile, kTangentForwardShared, stream>>>(pass);
    }
    else
    {
        const int grid = pair_grid(reinterpret_cast<const void*>(tangent_reverse_kernel), kTangentReverseShared, 256);
        tangent_reverse_kernel<<<grid, kTile, kTangentReverseShared, stream>>>(pass);
        ND_LAUNCH_CHECK();
        zero_tail_kernel<<<std::min<std::int64_t>(1184, blocks_for(s.capacity * 8)), kThreads, 0, stream>>>(
            pass.rows, s.capacity, pass.counters);
    }
    ND_LAUNCH_CHECK();
    ND_CUDA_TRY(cudaMemcpyAsync(s.status, pass.counters, 4 * sizeof(int), cudaMemcpyDeviceToDevice, stream));
    return ND_OK;
}

}  // extern "C"
