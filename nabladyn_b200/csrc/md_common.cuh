// Device pieces shared by the MD engine (md.cu) and the replica server (serve.cu): the atom
// vector, Lennard-Jones pair parameters, the chunked neighbor-list layout and its writers, and
// the Nose-Hoover chain half step.

#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"

namespace nd {

template <typename T>
struct alignas(4 * sizeof(T)) Pos4
{
    T x, y, z, w;
};

// Offsets into the float64 thermostat block.
enum Thermo : int
{
    kChainA = 0,      // q[3], p[3] after the last closing half step
    kKineticA = 6,    // carried K after the last closing half step
    kChainB = 7,      // q[3], p[3] after this step's opening half step
    kKineticB = 13,   // carried K after the opening
    kPendingScale = 14,  // the closing factor not yet applied to the stored velocities
    kOpenScale = 15,  // this step's opening factor
    kChainMass = 16,  // Q[3]
    kThermalEnergy = 19,  // kT
    kDegrees = 20,    // g = 3N - 3
    kTimestep = 21,
    kThermoSize = 24,
};

// ---------------------------------------------------------------------------------------
// Lennard-Jones parameters of a type pair, prepared once per block.

template <typename T>
struct PairParams
{
    T s2;     // sigma^2
    T e4;     // 4 eps
    T e24;    // 24 eps
    T shift;  // u(r_c)
};

template <typename T>
__device__ __forceinline__ PairParams<T> pair_params(T sigma, T epsilon, T cutoff_squared)
{
    PairParams<T> p;
    p.s2 = sigma * sigma;
    p.e4 = T(4) * epsilon;
    p.e24 = T(24) * epsilon;
    const T q = p.s2 / cutoff_squared;
    const T q6 = q * q * q;
    p.shift = p.e4 * (q6 * q6 - q6);
    return p;
}

// 1 / x by the hardware's approximate reciprocal (at most 1 ulp off). The .ftz form is the
// single instruction; it differs from the plain form only for subnormal inputs or results,
// which a squared distance between 1e-19 nm and 1e18 nm (the far sentinel) never produces.
__device__ __forceinline__ float fast_reciprocal(float x)
{
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

__device__ __forceinline__ double fast_reciprocal(double x)
{
    return 1.0 / x;
}

__device__ __forceinline__ int type_pair_row(int a, int b, int num_types)
{
    const int low = a < b ? a : b;
    const int high = a < b ? b : a;
    return low * (2 * num_types - low - 1) / 2 + high;
}

// The sentinel: an atom so far away that every distance to it fails the cutoff, yet stays
// finite in float32 (1e18 nm squared is 3e36), so its masked force is an exact zero.
template <typename T>
__device__ __forceinline__ Pos4<T> far_atom()
{
    return Pos4<T>{T(1e18), T(1e18), T(1e18), T(0)};
}

// The geometry of one brick's tile in shared memory. Row r = 3 (dz + 1) + (dy + 1) holds the
// tile cells c = 0 .. cells_per_row - 1 at x = x0 - 1 + c. start[r * cells_per_row + c] is
// the tile slot of the cell's first atom (the last entry is the tile size), first[...] the
// cell's first cell-order slot.
struct TileShape
{
    int cells_per_row;
    int size;
    int home_first;  // cell-order slots [home_first, home_end) are the brick's centers
    int home_end;
    int x0, x1, y, z;  // the brick: home cells x0 <= x < x1 of row (y, z)
    int pairs;         // center pairs of the home cells (two per pair, none across cells)
};

// The list stores each center's entries in chunks of kChunk uint16 indices, one 16-B word per
// chunk, interleaved by warps of 32 cell-order slots: chunk c of center i is word
// ((i / 32) * (width / kChunk) + c) * 32 + i % 32. A lane reads 8 neighbors with one load and
// a warp reads 512 contiguous bytes; a partial last chunk is padded with the sentinel.
constexpr int kChunk = 8;

__device__ __forceinline__ std::int64_t chunk_index(int center, int chunk, int width)
{
    return ((static_cast<std::int64_t>(center) >> 5) * (width / kChunk) + chunk) * kWarp +
           (center & 31);
}

// Collects one center's entries in registers and stores them a chunk at a time; unused slots
// of a chunk hold `pad`, the sentinel.
struct ListWriter
{
    uint4* chunks;
    int width;
    int center;
    unsigned long long pad;
    unsigned long long lo;
    unsigned long long hi;
    int count;

    __device__ __forceinline__ ListWriter(std::uint16_t* list, int width_, int center_,
                                          unsigned pad_index)
        : chunks(reinterpret_cast<uint4*>(list)), width(width_), center(center_),
          pad(0x0001000100010001ull * pad_index), lo(pad), hi(pad), count(0)
    {
    }

    __device__ __forceinline__ void add(unsigned index)
    {
        if (count < width)
        {
            const int r = count & (kChunk - 1);
            const unsigned long long value = index;
            const int shift = 16 * (r & 3);
            if (r < 4)
            {
                lo = (lo & ~(0xffffull << shift)) | (value << shift);
            }
            else
            {
                hi = (hi & ~(0xffffull << shift)) | (value << shift);
            }
            if (r == kChunk - 1)
            {
                store(count / kChunk);
            }
        }
        ++count;
    }

    __device__ __forceinline__ void store(int chunk)
    {
        chunks[chunk_index(center, chunk, width)] =
            make_uint4(static_cast<unsigned>(lo), static_cast<unsigned>(lo >> 32),
                       static_cast<unsigned>(hi), static_cast<unsigned>(hi >> 32));
        lo = pad;
        hi = pad;
    }

    __device__ __forceinline__ void finish()
    {
        const int stored = count < width ? count : width;
        if (stored % kChunk != 0)
        {
            store(stored / kChunk);
        }
    }
};

// The same chunks, staged per lane in 16 bytes of shared memory: a hit is one 2-byte store, and
// every eighth hit stores the chunk to global memory in one 16-byte write. The brick list build
// uses it; its hits are sparse and divergent, so the per-hit work is what the warp pays.
struct StagedListWriter
{
    uint4* chunks;
    std::uint16_t* staged;  // this lane's 8 slots
    int width;
    int center;
    int count;

    __device__ __forceinline__ StagedListWriter(std::uint16_t* list, std::uint16_t* lane_slots,
                                                int width_, int center_)
        : chunks(reinterpret_cast<uint4*>(list)), staged(lane_slots), width(width_),
          center(center_), count(0)
    {
    }

    __device__ __forceinline__ void add(unsigned index)
    {
        if (count < width)
        {
            const int r = count & (kChunk - 1);
            staged[r] = static_cast<std::uint16_t>(index);
            if (r == kChunk - 1)
            {
                chunks[chunk_index(center, count / kChunk, width)] =
                    *reinterpret_cast<const uint4*>(staged);
            }
        }
        ++count;
    }

    // Stores a partial last chunk, its unused slots set to `pad`.
    __device__ __forceinline__ void finish(unsigned pad)
    {
        const int stored = count < width ? count : width;
        if (stored % kChunk != 0)
        {
            for (int r = stored % kChunk; r < kChunk; ++r)
            {
                staged[r] = static_cast<std::uint16_t>(pad);
            }
            chunks[chunk_index(center, stored / kChunk, width)] =
                *reinterpret_cast<const uint4*>(staged);
        }
    }
};

// The Nose-Hoover chain of three, advanced by half a step against the kinetic energy K
// (Martyna, Tuckerman, Tobias and Klein 1996; src/nabladyn/md/_ensembles/_chain.py:36-83).
// Returns the velocity scale; q and p advance in place and K is scaled. `inverse` holds 1 / Q
// of each link: the update is one dependent chain, and a product in place of each quotient
// p / Q takes the divisions off it (a difference in the last bit of float64).
__device__ inline double chain_half_step_inverse(double& kinetic, double* q, double* p,
                                                 const double* inverse, double degrees,
                                                 double kT, double dt)
{
    const double quarter = 0.25 * dt, eighth = 0.125 * dt;
    auto driving = [&](int k, double energy) {
        return k == 0 ? 2.0 * energy - degrees * kT : p[k - 1] * p[k - 1] * inverse[k - 1] - kT;
    };
    double damping[2];
    for (int k = 2; k >= 0; --k)
    {
        if (k == 2)
        {
            p[k] = p[k] + quarter * driving(k, kinetic);
        }
        else
        {
            const double kick = quarter * driving(k, kinetic);
            p[k] = damping[k] * (damping[k] * p[k] + kick);
        }
        if (k > 0)
        {
            damping[k - 1] = exp(-eighth * p[k] * inverse[k]);
        }
    }
    const double factor = exp(-0.5 * dt * p[0] * inverse[0]);
    double scaled = kinetic * (factor * factor);
    for (int k = 0; k < 3; ++k)
    {
        q[k] = q[k] + 0.5 * dt * p[k] * inverse[k];
    }
    for (int k = 0; k < 3; ++k)
    {
        if (k == 2)
        {
            p[k] = p[k] + quarter * driving(k, scaled);
        }
        else
        {
            const double kick = quarter * driving(k, scaled);
            p[k] = damping[k] * (damping[k] * p[k] + kick);
        }
    }
    kinetic = scaled;
    return factor;
}

// The same from the links' masses Q.
__device__ inline double chain_half_step(double& kinetic, double* q, double* p, const double* mass,
                                         double degrees, double kT, double dt)
{
    const double inverse[3] = {1.0 / mass[0], 1.0 / mass[1], 1.0 / mass[2]};
    return chain_half_step_inverse(kinetic, q, p, inverse, degrees, kT, dt);
}

}  // namespace nd
