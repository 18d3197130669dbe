// Periodic geometry shared by the neighbor operator and the MD engine.

#pragma once

#include "common.cuh"

namespace nd {

// r^2 of a displacement, with the contraction pinned: fma(dz, dz, fma(dx, dx, dy * dy)).
template <typename T>
__host__ __device__ __forceinline__ T squared_norm(T dx, T dy, T dz)
{
    return fma(dz, dz, fma(dx, dx, dy * dy));
}

// The bin of coordinate x in [0, L) along an axis of `count` bins of `width`; the quotient
// can round up to `count` at the far face, so the bin is clamped
// (reference: src/nabladyn/neighbors/csrc/grid/grid.cuh:10-20). The clamp is taken on the
// floating quotient, so a non-finite coordinate still lands in a valid bin (the status word
// reports it); for finite coordinates the bin is the reference's.
template <typename T>
__device__ __forceinline__ index_t axis_bin(T x, T width, index_t count)
{
    const T q = floor(x / width);
    return q >= static_cast<T>(count) ? count - 1 : (q >= T(0) ? static_cast<index_t>(q) : 0);
}

// center - other under the minimum image of a period `length`: the coordinate on the far side
// moves by L first, which is exact, so the difference is rounded once
// (reference: src/nabladyn/neighbors/csrc/common/traversal.cuh:31-38).
template <typename T>
__device__ __forceinline__ T min_image(T center, T other, T length)
{
    const T raw = center - other;
    const T half = T(0.5) * length;
    return raw > half ? (center - length) - other : (raw < -half ? center - (other - length) : raw);
}

// Wraps x into [0, L) and returns the lattice crossings, as src/nabladyn/space.py:22-38 does:
// floor of the quotient, then the two fix-ups in that order.
template <typename T>
__device__ __forceinline__ T wrap_axis(T x, T length, long long& crossings)
{
    T c = floor(x / length);
    T wrapped = x - c * length;
    if (wrapped < T(0))
    {
        wrapped += length;
        c -= T(1);
    }
    if (wrapped >= length)
    {
        wrapped -= length;
        c += T(1);
    }
    crossings = static_cast<long long>(c);
    return wrapped;
}

}  // namespace nd
