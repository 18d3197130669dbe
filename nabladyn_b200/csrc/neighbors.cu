// The neighbor operator: a cell-list half list of the pairs closer than the list radius,
// with the on-GPU skin-reuse check, behind the C-ABI of include/nabladyn_b200.h.
//
// The operator keeps the reference's contract exactly (src/nabladyn/neighbors/csrc/ops.h:12-89,
// entry_points.cu:284-508): the same buffers, the same status bits, the same pair set (each
// pair found once, from the lower sorted index), padding columns k holding (k mod N, k mod N),
// and every rebuild kernel gated by a device flag so one CUDA Graph holds the whole update.
//
// What differs is how a build runs on the GPU:
//   * binning takes its in-bin slot from the counting atomic, so the scatter needs no atomics;
//   * one warp per bin orders the bin by atom id with register shuffles and gathers the sorted
//     positions in the same pass (the reference ranks from global memory, then gathers);
//   * the scans are our own gated kernels (scan.cuh), so an update that reuses its pairs runs
//     no scan at all;
//   * the pair total and the padding share one launch.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <limits>

#include "common.cuh"
#include "geometry.cuh"
#include "scan.cuh"

namespace nd {

// ---------------------------------------------------------------------------------------
// The traversal.

// One neighbor bin along one axis of a 27-bin stencil: its index and the image split of its
// shift s in {-L, 0, L}: the difference is (center - lead) - (other + trail), where lead = s
// when s > 0 and trail = s when s < 0, so each side moves by an exact multiple of L and the
// difference rounds once (reference: traversal.cuh:9-28, 40-57).
template <typename T>
struct StencilAxis
{
    index_t bin[3];
    T lead[3];   // center - lead, per step -1, 0, +1
    T trail[3];  // other + trail

    __device__ __forceinline__ StencilAxis(index_t home, index_t count, T center, T length)
    {
#pragma unroll
        for (int s = 0; s < 3; ++s)
        {
            const index_t raw = home + s - 1;
            const T shift = raw < 0 ? -length : (raw >= count ? length : T(0));
            bin[s] = raw < 0 ? raw + count : (raw >= count ? raw - count : raw);
            lead[s] = shift > T(0) ? center - shift : center;
            trail[s] = shift < T(0) ? shift : T(0);
        }
    }
};

// Calls visit(k) for every sorted atom k > center, in the 27 (or, on short axes, all) bins
// around the center's bin, that lies closer than sqrt(radius_squared). With three or more bins
// on every axis each stencil bin has a fixed image; otherwise every candidate takes its minimum
// image. The visiting order (z, y, x bins; ascending sorted index) fixes the fill order.
template <typename T, typename Visit>
__device__ __forceinline__ void visit_listed(
    const T* __restrict__ sorted_positions,
    const index_t* __restrict__ sorted_ids,
    const index_t* __restrict__ atom_bin,
    const index_t* __restrict__ bin_offsets,
    const index_t* __restrict__ dims,
    const T* __restrict__ cell,
    T radius_squared,
    index_t center,
    Visit& visit
)
{
    const T cx = sorted_positions[3LL * center];
    const T cy = sorted_positions[3LL * center + 1];
    const T cz = sorted_positions[3LL * center + 2];
    const index_t nx = dims[0], ny = dims[1], nz = dims[2];
    const index_t home = atom_bin[sorted_ids[center]];
    const index_t hx = home % nx, hy = (home / nx) % ny, hz = home / (nx * ny);
    if (nx >= 3 && ny >= 3 && nz >= 3)
    {
        const StencilAxis<T> ax(hx, nx, cx, cell[0]);
        const StencilAxis<T> ay(hy, ny, cy, cell[1]);
        const StencilAxis<T> az(hz, nz, cz, cell[2]);
#pragma unroll
        for (int sz = 0; sz < 3; ++sz)
        {
#pragma unroll
            for (int sy = 0; sy < 3; ++sy)
            {
                const index_t row = nx * (ay.bin[sy] + ny * az.bin[sz]);
#pragma unroll
                for (int sx = 0; sx < 3; ++sx)
                {
                    const index_t bin = ax.bin[sx] + row;
                    const index_t first = bin_offsets[bin];
                    const index_t end = bin_offsets[bin + 1];
                    for (index_t k = first > center ? first : center + 1; k < end; ++k)
                    {
                        const T* p = sorted_positions + 3LL * k;
                        const T dx = ax.lead[sx] - (p[0] + ax.trail[sx]);
                        const T dy = ay.lead[sy] - (p[1] + ay.trail[sy]);
                        const T dz = az.lead[sz] - (p[2] + az.trail[sz]);
                        if (squared_norm(dx, dy, dz) < radius_squared)
                        {
                            visit(k);
                        }
                    }
                }
            }
        }
        return;
    }
    // An axis with fewer than three bins is searched whole; one with three or more, around home.
    const int span_x = nx >= 3 ? 3 : nx, span_y = ny >= 3 ? 3 : ny, span_z = nz >= 3 ? 3 : nz;
    auto around = [](index_t h, int step, index_t count) {
        const index_t raw = h + step - 1;
        return raw < 0 ? raw + count : (raw >= count ? raw - count : raw);
    };
    for (int iz = 0; iz < span_z; ++iz)
    {
        const index_t bz = nz >= 3 ? around(hz, iz, nz) : iz;
        for (int iy = 0; iy < span_y; ++iy)
        {
            const index_t by = ny >= 3 ? around(hy, iy, ny) : iy;
            for (int ix = 0; ix < span_x; ++ix)
            {
                const index_t bin = (nx >= 3 ? around(hx, ix, nx) : ix) + nx * (by + ny * bz);
                const index_t first = bin_offsets[bin];
                const index_t end = bin_offsets[bin + 1];
                for (index_t k = first > center ? first : center + 1; k < end; ++k)
                {
                    const T* p = sorted_positions + 3LL * k;
                    const T dx = min_image(cx, p[0], cell[0]);
                    const T dy = min_image(cy, p[1], cell[1]);
                    const T dz = min_image(cz, p[2], cell[2]);
                    if (squared_norm(dx, dy, dz) < radius_squared)
                    {
                        visit(k);
                    }
                }
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// Grid: counting sort of the atoms by bin, ordered by atom id inside each bin.

// Bins each atom and takes its slot in the bin from the counting atomic. The slots are parked
// in `slots` (the pair_counts buffer, rewritten by the count that follows).
template <typename T>
__global__ void bin_atoms_kernel(
    const T* __restrict__ positions,
    const index_t* __restrict__ dims,
    const T* __restrict__ widths,
    index_t num_atoms,
    index_t* __restrict__ atom_bin,
    index_t* __restrict__ bin_counts,
    index_t* __restrict__ slots,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t atom = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (atom >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    const T* p = positions + 3 * atom;
    const index_t nx = dims[0], ny = dims[1], nz = dims[2];
    const index_t bin = axis_bin(p[0], widths[0], nx) +
                        nx * (axis_bin(p[1], widths[1], ny) + ny * axis_bin(p[2], widths[2], nz));
    atom_bin[atom] = bin;
    slots[atom] = atomicAdd(bin_counts + bin, 1);
}

// Places each atom at its bin's offset plus its slot and returns the counts to zero for the
// next build.
__global__ void place_atoms_kernel(
    const index_t* __restrict__ atom_bin,
    const index_t* __restrict__ slots,
    const index_t* __restrict__ bin_offsets,
    index_t num_atoms,
    index_t* __restrict__ bin_counts,
    index_t* __restrict__ unordered_ids,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t atom = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (atom >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    const index_t bin = atom_bin[atom];
    unordered_ids[bin_offsets[bin] + slots[atom]] = static_cast<index_t>(atom);
    bin_counts[bin] = 0;
}

// One warp per bin: each atom's rank is the number of smaller ids in its bin, counted with
// shuffles; the warp writes the sorted ids and gathers the sorted positions.
template <typename T>
__global__ void order_bins_kernel(
    const T* __restrict__ positions,
    const index_t* __restrict__ unordered_ids,
    const index_t* __restrict__ bin_offsets,
    std::int64_t num_bins,
    index_t* __restrict__ sorted_ids,
    T* __restrict__ sorted_positions,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t bin =
        (static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp;
    const int lane = threadIdx.x % kWarp;
    if (bin >= num_bins || !rebuilding(rebuild, status))
    {
        return;  // whole warps return together
    }
    const index_t begin = bin_offsets[bin];
    const index_t count = bin_offsets[bin + 1] - begin;
    for (index_t mine = 0; mine < count; mine += kWarp)
    {
        const bool active = mine + lane < count;
        const index_t id = active ? unordered_ids[begin + mine + lane] : 0;
        index_t rank = 0;
        for (index_t base = 0; base < count; base += kWarp)
        {
            const index_t other =
                base + lane < count ? unordered_ids[begin + base + lane] : 0x7fffffff;
            const int valid = count - base < kWarp ? count - base : kWarp;
            for (int s = 0; s < valid; ++s)
            {
                rank += __shfl_sync(kFullMask, other, s) < id;
            }
        }
        if (active)
        {
            const index_t slot = begin + rank;
            sorted_ids[slot] = id;
            sorted_positions[3LL * slot] = positions[3LL * id];
            sorted_positions[3LL * slot + 1] = positions[3LL * id + 1];
            sorted_positions[3LL * slot + 2] = positions[3LL * id + 2];
        }
    }
}

// ---------------------------------------------------------------------------------------
// Pairs on the grid path.

struct CountVisit
{
    index_t count;
    __device__ __forceinline__ void operator()(index_t) { ++count; }
};

// Writes (center id, neighbor id) from the center's first column; columns at or past the
// capacity are counted but not written.
struct FillVisit
{
    const index_t* __restrict__ sorted_ids;
    index_t center_id;
    std::int64_t column;
    std::int64_t capacity;
    index_t* __restrict__ pairs;

    __device__ __forceinline__ void operator()(index_t neighbor)
    {
        if (column < capacity)
        {
            pairs[column] = center_id;
            pairs[capacity + column] = sorted_ids[neighbor];
        }
        ++column;
    }
};

template <typename T>
__global__ void count_pairs_kernel(
    const T* __restrict__ sorted_positions,
    const index_t* __restrict__ sorted_ids,
    const index_t* __restrict__ atom_bin,
    const index_t* __restrict__ bin_offsets,
    const index_t* __restrict__ dims,
    const T* __restrict__ cell,
    T radius_squared,
    index_t num_atoms,
    index_t* __restrict__ pair_counts,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t center = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (center >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    CountVisit visit{0};
    visit_listed(sorted_positions, sorted_ids, atom_bin, bin_offsets, dims, cell, radius_squared,
                 static_cast<index_t>(center), visit);
    pair_counts[center] = visit.count;
}

template <typename T>
__global__ void fill_pairs_kernel(
    const T* __restrict__ sorted_positions,
    const index_t* __restrict__ sorted_ids,
    const index_t* __restrict__ atom_bin,
    const index_t* __restrict__ bin_offsets,
    const index_t* __restrict__ dims,
    const T* __restrict__ cell,
    const index_t* __restrict__ pair_offsets,
    T radius_squared,
    index_t num_atoms,
    index_t capacity,
    index_t* __restrict__ pairs,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t center = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (center >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    FillVisit visit{sorted_ids, sorted_ids[center], pair_offsets[center], capacity, pairs};
    visit_listed(sorted_positions, sorted_ids, atom_bin, bin_offsets, dims, cell, radius_squared,
                 static_cast<index_t>(center), visit);
}

// ---------------------------------------------------------------------------------------
// The all-pairs path, for lists whose first grid has at most three bins on every axis.

__host__ __device__ __forceinline__ std::int64_t bit_words(std::int64_t num_atoms)
{
    return (num_atoms + kWarp - 1) / kWarp;
}

constexpr int kAllPairsThreads = 128;

// One warp per atom: every atom with a higher id is tested once, 32 per ballot, and the hits
// are kept as the atom's bit row, so the fill computes no distance again.
template <typename T>
__global__ void test_all_pairs_kernel(
    const T* __restrict__ positions,
    const T* __restrict__ cell,
    T radius_squared,
    index_t num_atoms,
    std::uint32_t* __restrict__ bits,
    index_t* __restrict__ pair_counts,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t thread = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const std::int64_t center = thread / kWarp;
    if (center >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    const int lane = static_cast<int>(thread % kWarp);
    const std::int64_t words = bit_words(num_atoms);
    const T cx = positions[3 * center], cy = positions[3 * center + 1],
            cz = positions[3 * center + 2];
    const T lx = cell[0], ly = cell[1], lz = cell[2];
    index_t count = 0;
    for (std::int64_t word = (center + 1) / kWarp; word < words; ++word)
    {
        const std::int64_t other = word * kWarp + lane;
        bool hit = false;
        if (other > center && other < num_atoms)
        {
            const T* p = positions + 3 * other;
            hit = squared_norm(min_image(cx, p[0], lx), min_image(cy, p[1], ly),
                               min_image(cz, p[2], lz)) < radius_squared;
        }
        const unsigned hits = __ballot_sync(kFullMask, hit);
        if (lane == 0)
        {
            bits[center * words + word] = hits;
        }
        count += __popc(hits);
    }
    if (lane == 0)
    {
        pair_counts[center] = count;
    }
}

// Writes each atom's pairs from its bit row, from its first column on, in lane order.
__global__ void fill_all_pairs_kernel(
    const std::uint32_t* __restrict__ bits,
    const index_t* __restrict__ pair_offsets,
    index_t num_atoms,
    index_t capacity,
    index_t* __restrict__ pairs,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t thread = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    const std::int64_t center = thread / kWarp;
    if (center >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    const int lane = static_cast<int>(thread % kWarp);
    const unsigned below = (1u << lane) - 1u;
    const std::int64_t words = bit_words(num_atoms);
    std::int64_t column = pair_offsets[center];
    for (std::int64_t word = (center + 1) / kWarp; word < words; ++word)
    {
        const unsigned hits = bits[center * words + word];
        if ((hits >> lane) & 1u)
        {
            const std::int64_t slot = column + __popc(hits & below);
            if (slot < capacity)
            {
                pairs[slot] = static_cast<index_t>(center);
                pairs[capacity + slot] = static_cast<index_t>(word * kWarp + lane);
            }
        }
        column += __popc(hits);
    }
}

// ---------------------------------------------------------------------------------------
// Total, overflow and padding, in one launch over the capacity.

// Every thread derives the total from the last count and offset. Column k at or past the
// total holds the self-pair (k mod N, k mod N), spreading their zero gradients over the atoms.
// Thread 0 stores the total and, above the capacity, the overflow bit and the pairs needed;
// with an overflow there is no padding column, so the gate's read of the status cannot race.
__global__ void total_and_pad_kernel(
    const index_t* __restrict__ pair_counts,
    const index_t* __restrict__ pair_offsets,
    index_t num_atoms,
    index_t capacity,
    index_t* __restrict__ pair_total,
    index_t* __restrict__ pairs,
    index_t* __restrict__ status,
    const index_t* __restrict__ rebuild
)
{
    const std::int64_t column = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (!rebuilding(rebuild, status))
    {
        return;
    }
    const index_t total = pair_offsets[num_atoms - 1] + pair_counts[num_atoms - 1];
    if (column == 0)
    {
        pair_total[0] = total;
        if (total > capacity)
        {
            status[0] |= kOverflow;
            status[1] = total > status[1] ? total : status[1];
        }
    }
    if (column < capacity && column >= total)
    {
        const index_t atom = static_cast<index_t>(column % num_atoms);
        pairs[column] = atom;
        pairs[capacity + column] = atom;
    }
}

// ---------------------------------------------------------------------------------------
// The update: the cell check, the reuse rule and the commit of a rebuild
// (reference: src/nabladyn/neighbors/csrc/update/update.cuh:21-145).
//
// A rebuild stores the wrapped positions x0 and the cell L0. In a cell L, with s = L / L0 per
// axis, atom i has moved d_i = min image of x_i - s x0_i; the pairs are reused while every
// |d_i|^2 < ((R min(s) - cutoff - 32 eps L_max) / 2)^2.

constexpr int kThresholdSquared = 0;
constexpr int kScale = 1;

template <typename T>
__global__ void prepare_update_kernel(
    const T* __restrict__ cell,
    const T* __restrict__ reference_cell,
    T cutoff,
    T radius,
    T epsilon,
    const index_t* __restrict__ limits,
    index_t* __restrict__ dims,
    T* __restrict__ widths,
    T* __restrict__ reuse,
    index_t* __restrict__ rebuild,
    index_t* __restrict__ status
)
{
    rebuild[0] = 0;
    if (status[0] != 0)
    {
        return;
    }
    T smallest = cell[0] / reference_cell[0];
    T longest = cell[0];
    for (int axis = 0; axis < 3; ++axis)
    {
        const T length = cell[axis];
        if (!(isfinite(length) && length > 2 * cutoff))
        {
            status[0] |= kInvalidCell;
            return;
        }
        const T scale = length / reference_cell[axis];
        reuse[kScale + axis] = scale;
        smallest = scale < smallest ? scale : smallest;
        longest = length > longest ? length : longest;
        // Each bin keeps a margin of a few roundings of L.
        const T fit = floor(length / fma(T(4) * epsilon, length, radius));
        const index_t count =
            fit < 1 ? 1 : (fit > limits[axis] ? limits[axis] : static_cast<index_t>(fit));
        dims[axis] = count;
        widths[axis] = length / count;
    }
    const T allowance = fma(-(T(32) * epsilon), longest, fma(radius, smallest, -cutoff));
    if (allowance <= 0)
    {
        rebuild[0] = 1;
        return;
    }
    reuse[kThresholdSquared] = allowance * allowance / 4;
}

template <typename T>
__global__ void check_reuse_kernel(
    const T* __restrict__ positions,
    const T* __restrict__ reference_positions,
    const T* __restrict__ cell,
    const T* __restrict__ reuse,
    index_t num_atoms,
    index_t* __restrict__ rebuild,
    index_t* __restrict__ status
)
{
    const std::int64_t atom = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (atom >= num_atoms || status[0] != 0)
    {
        return;
    }
    const T* x = positions + 3 * atom;
    const T* x0 = reference_positions + 3 * atom;
    if (!(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2])))
    {
        atomicOr(status, kNonFinite);
        return;
    }
    if (rebuild[0] != 0)
    {
        return;
    }
    T moved = 0;
    for (int axis = 0; axis < 3; ++axis)
    {
        const T d = min_image(x[axis], reuse[kScale + axis] * x0[axis], cell[axis]);
        moved = fma(d, d, moved);
    }
    if (moved >= reuse[kThresholdSquared])
    {
        rebuild[0] = 1;  // every writer stores the same value
    }
}

template <typename T>
__global__ void commit_rebuild_kernel(
    const T* __restrict__ positions,
    const T* __restrict__ cell,
    index_t num_atoms,
    T* __restrict__ reference_positions,
    T* __restrict__ reference_cell,
    index_t* __restrict__ rebuild_count,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t index = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (index >= 3LL * num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    reference_positions[index] = positions[index];
    if (index < 3)
    {
        reference_cell[index] = cell[index];
    }
    if (index == 0)
    {
        ++rebuild_count[0];
    }
}

// ---------------------------------------------------------------------------------------
// Host launchers.

struct List
{
    const nd_neighbor_buffers* b;
    const index_t* rebuild;  // null: a build from allocate, which always runs

    bool all_pairs() const { return b->bits_numel > 0; }
    index_t* status() const { return b->status; }
};

template <typename T>
int launch_grid(const T* positions, std::int64_t n, const List& list, cudaStream_t stream)
{
    const nd_neighbor_buffers& b = *list.b;
    const auto num_atoms = static_cast<index_t>(n);
    bin_atoms_kernel<T><<<blocks_for(n), kThreads, 0, stream>>>(
        positions, b.dims, static_cast<const T*>(b.widths), num_atoms, b.atom_bin, b.bin_counts,
        b.pair_counts, list.rebuild, b.status);
    ND_LAUNCH_CHECK();
    ND_CUDA_TRY(scan_exclusive(b.bin_counts, b.bin_offsets, b.num_bin_slots, b.scan_temp,
                               list.rebuild, b.status, stream));
    place_atoms_kernel<<<blocks_for(n), kThreads, 0, stream>>>(
        b.atom_bin, b.pair_counts, b.bin_offsets, num_atoms, b.bin_counts, b.unordered_ids,
        list.rebuild, b.status);
    ND_LAUNCH_CHECK();
    const std::int64_t bins = b.num_bin_slots - 1;
    order_bins_kernel<T><<<blocks_for(bins * kWarp), kThreads, 0, stream>>>(
        positions, b.unordered_ids, b.bin_offsets, bins, b.sorted_ids,
        static_cast<T*>(b.sorted_positions), list.rebuild, b.status);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

template <typename T>
int launch_count(const T* positions, const T* cell, std::int64_t n, double radius,
                 const List& list, cudaStream_t stream)
{
    const nd_neighbor_buffers& b = *list.b;
    const auto num_atoms = static_cast<index_t>(n);
    const T r = static_cast<T>(radius);
    if (list.all_pairs())
    {
        test_all_pairs_kernel<T><<<blocks_for(n * kWarp, kAllPairsThreads), kAllPairsThreads, 0,
                                   stream>>>(
            positions, cell, r * r, num_atoms, reinterpret_cast<std::uint32_t*>(b.bits),
            b.pair_counts, list.rebuild, b.status);
    }
    else
    {
        count_pairs_kernel<T><<<blocks_for(n), kThreads, 0, stream>>>(
            static_cast<const T*>(b.sorted_positions), b.sorted_ids, b.atom_bin, b.bin_offsets,
            b.dims, cell, r * r, num_atoms, b.pair_counts, list.rebuild, b.status);
    }
    ND_LAUNCH_CHECK();
    ND_CUDA_TRY(scan_exclusive(b.pair_counts, b.pair_offsets, n, b.scan_temp, list.rebuild,
                               b.status, stream));
    return ND_OK;
}

template <typename T>
int launch_fill(const T* cell, std::int64_t n, double radius, const List& list,
                cudaStream_t stream)
{
    const nd_neighbor_buffers& b = *list.b;
    const auto num_atoms = static_cast<index_t>(n);
    const auto capacity = static_cast<index_t>(b.capacity);
    const T r = static_cast<T>(radius);
    if (list.all_pairs())
    {
        fill_all_pairs_kernel<<<blocks_for(n * kWarp, kAllPairsThreads), kAllPairsThreads, 0,
                                stream>>>(
            reinterpret_cast<const std::uint32_t*>(b.bits), b.pair_offsets, num_atoms, capacity,
            b.pairs, list.rebuild, b.status);
    }
    else
    {
        fill_pairs_kernel<T><<<blocks_for(n), kThreads, 0, stream>>>(
            static_cast<const T*>(b.sorted_positions), b.sorted_ids, b.atom_bin, b.bin_offsets,
            b.dims, cell, b.pair_offsets, r * r, num_atoms, capacity, b.pairs, list.rebuild,
            b.status);
    }
    ND_LAUNCH_CHECK();
    total_and_pad_kernel<<<blocks_for(b.capacity), kThreads, 0, stream>>>(
        b.pair_counts, b.pair_offsets, num_atoms, capacity, b.pair_total, b.pairs, b.status,
        list.rebuild);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

int check_buffers(int dtype, std::int64_t n, const nd_neighbor_buffers* b)
{
    ND_REQUIRE(dtype == ND_FLOAT32 || dtype == ND_FLOAT64, "positions must be float32 or float64");
    ND_REQUIRE(b != nullptr, "the list's buffers are missing");
    ND_REQUIRE(n >= 1 && n <= INT32_MAX, "positions must have shape [N, 3] with 1 <= N < 2**31");
    ND_REQUIRE(b->num_bin_slots >= 2 && b->num_bin_slots <= INT32_MAX,
               "the list's buffers do not match the positions");
    ND_REQUIRE(b->capacity >= 1 && b->capacity <= INT32_MAX, "pairs must be [2, C] with int32 C");
    ND_REQUIRE(b->bits_numel == 0 || b->bits_numel == n * bit_words(n),
               "bits must be empty or hold N rows of ceil(N / 32) words");
    const std::int64_t need = scan_scratch_bytes(b->num_bin_slots > n ? b->num_bin_slots : n);
    ND_REQUIRE(b->scan_temp_bytes >= need, "scan_temp is smaller than scan_temp_bytes asks");
    ND_REQUIRE(b->dims && b->widths && b->atom_bin && b->bin_counts && b->bin_offsets &&
                   b->unordered_ids && b->sorted_ids && b->sorted_positions && b->scan_temp &&
                   b->pair_counts && b->pair_offsets && b->pair_total && b->status && b->pairs &&
                   (b->bits_numel == 0 || b->bits),
               "a buffer of the list is null");
    return ND_OK;
}

template <typename T>
int count_first_frame(const void* positions, const void* cell, std::int64_t n, double radius,
                      const nd_neighbor_buffers* b, cudaStream_t stream)
{
    const List list{b, nullptr};
    const auto* x = static_cast<const T*>(positions);
    if (!list.all_pairs())
    {
        const int rc = launch_grid<T>(x, n, list, stream);
        if (rc != ND_OK)
        {
            return rc;
        }
    }
    return launch_count<T>(x, static_cast<const T*>(cell), n, radius, list, stream);
}

template <typename T>
int update(const void* positions, const void* cell, std::int64_t n, double cutoff, double radius,
           const nd_reuse_buffers* r, const nd_neighbor_buffers* b, cudaStream_t stream)
{
    const List list{b, r->rebuild};
    const auto* x = static_cast<const T*>(positions);
    const auto* box = static_cast<const T*>(cell);
    const auto num_atoms = static_cast<index_t>(n);
    prepare_update_kernel<T><<<1, 1, 0, stream>>>(
        box, static_cast<const T*>(r->reference_cell), static_cast<T>(cutoff),
        static_cast<T>(radius), std::numeric_limits<T>::epsilon(), r->limits, b->dims,
        static_cast<T*>(b->widths), static_cast<T*>(r->reuse), r->rebuild, b->status);
    ND_LAUNCH_CHECK();
    check_reuse_kernel<T><<<blocks_for(n), kThreads, 0, stream>>>(
        x, static_cast<const T*>(r->reference_positions), box, static_cast<const T*>(r->reuse),
        num_atoms, r->rebuild, b->status);
    ND_LAUNCH_CHECK();
    int rc = ND_OK;
    if (!list.all_pairs() && (rc = launch_grid<T>(x, n, list, stream)) != ND_OK)
    {
        return rc;
    }
    if ((rc = launch_count<T>(x, box, n, radius, list, stream)) != ND_OK)
    {
        return rc;
    }
    if ((rc = launch_fill<T>(box, n, radius, list, stream)) != ND_OK)
    {
        return rc;
    }
    commit_rebuild_kernel<T><<<blocks_for(3 * n), kThreads, 0, stream>>>(
        x, box, num_atoms, static_cast<T*>(r->reference_positions),
        static_cast<T*>(r->reference_cell), r->rebuild_count, r->rebuild, b->status);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

}  // namespace nd

// ---------------------------------------------------------------------------------------
// C-ABI.

extern "C" {

int nd_neighbors_scan_temp_bytes(std::int64_t items, std::int64_t* bytes)
{
    ND_REQUIRE(items > 0 && items <= INT32_MAX, "the scan length must fit int32");
    ND_REQUIRE(bytes != nullptr, "bytes is null");
    *bytes = nd::scan_scratch_bytes(items);
    return ND_OK;
}

int nd_neighbors_count_first_frame(int dtype, const void* positions, const void* cell,
                                   std::int64_t num_atoms, double radius,
                                   const nd_neighbor_buffers* buffers, nd_stream_t stream)
{
    const int rc = nd::check_buffers(dtype, num_atoms, buffers);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(positions && cell, "positions and cell must not be null");
    auto s = static_cast<cudaStream_t>(stream);
    return dtype == ND_FLOAT32
               ? nd::count_first_frame<float>(positions, cell, num_atoms, radius, buffers, s)
               : nd::count_first_frame<double>(positions, cell, num_atoms, radius, buffers, s);
}

int nd_neighbors_fill_first_frame(int dtype, const void* positions, const void* cell,
                                  std::int64_t num_atoms, double radius,
                                  const nd_neighbor_buffers* buffers, nd_stream_t stream)
{
    const int rc = nd::check_buffers(dtype, num_atoms, buffers);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(positions && cell, "positions and cell must not be null");
    const nd::List list{buffers, nullptr};
    auto s = static_cast<cudaStream_t>(stream);
    return dtype == ND_FLOAT32
               ? nd::launch_fill<float>(static_cast<const float*>(cell), num_atoms, radius, list, s)
               : nd::launch_fill<double>(static_cast<const double*>(cell), num_atoms, radius,
                                         list, s);
}

int nd_neighbors_update(int dtype, const void* positions, const void* cell,
                        std::int64_t num_atoms, double cutoff, double radius,
                        const nd_reuse_buffers* reuse, const nd_neighbor_buffers* buffers,
                        nd_stream_t stream)
{
    const int rc = nd::check_buffers(dtype, num_atoms, buffers);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(positions && cell, "positions and cell must not be null");
    ND_REQUIRE(reuse && reuse->reference_positions && reuse->reference_cell && reuse->limits &&
                   reuse->reuse && reuse->rebuild && reuse->rebuild_count,
               "the list's update buffers do not match the positions");
    auto s = static_cast<cudaStream_t>(stream);
    return dtype == ND_FLOAT32
               ? nd::update<float>(positions, cell, num_atoms, cutoff, radius, reuse, buffers, s)
               : nd::update<double>(positions, cell, num_atoms, cutoff, radius, reuse, buffers,
                                    s);
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// The pair build without allocation.
//
// Some callers cannot call cudaMalloc at all: code running inside another framework's CUDA
// Graph capture or memory pool, plugins whose host forbids allocation, or embedded drivers
// with a fixed memory map. For them, nd_neighbors_build_no_alloc builds one frame's pair list
// with every intermediate buffer (bins, sorted ids and positions, counts, offsets, scan tiles,
// the all-pairs bit rows) in one file-scope device array of fixed size, kNoAllocBytes, which
// every GPU that loads this library holds until the process exits. The caller passes only
// the positions, the cell and the outputs.

namespace nd {

constexpr std::int64_t kNoAllocMaxAtoms = 16384;
constexpr std::int64_t kNoAllocMaxBins = 16384;
constexpr std::int64_t kNoAllocMaxAllPairsAtoms = 2048;

constexpr std::int64_t round_up_256(std::int64_t bytes)
{
    return (bytes + 255) / 256 * 256;
}

// The layout of the array, in bytes from its start.
struct NoAllocLayout
{
    static constexpr std::int64_t dims = 0;
    static constexpr std::int64_t widths = 256;  // three doubles at most
    static constexpr std::int64_t atom_bin = 512;
    static constexpr std::int64_t bin_counts = atom_bin + round_up_256(4 * kNoAllocMaxAtoms);
    static constexpr std::int64_t bin_offsets = bin_counts + round_up_256(4 * (kNoAllocMaxBins + 1));
    static constexpr std::int64_t unordered_ids =
        bin_offsets + round_up_256(4 * (kNoAllocMaxBins + 1));
    static constexpr std::int64_t sorted_ids = unordered_ids + round_up_256(4 * kNoAllocMaxAtoms);
    static constexpr std::int64_t sorted_positions =
        sorted_ids + round_up_256(4 * kNoAllocMaxAtoms);
    static constexpr std::int64_t pair_counts =
        sorted_positions + round_up_256(3 * 8 * kNoAllocMaxAtoms);
    static constexpr std::int64_t pair_offsets = pair_counts + round_up_256(4 * kNoAllocMaxAtoms);
    static constexpr std::int64_t scan_temp = pair_offsets + round_up_256(4 * kNoAllocMaxAtoms);
    static constexpr std::int64_t bits =
        scan_temp + round_up_256((kNoAllocMaxAtoms + 1 + kTileItems - 1) / kTileItems * 4 + 16);
    static constexpr std::int64_t size =
        bits + round_up_256(4 * kNoAllocMaxAllPairsAtoms * ((kNoAllocMaxAllPairsAtoms + 31) / 32));
};

constexpr std::int64_t kNoAllocBytes = NoAllocLayout::size;

// The scratch itself. In host code this name is only a stand-in for the symbol: its device
// address comes from cudaGetSymbolAddress, per device.
static __device__ __align__(256) unsigned char no_alloc_scratch[kNoAllocBytes];

template <typename T>
__global__ void store_grid_kernel(index_t* dims, T* widths, int nx, int ny, int nz, double wx,
                                  double wy, double wz)
{
    dims[0] = nx;
    dims[1] = ny;
    dims[2] = nz;
    widths[0] = static_cast<T>(wx);
    widths[1] = static_cast<T>(wy);
    widths[2] = static_cast<T>(wz);
}

// The array's device address on the current device, looked up once per device.
int no_alloc_scratch_address(unsigned char** address)
{
    constexpr int kMaxDevices = 64;
    static unsigned char* addresses[kMaxDevices] = {};
    int device = 0;
    ND_CUDA_TRY(cudaGetDevice(&device));
    ND_REQUIRE(device >= 0 && device < kMaxDevices, "the device index is out of range");
    if (addresses[device] == nullptr)
    {
        void* found = nullptr;
        ND_CUDA_TRY(cudaGetSymbolAddress(&found, no_alloc_scratch));
        addresses[device] = static_cast<unsigned char*>(found);
    }
    *address = addresses[device];
    return ND_OK;
}

template <typename T>
int build_no_alloc(const void* positions, const void* cell, std::int64_t n, double radius,
                   const std::int32_t* dims, const double* widths, std::int32_t* pairs,
                   std::int64_t capacity, std::int32_t* pair_total, std::int32_t* status,
                   cudaStream_t stream)
{
    unsigned char* base = nullptr;
    const int found = no_alloc_scratch_address(&base);
    if (found != ND_OK)
    {
        return found;
    }
    const std::int64_t bins = static_cast<std::int64_t>(dims[0]) * dims[1] * dims[2];
    const bool all_pairs = dims[0] <= 3 && dims[1] <= 3 && dims[2] <= 3;
    nd_neighbor_buffers b{};
    b.dims = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::dims);
    b.widths = base + NoAllocLayout::widths;
    b.atom_bin = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::atom_bin);
    b.bin_counts = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::bin_counts);
    b.bin_offsets = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::bin_offsets);
    b.num_bin_slots = bins + 1;
    b.unordered_ids = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::unordered_ids);
    b.sorted_ids = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::sorted_ids);
    b.sorted_positions = base + NoAllocLayout::sorted_positions;
    b.scan_temp = base + NoAllocLayout::scan_temp;
    b.scan_temp_bytes = NoAllocLayout::bits - NoAllocLayout::scan_temp;
    b.pair_counts = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::pair_counts);
    b.pair_offsets = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::pair_offsets);
    b.pair_total = pair_total;
    b.status = status;
    b.pairs = pairs;
    b.capacity = capacity;
    b.bits = all_pairs ? reinterpret_cast<std::int32_t*>(base + NoAllocLayout::bits) : nullptr;
    b.bits_numel = all_pairs ? n * bit_words(n) : 0;
    // What must start at zero: the bin counts (a build returns them to zero, but an earlier
    // call may have stopped short), the outputs' total and status.
    ND_CUDA_TRY(cudaMemsetAsync(b.bin_counts, 0, sizeof(std::int32_t) * (bins + 1), stream));
    ND_CUDA_TRY(cudaMemsetAsync(pair_total, 0, sizeof(std::int32_t), stream));
    ND_CUDA_TRY(cudaMemsetAsync(status, 0, 2 * sizeof(std::int32_t), stream));
    store_grid_kernel<T><<<1, 1, 0, stream>>>(b.dims, static_cast<T*>(b.widths), dims[0], dims[1],
                                              dims[2], widths[0], widths[1], widths[2]);
    ND_LAUNCH_CHECK();
    const int counted = count_first_frame<T>(positions, cell, n, radius, &b, stream);
    if (counted != ND_OK)
    {
        return counted;
    }
    const List list{&b, nullptr};
    return launch_fill<T>(static_cast<const T*>(cell), n, radius, list, stream);
}

}  // namespace nd

extern "C" int nd_neighbors_build_no_alloc(int dtype, const void* positions, const void* cell,
                                           int64_t num_atoms, double radius,
                                           const int32_t* dims, const double* widths,
                                           int32_t* pairs, int64_t capacity,
                                           int32_t* pair_total, int32_t* status,
                                           nd_stream_t stream)
{
    ND_REQUIRE(dtype == ND_FLOAT32 || dtype == ND_FLOAT64, "positions must be float32 or float64");
    ND_REQUIRE(positions && cell && dims && widths && pairs && pair_total && status,
               "a required pointer is null");
    ND_REQUIRE(num_atoms >= 1 && num_atoms <= nd::kNoAllocMaxAtoms,
               "nd_neighbors_build_no_alloc takes at most 16384 atoms");
    ND_REQUIRE(dims[0] >= 1 && dims[1] >= 1 && dims[2] >= 1, "dims must be positive");
    const std::int64_t bins = static_cast<std::int64_t>(dims[0]) * dims[1] * dims[2];
    ND_REQUIRE(bins <= nd::kNoAllocMaxBins, "nd_neighbors_build_no_alloc takes at most 16384 bins");
    const bool all_pairs = dims[0] <= 3 && dims[1] <= 3 && dims[2] <= 3;
    ND_REQUIRE(!all_pairs || num_atoms <= nd::kNoAllocMaxAllPairsAtoms,
               "with at most three bins per axis nd_neighbors_build_no_alloc takes at most 2048 "
               "atoms");
    ND_REQUIRE(capacity >= 1 && capacity <= INT32_MAX, "pairs must be [2, C] with int32 C");
    auto s = static_cast<cudaStream_t>(stream);
    return dtype == ND_FLOAT32
               ? nd::build_no_alloc<float>(positions, cell, num_atoms, radius, dims, widths, pairs,
                                           capacity, pair_total, status, s)
               : nd::build_no_alloc<double>(positions, cell, num_atoms, radius, dims, widths,
                                            pairs, capacity, pair_total, status, s);
}
