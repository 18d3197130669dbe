// The neighbor operator: a cell-list half list of the pairs closer than the list radius,
// with the on-GPU skin-reuse check, behind the C-ABI of include/nabladyn_b200.h.
//
// The contract is the reference's (src/nabladyn/neighbors/csrc/ops.h:12-89,
// runtime/entry_points.cu:284-508): the same 15 buffers, the same status bits, the same pair
// set (each pair once, listed from the atom earlier in bin order), pair columns grouped by that
// atom from its offset in the scan of the counts, padding column k = (k mod N, k mod N), and
// every rebuild kernel gated by a device flag so one CUDA Graph holds a whole update. Two
// rules decide the pair set bit for bit and are kept: the grid (bins of width L / n_a, atoms
// ordered by bin, then by id) and the rounding of a displacement and its square (one rounding
// per difference, r^2 = fma(dz, dz, fma(dx, dx, dy * dy))).
//
// How the GPU builds it is this file's own design:
//   * binning takes each atom's in-bin slot from the counting atomic, and one warp per bin
//     orders the bin by id with shuffles while gathering the sorted positions;
//   * the pairs are built per HOME BIN, one warp each. Every candidate of a home bin's atoms
//     sits in the home bin itself (after the atom) or in a stencil bin that comes later in bin
//     order; the warp stages exactly those bins into shared memory as 16-B (x, y, z, id) slots,
//     each bin's coordinates already moved by its image where the move is exact. The lanes are
//     the home bin's atoms: each staged candidate is read once (a broadcast) and tested against
//     all of them, and a lane sets one bit per hit in a word of 32 candidates, so the count is
//     a popcount per word and only the fill's writes diverge;
//   * small boxes (at most three bins per axis) keep a word-major bit matrix: one thread per
//     (center, 32-candidate word) with the word's candidates staged in shared memory, so
//     threads of a block store consecutive words;
//   * the update opens with one warp that checks the cell and sets the grid and the reuse
//     threshold, checks reuse with one atomic per warp, and commits the new reference frame
//     inside the fill; the scans are our own gated kernels (scan.cuh), so an update that
//     reuses its pairs runs no scan; the pair total and the padding share one launch.

#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <cstdint>
#include <limits>

#include "common.cuh"
#include "geometry.cuh"
#include "scan.cuh"

namespace nd {

// A staged candidate: coordinates in the list's dtype and the atom id in the fourth word.
template <typename T>
struct alignas(4 * sizeof(T)) Slot
{
    T x, y, z, w;
};

__device__ __forceinline__ float id_word(float, index_t id) { return __int_as_float(id); }
__device__ __forceinline__ double id_word(double, index_t id)
{
    return __longlong_as_double(static_cast<long long>(id));
}
__device__ __forceinline__ index_t word_id(float w) { return __float_as_int(w); }
__device__ __forceinline__ index_t word_id(double w)
{
    return static_cast<index_t>(__double_as_longlong(w));
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
// Pairs on the grid path: one warp per home bin.

constexpr int kHoodWarps = 4;                 // bins per CTA, one per warp
constexpr int kHoodThreads = kHoodWarps * kWarp;
constexpr int kHoodBins = 27;                 // the home bin and its stencil, at most

// Shared-memory slots of one warp's neighborhood: 8 KB in either dtype (512 float32 or 256
// float64 candidates; a liquid at 21 atoms/nm^3 with 1.1 nm bins needs about 410). A larger
// neighborhood is read from global memory instead, with the same arithmetic.
template <typename T>
struct HoodSlots
{
    static constexpr int value = 8192 / static_cast<int>(sizeof(Slot<T>));
};

// The part of a home bin's stencil that holds candidates: the home bin (its atoms after the
// center) and each stencil bin that comes later in bin order (all its atoms). With three or
// more bins per axis each bin has a fixed image: `ahead` marks the axes on which the bin lies
// past the upper face, where the center moves by -L (the rounding of center - L, then of the
// difference), `behind` those on which it lies past the lower face, where the candidate moves
// by -L when staged. Otherwise every candidate takes the minimum image per axis.
struct Hood
{
    int count;                    // bins kept, the home bin first
    int total;                    // candidates in them
    int first[kHoodBins];         // sorted index of each bin's first atom
    int size[kHoodBins];          // atoms per bin
    int slot[kHoodBins + 1];      // first slot of each bin in the staged list
    unsigned char ahead[kHoodBins];
    unsigned char behind[kHoodBins];
};

// One warp lists the home bin's stencil. Lane s takes stencil bin s; the kept bins follow the
// home bin in stencil order, placed by a ballot.
__device__ __forceinline__ void plan_hood(
    Hood& hood,
    index_t home,
    const index_t* __restrict__ dims,
    const index_t* __restrict__ bin_offsets,
    bool fixed_images
)
{
    const int lane = threadIdx.x % kWarp;
    const index_t n[3] = {dims[0], dims[1], dims[2]};
    const index_t h[3] = {home % n[0], (home / n[0]) % n[1], home / (n[0] * n[1])};
    // Stencil bins per axis: three around home, or the whole axis when it has fewer bins.
    int span[3];
    for (int a = 0; a < 3; ++a)
    {
        span[a] = n[a] >= 3 ? 3 : n[a];
    }
    bool keep = false;
    index_t bin = 0;
    unsigned ahead = 0, behind = 0;
    if (lane < span[0] * span[1] * span[2])
    {
        const int s[3] = {lane % span[0], (lane / span[0]) % span[1], lane / (span[0] * span[1])};
        index_t b[3];
        for (int a = 0; a < 3; ++a)
        {
            if (n[a] >= 3)
            {
                const index_t raw = h[a] + s[a] - 1;
                b[a] = raw < 0 ? raw + n[a] : (raw >= n[a] ? raw - n[a] : raw);
                if (fixed_images)
                {
                    ahead |= raw >= n[a] ? 1u << a : 0u;
                    behind |= raw < 0 ? 1u << a : 0u;
                }
            }
            else
            {
                b[a] = s[a];
            }
        }
        bin = b[0] + n[0] * (b[1] + n[1] * b[2]);
        keep = bin > home;
    }
    const unsigned kept = __ballot_sync(kFullMask, keep);
    const int count = 1 + __popc(kept);
    if (keep)
    {
        const int at = 1 + __popc(kept & ((1u << lane) - 1u));
        const index_t begin = bin_offsets[bin];
        hood.first[at] = begin;
        hood.size[at] = bin_offsets[bin + 1] - begin;
        hood.ahead[at] = static_cast<unsigned char>(ahead);
        hood.behind[at] = static_cast<unsigned char>(behind);
    }
    if (lane == 0)
    {
        const index_t begin = bin_offsets[home];
        hood.first[0] = begin;
        hood.size[0] = bin_offsets[home + 1] - begin;
        hood.ahead[0] = 0;
        hood.behind[0] = 0;
        hood.count = count;
    }
    __syncwarp();
    // Slots: an exclusive scan of the kept bins' sizes, in their order.
    const int value = lane < count ? hood.size[lane] : 0;
    int inclusive = value;
#pragma unroll
    for (int offset = 1; offset < kWarp; offset *= 2)
    {
        const int up = __shfl_up_sync(kFullMask, inclusive, offset);
        inclusive += lane >= offset ? up : 0;
    }
    if (lane < count)
    {
        hood.slot[lane] = inclusive - value;
    }
    if (lane == count - 1)
    {
        hood.slot[count] = inclusive;
        hood.total = inclusive;
    }
    __syncwarp();
}

// Candidate `k` of kept bin `g`, in the list's arithmetic: the coordinate moved by -L on the
// axes where the bin lies past the lower face (an exact move), and the atom id.
template <typename T>
__device__ __forceinline__ Slot<T> hood_candidate(
    const Hood& hood, int g, int k,
    const T* __restrict__ sorted_positions,
    const index_t* __restrict__ sorted_ids,
    T lx, T ly, T lz
)
{
    const std::int64_t atom = hood.first[g] + k;
    const T* p = sorted_positions + 3 * atom;
    const unsigned behind = hood.behind[g];
    Slot<T> out;
    out.x = (behind & 1u) ? p[0] + (-lx) : p[0];
    out.y = (behind & 2u) ? p[1] + (-ly) : p[1];
    out.z = (behind & 4u) ? p[2] + (-lz) : p[2];
    out.w = id_word(T(0), sorted_ids[atom]);
    return out;
}

// One word of the lane's center against 32 consecutive candidates of kept bin `g` (each read
// once for the whole warp): bit j is set when candidate base + j is closer than the radius.
template <typename T, bool kFixed, bool kStaged>
__device__ __forceinline__ unsigned hit_word(
    const Hood& hood, const Slot<T>* __restrict__ staged,
    const T* __restrict__ sorted_positions, const index_t* __restrict__ sorted_ids,
    int g, int base, int size, const Slot<T>& c, T ax, T ay, T az, T lx, T ly, T lz,
    T radius_squared)
{
    auto test = [&](int j) {
        const int k = base + j;
        const Slot<T> p = kStaged ? staged[hood.slot[g] + k]
                                  : hood_candidate(hood, g, k, sorted_positions, sorted_ids,
                                                   lx, ly, lz);
        T dx, dy, dz;
        if (kFixed)
        {
            dx = ax - p.x;
            dy = ay - p.y;
            dz = az - p.z;
        }
        else
        {
            dx = min_image(c.x, p.x, lx);
            dy = min_image(c.y, p.y, ly);
            dz = min_image(c.z, p.z, lz);
        }
        return squared_norm(dx, dy, dz) < radius_squared;
    };
    unsigned hits = 0;
    if (size == kWarp)
    {
#pragma unroll
        for (int j = 0; j < kWarp; ++j)
        {
            hits |= test(j) ? 1u << j : 0u;
        }
    }
    else
    {
        for (int j = 0; j < size; ++j)
        {
            hits |= test(j) ? 1u << j : 0u;
        }
    }
    return hits;
}

// One warp, one home bin: the lanes are the bin's atoms (32 at a time), every candidate is
// read once per warp and tested against all of them. Each lane keeps a word of hits per 32
// candidates: the count adds its popcount; the fill writes its set bits from the lane's next
// column (only the writes diverge).
template <typename T, bool kFill, bool kFixed, bool kStaged>
__device__ __forceinline__ void hood_lanes(
    const Hood& hood, const Slot<T>* __restrict__ staged,
    const T* __restrict__ sorted_positions, const index_t* __restrict__ sorted_ids,
    T lx, T ly, T lz, T radius_squared,
    index_t* __restrict__ pair_counts, const index_t* __restrict__ pair_offsets,
    std::int64_t capacity, index_t* __restrict__ pairs)
{
    const int lane = threadIdx.x % kWarp;
    const int homes = hood.size[0];
    for (int group = 0; group < homes; group += kWarp)
    {
        const int h = group + lane;
        const bool active = h < homes;
        const Slot<T> c = !active ? Slot<T>{T(0), T(0), T(0), T(0)}
                          : kStaged ? staged[h]
                                    : hood_candidate(hood, 0, h, sorted_positions, sorted_ids,
                                                     lx, ly, lz);
        // The center past the lower face of a later bin's image: center - L, rounded once.
        const T cx_ahead = c.x - lx, cy_ahead = c.y - ly, cz_ahead = c.z - lz;
        const index_t center = hood.first[0] + h;
        index_t count = 0;
        std::int64_t column = kFill && active ? pair_offsets[center] : 0;
        const index_t center_id = kFill && active ? sorted_ids[center] : 0;
        // The home bin's candidates start after the group's first center.
        for (int g = 0; g < hood.count; ++g)
        {
            const unsigned ahead = hood.ahead[g];
            const T ax = (ahead & 1u) ? cx_ahead : c.x;
            const T ay = (ahead & 2u) ? cy_ahead : c.y;
            const T az = (ahead & 4u) ? cz_ahead : c.z;
            const int end = hood.size[g];
            for (int base = g == 0 ? group + 1 : 0; base < end; base += kWarp)
            {
                const int size = end - base < kWarp ? end - base : kWarp;
                unsigned hits = hit_word<T, kFixed, kStaged>(hood, staged, sorted_positions,
                                                             sorted_ids, g, base, size, c, ax,
                                                             ay, az, lx, ly, lz, radius_squared);
                if (g == 0)
                {
                    // Only candidates after the lane's own center: bits above h - base.
                    const int above = h - base + 1;
                    hits &= above <= 0 ? ~0u : (above >= kWarp ? 0u : ~0u << above);
                }
                hits = active ? hits : 0u;
                if (kFill)
                {
                    while (hits != 0)
                    {
                        const int j = __ffs(hits) - 1;
                        hits &= hits - 1;
                        if (column < capacity)
                        {
                            const index_t other =
                                kStaged ? word_id(staged[hood.slot[g] + base + j].w)
                                        : sorted_ids[hood.first[g] + base + j];
                            pairs[column] = center_id;
                            pairs[capacity + column] = other;
                        }
                        ++column;
                    }
                }
                else
                {
                    count += __popc(hits);
                }
            }
        }
        if (!kFill && active)
        {
            pair_counts[center] = count;
        }
    }
}

// Counts (kFill false) or writes (kFill true) the pairs of one home bin per warp. The fill of
// an update also stores the frame it was built from: each warp its home atoms' positions, the
// first warp the cell and the rebuild count.
template <typename T, bool kFill>
__global__ void __launch_bounds__(kHoodThreads) hood_pairs_kernel(
    const T* __restrict__ sorted_positions,
    const index_t* __restrict__ sorted_ids,
    const index_t* __restrict__ bin_offsets,
    const index_t* __restrict__ dims,
    const T* __restrict__ cell,
    T radius_squared,
    std::int64_t num_bins,
    index_t* __restrict__ pair_counts,
    const index_t* __restrict__ pair_offsets,
    index_t capacity,
    index_t* __restrict__ pairs,
    const T* __restrict__ positions,
    T* __restrict__ reference_positions,
    T* __restrict__ reference_cell,
    index_t* __restrict__ rebuild_count,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const std::int64_t home = static_cast<std::int64_t>(blockIdx.x) * kHoodWarps + warp;
    if (home >= num_bins || !rebuilding(rebuild, status))
    {
        return;  // whole warps; no block barrier follows
    }
    __shared__ Hood hoods[kHoodWarps];
    __shared__ Slot<T> tiles[kHoodWarps][HoodSlots<T>::value];
    Hood& hood = hoods[warp];
    Slot<T>* staged = tiles[warp];
    const bool fixed = dims[0] >= 3 && dims[1] >= 3 && dims[2] >= 3;
    const T lx = cell[0], ly = cell[1], lz = cell[2];
    plan_hood(hood, static_cast<index_t>(home), dims, bin_offsets, fixed);
    const int homes = hood.size[0];
    if (kFill && reference_positions != nullptr)
    {
        for (int k = lane; k < 3 * homes; k += kWarp)
        {
            const std::int64_t id = sorted_ids[hood.first[0] + k / 3];
            reference_positions[3 * id + k % 3] = positions[3 * id + k % 3];
        }
        if (home == 0 && lane < 3)
        {
            reference_cell[lane] = cell[lane];
        }
        if (home == 0 && lane == 0)
        {
            ++rebuild_count[0];
        }
    }
    if (homes == 0)
    {
        return;
    }
    const bool stage = hood.total <= HoodSlots<T>::value;
    if (stage)
    {
        for (int g = 0; g < hood.count; ++g)
        {
            for (int k = lane; k < hood.size[g]; k += kWarp)
            {
                staged[hood.slot[g] + k] =
                    hood_candidate(hood, g, k, sorted_positions, sorted_ids, lx, ly, lz);
            }
        }
        __syncwarp();
    }
    const std::int64_t cap = capacity;
    if (fixed)
    {
        stage ? hood_lanes<T, kFill, true, true>(hood, staged, sorted_positions, sorted_ids, lx,
                                                 ly, lz, radius_squared, pair_counts,
                                                 pair_offsets, cap, pairs)
              : hood_lanes<T, kFill, true, false>(hood, staged, sorted_positions, sorted_ids, lx,
                                                  ly, lz, radius_squared, pair_counts,
                                                  pair_offsets, cap, pairs);
    }
    else
    {
        stage ? hood_lanes<T, kFill, false, true>(hood, staged, sorted_positions, sorted_ids, lx,
                                                  ly, lz, radius_squared, pair_counts,
                                                  pair_offsets, cap, pairs)
              : hood_lanes<T, kFill, false, false>(hood, staged, sorted_positions, sorted_ids,
                                                   lx, ly, lz, radius_squared, pair_counts,
                                                   pair_offsets, cap, pairs);
    }
}

// ---------------------------------------------------------------------------------------
// The all-pairs path, for lists whose first grid has at most three bins on every axis.
//
// The hits live in a word-major bit matrix: word w of atom i, bits[w * N + i], holds bit b for
// atom 32 w + b, set when that atom comes after i and lies closer than the radius (minimum
// image per axis). Words that hold no atom after i are never written nor read.

__host__ __device__ __forceinline__ std::int64_t bit_words(std::int64_t num_atoms)
{
    return (num_atoms + kWarp - 1) / kWarp;
}

constexpr int kWordThreads = 128;

// Grid (centers / 128, words): the block stages word w's 32 candidates in shared memory and
// each thread builds one center's word from them.
template <typename T>
__global__ void __launch_bounds__(kWordThreads) pair_words_kernel(
    const T* __restrict__ positions,
    const T* __restrict__ cell,
    T radius_squared,
    index_t num_atoms,
    std::uint32_t* __restrict__ bits,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t word = blockIdx.y;
    const std::int64_t first_center = static_cast<std::int64_t>(blockIdx.x) * kWordThreads;
    if (first_center >= 32 * (word + 1) - 1 || !rebuilding(rebuild, status))
    {
        return;  // every center of the block comes at or after the word's last atom
    }
    __shared__ T candidates[3][kWarp];
    if (threadIdx.x < kWarp)
    {
        const std::int64_t j = 32 * word + threadIdx.x;
        const bool real = j < num_atoms;
        for (int a = 0; a < 3; ++a)
        {
            candidates[a][threadIdx.x] = real ? positions[3 * j + a] : T(0);
        }
    }
    __syncthreads();
    const std::int64_t center = first_center + threadIdx.x;
    if (center >= num_atoms || center >= 32 * (word + 1) - 1)
    {
        return;
    }
    const T cx = positions[3 * center], cy = positions[3 * center + 1],
            cz = positions[3 * center + 2];
    const T lx = cell[0], ly = cell[1], lz = cell[2];
    std::uint32_t hits = 0;
#pragma unroll 8
    for (int b = 0; b < kWarp; ++b)
    {
        const std::int64_t j = 32 * word + b;
        const T dx = min_image(cx, candidates[0][b], lx);
        const T dy = min_image(cy, candidates[1][b], ly);
        const T dz = min_image(cz, candidates[2][b], lz);
        const bool hit = j > center && j < num_atoms && squared_norm(dx, dy, dz) < radius_squared;
        hits |= hit ? 1u << b : 0u;
    }
    bits[word * num_atoms + center] = hits;
}

// One thread per center: its pair count from its words.
__global__ void row_counts_kernel(
    const std::uint32_t* __restrict__ bits,
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
    const std::int64_t words = bit_words(num_atoms);
    index_t count = 0;
    for (std::int64_t w = (center + 1) / kWarp; w < words; ++w)
    {
        count += __popc(bits[w * num_atoms + center]);
    }
    pair_counts[center] = count;
}

// One thread per center: its pairs from its words, in atom order, from its first column. The
// fill of an update also stores the center's position, and thread 0 the cell and the count.
template <typename T>
__global__ void row_fill_kernel(
    const std::uint32_t* __restrict__ bits,
    const index_t* __restrict__ pair_offsets,
    index_t num_atoms,
    index_t capacity,
    index_t* __restrict__ pairs,
    const T* __restrict__ positions,
    const T* __restrict__ cell,
    T* __restrict__ reference_positions,
    T* __restrict__ reference_cell,
    index_t* __restrict__ rebuild_count,
    const index_t* __restrict__ rebuild,
    const index_t* __restrict__ status
)
{
    const std::int64_t center = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (center >= num_atoms || !rebuilding(rebuild, status))
    {
        return;
    }
    if (reference_positions != nullptr)
    {
        for (int a = 0; a < 3; ++a)
        {
            reference_positions[3 * center + a] = positions[3 * center + a];
        }
        if (center == 0)
        {
            for (int a = 0; a < 3; ++a)
            {
                reference_cell[a] = cell[a];
            }
            ++rebuild_count[0];
        }
    }
    const std::int64_t words = bit_words(num_atoms);
    std::int64_t column = pair_offsets[center];
    for (std::int64_t w = (center + 1) / kWarp; w < words; ++w)
    {
        std::uint32_t hits = bits[w * num_atoms + center];
        while (hits != 0)
        {
            const int b = __ffs(hits) - 1;
            hits &= hits - 1;
            if (column < capacity)
            {
                pairs[column] = static_cast<index_t>(center);
                pairs[capacity + column] = static_cast<index_t>(32 * w + b);
            }
            ++column;
        }
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
// The update's gate (the rule of src/nabladyn/neighbors/csrc/update/update.cuh:13-20).
//
// A build stores the wrapped positions x0 and the cell L0. In a cell L, with s = L / L0 per
// axis, atom i has moved d_i = min image of x_i - s x0_i; the pairs are reused while every
// |d_i|^2 < ((R min(s) - cutoff - 32 eps L_max) / 2)^2. Entries of `reuse`: the squared
// threshold, then s per axis.

// One warp: lane a < 3 checks axis a of the cell and sets its grid (at most the first grid's
// bins, each wider than the radius with a margin of a few roundings of L) and its scale; lane 0
// then sets the threshold, or asks for a rebuild when there is no room to move. A list whose
// status holds an error stays as it is until it is allocated again.
template <typename T>
__global__ void open_update_kernel(
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
    const int lane = threadIdx.x;
    const bool sound = status[0] == 0;
    if (lane == 0)
    {
        rebuild[0] = 0;
    }
    const int axis = lane < 3 ? lane : 0;
    const T length = cell[axis];
    const T scale = length / reference_cell[axis];
    const bool valid = isfinite(length) && length > 2 * cutoff;
    const bool all_valid = __all_sync(kFullMask, valid);
    if (!sound)
    {
        return;
    }
    if (!all_valid)
    {
        if (lane == 0)
        {
            status[0] |= kInvalidCell;
        }
        return;
    }
    if (lane < 3)
    {
        reuse[1 + axis] = scale;
        const T fit = floor(length / fma(T(4) * epsilon, length, radius));
        const index_t count =
            fit < 1 ? 1 : (fit > limits[axis] ? limits[axis] : static_cast<index_t>(fit));
        dims[axis] = count;
        widths[axis] = length / count;
    }
    // The smallest scale and the longest length, over the three axes in lane order.
    const T s0 = __shfl_sync(kFullMask, scale, 0), s1 = __shfl_sync(kFullMask, scale, 1),
            s2 = __shfl_sync(kFullMask, scale, 2);
    const T l0 = __shfl_sync(kFullMask, length, 0), l1 = __shfl_sync(kFullMask, length, 1),
            l2 = __shfl_sync(kFullMask, length, 2);
    if (lane == 0)
    {
        T smallest = s0 < s1 ? s0 : s1;
        smallest = s2 < smallest ? s2 : smallest;
        T longest = l1 > l0 ? l1 : l0;
        longest = l2 > longest ? l2 : longest;
        const T allowance = fma(-(T(32) * epsilon), longest, fma(radius, smallest, -cutoff));
        if (allowance <= 0)
        {
            rebuild[0] = 1;
            return;
        }
        reuse[0] = allowance * allowance / 4;
    }
}

// One thread per atom, one atomic per warp: the non-finite bit, then the rebuild request when
// an atom has moved past the threshold.
template <typename T>
__global__ void reuse_check_kernel(
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
    if (status[0] != 0)
    {
        return;  // uniform: the open's verdict, read after its launch
    }
    const int lane = threadIdx.x % kWarp;
    bool bad = false, moved_far = false;
    if (atom < num_atoms)
    {
        const T* x = positions + 3 * atom;
        const T* x0 = reference_positions + 3 * atom;
        bad = !(isfinite(x[0]) && isfinite(x[1]) && isfinite(x[2]));
        T moved = 0;
        for (int axis = 0; axis < 3; ++axis)
        {
            const T d = min_image(x[axis], reuse[1 + axis] * x0[axis], cell[axis]);
            moved = fma(d, d, moved);
        }
        moved_far = !bad && moved >= reuse[0];
    }
    const unsigned bad_lanes = __ballot_sync(kFullMask, bad);
    const unsigned far_lanes = __ballot_sync(kFullMask, moved_far);
    if (lane == 0 && bad_lanes != 0)
    {
        atomicOr(status, kNonFinite);
    }
    if (lane == 0 && far_lanes != 0)
    {
        rebuild[0] = 1;  // every writer stores the same value
    }
}

// ---------------------------------------------------------------------------------------
// Host launchers.

struct List
{
    const nd_neighbor_buffers* b;
    const index_t* rebuild;  // null: a build from allocate, which always runs

    bool all_pairs() const { return b->bits_numel > 0; }
};

// Where an update's fill stores the frame it was built from; all null for allocate.
template <typename T>
struct Commit
{
    const T* positions = nullptr;
    T* reference_positions = nullptr;
    T* reference_cell = nullptr;
    index_t* rebuild_count = nullptr;
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

template <typename T, bool kFill>
void launch_hood(const T* cell, double radius, const List& list, const Commit<T>& commit,
                 cudaStream_t stream)
{
    const nd_neighbor_buffers& b = *list.b;
    const T r = static_cast<T>(radius);
    const std::int64_t bins = b.num_bin_slots - 1;
    hood_pairs_kernel<T, kFill><<<static_cast<unsigned>((bins + kHoodWarps - 1) / kHoodWarps),
                                  kHoodThreads, 0, stream>>>(
        static_cast<const T*>(b.sorted_positions), b.sorted_ids, b.bin_offsets, b.dims, cell,
        r * r, bins, b.pair_counts, b.pair_offsets, static_cast<index_t>(b.capacity), b.pairs,
        commit.positions, commit.reference_positions, commit.reference_cell,
        commit.rebuild_count, list.rebuild, b.status);
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
        auto* bits = reinterpret_cast<std::uint32_t*>(b.bits);
        const dim3 grid(blocks_for(n, kWordThreads), static_cast<unsigned>(bit_words(n)));
        pair_words_kernel<T><<<grid, kWordThreads, 0, stream>>>(positions, cell, r * r,
                                                               num_atoms, bits, list.rebuild,
                                                               b.status);
        ND_LAUNCH_CHECK();
        row_counts_kernel<<<blocks_for(n), kThreads, 0, stream>>>(bits, num_atoms, b.pair_counts,
                                                                  list.rebuild, b.status);
    }
    else
    {
        launch_hood<T, false>(cell, radius, list, Commit<T>{}, stream);
    }
    ND_LAUNCH_CHECK();
    ND_CUDA_TRY(scan_exclusive(b.pair_counts, b.pair_offsets, n, b.scan_temp, list.rebuild,
                               b.status, stream));
    return ND_OK;
}

template <typename T>
int launch_fill(const T* cell, std::int64_t n, double radius, const List& list,
                const Commit<T>& commit, cudaStream_t stream)
{
    const nd_neighbor_buffers& b = *list.b;
    const auto num_atoms = static_cast<index_t>(n);
    const auto capacity = static_cast<index_t>(b.capacity);
    if (list.all_pairs())
    {
        row_fill_kernel<T><<<blocks_for(n), kThreads, 0, stream>>>(
            reinterpret_cast<const std::uint32_t*>(b.bits), b.pair_offsets, num_atoms, capacity,
            b.pairs, commit.positions, cell, commit.reference_positions, commit.reference_cell,
            commit.rebuild_count, list.rebuild, b.status);
    }
    else
    {
        launch_hood<T, true>(cell, radius, list, commit, stream);
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
    ND_REQUIRE(b->bits_numel == 0 || bit_words(n) <= 65535,
               "the all-pairs path takes at most 2,097,120 atoms");
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
    open_update_kernel<T><<<1, kWarp, 0, stream>>>(
        box, static_cast<const T*>(r->reference_cell), static_cast<T>(cutoff),
        static_cast<T>(radius), std::numeric_limits<T>::epsilon(), r->limits, b->dims,
        static_cast<T*>(b->widths), static_cast<T*>(r->reuse), r->rebuild, b->status);
    ND_LAUNCH_CHECK();
    reuse_check_kernel<T><<<blocks_for(n), kThreads, 0, stream>>>(
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
    Commit<T> commit;
    commit.positions = x;
    commit.reference_positions = static_cast<T*>(r->reference_positions);
    commit.reference_cell = static_cast<T*>(r->reference_cell);
    commit.rebuild_count = r->rebuild_count;
    return launch_fill<T>(box, n, radius, list, commit, stream);
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
               ? nd::launch_fill<float>(static_cast<const float*>(cell), num_atoms, radius, list,
                                        nd::Commit<float>{}, s)
               : nd::launch_fill<double>(static_cast<const double*>(cell), num_atoms, radius,
                                         list, nd::Commit<double>{}, s);
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
// the all-pairs bit matrix) in one file-scope device array of fixed size, kNoAllocBytes, which
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
    static constexpr std::int64_t go = 128;      // the build's gate, set by store_grid_kernel
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

// The grid of the frame: the caller's bins per axis, each of width L / n as allocate chooses.
// A bin narrower than the radius would lose pairs: the build is then not run and the status
// reports an invalid cell. `go` gates the build's kernels as an update's rebuild flag does.
template <typename T>
__global__ void store_grid_kernel(index_t* dims, T* widths, const T* cell, T radius, int nx,
                                  int ny, int nz, index_t* go, index_t* status)
{
    const int n[3] = {nx, ny, nz};
    bool narrow = false;
    for (int a = 0; a < 3; ++a)
    {
        dims[a] = n[a];
        widths[a] = cell[a] / n[a];
        narrow = narrow || !(widths[a] >= radius);
    }
    go[0] = 1;
    status[0] = narrow ? kInvalidCell : 0;
    status[1] = 0;
}

// The array's device address on the current device, looked up once per device; concurrent
// first calls from several host threads store the same address.
int no_alloc_scratch_address(unsigned char** address)
{
    constexpr int kMaxDevices = 64;
    static std::atomic<unsigned char*> addresses[kMaxDevices] = {};
    int device = 0;
    ND_CUDA_TRY(cudaGetDevice(&device));
    ND_REQUIRE(device >= 0 && device < kMaxDevices, "the device index is out of range");
    unsigned char* known = addresses[device].load(std::memory_order_acquire);
    if (known == nullptr)
    {
        void* found = nullptr;
        ND_CUDA_TRY(cudaGetSymbolAddress(&found, no_alloc_scratch));
        known = static_cast<unsigned char*>(found);
        addresses[device].store(known, std::memory_order_release);
    }
    *address = known;
    return ND_OK;
}

template <typename T>
int build_no_alloc(const void* positions, const void* cell, std::int64_t n, double radius,
                   const std::int32_t* dims, std::int32_t* pairs, std::int64_t capacity,
                   std::int32_t* pair_total, std::int32_t* status, cudaStream_t stream)
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
    // call may have stopped short) and the total; the grid kernel sets the status and the gate.
    auto* go = reinterpret_cast<std::int32_t*>(base + NoAllocLayout::go);
    ND_CUDA_TRY(cudaMemsetAsync(b.bin_counts, 0, sizeof(std::int32_t) * (bins + 1), stream));
    ND_CUDA_TRY(cudaMemsetAsync(pair_total, 0, sizeof(std::int32_t), stream));
    store_grid_kernel<T><<<1, 1, 0, stream>>>(b.dims, static_cast<T*>(b.widths),
                                              static_cast<const T*>(cell),
                                              static_cast<T>(radius), dims[0], dims[1], dims[2],
                                              go, status);
    ND_LAUNCH_CHECK();
    const List list{&b, go};
    const auto* x = static_cast<const T*>(positions);
    const auto* box = static_cast<const T*>(cell);
    int rc = ND_OK;
    if (!all_pairs && (rc = launch_grid<T>(x, n, list, stream)) != ND_OK)
    {
        return rc;
    }
    if ((rc = launch_count<T>(x, box, n, radius, list, stream)) != ND_OK)
    {
        return rc;
    }
    return launch_fill<T>(box, n, radius, list, Commit<T>{}, stream);
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
    ND_REQUIRE(std::isfinite(radius) && radius > 0, "the radius must be positive and finite");
    ND_REQUIRE(dims[0] >= 1 && dims[1] >= 1 && dims[2] >= 1, "dims must be positive");
    for (int a = 0; a < 3; ++a)
    {
        ND_REQUIRE(std::isfinite(widths[a]) && widths[a] > 0,
                   "widths must be positive and finite");
        ND_REQUIRE(widths[a] >= radius, "a bin must be at least the radius wide");
    }
    const std::int64_t bins = static_cast<std::int64_t>(dims[0]) * dims[1] * dims[2];
    ND_REQUIRE(bins <= nd::kNoAllocMaxBins, "nd_neighbors_build_no_alloc takes at most 16384 bins");
    const bool all_pairs = dims[0] <= 3 && dims[1] <= 3 && dims[2] <= 3;
    ND_REQUIRE(!all_pairs || num_atoms <= nd::kNoAllocMaxAllPairsAtoms,
               "with at most three bins per axis nd_neighbors_build_no_alloc takes at most 2048 "
               "atoms");
    ND_REQUIRE(capacity >= 1 && capacity <= INT32_MAX, "pairs must be [2, C] with int32 C");
    auto s = static_cast<cudaStream_t>(stream);
    return dtype == ND_FLOAT32
               ? nd::build_no_alloc<float>(positions, cell, num_atoms, radius, dims, pairs,
                                           capacity, pair_total, status, s)
               : nd::build_no_alloc<double>(positions, cell, num_atoms, radius, dims, pairs,
                                            capacity, pair_total, status, s);
}
