// The MD engine: velocity-Verlet / Nose-Hoover steps of a Lennard-Jones system, with the
// neighbor rebuild decided on the GPU, in a handful of kernels per step.
//
// It replaces, for one simulation, the reference's step of three compiled programs around the
// neighbor operator (src/nabladyn/md/_simulation.py:316-364): programs[0] (chain half step,
// half kick, drift, wrap), NeighborList._update_wrapped, programs[1] (LJ E/F by torch.func
// and the second half kick, plus K for NVT) and programs[2] (the closing chain half step).
//
// Layout in HBM. The engine keeps every per-atom array in "cell order": the order of the last
// rebuild, atoms sorted by cell, within a cell by their 4 x 4 x 4 sub-cell in Morton order and
// then by atom id, so a cell's atoms are one contiguous range and neighbours in it are close. A rebuild re-sorts and permutes the state (positions, velocities, masses,
// images, ids, types); the forces are recomputed in the new order right after it. `ids` maps a
// slot back to the caller's atom. Positions are
// [N] x (x, y, z, type) vectors, 16 B in float32, so one load fetches an atom. Between rebuilds
// positions are NOT wrapped: an atom keeps the image it was binned in, which keeps every
// precomputed cell image valid; a rebuild wraps them and counts the crossings.
//
// Bricks and tiles. Cells of at least the list radius are grouped along x into bricks of a few
// cells. One CTA per brick stages the brick's 3 x 3 rows of neighbor cells (x extended by one
// cell each way) into shared memory, each cell already shifted by its periodic image and the
// brick's frame (brick_frame: every displacement rounds once), with coalesced 16-B loads. The
// neighbor list is a full list (both directions, no atomics) of uint16 tile-local indices, kept
// per PAIR of centers: consecutive centers of a brick share one list of the tile atoms closer
// than the radius to either of them (166 entries per pair on the 1M-atom argon box, against
// 2 x 125 for two lists), split into two halves, one per lane, and every neighbor read from
// shared memory is evaluated against both centers, the two as the halves of packed f32x2
// instructions. The halves are list rows, interleaved by warps of 32 rows:
//     entry (row, k) lives at ((row / 32) * width + k) * 32 + row % 32.
// The force kernel re-stages the same tile from the current positions and reads every
// neighbor from shared memory, so the only per-pair global traffic is the 2-B index.
//
// Small boxes (fewer than three cells on an axis) use one tile holding the whole system and
// the minimum image per pair, as the reference's all-pairs path does.
//
// Reductions. Pair arithmetic is in the system's dtype; each block reduces its energy,
// kinetic energy and virial in float64 into its own slot, and the last block to finish sums
// the slots in a fixed order (deterministic totals) and runs the scalar tail: the Nose-Hoover
// closing half step in float64 (src/nabladyn/md/_ensembles/_chain.py:36-83).

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <type_traits>

#include "common.cuh"
#include "geometry.cuh"
#include "md_common.cuh"
#include "scan.cuh"

namespace nd {

constexpr int kMDThreads = 256;
constexpr int kWarpsPerBlock = kMDThreads / kWarp;
constexpr int kMaxBrickCells = 14;                  // home cells per brick, at most
constexpr int kMaxRowCells = kMaxBrickCells + 2;    // tile cells per row
constexpr int kTileCells = 9 * kMaxRowCells;        // tile cells, at most
constexpr int kReduced = 8;                         // E, K, W xx yy zz xy xz yz
constexpr int kSmallLanes = 16;  // small-box forces: lanes sharing one atom's list

// The device view of one system, built from nd_md_system.
template <typename T>
struct System
{
    Pos4<T>* pos;
    T* vel;
    T* force;
    T* inv_mass;
    T* mass;
    long long* images;
    index_t* ids;
    Pos4<T>* ref_pos;
    Pos4<T>* pos_b;
    T* vel_b;
    T* inv_mass_b;
    T* mass_b;
    long long* images_b;
    index_t* ids_b;
    index_t* cell_counts;
    index_t* cell_offsets;
    index_t* atom_cell;
    index_t* slot;
    index_t* unordered;
    index_t* order;
    void* scan_temp;
    std::uint16_t* nbr;
    index_t* nbr_count;
    index_t* pair_order;
    index_t* rebuild;
    index_t* rebuild_count;
    index_t* status;
    double* partials;
    double* totals;
    double* thermo;
    const T* sigma;
    const T* epsilon;
    index_t n;
    index_t dims[3];
    T length[3];
    T widths[3];
    index_t bricks_x;
    index_t num_bricks;
    index_t force_blocks;  // the force kernel's grid: bricks, or kSmallLanes lanes per atom
    index_t width;
    index_t tile_cap;
    index_t sentinel;  // the tile slot of the far-away atom that pads partial list chunks
    int small;
    int num_types;
    T dt;
    T half_dt;
    T threshold_squared;
    T radius_squared;
    T cutoff_squared;
};

// ---------------------------------------------------------------------------------------
// Bulk asynchronous copies into shared memory, completed on an mbarrier (sm_90+ PTX).

constexpr index_t kStageTimeout = 16;  // status bit: a tile copy did not complete in time
constexpr int kWaitLimit = 1 << 22;    // mbarrier polls before a copy counts as lost

__device__ __forceinline__ unsigned shared_address(const void* pointer)
{
    return static_cast<unsigned>(__cvta_generic_to_shared(pointer));
}

__device__ __forceinline__ void barrier_init(std::uint64_t* barrier)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(shared_address(barrier)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void barrier_expect_bytes(std::uint64_t* barrier, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
                     shared_address(barrier)),
                 "r"(bytes)
                 : "memory");
}

// Copies `bytes` (a multiple of 16, both addresses 16-B aligned) from global memory of this
// GPU into this CTA's shared memory; completion counts on the barrier. No multicast.
__device__ __forceinline__ void bulk_load(void* destination, const void* source, unsigned bytes,
                                          std::uint64_t* barrier)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(shared_address(destination)),
        "l"(source), "r"(bytes), "r"(shared_address(barrier))
        : "memory");
}

__device__ __forceinline__ bool barrier_try_wait(std::uint64_t* barrier, unsigned phase)
{
    unsigned done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}"
        : "=r"(done)
        : "r"(shared_address(barrier)), "r"(phase)
        : "memory");
    return done != 0;
}

// Waits for phase 0 of the barrier, at most kWaitLimit polls and 0.5 s (a poll may suspend
// the thread for a while); false when it gave up.
__device__ __forceinline__ bool barrier_wait_bounded(std::uint64_t* barrier)
{
    std::uint64_t start;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(start));
    for (int poll = 0; poll < kWaitLimit; ++poll)
    {
        if (barrier_try_wait(barrier, 0))
        {
            return true;
        }
        std::uint64_t now;
        asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
        if (now - start > 500000000ull)
        {
            return false;
        }
    }
    return false;
}

// ---------------------------------------------------------------------------------------
// Tiles.

// The brick's frame: an offset per axis, 0 or -L, added to every coordinate of its tile and
// to its centers, so that each displacement is rounded once, as the reference's image rule
// does (src/nabladyn/neighbors/csrc/common/traversal.cuh:9-28). A tile cell past the upper
// face needs +L: x + L rounds at the ulp of L (1.9e-6 nm at L = 36.8 nm, which alone gives a
// force error of 1.2e-5 of FP64 on the 1M-atom box). So a brick whose tile crosses only the
// upper face along an axis moves its frame by -L there: its own cells then take x - L, exact
// by Sterbenz's lemma for x >= L/2, and the cells past the face keep x unchanged. A brick that
// crosses only the lower face (shift -L, x near L, exact) or no face keeps offset 0; a brick
// crossing both (a row of one brick) keeps 0 and rounds its +L cells.
template <typename T>
struct BrickFrame
{
    T x, y, z;
};

template <typename T>
__device__ __forceinline__ BrickFrame<T> brick_frame(const System<T>& s, const TileShape& shape)
{
    BrickFrame<T> frame;
    frame.x = (shape.x1 == s.dims[0] && shape.x0 > 0) ? -s.length[0] : T(0);
    frame.y = (shape.y == s.dims[1] - 1 && shape.y > 0) ? -s.length[1] : T(0);
    frame.z = (shape.z == s.dims[2] - 1 && shape.z > 0) ? -s.length[2] : T(0);
    return frame;
}

// Stages one brick's tile. The tile cells of a row are consecutive cells of the cell order
// (apart from a wrap along x), so each maximal run of cells whose atoms are adjacent in memory
// is one bulk copy, issued by the first warp; every thread then waits on the barrier, and the
// cells across a periodic boundary get their image shift in shared memory.
//
// `between(shape)` runs on every thread after the copies are issued and before the wait (only
// when the tile fits): work that needs the brick's shape but not its tile, such as the loads a
// CTA's first pass over its centers starts with, overlaps the copies.
template <typename T, typename Between>
__device__ __forceinline__ TileShape stage_brick(
    const System<T>& s,
    int brick,
    const Pos4<T>* __restrict__ positions,
    Pos4<T>* tile,
    int* start,
    int* first,
    Between&& between
)
{
    __shared__ std::uint64_t copied;
    const int nx = s.dims[0], ny = s.dims[1], nz = s.dims[2];
    const int bx = brick % s.bricks_x;
    const int x0 = bx * nx / s.bricks_x;
    const int x1 = (bx + 1) * nx / s.bricks_x;
    const int y = (brick / s.bricks_x) % ny;
    const int z = brick / (s.bricks_x * ny);
    if (threadIdx.x == 0)
    {
        tile[s.sentinel] = far_atom<T>();
        barrier_init(&copied);
    }
    const int per_row = x1 - x0 + 2;
    const int cells = 9 * per_row;
    // Per tile cell: its cell-order range.
    for (int t = threadIdx.x; t < cells; t += blockDim.x)
    {
        const int r = t / per_row, c = t % per_row;
        int cx = x0 - 1 + c, cy = y + r % 3 - 1, cz = z + r / 3 - 1;
        cx = cx < 0 ? cx + nx : (cx >= nx ? cx - nx : cx);
        cy = cy < 0 ? cy + ny : (cy >= ny ? cy - ny : cy);
        cz = cz < 0 ? cz + nz : (cz >= nz ? cz - nz : cz);
        const int cell = cx + nx * (cy + ny * cz);
        const int begin = s.cell_offsets[cell];
        first[t] = begin;
        start[t] = s.cell_offsets[cell + 1] - begin;  // the count, scanned below
    }
    __syncthreads();
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    // Exclusive scan of the counts by the first warp, which also counts the home cells' pairs.
    __shared__ int home_pairs;
    const int home_row = 4 * per_row;
    if (warp == 0)
    {
        int carry = 0;
        int pairs = 0;
        for (int base = 0; base < cells; base += kWarp)
        {
            const int t = base + lane;
            const int count = t < cells ? start[t] : 0;
            pairs += t > home_row && t < home_row + per_row - 1 ? (count + 1) / 2 : 0;
            int inclusive = count;
#pragma unroll
            for (int offset = 1; offset < kWarp; offset *= 2)
            {
                const int up = __shfl_up_sync(kFullMask, inclusive, offset);
                inclusive += lane >= offset ? up : 0;
            }
            if (t < cells)
            {
                start[t] = carry + inclusive - count;
            }
            carry += __shfl_sync(kFullMask, inclusive, kWarp - 1);
        }
        pairs = __reduce_add_sync(kFullMask, pairs);
        if (lane == 0)
        {
            start[cells] = carry;
            home_pairs = pairs;
        }
    }
    __syncthreads();
    TileShape shape;
    shape.cells_per_row = per_row;
    shape.size = start[cells];
    shape.pairs = home_pairs;
    shape.x0 = x0;
    shape.x1 = x1;
    shape.y = y;
    shape.z = z;
    shape.home_first = first[home_row + 1];
    shape.home_end = first[home_row + per_row - 2] + (start[home_row + per_row - 1] -
                                                      start[home_row + per_row - 2]);
    if (shape.size > s.tile_cap)
    {
        return shape;  // the caller flags the overflow; nothing is staged
    }
    if (warp == 0)
    {
        if (lane == 0)
        {
            barrier_expect_bytes(&copied, static_cast<unsigned>(shape.size * sizeof(Pos4<T>)));
        }
        __syncwarp();
        // A run starts at a cell whose atoms do not follow the previous cell's in memory.
        auto follows = [&](int t) { return first[t] == first[t - 1] + (start[t] - start[t - 1]); };
        for (int base = 0; base < cells; base += kWarp)
        {
            const int t = base + lane;
            if (t < cells && (t == 0 || !follows(t)))
            {
                int end = t + 1;
                while (end < cells && follows(end))
                {
                    ++end;
                }
                const unsigned bytes = (start[end] - start[t]) * sizeof(Pos4<T>);
                if (bytes > 0)
                {
                    bulk_load(tile + start[t], positions + first[t], bytes, &copied);
                }
            }
        }
    }
    between(static_cast<const TileShape&>(shape));
    // The first warp polls the barrier while the others wait at the block barrier (no issue
    // slots spent polling); then every warp observes the completed phase once, which makes
    // the copied bytes visible to it. One decision for the whole block, so every thread takes
    // the same path below.
    const bool arrived = warp != 0 || barrier_wait_bounded(&copied);
    if (!__syncthreads_and(arrived) || !barrier_try_wait(&copied, 0))
    {
        // Lost copies: flag it, give them one more bounded wait, and compute nothing. The
        // copies write only this CTA's own tile, so a copy still in flight after both waits
        // (a second, then another 0.5 s) can reach no other CTA's data; but a CTA that exits
        // with one outstanding leaves its shared memory to a late write, which is undefined.
        // That point means the copy engine has stopped: the status bit fails the run at its
        // next host read and no later result is used; an unbounded wait here would instead
        // hang the GPU, so the CTA leaves after the second bound.
        if (threadIdx.x == 0)
        {
            atomicOr(s.status, kStageTimeout);
        }
        barrier_wait_bounded(&copied);
        shape.size = s.tile_cap + 1;
        return shape;
    }
    // Each cell's image shift plus the brick's frame, one warp per cell that moves. A brick
    // whose tile crosses no periodic face has no shift at all (its frame is zero too): it
    // skips the loop, a block-uniform decision.
    const BrickFrame<T> frame = brick_frame(s, shape);
    const bool inside = x0 > 0 && x1 < nx && y > 0 && y < ny - 1 && z > 0 && z < nz - 1;
    if (inside)
    {
        return shape;  // no barrier is needed: nothing was written after the copies landed
    }
    int r = 0, c = warp;  // tile cell t = r * per_row + c, stepped without a division
    while (c >= per_row)
    {
        c -= per_row;
        ++r;
    }
    for (int t = warp; t < cells; t += kWarpsPerBlock)
    {
        const int cx = x0 - 1 + c, cy = y + r % 3 - 1, cz = z + r / 3 - 1;
        const T sx = (cx < 0 ? -s.length[0] : (cx >= nx ? s.length[0] : T(0))) + frame.x;
        const T sy = (cy < 0 ? -s.length[1] : (cy >= ny ? s.length[1] : T(0))) + frame.y;
        const T sz = (cz < 0 ? -s.length[2] : (cz >= nz ? s.length[2] : T(0))) + frame.z;
        if (sx != T(0) || sy != T(0) || sz != T(0))
        {
            for (int k = start[t] + lane; k < start[t + 1]; k += kWarp)
            {
                tile[k].x += sx;
                tile[k].y += sy;
                tile[k].z += sz;
            }
        }
        c += kWarpsPerBlock;
        while (c >= per_row)
        {
            c -= per_row;
            ++r;
        }
    }
    __syncthreads();
    return shape;
}

template <typename T>
__device__ __forceinline__ TileShape stage_brick(const System<T>& s, int brick,
                                                 const Pos4<T>* __restrict__ positions,
                                                 Pos4<T>* tile, int* start, int* first)
{
    return stage_brick(s, brick, positions, tile, start, first, [](const TileShape&) {});
}

__device__ __forceinline__ void flag_overflow(index_t* status, int word, int needed)
{
    atomicOr(status, kOverflow);
    atomicMax(status + word, needed);
}

// Center pairs. On the brick path a cell's atoms, cell-order slots [o, o + n), are taken two
// at a time: pair q holds slots o + 2q and o + 2q + 1 (the second missing when n is odd), so a
// pair never spans two cells. Pair q of cell g is P = o / 2 + g + q, and its list has two
// halves, rows 2P and 2P + 1. Cells come in cell order, so cell g's pairs end at or before
// cell g + 1's first (ceil(n / 2) <= n / 2 + 1 makes up for the rounded halves), and the rows
// of a system are fewer than N + 2 cells + 2.
__device__ __forceinline__ int cell_pair(int offset, int cell, int q)
{
    return offset / 2 + cell + q;
}

// A brick's pairs: the first home cell's first pair and the count over its home cells. The
// brick's entries of the pair order start at `first` and never reach the next brick's.
struct BrickPairs
{
    int first;
    int count;
};

template <typename T>
__device__ __forceinline__ BrickPairs brick_pairs(const System<T>& s, const TileShape& shape,
                                                  const int* start, const int* first)
{
    BrickPairs b;
    b.first = first[4 * shape.cells_per_row + 1] / 2 + shape.x0 +
              s.dims[0] * (shape.y + s.dims[1] * shape.z);
    b.count = shape.pairs;
    return b;
}

// One entry of a brick's pair order: the pair's index P and its first center's cell-order
// slot, shifted left by one, its low bit set when the pair has a second center.
struct PairEntry
{
    int pair;
    int centers;
};

// Shifts into `bits` from the right one bit: set when p lies closer than sqrt(r2max) to
// center a or to center b. The bit is the sign of min(r2) - r2max (negative exactly when
// r2 < r2max), taken by one funnel shift.
template <typename T>
__device__ __forceinline__ unsigned shift_in_hit(const Pos4<T>& a, const Pos4<T>& b,
                                                 const Pos4<T>& p, T r2max, unsigned bits)
{
    const T ra = squared_norm(a.x - p.x, a.y - p.y, a.z - p.z);
    const T rb = squared_norm(b.x - p.x, b.y - p.y, b.z - p.z);
    const T d = (ra < rb ? ra : rb) - r2max;
    return (bits << 1) | static_cast<unsigned>(d < T(0));
}

// The same test with the two centers as the halves of packed f32x2 instructions (sm_100):
// each half rounds as the scalar test, p - x being the exact negative of x - p.
__device__ __forceinline__ unsigned shift_in_hit(const Pos4<float>& a, const Pos4<float>& b,
                                                 const Pos4<float>& p, float r2max,
                                                 unsigned bits)
{
    const float2 dx = __fadd2_rn(make_float2(p.x, p.x), make_float2(-a.x, -b.x));
    const float2 dy = __fadd2_rn(make_float2(p.y, p.y), make_float2(-a.y, -b.y));
    const float2 dz = __fadd2_rn(make_float2(p.z, p.z), make_float2(-a.z, -b.z));
    const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
    const float d = fminf(r2.x, r2.y) - r2max;
    return __funnelshift_l(__float_as_uint(d), bits, 1);
}

// ---------------------------------------------------------------------------------------
// The list build, one CTA per brick (grid) or per 128 centers (small box).

template <typename T>
__global__ void __launch_bounds__(kMDThreads) build_list_kernel(System<T> s, int gated)
{
    if (gated && !rebuilding(s.rebuild, s.status))
    {
        return;
    }
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* tile = reinterpret_cast<Pos4<T>*>(smem_raw);
    __shared__ int start[kTileCells + 1];
    __shared__ int first[kTileCells];
    __shared__ __align__(16) std::uint16_t lane_slots[kMDThreads][kChunk];
    const T r2max = s.radius_squared;
    if (s.small)
    {
        // The whole system, unshifted; the minimum image per candidate.
        for (int k = threadIdx.x; k < s.n; k += blockDim.x)
        {
            tile[k] = s.pos[k];
        }
        __syncthreads();
        (void)first;
        const int center = blockIdx.x * blockDim.x + threadIdx.x;
        if (center >= s.n)
        {
            return;
        }
        const Pos4<T> c = tile[center];
        ListWriter list(s.nbr, s.width, center, s.sentinel);
        for (int k = 0; k < s.n; ++k)
        {
            if (k == center)
            {
                continue;
            }
            const Pos4<T> p = tile[k];
            const T dx = min_image(c.x, p.x, s.length[0]);
            const T dy = min_image(c.y, p.y, s.length[1]);
            const T dz = min_image(c.z, p.z, s.length[2]);
            if (squared_norm(dx, dy, dz) < r2max)
            {
                list.add(k);
            }
        }
        list.finish();
        s.nbr_count[center] = list.count;
        if (list.count > s.width)
        {
            flag_overflow(s.status, 1, list.count);
        }
        return;
    }
    const TileShape shape = stage_brick(s, blockIdx.x, s.pos, tile, start, first);
    if (threadIdx.x == 0)
    {
        atomicMax(s.status + 3, shape.size);  // the largest tile of this build, for sizing
    }
    if (shape.size > s.tile_cap)
    {
        if (threadIdx.x == 0)
        {
            flag_overflow(s.status, 2, shape.size);
        }
        return;
    }
    // Pair lists (see cell_pair). A pair's list holds every tile atom closer than the radius
    // to either center, the two centers themselves excepted, in two halves: candidates at even
    // and at odd offsets of a 32-candidate word. One warp per home cell builds the lists of
    // the cell's pairs, 16 at a time: lanes 0-15 the even halves, lanes 16-31 the odd ones.
    // Every candidate row is the x-run of three tile cells around the home cell, so a
    // candidate is one broadcast read per half-warp (the two half-warps read adjacent slots)
    // and the tests do not diverge; a lane tests its candidate against both of its centers and
    // keeps one bit per hit, then appends the word's hits.
    const int per_row = shape.cells_per_row;
    const int home_row = 4 * per_row;
    const int row_cell = shape.x0 + s.dims[0] * (shape.y + s.dims[1] * shape.z);
    const int warp = threadIdx.x / kWarp, lane = threadIdx.x % kWarp;
    const int part = lane >> 4;
    const Pos4<T> far = far_atom<T>();
    for (int c = 1 + warp; c < per_row - 1; c += kWarpsPerBlock)
    {
        const int cell = row_cell + c - 1;
        const int offset = first[home_row + c];
        const int tile_first = start[home_row + c];
        const int cell_count = start[home_row + c + 1] - tile_first;
        const int cell_pairs = (cell_count + 1) / 2;
        for (int group = 0; group * 16 < cell_pairs; ++group)
        {
            const int q = group * 16 + (lane & 15);
            const bool active = q < cell_pairs;
            const bool second = active && 2 * q + 1 < cell_count;
            const int self_a = active ? tile_first + 2 * q : -1;
            const int self_b = second ? self_a + 1 : -1;
            const Pos4<T> a = active ? tile[self_a] : far;
            const Pos4<T> b = second ? tile[self_b] : far;
            const int row = 2 * cell_pair(offset, cell, q) + part;
            StagedListWriter list(s.nbr, lane_slots[threadIdx.x], s.width, row);
            for (int r = 0; r < 9; ++r)
            {
                const int begin = start[r * per_row + c - 1];
                const int end = start[r * per_row + c + 2];
                for (int word = begin; word < end; word += kWarp)
                {
                    // This half's candidates are word + part + 2 jj; candidate jj's hit ends
                    // up in bit 15 - jj.
                    const int size = end - word < kWarp ? end - word : kWarp;
                    const int tests = (size - part + 1) / 2;
                    const Pos4<T>* candidates = tile + word + part;
                    unsigned bits = 0;
                    if (tests == kWarp / 2)
                    {
#pragma unroll
                        for (int jj = 0; jj < kWarp / 2; ++jj)
                        {
                            bits = shift_in_hit(a, b, candidates[2 * jj], r2max, bits);
                        }
                    }
                    else
                    {
                        for (int jj = 0; jj < tests; ++jj)
                        {
                            bits = shift_in_hit(a, b, candidates[2 * jj], r2max, bits);
                        }
                        bits <<= kWarp / 2 - tests;
                    }
                    // Not the centers themselves.
                    const unsigned off_a = static_cast<unsigned>(self_a - word - part);
                    const unsigned off_b = static_cast<unsigned>(self_b - word - part);
                    bits &= off_a < kWarp && !(off_a & 1u) ? ~(0x8000u >> (off_a >> 1)) : ~0u;
                    bits &= off_b < kWarp && !(off_b & 1u) ? ~(0x8000u >> (off_b >> 1)) : ~0u;
                    bits = active ? bits : 0u;
                    while (bits != 0)
                    {
                        const int top = 31 - __clz(bits);
                        bits &= ~(1u << top);
                        list.add(word + part + 2 * (15 - top));
                    }
                }
            }
            if (active)
            {
                list.finish(s.sentinel);
                s.nbr_count[row] = list.count;
                if (list.count > s.width)
                {
                    flag_overflow(s.status, 1, list.count);
                }
            }
        }
    }
    // The order in which the force kernel takes the brick's pairs: longest list first (ties
    // by enumeration order), so the lanes of a warp walk lists of about one length. The tile's
    // memory is free now; the pairs are enumerated cell by cell.
    __syncthreads();
    const BrickPairs pairs = brick_pairs(s, shape, start, first);
    auto* lengths = reinterpret_cast<int*>(smem_raw);
    int longest = 0;
    for (int k = threadIdx.x; k < pairs.count; k += blockDim.x)
    {
        int c = 1, q = k;
        for (int cell_pairs; c < per_row - 1; ++c)
        {
            cell_pairs = (start[home_row + c + 1] - start[home_row + c] + 1) / 2;
            if (q < cell_pairs)
            {
                break;
            }
            q -= cell_pairs;
        }
        const int row = 2 * cell_pair(first[home_row + c], row_cell + c - 1, q);
        const int even = s.nbr_count[row], odd = s.nbr_count[row + 1];
        lengths[k] = even > odd ? even : odd;
        if (s.width == kChunk)
        {
            // The sizing build (the smallest width): status[1] gets the longest whole pair
            // list, the bound a half can reach once the pair's centers drift apart.
            longest = even + odd > longest ? even + odd : longest;
        }
    }
    if (s.width == kChunk)
    {
        longest = __reduce_max_sync(kFullMask, longest);
        if (lane == 0 && longest > 0)
        {
            atomicMax(s.status + 1, longest);
        }
    }
    __syncthreads();
    auto* order = reinterpret_cast<PairEntry*>(s.pair_order);
    for (int k = threadIdx.x; k < pairs.count; k += blockDim.x)
    {
        const int mine = lengths[k];
        int rank = 0;
        for (int other = 0; other < pairs.count; ++other)
        {
            const int length = lengths[other];
            rank += length > mine || (length == mine && other < k);
        }
        int c = 1, q = k;
        int cell_count = 0;
        for (; c < per_row - 1; ++c)
        {
            cell_count = start[home_row + c + 1] - start[home_row + c];
            if (q < (cell_count + 1) / 2)
            {
                break;
            }
            q -= (cell_count + 1) / 2;
        }
        const int offset = first[home_row + c];
        PairEntry entry;
        entry.pair = cell_pair(offset, row_cell + c - 1, q);
        entry.centers = ((offset + 2 * q) << 1) | (2 * q + 1 < cell_count ? 1 : 0);
        order[pairs.first + rank] = entry;
    }
}

// ---------------------------------------------------------------------------------------
// Forces, the second half kick and the step's reductions.

// The per-atom results of the pair loop, for one center.
template <typename T>
struct CenterSums
{
    T fx, fy, fz;  // single type: in units of 24 eps; several types: kJ/mol/nm
    T energy;      // single type: sum of p6^2 - p6; several types: kJ/mol
    T inside;      // single type: pairs inside the cutoff
    T w[6];        // like the force
};

// One pair term, center `me` against neighbor p, added to the center's sums: no branch on the
// cutoff (a pair outside contributes an exact zero). With one atom type the constants 24 eps,
// 4 eps and u(r_c) are applied once per center, not per pair.
template <typename T, bool kMulti, bool kVirial, bool kEnergy>
__device__ __forceinline__ void add_pair_term(CenterSums<T>& c, const Pos4<T>& me,
                                              const Pos4<T>& p,
                                              const PairParams<T>* __restrict__ params, T s2,
                                              T cutoff_squared, int num_types)
{
    const T dx = me.x - p.x;
    const T dy = me.y - p.y;
    const T dz = me.z - p.z;
    const T r2 = squared_norm(dx, dy, dz);
    const bool inside = r2 < cutoff_squared;
    const T inv_r2 = fast_reciprocal(r2);
    PairParams<T> pp;
    if (kMulti)
    {
        pp = params[type_pair_row(static_cast<int>(me.w), static_cast<int>(p.w), num_types)];
    }
    const T q = (kMulti ? pp.s2 : s2) * inv_r2;
    const T p6 = q * q * q;
    const T mask = inside ? T(1) : T(0);
    T fs = mask * (inv_r2 * (p6 * fma(T(2), p6, T(-1))));
    if (kMulti)
    {
        fs *= pp.e24;
    }
    if (kEnergy)
    {
        const T u = fma(p6, p6, -p6);
        if (kMulti)
        {
            c.energy = fma(mask, fma(pp.e4, u, -pp.shift), c.energy);
        }
        else
        {
            c.energy = fma(mask, u, c.energy);
            c.inside += mask;
        }
    }
    c.fx = fma(fs, dx, c.fx);
    c.fy = fma(fs, dy, c.fy);
    c.fz = fma(fs, dz, c.fz);
    if (kVirial)
    {
        c.w[0] = fma(fs * dx, dx, c.w[0]);
        c.w[1] = fma(fs * dy, dy, c.w[1]);
        c.w[2] = fma(fs * dz, dz, c.w[2]);
        c.w[3] = fma(fs * dx, dy, c.w[3]);
        c.w[4] = fma(fs * dx, dz, c.w[4]);
        c.w[5] = fma(fs * dy, dz, c.w[5]);
    }
}

// Walks one half of a pair's list (8 neighbors per 16-B word, every neighbor read from the
// tile in shared memory, two words in flight since the list streams from HBM; partial chunks
// are padded with the far sentinel), each neighbor against both centers.
template <typename T, bool kMulti, bool kVirial, bool kEnergy>
__device__ __forceinline__ void half_list(const System<T>& s, const Pos4<T>* __restrict__ tile,
                                          const PairParams<T>* __restrict__ params,
                                          const Pos4<T>& a, const Pos4<T>& b, int row, int count,
                                          uint4 next, uint4 after, CenterSums<T>& ca,
                                          CenterSums<T>& cb)
{
    const int used = count < s.width ? count : s.width;
    const int num_chunks = (used + kChunk - 1) / kChunk;
    const uint4* chunks = reinterpret_cast<const uint4*>(s.nbr) + chunk_index(row, 0, s.width);
    const T cutoff_squared = s.cutoff_squared;
    const T s2 = params[0].s2;
    for (int chunk = 0; chunk < num_chunks; ++chunk)
    {
        const uint4 word = next;
        next = after;
        if (chunk + 2 < num_chunks)
        {
            after = chunks[static_cast<std::int64_t>(chunk + 2) * kWarp];
        }
        const unsigned packed[4] = {word.x, word.y, word.z, word.w};
#pragma unroll
        for (int r = 0; r < kChunk; ++r)
        {
            const Pos4<T> p = tile[(packed[r / 2] >> (16 * (r % 2))) & 0xffffu];
            add_pair_term<T, kMulti, kVirial, kEnergy>(ca, a, p, params, s2, cutoff_squared,
                                                       s.num_types);
            add_pair_term<T, kMulti, kVirial, kEnergy>(cb, b, p, params, s2, cutoff_squared,
                                                       s.num_types);
        }
    }
}

// One 16-B tile slot by a single 128-bit shared load, at a shared-window byte address.
__device__ __forceinline__ float4 load_slot(unsigned address)
{
    float4 v;
    asm("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
        : "=f"(v.x), "=f"(v.y), "=f"(v.z), "=f"(v.w)
        : "r"(address));
    return v;
}

// The step's half-list walk for one float32 atom type (forces only: a step needs neither
// energy nor virial). The two centers are the two halves of every packed f32x2 instruction
// (sm_100): a neighbor is read once and its displacement to both centers is three packed adds,
// its r^2 three packed products, the force factor a packed chain and the force sums three
// packed FMAs. The displacement is taken as p - me, the exact negative of me - p, and the
// sums are negated back, so each term is add_pair_term's up to the order of the force sums.
__device__ __forceinline__ void step_half_list(const System<float>& s,
                                               const Pos4<float>* __restrict__ tile,
                                               const PairParams<float>* __restrict__ params,
                                               const Pos4<float>& a, const Pos4<float>& b,
                                               int row, int count, uint4 next, uint4 after,
                                               CenterSums<float>& ca, CenterSums<float>& cb)
{
    const int used = count < s.width ? count : s.width;
    const int num_chunks = (used + kChunk - 1) / kChunk;
    const uint4* chunks = reinterpret_cast<const uint4*>(s.nbr) + chunk_index(row, 0, s.width);
    const float cutoff_squared = s.cutoff_squared;
    const float2 s2 = make_float2(params[0].s2, params[0].s2);
    const float2 two = make_float2(2.0f, 2.0f), minus_one = make_float2(-1.0f, -1.0f);
    const float2 back_x = make_float2(-a.x, -b.x);
    const float2 back_y = make_float2(-a.y, -b.y);
    const float2 back_z = make_float2(-a.z, -b.z);
    const unsigned base = shared_address(tile);
    float2 gx = make_float2(0.0f, 0.0f), gy = gx, gz = gx;  // sums of fs (p - me)
    for (int chunk = 0; chunk < num_chunks; ++chunk)
    {
        const uint4 word = next;
        next = after;
        if (chunk + 2 < num_chunks)
        {
            after = chunks[static_cast<std::int64_t>(chunk + 2) * kWarp];
        }
        const unsigned packed[4] = {word.x, word.y, word.z, word.w};
#pragma unroll
        for (int r = 0; r < kChunk; ++r)
        {
            const unsigned index = (packed[r / 2] >> (16 * (r % 2))) & 0xffffu;
            const float4 p = load_slot(base + (index << 4));
            const float2 dx = __fadd2_rn(make_float2(p.x, p.x), back_x);
            const float2 dy = __fadd2_rn(make_float2(p.y, p.y), back_y);
            const float2 dz = __fadd2_rn(make_float2(p.z, p.z), back_z);
            const float2 r2 = __ffma2_rn(dz, dz, __ffma2_rn(dx, dx, __fmul2_rn(dy, dy)));
            const float2 inv = make_float2(fast_reciprocal(r2.x), fast_reciprocal(r2.y));
            const float2 inside = make_float2(r2.x < cutoff_squared ? 1.0f : 0.0f,
                                              r2.y < cutoff_squared ? 1.0f : 0.0f);
            const float2 q = __fmul2_rn(__fmul2_rn(inv, s2), inside);  // zero outside
            const float2 p6 = __fmul2_rn(__fmul2_rn(q, q), q);
            const float2 fs = __fmul2_rn(inv, __fmul2_rn(p6, __ffma2_rn(two, p6, minus_one)));
            gx = __ffma2_rn(fs, dx, gx);
            gy = __ffma2_rn(fs, dy, gy);
            gz = __ffma2_rn(fs, dz, gz);
        }
    }
    ca.fx -= gx.x;
    ca.fy -= gy.x;
    ca.fz -= gz.x;
    cb.fx -= gx.y;
    cb.fy -= gy.y;
    cb.fz -= gz.y;
}

// The stand-in for the missing second center of a brick's last pair (an odd number of
// centers): far from every tile atom and from the far sentinel alike, so every one of its
// terms is an exact zero.
template <typename T>
__device__ __forceinline__ Pos4<T> absent_center()
{
    return Pos4<T>{T(-1e18), T(-1e18), T(-1e18), T(0)};
}

// What the second half kick of a center needs, loaded before its list is walked so that the
// loads' latency hides behind the pair work.
template <typename T>
struct KickInputs
{
    T vx, vy, vz, inverse_mass, mass;
};

template <typename T, bool kKickStep, bool kThermostat>
__device__ __forceinline__ KickInputs<T> load_kick(const System<T>& s, int center, bool valid)
{
    KickInputs<T> k{};
    if (kKickStep && valid)
    {
        const T* v = s.vel + 3LL * center;
        k.vx = v[0];
        k.vy = v[1];
        k.vz = v[2];
        k.inverse_mass = s.inv_mass[center];
        if (kThermostat)
        {
            k.mass = s.mass[center];
        }
    }
    return k;
}

// Writes a center's force, kicks its velocity (steps) and adds its kinetic energy (NVT).
template <typename T, bool kKickStep, bool kThermostat>
__device__ __forceinline__ void finish_center(const System<T>& s, int center,
                                              const KickInputs<T>& in, T fx, T fy, T fz,
                                              double* sums)
{
    T* f = s.force + 3LL * center;
    f[0] = fx;
    f[1] = fy;
    f[2] = fz;
    if (kKickStep)
    {
        const T kick = s.half_dt * in.inverse_mass;
        T* v = s.vel + 3LL * center;
        const T vx = fma(kick, fx, in.vx);
        const T vy = fma(kick, fy, in.vy);
        const T vz = fma(kick, fz, in.vz);
        v[0] = vx;
        v[1] = vy;
        v[2] = vz;
        if (kThermostat)
        {
            sums[1] += 0.5 * double(in.mass) * (double(vx) * vx + double(vy) * vy + double(vz) * vz);
        }
    }
}

// What a lane needs before walking its half of a pair's list: the pair (from the brick's
// longest-first order), its half's length and its first two list words. None of it needs the
// tile, so a CTA's first pass loads it while the tile's copies are in flight.
struct PairStart
{
    int row;     // this lane's half of the pair's list
    int center;  // the pair's first center (cell-order slot)
    bool live;   // the lane has a pair
    bool has_b;  // the pair has a second center
    int count;
    uint4 first_word, second_word;
};

// Lane `lane_index` of a brick's CTA takes the half (lane_index & 1) of the brick's pair
// lane_index / 2 in its longest-first order.
template <typename T>
__device__ __forceinline__ PairStart pair_start(const System<T>& s, const BrickPairs& pairs,
                                                int lane_index)
{
    PairStart p;
    p.live = lane_index < 2 * pairs.count;
    PairEntry entry{0, 0};
    if (p.live)
    {
        entry = reinterpret_cast<const PairEntry*>(s.pair_order)[pairs.first + (lane_index >> 1)];
    }
    p.row = 2 * entry.pair + (lane_index & 1);
    p.center = entry.centers >> 1;
    p.has_b = p.live && (entry.centers & 1) != 0;
    const uint4* chunks = reinterpret_cast<const uint4*>(s.nbr) + chunk_index(p.row, 0, s.width);
    const uint4 zero = make_uint4(0, 0, 0, 0);
    // A row holds width / 8 >= 1 words; the first two are loaded without waiting for the count.
    p.count = p.live ? s.nbr_count[p.row] : 0;
    p.first_word = p.live ? chunks[0] : zero;
    p.second_word = p.live && s.width > kChunk ? chunks[kWarp] : zero;
    return p;
}

// One center pair of a brick, one half of its list per lane: lanes 2k and 2k + 1 of a warp
// hold the two halves of pair q, add their force sums with one shuffle each, add the term
// between the two centers (kept out of the list) and write one center each. Every lane of the
// warp calls this, `live` false past the brick's last pair, so the shuffles see a full warp.
// Energy and virial: each pair of atoms is met from both ends, half from each; the term
// between the two centers is added, whole, by lane 2k alone.
template <typename T, bool kMulti, bool kVirial, bool kKickStep, bool kThermostat>
__device__ __forceinline__ void force_pair(
    const System<T>& s,
    const Pos4<T>* __restrict__ tile,
    const PairParams<T>* __restrict__ params,
    const BrickFrame<T>& frame,
    const PairStart& start,
    int part,
    double* sums
)
{
    constexpr bool kEnergy = !kKickStep;  // a step needs no energy; a frame's evaluation does
    const bool live = start.live, has_b = start.has_b;
    const int center_a = start.center;
    // The centers in the brick's frame, by the same additions their tile copies took.
    Pos4<T> a = live ? s.pos[center_a] : absent_center<T>();
    Pos4<T> b = has_b ? s.pos[center_a + 1] : absent_center<T>();
    if (live)
    {
        a.x += frame.x;
        a.y += frame.y;
        a.z += frame.z;
    }
    if (has_b)
    {
        b.x += frame.x;
        b.y += frame.y;
        b.z += frame.z;
    }
    // The center this lane finishes: the first for lane 2k, the second for lane 2k + 1.
    const KickInputs<T> kick =
        load_kick<T, kKickStep, kThermostat>(s, center_a + part, part == 0 ? live : has_b);
    CenterSums<T> ca{}, cb{};
    if (live)
    {
        const int row = start.row;
        if constexpr (std::is_same_v<T, float> && !kMulti && !kVirial && !kEnergy)
        {
            step_half_list(s, tile, params, a, b, row, start.count, start.first_word,
                           start.second_word, ca, cb);
        }
        else
        {
            half_list<T, kMulti, kVirial, kEnergy>(s, tile, params, a, b, row, start.count,
                                                   start.first_word, start.second_word, ca,
                                                   cb);
        }
    }
    ca.fx += __shfl_xor_sync(kFullMask, ca.fx, 1);
    ca.fy += __shfl_xor_sync(kFullMask, ca.fy, 1);
    ca.fz += __shfl_xor_sync(kFullMask, ca.fz, 1);
    cb.fx += __shfl_xor_sync(kFullMask, cb.fx, 1);
    cb.fy += __shfl_xor_sync(kFullMask, cb.fy, 1);
    cb.fz += __shfl_xor_sync(kFullMask, cb.fz, 1);
    if (!live)
    {
        return;
    }
    if (has_b)
    {
        // The term between the two centers: the forces in both lanes, energy and virial once.
        CenterSums<T> ab{};
        add_pair_term<T, kMulti, kVirial, kEnergy>(ab, a, b, params, params[0].s2,
                                                   s.cutoff_squared, s.num_types);
        ca.fx += ab.fx;
        ca.fy += ab.fy;
        ca.fz += ab.fz;
        cb.fx -= ab.fx;
        cb.fy -= ab.fy;
        cb.fz -= ab.fz;
        if (part == 0)
        {
            ca.energy += T(2) * ab.energy;
            ca.inside += T(2) * ab.inside;
#pragma unroll
            for (int k = 0; k < 6; ++k)
            {
                ca.w[k] += T(2) * ab.w[k];
            }
        }
    }
    T scale = T(1);  // kJ/mol/nm per unit of the accumulated force
    double energy;
    if (kMulti)
    {
        energy = double(ca.energy) + double(cb.energy);
    }
    else
    {
        scale = params[0].e24;
        energy = double(params[0].e4) * (double(ca.energy) + double(cb.energy)) -
                 double(params[0].shift) * (double(ca.inside) + double(cb.inside));
    }
    if (kEnergy)
    {
        sums[0] += 0.5 * energy;
    }
    if (kVirial)
    {
#pragma unroll
        for (int k = 0; k < 6; ++k)
        {
            sums[2 + k] += 0.5 * (double(ca.w[k] * scale) + double(cb.w[k] * scale));
        }
    }
    if (part == 0)
    {
        finish_center<T, kKickStep, kThermostat>(s, center_a, kick, ca.fx * scale,
                                                 ca.fy * scale, ca.fz * scale, sums);
    }
    else if (has_b)
    {
        finish_center<T, kKickStep, kThermostat>(s, center_a + 1, kick, cb.fx * scale,
                                                 cb.fy * scale, cb.fz * scale, sums);
    }
}

// Each warp reduces its sums in float64 into shared memory and arrives on a block counter; the
// block's last warp adds the warps' sums in a fixed order into the block's slot of `partials`.
// No block barrier: a warp leaves as soon as its own centers are done. `arrivals` starts at
// zero and is made visible by a barrier before any warp arrives.
// Only the sums in kMask (bit k for sums[k]) are reduced; the others are stored as zeros.
template <unsigned kMask = 0xffu>
__device__ __forceinline__ void block_partial(const double* sums, double* partials,
                                              unsigned* arrivals,
                                              double (*warp_sums)[kReduced])
{
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
#pragma unroll
    for (int k = 0; k < kReduced; ++k)
    {
        const double v = (kMask >> k) & 1u ? warp_sum(sums[k]) : 0.0;
        if (lane == 0)
        {
            warp_sums[warp][k] = v;
        }
    }
    __threadfence_block();
    unsigned arrived = 0;
    if (lane == 0)
    {
        arrived = atomicAdd(arrivals, 1u);
    }
    arrived = __shfl_sync(kFullMask, arrived, 0);
    if (arrived != kWarpsPerBlock - 1)
    {
        return;
    }
    __threadfence_block();
    if (lane < kReduced)
    {
        const volatile double* shared = &warp_sums[0][0];
        double total = 0;
        for (int w = 0; w < kWarpsPerBlock; ++w)
        {
            total += shared[w * kReduced + lane];
        }
        partials[static_cast<std::int64_t>(blockIdx.x) * kReduced + lane] = total;
    }
}

constexpr int kFinalizeThreads = 1024;

// One block: the fixed-order sum of the block slots into `totals`, then the scalar tail of a
// step: the rebuild flag cleared for the next check and, for NVT, the closing half step of the
// chain against this step's K, whose factor the next drift (or a frame read) applies.
template <bool kThermostat, bool kStep>
__global__ void __launch_bounds__(kFinalizeThreads) finalize_kernel(const double* partials,
                                                                    int blocks, double* totals,
                                                                    double* thermo,
                                                                    index_t* rebuild)
{
    __shared__ double warp_sums[kFinalizeThreads / kWarp][kReduced];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    double mine[kReduced] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int b = threadIdx.x; b < blocks; b += kFinalizeThreads)
    {
#pragma unroll
        for (int k = 0; k < kReduced; ++k)
        {
            mine[k] += partials[static_cast<std::int64_t>(b) * kReduced + k];
        }
    }
#pragma unroll
    for (int k = 0; k < kReduced; ++k)
    {
        const double v = warp_sum(mine[k]);
        if (lane == 0)
        {
            warp_sums[warp][k] = v;
        }
    }
    __syncthreads();
    if (warp != 0)
    {
        return;
    }
    double total[kReduced];
#pragma unroll
    for (int k = 0; k < kReduced; ++k)
    {
        total[k] = warp_sum(warp_sums[lane][k]);
    }
    if (lane != 0)
    {
        return;
    }
    for (int k = 0; k < kReduced; ++k)
    {
        totals[k] = total[k];
    }
    if (kStep)
    {
        rebuild[0] = 0;  // the next step's check starts clean
    }
    if (kThermostat)
    {
        double kinetic = total[1];
        double q[3], p[3];
        for (int k = 0; k < 3; ++k)
        {
            q[k] = thermo[kChainB + k];
            p[k] = thermo[kChainB + 3 + k];
        }
        const double factor = chain_half_step(kinetic, q, p, thermo + kChainMass,
                                              thermo[kDegrees], thermo[kThermalEnergy],
                                              thermo[kTimestep]);
        for (int k = 0; k < 3; ++k)
        {
            thermo[kChainA + k] = q[k];
            thermo[kChainA + 3 + k] = p[k];
        }
        thermo[kKineticA] = kinetic;
        thermo[kPendingScale] = factor;
    }
}

// The small box's pair loop split over kSmallLanes lanes: lane `part` takes chunks part,
// part + kSmallLanes, ...; the lanes' sums meet in a fixed shuffle tree, so a box of a few
// hundred atoms fills many SMs instead of two.
template <typename T, bool kMulti, bool kVirial, bool kKickStep, bool kThermostat>
__device__ __forceinline__ void force_center_split(const System<T>& s,
                                                   const Pos4<T>* __restrict__ tile,
                                                   const PairParams<T>* __restrict__ params,
                                                   int center, int part, double* sums)
{
    CenterSums<T> c{};
    const bool real = center < s.n;
    const Pos4<T> me = real ? tile[center] : far_atom<T>();
    if (real)
    {
        const int count = s.nbr_count[center];
        const int used = count < s.width ? count : s.width;
        const int num_chunks = (used + kChunk - 1) / kChunk;
        const uint4* chunks =
            reinterpret_cast<const uint4*>(s.nbr) + chunk_index(center, 0, s.width);
        const T cutoff_squared = s.cutoff_squared;
        const T s2 = params[0].s2;
        for (int chunk = part; chunk < num_chunks; chunk += kSmallLanes)
        {
            const uint4 word = chunks[static_cast<std::int64_t>(chunk) * kWarp];
            const unsigned packed[4] = {word.x, word.y, word.z, word.w};
#pragma unroll
            for (int r = 0; r < kChunk; ++r)
            {
                const Pos4<T> p = tile[(packed[r / 2] >> (16 * (r % 2))) & 0xffffu];
                const T dx = min_image(me.x, p.x, s.length[0]);
                const T dy = min_image(me.y, p.y, s.length[1]);
                const T dz = min_image(me.z, p.z, s.length[2]);
                const T r2 = squared_norm(dx, dy, dz);
                const bool inside = r2 < cutoff_squared;
                const T inv_r2 = fast_reciprocal(r2);
                PairParams<T> pp;
                if (kMulti)
                {
                    pp = params[type_pair_row(static_cast<int>(me.w), static_cast<int>(p.w),
                                              s.num_types)];
                }
                const T q = (kMulti ? pp.s2 : s2) * inv_r2;
                const T p6 = q * q * q;
                const T mask = inside ? T(1) : T(0);
                T fs = mask * (inv_r2 * (p6 * fma(T(2), p6, T(-1))));
                const T u = fma(p6, p6, -p6);
                if (kMulti)
                {
                    fs *= pp.e24;
                    c.energy = fma(mask, fma(pp.e4, u, -pp.shift), c.energy);
                }
                else
                {
                    c.energy = fma(mask, u, c.energy);
                    c.inside += mask;
                }
                c.fx = fma(fs, dx, c.fx);
                c.fy = fma(fs, dy, c.fy);
                c.fz = fma(fs, dz, c.fz);
                if (kVirial)
                {
                    c.w[0] = fma(fs * dx, dx, c.w[0]);
                    c.w[1] = fma(fs * dy, dy, c.w[1]);
                    c.w[2] = fma(fs * dz, dz, c.w[2]);
                    c.w[3] = fma(fs * dx, dy, c.w[3]);
                    c.w[4] = fma(fs * dx, dz, c.w[4]);
                    c.w[5] = fma(fs * dy, dz, c.w[5]);
                }
            }
        }
    }
#pragma unroll
    for (int offset = kSmallLanes / 2; offset > 0; offset /= 2)
    {
        c.fx += __shfl_xor_sync(kFullMask, c.fx, offset);
        c.fy += __shfl_xor_sync(kFullMask, c.fy, offset);
        c.fz += __shfl_xor_sync(kFullMask, c.fz, offset);
        c.energy += __shfl_xor_sync(kFullMask, c.energy, offset);
        c.inside += __shfl_xor_sync(kFullMask, c.inside, offset);
        if (kVirial)
        {
#pragma unroll
            for (int k = 0; k < 6; ++k)
            {
                c.w[k] += __shfl_xor_sync(kFullMask, c.w[k], offset);
            }
        }
    }
    if (!real || part != 0)
    {
        return;
    }
    T scale = T(1);
    double energy;
    if (kMulti)
    {
        energy = double(c.energy);
    }
    else
    {
        scale = params[0].e24;
        energy = double(params[0].e4) * double(c.energy) - double(params[0].shift) * double(c.inside);
    }
    const T fx = c.fx * scale, fy = c.fy * scale, fz = c.fz * scale;
    sums[0] += 0.5 * energy;
    if (kVirial)
    {
#pragma unroll
        for (int k = 0; k < 6; ++k)
        {
            sums[2 + k] += 0.5 * double(c.w[k] * scale);
        }
    }
    T* f = s.force + 3LL * center;
    f[0] = fx;
    f[1] = fy;
    f[2] = fz;
    if (kKickStep)
    {
        const T kick = s.half_dt * s.inv_mass[center];
        T* v = s.vel + 3LL * center;
        const T vx = fma(kick, fx, v[0]);
        const T vy = fma(kick, fy, v[1]);
        const T vz = fma(kick, fz, v[2]);
        v[0] = vx;
        v[1] = vy;
        v[2] = vz;
        if (kThermostat)
        {
            sums[1] += 0.5 * double(s.mass[center]) *
                       (double(vx) * vx + double(vy) * vy + double(vz) * vz);
        }
    }
}

// Float32 steps are held to 64 registers, so four CTAs share an SM (as their shared memory
// allows); the other forms keep the registers they need.
// Whether a force launch reduces anything (and so has a finalize): a frame evaluation always,
// a step for the thermostat's K or the virial; an NVE step without the virial does not.
template <bool kVirial, bool kKickStep, bool kThermostat>
constexpr bool kStepReduces = !kKickStep || kThermostat || kVirial;

template <typename T, bool kKickStep>
constexpr int force_blocks_per_sm()
{
    return std::is_same_v<T, float> && kKickStep ? 4 : 1;
}

template <typename T, bool kSmall, bool kMulti, bool kVirial, bool kKickStep, bool kThermostat>
__global__ void __launch_bounds__(kMDThreads, force_blocks_per_sm<T, kKickStep>())
    force_kernel(System<T> s)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* tile = reinterpret_cast<Pos4<T>*>(smem_raw);
    __shared__ int start[kTileCells + 1];
    __shared__ int first[kTileCells];
    __shared__ PairParams<T> params[36];
    __shared__ unsigned arrivals;
    __shared__ double warp_sums[kWarpsPerBlock][kReduced];
    const int rows = s.num_types * (s.num_types + 1) / 2;
    for (int k = threadIdx.x; k < rows; k += blockDim.x)
    {
        params[k] = pair_params(s.sigma[k], s.epsilon[k], s.cutoff_squared);
    }
    if (threadIdx.x == 0)
    {
        arrivals = 0;
    }
    if constexpr (!kStepReduces<kVirial, kKickStep, kThermostat>)
    {
        // A step that reduces nothing launches no finalize, so the reuse flag is cleared here
        // for the next step's check (no kernel reads it after the step's rebuild).
        if (blockIdx.x == 0 && threadIdx.x == 0)
        {
            s.rebuild[0] = 0;
        }
    }
    double sums[kReduced] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (kSmall)
    {
        for (int k = threadIdx.x; k < s.n; k += blockDim.x)
        {
            tile[k] = s.pos[k];
        }
        if (threadIdx.x == 0)
        {
            tile[s.sentinel] = far_atom<T>();
        }
        __syncthreads();
        const int global = blockIdx.x * blockDim.x + threadIdx.x;
        force_center_split<T, kMulti, kVirial, kKickStep, kThermostat>(
            s, tile, params, global / kSmallLanes, global % kSmallLanes, sums);
    }
    else
    {
        PairStart prefetched{};
        BrickPairs pairs{0, 0};
        const TileShape shape =
            stage_brick(s, blockIdx.x, s.pos, tile, start, first, [&](const TileShape& planned) {
                pairs = brick_pairs(s, planned, start, first);
                prefetched = pair_start(s, pairs, threadIdx.x);
            });
        if (shape.size <= s.tile_cap)
        {
            const BrickFrame<T> frame = brick_frame(s, shape);
            const int lanes = 2 * pairs.count;
            for (int base = 0; base < lanes; base += blockDim.x)
            {
                if (base + (threadIdx.x & ~(kWarp - 1)) >= lanes)
                {
                    break;  // the whole warp is past the last pair
                }
                const int t = base + threadIdx.x;
                const PairStart pair = base == 0 ? prefetched : pair_start(s, pairs, t);
                force_pair<T, kMulti, kVirial, kKickStep, kThermostat>(s, tile, params, frame,
                                                                       pair, t & 1, sums);
            }
        }
        else if (threadIdx.x == 0)
        {
            flag_overflow(s.status, 2, shape.size);
        }
    }
    // A step reduces only what its tail reads: K for NVT, the virial when asked; an NVE step
    // without the virial reduces nothing (its finalize only clears the rebuild flag).
    if constexpr (!kKickStep)
    {
        block_partial(sums, s.partials, &arrivals, warp_sums);
    }
    else if constexpr (kThermostat || kVirial)
    {
        block_partial<(kThermostat ? 0x2u : 0u) | (kVirial ? 0xfcu : 0u)>(sums, s.partials,
                                                                          &arrivals, warp_sums);
    }
}

// ---------------------------------------------------------------------------------------
// The first half of a step: the deferred thermostat scales, the half kick, the drift, the
// finiteness check and the reuse check, per atom. With kCondition (a step graph's drift), the
// block that finishes last also sets the graph's rebuild condition from the flag, once every
// block's reuse check is visible to it: each block's first thread fences and takes a ticket
// from rebuild[1]; the last ticket fences again, reads the flag and the status, sets the
// condition and puts the count back to zero for the next step (the fence-and-counter pattern
// of a last-block reduction).

template <typename T, bool kThermostat, bool kCondition>
__global__ void drift_kernel(System<T> s, cudaGraphConditionalHandle handle)
{
    __shared__ T scales[2];
    if (kThermostat)
    {
        // Every block advances the chain's opening half step from the same inputs; block 0
        // stores it. The closing factor of the previous step is applied first, as there.
        if (threadIdx.x == 0)
        {
            const double* th = s.thermo;
            double kinetic = th[kKineticA];
            double q[3], p[3];
            for (int k = 0; k < 3; ++k)
            {
                q[k] = th[kChainA + k];
                p[k] = th[kChainA + 3 + k];
            }
            const double factor = chain_half_step(kinetic, q, p, th + kChainMass, th[kDegrees],
                                                  th[kThermalEnergy], th[kTimestep]);
            scales[0] = static_cast<T>(th[kPendingScale]);
            scales[1] = static_cast<T>(factor);
            if (blockIdx.x == 0)
            {
                double* out = s.thermo;
                for (int k = 0; k < 3; ++k)
                {
                    out[kChainB + k] = q[k];
                    out[kChainB + 3 + k] = p[k];
                }
                out[kKineticB] = kinetic;
                out[kOpenScale] = factor;
            }
        }
        __syncthreads();
    }
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < s.n)
    {
        T* v = s.vel + 3 * i;
        const T* f = s.force + 3 * i;
        const T kick = s.half_dt * s.inv_mass[i];
        T vx = v[0], vy = v[1], vz = v[2];
        if (kThermostat)
        {
            vx = (vx * scales[0]) * scales[1];
            vy = (vy * scales[0]) * scales[1];
            vz = (vz * scales[0]) * scales[1];
        }
        vx = fma(kick, f[0], vx);
        vy = fma(kick, f[1], vy);
        vz = fma(kick, f[2], vz);
        Pos4<T> p = s.pos[i];
        p.x = fma(s.dt, vx, p.x);
        p.y = fma(s.dt, vy, p.y);
        p.z = fma(s.dt, vz, p.z);
        v[0] = vx;
        v[1] = vy;
        v[2] = vz;
        s.pos[i] = p;
        if (!(isfinite(p.x) && isfinite(p.y) && isfinite(p.z)))
        {
            atomicOr(s.status, kNonFinite);
        }
        else
        {
            const Pos4<T> r = s.ref_pos[i];
            if (squared_norm(p.x - r.x, p.y - r.y, p.z - r.z) >= s.threshold_squared)
            {
                s.rebuild[0] = 1;  // every writer stores the same value
            }
        }
    }
    if constexpr (kCondition)
    {
        __syncthreads();
        if (threadIdx.x == 0)
        {
            __threadfence();
            auto* count = reinterpret_cast<unsigned*>(s.rebuild + 1);
            if (atomicAdd(count, 1u) == gridDim.x - 1)
            {
                __threadfence();
                const volatile index_t* flag = s.rebuild;
                const volatile index_t* status = s.status;
                cudaGraphSetConditional(handle, flag[0] != 0 && status[0] == 0 ? 1u : 0u);
                *count = 0;
            }
        }
    }
}

// ---------------------------------------------------------------------------------------
// The rebuild: wrap, bin, sort by cell and id, permute the state, build the list.

template <typename T>
__global__ void wrap_and_bin_kernel(System<T> s, int gated)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= s.n || (gated && !rebuilding(s.rebuild, s.status)))
    {
        return;
    }
    Pos4<T> p = s.pos[i];
    long long cx, cy, cz;
    p.x = wrap_axis(p.x, s.length[0], cx);
    p.y = wrap_axis(p.y, s.length[1], cy);
    p.z = wrap_axis(p.z, s.length[2], cz);
    if (cx | cy | cz)
    {
        long long* image = s.images + 3 * i;
        image[0] += cx;
        image[1] += cy;
        image[2] += cz;
    }
    s.pos[i] = p;
    if (s.small)
    {
        s.ref_pos[i] = p;
        return;
    }
    const index_t nx = s.dims[0], ny = s.dims[1], nz = s.dims[2];
    const index_t cell = axis_bin(p.x, s.widths[0], nx) +
                         nx * (axis_bin(p.y, s.widths[1], ny) + ny * axis_bin(p.z, s.widths[2], nz));
    s.atom_cell[i] = cell;
    s.slot[i] = atomicAdd(s.cell_counts + cell, 1);
}

template <typename T>
__global__ void place_kernel(System<T> s, int gated)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= s.n || (gated && !rebuilding(s.rebuild, s.status)))
    {
        return;
    }
    const index_t cell = s.atom_cell[i];
    s.unordered[s.cell_offsets[cell] + s.slot[i]] = static_cast<index_t>(i);
    s.cell_counts[cell] = 0;
}

// One warp per cell: rank each atom by its key among the cell's atoms; order[new] = old slot.
template <typename T>
__global__ void order_kernel(System<T> s, std::int64_t num_cells, int gated)
{
    const std::int64_t cell =
        (static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) / kWarp;
    const int lane = threadIdx.x % kWarp;
    if (cell >= num_cells || (gated && !rebuilding(s.rebuild, s.status)))
    {
        return;
    }
    const index_t begin = s.cell_offsets[cell];
    const index_t count = s.cell_offsets[cell + 1] - begin;
    // The key: the atom's 4 x 4 x 4 sub-cell in Morton order, then its id, so consecutive
    // atoms of a cell are close and the engine's center pairs are tight.
    const index_t nx = s.dims[0], ny = s.dims[1];
    const T origin[3] = {T(cell % nx) * s.widths[0], T((cell / nx) % ny) * s.widths[1],
                         T(cell / (static_cast<std::int64_t>(nx) * ny)) * s.widths[2]};
    auto key_of = [&](index_t slot) -> unsigned long long {
        const Pos4<T> p = s.pos[slot];
        const T c[3] = {p.x, p.y, p.z};
        unsigned code = 0;
        for (int a = 0; a < 3; ++a)
        {
            int q = static_cast<int>((c[a] - origin[a]) * (T(4) / s.widths[a]));
            q = q < 0 ? 0 : (q > 3 ? 3 : q);
            code |= (q & 1u) << a;
            code |= ((q >> 1) & 1u) << (3 + a);
        }
        return (static_cast<unsigned long long>(code) << 32) |
               static_cast<unsigned>(s.ids[slot]);
    };
    for (index_t mine = 0; mine < count; mine += kWarp)
    {
        const bool active = mine + lane < count;
        const index_t old = active ? s.unordered[begin + mine + lane] : 0;
        const unsigned long long key = active ? key_of(old) : 0;
        index_t rank = 0;
        for (index_t base = 0; base < count; base += kWarp)
        {
            const unsigned long long other =
                base + lane < count ? key_of(s.unordered[begin + base + lane]) : ~0ull;
            const int valid = count - base < kWarp ? count - base : kWarp;
            for (int t = 0; t < valid; ++t)
            {
                rank += __shfl_sync(kFullMask, other, t) < key;
            }
        }
        if (active)
        {
            s.order[begin + rank] = old;
        }
    }
}

template <typename T>
__global__ void permute_kernel(System<T> s, int gated)
{
    const std::int64_t k = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= s.n || (gated && !rebuilding(s.rebuild, s.status)))
    {
        return;
    }
    const index_t old = s.order[k];
    s.pos_b[k] = s.pos[old];
    for (int a = 0; a < 3; ++a)
    {
        s.vel_b[3 * k + a] = s.vel[3LL * old + a];
        s.images_b[3 * k + a] = s.images[3LL * old + a];
    }
    s.inv_mass_b[k] = s.inv_mass[old];
    s.mass_b[k] = s.mass[old];
    s.ids_b[k] = s.ids[old];
}

template <typename T>
__global__ void commit_kernel(System<T> s, int gated)
{
    const std::int64_t k = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= s.n || (gated && !rebuilding(s.rebuild, s.status)))
    {
        return;
    }
    if (k == 0)
    {
        ++s.rebuild_count[0];
    }
    if (s.small)
    {
        return;  // the wrap stored the reference already; the order is unchanged
    }
    const Pos4<T> p = s.pos_b[k];
    s.pos[k] = p;
    s.ref_pos[k] = p;
    for (int a = 0; a < 3; ++a)
    {
        s.vel[3 * k + a] = s.vel_b[3 * k + a];
        s.images[3 * k + a] = s.images_b[3 * k + a];
    }
    s.inv_mass[k] = s.inv_mass_b[k];
    s.mass[k] = s.mass_b[k];
    s.ids[k] = s.ids_b[k];
}

// ---------------------------------------------------------------------------------------
// Import and export in the caller's atom order.

template <typename T>
__global__ void import_kernel(System<T> s, const T* __restrict__ positions,
                              const T* __restrict__ velocities, const T* __restrict__ masses,
                              const long long* __restrict__ images,
                              const index_t* __restrict__ types)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= s.n)
    {
        return;
    }
    Pos4<T> p;
    p.x = positions[3 * i];
    p.y = positions[3 * i + 1];
    p.z = positions[3 * i + 2];
    p.w = types != nullptr ? static_cast<T>(types[i]) : T(0);
    s.pos[i] = p;
    for (int a = 0; a < 3; ++a)
    {
        s.vel[3 * i + a] = velocities[3 * i + a];
        s.force[3 * i + a] = T(0);
        s.images[3 * i + a] = images[3 * i + a];
    }
    s.mass[i] = masses[i];
    s.inv_mass[i] = T(1) / masses[i];
    s.ids[i] = static_cast<index_t>(i);
}

// Writes the frame in the caller's order: positions wrapped into [0, L) with the crossings
// added to the images, velocities with the pending thermostat scale applied, forces.
template <typename T>
__global__ void export_kernel(System<T> s, T* __restrict__ positions, T* __restrict__ velocities,
                              T* __restrict__ forces, long long* __restrict__ images,
                              int thermostat)
{
    const std::int64_t k = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= s.n)
    {
        return;
    }
    const index_t i = s.ids[k];
    const Pos4<T> p = s.pos[k];
    long long c[3];
    const T w[3] = {wrap_axis(p.x, s.length[0], c[0]), wrap_axis(p.y, s.length[1], c[1]),
                    wrap_axis(p.z, s.length[2], c[2])};
    const T scale = thermostat ? static_cast<T>(s.thermo[kPendingScale]) : T(1);
    for (int a = 0; a < 3; ++a)
    {
        if (positions)
        {
            positions[3LL * i + a] = w[a];
        }
        if (images)
        {
            images[3LL * i + a] = s.images[3 * k + a] + c[a];
        }
        if (velocities)
        {
            velocities[3LL * i + a] = thermostat ? s.vel[3 * k + a] * scale : s.vel[3 * k + a];
        }
        if (forces)
        {
            forces[3LL * i + a] = s.force[3 * k + a];
        }
    }
}

// K = sum m v^2 / 2 of the stored velocities times the pending scale, in float64, into
// totals[1]; deterministic: per-block slots, fixed-order final sum by the last block.
template <typename T>
__global__ void __launch_bounds__(kMDThreads) kinetic_kernel(System<T> s, int thermostat)
{
    __shared__ unsigned arrivals;
    __shared__ double warp_sums[kWarpsPerBlock][kReduced];
    if (threadIdx.x == 0)
    {
        arrivals = 0;
    }
    __syncthreads();
    double sums[kReduced] = {0, 0, 0, 0, 0, 0, 0, 0};
    const std::int64_t k = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k < s.n)
    {
        const double scale = thermostat ? double(static_cast<T>(s.thermo[kPendingScale])) : 1.0;
        double v2 = 0;
        for (int a = 0; a < 3; ++a)
        {
            const double v = thermostat ? double(s.vel[3 * k + a] * static_cast<T>(scale))
                                        : double(s.vel[3 * k + a]);
            v2 += v * v;
        }
        sums[1] = 0.5 * double(s.mass[k]) * v2;
    }
    block_partial(sums, s.partials, &arrivals, warp_sums);
}

// ---------------------------------------------------------------------------------------
// Host side.

template <typename T>
System<T> view(const nd_md_system* m)
{
    System<T> s;
    s.pos = static_cast<Pos4<T>*>(m->positions);
    s.vel = static_cast<T*>(m->velocities);
    s.force = static_cast<T*>(m->forces);
    s.inv_mass = static_cast<T*>(m->inverse_masses);
    s.mass = static_cast<T*>(m->masses);
    s.images = reinterpret_cast<long long*>(m->images);
    s.ids = m->ids;
    s.ref_pos = static_cast<Pos4<T>*>(m->reference_positions);
    s.pos_b = static_cast<Pos4<T>*>(m->shadow_positions);
    s.vel_b = static_cast<T*>(m->shadow_velocities);
    s.inv_mass_b = static_cast<T*>(m->shadow_inverse_masses);
    s.mass_b = static_cast<T*>(m->shadow_masses);
    s.images_b = reinterpret_cast<long long*>(m->shadow_images);
    s.ids_b = m->shadow_ids;
    s.cell_counts = m->cell_counts;
    s.cell_offsets = m->cell_offsets;
    s.atom_cell = m->atom_cell;
    s.slot = m->slots;
    s.unordered = m->unordered;
    s.order = m->order;
    s.scan_temp = m->scan_temp;
    s.nbr = m->neighbors;
    s.nbr_count = m->neighbor_counts;
    s.pair_order = m->pair_order;
    s.rebuild = m->rebuild;
    s.rebuild_count = m->rebuild_count;
    s.status = m->status;
    s.partials = m->partials;
    s.totals = m->totals;
    s.thermo = m->thermostat;
    s.sigma = static_cast<const T*>(m->sigma);
    s.epsilon = static_cast<const T*>(m->epsilon);
    s.n = static_cast<index_t>(m->num_atoms);
    for (int a = 0; a < 3; ++a)
    {
        s.dims[a] = m->dims[a];
        s.length[a] = static_cast<T>(m->cell[a]);
        s.widths[a] = static_cast<T>(m->widths[a]);
    }
    s.bricks_x = m->bricks_x;
    s.small = m->small;
    s.num_bricks = s.small ? static_cast<index_t>((m->num_atoms + kMDThreads - 1) / kMDThreads)
                           : m->bricks_x * m->dims[1] * m->dims[2];
    s.force_blocks =
        s.small ? static_cast<index_t>((m->num_atoms * kSmallLanes + kMDThreads - 1) / kMDThreads)
                : s.num_bricks;
    s.width = m->width;
    s.tile_cap = m->tile_capacity;
    s.sentinel = m->small ? static_cast<index_t>(m->num_atoms) : m->tile_capacity;
    s.num_types = m->num_types;
    s.dt = static_cast<T>(m->timestep);
    s.half_dt = static_cast<T>(0.5 * m->timestep);
    s.threshold_squared = static_cast<T>(m->threshold_squared);
    s.radius_squared = static_cast<T>(m->radius) * static_cast<T>(m->radius);
    s.cutoff_squared = static_cast<T>(m->cutoff) * static_cast<T>(m->cutoff);
    return s;
}

template <typename T>
std::size_t tile_bytes(const System<T>& s)
{
    return static_cast<std::size_t>(s.sentinel + 1) * sizeof(Pos4<T>);
}

template <typename T>
int launch_build(const System<T>& s, int gated, cudaStream_t stream)
{
    const std::size_t bytes = tile_bytes(s);
    static DeviceGrant grant;  // per device; the first launch happens outside graph capture
    ND_CUDA_TRY(grant.allow(build_list_kernel<T>, bytes));
    build_list_kernel<T><<<s.num_bricks, kMDThreads, bytes, stream>>>(s, gated);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

template <typename T>
int launch_rebuild(const System<T>& s, std::int64_t num_cells, int gated, cudaStream_t stream)
{
    const unsigned atoms = blocks_for(s.n);
    wrap_and_bin_kernel<T><<<atoms, kThreads, 0, stream>>>(s, gated);
    ND_LAUNCH_CHECK();
    const index_t* gate = gated ? s.rebuild : nullptr;
    if (!s.small)
    {
        ND_CUDA_TRY(scan_exclusive(s.cell_counts, s.cell_offsets, num_cells + 1, s.scan_temp,
                                   gate, s.status, stream));
        place_kernel<T><<<atoms, kThreads, 0, stream>>>(s, gated);
        ND_LAUNCH_CHECK();
        order_kernel<T><<<blocks_for(num_cells * kWarp), kThreads, 0, stream>>>(s, num_cells,
                                                                               gated);
        ND_LAUNCH_CHECK();
        permute_kernel<T><<<atoms, kThreads, 0, stream>>>(s, gated);
        ND_LAUNCH_CHECK();
    }
    commit_kernel<T><<<atoms, kThreads, 0, stream>>>(s, gated);
    ND_LAUNCH_CHECK();
    return launch_build(s, gated, stream);
}

template <typename T, bool kVirial, bool kKickStep, bool kThermostat>
int launch_force_variant(const System<T>& s, cudaStream_t stream)
{
    const std::size_t bytes = tile_bytes(s);
    const bool multi = s.num_types > 1;
#define ND_FORCE_CASE(SMALL, MULTI)                                                         \
    if (s.small == SMALL && multi == MULTI)                                                 \
    {                                                                                       \
        auto kernel = force_kernel<T, SMALL, MULTI, kVirial, kKickStep, kThermostat>;       \
        static DeviceGrant grant;                                                           \
        ND_CUDA_TRY(grant.allow(kernel, bytes));                                            \
        kernel<<<s.force_blocks, kMDThreads, bytes, stream>>>(s);                           \
        ND_LAUNCH_CHECK();                                                                  \
        if constexpr (kStepReduces<kVirial, kKickStep, kThermostat>)                       \
        {                                                                                   \
            finalize_kernel<kThermostat, kKickStep><<<1, kFinalizeThreads, 0, stream>>>(     \
                s.partials, s.force_blocks, s.totals, s.thermo, s.rebuild);                 \
            ND_LAUNCH_CHECK();                                                              \
        }                                                                                   \
        return ND_OK;                                                                       \
    }
    ND_FORCE_CASE(1, true)
    ND_FORCE_CASE(1, false)
    ND_FORCE_CASE(0, true)
    ND_FORCE_CASE(0, false)
#undef ND_FORCE_CASE
    return ND_OK;
}

template <typename T>
int launch_forces(const System<T>& s, int virial, cudaStream_t stream)
{
    return virial ? launch_force_variant<T, true, false, false>(s, stream)
                  : launch_force_variant<T, false, false, false>(s, stream);
}

// The three phases of a step: 0 the drift with the reuse check, 1 the gated rebuild, 2 the
// forces with the second half kick and the tail. -1 runs all three.
template <typename T>
int launch_step(const System<T>& s, std::int64_t num_cells, int thermostat, int virial,
                int phase, cudaStream_t stream)
{
    if (phase < 0 || phase == 0)
    {
        const unsigned atoms = blocks_for(s.n);
        if (thermostat)
        {
            drift_kernel<T, true, false><<<atoms, kThreads, 0, stream>>>(s, 0);
        }
        else
        {
            drift_kernel<T, false, false><<<atoms, kThreads, 0, stream>>>(s, 0);
        }
        ND_LAUNCH_CHECK();
    }
    if (phase < 0 || phase == 1)
    {
        const int rc = launch_rebuild(s, num_cells, 1, stream);
        if (rc != ND_OK)
        {
            return rc;
        }
    }
    if (phase < 0 || phase == 2)
    {
        if (thermostat)
        {
            return virial ? launch_force_variant<T, true, true, true>(s, stream)
                          : launch_force_variant<T, false, true, true>(s, stream);
        }
        return virial ? launch_force_variant<T, true, true, false>(s, stream)
                      : launch_force_variant<T, false, true, false>(s, stream);
    }
    return ND_OK;
}

// The kernels one NVE step without the virial launches, as launch_step issues them.
std::int64_t step_launches(const nd_md_system* m)
{
    const std::int64_t cells = static_cast<std::int64_t>(m->dims[0]) * m->dims[1] * m->dims[2];
    std::int64_t rebuild = 3;  // wrap_and_bin, commit, build_list
    if (!m->small)
    {
        rebuild += (scan_tiles(cells + 1) <= 1 ? 1 : 3) + 3;  // scan, place, order, permute
    }
    return 1 + rebuild + 1;  // drift, rebuild, forces (an NVT step adds the finalize)
}

// ---------------------------------------------------------------------------------------
// Small boxes in one thread-block cluster: many whole steps per launch.
//
// A small box's step is a few microseconds of work spread over six launches (drift, the three
// gated rebuild launches, forces, finalize), so the launches bound it. Here one cluster of up
// to kRunCluster CTAs runs `steps` steps back to back, each CTA owning a contiguous range of
// atoms, the phases separated by cluster barriers (release/acquire at cluster scope), with the
// same arithmetic as those kernels: the chain's opening half step and the drift with the reuse
// check; on a rebuild the wrap and each CTA's centers' lists over all atoms; the forces with
// the second half kick (each atom's list over kSmallLanes lanes); the CTAs' float64 E and K
// summed in CTA order, then the chain's closing half step.
//
// A step is bound by latency, not by work (a few thousand pair terms per SM), so nothing of it
// goes through global memory: every CTA holds the whole system's positions in its shared
// memory and the owner of an atom writes its new position into every CTA's copy (distributed
// shared memory); the reuse and failure flags and the E and K partials travel the same way,
// each CTA writing its own slot in every CTA. The CTA's centers' lists live in its shared
// memory when they fit, else in the global list. The state (positions, velocities, forces,
// references, lists, chain, totals) is loaded at the start and stored at the end; only the
// rare events (a wrap's image crossings, a failure's status bits) write global memory on the
// way. Every CTA keeps the chain's state and closes it from the same sums, so a step needs
// two cluster barriers (three with a rebuild). Every branch around a cluster barrier is decided
// from values all CTAs read after the same barrier, so every CTA takes the same barriers. A
// failure (a status bit) stops the rebuilds, as in the per-step path; the host reads it.

constexpr int kRunThreads = 512;
constexpr int kRunMaxAtoms = 4096;
constexpr int kRunCluster = 16;  // CTAs of the largest cluster (past 8: non-portable)
static_assert(kRunCluster <= kWarp, "a warp reads every CTA's flag slot in one vote");

__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// The address of `local` (this CTA's shared memory) in CTA `rank` of the cluster.
template <typename V>
__device__ __forceinline__ V* cluster_peer(V* local, unsigned rank)
{
    unsigned long long remote;
    asm volatile("mapa.u64 %0, %1, %2;" : "=l"(remote) : "l"(local), "r"(rank));
    return reinterpret_cast<V*>(remote);
}

// One center's list on the small-box path by a whole warp, 32 candidates a round: the hits of a
// round are ranked by ballot, so the list holds them in ascending index order, as the per-step
// build's scan of all atoms stores them; a partial last chunk is padded with the sentinel.
// `entry(e)` is the list's e-th slot. Returns the count (entries past the width not stored).
template <typename T, typename Entry>
__device__ __forceinline__ int warp_center_list(const System<T>& s,
                                                const Pos4<T>* __restrict__ tile, int center,
                                                Entry&& entry)
{
    const int lane = threadIdx.x % kWarp;
    const Pos4<T> c = tile[center];
    const T r2max = s.radius_squared;
    int count = 0;
    for (int base = 0; base < s.n; base += kWarp)
    {
        const int k = base + lane;
        bool hit = false;
        if (k < s.n && k != center)
        {
            const Pos4<T> p = tile[k];
            const T dx = min_image(c.x, p.x, s.length[0]);
            const T dy = min_image(c.y, p.y, s.length[1]);
            const T dz = min_image(c.z, p.z, s.length[2]);
            hit = squared_norm(dx, dy, dz) < r2max;
        }
        const unsigned hits = __ballot_sync(kFullMask, hit);
        const int e = count + __popc(hits & ((1u << lane) - 1u));
        if (hit && e < s.width)
        {
            *entry(e) = static_cast<std::uint16_t>(k);
        }
        count += __popc(hits);
    }
    const int stored = count < s.width ? count : s.width;
    const int padded = (stored + kChunk - 1) / kChunk * kChunk;
    if (stored + lane < padded)
    {
        *entry(stored + lane) = static_cast<std::uint16_t>(s.sentinel);
    }
    return count;
}

// One center's pair loop on the small-box path, its lanes' sums met in force_center_split's
// shuffle tree and with its arithmetic; chunk c of its list is chunks[c * stride], `count` its
// length. Returns the force (lane `part` 0 only) and adds half the pair energy to `energy`.
template <typename T, bool kMulti>
__device__ __forceinline__ void run_center_forces(const System<T>& s,
                                                  const Pos4<T>* __restrict__ tile,
                                                  const PairParams<T>* __restrict__ params,
                                                  const uint4* __restrict__ chunks, int stride,
                                                  int count, int center, int part,
                                                  T (&force)[3], double& energy)
{
    CenterSums<T> c{};
    const bool real = center < s.n;
    const Pos4<T> me = real ? tile[center] : far_atom<T>();
    if (real)
    {
        const int stored_chunks = s.width / kChunk;
        uint4 next = part < stored_chunks ? chunks[part * stride] : make_uint4(0, 0, 0, 0);
        const int used = count < s.width ? count : s.width;
        const int num_chunks = (used + kChunk - 1) / kChunk;
        const T cutoff_squared = s.cutoff_squared;
        const T s2 = params[0].s2;
        for (int chunk = part; chunk < num_chunks; chunk += kSmallLanes)
        {
            const uint4 word = next;
            if (chunk + kSmallLanes < num_chunks)
            {
                next = chunks[(chunk + kSmallLanes) * stride];
            }
            const unsigned packed[4] = {word.x, word.y, word.z, word.w};
#pragma unroll
            for (int r = 0; r < kChunk; ++r)
            {
                const Pos4<T> p = tile[(packed[r / 2] >> (16 * (r % 2))) & 0xffffu];
                const T dx = min_image(me.x, p.x, s.length[0]);
                const T dy = min_image(me.y, p.y, s.length[1]);
                const T dz = min_image(me.z, p.z, s.length[2]);
                const T r2 = squared_norm(dx, dy, dz);
                const bool inside = r2 < cutoff_squared;
                const T inv_r2 = fast_reciprocal(r2);
                PairParams<T> pp;
                if (kMulti)
                {
                    pp = params[type_pair_row(static_cast<int>(me.w), static_cast<int>(p.w),
                                              s.num_types)];
                }
                const T q = (kMulti ? pp.s2 : s2) * inv_r2;
                const T p6 = q * q * q;
                const T mask = inside ? T(1) : T(0);
                T fs = mask * (inv_r2 * (p6 * fma(T(2), p6, T(-1))));
                const T u = fma(p6, p6, -p6);
                if (kMulti)
                {
                    fs *= pp.e24;
                    c.energy = fma(mask, fma(pp.e4, u, -pp.shift), c.energy);
                }
                else
                {
                    c.energy = fma(mask, u, c.energy);
                    c.inside += mask;
                }
                c.fx = fma(fs, dx, c.fx);
                c.fy = fma(fs, dy, c.fy);
                c.fz = fma(fs, dz, c.fz);
            }
        }
    }
#pragma unroll
    for (int offset = kSmallLanes / 2; offset > 0; offset /= 2)
    {
        c.fx += __shfl_xor_sync(kFullMask, c.fx, offset);
        c.fy += __shfl_xor_sync(kFullMask, c.fy, offset);
        c.fz += __shfl_xor_sync(kFullMask, c.fz, offset);
        c.energy += __shfl_xor_sync(kFullMask, c.energy, offset);
        c.inside += __shfl_xor_sync(kFullMask, c.inside, offset);
    }
    if (!real || part != 0)
    {
        return;
    }
    T scale = T(1);
    double e;
    if (kMulti)
    {
        e = double(c.energy);
    }
    else
    {
        scale = params[0].e24;
        e = double(params[0].e4) * double(c.energy) - double(params[0].shift) * double(c.inside);
    }
    force[0] = c.fx * scale;
    force[1] = c.fy * scale;
    force[2] = c.fz * scale;
    energy += 0.5 * e;
}

// The dynamic shared memory of a one-launch run: every atom's position (slots 0 .. sentinel),
// then, with the lists in shared memory, `centers` lists of `width` entries and their counts.
template <typename T>
std::size_t run_shared_bytes(const System<T>& s, int centers, bool shared_lists)
{
    std::size_t bytes = static_cast<std::size_t>(s.sentinel + 1) * sizeof(Pos4<T>);
    if (shared_lists)
    {
        bytes += static_cast<std::size_t>(centers) * s.width * sizeof(std::uint16_t);
        bytes += static_cast<std::size_t>(centers) * sizeof(int);
    }
    return bytes;
}

template <typename T, bool kMulti, bool kThermostat, bool kSharedLists>
__global__ void __launch_bounds__(kRunThreads, 1) small_run_kernel(System<T> s, int steps)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto* tile = reinterpret_cast<Pos4<T>*>(smem_raw);
    __shared__ PairParams<T> params[36];
    __shared__ double warp_sums[kRunThreads / kWarp][2];
    __shared__ T forces[kRunThreads][3];  // this step's force on each owned atom
    __shared__ T scales[2];
    __shared__ double thermo[kThermoSize];  // the chain's slots, stored at the end
    __shared__ double totals[2];            // the last step's E and K, stored at the end
    // Written by CTA r into slot r of every CTA: its E and K; the stamp (step + 1) of a step in
    // which one of its atoms moved past the reuse threshold; whether it saw a failure.
    __shared__ double partials[kRunCluster][2];
    __shared__ int moved[kRunCluster];
    __shared__ int failed[kRunCluster];
    const int rows = s.num_types * (s.num_types + 1) / 2;
    for (int k = threadIdx.x; k < rows; k += blockDim.x)
    {
        params[k] = pair_params(s.sigma[k], s.epsilon[k], s.cutoff_squared);
    }
    const int n = s.n;
    const int ctas = gridDim.x;
    const int rank = blockIdx.x;  // the grid is one cluster
    const int first = static_cast<int>(static_cast<std::int64_t>(n) * rank / ctas);
    const int last = static_cast<int>(static_cast<std::int64_t>(n) * (rank + 1) / ctas);
    const int centers = last - first;
    const int words = s.width / kChunk;  // chunks per list
    auto* lists = reinterpret_cast<std::uint16_t*>(tile + s.sentinel + 1);
    auto* counts = reinterpret_cast<int*>(lists + static_cast<std::size_t>(centers) * s.width);
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    // Thread t owns atom first + t (at most kRunThreads per CTA): its state stays in registers
    // for the whole launch and is stored back at the end.
    const int mine = first + static_cast<int>(threadIdx.x);
    const bool owner = mine < last;
    Pos4<T> position{}, reference{};
    T velocity[3] = {T(0), T(0), T(0)};
    T inv_mass = T(0), mass = T(0);
    if (owner)
    {
        position = s.pos[mine];
        reference = s.ref_pos[mine];
        for (int a = 0; a < 3; ++a)
        {
            velocity[a] = s.vel[3LL * mine + a];
            forces[threadIdx.x][a] = s.force[3LL * mine + a];
        }
        inv_mass = s.inv_mass[mine];
        mass = s.mass[mine];
    }
    for (int i = threadIdx.x; i < n; i += blockDim.x)
    {
        tile[i] = s.pos[i];
    }
    if (kSharedLists)
    {
        for (int i = threadIdx.x; i < centers; i += blockDim.x)
        {
            counts[i] = s.nbr_count[first + i];
        }
        const uint4* stored = reinterpret_cast<const uint4*>(s.nbr);
        for (int w = threadIdx.x; w < centers * words; w += blockDim.x)
        {
            reinterpret_cast<uint4*>(lists)[w] =
                stored[chunk_index(first + w / words, w % words, s.width)];
        }
    }
    if (threadIdx.x < kRunCluster)
    {
        moved[threadIdx.x] = 0;
        failed[threadIdx.x] = 0;
    }
    // Thread 0's chain state and constants (1 / Q, g, kT, dt), in registers for the launch.
    double chain_q[3] = {0, 0, 0}, chain_p[3] = {0, 0, 0}, chain_kinetic = 0, pending = 1;
    double inverse[3] = {0, 0, 0}, degrees = 0, thermal = 0, chain_dt = 0;
    if (threadIdx.x == 0)
    {
        tile[s.sentinel] = far_atom<T>();
        if (kThermostat)
        {
            for (int k = 0; k < kThermoSize; ++k)
            {
                thermo[k] = s.thermo[k];
            }
            for (int k = 0; k < 3; ++k)
            {
                chain_q[k] = thermo[kChainA + k];
                chain_p[k] = thermo[kChainA + 3 + k];
                inverse[k] = 1.0 / thermo[kChainMass + k];
            }
            chain_kinetic = thermo[kKineticA];
            pending = thermo[kPendingScale];
            degrees = thermo[kDegrees];
            thermal = thermo[kThermalEnergy];
            chain_dt = thermo[kTimestep];
        }
    }
    const bool failed_before = s.status[0] != 0;  // a latched failure stops the rebuilds
    int rebuilds = 0;
    const T kick = s.half_dt * inv_mass;
    // No CTA writes into another before every CTA has set up its shared memory.
    cluster_barrier();
    for (int step = 0; step < steps; ++step)
    {
        // The chain's opening half step (as every drift block computes it).
        if (kThermostat && threadIdx.x == 0)
        {
            const double factor =
                chain_half_step_inverse(chain_kinetic, chain_q, chain_p, inverse, degrees,
                                        thermal, chain_dt);
            scales[0] = static_cast<T>(pending);
            scales[1] = static_cast<T>(factor);
            for (int k = 0; k < 3; ++k)
            {
                thermo[kChainB + k] = chain_q[k];
                thermo[kChainB + 3 + k] = chain_p[k];
            }
            thermo[kKineticB] = chain_kinetic;
            thermo[kOpenScale] = factor;
        }
        __syncthreads();
        // The drift of the owned atom, from registers and this CTA's forces.
        if (owner)
        {
            T vx = velocity[0], vy = velocity[1], vz = velocity[2];
            if (kThermostat)
            {
                vx = (vx * scales[0]) * scales[1];
                vy = (vy * scales[0]) * scales[1];
                vz = (vz * scales[0]) * scales[1];
            }
            vx = fma(kick, forces[threadIdx.x][0], vx);
            vy = fma(kick, forces[threadIdx.x][1], vy);
            vz = fma(kick, forces[threadIdx.x][2], vz);
            position.x = fma(s.dt, vx, position.x);
            position.y = fma(s.dt, vy, position.y);
            position.z = fma(s.dt, vz, position.z);
            velocity[0] = vx;
            velocity[1] = vy;
            velocity[2] = vz;
            for (int r = 0; r < ctas; ++r)
            {
                cluster_peer(tile, r)[mine] = position;
            }
            if (!(isfinite(position.x) && isfinite(position.y) && isfinite(position.z)))
            {
                atomicOr(s.status, kNonFinite);
                for (int r = 0; r < ctas; ++r)
                {
                    cluster_peer(failed, r)[rank] = 1;
                }
            }
            else if (squared_norm(position.x - reference.x, position.y - reference.y,
                                  position.z - reference.z) >= s.threshold_squared)
            {
                for (int r = 0; r < ctas; ++r)
                {
                    cluster_peer(moved, r)[rank] = step + 1;  // every writer stores the same
                }
            }
        }
        cluster_barrier();
        // Every CTA reads the same flags here: this step's writers are all before the barrier,
        // the next step's after the next one, which no CTA passes before reading these. Lane
        // r of each warp reads slot r (slots past the cluster's CTAs stay zero).
        const bool rebuild =
            __any_sync(kFullMask, lane < kRunCluster && moved[lane % kRunCluster] == step + 1);
        const bool stop =
            failed_before ||
            __any_sync(kFullMask, lane < kRunCluster && failed[lane % kRunCluster] != 0);
        if (rebuild && !stop)
        {
            ++rebuilds;
            if (owner)
            {
                long long cx, cy, cz;
                position.x = wrap_axis(position.x, s.length[0], cx);
                position.y = wrap_axis(position.y, s.length[1], cy);
                position.z = wrap_axis(position.z, s.length[2], cz);
                if (cx | cy | cz)
                {
                    long long* image = s.images + 3LL * mine;
                    image[0] += cx;
                    image[1] += cy;
                    image[2] += cz;
                }
                reference = position;
                for (int r = 0; r < ctas; ++r)
                {
                    cluster_peer(tile, r)[mine] = position;
                }
            }
            cluster_barrier();
            // A warp per center: the ballot build stores what the per-step build's scan does.
            for (int local = warp; local < centers; local += kRunThreads / kWarp)
            {
                const int center = first + local;
                int count;
                if (kSharedLists)
                {
                    std::uint16_t* entries = lists + static_cast<std::size_t>(local) * s.width;
                    count = warp_center_list(s, tile, center, [&](int e) { return entries + e; });
                    if (lane == 0)
                    {
                        counts[local] = count;
                    }
                }
                else
                {
                    auto* entries = reinterpret_cast<std::uint16_t*>(s.nbr);
                    count = warp_center_list(s, tile, center, [&](int e) {
                        return entries + chunk_index(center, e / kChunk, s.width) * kChunk +
                               e % kChunk;
                    });
                    if (lane == 0)
                    {
                        s.nbr_count[center] = count;
                    }
                }
                if (lane == 0 && count > s.width)
                {
                    flag_overflow(s.status, 1, count);
                    for (int r = 0; r < ctas; ++r)
                    {
                        cluster_peer(failed, r)[rank] = 1;
                    }
                }
            }
            __syncthreads();
        }
        // This CTA's centers over kSmallLanes lanes each; the forces meet in shared memory.
        double sums[2] = {0.0, 0.0};
        const int tasks = centers * kSmallLanes;
        for (int base = 0; base < tasks; base += blockDim.x)
        {
            const int task = base + threadIdx.x;
            const int center = task < tasks ? first + task / kSmallLanes : n;  // n: no center
            const int local = center - first;
            const uint4* chunks = nullptr;
            int stride = 0, count = 0;
            if (center < n)
            {
                if (kSharedLists)
                {
                    chunks = reinterpret_cast<const uint4*>(lists) +
                             static_cast<std::size_t>(local) * words;
                    stride = 1;
                    count = counts[local];
                }
                else
                {
                    chunks = reinterpret_cast<const uint4*>(s.nbr) + chunk_index(center, 0, s.width);
                    stride = kWarp;
                    count = s.nbr_count[center];
                }
            }
            T force[3];
            run_center_forces<T, kMulti>(s, tile, params, chunks, stride, count, center,
                                         task % kSmallLanes, force, sums[0]);
            if (center < n && task % kSmallLanes == 0)
            {
                for (int a = 0; a < 3; ++a)
                {
                    forces[local][a] = force[a];
                }
            }
        }
        __syncthreads();
        // The second half kick of the owned atom, and its kinetic energy.
        if (owner)
        {
            const T vx = fma(kick, forces[threadIdx.x][0], velocity[0]);
            const T vy = fma(kick, forces[threadIdx.x][1], velocity[1]);
            const T vz = fma(kick, forces[threadIdx.x][2], velocity[2]);
            velocity[0] = vx;
            velocity[1] = vy;
            velocity[2] = vz;
            if (kThermostat)
            {
                sums[1] += 0.5 * double(mass) * (double(vx) * vx + double(vy) * vy + double(vz) * vz);
            }
        }
        const double e = warp_sum(sums[0]);
        const double k = warp_sum(sums[1]);
        if (lane == 0)
        {
            warp_sums[warp][0] = e;
            warp_sums[warp][1] = k;
        }
        __syncthreads();
        if (threadIdx.x == 0)
        {
            double sum[2] = {0.0, 0.0};
            for (int w = 0; w < kRunThreads / kWarp; ++w)
            {
                sum[0] += warp_sums[w][0];
                sum[1] += warp_sums[w][1];
            }
            for (int r = 0; r < ctas; ++r)
            {
                double* slot = cluster_peer(&partials[rank][0], r);
                slot[0] = sum[0];
                slot[1] = sum[1];
            }
        }
        cluster_barrier();
        // Every CTA: the totals in CTA order and the chain's closing half step
        // (finalize_kernel's). The next step's partials are written only after its drift
        // barrier, which every CTA reaches after reading these.
        if (threadIdx.x == 0)
        {
            double energy = 0.0, kinetic = 0.0;
            for (int c = 0; c < ctas; ++c)
            {
                energy += partials[c][0];
                kinetic += partials[c][1];
            }
            totals[0] = energy;
            totals[1] = kinetic;
            if (kThermostat)
            {
                chain_kinetic = kinetic;
                pending = chain_half_step_inverse(chain_kinetic, chain_q, chain_p, inverse,
                                                  degrees, thermal, chain_dt);
                for (int r = 0; r < 3; ++r)
                {
                    thermo[kChainA + r] = chain_q[r];
                    thermo[kChainA + 3 + r] = chain_p[r];
                }
                thermo[kKineticA] = chain_kinetic;
                thermo[kPendingScale] = pending;
            }
        }
    }
    // The state back to global memory; no CTA touches another's shared memory after the last
    // step's second barrier.
    if (owner)
    {
        s.pos[mine] = position;
        s.ref_pos[mine] = reference;
        for (int a = 0; a < 3; ++a)
        {
            s.vel[3LL * mine + a] = velocity[a];
            s.force[3LL * mine + a] = forces[threadIdx.x][a];
        }
    }
    if (kSharedLists && rebuilds > 0)
    {
        for (int i = threadIdx.x; i < centers; i += blockDim.x)
        {
            s.nbr_count[first + i] = counts[i];
        }
        uint4* stored = reinterpret_cast<uint4*>(s.nbr);
        for (int w = threadIdx.x; w < centers * words; w += blockDim.x)
        {
            const int local = w / words, chunk = w % words;
            if (chunk * kChunk < counts[local])
            {
                stored[chunk_index(first + local, chunk, s.width)] =
                    reinterpret_cast<const uint4*>(lists)[w];
            }
        }
    }
    if (rank == 0 && threadIdx.x == 0)
    {
        s.totals[0] = totals[0];
        s.totals[1] = totals[1];
        for (int r = 2; r < kReduced; ++r)
        {
            s.totals[r] = 0.0;
        }
        if (kThermostat)
        {
            for (int k = 0; k < kChainMass; ++k)
            {
                s.thermo[k] = thermo[k];
            }
        }
        s.rebuild_count[0] += rebuilds;
        s.rebuild[0] = 0;  // the reuse flag starts clean, as after a per-step rebuild
    }
}

// Launches one variant on `ctas` CTAs (one cluster); `placed` false when the GPU cannot hold
// a cluster that size (sizes past 8 are non-portable), nothing launched.
template <typename T, bool kMulti, bool kThermostat, bool kSharedLists>
cudaError_t launch_run_variant(const System<T>& s, int steps, int ctas, std::size_t bytes,
                               cudaStream_t stream, bool& placed)
{
    auto kernel = small_run_kernel<T, kMulti, kThermostat, kSharedLists>;
    // Set on every launch (a launch runs up to a thousand steps and is never graph-captured):
    // the static bytes count against the 48 KB a kernel gets without the grant.
    cudaError_t rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          static_cast<int>(bytes));
    if (rc == cudaSuccess && ctas > 8)
    {
        rc = cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    }
    if (rc != cudaSuccess)
    {
        return rc;
    }
    cudaLaunchConfig_t config = {};
    config.gridDim = dim3(ctas);
    config.blockDim = dim3(kRunThreads);
    config.dynamicSmemBytes = bytes;
    config.stream = stream;
    cudaLaunchAttribute attribute[1];
    attribute[0].id = cudaLaunchAttributeClusterDimension;
    attribute[0].val.clusterDim.x = ctas;
    attribute[0].val.clusterDim.y = 1;
    attribute[0].val.clusterDim.z = 1;
    config.attrs = attribute;
    config.numAttrs = 1;
    if (ctas > 8)
    {
        int clusters = 0;
        rc = cudaOccupancyMaxActiveClusters(&clusters, kernel, &config);
        if (rc != cudaSuccess)
        {
            return rc;
        }
        if (clusters < 1)
        {
            placed = false;
            return cudaSuccess;
        }
    }
    placed = true;
    return cudaLaunchKernelEx(&config, kernel, s, steps);
}

template <typename T>
cudaError_t launch_run_dispatch(const System<T>& s, bool multi, bool thermostat,
                                bool shared_lists, int steps, int ctas, std::size_t bytes,
                                cudaStream_t stream, bool& placed)
{
#define ND_RUN_CASE(MULTI, THERMO, SHARED)                                                   \
    if (multi == MULTI && thermostat == THERMO && shared_lists == SHARED)                    \
    {                                                                                        \
        return launch_run_variant<T, MULTI, THERMO, SHARED>(s, steps, ctas, bytes, stream,   \
                                                            placed);                         \
    }
    ND_RUN_CASE(false, false, true)
    ND_RUN_CASE(false, true, true)
    ND_RUN_CASE(true, false, true)
    ND_RUN_CASE(true, true, true)
    ND_RUN_CASE(false, false, false)
    ND_RUN_CASE(false, true, false)
    ND_RUN_CASE(true, false, false)
    ND_RUN_CASE(true, true, false)
#undef ND_RUN_CASE
    return cudaErrorInvalidValue;
}

template <typename T>
int launch_small_run(const System<T>& s, int thermostat, int steps, cudaStream_t stream)
{
    // A CTA per 32 atoms up to the largest cluster, a portable 8 when the GPU cannot place
    // that; the CTA's lists in shared memory when they fit beside the positions and the
    // kernel's static shared memory (about 14 KB in float64), else in the global list.
    constexpr std::size_t kSharedBudget = 200 * 1024;
    const int wanted = static_cast<int>((s.n + kWarp - 1) / kWarp);
    for (const int limit : {kRunCluster, 8})
    {
        const int ctas = std::max(1, std::min(limit, wanted));
        const int centers = static_cast<int>((s.n + ctas - 1) / ctas);
        const bool shared_lists = run_shared_bytes(s, centers, true) <= kSharedBudget;
        const std::size_t bytes = run_shared_bytes(s, centers, shared_lists);
        bool placed = false;
        ND_CUDA_TRY(launch_run_dispatch(s, s.num_types > 1, thermostat != 0, shared_lists, steps,
                                        ctas, bytes, stream, placed));
        if (placed)
        {
            return ND_OK;
        }
    }
    set_error("no cluster of 8 CTAs fits on this GPU for a one-launch run");
    return ND_ECUDA;
}

// Sets the rebuild branch of a step graph from the device flag the drift kernel wrote.
// A graph of `steps` steps in which each step's rebuild kernels sit in the body of a
// conditional IF node whose condition the drift kernel sets from the device flag, so a step
// that reuses the list launches only the drift and the forces (and their finalize, when the
// step reduces anything). Built by capture into a graph we own (the body by capture into the node's graph).
template <typename T>
int build_step_graph(const System<T>& s, std::int64_t num_cells, int thermostat, int steps,
                     cudaGraph_t graph)
{
    cudaStream_t main = nullptr, body_stream = nullptr;
    ND_CUDA_TRY(cudaStreamCreateWithFlags(&main, cudaStreamNonBlocking));
    const cudaError_t created = cudaStreamCreateWithFlags(&body_stream, cudaStreamNonBlocking);
    if (created != cudaSuccess)
    {
        cudaStreamDestroy(main);
        ND_CUDA_TRY(created);
    }
    auto fail = [&](int rc) {
        cudaGraph_t partial = nullptr;
        cudaStreamEndCapture(body_stream, &partial);
        cudaStreamEndCapture(main, &partial);
        cudaGetLastError();
        cudaStreamDestroy(body_stream);
        cudaStreamDestroy(main);
        return rc;
    };
    if (cudaStreamBeginCaptureToGraph(main, graph, nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal) != cudaSuccess)
    {
        set_error("a step graph could not begin its capture");
        return fail(ND_ECUDA);
    }
    for (int step = 0; step < steps; ++step)
    {
        cudaGraphConditionalHandle handle;
        if (cudaGraphConditionalHandleCreate(&handle, graph, 0, cudaGraphCondAssignDefault) !=
            cudaSuccess)
        {
            set_error("a step graph could not create its conditional handle");
            return fail(ND_ECUDA);
        }
        const unsigned atoms = blocks_for(s.n);
        if (thermostat)
        {
            drift_kernel<T, true, true><<<atoms, kThreads, 0, main>>>(s, handle);
        }
        else
        {
            drift_kernel<T, false, true><<<atoms, kThreads, 0, main>>>(s, handle);
        }
        if (cudaGetLastError() != cudaSuccess)
        {
            set_error("a step graph could not capture its drift");
            return fail(ND_ECUDA);
        }
        cudaStreamCaptureStatus capture_status;
        const cudaGraphNode_t* dependencies = nullptr;
        std::size_t count = 0;
        if (cudaStreamGetCaptureInfo(main, &capture_status, nullptr, nullptr, &dependencies,
                                     &count) != cudaSuccess)
        {
            set_error("a step graph could not read its capture");
            return fail(ND_ECUDA);
        }
        cudaGraphNodeParams params = {};
        params.type = cudaGraphNodeTypeConditional;
        params.conditional.handle = handle;
        params.conditional.type = cudaGraphCondTypeIf;
        params.conditional.size = 1;
        cudaGraphNode_t node;
        if (cudaGraphAddNode(&node, graph, dependencies, count, &params) != cudaSuccess ||
            cudaStreamUpdateCaptureDependencies(main, &node, 1,
                                                cudaStreamSetCaptureDependencies) != cudaSuccess)
        {
            set_error("a step graph could not add its conditional rebuild");
            return fail(ND_ECUDA);
        }
        cudaGraph_t body = params.conditional.phGraph_out[0];
        if (cudaStreamBeginCaptureToGraph(body_stream, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        {
            set_error("a step graph could not capture its rebuild");
            return fail(ND_ECUDA);
        }
        int rc = launch_rebuild(s, num_cells, 1, body_stream);
        if (rc != ND_OK)
        {
            return fail(rc);
        }
        if (cudaStreamEndCapture(body_stream, &body) != cudaSuccess)
        {
            set_error("a step graph could not end its rebuild capture");
            return fail(ND_ECUDA);
        }
        rc = launch_step(s, num_cells, thermostat, 0, 2, main);
        if (rc != ND_OK)
        {
            return fail(rc);
        }
    }
    cudaGraph_t captured = graph;
    const cudaError_t ended = cudaStreamEndCapture(main, &captured);
    cudaStreamDestroy(body_stream);
    cudaStreamDestroy(main);
    ND_CUDA_TRY(ended);
    return ND_OK;
}

int check_system(const nd_md_system* m)
{
    ND_REQUIRE(m != nullptr, "the system is null");
    ND_REQUIRE(m->dtype == ND_FLOAT32 || m->dtype == ND_FLOAT64,
               "the system must be float32 or float64");
    ND_REQUIRE(m->num_atoms >= 2 && m->num_atoms <= INT32_MAX, "N must be in [2, 2**31)");
    ND_REQUIRE(m->num_types >= 1 && m->num_types <= 8, "1 to 8 atom types are supported");
    ND_REQUIRE(m->width >= 8 && m->width % 8 == 0, "the list width must be a positive multiple of 8");
    const std::size_t pos_bytes = m->dtype == ND_FLOAT32 ? 16 : 32;
    if (m->small)
    {
        ND_REQUIRE(m->num_atoms <= 65534, "a small-box system holds at most 65534 atoms");
        ND_REQUIRE(static_cast<std::size_t>(m->num_atoms + 1) * pos_bytes <= 200 * 1024,
                   "a small-box system must fit one shared-memory tile");
    }
    else
    {
        ND_REQUIRE(m->dims[0] >= 3 && m->dims[1] >= 3 && m->dims[2] >= 3,
                   "the cell grid needs three or more cells per axis");
        ND_REQUIRE(m->bricks_x >= 1 && m->bricks_x <= m->dims[0], "bricks_x out of range");
        ND_REQUIRE((m->dims[0] + m->bricks_x - 1) / m->bricks_x <= kMaxBrickCells,
                   "a brick spans too many cells");
        ND_REQUIRE(m->tile_capacity >= 1 && m->tile_capacity <= 65534 &&
                       static_cast<std::size_t>(m->tile_capacity + 1) * pos_bytes <= 200 * 1024,
                   "the tile capacity must fit shared memory and uint16 indices");
    }
    return ND_OK;
}

}  // namespace nd

// ---------------------------------------------------------------------------------------
// C-ABI.

#define ND_MD_DISPATCH(m, call)                                                 \
    ((m)->dtype == ND_FLOAT32 ? [&] { auto s = nd::view<float>(m); return call; }() \
                              : [&] { auto s = nd::view<double>(m); return call; }())

extern "C" {

int nd_md_import(const nd_md_system* system, const void* positions, const void* velocities,
                 const void* masses, const int64_t* images, const int32_t* types,
                 nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(positions && velocities && masses && images, "a frame pointer is null");
    auto st = static_cast<cudaStream_t>(stream);
    return ND_MD_DISPATCH(system, ([&] {
        using T = std::remove_pointer_t<decltype(s.vel)>;
        nd::import_kernel<T><<<nd::blocks_for(s.n), nd::kThreads, 0, st>>>(
            s, static_cast<const T*>(positions), static_cast<const T*>(velocities),
            static_cast<const T*>(masses), reinterpret_cast<const long long*>(images),
            system->num_types > 1 ? types : nullptr);
        ND_LAUNCH_CHECK();
        return ND_OK;
    }()));
}

int nd_md_rebuild(const nd_md_system* system, nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    const std::int64_t cells =
        static_cast<std::int64_t>(system->dims[0]) * system->dims[1] * system->dims[2];
    return ND_MD_DISPATCH(system, nd::launch_rebuild(s, cells, 0, st));
}

int nd_md_forces(const nd_md_system* system, int virial, nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return ND_MD_DISPATCH(system, nd::launch_forces(s, virial, st));
}

int nd_md_step(const nd_md_system* system, int thermostat, int virial, nd_stream_t stream)
{
    return nd_md_step_phase(system, -1, thermostat, virial, stream);
}

int nd_md_step_phase(const nd_md_system* system, int phase, int thermostat, int virial,
                     nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(phase >= -1 && phase <= 2, "the phase must be -1 (all), 0, 1 or 2");
    auto st = static_cast<cudaStream_t>(stream);
    const std::int64_t cells =
        static_cast<std::int64_t>(system->dims[0]) * system->dims[1] * system->dims[2];
    return ND_MD_DISPATCH(system, nd::launch_step(s, cells, thermostat, virial, phase, st));
}

int nd_md_run_small(const nd_md_system* system, int thermostat, int steps, nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(system->small, "only small-box systems (fewer than three cells on an axis) run in one launch");
    ND_REQUIRE(system->num_atoms <= nd::kRunMaxAtoms, "a one-launch run takes at most 4096 atoms");
    ND_REQUIRE(steps >= 0, "steps must be nonnegative");
    if (steps == 0)
    {
        return ND_OK;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return ND_MD_DISPATCH(system, nd::launch_small_run(s, thermostat, steps, st));
}

int nd_md_step_launches(const nd_md_system* system, int64_t* launches)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(launches != nullptr, "launches is null");
    *launches = nd::step_launches(system);
    return ND_OK;
}

int nd_md_graph_create(const nd_md_system* system, int thermostat, int steps, void** graph_out)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(steps >= 1 && steps <= 4096, "steps must lie in [1, 4096]");
    ND_REQUIRE(graph_out != nullptr, "graph_out is null");
    const std::int64_t cells =
        static_cast<std::int64_t>(system->dims[0]) * system->dims[1] * system->dims[2];
    cudaGraph_t graph = nullptr;
    ND_CUDA_TRY(cudaGraphCreate(&graph, 0));
    const int built = ND_MD_DISPATCH(system,
                                     nd::build_step_graph(s, cells, thermostat, steps, graph));
    if (built != ND_OK)
    {
        cudaGraphDestroy(graph);
        return built;
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t instantiated = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    ND_CUDA_TRY(instantiated);
    *graph_out = exec;
    return ND_OK;
}

int nd_md_graph_launch(void* graph, nd_stream_t stream)
{
    ND_REQUIRE(graph != nullptr, "the graph is null");
    ND_CUDA_TRY(cudaGraphLaunch(static_cast<cudaGraphExec_t>(graph),
                                static_cast<cudaStream_t>(stream)));
    return ND_OK;
}

int nd_md_graph_destroy(void* graph)
{
    if (graph != nullptr)
    {
        ND_CUDA_TRY(cudaGraphExecDestroy(static_cast<cudaGraphExec_t>(graph)));
    }
    return ND_OK;
}

int nd_md_export(const nd_md_system* system, void* positions, void* velocities, void* forces,
                 int64_t* images, int thermostat, nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return ND_MD_DISPATCH(system, ([&] {
        using T = std::remove_pointer_t<decltype(s.vel)>;
        nd::export_kernel<T><<<nd::blocks_for(s.n), nd::kThreads, 0, st>>>(
            s, static_cast<T*>(positions), static_cast<T*>(velocities), static_cast<T*>(forces),
            reinterpret_cast<long long*>(images), thermostat);
        ND_LAUNCH_CHECK();
        return ND_OK;
    }()));
}

int nd_md_kinetic(const nd_md_system* system, int thermostat, nd_stream_t stream)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return ND_MD_DISPATCH(system, ([&] {
        using T = std::remove_pointer_t<decltype(s.vel)>;
        const unsigned blocks = nd::blocks_for(s.n, nd::kMDThreads);
        nd::kinetic_kernel<T><<<blocks, nd::kMDThreads, 0, st>>>(s, thermostat);
        ND_LAUNCH_CHECK();
        nd::finalize_kernel<false, false><<<1, nd::kFinalizeThreads, 0, st>>>(
            s.partials, static_cast<int>(blocks), s.totals + nd::kReduced, s.thermo, s.rebuild);
        ND_LAUNCH_CHECK();
        return ND_OK;
    }()));
}

int nd_md_partial_slots(const nd_md_system* system, int64_t* slots)
{
    const int rc = nd::check_system(system);
    if (rc != ND_OK)
    {
        return rc;
    }
    ND_REQUIRE(slots != nullptr, "slots is null");
    const std::int64_t bricks =
        system->small
            ? (system->num_atoms * nd::kSmallLanes + nd::kMDThreads - 1) / nd::kMDThreads
            : static_cast<std::int64_t>(system->bricks_x) * system->dims[1] * system->dims[2];
    const std::int64_t atoms = (system->num_atoms + nd::kMDThreads - 1) / nd::kMDThreads;
    *slots = (bricks > atoms ? bricks : atoms) * nd::kReduced;
    return ND_OK;
}

}  // extern "C"
