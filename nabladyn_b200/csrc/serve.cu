// The replica server: many independent Lennard-Jones NVT replicas (tens to thousands of atoms
// each) resident in one pool, advanced by a persistent kernel in which each CTA owns one
// replica and runs a whole budget of steps: the chain half steps, the drift, the on-GPU reuse
// check, the rebuild, the forces and the second half kick, separated by block barriers only.
// No per-step launch, no grid-wide synchronisation: replicas never wait on each other, so a
// replica's arithmetic (and its result, bit for bit) does not depend on its batch-mates.
//
// It serves the same step as the MD engine (src/nabladyn/md/_ensembles/_nvt.py:88-129,
// _nve.py:39-58, _chain.py:36-83, the reuse rule of src/nabladyn/neighbors/csrc/update/
// update.cuh:21-116) for systems too small to fill a GPU one at a time. Positions stay unwrapped
// between rebuilds and every pair takes its minimum image. The neighbor list is the engine's
// chunked full list of uint16 replica-local indices; a rebuild sorts the replica into cells
// (deterministically, by atom index within a cell) in the CTA, or tests all pairs when an axis
// has fewer than three cells.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "geometry.cuh"
#include "md_common.cuh"

namespace nd {

constexpr int kServeThreads = 512;
constexpr int kServeWarps = kServeThreads / kWarp;
constexpr int kServeMaxCells = 4096;

struct ServePool
{
    nd_replica* replicas;
    Pos4<float>* pos;
    float* vel;
    float* force;
    float* mass;
    float* inv_mass;
    long long* images;
    Pos4<float>* ref_pos;
    std::uint16_t* nbr;
    index_t* nbr_count;
    index_t* sorted;
    index_t* scratch;
    index_t* cell_start;
    Pos4<float>* ordered;
};

// The scalar fields of one replica, in shared memory for the CTA.
struct ReplicaScalars
{
    int n;
    int width;
    int dims[3];
    int cells;
    float cell[3];
    float widths[3];
    float cutoff_squared;
    float radius_squared;
    float threshold_squared;
    float dt;
    float half_dt;
    PairParams<float> lj;
    int status;
    int rebuild_count;
    int steps_left;
};

// Block sum of one double per thread, in a fixed order; every thread gets the total.
__device__ double block_sum(double value, double* warp_sums)
{
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    value = warp_sum(value);
    if (lane == 0)
    {
        warp_sums[warp] = value;
    }
    __syncthreads();
    double total = 0;
    for (int w = 0; w < kServeWarps; ++w)
    {
        total += warp_sums[w];
    }
    __syncthreads();
    return total;
}

// Exclusive scan of counts[0, cells) in place (counts[cells] gets the total), kServeMaxCells at
// most: each thread owns 8 consecutive counts, the 512 thread sums are scanned by warps.
__device__ void block_scan_cells(int* counts, int cells, int* warp_totals)
{
    constexpr int kPer = kServeMaxCells / kServeThreads;
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    const int base = threadIdx.x * kPer;
    int local[kPer];
    int sum = 0;
#pragma unroll
    for (int k = 0; k < kPer; ++k)
    {
        local[k] = base + k < cells ? counts[base + k] : 0;
        sum += local[k];
    }
    int inclusive = sum;
#pragma unroll
    for (int offset = 1; offset < kWarp; offset *= 2)
    {
        const int up = __shfl_up_sync(kFullMask, inclusive, offset);
        inclusive += lane >= offset ? up : 0;
    }
    if (lane == kWarp - 1)
    {
        warp_totals[warp] = inclusive;
    }
    __syncthreads();
    int before = 0;
    for (int w = 0; w < warp; ++w)
    {
        before += warp_totals[w];
    }
    int running = before + inclusive - sum;
#pragma unroll
    for (int k = 0; k < kPer; ++k)
    {
        if (base + k < cells)
        {
            counts[base + k] = running;
        }
        running += local[k];
    }
    if (threadIdx.x == kServeThreads - 1)
    {
        counts[cells] = running;
    }
    __syncthreads();
}

// Adds to `list` the atoms k = begin .. end - 1 closer to `me` (atom i) than the list radius
// under the minimum image, in k order (the all-pairs path of a replica with fewer than three
// cells along an axis). Four candidates at a time, loaded before any is tested.
__device__ __forceinline__ void scan_candidates(const ReplicaScalars& r, const Pos4<float>& me,
                                                int i, int begin, int end,
                                                const Pos4<float>* pos, ListWriter& list)
{
    constexpr int kGroup = 4;
    for (int k = begin; k < end; k += kGroup)
    {
        int j[kGroup];
        Pos4<float> p[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u)
        {
            j[u] = k + u < end ? k + u : -1;
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u)
        {
            p[u] = j[u] >= 0 ? pos[j[u]] : me;
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u)
        {
            const float d2 = squared_norm(min_image(me.x, p[u].x, r.cell[0]),
                                          min_image(me.y, p[u].y, r.cell[1]),
                                          min_image(me.z, p[u].z, r.cell[2]));
            if (j[u] >= 0 && j[u] != i && d2 < r.radius_squared)
            {
                list.add(j[u]);
            }
        }
    }
}

// The image of one stencil cell along an axis: the cell index h + d wrapped into [0, dims),
// and which side of the displacement takes the period. Past the upper face the center moves
// (center - L), past the lower face the candidate does (candidate - L): the two forms the
// minimum image rounds (min_image), so every candidate within the radius gets the bits the
// per-candidate minimum image gives it (the radius is below half the period: on a grid every
// axis has at least three cells at least one radius wide, and a displacement under the radius
// along an axis has one image within half the period).
struct AxisImage
{
    int cell;
    float center_shift;
    float candidate_shift;
};

__device__ __forceinline__ AxisImage axis_image(int h, int d, int dims, float length)
{
    AxisImage a{h + d, 0.0f, 0.0f};
    if (a.cell < 0)
    {
        a.cell += dims;
        a.candidate_shift = length;
    }
    else if (a.cell >= dims)
    {
        a.cell -= dims;
        a.center_shift = length;
    }
    return a;
}

// Adds to `list` the candidates of one stencil cell, k = begin .. end - 1 of the cell-ordered
// copy (x, y, z, and the atom's index in w), that lie closer than the list radius to the
// center (cell-order row `self`), in k order: one 16-B load per candidate, no index lookup
// and no per-candidate image choice. Eight candidates at a time, all loaded before any is
// tested; their hits are kept as bits and appended lowest first (one append loop per group
// instead of a branch per candidate; groups of 4 and 16 measured slower).
__device__ __forceinline__ void scan_cell(const ReplicaScalars& r, float cx, float cy, float cz,
                                          float sx, float sy, float sz, int self,
                                          const Pos4<float>* __restrict__ ordered, int begin,
                                          int end, StagedListWriter& list)
{
    constexpr int kGroup = 8;
    for (int k = begin; k < end; k += kGroup)
    {
        Pos4<float> p[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u)
        {
            p[u] = k + u < end ? ordered[k + u] : far_atom<float>();
        }
        unsigned hits = 0;
#pragma unroll
        for (int u = 0; u < kGroup; ++u)
        {
            const float d2 = squared_norm(cx - (p[u].x - sx), cy - (p[u].y - sy),
                                          cz - (p[u].z - sz));
            hits |= static_cast<unsigned>(k + u != self && d2 < r.radius_squared) << u;
        }
        while (hits != 0)
        {
            const int u = __ffs(hits) - 1;
            hits &= hits - 1;
            list.add(static_cast<unsigned>(reinterpret_cast<const int*>(ordered + k + u)[3]));
        }
    }
}

// Wraps the positions (counting crossings into the images), stores the reference frame and
// rebuilds the list. Called by the whole CTA. On a grid, `ordered` receives the wrapped
// positions in cell order with each atom's index in w, which the candidate scan reads.
__device__ void rebuild_replica(const ReplicaScalars& r, Pos4<float>* pos, Pos4<float>* ref,
                                long long* images, std::uint16_t* nbr, index_t* nbr_count,
                                index_t* sorted, index_t* scratch, index_t* cell_start,
                                Pos4<float>* ordered, int* counts, int* warp_totals,
                                int* status_flags)
{
    const int n = r.n;
    for (int i = threadIdx.x; i < n; i += kServeThreads)
    {
        Pos4<float> p = pos[i];
        long long c[3];
        p.x = wrap_axis(p.x, r.cell[0], c[0]);
        p.y = wrap_axis(p.y, r.cell[1], c[1]);
        p.z = wrap_axis(p.z, r.cell[2], c[2]);
        if (c[0] | c[1] | c[2])
        {
            images[3LL * i] += c[0];
            images[3LL * i + 1] += c[1];
            images[3LL * i + 2] += c[2];
        }
        pos[i] = p;
        ref[i] = p;
    }
    const bool grid = r.dims[0] >= 3 && r.dims[1] >= 3 && r.dims[2] >= 3;
    if (grid)
    {
        // Counting sort by cell (the slot parked in nbr_count, rewritten by the list below),
        // then each cell's range ordered by atom index, so the order is deterministic.
        for (int c = threadIdx.x; c <= r.cells; c += kServeThreads)
        {
            counts[c] = 0;
        }
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += kServeThreads)
        {
            const Pos4<float> p = pos[i];
            const int c = axis_bin(p.x, r.widths[0], r.dims[0]) +
                          r.dims[0] * (axis_bin(p.y, r.widths[1], r.dims[1]) +
                                       r.dims[1] * axis_bin(p.z, r.widths[2], r.dims[2]));
            scratch[i] = c;
            nbr_count[i] = atomicAdd(counts + c, 1);
        }
        __syncthreads();
        block_scan_cells(counts, r.cells, warp_totals);
        for (int c = threadIdx.x; c <= r.cells; c += kServeThreads)
        {
            cell_start[c] = counts[c];
        }
        for (int i = threadIdx.x; i < n; i += kServeThreads)
        {
            sorted[counts[scratch[i]] + nbr_count[i]] = i;
        }
        __syncthreads();
        for (int c = threadIdx.x; c < r.cells; c += kServeThreads)
        {
            const int begin = counts[c], end = counts[c + 1];
            for (int k = begin + 1; k < end; ++k)
            {
                const int atom = sorted[k];
                int m = k - 1;
                while (m >= begin && sorted[m] > atom)
                {
                    sorted[m + 1] = sorted[m];
                    --m;
                }
                sorted[m + 1] = atom;
            }
        }
        __syncthreads();
        for (int row = threadIdx.x; row < n; row += kServeThreads)
        {
            const int atom = sorted[row];
            Pos4<float> p = pos[atom];
            p.w = __int_as_float(atom);
            ordered[row] = p;
        }
    }
    __syncthreads();
    // The list: every neighbor j != i closer than the list radius, minimum image. Row `row`
    // holds the list of atom sorted[row] on a grid (the lanes of a warp take atoms of one or
    // two cells, whose candidates they share), of atom `row` otherwise. On a grid the stencil
    // is scanned in two passes, each in stencil order with candidates in cell order: first the
    // cells that need no image, whose entries (the "direct" ones) keep the plain difference as
    // their minimum image until the next rebuild, then the cells across a face. Each cell is
    // scanned with its image, so the entries are those of a scan of every candidate with its
    // own minimum image. nbr_count[row] holds the count in its low 16 bits and the direct
    // entries in its high 16 bits (a count is at most N - 1 < 2^16).
    // A row's entries go through 16 bytes of shared memory per thread, a chunk at a time to
    // global memory (the staged writer measured 14 % faster than packing them in registers).
    __shared__ __align__(16) std::uint16_t lane_slots[kServeThreads][kChunk];
    for (int row = threadIdx.x; row < n; row += kServeThreads)
    {
        StagedListWriter list(nbr, lane_slots[threadIdx.x], r.width, row);
        int direct = 0;
        if (grid)
        {
            const Pos4<float> me = ordered[row];
            const int hx = axis_bin(me.x, r.widths[0], r.dims[0]);
            const int hy = axis_bin(me.y, r.widths[1], r.dims[1]);
            const int hz = axis_bin(me.z, r.widths[2], r.dims[2]);
            for (int pass = 0; pass < 2; ++pass)
            {
                for (int dz = -1; dz <= 1; ++dz)
                {
                    const AxisImage iz = axis_image(hz, dz, r.dims[2], r.cell[2]);
                    const float cz = me.z - iz.center_shift;
                    for (int dy = -1; dy <= 1; ++dy)
                    {
                        const AxisImage iy = axis_image(hy, dy, r.dims[1], r.cell[1]);
                        const float cy = me.y - iy.center_shift;
                        for (int dx = -1; dx <= 1; ++dx)
                        {
                            const AxisImage ix = axis_image(hx, dx, r.dims[0], r.cell[0]);
                            const bool imaged = hx + dx != ix.cell || hy + dy != iy.cell ||
                                                hz + dz != iz.cell;
                            if (imaged != (pass == 1))
                            {
                                continue;
                            }
                            const int c = ix.cell + r.dims[0] * (iy.cell + r.dims[1] * iz.cell);
                            scan_cell(r, me.x - ix.center_shift, cy, cz, ix.candidate_shift,
                                      iy.candidate_shift, iz.candidate_shift, row, ordered,
                                      counts[c], counts[c + 1], list);
                        }
                    }
                }
                if (pass == 0)
                {
                    direct = list.count;
                }
            }
            list.finish(0xffffu);
        }
        else
        {
            ListWriter all(nbr, r.width, row, 0xffffu);
            scan_candidates(r, pos[row], row, 0, n, pos, all);
            all.finish();
            list.count = all.count;
        }
        nbr_count[row] = list.count | (direct << 16);
        if (list.count > r.width)
        {
            atomicOr(status_flags, kOverflow);
        }
    }
    __syncthreads();
}

// One list entry's pair term, added to the center's sums (an exact zero outside the cutoff).
// With kImage the displacement takes the minimum image; without, it is the plain difference,
// which is what the minimum image gives a direct entry (see rebuild_replica): the entry was
// within the list radius with no image at the rebuild, neither atom has moved half the skin
// since, and the period is more than twice the radius plus the skin on a grid.
template <bool kEnergy, bool kImage>
__device__ __forceinline__ void serve_pair(const ReplicaScalars& r, const Pos4<float>& me,
                                           const Pos4<float>& p, float& fx, float& fy, float& fz,
                                           float& esum, float& inside_count)
{
    const float dx = kImage ? min_image(me.x, p.x, r.cell[0]) : me.x - p.x;
    const float dy = kImage ? min_image(me.y, p.y, r.cell[1]) : me.y - p.y;
    const float dz = kImage ? min_image(me.z, p.z, r.cell[2]) : me.z - p.z;
    const float r2 = squared_norm(dx, dy, dz);
    const float mask = r2 < r.cutoff_squared ? 1.0f : 0.0f;
    const float inv_r2 = fast_reciprocal(r2);
    const float q = r.lj.s2 * inv_r2;
    const float p6 = q * q * q;
    const float fs = mask * (inv_r2 * (p6 * fmaf(2.0f, p6, -1.0f)));
    if (kEnergy)
    {
        esum = fmaf(mask, fmaf(p6, p6, -p6), esum);
        inside_count += mask;
    }
    fx = fmaf(fs, dx, fx);
    fy = fmaf(fs, dy, fy);
    fz = fmaf(fs, dz, fz);
}

// The eight entries of one list word.
template <bool kEnergy, bool kImage>
__device__ __forceinline__ void serve_chunk(const ReplicaScalars& r, const Pos4<float>* pos,
                                            const Pos4<float>& me, const uint4& word, float& fx,
                                            float& fy, float& fz, float& esum,
                                            float& inside_count)
{
    const unsigned packed[4] = {word.x, word.y, word.z, word.w};
#pragma unroll
    for (int k = 0; k < kChunk; ++k)
    {
        const Pos4<float> p = pos[(packed[k / 2] >> (16 * (k % 2))) & 0xffffu];
        serve_pair<kEnergy, kImage>(r, me, p, fx, fy, fz, esum, inside_count);
    }
}

// Forces at the current positions; with `kKick`, also the second half kick, returning the
// thread's part of K (float64); with `kEnergy`, the thread's part of E (a step needs E only
// when its energy is reported: the last step of a round). Whole chunks of the list go through
// without a bound check; only the last, partial chunk checks the count.
template <bool kKick, bool kEnergy>
__device__ void replica_forces(const ReplicaScalars& r, const Pos4<float>* pos, float* vel,
                               float* force, const float* mass, const float* inv_mass,
                               const std::uint16_t* nbr, const index_t* nbr_count,
                               const index_t* order, double& kinetic, double& energy)
{
    for (int base = 0; base < r.n; base += kServeThreads)
    {
        const int row = base + static_cast<int>(threadIdx.x);
        const unsigned active = __ballot_sync(kFullMask, row < r.n);
        if (row >= r.n)
        {
            break;
        }
        const int i = order != nullptr ? order[row] : row;  // the list row's atom
        const Pos4<float> me = pos[i];
        const int listed = nbr_count[row] & 0xffff;
        const int count = listed < r.width ? listed : r.width;
        const uint4* chunks = reinterpret_cast<const uint4*>(nbr) + chunk_index(row, 0, r.width);
        // The kick's inputs are loaded before the pairs, so their latency hides behind them.
        float v[3] = {0.0f, 0.0f, 0.0f}, w = 0.0f, m = 0.0f;
        if (kKick)
        {
            const float* vi = vel + 3LL * i;
            v[0] = vi[0];
            v[1] = vi[1];
            v[2] = vi[2];
            w = inv_mass[i];
            m = mass[i];
        }
        float fx = 0, fy = 0, fz = 0, esum = 0, inside_count = 0;
        const int full = count / kChunk;
        const int chunk_count = (count + kChunk - 1) / kChunk;
        // The whole words of direct entries come first; the word that holds the last direct
        // entry and every later one take the minimum image (which gives a direct entry the
        // same bits as the plain difference).
        const int direct_words = min((nbr_count[row] >> 16) / kChunk, full);
        // Each chunk's word is loaded one chunk ahead: a pool's lists are far larger than L2,
        // so a word comes from DRAM, and its latency now overlaps the previous chunk's pairs.
        uint4 next = chunk_count > 0 ? chunks[0] : make_uint4(0, 0, 0, 0);
        auto advance = [&](int chunk) {
            const uint4 word = next;
            if (chunk + 1 < chunk_count)
            {
                next = chunks[static_cast<std::int64_t>(chunk + 1) * kWarp];
            }
            return word;
        };
        // One vote per word keeps the choice uniform over the warp, whose rows are the atoms of
        // one or two cells: the plain difference when every lane's word is direct.
        const int warp_full = __reduce_max_sync(active, full);
        for (int chunk = 0; chunk < warp_full; ++chunk)
        {
            const bool mine = chunk < full;
            const bool direct = __all_sync(active, !mine || chunk < direct_words);
            if (mine)
            {
                const uint4 word = advance(chunk);
                if (direct)
                {
                    serve_chunk<kEnergy, false>(r, pos, me, word, fx, fy, fz, esum,
                                                inside_count);
                }
                else
                {
                    serve_chunk<kEnergy, true>(r, pos, me, word, fx, fy, fz, esum,
                                               inside_count);
                }
            }
        }
        if (full < chunk_count)
        {
            const unsigned packed[4] = {next.x, next.y, next.z, next.w};
#pragma unroll
            for (int k = 0; k < kChunk; ++k)
            {
                if (full * kChunk + k < count)
                {
                    const Pos4<float> p = pos[(packed[k / 2] >> (16 * (k % 2))) & 0xffffu];
                    serve_pair<kEnergy, true>(r, me, p, fx, fy, fz, esum, inside_count);
                }
            }
        }
        fx *= r.lj.e24;
        fy *= r.lj.e24;
        fz *= r.lj.e24;
        if (kEnergy)
        {
            energy += 0.5 * (double(r.lj.e4) * esum - double(r.lj.shift) * inside_count);
        }
        float* f = force + 3LL * i;
        f[0] = fx;
        f[1] = fy;
        f[2] = fz;
        if (kKick)
        {
            const float kick = r.half_dt * w;
            const float vx = fmaf(kick, fx, v[0]);
            const float vy = fmaf(kick, fy, v[1]);
            const float vz = fmaf(kick, fz, v[2]);
            float* vi = vel + 3LL * i;
            vi[0] = vx;
            vi[1] = vy;
            vi[2] = vz;
            kinetic += 0.5 * double(m) * (double(vx) * vx + double(vy) * vy + double(vz) * vz);
        }
    }
}

// mode 0: wrap, rebuild and the first forces of newly admitted replicas. mode 1: run each
// listed replica for min(budget, steps left) NVT steps. One CTA per SM, up to 128 registers a
// thread: held to two CTAs (64 registers) the kernel spills, and measured slower.
__global__ void __launch_bounds__(kServeThreads, 1) serve_kernel(ServePool p, const int* slots,
                                                              const int* budgets, int mode)
{
    __shared__ ReplicaScalars r;
    __shared__ double thermo[kThermoSize];
    __shared__ int counts[kServeMaxCells + 1];
    __shared__ double warp_sums[kServeWarps];
    __shared__ float scales[2];
    __shared__ int flags;
    __shared__ int warp_totals[kServeWarps];
    nd_replica* replica = p.replicas + slots[blockIdx.x];
    if (threadIdx.x == 0)
    {
        r.n = replica->num_atoms;
        r.width = replica->width;
        r.cells = 1;
        for (int a = 0; a < 3; ++a)
        {
            r.dims[a] = replica->dims[a];
            r.cells *= replica->dims[a];
            r.cell[a] = replica->cell[a];
            r.widths[a] = replica->widths[a];
        }
        r.cutoff_squared = replica->cutoff * replica->cutoff;
        r.radius_squared = replica->radius * replica->radius;
        r.threshold_squared = replica->threshold_squared;
        r.dt = replica->timestep;
        r.half_dt = 0.5f * replica->timestep;
        r.lj = pair_params(replica->sigma, replica->epsilon, r.cutoff_squared);
        r.status = replica->status;
        r.rebuild_count = replica->rebuild_count;
        r.steps_left = replica->steps_left;
        flags = 0;
    }
    for (int k = threadIdx.x; k < kThermoSize; k += kServeThreads)
    {
        thermo[k] = replica->thermostat[k];
    }
    __syncthreads();
    const std::int64_t a0 = replica->atom_offset;
    Pos4<float>* pos = p.pos + a0;
    Pos4<float>* ref = p.ref_pos + a0;
    float* vel = p.vel + 3 * a0;
    float* force = p.force + 3 * a0;
    const float* mass = p.mass + a0;
    const float* inv_mass = p.inv_mass + a0;
    long long* images = p.images + 3 * a0;
    std::uint16_t* nbr = p.nbr + replica->list_offset;
    index_t* nbr_count = p.nbr_count + a0;
    index_t* sorted = p.sorted + a0;
    index_t* scratch = p.scratch + a0;
    index_t* cell_start = p.cell_start + replica->cell_offset;
    Pos4<float>* ordered = p.ordered + a0;
    // List rows follow the cell order on a grid (set by every rebuild), else the atoms.
    const bool grid = r.dims[0] >= 3 && r.dims[1] >= 3 && r.dims[2] >= 3;
    const index_t* order = grid ? sorted : nullptr;

    if (mode == 0)
    {
        rebuild_replica(r, pos, ref, images, nbr, nbr_count, sorted, scratch, cell_start, ordered,
                        counts, warp_totals, &flags);
        double kinetic = 0, energy = 0;
        replica_forces<false, true>(r, pos, vel, force, mass, inv_mass, nbr, nbr_count, order,
                                    kinetic, energy);
        energy = block_sum(energy, warp_sums);
        if (threadIdx.x == 0)
        {
            replica->status = r.status | flags;
            replica->rebuild_count = r.rebuild_count + 1;
            replica->energy = energy;
        }
        return;
    }
    const int budget = budgets[blockIdx.x] < r.steps_left ? budgets[blockIdx.x] : r.steps_left;
    int done = 0;
    double last_energy = replica->energy;  // thread 0's copy
    for (; done < budget; ++done)
    {
        if (r.status != 0)
        {
            break;
        }
        if (threadIdx.x == 0)
        {
            // The opening chain half step; the previous closing factor is still pending.
            double kinetic = thermo[kKineticA];
            double q[3], pc[3];
            for (int k = 0; k < 3; ++k)
            {
                q[k] = thermo[kChainA + k];
                pc[k] = thermo[kChainA + 3 + k];
            }
            const double factor = chain_half_step(kinetic, q, pc, thermo + kChainMass,
                                                  thermo[kDegrees], thermo[kThermalEnergy],
                                                  thermo[kTimestep]);
            scales[0] = static_cast<float>(thermo[kPendingScale]);
            scales[1] = static_cast<float>(factor);
            for (int k = 0; k < 3; ++k)
            {
                thermo[kChainB + k] = q[k];
                thermo[kChainB + 3 + k] = pc[k];
            }
        }
        __syncthreads();
        int moved = 0, bad = 0;
        for (int i = threadIdx.x; i < r.n; i += kServeThreads)
        {
            float* v = vel + 3LL * i;
            const float* f = force + 3LL * i;
            const float kick = r.half_dt * inv_mass[i];
            const float vx = fmaf(kick, f[0], (v[0] * scales[0]) * scales[1]);
            const float vy = fmaf(kick, f[1], (v[1] * scales[0]) * scales[1]);
            const float vz = fmaf(kick, f[2], (v[2] * scales[0]) * scales[1]);
            v[0] = vx;
            v[1] = vy;
            v[2] = vz;
            Pos4<float> x = pos[i];
            x.x = fmaf(r.dt, vx, x.x);
            x.y = fmaf(r.dt, vy, x.y);
            x.z = fmaf(r.dt, vz, x.z);
            pos[i] = x;
            bad |= !(isfinite(x.x) && isfinite(x.y) && isfinite(x.z));
            const Pos4<float> x0 = ref[i];
            moved |= squared_norm(x.x - x0.x, x.y - x0.y, x.z - x0.z) >= r.threshold_squared;
        }
        if (__syncthreads_or(bad))
        {
            if (threadIdx.x == 0)
            {
                r.status |= kNonFinite;
            }
            __syncthreads();
            break;
        }
        if (__syncthreads_or(moved))
        {
            rebuild_replica(r, pos, ref, images, nbr, nbr_count, sorted, scratch, cell_start,
                            ordered, counts, warp_totals, &flags);
            if (threadIdx.x == 0)
            {
                ++r.rebuild_count;
                r.status |= flags;
            }
        }
        double kinetic = 0, energy = 0;
        const bool reported = done + 1 == budget;  // the round's last step reports its energy
        if (reported)
        {
            replica_forces<true, true>(r, pos, vel, force, mass, inv_mass, nbr, nbr_count,
                                       order, kinetic, energy);
        }
        else
        {
            replica_forces<true, false>(r, pos, vel, force, mass, inv_mass, nbr, nbr_count,
                                        order, kinetic, energy);
        }
        kinetic = block_sum(kinetic, warp_sums);
        if (reported)
        {
            energy = block_sum(energy, warp_sums);
        }
        if (threadIdx.x == 0)
        {
            if (reported)
            {
                last_energy = energy;
            }
            // The closing chain half step against this step's K.
            double q[3], pc[3];
            for (int k = 0; k < 3; ++k)
            {
                q[k] = thermo[kChainB + k];
                pc[k] = thermo[kChainB + 3 + k];
            }
            const double factor = chain_half_step(kinetic, q, pc, thermo + kChainMass,
                                                  thermo[kDegrees], thermo[kThermalEnergy],
                                                  thermo[kTimestep]);
            for (int k = 0; k < 3; ++k)
            {
                thermo[kChainA + k] = q[k];
                thermo[kChainA + 3 + k] = pc[k];
            }
            thermo[kKineticA] = kinetic;
            thermo[kPendingScale] = factor;
        }
        __syncthreads();
    }
    for (int k = threadIdx.x; k < kThermoSize; k += kServeThreads)
    {
        replica->thermostat[k] = thermo[k];
    }
    if (threadIdx.x == 0)
    {
        replica->steps_left = r.steps_left - done;
        replica->status = r.status;
        replica->rebuild_count = r.rebuild_count;
        replica->energy = last_energy;
    }
}

}  // namespace nd

extern "C" int nd_serve_run(const nd_replica_pool* pool, const int32_t* slots,
                            const int32_t* budgets, int32_t count, int32_t mode,
                            nd_stream_t stream)
{
    ND_REQUIRE(pool != nullptr && slots != nullptr, "the pool or the slot list is null");
    ND_REQUIRE(mode == 0 || (mode == 1 && budgets != nullptr), "mode is 0 (admit) or 1 (run)");
    ND_REQUIRE(count >= 0 && count <= 1 << 20, "count out of range");
    ND_REQUIRE(pool->replicas && pool->positions && pool->velocities && pool->forces &&
                   pool->masses && pool->inverse_masses && pool->images &&
                   pool->reference_positions && pool->neighbors && pool->neighbor_counts &&
                   pool->sorted && pool->scratch && pool->cell_starts &&
                   pool->ordered_positions,
               "a pool buffer is null");
    if (count == 0)
    {
        return ND_OK;
    }
    nd::ServePool p;
    p.replicas = pool->replicas;
    p.pos = static_cast<nd::Pos4<float>*>(pool->positions);
    p.vel = static_cast<float*>(pool->velocities);
    p.force = static_cast<float*>(pool->forces);
    p.mass = static_cast<float*>(pool->masses);
    p.inv_mass = static_cast<float*>(pool->inverse_masses);
    p.images = reinterpret_cast<long long*>(pool->images);
    p.ref_pos = static_cast<nd::Pos4<float>*>(pool->reference_positions);
    p.nbr = pool->neighbors;
    p.nbr_count = pool->neighbor_counts;
    p.sorted = pool->sorted;
    p.scratch = pool->scratch;
    p.cell_start = pool->cell_starts;
    p.ordered = static_cast<nd::Pos4<float>*>(pool->ordered_positions);
    nd::serve_kernel<<<count, nd::kServeThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        p, slots, budgets, mode);
    ND_LAUNCH_CHECK();
    return ND_OK;
}
