/*
 * ORACLE (test infrastructure only): a CPU restatement of the reference's neighbor operator.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may load this file's
 * library, and only as the checker. It restates, one thread at a time and in the same floating
 * point operations, the reference's CUDA kernels:
 *   binning          src/nabladyn/neighbors/csrc/grid/grid.cuh:10-49 (floor(x / w), clamped)
 *   in-bin order     grid.cuh:51-100 (ascending atom id)
 *   traversal        src/nabladyn/neighbors/csrc/common/traversal.cuh:12-147
 *   count / fill     src/nabladyn/neighbors/csrc/pairs/pairs.cuh:44-112, 140-157
 *   all-pairs path   src/nabladyn/neighbors/csrc/pairs/all_pairs.cuh:30-114
 *   reuse rule       src/nabladyn/neighbors/csrc/update/update.cuh:28-116
 * The reference compiles with nvcc's default contraction; the one contraction that decides the
 * pair set, r^2 = dx dx + dy dy + dz dz, is written here as fma(dz, dz, fma(dx, dx, dy * dy))
 * and pinned by the GPU parity tests. Build with -ffp-contract=off so the compiler adds no
 * other contraction.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define DEFINE_ORACLE(T, SUFFIX, FMA, FLOOR)                                                      \
    static T squared_norm_##SUFFIX(T dx, T dy, T dz) { return FMA(dz, dz, FMA(dx, dx, dy * dy)); } \
                                                                                                  \
    static T min_image_##SUFFIX(T center, T other, T length)                                      \
    {                                                                                             \
        const T raw = center - other;                                                             \
        const T half = (T)0.5 * length;                                                           \
        return raw > half ? (center - length) - other                                             \
                          : (raw < -half ? center - (other - length) : raw);                      \
    }                                                                                             \
                                                                                                  \
    static int32_t axis_bin_##SUFFIX(T x, T width, int32_t count)                                 \
    {                                                                                             \
        const int32_t bin = (int32_t)FLOOR(x / width);                                            \
        return bin < 0 ? 0 : (bin >= count ? count - 1 : bin);                                   \
    }                                                                                             \
                                                                                                  \
    typedef struct                                                                                \
    {                                                                                             \
        int32_t id;                                                                               \
        int32_t bin;                                                                              \
    } Entry_##SUFFIX;                                                                             \
                                                                                                  \
    static int compare_##SUFFIX(const void* a, const void* b)                                     \
    {                                                                                             \
        const Entry_##SUFFIX* x = (const Entry_##SUFFIX*)a;                                       \
        const Entry_##SUFFIX* y = (const Entry_##SUFFIX*)b;                                       \
        if (x->bin != y->bin) return x->bin < y->bin ? -1 : 1;                                    \
        return x->id < y->id ? -1 : (x->id > y->id);                                              \
    }                                                                                             \
                                                                                                  \
    /* Grid path. Writes up to `capacity` pairs (first, second) and returns the pair count. */    \
    int64_t oracle_grid_pairs_##SUFFIX(const T* positions, const T* cell, int64_t n,             \
                                       const int32_t* dims, const T* widths, double radius,       \
                                       int32_t* first, int32_t* second, int64_t capacity,         \
                                       int32_t* sorted_ids_out)                                   \
    {                                                                                             \
        const int32_t nx = dims[0], ny = dims[1], nz = dims[2];                                   \
        const int64_t bins = (int64_t)nx * ny * nz;                                               \
        Entry_##SUFFIX* entries = (Entry_##SUFFIX*)malloc(sizeof(Entry_##SUFFIX) * n);            \
        int32_t* offsets = (int32_t*)calloc(bins + 1, sizeof(int32_t));                           \
        T* sorted = (T*)malloc(sizeof(T) * 3 * n);                                                \
        int32_t* home_of = (int32_t*)malloc(sizeof(int32_t) * n);                                 \
        for (int64_t i = 0; i < n; ++i)                                                           \
        {                                                                                         \
            const T* p = positions + 3 * i;                                                       \
            entries[i].id = (int32_t)i;                                                           \
            entries[i].bin = axis_bin_##SUFFIX(p[0], widths[0], nx) +                             \
                             nx * (axis_bin_##SUFFIX(p[1], widths[1], ny) +                       \
                                   ny * axis_bin_##SUFFIX(p[2], widths[2], nz));                  \
            offsets[entries[i].bin + 1] += 1;                                                     \
        }                                                                                         \
        for (int64_t b = 0; b < bins; ++b) offsets[b + 1] += offsets[b];                          \
        qsort(entries, (size_t)n, sizeof(Entry_##SUFFIX), compare_##SUFFIX);                      \
        for (int64_t k = 0; k < n; ++k)                                                           \
        {                                                                                         \
            const int32_t id = entries[k].id;                                                     \
            memcpy(sorted + 3 * k, positions + 3 * (int64_t)id, sizeof(T) * 3);                   \
            home_of[k] = entries[k].bin;                                                          \
            if (sorted_ids_out) sorted_ids_out[k] = id;                                           \
        }                                                                                         \
        const T r = (T)radius;                                                                    \
        const T r2 = r * r;                                                                       \
        int64_t column = 0;                                                                       \
        const int stencil = nx >= 3 && ny >= 3 && nz >= 3;                                        \
        for (int64_t c = 0; c < n; ++c)                                                           \
        {                                                                                         \
            const T cx = sorted[3 * c], cy = sorted[3 * c + 1], cz = sorted[3 * c + 2];          \
            const int32_t home = home_of[c];                                                      \
            const int32_t h[3] = {home % nx, (home / nx) % ny, home / (nx * ny)};                 \
            const int32_t count[3] = {nx, ny, nz};                                                \
            const T length[3] = {cell[0], cell[1], cell[2]};                                      \
            const T center[3] = {cx, cy, cz};                                                     \
            const int span[3] = {stencil ? 3 : (nx >= 3 ? 3 : nx), stencil ? 3 : (ny >= 3 ? 3 : ny), \
                                 stencil ? 3 : (nz >= 3 ? 3 : nz)};                               \
            for (int iz = 0; iz < span[2]; ++iz)                                                  \
                for (int iy = 0; iy < span[1]; ++iy)                                              \
                    for (int ix = 0; ix < span[0]; ++ix)                                          \
                    {                                                                             \
                        const int step[3] = {ix, iy, iz};                                         \
                        int32_t b[3];                                                             \
                        T lead[3], trail[3];                                                      \
                        for (int a = 0; a < 3; ++a)                                               \
                        {                                                                         \
                            if (count[a] >= 3)                                                    \
                            {                                                                     \
                                const int32_t raw = h[a] + step[a] - 1;                           \
                                const T shift = raw < 0 ? -length[a]                              \
                                                        : (raw >= count[a] ? length[a] : (T)0);   \
                                b[a] = raw < 0 ? raw + count[a]                                   \
                                               : (raw >= count[a] ? raw - count[a] : raw);        \
                                lead[a] = shift > (T)0 ? center[a] - shift : center[a];           \
                                trail[a] = shift < (T)0 ? shift : (T)0;                           \
                            }                                                                     \
                            else                                                                  \
                            {                                                                     \
                                b[a] = step[a];                                                   \
                                lead[a] = center[a];                                              \
                                trail[a] = (T)0;                                                  \
                            }                                                                     \
                        }                                                                         \
                        const int32_t bin = b[0] + nx * (b[1] + ny * b[2]);                       \
                        const int32_t begin = offsets[bin], end = offsets[bin + 1];               \
                        for (int64_t k = begin > c ? begin : c + 1; k < end; ++k)                 \
                        {                                                                         \
                            const T* p = sorted + 3 * k;                                          \
                            T dx, dy, dz;                                                         \
                            if (stencil)                                                          \
                            {                                                                     \
                                dx = lead[0] - (p[0] + trail[0]);                                 \
                                dy = lead[1] - (p[1] + trail[1]);                                 \
                                dz = lead[2] - (p[2] + trail[2]);                                 \
                            }                                                                     \
                            else                                                                  \
                            {                                                                     \
                                dx = min_image_##SUFFIX(cx, p[0], cell[0]);                       \
                                dy = min_image_##SUFFIX(cy, p[1], cell[1]);                       \
                                dz = min_image_##SUFFIX(cz, p[2], cell[2]);                       \
                            }                                                                     \
                            if (squared_norm_##SUFFIX(dx, dy, dz) < r2)                           \
                            {                                                                     \
                                if (column < capacity)                                            \
                                {                                                                 \
                                    first[column] = entries[c].id;                                \
                                    second[column] = entries[k].id;                               \
                                }                                                                 \
                                ++column;                                                         \
                            }                                                                     \
                        }                                                                         \
                    }                                                                             \
        }                                                                                         \
        free(entries);                                                                            \
        free(offsets);                                                                            \
        free(sorted);                                                                             \
        free(home_of);                                                                            \
        return column;                                                                            \
    }                                                                                             \
                                                                                                  \
    /* All-pairs path: every (i, j), i < j, closer than the radius under the minimum image. */    \
    int64_t oracle_all_pairs_##SUFFIX(const T* positions, const T* cell, int64_t n,              \
                                      double radius, int32_t* first, int32_t* second,             \
                                      int64_t capacity)                                           \
    {                                                                                             \
        const T r = (T)radius;                                                                    \
        const T r2 = r * r;                                                                       \
        int64_t column = 0;                                                                       \
        for (int64_t i = 0; i < n; ++i)                                                           \
        {                                                                                         \
            const T* c = positions + 3 * i;                                                       \
            for (int64_t j = i + 1; j < n; ++j)                                                   \
            {                                                                                     \
                const T* p = positions + 3 * j;                                                   \
                const T d2 = squared_norm_##SUFFIX(min_image_##SUFFIX(c[0], p[0], cell[0]),       \
                                                   min_image_##SUFFIX(c[1], p[1], cell[1]),       \
                                                   min_image_##SUFFIX(c[2], p[2], cell[2]));      \
                if (d2 < r2)                                                                      \
                {                                                                                 \
                    if (column < capacity)                                                        \
                    {                                                                             \
                        first[column] = (int32_t)i;                                               \
                        second[column] = (int32_t)j;                                              \
                    }                                                                             \
                    ++column;                                                                     \
                }                                                                                 \
            }                                                                                     \
        }                                                                                         \
        return column;                                                                            \
    }                                                                                             \
                                                                                                  \
    /* The reuse rule: returns 1 to rebuild, 0 to reuse, -1 for a bad cell, -2 non-finite.       \
       Also writes the grid dims and widths an update would use. */                             \
    int oracle_reuse_##SUFFIX(const T* positions, const T* reference_positions, const T* cell,    \
                              const T* reference_cell, int64_t n, double cutoff, double radius,   \
                              const int32_t* limits, int32_t* dims, T* widths)                    \
    {                                                                                             \
        const T eps = sizeof(T) == 4 ? (T)1.1920928955078125e-07 : (T)2.220446049250313e-16;     \
        const T rc = (T)cutoff, rr = (T)radius;                                                   \
        T scale[3];                                                                               \
        T smallest = cell[0] / reference_cell[0];                                                 \
        T longest = cell[0];                                                                      \
        for (int a = 0; a < 3; ++a)                                                               \
        {                                                                                         \
            const T length = cell[a];                                                             \
            if (!(isfinite(length) && length > 2 * rc)) return -1;                                \
            scale[a] = length / reference_cell[a];                                                \
            smallest = scale[a] < smallest ? scale[a] : smallest;                                 \
            longest = length > longest ? length : longest;                                        \
            const T fit = FLOOR(length / FMA((T)4 * eps, length, rr));                            \
            const int32_t count = fit < 1 ? 1 : (fit > limits[a] ? limits[a] : (int32_t)fit);     \
            dims[a] = count;                                                                      \
            widths[a] = length / count;                                                           \
        }                                                                                         \
        for (int64_t i = 0; i < 3 * n; ++i)                                                       \
            if (!isfinite(positions[i])) return -2;                                               \
        const T allowance = FMA(-((T)32 * eps), longest, FMA(rr, smallest, -rc));                 \
        if (allowance <= 0) return 1;                                                             \
        const T threshold = allowance * allowance / 4;                                            \
        for (int64_t i = 0; i < n; ++i)                                                           \
        {                                                                                         \
            T moved = 0;                                                                          \
            for (int a = 0; a < 3; ++a)                                                           \
            {                                                                                     \
                const T d = min_image_##SUFFIX(positions[3 * i + a],                              \
                                               scale[a] * reference_positions[3 * i + a],         \
                                               cell[a]);                                          \
                moved = FMA(d, d, moved);                                                         \
            }                                                                                     \
            if (moved >= threshold) return 1;                                                     \
        }                                                                                         \
        return 0;                                                                                 \
    }

DEFINE_ORACLE(float, f32, fmaf, floorf)
DEFINE_ORACLE(double, f64, fma, floor)
