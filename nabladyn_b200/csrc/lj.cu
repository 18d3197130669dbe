// Lennard-Jones energy, forces, virial (and parameter gradients) over a [2, C] pair index,
// the NeighborPairs contract of src/nabladyn/neighbors/_pairs.py:8-22.
//
// It restates src/nabladyn/potential/_lennard_jones/_potential.py:209-234 with the
// derivatives written out instead of taken by torch.func (src/nabladyn/quantity.py:160-184):
// for a valid column (i != j, r^2 < r_c^2) with p6 = (sigma^2 / r^2)^3,
//     u   = 4 eps (p6^2 - p6) - u_c,                  u_c = u at r_c, unshifted,
//     f_s = 24 eps (2 p6^2 - p6) / r^2,               F_i += f_s d, F_j -= f_s d,
//     W  += f_s d (x) d,                               (W = -dE/dstrain at zero strain)
//     dE/deps   += 4 (p6^2 - p6) - 4 (pc6^2 - pc6),
//     dE/dsigma += 24 eps / sigma (2 p6^2 - p6 - 2 pc6^2 + pc6),
// with d the minimum-image vector x_i - x_j of src/nabladyn/space.py:11-19. Under a strain
// eps_s (src/nabladyn/space.py:51-64) every vector is deformed first, d' = (I + eps_s) d; then
// F_i = f_s (I + eps_s)^T d' and W_ab = f_s d'_a d_b, the derivatives of the strained energy.
//
// One pass computes everything; pair arithmetic runs in the positions' dtype and the totals
// (E, W, parameter gradients) are reduced in float64: per-thread partials, warp shuffles,
// one float64 atomic per block.

#include <cuda_runtime.h>

#include <cstdint>

#include "common.cuh"

namespace nd {

constexpr int kLJThreads = 256;
constexpr int kMaxRows = 36;  // T(T+1)/2 rows for up to 8 atom types

// The minimum-image vector left - right for coordinates in [0, L): the far coordinate moves
// by L first (src/nabladyn/space.py:11-19).
template <typename T>
__device__ __forceinline__ T displacement(T left, T right, T length)
{
    const T raw = left - right;
    const T half = T(0.5) * length;
    const T left_shift = raw > half ? length : T(0);
    const T right_shift = raw < -half ? length : T(0);
    return (left - left_shift) - (right - right_shift);
}

__device__ __forceinline__ int pair_row(int a, int b, int num_types)
{
    const int low = a < b ? a : b;
    const int high = a < b ? b : a;
    return low * (2 * num_types - low - 1) / 2 + high;
}

template <typename T>
struct LJAccumulators
{
    T energy = 0;
    T w[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};  // row-major W
};

template <typename T, bool kParameterGrads, bool kStrained>
__global__ void __launch_bounds__(kLJThreads) lj_pairs_kernel(
    const T* __restrict__ positions,
    const T* __restrict__ cell,
    const index_t* __restrict__ pairs,
    std::int64_t capacity,
    index_t num_atoms,
    const index_t* __restrict__ atom_types,  // null: one type
    int num_types,
    const T* __restrict__ sigma,
    const T* __restrict__ epsilon,
    const T* __restrict__ strain,
    T cutoff_squared,
    double* __restrict__ energy,
    T* __restrict__ forces,
    double* __restrict__ virial,
    double* __restrict__ sigma_grad,
    double* __restrict__ epsilon_grad
)
{
    // Frame blockIdx.y of a batch of frames with the same atoms and capacity.
    const std::int64_t frame = blockIdx.y;
    positions += frame * 3 * num_atoms;
    cell += frame * 3;
    pairs += frame * 2 * capacity;
    energy += frame;
    forces += frame * 3 * num_atoms;
    virial += frame * 9;
    const int rows = num_types * (num_types + 1) / 2;
    __shared__ double row_grads[2 * kMaxRows];
    if (kParameterGrads)
    {
        for (int k = threadIdx.x; k < 2 * rows; k += blockDim.x)
        {
            row_grads[k] = 0.0;
        }
        __syncthreads();
    }
    const T lx = cell[0], ly = cell[1], lz = cell[2];
    T e[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    if (kStrained)
    {
#pragma unroll
        for (int k = 0; k < 9; ++k)
        {
            e[k] = strain[k];
        }
    }
    LJAccumulators<T> acc;
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t column = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         column < capacity; column += stride)
    {
        const index_t i = pairs[column];
        const index_t j = pairs[capacity + column];
        // Self-pairs are padding; an index outside [0, N) is skipped, never read.
        if (i == j || static_cast<unsigned>(i) >= static_cast<unsigned>(num_atoms) ||
            static_cast<unsigned>(j) >= static_cast<unsigned>(num_atoms))
        {
            continue;
        }
        const T ux = displacement(positions[3LL * i], positions[3LL * j], lx);
        const T uy = displacement(positions[3LL * i + 1], positions[3LL * j + 1], ly);
        const T uz = displacement(positions[3LL * i + 2], positions[3LL * j + 2], lz);
        T dx = ux, dy = uy, dz = uz;
        if (kStrained)
        {
            dx = ux + ux * e[0] + uy * e[1] + uz * e[2];
            dy = uy + ux * e[3] + uy * e[4] + uz * e[5];
            dz = uz + ux * e[6] + uy * e[7] + uz * e[8];
        }
        const T r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < cutoff_squared))
        {
            continue;
        }
        const int row = atom_types == nullptr ? 0 : pair_row(atom_types[i], atom_types[j], num_types);
        const T s = sigma[row];
        const T eps = epsilon[row];
        const T s2 = s * s;
        const T inv_r2 = T(1) / r2;
        const T q = s2 * inv_r2;
        const T p6 = q * q * q;
        const T qc = s2 / cutoff_squared;
        const T pc6 = qc * qc * qc;
        const T shift = T(4) * eps * (pc6 * pc6 - pc6);
        acc.energy += T(4) * eps * (p6 * p6 - p6) - shift;
        const T fs = T(24) * eps * (T(2) * p6 * p6 - p6) * inv_r2;
        T fx = fs * dx, fy = fs * dy, fz = fs * dz;
        if (kStrained)
        {
            acc.w[0] += fx * ux;
            acc.w[1] += fx * uy;
            acc.w[2] += fx * uz;
            acc.w[3] += fy * ux;
            acc.w[4] += fy * uy;
            acc.w[5] += fy * uz;
            acc.w[6] += fz * ux;
            acc.w[7] += fz * uy;
            acc.w[8] += fz * uz;
            // The force on the undeformed positions: (I + eps_s)^T f.
            const T gx = fx + e[0] * fx + e[3] * fy + e[6] * fz;
            const T gy = fy + e[1] * fx + e[4] * fy + e[7] * fz;
            const T gz = fz + e[2] * fx + e[5] * fy + e[8] * fz;
            fx = gx;
            fy = gy;
            fz = gz;
        }
        else
        {
            acc.w[0] += fx * dx;
            acc.w[4] += fy * dy;
            acc.w[8] += fz * dz;
            acc.w[1] += fx * dy;
            acc.w[2] += fx * dz;
            acc.w[5] += fy * dz;
        }
        atomicAdd(forces + 3LL * i, fx);
        atomicAdd(forces + 3LL * i + 1, fy);
        atomicAdd(forces + 3LL * i + 2, fz);
        atomicAdd(forces + 3LL * j, -fx);
        atomicAdd(forces + 3LL * j + 1, -fy);
        atomicAdd(forces + 3LL * j + 2, -fz);
        if (kParameterGrads)
        {
            const double de = 4.0 * (double(p6) * p6 - p6) - 4.0 * (double(pc6) * pc6 - pc6);
            const double ds = 24.0 * double(eps) / double(s) *
                              (2.0 * double(p6) * p6 - p6 - 2.0 * double(pc6) * pc6 + pc6);
            atomicAdd(row_grads + row, ds);
            atomicAdd(row_grads + rows + row, de);
        }
    }
    // Block totals in float64: warp shuffles, then one warp over the per-warp sums. Without a
    // strain only the upper triangle was accumulated; the lower one mirrors it.
    if (!kStrained)
    {
        acc.w[3] = acc.w[1];
        acc.w[6] = acc.w[2];
        acc.w[7] = acc.w[5];
    }
    __shared__ double partial[10][kLJThreads / kWarp];
    const int lane = threadIdx.x % kWarp, warp = threadIdx.x / kWarp;
    double values[10];
    values[0] = double(acc.energy);
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        values[k + 1] = double(acc.w[k]);
    }
#pragma unroll
    for (int k = 0; k < 10; ++k)
    {
        values[k] = warp_sum(values[k]);
        if (lane == 0)
        {
            partial[k][warp] = values[k];
        }
    }
    __syncthreads();
    if (warp == 0)
    {
#pragma unroll
        for (int k = 0; k < 10; ++k)
        {
            double v = lane < kLJThreads / kWarp ? partial[k][lane] : 0.0;
            v = warp_sum(v);
            if (lane == 0)
            {
                atomicAdd(k == 0 ? energy : virial + (k - 1), v);
            }
        }
    }
    if (kParameterGrads)
    {
        __syncthreads();
        for (int k = threadIdx.x; k < rows; k += blockDim.x)
        {
            atomicAdd(sigma_grad + k, row_grads[k]);
            atomicAdd(epsilon_grad + k, row_grads[rows + k]);
        }
    }
}

template <typename T>
int lj_pairs(const nd_lj_pairs_args* a, cudaStream_t stream)
{
    const std::int64_t n = a->num_atoms;
    ND_CUDA_TRY(cudaMemsetAsync(a->forces, 0, sizeof(T) * 3 * n, stream));
    ND_CUDA_TRY(cudaMemsetAsync(a->energy, 0, sizeof(double), stream));
    ND_CUDA_TRY(cudaMemsetAsync(a->virial, 0, sizeof(double) * 9, stream));
    const int rows = a->num_types * (a->num_types + 1) / 2;
    const bool grads = a->sigma_grad != nullptr;
    if (grads)
    {
        ND_CUDA_TRY(cudaMemsetAsync(a->sigma_grad, 0, sizeof(double) * rows, stream));
        ND_CUDA_TRY(cudaMemsetAsync(a->epsilon_grad, 0, sizeof(double) * rows, stream));
    }
    int device = 0, sms = 148;
    ND_CUDA_TRY(cudaGetDevice(&device));
    ND_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const std::int64_t wanted = (a->capacity + kLJThreads - 1) / kLJThreads;
    const std::int64_t most = static_cast<std::int64_t>(sms) * 8;
    const auto blocks = static_cast<unsigned>(wanted < most ? (wanted > 0 ? wanted : 1) : most);
    const T rc = static_cast<T>(a->cutoff);
    const auto* types = a->num_types > 1 ? a->atom_types : nullptr;
    const auto* strain = static_cast<const T*>(a->strain);
#define ND_LJ_LAUNCH(GRADS, STRAINED)                                                         \
    lj_pairs_kernel<T, GRADS, STRAINED><<<blocks, kLJThreads, 0, stream>>>(                  \
        static_cast<const T*>(a->positions), static_cast<const T*>(a->cell), a->pairs,       \
        a->capacity, static_cast<index_t>(a->num_atoms), types, a->num_types, static_cast<const T*>(a->sigma),                   \
        static_cast<const T*>(a->epsilon), strain, rc * rc, a->energy,                        \
        static_cast<T*>(a->forces), a->virial, a->sigma_grad, a->epsilon_grad)
    if (grads)
    {
        if (strain)
        {
            ND_LJ_LAUNCH(true, true);
        }
        else
        {
            ND_LJ_LAUNCH(true, false);
        }
    }
    else
    {
        if (strain)
        {
            ND_LJ_LAUNCH(false, true);
        }
        else
        {
            ND_LJ_LAUNCH(false, false);
        }
    }
#undef ND_LJ_LAUNCH
    ND_LAUNCH_CHECK();
    return ND_OK;
}

// The parameter backward of a batch: given the loss's gradients with respect to each frame's
// energy, forces and virial, accumulates dLoss/dsigma and dLoss/depsilon per type-pair row.
// For a valid column with d = x_i - x_j and f_s = 24 eps (2 p6^2 - p6) / r^2 (so F_i = f_s d,
// F_j = -f_s d, W = f_s d (x) d), the pair adds
//     g_E du/dtheta + (d . (g_F[i] - g_F[j]) + d^T g_W d) df_s/dtheta,
// with du/deps = 4 (p6^2 - p6) - 4 (pc6^2 - pc6), du/dsigma = 24 eps / sigma (2 p6^2 - p6 -
// 2 pc6^2 + pc6), df_s/deps = f_s / eps and df_s/dsigma = 144 eps p6 (4 p6 - 1) / (sigma r^2).
// This is the double backward the reference takes through torch.func
// (src/nabladyn/training/_fit.py:245-271), written out. Per-row sums are float64.
template <typename T>
__global__ void __launch_bounds__(kLJThreads) lj_parameter_backward_kernel(
    const T* __restrict__ positions,
    const T* __restrict__ cell,
    const index_t* __restrict__ pairs,
    std::int64_t capacity,
    index_t num_atoms,
    const index_t* __restrict__ atom_types,
    int num_types,
    const T* __restrict__ sigma,
    const T* __restrict__ epsilon,
    T cutoff_squared,
    const double* __restrict__ energy_grad,
    const T* __restrict__ forces_grad,
    const double* __restrict__ virial_grad,
    double* __restrict__ sigma_grad,
    double* __restrict__ epsilon_grad
)
{
    const std::int64_t frame = blockIdx.y;
    positions += frame * 3 * num_atoms;
    cell += frame * 3;
    pairs += frame * 2 * capacity;
    forces_grad += frame * 3 * num_atoms;
    const double ge = energy_grad[frame];
    double gw[9];
#pragma unroll
    for (int k = 0; k < 9; ++k)
    {
        gw[k] = virial_grad[frame * 9 + k];
    }
    const int rows = num_types * (num_types + 1) / 2;
    __shared__ double row_grads[2 * kMaxRows];
    for (int k = threadIdx.x; k < 2 * rows; k += blockDim.x)
    {
        row_grads[k] = 0.0;
    }
    __syncthreads();
    const T lx = cell[0], ly = cell[1], lz = cell[2];
    const std::int64_t stride = static_cast<std::int64_t>(gridDim.x) * blockDim.x;
    for (std::int64_t column = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
         column < capacity; column += stride)
    {
        const index_t i = pairs[column];
        const index_t j = pairs[capacity + column];
        if (i == j || static_cast<unsigned>(i) >= static_cast<unsigned>(num_atoms) ||
            static_cast<unsigned>(j) >= static_cast<unsigned>(num_atoms))
        {
            continue;
        }
        const T dx = displacement(positions[3LL * i], positions[3LL * j], lx);
        const T dy = displacement(positions[3LL * i + 1], positions[3LL * j + 1], ly);
        const T dz = displacement(positions[3LL * i + 2], positions[3LL * j + 2], lz);
        const T r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < cutoff_squared))
        {
            continue;
        }
        const int row = atom_types == nullptr ? 0 : pair_row(atom_types[i], atom_types[j], num_types);
        const double s = sigma[row];
        const double eps = epsilon[row];
        const double inv_r2 = 1.0 / double(r2);
        const double q = s * s * inv_r2;
        const double p6 = q * q * q;
        const double qc = s * s / double(cutoff_squared);
        const double pc6 = qc * qc * qc;
        const double fs = 24.0 * eps * (2.0 * p6 * p6 - p6) * inv_r2;
        const double x = dx, y = dy, z = dz;
        const double dgx = double(forces_grad[3LL * i]) - double(forces_grad[3LL * j]);
        const double dgy = double(forces_grad[3LL * i + 1]) - double(forces_grad[3LL * j + 1]);
        const double dgz = double(forces_grad[3LL * i + 2]) - double(forces_grad[3LL * j + 2]);
        const double g = x * dgx + y * dgy + z * dgz +
                         x * (gw[0] * x + gw[1] * y + gw[2] * z) +
                         y * (gw[3] * x + gw[4] * y + gw[5] * z) +
                         z * (gw[6] * x + gw[7] * y + gw[8] * z);
        const double du_deps = 4.0 * (p6 * p6 - p6) - 4.0 * (pc6 * pc6 - pc6);
        const double du_dsigma = 24.0 * eps / s * (2.0 * p6 * p6 - p6 - 2.0 * pc6 * pc6 + pc6);
        const double dfs_deps = fs / eps;
        const double dfs_dsigma = 144.0 * eps * p6 * (4.0 * p6 - 1.0) * inv_r2 / s;
        atomicAdd(row_grads + row, ge * du_dsigma + g * dfs_dsigma);
        atomicAdd(row_grads + rows + row, ge * du_deps + g * dfs_deps);
    }
    __syncthreads();
    for (int k = threadIdx.x; k < rows; k += blockDim.x)
    {
        atomicAdd(sigma_grad + k, row_grads[k]);
        atomicAdd(epsilon_grad + k, row_grads[rows + k]);
    }
}

unsigned pair_blocks(std::int64_t capacity, std::int64_t frames)
{
    int device = 0, sms = 148;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const std::int64_t wanted = (capacity + kLJThreads - 1) / kLJThreads;
    std::int64_t most = static_cast<std::int64_t>(sms) * 8 / (frames > 0 ? frames : 1);
    most = most < 1 ? 1 : most;
    return static_cast<unsigned>(wanted < most ? (wanted > 0 ? wanted : 1) : most);
}

template <typename T>
int lj_batch_forward(const nd_lj_batch_args* a, cudaStream_t stream)
{
    const std::int64_t n = a->num_atoms, frames = a->frames;
    ND_CUDA_TRY(cudaMemsetAsync(a->forces, 0, sizeof(T) * 3 * n * frames, stream));
    ND_CUDA_TRY(cudaMemsetAsync(a->energy, 0, sizeof(double) * frames, stream));
    ND_CUDA_TRY(cudaMemsetAsync(a->virial, 0, sizeof(double) * 9 * frames, stream));
    const T rc = static_cast<T>(a->cutoff);
    const auto* types = a->num_types > 1 ? a->atom_types : nullptr;
    const dim3 grid(pair_blocks(a->capacity, frames), static_cast<unsigned>(frames));
    lj_pairs_kernel<T, false, false><<<grid, kLJThreads, 0, stream>>>(
        static_cast<const T*>(a->positions), static_cast<const T*>(a->cells), a->pairs,
        a->capacity, static_cast<index_t>(n), types, a->num_types,
        static_cast<const T*>(a->sigma), static_cast<const T*>(a->epsilon), nullptr, rc * rc,
        a->energy, static_cast<T*>(a->forces), a->virial, nullptr, nullptr);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

template <typename T>
int lj_batch_parameter_backward(const nd_lj_batch_args* a, cudaStream_t stream)
{
    const int rows = a->num_types * (a->num_types + 1) / 2;
    ND_CUDA_TRY(cudaMemsetAsync(a->sigma_grad, 0, sizeof(double) * rows, stream));
    ND_CUDA_TRY(cudaMemsetAsync(a->epsilon_grad, 0, sizeof(double) * rows, stream));
    const T rc = static_cast<T>(a->cutoff);
    const auto* types = a->num_types > 1 ? a->atom_types : nullptr;
    const dim3 grid(pair_blocks(a->capacity, a->frames), static_cast<unsigned>(a->frames));
    lj_parameter_backward_kernel<T><<<grid, kLJThreads, 0, stream>>>(
        static_cast<const T*>(a->positions), static_cast<const T*>(a->cells), a->pairs,
        a->capacity, static_cast<index_t>(a->num_atoms), types, a->num_types,
        static_cast<const T*>(a->sigma), static_cast<const T*>(a->epsilon), rc * rc,
        a->energy_grad, static_cast<const T*>(a->forces_grad), a->virial_grad, a->sigma_grad,
        a->epsilon_grad);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

int check_batch(const nd_lj_batch_args* a, bool backward)
{
    ND_REQUIRE(a != nullptr, "the arguments are null");
    ND_REQUIRE(a->dtype == ND_FLOAT32 || a->dtype == ND_FLOAT64, "positions must be float32 or float64");
    ND_REQUIRE(a->frames >= 1 && a->frames <= 65535, "1 to 65535 frames per batch");
    ND_REQUIRE(a->num_atoms >= 1 && a->num_atoms <= INT32_MAX, "N must be in [1, 2**31)");
    ND_REQUIRE(a->capacity >= 1 && a->capacity <= INT32_MAX, "pairs must be [F, 2, C]");
    ND_REQUIRE(a->num_types >= 1 && a->num_types <= 8, "1 to 8 atom types are supported");
    ND_REQUIRE(a->num_types == 1 || a->atom_types != nullptr, "atom_types is null");
    ND_REQUIRE(a->cutoff > 0, "the cutoff must be positive");
    ND_REQUIRE(a->positions && a->cells && a->pairs && a->sigma && a->epsilon,
               "a required pointer is null");
    if (backward)
    {
        ND_REQUIRE(a->energy_grad && a->forces_grad && a->virial_grad && a->sigma_grad &&
                       a->epsilon_grad,
                   "a gradient pointer is null");
    }
    else
    {
        ND_REQUIRE(a->energy && a->forces && a->virial, "an output pointer is null");
    }
    return ND_OK;
}

}  // namespace nd

extern "C" int nd_lj_batch_forward(const nd_lj_batch_args* args, nd_stream_t stream)
{
    const int rc = nd::check_batch(args, false);
    if (rc != ND_OK)
    {
        return rc;
    }
    auto s = static_cast<cudaStream_t>(stream);
    return args->dtype == ND_FLOAT32 ? nd::lj_batch_forward<float>(args, s)
                                     : nd::lj_batch_forward<double>(args, s);
}

extern "C" int nd_lj_batch_parameter_backward(const nd_lj_batch_args* args, nd_stream_t stream)
{
    const int rc = nd::check_batch(args, true);
    if (rc != ND_OK)
    {
        return rc;
    }
    auto s = static_cast<cudaStream_t>(stream);
    return args->dtype == ND_FLOAT32 ? nd::lj_batch_parameter_backward<float>(args, s)
                                     : nd::lj_batch_parameter_backward<double>(args, s);
}

extern "C" int nd_lj_energy_force_virial(const nd_lj_pairs_args* args, nd_stream_t stream)
{
    ND_REQUIRE(args != nullptr, "the arguments are null");
    ND_REQUIRE(args->dtype == ND_FLOAT32 || args->dtype == ND_FLOAT64,
               "positions must be float32 or float64");
    ND_REQUIRE(args->num_atoms >= 1 && args->num_atoms <= INT32_MAX, "N must be in [1, 2**31)");
    ND_REQUIRE(args->capacity >= 1 && args->capacity <= INT32_MAX, "pairs must be [2, C]");
    ND_REQUIRE(args->num_types >= 1 && args->num_types <= 8, "1 to 8 atom types are supported");
    ND_REQUIRE(args->num_types == 1 || args->atom_types != nullptr, "atom_types is null");
    ND_REQUIRE(args->cutoff > 0, "the cutoff must be positive");
    ND_REQUIRE(args->positions && args->cell && args->pairs && args->sigma && args->epsilon &&
                   args->energy && args->forces && args->virial,
               "a required pointer is null");
    ND_REQUIRE((args->sigma_grad == nullptr) == (args->epsilon_grad == nullptr),
               "sigma_grad and epsilon_grad come together");
    auto s = static_cast<cudaStream_t>(stream);
    return args->dtype == ND_FLOAT32 ? nd::lj_pairs<float>(args, s) : nd::lj_pairs<double>(args, s);
}
