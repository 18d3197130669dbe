// Velocity Verlet and the Nose-Hoover chain for a frame kept in the caller's order, whatever
// potential gives the forces: the integrator of the pair engine (models other than
// Lennard-Jones, whose engine in md.cu fuses these steps into its own kernels).
//
// A step is, as src/nabladyn/md/_simulation.py:331-348 orders the ensemble halves
// (src/nabladyn/md/_ensembles/_nve.py:39-58, _nvt.py:88-129):
//   open   NVT: the chain's opening half step against the carried K; then every atom
//          v = s v + dt/2 F/m, x = wrap(x + dt v) with its image count, the non-finite check;
//   (the caller's neighbor update and forces)
//   close  v += dt/2 F/m with per-block float64 sums of m v^2, then one block sums them in a
//          fixed order into K and, for NVT, runs the closing half step; its factor stays
//          pending and the next open (or a frame read) applies it.
// The thermostat block has the layout of the MD engine's (enum Thermo in md_common.cuh).
//
// NPT (src/nabladyn/md/_ensembles/_npt.py:66-251, isotropic MTK with chains on the particles
// and on the barostat, Tuckerman et al. 2006 operator order) adds, all in float64 on the GPU:
//   open   the barostat's chain half step against p_eps^2 / 2M, the particles' chain,
//          p_eps += dt/2 G with G = alpha 2K + tr W - 3 P V, then the drag exp(-alpha v_eps
//          dt/2) folded into the velocity scale, the half kick, and the drift with box and
//          positions grown by exp(v_eps dt/2) before and after it: x = (x g + dt v) g, L *= g^2;
//   close  v = (v + dt/2 F/m) drag with K in float64, p_eps += dt/2 G, the particles' chain
//          (its factor pending, as for NVT), the barostat's chain.

#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "md_common.cuh"

namespace nd {
namespace {

constexpr int kIntegrateThreads = 256;
constexpr int kCloseThreads = 1024;

// Integration modes (the `mode` argument of the entry points).
constexpr int kNVE = 0, kNVT = 1, kNPT = 2;

// Offsets into the float64 barostat block (nd_integrator.barostat).
enum Barostat : int
{
    kBoxMomentum = 0,    // p_eps
    kBoxChain = 1,       // q[3], p[3] of the barostat's chain
    kBoxChainMass = 7,   // its masses [3]
    kBoxMass = 10,       // M = 3 (N + 1) kT tau_b^2
    kPressure = 11,      // P in kJ/mol/nm^3
    kAlpha = 12,         // 1 + 1/N
    kMasterCell = 13,    // the cell [3], float64
    kDrag = 16,          // exp(-alpha v_eps dt/2) of this step
    kGrowth = 17,        // exp(v_eps dt/2) of this step
    kBarostatSize = 32,
};

template <typename T>
struct Frame
{
    std::int64_t n;
    T* x;
    T* v;
    const T* f;
    const T* m;
    std::int64_t* images;
    T* cell;
    double* thermo;
    double* box;
    const double* virial;
    double* partials;
    double* totals;
    index_t* status;
    T dt;
};

template <typename T>
Frame<T> frame_of(const nd_integrator& s)
{
    return Frame<T>{s.num_atoms,
                    static_cast<T*>(s.positions),
                    static_cast<T*>(s.velocities),
                    static_cast<const T*>(s.forces),
                    static_cast<const T*>(s.masses),
                    s.images,
                    static_cast<T*>(s.cell),
                    s.thermostat,
                    s.barostat,
                    s.virial,
                    s.partials,
                    s.totals,
                    s.status,
                    static_cast<T>(s.timestep)};
}

__global__ void open_chain_kernel(double* thermo)
{
    double kinetic = thermo[kKineticA];
    double q[3], p[3];
    for (int k = 0; k < 3; ++k)
    {
        q[k] = thermo[kChainA + k];
        p[k] = thermo[kChainA + 3 + k];
    }
    const double factor = chain_half_step(kinetic, q, p, thermo + kChainMass, thermo[kDegrees],
                                          thermo[kThermalEnergy], thermo[kTimestep]);
    for (int k = 0; k < 3; ++k)
    {
        thermo[kChainB + k] = q[k];
        thermo[kChainB + 3 + k] = p[k];
    }
    thermo[kKineticB] = kinetic;
    thermo[kOpenScale] = thermo[kPendingScale] * factor;
    thermo[kPendingScale] = 1.0;
}

// The barostat's chain (one degree of freedom) by half a step against p_eps^2 / 2M; scales
// p_eps.
__device__ inline void box_chain_half_step(double* box, const double* thermo)
{
    double kinetic = box[kBoxMomentum] * box[kBoxMomentum] / (2.0 * box[kBoxMass]);
    const double factor = chain_half_step(kinetic, box + kBoxChain, box + kBoxChain + 3,
                                          box + kBoxChainMass, 1.0, thermo[kThermalEnergy],
                                          thermo[kTimestep]);
    box[kBoxMomentum] *= factor;
}

// G = alpha 2K + tr W - 3 P V, with the master cell's volume.
__device__ inline double box_force(const double* box, const double* virial, double kinetic)
{
    const double volume = box[kMasterCell] * box[kMasterCell + 1] * box[kMasterCell + 2];
    return box[kAlpha] * 2.0 * kinetic + (virial[0] + virial[4] + virial[8]) -
           3.0 * box[kPressure] * volume;
}

template <typename T>
__global__ void open_npt_kernel(Frame<T> s)
{
    double* thermo = s.thermo;
    double* box = s.box;
    const double dt = thermo[kTimestep];
    box_chain_half_step(box, thermo);
    double kinetic = thermo[kKineticA];
    double q[3], p[3];
    for (int k = 0; k < 3; ++k)
    {
        q[k] = thermo[kChainA + k];
        p[k] = thermo[kChainA + 3 + k];
    }
    const double factor = chain_half_step(kinetic, q, p, thermo + kChainMass, thermo[kDegrees],
                                          thermo[kThermalEnergy], dt);
    for (int k = 0; k < 3; ++k)
    {
        thermo[kChainB + k] = q[k];
        thermo[kChainB + 3 + k] = p[k];
    }
    thermo[kKineticB] = kinetic;
    box[kBoxMomentum] += 0.5 * dt * box_force(box, s.virial, kinetic);
    const double rate = box[kBoxMomentum] / box[kBoxMass];
    const double drag = exp(-box[kAlpha] * rate * 0.5 * dt);
    const double growth = exp(rate * 0.5 * dt);
    box[kDrag] = drag;
    box[kGrowth] = growth;
    // The chain's scale for the drift (the pending closing factor and this opening factor);
    // the drag follows it there, then the kick.
    thermo[kOpenScale] = thermo[kPendingScale] * factor;
    thermo[kPendingScale] = 1.0;
    for (int axis = 0; axis < 3; ++axis)
    {
        box[kMasterCell + axis] = box[kMasterCell + axis] * growth * growth;
        s.cell[axis] = static_cast<T>(box[kMasterCell + axis]);
    }
}

// x - floor(x / L) L with the two fix-ups of src/nabladyn/space.py:22-38, and the crossings.
template <typename T>
__device__ __forceinline__ T wrap_coordinate(T x, T length, std::int64_t& crossings)
{
    T c = floor(x / length);
    T w = x - c * length;
    if (w < T(0))
    {
        w += length;
        c -= T(1);
    }
    if (w >= length)
    {
        w -= length;
        c += T(1);
    }
    crossings += static_cast<std::int64_t>(c);
    return w;
}

template <typename T, bool kThermostat>
__global__ void __launch_bounds__(kIntegrateThreads) drift_kernel(Frame<T> s)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= s.n)
    {
        return;
    }
    const T scale = kThermostat ? static_cast<T>(s.thermo[kOpenScale]) : T(1);
    const T kick = T(0.5) * s.dt / s.m[i];
    bool finite = true;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis)
    {
        const std::int64_t k = 3 * i + axis;
        const T v = scale * s.v[k] + kick * s.f[k];
        const T moved = s.x[k] + s.dt * v;
        finite = finite && isfinite(moved);
        std::int64_t crossings = s.images[k];
        const T wrapped = finite ? wrap_coordinate(moved, s.cell[axis], crossings) : moved;
        s.v[k] = v;
        s.x[k] = wrapped;
        s.images[k] = crossings;
    }
    if (!finite)
    {
        atomicOr(s.status, kNonFinite);
    }
}

// NPT drift: v = (f s v) d + dt/2 F/m, x = (x g + dt v) g, wrapped into the grown cell.
template <typename T>
__global__ void __launch_bounds__(kIntegrateThreads) drift_npt_kernel(Frame<T> s)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= s.n)
    {
        return;
    }
    const T scale = static_cast<T>(s.thermo[kOpenScale]);
    const T growth = static_cast<T>(s.box[kGrowth]);
    const T drag = static_cast<T>(s.box[kDrag]);
    const T kick = T(0.5) * s.dt / s.m[i];
    bool finite = true;
#pragma unroll
    for (int axis = 0; axis < 3; ++axis)
    {
        const std::int64_t k = 3 * i + axis;
        const T v = (scale * s.v[k]) * drag + kick * s.f[k];
        const T moved = (s.x[k] * growth + s.dt * v) * growth;
        finite = finite && isfinite(moved);
        std::int64_t crossings = s.images[k];
        const T wrapped = finite ? wrap_coordinate(moved, s.cell[axis], crossings) : moved;
        s.v[k] = v;
        s.x[k] = wrapped;
        s.images[k] = crossings;
    }
    if (!finite)
    {
        atomicOr(s.status, kNonFinite);
    }
}

// v += dt/2 F/m (kick) or v scaled by the pending factor (read only); per-block sums of m v^2.
template <typename T, bool kKick, bool kScaled, bool kWithDrag = false>
__global__ void __launch_bounds__(kIntegrateThreads) kinetic_kernel(Frame<T> s)
{
    const std::int64_t i = static_cast<std::int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    double twice = 0.0;
    if (i < s.n)
    {
        const T kick = T(0.5) * s.dt / s.m[i];
        const T scale = kScaled ? static_cast<T>(s.thermo[kPendingScale]) : T(1);
        const T drag = kWithDrag ? static_cast<T>(s.box[Barostat::kDrag]) : T(1);
#pragma unroll
        for (int axis = 0; axis < 3; ++axis)
        {
            const std::int64_t k = 3 * i + axis;
            T v = s.v[k];
            if (kKick)
            {
                v += kick * s.f[k];
                if (kWithDrag)
                {
                    v *= drag;
                }
                s.v[k] = v;
            }
            v *= scale;
            twice += static_cast<double>(s.m[i]) * static_cast<double>(v) * static_cast<double>(v);
        }
    }
    __shared__ double warps[kIntegrateThreads / kWarp];
    twice = warp_sum(twice);
    if (threadIdx.x % kWarp == 0)
    {
        warps[threadIdx.x / kWarp] = twice;
    }
    __syncthreads();
    if (threadIdx.x == 0)
    {
        double block = 0.0;
        for (int w = 0; w < kIntegrateThreads / kWarp; ++w)
        {
            block += warps[w];
        }
        s.partials[blockIdx.x] = block;
    }
}

// K = sum / 2 in a fixed order into totals[slot]; for a step's close with NVT, the closing
// half step of the chain.
template <bool kChain>
__global__ void __launch_bounds__(kCloseThreads) close_kernel(const double* partials, int blocks,
                                                              double* totals, int slot,
                                                              double* thermo)
{
    __shared__ double warps[kCloseThreads / kWarp];
    double mine = 0.0;
    for (int b = threadIdx.x; b < blocks; b += kCloseThreads)
    {
        mine += partials[b];
    }
    mine = warp_sum(mine);
    if (threadIdx.x % kWarp == 0)
    {
        warps[threadIdx.x / kWarp] = mine;
    }
    __syncthreads();
    if (threadIdx.x >= kWarp)
    {
        return;
    }
    const double total = warp_sum(warps[threadIdx.x]);
    if (threadIdx.x != 0)
    {
        return;
    }
    double kinetic = 0.5 * total;
    totals[slot] = kinetic;
    if (kChain)
    {
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

// The NPT close: K in a fixed order, p_eps += dt/2 G, the particles' closing half step (its
// factor pending), the barostat's chain.
__global__ void __launch_bounds__(kCloseThreads) close_npt_kernel(const double* partials,
                                                                  int blocks, double* totals,
                                                                  double* thermo, double* box,
                                                                  const double* virial)
{
    __shared__ double warps[kCloseThreads / kWarp];
    double mine = 0.0;
    for (int b = threadIdx.x; b < blocks; b += kCloseThreads)
    {
        mine += partials[b];
    }
    mine = warp_sum(mine);
    if (threadIdx.x % kWarp == 0)
    {
        warps[threadIdx.x / kWarp] = mine;
    }
    __syncthreads();
    if (threadIdx.x >= kWarp)
    {
        return;
    }
    const double total = warp_sum(warps[threadIdx.x]);
    if (threadIdx.x != 0)
    {
        return;
    }
    double kinetic = 0.5 * total;
    totals[1] = kinetic;
    const double dt = thermo[kTimestep];
    box[kBoxMomentum] += 0.5 * dt * box_force(box, virial, kinetic);
    double q[3], p[3];
    for (int k = 0; k < 3; ++k)
    {
        q[k] = thermo[kChainB + k];
        p[k] = thermo[kChainB + 3 + k];
    }
    const double factor = chain_half_step(kinetic, q, p, thermo + kChainMass, thermo[kDegrees],
                                          thermo[kThermalEnergy], dt);
    for (int k = 0; k < 3; ++k)
    {
        thermo[kChainA + k] = q[k];
        thermo[kChainA + 3 + k] = p[k];
    }
    thermo[kKineticA] = kinetic;
    thermo[kPendingScale] = factor;
    box_chain_half_step(box, thermo);
}

int check(const nd_integrator* s, int mode)
{
    ND_REQUIRE(s != nullptr, "integrator is null");
    ND_REQUIRE(s->dtype == ND_FLOAT32 || s->dtype == ND_FLOAT64, "dtype must be float32 or float64");
    ND_REQUIRE(s->num_atoms >= 1, "num_atoms must be positive");
    ND_REQUIRE(s->positions && s->velocities && s->forces && s->masses && s->images && s->cell &&
                   s->thermostat && s->partials && s->totals && s->status,
               "a buffer of the integrator is null");
    ND_REQUIRE(mode >= kNVE && mode <= kNPT, "mode must be 0 (NVE), 1 (NVT) or 2 (NPT)");
    ND_REQUIRE(mode != kNPT || (s->barostat != nullptr && s->virial != nullptr),
               "NPT needs the barostat block and the virial");
    return ND_OK;
}

unsigned int integrate_blocks(std::int64_t n)
{
    return blocks_for(n, kIntegrateThreads);
}

template <typename T>
int open_step(const nd_integrator& s, int mode, cudaStream_t stream)
{
    const Frame<T> frame = frame_of<T>(s);
    const unsigned int blocks = integrate_blocks(s.num_atoms);
    if (mode == kNPT)
    {
        open_npt_kernel<T><<<1, 1, 0, stream>>>(frame);
        ND_LAUNCH_CHECK();
        drift_npt_kernel<T><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
    }
    else if (mode == kNVT)
    {
        open_chain_kernel<<<1, 1, 0, stream>>>(s.thermostat);
        ND_LAUNCH_CHECK();
        drift_kernel<T, true><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
    }
    else
    {
        drift_kernel<T, false><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
    }
    ND_LAUNCH_CHECK();
    return ND_OK;
}

template <typename T>
int close_step(const nd_integrator& s, int mode, cudaStream_t stream)
{
    const Frame<T> frame = frame_of<T>(s);
    const unsigned int blocks = integrate_blocks(s.num_atoms);
    if (mode == kNPT)
    {
        kinetic_kernel<T, true, false, true><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
        ND_LAUNCH_CHECK();
        close_npt_kernel<<<1, kCloseThreads, 0, stream>>>(s.partials, blocks, s.totals,
                                                          s.thermostat, s.barostat, s.virial);
    }
    else
    {
        kinetic_kernel<T, true, false><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
        ND_LAUNCH_CHECK();
        if (mode == kNVT)
        {
            close_kernel<true><<<1, kCloseThreads, 0, stream>>>(s.partials, blocks, s.totals, 1,
                                                                s.thermostat);
        }
        else
        {
            close_kernel<false><<<1, kCloseThreads, 0, stream>>>(s.partials, blocks, s.totals, 1,
                                                                 s.thermostat);
        }
    }
    ND_LAUNCH_CHECK();
    return ND_OK;
}

template <typename T>
int kinetic_now(const nd_integrator& s, int mode, cudaStream_t stream)
{
    const bool thermostat = mode != kNVE;
    const Frame<T> frame = frame_of<T>(s);
    const unsigned int blocks = integrate_blocks(s.num_atoms);
    if (thermostat)
    {
        kinetic_kernel<T, false, true><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
    }
    else
    {
        kinetic_kernel<T, false, false><<<blocks, kIntegrateThreads, 0, stream>>>(frame);
    }
    ND_LAUNCH_CHECK();
    close_kernel<false><<<1, kCloseThreads, 0, stream>>>(s.partials, blocks, s.totals, 9,
                                                         s.thermostat);
    ND_LAUNCH_CHECK();
    return ND_OK;
}

}  // namespace
}  // namespace nd

extern "C" {

int nd_integrate_partial_slots(int64_t num_atoms, int64_t* slots)
{
    ND_REQUIRE(num_atoms >= 1 && slots != nullptr, "num_atoms must be positive");
    *slots = static_cast<int64_t>(nd::integrate_blocks(num_atoms));
    return ND_OK;
}

int nd_integrate_open(const nd_integrator* s, int mode, nd_stream_t stream)
{
    if (const int rc = nd::check(s, mode); rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return s->dtype == ND_FLOAT32 ? nd::open_step<float>(*s, mode, st)
                                  : nd::open_step<double>(*s, mode, st);
}

int nd_integrate_close(const nd_integrator* s, int mode, nd_stream_t stream)
{
    if (const int rc = nd::check(s, mode); rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return s->dtype == ND_FLOAT32 ? nd::close_step<float>(*s, mode, st)
                                  : nd::close_step<double>(*s, mode, st);
}

int nd_integrate_kinetic(const nd_integrator* s, int mode, nd_stream_t stream)
{
    if (const int rc = nd::check(s, mode); rc != ND_OK)
    {
        return rc;
    }
    auto st = static_cast<cudaStream_t>(stream);
    return s->dtype == ND_FLOAT32 ? nd::kinetic_now<float>(*s, mode, st)
                                  : nd::kinetic_now<double>(*s, mode, st);
}

}  // extern "C"
