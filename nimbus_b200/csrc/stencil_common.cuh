// Shared device helpers for the C-grid hot-path kernels (sm_100a).
//
// Layout: [nx][ny][nz] float, k fastest; cell (i,j,k) at (i*ny + j)*nz + k.
// Every kernel here is a bandwidth-bound stencil (no tensor-core work), so
// the design points are coalesced k-contiguous access, grids sized in
// multiples of the SM count, and as few passes over HBM as the method's
// dependencies allow.
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>
#include <cuda_runtime.h>

namespace nimbus
{

// Physical constants: include/core/infra/physical_constants.hpp:15-34.
constexpr double kRd = 287.0;
constexpr double kCpd = 1004.0;
constexpr double kP00 = 100000.0;
// KW78 phase speed: boundary_conditions_cartesian_cgrid.cpp:266.
constexpr float kCStar = 30.0f;

enum : int
{
    kBcPeriodic = 0,
    kBcRadiative = 1,
    kBcRigid = 2,
    kBcRigidSlip = 3,
    kBcZeroGradient = 4,
};
enum : int
{
    kBottomNoSlip = 0,
    kBottomSlip = 1,
};
enum : int
{
    kTopRigid = 0,
    kTopSponge = 1,
    kTopOpen = 2,
};

// Device status word bits (OR-accumulated; read and cleared by the host).
enum : unsigned
{
    kStatusNonfiniteMassFlux = 1u << 0,
    kStatusNonfiniteTransport = 1u << 1,
    kStatusInvalidEos = 1u << 2,
    kStatusSgsInvalid = 1u << 3,
    kStatusInvalidState = 1u << 4,  // a pressure or density failed the CFL scan (non-finite or <= 0)
    kStatusStagingTimeout = 1u << 5,  // a bulk-staged tile's copies did not complete (the step is void)
};

struct Dims
{
    int nx, ny, nz;
    // Division by nz and ny as (x * magic) >> 32 with magic = ceil(2^32 / d)
    // = (2^32 + e) / d: floor(x*magic / 2^32) = floor(x / d) whenever
    // x * e < 2^32, since the excess x*e/(d*2^32) then stays below 1/d.
    // make_dims() checks that bound for the largest dividend and leaves the
    // magic at 0 (plain division) when it does not hold.
    unsigned nz_magic = 0, ny_magic = 0;
    __host__ __device__ __forceinline__ int cells() const { return nx * ny * nz; }
    __host__ __device__ __forceinline__ int at(int i, int j, int k) const { return (i * ny + j) * nz + k; }
    __host__ __device__ __forceinline__ int sx() const { return ny * nz; }  // stride of i
    __host__ __device__ __forceinline__ int sy() const { return nz; }       // stride of j
};

__host__ __device__ __forceinline__ unsigned div_magic(unsigned d)
{
    return (unsigned)((0x100000000ull + d - 1) / d);
}

// Magic for dividing every x <= x_max by d, or 0 if the bound fails.
__host__ __device__ __forceinline__ unsigned checked_magic(unsigned d, unsigned long long x_max)
{
    if (d == 0) return 0;
    const unsigned m = div_magic(d);
    const unsigned long long e = (unsigned long long)m * d - 0x100000000ull;
    return (x_max * e < 0x100000000ull) ? m : 0u;
}

__host__ __device__ __forceinline__ Dims make_dims(int nx, int ny, int nz)
{
    Dims d;
    d.nx = nx;
    d.ny = ny;
    d.nz = nz;
    const unsigned long long cells = (unsigned long long)nx * ny * nz;
    d.nz_magic = checked_magic((unsigned)nz, cells);
    d.ny_magic = checked_magic((unsigned)ny, (unsigned long long)nx * ny);
    if (d.nz_magic == 0 || d.ny_magic == 0) d.nz_magic = d.ny_magic = 0;
    return d;
}

__device__ __forceinline__ void decompose(const Dims& d, int c, int& i, int& j, int& k)
{
    if (d.nz_magic != 0)
    {
        const int t = (int)__umulhi((unsigned)c, d.nz_magic);
        k = c - t * d.nz;
        i = (int)__umulhi((unsigned)t, d.ny_magic);
        j = t - i * d.ny;
        return;
    }
    k = c % d.nz;
    const int t = c / d.nz;
    j = t % d.ny;
    i = t / d.ny;
}

__device__ __forceinline__ double finite_or_zero(double v) { return isfinite(v) ? v : 0.0; }
__device__ __forceinline__ double safe_rho(double v) { return (isfinite(v) && v > 1.0e-6) ? v : 1.0; }

// std::clamp after a non-finite fallback (acoustic_cgrid_fast.cpp:38-43).
__device__ __forceinline__ float clamp_value(float v, float fallback, float lo, float hi)
{
    if (!isfinite(v)) v = fallback;
    return v < lo ? lo : (hi < v ? hi : v);
}

// ---- Acoustic speed scan ------------------------------------------------
// Before every large step the reference samples c_max = max sqrt(gamma p / rho)
// over the state (the flat Cartesian CFL scan, src/numerics/runtime.cpp:346-401,
// the product formed as (gamma * p) / rho in FP64) and derives the substep
// count from it.  sqrt is monotone and correctly rounded, so the maximum of
// (gamma p) / rho followed by one sqrt is that maximum exactly; a
// non-negative double's bits order like its value, so the maximum is an
// integer atomicMax.

// (gamma p) / rho of one cell as ordered double bits; 0 and an invalid-state
// flag where p or rho is non-finite or non-positive (where the reference throws).
__device__ __forceinline__ unsigned long long sound_speed_sq_bits(double gamma, float p, float rho, unsigned& flags)
{
    const double ph = (double)p, rh = (double)rho;
    if (!(isfinite(ph) && ph > 0.0 && isfinite(rh) && rh > 0.0))
    {
        flags |= kStatusInvalidState;
        return 0ull;
    }
    return (unsigned long long)__double_as_longlong(gamma * ph / rh);
}

// Maximum of v over the block, valid in thread 0.  Every thread of the block
// calls it (it synchronises the block).
__device__ __forceinline__ unsigned long long block_max_u64(unsigned long long v)
{
    __shared__ unsigned long long part[32];
    for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    __syncthreads();  // an earlier call may still read part[]
    if (lane == 0) part[warp] = v;
    __syncthreads();
    if (warp == 0)
    {
        const int warps = (blockDim.x + 31) >> 5;
        v = lane < warps ? part[lane] : 0ull;
        for (int o = 16; o > 0; o >>= 1) v = max(v, __shfl_xor_sync(0xffffffffu, v, o));
    }
    return v;
}

// Grid-stride scan of one field pair: the maximum into *out (atomicMax of
// the ordered bits), invalid cells into *status.
static __global__ void __launch_bounds__(256) max_sound_speed_kernel(const float* __restrict__ p,
                                                                     const float* __restrict__ rho, long long n,
                                                                     double gamma, unsigned long long* out,
                                                                     unsigned* status)
{
    unsigned long long best = 0;
    unsigned flags = 0;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
        best = max(best, sound_speed_sq_bits(gamma, p[c], rho[c], flags));
    best = block_max_u64(best);
    if (threadIdx.x == 0 && best) atomicMax(out, best);
    if (flags) atomicOr(status, flags);
}

}  // namespace nimbus

namespace nimbus_host
{
// SplitExplicitScheme::resolve_substep_count
// (src/numerics/time_stepping/schemes/split_explicit/split_explicit.cpp:67-170)
// with a positive minimum spacing: N = max(requested, max(ceil(dt c_max /
// (0.5 min_spacing)) + 1, 2)), requested <= 0 meaning the CFL rule alone;
// -1 where the reference throws.
inline int resolve_substep_count(double dt_large, double c_max, double min_spacing, int requested)
{
    if (!(dt_large > 0.0) || !std::isfinite(dt_large)) return -1;
    if (!(c_max > 0.0) || !std::isfinite(c_max)) return -1;
    if (!(min_spacing > 0.0) || !std::isfinite(min_spacing)) return -1;
    const double required_real = dt_large * c_max / (0.5 * min_spacing);
    if (!std::isfinite(required_real) || required_real >= 2147483646.0) return -1;
    int required = static_cast<int>(std::ceil(required_real)) + 1;
    if (required < 2) required = 2;
    return requested > 0 ? (requested > required ? requested : required) : required;
}

// Largest sqrt(gamma p0 / rho0) of the base columns (runtime.cpp:854-870).
inline double base_sound_speed(const double* p0, const double* rho0, int nz, double gamma)
{
    double best = 0.0;
    for (int k = 0; k < nz; ++k)
    {
        const double s = std::sqrt(gamma * p0[k] / rho0[k]);
        if (best < s) best = s;
    }
    return best;
}

inline double ordered_bits_to_double(unsigned long long b)
{
    double x;
    std::memcpy(&x, &b, sizeof x);
    return x;
}
}  // namespace nimbus_host
