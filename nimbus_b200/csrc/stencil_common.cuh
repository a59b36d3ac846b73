// Shared device helpers for the C-grid hot-path kernels (sm_100a).
//
// Layout: [nx][ny][nz] float, k fastest; cell (i,j,k) at (i*ny + j)*nz + k.
// Every kernel here is a bandwidth-bound stencil (no tensor-core work), so
// the design points are coalesced k-contiguous access, grids sized in
// multiples of the SM count, and as few passes over HBM as the method's
// dependencies allow.
#pragma once

#include <cstdint>
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

}  // namespace nimbus
