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
};

struct Dims
{
    int nx, ny, nz;
    __host__ __device__ __forceinline__ int cells() const { return nx * ny * nz; }
    __host__ __device__ __forceinline__ int at(int i, int j, int k) const { return (i * ny + j) * nz + k; }
    __host__ __device__ __forceinline__ int sx() const { return ny * nz; }  // stride of i
    __host__ __device__ __forceinline__ int sy() const { return nz; }       // stride of j
};

__device__ __forceinline__ void decompose(const Dims& d, int c, int& i, int& j, int& k)
{
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
