// Acoustic substep kernels of the Klemp-Wilhelmson split-explicit loop on
// the flat Cartesian C-grid, reference-precision form: FP32 storage, FP64
// interior arithmetic in the reference's own operation order.  This file is
// compiled with --fmad=false so no multiply-add is contracted, which keeps
// every stored value identical to the reference CPU solver's.
//
// One substep is two full-grid passes plus three boundary passes:
//   continuity_eos : retained mass-flux accumulation from the pre-substep
//                    state, continuity tendency, rho forward Euler + clamp,
//                    EOS pressure + clamp.  rho is written to the other half
//                    of a ping-pong pair (neighbours still need the old rho);
//                    p is written in place (the old p is never read).
//   momentum       : u,v,w forward Euler from the new pressure gradient.
//   bc_we, bc_sn, bc_vertical : the boundary closure in the reference's
//                    face order W,E -> S,N -> vertical.  Each thread owns one
//                    boundary row, so within a kernel W precedes E (and S
//                    precedes N) exactly as in the reference's sequential loops.
#pragma once

#include "stencil_common.cuh"

namespace nimbus
{

struct AcousticParams
{
    Dims d;
    double inv_dx, inv_dy, inv_dz;
    double dt_small;
    double gamma;
    float rho_min, rho_max, p_min, p_max, p_ref_fallback, wind_h, wind_v;
    // Retained mass flux (accumulated when mfx != nullptr).
    double weight;
    double frame_u, frame_v;
    int top_open;
};

// Pass 1+2 of acoustic_cgrid_fast.cpp:47-157 and the Host-precision flux
// accumulation of advection_cartesian.cpp:743-849 (cartesian_mass_flux.hpp:57-75,381-393).
static __global__ void __launch_bounds__(256) acoustic_continuity_eos_kernel(
    AcousticParams P, const float* __restrict__ rho, const float* __restrict__ u, const float* __restrict__ v,
    const float* __restrict__ w, const float* __restrict__ theta, const double* __restrict__ rho0,
    float* __restrict__ rho_out, float* __restrict__ p_out, float* __restrict__ drho_out,
    float* __restrict__ mfx, float* __restrict__ mfy, float* __restrict__ mfz, unsigned* __restrict__ status)
{
    const Dims d = P.d;
    const int n = d.cells();
    const int sx = d.sx(), sy = d.sy();
    unsigned flags = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        const double rc = (double)rho[c];

        if (mfx != nullptr)
        {
            const double weight = P.weight;
            if (i < d.nx - 1)
            {
                const double vel = (double)u[c] - P.frame_u;
                const double flux = 0.5 * (rc + (double)rho[c + sx]) * vel;
                const double next = (double)mfx[c] + weight * flux;
                const float stored = (float)next;
                if (isfinite(next) && isfinite(stored)) mfx[c] = stored;
                else flags |= kStatusNonfiniteMassFlux;
            }
            if (j < d.ny - 1)
            {
                const double vel = (double)v[c] - P.frame_v;
                const double flux = 0.5 * (rc + (double)rho[c + sy]) * vel;
                const double next = (double)mfy[c] + weight * flux;
                const float stored = (float)next;
                if (isfinite(next) && isfinite(stored)) mfy[c] = stored;
                else flags |= kStatusNonfiniteMassFlux;
            }
            double zflux;
            if (k == d.nz - 1) zflux = P.top_open ? rc * (double)w[c] : 0.0;
            else zflux = 0.5 * (rc + (double)rho[c + 1]) * (double)w[c];
            const double znext = (double)mfz[c] + weight * zflux;
            const float zstored = (float)znext;
            if (isfinite(znext) && isfinite(zstored)) mfz[c] = zstored;
            else flags |= kStatusNonfiniteMassFlux;
        }

        double drho = 0.0;
        if (i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1)
        {
            const double fx_pos = 0.5 * (rc + (double)rho[c + sx]) * (double)u[c];
            const double fx_neg = 0.5 * ((double)rho[c - sx] + rc) * (double)u[c - sx];
            const double fy_pos = 0.5 * (rc + (double)rho[c + sy]) * (double)v[c];
            const double fy_neg = 0.5 * ((double)rho[c - sy] + rc) * (double)v[c - sy];
            const double fz_pos = (k + 1 < d.nz) ? 0.5 * (rc + (double)rho[c + 1]) * (double)w[c] : rc * (double)w[c];
            const double fz_neg = (k > 0) ? 0.5 * ((double)rho[c - 1] + rc) * (double)w[c - 1] : 0.0;
            drho = -((fx_pos - fx_neg) * P.inv_dx + (fy_pos - fy_neg) * P.inv_dy + (fz_pos - fz_neg) * P.inv_dz);
        }
        const float drho_stored = (float)finite_or_zero(drho);
        if (drho_out != nullptr) drho_out[c] = drho_stored;

        double rho_new = rc + (double)drho_stored * P.dt_small;
        if (!isfinite(rho_new) || rho_new <= 0.0)
        {
            const double base = rho0[k];
            rho_new = (0.1 < base) ? base : 0.1;
        }
        const float rho_stored = clamp_value((float)rho_new, 1.0f, P.rho_min, P.rho_max);
        rho_out[c] = rho_stored;

        double p_new = (double)P.p_ref_fallback;
        const double th = (double)theta[c];
        if (th > 0.0) p_new = kP00 * pow((double)rho_stored * kRd * th / kP00, P.gamma);
        if (!isfinite(p_new) || p_new <= 0.0) p_new = (double)P.p_ref_fallback;
        p_out[c] = clamp_value((float)p_new, 101325.0f, P.p_min, P.p_max);
    }
    if (flags) atomicOr(status, flags);
}

// Pass 3 of acoustic_cgrid_fast.cpp:159-215, in place on u,v,w.
static __global__ void __launch_bounds__(256) acoustic_momentum_kernel(
    AcousticParams P, const float* __restrict__ rho, const float* __restrict__ p, const double* __restrict__ p0,
    float* __restrict__ u, float* __restrict__ v, float* __restrict__ w)
{
    const Dims d = P.d;
    const int n = d.cells();
    const int sx = d.sx(), sy = d.sy();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        float du = 0.0f, dv = 0.0f, dw = 0.0f;
        if (i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1)
        {
            const double rc = (double)rho[c];
            const double rho_x = 0.5 * (rc + (double)rho[c + sx]);
            const double rho_y = 0.5 * (rc + (double)rho[c + sy]);
            const double rho_z = 0.5 * (rc + (double)rho[c + 1]);
            const double dp0_dz = (p0[k + 1] - p0[k]) * P.inv_dz;
            const double pc = (double)p[c];
            du = (float)finite_or_zero(-((double)p[c + sx] - pc) * P.inv_dx / safe_rho(rho_x));
            dv = (float)finite_or_zero(-((double)p[c + sy] - pc) * P.inv_dy / safe_rho(rho_y));
            dw = (float)finite_or_zero(-((((double)p[c + 1] - pc) * P.inv_dz) - dp0_dz) / safe_rho(rho_z));
        }
        u[c] = clamp_value((float)((double)u[c] + (double)du * P.dt_small), 0.0f, -P.wind_h, P.wind_h);
        v[c] = clamp_value((float)((double)v[c] + (double)dv * P.dt_small), 0.0f, -P.wind_h, P.wind_h);
        w[c] = clamp_value((float)((double)w[c] + (double)dw * P.dt_small), 0.0f, -P.wind_v, P.wind_v);
    }
}

struct BoundaryParams
{
    Dims d;
    int west, east, south, north, bottom, top;
    float dt_rad;     // (float)dt_small; 0 = refresh only
    float inv_dx, inv_dy;
    float frame_u, frame_v;
};

// include/dynamics/radiative_face.hpp: four separately rounded FP32 operations.
__device__ __forceinline__ float kw78_updated_face(float previous, float phase, float gradient, float dt_rad,
                                                   float inv_spacing, bool negative_outgoing)
{
    if (negative_outgoing ? phase >= 0.0f : phase <= 0.0f) return previous;
    const float dt_phase = __fmul_rn(dt_rad, phase);
    const float tendency = __fmul_rn(dt_phase, gradient);
    const float increment = __fmul_rn(tendency, inv_spacing);
    return __fsub_rn(previous, increment);
}

// West then east faces for one (j,k) row r: boundary_conditions_cartesian_cgrid.cpp:927-1032.
__device__ __forceinline__ void bc_we_row(const BoundaryParams& B, float* __restrict__ u, float* __restrict__ v,
                                          float* __restrict__ w, float* __restrict__ rho, float* __restrict__ p,
                                          float* __restrict__ u_west, float* __restrict__ u_east, int r)
{
    const Dims d = B.d;
    const bool radiate = B.dt_rad > 0.0f;
    {
        const int j = r / d.nz, k = r % d.nz;
        // ---- West: ghost i=0, wall face u[0] ----
        {
            const int g = d.at(0, j, k), in = d.at(1, j, k);
            if (B.west == kBcPeriodic)
            {
                const int s = d.at(d.nx - 2, j, k);
                u[g] = u[s]; v[g] = v[s]; w[g] = w[s]; rho[g] = rho[s]; p[g] = p[s];
            }
            else
            {
                if (B.west == kBcRadiative)
                {
                    if (radiate)
                    {
                        const float up = u_west[r];
                        const float phase = __fsub_rn(__fsub_rn(up, B.frame_u), kCStar);
                        const float un = kw78_updated_face(up, phase, __fsub_rn(u[in], up), B.dt_rad, B.inv_dx, true);
                        u[g] = un;
                        u_west[r] = un;
                    }
                }
                else if (B.west == kBcZeroGradient) u[g] = u[in];
                else u[g] = B.frame_u;
                if (B.west == kBcRigid) { v[g] = B.frame_v; w[g] = 0.0f; }
                else { v[g] = v[in]; w[g] = w[in]; }
                rho[g] = rho[in]; p[g] = p[in];
            }
        }
        // ---- East: ghost i=nx-1, wall face u[nx-2] ----
        {
            const int g = d.at(d.nx - 1, j, k), a = d.at(d.nx - 2, j, k), am = d.at(d.nx - 3, j, k);
            if (B.east == kBcPeriodic)
            {
                const int s = d.at(1, j, k);
                u[g] = u[s]; v[g] = v[s]; w[g] = w[s]; rho[g] = rho[s]; p[g] = p[s];
            }
            else
            {
                if (B.east == kBcRigid || B.east == kBcRigidSlip) u[a] = B.frame_u;
                if (B.east == kBcRadiative && radiate)
                {
                    const float up = u_east[r];
                    const float phase = __fadd_rn(__fsub_rn(up, B.frame_u), kCStar);
                    const float un = kw78_updated_face(up, phase, __fsub_rn(up, u[am]), B.dt_rad, B.inv_dx, false);
                    u[a] = un;
                    u_east[r] = un;
                }
                else if (B.east == kBcZeroGradient) u[a] = u[am];
                u[g] = (B.east == kBcRadiative || B.east == kBcZeroGradient) ? u[a] : B.frame_u;
                if (B.east == kBcRigid) { v[g] = B.frame_v; w[g] = 0.0f; }
                else { v[g] = v[a]; w[g] = w[a]; }
                rho[g] = rho[a]; p[g] = p[a];
            }
        }
    }
}

static __global__ void acoustic_bc_we_kernel(BoundaryParams B, float* __restrict__ u, float* __restrict__ v,
                                      float* __restrict__ w, float* __restrict__ rho, float* __restrict__ p,
                                      float* __restrict__ u_west, float* __restrict__ u_east)
{
    const int rows = B.d.ny * B.d.nz;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
        bc_we_row(B, u, v, w, rho, p, u_west, u_east, r);
}

// South then north faces for one (i,k) row r: boundary_conditions_cartesian_cgrid.cpp:1034-1121.
__device__ __forceinline__ void bc_sn_row(const BoundaryParams& B, float* __restrict__ u, float* __restrict__ v,
                                          float* __restrict__ w, float* __restrict__ rho, float* __restrict__ p,
                                          float* __restrict__ v_south, float* __restrict__ v_north, int r)
{
    const Dims d = B.d;
    const bool radiate = B.dt_rad > 0.0f;
    {
        const int i = r / d.nz, k = r % d.nz;
        {
            const int g = d.at(i, 0, k), in = d.at(i, 1, k);
            if (B.south == kBcPeriodic)
            {
                const int s = d.at(i, d.ny - 2, k);
                v[g] = v[s]; u[g] = u[s]; w[g] = w[s]; rho[g] = rho[s]; p[g] = p[s];
            }
            else
            {
                if (B.south == kBcRadiative)
                {
                    if (radiate)
                    {
                        const float vp = v_south[r];
                        const float phase = __fsub_rn(__fsub_rn(vp, B.frame_v), kCStar);
                        const float vn = kw78_updated_face(vp, phase, __fsub_rn(v[in], vp), B.dt_rad, B.inv_dy, true);
                        v[g] = vn;
                        v_south[r] = vn;
                    }
                }
                else if (B.south == kBcZeroGradient) v[g] = v[in];
                else v[g] = B.frame_v;
                if (B.south == kBcRigid) { u[g] = B.frame_u; w[g] = 0.0f; }
                else { u[g] = u[in]; w[g] = w[in]; }
                rho[g] = rho[in]; p[g] = p[in];
            }
        }
        {
            const int g = d.at(i, d.ny - 1, k), a = d.at(i, d.ny - 2, k), am = d.at(i, d.ny - 3, k);
            if (B.north == kBcPeriodic)
            {
                const int s = d.at(i, 1, k);
                v[g] = v[s]; u[g] = u[s]; w[g] = w[s]; rho[g] = rho[s]; p[g] = p[s];
            }
            else
            {
                if (B.north == kBcRigid || B.north == kBcRigidSlip) v[a] = B.frame_v;
                if (B.north == kBcRadiative && radiate)
                {
                    const float vp = v_north[r];
                    const float phase = __fadd_rn(__fsub_rn(vp, B.frame_v), kCStar);
                    const float vn = kw78_updated_face(vp, phase, __fsub_rn(vp, v[am]), B.dt_rad, B.inv_dy, false);
                    v[a] = vn;
                    v_north[r] = vn;
                }
                else if (B.north == kBcZeroGradient) v[a] = v[am];
                v[g] = (B.north == kBcRadiative || B.north == kBcZeroGradient) ? v[a] : B.frame_v;
                if (B.north == kBcRigid) { u[g] = B.frame_u; w[g] = 0.0f; }
                else { u[g] = u[a]; w[g] = w[a]; }
                rho[g] = rho[a]; p[g] = p[a];
            }
        }
    }
}

static __global__ void acoustic_bc_sn_kernel(BoundaryParams B, float* __restrict__ u, float* __restrict__ v,
                                      float* __restrict__ w, float* __restrict__ rho, float* __restrict__ p,
                                      float* __restrict__ v_south, float* __restrict__ v_north)
{
    const int rows = B.d.nx * B.d.nz;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
        bc_sn_row(B, u, v, w, rho, p, v_south, v_north, r);
}

// Vertical closure for one (i,j) column: boundary_conditions_cartesian_cgrid.cpp:1124-1175.
__device__ __forceinline__ void bc_vertical_column(const BoundaryParams& B, float* __restrict__ u,
                                                   float* __restrict__ v, float* __restrict__ w, int col)
{
    const Dims d = B.d;
    {
        const int base = col * d.nz;
        if (B.bottom == kBottomNoSlip)
        {
            u[base] = 0.0f;
            v[base] = 0.0f;
        }
        const int kt = base + d.nz - 1, km = base + d.nz - 2;
        w[kt] = (B.top == kTopOpen) ? w[km] : 0.0f;
        u[kt] = u[km];
        v[kt] = v[km];
    }
}

static __global__ void acoustic_bc_vertical_kernel(BoundaryParams B, float* __restrict__ u, float* __restrict__ v,
                                            float* __restrict__ w)
{
    const int cols = B.d.nx * B.d.ny;
    for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < cols; col += gridDim.x * blockDim.x)
        bc_vertical_column(B, u, v, w, col);
}

// seed_radiative_state (boundary_conditions_cartesian_cgrid.cpp:798-822) for
// history slot r of the west/east (r < ny*nz) and south/north rows.
__device__ __forceinline__ void seed_radiation_row(const Dims& d, const float* __restrict__ u,
                                                   const float* __restrict__ v, float* __restrict__ wave, int r)
{
    const int yz = d.ny * d.nz, xz = d.nx * d.nz;
    {
        if (r < yz)
        {
            const int j = r / d.nz, k = r % d.nz;
            wave[r] = u[d.at(0, j, k)];
            wave[yz + r] = u[d.at(d.nx - 2, j, k)];
        }
        else
        {
            const int q = r - yz;
            const int i = q / d.nz, k = q % d.nz;
            wave[2 * yz + q] = v[d.at(i, 0, k)];
            wave[2 * yz + xz + q] = v[d.at(i, d.ny - 2, k)];
        }
    }
}

static __global__ void acoustic_seed_radiation_kernel(Dims d, const float* __restrict__ u, const float* __restrict__ v,
                                               float* __restrict__ wave)
{
    const int rows = d.ny * d.nz + d.nx * d.nz;
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < rows; r += gridDim.x * blockDim.x)
        seed_radiation_row(d, u, v, wave, r);
}

}  // namespace nimbus
