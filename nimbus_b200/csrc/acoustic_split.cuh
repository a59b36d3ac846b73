// Two-launch acoustic substep (one thread per cell, grid-stride), templated on
// the precision policy of acoustic_fused.cuh:
//   split_continuity_eos : retained mass flux from the old state, continuity,
//                          rho forward Euler, EOS; new rho to a ping-pong
//                          buffer, p in place.
//   split_momentum       : u,v,w forward Euler from the new pressure gradient,
//                          written to ping-pong buffers.
// No shared memory and no barriers: neighbour reuse comes from L1/L2 and
// latency is hidden by full occupancy.  It moves 84 B/cell (u,v,w are read
// twice, the new rho/p written then re-read) against the fused form's
// 64 B/cell, but issues fewer instructions per cell; the autotuner picks
// between the two per grid shape.
#pragma once

#include "acoustic_fused.cuh"

namespace nimbus
{

// First substep of a large step writes the retained flux instead of adding to
// it: float(0.0 + w*flux) is bit-identical to accumulating into a zeroed slot
// (the +0.0 turns a -0.0 product into +0.0 exactly as the add would).
__device__ __forceinline__ void fused_store(float* slot, double weight, double flux, unsigned& flags)
{
    const float st = (float)(0.0 + weight * flux);
    if (isfinite(st)) *slot = st;
    else
    {
        *slot = 0.0f;
        flags |= kStatusNonfiniteMassFlux;
    }
}

__device__ __forceinline__ void retain_flux(float* slot, double weight, double flux, unsigned& flags, bool store)
{
    if (store) fused_store(slot, weight, flux, flags);
    else fused_accumulate(slot, weight, flux, flags);
}

// Continuity, rho forward Euler and EOS for cell c.  With store_flux the
// retained fluxes are written rather than accumulated and rho_copy (when
// given) receives the pre-substep density (the transport context's
// beginning density).
template <class Policy>
__device__ __forceinline__ void continuity_eos_cell(const FusedParams& P, const float* __restrict__ rho,
                                                    const float* __restrict__ u, const float* __restrict__ v,
                                                    const float* __restrict__ w, const float* __restrict__ theta,
                                                    const double* __restrict__ rho0,
                                                    const float4* __restrict__ eos0, float* __restrict__ rho_out,
                                                    float* __restrict__ p_out, float* __restrict__ drho_out,
                                                    float* __restrict__ mfx, float* __restrict__ mfy,
                                                    float* __restrict__ mfz, int c, unsigned& flags, bool store_flux,
                                                    float* __restrict__ rho_copy)
{
    using real = typename Policy::real;
    const Dims d = P.d;
    const int sx = d.sx(), sy = d.sy();
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        const float rho_c = rho[c];
        if (rho_copy != nullptr) rho_copy[c] = rho_c;
        if (mfx != nullptr)
        {
            if constexpr (sizeof(real) == 8)
            {
                const double rc = (double)rho_c;
                if (i < d.nx - 1) retain_flux(mfx + c, P.weight, 0.5 * (rc + (double)rho[c + sx]) * ((double)u[c] - P.frame_u), flags, store_flux);
                if (j < d.ny - 1) retain_flux(mfy + c, P.weight, 0.5 * (rc + (double)rho[c + sy]) * ((double)v[c] - P.frame_v), flags, store_flux);
                const double zf = (k == d.nz - 1) ? (P.top_open ? rc * (double)w[c] : 0.0)
                                                  : 0.5 * (rc + (double)rho[c + 1]) * (double)w[c];
                retain_flux(mfz + c, P.weight, zf, flags, store_flux);
            }
            else
            {
                if (i < d.nx - 1)
                    retain_flux_f32(mfx + c, P.weight_f, 0.5f * (rho_c + rho[c + sx]) * (u[c] - P.frame_u_f), flags,
                                    store_flux);
                if (j < d.ny - 1)
                    retain_flux_f32(mfy + c, P.weight_f, 0.5f * (rho_c + rho[c + sy]) * (v[c] - P.frame_v_f), flags,
                                    store_flux);
                const float zf = (k == d.nz - 1) ? (P.top_open ? rho_c * w[c] : 0.0f) : 0.5f * (rho_c + rho[c + 1]) * w[c];
                retain_flux_f32(mfz + c, P.weight_f, zf, flags, store_flux);
            }
        }
        real drho = (real)0;
        if (i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1)
        {
            const real rc = (real)rho_c;
            const real half = (real)0.5;
            const real fx_pos = half * (rc + (real)rho[c + sx]) * (real)u[c];
            const real fx_neg = half * ((real)rho[c - sx] + rc) * (real)u[c - sx];
            const real fy_pos = half * (rc + (real)rho[c + sy]) * (real)v[c];
            const real fy_neg = half * ((real)rho[c - sy] + rc) * (real)v[c - sy];
            const real fz_pos = (k + 1 < d.nz) ? half * (rc + (real)rho[c + 1]) * (real)w[c] : rc * (real)w[c];
            const real fz_neg = (k > 0) ? half * ((real)rho[c - 1] + rc) * (real)w[c - 1] : (real)0;
            if constexpr (sizeof(real) == 8)
                drho = -((fx_pos - fx_neg) * P.inv_dx + (fy_pos - fy_neg) * P.inv_dy + (fz_pos - fz_neg) * P.inv_dz);
            else
                drho = -((fx_pos - fx_neg) * P.inv_dx_f + (fy_pos - fy_neg) * P.inv_dy_f +
                         (fz_pos - fz_neg) * P.inv_dz_f);
        }
        float drho_stored;
        if constexpr (sizeof(real) == 8) drho_stored = (float)finite_or_zero(drho);
        else drho_stored = isfinite(drho) ? drho : 0.0f;
        if (drho_out != nullptr) drho_out[c] = drho_stored;
        const float rho_stored = substep_density<Policy>(P, rho_c, drho_stored, rho0, k);
        rho_out[c] = rho_stored;
        p_out[c] = substep_pressure<Policy>(P, eos0, k, rho_stored, theta[c]);
    }
}

template <class Policy>
static __global__ void __launch_bounds__(256) split_continuity_eos_kernel(
    FusedParams P, const float* __restrict__ rho, const float* __restrict__ u, const float* __restrict__ v,
    const float* __restrict__ w, const float* __restrict__ theta, const double* __restrict__ rho0,
    const float4* __restrict__ eos0, float* __restrict__ rho_out, float* __restrict__ p_out,
    float* __restrict__ drho_out, float* __restrict__ mfx, float* __restrict__ mfy, float* __restrict__ mfz,
    unsigned* __restrict__ status)
{
    const int n = P.d.cells();
    unsigned flags = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        continuity_eos_cell<Policy>(P, rho, u, v, w, theta, rho0, eos0, rho_out, p_out, drho_out, mfx, mfy, mfz, c,
                                    flags, false, nullptr);
    if (flags) atomicOr(status, flags);
}

// Momentum forward Euler for the faces of cell c.  Face c reads only its own
// old velocity, so u_out may alias u (in-place update).
template <class Policy>
__device__ __forceinline__ void momentum_cell(const FusedParams& P, const float* __restrict__ rho,
                                              const float* __restrict__ p, const double* __restrict__ p0,
                                              const float2* __restrict__ dp0_split, const float* u, const float* v,
                                              const float* w, float* u_out, float* v_out, float* w_out, int c)
{
    using real = typename Policy::real;
    const Dims d = P.d;
    const int sx = d.sx(), sy = d.sy();
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        float du = 0.0f, dv = 0.0f, dw = 0.0f;
        if (i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1)
        {
            if constexpr (sizeof(real) == 8)
            {
                const double rc = (double)rho[c];
                const double rho_x = 0.5 * (rc + (double)rho[c + sx]);
                const double rho_y = 0.5 * (rc + (double)rho[c + sy]);
                const double rho_z = 0.5 * (rc + (double)rho[c + 1]);
                const double pc = (double)p[c];
                const double dp0_dz = (p0[k + 1] - p0[k]) * P.inv_dz;
                du = (float)finite_or_zero(-((double)p[c + sx] - pc) * P.inv_dx / safe_rho(rho_x));
                dv = (float)finite_or_zero(-((double)p[c + sy] - pc) * P.inv_dy / safe_rho(rho_y));
                dw = (float)finite_or_zero(-((((double)p[c + 1] - pc) * P.inv_dz) - dp0_dz) / safe_rho(rho_z));
            }
            else
            {
                const float rc = rho[c];
                const float rho_x = 0.5f * (rc + rho[c + sx]);
                const float rho_y = 0.5f * (rc + rho[c + sy]);
                const float rho_z = 0.5f * (rc + rho[c + 1]);
                const float pc = p[c];
                const float2 dp0 = dp0_split[k];
                const float dpz = ((p[c + 1] - pc) - dp0.x) - dp0.y;
                const float sxr = (isfinite(rho_x) && rho_x > 1.0e-6f) ? rho_x : 1.0f;
                const float syr = (isfinite(rho_y) && rho_y > 1.0e-6f) ? rho_y : 1.0f;
                const float szr = (isfinite(rho_z) && rho_z > 1.0e-6f) ? rho_z : 1.0f;
                const float a = __fdividef(-(p[c + sx] - pc) * P.inv_dx_f, sxr);
                const float b = __fdividef(-(p[c + sy] - pc) * P.inv_dy_f, syr);
                const float cz = __fdividef(-dpz * P.inv_dz_f, szr);
                du = isfinite(a) ? a : 0.0f;
                dv = isfinite(b) ? b : 0.0f;
                dw = isfinite(cz) ? cz : 0.0f;
            }
        }
        if constexpr (sizeof(real) == 8)
        {
            u_out[c] = clamp_value((float)((double)u[c] + (double)du * P.dt_small), 0.0f, -P.wind_h, P.wind_h);
            v_out[c] = clamp_value((float)((double)v[c] + (double)dv * P.dt_small), 0.0f, -P.wind_h, P.wind_h);
            w_out[c] = clamp_value((float)((double)w[c] + (double)dw * P.dt_small), 0.0f, -P.wind_v, P.wind_v);
        }
        else
        {
            const float dt = P.dt_f;
            u_out[c] = clamp_value(__fmaf_rn(du, dt, u[c]), 0.0f, -P.wind_h, P.wind_h);
            v_out[c] = clamp_value(__fmaf_rn(dv, dt, v[c]), 0.0f, -P.wind_h, P.wind_h);
            w_out[c] = clamp_value(__fmaf_rn(dw, dt, w[c]), 0.0f, -P.wind_v, P.wind_v);
        }
    }
}

template <class Policy>
static __global__ void __launch_bounds__(256) split_momentum_kernel(
    FusedParams P, const float* __restrict__ rho, const float* __restrict__ p, const double* __restrict__ p0,
    const float2* __restrict__ dp0_split, const float* __restrict__ u, const float* __restrict__ v,
    const float* __restrict__ w, float* __restrict__ u_out, float* __restrict__ v_out, float* __restrict__ w_out)
{
    const int n = P.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        momentum_cell<Policy>(P, rho, p, p0, dp0_split, u, v, w, u_out, v_out, w_out, c);
}

}  // namespace nimbus
