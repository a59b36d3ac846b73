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

// Retained-flux update from an already loaded slot value.  Reference policy:
// the FP64 weighted sum rounded once to the FP32 slot (fused_accumulate);
// FP32 policy: one FMA (retain_flux_f32).  With store the slot starts from
// zero -- the first substep of a large step writes instead of accumulating,
// bit-identical to accumulating into a zeroed slot (the 0.0 + product turns a
// -0.0 into +0.0 exactly as the add would).
template <class Policy>
__device__ __forceinline__ void retain_flux_from(float* slot, float old, const FusedParams& P, double flux64,
                                                 float flux32, unsigned& flags, bool store)
{
    if constexpr (Policy::exact_pow)
    {
        const float st = (float)((store ? 0.0 : (double)old) + P.weight * flux64);
        if (isfinite(st)) *slot = st;
        else
        {
            if (store) *slot = 0.0f;
            flags |= kStatusNonfiniteMassFlux;
        }
    }
    else
    {
        const float st = __fmaf_rn(P.weight_f, flux32, store ? 0.0f : old);
        if (isfinite(st)) *slot = st;
        else
        {
            if (store) *slot = 0.0f;
            flags |= kStatusNonfiniteMassFlux;
        }
    }
}

// Continuity, rho forward Euler and EOS for cell c.  With store_flux the
// retained fluxes are written rather than accumulated and rho_copy (when
// given) receives the pre-substep density (the transport context's
// beginning density).  Every load is issued before any arithmetic (indices of
// neighbours outside the grid are clamped to the cell; those values are not
// used), so a thread has all of its memory requests in flight at once.
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
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool xlo = i >= 1, xhi = i < d.nx - 1, ylo = j >= 1, yhi = j < d.ny - 1;
    const bool zlo = k > 0, zhi = k + 1 < d.nz;
    const float rho_c = rho[c];
    const float rxp = rho[xhi ? c + sx : c], rxm = rho[xlo ? c - sx : c];
    const float ryp = rho[yhi ? c + sy : c], rym = rho[ylo ? c - sy : c];
    const float rzp = rho[zhi ? c + 1 : c], rzm = rho[zlo ? c - 1 : c];
    const float uc = u[c], uxm = u[xlo ? c - sx : c];
    const float vc = v[c], vym = v[ylo ? c - sy : c];
    const float wc = w[c], wzm = w[zlo ? c - 1 : c];
    const float th = theta[c];
    const bool flux = mfx != nullptr;
    const bool acc = flux && !store_flux;
    const float mx = acc ? mfx[c] : 0.0f, my = acc ? mfy[c] : 0.0f, mz = acc ? mfz[c] : 0.0f;

    if (rho_copy != nullptr) rho_copy[c] = rho_c;
    if (flux)
    {
        if constexpr (sizeof(real) == 8)
        {
            const double rc = (double)rho_c;
            if (xhi)
                retain_flux_from<Policy>(mfx + c, mx, P, 0.5 * (rc + (double)rxp) * ((double)uc - P.frame_u), 0.0f,
                                         flags, store_flux);
            if (yhi)
                retain_flux_from<Policy>(mfy + c, my, P, 0.5 * (rc + (double)ryp) * ((double)vc - P.frame_v), 0.0f,
                                         flags, store_flux);
            const double zf = !zhi ? (P.top_open ? rc * (double)wc : 0.0) : 0.5 * (rc + (double)rzp) * (double)wc;
            retain_flux_from<Policy>(mfz + c, mz, P, zf, 0.0f, flags, store_flux);
        }
        else
        {
            if (xhi)
                retain_flux_from<Policy>(mfx + c, mx, P, 0.0, 0.5f * (rho_c + rxp) * (uc - P.frame_u_f), flags,
                                         store_flux);
            if (yhi)
                retain_flux_from<Policy>(mfy + c, my, P, 0.0, 0.5f * (rho_c + ryp) * (vc - P.frame_v_f), flags,
                                         store_flux);
            const float zf = !zhi ? (P.top_open ? rho_c * wc : 0.0f) : 0.5f * (rho_c + rzp) * wc;
            retain_flux_from<Policy>(mfz + c, mz, P, 0.0, zf, flags, store_flux);
        }
    }
    real drho = (real)0;
    if (xlo && xhi && ylo && yhi)
    {
        const real rc = (real)rho_c;
        const real half = (real)0.5;
        const real fx_pos = half * (rc + (real)rxp) * (real)uc;
        const real fx_neg = half * ((real)rxm + rc) * (real)uxm;
        const real fy_pos = half * (rc + (real)ryp) * (real)vc;
        const real fy_neg = half * ((real)rym + rc) * (real)vym;
        const real fz_pos = zhi ? half * (rc + (real)rzp) * (real)wc : rc * (real)wc;
        const real fz_neg = zlo ? half * ((real)rzm + rc) * (real)wzm : (real)0;
        if constexpr (sizeof(real) == 8)
            drho = -((fx_pos - fx_neg) * P.inv_dx + (fy_pos - fy_neg) * P.inv_dy + (fz_pos - fz_neg) * P.inv_dz);
        else
            drho = -((fx_pos - fx_neg) * P.inv_dx_f + (fy_pos - fy_neg) * P.inv_dy_f + (fz_pos - fz_neg) * P.inv_dz_f);
    }
    float drho_stored;
    if constexpr (sizeof(real) == 8) drho_stored = (float)finite_or_zero(drho);
    else drho_stored = isfinite(drho) ? drho : 0.0f;
    if (drho_out != nullptr) drho_out[c] = drho_stored;
    const float rho_stored = substep_density<Policy>(P, rho_c, drho_stored, rho0, k);
    rho_out[c] = rho_stored;
    p_out[c] = substep_pressure<Policy>(P, eos0, k, rho_stored, th);
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
// Stores the new face velocities of cell c, with the vertical closure of its
// column when fuse_vertical asks for it (see momentum_cell).  (Handing the
// top values to the cell above through a warp shuffle, so that every lane
// stores its own cell, measured slower than these scattered stores.)
__device__ __forceinline__ void momentum_store(const Dims& d, int i, int j, int k, int c, int fuse_vertical, float un,
                                               float vn, float wn, float* u_out, float* v_out, float* w_out)
{
    if ((fuse_vertical & 1) && i >= 1 && i <= d.nx - 3 && j >= 1 && j <= d.ny - 3)
    {
        if (k == d.nz - 1) return;  // written by the cell below
        if (k == 0 && (fuse_vertical & 2))
        {
            un = 0.0f;
            vn = 0.0f;
        }
        if (k == d.nz - 2)
        {
            u_out[c + 1] = un;
            v_out[c + 1] = vn;
            w_out[c + 1] = (fuse_vertical & 4) ? wn : 0.0f;
        }
    }
    u_out[c] = un;
    v_out[c] = vn;
    w_out[c] = wn;
}

// fuse_vertical (kFuse* bits): the momentum pass also applies the vertical
// closure (bc_vertical_column) to the columns no lateral closure writes
// (1 <= i <= nx-3, 1 <= j <= ny-3): the no-slip bottom zeros u and v at k = 0,
// the cell at k = nz-2 writes its new u, v and w (or 0 under a rigid top)
// into level nz-1 as well, and the cell at nz-1 does not store.  The lateral
// closures that run in between neither write nor depend on those columns'
// levels 0 and nz-1 for any value that survives the closure of their own
// columns, so the state is the one the separate closure pass gives.
enum : int
{
    kFuseVertical = 1,
    kFuseNoSlipBottom = 2,
    kFuseOpenTop = 4
};

template <class Policy>
__device__ __forceinline__ void momentum_cell(const FusedParams& P, const float* __restrict__ rho,
                                              const float* __restrict__ p, const double* __restrict__ p0,
                                              const float2* __restrict__ dp0_split, const float* u, const float* v,
                                              const float* w, float* u_out, float* v_out, float* w_out, int c,
                                              int fuse_vertical = 0)
{
    using real = typename Policy::real;
    const Dims d = P.d;
    const int sx = d.sx(), sy = d.sy();
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool interior = i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1;
    // Every load first; outside the interior the neighbour indices fall back
    // to the cell itself (those values are not used).
    const int cx = interior ? c + sx : c, cy = interior ? c + sy : c, cz1 = interior ? c + 1 : c;
    const float rc = rho[c], rx = rho[cx], ry = rho[cy], rz = rho[cz1];
    const float pc = p[c], px = p[cx], py = p[cy], pz = p[cz1];
    const float uc = u[c], vc = v[c], wc = w[c];
    float du = 0.0f, dv = 0.0f, dw = 0.0f;
    if constexpr (sizeof(real) == 8)
    {
        if (interior)
        {
            const double rcd = (double)rc;
            const double rho_x = 0.5 * (rcd + (double)rx);
            const double rho_y = 0.5 * (rcd + (double)ry);
            const double rho_z = 0.5 * (rcd + (double)rz);
            const double pcd = (double)pc;
            const double dp0_dz = (p0[k + 1] - p0[k]) * P.inv_dz;
            du = (float)finite_or_zero(-((double)px - pcd) * P.inv_dx / safe_rho(rho_x));
            dv = (float)finite_or_zero(-((double)py - pcd) * P.inv_dy / safe_rho(rho_y));
            dw = (float)finite_or_zero(-((((double)pz - pcd) * P.inv_dz) - dp0_dz) / safe_rho(rho_z));
        }
        momentum_store(d, i, j, k, c, fuse_vertical,
                       clamp_value((float)((double)uc + (double)du * P.dt_small), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value((float)((double)vc + (double)dv * P.dt_small), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value((float)((double)wc + (double)dw * P.dt_small), 0.0f, -P.wind_v, P.wind_v), u_out,
                       v_out, w_out);
    }
    else
    {
        const float2 dp0 = dp0_split[k];
        if (interior)
        {
            const float rho_x = 0.5f * (rc + rx);
            const float rho_y = 0.5f * (rc + ry);
            const float rho_z = 0.5f * (rc + rz);
            const float dpz = ((pz - pc) - dp0.x) - dp0.y;
            const float sxr = (isfinite(rho_x) && rho_x > 1.0e-6f) ? rho_x : 1.0f;
            const float syr = (isfinite(rho_y) && rho_y > 1.0e-6f) ? rho_y : 1.0f;
            const float szr = (isfinite(rho_z) && rho_z > 1.0e-6f) ? rho_z : 1.0f;
            const float a = __fdividef(-(px - pc) * P.inv_dx_f, sxr);
            const float b = __fdividef(-(py - pc) * P.inv_dy_f, syr);
            const float cz = __fdividef(-dpz * P.inv_dz_f, szr);
            du = isfinite(a) ? a : 0.0f;
            dv = isfinite(b) ? b : 0.0f;
            dw = isfinite(cz) ? cz : 0.0f;
        }
        const float dt = P.dt_f;
        momentum_store(d, i, j, k, c, fuse_vertical, clamp_value(__fmaf_rn(du, dt, uc), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value(__fmaf_rn(dv, dt, vc), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value(__fmaf_rn(dw, dt, wc), 0.0f, -P.wind_v, P.wind_v), u_out, v_out, w_out);
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
