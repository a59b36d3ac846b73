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

// The old-state neighbourhood one cell's continuity reads: density at the
// cell and its six face neighbours, the velocities on the cell's upper and
// lower faces, theta, and the stored retained-flux sums.  Neighbours outside
// the grid hold the cell's own value (they are never used).
struct ContinuityStencil
{
    float rho_c, rxp, rxm, ryp, rym, rzp, rzm;
    float uc, uxm, vc, vym, wc, wzm;
    float th;
    float mx, my, mz;
};

// Continuity, rho forward Euler and EOS of cell c = (i, j, k) from its loaded
// stencil: the retained fluxes of its three upper faces (written when
// store_flux, else accumulated), the new density into rho_out[c] and the
// pressure into p_out[c].  Every way of loading the stencil (one thread per
// cell, or marching along i) ends here, so the arithmetic is one sequence.
template <class Policy>
__device__ __forceinline__ void continuity_eos_values(const FusedParams& P, const ContinuityStencil& s, int i, int j,
                                                      int k, int c, const double* __restrict__ rho0,
                                                      const float4* __restrict__ eos0, float* __restrict__ rho_out,
                                                      float* __restrict__ p_out, float* __restrict__ drho_out,
                                                      float* __restrict__ mfx, float* __restrict__ mfy,
                                                      float* __restrict__ mfz, unsigned& flags, bool store_flux,
                                                      float* __restrict__ rho_copy)
{
    using real = typename Policy::real;
    const Dims d = P.d;
    const bool xlo = i >= 1, xhi = i < d.nx - 1, ylo = j >= 1, yhi = j < d.ny - 1;
    const bool zlo = k > 0, zhi = k + 1 < d.nz;
    const float rho_c = s.rho_c;
    const bool flux = mfx != nullptr;

    if (rho_copy != nullptr) rho_copy[c] = rho_c;
    if (flux)
    {
        if constexpr (sizeof(real) == 8)
        {
            const double rc = (double)rho_c;
            if (xhi)
                retain_flux_from<Policy>(mfx + c, s.mx, P, 0.5 * (rc + (double)s.rxp) * ((double)s.uc - P.frame_u),
                                         0.0f, flags, store_flux);
            if (yhi)
                retain_flux_from<Policy>(mfy + c, s.my, P, 0.5 * (rc + (double)s.ryp) * ((double)s.vc - P.frame_v),
                                         0.0f, flags, store_flux);
            const double zf =
                !zhi ? (P.top_open ? rc * (double)s.wc : 0.0) : 0.5 * (rc + (double)s.rzp) * (double)s.wc;
            retain_flux_from<Policy>(mfz + c, s.mz, P, zf, 0.0f, flags, store_flux);
        }
        else
        {
            if (xhi)
                retain_flux_from<Policy>(mfx + c, s.mx, P, 0.0, 0.5f * (rho_c + s.rxp) * (s.uc - P.frame_u_f), flags,
                                         store_flux);
            if (yhi)
                retain_flux_from<Policy>(mfy + c, s.my, P, 0.0, 0.5f * (rho_c + s.ryp) * (s.vc - P.frame_v_f), flags,
                                         store_flux);
            const float zf = !zhi ? (P.top_open ? rho_c * s.wc : 0.0f) : 0.5f * (rho_c + s.rzp) * s.wc;
            retain_flux_from<Policy>(mfz + c, s.mz, P, 0.0, zf, flags, store_flux);
        }
    }
    real drho = (real)0;
    if (xlo && xhi && ylo && yhi)
    {
        const real rc = (real)rho_c;
        const real half = (real)0.5;
        const real fx_pos = half * (rc + (real)s.rxp) * (real)s.uc;
        const real fx_neg = half * ((real)s.rxm + rc) * (real)s.uxm;
        const real fy_pos = half * (rc + (real)s.ryp) * (real)s.vc;
        const real fy_neg = half * ((real)s.rym + rc) * (real)s.vym;
        const real fz_pos = zhi ? half * (rc + (real)s.rzp) * (real)s.wc : rc * (real)s.wc;
        const real fz_neg = zlo ? half * ((real)s.rzm + rc) * (real)s.wzm : (real)0;
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
    p_out[c] = substep_pressure<Policy>(P, eos0, k, rho_stored, s.th);
}

// Loads cell c = (i, j, k)'s continuity stencil (acc: the stored retained-flux
// sums too).  Neighbours outside the grid read the cell itself.
__device__ __forceinline__ ContinuityStencil continuity_load(const Dims& d, const float* __restrict__ rho,
                                                             const float* __restrict__ u,
                                                             const float* __restrict__ v,
                                                             const float* __restrict__ w,
                                                             const float* __restrict__ theta, const float* mfx,
                                                             const float* mfy, const float* mfz, bool acc, int c,
                                                             int i, int j, int k)
{
    const int sx = d.sx(), sy = d.sy();
    const bool xlo = i >= 1, xhi = i < d.nx - 1, ylo = j >= 1, yhi = j < d.ny - 1;
    const bool zlo = k > 0, zhi = k + 1 < d.nz;
    ContinuityStencil s;
    s.rho_c = rho[c];
    s.rxp = rho[xhi ? c + sx : c];
    s.rxm = rho[xlo ? c - sx : c];
    s.ryp = rho[yhi ? c + sy : c];
    s.rym = rho[ylo ? c - sy : c];
    s.rzp = rho[zhi ? c + 1 : c];
    s.rzm = rho[zlo ? c - 1 : c];
    s.uc = u[c];
    s.uxm = u[xlo ? c - sx : c];
    s.vc = v[c];
    s.vym = v[ylo ? c - sy : c];
    s.wc = w[c];
    s.wzm = w[zlo ? c - 1 : c];
    s.th = theta[c];
    s.mx = acc ? mfx[c] : 0.0f;
    s.my = acc ? mfy[c] : 0.0f;
    s.mz = acc ? mfz[c] : 0.0f;
    return s;
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
    int i, j, k;
    decompose(P.d, c, i, j, k);
    const ContinuityStencil s =
        continuity_load(P.d, rho, u, v, w, theta, mfx, mfy, mfz, mfx != nullptr && !store_flux, c, i, j, k);
    continuity_eos_values<Policy>(P, s, i, j, k, c, rho0, eos0, rho_out, p_out, drho_out, mfx, mfy, mfz, flags,
                                  store_flux, rho_copy);
}

// The same continuity for the cells (i0 .. i1-1, j, k) of one grid row along
// x, marching in i: the density of planes i-1, i and the x-velocity of plane
// i-1 carry over in registers from the previous cell, so a cell loads one new
// x-neighbour instead of three, and its neighbour offsets and boundary flags
// in j and k are formed once per row.  q = j nz + k.
template <class Policy>
__device__ __forceinline__ void continuity_eos_march(const FusedParams& P, const float* __restrict__ rho,
                                                     const float* __restrict__ u, const float* __restrict__ v,
                                                     const float* __restrict__ w, const float* __restrict__ theta,
                                                     const double* __restrict__ rho0,
                                                     const float4* __restrict__ eos0, float* __restrict__ rho_out,
                                                     float* __restrict__ p_out, float* __restrict__ mfx,
                                                     float* __restrict__ mfy, float* __restrict__ mfz, int i0, int i1,
                                                     int j, int k, int q, unsigned& flags, bool store_flux,
                                                     float* __restrict__ rho_copy)
{
    const Dims d = P.d;
    const int sx = d.sx();
    const int oyp = j < d.ny - 1 ? d.nz : 0, oym = j >= 1 ? -d.nz : 0;
    const int ozp = k + 1 < d.nz ? 1 : 0, ozm = k > 0 ? -1 : 0;
    const bool acc = mfx != nullptr && !store_flux;
    int c = i0 * sx + q;
    float r_m = rho[i0 >= 1 ? c - sx : c];
    float r_c = rho[c];
    float u_m = u[i0 >= 1 ? c - sx : c];
    for (int i = i0; i < i1; ++i, c += sx)
    {
        ContinuityStencil s;
        s.rho_c = r_c;
        s.rxm = r_m;
        s.rxp = rho[i < d.nx - 1 ? c + sx : c];
        s.ryp = rho[c + oyp];
        s.rym = rho[c + oym];
        s.rzp = rho[c + ozp];
        s.rzm = rho[c + ozm];
        s.uc = u[c];
        s.uxm = u_m;
        s.vc = v[c];
        s.vym = v[c + oym];
        s.wc = w[c];
        s.wzm = w[c + ozm];
        s.th = theta[c];
        s.mx = acc ? mfx[c] : 0.0f;
        s.my = acc ? mfy[c] : 0.0f;
        s.mz = acc ? mfz[c] : 0.0f;
        continuity_eos_values<Policy>(P, s, i, j, k, c, rho0, eos0, rho_out, p_out, nullptr, mfx, mfy, mfz, flags,
                                      store_flux, rho_copy);
        r_m = r_c;
        r_c = s.rxp;
        u_m = s.uc;
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

// The new-state neighbourhood of one cell's momentum: density and pressure at
// the cell and its upper x, y and z neighbours, and the cell's old face
// velocities.
struct MomentumStencil
{
    float rc, rx, ry, rz;
    float pc, px, py, pz;
    float uc, vc, wc;
};

// Momentum forward Euler of the faces of cell c = (i, j, k) from its loaded
// stencil (see momentum_cell).
template <class Policy>
__device__ __forceinline__ void momentum_values(const FusedParams& P, const MomentumStencil& s, int i, int j, int k,
                                                int c, const double* __restrict__ p0,
                                                const float2* __restrict__ dp0_split, float* u_out, float* v_out,
                                                float* w_out, int fuse_vertical)
{
    using real = typename Policy::real;
    const Dims d = P.d;
    const bool interior = i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1;
    float du = 0.0f, dv = 0.0f, dw = 0.0f;
    if constexpr (sizeof(real) == 8)
    {
        if (interior)
        {
            const double rcd = (double)s.rc;
            const double rho_x = 0.5 * (rcd + (double)s.rx);
            const double rho_y = 0.5 * (rcd + (double)s.ry);
            const double rho_z = 0.5 * (rcd + (double)s.rz);
            const double pcd = (double)s.pc;
            const double dp0_dz = (p0[k + 1] - p0[k]) * P.inv_dz;
            du = (float)finite_or_zero(-((double)s.px - pcd) * P.inv_dx / safe_rho(rho_x));
            dv = (float)finite_or_zero(-((double)s.py - pcd) * P.inv_dy / safe_rho(rho_y));
            dw = (float)finite_or_zero(-((((double)s.pz - pcd) * P.inv_dz) - dp0_dz) / safe_rho(rho_z));
        }
        momentum_store(d, i, j, k, c, fuse_vertical,
                       clamp_value((float)((double)s.uc + (double)du * P.dt_small), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value((float)((double)s.vc + (double)dv * P.dt_small), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value((float)((double)s.wc + (double)dw * P.dt_small), 0.0f, -P.wind_v, P.wind_v),
                       u_out, v_out, w_out);
    }
    else
    {
        const float2 dp0 = dp0_split[k];
        if (interior)
        {
            const float rho_x = 0.5f * (s.rc + s.rx);
            const float rho_y = 0.5f * (s.rc + s.ry);
            const float rho_z = 0.5f * (s.rc + s.rz);
            const float dpz = ((s.pz - s.pc) - dp0.x) - dp0.y;
            const float sxr = (isfinite(rho_x) && rho_x > 1.0e-6f) ? rho_x : 1.0f;
            const float syr = (isfinite(rho_y) && rho_y > 1.0e-6f) ? rho_y : 1.0f;
            const float szr = (isfinite(rho_z) && rho_z > 1.0e-6f) ? rho_z : 1.0f;
            const float a = __fdividef(-(s.px - s.pc) * P.inv_dx_f, sxr);
            const float b = __fdividef(-(s.py - s.pc) * P.inv_dy_f, syr);
            const float cz = __fdividef(-dpz * P.inv_dz_f, szr);
            du = isfinite(a) ? a : 0.0f;
            dv = isfinite(b) ? b : 0.0f;
            dw = isfinite(cz) ? cz : 0.0f;
        }
        const float dt = P.dt_f;
        momentum_store(d, i, j, k, c, fuse_vertical, clamp_value(__fmaf_rn(du, dt, s.uc), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value(__fmaf_rn(dv, dt, s.vc), 0.0f, -P.wind_h, P.wind_h),
                       clamp_value(__fmaf_rn(dw, dt, s.wc), 0.0f, -P.wind_v, P.wind_v), u_out, v_out, w_out);
    }
}

// Loads cell c = (i, j, k)'s momentum stencil; outside the interior the
// neighbour indices fall back to the cell itself (those values are not used).
__device__ __forceinline__ MomentumStencil momentum_load(const Dims& d, const float* __restrict__ rho,
                                                         const float* __restrict__ p, const float* u, const float* v,
                                                         const float* w, int c, int i, int j, int k)
{
    const bool interior = i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1;
    const int cx = interior ? c + d.sx() : c, cy = interior ? c + d.sy() : c, cz1 = interior ? c + 1 : c;
    MomentumStencil s;
    s.rc = rho[c];
    s.rx = rho[cx];
    s.ry = rho[cy];
    s.rz = rho[cz1];
    s.pc = p[c];
    s.px = p[cx];
    s.py = p[cy];
    s.pz = p[cz1];
    s.uc = u[c];
    s.vc = v[c];
    s.wc = w[c];
    return s;
}

template <class Policy>
__device__ __forceinline__ void momentum_cell(const FusedParams& P, const float* __restrict__ rho,
                                              const float* __restrict__ p, const double* __restrict__ p0,
                                              const float2* __restrict__ dp0_split, const float* u, const float* v,
                                              const float* w, float* u_out, float* v_out, float* w_out, int c,
                                              int fuse_vertical = 0)
{
    int i, j, k;
    decompose(P.d, c, i, j, k);
    const MomentumStencil s = momentum_load(P.d, rho, p, u, v, w, c, i, j, k);
    momentum_values<Policy>(P, s, i, j, k, c, p0, dp0_split, u_out, v_out, w_out, fuse_vertical);
}

// The same momentum for the cells (i0 .. i1-1, j, k) of one row along x,
// marching in i: the new density and pressure of plane i+1 loaded for cell i
// are those of cell i+1, so they carry over in registers.  q = j nz + k.
template <class Policy>
__device__ __forceinline__ void momentum_march(const FusedParams& P, const float* __restrict__ rho,
                                               const float* __restrict__ p, const double* __restrict__ p0,
                                               const float2* __restrict__ dp0_split, float* u, float* v, float* w,
                                               int i0, int i1, int j, int k, int q, int fuse_vertical)
{
    const Dims d = P.d;
    const int sx = d.sx();
    const int oy = j < d.ny - 1 ? d.nz : 0, oz = k < d.nz - 1 ? 1 : 0;
    int c = i0 * sx + q;
    float rc = rho[c], pc = p[c];
    for (int i = i0; i < i1; ++i, c += sx)
    {
        MomentumStencil s;
        const int cx = i < d.nx - 1 ? c + sx : c;
        s.rc = rc;
        s.pc = pc;
        s.rx = rho[cx];
        s.px = p[cx];
        s.ry = rho[c + oy];
        s.py = p[c + oy];
        s.rz = rho[c + oz];
        s.pz = p[c + oz];
        s.uc = u[c];
        s.vc = v[c];
        s.wc = w[c];
        momentum_values<Policy>(P, s, i, j, k, c, p0, dp0_split, u, v, w, fuse_vertical);
        rc = s.rx;
        pc = s.px;
    }
}

// ---- Two vertically adjacent cells per thread ------------------------------
// Cells c and c + 1 with c even, of a grid whose nz is even: both lie in one
// column (k even, k + 1 <= nz - 1), share i and j, and every field's values at
// the pair and at the pair shifted by +-sx or +-sy are one aligned 8-byte load
// (member fields start on 256-byte boundaries; sx and sy are even).  Each
// cell's stencil holds the values the one-cell loads give wherever its
// arithmetic reads them (a neighbour outside the grid or the interior may
// hold another in-range value), and its arithmetic is the one-cell form's.
__device__ __forceinline__ float2 load_pair(const float* __restrict__ f, int c)
{
    return *reinterpret_cast<const float2*>(f + c);
}

template <class Policy>
__device__ __forceinline__ void continuity_eos_kpair(const FusedParams& P, const float* __restrict__ rho,
                                                     const float* __restrict__ u, const float* __restrict__ v,
                                                     const float* __restrict__ w, const float* __restrict__ theta,
                                                     const double* __restrict__ rho0,
                                                     const float4* __restrict__ eos0, float* __restrict__ rho_out,
                                                     float* __restrict__ p_out, float* __restrict__ mfx,
                                                     float* __restrict__ mfy, float* __restrict__ mfz, int c,
                                                     unsigned& flags, bool store_flux, float* __restrict__ rho_copy)
{
    const Dims d = P.d;
    int i, j, k;
    decompose(d, c, i, j, k);
    const int sx = d.sx(), sy = d.sy();
    const bool xlo = i >= 1, xhi = i < d.nx - 1, ylo = j >= 1, yhi = j < d.ny - 1;
    const bool acc = mfx != nullptr && !store_flux;
    const float2 r = load_pair(rho, c);
    const float2 rxp = load_pair(rho, xhi ? c + sx : c), rxm = load_pair(rho, xlo ? c - sx : c);
    const float2 ryp = load_pair(rho, yhi ? c + sy : c), rym = load_pair(rho, ylo ? c - sy : c);
    const float rzm = rho[k > 0 ? c - 1 : c];
    const float rzp = rho[k + 2 < d.nz ? c + 2 : c + 1];
    const float2 uc = load_pair(u, c), uxm = load_pair(u, xlo ? c - sx : c);
    const float2 vc = load_pair(v, c), vym = load_pair(v, ylo ? c - sy : c);
    const float2 wc = load_pair(w, c);
    const float wzm = w[k > 0 ? c - 1 : c];
    const float2 th = load_pair(theta, c);
    float2 mx = make_float2(0.0f, 0.0f), my = mx, mz = mx;
    if (acc)
    {
        mx = load_pair(mfx, c);
        my = load_pair(mfy, c);
        mz = load_pair(mfz, c);
    }
    ContinuityStencil a, b;
    a.rho_c = r.x; a.rxp = rxp.x; a.rxm = rxm.x; a.ryp = ryp.x; a.rym = rym.x; a.rzp = r.y; a.rzm = rzm;
    a.uc = uc.x; a.uxm = uxm.x; a.vc = vc.x; a.vym = vym.x; a.wc = wc.x; a.wzm = wzm; a.th = th.x;
    a.mx = mx.x; a.my = my.x; a.mz = mz.x;
    b.rho_c = r.y; b.rxp = rxp.y; b.rxm = rxm.y; b.ryp = ryp.y; b.rym = rym.y; b.rzp = rzp; b.rzm = r.x;
    b.uc = uc.y; b.uxm = uxm.y; b.vc = vc.y; b.vym = vym.y; b.wc = wc.y; b.wzm = wc.x; b.th = th.y;
    b.mx = mx.y; b.my = my.y; b.mz = mz.y;
    continuity_eos_values<Policy>(P, a, i, j, k, c, rho0, eos0, rho_out, p_out, nullptr, mfx, mfy, mfz, flags,
                                  store_flux, rho_copy);
    continuity_eos_values<Policy>(P, b, i, j, k + 1, c + 1, rho0, eos0, rho_out, p_out, nullptr, mfx, mfy, mfz, flags,
                                  store_flux, rho_copy);
}

// Momentum of the pair (c, c + 1), in place.  Both stencils are loaded before
// either cell stores: under the vertical closure the cell at nz - 2 writes
// level nz - 1, which is the pair's second cell when nz - 2 is even, and that
// cell stores nothing.
template <class Policy>
__device__ __forceinline__ void momentum_kpair(const FusedParams& P, const float* __restrict__ rho,
                                               const float* __restrict__ p, const double* __restrict__ p0,
                                               const float2* __restrict__ dp0_split, float* u, float* v, float* w,
                                               int c, int fuse_vertical)
{
    const Dims d = P.d;
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool ij = i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1;
    const int cx = ij ? c + d.sx() : c, cy = ij ? c + d.sy() : c;
    const float2 r = load_pair(rho, c), rx = load_pair(rho, cx), ry = load_pair(rho, cy);
    const float2 pc = load_pair(p, c), px = load_pair(p, cx), py = load_pair(p, cy);
    const int cz2 = ij && k + 2 < d.nz ? c + 2 : c + 1;
    const float rz2 = rho[cz2], pz2 = p[cz2];
    const float2 uc = load_pair(u, c), vc = load_pair(v, c), wc = load_pair(w, c);
    MomentumStencil a, b;
    a.rc = r.x; a.rx = rx.x; a.ry = ry.x; a.rz = r.y;
    a.pc = pc.x; a.px = px.x; a.py = py.x; a.pz = pc.y;
    a.uc = uc.x; a.vc = vc.x; a.wc = wc.x;
    b.rc = r.y; b.rx = rx.y; b.ry = ry.y; b.rz = rz2;
    b.pc = pc.y; b.px = px.y; b.py = py.y; b.pz = pz2;
    b.uc = uc.y; b.vc = vc.y; b.wc = wc.y;
    momentum_values<Policy>(P, a, i, j, k, c, p0, dp0_split, u, v, w, fuse_vertical);
    momentum_values<Policy>(P, b, i, j, k + 1, c + 1, p0, dp0_split, u, v, w, fuse_vertical);
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
