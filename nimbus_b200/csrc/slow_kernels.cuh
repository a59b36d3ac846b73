// Slow (advective) tendencies of the flat C-grid KW scheme and the Heun slow
// step, sm_100a.
//
// One slow step is two launches:
//   slow_predict : k1 = L(u^n); writes k1 and the predictor state
//                  x* = x^n + dt*k1 (u, v, w, p)            [prepare_slow_rk2_tendencies]
//   slow_correct : k2 = L(x*); t = 0.5f*(k2 + k1) in FP32 as the reference
//                  averages; x^n += dt*t                      [apply_slow_tendencies]
// L is CartesianCGrid3DScheme::compute_slow_tendencies
// (cartesian_cgrid_3d.cpp:1026-1401): fd5/fd3/fd1 upwind-biased momentum
// advection (derivative_operators.hpp:324-395), f-plane Coriolis on the
// perturbation wind, buoyancy -g(rho-rho0)/rho with vapour and hydrometeor
// loading on w, and centred -u.grad p for p.
#pragma once

#include "acoustic_fused.cuh"

namespace nimbus
{

struct SlowParams
{
    Dims d;
    double inv_dx, inv_dy, inv_dz;
    double dt;
    double coriolis_f;
    double frame_u, frame_v;
    double gravity;
    int moist;    // qv and qv0 present
    int loading;  // qc, qr present
    // FP32 form: the scalars above rounded once.
    float inv_dx_f, inv_dy_f, inv_dz_f, half_inv_dx_f, half_inv_dy_f, half_inv_dz_f, dt_f, coriolis_f_f, frame_u_f,
        frame_v_f, gravity_f;
    // fd3 / fd5 stencil scales inv_d / 6 and inv_d / 60 per axis (x, y, z),
    // formed once on the host exactly as the derivative operators form them.
    double d6[3], d60[3];
    float d6_f[3], d60_f[3];
};

__host__ __device__ inline void finish_fp32(SlowParams& S)
{
    S.inv_dx_f = (float)S.inv_dx;
    S.inv_dy_f = (float)S.inv_dy;
    S.inv_dz_f = (float)S.inv_dz;
    S.half_inv_dx_f = (float)(0.5 * S.inv_dx);
    S.half_inv_dy_f = (float)(0.5 * S.inv_dy);
    S.half_inv_dz_f = (float)(0.5 * S.inv_dz);
    S.dt_f = (float)S.dt;
    S.coriolis_f_f = (float)S.coriolis_f;
    S.frame_u_f = (float)S.frame_u;
    S.frame_v_f = (float)S.frame_v;
    S.gravity_f = (float)S.gravity;
    const double inv[3] = {S.inv_dx, S.inv_dy, S.inv_dz};
    const float inv_f[3] = {S.inv_dx_f, S.inv_dy_f, S.inv_dz_f};
    for (int a = 0; a < 3; ++a)
    {
        S.d6[a] = inv[a] / 6.0;
        S.d60[a] = inv[a] / 60.0;
        S.d6_f[a] = inv_f[a] / 6.0f;
        S.d60_f[a] = inv_f[a] / 60.0f;
    }
}

// upwind_dx/dy/dz (derivative_operators.hpp:324-395): fd5 upwind-biased in
// the interior, fd3 two points from a boundary, fd1 next to it, 0 on it.
// Away from the boundary the side is selected, not branched on: the a < 0
// stencils of fd5 and fd1 are the a >= 0 ones on the mirrored points with
// every intermediate negated (the reference's own operation order, so the
// result is bit-identical), and lanes with opposite winds do not diverge.
template <class real>
__device__ __forceinline__ real upwind_from(int half, real cc, real m1, real p1, real m2, real p2, real m3, real p3,
                                            real a, real inv_d, real inv_d6, real inv_d60)
{
    if (half <= 0) return (real)0;
    const bool pos = a >= (real)0;
    if (half == 1)
    {
        const real v = (cc - (pos ? m1 : p1)) * inv_d;
        return pos ? v : -v;
    }
    if (half == 2)
        return pos ? ((real)2 * p1 + (real)3 * cc - (real)6 * m1 + m2) * inv_d6
                   : (-p2 + (real)6 * p1 - (real)3 * cc - (real)2 * m1) * inv_d6;
    const real x1 = pos ? m1 : p1, x2 = pos ? m2 : p2, x3 = pos ? m3 : p3;
    const real y1 = pos ? p1 : m1, y2 = pos ? p2 : m2;
    const real v = ((real)-2 * x3 + (real)15 * x2 - (real)60 * x1 + (real)20 * cc + (real)30 * y1 - (real)3 * y2) *
                   inv_d60;
    return pos ? v : -v;
}

// The velocity and pressure fields seen from one cell: uvw(off) / p(off) are
// the values `off` cells away (k fastest).  PlanarState reads four arrays;
// PackedState one array of float4 {u, v, w, p} cells (the member engine's
// Heun predictor), where a stencil point's three velocities are one 16-byte
// load.
struct PlanarState
{
    const float* __restrict__ u;  // each at the cell
    const float* __restrict__ v;
    const float* __restrict__ w;
    const float* __restrict__ pr;
    __device__ __forceinline__ float3 uvw(int o) const { return make_float3(u[o], v[o], w[o]); }
    __device__ __forceinline__ float U(int o) const { return u[o]; }
    __device__ __forceinline__ float V(int o) const { return v[o]; }
    __device__ __forceinline__ float W(int o) const { return w[o]; }
    __device__ __forceinline__ float P(int o) const { return pr[o]; }
};

struct PackedState
{
    const float4* __restrict__ x;  // at the cell
    __device__ __forceinline__ float3 uvw(int o) const
    {
        const float4 t = x[o];
        return make_float3(t.x, t.y, t.z);
    }
    __device__ __forceinline__ float U(int o) const { return x[o].x; }
    __device__ __forceinline__ float V(int o) const { return x[o].y; }
    __device__ __forceinline__ float W(int o) const { return x[o].z; }
    __device__ __forceinline__ float P(int o) const { return x[o].w; }
};

// The upwind derivatives of u, v and w along one axis (stride, index idx of
// n), each with its own advecting wind: one set of stencil-point loads for
// the three fields.  Only points inside the grid are read (the half-width
// decides the order, as in the reference).
template <class real, class State>
__device__ __forceinline__ void upwind3(const State& X, int stride, int idx, int n, real au, real av, real aw,
                                        real inv_d, real inv_d6, real inv_d60, real& du, real& dv, real& dw)
{
    const int half = min(idx, n - 1 - idx);
    if (half <= 0)
    {
        du = dv = dw = (real)0;
        return;
    }
    const float3 cc = X.uvw(0), m1 = X.uvw(-stride), p1 = X.uvw(stride);
    float3 m2 = cc, p2 = cc, m3 = cc, p3 = cc;
    if (half >= 2)
    {
        m2 = X.uvw(-2 * stride);
        p2 = X.uvw(2 * stride);
    }
    if (half >= 3)
    {
        m3 = X.uvw(-3 * stride);
        p3 = X.uvw(3 * stride);
    }
    du = upwind_from<real>(half, cc.x, m1.x, p1.x, m2.x, p2.x, m3.x, p3.x, au, inv_d, inv_d6, inv_d60);
    dv = upwind_from<real>(half, cc.y, m1.y, p1.y, m2.y, p2.y, m3.y, p3.y, av, inv_d, inv_d6, inv_d60);
    dw = upwind_from<real>(half, cc.z, m1.z, p1.z, m2.z, p2.z, m3.z, p3.z, aw, inv_d, inv_d6, inv_d60);
}

// The four slow tendencies of cell c (zero outside their index ranges).
// Reference policy: the reference's FP64 interior arithmetic and order.  FP32
// policy: the same stencils in FP32, the base-state face averages formed in
// FP64 and rounded once.
template <class Policy, class State>
__device__ __forceinline__ void slow_tendencies_at(const SlowParams& S, int c, int i, int j, int k, const State& X,
                                                   const float* __restrict__ rho, const float* __restrict__ qv,
                                                   const float* __restrict__ qc, const float* __restrict__ qr,
                                                   const double* __restrict__ rho0, const double* __restrict__ qv0,
                                                   const double* __restrict__ u0, const double* __restrict__ v0,
                                                   float& out_u, float& out_v, float& out_w, float& out_p)
{
    using real = typename Policy::real;
    constexpr bool f32 = sizeof(real) == 4;
    const Dims d = S.d;
    out_u = out_v = out_w = out_p = 0.0f;
    if (!(i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1)) return;
    const int sx = d.sx(), sy = d.sy();
    const real q = (real)0.25, h = (real)0.5;
    real inv_dx, inv_dy, inv_dz, fu, fv, cf, x6, y6, z6, x60, y60, z60;
    if constexpr (f32)
    {
        inv_dx = S.inv_dx_f; inv_dy = S.inv_dy_f; inv_dz = S.inv_dz_f;
        fu = S.frame_u_f; fv = S.frame_v_f; cf = S.coriolis_f_f;
        x6 = S.d6_f[0]; y6 = S.d6_f[1]; z6 = S.d6_f[2];
        x60 = S.d60_f[0]; y60 = S.d60_f[1]; z60 = S.d60_f[2];
    }
    else
    {
        inv_dx = S.inv_dx; inv_dy = S.inv_dy; inv_dz = S.inv_dz;
        fu = S.frame_u; fv = S.frame_v; cf = S.coriolis_f;
        x6 = S.d6[0]; y6 = S.d6[1]; z6 = S.d6[2];
        x60 = S.d60[0]; y60 = S.d60[1]; z60 = S.d60[2];
    }
    auto store = [](real t) -> float {
        if constexpr (f32) return isfinite(t) ? t : 0.0f;
        else return (float)finite_or_zero((double)t);
    };
    // Advecting winds of du (x-face), dv (y-face) and dw (z-face).
    const real ux_u = (real)X.U(0);
    const real uy_u = q * ((real)X.V(-sy) + (real)X.V(0) + (real)X.V(sx - sy) + (real)X.V(sx));
    const real tux_u = ux_u - fu, tuy_u = uy_u - fv;
    const real wx = (k == 0) ? q * ((real)X.W(0) + (real)X.W(sx))
                             : q * ((real)X.W(-1) + (real)X.W(0) + (real)X.W(sx - 1) + (real)X.W(sx));
    const real vy = (real)X.V(0);
    const real ux_v = q * ((real)X.U(-sx) + (real)X.U(0) + (real)X.U(sy - sx) + (real)X.U(sy));
    const real tvy = vy - fv, tux_v = ux_v - fu;
    const real wy = (k == 0) ? q * ((real)X.W(0) + (real)X.W(sy))
                             : q * ((real)X.W(-1) + (real)X.W(0) + (real)X.W(sy - 1) + (real)X.W(sy));
    const real wz = (real)X.W(0);
    const real ux_w = q * ((real)X.U(-sx) + (real)X.U(0) + (real)X.U(1 - sx) + (real)X.U(1));
    const real uy_w = q * ((real)X.V(-sy) + (real)X.V(0) + (real)X.V(1 - sy) + (real)X.V(1));
    const real tux_w = ux_w - fu, tuy_w = uy_w - fv;
    // Upwind derivatives, one axis at a time for the three fields.
    real dxu, dxv, dxw, dyu, dyv, dyw, dzu, dzv, dzw;
    upwind3<real>(X, sx, i, d.nx, tux_u, tux_v, tux_w, inv_dx, x6, x60, dxu, dxv, dxw);
    upwind3<real>(X, sy, j, d.ny, tuy_u, tvy, tuy_w, inv_dy, y6, y60, dyu, dyv, dyw);
    if (k == 0)
    {
        dzu = (wx >= (real)0) ? (real)0 : ((real)X.U(1) - (real)X.U(0)) * inv_dz;
        dzv = (wy >= (real)0) ? (real)0 : ((real)X.V(1) - (real)X.V(0)) * inv_dz;
        dzw = (wz >= (real)0) ? ((real)X.W(0) - (real)0) * inv_dz : ((real)X.W(1) - (real)X.W(0)) * inv_dz;
    }
    else upwind3<real>(X, 1, k, d.nz, wx, wy, wz, inv_dz, z6, z60, dzu, dzv, dzw);
    // du at the x-face
    {
        const real v0k = v0 ? (real)v0[k] : (real)0;
        const real du = -tux_u * dxu - tuy_u * dyu - wx * dzu + cf * (uy_u - v0k);
        out_u = store(du);
    }
    // dv at the y-face
    {
        const real u0k = u0 ? (real)u0[k] : (real)0;
        const real dv = -tux_v * dxv - tvy * dyv - wy * dzv - cf * (ux_v - u0k);
        out_v = store(dv);
    }
    // dw at the z-face
    {
        if constexpr (f32)
        {
            const float g = S.gravity_f;
            const float rho_face = 0.5f * (rho[c] + rho[c + 1]);
            const float rho_s = (isfinite(rho_face) && rho_face > 1.0e-6f) ? rho_face : 1.0f;
            const float rho0_face = (float)(0.5 * (rho0[k] + rho0[k + 1]));
            float forcing = -g * (rho_face - rho0_face) / rho_s;
            if (S.moist)
            {
                const float qf = 0.5f * (qv[c] + qv[c + 1]);
                const float q0f = (float)(0.5 * ((double)(float)qv0[k] + (double)(float)qv0[k + 1]));
                forcing += g * 0.608f * (qf - q0f);
            }
            if (S.loading)
                forcing += -g * (0.5f * ((qc[c] + qr[c]) + (qc[c + 1] + qr[c + 1])));
            const real dw = -tux_w * dxw - tuy_w * dyw - wz * dzw + forcing;
            out_w = store(dw);
        }
        else
        {
            const double rho_face = 0.5 * ((double)rho[c] + (double)rho[c + 1]);
            const double rho_s = safe_rho(rho_face);
            const double rho0_face = 0.5 * (rho0[k] + rho0[k + 1]);
            const double g = S.gravity;
            const double buoy = -g * (rho_face - rho0_face) / rho_s;
            double moist = 0.0;
            if (S.moist)
            {
                const double qf = 0.5 * ((double)qv[c] + (double)qv[c + 1]);
                const double q0f = 0.5 * ((double)(float)qv0[k] + (double)(float)qv0[k + 1]);
                moist = g * 0.608 * (qf - q0f);
            }
            double load = 0.0;
            if (S.loading)
            {
                const double lo = (double)qc[c] + (double)qr[c] + 0.0 + 0.0 + 0.0 + 0.0;
                const double hi = (double)qc[c + 1] + (double)qr[c + 1] + 0.0 + 0.0 + 0.0 + 0.0;
                load = -g * (0.5 * (lo + hi));
            }
            const real dw = -tux_w * dxw - tuy_w * dyw - wz * dzw + (real)buoy + (real)moist + (real)load;
            out_w = store(dw);
        }
    }
    // dp at the centre
    if (k >= 1)
    {
        const real uc = h * ((real)X.U(0) + (real)X.U(-sx));
        const real vc = h * ((real)X.V(0) + (real)X.V(-sy));
        const real tuc = uc - fu, tvc = vc - fv;
        const real wc = h * ((real)X.W(0) + (real)X.W(-1));
        real hx, hy, hz;
        if constexpr (f32)
        {
            hx = S.half_inv_dx_f; hy = S.half_inv_dy_f; hz = S.half_inv_dz_f;
        }
        else
        {
            hx = (real)(0.5 * S.inv_dx); hy = (real)(0.5 * S.inv_dy); hz = (real)(0.5 * S.inv_dz);
        }
        const real dpdx = ((real)X.P(sx) - (real)X.P(-sx)) * hx;
        const real dpdy = ((real)X.P(sy) - (real)X.P(-sy)) * hy;
        const real dpdz = ((real)X.P(1) - (real)X.P(-1)) * hz;
        out_p = store(-tuc * dpdx - tvc * dpdy - wc * dpdz);
    }
}

// x + dt * t (apply_slow_tendencies_cpu, dynamics.cpp:1955-2080: a
// non-finite tendency counts as zero).  Reference policy: FP64 add rounded
// once; FP32 policy: one FMA.
template <class Policy>
__device__ __forceinline__ float slow_apply_one(const SlowParams& S, float x, float t)
{
    if constexpr (sizeof(typename Policy::real) == 4) return __fmaf_rn(isfinite(t) ? t : 0.0f, S.dt_f, x);
    else return (float)((double)x + finite_or_zero((double)t) * S.dt);
}

// The slow tendencies applied over dt with the CPU's arithmetic
// (apply_slow_tendencies_cpu, dynamics.cpp:1955-2095): the horizontal
// tendencies gain the boundary-layer ones (du + du_pbl in FP64; a missing
// field counts as zero, added all the same so that a -0.0 sums as it does
// there), a non-finite tendency counts as zero when sanitize is on, and each
// field takes x + t dt in FP64 rounded once to FP32.
static __global__ void __launch_bounds__(256) slow_apply_kernel(
    float* __restrict__ u, float* __restrict__ v, float* __restrict__ w, float* __restrict__ p,
    const float* __restrict__ du, const float* __restrict__ dv, const float* __restrict__ dw,
    const float* __restrict__ dp, const float* __restrict__ du_pbl, const float* __restrict__ dv_pbl, long long n,
    double dt, int sanitize)
{
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    {
        double tu = (double)du[c] + (du_pbl ? (double)du_pbl[c] : 0.0);
        double tv = (double)dv[c] + (dv_pbl ? (double)dv_pbl[c] : 0.0);
        double tw = (double)dw[c];
        double tp = (double)dp[c];
        if (sanitize)
        {
            tu = finite_or_zero(tu);
            tv = finite_or_zero(tv);
            tw = finite_or_zero(tw);
            tp = finite_or_zero(tp);
        }
        u[c] = (float)((double)u[c] + tu * dt);
        v[c] = (float)((double)v[c] + tv * dt);
        w[c] = (float)((double)w[c] + tw * dt);
        p[c] = (float)((double)p[c] + tp * dt);
    }
}

// k1 at cell c and, when su is given, the predictor state x* = x + dt*k1.
// Also the plain tendency evaluation (su == null).
template <class Policy>
__device__ __forceinline__ void slow_predict_cell(
    const SlowParams& S, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const float* __restrict__ rho, const float* __restrict__ p, const float* __restrict__ qv,
    const float* __restrict__ qc, const float* __restrict__ qr, const double* __restrict__ rho0,
    const double* __restrict__ qv0, const double* __restrict__ u0, const double* __restrict__ v0,
    float* __restrict__ k1u, float* __restrict__ k1v, float* __restrict__ k1w, float* __restrict__ k1p,
    float* __restrict__ su, float* __restrict__ sv, float* __restrict__ sw, float* __restrict__ sp, int c)
{
    int i, j, k;
    decompose(S.d, c, i, j, k);
    float tu, tv, tw, tp;
    slow_tendencies_at<Policy>(S, c, i, j, k, PlanarState{u + c, v + c, w + c, p + c}, rho, qv, qc, qr, rho0, qv0, u0,
                               v0, tu, tv, tw, tp);
    k1u[c] = tu;
    k1v[c] = tv;
    k1w[c] = tw;
    k1p[c] = tp;
    if (su != nullptr)
    {
        su[c] = slow_apply_one<Policy>(S, u[c], tu);
        sv[c] = slow_apply_one<Policy>(S, v[c], tv);
        sw[c] = slow_apply_one<Policy>(S, w[c], tw);
        sp[c] = slow_apply_one<Policy>(S, p[c], tp);
    }
}

template <class Policy>
static __global__ void __launch_bounds__(256) slow_predict_kernel(
    SlowParams S, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const float* __restrict__ rho, const float* __restrict__ p, const float* __restrict__ qv,
    const float* __restrict__ qc, const float* __restrict__ qr, const double* __restrict__ rho0,
    const double* __restrict__ qv0, const double* __restrict__ u0, const double* __restrict__ v0,
    float* __restrict__ k1u, float* __restrict__ k1v, float* __restrict__ k1w, float* __restrict__ k1p,
    float* __restrict__ su, float* __restrict__ sv, float* __restrict__ sw, float* __restrict__ sp)
{
    const int n = S.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        slow_predict_cell<Policy>(S, u, v, w, rho, p, qv, qc, qr, rho0, qv0, u0, v0, k1u, k1v, k1w, k1p, su, sv, sw,
                                  sp, c);
}

// k2 at the predictor state, the FP32 Heun average and its application to
// cell c's own u, v, w, p (in place: the stencil reads only the predictor).
template <class Policy>
__device__ __forceinline__ void slow_correct_cell(
    const SlowParams& S, const float* __restrict__ su, const float* __restrict__ sv, const float* __restrict__ sw,
    const float* __restrict__ rho, const float* __restrict__ sp, const float* __restrict__ qv,
    const float* __restrict__ qc, const float* __restrict__ qr, const double* __restrict__ rho0,
    const double* __restrict__ qv0, const double* __restrict__ u0, const double* __restrict__ v0,
    const float* __restrict__ k1u, const float* __restrict__ k1v, const float* __restrict__ k1w,
    const float* __restrict__ k1p, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
    float* __restrict__ p, float* __restrict__ tu_out, float* __restrict__ tv_out, float* __restrict__ tw_out,
    float* __restrict__ tp_out, int c)
{
    int i, j, k;
    decompose(S.d, c, i, j, k);
    float tu, tv, tw, tp;
    slow_tendencies_at<Policy>(S, c, i, j, k, PlanarState{su + c, sv + c, sw + c, sp + c}, rho, qv, qc, qr, rho0, qv0,
                               u0, v0, tu, tv, tw, tp);
    tu = __fmul_rn(0.5f, __fadd_rn(tu, k1u[c]));
    tv = __fmul_rn(0.5f, __fadd_rn(tv, k1v[c]));
    tw = __fmul_rn(0.5f, __fadd_rn(tw, k1w[c]));
    tp = __fmul_rn(0.5f, __fadd_rn(tp, k1p[c]));
    if (tu_out != nullptr)
    {
        tu_out[c] = tu;
        tv_out[c] = tv;
        tw_out[c] = tw;
        tp_out[c] = tp;
    }
    u[c] = slow_apply_one<Policy>(S, u[c], tu);
    v[c] = slow_apply_one<Policy>(S, v[c], tv);
    w[c] = slow_apply_one<Policy>(S, w[c], tw);
    p[c] = slow_apply_one<Policy>(S, p[c], tp);
}

// The member engine's form: k1 and the predictor as one float4 {u, v, w, p}
// per cell, so the corrector reads a stencil point's predictor velocities
// with one load.  Same arithmetic as slow_predict_cell / slow_correct_cell.
template <class Policy>
__device__ __forceinline__ void slow_predict_packed(
    const SlowParams& S, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const float* __restrict__ rho, const float* __restrict__ p, const float* __restrict__ qv,
    const float* __restrict__ qc, const float* __restrict__ qr, const double* __restrict__ rho0,
    const double* __restrict__ qv0, const double* __restrict__ u0, const double* __restrict__ v0,
    float4* __restrict__ k1, float4* __restrict__ xs, int c)
{
    int i, j, k;
    decompose(S.d, c, i, j, k);
    float tu, tv, tw, tp;
    slow_tendencies_at<Policy>(S, c, i, j, k, PlanarState{u + c, v + c, w + c, p + c}, rho, qv, qc, qr, rho0, qv0, u0,
                               v0, tu, tv, tw, tp);
    k1[c] = make_float4(tu, tv, tw, tp);
    xs[c] = make_float4(slow_apply_one<Policy>(S, u[c], tu), slow_apply_one<Policy>(S, v[c], tv),
                        slow_apply_one<Policy>(S, w[c], tw), slow_apply_one<Policy>(S, p[c], tp));
}

template <class Policy>
__device__ __forceinline__ void slow_correct_packed(
    const SlowParams& S, const float4* __restrict__ xs, const float* __restrict__ rho, const float* __restrict__ qv,
    const float* __restrict__ qc, const float* __restrict__ qr, const double* __restrict__ rho0,
    const double* __restrict__ qv0, const double* __restrict__ u0, const double* __restrict__ v0,
    const float4* __restrict__ k1, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
    float* __restrict__ p, int c)
{
    int i, j, k;
    decompose(S.d, c, i, j, k);
    float tu, tv, tw, tp;
    slow_tendencies_at<Policy>(S, c, i, j, k, PackedState{xs + c}, rho, qv, qc, qr, rho0, qv0, u0, v0, tu, tv, tw, tp);
    const float4 a = k1[c];
    tu = __fmul_rn(0.5f, __fadd_rn(tu, a.x));
    tv = __fmul_rn(0.5f, __fadd_rn(tv, a.y));
    tw = __fmul_rn(0.5f, __fadd_rn(tw, a.z));
    tp = __fmul_rn(0.5f, __fadd_rn(tp, a.w));
    u[c] = slow_apply_one<Policy>(S, u[c], tu);
    v[c] = slow_apply_one<Policy>(S, v[c], tv);
    w[c] = slow_apply_one<Policy>(S, w[c], tw);
    p[c] = slow_apply_one<Policy>(S, p[c], tp);
}

template <class Policy>
static __global__ void __launch_bounds__(256) slow_correct_kernel(
    SlowParams S, const float* __restrict__ su, const float* __restrict__ sv, const float* __restrict__ sw,
    const float* __restrict__ rho, const float* __restrict__ sp, const float* __restrict__ qv,
    const float* __restrict__ qc, const float* __restrict__ qr, const double* __restrict__ rho0,
    const double* __restrict__ qv0, const double* __restrict__ u0, const double* __restrict__ v0,
    const float* __restrict__ k1u, const float* __restrict__ k1v, const float* __restrict__ k1w,
    const float* __restrict__ k1p, float* __restrict__ u, float* __restrict__ v, float* __restrict__ w,
    float* __restrict__ p, float* __restrict__ tu_out, float* __restrict__ tv_out, float* __restrict__ tw_out,
    float* __restrict__ tp_out)
{
    const int n = S.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        slow_correct_cell<Policy>(S, su, sv, sw, rho, sp, qv, qc, qr, rho0, qv0, u0, v0, k1u, k1v, k1w, k1p, u, v, w,
                                  p, tu_out, tv_out, tw_out, tp_out, c);
}

// ---- The slow-tendency operator of the device route ------------------------
//
// CartesianCGrid3DScheme::compute_slow_tendencies (cartesian_cgrid_3d.cpp:835-925)
// hands a supporting backend dispatch_cartesian_cgrid_slow_tendencies: FP32
// fields, FP32 base profiles (rho0, qv0, u0, v0 -- the wind profiles one zero
// when the sounding has none), the host-summed hydrometeor loading, FP32
// spacings, f at grid y = 0 and the beta-plane df/dy.  The operator's
// arithmetic is the reference's device form of the scheme
// (vulkan/shaders/compute/dynamics/cartesian_cgrid_slow_tendencies.comp:139-391):
// the same upwind-biased momentum advection and centred pressure advection
// as the CPU route, in FP32, every output written (zero where the scheme
// does not act; drho_dt is zero on this path).
struct SlowDispatchParams
{
    Dims d;
    float inv_dx, inv_dy, inv_dz, inv_2dx, inv_2dy, inv_2dz;
    float d6[3], d60[3];  // inv_d / 6 and inv_d / 60 per axis, as the operator forms them
    float dy, g, f0, beta, frame_u, frame_v;
    int has_moisture, has_loading, wind_profiles, emit_advection;
};

static __global__ void __launch_bounds__(256) slow_tendencies_dispatch_kernel(
    SlowDispatchParams S, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const float* __restrict__ rho, const float* __restrict__ p, const float* __restrict__ rho0,
    const float* __restrict__ qv0, const float* __restrict__ u0, const float* __restrict__ v0,
    const float* __restrict__ qv, const float* __restrict__ loading, float* __restrict__ du_dt,
    float* __restrict__ dv_dt, float* __restrict__ dw_dt, float* __restrict__ drho_dt, float* __restrict__ dp_dt,
    float* __restrict__ du_adv, float* __restrict__ dv_adv, float* __restrict__ dw_adv)
{
    const Dims d = S.d;
    const int n = d.cells(), sx = d.sx(), sy = d.sy();
    auto clean = [](float t) { return isfinite(t) ? t : 0.0f; };
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        float du = 0.0f, dv = 0.0f, dw = 0.0f, dp = 0.0f, au = 0.0f, av = 0.0f, aw = 0.0f;
        if (i >= 1 && i <= d.nx - 2 && j >= 1 && j <= d.ny - 2 && k <= d.nz - 2)
        {
            const PlanarState X{u + c, v + c, w + c, p + c};
            const float u0k = S.wind_profiles ? u0[k] : 0.0f, v0k = S.wind_profiles ? v0[k] : 0.0f;
            // Advecting winds at the x-, y- and z-faces.
            const float ux = X.U(0);
            const float uy_x = 0.25f * (X.V(-sy) + X.V(0) + X.V(sx - sy) + X.V(sx));
            const float w_x = (k == 0) ? 0.25f * (X.W(0) + X.W(sx))
                                       : 0.25f * (X.W(-1) + X.W(0) + X.W(sx - 1) + X.W(sx));
            const float vy = X.V(0);
            const float ux_y = 0.25f * (X.U(-sx) + X.U(0) + X.U(sy - sx) + X.U(sy));
            const float w_y = (k == 0) ? 0.25f * (X.W(0) + X.W(sy))
                                       : 0.25f * (X.W(-1) + X.W(0) + X.W(sy - 1) + X.W(sy));
            const float wz = X.W(0);
            const float ux_w = 0.25f * (X.U(-sx) + X.U(0) + X.U(1 - sx) + X.U(1));
            const float uy_w = 0.25f * (X.V(-sy) + X.V(0) + X.V(1 - sy) + X.V(1));
            float dxu, dxv, dxw, dyu, dyv, dyw, dzu, dzv, dzw;
            upwind3<float>(X, sx, i, d.nx, ux, ux_y, ux_w, S.inv_dx, S.d6[0], S.d60[0], dxu, dxv, dxw);
            upwind3<float>(X, sy, j, d.ny, uy_x, vy, uy_w, S.inv_dy, S.d6[1], S.d60[1], dyu, dyv, dyw);
            if (k == 0)
            {
                dzu = (w_x >= 0.0f) ? 0.0f : (X.U(1) - ux) * S.inv_dz;
                dzv = (w_y >= 0.0f) ? 0.0f : (X.V(1) - vy) * S.inv_dz;
                dzw = (wz >= 0.0f) ? X.W(0) * S.inv_dz : (X.W(1) - X.W(0)) * S.inv_dz;
            }
            else upwind3<float>(X, 1, k, d.nz, w_x, w_y, wz, S.inv_dz, S.d6[2], S.d60[2], dzu, dzv, dzw);
            // du at the x-face
            au = -(ux - S.frame_u) * dxu - (uy_x - S.frame_v) * dyu - w_x * dzu;
            float cor_x = S.f0 * (uy_x - v0k);
            if (S.beta != 0.0f)
            {
                const float f_lo = S.f0 + S.beta * ((float)j + 0.25f) * S.dy;
                const float f_hi = S.f0 + S.beta * ((float)j + 0.75f) * S.dy;
                cor_x = 0.25f * (f_lo * (X.V(-sy) + X.V(sx - sy) - 2.0f * v0k) +
                                 f_hi * (X.V(0) + X.V(sx) - 2.0f * v0k));
            }
            du = au + cor_x;
            // dv at the y-face
            av = -(ux_y - S.frame_u) * dxv - (vy - S.frame_v) * dyv - w_y * dzv;
            float cor_y = S.f0 * (ux_y - u0k);
            if (S.beta != 0.0f)
            {
                const float f_lo = S.f0 + S.beta * ((float)j + 0.75f) * S.dy;
                const float f_hi = S.f0 + S.beta * ((float)j + 1.25f) * S.dy;
                cor_y = 0.25f * (f_lo * (X.U(-sx) + X.U(0) - 2.0f * u0k) + f_hi * (X.U(sy - sx) + X.U(sy) - 2.0f * u0k));
            }
            dv = av - cor_y;
            // dw at the z-face: advection, buoyancy, vapour and loading
            aw = -(ux_w - S.frame_u) * dxw - (uy_w - S.frame_v) * dyw - wz * dzw;
            const float rho_face = 0.5f * (rho[c] + rho[c + 1]);
            const float rho_safe = (isfinite(rho_face) && rho_face > 1.0e-6f) ? rho_face : 1.0f;
            const float rho0_face = 0.5f * (rho0[k] + rho0[k + 1]);
            const float buoyancy = -S.g * (rho_face - rho0_face) / rho_safe;
            float moisture = 0.0f, load = 0.0f;
            if (S.has_moisture)
                moisture = S.g * 0.608f * (0.5f * (qv[c] + qv[c + 1]) - 0.5f * (qv0[k] + qv0[k + 1]));
            if (S.has_loading) load = -S.g * 0.5f * (loading[c] + loading[c + 1]);
            dw = aw + buoyancy + moisture + load;
            // dp at the cell centre (centred advection), levels 1 .. nz-2
            if (k >= 1)
            {
                const float uc = 0.5f * (X.U(0) + X.U(-sx));
                const float vc = 0.5f * (X.V(0) + X.V(-sy));
                const float wc = 0.5f * (X.W(0) + X.W(-1));
                const float dpdx = (X.P(sx) - X.P(-sx)) * S.inv_2dx;
                const float dpdy = (X.P(sy) - X.P(-sy)) * S.inv_2dy;
                const float dpdz = (X.P(1) - X.P(-1)) * S.inv_2dz;
                dp = -(uc - S.frame_u) * dpdx - (vc - S.frame_v) * dpdy - wc * dpdz;
            }
        }
        du_dt[c] = clean(du);
        dv_dt[c] = clean(dv);
        dw_dt[c] = clean(dw);
        dp_dt[c] = clean(dp);
        if (drho_dt) drho_dt[c] = 0.0f;
        if (S.emit_advection)
        {
            du_adv[c] = clean(au);
            dv_adv[c] = clean(av);
            dw_adv[c] = clean(aw);
        }
    }
}

}  // namespace nimbus
