// Smagorinsky SGS closure on a flat C-grid (stability correction "none"):
// eddy coefficients, conservative live-density stress and scalar diffusion
// tendencies, the forward-Euler application and the explicit stability
// reductions.  Reference: SmagorinskyScheme::compute_eddy_coefficients
// (src/turbulence/schemes/smagorinsky/smagorinsky.cpp:494-571),
// compute_directional_strain_sq_centered, compute_momentum_diffusion_tendencies
// and compute_scalar_diffusion_tendencies
// (src/turbulence/base/eddy_viscosity.cpp:1253-1400,1532-2090),
// apply_sgs_tendencies_cpu and compute_sgs_explicit_stability
// (src/core/orchestration/dynamics/sgs_apply.cpp:436-956,1483-1973).
//
// FP64 arithmetic over FP32 storage in the reference's operation order
// (compiled without FMA contraction): bit-identical to the CPU solver.  The
// closure kernels are templated on their arithmetic type R: R = double is that
// reference form, R = float the FP32 form (same operations in FP32).  Every
// stress or flux the reference carries along a column (its rolling lower
// T13 / T23 / T33) is recomputed here from the same expression, which gives
// the same binary64 value, so each cell is independent: one thread per cell;
// within a cell the three corner edge stresses two faces share are formed once.
#pragma once

#include "stencil_common.cuh"

namespace nimbus
{

struct SgsParams
{
    Dims d;
    double dx, dy;
    const double* dz;     // [nz] cell thickness (device)
    const double* delta;  // [nz] filter width (device, formed on the host)
    int use_h, use_v;
    int px, py;           // periodic x / y
    int open[4];          // W, E, S, N lateral faces open (scalar fluxes pass)
    double Cs, Pr_t, Sc_t, nu_max, K_max;
    // FP32 form: reciprocals of the spacings (it multiplies where the
    // reference form divides).
    float inv_dx_f, inv_dy_f;
    const float* inv_dz_f;   // [nz] (device)
    const float* inv_dzc_f;  // [nz] (device): 1 / distance between centres k and k+1
};

// A divisor: the reference form divides by d; the FP32 form multiplies by the
// FP32 reciprocal (one rounding more, no division sequence).
template <class R>
struct Recip
{
    double d;
    float inv;
};

template <class R>
__device__ __forceinline__ R operator/(R x, Recip<R> r)
{
    if constexpr (sizeof(R) == sizeof(float))
        return x * r.inv;
    else
        return x / R(r.d);
}

// Neighbour rows (eddy_viscosity.cpp:69-105): clamped to the allocated
// range, or on a periodic axis wrapped over the physical rows 1..n-2.
__device__ __forceinline__ int sgs_prev(int i, int n, int periodic)
{
    if (!periodic) return i > 0 ? i - 1 : 0;
    return i <= 1 ? n - 2 : (i - 1 < n - 2 ? i - 1 : n - 2);
}

__device__ __forceinline__ int sgs_next(int i, int n, int periodic)
{
    if (!periodic) return i + 1 < n - 1 ? i + 1 : n - 1;
    return i >= n - 2 ? 1 : (i + 1 > 1 ? i + 1 : 1);
}

template <class R>
struct SgsAt
{
    const SgsParams& P;
    __device__ __forceinline__ int at(int i, int j, int k) const { return P.d.at(i, j, k); }
    __device__ __forceinline__ R f(const float* x, int i, int j, int k) const
    {
        return (R)__ldg(x + at(i, j, k));
    }
    // w with the implicit ground face w[-1] = 0.
    __device__ __forceinline__ R wf(const float* w, int i, int j, int k) const
    {
        return k < 0 ? R(0.0) : f(w, i, j, k);
    }
    __device__ __forceinline__ Recip<R> DX() const { return {P.dx, P.inv_dx_f}; }
    __device__ __forceinline__ Recip<R> DY() const { return {P.dy, P.inv_dy_f}; }
    __device__ __forceinline__ Recip<R> DZ(int k) const { return {P.dz[k], P.inv_dz_f[k]}; }
    // Distance between centres k and k+1 as a divisor (the reference form
    // divides by 0.5 (dz_k + dz_k+1)).  Defined for k < nz - 1 only: every
    // caller guards that; the FP32 table holds NaN at nz - 1 and dz has no
    // element nz.
    __device__ __forceinline__ Recip<R> DZC(int k) const { return {0.5 * (P.dz[k] + P.dz[k + 1]), P.inv_dzc_f[k]}; }
    __device__ __forceinline__ R dzc(int k) const { return R(0.5) * (R(P.dz[k]) + R(P.dz[k + 1])); }
    // mu = rho nu at a centre; on an xy edge (four-point mean); on an xz or yz
    // edge (pair means of the two levels, weighted by the other level's
    // thickness).
    __device__ __forceinline__ R mu(const float* rho, const float* nu, int i, int j, int k) const
    {
        return f(rho, i, j, k) * f(nu, i, j, k);
    }
    __device__ __forceinline__ R mu_xy(const float* rho, const float* nu, int i, int j, int k) const
    {
        const int i1 = sgs_next(i, P.d.nx, P.px), j1 = sgs_next(j, P.d.ny, P.py);
        return R(0.25) * (mu(rho, nu, i, j, k) + mu(rho, nu, i1, j, k) + mu(rho, nu, i, j1, k) + mu(rho, nu, i1, j1, k));
    }
    __device__ __forceinline__ R mu_z(const float* rho, const float* nu, int i, int j, int i1, int j1,
                                           int k) const
    {
        const R lo = R(0.5) * (mu(rho, nu, i, j, k) + mu(rho, nu, i1, j1, k));
        const R up = R(0.5) * (mu(rho, nu, i, j, k + 1) + mu(rho, nu, i1, j1, k + 1));
        return (R(P.dz[k + 1]) * lo + R(P.dz[k]) * up) / (R(P.dz[k]) + R(P.dz[k + 1]));
    }
};

// Strain-rate square at a scalar centre (compute_directional_strain_sq_centered).
template <class R>
__device__ R sgs_strain_sq(const SgsParams& P, const float* u, const float* v, const float* w, int i, int j,
                                int k)
{
    const SgsAt<R> A{P};
    const int nx = P.d.nx, ny = P.d.ny, nz = P.d.nz;
    const int jm = sgs_prev(j, ny, P.py), im = sgs_prev(i, nx, P.px);
    const R s11 = (A.f(u, i, j, k) - A.f(u, im, j, k)) / A.DX();
    const R s22 = (A.f(v, i, j, k) - A.f(v, i, jm, k)) / A.DY();
    const R s33 = (A.wf(w, i, j, k) - A.wf(w, i, j, k - 1)) / A.DZ(k);
    R s12[4];
    {
        const int ie[4] = {im, im, i, i}, je[4] = {jm, j, jm, j};
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
            const int ii = ie[e], jj = je[e];
            const int jj1 = sgs_next(jj, ny, P.py), ii1 = sgs_next(ii, nx, P.px);
            const R dudy = (A.f(u, ii, jj1, k) - A.f(u, ii, jj, k)) / A.DY();
            const R dvdx = (A.f(v, ii1, jj, k) - A.f(v, ii, jj, k)) / A.DX();
            s12[e] = R(0.5) * (dudy + dvdx);
        }
    }
    R xz0[4], xz1[4], yz0[4], yz1[4];
    {
        const int xi[4] = {im, im, i, i}, yj[4] = {jm, jm, j, j}, ke[4] = {k - 1, k, k - 1, k};
#pragma unroll
        for (int e = 0; e < 4; ++e)
        {
            const int kk = ke[e];
            if (kk < 0 || kk >= nz - 1)
            {
                xz0[e] = xz1[e] = yz0[e] = yz1[e] = R(0.0);
                continue;
            }
            const Recip<R> dzc = A.DZC(kk);
            const int ii = xi[e], ii1 = sgs_next(ii, nx, P.px);
            xz0[e] = (A.f(u, ii, j, kk + 1) - A.f(u, ii, j, kk)) / dzc;
            xz1[e] = (A.wf(w, ii1, j, kk) - A.wf(w, ii, j, kk)) / A.DX();
            const int jj = yj[e], jj1 = sgs_next(jj, ny, P.py);
            yz0[e] = (A.f(v, i, jj, kk + 1) - A.f(v, i, jj, kk)) / dzc;
            yz1[e] = (A.wf(w, i, jj1, kk) - A.wf(w, i, jj, kk)) / A.DY();
        }
    }
    const R s12_sq = R(0.25) * (s12[0] * s12[0] + s12[1] * s12[1] + s12[2] * s12[2] + s12[3] * s12[3]);
    auto avg_sq = [](const R (&g)[4]) { return R(0.25) * (g[0] * g[0] + g[1] * g[1] + g[2] * g[2] + g[3] * g[3]); };
    if (P.use_h && !P.use_v) return R(2.0) * (s11 * s11 + s22 * s22) + R(4.0) * s12_sq + avg_sq(xz1) + avg_sq(yz1);
    if (P.use_v && !P.use_h) return avg_sq(xz0) + avg_sq(yz0) + R(2.0) * s33 * s33;
    R sxz[4], syz[4];
#pragma unroll
    for (int e = 0; e < 4; ++e)
    {
        const R a = R(0.5) * (xz0[e] + xz1[e]);
        const R b = R(0.5) * (yz0[e] + yz1[e]);
        sxz[e] = a * a;
        syz[e] = b * b;
    }
    const R s13_sq = R(0.25) * (sxz[0] + sxz[1] + sxz[2] + sxz[3]);
    const R s23_sq = R(0.25) * (syz[0] + syz[1] + syz[2] + syz[3]);
    return R(2.0) * (s11 * s11 + s22 * s22 + s33 * s33) + R(4.0) * (s12_sq + s13_sq + s23_sq);
}

template <class R>
__device__ __forceinline__ R sgs_min(R a, R b) { return b < a ? b : a; }  // std::min

// Eddy coefficients of every cell; a cell whose inputs break the reference's
// field contract (validate_scheme_inputs, eddy_viscosity.cpp:1088-1175) or
// whose coefficient is not finite raises kStatusSgsInvalid.
template <class R>
__global__ void __launch_bounds__(256, 3) sgs_coefficients_kernel(SgsParams P, const float* __restrict__ u,
                                                               const float* __restrict__ v,
                                                               const float* __restrict__ w,
                                                               const float* __restrict__ theta,
                                                               const float* __restrict__ qv,
                                                               const float* __restrict__ rho, float* __restrict__ nu_t,
                                                               float* __restrict__ K_theta, float* __restrict__ K_q,
                                                               unsigned* status)
{
    const int n = P.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(P.d, c, i, j, k);
        const float th = theta[c], r = rho[c];
        bool bad = !isfinite(u[c]) || !isfinite(v[c]) || !isfinite(w[c]) || !isfinite(th) || !(th > 0.0f) ||
                   !isfinite(r) || !(r > 0.0f) || (qv && (!isfinite(qv[c]) || qv[c] < 0.0f));
        const R strain = sqrt(sgs_strain_sq<R>(P, u, v, w, i, j, k));
        R nu = R(P.Cs) * R(P.Cs) * R(P.delta[k]) * R(P.delta[k]) * strain * R(1.0);
        bad |= !isfinite(strain) || !isfinite(nu);
        nu = sgs_min(nu, R(P.nu_max));
        const R kt = nu / R(P.Pr_t), kq = nu / R(P.Sc_t);
        bad |= !isfinite(kt) || !isfinite(kq);
        if (bad) atomicOr(status, kStatusSgsInvalid);
        nu_t[c] = (float)nu;
        K_theta[c] = (float)sgs_min(kt, R(P.K_max));
        K_q[c] = (float)sgs_min(kq, R(P.K_max));
    }
}

// Scalar diffusion tendency at one cell (compute_scalar_diffusion_tendencies).
template <class R>
__device__ R sgs_scalar_rate(const SgsParams& P, const float* rho, const float* K, const float* phi, int i,
                                  int j, int k)
{
    const SgsAt<R> A{P};
    const int nx = P.d.nx, ny = P.d.ny, nz = P.d.nz;
    const int jmm = !P.py && !P.open[2] && j == 1 ? j : sgs_prev(j, ny, P.py);
    const int jpp = !P.py && !P.open[3] && j == ny - 2 ? j : sgs_next(j, ny, P.py);
    const int imm = !P.px && !P.open[0] && i == 1 ? i : sgs_prev(i, nx, P.px);
    const int ipp = !P.px && !P.open[1] && i == nx - 2 ? i : sgs_next(i, nx, P.px);
    auto tr = [&](int ii, int jj, int kk) { return A.f(rho, ii, jj, kk) * A.f(K, ii, jj, kk); };
    R div = R(0.0);
    if (P.use_h)
    {
        const R ph = A.f(phi, i, j, k), tc = tr(i, j, k);
        const R fe = R(0.5) * (tc + tr(ipp, j, k)) * (A.f(phi, ipp, j, k) - ph) / A.DX();
        const R fw = R(0.5) * (tr(imm, j, k) + tc) * (ph - A.f(phi, imm, j, k)) / A.DX();
        const R fn = R(0.5) * (tc + tr(i, jpp, k)) * (A.f(phi, i, jpp, k) - ph) / A.DY();
        const R fs = R(0.5) * (tr(i, jmm, k) + tc) * (ph - A.f(phi, i, jmm, k)) / A.DY();
        div += (fe - fw) / A.DX() + (fn - fs) / A.DY();
    }
    if (P.use_v)
    {
        const R ft = k < nz - 1 ? R(0.5) * (tr(i, j, k) + tr(i, j, k + 1)) *
                                           (A.f(phi, i, j, k + 1) - A.f(phi, i, j, k)) / A.DZC(k)
                                     : R(0.0);
        const R fb = k > 0 ? R(0.5) * (tr(i, j, k - 1) + tr(i, j, k)) *
                                      (A.f(phi, i, j, k) - A.f(phi, i, j, k - 1)) / A.DZC(k - 1)
                                : R(0.0);
        div += (ft - fb) / A.DZ(k);
    }
    return div / A.f(rho, i, j, k);
}

// The stresses on the three edges that meet at cell (i, j, k)'s upper-east-
// north corner, each used by two of the cell's faces with the same binary64
// value: T12 on the xy edge (x-face i, y-face j), shared by du (its north
// edge) and dv (its east edge); T13 on the xz edge (x-face i, z-face k),
// shared by du (its upper edge) and dw (its east edge); T23 likewise on the
// yz edge.  In each stress mode the reference's du / dw (dv / dw) forms of
// T13 (T23) reduce to the same expression.
template <class R>
__device__ __forceinline__ R sgs_t12(const SgsParams& P, const float* u, const float* v, const float* rho,
                                          const float* nu, int i, int j, int k)
{
    const SgsAt<R> A{P};
    const int i1 = sgs_next(i, P.d.nx, P.px), j1 = sgs_next(j, P.d.ny, P.py);
    const R s12 =
        R(0.5) * ((A.f(u, i, j1, k) - A.f(u, i, j, k)) / A.DY() + (A.f(v, i1, j, k) - A.f(v, i, j, k)) / A.DX());
    return R(2.0) * A.mu_xy(rho, nu, i, j, k) * s12;
}

template <class R>
__device__ __forceinline__ R sgs_t13(const SgsParams& P, const float* u, const float* w, const float* rho,
                                          const float* nu, int i, int j, int k)
{
    const SgsAt<R> A{P};
    const int i1 = sgs_next(i, P.d.nx, P.px);
    const R dwdx = (A.wf(w, i1, j, k) - A.wf(w, i, j, k)) / A.DX();
    R grad = dwdx;
    if (P.use_v)
    {
        const R dudz = (A.f(u, i, j, k + 1) - A.f(u, i, j, k)) / A.DZC(k);
        grad = P.use_h ? dudz + dwdx : dudz;
    }
    return A.mu_z(rho, nu, i, j, i1, j, k) * grad;
}

template <class R>
__device__ __forceinline__ R sgs_t23(const SgsParams& P, const float* v, const float* w, const float* rho,
                                          const float* nu, int i, int j, int k)
{
    const SgsAt<R> A{P};
    const int j1 = sgs_next(j, P.d.ny, P.py);
    const R dwdy = (A.wf(w, i, j1, k) - A.wf(w, i, j, k)) / A.DY();
    R grad = dwdy;
    if (P.use_v)
    {
        const R dvdz = (A.f(v, i, j, k + 1) - A.f(v, i, j, k)) / A.DZC(k);
        grad = P.use_h ? dvdz + dwdy : dvdz;
    }
    return A.mu_z(rho, nu, i, j, i, j1, k) * grad;
}

// du/dt at x-face (i, j, k) (compute_momentum_diffusion_tendencies, first
// loop); t12 / t13: the shared corner stresses above.
template <class R>
__device__ R sgs_du(const SgsParams& P, const float* u, const float* v, const float* w, const float* rho,
                         const float* nu, int i, int j, int k, R t12, R t13)
{
    const SgsAt<R> A{P};
    const int nx = P.d.nx, ny = P.d.ny;
    const int jmm = sgs_prev(j, ny, P.py), imm = sgs_prev(i, nx, P.px), ipp = sgs_next(i, nx, P.px);
    R div = R(0.0);
    if (P.use_h)
    {
        const R s_r = (A.f(u, ipp, j, k) - A.f(u, i, j, k)) / A.DX();
        const R s_l = (A.f(u, i, j, k) - A.f(u, imm, j, k)) / A.DX();
        div += (R(2.0) * A.mu(rho, nu, ipp, j, k) * s_r - R(2.0) * A.mu(rho, nu, i, j, k) * s_l) / A.DX();
        div += (t12 - sgs_t12<R>(P, u, v, rho, nu, i, jmm, k)) / A.DY();
    }
    if (P.use_v)
    {
        // T13 on the z-faces k (upper) and k-1 (lower; zero at the ground).
        const R lower = k > 0 ? sgs_t13<R>(P, u, w, rho, nu, i, j, k - 1) : R(0.0);
        div += (t13 - lower) / A.DZ(k);
    }
    return div / (R(0.5) * (A.f(rho, i, j, k) + A.f(rho, ipp, j, k)));
}

// dv/dt at y-face (i, j, k) (second loop).
template <class R>
__device__ R sgs_dv(const SgsParams& P, const float* u, const float* v, const float* w, const float* rho,
                         const float* nu, int i, int j, int k, R t12, R t23)
{
    const SgsAt<R> A{P};
    const int nx = P.d.nx, ny = P.d.ny;
    const int jmm = sgs_prev(j, ny, P.py), jpp = sgs_next(j, ny, P.py), imm = sgs_prev(i, nx, P.px);
    R div = R(0.0);
    if (P.use_h)
    {
        const R s_n = (A.f(v, i, jpp, k) - A.f(v, i, j, k)) / A.DY();
        const R s_s = (A.f(v, i, j, k) - A.f(v, i, jmm, k)) / A.DY();
        div += (R(2.0) * A.mu(rho, nu, i, jpp, k) * s_n - R(2.0) * A.mu(rho, nu, i, j, k) * s_s) / A.DY();
        div += (t12 - sgs_t12<R>(P, u, v, rho, nu, imm, j, k)) / A.DX();
    }
    if (P.use_v)
    {
        const R lower = k > 0 ? sgs_t23<R>(P, v, w, rho, nu, i, j, k - 1) : R(0.0);
        div += (t23 - lower) / A.DZ(k);
    }
    return div / (R(0.5) * (A.f(rho, i, j, k) + A.f(rho, i, jpp, k)));
}

// dw/dt at z-face (i, j, k) (third loop): stress divergence over the dual
// column mass.
template <class R>
__device__ R sgs_dw(const SgsParams& P, const float* u, const float* v, const float* w, const float* rho,
                         const float* nu, int i, int j, int k, R t13, R t23)
{
    const SgsAt<R> A{P};
    const int imm = sgs_prev(i, P.d.nx, P.px), jmm = sgs_prev(j, P.d.ny, P.py);
    const R dzb = R(P.dz[k]), dzt = R(P.dz[k + 1]), dzd = A.dzc(k);
    const R mass = R(0.5) * (A.f(rho, i, j, k) * dzb + A.f(rho, i, j, k + 1) * dzt);
    R force = R(0.0);
    if (P.use_v)
    {
        const R t33_t = R(2.0) * A.mu(rho, nu, i, j, k + 1) * ((A.wf(w, i, j, k + 1) - A.wf(w, i, j, k)) / A.DZ(k + 1));
        const R t33_b = R(2.0) * A.mu(rho, nu, i, j, k) * ((A.wf(w, i, j, k) - A.wf(w, i, j, k - 1)) / A.DZ(k));
        force += t33_t - t33_b;
    }
    if (P.use_h)
    {
        force += dzd * (t13 - sgs_t13<R>(P, u, w, rho, nu, imm, j, k)) / A.DX();
        force += dzd * (t23 - sgs_t23<R>(P, v, w, rho, nu, i, jmm, k)) / A.DY();
    }
    return force / mass;
}

// The five tendencies of every cell; zero where the reference leaves its
// pre-cleared outputs untouched.
template <class R>
__global__ void __launch_bounds__(256, 4) sgs_tendencies_kernel(
    SgsParams P, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const float* __restrict__ theta, const float* __restrict__ qv, const float* __restrict__ rho,
    const float* __restrict__ nu_t, const float* __restrict__ K_theta, const float* __restrict__ K_q,
    float* __restrict__ dudt, float* __restrict__ dvdt, float* __restrict__ dwdt, float* __restrict__ dthdt,
    float* __restrict__ dqvdt)
{
    const int n = P.d.cells();
    const int nx = P.d.nx, ny = P.d.ny, nz = P.d.nz;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        int i, j, k;
        decompose(P.d, c, i, j, k);
        const bool column = i >= 1 && i <= nx - 2 && j >= 1 && j <= ny - 2;
        const bool below_lid = k <= nz - 2;
        float ru = 0.0f, rv = 0.0f, rw = 0.0f, rt = 0.0f, rq = 0.0f;
        if (column && below_lid)
        {
            const bool du_on = i <= (P.px ? nx - 2 : nx - 3);
            const bool dv_on = j <= (P.py ? ny - 2 : ny - 3);
            const R t12 = P.use_h && (du_on || dv_on) ? sgs_t12<R>(P, u, v, rho, nu_t, i, j, k) : R(0.0);
            const R t13 = (du_on && P.use_v) || P.use_h ? sgs_t13<R>(P, u, w, rho, nu_t, i, j, k) : R(0.0);
            const R t23 = (dv_on && P.use_v) || P.use_h ? sgs_t23<R>(P, v, w, rho, nu_t, i, j, k) : R(0.0);
            if (du_on) ru = (float)sgs_du<R>(P, u, v, w, rho, nu_t, i, j, k, t12, t13);
            if (dv_on) rv = (float)sgs_dv<R>(P, u, v, w, rho, nu_t, i, j, k, t12, t23);
            rw = (float)sgs_dw<R>(P, u, v, w, rho, nu_t, i, j, k, t13, t23);
        }
        if (column)
        {
            rt = (float)sgs_scalar_rate<R>(P, rho, K_theta, theta, i, j, k);
            if (qv) rq = (float)sgs_scalar_rate<R>(P, rho, K_q, qv, i, j, k);
        }
        dudt[c] = ru;
        dvdt[c] = rv;
        dwdt[c] = rw;
        dthdt[c] = rt;
        if (dqvdt) dqvdt[c] = rq;
    }
}

struct SgsApplyParams
{
    int n, nz;
    double dt;
    int repairs;
    double theta_ref;
    float theta_lo, theta_hi, qv_hi, wind_h, wind_v;
    const double* theta0;  // [nz] base theta or null (device)
};

// sanitize_value (include/core/field/field_bounds.hpp:40-56).
__device__ __forceinline__ float sgs_sanitize(float x, int repairs, float fallback, float lo, float hi)
{
    if (!repairs) return x;
    if (!isfinite(x)) return fallback;
    return x < lo ? lo : (hi < x ? hi : x);
}

__device__ __forceinline__ double sgs_rate(float r, int repairs)
{
    const double x = (double)r;
    return repairs && !isfinite(x) ? 0.0 : x;
}

// Forward Euler of every cell (apply_sgs_tendencies_cpu without the work
// ledger): x += dt dx/dt in FP64, rounded once, clamped and repaired.
__global__ void __launch_bounds__(256) sgs_apply_kernel(SgsApplyParams A, float* __restrict__ u,
                                                        float* __restrict__ v, float* __restrict__ w,
                                                        float* __restrict__ theta, float* __restrict__ qv,
                                                        float* __restrict__ tke, const float* __restrict__ dudt,
                                                        const float* __restrict__ dvdt, const float* __restrict__ dwdt,
                                                        const float* __restrict__ dthdt,
                                                        const float* __restrict__ dqvdt,
                                                        const float* __restrict__ dtkedt,
                                                        const float* __restrict__ dtke_pbl)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < A.n; c += gridDim.x * blockDim.x)
    {
        float* wind[3] = {u, v, w};
        const float* rate[3] = {dudt, dvdt, dwdt};
#pragma unroll
        for (int f = 0; f < 3; ++f)
        {
            double x = (double)wind[f][c] + sgs_rate(rate[f][c], A.repairs) * A.dt;
            if (A.repairs && !isfinite(x)) x = 0.0;
            const float lim = f == 2 ? A.wind_v : A.wind_h;
            wind[f][c] = sgs_sanitize((float)x, A.repairs, 0.0f, -lim, lim);
        }
        const double th_old = (double)theta[c];
        double th = th_old + sgs_rate(dthdt[c], A.repairs) * A.dt;
        if (A.repairs && !isfinite(th))
            th = isfinite(th_old) ? th_old : (A.theta0 ? A.theta0[c % A.nz] : A.theta_ref);
        theta[c] = sgs_sanitize((float)th, A.repairs, (float)A.theta_ref, A.theta_lo, A.theta_hi);
        if (qv)
        {
            double q = (double)qv[c] + sgs_rate(dqvdt[c], A.repairs) * A.dt;
            if (A.repairs && !isfinite(q)) q = 0.0;
            qv[c] = sgs_sanitize((float)q, A.repairs, 0.0f, 0.0f, A.qv_hi);
        }
        if (tke)
        {
            const double old = (double)tke[c];
            double t = old + (sgs_rate(dtkedt[c], A.repairs) + sgs_rate(dtke_pbl[c], A.repairs)) * A.dt;
            if (A.repairs && !isfinite(t)) t = isfinite(old) ? old : 0.0;
            tke[c] = (float)(A.repairs ? (t < 0.0 ? 0.0 : t) : t);
        }
    }
}

// ---- explicit stability (closed or periodic lateral faces) ----

// One warp per physical x-slab i: the slab's momentum power and
// acceleration norm summed serially in j-k order (the reference's
// deterministic slab reduction), its theta / qv extrema, and its part of the
// input check.  partial: [slab][6] = power, norm, theta min, max, qv min, max.
// The lanes load 32 consecutive levels of a row (coalesced) and form each
// cell's six terms (mass * velocity * acceleration and mass * acceleration^2
// of its u, v and w faces) in parallel; lanes 0 and 1 then add them to the
// power and norm sums (one each) in the reference's order, while the lanes
// already hold the next chunk's loads.  A face the reference skips contributes +0.0, which
// leaves a sum that started at +0.0 unchanged bit for bit.
constexpr int kSlabWarps = 4;

struct SlabChunk
{
    float u, v, w, r, ri, rj, rk, du, dv, dw, th, dth, q, dq;
};

__device__ __forceinline__ SlabChunk slab_load(const SgsParams& P, const float* u, const float* v, const float* w,
                                               const float* theta, const float* qv, const float* rho,
                                               const float* dudt, const float* dvdt, const float* dwdt,
                                               const float* dthdt, const float* dqvdt, int i, int i1, int j, int j1,
                                               int k)
{
    SlabChunk x{};
    if (k >= P.d.nz) return x;
    const int c = P.d.at(i, j, k);
    x.u = __ldg(u + c);
    x.v = __ldg(v + c);
    x.w = __ldg(w + c);
    x.r = __ldg(rho + c);
    x.ri = __ldg(rho + P.d.at(i1, j, k));
    x.rj = __ldg(rho + P.d.at(i, j1, k));
    x.rk = k + 1 < P.d.nz ? __ldg(rho + c + 1) : 1.0f;
    x.du = __ldg(dudt + c);
    x.dv = __ldg(dvdt + c);
    x.dw = __ldg(dwdt + c);
    x.th = __ldg(theta + c);
    x.dth = __ldg(dthdt + c);
    if (qv)
    {
        x.q = __ldg(qv + c);
        x.dq = __ldg(dqvdt + c);
    }
    return x;
}

__global__ void __launch_bounds__(32 * kSlabWarps) sgs_stability_slab_kernel(
    SgsParams P, const float* __restrict__ u, const float* __restrict__ v, const float* __restrict__ w,
    const float* __restrict__ theta, const float* __restrict__ qv, const float* __restrict__ rho,
    const float* __restrict__ dudt, const float* __restrict__ dvdt, const float* __restrict__ dwdt,
    const float* __restrict__ dthdt, const float* __restrict__ dqvdt, double* __restrict__ partial,
    unsigned* status)
{
    __shared__ double terms[kSlabWarps][6][32];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int slab = blockIdx.x * kSlabWarps + wib;
    const int nx = P.d.nx, ny = P.d.ny, nz = P.d.nz;
    if (slab >= nx - 2) return;  // uniform across the warp
    const int i = slab + 1;
    const double area = P.dx * P.dy;
    const int i1 = P.px && i >= nx - 2 ? 1 : i + 1;
    const bool has_u = P.px || i <= nx - 3;
    double (*t)[32] = terms[wib];
    double p = 0.0, a = 0.0, tlo = INFINITY, thi = -INFINITY, qlo = INFINITY, qhi = -INFINITY;
    bool bad = false;
    const int chunks = (nz + 31) / 32;
    const int total = (ny - 2) * chunks;
    // Chunk n covers row j = 1 + n / chunks, levels (n % chunks) * 32 + lane.
    auto row_of = [&](int n, int& j, int& j1, int& k) {
        j = 1 + n / chunks;
        j1 = P.py && j >= ny - 2 ? 1 : j + 1;
        k = (n % chunks) * 32 + lane;
    };
    int j, j1, k;
    // Two chunks in flight ahead of the one being summed.
    int jb = 0, j1b = 0, kb = 0;
    row_of(0, j, j1, k);
    SlabChunk x = slab_load(P, u, v, w, theta, qv, rho, dudt, dvdt, dwdt, dthdt, dqvdt, i, i1, j, j1, k);
    SlabChunk y{};
    if (total > 1)
    {
        row_of(1, jb, j1b, kb);
        y = slab_load(P, u, v, w, theta, qv, rho, dudt, dvdt, dwdt, dthdt, dqvdt, i, i1, jb, j1b, kb);
    }
    for (int n = 0; n < total; ++n)
    {
        const int jc = j, kc = k;
        const SlabChunk cur = x;
        x = y;
        j = jb;
        j1 = j1b;
        k = kb;
        if (n + 2 < total)
        {
            row_of(n + 2, jb, j1b, kb);
            y = slab_load(P, u, v, w, theta, qv, rho, dudt, dvdt, dwdt, dthdt, dqvdt, i, i1, jb, j1b, kb);
        }
        double tm[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        if (kc < nz)
        {
            const double r = cur.r, th = cur.th;
            bad |= !isfinite(r) || !isfinite(cur.u) || !isfinite(cur.v) || !isfinite(cur.w) || !isfinite(th) ||
                   !isfinite(cur.du) || !isfinite(cur.dv) || !isfinite(cur.dw) || !isfinite(cur.dth) ||
                   !(r > 0.0) || !(th > 0.0);
            if (kc < nz - 1)
            {
                const double vol = area * P.dz[kc];
                if (has_u)
                {
                    const double m = 0.5 * (r * vol + (double)cur.ri * vol);
                    const double acc = cur.du;
                    tm[0] = m * (double)cur.u * acc;
                    tm[1] = m * acc * acc;
                }
                if (P.py || jc < ny - 2)
                {
                    const double m = 0.5 * (r * vol + (double)cur.rj * vol);
                    const double acc = cur.dv;
                    tm[2] = m * (double)cur.v * acc;
                    tm[3] = m * acc * acc;
                }
                const double m = 0.5 * (r * vol + (double)cur.rk * (area * P.dz[kc + 1]));
                const double acc = cur.dw;
                tm[4] = m * (double)cur.w * acc;
                tm[5] = m * acc * acc;
            }
            tlo = th < tlo ? th : tlo;
            thi = thi < th ? th : thi;
            if (qv)
            {
                const double q = cur.q;
                bad |= !isfinite(q) || q < 0.0 || !isfinite(cur.dq);
                qlo = q < qlo ? q : qlo;
                qhi = qhi < q ? q : qhi;
            }
        }
#pragma unroll
        for (int q = 0; q < 6; ++q) t[q][lane] = tm[q];
        __syncwarp();
        if (lane < 2)
        {
            // Lane 0 carries the power sum, lane 1 the norm sum: two
            // independent serial chains, each in the reference's order.
            const int cells = min(32, nz - (kc - lane));
            double acc = lane == 0 ? p : a;
            for (int c = 0; c < cells; ++c)
            {
                acc += t[lane][c];
                acc += t[lane + 2][c];
                acc += t[lane + 4][c];
            }
            if (lane == 0)
                p = acc;
            else
                a = acc;
        }
        __syncwarp();
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        tlo = fmin(tlo, __shfl_down_sync(0xffffffffu, tlo, off));
        thi = fmax(thi, __shfl_down_sync(0xffffffffu, thi, off));
        qlo = fmin(qlo, __shfl_down_sync(0xffffffffu, qlo, off));
        qhi = fmax(qhi, __shfl_down_sync(0xffffffffu, qhi, off));
    }
    bad = __any_sync(0xffffffffu, bad);
    a = __shfl_sync(0xffffffffu, a, 1);
    if (lane == 0)
    {
        if (bad) atomicOr(status, kStatusSgsInvalid);
        double* o = partial + 6 * slab;
        o[0] = p;
        o[1] = a;
        o[2] = tlo;
        o[3] = thi;
        o[4] = qlo;
        o[5] = qhi;
    }
}

// Merge of the slab partials in increasing i: compensated sums of power and
// norm (CompensatedSum, include/diagnostics/deterministic_reduction.hpp:28-53)
// and the extrema.  out: power, norm, theta min, max, qv min, max; one thread.
__global__ void sgs_stability_merge_kernel(int slabs, const double* __restrict__ partial, double* __restrict__ out)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double sums[2] = {0.0, 0.0}, corr[2] = {0.0, 0.0};
    double tlo = INFINITY, thi = -INFINITY, qlo = INFINITY, qhi = -INFINITY;
    for (int s = 0; s < slabs; ++s)
    {
        const double* o = partial + 6 * s;
#pragma unroll
        for (int q = 0; q < 2; ++q)
        {
            const double x = o[q], next = sums[q] + x;
            if (fabs(sums[q]) >= fabs(x))
                corr[q] += (sums[q] - next) + x;
            else
                corr[q] += (x - next) + sums[q];
            sums[q] = next;
        }
        tlo = o[2] < tlo ? o[2] : tlo;
        thi = thi < o[3] ? o[3] : thi;
        qlo = o[4] < qlo ? o[4] : qlo;
        qhi = qhi < o[5] ? o[5] : qhi;
    }
    out[0] = sums[0] + corr[0];
    out[1] = sums[1] + corr[1];
    out[2] = tlo;
    out[3] = thi;
    out[4] = qlo;
    out[5] = qhi;
}

// The theta / qv monotonic limits: min over the physical cells of the time to
// reach the field's current extremum.  Every candidate is >= 0, so the
// minimum is an unsigned min over the bit patterns (atomicMin).  ext: the
// merged extrema (out[2..5] above); lim: two u64 slots preset to +inf.
__global__ void __launch_bounds__(256) sgs_stability_limit_kernel(SgsParams P, const float* __restrict__ theta,
                                                                  const float* __restrict__ qv,
                                                                  const float* __restrict__ dthdt,
                                                                  const float* __restrict__ dqvdt,
                                                                  const double* __restrict__ ext,
                                                                  unsigned long long* lim)
{
    const int nx = P.d.nx, ny = P.d.ny, nz = P.d.nz;
    const int n = (nx - 2) * (ny - 2) * nz;
    double tl = INFINITY, ql = INFINITY;
    for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x)
    {
        const int k = t % nz, col = t / nz;
        const int j = 1 + col % (ny - 2), i = 1 + col / (ny - 2);
        const int c = P.d.at(i, j, k);
        const double th = theta[c], r = dthdt[c];
        if (r > 0.0)
            tl = fmin(tl, (ext[1] - th) / r);
        else if (r < 0.0)
            tl = fmin(tl, (th - ext[0]) / -r);
        if (qv)
        {
            const double q = qv[c], rq = dqvdt[c];
            if (rq > 0.0)
                ql = fmin(ql, (ext[3] - q) / rq);
            else if (rq < 0.0)
                ql = fmin(ql, (q - ext[2]) / -rq);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1)
    {
        tl = fmin(tl, __shfl_down_sync(0xffffffffu, tl, off));
        ql = fmin(ql, __shfl_down_sync(0xffffffffu, ql, off));
    }
    if ((threadIdx.x & 31) == 0)
    {
        atomicMin(lim, (unsigned long long)__double_as_longlong(tl));
        atomicMin(lim + 1, (unsigned long long)__double_as_longlong(ql));
    }
}

}  // namespace nimbus
