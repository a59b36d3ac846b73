// Conservative flux-form scalar transport on the retained C-grid context,
// reference-precision form (FP64 face arithmetic, FP32 face scratch as the
// reference's Field3D scratch stores it).  Compiled with --fmad=false.
//
// Three passes per scalar batch (blockIdx.y = scalar):
//   faces   : SF = M * phi_face on each cell's owned +x/+y/+z faces; phi_face
//             from WENO5-JS where the 5-point upwind stencil fits, else the
//             MC-limited slope (advection_cartesian.cpp:1943-2172).
//   limiter : positive-definite donor ratio per cell (:2174-2240).
//   update  : donor-limited divergence and density recovery (:2465-2640).
#pragma once

#include "stencil_common.cuh"

#include <type_traits>

namespace nimbus
{

constexpr int kMaxScalars = 16;

struct TransportParams
{
    Dims d;
    double inv_dx, inv_dy, inv_dz;
    double dt;
    double rho_floor;
    int weno;
    int top_open;
    int n_scalars;
    const float* q_in[kMaxScalars];
    float* q_out[kMaxScalars];
    int positive_definite[kMaxScalars];
    // FP32 form: the scalars above rounded once.
    float inv_dx_f, inv_dy_f, inv_dz_f, dt_f, inv_dt_f, rho_floor_f;
};

// The fields of TransportParams the interleaved (float4) cell functions read:
// geometry, spacings, dt, the density floor, the reconstruction and top
// flags and the first four scalars' positive-definite flags.
struct TransportCompact
{
    Dims d;
    double inv_dx, inv_dy, inv_dz;
    double dt;
    double rho_floor;
    int weno;
    int top_open;
    int positive_definite[4];
    float inv_dx_f, inv_dy_f, inv_dz_f, dt_f, inv_dt_f, rho_floor_f;
};

__host__ __device__ inline void finish_fp32(TransportParams& T)
{
    T.inv_dx_f = (float)T.inv_dx;
    T.inv_dy_f = (float)T.inv_dy;
    T.inv_dz_f = (float)T.inv_dz;
    T.dt_f = (float)T.dt;
    T.inv_dt_f = (float)(1.0 / T.dt);
    T.rho_floor_f = (float)T.rho_floor;
}

// weno5_face_value (include/numerics/advection/weno5_face.hpp:43-86).
__device__ __forceinline__ double weno5_face(double a, double b, double c, double d, double e)
{
    const double p0 = (1.0 / 3.0) * a - (7.0 / 6.0) * b + (11.0 / 6.0) * c;
    const double p1 = -(1.0 / 6.0) * b + (5.0 / 6.0) * c + (1.0 / 3.0) * d;
    const double p2 = (1.0 / 3.0) * c + (5.0 / 6.0) * d - (1.0 / 6.0) * e;
    const double s0a = a - 2.0 * b + c;
    const double s0b = a - 4.0 * b + 3.0 * c;
    const double s1a = b - 2.0 * c + d;
    const double s1b = b - d;
    const double s2a = c - 2.0 * d + e;
    const double s2b = 3.0 * c - 4.0 * d + e;
    const double b0 = (13.0 / 12.0) * s0a * s0a + 0.25 * s0b * s0b;
    const double b1 = (13.0 / 12.0) * s1a * s1a + 0.25 * s1b * s1b;
    const double b2 = (13.0 / 12.0) * s2a * s2a + 0.25 * s2b * s2b;
    const double aa = a * a, bb = b * b, cc = c * c, dd = d * d, ee = e * e;
    const double m_ab = (aa < bb) ? bb : aa;
    const double m_cd = (cc < dd) ? dd : cc;
    const double m_abcd = (m_ab < m_cd) ? m_cd : m_ab;
    const double q2max = (m_abcd < ee) ? ee : m_abcd;
    const double eps = 1.0e-6 * q2max + 1.0e-40;
    const double a0 = (1.0 / 10.0) / ((eps + b0) * (eps + b0));
    const double a1 = (6.0 / 10.0) / ((eps + b1) * (eps + b1));
    const double a2 = (3.0 / 10.0) / ((eps + b2) * (eps + b2));
    const double sum = a0 + a1 + a2;
    if (!(sum > 0.0) || !isfinite(sum)) return c;
    const double face = (a0 * p0 + a1 * p1 + a2 * p2) / sum;
    return isfinite(face) ? face : c;
}

// minmod3 / mc_limited_slope (advection_cartesian.cpp:136-170).
__device__ __forceinline__ double mc_slope(double qm, double q0, double qp)
{
    const double right = qp - q0, left = q0 - qm;
    const double a = 0.5 * (right + left), b = 2.0 * right, c = 2.0 * left;
    if (a > 0.0 && b > 0.0 && c > 0.0) return fmin(a, fmin(b, c));
    if (a < 0.0 && b < 0.0 && c < 0.0) return fmax(a, fmax(b, c));
    return 0.0;
}

// Lane arithmetic for the FP32 face offset: one scalar stencil (float) or two
// independent stencils at once (float2, Blackwell's paired f32x2 FMA / MUL /
// ADD: two IEEE round-to-nearest operations per instruction).  Every operation
// is an explicit round-to-nearest intrinsic, so the scalar and paired forms
// run the same operation sequence and give the same bits; only the
// reciprocals, the final quotient and the finiteness test act per lane.
template <class V>
struct Lanes;

template <>
struct Lanes<float>
{
    static __device__ __forceinline__ float splat(float x) { return x; }
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
    static __device__ __forceinline__ float maxf(float a, float b) { return fmaxf(a, b); }
    static __device__ __forceinline__ float absf(float a) { return fabsf(a); }
    static __device__ __forceinline__ float rcp(float a) { return __fdividef(1.0f, a); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
    static __device__ __forceinline__ float finite_or_zero(float a) { return isfinite(a) ? a : 0.0f; }
};

template <>
struct Lanes<float2>
{
    static __device__ __forceinline__ float2 splat(float x) { return make_float2(x, x); }
    static __device__ __forceinline__ float2 add(float2 a, float2 b) { return __fadd2_rn(a, b); }
    static __device__ __forceinline__ float2 mul(float2 a, float2 b) { return __fmul2_rn(a, b); }
    static __device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
    static __device__ __forceinline__ float2 maxf(float2 a, float2 b)
    {
        return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y));
    }
    static __device__ __forceinline__ float2 absf(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
    static __device__ __forceinline__ float2 rcp(float2 a)
    {
        return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y));
    }
    static __device__ __forceinline__ float2 div(float2 a, float2 b)
    {
        return make_float2(__fdividef(a.x, b.x), __fdividef(a.y, b.y));
    }
    static __device__ __forceinline__ float2 finite_or_zero(float2 a)
    {
        return make_float2(isfinite(a.x) ? a.x : 0.0f, isfinite(a.y) ? a.y : 0.0f);
    }
};

// FP32 face offset from the donor value c (face = c + offset): WENO5-JS on
// the stencil normalised by its largest magnitude, as the reference's FP32
// GPU form normalises it (weno5_face_offset_fp32,
// include/numerics/advection/weno5_face.hpp:88-120: differences from the
// donor, eps = 1e-6 * relative^2 + (1e-20 / scale)^2, ideal weights 1/10,
// 6/10, 3/10, p = 2), so moisture-scale fields keep their nonlinear weights.
// After normalisation every eps + beta_k is at least 1e-6, so the weights
// d_k / (eps + beta_k)^2 are formed directly from approximate reciprocals
// instead of the reference's min-normalised ratios: the same weights to FP32
// rounding in about half the instructions.  A non-finite result falls back to
// the donor value (offset 0).  V = float2 evaluates two stencils at once.
template <class V>
__device__ __forceinline__ V weno5_offset_lanes(V a, V b, V c, V d, V e)
{
    using L = Lanes<V>;
    const V magnitude = L::maxf(L::maxf(L::maxf(L::absf(a), L::absf(b)), L::maxf(L::absf(c), L::absf(d))),
                                L::absf(e));
    const V scale = L::maxf(magnitude, L::splat(1e-20f));
    const V inv = L::rcp(scale);
    const V m1 = L::splat(-1.0f);
    const V ac = L::mul(L::fma(c, m1, a), inv), bc = L::mul(L::fma(c, m1, b), inv);
    const V dc = L::mul(L::fma(c, m1, d), inv), ec = L::mul(L::fma(c, m1, e), inv);
    const V p0 = L::fma(ac, L::splat(1.0f / 3.0f), L::mul(bc, L::splat(-7.0f / 6.0f)));
    const V p1 = L::fma(dc, L::splat(1.0f / 3.0f), L::mul(bc, L::splat(-1.0f / 6.0f)));
    const V p2 = L::fma(dc, L::splat(5.0f / 6.0f), L::mul(ec, L::splat(-1.0f / 6.0f)));
    const V s0a = L::fma(bc, L::splat(-2.0f), ac), s0b = L::fma(bc, L::splat(-4.0f), ac);
    const V s1a = L::add(bc, dc), s1b = L::fma(dc, m1, bc);
    const V s2a = L::fma(dc, L::splat(-2.0f), ec), s2b = L::fma(dc, L::splat(-4.0f), ec);
    const V k13 = L::splat(13.0f / 12.0f), quarter = L::splat(0.25f);
    const V b0 = L::fma(L::mul(s0a, k13), s0a, L::mul(L::mul(s0b, quarter), s0b));
    const V b1 = L::fma(L::mul(s1a, k13), s1a, L::mul(L::mul(s1b, quarter), s1b));
    const V b2 = L::fma(L::mul(s2a, k13), s2a, L::mul(L::mul(s2b, quarter), s2b));
    const V relative = L::mul(magnitude, inv);
    const V flo = L::mul(L::splat(1e-20f), inv);
    const V epsilon = L::fma(L::mul(relative, L::splat(1e-6f)), relative, L::mul(flo, flo));
    const V r0 = L::rcp(L::add(epsilon, b0)), r1 = L::rcp(L::add(epsilon, b1)), r2 = L::rcp(L::add(epsilon, b2));
    const V a0 = L::mul(L::mul(r0, L::splat(0.1f)), r0);
    const V a1 = L::mul(L::mul(r1, L::splat(0.6f)), r1);
    const V a2 = L::mul(L::mul(r2, L::splat(0.3f)), r2);
    const V num = L::fma(a2, p2, L::fma(a1, p1, L::mul(a0, p0)));
    const V den = L::add(L::add(a0, a1), a2);
    return L::finite_or_zero(L::mul(scale, L::div(num, den)));
}

__device__ __forceinline__ float weno5_offset_f32(float a, float b, float c, float d, float e)
{
    return weno5_offset_lanes<float>(a, b, c, d, e);
}

__device__ __forceinline__ float mc_slope_f32(float qm, float q0, float qp)
{
    const float right = qp - q0, left = q0 - qm;
    const float a = 0.5f * (right + left), b = 2.0f * right, c = 2.0f * left;
    if (a > 0.0f && b > 0.0f && c > 0.0f) return fminf(a, fminf(b, c));
    if (a < 0.0f && b < 0.0f && c < 0.0f) return fmaxf(a, fmaxf(b, c));
    return 0.0f;
}

// The stencil of one face, shared by every scalar (the upwind side follows
// the mass flux, which all scalars share): the five cell offsets of the WENO5
// stencil (donor - 2s .. donor + 2s), or for the MC fallback near a wall the
// donor (o[2]) and its two neighbours in the reference's argument order.
struct FaceStencil
{
    int o[5];
    bool pos;    // mflux >= 0
    bool weno;   // the 5-point stencil fits
    bool slope;  // MC: the slope's neighbours exist
};

__device__ __forceinline__ FaceStencil face_stencil(int base, int stride, int l, int n, bool mflux_pos, int weno)
{
    FaceStencil f;
    f.pos = mflux_pos;
    const int donor = f.pos ? l : l + 1;
    const int s = f.pos ? stride : -stride;
    f.weno = weno && donor - 2 >= 0 && donor + 2 <= n - 1;
    const int cd = base + donor * stride;
    if (f.weno)
    {
        f.o[0] = cd - 2 * s; f.o[1] = cd - s; f.o[2] = cd; f.o[3] = cd + s; f.o[4] = cd + 2 * s;
        f.slope = false;
    }
    else
    {
        // advection_cartesian.cpp:1971-2008: positive side
        // mc(q[l-1], q[l], q[l+1]) when l >= 1, negative side
        // mc(q[l], q[l+1], q[l+2]) when l + 1 <= n - 2.
        f.slope = f.pos ? (l >= 1) : (l + 1 <= n - 2);
        const int lo = f.pos ? l - 1 : l, hi = f.pos ? l + 1 : l + 2;
        f.o[0] = f.slope ? base + lo * stride : cd;
        f.o[1] = f.o[0]; f.o[2] = cd; f.o[3] = f.slope ? base + hi * stride : cd; f.o[4] = f.o[3];
    }
    return f;
}

// The face flux of one scalar on a prepared stencil
// (advection_cartesian.cpp:1943-2172).  FP32 form: M * donor + M * offset
// with the normalised WENO5 offset; reference precision: M times the FP64
// face value (WENO5 where the stencil fits, else donor +- half the MC
// slope), rounded once to the FP32 scratch.
// The same from the five stencil values v[m] = q[f.o[m]] (for the MC
// fallback v[0], v[2], v[3] are the slope's points).
template <bool kFp32>
__device__ __forceinline__ float stencil_flux_values(const float (&v)[5], const FaceStencil& f, float mflux)
{
    if constexpr (kFp32)
    {
        const float q0 = v[2];
        float offset;
        if (f.weno) offset = weno5_offset_f32(v[0], v[1], q0, v[3], v[4]);
        else
        {
            const float sl = f.slope ? mc_slope_f32(v[0], q0, v[3]) : 0.0f;
            offset = (f.pos ? 0.5f : -0.5f) * sl;
        }
        return __fmaf_rn(mflux, q0, mflux * offset);
    }
    else
    {
        const double q0 = (double)v[2];
        double face;
        if (f.weno) face = weno5_face((double)v[0], (double)v[1], q0, (double)v[3], (double)v[4]);
        else
        {
            const double sl = f.slope ? mc_slope((double)v[0], q0, (double)v[3]) : 0.0;
            face = f.pos ? q0 + 0.5 * sl : q0 - 0.5 * sl;
        }
        return (float)((double)mflux * face);
    }
}

template <bool kFp32>
__device__ __forceinline__ float stencil_flux(const float* __restrict__ q, const FaceStencil& f, float mflux)
{
    const float v[5] = {q[f.o[0]], q[f.o[1]], q[f.o[2]], q[f.o[3]], q[f.o[4]]};
    return stencil_flux_values<kFp32>(v, f, mflux);
}

// FP32 face fluxes of two scalars on one stencil (same donor, same mass
// flux): the WENO5 arithmetic of both in paired f32x2 instructions, with the
// same bits as two stencil_flux<true> calls.
__device__ __forceinline__ float2 stencil_flux_pair_values(const float2 (&v)[5], const FaceStencil& f, float mflux)
{
    const float2 q0 = v[2];
    float2 offset;
    if (f.weno) offset = weno5_offset_lanes<float2>(v[0], v[1], q0, v[3], v[4]);
    else
    {
        const float h = f.pos ? 0.5f : -0.5f;
        const float sa = f.slope ? mc_slope_f32(v[0].x, q0.x, v[3].x) : 0.0f;
        const float sb = f.slope ? mc_slope_f32(v[0].y, q0.y, v[3].y) : 0.0f;
        offset = make_float2(h * sa, h * sb);
    }
    const float2 m = make_float2(mflux, mflux);
    return __ffma2_rn(m, q0, __fmul2_rn(m, offset));
}

__device__ __forceinline__ float2 stencil_flux_pair(const float* __restrict__ qa, const float* __restrict__ qb,
                                                    const FaceStencil& f, float mflux)
{
    float2 v[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) v[m] = make_float2(qa[f.o[m]], qb[f.o[m]]);
    return stencil_flux_pair_values(v, f, mflux);
}

// Face fluxes owned by cell c (its +x, +y and +z faces) for every scalar:
// the cell's index, mass fluxes and face stencils are formed once and the
// scalars follow.  kFp32 selects the FP32 form, otherwise FP64 face values
// rounded once to the FP32 scratch.  q(s) gives scalar s's field; sf is the
// [scalars][3][cells] face-flux scratch (x, y, z).
template <bool kFp32, class QIn>
__device__ __forceinline__ void transport_faces_cell(const TransportParams& T, int scalars, QIn&& q_of,
                                                     const float* __restrict__ mfx, const float* __restrict__ mfy,
                                                     const float* __restrict__ mfz, float* __restrict__ sf, int c)
{
    const Dims d = T.d;
    const size_t n = (size_t)d.cells();
    const int kz_end = T.top_open ? d.nz : d.nz - 1;
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool hx = i <= d.nx - 2, hy = j <= d.ny - 2, hz = k < kz_end, top = k == d.nz - 1;
    const float fx = hx ? mfx[c] : 0.0f, fy = hy ? mfy[c] : 0.0f, fz = hz ? mfz[c] : 0.0f;
    const FaceStencil sx = face_stencil(c - i * d.sx(), d.sx(), i, d.nx, fx >= 0.0f, T.weno);
    const FaceStencil sy = face_stencil(c - j * d.sy(), d.sy(), j, d.ny, fy >= 0.0f, T.weno);
    const FaceStencil sz = face_stencil(c - k, 1, top ? k - 1 : k, d.nz, fz >= 0.0f, T.weno);
    int s = 0;
    if constexpr (kFp32)
    {
        for (; s + 1 < scalars; s += 2)
        {
            const float* __restrict__ qa = q_of(s);
            const float* __restrict__ qb = q_of(s + 1);
            float* __restrict__ sfx = sf + (size_t)s * 3 * n;
            float* __restrict__ sfy = sfx + n;
            float* __restrict__ sfz = sfy + n;
            float* __restrict__ tfx = sfz + n;  // scalar s + 1
            float* __restrict__ tfy = tfx + n;
            float* __restrict__ tfz = tfy + n;
            if (hx)
            {
                const float2 r = stencil_flux_pair(qa, qb, sx, fx);
                sfx[c] = r.x;
                tfx[c] = r.y;
            }
            if (hy)
            {
                const float2 r = stencil_flux_pair(qa, qb, sy, fy);
                sfy[c] = r.x;
                tfy[c] = r.y;
            }
            if (hz)
            {
                if (top)
                {
                    sfz[c] = fz * qa[c];
                    tfz[c] = fz * qb[c];
                }
                else
                {
                    const float2 r = stencil_flux_pair(qa, qb, sz, fz);
                    sfz[c] = r.x;
                    tfz[c] = r.y;
                }
            }
        }
    }
    for (; s < scalars; ++s)
    {
        const float* __restrict__ q = q_of(s);
        float* __restrict__ sfx = sf + (size_t)s * 3 * n;
        float* __restrict__ sfy = sfx + n;
        float* __restrict__ sfz = sfy + n;
        if (hx) sfx[c] = stencil_flux<kFp32>(q, sx, fx);
        if (hy) sfy[c] = stencil_flux<kFp32>(q, sy, fy);
        if (hz)
        {
            if (top) sfz[c] = kFp32 ? fz * q[c] : (float)((double)fz * (double)q[c]);
            else sfz[c] = stencil_flux<kFp32>(q, sz, fz);
        }
    }
}

template <bool kFp32>
static __global__ void __launch_bounds__(256) transport_faces_kernel(TransportParams T, const float* __restrict__ mfx,
                                                                     const float* __restrict__ mfy,
                                                                     const float* __restrict__ mfz,
                                                                     float* __restrict__ sf)
{
    const int n = T.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        transport_faces_cell<kFp32>(T, T.n_scalars, [&](int s) { return T.q_in[s]; }, mfx, mfy, mfz, sf, c);
}

// conservative_pd_limiter_factor (advection_cartesian.hpp:101-108), non-support path.
__device__ __forceinline__ float pd_limiter_factor(double r)
{
    if (!(r > 0.0 && r < 1.0)) return (float)r;
    const float roundoff = 1.0f - 32.0f * 1.1920928955078125e-7f;
    const float stored = (float)r;
    return nextafterf(__fmul_rn(stored, roundoff), 0.0f);
}

// Positive-definite donor ratio of one scalar at a cell from its six face
// fluxes (advection_cartesian.cpp:2174-2240): x+, x-, y+, y-, z+, z- faces,
// each counted only where it exists (the has_* flags).  kFp32: the same sums
// in FP32 (the reference's FP32 GPU form); the factor's 32-ulp roundoff
// margin covers the FP32 rounding of the update.
template <bool kFp32, class TP>
__device__ __forceinline__ float limiter_factor(const TP& T, float fxp, float fxm, float fyp, float fym,
                                                float fzp, float fzm, bool xp, bool xm, bool yp, bool ym, bool zp,
                                                bool zm, float rho_b, float q)
{
    using real = typename std::conditional<kFp32, float, double>::type;
    const real rb = (real)rho_b;
    const real idx = kFp32 ? (real)T.inv_dx_f : (real)T.inv_dx;
    const real idy = kFp32 ? (real)T.inv_dy_f : (real)T.inv_dy;
    const real idz = kFp32 ? (real)T.inv_dz_f : (real)T.inv_dz;
    real out = 0;
    if (xp && fxp > 0.0f) out += (real)fxp * idx;
    if (xm && fxm < 0.0f) out -= (real)fxm * idx;
    if (yp && fyp > 0.0f) out += (real)fyp * idy;
    if (ym && fym < 0.0f) out -= (real)fym * idy;
    if (zp && fzp > 0.0f) out += (real)fzp * idz;
    if (zm && fzm < 0.0f) out -= (real)fzm * idz;
    if constexpr (kFp32)
    {
        float r = 1.0f;
        if (out > 0.0f)
        {
            const float available = rb * ((q < 0.0f) ? 0.0f : q) * T.inv_dt_f;
            const float ratio = __fdividef(available, out);
            r = (ratio < 1.0f) ? ratio : 1.0f;
        }
        return (r > 0.0f && r < 1.0f) ? nextafterf(__fmul_rn(r, 1.0f - 32.0f * 1.1920928955078125e-7f), 0.0f) : r;
    }
    else
    {
        double r = 1.0;
        if (out > 0.0)
        {
            const double qc = (double)q;
            const double available = rb * ((qc < 0.0) ? 0.0 : qc) / T.dt;  // std::max(q, 0.0)
            const double ratio = available / out;
            r = (ratio < 1.0) ? ratio : 1.0;  // std::min(1.0, ratio), NaN -> 1
        }
        return pd_limiter_factor(r);
    }
}

// The limiter factor of every positive-definite scalar at cell c; sf is
// [scalars][3][cells], rl [scalars][cells].
template <bool kFp32, class QIn>
__device__ __forceinline__ void transport_limiter_cell(const TransportParams& T, int scalars, QIn&& q_of,
                                                       const float* __restrict__ rho_begin,
                                                       const float* __restrict__ sf, float* __restrict__ rl, int c)
{
    const Dims d = T.d;
    const size_t n = (size_t)d.cells();
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool xm = i >= 1, xp = i <= d.nx - 2, ym = j >= 1, yp = j <= d.ny - 2, zm = k >= 1;
    const bool zp = k <= d.nz - 2 || (T.top_open && k == d.nz - 1);
    const int cxm = xm ? c - d.sx() : c, cym = ym ? c - d.sy() : c, czm = zm ? c - 1 : c;
    const float rb = rho_begin[c];
    for (int s = 0; s < scalars; ++s)
    {
        if (!T.positive_definite[s]) continue;
        const float* __restrict__ sfx = sf + (size_t)s * 3 * n;
        const float* __restrict__ sfy = sfx + n;
        const float* __restrict__ sfz = sfy + n;
        rl[(size_t)s * n + c] = limiter_factor<kFp32>(T, sfx[c], sfx[cxm], sfy[c], sfy[cym], sfz[c], sfz[czm], xp,
                                                      xm, yp, ym, zp, zm, rb, q_of(s)[c]);
    }
}

template <bool kFp32>
static __global__ void __launch_bounds__(256) transport_limiter_kernel(TransportParams T,
                                                                       const float* __restrict__ rho_begin,
                                                                       const float* __restrict__ sf,
                                                                       float* __restrict__ rl)
{
    const int n = T.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        transport_limiter_cell<kFp32>(T, T.n_scalars, [&](int s) { return T.q_in[s]; }, rho_begin, sf, rl, c);
}

// The donor-side factor of a face (limited_flux in the reference): the factor
// of the cell the flux leaves.
template <bool kFp32>
__device__ __forceinline__ typename std::conditional<kFp32, float, double>::type limited_face(float raw, bool pd,
                                                                                             float r_lo, float r_hi)
{
    if (!pd || raw == 0.0f) return raw;
    const float r = raw > 0.0f ? r_lo : r_hi;
    if constexpr (kFp32) return raw * r;
    else return (double)raw * (double)r;
}

// The new value of one scalar at an interior cell from its six face fluxes
// (x+, x-, y+, y-, z+, z-), the limiter factors of the cell and its six
// neighbours (positive-definite scalars only) and its old value
// (advection_cartesian.cpp:2465-2640).  kFp32: the same sums in FP32.
template <bool kFp32, class TP>
__device__ __forceinline__ float update_value(const TP& T, bool pd, float fxp, float fxm, float fyp,
                                              float fym, float fzp, float fzm, float rc, float rxp, float rxm,
                                              float ryp, float rym, float rzp, float rzm, float qraw, bool has_top,
                                              bool has_bottom, float rho_e, float rho_b, unsigned& flags)
{
    using real = typename std::conditional<kFp32, float, double>::type;
    const real re = (real)rho_e;
    const real rb = (real)rho_b;
    const real floor_ = kFp32 ? (real)T.rho_floor_f : (real)T.rho_floor;
    const real denom = (re > floor_) ? re : floor_;
    const real idx = kFp32 ? (real)T.inv_dx_f : (real)T.inv_dx;
    const real idy = kFp32 ? (real)T.inv_dy_f : (real)T.inv_dy;
    const real idz = kFp32 ? (real)T.inv_dz_f : (real)T.inv_dz;
    const real dt = kFp32 ? (real)T.dt_f : (real)T.dt;
    const real sxp = limited_face<kFp32>(fxp, pd, rc, rxp);
    const real sxm = limited_face<kFp32>(fxm, pd, rxm, rc);
    const real syp = limited_face<kFp32>(fyp, pd, rc, ryp);
    const real sym = limited_face<kFp32>(fym, pd, rym, rc);
    const real szp = has_top ? limited_face<kFp32>(fzp, pd, rc, rzp) : (real)0;
    const real szm = has_bottom ? limited_face<kFp32>(fzm, pd, rzm, rc) : (real)0;
    const real qc = (real)qraw;
    real rho_phi;
    if (pd)
    {
        real outgoing = 0, incoming = 0;
        if (sxp >= 0) outgoing += sxp * idx; else incoming -= sxp * idx;
        if (sxm <= 0) outgoing -= sxm * idx; else incoming += sxm * idx;
        if (syp >= 0) outgoing += syp * idy; else incoming -= syp * idy;
        if (sym <= 0) outgoing -= sym * idy; else incoming += sym * idy;
        if (has_top) { if (szp >= 0) outgoing += szp * idz; else incoming -= szp * idz; }
        if (has_bottom) { if (szm <= 0) outgoing -= szm * idz; else incoming += szm * idz; }
        rho_phi = (rb * qc - dt * outgoing) + dt * incoming;
    }
    else
    {
        const real div = (sxp - sxm) * idx + (syp - sym) * idy + (szp - szm) * idz;
        if constexpr (kFp32)
        {
            // (rb q - dt div) / denom as q + ((rb - denom) q - dt div) / denom:
            // the small increment carries the FP32 rounding instead of the
            // full value (theta ~ 300 K would lose its perturbation bits).
            rho_phi = (rb - denom) * qc - dt * div;
        }
        else rho_phi = rb * qc - dt * div;
    }
    float out;
    if constexpr (kFp32) out = pd ? __fdividef(rho_phi, denom) : qc + __fdividef(rho_phi, denom);
    else out = (float)(rho_phi / denom);
    if (!isfinite(out)) flags |= kStatusNonfiniteTransport;
    return out;
}

// Donor-limited divergence and density recovery at cell c for every scalar
// (advection_cartesian.cpp:2465-2640).  The output may alias the input: cell
// c reads only its own old value, the fluxes live in the scratch.
template <bool kFp32, class QIn, class QOut>
__device__ __forceinline__ void transport_update_cell(const TransportParams& T, int scalars, QIn&& q_of,
                                                      QOut&& qo_of, const float* __restrict__ rho_end,
                                                      const float* __restrict__ rho_begin,
                                                      const float* __restrict__ sf, const float* __restrict__ rl,
                                                      int c, unsigned& flags)
{
    const Dims d = T.d;
    const size_t n = (size_t)d.cells();
    int i, j, k;
    decompose(d, c, i, j, k);
    if (!(i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1))
    {
        for (int s = 0; s < scalars; ++s)
        {
            const float* q = q_of(s);
            float* qo = qo_of(s);
            if (q != qo) qo[c] = q[c];  // seed_destination_from_source
        }
        return;
    }
    const int cxm = c - d.sx(), cxp = c + d.sx(), cym = c - d.sy(), cyp = c + d.sy();
    const bool has_top = k <= d.nz - 2 || (T.top_open && k == d.nz - 1);
    const float re = rho_end[c], rb = rho_begin[c];
    // Every candidate is loaded up front, so no load waits on a flux sign.
    const int czp = k < d.nz - 1 ? c + 1 : c, czm = k >= 1 ? c - 1 : c;
    for (int s = 0; s < scalars; ++s)
    {
        const bool pd = T.positive_definite[s] != 0;
        const float* __restrict__ sfx = sf + (size_t)s * 3 * n;
        const float* __restrict__ sfy = sfx + n;
        const float* __restrict__ sfz = sfy + n;
        const float* __restrict__ r = rl + (size_t)s * n;
        const float fxp = sfx[c], fxm = sfx[cxm], fyp = sfy[c], fym = sfy[cym];
        const float fzp = sfz[c], fzm = sfz[czm];
        const float qraw = q_of(s)[c];
        float rc = 1.0f, rxp = 1.0f, rxm = 1.0f, ryp = 1.0f, rym = 1.0f, rzp = 1.0f, rzm = 1.0f;
        if (pd)
        {
            rc = r[c]; rxp = r[cxp]; rxm = r[cxm]; ryp = r[cyp]; rym = r[cym]; rzp = r[czp]; rzm = r[czm];
        }
        qo_of(s)[c] = update_value<kFp32>(T, pd, fxp, fxm, fyp, fym, fzp, fzm, rc, rxp, rxm, ryp, rym, rzp, rzm, qraw,
                                          has_top, k >= 1, re, rb, flags);
    }
}

template <bool kFp32>
static __global__ void __launch_bounds__(256) transport_update_kernel(TransportParams T,
                                                                      const float* __restrict__ rho_end,
                                                                      const float* __restrict__ rho_begin,
                                                                      const float* __restrict__ sf,
                                                                      const float* __restrict__ rl, unsigned* status)
{
    const int n = T.d.cells();
    unsigned flags = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        transport_update_cell<kFp32>(T, T.n_scalars, [&](int s) { return T.q_in[s]; }, [&](int s) { return T.q_out[s]; },
                              rho_end, rho_begin, sf, rl, c, flags);
    if (flags) atomicOr(status, flags);
}

// ---- Four scalars interleaved (the member engine) -------------------------
// The engine transports exactly four scalars (theta, qv, qc, qr).  It reads
// them from q4, a [cells] float4 copy of their values before transport (one
// 16-byte load per stencil point instead of four), keeps their face fluxes as
// [3][cells] float4 (x, y, z faces; one lane per scalar) and their limiter
// factors as [cells] float4.  The arithmetic is the per-scalar helpers above,
// so the values equal the planar form's.

__device__ __forceinline__ float lane4(const float4& v, int s)
{
    return s == 0 ? v.x : (s == 1 ? v.y : (s == 2 ? v.z : v.w));
}

// The four face fluxes of one face from its stencil: q4 holds the four
// scalars of every cell.
template <bool kFp32>
__device__ __forceinline__ float4 stencil_flux4(const float4* __restrict__ q4, const FaceStencil& f, float mflux)
{
    float4 p[5];
#pragma unroll
    for (int m = 0; m < 5; ++m) p[m] = q4[f.o[m]];
    if constexpr (kFp32)
    {
        float2 a[5], b[5];
#pragma unroll
        for (int m = 0; m < 5; ++m)
        {
            a[m] = make_float2(p[m].x, p[m].y);
            b[m] = make_float2(p[m].z, p[m].w);
        }
        const float2 ra = stencil_flux_pair_values(a, f, mflux), rb = stencil_flux_pair_values(b, f, mflux);
        return make_float4(ra.x, ra.y, rb.x, rb.y);
    }
    else
    {
        float r[4];
#pragma unroll
        for (int s = 0; s < 4; ++s)
        {
            const float v[5] = {lane4(p[0], s), lane4(p[1], s), lane4(p[2], s), lane4(p[3], s), lane4(p[4], s)};
            r[s] = stencil_flux_values<false>(v, f, mflux);
        }
        return make_float4(r[0], r[1], r[2], r[3]);
    }
}

// The cell functions below take the transport parameters as any type with
// TransportParams' geometry and flag fields (the member engine passes a
// compact copy through the constant bank).
template <bool kFp32, class TP>
__device__ __forceinline__ void transport_faces_cell4(const TP& T, const float4* __restrict__ q4,
                                                      const float* __restrict__ mfx, const float* __restrict__ mfy,
                                                      const float* __restrict__ mfz, float4* __restrict__ sf4, int c)
{
    const Dims d = T.d;
    const size_t n = (size_t)d.cells();
    const int kz_end = T.top_open ? d.nz : d.nz - 1;
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool hx = i <= d.nx - 2, hy = j <= d.ny - 2, hz = k < kz_end, top = k == d.nz - 1;
    const float fx = hx ? mfx[c] : 0.0f, fy = hy ? mfy[c] : 0.0f, fz = hz ? mfz[c] : 0.0f;
    const FaceStencil sx = face_stencil(c - i * d.sx(), d.sx(), i, d.nx, fx >= 0.0f, T.weno);
    const FaceStencil sy = face_stencil(c - j * d.sy(), d.sy(), j, d.ny, fy >= 0.0f, T.weno);
    const FaceStencil sz = face_stencil(c - k, 1, top ? k - 1 : k, d.nz, fz >= 0.0f, T.weno);
    float4 ox = make_float4(0.0f, 0.0f, 0.0f, 0.0f), oy = ox, oz = ox;
    if (hx) ox = stencil_flux4<kFp32>(q4, sx, fx);
    if (hy) oy = stencil_flux4<kFp32>(q4, sy, fy);
    if (hz)
    {
        if (top)
        {
            const float4 q = q4[c];
            if constexpr (kFp32) oz = make_float4(fz * q.x, fz * q.y, fz * q.z, fz * q.w);
            else
            {
                const double f = (double)fz;
                oz = make_float4((float)(f * (double)q.x), (float)(f * (double)q.y), (float)(f * (double)q.z),
                                 (float)(f * (double)q.w));
            }
        }
        else oz = stencil_flux4<kFp32>(q4, sz, fz);
    }
    sf4[c] = ox;
    sf4[n + c] = oy;
    sf4[2 * n + c] = oz;
}

template <bool kFp32, class TP>
__device__ __forceinline__ void transport_limiter_cell4(const TP& T, const float4* __restrict__ q4,
                                                        const float* __restrict__ rho_begin,
                                                        const float4* __restrict__ sf4, float4* __restrict__ rl4,
                                                        int c)
{
    const Dims d = T.d;
    const size_t n = (size_t)d.cells();
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool xm = i >= 1, xp = i <= d.nx - 2, ym = j >= 1, yp = j <= d.ny - 2, zm = k >= 1;
    const bool zp = k <= d.nz - 2 || (T.top_open && k == d.nz - 1);
    const int cxm = xm ? c - d.sx() : c, cym = ym ? c - d.sy() : c, czm = zm ? c - 1 : c;
    const float4 fxp = sf4[c], fxm = sf4[cxm], fyp = sf4[n + c], fym = sf4[n + cym];
    const float4 fzp = sf4[2 * n + c], fzm = sf4[2 * n + czm];
    const float rb = rho_begin[c];
    const float4 q = q4[c];
    float r[4];
#pragma unroll
    for (int s = 0; s < 4; ++s)
        r[s] = T.positive_definite[s]
                   ? limiter_factor<kFp32>(T, lane4(fxp, s), lane4(fxm, s), lane4(fyp, s), lane4(fym, s),
                                           lane4(fzp, s), lane4(fzm, s), xp, xm, yp, ym, zp, zm, rb, lane4(q, s))
                   : 1.0f;
    rl4[c] = make_float4(r[0], r[1], r[2], r[3]);
}

template <bool kFp32, class TP, class QIn, class QOut>
__device__ __forceinline__ void transport_update_cell4(const TP& T, const float4* __restrict__ q4,
                                                       QIn&& q_of, QOut&& qo_of,
                                                       const float* __restrict__ rho_end,
                                                       const float* __restrict__ rho_begin,
                                                       const float4* __restrict__ sf4,
                                                       const float4* __restrict__ rl4, int c, unsigned& flags)
{
    const Dims d = T.d;
    const size_t n = (size_t)d.cells();
    int i, j, k;
    decompose(d, c, i, j, k);
    if (!(i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1))
    {
#pragma unroll
        for (int s = 0; s < 4; ++s)
        {
            const float* q = q_of(s);
            float* qo = qo_of(s);
            if (q != qo) qo[c] = q[c];  // seed_destination_from_source
        }
        return;
    }
    const int cxm = c - d.sx(), cxp = c + d.sx(), cym = c - d.sy(), cyp = c + d.sy();
    const int czp = k < d.nz - 1 ? c + 1 : c, czm = k >= 1 ? c - 1 : c;
    const bool has_top = k <= d.nz - 2 || (T.top_open && k == d.nz - 1);
    const float4 fxp = sf4[c], fxm = sf4[cxm], fyp = sf4[n + c], fym = sf4[n + cym];
    const float4 fzp = sf4[2 * n + c], fzm = sf4[2 * n + czm];
    const float4 rc = rl4[c], rxp = rl4[cxp], rxm = rl4[cxm], ryp = rl4[cyp], rym = rl4[cym];
    const float4 rzp = rl4[czp], rzm = rl4[czm];
    const float re = rho_end[c], rb = rho_begin[c];
    const float4 q = q4[c];
    const float qraw[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int s = 0; s < 4; ++s)
    {
        const bool pd = T.positive_definite[s] != 0;
        qo_of(s)[c] = update_value<kFp32>(
            T, pd, lane4(fxp, s), lane4(fxm, s), lane4(fyp, s), lane4(fym, s), lane4(fzp, s), lane4(fzm, s),
            pd ? lane4(rc, s) : 1.0f, pd ? lane4(rxp, s) : 1.0f, pd ? lane4(rxm, s) : 1.0f, pd ? lane4(ryp, s) : 1.0f,
            pd ? lane4(rym, s) : 1.0f, pd ? lane4(rzp, s) : 1.0f, pd ? lane4(rzm, s) : 1.0f, qraw[s], has_top, k >= 1,
            re, rb, flags);
    }
}

}  // namespace nimbus
