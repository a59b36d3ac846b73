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
};

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

// Face value for face l+1/2 on an axis of extent n, cells at q[base + m*stride].
__device__ __forceinline__ double face_value(const float* __restrict__ q, int base, int stride, int l, int n,
                                             double mflux, int weno)
{
#define NQ(m) ((double)q[base + (m) * stride])
    if (mflux >= 0.0)
    {
        const double q0 = NQ(l);
        if (weno && l >= 2 && l + 2 <= n - 1) return weno5_face(NQ(l - 2), NQ(l - 1), q0, NQ(l + 1), NQ(l + 2));
        const double sl = (l >= 1) ? mc_slope(NQ(l - 1), q0, NQ(l + 1)) : 0.0;
        return q0 + 0.5 * sl;
    }
    const double q0 = NQ(l + 1);
    if (weno && l - 1 >= 0 && l + 3 <= n - 1) return weno5_face(NQ(l + 3), NQ(l + 2), q0, NQ(l), NQ(l - 1));
    const double sl = (l + 1 <= n - 2) ? mc_slope(NQ(l), q0, NQ(l + 2)) : 0.0;
    return q0 - 0.5 * sl;
#undef NQ
}

// FP32 face offset from the donor value: weno5_face_offset_fp32
// (include/numerics/advection/weno5_face.hpp:88-120), the reference's own FP32
// GPU reconstruction (scale-normalised, so moisture-scale fields keep their
// nonlinear weights).
__device__ __forceinline__ float weno5_offset_f32(float a, float b, float c, float d, float e)
{
    const float magnitude = fmaxf(fmaxf(fmaxf(fabsf(a), fabsf(b)), fmaxf(fabsf(c), fabsf(d))), fabsf(e));
    const float scale = fmaxf(magnitude, 1e-20f);
    if (!isfinite(scale)) return 0.0f;
    const float inv = __frcp_rn(scale);
    auto diff = [&](float value) {
        const float delta = value - c;
        return isfinite(delta) ? delta * inv : value * inv - c * inv;
    };
    const float ac = diff(a), bc = diff(b), dc = diff(d), ec = diff(e);
    const float p0 = (1.0f / 3.0f) * ac - (7.0f / 6.0f) * bc;
    const float p1 = -(1.0f / 6.0f) * bc + (1.0f / 3.0f) * dc;
    const float p2 = (5.0f / 6.0f) * dc - (1.0f / 6.0f) * ec;
    const float s0a = ac - 2.0f * bc, s0b = ac - 4.0f * bc;
    const float s1a = bc + dc, s1b = bc - dc;
    const float s2a = ec - 2.0f * dc, s2b = ec - 4.0f * dc;
    const float b0 = (13.0f / 12.0f) * s0a * s0a + 0.25f * s0b * s0b;
    const float b1 = (13.0f / 12.0f) * s1a * s1a + 0.25f * s1b * s1b;
    const float b2 = (13.0f / 12.0f) * s2a * s2a + 0.25f * s2b * s2b;
    const float relative = magnitude * inv;
    const float flo = 1e-20f * inv;
    const float epsilon = 1e-6f * relative * relative + flo * flo;
    const float e0 = epsilon + b0, e1 = epsilon + b1, e2 = epsilon + b2;
    const float minimum = fminf(fminf(e0, e1), e2);
    const float r0 = __fdividef(minimum, e0), r1 = __fdividef(minimum, e1), r2 = __fdividef(minimum, e2);
    const float a0 = 0.1f * r0 * r0, a1 = 0.6f * r1 * r1, a2 = 0.3f * r2 * r2;
    const float sum = a0 + a1 + a2;
    const float offset = scale * __fdividef(a0 * p0 + a1 * p1 + a2 * p2, sum);
    return isfinite(offset) ? offset : 0.0f;
}

__device__ __forceinline__ float mc_slope_f32(float qm, float q0, float qp)
{
    const float right = qp - q0, left = q0 - qm;
    const float a = 0.5f * (right + left), b = 2.0f * right, c = 2.0f * left;
    if (a > 0.0f && b > 0.0f && c > 0.0f) return fminf(a, fminf(b, c));
    if (a < 0.0f && b < 0.0f && c < 0.0f) return fmaxf(a, fmaxf(b, c));
    return 0.0f;
}

// FP32 scalar face flux M*phi as M*base + M*offset (the reference's FP32 GPU form).
__device__ __forceinline__ float face_flux_f32(const float* __restrict__ q, int base, int stride, int l, int n,
                                               float mflux, int weno)
{
#define NQ(m) (q[base + (m) * stride])
    float donor, offset;
    if (mflux >= 0.0f)
    {
        donor = NQ(l);
        if (weno && l >= 2 && l + 2 <= n - 1) offset = weno5_offset_f32(NQ(l - 2), NQ(l - 1), donor, NQ(l + 1), NQ(l + 2));
        else offset = 0.5f * ((l >= 1) ? mc_slope_f32(NQ(l - 1), donor, NQ(l + 1)) : 0.0f);
    }
    else
    {
        donor = NQ(l + 1);
        if (weno && l - 1 >= 0 && l + 3 <= n - 1) offset = weno5_offset_f32(NQ(l + 3), NQ(l + 2), donor, NQ(l), NQ(l - 1));
        else offset = -0.5f * ((l + 1 <= n - 2) ? mc_slope_f32(NQ(l), donor, NQ(l + 2)) : 0.0f);
    }
    return __fmaf_rn(mflux, donor, mflux * offset);
#undef NQ
}

// Face fluxes of scalar s owned by cell c (its +x, +y and +z faces).
// kFp32 selects the reference's FP32 GPU form (face_flux_f32), otherwise FP64
// face values rounded once to the FP32 scratch.
// sf points at the scalar's [3][cells] face-flux scratch (x, y, z).
template <bool kFp32>
__device__ __forceinline__ void transport_faces_cell(const TransportParams& T, const float* __restrict__ q,
                                                     const float* __restrict__ mfx, const float* __restrict__ mfy,
                                                     const float* __restrict__ mfz, float* __restrict__ sf, int c)
{
    const Dims d = T.d;
    const int n = d.cells();
    float* __restrict__ sfx = sf;
    float* __restrict__ sfy = sfx + n;
    float* __restrict__ sfz = sfy + n;
    const int kz_end = T.top_open ? d.nz : d.nz - 1;
    int i, j, k;
    decompose(d, c, i, j, k);
    if constexpr (kFp32)
    {
        if (i <= d.nx - 2) sfx[c] = face_flux_f32(q, c - i * d.sx(), d.sx(), i, d.nx, mfx[c], T.weno);
        if (j <= d.ny - 2) sfy[c] = face_flux_f32(q, c - j * d.sy(), d.sy(), j, d.ny, mfy[c], T.weno);
        if (k < kz_end)
        {
            const float mf = mfz[c];
            sfz[c] = (k == d.nz - 1) ? mf * q[c] : face_flux_f32(q, c - k, 1, k, d.nz, mf, T.weno);
        }
    }
    else
    {
        if (i <= d.nx - 2)
        {
            const double mf = (double)mfx[c];
            sfx[c] = (float)(mf * face_value(q, c - i * d.sx(), d.sx(), i, d.nx, mf, T.weno));
        }
        if (j <= d.ny - 2)
        {
            const double mf = (double)mfy[c];
            sfy[c] = (float)(mf * face_value(q, c - j * d.sy(), d.sy(), j, d.ny, mf, T.weno));
        }
        if (k < kz_end)
        {
            const double mf = (double)mfz[c];
            if (k == d.nz - 1) sfz[c] = (float)(mf * (double)q[c]);
            else sfz[c] = (float)(mf * face_value(q, c - k, 1, k, d.nz, mf, T.weno));
        }
    }
}

template <bool kFp32>
static __global__ void __launch_bounds__(256) transport_faces_kernel(TransportParams T, const float* __restrict__ mfx,
                                                              const float* __restrict__ mfy,
                                                              const float* __restrict__ mfz, float* __restrict__ sf)
{
    const int n = T.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        transport_faces_cell<kFp32>(T, T.q_in[blockIdx.y], mfx, mfy, mfz, sf + (size_t)blockIdx.y * 3 * n, c);
}

// conservative_pd_limiter_factor (advection_cartesian.hpp:101-108), non-support path.
__device__ __forceinline__ float pd_limiter_factor(double r)
{
    if (!(r > 0.0 && r < 1.0)) return (float)r;
    const float roundoff = 1.0f - 32.0f * 1.1920928955078125e-7f;
    const float stored = (float)r;
    return nextafterf(__fmul_rn(stored, roundoff), 0.0f);
}

// Positive-definite donor ratio of scalar s at cell c (advection_cartesian.cpp:2174-2240).
// sf is the scalar's face-flux scratch, rl its [cells] limiter factors.
__device__ __forceinline__ void transport_limiter_cell(const TransportParams& T, const float* __restrict__ q,
                                                       const float* __restrict__ rho_begin,
                                                       const float* __restrict__ sf, float* __restrict__ r_out, int c)
{
    const Dims d = T.d;
    const int n = d.cells();
    const float* __restrict__ sfx = sf;
    const float* __restrict__ sfy = sfx + n;
    const float* __restrict__ sfz = sfy + n;
    int i, j, k;
    decompose(d, c, i, j, k);
    double out = 0.0;
    if (i <= d.nx - 2 && sfx[c] > 0.0f) out += (double)sfx[c] * T.inv_dx;
    if (i >= 1 && sfx[c - d.sx()] < 0.0f) out -= (double)sfx[c - d.sx()] * T.inv_dx;
    if (j <= d.ny - 2 && sfy[c] > 0.0f) out += (double)sfy[c] * T.inv_dy;
    if (j >= 1 && sfy[c - d.sy()] < 0.0f) out -= (double)sfy[c - d.sy()] * T.inv_dy;
    if ((k <= d.nz - 2 || (T.top_open && k == d.nz - 1)) && sfz[c] > 0.0f) out += (double)sfz[c] * T.inv_dz;
    if (k >= 1 && sfz[c - 1] < 0.0f) out -= (double)sfz[c - 1] * T.inv_dz;
    double r = 1.0;
    if (out > 0.0)
    {
        const double qc = (double)q[c];
        const double available = (double)rho_begin[c] * ((qc < 0.0) ? 0.0 : qc) / T.dt;  // std::max(q, 0.0)
        const double ratio = available / out;
        r = (ratio < 1.0) ? ratio : 1.0;  // std::min(1.0, ratio), NaN -> 1
    }
    r_out[c] = pd_limiter_factor(r);
}

static __global__ void __launch_bounds__(256) transport_limiter_kernel(TransportParams T, const float* __restrict__ rho_begin,
                                                                const float* __restrict__ sf, float* __restrict__ rl)
{
    const int s = blockIdx.y;
    if (!T.positive_definite[s]) return;
    const int n = T.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        transport_limiter_cell(T, T.q_in[s], rho_begin, sf + (size_t)s * 3 * n, rl + (size_t)s * n, c);
}

__device__ __forceinline__ double limited_flux(float raw, bool pd, const float* __restrict__ rl, int lo, int hi)
{
    if (!pd || raw == 0.0f) return (double)raw;
    const float r = raw > 0.0f ? rl[lo] : rl[hi];
    return (double)raw * (double)r;
}

// Donor-limited divergence and density recovery of scalar s at cell c
// (advection_cartesian.cpp:2465-2640).  q_out may alias q_in: cell c reads
// only its own old value, the fluxes live in the scratch.
__device__ __forceinline__ void transport_update_cell(const TransportParams& T, bool pd, const float* q, float* qo,
                                                      const float* __restrict__ rho_end,
                                                      const float* __restrict__ rho_begin,
                                                      const float* __restrict__ sf, const float* __restrict__ r,
                                                      int c, unsigned& flags)
{
    const Dims d = T.d;
    const int n = d.cells();
    const float* __restrict__ sfx = sf;
    const float* __restrict__ sfy = sfx + n;
    const float* __restrict__ sfz = sfy + n;
    int i, j, k;
    decompose(d, c, i, j, k);
    if (!(i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1))
    {
        if (q != qo) qo[c] = q[c];  // seed_destination_from_source
        return;
    }
    const int cxm = c - d.sx(), cxp = c + d.sx(), cym = c - d.sy(), cyp = c + d.sy();
    const bool has_top = k <= d.nz - 2 || (T.top_open && k == d.nz - 1);
    const double sxp = limited_flux(sfx[c], pd, r, c, cxp);
    const double sxm = limited_flux(sfx[cxm], pd, r, cxm, c);
    const double syp = limited_flux(sfy[c], pd, r, c, cyp);
    const double sym = limited_flux(sfy[cym], pd, r, cym, c);
    const double szp = has_top ? limited_flux(sfz[c], pd, r, c, k < d.nz - 1 ? c + 1 : c) : 0.0;
    const double szm = (k >= 1) ? limited_flux(sfz[c - 1], pd, r, c - 1, c) : 0.0;
    const double re = (double)rho_end[c];
    const double rb = (double)rho_begin[c];
    const double qc = (double)q[c];
    double rho_phi;
    if (pd)
    {
        double outgoing = 0.0, incoming = 0.0;
        if (sxp >= 0.0) outgoing += sxp * T.inv_dx; else incoming -= sxp * T.inv_dx;
        if (sxm <= 0.0) outgoing -= sxm * T.inv_dx; else incoming += sxm * T.inv_dx;
        if (syp >= 0.0) outgoing += syp * T.inv_dy; else incoming -= syp * T.inv_dy;
        if (sym <= 0.0) outgoing -= sym * T.inv_dy; else incoming += sym * T.inv_dy;
        if (has_top) { if (szp >= 0.0) outgoing += szp * T.inv_dz; else incoming -= szp * T.inv_dz; }
        if (k >= 1) { if (szm <= 0.0) outgoing -= szm * T.inv_dz; else incoming += szm * T.inv_dz; }
        rho_phi = (rb * qc - T.dt * outgoing) + T.dt * incoming;
    }
    else
    {
        const double div = (sxp - sxm) * T.inv_dx + (syp - sym) * T.inv_dy + (szp - szm) * T.inv_dz;
        rho_phi = rb * qc - T.dt * div;
    }
    const double denom = (re > T.rho_floor) ? re : T.rho_floor;
    const float out = (float)(rho_phi / denom);
    if (!isfinite(out)) flags |= kStatusNonfiniteTransport;
    qo[c] = out;
}

static __global__ void __launch_bounds__(256) transport_update_kernel(TransportParams T, const float* __restrict__ rho_end,
                                                               const float* __restrict__ rho_begin,
                                                               const float* __restrict__ sf,
                                                               const float* __restrict__ rl, unsigned* status)
{
    const int n = T.d.cells();
    unsigned flags = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        const int s = blockIdx.y;
        transport_update_cell(T, T.positive_definite[s] != 0, T.q_in[s], T.q_out[s], rho_end, rho_begin,
                              sf + (size_t)s * 3 * n, rl + (size_t)s * n, c, flags);
    }
    if (flags) atomicOr(status, flags);
}

}  // namespace nimbus
