// One-launch acoustic substep (continuity, EOS, momentum and the retained
// mass-flux accumulation) for the flat Cartesian C-grid, sm_100a.
//
// Decomposition ("2.5-D" marching): a CTA owns a strip of TJ consecutive
// j-rows with the full vertical column (for a fixed i that strip is one
// contiguous run of TJ*nz floats, so every plane load is one contiguous,
// perfectly coalesced copy) and marches along i over a chunk of planes.
// Old-state planes stream into rolling shared-memory slots with cp.async
// (16-byte LDGSTS, bypassing registers); the copies for plane i+2 are in
// flight while plane i+1's new density and pressure and plane i's momentum
// are computed.  New rho/p are formed once per plane on the strip plus one
// halo row (the only redundant work); halo rows of the old state come from
// L2, so DRAM sees each field close to once per substep.
//
// Precision policies:
//   RefPolicy   FP64 interior arithmetic in the reference's operation order
//               (acoustic_cgrid_fast.cpp:47-215), EOS via pow(): bit-identical
//               to the CPU solver when compiled with --fmad=false.
//   Fp32Policy  FP32 arithmetic throughout; the base state enters in FP64 (the
//               hydrostatic difference p0[k+1]-p0[k] as an FP32 hi+lo pair, so
//               the w equation's cancellation stays exact to ~1e-7); the EOS is
//               the compensated binomial form of substep_pressure (within
//               about half an FP32 ulp of FP64), and the retained mass-flux
//               sums and the density update are single-rounding FMAs.
#pragma once

#include "stencil_common.cuh"

namespace nimbus
{

struct FusedParams
{
    Dims d;
    double inv_dx, inv_dy, inv_dz;
    double dt_small;
    double gamma;
    float rho_min, rho_max, p_min, p_max, p_ref_fallback, wind_h, wind_v;
    double weight;           // mass-flux weight; mfx == nullptr disables accumulation
    double frame_u, frame_v;
    int top_open;
    int chunk;               // i-planes per CTA
    unsigned nz_magic;       // fast t / nz (see fused_nz_magic)
    int vec4;                // 1: 16-byte copies (nz % 4 == 0 and 16-byte aligned bases)
    // FP32 form: the scalars above rounded once, and the binomial-series
    // coefficients binom(gamma, n), n = 1..6, of the EOS (substep_pressure).
    float inv_dx_f, inv_dy_f, inv_dz_f, dt_f, weight_f, frame_u_f, frame_v_f;
    float eos_c[6];
};

// Derives the FP32 copies of a filled parameter block.
__host__ __device__ inline void finish_fp32(FusedParams& P)
{
    P.inv_dx_f = (float)P.inv_dx;
    P.inv_dy_f = (float)P.inv_dy;
    P.inv_dz_f = (float)P.inv_dz;
    P.dt_f = (float)P.dt_small;
    P.weight_f = (float)P.weight;
    P.frame_u_f = (float)P.frame_u;
    P.frame_v_f = (float)P.frame_v;
    double c = 1.0;
    for (int n = 1; n <= 6; ++n)
    {
        c *= (P.gamma - (n - 1)) / n;
        P.eos_c[n - 1] = (float)c;
    }
}

struct RefPolicy
{
    using real = double;
    static constexpr bool exact_pow = true;
};
struct Fp32Policy
{
    using real = float;
    static constexpr bool exact_pow = false;
};

// floor(t / nz) as (t * magic) >> 32 with magic = ceil(2^32 / nz); exact for
// t < 2^32 / nz, far above the TJ*nz*4 window indices used here.
__host__ __device__ __forceinline__ unsigned fused_nz_magic(unsigned nz)
{
    return (unsigned)((0x100000000ull + nz - 1) / nz);
}
__device__ __forceinline__ int fast_div(int t, unsigned magic) { return (int)__umulhi((unsigned)t, magic); }

__device__ __forceinline__ void cp_async16(float* smem, const float* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(float* smem, const float* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_0() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Stores the FP64 weighted sum into an FP32 mass-flux slot; a non-finite
// result (of the sum or of its rounding) leaves the slot and flags the call
// (advection_cartesian.cpp:743-758).
__device__ __forceinline__ void fused_accumulate(float* slot, double weight, double flux, unsigned& flags)
{
    const float st = (float)((double)*slot + weight * flux);
    if (isfinite(st)) *slot = st;
    else flags |= kStatusNonfiniteMassFlux;
}

// Per-level base data, from the FP64 pressure profile: the hydrostatic
// difference p0[k+1] - p0[k] as an FP32 hi+lo pair (the w equation of the
// FP32 form), and for the FP32 EOS p0 and b = (R_d / p00) / x0 as hi+lo pairs,
// where x0 = (p0 / p00)^(1/gamma) is the EOS argument at the base pressure.
static __global__ void level_base_kernel(const double* __restrict__ p0, int nz, double gamma,
                                         float2* __restrict__ dp0, float4* __restrict__ eos0)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nz) return;
    const double dp = (k + 1 < nz) ? p0[k + 1] - p0[k] : 0.0;
    const float hi = (float)dp;
    dp0[k] = make_float2(hi, (float)(dp - (double)hi));
    const double x0 = pow(p0[k] / kP00, 1.0 / gamma);
    const double b = (kRd / kP00) / x0;
    const float ph = (float)p0[k], bh = (float)b;
    eos0[k] = make_float4(ph, (float)(p0[k] - (double)ph), bh, (float)(b - (double)bh));
}

// The retained mass-flux increment of the FP32 form: one FMA, the weighted
// flux added to the stored sum and rounded once to the FP32 slot -- the same
// single rounding as the reference's FP64 add stored to FP32
// (advection_cartesian.cpp:768-775), without leaving FP32.  With store the
// slot starts from zero (first substep of a large step).
__device__ __forceinline__ void retain_flux_f32(float* slot, float weight, float flux, unsigned& flags, bool store)
{
    const float st = __fmaf_rn(weight, flux, store ? 0.0f : *slot);
    if (isfinite(st)) *slot = st;
    else
    {
        if (store) *slot = 0.0f;
        flags |= kStatusNonfiniteMassFlux;
    }
}

// rho forward Euler + fallback + clamp (acoustic_cgrid_fast.cpp:120-135).
// Reference policy: FP64 add rounded once; FP32 policy: one FMA.
template <class Policy>
__device__ __forceinline__ float substep_density(const FusedParams& P, float rho_c, float drho_stored,
                                                 const double* __restrict__ rho0, int k)
{
    if constexpr (Policy::exact_pow)
    {
        double rho_new = (double)rho_c + (double)drho_stored * P.dt_small;
        if (!isfinite(rho_new) || rho_new <= 0.0)
        {
            const double b = rho0[k];
            rho_new = (0.1 < b) ? b : 0.1;
        }
        return clamp_value((float)rho_new, 1.0f, P.rho_min, P.rho_max);
    }
    else
    {
        float rn = __fmaf_rn(drho_stored, P.dt_f, rho_c);
        if (!isfinite(rn) || rn <= 0.0f)
        {
            const double b = rho0[k];
            rn = (float)((0.1 < b) ? b : 0.1);
        }
        return clamp_value(rn, 1.0f, P.rho_min, P.rho_max);
    }
}

// EOS pressure p = p00 (rho R_d theta / p00)^gamma + fallback + clamp
// (acoustic_cgrid_fast.cpp:136-157).  Reference policy: pow in FP64.  FP32
// policy: p = p0 (1 + d)^gamma with 1 + d = rho theta b, the product formed
// exactly as an FP32 hi+lo pair so d keeps full precision, and (1 + d)^gamma - 1
// summed by its binomial series to the sixth power (|d| <= 1/16: the
// truncation is below 2e-11 relative); the result is within about half an
// FP32 ulp of the FP64 value.  Larger |d| take the FP64 route.
template <class Policy>
__device__ __forceinline__ float substep_pressure(const FusedParams& P, const float4* __restrict__ eos0, int k,
                                                  float rho_stored, float th)
{
    if constexpr (Policy::exact_pow)
    {
        double p_new = (double)P.p_ref_fallback;
        const double thv = (double)th;
        if (thv > 0.0)
        {
            const double x = (double)rho_stored * kRd * thv / kP00;
            p_new = kP00 * pow(x, P.gamma);
        }
        if (!isfinite(p_new) || p_new <= 0.0) p_new = (double)P.p_ref_fallback;
        return clamp_value((float)p_new, 101325.0f, P.p_min, P.p_max);
    }
    else
    {
        float p = P.p_ref_fallback;
        if (th > 0.0f)
        {
            const float4 e = eos0[k];
            const float rt = rho_stored * th;
            const float rt_lo = __fmaf_rn(rho_stored, th, -rt);
            const float r = rt * e.z;
            const float r_lo = __fmaf_rn(rt, e.z, -r) + __fmaf_rn(rt, e.w, rt_lo * e.z);
            const float dl = (r - 1.0f) + r_lo;
            if (fabsf(dl) <= 0.0625f)
            {
                float sum = P.eos_c[5];
                for (int n = 4; n >= 0; --n) sum = __fmaf_rn(sum, dl, P.eos_c[n]);
                p = e.x + __fmaf_rn(e.x, sum * dl, e.y);
            }
            else
            {
                double pd = kP00 * exp(P.gamma * log((double)rho_stored * kRd * (double)th / kP00));
                if (!isfinite(pd) || pd <= 0.0) pd = (double)P.p_ref_fallback;
                p = (float)pd;
            }
        }
        return clamp_value(p, 101325.0f, P.p_min, P.p_max);
    }
}

template <int TJ>
struct FusedSmem
{
    // Rolling plane slots, each [rows][nz]:
    //   rho_old 4 slots, rows j0-1 .. j0+TJ+1 (TJ+3)
    //   u_old   3 slots, rows j0 .. j0+TJ     (TJ+1)
    //   v_old   3 slots, rows j0-1 .. j0+TJ   (TJ+2)
    //   w_old   3 slots, rows j0 .. j0+TJ     (TJ+1)
    //   theta   2 slots, rows j0 .. j0+TJ     (TJ+1)
    //   rho_new, p_new 2 slots each           (TJ+1)
    static constexpr int rows_rho = TJ + 3, rows_e = TJ + 1, rows_v = TJ + 2;
    static constexpr int slots_rho = 4, slots_uvw = 3, slots_th = 2, slots_new = 2;
    static size_t floats(int nz)
    {
        return (size_t)nz * (slots_rho * rows_rho + slots_uvw * (rows_e + rows_v + rows_e) + slots_th * rows_e +
                             2 * slots_new * rows_e);
    }
};

template <int TJ, int BLOCK, class Policy>
static __global__ void __launch_bounds__(BLOCK, 3) acoustic_substep_fused_kernel(
    FusedParams P, const float* __restrict__ rho_in, const float* __restrict__ u_in, const float* __restrict__ v_in,
    const float* __restrict__ w_in, const float* __restrict__ theta, const double* __restrict__ rho0,
    const double* __restrict__ p0, const float2* __restrict__ dp0_split, const float4* __restrict__ eos0,
    float* __restrict__ drho_out,
    float* __restrict__ rho_out, float* __restrict__ p_out, float* __restrict__ u_out, float* __restrict__ v_out,
    float* __restrict__ w_out, float* __restrict__ mfx, float* __restrict__ mfy, float* __restrict__ mfz,
    unsigned* __restrict__ status)
{
    using real = typename Policy::real;
    using S = FusedSmem<TJ>;
    extern __shared__ __align__(16) float smem[];
    const Dims d = P.d;
    const int nz = d.nz;
    const int sx = d.sx();
    const unsigned magic = P.nz_magic;
    const int strips = (d.ny + TJ - 1) / TJ;
    const int strip = blockIdx.x % strips;
    const int chunk_id = blockIdx.x / strips;
    const int j0 = strip * TJ;
    const int i_begin = chunk_id * P.chunk;
    if (i_begin >= d.nx) return;
    const int i_end = min(d.nx, i_begin + P.chunk);
    const int tj = min(TJ, d.ny - j0);  // rows owned by this strip

    const int plane_rho = S::rows_rho * nz, plane_e = S::rows_e * nz, plane_v = S::rows_v * nz;
    float* s_rho = smem;
    float* s_u = s_rho + S::slots_rho * plane_rho;
    float* s_v = s_u + S::slots_uvw * plane_e;
    float* s_w = s_v + S::slots_uvw * plane_v;
    float* s_th = s_w + S::slots_uvw * plane_e;
    float* s_rn = s_th + S::slots_th * plane_e;
    float* s_pn = s_rn + S::slots_new * plane_e;

    // Plane slots; plane indices are >= -1.
    auto rho_slot = [&](int i) { return s_rho + ((i + 4) & 3) * plane_rho; };
    auto u_slot = [&](int i) { return s_u + ((i + 3) % 3) * plane_e; };
    auto v_slot = [&](int i) { return s_v + ((i + 3) % 3) * plane_v; };
    auto w_slot = [&](int i) { return s_w + ((i + 3) % 3) * plane_e; };
    auto th_slot = [&](int i) { return s_th + ((i + 2) & 1) * plane_e; };
    auto rn_slot = [&](int i) { return s_rn + ((i + 2) & 1) * plane_e; };
    auto pn_slot = [&](int i) { return s_pn + ((i + 2) & 1) * plane_e; };

    // Asynchronously copy rows (j0-first) .. (j0-first+rows-1) of plane i into
    // dst; rows outside the domain (and planes outside [0,nx)) are zero-filled.
    auto stage = [&](float* dst, const float* __restrict__ src, int i, int first, int rows) {
        const int jlo = j0 - first;
        const int n = rows * nz;
        int r_lo = 0, r_hi = 0;
        if (i >= 0 && i < d.nx)
        {
            r_lo = max(0, -jlo);
            r_hi = max(r_lo, min(rows, d.ny - jlo));
        }
        const int z_lo = r_lo * nz, z_hi = r_hi * nz;
        for (int t = threadIdx.x; t < z_lo; t += BLOCK) dst[t] = 0.0f;
        for (int t = z_hi + threadIdx.x; t < n; t += BLOCK) dst[t] = 0.0f;
        if (z_hi > z_lo)
        {
            const float* base = src + (size_t)i * sx + (size_t)(jlo + r_lo) * nz;
            float* out = dst + z_lo;
            const int m = z_hi - z_lo;
            if (P.vec4)
            {
                for (int t = threadIdx.x; t < (m >> 2); t += BLOCK) cp_async16(out + 4 * t, base + 4 * t);
            }
            else
            {
                for (int t = threadIdx.x; t < m; t += BLOCK) cp_async4(out + t, base + t);
            }
        }
    };
    // Old-state inputs of plane i's continuity (rho of plane i+1 included).
    auto stage_plane = [&](int i) {
        stage(rho_slot(i + 1), rho_in, i + 1, 1, S::rows_rho);
        stage(u_slot(i), u_in, i, 0, S::rows_e);
        stage(v_slot(i), v_in, i, 1, S::rows_v);
        stage(w_slot(i), w_in, i, 0, S::rows_e);
        stage(th_slot(i), theta, i, 0, S::rows_e);
    };

    // New density and pressure of plane i on rows j0 .. j0+tj (strip + halo row).
    // Window index t = r*nz + k for the u/w/theta/new windows; the rho and v
    // windows start one row above the strip, so their index is t + nz.
    auto form_rho_p = [&](int i) {
        const float* rm = rho_slot(i - 1);
        const float* rc_ = rho_slot(i);
        const float* rp = rho_slot(i + 1);
        const float* uc = u_slot(i);
        const float* um = u_slot(i - 1);
        const float* vc = v_slot(i);
        const float* wc = w_slot(i);
        const float* th = th_slot(i);
        float* rn = rn_slot(i);
        float* pn = pn_slot(i);
        const int rows = min(tj + 1, d.ny - j0);
        const int n = rows * nz;
        const bool interior_i = i >= 1 && i < d.nx - 1;
        for (int t = threadIdx.x; t < n; t += BLOCK)
        {
            const int r = fast_div(t, magic), k = t - r * nz;
            const int j = j0 + r;
            const int cr = t + nz;
            const float rho_c = rc_[cr];
            double drho = 0.0;
            if (interior_i && j >= 1 && j < d.ny - 1)
            {
                const real rcv = (real)rho_c;
                const real half = (real)0.5;
                const real fx_pos = half * (rcv + (real)rp[cr]) * (real)uc[t];
                const real fx_neg = half * ((real)rm[cr] + rcv) * (real)um[t];
                const real fy_pos = half * (rcv + (real)rc_[cr + nz]) * (real)vc[cr];
                const real fy_neg = half * ((real)rc_[cr - nz] + rcv) * (real)vc[cr - nz];
                const real fz_pos = (k + 1 < nz) ? half * (rcv + (real)rc_[cr + 1]) * (real)wc[t] : rcv * (real)wc[t];
                const real fz_neg = (k > 0) ? half * ((real)rc_[cr - 1] + rcv) * (real)wc[t - 1] : (real)0;
                drho = (double)(-((fx_pos - fx_neg) * (real)P.inv_dx + (fy_pos - fy_neg) * (real)P.inv_dy +
                                  (fz_pos - fz_neg) * (real)P.inv_dz));
            }
            const float drho_stored = (float)finite_or_zero(drho);
            if (drho_out != nullptr && r < tj) drho_out[(size_t)i * sx + (size_t)j * nz + k] = drho_stored;
            const float rho_stored = substep_density<Policy>(P, rho_c, drho_stored, rho0, k);
            rn[t] = rho_stored;
            pn[t] = substep_pressure<Policy>(P, eos0, k, rho_stored, th[t]);
        }
    };

    // ---- prologue ----
    stage(rho_slot(i_begin - 1), rho_in, i_begin - 1, 1, S::rows_rho);
    stage(rho_slot(i_begin), rho_in, i_begin, 1, S::rows_rho);
    stage(u_slot(i_begin - 1), u_in, i_begin - 1, 0, S::rows_e);
    stage_plane(i_begin);
    cp_async_commit();
    stage_plane(i_begin + 1);
    cp_async_commit();
    cp_async_wait_1();
    __syncthreads();
    form_rho_p(i_begin);

    unsigned flags = 0;
    const int n_owned = tj * nz;
    for (int i = i_begin; i < i_end; ++i)
    {
        // Slots written now (plane i+2, rho plane i+3) were last read before
        // the previous iteration's closing barrier.
        stage_plane(i + 2);  // zero-filled past the last plane
        cp_async_commit();
        cp_async_wait_1();   // plane i+1 has landed
        __syncthreads();
        // Retained mass flux from the old state of plane i; publish rho/p of plane i.
        {
            const float* rc_ = rho_slot(i);
            const float* rp = rho_slot(i + 1);
            const float* uc = u_slot(i);
            const float* vc = v_slot(i);
            const float* wc = w_slot(i);
            const float* rn = rn_slot(i);
            const float* pn = pn_slot(i);
            const size_t plane_base = (size_t)i * sx + (size_t)j0 * nz;
            for (int t = threadIdx.x; t < n_owned; t += BLOCK)
            {
                const size_t g = plane_base + t;
                if (mfx != nullptr)
                {
                    const int r = fast_div(t, magic), k = t - r * nz;
                    const int j = j0 + r;
                    const int cr = t + nz;
                    const float rho_c = rc_[cr];
                    if constexpr (sizeof(real) == 8)
                    {
                        const double rcd = (double)rho_c;
                        if (i < d.nx - 1)
                            fused_accumulate(mfx + g, P.weight, 0.5 * (rcd + (double)rp[cr]) * ((double)uc[t] - P.frame_u), flags);
                        if (j < d.ny - 1)
                            fused_accumulate(mfy + g, P.weight, 0.5 * (rcd + (double)rc_[cr + nz]) * ((double)vc[cr] - P.frame_v), flags);
                        const double zf = (k == nz - 1) ? (P.top_open ? rcd * (double)wc[t] : 0.0)
                                                        : 0.5 * (rcd + (double)rc_[cr + 1]) * (double)wc[t];
                        fused_accumulate(mfz + g, P.weight, zf, flags);
                    }
                    else
                    {
                        if (i < d.nx - 1)
                            retain_flux_f32(mfx + g, P.weight_f, 0.5f * (rho_c + rp[cr]) * (uc[t] - P.frame_u_f), flags, false);
                        if (j < d.ny - 1)
                            retain_flux_f32(mfy + g, P.weight_f, 0.5f * (rho_c + rc_[cr + nz]) * (vc[cr] - P.frame_v_f), flags, false);
                        const float zf = (k == nz - 1) ? (P.top_open ? rho_c * wc[t] : 0.0f) : 0.5f * (rho_c + rc_[cr + 1]) * wc[t];
                        retain_flux_f32(mfz + g, P.weight_f, zf, flags, false);
                    }
                }
                rho_out[g] = rn[t];
                p_out[g] = pn[t];
            }
        }
        if (i + 1 < d.nx) form_rho_p(i + 1);
        __syncthreads();
        // Momentum of plane i from the new rho/p of planes i and i+1.
        {
            const float* rn = rn_slot(i);
            const float* pn = pn_slot(i);
            const float* rnx = rn_slot(i + 1);
            const float* pnx = pn_slot(i + 1);
            const float* uc = u_slot(i);
            const float* vc = v_slot(i);
            const float* wc = w_slot(i);
            const size_t plane_base = (size_t)i * sx + (size_t)j0 * nz;
            const bool interior_i = i >= 1 && i < d.nx - 1;
            for (int t = threadIdx.x; t < n_owned; t += BLOCK)
            {
                const int r = fast_div(t, magic), k = t - r * nz;
                const int j = j0 + r;
                float du = 0.0f, dv = 0.0f, dw = 0.0f;
                if (interior_i && j >= 1 && j < d.ny - 1 && k < nz - 1)
                {
                    if constexpr (sizeof(real) == 8)
                    {
                        const double rc = (double)rn[t];
                        const double rho_x = 0.5 * (rc + (double)rnx[t]);
                        const double rho_y = 0.5 * (rc + (double)rn[t + nz]);
                        const double rho_z = 0.5 * (rc + (double)rn[t + 1]);
                        const double pc = (double)pn[t];
                        const double dp0_dz = (p0[k + 1] - p0[k]) * P.inv_dz;
                        du = (float)finite_or_zero(-((double)pnx[t] - pc) * P.inv_dx / safe_rho(rho_x));
                        dv = (float)finite_or_zero(-((double)pn[t + nz] - pc) * P.inv_dy / safe_rho(rho_y));
                        dw = (float)finite_or_zero(-((((double)pn[t + 1] - pc) * P.inv_dz) - dp0_dz) / safe_rho(rho_z));
                    }
                    else
                    {
                        const float rc = rn[t];
                        const float rho_x = 0.5f * (rc + rnx[t]);
                        const float rho_y = 0.5f * (rc + rn[t + nz]);
                        const float rho_z = 0.5f * (rc + rn[t + 1]);
                        const float pc = pn[t];
                        // (p[k+1]-p[k]) - (p0[k+1]-p0[k]) with the base difference as FP32 hi+lo.
                        const float2 dp0 = dp0_split[k];
                        const float dpz = ((pn[t + 1] - pc) - dp0.x) - dp0.y;
                        const float sxr = (isfinite(rho_x) && rho_x > 1.0e-6f) ? rho_x : 1.0f;
                        const float syr = (isfinite(rho_y) && rho_y > 1.0e-6f) ? rho_y : 1.0f;
                        const float szr = (isfinite(rho_z) && rho_z > 1.0e-6f) ? rho_z : 1.0f;
                        const float a = __fdividef(-(pnx[t] - pc) * P.inv_dx_f, sxr);
                        const float b = __fdividef(-(pn[t + nz] - pc) * P.inv_dy_f, syr);
                        const float c = __fdividef(-dpz * P.inv_dz_f, szr);
                        du = isfinite(a) ? a : 0.0f;
                        dv = isfinite(b) ? b : 0.0f;
                        dw = isfinite(c) ? c : 0.0f;
                    }
                }
                const size_t g = plane_base + t;
                if constexpr (sizeof(real) == 8)
                {
                    u_out[g] = clamp_value((float)((double)uc[t] + (double)du * P.dt_small), 0.0f, -P.wind_h, P.wind_h);
                    v_out[g] = clamp_value((float)((double)vc[t + nz] + (double)dv * P.dt_small), 0.0f, -P.wind_h, P.wind_h);
                    w_out[g] = clamp_value((float)((double)wc[t] + (double)dw * P.dt_small), 0.0f, -P.wind_v, P.wind_v);
                }
                else
                {
                    const float dt = P.dt_f;
                    u_out[g] = clamp_value(__fmaf_rn(du, dt, uc[t]), 0.0f, -P.wind_h, P.wind_h);
                    v_out[g] = clamp_value(__fmaf_rn(dv, dt, vc[t + nz]), 0.0f, -P.wind_h, P.wind_h);
                    w_out[g] = clamp_value(__fmaf_rn(dw, dt, wc[t]), 0.0f, -P.wind_v, P.wind_v);
                }
            }
        }
        __syncthreads();
    }
    cp_async_wait_0();
    if (flags) atomicOr(status, flags);
}

}  // namespace nimbus
