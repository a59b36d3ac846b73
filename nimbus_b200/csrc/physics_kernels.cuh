// Kessler warm-rain microphysics and the EOS pressure re-projection, sm_100a.
//
// Kessler (KesslerScheme::compute_tendencies, kessler.cpp:103-520) is one
// thread per cell, k fastest.  The sedimentation's column coupling -- cell k
// loses its own fall flux and gains its upper neighbour's, in that order
// (kessler.cpp:479-518) -- is a per-cell formula, so each thread recomputes
// the flux of cell k+1 from the original qr and densities instead of walking
// the column: (pre_k - own_k) + recv_{k+1}, the reference's exact FP32 order.
// The step form applies the tendencies in the same launch (theta, qv, qc in
// place; qr to a separate buffer, because the thread below still reads the
// original qr of this cell).
#pragma once

#include "stencil_common.cuh"

namespace nimbus
{

struct KesslerParams
{
    Dims d;
    double dz;
    double dt;
    int i0, i1, j0, j1, k0, k1;  // cell domain
    double qc0, c_auto, c_accr, evap_eff, vt_max;
    // FP32 form: the scalars above rounded once.
    float dz_f, dt_f, qc0_f, c_auto_f, c_accr_f, evap_eff_f, vt_max_f;
};

__host__ __device__ inline void finish_fp32(KesslerParams& K)
{
    K.dz_f = (float)K.dz;
    K.dt_f = (float)K.dt;
    K.qc0_f = (float)K.qc0;
    K.c_auto_f = (float)K.c_auto;
    K.c_accr_f = (float)K.c_accr;
    K.evap_eff_f = (float)K.evap_eff;
    K.vt_max_f = (float)K.vt_max;
}

// Constants: microphysics_base.hpp:1073-1080, fall_speeds.hpp:60-68.
constexpr double kKT0 = 273.15, kKLv = 2.5e6, kKCp = 1004.0, kKRv = 461.5, kKRd = 287.0, kKP0 = 100000.0;
constexpr double kThetaStepMax = 50.0, kTheta0 = 300.0;  // max_theta_step_change_k, theta_reference_k
constexpr double kRainA = 36.34, kRainB = 0.1346, kRainMinQ = 1.0e-9, kFallRho = 1.2;

__device__ __forceinline__ double kclamp(double v, double lo, double hi) { return v < lo ? lo : (hi < v ? hi : v); }
__device__ __forceinline__ double kmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double kmin(double a, double b) { return b < a ? b : a; }

__device__ __forceinline__ double k_theta_to_temperature(double theta, double p)
{
    if (!isfinite(theta) || !isfinite(p)) return kKT0;
    const double th = kclamp(theta, 150.0, 700.0), ps = kclamp(p, 100.0, 200000.0);
    const double T = th * pow(ps / kKP0, kKRd / kKCp);
    return isfinite(T) ? T : kKT0;
}

__device__ __forceinline__ double k_qvs_water(double T, double p)
{
    double e = 0.0;
    if (isfinite(T))
    {
        const double tc = kclamp(T, 150.0, 400.0) - kKT0;
        const double value = 611.21 * exp((18.678 - tc / 234.5) * tc / (257.14 + tc));
        e = isfinite(value) ? kmax(0.0, value) : 0.0;
    }
    if (!isfinite(e) || !isfinite(p)) return 0.0;
    const double ps = kclamp(p, 100.0, 200000.0);
    return kclamp(0.62198 * e / kmax(ps - e, 1.0), 0.0, 0.2);
}

__device__ __forceinline__ double k_sat_slope(double temperature, double saturation, double p)
{
    if (!(temperature > 150.0 && temperature < 400.0) || !(saturation > 0.0 && saturation < 0.2)) return 0.0;
    const double pressure = kclamp(p, 100.0, 200000.0);
    const double vapor = saturation * pressure / (0.62198 + saturation);
    const double tc = temperature - kKT0;
    const double den = 257.14 + tc;
    const double num = (18.678 - tc / 234.5) * tc;
    const double num_slope = 18.678 - 2.0 * tc / 234.5;
    const double lps = (num_slope * den - num) / (den * den);
    return saturation * pressure / kmax(pressure - vapor, 1.0) * lps;
}

// Coupled saturation adjustment (thermodynamics.hpp:282-466).
static __device__ double k_saturation_adjustment(double T_in, double p, double& qv, double& qc)
{
    double T = isfinite(T_in) ? kclamp(T_in, 150.0, 400.0) : kKT0;
    qv = isfinite(qv) ? kmax(0.0, qv) : 0.0;
    qc = isfinite(qc) ? kmax(0.0, qc) : 0.0;
    double qvs = k_qvs_water(T, p);
    if (!isfinite(qvs) || qvs < 0.0) qvs = 0.0;
    const double L = kKLv / kKCp;
    const double eps8 = 8.0 * 2.220446049250313e-16;
    if (qv > qvs)
    {
        const double maximum = kmin(qv, kmax(0.0, (400.0 - T) / L));
        double condensed = maximum;
        if (qv - maximum - k_qvs_water(T + L * maximum, p) <= 0.0)
        {
            double lower = 0.0, upper = maximum;
            condensed = kclamp((qv - qvs) / (1.0 + L * k_sat_slope(T, qvs, p)), lower, upper);
            for (int it = 0; it < 10; ++it)
            {
                const double ta = T + L * condensed;
                const double sa = k_qvs_water(ta, p);
                const double value = qv - condensed - sa;
                if (fabs(value) <= eps8 * kmax(kmax(1.0, fabs(qv)), fabs(sa))) break;
                if (value > 0.0) lower = condensed;
                else upper = condensed;
                const double derivative = -1.0 - L * k_sat_slope(ta, sa, p);
                const double candidate = condensed - value / derivative;
                condensed = (candidate > lower && candidate < upper) ? candidate : 0.5 * (lower + upper);
            }
        }
        qv -= condensed;
        qc += condensed;
        T += L * condensed;
    }
    else if (qv < qvs && qc > 0.0)
    {
        const double maximum = kmin(qc, kmax(0.0, (T - 150.0) / L));
        double evaporated = maximum;
        if (qv + maximum - k_qvs_water(T - L * maximum, p) >= 0.0)
        {
            double lower = 0.0, upper = maximum;
            evaporated = kclamp((qvs - qv) / (1.0 + L * k_sat_slope(T, qvs, p)), lower, upper);
            for (int it = 0; it < 10; ++it)
            {
                const double ta = T - L * evaporated;
                const double sa = k_qvs_water(ta, p);
                const double value = qv + evaporated - sa;
                if (fabs(value) <= eps8 * kmax(kmax(1.0, fabs(qv)), fabs(sa))) break;
                if (value < 0.0) lower = evaporated;
                else upper = evaporated;
                const double derivative = 1.0 + L * k_sat_slope(ta, sa, p);
                const double candidate = evaporated - value / derivative;
                evaporated = (candidate > lower && candidate < upper) ? candidate : 0.5 * (lower + upper);
            }
        }
        qc -= evaporated;
        qv += evaporated;
        T -= L * evaporated;
    }
    qc = kmax(0.0, qc);
    qv = kmax(0.0, qv);
    return T;
}

// Rain fall flux Vt*qr of one cell, rounded to FP32 as the reference stores it.
__device__ __forceinline__ float k_sed_flux(const KesslerParams& K, double qr_raw, double rho_k)
{
    const double q = kmax(0.0, qr_raw);
    if (!(q > 0.0)) return 0.0f;
    const double fall = sqrt(kFallRho / rho_k);
    const double vt0 = (q < kRainMinQ) ? 0.0 : kRainA * pow(1.0e-3 * rho_k * q, kRainB);
    const double vt = kmin(vt0 * fall, K.vt_max);
    return (float)(vt * q);
}

// Kessler tendencies of cell c and, with kApply, their application (theta,
// qv, qc in place; the new qr to qr_out, since the cell below still reads
// this cell's old qr for its sedimentation inflow).
// With `fresh` the applied state of the cell (theta, qv, qc, qr) is also
// returned, for a pass that continues from it in registers.
template <bool kApply>
__device__ __forceinline__ void kessler_cell(const KesslerParams& K, float* __restrict__ theta,
                                             float* __restrict__ qv, float* __restrict__ qc,
                                             const float* __restrict__ qr, const float* __restrict__ p,
                                             const float* __restrict__ rho, float* __restrict__ qr_out,
                                             float* __restrict__ dth_out, float* __restrict__ dqv_out,
                                             float* __restrict__ dqc_out, float* __restrict__ dqr_out, int c,
                                             float4* fresh = nullptr)
{
    const Dims d = K.d;
    const double dt = K.dt;
    {
        int i, j, k;
        decompose(d, c, i, j, k);
        const bool inside = i >= K.i0 && i < K.i1 && j >= K.j0 && j < K.j1 && k >= K.k0 && k < K.k1;
        float dth = 0.0f, dqv = 0.0f, dqc = 0.0f, dqr = 0.0f;
        const float qr_c = qr[c];
        if (inside && dt > 0.0)
        {
            const float p_c = p[c];
            const float qv_c = qv[c], qc_c = qc[c];
            // Saturation adjustment.
            const float tv = (float)k_theta_to_temperature((double)theta[c], (double)p_c);
            double qvd = (double)qv_c, qcd = (double)qc_c;
            const float temp = (float)k_saturation_adjustment((double)tv, (double)p_c, qvd, qcd);
            const float qv_adj = (float)qvd, qc_adj = (float)qcd;
            const double dqa = (double)qc_adj - (double)qc_c;
            if (dqa != 0.0)
            {
                const double rate = dqa * (1.0 / dt);
                dqc = __fadd_rn(dqc, (float)rate);
                dqv = __fsub_rn(dqv, (float)rate);
                dth = __fadd_rn(dth, (float)(kKLv / kKCp * rate));
            }
            // Autoconversion + accretion, then rain evaporation.
            float prod = 0.0f;
            if (qc_adj > 0.0f)
            {
                const double factor =
                    1.0 / (1.0 + K.c_accr * dt * pow((double)(0.0f < qr_c ? qr_c : 0.0f), 0.875));
                const double amount =
                    (double)qc_adj * (1.0 - factor) + factor * K.c_auto * dt * kmax((double)qc_adj - K.qc0, 0.0);
                prod = (float)(kclamp(amount, 0.0, (double)qc_adj) / dt);
                dqc = __fsub_rn(dqc, prod);
                dqr = __fadd_rn(dqr, prod);
            }
            if (qr_c > 0.0f || prod > 0.0f)
            {
                const double pv = (double)p_c, rv = (double)rho[c];
                const double qvsat = k_qvs_water((double)temp, pv);
                if (qvsat > 0.0 && (double)qv_adj < qvsat && rv > 0.0 && pv > 0.0)
                {
                    const double qr_av = (double)qr_c + (double)prod * dt;
                    const double rcgs = 1.0e-3 * rv;
                    const double rain = rcgs * kmax(qr_av, 0.0);
                    const double vent = (1.6 + 124.9 * pow(rain, 0.2046)) * pow(rain, 0.525);
                    const double resist = 2.55e8 / (pv * qvsat) + 5.4e5;
                    const double raw = K.evap_eff * (vent / resist) * ((qvsat - (double)qv_adj) / (rcgs * qvsat));
                    const double gsat =
                        (kKLv * kKLv * qvsat) / (kKCp * kKRv * kmax((double)temp * (double)temp, 1.0));
                    const double bound = (qvsat - (double)qv_adj) / (1.0 + gsat);
                    const double evap = kclamp(raw, 0.0, kmin(bound / dt, qr_av / dt));
                    // Field3D's element proxy rounds the double operand to float first.
                    dqv = __fadd_rn(dqv, (float)evap);
                    dqr = __fsub_rn(dqr, (float)evap);
                    dth = __fsub_rn(dth, (float)(kKLv / kKCp * evap));
                }
            }
            // Sedimentation: lose the own fall flux, then gain the upper neighbour's.
            const double rho_k = (double)rho[c];
            if (kmax(0.0, (double)qr_c) > 0.0)
                dqr = __fsub_rn(dqr, (float)((double)k_sed_flux(K, (double)qr_c, rho_k) / K.dz));
            if (k + 1 < K.k1)
            {
                const double qr_up = (double)qr[c + 1];
                if (kmax(0.0, qr_up) > 0.0)
                {
                    const double rho_up = (double)rho[c + 1];
                    const float up = k_sed_flux(K, qr_up, rho_up);
                    const double recv = rho_up / rho_k;
                    dqr = __fadd_rn(dqr, (float)(recv * (double)up / K.dz));
                }
            }
            // Temperature tendency to theta tendency.
            {
                const double dT = (double)dth, pv = (double)p_c;
                double r = 0.0;
                if (isfinite(dT) && isfinite(pv))
                {
                    // The factor is finite and positive (ps is clamped), so a
                    // zero tendency keeps its own signed zero without it.
                    if (dT == 0.0) r = dT;
                    else
                    {
                        const double ps = kclamp(pv, 100.0, 200000.0);
                        r = dT * pow(kKP0 / ps, kKRd / kKCp);
                        if (!isfinite(r)) r = 0.0;
                    }
                }
                dth = (float)r;
            }
        }
        if (dth_out != nullptr)
        {
            dth_out[c] = dth;
            dqv_out[c] = dqv;
            dqc_out[c] = dqc;
            dqr_out[c] = dqr;
        }
        if (kApply)
        {
            float qr_new = qr_c;
            float th_new, qv_new, qc_new;
            if (!inside)
            {
                if (fresh)
                {
                    th_new = theta[c];
                    qv_new = qv[c];
                    qc_new = qc[c];
                }
            }
            else
            {
                // The CPU commit of step_microphysics_once with radiation,
                // boundary layer and stochastic multipliers off
                // (microphysics_step.cpp:3026-3245).
                auto water = [&](float q, float dq) {
                    const double dqs = isfinite(dq) ? (double)dq : 0.0;
                    const float raw = (float)((double)q + dqs * dt);
                    return !isfinite(raw) ? 0.0f : (raw < 0.0f ? 0.0f : (0.05f < raw ? 0.05f : raw));
                };
                qv_new = water(qv[c], dqv);
                qc_new = water(qc[c], dqc);
                qv[c] = qv_new;
                qc[c] = qc_new;
                qr_new = water(qr_c, dqr);
                const double told = (double)theta[c];
                double total = (isfinite(dth) ? (double)dth : 0.0) * dt;
                if (!isfinite(total)) total = 0.0;
                const double limited = kclamp(total, -kThetaStepMax, kThetaStepMax);
                double tn = told + limited;
                if (!isfinite(tn)) tn = isfinite(told) ? told : kTheta0;
                const float stored = (float)tn;
                th_new = clamp_value(stored, (float)kTheta0, 200.0f, 700.0f);
                theta[c] = th_new;
            }
            qr_out[c] = qr_new;
            if (fresh) *fresh = make_float4(th_new, qv_new, qc_new, qr_new);
        }
    }
}

// ---- FP32 form -------------------------------------------------------------
// The same scheme in FP32 arithmetic (the reference's GPU microphysics
// dispatch takes FP32 parameters, src/compute/dispatch/microphysics.cpp):
// the same clamps, branches and order, FP32 powf/expf/sqrtf, and a saturation
// adjustment whose Newton iteration stops at a few FP32 ulps of the vapour
// rather than at the FP64 epsilon.  Used by the FP32 precision form only.
constexpr float kfT0 = 273.15f, kfP0 = 100000.0f;
constexpr float kfKappa = (float)(kKRd / kKCp), kfLvCp = (float)(kKLv / kKCp);
constexpr float kfLv2CpRv = (float)(kKLv * kKLv / (kKCp * kKRv));

__device__ __forceinline__ float kfclamp(float v, float lo, float hi) { return v < lo ? lo : (hi < v ? hi : v); }

__device__ __forceinline__ float kf_theta_to_temperature(float theta, float p)
{
    if (!isfinite(theta) || !isfinite(p)) return kfT0;
    const float th = kfclamp(theta, 150.0f, 700.0f), ps = kfclamp(p, 100.0f, 200000.0f);
    const float T = th * powf(ps / kfP0, kfKappa);
    return isfinite(T) ? T : kfT0;
}

__device__ __forceinline__ float kf_qvs_water(float T, float p)
{
    float e = 0.0f;
    if (isfinite(T))
    {
        const float tc = kfclamp(T, 150.0f, 400.0f) - kfT0;
        const float value = 611.21f * expf((18.678f - tc / 234.5f) * tc / (257.14f + tc));
        e = isfinite(value) ? fmaxf(0.0f, value) : 0.0f;
    }
    if (!isfinite(e) || !isfinite(p)) return 0.0f;
    const float ps = kfclamp(p, 100.0f, 200000.0f);
    return kfclamp(0.62198f * e / fmaxf(ps - e, 1.0f), 0.0f, 0.2f);
}

__device__ __forceinline__ float kf_sat_slope(float temperature, float saturation, float p)
{
    if (!(temperature > 150.0f && temperature < 400.0f) || !(saturation > 0.0f && saturation < 0.2f)) return 0.0f;
    const float pressure = kfclamp(p, 100.0f, 200000.0f);
    const float vapor = saturation * pressure / (0.62198f + saturation);
    const float tc = temperature - kfT0;
    const float den = 257.14f + tc;
    const float num = (18.678f - tc / 234.5f) * tc;
    const float num_slope = 18.678f - 2.0f * tc / 234.5f;
    const float lps = (num_slope * den - num) / (den * den);
    return saturation * pressure / fmaxf(pressure - vapor, 1.0f) * lps;
}

// One Newton-bisection solve of the coupled adjustment (k_saturation_adjustment
// in FP32): sign = +1 condenses vapour, -1 evaporates cloud.
__device__ __forceinline__ float kf_adjust(float T, float p, float qv, float qvs, float maximum, float sign)
{
    const float L = kfLvCp;
    float amount = maximum;
    if (sign * (qv - sign * maximum - kf_qvs_water(T + sign * L * maximum, p)) <= 0.0f)
    {
        float lower = 0.0f, upper = maximum;
        amount = kfclamp(sign * (qv - qvs) / (1.0f + L * kf_sat_slope(T, qvs, p)), lower, upper);
        for (int it = 0; it < 10; ++it)
        {
            const float ta = T + sign * L * amount;
            const float sa = kf_qvs_water(ta, p);
            const float value = qv - sign * amount - sa;
            if (fabsf(value) <= 4.0f * 1.1920929e-7f * fmaxf(fmaxf(fabsf(qv), fabsf(sa)), 1.0e-12f)) break;
            if (sign * value > 0.0f) lower = amount;
            else upper = amount;
            const float derivative = -1.0f - L * kf_sat_slope(ta, sa, p);
            const float candidate = amount + sign * value / (-derivative);
            amount = (candidate > lower && candidate < upper) ? candidate : 0.5f * (lower + upper);
        }
    }
    return amount;
}

static __device__ float kf_saturation_adjustment(float T_in, float p, float& qv, float& qc)
{
    float T = isfinite(T_in) ? kfclamp(T_in, 150.0f, 400.0f) : kfT0;
    qv = isfinite(qv) ? fmaxf(0.0f, qv) : 0.0f;
    qc = isfinite(qc) ? fmaxf(0.0f, qc) : 0.0f;
    float qvs = kf_qvs_water(T, p);
    if (!isfinite(qvs) || qvs < 0.0f) qvs = 0.0f;
    const float L = kfLvCp;
    if (qv > qvs)
    {
        const float condensed = kf_adjust(T, p, qv, qvs, fminf(qv, fmaxf(0.0f, (400.0f - T) / L)), 1.0f);
        qv -= condensed;
        qc += condensed;
        T += L * condensed;
    }
    else if (qv < qvs && qc > 0.0f)
    {
        const float evaporated = kf_adjust(T, p, qv, qvs, fminf(qc, fmaxf(0.0f, (T - 150.0f) / L)), -1.0f);
        qc -= evaporated;
        qv += evaporated;
        T -= L * evaporated;
    }
    qc = fmaxf(0.0f, qc);
    qv = fmaxf(0.0f, qv);
    return T;
}

__device__ __forceinline__ float kf_sed_flux(const KesslerParams& K, float qr_raw, float rho_k)
{
    const float q = fmaxf(0.0f, qr_raw);
    if (!(q > 0.0f)) return 0.0f;
    const float fall = sqrtf((float)kFallRho / rho_k);
    const float vt0 = (q < (float)kRainMinQ) ? 0.0f : (float)kRainA * powf(1.0e-3f * rho_k * q, (float)kRainB);
    return fminf(vt0 * fall, K.vt_max_f) * q;
}

template <bool kApply>
__device__ __forceinline__ void kessler_cell_f32(const KesslerParams& K, float* __restrict__ theta,
                                                 float* __restrict__ qv, float* __restrict__ qc,
                                                 const float* __restrict__ qr, const float* __restrict__ p,
                                                 const float* __restrict__ rho, float* __restrict__ qr_out,
                                                 float* __restrict__ dth_out, float* __restrict__ dqv_out,
                                                 float* __restrict__ dqc_out, float* __restrict__ dqr_out, int c,
                                                 float4* fresh = nullptr)
{
    const Dims d = K.d;
    const float dt = K.dt_f;
    int i, j, k;
    decompose(d, c, i, j, k);
    const bool inside = i >= K.i0 && i < K.i1 && j >= K.j0 && j < K.j1 && k >= K.k0 && k < K.k1;
    float dth = 0.0f, dqv = 0.0f, dqc = 0.0f, dqr = 0.0f;
    const float qr_c = qr[c];
    const float th_c = theta[c], qv_c = qv[c], qc_c = qc[c];
    if (inside && dt > 0.0f)
    {
        const float p_c = p[c], rho_k = rho[c];
        const bool up_exists = k + 1 < K.k1;
        const float qr_up = up_exists ? qr[c + 1] : 0.0f, rho_up = up_exists ? rho[c + 1] : 1.0f;
        // Saturation adjustment.
        float qv_adj = qv_c, qc_adj = qc_c;
        const float temp = kf_saturation_adjustment(kf_theta_to_temperature(th_c, p_c), p_c, qv_adj, qc_adj);
        const float dqa = qc_adj - qc_c;
        if (dqa != 0.0f)
        {
            const float rate = dqa / dt;
            dqc += rate;
            dqv -= rate;
            dth += kfLvCp * rate;
        }
        // Autoconversion + accretion, then rain evaporation.
        float prod = 0.0f;
        if (qc_adj > 0.0f)
        {
            const float factor = 1.0f / (1.0f + K.c_accr_f * dt * powf(fmaxf(qr_c, 0.0f), 0.875f));
            const float amount = qc_adj * (1.0f - factor) + factor * K.c_auto_f * dt * fmaxf(qc_adj - K.qc0_f, 0.0f);
            prod = kfclamp(amount, 0.0f, qc_adj) / dt;
            dqc -= prod;
            dqr += prod;
        }
        if (qr_c > 0.0f || prod > 0.0f)
        {
            const float qvsat = kf_qvs_water(temp, p_c);
            if (qvsat > 0.0f && qv_adj < qvsat && rho_k > 0.0f && p_c > 0.0f)
            {
                const float qr_av = qr_c + prod * dt;
                const float rcgs = 1.0e-3f * rho_k;
                const float rain = rcgs * fmaxf(qr_av, 0.0f);
                const float vent = (1.6f + 124.9f * powf(rain, 0.2046f)) * powf(rain, 0.525f);
                const float resist = 2.55e8f / (p_c * qvsat) + 5.4e5f;
                const float raw = K.evap_eff_f * (vent / resist) * ((qvsat - qv_adj) / (rcgs * qvsat));
                const float gsat = kfLv2CpRv * qvsat / fmaxf(temp * temp, 1.0f);
                const float bound = (qvsat - qv_adj) / (1.0f + gsat);
                const float evap = kfclamp(raw, 0.0f, fminf(bound / dt, qr_av / dt));
                dqv += evap;
                dqr -= evap;
                dth -= kfLvCp * evap;
            }
        }
        // Sedimentation: lose the own fall flux, then gain the upper neighbour's.
        if (qr_c > 0.0f) dqr -= kf_sed_flux(K, qr_c, rho_k) / K.dz_f;
        if (up_exists && qr_up > 0.0f) dqr += (rho_up / rho_k) * kf_sed_flux(K, qr_up, rho_up) / K.dz_f;
        // Temperature tendency to theta tendency (a zero tendency needs no factor).
        if (isfinite(dth) && isfinite(p_c))
        {
            if (dth != 0.0f)
            {
                const float r = dth * powf(kfP0 / kfclamp(p_c, 100.0f, 200000.0f), kfKappa);
                dth = isfinite(r) ? r : 0.0f;
            }
        }
        else dth = 0.0f;
    }
    if (dth_out != nullptr)
    {
        dth_out[c] = dth;
        dqv_out[c] = dqv;
        dqc_out[c] = dqc;
        dqr_out[c] = dqr;
    }
    if (kApply)
    {
        float th_new = th_c, qv_new = qv_c, qc_new = qc_c, qr_new = qr_c;
        if (inside)
        {
            // step_microphysics_once's commit (microphysics_step.cpp:3026-3245).
            auto water = [&](float q, float dq) {
                const float raw = __fmaf_rn(isfinite(dq) ? dq : 0.0f, dt, q);
                return !isfinite(raw) ? 0.0f : (raw < 0.0f ? 0.0f : (0.05f < raw ? 0.05f : raw));
            };
            qv_new = water(qv_c, dqv);
            qc_new = water(qc_c, dqc);
            qr_new = water(qr_c, dqr);
            float total = (isfinite(dth) ? dth : 0.0f) * dt;
            if (!isfinite(total)) total = 0.0f;
            float tn = th_c + kfclamp(total, -(float)kThetaStepMax, (float)kThetaStepMax);
            if (!isfinite(tn)) tn = isfinite(th_c) ? th_c : (float)kTheta0;
            th_new = clamp_value(tn, (float)kTheta0, 200.0f, 700.0f);
            theta[c] = th_new;
            qv[c] = qv_new;
            qc[c] = qc_new;
        }
        qr_out[c] = qr_new;
        if (fresh) *fresh = make_float4(th_new, qv_new, qc_new, qr_new);
    }
}

template <bool kApply>
static __global__ void __launch_bounds__(256) kessler_f32_kernel(KesslerParams K, float* __restrict__ theta,
                                                                 float* __restrict__ qv, float* __restrict__ qc,
                                                                 const float* __restrict__ qr,
                                                                 const float* __restrict__ p,
                                                                 const float* __restrict__ rho,
                                                                 float* __restrict__ qr_out,
                                                                 float* __restrict__ dth_out,
                                                                 float* __restrict__ dqv_out,
                                                                 float* __restrict__ dqc_out,
                                                                 float* __restrict__ dqr_out)
{
    const int n = K.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        kessler_cell_f32<kApply>(K, theta, qv, qc, qr, p, rho, qr_out, dth_out, dqv_out, dqc_out, dqr_out, c);
}

template <bool kApply>
static __global__ void __launch_bounds__(256) kessler_kernel(KesslerParams K, float* __restrict__ theta, float* __restrict__ qv,
                                                      float* __restrict__ qc, const float* __restrict__ qr,
                                                      const float* __restrict__ p, const float* __restrict__ rho,
                                                      float* __restrict__ qr_out, float* __restrict__ dth_out,
                                                      float* __restrict__ dqv_out, float* __restrict__ dqc_out,
                                                      float* __restrict__ dqr_out)
{
    const int n = K.d.cells();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        kessler_cell<kApply>(K, theta, qv, qc, qr, p, rho, qr_out, dth_out, dqv_out, dqc_out, dqr_out, c);
}

// EOS pressure re-projection (eos_apply.cpp:50-175, pressure_fp64 in
// eos_pressure.hpp:30-38): candidate p = clamp(float(p00 (rho R_d theta /
// p00)^gamma)) for every cell.  With qv/qc/qr given, the cells of the
// attributed domain (physical_scalar_domain: the one-cell lateral ring dropped
// where the extent is >= 3, every level) are also checked as the energy
// attribution checks them (eos_apply.cpp:139-158): old p finite and positive,
// qv finite and non-negative, qc + qr (FP64) finite and non-negative.  Any
// failure sets the status bit; eos_publish_kernel then leaves p untouched.
// The candidate pressure of cell c from its values; sets the refusal bit and
// returns false for an invalid cell.  moist adds the attributed-domain checks.
__device__ __forceinline__ bool eos_candidate_value(const Dims& d, int c, float r, float th, double gamma, bool moist,
                                                    float po, float q, float qc, float qr, float& p_new,
                                                    unsigned& flags)
{
    const double diagnosed = kP00 * pow((double)r * kRd * (double)th / kP00, gamma);
    if (!isfinite(r) || !(r > 0.0f) || !isfinite(th) || !(th > 0.0f) || !isfinite(diagnosed) || diagnosed <= 0.0 ||
        !isfinite((float)diagnosed))
    {
        flags |= kStatusInvalidEos;
        return false;
    }
    p_new = clamp_value((float)diagnosed, 101325.0f, 1000.0f, 200000.0f);
    if (moist)
    {
        const int ih = d.nx >= 3, jh = d.ny >= 3;
        int i, j, k;
        decompose(d, c, i, j, k);
        if (i >= ih && i < d.nx - ih && j >= jh && j < d.ny - jh)
        {
            const double liquid = (double)qc + (double)qr;
            if (!isfinite(po) || po <= 0.0f || !isfinite(q) || q < 0.0f || !isfinite(liquid) || liquid < 0.0)
                flags |= kStatusInvalidEos;
        }
    }
    return true;
}

// The binomial-series coefficients binom(gamma, n), n = 1..6, rounded once.
struct EosSeries
{
    float c[6];
};

__host__ inline EosSeries eos_series(double gamma)
{
    EosSeries e;
    double c = 1.0;
    for (int n = 1; n <= 6; ++n)
    {
        c *= (gamma - (n - 1)) / n;
        e.c[n - 1] = (float)c;
    }
    return e;
}

// FP32 form of eos_candidate_value: p = p0 (1 + d)^gamma around the level's
// base state (eos0[k] = {p0 hi, p0 lo, b hi, b lo}, b = R_d / (p00 x0),
// x0 = (p0 / p00)^(1/gamma)), with 1 + d = rho theta b formed exactly as a
// hi+lo pair and the series summed to the sixth power for |d| <= 1/16 (within
// about half an FP32 ulp of the FP64 value; larger |d| take FP64).  The same
// refusal rules and clamp as the FP64 form.
__device__ __forceinline__ bool eos_candidate_value_f32(const Dims& d, int c, int k, float r, float th,
                                                        const float4* __restrict__ eos0, const EosSeries& series,
                                                        double gamma, bool moist, float po, float q, float qc,
                                                        float qr, float& p_new, unsigned& flags)
{
    bool ok = isfinite(r) && r > 0.0f && isfinite(th) && th > 0.0f;
    float pressure = 0.0f;
    if (ok)
    {
        const float4 e = eos0[k];
        const float rt = r * th;
        const float rt_lo = __fmaf_rn(r, th, -rt);
        const float x = rt * e.z;
        const float x_lo = __fmaf_rn(rt, e.z, -x) + __fmaf_rn(rt, e.w, rt_lo * e.z);
        const float dl = (x - 1.0f) + x_lo;
        if (fabsf(dl) <= 0.0625f)
        {
            float sum = series.c[5];
            for (int n = 4; n >= 0; --n) sum = __fmaf_rn(sum, dl, series.c[n]);
            pressure = e.x + __fmaf_rn(e.x, sum * dl, e.y);
        }
        else
        {
            const double diagnosed = kP00 * pow((double)r * kRd * (double)th / kP00, gamma);
            ok = isfinite(diagnosed) && diagnosed > 0.0 && isfinite((float)diagnosed);
            pressure = (float)diagnosed;
        }
    }
    if (!ok)
    {
        flags |= kStatusInvalidEos;
        return false;
    }
    p_new = clamp_value(pressure, 101325.0f, 1000.0f, 200000.0f);
    if (moist)
    {
        const int ih = d.nx >= 3, jh = d.ny >= 3;
        int i, j, kk;
        decompose(d, c, i, j, kk);
        if (i >= ih && i < d.nx - ih && j >= jh && j < d.ny - jh)
        {
            const double liquid = (double)qc + (double)qr;
            if (!isfinite(po) || po <= 0.0f || !isfinite(q) || q < 0.0f || !isfinite(liquid) || liquid < 0.0)
                flags |= kStatusInvalidEos;
        }
    }
    return true;
}

static __global__ void __launch_bounds__(256) eos_candidate_f32_kernel(
    Dims d, const float* __restrict__ rho, const float* __restrict__ theta, const float* __restrict__ p_old,
    const float* __restrict__ qv, const float* __restrict__ qc, const float* __restrict__ qr,
    const float4* __restrict__ eos0, EosSeries series, double gamma, float* __restrict__ p_candidate,
    unsigned* __restrict__ status)
{
    const int n = (int)d.cells();
    const bool moist = qv != nullptr;
    unsigned flags = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
    {
        const int k = c % d.nz;
        float p_new;
        if (eos_candidate_value_f32(d, c, k, rho[c], theta[c], eos0, series, gamma, moist, moist ? p_old[c] : 0.0f,
                                    moist ? qv[c] : 0.0f, moist ? qc[c] : 0.0f, moist ? qr[c] : 0.0f, p_new, flags))
            p_candidate[c] = p_new;
    }
    if (flags) atomicOr(status, flags);
}

__device__ __forceinline__ void eos_candidate_cell(const Dims& d, const float* __restrict__ rho,
                                                   const float* __restrict__ theta, const float* __restrict__ p_old,
                                                   const float* __restrict__ qv, const float* __restrict__ qc,
                                                   const float* __restrict__ qr, double gamma,
                                                   float* __restrict__ p_candidate, int c, unsigned& flags)
{
    const bool moist = qv != nullptr;
    float p_new;
    if (eos_candidate_value(d, c, rho[c], theta[c], gamma, moist, moist ? p_old[c] : 0.0f, moist ? qv[c] : 0.0f,
                            moist ? qc[c] : 0.0f, moist ? qr[c] : 0.0f, p_new, flags))
        p_candidate[c] = p_new;
}

static __global__ void __launch_bounds__(256) eos_candidate_kernel(Dims d, const float* __restrict__ rho,
                                                            const float* __restrict__ theta,
                                                            const float* __restrict__ p_old,
                                                            const float* __restrict__ qv, const float* __restrict__ qc,
                                                            const float* __restrict__ qr, double gamma,
                                                            float* __restrict__ p_candidate,
                                                            unsigned* __restrict__ status)
{
    const int n = (int)d.cells();
    unsigned flags = 0;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x)
        eos_candidate_cell(d, rho, theta, p_old, qv, qc, qr, gamma, p_candidate, c, flags);
    if (flags) atomicOr(status, flags);
}

// Publishes the candidate pressure unless the projection was refused.
static __global__ void __launch_bounds__(256) eos_publish_kernel(long long n, const float* __restrict__ p_candidate,
                                                          float* __restrict__ p, const unsigned* __restrict__ status)
{
    if (*status & kStatusInvalidEos) return;
    const long long n4 = n / 4;
    const float4* src = reinterpret_cast<const float4*>(p_candidate);
    float4* dst = reinterpret_cast<float4*>(p);
    const long long stride = (long long)gridDim.x * blockDim.x;
    const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if ((reinterpret_cast<uintptr_t>(p) & 15) == 0)
    {
        for (long long c = t; c < n4; c += stride) dst[c] = src[c];
        for (long long c = 4 * n4 + t; c < n; c += stride) p[c] = p_candidate[c];
    }
    else
    {
        for (long long c = t; c < n; c += stride) p[c] = p_candidate[c];
    }
}

// ---- The Kessler dispatches of the device route ---------------------------
//
// KesslerScheme::compute_tendencies (kessler.cpp:152-300) has a second route
// when the active backend supports the Kessler operators: it runs the
// saturation adjustment on the host, hands the adjusted temperature, qv and
// qc to dispatch_kessler_pointwise (warm-rain production and rain
// evaporation, FP32, outputs written over the whole grid, zero outside the
// cell domain), books the adjustment's tendencies itself and then calls
// dispatch_kessler_sedimentation, which adds the rain fallout to dqr_dt in
// place.  The operators' arithmetic is the reference's device form of them
// (vulkan/shaders/compute/microphysics/kessler_pointwise.comp:70-172,
// kessler_sedimentation.comp:44-117): FP32 throughout.

struct KesslerPointwiseParams
{
    int nx, ny, nz;
    int i0, i1, j0, j1, k0, k1;
    float qc0, c_auto, c_accr, evaporation_efficiency, lv_cp, t0, dt;
};

// Buck's saturation vapour pressure over water (all temperatures) and the
// saturation mixing ratio bounded to [0, 0.2] (kessler_pointwise.comp:55-69).
__device__ __forceinline__ float kessler_qvsat_f32(float T, float p, float t0)
{
    const float tc = T - t0;
    const float es = 611.21f * expf((18.678f - tc / 234.5f) * tc / (257.14f + tc));
    const float denom = fmaxf(p - es, 1.0f);
    return fminf(fmaxf(0.62198f * es / denom, 0.0f), 0.2f);
}

static __global__ void __launch_bounds__(256) kessler_pointwise_kernel(
    KesslerPointwiseParams P, const float* __restrict__ temperature, const float* __restrict__ pres,
    const float* __restrict__ qv, const float* __restrict__ qc, const float* __restrict__ qr,
    const float* __restrict__ rho_d, float* __restrict__ dth, float* __restrict__ dqv, float* __restrict__ dqc,
    float* __restrict__ dqr, float* __restrict__ dqg, float* __restrict__ dqh)
{
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    {
        const int k = (int)(c % P.nz);
        const long long col = c / P.nz;
        const int j = (int)(col % P.ny), i = (int)(col / P.ny);
        float d_th = 0.0f, d_qv = 0.0f, d_qc = 0.0f, d_qr = 0.0f;
        if (i >= P.i0 && i < P.i1 && j >= P.j0 && j < P.j1 && k >= P.k0 && k < P.k1)
        {
            const float T = temperature[c], pv = pres[c], qvv = qv[c], qcv = qc[c], qrv = qr[c], rho = rho_d[c];
            const float dt = P.dt;
            // Finite-step production: implicit accretion plus autoconversion.
            float production = 0.0f;
            if (dt > 0.0f && qcv > 0.0f)
            {
                const float factor = 1.0f / (1.0f + P.c_accr * dt * powf(fmaxf(qrv, 0.0f), 0.875f));
                float amount = qcv * (1.0f - factor) + factor * P.c_auto * dt * fmaxf(qcv - P.qc0, 0.0f);
                amount = fminf(fmaxf(amount, 0.0f), qcv);
                production = amount / dt;
                d_qc -= production;
                d_qr += production;
            }
            // Rain evaporation in sub-saturated air, bounded by the
            // saturation deficit and the rain available over the step.
            if (qrv > 0.0f || production > 0.0f)
            {
                const float qvsat = kessler_qvsat_f32(T, pv, P.t0);
                if (qvsat > 0.0f && qvv < qvsat && rho > 0.0f && pv > 0.0f)
                {
                    const float available = qrv + production * dt;
                    const float rcgs = 1.0e-3f * rho;
                    const float content = rcgs * fmaxf(available, 0.0f);
                    const float ventilation = (1.6f + 124.9f * powf(content, 0.2046f)) * powf(content, 0.525f);
                    const float resistance = 2.55e8f / (pv * qvsat) + 5.4e5f;
                    const float raw = P.evaporation_efficiency * (ventilation / resistance) *
                                      ((qvsat - qvv) / (rcgs * qvsat));
                    const float gamma_sat = P.lv_cp * (2.5e6f / 461.5f) * qvsat / fmaxf(T * T, 1.0f);
                    const float bound = (qvsat - qvv) / (1.0f + gamma_sat);
                    const float evap = fminf(fmaxf(raw, 0.0f), fminf(bound / dt, available / dt));
                    d_qv += evap;
                    d_qr -= evap;
                    d_th -= P.lv_cp * evap;
                }
            }
        }
        dth[c] = d_th;
        dqv[c] = d_qv;
        dqc[c] = d_qc;
        dqr[c] = d_qr;
        if (dqg) dqg[c] = 0.0f;
        if (dqh) dqh[c] = 0.0f;
    }
}

struct KesslerSedimentationParams
{
    int nx, ny, nz;
    int i0, i1, j0, j1, k0, k1;
    float dz, vt_max, vt_cap;
};

// The rain fallout out of level k (kessler_sedimentation.comp:83-115): zero
// below the species threshold; *donor_dz and *recv_scale receive the donor
// layer's thickness and the density weight over the receiver's thickness.
__device__ __forceinline__ float kessler_fallout_f32(const KesslerSedimentationParams& P, const float* qr,
                                                     const float* rho_d, const float* layers, long long idx, int k,
                                                     float& donor_dz, float& recv_scale_num, float& receiver_dz)
{
    donor_dz = P.dz;
    receiver_dz = P.dz;
    if (layers)
    {
        donor_dz = layers[idx];
        receiver_dz = k > P.k0 ? layers[idx - 1] : donor_dz;
    }
    float fall = 1.0f, weight = 1.0f, rho_air = 1.2f;
    if (rho_d)
    {
        const float rk = rho_d[idx];
        const float rkm = k > P.k0 ? rho_d[idx - 1] : rk;
        fall = sqrtf(1.2f / rk);
        weight = rk / rkm;
        rho_air = rk;
    }
    recv_scale_num = weight;
    const float q = fmaxf(qr[idx], 0.0f);
    if (!(q > 1.0e-9f)) return 0.0f;
    float vt = 36.34f * powf(1.0e-3f * rho_air * q, 0.1346f);
    vt = fminf(vt * fall, P.vt_max);
    vt = fminf(vt, P.vt_cap);
    return vt * q;
}

// One thread per cell of the domain: the column's sequential update of
// dqr_dt[k] is (dqr - fallout_k / donor_dz_k) + w_{k+1} fallout_{k+1} /
// receiver_dz_{k+1}, evaluated here per level in that order.
static __global__ void __launch_bounds__(256) kessler_sedimentation_kernel(
    KesslerSedimentationParams P, const float* __restrict__ qr, const float* __restrict__ rho_d,
    const float* __restrict__ layers, float* __restrict__ dqr)
{
    const long long n = (long long)P.nx * P.ny * P.nz;
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < n; c += (long long)gridDim.x * blockDim.x)
    {
        const int k = (int)(c % P.nz);
        const long long col = c / P.nz;
        const int j = (int)(col % P.ny), i = (int)(col / P.ny);
        if (i < P.i0 || i >= P.i1 || j < P.j0 || j >= P.j1 || k < P.k0 || k >= P.k1) continue;
        float donor, weight, receiver;
        const float out = kessler_fallout_f32(P, qr, rho_d, layers, c, k, donor, weight, receiver);
        float t = dqr[c];
        if (fmaxf(qr[c], 0.0f) > 1.0e-9f) t -= out / donor;
        if (k + 1 < P.k1)
        {
            float d2, w2, r2;
            const float in = kessler_fallout_f32(P, qr, rho_d, layers, c + 1, k + 1, d2, w2, r2);
            if (fmaxf(qr[c + 1], 0.0f) > 1.0e-9f) t += w2 * in / r2;
        }
        dqr[c] = t;
    }
}

}  // namespace nimbus
