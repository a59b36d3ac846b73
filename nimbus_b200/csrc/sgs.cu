// C-ABI of the Smagorinsky SGS path (include/nimbus_cuda.h): the fused
// closure, the forward-Euler application, the explicit stability limit and
// the substepped SGS integration of one large step.
#include "../../include/nimbus_cuda.h"
#include "context.cuh"
#include "sgs_kernels.cuh"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <string>
#include <vector>

using namespace nimbus;
using namespace nimbus_host;

namespace
{

// validate_scheme_inputs' configuration contract (eddy_viscosity.cpp:1088-1175)
// plus the flat filter widths it implies.
const char* check_closure(const nimbus_smagorinsky_args* a, std::vector<double>& delta)
{
    if (!a->u || !a->v || !a->w || !a->theta || !a->rho || !a->dz) return "a required field pointer is null";
    if (a->nx < 3 || a->ny < 3 || a->nz < 2) return "SGS diffusion requires a C-grid of at least 3x3x2";
    if (!cells_fit(a->nx, a->ny, a->nz)) return "grid too large for one dispatch";
    if (!a->use_horizontal && !a->use_vertical) return "unsupported turbulence mode";
    if (a->filter_mode != 0 && a->filter_mode != 1) return "unsupported turbulence filter width";
    if (!finite_positive(a->dx) || !finite_positive(a->dy)) return "grid spacing must be finite and positive";
    if (!std::isfinite(a->Cs) || a->Cs < 0.0 || !finite_positive(a->Pr_t) || !finite_positive(a->Sc_t) ||
        !std::isfinite(a->nu_t_max) || a->nu_t_max < 0.0 || !std::isfinite(a->K_max) || a->K_max < 0.0)
        return "turbulence configuration violates the implemented coefficient contract";
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE) return "unknown memory kind";
    delta.resize(static_cast<size_t>(a->nz));
    for (int k = 0; k < a->nz; ++k)
    {
        if (!finite_positive(a->dz[k])) return "vertical metric spacing must be positive and finite";
        delta[k] = a->filter_mode == 1 ? std::sqrt(a->dx * a->dy) : std::cbrt(a->dx * a->dy * a->dz[k]);
        if (!finite_positive(delta[k])) return "filter width must be finite and positive";
    }
    return nullptr;
}

// Device copies of dz and the filter widths, back to back.
nimbus_status stage_tables(nimbus_cuda_context* ctx, cudaStream_t st, const double* dz,
                           const std::vector<double>& delta, SgsParams& P)
{
    const size_t nz = delta.size();
    double* dev = nullptr;
    NB_TRY(ensure(ctx, kSgsTables, 3 * nz, &dev));  // dz, delta, then the FP32 reciprocals of dz and dzc
    std::vector<float> inv(2 * nz, 0.0f);
    for (size_t k = 0; k < nz; ++k) inv[k] = static_cast<float>(1.0 / dz[k]);
    for (size_t k = 0; k + 1 < nz; ++k) inv[nz + k] = static_cast<float>(1.0 / (0.5 * (dz[k] + dz[k + 1])));
    // No centre above the top level: a use of DZC(nz - 1) shows up as NaN.
    inv[2 * nz - 1] = std::numeric_limits<float>::quiet_NaN();
    NB_CUDA(ctx, cudaMemcpyAsync(dev, dz, nz * sizeof(double), cudaMemcpyHostToDevice, st));
    NB_CUDA(ctx, cudaMemcpyAsync(dev + nz, delta.data(), nz * sizeof(double), cudaMemcpyHostToDevice, st));
    float* inv_dev = reinterpret_cast<float*>(dev + 2 * nz);
    NB_CUDA(ctx, cudaMemcpyAsync(inv_dev, inv.data(), 2 * nz * sizeof(float), cudaMemcpyHostToDevice, st));
    P.dz = dev;
    P.delta = dev + nz;
    P.inv_dz_f = inv_dev;
    P.inv_dzc_f = inv_dev + nz;
    return NIMBUS_OK;
}

SgsParams params_of(const nimbus_smagorinsky_args* a)
{
    SgsParams P{};
    P.d = make_dims(a->nx, a->ny, a->nz);
    P.dx = a->dx;
    P.dy = a->dy;
    P.use_h = a->use_horizontal ? 1 : 0;
    P.use_v = a->use_vertical ? 1 : 0;
    P.px = a->periodic_x ? 1 : 0;
    P.py = a->periodic_y ? 1 : 0;
    for (int f = 0; f < 4; ++f) P.open[f] = a->open_lateral[f] ? 1 : 0;
    P.Cs = a->Cs;
    P.Pr_t = a->Pr_t;
    P.Sc_t = a->Sc_t;
    P.nu_max = a->nu_t_max;
    P.K_max = a->K_max;
    P.inv_dx_f = static_cast<float>(1.0 / a->dx);
    P.inv_dy_f = static_cast<float>(1.0 / a->dy);
    return P;
}

// Device pointers of one closure evaluation.
struct ClosureDevice
{
    const float *u, *v, *w, *theta, *qv, *rho;
    float *nu, *kt, *kq;
    float *du, *dv, *dw, *dth, *dqv;
};

nimbus_status launch_closure(nimbus_cuda_context* ctx, cudaStream_t st, const SgsParams& P, const ClosureDevice& D,
                             unsigned* status)
{
    const int grid = grid_for(ctx, P.d.cells());
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_SGS);
    if (ctx->precision == NIMBUS_PRECISION_FP32)
    {
        sgs_coefficients_kernel<float><<<grid, kThreads, 0, st>>>(P, D.u, D.v, D.w, D.theta, D.qv, D.rho, D.nu,
                                                                  D.kt, D.kq, status);
        sgs_tendencies_kernel<float><<<grid, kThreads, 0, st>>>(P, D.u, D.v, D.w, D.theta, D.qv, D.rho, D.nu, D.kt,
                                                                D.kq, D.du, D.dv, D.dw, D.dth, D.dqv);
    }
    else
    {
        sgs_coefficients_kernel<double><<<grid, kThreads, 0, st>>>(P, D.u, D.v, D.w, D.theta, D.qv, D.rho, D.nu,
                                                                   D.kt, D.kq, status);
        sgs_tendencies_kernel<double><<<grid, kThreads, 0, st>>>(P, D.u, D.v, D.w, D.theta, D.qv, D.rho, D.nu, D.kt,
                                                                 D.kq, D.du, D.dv, D.dw, D.dth, D.dqv);
    }
    ctx->launches += 2;
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

// Scratch of one stability evaluation: slab partials, merged sums / extrema,
// the two limit minima and a status word.
struct StabilityScratch
{
    double* partial;
    double* merged;
    unsigned long long* lim;
    unsigned* status;
};

nimbus_status stability_scratch(nimbus_cuda_context* ctx, int nx, StabilityScratch& S)
{
    const size_t slabs = static_cast<size_t>(nx - 2);
    unsigned char* base = nullptr;
    const size_t bytes = (6 * slabs + 6) * sizeof(double) + 2 * sizeof(unsigned long long) + 16;
    NB_TRY(ensure(ctx, kSgsScratch, bytes, &base));
    S.partial = reinterpret_cast<double*>(base);
    S.merged = S.partial + 6 * slabs;
    S.lim = reinterpret_cast<unsigned long long*>(S.merged + 6);
    S.status = reinterpret_cast<unsigned*>(S.lim + 2);
    return NIMBUS_OK;
}

// The state / rates the stability and the closure read, on the device.
struct Rates
{
    const float *du, *dv, *dw, *dth, *dqv;
};

// Enqueues the stability reductions and waits for them; finishes on the
// host as compute_sgs_explicit_stability does.  `closure_status` (device, may
// be null) is read in the same copy: the closure's contract flag.
nimbus_status run_stability(nimbus_cuda_context* ctx, cudaStream_t st, const SgsParams& P, const ClosureDevice& D,
                            const Rates& R, const StabilityScratch& S, const unsigned* closure_status,
                            nimbus_sgs_stability* out)
{
    const int slabs = P.d.nx - 2;
    const unsigned long long inf_bits = 0x7ff0000000000000ull;
    const unsigned long long init[2] = {inf_bits, inf_bits};
    NB_CUDA(ctx, cudaMemcpyAsync(S.lim, init, sizeof(init), cudaMemcpyHostToDevice, st));
    NB_CUDA(ctx, cudaMemsetAsync(S.status, 0, sizeof(unsigned), st));
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_SGS);
        sgs_stability_slab_kernel<<<(slabs + kSlabWarps - 1) / kSlabWarps, 32 * kSlabWarps, 0, st>>>(
            P, D.u, D.v, D.w, D.theta, D.qv, D.rho, R.du, R.dv, R.dw, R.dth, R.dqv, S.partial, S.status);
        sgs_stability_merge_kernel<<<1, 32, 0, st>>>(slabs, S.partial, S.merged);
        const long long cells = static_cast<long long>(slabs) * (P.d.ny - 2) * P.d.nz;
        sgs_stability_limit_kernel<<<grid_for(ctx, cells), kThreads, 0, st>>>(P, D.theta, D.qv, R.dth, R.dqv,
                                                                            S.merged + 2, S.lim);
        ctx->launches += 3;
    }
    NB_CUDA(ctx, cudaGetLastError());
    double merged[6];
    unsigned long long lim[2];
    unsigned flags[2] = {0, 0};
    NB_CUDA(ctx, cudaMemcpyAsync(merged, S.merged, sizeof(merged), cudaMemcpyDeviceToHost, st));
    NB_CUDA(ctx, cudaMemcpyAsync(lim, S.lim, sizeof(lim), cudaMemcpyDeviceToHost, st));
    NB_CUDA(ctx, cudaMemcpyAsync(&flags[0], S.status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    if (closure_status)
        NB_CUDA(ctx, cudaMemcpyAsync(&flags[1], closure_status, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    if (flags[1]) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "turbulence field violates its finite physical domain");
    if (flags[0])
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT,
                    "SGS stability evaluation requires finite physical state and tendencies");
    const double linear = merged[0], norm = merged[1];
    if (!std::isfinite(linear) || !std::isfinite(norm) || norm < 0.0)
        return fail(ctx, NIMBUS_ERR_NONFINITE, "SGS momentum stability reduction produced an invalid result");
    constexpr double safety = 0.9;
    nimbus_sgs_stability r{};
    r.momentum_energy_timestep_s = std::numeric_limits<double>::infinity();
    if (norm > 0.0)
    {
        if (!(linear < 0.0)) return fail(ctx, NIMBUS_ERR_NONFINITE, "realized SGS momentum tendency is not dissipative");
        r.momentum_irreversible_dissipation_w = -linear;
        r.momentum_energy_timestep_s = safety * (-2.0 * linear / norm);
    }
    double limits[2];
    for (int q = 0; q < 2; ++q)
    {
        double raw;
        std::memcpy(&raw, &lim[q], sizeof(raw));
        if (std::isinf(raw) || raw >= 0.5 * DBL_MAX)
            limits[q] = std::numeric_limits<double>::infinity();
        else if (!std::isfinite(raw) || raw <= 0.0)
            return fail(ctx, NIMBUS_ERR_NONFINITE, "realized SGS tendency has no positive monotonic timestep");
        else
            limits[q] = safety * raw;
    }
    r.theta_monotonic_timestep_s = limits[0];
    r.qv_monotonic_timestep_s = limits[1];
    r.maximum_timestep_s = std::min({r.momentum_energy_timestep_s, limits[0], limits[1]});
    if (!(r.maximum_timestep_s > 0.0))
        return fail(ctx, NIMBUS_ERR_NONFINITE, "realized SGS explicit stability limit is invalid");
    *out = r;
    return NIMBUS_OK;
}

bool open_stress_boundary(const nimbus_smagorinsky_args* a)
{
    const bool lateral = a->open_lateral[0] || a->open_lateral[1] || a->open_lateral[2] || a->open_lateral[3];
    return lateral || (a->open_top && a->use_vertical);
}

struct ApplyDevice
{
    float *u, *v, *w, *theta, *qv, *tke;
    const float *du, *dv, *dw, *dth, *dqv, *dtke, *dtke_pbl;
};

nimbus_status launch_apply(nimbus_cuda_context* ctx, cudaStream_t st, int n, int nz, double dt, int sanitize,
                           double theta_ref, float th_lo, float th_hi, float qv_hi, float wind_h, float wind_v,
                           const double* theta0_dev, const ApplyDevice& D)
{
    SgsApplyParams A{n, nz, dt, sanitize ? 1 : 0, theta_ref, th_lo, th_hi, qv_hi, wind_h, wind_v, theta0_dev};
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_SGS);
        sgs_apply_kernel<<<grid_for(ctx, n), kThreads, 0, st>>>(A, D.u, D.v, D.w, D.theta, D.qv, D.tke, D.du, D.dv,
                                                               D.dw, D.dth, D.dqv, D.dtke, D.dtke_pbl);
        ctx->launches += 1;
    }
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

// theta0_base on the device (nz doubles).
nimbus_status stage_theta0(nimbus_cuda_context* ctx, cudaStream_t st, const double* host, int nz, double** dev)
{
    *dev = nullptr;
    if (!host) return NIMBUS_OK;
    double* base = nullptr;
    NB_TRY(ensure(ctx, kSgsTheta0, static_cast<size_t>(nz), &base));
    NB_CUDA(ctx, cudaMemcpyAsync(base, host, static_cast<size_t>(nz) * sizeof(double), cudaMemcpyHostToDevice, st));
    *dev = base;
    return NIMBUS_OK;
}

// Closure device pointers: the caller's (device memory) or workspace for
// the missing coefficient / rate outputs.
nimbus_status closure_device(nimbus_cuda_context* ctx, const nimbus_smagorinsky_args* a, ClosureDevice& D)
{
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    float* coef = nullptr;
    float* rates = nullptr;
    NB_TRY(ensure(ctx, kSgsCoef, 3 * n, &coef));
    NB_TRY(ensure(ctx, kSgsRates, 5 * n, &rates));
    D = ClosureDevice{a->u, a->v, a->w, a->theta, a->qv, a->rho, a->nu_t ? a->nu_t : coef,
                      a->K_theta ? a->K_theta : coef + n, a->K_q ? a->K_q : coef + 2 * n,
                      a->dudt_sgs ? a->dudt_sgs : rates, a->dvdt_sgs ? a->dvdt_sgs : rates + n,
                      a->dwdt_sgs ? a->dwdt_sgs : rates + 2 * n, a->dthetadt_sgs ? a->dthetadt_sgs : rates + 3 * n,
                      a->dqvdt_sgs ? a->dqvdt_sgs : rates + 4 * n};
    return NIMBUS_OK;
}

}  // namespace

extern "C" {

nimbus_status nimbus_cuda_smagorinsky_fused(nimbus_cuda_context* ctx, const nimbus_smagorinsky_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    std::vector<double> delta;
    if (const char* why = check_closure(a, delta)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (!a->dudt_sgs || !a->dvdt_sgs || !a->dwdt_sgs || !a->dthetadt_sgs || (a->qv && !a->dqvdt_sgs))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "a tendency output is null");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE && a->stream) st = static_cast<cudaStream_t>(a->stream);
    SgsParams P = params_of(a);
    NB_TRY(stage_tables(ctx, st, a->dz, delta, P));
    const size_t n = static_cast<size_t>(P.d.cells());
    const size_t bytes = n * sizeof(float);
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        ClosureDevice D;
        NB_TRY(closure_device(ctx, a, D));
        return launch_closure(ctx, st, P, D, ctx->status);
    }
    // Host memory: stage the state, run, and publish only a valid result.
    float *u, *v, *w, *th, *qv = nullptr, *rho, *coef, *rates;
    NB_TRY(ensure(ctx, kU, n, &u));
    NB_TRY(ensure(ctx, kV, n, &v));
    NB_TRY(ensure(ctx, kW, n, &w));
    NB_TRY(ensure(ctx, kTheta, n, &th));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kSgsCoef, 3 * n, &coef));
    NB_TRY(ensure(ctx, kSgsRates, 5 * n, &rates));
    NB_TRY(upload(ctx, u, a->u, bytes));
    NB_TRY(upload(ctx, v, a->v, bytes));
    NB_TRY(upload(ctx, w, a->w, bytes));
    NB_TRY(upload(ctx, th, a->theta, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    if (a->qv)
    {
        NB_TRY(ensure(ctx, kQv, n, &qv));
        NB_TRY(upload(ctx, qv, a->qv, bytes));
    }
    StabilityScratch S;
    NB_TRY(stability_scratch(ctx, a->nx, S));
    NB_CUDA(ctx, cudaMemsetAsync(S.status, 0, sizeof(unsigned), st));
    const ClosureDevice D{u, v, w, th, qv, rho, coef, coef + n, coef + 2 * n,
                          rates, rates + n, rates + 2 * n, rates + 3 * n, rates + 4 * n};
    NB_TRY(launch_closure(ctx, st, P, D, S.status));
    unsigned flag = 0;
    NB_CUDA(ctx, cudaMemcpyAsync(&flag, S.status, sizeof(flag), cudaMemcpyDeviceToHost, st));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    if (flag)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT,
                    "turbulence field violates its finite physical domain or a coefficient is not finite");
    float* outs[8] = {a->nu_t, a->K_theta, a->K_q, a->dudt_sgs, a->dvdt_sgs, a->dwdt_sgs, a->dthetadt_sgs,
                      a->dqvdt_sgs};
    const float* srcs[8] = {coef, coef + n, coef + 2 * n, rates, rates + n, rates + 2 * n, rates + 3 * n,
                            rates + 4 * n};
    for (int f = 0; f < 8; ++f)
        if (outs[f]) NB_TRY(download(ctx, outs[f], srcs[f], bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_sgs_apply(nimbus_cuda_context* ctx, const nimbus_sgs_apply_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->u || !a->v || !a->w || !a->theta || !a->dudt || !a->dvdt || !a->dwdt || !a->dthetadt ||
        (a->qv && !a->dqvdt) || (a->tke && (!a->dtkedt || !a->dtkedt_pbl)))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "a required SGS apply pointer is null");
    if (a->nx < 1 || a->ny < 1 || a->nz < 1 || !cells_fit(a->nx, a->ny, a->nz))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid SGS apply grid");
    if (!finite_positive(a->dt))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "SGS apply requires a positive finite timestep");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE && a->stream) st = static_cast<cudaStream_t>(a->stream);
    double* theta0 = nullptr;
    NB_TRY(stage_theta0(ctx, st, a->theta0_base, a->nz, &theta0));
    const int n = a->nx * a->ny * a->nz;
    const size_t bytes = static_cast<size_t>(n) * sizeof(float);
    ApplyDevice D{a->u, a->v, a->w, a->theta, a->qv, a->tke, a->dudt, a->dvdt, a->dwdt, a->dthetadt, a->dqvdt,
                  a->dtkedt, a->dtkedt_pbl};
    if (a->memory == NIMBUS_MEMORY_HOST)
    {
        float *f[6] = {}, *r[7] = {};
        const Slot fs[6] = {kU, kV, kW, kTheta, kQv, kTke};
        float* const hf[6] = {a->u, a->v, a->w, a->theta, a->qv, a->tke};
        for (int q = 0; q < 6; ++q)
        {
            if (!hf[q]) continue;
            NB_TRY(ensure(ctx, fs[q], static_cast<size_t>(n), &f[q]));
            NB_TRY(upload(ctx, f[q], hf[q], bytes));
        }
        float* rates = nullptr;
        float* tke_rates = nullptr;
        NB_TRY(ensure(ctx, kSgsRates, 5 * static_cast<size_t>(n), &rates));
        if (a->tke) NB_TRY(ensure(ctx, kTkeRates, 2 * static_cast<size_t>(n), &tke_rates));
        const float* hr[7] = {a->dudt, a->dvdt, a->dwdt, a->dthetadt, a->dqvdt, a->dtkedt, a->dtkedt_pbl};
        for (int q = 0; q < 7; ++q)
        {
            if (!hr[q] || (q == 4 && !a->qv) || (q >= 5 && !a->tke)) continue;
            r[q] = q < 5 ? rates + static_cast<size_t>(q) * n : tke_rates + static_cast<size_t>(q - 5) * n;
            NB_TRY(upload(ctx, r[q], hr[q], bytes));
        }
        D = ApplyDevice{f[0], f[1], f[2], f[3], f[4], f[5], r[0], r[1], r[2], r[3], r[4], r[5], r[6]};
    }
    NB_TRY(launch_apply(ctx, st, n, a->nz, a->dt, a->sanitize, a->theta_reference, a->theta_min, a->theta_max,
                        a->qv_max, a->wind_h_max, a->wind_v_max, theta0, D));
    if (a->memory == NIMBUS_MEMORY_HOST)
    {
        float* const hf[6] = {a->u, a->v, a->w, a->theta, a->qv, a->tke};
        float* const df[6] = {D.u, D.v, D.w, D.theta, D.qv, D.tke};
        for (int q = 0; q < 6; ++q)
            if (hf[q]) NB_TRY(download(ctx, hf[q], df[q], bytes));
        NB_CUDA(ctx, cudaStreamSynchronize(st));
    }
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_sgs_stability(nimbus_cuda_context* ctx, const nimbus_smagorinsky_args* a,
                                        nimbus_sgs_stability* out)
{
    if (!ctx || !a || !out) return NIMBUS_ERR_INVALID_ARGUMENT;
    std::vector<double> delta;
    if (const char* why = check_closure(a, delta)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (!a->dudt_sgs || !a->dvdt_sgs || !a->dwdt_sgs || !a->dthetadt_sgs || (a->qv && !a->dqvdt_sgs))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "a tendency input is null");
    if (open_stress_boundary(a))
        return fail(ctx, NIMBUS_ERR_UNSUPPORTED, "open stress boundaries need the realized boundary-power term");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE && a->stream) st = static_cast<cudaStream_t>(a->stream);
    SgsParams P = params_of(a);
    NB_TRY(stage_tables(ctx, st, a->dz, delta, P));
    const size_t n = static_cast<size_t>(P.d.cells());
    const size_t bytes = n * sizeof(float);
    ClosureDevice D{a->u, a->v, a->w, a->theta, a->qv, a->rho, nullptr, nullptr, nullptr,
                    a->dudt_sgs, a->dvdt_sgs, a->dwdt_sgs, a->dthetadt_sgs, a->dqvdt_sgs};
    if (a->memory == NIMBUS_MEMORY_HOST)
    {
        float *u, *v, *w, *th, *qv = nullptr, *rho, *rates;
        NB_TRY(ensure(ctx, kU, n, &u));
        NB_TRY(ensure(ctx, kV, n, &v));
        NB_TRY(ensure(ctx, kW, n, &w));
        NB_TRY(ensure(ctx, kTheta, n, &th));
        NB_TRY(ensure(ctx, kRho, n, &rho));
        NB_TRY(ensure(ctx, kSgsRates, 5 * n, &rates));
        const float* hs[5] = {a->u, a->v, a->w, a->theta, a->rho};
        float* ds[5] = {u, v, w, th, rho};
        for (int q = 0; q < 5; ++q) NB_TRY(upload(ctx, ds[q], hs[q], bytes));
        if (a->qv)
        {
            NB_TRY(ensure(ctx, kQv, n, &qv));
            NB_TRY(upload(ctx, qv, a->qv, bytes));
        }
        const float* hr[5] = {a->dudt_sgs, a->dvdt_sgs, a->dwdt_sgs, a->dthetadt_sgs, a->dqvdt_sgs};
        for (int q = 0; q < 5; ++q)
            if (hr[q] && (q < 4 || a->qv)) NB_TRY(upload(ctx, rates + q * n, hr[q], bytes));
        D = ClosureDevice{u, v, w, th, qv, rho, nullptr, nullptr, nullptr,
                          rates, rates + n, rates + 2 * n, rates + 3 * n, rates + 4 * n};
    }
    StabilityScratch S;
    NB_TRY(stability_scratch(ctx, a->nx, S));
    const Rates R{D.du, D.dv, D.dw, D.dth, D.dqv};
    return run_stability(ctx, st, P, D, R, S, nullptr, out);
}

nimbus_status nimbus_cuda_sgs_step(nimbus_cuda_context* ctx, const nimbus_sgs_step_args* a, int* substeps,
                                   double* stability_limit_s)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    const nimbus_smagorinsky_args* c = &a->closure;
    std::vector<double> delta;
    if (const char* why = check_closure(c, delta)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (c->memory != NIMBUS_MEMORY_DEVICE) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "SGS step needs device memory");
    if (!finite_positive(a->dt) || !finite_positive(a->dt_sgs) || !std::isfinite(a->time_s))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "SGS step needs finite positive dt and dt_sgs");
    if (open_stress_boundary(c))
        return fail(ctx, NIMBUS_ERR_UNSUPPORTED, "open stress boundaries need the realized boundary-power term");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = c->stream ? static_cast<cudaStream_t>(c->stream) : ctx->stream;
    SgsParams P = params_of(c);
    NB_TRY(stage_tables(ctx, st, c->dz, delta, P));
    double* theta0 = nullptr;
    NB_TRY(stage_theta0(ctx, st, a->theta0_base, c->nz, &theta0));
    ClosureDevice D;
    NB_TRY(closure_device(ctx, c, D));
    StabilityScratch S;
    NB_TRY(stability_scratch(ctx, c->nx, S));
    unsigned* closure_flag = S.status + 1;
    const Rates R{D.du, D.dv, D.dw, D.dth, D.dqv};
    const ApplyDevice A{const_cast<float*>(c->u), const_cast<float*>(c->v), const_cast<float*>(c->w),
                        const_cast<float*>(c->theta), const_cast<float*>(c->qv), nullptr,
                        D.du, D.dv, D.dw, D.dth, D.dqv, nullptr, nullptr};
    const int n = P.d.cells();
    // The reference's explicit SGS loop (dynamics.cpp:7159-7217).
    const double dt = a->dt;
    const double floor_s = 64.0 * std::numeric_limits<double>::epsilon() * std::max({1.0, dt, std::abs(a->time_s)});
    double advanced = 0.0, seen = std::numeric_limits<double>::infinity();
    int count = 0;
    while (advanced < dt)
    {
        NB_CUDA(ctx, cudaMemsetAsync(closure_flag, 0, sizeof(unsigned), st));
        NB_TRY(launch_closure(ctx, st, P, D, closure_flag));
        nimbus_sgs_stability stab;
        NB_TRY(run_stability(ctx, st, P, D, R, S, closure_flag, &stab));
        seen = std::min(seen, stab.maximum_timestep_s);
        const double remaining = dt - advanced;
        const double sub = std::min({remaining, a->dt_sgs, stab.maximum_timestep_s});
        if (!std::isfinite(sub) || sub <= floor_s || ++count > 1000000)
            return fail(ctx, NIMBUS_ERR_NONFINITE, "SGS explicit integration cannot make stable progress");
        NB_TRY(launch_apply(ctx, st, n, c->nz, sub, a->sanitize, 300.0, 200.0f, 700.0f, 0.05f, 180.0f, 120.0f,
                            theta0, A));
        advanced += sub;
        if (dt - advanced <= floor_s) advanced = dt;
    }
    if (substeps) *substeps = count;
    if (stability_limit_s) *stability_limit_s = seen;
    return NIMBUS_OK;
}

}  // extern "C"
