// C-ABI of the B200 CUDA backend (include/nimbus_cuda.h).
//
// Host-memory calls stage through a per-context device workspace and return
// fence-confirmed, leaving host arrays untouched on any refusal or failure
// (include/compute/dispatch/dynamics.hpp:682-683).  Device-memory calls only
// enqueue; nimbus_cuda_synchronize() reports their status word.
#include "../../include/nimbus_cuda.h"
#include "context.cuh"
#include "launch.cuh"

#include "acoustic_fused.cuh"
#include "acoustic_kernels.cuh"
#include "acoustic_split.cuh"
#include "slow_kernels.cuh"
#include "physics_kernels.cuh"
#include "relaxation_kernels.cuh"
#include "transport_kernels.cuh"

#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

using namespace nimbus;
using namespace nimbus_host;

namespace
{

// Mirrors valid_acoustic_cgrid_dispatch (src/compute/cpu/acoustic_cgrid.cpp:11-46).
const char* check_acoustic_common(const float* u, const float* v, const float* w, const float* rho, const float* p,
                                  const float* theta, const double* rho0, const double* p0, int base_len, int nx,
                                  int ny, int nz, double dx, double dy, double dz, double dt, double gamma,
                                  float rho_min, float rho_max, float p_min, float p_max, float p_ref,
                                  float wind_h, float wind_v)
{
    if (!u || !v || !w || !rho || !p || !theta || !rho0 || !p0) return "a required field pointer is null";
    if (nx < 3 || ny < 3 || nz < 2) return "grid must be at least 3x3x2";
    if (!cells_fit(nx, ny, nz)) return "grid too large for one dispatch";
    if (base_len < nz) return "base profiles shorter than nz";
    if (!finite_positive(dx) || !finite_positive(dy) || !finite_positive(dz)) return "grid spacing must be finite and positive";
    if (!finite_positive(dt)) return "dt_small must be finite and positive";
    if (!finite_positive(gamma)) return "gamma must be finite and positive";
    if (!valid_bounds(rho_min, rho_max) || !valid_bounds(p_min, p_max)) return "invalid clamp bounds";
    if (!finite_positive(p_ref)) return "p_ref_fallback must be finite and positive";
    if (!std::isfinite(wind_h) || wind_h < 0.0f || !std::isfinite(wind_v) || wind_v < 0.0f) return "invalid wind clamps";
    const void* outs[] = {u, v, w, rho, p};
    for (int a = 0; a < 5; ++a)
    {
        if (outs[a] == theta) return "theta aliases an output field";
        for (int b = 0; b < a; ++b)
            if (outs[a] == outs[b]) return "output fields alias";
    }
    return nullptr;
}

AcousticParams acoustic_params(int nx, int ny, int nz, double dx, double dy, double dz, double dt, double gamma,
                               float rho_min, float rho_max, float p_min, float p_max, float p_ref, float wind_h,
                               float wind_v)
{
    AcousticParams P{};
    P.d = make_dims(nx, ny, nz);
    P.inv_dx = 1.0 / dx;
    P.inv_dy = 1.0 / dy;
    P.inv_dz = 1.0 / dz;
    P.dt_small = dt;
    P.gamma = gamma;
    P.rho_min = rho_min;
    P.rho_max = rho_max;
    P.p_min = p_min;
    P.p_max = p_max;
    P.p_ref_fallback = p_ref;
    P.wind_h = wind_h;
    P.wind_v = wind_v;
    return P;
}

// ---------------------------------------------------------------------------
// Device-side sequences (all pointers device memory).
// ---------------------------------------------------------------------------

struct AcousticDevice
{
    float *u, *v, *w, *rho, *p;
    const float* theta;
    const double *rho0, *p0;
    float* rho_alt;   // ping-pong partner of rho
    float* drho;      // optional
    float *mfx, *mfy, *mfz;  // optional (all or none)
    float *u_alt, *v_alt, *w_alt;  // ping-pong partners of u, v, w (fused substep)
};

nimbus_status ensure_alts(nimbus_cuda_context* ctx, size_t n, AcousticDevice& D)
{
    NB_TRY(ensure(ctx, kRhoAlt, n, &D.rho_alt));
    NB_TRY(ensure(ctx, kUAlt, n, &D.u_alt));
    NB_TRY(ensure(ctx, kVAlt, n, &D.v_alt));
    NB_TRY(ensure(ctx, kWAlt, n, &D.w_alt));
    return NIMBUS_OK;
}

int resolve_form(const nimbus_cuda_context* ctx, const Dims& d)
{
    if (ctx->substep_form != NIMBUS_SUBSTEP_AUTO) return ctx->substep_form;
    for (const auto& e : ctx->tuned)
        if (e.nx == d.nx && e.ny == d.ny && e.nz == d.nz && e.precision == ctx->precision) return e.form;
    return NIMBUS_SUBSTEP_SPLIT;
}

nimbus_status launch_fused(nimbus_cuda_context* ctx, cudaStream_t st, const FusedParams& F, const Prognostic& in,
                           const Prognostic& out, float* p, const float* theta, const double* rho0, const double* p0,
                           const float2* dp0, const float4* eos0, float* drho, float* mfx, float* mfy, float* mfz)
{
    const bool fp32 = ctx->precision == NIMBUS_PRECISION_FP32;
    if (resolve_form(ctx, F.d) == NIMBUS_SUBSTEP_SPLIT)
    {
        if (fp32) return nimbus_fp32::launch_split(ctx, st, F, in, out, p, theta, rho0, p0, dp0, eos0, drho, mfx, mfy, mfz);
        return launch_split_impl<RefPolicy>(ctx, st, F, in, out, p, theta, rho0, p0, dp0, eos0, drho, mfx, mfy, mfz);
    }
    if (fp32) return nimbus_fp32::launch_fused(ctx, st, F, in, out, p, theta, rho0, p0, dp0, eos0, drho, mfx, mfy, mfz);
    return launch_fused_impl<RefPolicy>(ctx, st, F, in, out, p, theta, rho0, p0, dp0, eos0, drho, mfx, mfy, mfz);
}

// Resting state for the autotuner: rho=1.1, u=v=w=0, p=9e4, theta=300, zero
// fluxes; profiles rho0=1.1, p0=9e4 and a zero hydrostatic difference.
__global__ void fill_tuning_state(float* buf, size_t n, double* prof, int nz, float2* dp0)
{
    for (size_t c = blockIdx.x * (size_t)blockDim.x + threadIdx.x; c < n; c += (size_t)gridDim.x * blockDim.x)
    {
        buf[c] = 0.0f;            // u
        buf[n + c] = 0.0f;        // v
        buf[2 * n + c] = 0.0f;    // w
        buf[3 * n + c] = 1.1f;    // rho
        buf[4 * n + c] = 0.0f;
        buf[5 * n + c] = 0.0f;
        buf[6 * n + c] = 0.0f;
        buf[7 * n + c] = 1.1f;
        buf[8 * n + c] = 90000.0f;  // p
        buf[9 * n + c] = 300.0f;    // theta
        buf[10 * n + c] = 0.0f;
        buf[11 * n + c] = 0.0f;
        buf[12 * n + c] = 0.0f;
    }
    if (blockIdx.x == 0)
        for (int k = threadIdx.x; k < nz; k += blockDim.x)
        {
            prof[k] = 1.1;
            prof[nz + k] = 90000.0;
            dp0[k] = make_float2(0.0f, 0.0f);
        }
}

FusedParams fused_params(const nimbus_cuda_context* ctx, int nx, int ny, int nz, double dx, double dy, double dz,
                         double dt, double gamma, float rho_min, float rho_max, float p_min, float p_max, float p_ref,
                         float wind_h, float wind_v)
{
    FusedParams F{};
    F.d = make_dims(nx, ny, nz);
    F.inv_dx = 1.0 / dx;
    F.inv_dy = 1.0 / dy;
    F.inv_dz = 1.0 / dz;
    F.dt_small = dt;
    F.gamma = gamma;
    F.rho_min = rho_min;
    F.rho_max = rho_max;
    F.p_min = p_min;
    F.p_max = p_max;
    F.p_ref_fallback = p_ref;
    F.wind_h = wind_h;
    F.wind_v = wind_v;
    F.chunk = 1;  // set at launch from the kernel's occupancy
    finish_fp32(F);
    return F;
}

void launch_boundaries(nimbus_cuda_context* ctx, cudaStream_t st, const BoundaryParams& B, const AcousticDevice& D,
                       float* rho, float* wave)
{
    const Dims d = B.d;
    const int yz = d.ny * d.nz, xz = d.nx * d.nz;
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_ACOUSTIC_BOUNDARY);
    acoustic_bc_we_kernel<<<grid_for(ctx, yz), kThreads, 0, st>>>(B, D.u, D.v, D.w, rho, D.p, wave, wave + yz);
    acoustic_bc_sn_kernel<<<grid_for(ctx, xz), kThreads, 0, st>>>(B, D.u, D.v, D.w, rho, D.p, wave + 2 * yz,
                                                                  wave + 2 * yz + xz);
    acoustic_bc_vertical_kernel<<<grid_for(ctx, d.nx * d.ny), kThreads, 0, st>>>(B, D.u, D.v, D.w);
    ctx->launches += 3;
}

nimbus_status run_batched_device(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus_acoustic_batched_args* a,
                                 const AcousticDevice& D, float* wave, const float* wave_in, float* density_begin)
{
    const Dims d = make_dims(a->nx, a->ny, a->nz);
    const size_t n = static_cast<size_t>(d.cells());
    const int yz = d.ny * d.nz, xz = d.nx * d.nz;
    if (wave_in == nullptr)
    {
        acoustic_seed_radiation_kernel<<<grid_for(ctx, yz + xz), kThreads, 0, st>>>(d, D.u, D.v, wave);
        ctx->launches += 1;
    }
    else if (wave_in != wave)
    {
        NB_CUDA(ctx, cudaMemcpyAsync(wave, wave_in, sizeof(float) * 2 * (yz + xz), cudaMemcpyDeviceToDevice, st));
    }
    if (density_begin)
        NB_CUDA(ctx, cudaMemcpyAsync(density_begin, D.rho, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));

    FusedParams F = fused_params(ctx, a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small, a->gamma, a->rho_min,
                                 a->rho_max, a->p_min, a->p_max, a->p_ref_fallback, a->wind_clamp_h, a->wind_clamp_v);
    F.weight = a->mass_flux_weight;
    F.frame_u = a->frame_velocity_u_ms;
    F.frame_v = a->frame_velocity_v_ms;
    F.top_open = a->bc_top == kTopOpen;
    finish_fp32(F);

    BoundaryParams B{};
    B.d = d;
    B.west = a->bc_west; B.east = a->bc_east; B.south = a->bc_south; B.north = a->bc_north;
    B.bottom = a->bc_bottom; B.top = a->bc_top;
    B.dt_rad = static_cast<float>(a->dt_small);
    B.inv_dx = 1.0f / static_cast<float>(a->dx);
    B.inv_dy = 1.0f / static_cast<float>(a->dy);
    B.frame_u = a->frame_velocity_u_ms;
    B.frame_v = a->frame_velocity_v_ms;

    float2* dp0 = nullptr;
    float4* eos0 = nullptr;
    NB_TRY(ensure(ctx, kDp0, static_cast<size_t>(d.nz), &dp0));
    NB_TRY(ensure(ctx, kEos0, static_cast<size_t>(d.nz), &eos0));
    level_base_kernel<<<(d.nz + 127) / 128, 128, 0, st>>>(D.p0, d.nz, F.gamma, dp0, eos0);
    ctx->launches += 1;
    Prognostic user{D.u, D.v, D.w, D.rho};
    Prognostic work{D.u_alt, D.v_alt, D.w_alt, D.rho_alt};
    Prognostic cur = user, alt = work;
    for (int s = 0; s < a->n_substeps; ++s)
    {
        NB_TRY(launch_fused(ctx, st, F, cur, alt, D.p, D.theta, D.rho0, D.p0, dp0, eos0, nullptr, D.mfx, D.mfy,
                            D.mfz));
        AcousticDevice E = D;
        E.u = alt.u; E.v = alt.v; E.w = alt.w;
        launch_boundaries(ctx, st, B, E, alt.rho, wave);
        std::swap(cur, alt);
    }
    if (cur.u != user.u)
    {
        NB_CUDA(ctx, cudaMemcpyAsync(user.u, cur.u, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        NB_CUDA(ctx, cudaMemcpyAsync(user.v, cur.v, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        NB_CUDA(ctx, cudaMemcpyAsync(user.w, cur.w, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        NB_CUDA(ctx, cudaMemcpyAsync(user.rho, cur.rho, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    }
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

// One fused substep on device memory, result back in the caller's arrays.
nimbus_status run_fused_device(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus_acoustic_fused_args* a,
                               const AcousticDevice& D)
{
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    FusedParams F = fused_params(ctx, a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small, a->gamma, a->rho_min,
                                 a->rho_max, a->p_min, a->p_max, a->p_ref_fallback, a->wind_clamp_h, a->wind_clamp_v);
    float2* dp0 = nullptr;
    float4* eos0 = nullptr;
    NB_TRY(ensure(ctx, kDp0, static_cast<size_t>(a->nz), &dp0));
    NB_TRY(ensure(ctx, kEos0, static_cast<size_t>(a->nz), &eos0));
    level_base_kernel<<<(a->nz + 127) / 128, 128, 0, st>>>(D.p0, a->nz, F.gamma, dp0, eos0);
    ctx->launches += 1;
    Prognostic user{D.u, D.v, D.w, D.rho};
    Prognostic work{D.u_alt, D.v_alt, D.w_alt, D.rho_alt};
    NB_TRY(launch_fused(ctx, st, F, user, work, D.p, D.theta, D.rho0, D.p0, dp0, eos0, D.drho, nullptr, nullptr,
                        nullptr));
    NB_CUDA(ctx, cudaMemcpyAsync(user.u, work.u, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    NB_CUDA(ctx, cudaMemcpyAsync(user.v, work.v, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    NB_CUDA(ctx, cudaMemcpyAsync(user.w, work.w, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    NB_CUDA(ctx, cudaMemcpyAsync(user.rho, work.rho, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

const char* check_batched(const nimbus_acoustic_batched_args* a)
{
    const char* why = check_acoustic_common(a->u, a->v, a->w, a->rho, a->p, a->theta, a->rho0_base, a->p0_base,
                                            a->base_len, a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small,
                                            a->gamma, a->rho_min, a->rho_max, a->p_min, a->p_max,
                                            a->p_ref_fallback, a->wind_clamp_h, a->wind_clamp_v);
    if (why) return why;
    if (a->nx < 4 || a->ny < 4) return "batched acoustic loop needs nx>=4 and ny>=4";
    if (a->n_substeps < 1 || a->n_substeps > 4096) return "n_substeps must be in [1, 4096]";
    for (int bc : {a->bc_west, a->bc_east, a->bc_south, a->bc_north})
        if (bc < 0 || bc > 4) return "lateral boundary code out of range";
    if (a->bc_bottom < 0 || a->bc_bottom > 1 || a->bc_top < 0 || a->bc_top > 2) return "vertical boundary code out of range";
    if (!a->wave_history_output) return "wave_history_output is required";
    if (a->accumulate_mass_flux)
    {
        if (!a->mass_flux_x || !a->mass_flux_y || !a->mass_flux_z) return "mass flux outputs are required";
        if (!finite_positive(a->mass_flux_weight)) return "mass_flux_weight must be finite and positive";
    }
    if (!std::isfinite(a->frame_velocity_u_ms) || !std::isfinite(a->frame_velocity_v_ms)) return "frame velocity must be finite";
    return nullptr;
}

const char* check_transport(const nimbus_scalar_transport_args* a)
{
    if (a->n_scalars < 0 || a->n_scalars > kMaxScalars) return "n_scalars must be in [0, 16]";
    if (a->n_scalars == 0) return nullptr;
    if (!a->q_in || !a->q_out || !a->positive_definite) return "scalar pointer arrays are required";
    if (!a->rho_end || !a->rho_begin || !a->mass_flux_x || !a->mass_flux_y || !a->mass_flux_z)
        return "density and mass-flux pointers are required";
    if (a->nx < 3 || a->ny < 3 || a->nz < 2) return "grid must be at least 3x3x2";
    if (!cells_fit(a->nx, a->ny, a->nz)) return "grid too large for one dispatch";
    if (!finite_positive(a->dx) || !finite_positive(a->dy) || !finite_positive(a->dz) || !finite_positive(a->dt))
        return "spacing and dt must be finite and positive";
    if (!(std::isfinite(a->rho_floor) && a->rho_floor > 0.0f)) return "rho_floor must be finite and positive";
    for (int s = 0; s < a->n_scalars; ++s)
    {
        if (!a->q_in[s] || !a->q_out[s]) return "null scalar field";
        for (int t = 0; t < s; ++t)
            if (a->q_out[s] == a->q_out[t] || a->q_in[s] == a->q_in[t]) return "duplicate scalar field";
    }
    return nullptr;
}

TransportParams transport_params(const nimbus_scalar_transport_args* a)
{
    TransportParams T{};
    T.d = make_dims(a->nx, a->ny, a->nz);
    T.inv_dx = 1.0 / a->dx;
    T.inv_dy = 1.0 / a->dy;
    T.inv_dz = 1.0 / a->dz;
    T.dt = a->dt;
    T.rho_floor = static_cast<double>(a->rho_floor);
    T.weno = a->weno != 0;
    T.top_open = a->top_open != 0;
    T.n_scalars = a->n_scalars;
    for (int s = 0; s < a->n_scalars; ++s) T.positive_definite[s] = a->positive_definite[s] != 0;
    finish_fp32(T);
    return T;
}

nimbus_status run_transport_device(nimbus_cuda_context* ctx, cudaStream_t st, const TransportParams& T,
                                   const float* rho_end, const float* rho_begin, const float* mfx, const float* mfy,
                                   const float* mfz)
{
    const size_t n = static_cast<size_t>(T.d.cells());
    float* sf = nullptr;
    float* rl = nullptr;
    NB_TRY(ensure(ctx, kSf, 3 * n * T.n_scalars, &sf));
    NB_TRY(ensure(ctx, kRl, n * T.n_scalars, &rl));
    if (ctx->precision == NIMBUS_PRECISION_FP32)
        return nimbus_fp32::launch_transport(ctx, st, T, rho_end, rho_begin, mfx, mfy, mfz, sf, rl);
    return launch_transport_impl<false>(ctx, st, T, rho_end, rho_begin, mfx, mfy, mfz, sf, rl);
}

const char* check_slow(const nimbus_slow_args* a, bool step)
{
    if (!a->u || !a->v || !a->w || !a->p || !a->rho || !a->rho0_base) return "a required field pointer is null";
    if (a->nx < 3 || a->ny < 3 || a->nz < 2) return "grid must be at least 3x3x2";
    if (!cells_fit(a->nx, a->ny, a->nz)) return "grid too large for one dispatch";
    if (a->base_len < a->nz) return "base profiles shorter than nz";
    if (!finite_positive(a->dx) || !finite_positive(a->dy) || !finite_positive(a->dz)) return "invalid spacing";
    if (step && !finite_positive(a->dt_large)) return "dt_large must be finite and positive";
    if (!std::isfinite(a->gravity) || !std::isfinite(a->coriolis_f)) return "gravity and coriolis_f must be finite";
    if (a->qv && !a->qv0_base) return "qv requires qv0_base";
    if ((a->qc == nullptr) != (a->qr == nullptr)) return "qc and qr come together";
    const bool outs = a->du_dt && a->dv_dt && a->dw_dt && a->dp_dt;
    const bool none = !a->du_dt && !a->dv_dt && !a->dw_dt && !a->dp_dt;
    if (!step && !outs) return "tendency outputs are required";
    if (step && !outs && !none) return "tendency outputs come together";
    return nullptr;
}

SlowParams slow_params(const nimbus_slow_args* a)
{
    SlowParams S{};
    S.d = make_dims(a->nx, a->ny, a->nz);
    S.inv_dx = 1.0 / a->dx;
    S.inv_dy = 1.0 / a->dy;
    S.inv_dz = 1.0 / a->dz;
    S.dt = a->dt_large;
    S.coriolis_f = a->coriolis_f;
    S.frame_u = a->frame_velocity_u_ms;
    S.frame_v = a->frame_velocity_v_ms;
    S.gravity = a->gravity;
    S.moist = a->qv != nullptr;
    S.loading = a->qc != nullptr;
    finish_fp32(S);
    return S;
}

nimbus_status slow_entry(nimbus_cuda_context* ctx, const nimbus_slow_args* a, bool step)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (const char* why = check_slow(a, step)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const SlowParams S = slow_params(a);
    const bool fp32 = ctx->precision == NIMBUS_PRECISION_FP32;
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
        SlowDevice D{a->u, a->v, a->w, a->p, a->rho, a->qv, a->qc, a->qr, a->rho0_base, a->qv0_base, a->u0_base,
                     a->v0_base, a->du_dt, a->dv_dt, a->dw_dt, a->dp_dt};
        return fp32 ? nimbus_fp32::run_slow(ctx, st, S, D, step) : run_slow_device<RefPolicy>(ctx, st, S, D, step);
    }
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const size_t bytes = n * sizeof(float);
    const size_t nzb = sizeof(double) * static_cast<size_t>(a->nz);
    float *u, *v, *w, *p, *rho, *qv = nullptr, *qc = nullptr, *qr = nullptr, *out = nullptr;
    double *rho0, *qv0 = nullptr, *u0 = nullptr, *v0 = nullptr;
    NB_TRY(ensure(ctx, kU, n, &u));
    NB_TRY(ensure(ctx, kV, n, &v));
    NB_TRY(ensure(ctx, kW, n, &w));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kRho0, static_cast<size_t>(a->nz), &rho0));
    NB_TRY(upload(ctx, u, a->u, bytes));
    NB_TRY(upload(ctx, v, a->v, bytes));
    NB_TRY(upload(ctx, w, a->w, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    NB_TRY(upload(ctx, rho0, a->rho0_base, nzb));
    if (a->qv)
    {
        NB_TRY(ensure(ctx, kQv, n, &qv));
        NB_TRY(ensure(ctx, kQv0, static_cast<size_t>(a->nz), &qv0));
        NB_TRY(upload(ctx, qv, a->qv, bytes));
        NB_TRY(upload(ctx, qv0, a->qv0_base, nzb));
    }
    if (a->qc)
    {
        NB_TRY(ensure(ctx, kQc, n, &qc));
        NB_TRY(ensure(ctx, kQr, n, &qr));
        NB_TRY(upload(ctx, qc, a->qc, bytes));
        NB_TRY(upload(ctx, qr, a->qr, bytes));
    }
    if (a->u0_base)
    {
        NB_TRY(ensure(ctx, kU0, static_cast<size_t>(a->nz), &u0));
        NB_TRY(upload(ctx, u0, a->u0_base, nzb));
    }
    if (a->v0_base)
    {
        NB_TRY(ensure(ctx, kV0, static_cast<size_t>(a->nz), &v0));
        NB_TRY(upload(ctx, v0, a->v0_base, nzb));
    }
    const bool want_out = a->du_dt != nullptr;
    if (want_out) NB_TRY(ensure(ctx, kSlowOut, 4 * n, &out));
    SlowDevice D{u, v, w, p, rho, qv, qc, qr, rho0, qv0, u0, v0, out, out ? out + n : nullptr,
                 out ? out + 2 * n : nullptr, out ? out + 3 * n : nullptr};
    NB_TRY(fp32 ? nimbus_fp32::run_slow(ctx, st, S, D, step) : run_slow_device<RefPolicy>(ctx, st, S, D, step));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    if (step)
    {
        NB_TRY(download(ctx, a->u, u, bytes));
        NB_TRY(download(ctx, a->v, v, bytes));
        NB_TRY(download(ctx, a->w, w, bytes));
        NB_TRY(download(ctx, a->p, p, bytes));
    }
    if (want_out)
    {
        NB_TRY(download(ctx, a->du_dt, out, bytes));
        NB_TRY(download(ctx, a->dv_dt, out + n, bytes));
        NB_TRY(download(ctx, a->dw_dt, out + 2 * n, bytes));
        NB_TRY(download(ctx, a->dp_dt, out + 3 * n, bytes));
    }
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

const char* check_kessler(const nimbus_kessler_args* a, bool step)
{
    if (!a->theta || !a->qv || !a->qc || !a->qr || !a->p || !a->rho) return "a required field pointer is null";
    if (a->nx < 1 || a->ny < 1 || a->nz < 1 || !cells_fit(a->nx, a->ny, a->nz)) return "invalid grid";
    if (!finite_positive(a->dz)) return "dz must be finite and positive";
    if (!std::isfinite(a->dt) || a->dt < 0.0) return "dt must be finite and non-negative";
    const int* d = a->domain;
    if (d[0] < 0 || d[1] > a->nx || d[0] >= d[1] || d[2] < 0 || d[3] > a->ny || d[2] >= d[3] || d[4] < 0 ||
        d[5] > a->nz || d[4] >= d[5])
        return "cell domain is empty or outside the grid";
    const bool outs = a->dtheta_dt && a->dqv_dt && a->dqc_dt && a->dqr_dt;
    const bool none = !a->dtheta_dt && !a->dqv_dt && !a->dqc_dt && !a->dqr_dt;
    if (!step && !outs) return "tendency outputs are required";
    if (step && !outs && !none) return "tendency outputs come together";
    return nullptr;
}

KesslerParams kessler_params(const nimbus_kessler_args* a)
{
    KesslerParams K{};
    K.d = make_dims(a->nx, a->ny, a->nz);
    K.dz = a->dz;
    K.dt = a->dt;
    K.i0 = a->domain[0]; K.i1 = a->domain[1];
    K.j0 = a->domain[2]; K.j1 = a->domain[3];
    K.k0 = a->domain[4]; K.k1 = a->domain[5];
    // KesslerScheme defaults (kessler.hpp:40-46, microphysics/config.hpp:11-18).
    K.qc0 = 1.0e-3;
    K.c_auto = 1.0e-3;
    K.c_accr = 2.2;
    K.evap_eff = 1.0;
    K.vt_max = 20.0;
    finish_fp32(K);
    return K;
}

// Kessler on device memory; in the step form qr is rewritten through the
// workspace ping-pong buffer.
nimbus_status run_kessler_device(nimbus_cuda_context* ctx, cudaStream_t st, const KesslerParams& K, float* theta,
                                 float* qv, float* qc, float* qr, const float* p, const float* rho, float* dth,
                                 float* dqv, float* dqc, float* dqr, bool step)
{
    const size_t n = static_cast<size_t>(K.d.cells());
    const int blocks = grid_for(ctx, static_cast<long long>(n));
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_MICROPHYSICS);
    const bool fp32 = ctx->precision == NIMBUS_PRECISION_FP32;
    if (!step)
    {
        if (fp32)
            kessler_f32_kernel<false><<<blocks, kThreads, 0, st>>>(K, theta, qv, qc, qr, p, rho, nullptr, dth, dqv, dqc,
                                                                  dqr);
        else
            kessler_kernel<false><<<blocks, kThreads, 0, st>>>(K, theta, qv, qc, qr, p, rho, nullptr, dth, dqv, dqc,
                                                              dqr);
        ctx->launches += 1;
    }
    else
    {
        float* qr_new = nullptr;
        NB_TRY(ensure(ctx, kQrAlt, n, &qr_new));
        if (fp32)
            kessler_f32_kernel<true><<<blocks, kThreads, 0, st>>>(K, theta, qv, qc, qr, p, rho, qr_new, dth, dqv, dqc,
                                                                 dqr);
        else
            kessler_kernel<true><<<blocks, kThreads, 0, st>>>(K, theta, qv, qc, qr, p, rho, qr_new, dth, dqv, dqc,
                                                             dqr);
        NB_CUDA(ctx, cudaMemcpyAsync(qr, qr_new, sizeof(float) * n, cudaMemcpyDeviceToDevice, st));
        ctx->launches += 1;
    }
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

nimbus_status kessler_entry(nimbus_cuda_context* ctx, const nimbus_kessler_args* a, bool step)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (const char* why = check_kessler(a, step)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const KesslerParams K = kessler_params(a);
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
        return run_kessler_device(ctx, st, K, a->theta, a->qv, a->qc, a->qr, a->p, a->rho, a->dtheta_dt, a->dqv_dt,
                                  a->dqc_dt, a->dqr_dt, step);
    }
    const size_t n = static_cast<size_t>(K.d.cells());
    const size_t bytes = n * sizeof(float);
    float *th, *qv, *qc, *qr, *p, *rho, *out = nullptr;
    NB_TRY(ensure(ctx, kTheta, n, &th));
    NB_TRY(ensure(ctx, kQv, n, &qv));
    NB_TRY(ensure(ctx, kQc, n, &qc));
    NB_TRY(ensure(ctx, kQr, n, &qr));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(upload(ctx, th, a->theta, bytes));
    NB_TRY(upload(ctx, qv, a->qv, bytes));
    NB_TRY(upload(ctx, qc, a->qc, bytes));
    NB_TRY(upload(ctx, qr, a->qr, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    const bool want_out = a->dtheta_dt != nullptr;
    if (want_out) NB_TRY(ensure(ctx, kKesslerOut, 4 * n, &out));
    NB_TRY(run_kessler_device(ctx, st, K, th, qv, qc, qr, p, rho, out, out ? out + n : nullptr,
                              out ? out + 2 * n : nullptr, out ? out + 3 * n : nullptr, step));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    if (step)
    {
        NB_TRY(download(ctx, a->theta, th, bytes));
        NB_TRY(download(ctx, a->qv, qv, bytes));
        NB_TRY(download(ctx, a->qc, qc, bytes));
        NB_TRY(download(ctx, a->qr, qr, bytes));
    }
    if (want_out)
    {
        NB_TRY(download(ctx, a->dtheta_dt, out, bytes));
        NB_TRY(download(ctx, a->dqv_dt, out + n, bytes));
        NB_TRY(download(ctx, a->dqc_dt, out + 2 * n, bytes));
        NB_TRY(download(ctx, a->dqr_dt, out + 3 * n, bytes));
    }
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

nimbus_status run_eos_device(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus_eos_args* a, float* p,
                             const float* rho, const float* theta, const float* qv, const float* qc,
                             const float* qr, const double* p0_device)
{
    const Dims d = make_dims(a->nx, a->ny, a->nz);
    const long long n = d.cells();
    float* candidate = nullptr;
    NB_TRY(ensure(ctx, kEosCandidate, static_cast<size_t>(n), &candidate));
    // The FP32 form evaluates the EOS around the base pressure profile when
    // the caller gives it (the compensated form of the acoustic substeps).
    const bool fp32 = ctx->precision == NIMBUS_PRECISION_FP32 && p0_device != nullptr;
    float4* eos0 = nullptr;
    if (fp32)
    {
        float2* dp0 = nullptr;
        NB_TRY(ensure(ctx, kDp0, static_cast<size_t>(d.nz), &dp0));
        NB_TRY(ensure(ctx, kEos0, static_cast<size_t>(d.nz), &eos0));
        level_base_kernel<<<(d.nz + 127) / 128, 128, 0, st>>>(p0_device, d.nz, a->gamma, dp0, eos0);
        ctx->launches += 1;
    }
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_MICROPHYSICS);
    if (fp32)
        eos_candidate_f32_kernel<<<grid_for(ctx, n), kThreads, 0, st>>>(d, rho, theta, p, qv, qc, qr, eos0,
                                                                         eos_series(a->gamma), a->gamma, candidate,
                                                                         ctx->status);
    else
        eos_candidate_kernel<<<grid_for(ctx, n), kThreads, 0, st>>>(d, rho, theta, p, qv, qc, qr, a->gamma,
                                                                     candidate, ctx->status);
    eos_publish_kernel<<<grid_for(ctx, (n + 3) / 4), kThreads, 0, st>>>(n, candidate, p, ctx->status);
    ctx->launches += 2;
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// Exported entry points.
// ---------------------------------------------------------------------------

extern "C" {

int nimbus_cuda_abi_version(void) { return NIMBUS_CUDA_ABI_VERSION; }

nimbus_status nimbus_cuda_create(int device, nimbus_cuda_context** out)
{
    if (!out) return NIMBUS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0 || device < 0 || device >= count)
        return NIMBUS_ERR_NO_DEVICE;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) return NIMBUS_ERR_NO_DEVICE;
    if (prop.major != 10) return NIMBUS_ERR_NO_DEVICE;  // built for sm_100a only
    auto* ctx = new (std::nothrow) nimbus_cuda_context();
    if (!ctx) return NIMBUS_ERR_OUT_OF_MEMORY;
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaSetDevice(device) != cudaSuccess || cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
        cudaMalloc(&ctx->status, sizeof(unsigned)) != cudaSuccess || cudaMemset(ctx->status, 0, sizeof(unsigned)) != cudaSuccess)
    {
        nimbus_cuda_destroy(ctx);
        return NIMBUS_ERR_CUDA;
    }
    *out = ctx;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_device_info(nimbus_cuda_context* ctx, nimbus_device_info* out)
{
    if (!ctx || !out) return NIMBUS_ERR_INVALID_ARGUMENT;
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaDeviceProp prop{};
    NB_CUDA(ctx, cudaGetDeviceProperties(&prop, ctx->device));
    size_t free_b = 0, total_b = 0;
    NB_CUDA(ctx, cudaMemGetInfo(&free_b, &total_b));
    *out = nimbus_device_info{};
    std::strncpy(out->name, prop.name, sizeof(out->name) - 1);
    out->sm_count = prop.multiProcessorCount;
    out->cc_major = prop.major;
    out->cc_minor = prop.minor;
    out->total_bytes = total_b;
    out->free_bytes = free_b;
    return NIMBUS_OK;
}

void nimbus_cuda_destroy(nimbus_cuda_context* ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    drain_timing(ctx);
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    for (auto& b : ctx->ws)
        if (b.ptr) cudaFree(b.ptr);
    if (ctx->status) cudaFree(ctx->status);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    delete ctx;
}

const char* nimbus_cuda_last_error(const nimbus_cuda_context* ctx) { return ctx ? ctx->error.c_str() : "null context"; }
uint64_t nimbus_cuda_kernel_launches(const nimbus_cuda_context* ctx) { return ctx ? ctx->launches.load() : 0; }
void* nimbus_cuda_stream(const nimbus_cuda_context* ctx) { return ctx ? static_cast<void*>(ctx->stream) : nullptr; }

nimbus_status nimbus_cuda_synchronize(nimbus_cuda_context* ctx)
{
    if (!ctx) return NIMBUS_ERR_INVALID_ARGUMENT;
    unsigned flags = 0;
    NB_TRY(read_status(ctx, ctx->stream, &flags));
    if (flags & kStatusNonfiniteMassFlux) return fail(ctx, NIMBUS_ERR_NONFINITE, "non-finite retained face mass flux");
    if (flags & kStatusNonfiniteTransport) return fail(ctx, NIMBUS_ERR_NONFINITE, "non-finite transported scalar");
    if (flags & kStatusInvalidEos) return fail(ctx, NIMBUS_ERR_NONFINITE, "EOS projection met an invalid state");
    if (flags & kStatusSgsInvalid)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT,
                    "SGS closure met a state outside its contract or a non-finite coefficient");
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_slow_tendencies(nimbus_cuda_context* ctx, const nimbus_slow_args* a)
{
    return slow_entry(ctx, a, false);
}

nimbus_status nimbus_cuda_slow_step(nimbus_cuda_context* ctx, const nimbus_slow_args* a)
{
    return slow_entry(ctx, a, true);
}

nimbus_status nimbus_cuda_acoustic_boundaries(nimbus_cuda_context* ctx, const nimbus_boundary_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->u || !a->v || !a->w || !a->rho || !a->p) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "a field pointer is null");
    if (a->nx < 4 || a->ny < 4 || a->nz < 2 || !cells_fit(a->nx, a->ny, a->nz))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "boundary closure needs a grid of at least 4x4x2");
    if (!finite_positive(a->dx) || !finite_positive(a->dy) || !std::isfinite(a->dt_small) || a->dt_small < 0.0)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid spacing or dt_small");
    for (int bc : {a->bc_west, a->bc_east, a->bc_south, a->bc_north})
        if (bc < 0 || bc > 4) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "lateral boundary code out of range");
    if (a->bc_bottom < 0 || a->bc_bottom > 1 || a->bc_top < 0 || a->bc_top > 2)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "vertical boundary code out of range");
    const bool radiative = a->bc_west == kBcRadiative || a->bc_east == kBcRadiative || a->bc_south == kBcRadiative ||
                           a->bc_north == kBcRadiative;
    if (a->dt_small > 0.0 && radiative && !a->wave_history)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "radiative faces need the wave history");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = a->stream ? static_cast<cudaStream_t>(a->stream) : ctx->stream;
    BoundaryParams B{};
    B.d = make_dims(a->nx, a->ny, a->nz);
    B.west = a->bc_west; B.east = a->bc_east; B.south = a->bc_south; B.north = a->bc_north;
    B.bottom = a->bc_bottom; B.top = a->bc_top;
    B.dt_rad = static_cast<float>(a->dt_small);
    B.inv_dx = 1.0f / static_cast<float>(a->dx);
    B.inv_dy = 1.0f / static_cast<float>(a->dy);
    B.frame_u = a->frame_velocity_u_ms;
    B.frame_v = a->frame_velocity_v_ms;
    AcousticDevice D{};
    D.u = a->u; D.v = a->v; D.w = a->w; D.rho = a->rho; D.p = a->p;
    // Without radiation the history is never read; any valid pointer will do.
    float* wave = a->wave_history ? a->wave_history : a->u;
    launch_boundaries(ctx, st, B, D, a->rho, wave);
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_kessler_tendencies(nimbus_cuda_context* ctx, const nimbus_kessler_args* a)
{
    return kessler_entry(ctx, a, false);
}

nimbus_status nimbus_cuda_kessler_step(nimbus_cuda_context* ctx, const nimbus_kessler_args* a)
{
    return kessler_entry(ctx, a, true);
}

nimbus_status nimbus_cuda_state_relaxation(nimbus_cuda_context* ctx, const nimbus_state_relaxation_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->u || !a->v || !a->w || !a->theta || a->nx < 1 || a->ny < 1 || a->nz < 1 ||
        !cells_fit(a->nx, a->ny, a->nz) || a->lateral_width < 0)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid state relaxation arguments");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    const int nz = a->nz;
    RelaxImage img;
    if (const char* why = build_relax_image(a->nx, a->ny, nz, a->alpha, a->upper_w_alpha, a->w_only_alpha, a->u_ref,
                                            a->v_ref, a->theta_ref, a->lateral_width, a->lateral_alpha, a->do_upper,
                                            a->do_w_only, a->do_lateral, a->staggered, a->implicit_mode, a->dt, img))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (!img.upper && !img.lid && !img.lateral) return NIMBUS_OK;

    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE && a->stream) st = static_cast<cudaStream_t>(a->stream);
    unsigned char* dev = nullptr;
    NB_TRY(ensure(ctx, kRelaxTables, img.bytes(), &dev));
    // Pageable sources: the call returns once the tables are staged.
    const size_t tab_bytes = img.tab.size() * sizeof(double);
    NB_CUDA(ctx, cudaMemcpyAsync(dev, img.tab.data(), tab_bytes, cudaMemcpyHostToDevice, st));
    NB_CUDA(ctx, cudaMemcpyAsync(dev + tab_bytes, img.on.data(), img.on.size(), cudaMemcpyHostToDevice, st));
    const RelaxTables R = relax_tables(img, dev, nz);
    const Dims d = make_dims(a->nx, a->ny, a->nz);
    const long long n = d.cells();
    float *u = a->u, *v = a->v, *w = a->w, *th = a->theta;
    const size_t bytes = static_cast<size_t>(n) * sizeof(float);
    if (a->memory == NIMBUS_MEMORY_HOST)
    {
        NB_TRY(ensure(ctx, kU, static_cast<size_t>(n), &u));
        NB_TRY(ensure(ctx, kV, static_cast<size_t>(n), &v));
        NB_TRY(ensure(ctx, kW, static_cast<size_t>(n), &w));
        NB_TRY(ensure(ctx, kTheta, static_cast<size_t>(n), &th));
        NB_TRY(upload(ctx, u, a->u, bytes));
        NB_TRY(upload(ctx, v, a->v, bytes));
        NB_TRY(upload(ctx, w, a->w, bytes));
        NB_TRY(upload(ctx, th, a->theta, bytes));
    }
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_MICROPHYSICS);
        state_relaxation_kernel<<<grid_for(ctx, n), kThreads, 0, st>>>(d, R, u, v, w, th);
        ctx->launches += 1;
    }
    NB_CUDA(ctx, cudaGetLastError());
    if (a->memory == NIMBUS_MEMORY_HOST)
    {
        NB_CUDA(ctx, cudaStreamSynchronize(st));
        NB_TRY(download(ctx, a->u, u, bytes));
        NB_TRY(download(ctx, a->v, v, bytes));
        NB_TRY(download(ctx, a->w, w, bytes));
        NB_TRY(download(ctx, a->theta, th, bytes));
        NB_CUDA(ctx, cudaStreamSynchronize(st));
    }
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_eos_projection(nimbus_cuda_context* ctx, const nimbus_eos_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->p || !a->rho || !a->theta || a->nx < 1 || a->ny < 1 || a->nz < 1 ||
        !cells_fit(a->nx, a->ny, a->nz) || !finite_positive(a->gamma))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid EOS projection arguments");
    const bool moist = a->qv && a->qc && a->qr;
    if (!moist && (a->qv || a->qc || a->qr)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "qv, qc, qr come together");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
        return run_eos_device(ctx, st, a, a->p, a->rho, a->theta, a->qv, a->qc, a->qr, a->p0_base);
    }
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const size_t bytes = n * sizeof(float);
    float *p, *rho, *th, *qv = nullptr, *qc = nullptr, *qr = nullptr;
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kTheta, n, &th));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    NB_TRY(upload(ctx, th, a->theta, bytes));
    if (moist)
    {
        NB_TRY(ensure(ctx, kQv, n, &qv));
        NB_TRY(ensure(ctx, kQc, n, &qc));
        NB_TRY(ensure(ctx, kQr, n, &qr));
        NB_TRY(upload(ctx, qv, a->qv, bytes));
        NB_TRY(upload(ctx, qc, a->qc, bytes));
        NB_TRY(upload(ctx, qr, a->qr, bytes));
    }
    double* p0 = nullptr;
    if (a->p0_base)
    {
        NB_TRY(ensure(ctx, kP0, static_cast<size_t>(a->nz), &p0));
        NB_TRY(upload(ctx, p0, a->p0_base, sizeof(double) * static_cast<size_t>(a->nz)));
    }
    NB_TRY(run_eos_device(ctx, st, a, p, rho, th, qv, qc, qr, p0));
    unsigned flags = 0;
    NB_TRY(read_status(ctx, st, &flags));
    if (flags & kStatusInvalidEos)
        return fail(ctx, NIMBUS_ERR_NONFINITE, "EOS pressure projection rejected an invalid physical state");
    NB_TRY(download(ctx, a->p, p, bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_slow_apply(nimbus_cuda_context* ctx, const nimbus_slow_apply_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->u || !a->v || !a->w || !a->p || !a->du_dt || !a->dv_dt || !a->dw_dt || !a->dp_dt || a->nx < 1 ||
        a->ny < 1 || a->nz < 1 || !cells_fit(a->nx, a->ny, a->nz) || !std::isfinite(a->dt_large))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid slow apply arguments");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const int blocks = grid_for(ctx, static_cast<long long>(n));
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        cudaStream_t st = a->stream ? static_cast<cudaStream_t>(a->stream) : ctx->stream;
        slow_apply_kernel<<<blocks, kThreads, 0, st>>>(a->u, a->v, a->w, a->p, a->du_dt, a->dv_dt, a->dw_dt, a->dp_dt,
                                                       a->du_dt_pbl, a->dv_dt_pbl, static_cast<long long>(n),
                                                       a->dt_large, a->sanitize);
        NB_CUDA(ctx, cudaGetLastError());
        ctx->launches += 1;
        return NIMBUS_OK;
    }
    const size_t bytes = n * sizeof(float);
    float *u, *v, *w, *p, *t, *pbl = nullptr;
    NB_TRY(ensure(ctx, kU, n, &u));
    NB_TRY(ensure(ctx, kV, n, &v));
    NB_TRY(ensure(ctx, kW, n, &w));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kSlowK1, 4 * n, &t));
    if (a->du_dt_pbl || a->dv_dt_pbl) NB_TRY(ensure(ctx, kSlowStar, 2 * n, &pbl));
    NB_TRY(upload(ctx, u, a->u, bytes));
    NB_TRY(upload(ctx, v, a->v, bytes));
    NB_TRY(upload(ctx, w, a->w, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, t, a->du_dt, bytes));
    NB_TRY(upload(ctx, t + n, a->dv_dt, bytes));
    NB_TRY(upload(ctx, t + 2 * n, a->dw_dt, bytes));
    NB_TRY(upload(ctx, t + 3 * n, a->dp_dt, bytes));
    if (a->du_dt_pbl) NB_TRY(upload(ctx, pbl, a->du_dt_pbl, bytes));
    if (a->dv_dt_pbl) NB_TRY(upload(ctx, pbl + n, a->dv_dt_pbl, bytes));
    slow_apply_kernel<<<blocks, kThreads, 0, ctx->stream>>>(u, v, w, p, t, t + n, t + 2 * n, t + 3 * n,
                                                            a->du_dt_pbl ? pbl : nullptr,
                                                            a->dv_dt_pbl ? pbl + n : nullptr,
                                                            static_cast<long long>(n), a->dt_large, a->sanitize);
    NB_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    NB_TRY(download(ctx, a->u, u, bytes));
    NB_TRY(download(ctx, a->v, v, bytes));
    NB_TRY(download(ctx, a->w, w, bytes));
    NB_TRY(download(ctx, a->p, p, bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return NIMBUS_OK;
}

namespace
{
bool domain_ok(int nx, int ny, int nz, int i0, int i1, int j0, int j1, int k0, int k1)
{
    return 0 <= i0 && i0 <= i1 && i1 <= nx && 0 <= j0 && j0 <= j1 && j1 <= ny && 0 <= k0 && k0 <= k1 && k1 <= nz;
}
}  // namespace

nimbus_status nimbus_cuda_kessler_pointwise(nimbus_cuda_context* ctx, const nimbus_kessler_pointwise_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->temperature || !a->p || !a->qv || !a->qc || !a->qr || !a->rho_d || !a->dtheta_dt || !a->dqv_dt ||
        !a->dqc_dt || !a->dqr_dt || a->nx < 1 || a->ny < 1 || a->nz < 1 || !cells_fit(a->nx, a->ny, a->nz) ||
        !domain_ok(a->nx, a->ny, a->nz, a->i_begin, a->i_end, a->j_begin, a->j_end, a->k_begin, a->k_end))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid Kessler pointwise arguments");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    KesslerPointwiseParams P{a->nx, a->ny, a->nz, a->i_begin, a->i_end, a->j_begin, a->j_end, a->k_begin, a->k_end,
                             a->qc0, a->c_auto, a->c_accr, a->evaporation_efficiency, a->lv_cp, a->t0, a->dt_step};
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const int blocks = grid_for(ctx, static_cast<long long>(n));
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        cudaStream_t st = a->stream ? static_cast<cudaStream_t>(a->stream) : ctx->stream;
        kessler_pointwise_kernel<<<blocks, kThreads, 0, st>>>(P, a->temperature, a->p, a->qv, a->qc, a->qr, a->rho_d,
                                                              a->dtheta_dt, a->dqv_dt, a->dqc_dt, a->dqr_dt,
                                                              a->dqg_dt, a->dqh_dt);
        NB_CUDA(ctx, cudaGetLastError());
        ctx->launches += 1;
        return NIMBUS_OK;
    }
    const size_t bytes = n * sizeof(float);
    float *T, *p, *qv, *qc, *qr, *rho, *out;
    NB_TRY(ensure(ctx, kTheta, n, &T));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kQv, n, &qv));
    NB_TRY(ensure(ctx, kQc, n, &qc));
    NB_TRY(ensure(ctx, kQr, n, &qr));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kKesslerOut, 4 * n, &out));
    NB_TRY(upload(ctx, T, a->temperature, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, qv, a->qv, bytes));
    NB_TRY(upload(ctx, qc, a->qc, bytes));
    NB_TRY(upload(ctx, qr, a->qr, bytes));
    NB_TRY(upload(ctx, rho, a->rho_d, bytes));
    kessler_pointwise_kernel<<<blocks, kThreads, 0, ctx->stream>>>(P, T, p, qv, qc, qr, rho, out, out + n, out + 2 * n,
                                                                   out + 3 * n, nullptr, nullptr);
    NB_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    NB_TRY(download(ctx, a->dtheta_dt, out, bytes));
    NB_TRY(download(ctx, a->dqv_dt, out + n, bytes));
    NB_TRY(download(ctx, a->dqc_dt, out + 2 * n, bytes));
    NB_TRY(download(ctx, a->dqr_dt, out + 3 * n, bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (a->dqg_dt) std::memset(a->dqg_dt, 0, bytes);
    if (a->dqh_dt) std::memset(a->dqh_dt, 0, bytes);
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_kessler_sedimentation(nimbus_cuda_context* ctx, const nimbus_kessler_sedimentation_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->qr || !a->dqr_dt || a->nx < 1 || a->ny < 1 || a->nz < 1 || !cells_fit(a->nx, a->ny, a->nz) ||
        !domain_ok(a->nx, a->ny, a->nz, a->i_begin, a->i_end, a->j_begin, a->j_end, a->k_begin, a->k_end) ||
        (!a->layer_thickness_m && !(a->dz > 0.0f)))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid Kessler sedimentation arguments");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    KesslerSedimentationParams P{a->nx, a->ny, a->nz, a->i_begin, a->i_end, a->j_begin, a->j_end, a->k_begin,
                                 a->k_end, a->dz, a->vt_max_rain, a->vt_cap};
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const int blocks = grid_for(ctx, static_cast<long long>(n));
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        cudaStream_t st = a->stream ? static_cast<cudaStream_t>(a->stream) : ctx->stream;
        kessler_sedimentation_kernel<<<blocks, kThreads, 0, st>>>(P, a->qr, a->rho_d, a->layer_thickness_m,
                                                                  a->dqr_dt);
        NB_CUDA(ctx, cudaGetLastError());
        ctx->launches += 1;
        return NIMBUS_OK;
    }
    const size_t bytes = n * sizeof(float);
    float *qr, *dqr, *rho = nullptr, *layers = nullptr;
    NB_TRY(ensure(ctx, kQr, n, &qr));
    NB_TRY(ensure(ctx, kKesslerOut, 4 * n, &dqr));
    NB_TRY(upload(ctx, qr, a->qr, bytes));
    NB_TRY(upload(ctx, dqr, a->dqr_dt, bytes));
    if (a->rho_d)
    {
        NB_TRY(ensure(ctx, kRho, n, &rho));
        NB_TRY(upload(ctx, rho, a->rho_d, bytes));
    }
    if (a->layer_thickness_m)
    {
        layers = dqr + n;
        NB_TRY(upload(ctx, layers, a->layer_thickness_m, bytes));
    }
    kessler_sedimentation_kernel<<<blocks, kThreads, 0, ctx->stream>>>(P, qr, rho, layers, dqr);
    NB_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    NB_TRY(download(ctx, a->dqr_dt, dqr, bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_cgrid_slow_tendencies(nimbus_cuda_context* ctx, const nimbus_cgrid_slow_tendencies_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    const bool adv = a->du_advection_dt || a->dv_advection_dt || a->dw_advection_dt;
    const bool winds = a->wind0_base_len >= a->nz;
    if (!a->u || !a->v || !a->w || !a->rho || !a->p || !a->rho0_base || !a->du_dt || !a->dv_dt || !a->dw_dt ||
        !a->dp_dt || a->nx < 3 || a->ny < 3 || a->nz < 2 || !cells_fit(a->nx, a->ny, a->nz) ||
        a->rho0_base_len < a->nz || (a->has_moisture && (!a->qv || !a->qv0_base || a->qv0_base_len < a->nz)) ||
        (a->has_loading && !a->loading) || (winds && (!a->u0_base || !a->v0_base)) ||
        (adv && !(a->du_advection_dt && a->dv_advection_dt && a->dw_advection_dt)) || !(a->dx > 0.0f) ||
        !(a->dy > 0.0f) || !(a->dz > 0.0f))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid slow tendency arguments");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    SlowDispatchParams S{};
    S.d = Dims{a->nx, a->ny, a->nz};
    // The operator's FP32 constants, formed as it forms them.
    S.inv_dx = 1.0f / a->dx;
    S.inv_dy = 1.0f / a->dy;
    S.inv_dz = 1.0f / a->dz;
    S.inv_2dx = 0.5f / a->dx;
    S.inv_2dy = 0.5f / a->dy;
    S.inv_2dz = 0.5f / a->dz;
    const float inv[3] = {S.inv_dx, S.inv_dy, S.inv_dz};
    for (int q = 0; q < 3; ++q)
    {
        S.d6[q] = inv[q] / 6.0f;
        S.d60[q] = inv[q] / 60.0f;
    }
    S.dy = a->dy;
    S.g = a->g;
    S.f0 = a->coriolis_f;
    S.beta = a->coriolis_beta;
    S.frame_u = a->frame_velocity_u;
    S.frame_v = a->frame_velocity_v;
    S.has_moisture = a->has_moisture ? 1 : 0;
    S.has_loading = a->has_loading ? 1 : 0;
    S.wind_profiles = winds ? 1 : 0;
    S.emit_advection = adv ? 1 : 0;
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const int blocks = grid_for(ctx, static_cast<long long>(n));
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        cudaStream_t st = a->stream ? static_cast<cudaStream_t>(a->stream) : ctx->stream;
        slow_tendencies_dispatch_kernel<<<blocks, kThreads, 0, st>>>(
            S, a->u, a->v, a->w, a->rho, a->p, a->rho0_base, a->qv0_base, a->u0_base, a->v0_base, a->qv, a->loading,
            a->du_dt, a->dv_dt, a->dw_dt, a->drho_dt, a->dp_dt, a->du_advection_dt, a->dv_advection_dt,
            a->dw_advection_dt);
        NB_CUDA(ctx, cudaGetLastError());
        ctx->launches += 1;
        return NIMBUS_OK;
    }
    const size_t bytes = n * sizeof(float);
    const size_t nzb = static_cast<size_t>(a->nz) * sizeof(float);
    float *u, *v, *w, *rho, *p, *prof, *qv = nullptr, *load = nullptr, *out, *advo = nullptr;
    NB_TRY(ensure(ctx, kU, n, &u));
    NB_TRY(ensure(ctx, kV, n, &v));
    NB_TRY(ensure(ctx, kW, n, &w));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kRelaxTables, 4 * static_cast<size_t>(a->nz), &prof));
    NB_TRY(ensure(ctx, kSlowK1, 4 * n, &out));
    NB_TRY(upload(ctx, u, a->u, bytes));
    NB_TRY(upload(ctx, v, a->v, bytes));
    NB_TRY(upload(ctx, w, a->w, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, prof, a->rho0_base, nzb));
    if (a->has_moisture)
    {
        NB_TRY(ensure(ctx, kQv, n, &qv));
        NB_TRY(upload(ctx, qv, a->qv, bytes));
        NB_TRY(upload(ctx, prof + a->nz, a->qv0_base, nzb));
    }
    if (winds)
    {
        NB_TRY(upload(ctx, prof + 2 * static_cast<size_t>(a->nz), a->u0_base, nzb));
        NB_TRY(upload(ctx, prof + 3 * static_cast<size_t>(a->nz), a->v0_base, nzb));
    }
    if (a->has_loading)
    {
        NB_TRY(ensure(ctx, kQc, n, &load));
        NB_TRY(upload(ctx, load, a->loading, bytes));
    }
    if (adv) NB_TRY(ensure(ctx, kSlowStar, 3 * n, &advo));
    slow_tendencies_dispatch_kernel<<<blocks, kThreads, 0, ctx->stream>>>(
        S, u, v, w, rho, p, prof, prof + a->nz, prof + 2 * static_cast<size_t>(a->nz),
        prof + 3 * static_cast<size_t>(a->nz), qv, load, out, out + n, out + 2 * n, nullptr, out + 3 * n,
        adv ? advo : nullptr, adv ? advo + n : nullptr, adv ? advo + 2 * n : nullptr);
    NB_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    NB_TRY(download(ctx, a->du_dt, out, bytes));
    NB_TRY(download(ctx, a->dv_dt, out + n, bytes));
    NB_TRY(download(ctx, a->dw_dt, out + 2 * n, bytes));
    NB_TRY(download(ctx, a->dp_dt, out + 3 * n, bytes));
    if (adv)
    {
        NB_TRY(download(ctx, a->du_advection_dt, advo, bytes));
        NB_TRY(download(ctx, a->dv_advection_dt, advo + n, bytes));
        NB_TRY(download(ctx, a->dw_advection_dt, advo + 2 * n, bytes));
    }
    NB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
    if (a->drho_dt) std::memset(a->drho_dt, 0, bytes);
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_max_sound_speed(nimbus_cuda_context* ctx, nimbus_sound_speed_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (!a->p || !a->rho || a->nx < 1 || a->ny < 1 || a->nz < 1 || !cells_fit(a->nx, a->ny, a->nz))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "invalid sound speed scan arguments");
    if ((a->p0_base == nullptr) != (a->rho0_base == nullptr))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "p0_base and rho0_base come together");
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const float* p = a->p;
    const float* rho = a->rho;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
    }
    else
    {
        float *dp, *drho;
        NB_TRY(ensure(ctx, kP, n, &dp));
        NB_TRY(ensure(ctx, kRho, n, &drho));
        NB_TRY(upload(ctx, dp, a->p, n * sizeof(float)));
        NB_TRY(upload(ctx, drho, a->rho, n * sizeof(float)));
        if (st != ctx->stream) NB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
        p = dp;
        rho = drho;
    }
    // Its own result slot and flag word: the context's status word keeps the
    // flags of work enqueued before this call for nimbus_cuda_synchronize.
    unsigned long long* slot = nullptr;
    NB_TRY(ensure(ctx, kSoundSpeed, 2, &slot));
    NB_CUDA(ctx, cudaMemsetAsync(slot, 0, 2 * sizeof(unsigned long long), st));
    const double gamma = kCpd / (kCpd - kRd);
    max_sound_speed_kernel<<<grid_for(ctx, static_cast<long long>(n)), kThreads, 0, st>>>(
        p, rho, static_cast<long long>(n), gamma, slot, reinterpret_cast<unsigned*>(slot + 1));
    NB_CUDA(ctx, cudaGetLastError());
    ctx->launches += 1;
    unsigned long long result[2] = {0, 0};
    NB_CUDA(ctx, cudaMemcpyAsync(result, slot, sizeof result, cudaMemcpyDeviceToHost, st));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    const unsigned long long bits = result[0];
    const unsigned flags = static_cast<unsigned>(result[1]);
    if (flags & kStatusInvalidState)
        return fail(ctx, NIMBUS_ERR_NONFINITE, "CFL scan requires finite wind and positive finite pressure/density");
    double c = std::sqrt(ordered_bits_to_double(bits));
    if (a->p0_base) c = std::max(c, base_sound_speed(a->p0_base, a->rho0_base, a->nz, gamma));
    a->max_sound_speed = c;
    return NIMBUS_OK;
}

int nimbus_cuda_resolve_substep_count(double dt_large, double max_sound_speed, double min_spacing, int requested)
{
    return resolve_substep_count(dt_large, max_sound_speed, min_spacing, requested);
}

nimbus_status nimbus_cuda_set_precision(nimbus_cuda_context* ctx, int precision)
{
    if (!ctx) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (precision != NIMBUS_PRECISION_REFERENCE && precision != NIMBUS_PRECISION_FP32)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown precision");
    ctx->precision = precision;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_set_substep_form(nimbus_cuda_context* ctx, int form)
{
    if (!ctx) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (form != NIMBUS_SUBSTEP_AUTO && form != NIMBUS_SUBSTEP_FUSED && form != NIMBUS_SUBSTEP_SPLIT)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown substep form");
    ctx->substep_form = form;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_autotune_substep(nimbus_cuda_context* ctx, int nx, int ny, int nz, int* chosen_form,
                                           double* ms_per_substep)
{
    if (!ctx) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (nx < 3 || ny < 3 || nz < 2 || !cells_fit(nx, ny, nz)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "bad shape");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = static_cast<size_t>(nx) * ny * nz;
    // Scratch state: a resting isothermal column is enough to exercise every
    // instruction path the timing depends on.
    float* buf = nullptr;
    double* prof = nullptr;
    float2* dp0 = nullptr;
    float4* eos0 = nullptr;
    NB_CUDA(ctx, cudaMalloc(&buf, sizeof(float) * n * 13));
    if (cudaMalloc(&prof, sizeof(double) * 2 * nz) != cudaSuccess || cudaMalloc(&dp0, sizeof(float2) * nz) != cudaSuccess ||
        cudaMalloc(&eos0, sizeof(float4) * nz) != cudaSuccess)
    {
        cudaFree(buf);
        if (prof) cudaFree(prof);
        if (dp0) cudaFree(dp0);
        return fail(ctx, NIMBUS_ERR_OUT_OF_MEMORY, "autotune scratch");
    }
    cudaStream_t st = ctx->stream;
    Prognostic a{buf, buf + n, buf + 2 * n, buf + 3 * n};
    Prognostic b{buf + 4 * n, buf + 5 * n, buf + 6 * n, buf + 7 * n};
    float* p = buf + 8 * n;
    float* theta = buf + 9 * n;
    float* mf = buf + 10 * n;
    fill_tuning_state<<<grid_for(ctx, static_cast<long long>(n)), kThreads, 0, st>>>(buf, n, prof, nz, dp0);
    FusedParams F = fused_params(ctx, nx, ny, nz, 250.0, 250.0, 250.0, 0.1, 1004.0 / 717.0, 0.05f, 2.0f, 1000.0f,
                                 200000.0f, 100000.0f, 180.0f, 120.0f);
    F.weight = 0.1;
    finish_fp32(F);
    level_base_kernel<<<(nz + 127) / 128, 128, 0, st>>>(prof + nz, nz, F.gamma, dp0, eos0);
    const int saved_form = ctx->substep_form;
    const bool saved_timing = ctx->timing;
    ctx->timing = false;
    int best = NIMBUS_SUBSTEP_SPLIT;
    double best_ms = 1e30;
    nimbus_status rc = NIMBUS_OK;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int form : {NIMBUS_SUBSTEP_SPLIT, NIMBUS_SUBSTEP_FUSED})
    {
        ctx->substep_form = form;
        const int reps = 6;
        for (int w = 0; w < 2 + reps && rc == NIMBUS_OK; ++w)
        {
            if (w == 2) cudaEventRecord(e0, st);
            rc = launch_fused(ctx, st, F, (w & 1) ? b : a, (w & 1) ? a : b, p, theta, prof, prof + nz, dp0, eos0,
                              nullptr, mf, mf + n, mf + 2 * n);
        }
        cudaEventRecord(e1, st);
        if (rc != NIMBUS_OK) break;
        if (cudaEventSynchronize(e1) != cudaSuccess) { rc = cuda_fail(ctx, cudaGetLastError(), "autotune"); break; }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double per = ms / reps;
        if (per < best_ms)
        {
            best_ms = per;
            best = form;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), st);
    cudaStreamSynchronize(st);
    cudaFree(buf);
    cudaFree(prof);
    cudaFree(dp0);
    cudaFree(eos0);
    ctx->substep_form = saved_form;
    ctx->timing = saved_timing;
    if (rc != NIMBUS_OK) return rc;
    bool found = false;
    for (auto& e : ctx->tuned)
        if (e.nx == nx && e.ny == ny && e.nz == nz && e.precision == ctx->precision)
        {
            e.form = best;
            found = true;
        }
    if (!found) ctx->tuned.push_back({nx, ny, nz, ctx->precision, best});
    if (chosen_form) *chosen_form = best;
    if (ms_per_substep) *ms_per_substep = best_ms;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_set_kernel_timing(nimbus_cuda_context* ctx, int enable)
{
    if (!ctx) return NIMBUS_ERR_INVALID_ARGUMENT;
    drain_timing(ctx);
    ctx->timing = enable != 0;
    for (int f = 0; f < NIMBUS_KERNEL_FAMILIES; ++f)
    {
        ctx->timed_launches[f] = 0;
        ctx->timed_ms[f] = 0.0;
    }
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_kernel_timing(nimbus_cuda_context* ctx, int family, uint64_t* launches, double* total_ms)
{
    if (!ctx || family < 0 || family >= NIMBUS_KERNEL_FAMILIES || !launches || !total_ms)
        return NIMBUS_ERR_INVALID_ARGUMENT;
    drain_timing(ctx);
    *launches = ctx->timed_launches[family];
    *total_ms = ctx->timed_ms[family];
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_acoustic_fused(nimbus_cuda_context* ctx, const nimbus_acoustic_fused_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (const char* why = check_acoustic_common(a->u, a->v, a->w, a->rho, a->p, a->theta, a->rho0_base, a->p0_base,
                                                a->base_len, a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small,
                                                a->gamma, a->rho_min, a->rho_max, a->p_min, a->p_max,
                                                a->p_ref_fallback, a->wind_clamp_h, a->wind_clamp_v))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const size_t bytes = n * sizeof(float);
    const AcousticParams P = acoustic_params(a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small, a->gamma,
                                             a->rho_min, a->rho_max, a->p_min, a->p_max, a->p_ref_fallback,
                                             a->wind_clamp_h, a->wind_clamp_v);
    AcousticDevice D{};
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
        D = {a->u, a->v, a->w, a->rho, a->p, a->theta, a->rho0_base, a->p0_base, nullptr, a->drho_scratch};
        NB_TRY(ensure_alts(ctx, n, D));
        return run_fused_device(ctx, st, a, D);
    }
    float *u, *v, *w, *rho, *p, *theta, *alt, *drho = nullptr;
    double *rho0, *p0;
    NB_TRY(ensure(ctx, kU, n, &u));
    NB_TRY(ensure(ctx, kV, n, &v));
    NB_TRY(ensure(ctx, kW, n, &w));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kTheta, n, &theta));
    NB_TRY(ensure(ctx, kRhoAlt, n, &alt));
    NB_TRY(ensure(ctx, kRho0, static_cast<size_t>(a->nz), &rho0));
    NB_TRY(ensure(ctx, kP0, static_cast<size_t>(a->nz), &p0));
    if (a->drho_scratch) NB_TRY(ensure(ctx, kDrho, n, &drho));
    NB_TRY(upload(ctx, u, a->u, bytes));
    NB_TRY(upload(ctx, v, a->v, bytes));
    NB_TRY(upload(ctx, w, a->w, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, theta, a->theta, bytes));
    NB_TRY(upload(ctx, rho0, a->rho0_base, sizeof(double) * a->nz));
    NB_TRY(upload(ctx, p0, a->p0_base, sizeof(double) * a->nz));
    D = {u, v, w, rho, p, theta, rho0, p0, alt, drho};
    NB_TRY(ensure_alts(ctx, n, D));
    NB_TRY(run_fused_device(ctx, st, a, D));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    NB_TRY(download(ctx, a->u, u, bytes));
    NB_TRY(download(ctx, a->v, v, bytes));
    NB_TRY(download(ctx, a->w, w, bytes));
    NB_TRY(download(ctx, a->rho, rho, bytes));
    NB_TRY(download(ctx, a->p, p, bytes));
    if (drho) NB_TRY(download(ctx, a->drho_scratch, drho, bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_acoustic_batched(nimbus_cuda_context* ctx, const nimbus_acoustic_batched_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (const char* why = check_batched(a)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = static_cast<size_t>(a->nx) * a->ny * a->nz;
    const size_t bytes = n * sizeof(float);
    const size_t waves = 2 * (static_cast<size_t>(a->nx) + a->ny) * a->nz;
    const bool mf = a->accumulate_mass_flux != 0;
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
        AcousticDevice D{a->u, a->v, a->w, a->rho, a->p, a->theta, a->rho0_base, a->p0_base, nullptr, nullptr,
                         mf ? a->mass_flux_x : nullptr, mf ? a->mass_flux_y : nullptr, mf ? a->mass_flux_z : nullptr};
        NB_TRY(ensure_alts(ctx, n, D));
        return run_batched_device(ctx, st, a, D, a->wave_history_output, a->wave_history, a->density_begin);
    }
    float *u, *v, *w, *rho, *p, *theta, *alt, *wave, *rb = nullptr, *mx = nullptr, *my = nullptr, *mz = nullptr;
    double *rho0, *p0;
    NB_TRY(ensure(ctx, kU, n, &u));
    NB_TRY(ensure(ctx, kV, n, &v));
    NB_TRY(ensure(ctx, kW, n, &w));
    NB_TRY(ensure(ctx, kRho, n, &rho));
    NB_TRY(ensure(ctx, kP, n, &p));
    NB_TRY(ensure(ctx, kTheta, n, &theta));
    NB_TRY(ensure(ctx, kRhoAlt, n, &alt));
    NB_TRY(ensure(ctx, kWave, waves, &wave));
    NB_TRY(ensure(ctx, kRho0, static_cast<size_t>(a->nz), &rho0));
    NB_TRY(ensure(ctx, kP0, static_cast<size_t>(a->nz), &p0));
    if (a->density_begin) NB_TRY(ensure(ctx, kRhoBegin, n, &rb));
    if (mf)
    {
        NB_TRY(ensure(ctx, kMfx, n, &mx));
        NB_TRY(ensure(ctx, kMfy, n, &my));
        NB_TRY(ensure(ctx, kMfz, n, &mz));
        NB_TRY(upload(ctx, mx, a->mass_flux_x, bytes));
        NB_TRY(upload(ctx, my, a->mass_flux_y, bytes));
        NB_TRY(upload(ctx, mz, a->mass_flux_z, bytes));
    }
    NB_TRY(upload(ctx, u, a->u, bytes));
    NB_TRY(upload(ctx, v, a->v, bytes));
    NB_TRY(upload(ctx, w, a->w, bytes));
    NB_TRY(upload(ctx, rho, a->rho, bytes));
    NB_TRY(upload(ctx, p, a->p, bytes));
    NB_TRY(upload(ctx, theta, a->theta, bytes));
    NB_TRY(upload(ctx, rho0, a->rho0_base, sizeof(double) * a->nz));
    NB_TRY(upload(ctx, p0, a->p0_base, sizeof(double) * a->nz));
    if (a->wave_history) NB_TRY(upload(ctx, wave, a->wave_history, sizeof(float) * waves));
    AcousticDevice D{u, v, w, rho, p, theta, rho0, p0, alt, nullptr, mx, my, mz};
    NB_TRY(ensure_alts(ctx, n, D));
    NB_TRY(run_batched_device(ctx, st, a, D, wave, a->wave_history ? wave : nullptr, rb));
    unsigned flags = 0;
    NB_TRY(read_status(ctx, st, &flags));
    if (flags & kStatusNonfiniteMassFlux)
        return fail(ctx, NIMBUS_ERR_NONFINITE, "non-finite retained face mass flux; host fields left untouched");
    NB_TRY(download(ctx, a->u, u, bytes));
    NB_TRY(download(ctx, a->v, v, bytes));
    NB_TRY(download(ctx, a->w, w, bytes));
    NB_TRY(download(ctx, a->rho, rho, bytes));
    NB_TRY(download(ctx, a->p, p, bytes));
    NB_TRY(download(ctx, a->wave_history_output, wave, sizeof(float) * waves));
    if (rb) NB_TRY(download(ctx, a->density_begin, rb, bytes));
    if (mf)
    {
        NB_TRY(download(ctx, a->mass_flux_x, mx, bytes));
        NB_TRY(download(ctx, a->mass_flux_y, my, bytes));
        NB_TRY(download(ctx, a->mass_flux_z, mz, bytes));
    }
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_scalar_transport(nimbus_cuda_context* ctx, const nimbus_scalar_transport_args* a)
{
    if (!ctx || !a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (const char* why = check_transport(a)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (a->n_scalars == 0) return NIMBUS_OK;
    if (a->memory != NIMBUS_MEMORY_HOST && a->memory != NIMBUS_MEMORY_DEVICE)
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown memory kind");
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    TransportParams T = transport_params(a);
    const size_t n = static_cast<size_t>(T.d.cells());
    const size_t bytes = n * sizeof(float);
    cudaStream_t st = ctx->stream;
    if (a->memory == NIMBUS_MEMORY_DEVICE)
    {
        if (a->stream) st = static_cast<cudaStream_t>(a->stream);
        for (int s = 0; s < a->n_scalars; ++s)
        {
            T.q_in[s] = a->q_in[s];
            T.q_out[s] = a->q_out[s];
        }
        return run_transport_device(ctx, st, T, a->rho_end, a->rho_begin, a->mass_flux_x, a->mass_flux_y,
                                    a->mass_flux_z);
    }
    float *re, *rb, *mx, *my, *mz;
    NB_TRY(ensure(ctx, kRhoEnd, n, &re));
    NB_TRY(ensure(ctx, kRhoBegin, n, &rb));
    NB_TRY(ensure(ctx, kMfx, n, &mx));
    NB_TRY(ensure(ctx, kMfy, n, &my));
    NB_TRY(ensure(ctx, kMfz, n, &mz));
    NB_TRY(upload(ctx, re, a->rho_end, bytes));
    NB_TRY(upload(ctx, rb, a->rho_begin, bytes));
    NB_TRY(upload(ctx, mx, a->mass_flux_x, bytes));
    NB_TRY(upload(ctx, my, a->mass_flux_y, bytes));
    NB_TRY(upload(ctx, mz, a->mass_flux_z, bytes));
    for (int s = 0; s < a->n_scalars; ++s)
    {
        float *qi, *qo;
        NB_TRY(ensure(ctx, static_cast<Slot>(kQ0 + 2 * s), n, &qi));
        NB_TRY(ensure(ctx, static_cast<Slot>(kQ0 + 2 * s + 1), n, &qo));
        NB_TRY(upload(ctx, qi, a->q_in[s], bytes));
        T.q_in[s] = qi;
        T.q_out[s] = qo;
    }
    NB_TRY(run_transport_device(ctx, st, T, re, rb, mx, my, mz));
    unsigned flags = 0;
    NB_TRY(read_status(ctx, st, &flags));
    if (flags & kStatusNonfiniteTransport)
        return fail(ctx, NIMBUS_ERR_NONFINITE, "non-finite transported scalar; host fields left untouched");
    for (int s = 0; s < a->n_scalars; ++s) NB_TRY(download(ctx, a->q_out[s], T.q_out[s], bytes));
    NB_CUDA(ctx, cudaStreamSynchronize(st));
    return NIMBUS_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// Fused acoustic substep with static scratch: no device allocation at all.
// ---------------------------------------------------------------------------
namespace
{

constexpr int kStaticScratchMaxDevices = 64;

// The density ping-pong partner for nimbus_cuda_acoustic_fused_static_scratch.
// Host code must not pass this symbol to a kernel: on the host it names a
// stand-in, not the device address, which is resolved per device below.
static __device__ __align__(256) float g_static_rho_scratch[NIMBUS_STATIC_SCRATCH_CELLS];

std::mutex g_static_scratch_mutex;
float* g_static_scratch_ptr[kStaticScratchMaxDevices] = {};
int g_static_scratch_sms[kStaticScratchMaxDevices] = {};

}  // namespace

extern "C" nimbus_status nimbus_cuda_acoustic_fused_static_scratch(const nimbus_acoustic_fused_args* a)
{
    if (!a) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (a->memory != NIMBUS_MEMORY_DEVICE) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (check_acoustic_common(a->u, a->v, a->w, a->rho, a->p, a->theta, a->rho0_base, a->p0_base, a->base_len,
                              a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small, a->gamma, a->rho_min,
                              a->rho_max, a->p_min, a->p_max, a->p_ref_fallback, a->wind_clamp_h,
                              a->wind_clamp_v) != nullptr)
        return NIMBUS_ERR_INVALID_ARGUMENT;
    const long long cells = static_cast<long long>(a->nx) * a->ny * a->nz;
    if (cells > NIMBUS_STATIC_SCRATCH_CELLS) return NIMBUS_ERR_TOO_LARGE;

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return NIMBUS_ERR_CUDA;
    if (dev < 0 || dev >= kStaticScratchMaxDevices) return NIMBUS_ERR_UNSUPPORTED;
    float* scratch = nullptr;
    int sms = 0;
    {
        std::lock_guard<std::mutex> lock(g_static_scratch_mutex);
        if (!g_static_scratch_ptr[dev])
        {
            // Set-up, once per device, with that device current.  A failed
            // set-up clears the error it raised, so that a later call of any
            // entry point does not report it as its own.
            void* ptr = nullptr;
            if (cudaGetSymbolAddress(&ptr, g_static_rho_scratch) != cudaSuccess || ptr == nullptr)
            {
                (void)cudaGetLastError();
                return NIMBUS_ERR_CUDA;
            }
            int count = 0;
            if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || count <= 0)
            {
                (void)cudaGetLastError();
                return NIMBUS_ERR_CUDA;
            }
            g_static_scratch_ptr[dev] = static_cast<float*>(ptr);
            g_static_scratch_sms[dev] = count;
        }
        scratch = g_static_scratch_ptr[dev];
        sms = g_static_scratch_sms[dev];
    }

    const AcousticParams P = acoustic_params(a->nx, a->ny, a->nz, a->dx, a->dy, a->dz, a->dt_small, a->gamma,
                                             a->rho_min, a->rho_max, a->p_min, a->p_max, a->p_ref_fallback,
                                             a->wind_clamp_h, a->wind_clamp_v);
    cudaStream_t st = static_cast<cudaStream_t>(a->stream);
    long long blocks = (cells + kThreads - 1) / kThreads;
    if (blocks > static_cast<long long>(sms) * 16) blocks = static_cast<long long>(sms) * 16;
    // An error left by earlier, unrelated work of the process is not this
    // call's failure: drop it before the first launch, then check each step.
    (void)cudaGetLastError();
    acoustic_continuity_eos_kernel<<<static_cast<int>(blocks), kThreads, 0, st>>>(
        P, a->rho, a->u, a->v, a->w, a->theta, a->rho0_base, scratch, a->p, a->drho_scratch, nullptr, nullptr,
        nullptr, nullptr);
    if (cudaGetLastError() != cudaSuccess) return NIMBUS_ERR_CUDA;
    acoustic_momentum_kernel<<<static_cast<int>(blocks), kThreads, 0, st>>>(P, scratch, a->p, a->p0_base, a->u,
                                                                             a->v, a->w);
    if (cudaGetLastError() != cudaSuccess) return NIMBUS_ERR_CUDA;
    // A failure from here on leaves p, u, v, w already advanced while rho
    // keeps its old values (the new density is still in the scratch array).
    if (cudaMemcpyAsync(a->rho, scratch, sizeof(float) * static_cast<size_t>(cells), cudaMemcpyDeviceToDevice, st) !=
        cudaSuccess)
        return NIMBUS_ERR_CUDA;
    return NIMBUS_OK;
}
