// Host-side launch sequences shared by the backend's translation units.
//
// The kernels of the two precision forms are instantiated in different
// translation units: the reference-precision ones in files compiled with
// --fmad=false (no contracted multiply-add, bit-exact to the CPU solver), the
// FP32 ones in fp32_kernels.cu, compiled with contraction on (the FP32 form
// has no bit-exactness contract, and a fused multiply-add is one instruction
// and one rounding instead of two).  The templates below are in an unnamed
// namespace so each translation unit owns its instantiations.
#pragma once

#include "context.cuh"
#include "acoustic_fused.cuh"
#include "acoustic_split.cuh"
#include "slow_kernels.cuh"
#include "transport_kernels.cuh"

struct nimbus_engine;

namespace nimbus_host
{

// The four prognostic fields an acoustic substep rewrites (one buffer set).
struct Prognostic
{
    float *u, *v, *w, *rho;
};

// Device pointers of one slow-step call.
struct SlowDevice
{
    float *u, *v, *w, *p;
    const float *rho, *qv, *qc, *qr;
    const double *rho0, *qv0, *u0, *v0;
    float *du, *dv, *dw, *dp;
};

}  // namespace nimbus_host

namespace
{

using namespace nimbus;
using namespace nimbus_host;

// Fused one-launch substep: reads (u,v,w,rho)[cur], writes (u,v,w,rho)[alt],
// p in place, mass fluxes in place.
constexpr int kFusedTJ = 8;
constexpr int kFusedBlock = 256;


bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

template <class Policy>
nimbus_status launch_fused_impl(nimbus_cuda_context* ctx, cudaStream_t st, FusedParams F, const Prognostic& in,
                                const Prognostic& out, float* p, const float* theta, const double* rho0,
                                const double* p0, const float2* dp0, const float4* eos0, float* drho, float* mfx,
                                float* mfy, float* mfz)
{
    const size_t smem = FusedSmem<kFusedTJ>::floats(F.d.nz) * sizeof(float);
    auto kernel = acoustic_substep_fused_kernel<kFusedTJ, kFusedBlock, Policy>;
    if (smem > 220 * 1024) return fail(ctx, NIMBUS_ERR_UNSUPPORTED, "nz too large for the fused substep's shared window");
    static int occupancy_cache[2][512] = {};
    const int pol = Policy::exact_pow ? 0 : 1;
    int& occ = occupancy_cache[pol][F.d.nz < 512 ? F.d.nz : 511];
    if (occ == 0)
    {
        NB_CUDA(ctx, cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 220 * 1024));
        int blocks = 0;
        NB_CUDA(ctx, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kFusedBlock, smem));
        occ = blocks > 0 ? blocks : 1;
    }
    // Chunk the i-march so the grid is about one full wave of resident CTAs
    // (each chunk recomputes one plane, so longer chunks waste less).
    const int strips = (F.d.ny + kFusedTJ - 1) / kFusedTJ;
    const int resident = ctx->sm_count * occ;
    int chunks = resident / strips;
    if (chunks < 1) chunks = 1;
    if (chunks > F.d.nx) chunks = F.d.nx;
    F.chunk = (F.d.nx + chunks - 1) / chunks;
    chunks = (F.d.nx + F.chunk - 1) / F.chunk;
    F.nz_magic = fused_nz_magic(static_cast<unsigned>(F.d.nz));
    F.vec4 = (F.d.nz % 4 == 0) && aligned16(in.rho) && aligned16(in.u) && aligned16(in.v) && aligned16(in.w) &&
             aligned16(theta);
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_ACOUSTIC_SUBSTEP);
    kernel<<<strips * chunks, kFusedBlock, smem, st>>>(F, in.rho, in.u, in.v, in.w, theta, rho0, p0, dp0, eos0, drho,
                                                       out.rho, p, out.u, out.v, out.w, mfx, mfy, mfz, ctx->status);
    ctx->launches += 1;
    return NIMBUS_OK;
}

template <class Policy>
nimbus_status launch_split_impl(nimbus_cuda_context* ctx, cudaStream_t st, FusedParams F, const Prognostic& in,
                                const Prognostic& out, float* p, const float* theta, const double* rho0,
                                const double* p0, const float2* dp0, const float4* eos0, float* drho, float* mfx,
                                float* mfy, float* mfz)
{
    const long long n = F.d.cells();
    long long blocks = (n + kThreads - 1) / kThreads;
    const long long cap = static_cast<long long>(ctx->sm_count) * 32;
    if (blocks > cap) blocks = cap;
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_ACOUSTIC_SUBSTEP);
        split_continuity_eos_kernel<Policy><<<static_cast<int>(blocks), kThreads, 0, st>>>(
            F, in.rho, in.u, in.v, in.w, theta, rho0, eos0, out.rho, p, drho, mfx, mfy, mfz, ctx->status);
    }
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_ACOUSTIC_MOMENTUM);
        split_momentum_kernel<Policy><<<static_cast<int>(blocks), kThreads, 0, st>>>(F, out.rho, p, p0, dp0, in.u,
                                                                                      in.v, in.w, out.u, out.v, out.w);
    }
    ctx->launches += 2;
    return NIMBUS_OK;
}


template <class Policy>
nimbus_status run_slow_device(nimbus_cuda_context* ctx, cudaStream_t st, const SlowParams& S, const SlowDevice& D,
                              bool step)
{
    const size_t n = static_cast<size_t>(S.d.cells());
    const int blocks = grid_for(ctx, static_cast<long long>(n));
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_SLOW);
    if (!step)
    {
        slow_predict_kernel<Policy><<<blocks, kThreads, 0, st>>>(S, D.u, D.v, D.w, D.rho, D.p, D.qv, D.qc, D.qr, D.rho0,
                                                                 D.qv0, D.u0, D.v0, D.du, D.dv, D.dw, D.dp, nullptr,
                                                                 nullptr, nullptr, nullptr);
        ctx->launches += 1;
        NB_CUDA(ctx, cudaGetLastError());
        return NIMBUS_OK;
    }
    float *k1 = nullptr, *xs = nullptr;
    NB_TRY(ensure(ctx, kSlowK1, 4 * n, &k1));
    NB_TRY(ensure(ctx, kSlowStar, 4 * n, &xs));
    slow_predict_kernel<Policy><<<blocks, kThreads, 0, st>>>(S, D.u, D.v, D.w, D.rho, D.p, D.qv, D.qc, D.qr, D.rho0,
                                                             D.qv0, D.u0, D.v0, k1, k1 + n, k1 + 2 * n, k1 + 3 * n, xs,
                                                             xs + n, xs + 2 * n, xs + 3 * n);
    slow_correct_kernel<Policy><<<blocks, kThreads, 0, st>>>(S, xs, xs + n, xs + 2 * n, D.rho, xs + 3 * n, D.qv, D.qc,
                                                             D.qr, D.rho0, D.qv0, D.u0, D.v0, k1, k1 + n, k1 + 2 * n,
                                                             k1 + 3 * n, D.u, D.v, D.w, D.p, D.du, D.dv, D.dw, D.dp);
    ctx->launches += 2;
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

// The three transport passes for the scalars of T (one thread per cell, every
// scalar of the cell).
template <bool kFp32>
nimbus_status launch_transport_impl(nimbus_cuda_context* ctx, cudaStream_t st, const TransportParams& T,
                                    const float* rho_end, const float* rho_begin, const float* mfx, const float* mfy,
                                    const float* mfz, float* sf, float* rl)
{
    const dim3 grid(grid_for(ctx, T.d.cells()));
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_TRANSPORT_FACES);
        transport_faces_kernel<kFp32><<<grid, kThreads, 0, st>>>(T, mfx, mfy, mfz, sf);
    }
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_TRANSPORT_LIMITER);
        transport_limiter_kernel<kFp32><<<grid, kThreads, 0, st>>>(T, rho_begin, sf, rl);
    }
    {
        LaunchTimer t(ctx, st, NIMBUS_KERNEL_TRANSPORT_UPDATE);
        transport_update_kernel<kFp32><<<grid, kThreads, 0, st>>>(T, rho_end, rho_begin, sf, rl, ctx->status);
    }
    ctx->launches += 3;
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

}  // namespace

// FP32-form launches, defined in fp32_kernels.cu.
namespace nimbus_fp32
{
nimbus_status launch_fused(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::FusedParams& F,
                           const nimbus_host::Prognostic& in, const nimbus_host::Prognostic& out, float* p,
                           const float* theta,
                           const double* rho0, const double* p0, const float2* dp0, const float4* eos0, float* drho,
                           float* mfx, float* mfy, float* mfz);
nimbus_status launch_split(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::FusedParams& F,
                           const nimbus_host::Prognostic& in, const nimbus_host::Prognostic& out, float* p,
                           const float* theta,
                           const double* rho0, const double* p0, const float2* dp0, const float4* eos0, float* drho,
                           float* mfx, float* mfy, float* mfz);
nimbus_status run_slow(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::SlowParams& S,
                       const nimbus_host::SlowDevice& D, bool step);
nimbus_status launch_transport(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::TransportParams& T,
                               const float* rho_end, const float* rho_begin, const float* mfx, const float* mfy,
                               const float* mfz, float* sf, float* rl);
// Part `part` of one large step of every engine member of a lane (FP32 form);
// returns the launch count.
int engine_enqueue(nimbus_engine* e, int lane, cudaStream_t st, int part);
}  // namespace nimbus_fp32
