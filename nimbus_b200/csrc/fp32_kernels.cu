// FP32-form launches of the per-operation entry points and of the member
// engine.  This translation unit is compiled with --fmad=true: the FP32 form
// has no bit-exactness contract, and a contracted multiply-add is one
// instruction and one rounding.  The reference-precision instantiations of the
// same kernel templates live in the --fmad=false units.
#include "launch.cuh"
#include "engine_internal.cuh"

namespace nimbus_fp32
{

nimbus_status launch_fused(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::FusedParams& F,
                           const nimbus_host::Prognostic& in, const nimbus_host::Prognostic& out, float* p,
                           const float* theta, const double* rho0, const double* p0, const float2* dp0,
                           const float4* eos0, float* drho, float* mfx, float* mfy, float* mfz)
{
    return launch_fused_impl<nimbus::Fp32Policy>(ctx, st, F, in, out, p, theta, rho0, p0, dp0, eos0, drho, mfx, mfy,
                                                 mfz);
}

nimbus_status launch_split(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::FusedParams& F,
                           const nimbus_host::Prognostic& in, const nimbus_host::Prognostic& out, float* p,
                           const float* theta, const double* rho0, const double* p0, const float2* dp0,
                           const float4* eos0, float* drho, float* mfx, float* mfy, float* mfz)
{
    return launch_split_impl<nimbus::Fp32Policy>(ctx, st, F, in, out, p, theta, rho0, p0, dp0, eos0, drho, mfx, mfy,
                                                 mfz);
}

nimbus_status run_slow(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::SlowParams& S,
                       const nimbus_host::SlowDevice& D, bool step)
{
    return run_slow_device<nimbus::Fp32Policy>(ctx, st, S, D, step);
}

nimbus_status launch_transport(nimbus_cuda_context* ctx, cudaStream_t st, const nimbus::TransportParams& T,
                               const float* rho_end, const float* rho_begin, const float* mfx, const float* mfy,
                               const float* mfz, float* sf, float* rl)
{
    return launch_transport_impl<true>(ctx, st, T, rho_end, rho_begin, mfx, mfy, mfz, sf, rl);
}

int engine_enqueue(nimbus_engine* e, int lane, cudaStream_t st, int part)
{
    return enqueue_step<nimbus::Fp32Policy, true>(e, lane, st, part);
}

}  // namespace nimbus_fp32
