// Host-side internals shared by the backend's translation units: the
// context behind nimbus_cuda_context, its device workspace, error reporting,
// launch timing and the staging helpers.
#pragma once

#include "../../include/nimbus_cuda.h"
#include "transport_kernels.cuh"

#include <atomic>
#include <cmath>
#include <cstdint>
#include <limits>
#include <string>
#include <vector>

#include <cuda_runtime.h>

namespace nimbus_host
{

using nimbus::kMaxScalars;

constexpr int kThreads = 256;

struct DeviceBuffer
{
    void* ptr = nullptr;
    size_t bytes = 0;
};

enum Slot
{
    kU, kV, kW, kRho, kP, kTheta, kRhoAlt, kDrho, kRho0, kP0, kMfx, kMfy, kMfz, kWave, kRhoBegin,
    kRhoEnd, kSf, kRl, kUAlt, kVAlt, kWAlt, kDp0, kSlowK1, kSlowStar, kSlowOut, kQv, kQc, kQr, kQv0, kU0, kV0,
    kQrAlt, kKesslerOut, kEosCandidate, kEos0, kRelaxTables, kCentre, kGround,
    kSgsTables, kSgsCoef, kSgsRates, kSgsScratch, kSgsTheta0, kTke, kTkeRates, kSoundSpeed,
    kQ0, kSlotCount = kQ0 + 2 * kMaxScalars
};

}  // namespace nimbus_host

struct TimedLaunch
{
    int family;
    cudaEvent_t start, stop;
};

struct nimbus_cuda_context
{
    int device = 0;
    int precision = NIMBUS_PRECISION_REFERENCE;
    int substep_form = NIMBUS_SUBSTEP_AUTO;
    struct TunedShape
    {
        int nx, ny, nz, precision, form;
    };
    std::vector<TunedShape> tuned;
    bool timing = false;
    std::vector<TimedLaunch> pending;
    std::vector<cudaEvent_t> event_pool;
    uint64_t timed_launches[NIMBUS_KERNEL_FAMILIES] = {};
    double timed_ms[NIMBUS_KERNEL_FAMILIES] = {};
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    unsigned* status = nullptr;  // device status word
    std::atomic<uint64_t> launches{0};  // engines of this context may step from their own host threads
    std::string error;
    nimbus_host::DeviceBuffer ws[nimbus_host::kSlotCount];
};

namespace nimbus_host
{

inline nimbus_status fail(nimbus_cuda_context* ctx, nimbus_status s, const std::string& msg)
{
    if (ctx) ctx->error = msg;
    return s;
}

inline nimbus_status cuda_fail(nimbus_cuda_context* ctx, cudaError_t e, const char* where)
{
    return fail(ctx, e == cudaErrorMemoryAllocation ? NIMBUS_ERR_OUT_OF_MEMORY : NIMBUS_ERR_CUDA,
                std::string(where) + ": " + cudaGetErrorString(e));
}

#define NB_CUDA(ctx, call)                                   \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(ctx, e_, #call); \
    } while (0)

template <class T>
inline nimbus_status ensure(nimbus_cuda_context* ctx, Slot slot, size_t count, T** out)
{
    DeviceBuffer& b = ctx->ws[slot];
    const size_t bytes = count * sizeof(T);
    if (b.bytes < bytes)
    {
        if (b.ptr) cudaFree(b.ptr);
        b.ptr = nullptr;
        b.bytes = 0;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "workspace allocation");
        b.ptr = p;
        b.bytes = bytes;
    }
    *out = static_cast<T*>(b.ptr);
    return NIMBUS_OK;
}

inline cudaEvent_t take_event(nimbus_cuda_context* ctx)
{
    if (!ctx->event_pool.empty())
    {
        cudaEvent_t e = ctx->event_pool.back();
        ctx->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets the launches issued between begin() and end() with CUDA events on
// their stream when kernel timing is enabled.
struct LaunchTimer
{
    nimbus_cuda_context* ctx;
    cudaStream_t stream;
    int family;
    cudaEvent_t start = nullptr;
    LaunchTimer(nimbus_cuda_context* c, cudaStream_t s, int f) : ctx(c), stream(s), family(f)
    {
        if (ctx->timing)
        {
            start = take_event(ctx);
            cudaEventRecord(start, stream);
        }
    }
    ~LaunchTimer()
    {
        if (start)
        {
            cudaEvent_t stop = take_event(ctx);
            cudaEventRecord(stop, stream);
            ctx->pending.push_back({family, start, stop});
        }
    }
};

inline void drain_timing(nimbus_cuda_context* ctx)
{
    for (auto& t : ctx->pending)
    {
        float ms = 0.0f;
        cudaEventSynchronize(t.stop);
        cudaEventElapsedTime(&ms, t.start, t.stop);
        ctx->timed_launches[t.family] += 1;
        ctx->timed_ms[t.family] += ms;
        ctx->event_pool.push_back(t.start);
        ctx->event_pool.push_back(t.stop);
    }
    ctx->pending.clear();
}

inline int grid_for(const nimbus_cuda_context* ctx, long long work)
{
    long long blocks = (work + kThreads - 1) / kThreads;
    const long long cap = static_cast<long long>(ctx->sm_count) * 16;
    if (blocks > cap) blocks = cap;
    return blocks < 1 ? 1 : static_cast<int>(blocks);
}

inline bool finite_positive(double v) { return std::isfinite(v) && v > 0.0; }
inline bool valid_bounds(float lo, float hi) { return std::isfinite(lo) && std::isfinite(hi) && lo > 0.0f && lo <= hi; }
inline bool cells_fit(int nx, int ny, int nz)
{
    return static_cast<long long>(nx) * ny * nz < static_cast<long long>(std::numeric_limits<int>::max()) / 4;
}

inline nimbus_status upload(nimbus_cuda_context* ctx, void* dst, const void* src, size_t bytes)
{
    NB_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream));
    return NIMBUS_OK;
}

inline nimbus_status download(nimbus_cuda_context* ctx, void* dst, const void* src, size_t bytes)
{
    NB_CUDA(ctx, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream));
    return NIMBUS_OK;
}

inline nimbus_status read_status(nimbus_cuda_context* ctx, cudaStream_t stream, unsigned* flags)
{
    unsigned h = 0;
    NB_CUDA(ctx, cudaMemcpyAsync(&h, ctx->status, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
    NB_CUDA(ctx, cudaMemsetAsync(ctx->status, 0, sizeof(unsigned), stream));
    NB_CUDA(ctx, cudaStreamSynchronize(stream));
    *flags = h;
    return NIMBUS_OK;
}

#define NB_TRY(expr)                         \
    do {                                     \
        nimbus_status s_ = (expr);           \
        if (s_ != NIMBUS_OK) return s_;      \
    } while (0)

}  // namespace nimbus_host
