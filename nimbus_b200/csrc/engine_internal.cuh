// Member-engine internals shared by the translation units that enqueue its
// large step (engine.cu for the reference-precision form, fp32_kernels.cu for
// the FP32 form, each compiled with its own contraction setting).
#pragma once

#include "context.cuh"
#include "engine_kernels.cuh"

#include <map>
#include <vector>

namespace nimbus_engine_detail
{
struct MemberSlot
{
    int id;
    nimbus_member_desc desc;  // profile pointers cleared after admission
    void* arena = nullptr;
    size_t bytes = 0;
    nimbus::EngineMember m;   // host view of the device entry (refreshed before use)
};
// The Kessler + EOS pass is FP64 in both forms and is launched from the
// uncontracted unit (engine.cu), so both forms and the per-operation path
// share its rounding.  Returns the launch count.
int launch_microphysics(nimbus_engine* e, cudaStream_t st, const nimbus::EngineMember* table,
                        const long long* prefix, long long tiles);
}  // namespace nimbus_engine_detail

struct nimbus_engine
{
    nimbus_cuda_context* ctx = nullptr;
    std::vector<nimbus_engine_detail::MemberSlot> slots;  // admission order
    std::vector<int> order;         // slot indices in table order
    int next_id = 1;
    bool dirty = true;              // table / graph need a rebuild
    bool table_current = true;      // host views match the device table
    bool use_graph = true;
    int built_precision = -1;
    nimbus::EngineMember* d_table = nullptr;
    size_t table_cap = 0;
    long long* d_prefix = nullptr;
    size_t prefix_cap = 0;
    std::vector<long long> prefix;  // [kItemKinds][members + 1]
    std::vector<int> active;        // members inside the loop at substep s
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches_per_step = 0;
    std::map<const void*, int> occupancy;
};

namespace
{

using namespace nimbus;
using namespace nimbus_host;

constexpr int kEngineBlock = 256;

int blocks_per_sm(nimbus_engine* e, const void* kernel)
{
    auto it = e->occupancy.find(kernel);
    if (it != e->occupancy.end()) return it->second;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kEngineBlock, 0) != cudaSuccess || blocks < 1)
        blocks = 1;
    e->occupancy[kernel] = blocks;
    return blocks;
}

// Persistent grid: one wave of resident CTAs, never more blocks than tiles.
unsigned engine_grid(nimbus_engine* e, const void* kernel, long long tiles)
{
    const long long wave = static_cast<long long>(e->ctx->sm_count) * blocks_per_sm(e, kernel);
    const long long g = tiles < wave ? tiles : wave;
    return static_cast<unsigned>(g < 1 ? 1 : g);
}

const long long* prefix_of(const nimbus_engine* e, int kind)
{
    return e->d_prefix + static_cast<size_t>(kind) * (e->order.size() + 1);
}

long long tiles_of(const nimbus_engine* e, int kind, int members)
{
    return e->prefix[static_cast<size_t>(kind) * (e->order.size() + 1) + members];
}

#define ENGINE_LAUNCH(family, kernel, tiles, gy, ...)                                                    \
    do {                                                                                                 \
        const long long tiles_ = (tiles);                                                                \
        if (tiles_ > 0)                                                                                  \
        {                                                                                                \
            LaunchTimer t_(ctx, st, family);                                                             \
            kernel<<<dim3(engine_grid(e, reinterpret_cast<const void*>(kernel), tiles_), gy), kEngineBlock, 0, \
                     st>>>(__VA_ARGS__);                                                                 \
            ++count;                                                                                     \
        }                                                                                                \
    } while (0)

// Enqueues one large step of every member; returns the number of launches.
template <class Policy, bool kFp32>
int enqueue_step(nimbus_engine* e, cudaStream_t st)
{
    nimbus_cuda_context* ctx = e->ctx;
    const int n = static_cast<int>(e->order.size());
    int count = 0;
    EngineMember* T = e->d_table;
    const long long* pc = prefix_of(e, kItemCells);
    const long long* pwe = prefix_of(e, kItemRowsWE);
    const long long* psn = prefix_of(e, kItemRowsSN);
    const long long* pcol = prefix_of(e, kItemColumns);
    const long long* phist = prefix_of(e, kItemHistory);
    const long long cells = tiles_of(e, kItemCells, n);

    // Heun slow step (prepare_slow_rk2_tendencies + apply_slow_tendencies).
    ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_predict_kernel<Policy>, cells, 1, T, pc, cells);
    ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_correct_kernel<Policy>, cells, 1, T, pc, cells);
    // seed_acoustic_radiation: apply_acoustic(0) then the KW78 seed.
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, kItemRowsWE, n), 1, T, pwe,
                  tiles_of(e, kItemRowsWE, n), 0, 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, kItemRowsSN, n), 1, T, psn,
                  tiles_of(e, kItemRowsSN, n), 0, 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_kernel, tiles_of(e, kItemColumns, n), 1, T,
                  pcol, tiles_of(e, kItemColumns, n));
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_seed_kernel, tiles_of(e, kItemHistory, n), 1, T, phist,
                  tiles_of(e, kItemHistory, n));
    // The acoustic loop: members still inside it are a prefix of the table.
    for (size_t s = 0; s < e->active.size(); ++s)
    {
        const int a = e->active[s];
        const int si = static_cast<int>(s);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, engine_continuity_kernel<Policy>, tiles_of(e, kItemCells, a), 1,
                      T, pc, tiles_of(e, kItemCells, a), si);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_kernel<Policy>, tiles_of(e, kItemCells, a), 1,
                      T, pc, tiles_of(e, kItemCells, a), si);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, kItemRowsWE, a), 1, T, pwe,
                      tiles_of(e, kItemRowsWE, a), si, 0);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, kItemRowsSN, a), 1, T, psn,
                      tiles_of(e, kItemRowsSN, a), si, 0);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_kernel, tiles_of(e, kItemColumns, a), 1, T,
                      pcol, tiles_of(e, kItemColumns, a));
    }
    engine_swap_kernel<<<(n + 127) / 128, 128, 0, st>>>(T, n, 0);
    ++count;
    // Conservative transport of theta, qv, qc, qr against the retained fluxes.
    ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_FACES, engine_transport_faces_kernel<kFp32>, cells, 1, T, pc,
                  cells);
    ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_LIMITER, engine_transport_limiter_kernel<kFp32>, cells, 1, T, pc,
                  cells);
    ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_UPDATE, engine_transport_update_kernel<kFp32>, cells, 1, T, pc,
                  cells);
    // Kessler step and the EOS pressure re-projection (one pass), then the
    // pointer rotation that publishes the new qr and pressure.
    count += nimbus_engine_detail::launch_microphysics(e, st, T, pc, cells);
    engine_swap_kernel<<<(n + 127) / 128, 128, 0, st>>>(T, n, 1);
    ++count;
    return count;
}

}  // namespace
