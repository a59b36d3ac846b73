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
    double c_base = 0.0;      // largest sound speed of the base columns (resolve_substeps members)
};
// A lane: a contiguous run of table rows whose members step together.  The
// members are split into size-balanced lanes; each lane's launches go to its
// own stream (forked from the engine stream and joined back, inside the one
// captured graph), so one lane's kernels fill the SMs that another's
// launch tails leave idle.  Within a lane rows are sorted by substep count,
// so the members still inside the acoustic loop are a prefix of it.
struct Lane
{
    int first = 0;            // first table row
    int members = 0;
    size_t prefix_first = 0;  // first entry of this lane's [kItemKinds][members + 1] prefix block
    std::vector<int> active;  // members of this lane inside the loop at substep s
    bool closing = false;     // some member ends its step with the boundary closure
};
// The Kessler + EOS pass (FP64 in the reference-precision form, FP32 in the
// FP32 form) is launched from the uncontracted unit (engine.cu), so the engine
// and the per-operation path share its rounding.  Returns the launch count.
int launch_microphysics(nimbus_engine* e, cudaStream_t st, const nimbus::EngineMember* table,
                        const long long* prefix, long long tiles);
}  // namespace nimbus_engine_detail

struct nimbus_engine
{
    nimbus_cuda_context* ctx = nullptr;
    cudaStream_t stream = nullptr;  // the engine's own stream (graphs, copies)
    bool mirror_exact = true;       // host views predict the device pointer rotations
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
    std::vector<long long> prefix;  // the lanes' prefix blocks, back to back
    std::vector<nimbus_engine_detail::Lane> lanes;
    int lane_target = 4;            // lanes when there are at least that many members
    std::vector<cudaStream_t> lane_streams;  // lanes 1.. (lane 0 runs on the engine stream)
    std::vector<cudaEvent_t> lane_done;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int launches_per_step = 0;
    std::map<const void*, int> occupancy;
    float* d_image = nullptr;       // device staging for the state image
    size_t image_cap = 0;           // bytes
    float* d_centre = nullptr;      // device staging for history frames
    size_t centre_cap = 0;          // bytes
    unsigned long long* d_c2 = nullptr;  // per table row: max (gamma p) / rho before a step
    unsigned long long* h_c2 = nullptr;  // pinned host copy
    size_t c2_cap = 0;                   // rows
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

const long long* prefix_of(const nimbus_engine* e, const nimbus_engine_detail::Lane& L, int kind)
{
    return e->d_prefix + L.prefix_first + static_cast<size_t>(kind) * (L.members + 1);
}

long long tiles_of(const nimbus_engine* e, const nimbus_engine_detail::Lane& L, int kind, int members)
{
    return e->prefix[L.prefix_first + static_cast<size_t>(kind) * (L.members + 1) + members];
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

// Enqueues one large step of the members of one lane on `st`; returns the
// number of launches.
template <class Policy, bool kFp32>
int enqueue_step(nimbus_engine* e, int lane, cudaStream_t st)
{
    nimbus_cuda_context* ctx = e->ctx;
    const nimbus_engine_detail::Lane& L = e->lanes[static_cast<size_t>(lane)];
    const int n = L.members;
    int count = 0;
    EngineMember* T = e->d_table + L.first;
    const long long* pc = prefix_of(e, L, kItemCells);
    const long long* pwe = prefix_of(e, L, kItemRowsWE);
    const long long* psn = prefix_of(e, L, kItemRowsSN);
    const long long* pcol = prefix_of(e, L, kItemColumns);
    const long long* phist = prefix_of(e, L, kItemHistory);
    const long long* pper = prefix_of(e, L, kItemPerimeter);
    const long long cells = tiles_of(e, L, kItemCells, n);

    // Heun slow step (prepare_slow_rk2_tendencies + apply_slow_tendencies).
    ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_predict_kernel<Policy>, cells, 1, T, pc, cells);
    ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_correct_kernel<Policy>, cells, 1, T, pc, cells);
    // seed_acoustic_radiation: apply_acoustic(0) then the KW78 seed.
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, L, kItemRowsWE, n), 1, T, pwe,
                  tiles_of(e, L, kItemRowsWE, n), 0, 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, L, kItemRowsSN, n), 1, T, psn,
                  tiles_of(e, L, kItemRowsSN, n), 0, 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_kernel, tiles_of(e, L, kItemColumns, n), 1, T,
                  pcol, tiles_of(e, L, kItemColumns, n), 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_seed_kernel, tiles_of(e, L, kItemHistory, n), 1, T, phist,
                  tiles_of(e, L, kItemHistory, n));
    // The acoustic loop: members still inside it are a prefix of the lane.
    for (size_t s = 0; s < L.active.size(); ++s)
    {
        const int a = L.active[s];
        const int si = static_cast<int>(s);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, engine_continuity_kernel<Policy>, tiles_of(e, L, kItemCells, a), 1,
                      T, pc, tiles_of(e, L, kItemCells, a), si);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_kernel<Policy>, tiles_of(e, L, kItemCells, a), 1,
                      T, pc, tiles_of(e, L, kItemCells, a), si);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, L, kItemRowsWE, a), 1, T, pwe,
                      tiles_of(e, L, kItemRowsWE, a), si, 0);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, L, kItemRowsSN, a), 1, T, psn,
                      tiles_of(e, L, kItemRowsSN, a), si, 0);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_perimeter_kernel,
                      tiles_of(e, L, kItemPerimeter, a), 1, T, pper, tiles_of(e, L, kItemPerimeter, a));
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
    // The closing boundary refresh (apply_full_attributed, after the sponge)
    // for the members that ask for it, on the published density and pressure.
    if (L.closing)
    {
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, L, kItemRowsWE, n), 1, T, pwe,
                      tiles_of(e, L, kItemRowsWE, n), 0, 2);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, L, kItemRowsSN, n), 1, T, psn,
                      tiles_of(e, L, kItemRowsSN, n), 0, 2);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_kernel, tiles_of(e, L, kItemColumns, n), 1,
                      T, pcol, tiles_of(e, L, kItemColumns, n), 2);
    }
    return count;
}

}  // namespace
