// Member-engine internals shared by the translation units that enqueue its
// large step (engine.cu for the reference-precision form, fp32_kernels.cu for
// the FP32 form, each compiled with its own contraction setting).
#pragma once

#include "context.cuh"
#include "engine_kernels.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
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
    int march_len = 16;             // i-planes per thread of the marching acoustic kernels
    int acoustic_form = NIMBUS_ACOUSTIC_CONST;  // nimbus_acoustic_form of the continuity pass
    int momentum_form = NIMBUS_ACOUSTIC_MARCH;  // and of the momentum pass (marching measured fastest)
    std::vector<cudaStream_t> lane_streams;  // lanes 1.. (lane 0 runs on the engine stream)
    std::vector<cudaEvent_t> lane_done;
    cudaEvent_t fork = nullptr;
    // One large step as two graphs: part 0 (Heun slow step, boundary refresh
    // and KW78 seed) needs no substep count; part 1 (the acoustic loop and the
    // rest of the step) does.  With resolve_substeps members, part 1 ends with
    // the acoustic speed scan of the state the next step starts from, so the
    // host reads the next step's counts while that step's part 0 runs.
    cudaGraph_t graph[2] = {nullptr, nullptr};
    cudaGraphExec_t exec[2] = {nullptr, nullptr};
    uint64_t exec_key[2] = {0, 0};  // topology key of exec (graph_topology_key)
    // Instantiated graphs of topologies used before (lane count and substep
    // counts come and go as runs are admitted and retire): a rebuild whose
    // topology matches one of them updates it in place instead of
    // instantiating anew.  Least recently used first out.
    struct CachedExec
    {
        uint64_t key;
        cudaGraphExec_t exec;
        uint64_t used;
    };
    std::vector<CachedExec> exec_cache[2];
    uint64_t exec_clock = 0;
    int launches_per_step = 0;
    int launches_part[2] = {0, 0};
    bool graphs_stale = true;       // the table changed since the graphs were captured
    uint64_t graph_instantiations = 0, graph_updates = 0;
    bool resolving = false;         // some member re-derives its substep count every step
    bool scan_pending = false;      // h_c2 will hold the current rows' scan once scan_done completes
    cudaEvent_t scan_done = nullptr;
    std::map<const void*, int> occupancy;
    std::map<std::pair<const void*, size_t>, int> occupancy_smem;  // (kernel, dynamic shared bytes)
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

// The slow Heun pair's and the transport passes' constant-bank forms (1) or
// member-table forms (0).
#ifndef NIMBUS_SLOW_CONST
#define NIMBUS_SLOW_CONST 1
#endif
#ifndef NIMBUS_TRANSPORT_CONST
#define NIMBUS_TRANSPORT_CONST 1
#endif

int blocks_per_sm(nimbus_engine* e, const void* kernel, int block = kEngineBlock)
{
    auto it = e->occupancy.find(kernel);
    if (it != e->occupancy.end()) return it->second;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, block, 0) != cudaSuccess || blocks < 1)
        blocks = 1;
    e->occupancy[kernel] = blocks;
    return blocks;
}

// Persistent grid: one wave of resident CTAs, never more blocks than tiles.
unsigned engine_grid(nimbus_engine* e, const void* kernel, long long tiles, int block = kEngineBlock)
{
    const long long wave = static_cast<long long>(e->ctx->sm_count) * blocks_per_sm(e, kernel, block);
    const long long g = tiles < wave ? tiles : wave;
    return static_cast<unsigned>(g < 1 ? 1 : g);
}

// The bulk-staged acoustic forms: dynamic shared memory of kBulkStages
// stages plus their barriers, at most kBulkSmemLimit (a lane whose members
// need more takes the constant-bank form).
constexpr size_t kBulkSmemLimit = 200 * 1024;
static_assert(kBulkTile == kEngineBlock * kItemsPerThread, "a bulk-staged tile is one cell tile");

size_t bulk_smem_bytes(int stage_floats)
{
    return kBulkBarrierBytes + static_cast<size_t>(kBulkStages) * stage_floats * sizeof(float);
}

// Persistent grid of a launch with dynamic shared memory.
unsigned engine_grid_smem(nimbus_engine* e, const void* kernel, long long tiles, size_t smem)
{
    const auto key = std::make_pair(kernel, smem);
    auto it = e->occupancy_smem.find(key);
    int blocks = 0;
    if (it != e->occupancy_smem.end()) blocks = it->second;
    else
    {
        // The opt-in limit is a ceiling only (occupancy follows each launch's
        // own size), so every size this kernel is launched with fits under it.
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(kBulkSmemLimit));
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, kernel, kEngineBlock, smem) != cudaSuccess ||
            blocks < 1)
            blocks = 1;
        e->occupancy_smem[key] = blocks;
    }
    const long long wave = static_cast<long long>(e->ctx->sm_count) * blocks;
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

#define ENGINE_LAUNCH_GRID(family, kernel, tiles, gy, block, ...)                                       \
    do {                                                                                                 \
        const long long tiles_ = (tiles);                                                                \
        if (tiles_ > 0)                                                                                  \
        {                                                                                                \
            LaunchTimer t_(ctx, st, family);                                                             \
            kernel<<<dim3(engine_grid(e, reinterpret_cast<const void*>(kernel), tiles_, (block)), gy),   \
                     (block), 0, st>>>(__VA_ARGS__);                                                     \
            ++count;                                                                                     \
        }                                                                                                \
    } while (0)
#define ENGINE_LAUNCH_SMEM(family, kernel, tiles, smem, ...)                                            \
    do {                                                                                                 \
        const long long tiles_ = (tiles);                                                                \
        if (tiles_ > 0)                                                                                  \
        {                                                                                                \
            LaunchTimer t_(ctx, st, family);                                                             \
            kernel<<<engine_grid_smem(e, reinterpret_cast<const void*>(kernel), tiles_, (smem)),         \
                     kEngineBlock, (smem), st>>>(__VA_ARGS__);                                           \
            ++count;                                                                                     \
        }                                                                                                \
    } while (0)
#define ENGINE_LAUNCH(family, kernel, tiles, gy, ...) \
    ENGINE_LAUNCH_GRID(family, kernel, tiles, gy, kEngineBlock, __VA_ARGS__)
#define ENGINE_LAUNCH_BLOCK(family, kernel, tiles, block, ...) \
    ENGINE_LAUNCH_GRID(family, kernel, tiles, 1, block, __VA_ARGS__)

// Enqueues part `part` of one large step of the members of one lane on `st`
// (0: Heun slow step, boundary refresh and KW78 seed; 1: the acoustic loop,
// transport, microphysics and EOS, the closing refresh); returns the number
// of launches.
template <class Policy, bool kFp32>
int enqueue_step(nimbus_engine* e, int lane, cudaStream_t st, int part)
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

    if (part == 0)
    {
    // Heun slow step (prepare_slow_rk2_tendencies + apply_slow_tendencies):
    // the constant-bank form for lanes of at most kSlowConstMembers members.
    if (NIMBUS_SLOW_CONST && n <= kSlowConstMembers)
    {
        std::unique_ptr<SlowLaunch> sl(new SlowLaunch());
        const long long* p = e->prefix.data() + L.prefix_first + static_cast<size_t>(kItemCells) * (n + 1);
        for (int r = 0; r <= n; ++r) sl->prefix[r] = p[r];
        for (int r = 0; r < n; ++r)
        {
            const EngineMember& H = e->slots[static_cast<size_t>(e->order[static_cast<size_t>(L.first + r)])].m;
            SlowConst& A = sl->m[r];
            A.S = H.S;
            A.u = H.u;
            A.v = H.v;
            A.w = H.w;
            A.theta = H.theta;
            A.qv = H.qv;
            A.qc = H.qc;
            A.k1 = reinterpret_cast<float4*>(H.k1);
            A.xs = reinterpret_cast<float4*>(H.xs);
            A.q4 = reinterpret_cast<float4*>(H.q4);
            A.rho0 = H.rho0;
            A.qv0 = H.qv0;
            A.u0 = H.u0;
            A.v0 = H.v0;
        }
        ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_predict_const_kernel<Policy>, cells, 1, *sl, T, cells);
        ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_correct_const_kernel<Policy>, cells, 1, *sl, T, cells);
    }
    else
    {
        ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_predict_kernel<Policy>, cells, 1, T, pc, cells);
        ENGINE_LAUNCH(NIMBUS_KERNEL_SLOW, engine_slow_correct_kernel<Policy>, cells, 1, T, pc, cells);
    }
    // seed_acoustic_radiation: apply_acoustic(0) then the KW78 seed.
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, L, kItemRowsWE, n), 1, T, pwe,
                  tiles_of(e, L, kItemRowsWE, n), 0, 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, L, kItemRowsSN, n), 1, T, psn,
                  tiles_of(e, L, kItemRowsSN, n), 0, 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_kernel, tiles_of(e, L, kItemColumns, n), 1, T,
                  pcol, tiles_of(e, L, kItemColumns, n), 1);
    ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_seed_kernel, tiles_of(e, L, kItemHistory, n), 1, T, phist,
                  tiles_of(e, L, kItemHistory, n));
    return count;
    }
    // The acoustic loop: members still inside it are a prefix of the lane.
    const long long* pm = prefix_of(e, L, kItemMarch);
    // The constant-bank forms: the lane's members' constants as one kernel
    // parameter (lanes of at most kConstMembers members; larger ones take the
    // member-table form).
    auto in_bank = [](int f) {
        return f == NIMBUS_ACOUSTIC_CONST || f == NIMBUS_ACOUSTIC_PAIR || f == NIMBUS_ACOUSTIC_BULK ||
               f == NIMBUS_ACOUSTIC_CMARCH;
    };
    // Bulk copies move 16-byte units between 16-byte-aligned addresses: every
    // member field starts on a 256-byte boundary of its arena, so the arenas
    // themselves must be 16-byte aligned.
    int sy4 = 4;
    bool arenas_aligned = true;
    for (int r = 0; r < n; ++r)
    {
        const nimbus_engine_detail::MemberSlot& slot =
            e->slots[static_cast<size_t>(e->order[static_cast<size_t>(L.first + r)])];
        sy4 = std::max(sy4, (slot.m.F.d.sy() + 3) & ~3);
        arenas_aligned = arenas_aligned && reinterpret_cast<uintptr_t>(slot.arena) % 16 == 0;
    }
    const size_t smem_cont = bulk_smem_bytes(continuity_stage_floats(sy4));
    const size_t smem_mom = bulk_smem_bytes(momentum_stage_floats(sy4));
    auto resolve_form = [&](int f) {
        if (in_bank(f) && n > kConstMembers) return static_cast<int>(NIMBUS_ACOUSTIC_TABLE);
        if (f == NIMBUS_ACOUSTIC_BULK && (smem_cont > kBulkSmemLimit || !arenas_aligned))
            return static_cast<int>(NIMBUS_ACOUSTIC_CONST);
        return f;
    };
    const int cform = resolve_form(e->acoustic_form), mform = resolve_form(e->momentum_form);
    std::unique_ptr<AcousticLaunch> al;
#ifndef NIMBUS_ACOUSTIC_SHARED
#define NIMBUS_ACOUSTIC_SHARED 1
#endif
    bool shared = NIMBUS_ACOUSTIC_SHARED != 0;  // every member's shared values equal al->shared
    if (in_bank(cform) || in_bank(mform))
    {
        al.reset(new AcousticLaunch());
        const long long* p = e->prefix.data() + L.prefix_first + static_cast<size_t>(kItemCells) * (n + 1);
        for (int r = 0; r <= n; ++r)
        {
            al->prefix[r] = p[r];
            al->prefix32[r] = static_cast<int>(p[r]);
        }
        const long long* pmr = e->prefix.data() + L.prefix_first + static_cast<size_t>(kItemMarch) * (n + 1);
        for (int r = 0; r <= n; ++r) al->march_prefix[r] = pmr[r];
        al->bulk_sy4 = sy4;
        for (int r = 0; r < n; ++r)
        {
            const EngineMember& H = e->slots[static_cast<size_t>(e->order[static_cast<size_t>(L.first + r)])].m;
            const AcousticShared own = acoustic_shared_of(H.F);
            if (r == 0) al->shared = own;
            else if (std::memcmp(&own, &al->shared, sizeof(AcousticShared)) != 0) shared = false;
        }
        for (int r = 0; r < n; ++r)
        {
            const EngineMember& H = e->slots[static_cast<size_t>(e->order[static_cast<size_t>(L.first + r)])].m;
            AcousticConst& A = al->m[r];
            A.F = H.F;
            A.u = H.u;
            A.v = H.v;
            A.w = H.w;
            A.theta = H.theta;
            A.mfx = H.mfx;
            A.mfy = H.mfy;
            A.mfz = H.mfz;
            A.rho_begin = H.rho_begin;
            A.status = H.status;
            A.rho0 = H.rho0;
            A.p0 = H.p0;
            A.dp0 = H.dp0;
            A.eos0 = H.eos0;
            A.vertical = kFuseVertical | (H.B.bottom == kBottomNoSlip ? kFuseNoSlipBottom : 0) |
                         (H.B.top == kTopOpen ? kFuseOpenTop : 0);
            A.march_len = H.march_len;
            A.march_blocks = H.march_blocks;
        }
    }
    for (size_t s = 0; s < L.active.size(); ++s)
    {
        const int a = L.active[s];
        const int si = static_cast<int>(s);
        const long long tiles = tiles_of(e, L, kItemCells, a);
        const long long march_tiles = tiles_of(e, L, kItemMarch, a);
        switch (cform)
        {
        case NIMBUS_ACOUSTIC_CONST:
            if (s == 0 && shared)
                ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_const_kernel<Policy, true, true>),
                              tiles, 1, *al, T, tiles, si);
            else if (s == 0)
                ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_const_kernel<Policy, true, false>),
                              tiles, 1, *al, T, tiles, si);
            else if (shared)
                ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_const_kernel<Policy, false, true>),
                              tiles, 1, *al, T, tiles, si);
            else
                ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_const_kernel<Policy, false, false>),
                              tiles, 1, *al, T, tiles, si);
            break;
        case NIMBUS_ACOUSTIC_PAIR:
            if (s == 0 && shared)
                ENGINE_LAUNCH_BLOCK(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP,
                                    (engine_continuity_pair_kernel<Policy, true, true>), tiles, kEngineBlock / 2, *al,
                                    T, tiles, si);
            else if (s == 0)
                ENGINE_LAUNCH_BLOCK(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP,
                                    (engine_continuity_pair_kernel<Policy, true, false>), tiles, kEngineBlock / 2, *al,
                                    T, tiles, si);
            else if (shared)
                ENGINE_LAUNCH_BLOCK(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP,
                                    (engine_continuity_pair_kernel<Policy, false, true>), tiles, kEngineBlock / 2, *al,
                                    T, tiles, si);
            else
                ENGINE_LAUNCH_BLOCK(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP,
                                    (engine_continuity_pair_kernel<Policy, false, false>), tiles, kEngineBlock / 2,
                                    *al, T, tiles, si);
            break;
        case NIMBUS_ACOUSTIC_MARCH:
            ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, engine_continuity_march_kernel<Policy>, march_tiles, 1, T,
                          pm, march_tiles, si);
            break;
        case NIMBUS_ACOUSTIC_CMARCH:
            if (s == 0)
                ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_cmarch_kernel<Policy, true>),
                              march_tiles, 1, *al, T, march_tiles, si);
            else
                ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_cmarch_kernel<Policy, false>),
                              march_tiles, 1, *al, T, march_tiles, si);
            break;
        case NIMBUS_ACOUSTIC_BULK:
            if (s == 0)
                ENGINE_LAUNCH_SMEM(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_bulk_kernel<Policy, true>),
                                   tiles, smem_cont, *al, T, tiles, si);
            else
                ENGINE_LAUNCH_SMEM(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, (engine_continuity_bulk_kernel<Policy, false>),
                                   tiles, smem_cont, *al, T, tiles, si);
            break;
        default:
            ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_SUBSTEP, engine_continuity_kernel<Policy>, tiles, 1, T, pc, tiles,
                          si);
        }
        switch (mform)
        {
        case NIMBUS_ACOUSTIC_CONST:
            ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_const_kernel<Policy>, tiles, 1, *al, T,
                          tiles, si);
            break;
        case NIMBUS_ACOUSTIC_PAIR:
            ENGINE_LAUNCH_BLOCK(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_pair_kernel<Policy>, tiles,
                                kEngineBlock / 2, *al, T, tiles, si);
            break;
        case NIMBUS_ACOUSTIC_MARCH:
            ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_march_kernel<Policy>, march_tiles, 1, T,
                          pm, march_tiles, si);
            break;
        case NIMBUS_ACOUSTIC_BULK:
            ENGINE_LAUNCH_SMEM(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_bulk_kernel<Policy>, tiles, smem_mom,
                               *al, T, tiles, si);
            break;
        case NIMBUS_ACOUSTIC_CMARCH:
            ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_cmarch_kernel<Policy>, march_tiles, 1, *al,
                          T, march_tiles, si);
            break;
        default:
            ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_MOMENTUM, engine_momentum_kernel<Policy>, tiles, 1, T, pc, tiles,
                          si);
        }
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_we_kernel, tiles_of(e, L, kItemRowsWE, a), 1, T, pwe,
                      tiles_of(e, L, kItemRowsWE, a), si, 0);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_sn_kernel, tiles_of(e, L, kItemRowsSN, a), 1, T, psn,
                      tiles_of(e, L, kItemRowsSN, a), si, 0);
        ENGINE_LAUNCH(NIMBUS_KERNEL_ACOUSTIC_BOUNDARY, engine_bc_vertical_perimeter_kernel,
                      tiles_of(e, L, kItemPerimeter, a), 1, T, pper, tiles_of(e, L, kItemPerimeter, a));
    }
    engine_swap_kernel<<<(n + 127) / 128, 128, 0, st>>>(T, n, 0);
    ++count;
    // Conservative transport of theta, qv, qc, qr against the retained fluxes
    // (the constant-bank form for lanes of at most kTransportConstMembers).
    if (NIMBUS_TRANSPORT_CONST && n <= kTransportConstMembers)
    {
        std::unique_ptr<TransportLaunch> tl(new TransportLaunch());
        const long long* p = e->prefix.data() + L.prefix_first + static_cast<size_t>(kItemCells) * (n + 1);
        for (int r = 0; r <= n; ++r) tl->prefix[r] = p[r];
        for (int r = 0; r < n; ++r)
        {
            const EngineMember& H = e->slots[static_cast<size_t>(e->order[static_cast<size_t>(L.first + r)])].m;
            TransportConst& A = tl->m[r];
            TransportCompact& C = A.T;
            C.d = H.T.d;
            C.inv_dx = H.T.inv_dx;
            C.inv_dy = H.T.inv_dy;
            C.inv_dz = H.T.inv_dz;
            C.dt = H.T.dt;
            C.rho_floor = H.T.rho_floor;
            C.weno = H.T.weno;
            C.top_open = H.T.top_open;
            for (int q = 0; q < 4; ++q) C.positive_definite[q] = H.T.positive_definite[q];
            C.inv_dx_f = H.T.inv_dx_f;
            C.inv_dy_f = H.T.inv_dy_f;
            C.inv_dz_f = H.T.inv_dz_f;
            C.dt_f = H.T.dt_f;
            C.inv_dt_f = H.T.inv_dt_f;
            C.rho_floor_f = H.T.rho_floor_f;
            A.q4 = reinterpret_cast<const float4*>(H.q4);
            A.mfx = H.mfx;
            A.mfy = H.mfy;
            A.mfz = H.mfz;
            A.rho_begin = H.rho_begin;
            A.sf = reinterpret_cast<float4*>(H.sf);
            A.rl = reinterpret_cast<float4*>(H.rl);
            A.theta = H.theta;
            A.qv = H.qv;
            A.qc = H.qc;
            A.status = H.status;
        }
        ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_FACES, engine_transport_faces_const_kernel<kFp32>, cells, 1, *tl, T,
                      cells);
        ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_LIMITER, engine_transport_limiter_const_kernel<kFp32>, cells, 1, *tl, T,
                      cells);
        ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_UPDATE, engine_transport_update_const_kernel<kFp32>, cells, 1, *tl, T,
                      cells);
    }
    else
    {
        ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_FACES, engine_transport_faces_kernel<kFp32>, cells, 1, T, pc, cells);
        ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_LIMITER, engine_transport_limiter_kernel<kFp32>, cells, 1, T, pc,
                      cells);
        ENGINE_LAUNCH(NIMBUS_KERNEL_TRANSPORT_UPDATE, engine_transport_update_kernel<kFp32>, cells, 1, T, pc, cells);
    }
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
    // The acoustic speed scan of the state the next step starts from.
    if (e->resolving)
        ENGINE_LAUNCH(NIMBUS_KERNEL_MICROPHYSICS, engine_sound_speed_kernel, tiles_of(e, L, kItemScan, n), 1, T,
                      prefix_of(e, L, kItemScan), tiles_of(e, L, kItemScan, n), e->d_c2 + L.first);
    return count;
}

}  // namespace
