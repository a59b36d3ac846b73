// Member engine (include/nimbus_cuda.h): resident runs advanced together, one
// batched launch per phase of the large step, replayed from a CUDA graph.
//
// Host bookkeeping.  Each member owns one device arena (state, retained
// transport context, scratch, profiles, status word).  The device member
// table is the authority for the ping-pong pointers (the swap kernels rotate
// them on the device every step), so any host-side change to the membership
// first waits for the stream and reads the table back.  The table is kept
// sorted by substep count, descending, so the members still inside their
// acoustic loop at substep s are a prefix of it.
#include "../../include/nimbus_cuda.h"
#include "context.cuh"
#include "engine_internal.cuh"
#include "launch.cuh"
#include "output_host.cuh"

#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

using namespace nimbus;
using namespace nimbus_host;

namespace
{

constexpr size_t kAlign = 256;

using nimbus_engine_detail::Lane;
using nimbus_engine_detail::MemberSlot;

size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// Byte layout of one member's arena.
struct ArenaLayout
{
    size_t cells, history;
    size_t off_state, off_ctxt, off_wave, off_sf, off_rl, off_q4, off_k1, off_xs, off_eos, off_status, off_prof, off_dp0,
        off_eos0, off_sponge, sponge_bytes, total;
};

ArenaLayout arena_layout(const nimbus_member_desc* d)
{
    ArenaLayout L{};
    L.cells = static_cast<size_t>(d->nx) * d->ny * d->nz;
    L.history = 2 * (static_cast<size_t>(d->nx) + d->ny) * d->nz;
    const size_t field = align_up(L.cells * sizeof(float));
    size_t off = 0;
    L.off_state = off;  off += 11 * field;                  // u v w rho rho_alt p theta qv qc qr qr_alt
    L.off_ctxt = off;   off += 4 * field;                   // rho_begin mfx mfy mfz
    L.off_wave = off;   off += align_up(L.history * sizeof(float));
    L.off_sf = off;     off += align_up(3 * kEngineScalars * L.cells * sizeof(float));
    L.off_rl = off;     off += align_up(kEngineScalars * L.cells * sizeof(float));
    L.off_q4 = off;     off += align_up(kEngineScalars * L.cells * sizeof(float));
    L.off_k1 = off;     off += align_up(4 * L.cells * sizeof(float));
    L.off_xs = off;     off += align_up(4 * L.cells * sizeof(float));
    L.off_eos = off;    off += field;
    L.off_status = off; off += kAlign;
    L.off_prof = off;   off += align_up(5 * static_cast<size_t>(d->nz) * sizeof(double));
    L.off_dp0 = off;    off += align_up(static_cast<size_t>(d->nz) * sizeof(float2));
    L.off_eos0 = off;   off += align_up(static_cast<size_t>(d->nz) * sizeof(float4));
    L.off_sponge = off;
    if (const nimbus_sponge_desc* sp = d->sponge)
    {
        // RelaxImage: 6 nz + max(width, 1) doubles, then 2 nz level flags.
        const int width = (sp->do_lateral && sp->lateral_width > 0) ? sp->lateral_width : 0;
        L.sponge_bytes = (6 * static_cast<size_t>(d->nz) + static_cast<size_t>(width > 0 ? width : 1)) *
                             sizeof(double) + 2 * static_cast<size_t>(d->nz);
        off += align_up(L.sponge_bytes);
    }
    L.total = off;
    return L;
}

const char* check_desc(const nimbus_member_desc* d)
{
    if (d->nx < 4 || d->ny < 4 || d->nz < 2) return "member grid must be at least 4x4x2";
    if (!cells_fit(d->nx, d->ny, d->nz)) return "member grid too large";
    if (!finite_positive(d->dx) || !finite_positive(d->dy) || !finite_positive(d->dz) || !finite_positive(d->dt))
        return "spacing and dt must be finite and positive";
    if (d->resolve_substeps != 0 && d->resolve_substeps != 1) return "resolve_substeps must be 0 or 1";
    if (d->resolve_substeps ? (d->n_substeps < 0 || d->n_substeps > 4096) : (d->n_substeps < 1 || d->n_substeps > 4096))
        return "n_substeps must be in [1, 4096] ([0, 4096] as the requested minimum of resolve_substeps)";
    for (int a = 0; a < 4; ++a)
        if (d->bc[a] < 0 || d->bc[a] > 4) return "lateral boundary code out of range";
    if (d->bc[4] < 0 || d->bc[4] > 1 || d->bc[5] < 0 || d->bc[5] > 2) return "vertical boundary code out of range";
    if (!std::isfinite(d->coriolis_f) || !std::isfinite(d->frame_velocity_u_ms) ||
        !std::isfinite(d->frame_velocity_v_ms))
        return "coriolis_f and frame velocity must be finite";
    if (d->microphysics != 0 && d->microphysics != 1) return "microphysics must be 0 (none) or 1 (Kessler)";
    if (d->final_closure != 0 && d->final_closure != 1) return "final_closure must be 0 or 1";
    // step_microphysics subcycles when the interval exceeds the sedimentation
    // limit 0.8 dz / max terminal velocity (microphysics_step.cpp:3500-3575,
    // 3686-3740); Kessler's fall speed is capped at 20 m/s, so dt <= 0.04 dz
    // guarantees the single call this engine makes.
    if (d->microphysics == 1 && d->dt > 0.8 * d->dz / 20.0)
        return "dt exceeds the Kessler sedimentation limit 0.8 dz / (20 m/s); the reference would subcycle";
    if (!d->rho0_base || !d->p0_base || !d->qv0_base) return "rho0, p0 and qv0 base profiles are required";
    if (const nimbus_sponge_desc* sp = d->sponge)
    {
        RelaxImage img;
        if (const char* why = build_relax_image(d->nx, d->ny, d->nz, sp->alpha, sp->upper_w_alpha, sp->w_only_alpha,
                                                sp->u_ref, sp->v_ref, sp->theta_ref, sp->lateral_width,
                                                sp->lateral_alpha, sp->do_upper, sp->do_w_only, sp->do_lateral,
                                                sp->staggered, sp->implicit_mode, d->dt, img))
            return why;
    }
    return nullptr;
}

// Parameter blocks of one member: the values the per-operation entry points
// receive from the reference-facing callers (dispatch constants of
// dynamics.cpp:4560-4586 and field_bounds.hpp).
void fill_params(EngineMember& M, const nimbus_member_desc* a)
{
    const double gamma = kCpd / (kCpd - kRd);
    const double dt_small = a->dt / a->n_substeps;
    FusedParams& F = M.F;
    F = FusedParams{};
    F.d = make_dims(a->nx, a->ny, a->nz);
    F.inv_dx = 1.0 / a->dx;
    F.inv_dy = 1.0 / a->dy;
    F.inv_dz = 1.0 / a->dz;
    F.dt_small = dt_small;
    F.gamma = gamma;
    F.rho_min = 0.05f;
    F.rho_max = 2.0f;
    F.p_min = 1000.0f;
    F.p_max = 200000.0f;
    F.p_ref_fallback = 100000.0f;
    F.wind_h = 180.0f;
    F.wind_v = 120.0f;
    F.weight = dt_small / a->dt;
    F.frame_u = a->frame_velocity_u_ms;
    F.frame_v = a->frame_velocity_v_ms;
    F.top_open = a->bc[5] == kTopOpen;
    F.chunk = 1;
    finish_fp32(F);

    BoundaryParams& B = M.B;
    B = BoundaryParams{};
    B.d = F.d;
    B.west = a->bc[0]; B.east = a->bc[1]; B.south = a->bc[2]; B.north = a->bc[3];
    B.bottom = a->bc[4]; B.top = a->bc[5];
    B.dt_rad = static_cast<float>(dt_small);
    B.inv_dx = 1.0f / static_cast<float>(a->dx);
    B.inv_dy = 1.0f / static_cast<float>(a->dy);
    B.frame_u = a->frame_velocity_u_ms;
    B.frame_v = a->frame_velocity_v_ms;

    TransportParams& T = M.T;
    T = TransportParams{};
    T.d = F.d;
    T.inv_dx = 1.0 / a->dx;
    T.inv_dy = 1.0 / a->dy;
    T.inv_dz = 1.0 / a->dz;
    T.dt = a->dt;
    T.rho_floor = static_cast<double>(0.05f);
    T.weno = 1;
    T.top_open = a->bc[5] == kTopOpen;
    T.n_scalars = kEngineScalars;
    T.positive_definite[0] = 0;  // theta (advection_batch.cpp:742-745)
    for (int s = 1; s < kEngineScalars; ++s) T.positive_definite[s] = 1;
    finish_fp32(T);

    SlowParams& S = M.S;
    S = SlowParams{};
    S.d = F.d;
    S.inv_dx = 1.0 / a->dx;
    S.inv_dy = 1.0 / a->dy;
    S.inv_dz = 1.0 / a->dz;
    S.dt = a->dt;
    S.coriolis_f = a->coriolis_f;
    S.frame_u = a->frame_velocity_u_ms;
    S.frame_v = a->frame_velocity_v_ms;
    S.gravity = 9.81;
    S.moist = 1;
    S.loading = 1;
    finish_fp32(S);

    KesslerParams& K = M.K;
    K = KesslerParams{};
    K.d = F.d;
    K.dz = a->dz;
    K.dt = a->dt;
    K.i0 = 1; K.i1 = a->nx - 1;  // physical_scalar_domain of the C-grid
    K.j0 = 1; K.j1 = a->ny - 1;
    K.k0 = 0; K.k1 = a->nz;
    K.qc0 = 1.0e-3;
    K.c_auto = 1.0e-3;
    K.c_accr = 2.2;
    K.evap_eff = 1.0;
    K.vt_max = 20.0;
    finish_fp32(K);

    M.gamma = gamma;
    M.eos_series = eos_series(gamma);
    M.n_substeps = a->n_substeps;
    M.microphysics = a->microphysics;
    M.items[kItemCells] = a->nx * a->ny * a->nz;
    M.items[kItemRowsWE] = a->ny * a->nz;
    M.items[kItemRowsSN] = a->nx * a->nz;
    M.items[kItemColumns] = a->nx * a->ny;
    M.items[kItemHistory] = (a->ny + a->nx) * a->nz;
    M.items[kItemPerimeter] = 3 * a->nx + 3 * (a->ny - 3);
    M.items[kItemScan] = (M.items[kItemCells] + kScanCells - 1) / kScanCells;
}

}  // namespace


namespace
{

// The host views track the device pointer rotations by replaying them
// (rotate_host_views) after every enqueued step; only a refused EOS
// projection (a member whose p is not rotated) makes them inexact, and then
// the device table is read back.
void rotate_host_views(nimbus_engine* e, int steps)
{
    for (auto& slot : e->slots)
    {
        EngineMember& M = slot.m;
        for (int s = 0; s < steps; ++s)
        {
            if (M.n_substeps & 1) std::swap(M.rho, M.rho_alt);
            if (M.microphysics) std::swap(M.qr, M.qr_alt);
            std::swap(M.p, M.eos);
        }
    }
}

// Makes the host views exact: when they already are (the mirror replayed
// every enqueued rotation), returns at once without waiting for the stream;
// otherwise waits for the stream and reads the table back.
nimbus_status sync_table_to_host(nimbus_engine* e)
{
    nimbus_cuda_context* ctx = e->ctx;
    if (e->table_current || e->order.empty()) return NIMBUS_OK;
    NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
    std::vector<EngineMember> host(e->order.size());
    NB_CUDA(ctx, cudaMemcpy(host.data(), e->d_table, sizeof(EngineMember) * host.size(), cudaMemcpyDeviceToHost));
    for (size_t r = 0; r < e->order.size(); ++r) e->slots[e->order[r]].m = host[r];
    e->table_current = true;
    return NIMBUS_OK;
}

// Free device memory for admission (the rule of
// include/compute/compute_memory_admission.hpp): cudaMemGetInfo's free bytes
// plus what the device's default memory pool holds reserved but unused
// (arenas of retired members freed in stream order return there first).
nimbus_status free_device_bytes(nimbus_cuda_context* ctx, size_t* out)
{
    size_t free_bytes = 0, total_bytes = 0;
    NB_CUDA(ctx, cudaMemGetInfo(&free_bytes, &total_bytes));
    cudaMemPool_t pool = nullptr;
    NB_CUDA(ctx, cudaDeviceGetDefaultMemPool(&pool, ctx->device));
    unsigned long long reserved = 0, used = 0;  // the attributes are 64-bit
    NB_CUDA(ctx, cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved));
    NB_CUDA(ctx, cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used));
    *out = free_bytes + static_cast<size_t>(reserved > used ? reserved - used : 0);
    return NIMBUS_OK;
}

// Lane streams and events live as long as the engine; grown on demand.
nimbus_status ensure_lane_streams(nimbus_engine* e, size_t extra)
{
    nimbus_cuda_context* ctx = e->ctx;
    if (extra && !e->fork) NB_CUDA(ctx, cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming));
    while (e->lane_streams.size() < extra)
    {
        cudaStream_t s = nullptr;
        NB_CUDA(ctx, cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        e->lane_streams.push_back(s);
        cudaEvent_t d = nullptr;
        NB_CUDA(ctx, cudaEventCreateWithFlags(&d, cudaEventDisableTiming));
        e->lane_done.push_back(d);
    }
    return NIMBUS_OK;
}

void destroy_graphs(nimbus_engine* e)
{
    for (int part = 0; part < 2; ++part)
    {
        if (e->exec[part]) cudaGraphExecDestroy(e->exec[part]);
        if (e->graph[part]) cudaGraphDestroy(e->graph[part]);
        e->exec[part] = nullptr;
        e->graph[part] = nullptr;
        for (auto& c : e->exec_cache[part]) cudaGraphExecDestroy(c.exec);
        e->exec_cache[part].clear();
    }
}

constexpr size_t kExecCache = 8;  // instantiated topologies kept per part

// Topology key of a captured graph: its node and edge counts and, in node
// order, each node's type and, for kernel nodes, the kernel.  Graphs with
// equal keys are captured by the same launch sequence; an update that the
// runtime refuses all the same only costs the instantiation it would have
// taken anyway.
uint64_t graph_topology_key(cudaGraph_t g)
{
    uint64_t h = 1469598103934665603ull;  // FNV-1a
    auto mix = [&](uint64_t v) {
        for (int b = 0; b < 8; ++b)
        {
            h ^= (v >> (8 * b)) & 0xffu;
            h *= 1099511628211ull;
        }
    };
    size_t n = 0, edges = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
    if (cudaGraphGetEdges(g, nullptr, nullptr, &edges) != cudaSuccess) return 0;
    mix(n);
    mix(edges);
    std::vector<cudaGraphNode_t> nodes(n);
    if (n && cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    for (cudaGraphNode_t node : nodes)
    {
        cudaGraphNodeType type;
        if (cudaGraphNodeGetType(node, &type) != cudaSuccess) return 0;
        mix(static_cast<uint64_t>(type));
        if (type == cudaGraphNodeTypeKernel)
        {
            cudaKernelNodeParams kp{};
            if (cudaGraphKernelNodeGetParams(node, &kp) != cudaSuccess) return 0;
            mix(reinterpret_cast<uint64_t>(kp.func));
        }
    }
    return h == 0 ? 1 : h;
}

// Makes exec (instantiated from a graph of the same key) run g; false when the
// runtime refuses the update.
bool update_exec(cudaGraphExec_t exec, cudaGraph_t g)
{
    cudaGraphExecUpdateResultInfo info{};
    if (cudaGraphExecUpdate(exec, g, &info) == cudaSuccess) return true;
    (void)cudaGetLastError();  // a refused update is not an error of the engine
    return false;
}

void park_exec(nimbus_engine* e, int part, uint64_t key, cudaGraphExec_t exec)
{
    auto& cache = e->exec_cache[part];
    if (key == 0)
    {
        cudaGraphExecDestroy(exec);
        return;
    }
    if (cache.size() >= kExecCache)
    {
        size_t oldest = 0;
        for (size_t i = 1; i < cache.size(); ++i)
            if (cache[i].used < cache[oldest].used) oldest = i;
        cudaGraphExecDestroy(cache[oldest].exec);
        cache.erase(cache.begin() + static_cast<std::ptrdiff_t>(oldest));
    }
    cache.push_back({key, exec, ++e->exec_clock});
}

cudaGraphExec_t take_exec(nimbus_engine* e, int part, uint64_t key)
{
    auto& cache = e->exec_cache[part];
    for (size_t i = 0; i < cache.size(); ++i)
        if (cache[i].key == key)
        {
            cudaGraphExec_t x = cache[i].exec;
            cache.erase(cache.begin() + static_cast<std::ptrdiff_t>(i));
            return x;
        }
    return nullptr;
}

nimbus_status rebuild_table(nimbus_engine* e)
{
    nimbus_cuda_context* ctx = e->ctx;
    NB_TRY(sync_table_to_host(e));
    const size_t n = e->slots.size();
    // Lanes: members placed largest first on the least loaded lane (work =
    // cells x (substeps + 3), the large step's cost in substep-equivalents),
    // then each lane sorted by substep count, longest first.
    const size_t lanes = std::min<size_t>(n, static_cast<size_t>(std::max(1, e->lane_target)));
    std::vector<int> by_work(n);
    for (size_t i = 0; i < n; ++i) by_work[i] = static_cast<int>(i);
    auto work = [&](int i) {
        return static_cast<double>(e->slots[i].m.items[kItemCells]) * (e->slots[i].m.n_substeps + 3);
    };
    std::stable_sort(by_work.begin(), by_work.end(), [&](int a, int b) { return work(a) > work(b); });
    std::vector<std::vector<int>> members(lanes);
    std::vector<double> load(lanes, 0.0);
    for (int i : by_work)
    {
        const size_t k = static_cast<size_t>(std::min_element(load.begin(), load.end()) - load.begin());
        members[k].push_back(i);
        load[k] += work(i);
    }
    e->order.clear();
    e->lanes.assign(lanes, Lane());
    size_t pre = 0;
    for (size_t k = 0; k < lanes; ++k)
    {
        auto& m = members[k];
        std::stable_sort(m.begin(), m.end(), [&](int a, int b) {
            const int na = e->slots[a].m.n_substeps, nb = e->slots[b].m.n_substeps;
            return na > nb || (na == nb && a < b);
        });
        Lane& L = e->lanes[k];
        L.first = static_cast<int>(e->order.size());
        L.members = static_cast<int>(m.size());
        L.prefix_first = pre;
        pre += static_cast<size_t>(kItemKinds) * (m.size() + 1);
        e->order.insert(e->order.end(), m.begin(), m.end());
    }
    NB_TRY(ensure_lane_streams(e, lanes ? lanes - 1 : 0));
    if (n > e->table_cap)
    {
        const size_t cap = std::max<size_t>(n, 2 * e->table_cap);
        NB_CUDA(ctx, cudaStreamSynchronize(e->stream));  // enqueued steps still read the old table
        if (e->d_table) cudaFree(e->d_table);
        e->d_table = nullptr;
        e->table_cap = 0;
        NB_CUDA(ctx, cudaMalloc(&e->d_table, sizeof(EngineMember) * cap));
        e->table_cap = cap;
    }
    if (pre > e->prefix_cap)
    {
        NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
        if (e->d_prefix) cudaFree(e->d_prefix);
        e->d_prefix = nullptr;
        e->prefix_cap = 0;
        NB_CUDA(ctx, cudaMalloc(&e->d_prefix, sizeof(long long) * (pre + 64)));
        e->prefix_cap = pre + 64;
    }
    long long image = 0;  // state-image offsets in admission order
    for (auto& slot : e->slots)
    {
        slot.m.image_offset = image;
        image += 9LL * slot.m.items[kItemCells];
        // Marching tiles: (j, k) blocks of one CTA times i-chunks of march_len planes.
        EngineMember& M = slot.m;
        const int blocks = (M.F.d.ny * M.F.d.nz + kEngineBlock - 1) / kEngineBlock;
        const int chunks = (M.F.d.nx + e->march_len - 1) / e->march_len;
        M.march_len = e->march_len;
        M.march_blocks = blocks;
        M.items[kItemMarch] = blocks * kEngineBlock * chunks;
    }
    std::vector<EngineMember> host(n);
    for (size_t r = 0; r < n; ++r) host[r] = e->slots[e->order[r]].m;
    e->prefix.assign(pre, 0);
    const int tile = kEngineBlock * kItemsPerThread;
    for (Lane& L : e->lanes)
    {
        const EngineMember* rows = host.data() + L.first;
        int max_n = 0;
        for (int r = 0; r < L.members; ++r) max_n = std::max(max_n, rows[r].n_substeps);
        for (int k = 0; k < kItemKinds; ++k)
        {
            long long* p = e->prefix.data() + L.prefix_first + static_cast<size_t>(k) * (L.members + 1);
            p[0] = 0;
            for (int r = 0; r < L.members; ++r) p[r + 1] = p[r] + (rows[r].items[k] + tile - 1) / tile;
        }
        L.closing = false;
        for (int r = 0; r < L.members; ++r) L.closing = L.closing || rows[r].close_step != 0;
        L.active.assign(max_n, 0);
        for (int st = 0; st < max_n; ++st)
        {
            int a = 0;
            while (a < L.members && rows[a].n_substeps > st) ++a;
            L.active[st] = a;
        }
    }
    if (n)
    {
        // Stream-ordered after every enqueued step (the host views already
        // include their rotations); pageable sources are staged before the
        // calls return, so the vectors may go.
        NB_CUDA(ctx, cudaMemcpyAsync(e->d_table, host.data(), sizeof(EngineMember) * n, cudaMemcpyHostToDevice,
                                     e->stream));
        NB_CUDA(ctx, cudaMemcpyAsync(e->d_prefix, e->prefix.data(), sizeof(long long) * pre,
                                     cudaMemcpyHostToDevice, e->stream));
    }
    e->table_current = true;
    e->graphs_stale = true;
    // The acoustic speed scan's per-row maxima (device) and their pinned host copy.
    e->resolving = false;
    for (const auto& slot : e->slots) e->resolving = e->resolving || slot.desc.resolve_substeps;
    e->scan_pending = false;  // rows moved: an earlier scan no longer matches them
    if (e->resolving && n > e->c2_cap)
    {
        NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
        if (e->d_c2) cudaFree(e->d_c2);
        if (e->h_c2) cudaFreeHost(e->h_c2);
        e->d_c2 = nullptr;
        e->h_c2 = nullptr;
        e->c2_cap = 0;
        const size_t cap = std::max<size_t>(2 * n, 64);
        NB_CUDA(ctx, cudaMalloc(&e->d_c2, cap * sizeof(unsigned long long)));
        NB_CUDA(ctx, cudaMallocHost(&e->h_c2, cap * sizeof(unsigned long long)));
        e->c2_cap = cap;
    }
    if (e->resolving && !e->scan_done) NB_CUDA(ctx, cudaEventCreateWithFlags(&e->scan_done, cudaEventDisableTiming));
    e->dirty = false;
    return NIMBUS_OK;
}

// The acoustic speed scan outside a step (after admissions, writes or
// uploads changed the state the next step starts from): every member's
// maximum (gamma p) / rho into d_c2 by table row, copied to the pinned h_c2.
// Inside a step the scan is part 1's last launch.
nimbus_status enqueue_scan(nimbus_engine* e)
{
    nimbus_cuda_context* ctx = e->ctx;
    const size_t n = e->order.size();
    NB_CUDA(ctx, cudaMemsetAsync(e->d_c2, 0, n * sizeof(unsigned long long), e->stream));
    for (const Lane& L : e->lanes)
    {
        const long long tiles = tiles_of(e, L, kItemScan, L.members);
        if (tiles <= 0) continue;
        engine_sound_speed_kernel<<<engine_grid(e, reinterpret_cast<const void*>(engine_sound_speed_kernel), tiles),
                                    kEngineBlock, 0, e->stream>>>(e->d_table + L.first, prefix_of(e, L, kItemScan),
                                                                  tiles, e->d_c2 + L.first);
        ctx->launches += 1;
    }
    NB_CUDA(ctx, cudaGetLastError());
    NB_CUDA(ctx, cudaMemcpyAsync(e->h_c2, e->d_c2, n * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                                 e->stream));
    NB_CUDA(ctx, cudaEventRecord(e->scan_done, e->stream));
    e->scan_pending = true;
    return NIMBUS_OK;
}

// Substep counts of the resolve_substeps members for the step whose part 0 is
// enqueued (the reference's choose_runtime_timestep + resolve_substep_count
// before every step): waits for the pending scan of that step's starting
// state and gives each member whose count changed its new count and substep
// parameters (the table and graphs are then rebuilt).
nimbus_status apply_scan(nimbus_engine* e)
{
    nimbus_cuda_context* ctx = e->ctx;
    NB_CUDA(ctx, cudaEventSynchronize(e->scan_done));
    e->scan_pending = false;
    for (size_t r = 0; r < e->order.size(); ++r)
    {
        MemberSlot& slot = e->slots[static_cast<size_t>(e->order[r])];
        if (!slot.desc.resolve_substeps) continue;
        // 0: every cell failed the scan (flagged in the member's status word);
        // the member keeps its count.
        if (e->h_c2[r] == 0) continue;
        const double c = std::max(std::sqrt(ordered_bits_to_double(e->h_c2[r])), slot.c_base);
        const double spacing = std::min({slot.desc.dx, slot.desc.dy, slot.desc.dz});
        const int count = resolve_substep_count(slot.desc.dt, c, spacing, slot.desc.n_substeps);
        if (count < 1 || count > 4096)
            return fail(ctx, NIMBUS_ERR_UNSUPPORTED, "a member's acoustic CFL needs an unsupported substep count");
        if (count == slot.m.n_substeps) continue;
        if (!e->dirty) NB_TRY(sync_table_to_host(e));  // exact host views before editing a row
        nimbus_member_desc d = slot.desc;
        d.n_substeps = count;
        fill_params(slot.m, &d);
        e->dirty = true;
    }
    return NIMBUS_OK;
}

int enqueue_lane(nimbus_engine* e, int lane, cudaStream_t st, int part)
{
    if (e->ctx->precision == NIMBUS_PRECISION_FP32) return nimbus_fp32::engine_enqueue(e, lane, st, part);
    return enqueue_step<RefPolicy, false>(e, lane, st, part);
}

// Part `part` of one large step of every lane: lanes 1.. forked from `st`
// onto their own streams and joined back (inside a capture this builds
// parallel branches of one graph).  Part 1 with resolving members ends with
// the copy of the scan maxima to the host.  Returns the launch count.
int enqueue(nimbus_engine* e, cudaStream_t st, int part)
{
    const size_t lanes = e->lanes.size();
    if (lanes == 0) return 0;
    const bool scan = part == 1 && e->resolving;
    if (scan) cudaMemsetAsync(e->d_c2, 0, e->order.size() * sizeof(unsigned long long), st);
    int count = 0;
    if (lanes == 1) count = enqueue_lane(e, 0, st, part);
    else
    {
        cudaEventRecord(e->fork, st);
        for (size_t k = 1; k < lanes; ++k)
        {
            cudaStream_t ls = e->lane_streams[k - 1];
            cudaStreamWaitEvent(ls, e->fork, 0);
            count += enqueue_lane(e, static_cast<int>(k), ls, part);
            cudaEventRecord(e->lane_done[k - 1], ls);
        }
        count += enqueue_lane(e, 0, st, part);
        for (size_t k = 1; k < lanes; ++k) cudaStreamWaitEvent(st, e->lane_done[k - 1], 0);
    }
    if (scan)
        cudaMemcpyAsync(e->h_c2, e->d_c2, e->order.size() * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st);
    return count;
}

// Captures both parts of a step.  An admission or retirement that keeps the
// graphs' shape (lanes, launches per lane) only changes launch parameters
// (grid sizes, table rows, tile counts): the instantiated graph is updated in
// place (cudaGraphExecUpdate) rather than instantiated again.
nimbus_status build_graphs(nimbus_engine* e)
{
    nimbus_cuda_context* ctx = e->ctx;
    cudaStream_t st = e->stream;
    if (e->built_precision != ctx->precision) destroy_graphs(e);
    for (int part = 0; part < 2; ++part)
    {
        NB_CUDA(ctx, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int launches = enqueue(e, st, part);
        cudaGraph_t g = nullptr;
        const cudaError_t end = cudaStreamEndCapture(st, &g);
        if (end != cudaSuccess) return cuda_fail(ctx, end, "engine graph capture");
        const uint64_t key = graph_topology_key(g);
        bool updated = false;
        if (e->exec[part] && key != 0 && e->exec_key[part] == key) updated = update_exec(e->exec[part], g);
        if (!updated && e->exec[part])
        {
            park_exec(e, part, e->exec_key[part], e->exec[part]);  // its topology may come back
            e->exec[part] = nullptr;
        }
        if (!updated && key != 0)
        {
            if (cudaGraphExec_t x = take_exec(e, part, key))
            {
                if (update_exec(x, g))
                {
                    e->exec[part] = x;
                    updated = true;
                }
                else
                    cudaGraphExecDestroy(x);
            }
        }
        if (!updated)
        {
            cudaGraphExec_t x = nullptr;
            const cudaError_t inst = cudaGraphInstantiate(&x, g, 0);
            if (inst != cudaSuccess)
            {
                cudaGraphDestroy(g);
                return cuda_fail(ctx, inst, "engine graph instantiation");
            }
            e->exec[part] = x;
            ++e->graph_instantiations;
        }
        else
            ++e->graph_updates;
        e->exec_key[part] = key;
        if (e->graph[part]) cudaGraphDestroy(e->graph[part]);
        e->graph[part] = g;
        e->launches_part[part] = launches;
    }
    e->graphs_stale = false;
    e->launches_per_step = e->launches_part[0] + e->launches_part[1];
    e->built_precision = ctx->precision;
    return NIMBUS_OK;
}

// Enqueues part `part` of one step (graph or eager launches).
nimbus_status launch_part(nimbus_engine* e, bool graph, int part)
{
    nimbus_cuda_context* ctx = e->ctx;
    if (graph) NB_CUDA(ctx, cudaGraphLaunch(e->exec[part], e->stream));
    else e->launches_part[part] = enqueue(e, e->stream, part);
    ctx->launches += static_cast<uint64_t>(e->launches_part[part]);
    return NIMBUS_OK;
}

MemberSlot* find_slot(nimbus_engine* e, int id, size_t* index = nullptr)
{
    for (size_t i = 0; i < e->slots.size(); ++i)
        if (e->slots[i].id == id)
        {
            if (index) *index = i;
            return &e->slots[i];
        }
    return nullptr;
}

size_t image_bytes_of(const nimbus_engine* e)
{
    size_t floats = 0;
    for (const auto& slot : e->slots) floats += 9ull * static_cast<size_t>(slot.m.items[kItemCells]);
    return floats * sizeof(float);
}

// Table current, staging allocated: the common part of the image copies.
nimbus_status prepare_image(nimbus_engine* e, size_t* bytes)
{
    nimbus_cuda_context* ctx = e->ctx;
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    if (e->dirty) NB_TRY(rebuild_table(e));
    *bytes = image_bytes_of(e);
    if (*bytes > e->image_cap)
    {
        NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
        if (e->d_image) cudaFree(e->d_image);
        e->d_image = nullptr;
        e->image_cap = 0;
        NB_CUDA(ctx, cudaMalloc(&e->d_image, *bytes));
        e->image_cap = *bytes;
    }
    return NIMBUS_OK;
}

void launch_image(nimbus_engine* e, int gather, float* image = nullptr)
{
    for (const Lane& L : e->lanes)
    {
        const long long tiles = tiles_of(e, L, kItemCells, L.members);
        if (tiles <= 0) continue;
        engine_image_kernel<<<engine_grid(e, reinterpret_cast<const void*>(engine_image_kernel), tiles), kEngineBlock,
                              0, e->stream>>>(e->d_table + L.first, prefix_of(e, L, kItemCells), tiles,
                                              image ? image : e->d_image, gather);
        e->ctx->launches += 1;
    }
}

const char* check_state(const nimbus_member_state* s)
{
    if (!s) return "state is null";
    if (!s->u || !s->v || !s->w || !s->rho || !s->p || !s->theta || !s->qv || !s->qc || !s->qr)
        return "a state array is null";
    return nullptr;
}

}  // namespace

int nimbus_engine_detail::launch_microphysics(nimbus_engine* e, cudaStream_t st, const nimbus::EngineMember* table,
                                              const long long* prefix, long long tiles)
{
    if (tiles <= 0) return 0;
    nimbus_cuda_context* ctx = e->ctx;
    LaunchTimer t(ctx, st, NIMBUS_KERNEL_MICROPHYSICS);
    if (ctx->precision == NIMBUS_PRECISION_FP32)
        engine_microphysics_eos_kernel<true>
            <<<engine_grid(e, reinterpret_cast<const void*>(engine_microphysics_eos_kernel<true>), tiles),
               kEngineBlock, 0, st>>>(table, prefix, tiles);
    else
        engine_microphysics_eos_kernel<false>
            <<<engine_grid(e, reinterpret_cast<const void*>(engine_microphysics_eos_kernel<false>), tiles),
               kEngineBlock, 0, st>>>(table, prefix, tiles);
    return 1;
}

extern "C" {

nimbus_status nimbus_cuda_engine_create(nimbus_cuda_context* ctx, nimbus_engine** out)
{
    if (!ctx || !out) return NIMBUS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    // Member arenas come from the device's default memory pool (stream-ordered
    // allocation); keep what retirements free there, so that admissions reuse
    // it without mapping memory again.  free_device_bytes counts it as free.
    {
        cudaMemPool_t pool = nullptr;
        NB_CUDA(ctx, cudaDeviceGetDefaultMemPool(&pool, ctx->device));
        unsigned long long keep = ~0ull;
        NB_CUDA(ctx, cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    }
    auto* e = new (std::nothrow) nimbus_engine();
    if (!e) return fail(ctx, NIMBUS_ERR_OUT_OF_MEMORY, "engine allocation failed");
    e->ctx = ctx;
    const cudaError_t err = cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking);
    if (err != cudaSuccess)
    {
        delete e;
        return cuda_fail(ctx, err, "engine stream");
    }
    *out = e;
    return NIMBUS_OK;
}

void nimbus_cuda_engine_destroy(nimbus_engine* e)
{
    if (!e) return;
    cudaStreamSynchronize(e->stream);
    destroy_graphs(e);
    if (e->scan_done) cudaEventDestroy(e->scan_done);
    for (auto& s : e->slots)
        if (s.arena) cudaFreeAsync(s.arena, e->stream);
    cudaStreamSynchronize(e->stream);
    if (e->d_table) cudaFree(e->d_table);
    if (e->d_prefix) cudaFree(e->d_prefix);
    if (e->d_image) cudaFree(e->d_image);
    if (e->d_centre) cudaFree(e->d_centre);
    if (e->d_c2) cudaFree(e->d_c2);
    if (e->h_c2) cudaFreeHost(e->h_c2);
    for (cudaStream_t ls : e->lane_streams) cudaStreamDestroy(ls);
    for (cudaEvent_t ev : e->lane_done) cudaEventDestroy(ev);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->stream) cudaStreamDestroy(e->stream);
    delete e;
}

size_t nimbus_cuda_engine_member_bytes(const nimbus_member_desc* desc)
{
    if (!desc || check_desc(desc)) return 0;
    return arena_layout(desc).total;
}

nimbus_status nimbus_cuda_engine_admit(nimbus_engine* e, const nimbus_member_desc* desc,
                                       const nimbus_member_state* initial, size_t reserve_bytes, int* member_id)
{
    if (!e || !desc || !member_id) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    if (const char* why = check_desc(desc)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    if (const char* why = check_state(initial)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    const ArenaLayout L = arena_layout(desc);
    size_t free_bytes = 0;
    NB_TRY(free_device_bytes(ctx, &free_bytes));
    if (L.total + reserve_bytes > free_bytes)
        return fail(ctx, NIMBUS_ERR_OUT_OF_MEMORY, "member does not fit the free device memory");

    // A resolve_substeps member starts with the count of its base columns'
    // sound speed; the device scan of its initial state, which runs before
    // its first step, settles the count of that step (admission does no pass
    // over the state on the host).
    nimbus_member_desc first = *desc;
    double c_base = 0.0;
    if (desc->resolve_substeps)
    {
        const double gamma = kCpd / (kCpd - kRd);
        for (int k = 0; k < desc->nz; ++k)
            if (!finite_positive(desc->p0_base[k]) || !finite_positive(desc->rho0_base[k]))
                return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "base pressure and density must be positive and finite");
        c_base = base_sound_speed(desc->p0_base, desc->rho0_base, desc->nz, gamma);
        const int count = resolve_substep_count(desc->dt, c_base, std::min({desc->dx, desc->dy, desc->dz}),
                                                desc->n_substeps);
        if (count < 1 || count > 4096)
            return fail(ctx, NIMBUS_ERR_UNSUPPORTED, "the acoustic CFL needs an unsupported substep count");
        first.n_substeps = count;
    }

    MemberSlot slot;
    slot.id = e->next_id;
    slot.desc = *desc;
    slot.c_base = c_base;
    slot.desc.rho0_base = slot.desc.p0_base = slot.desc.qv0_base = slot.desc.u0_base = slot.desc.v0_base = nullptr;
    slot.desc.sponge = nullptr;
    slot.bytes = L.total;
    {
        // Stream-ordered: the arena is ready for everything later on the
        // engine stream, and admission does not wait for enqueued steps.
        const cudaError_t err = cudaMallocAsync(&slot.arena, L.total, e->stream);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "member allocation");
    }
    char* base = static_cast<char*>(slot.arena);
    const size_t field = align_up(L.cells * sizeof(float));
    auto fld = [&](size_t off, int idx) { return reinterpret_cast<float*>(base + off + idx * field); };
    EngineMember& M = slot.m;
    M = EngineMember{};
    M.u = fld(L.off_state, 0);
    M.v = fld(L.off_state, 1);
    M.w = fld(L.off_state, 2);
    M.rho = fld(L.off_state, 3);
    M.rho_alt = fld(L.off_state, 4);
    M.p = fld(L.off_state, 5);
    M.theta = fld(L.off_state, 6);
    M.qv = fld(L.off_state, 7);
    M.qc = fld(L.off_state, 8);
    M.qr = fld(L.off_state, 9);
    M.qr_alt = fld(L.off_state, 10);
    M.rho_begin = fld(L.off_ctxt, 0);
    M.mfx = fld(L.off_ctxt, 1);
    M.mfy = fld(L.off_ctxt, 2);
    M.mfz = fld(L.off_ctxt, 3);
    M.wave = reinterpret_cast<float*>(base + L.off_wave);
    M.sf = reinterpret_cast<float*>(base + L.off_sf);
    M.rl = reinterpret_cast<float*>(base + L.off_rl);
    M.q4 = reinterpret_cast<float*>(base + L.off_q4);
    M.k1 = reinterpret_cast<float*>(base + L.off_k1);
    M.xs = reinterpret_cast<float*>(base + L.off_xs);
    M.eos = reinterpret_cast<float*>(base + L.off_eos);
    M.status = reinterpret_cast<unsigned*>(base + L.off_status);
    double* prof = reinterpret_cast<double*>(base + L.off_prof);
    const size_t nz = static_cast<size_t>(desc->nz);
    M.rho0 = prof;
    M.p0 = prof + nz;
    M.qv0 = prof + 2 * nz;
    M.u0 = prof + 3 * nz;
    M.v0 = prof + 4 * nz;
    float2* dp0 = reinterpret_cast<float2*>(base + L.off_dp0);
    float4* eos0 = reinterpret_cast<float4*>(base + L.off_eos0);
    M.dp0 = dp0;
    M.eos0 = eos0;
    fill_params(M, &first);

    // Profiles, the split hydrostatic difference and the initial state.
    std::vector<double> hp(5 * nz, 0.0);
    std::memcpy(hp.data(), desc->rho0_base, nz * sizeof(double));
    std::memcpy(hp.data() + nz, desc->p0_base, nz * sizeof(double));
    std::memcpy(hp.data() + 2 * nz, desc->qv0_base, nz * sizeof(double));
    if (desc->u0_base) std::memcpy(hp.data() + 3 * nz, desc->u0_base, nz * sizeof(double));
    if (desc->v0_base) std::memcpy(hp.data() + 4 * nz, desc->v0_base, nz * sizeof(double));
    const size_t bytes = L.cells * sizeof(float);
    cudaError_t err = cudaSuccess;
    const float* src[9] = {initial->u, initial->v, initial->w, initial->rho, initial->p, initial->theta,
                           initial->qv, initial->qc, initial->qr};
    float* dst[9] = {M.u, M.v, M.w, M.rho, M.p, M.theta, M.qv, M.qc, M.qr};
    // Pageable sources are staged before each call returns (the caller's
    // arrays and the local vectors may go); pinned ones are read by the copy.
    for (int f = 0; f < 9 && err == cudaSuccess; ++f)
        err = cudaMemcpyAsync(dst[f], src[f], bytes, cudaMemcpyHostToDevice, e->stream);
    if (err == cudaSuccess)
        err = cudaMemcpyAsync(prof, hp.data(), hp.size() * sizeof(double), cudaMemcpyHostToDevice, e->stream);
    M.R = RelaxTables{};
    M.close_step = desc->final_closure != 0;
    if (err == cudaSuccess && desc->sponge)
    {
        const nimbus_sponge_desc* sp = desc->sponge;
        RelaxImage img;  // validated by check_desc
        build_relax_image(desc->nx, desc->ny, desc->nz, sp->alpha, sp->upper_w_alpha, sp->w_only_alpha, sp->u_ref,
                          sp->v_ref, sp->theta_ref, sp->lateral_width, sp->lateral_alpha, sp->do_upper, sp->do_w_only,
                          sp->do_lateral, sp->staggered, sp->implicit_mode, desc->dt, img);
        unsigned char* dev = reinterpret_cast<unsigned char*>(base + L.off_sponge);
        const size_t tab_bytes = img.tab.size() * sizeof(double);
        err = cudaMemcpyAsync(dev, img.tab.data(), tab_bytes, cudaMemcpyHostToDevice, e->stream);
        if (err == cudaSuccess)
            err = cudaMemcpyAsync(dev + tab_bytes, img.on.data(), img.on.size(), cudaMemcpyHostToDevice, e->stream);
        M.R = relax_tables(img, dev, desc->nz);
    }
    if (err == cudaSuccess)
    {
        // The same per-level kernel the per-operation path runs, so both forms
        // see identical base data.
        level_base_kernel<<<(desc->nz + 127) / 128, 128, 0, e->stream>>>(M.p0, desc->nz, M.gamma, dp0, eos0);
        err = cudaGetLastError();
    }
    if (err == cudaSuccess) err = cudaMemsetAsync(M.status, 0, sizeof(unsigned), e->stream);
    // Scratch that a step reads before writing: none, but keep it defined.
    if (err == cudaSuccess) err = cudaMemsetAsync(M.wave, 0, L.history * sizeof(float), e->stream);
    if (err != cudaSuccess)
    {
        cudaFreeAsync(slot.arena, e->stream);
        return cuda_fail(ctx, err, "member upload");
    }
    e->slots.push_back(slot);
    ++e->next_id;
    e->dirty = true;
    *member_id = slot.id;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_retire(nimbus_engine* e, int member_id)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    size_t index = 0;
    if (!find_slot(e, member_id, &index)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    // Freed in stream order after the enqueued steps that still use it; no wait.
    NB_CUDA(ctx, cudaFreeAsync(e->slots[index].arena, e->stream));
    e->slots.erase(e->slots.begin() + static_cast<long>(index));
    e->dirty = true;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_read_async(nimbus_engine* e, int member_id, const nimbus_member_state* out)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    if (const char* why = check_state(out)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    MemberSlot* s = find_slot(e, member_id);
    if (!s) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    if (!e->mirror_exact) NB_TRY(sync_table_to_host(e));
    const EngineMember& M = s->m;
    const size_t bytes = static_cast<size_t>(M.items[kItemCells]) * sizeof(float);
    const float* src[9] = {M.u, M.v, M.w, M.rho, M.p, M.theta, M.qv, M.qc, M.qr};
    float* dst[9] = {out->u, out->v, out->w, out->rho, out->p, out->theta, out->qv, out->qc, out->qr};
    for (int f = 0; f < 9; ++f)
        NB_CUDA(ctx, cudaMemcpyAsync(dst[f], src[f], bytes, cudaMemcpyDeviceToHost, e->stream));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_write_async(nimbus_engine* e, int member_id, const nimbus_member_state* in)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    e->scan_pending = false;  // the next step's starting state changes
    nimbus_cuda_context* ctx = e->ctx;
    if (const char* why = check_state(in)) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, why);
    MemberSlot* s = find_slot(e, member_id);
    if (!s) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    if (!e->mirror_exact) NB_TRY(sync_table_to_host(e));
    const EngineMember& M = s->m;
    const size_t bytes = static_cast<size_t>(M.items[kItemCells]) * sizeof(float);
    const float* src[9] = {in->u, in->v, in->w, in->rho, in->p, in->theta, in->qv, in->qc, in->qr};
    float* dst[9] = {M.u, M.v, M.w, M.rho, M.p, M.theta, M.qv, M.qc, M.qr};
    for (int f = 0; f < 9; ++f)
        NB_CUDA(ctx, cudaMemcpyAsync(dst[f], src[f], bytes, cudaMemcpyHostToDevice, e->stream));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_history_async(nimbus_engine* e, int member_id, unsigned fields, void* host_image)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    if (fields & ~static_cast<unsigned>(NIMBUS_HISTORY_CORE))
        return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown history field bit");
    if (fields && !host_image) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "host_image is null");
    MemberSlot* s = find_slot(e, member_id);
    if (!s) return fail(ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    if (!fields) return NIMBUS_OK;
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!e->mirror_exact) NB_TRY(sync_table_to_host(e));
    const EngineMember& M = s->m;
    const size_t need = 3 * static_cast<size_t>(M.items[kItemCells]) * sizeof(float);
    if (need > e->centre_cap)
    {
        NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
        if (e->d_centre) cudaFree(e->d_centre);
        e->d_centre = nullptr;
        e->centre_cap = 0;
        NB_CUDA(ctx, cudaMalloc(&e->d_centre, need));
        e->centre_cap = need;
    }
    const float* src[kHistoryFields] = {M.u, M.v, M.w, M.rho, M.p, M.theta, M.qv, M.qc, M.qr};
    return enqueue_history(ctx, e->stream, src, fields, nullptr, s->desc.nx, s->desc.ny, s->desc.nz, e->d_centre,
                           static_cast<float*>(host_image));
}

nimbus_status nimbus_cuda_engine_read(nimbus_engine* e, int member_id, const nimbus_member_state* out)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    NB_TRY(sync_table_to_host(e));
    NB_TRY(nimbus_cuda_engine_read_async(e, member_id, out));
    NB_CUDA(e->ctx, cudaStreamSynchronize(e->stream));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_write(nimbus_engine* e, int member_id, const nimbus_member_state* in)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    NB_TRY(sync_table_to_host(e));
    NB_TRY(nimbus_cuda_engine_write_async(e, member_id, in));
    NB_CUDA(e->ctx, cudaStreamSynchronize(e->stream));
    return NIMBUS_OK;
}

void* nimbus_cuda_engine_stream(const nimbus_engine* e) { return e ? static_cast<void*>(e->stream) : nullptr; }

size_t nimbus_cuda_engine_image_bytes(const nimbus_engine* e) { return e ? image_bytes_of(e) : 0; }

size_t nimbus_cuda_engine_image_offset(const nimbus_engine* e, int member_id)
{
    if (!e) return static_cast<size_t>(-1);
    size_t floats = 0;
    for (const auto& slot : e->slots)
    {
        if (slot.id == member_id) return floats * sizeof(float);
        floats += 9ull * static_cast<size_t>(slot.m.items[kItemCells]);
    }
    return static_cast<size_t>(-1);
}

nimbus_status nimbus_cuda_engine_upload_image_async(nimbus_engine* e, const void* host_image)
{
    if (!e || !host_image) return NIMBUS_ERR_INVALID_ARGUMENT;
    e->scan_pending = false;  // the next step's starting state changes
    nimbus_cuda_context* ctx = e->ctx;
    size_t bytes = 0;
    NB_TRY(prepare_image(e, &bytes));
    if (!bytes) return NIMBUS_OK;
    NB_CUDA(ctx, cudaMemcpyAsync(e->d_image, host_image, bytes, cudaMemcpyHostToDevice, e->stream));
    launch_image(e, 0);
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_download_image_async(nimbus_engine* e, void* host_image)
{
    if (!e || !host_image) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    size_t bytes = 0;
    NB_TRY(prepare_image(e, &bytes));
    if (!bytes) return NIMBUS_OK;
    launch_image(e, 1);
    NB_CUDA(ctx, cudaGetLastError());
    NB_CUDA(ctx, cudaMemcpyAsync(host_image, e->d_image, bytes, cudaMemcpyDeviceToHost, e->stream));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_step(nimbus_engine* e, int n_steps)
{
    if (!e || n_steps < 0) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    if (e->dirty) NB_TRY(rebuild_table(e));
    if (e->slots.empty() || n_steps == 0) return NIMBUS_OK;
    const bool graph = e->use_graph && !ctx->timing;
    if (graph && (!e->exec[0] || e->graphs_stale || e->built_precision != ctx->precision)) NB_TRY(build_graphs(e));
    for (int i = 0; i < n_steps; ++i)
    {
        // Part 0 needs no substep count; with resolving members the counts
        // are derived while it runs, from the scan of the step's starting
        // state (part 1 of the previous step, or an explicit scan).
        if (e->resolving && !e->scan_pending) NB_TRY(enqueue_scan(e));
        NB_TRY(launch_part(e, graph, 0));
        if (e->resolving)
        {
            NB_TRY(apply_scan(e));
            if (e->dirty)
            {
                // The new rows take effect after part 0, whose work is per
                // member and independent of the row order.
                NB_TRY(rebuild_table(e));
                if (graph) NB_TRY(build_graphs(e));
            }
        }
        NB_TRY(launch_part(e, graph, 1));
        if (e->resolving)
        {
            NB_CUDA(ctx, cudaEventRecord(e->scan_done, e->stream));
            e->scan_pending = true;
        }
        e->launches_per_step = e->launches_part[0] + e->launches_part[1];
        rotate_host_views(e, 1);
        e->table_current = e->mirror_exact;
    }
    NB_CUDA(ctx, cudaGetLastError());
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_member_status_async(nimbus_engine* e, int member_id, unsigned* host_flags)
{
    if (!e || !host_flags) return NIMBUS_ERR_INVALID_ARGUMENT;
    MemberSlot* s = find_slot(e, member_id);
    if (!s) return fail(e->ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    NB_CUDA(e->ctx, cudaMemcpyAsync(host_flags, s->m.status, sizeof(unsigned), cudaMemcpyDeviceToHost, e->stream));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_graph_builds(const nimbus_engine* e, uint64_t* instantiations, uint64_t* updates)
{
    if (!e || !instantiations || !updates) return NIMBUS_ERR_INVALID_ARGUMENT;
    *instantiations = e->graph_instantiations;
    *updates = e->graph_updates;
    return NIMBUS_OK;
}

// The engine autotuner: times candidate launch configurations on the
// resident members themselves and keeps the fastest.  The members' states are
// saved before (a device copy through the state-image kernel) and restored
// after, so tuning leaves every run where it was.
nimbus_status nimbus_cuda_engine_autotune(nimbus_engine* e, int steps, nimbus_engine_tuning* out)
{
    if (!e || !out || steps < 1 || steps > 100) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    NB_CUDA(ctx, cudaSetDevice(ctx->device));
    *out = nimbus_engine_tuning{};
    if (e->dirty) NB_TRY(rebuild_table(e));
    if (e->slots.empty())
    {
        out->lanes = e->lane_target;
        out->acoustic_form = e->acoustic_form;
        out->momentum_form = e->momentum_form;
        out->march = e->march_len;
        return NIMBUS_OK;
    }
    const size_t bytes = image_bytes_of(e);
    float* backup = nullptr;
    NB_CUDA(ctx, cudaMallocAsync(reinterpret_cast<void**>(&backup), bytes, e->stream));
    launch_image(e, 1, backup);  // save
    struct Candidate
    {
        int lanes, form, momentum, march;
    };
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    NB_CUDA(ctx, cudaEventCreate(&t0));
    NB_CUDA(ctx, cudaEventCreate(&t1));
    const Candidate saved{e->lane_target, e->acoustic_form, e->momentum_form, e->march_len};
    double best = 1e300;
    Candidate chosen = saved;
    nimbus_status status = NIMBUS_OK;
    int n = 0;
    // Times one candidate; false when a step failed (status set).
    auto trial = [&](const Candidate& c) {
        e->lane_target = c.lanes;
        e->acoustic_form = c.form;
        e->momentum_form = c.momentum;
        e->march_len = c.march;
        e->dirty = true;
        status = nimbus_cuda_engine_step(e, 1);  // builds the table and graphs, warms up
        if (status != NIMBUS_OK) return false;
        cudaEventRecord(t0, e->stream);
        status = nimbus_cuda_engine_step(e, steps);
        if (status != NIMBUS_OK) return false;
        cudaEventRecord(t1, e->stream);
        if (cudaEventSynchronize(t1) != cudaSuccess)
        {
            status = cuda_fail(ctx, cudaGetLastError(), "autotune timing");
            return false;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, t0, t1);
        const double per_step = ms / steps;
        if (n < NIMBUS_TUNING_CANDIDATES)
        {
            out->candidate_lanes[n] = c.lanes;
            out->candidate_form[n] = c.form;
            out->candidate_momentum_form[n] = c.momentum;
            out->candidate_march[n] = c.march;
            out->candidate_ms[n] = per_step;
            ++n;
        }
        if (per_step < best)
        {
            best = per_step;
            chosen = c;
        }
        // Restore the saved states for the next candidate (rows may have
        // moved with the lane split: the image follows admission order).
        launch_image(e, 0, backup);
        return true;
    };
    // Lanes first (constant-bank form), then every pair of pass forms at the
    // fastest lane count.
    const int members = static_cast<int>(e->slots.size());
    bool ok = true;
    for (int lanes : {1, 2, 4, 6, 8})
    {
        if (lanes > members && lanes != 1) continue;
        if (!(ok = trial({lanes, NIMBUS_ACOUSTIC_CONST, NIMBUS_ACOUSTIC_CONST, saved.march}))) break;
    }
    const int forms[] = {NIMBUS_ACOUSTIC_CONST, NIMBUS_ACOUSTIC_PAIR, NIMBUS_ACOUSTIC_TABLE, NIMBUS_ACOUSTIC_MARCH,
                         NIMBUS_ACOUSTIC_BULK, NIMBUS_ACOUSTIC_CMARCH};
    const int lanes = chosen.lanes;
    for (int cf : forms)
    {
        if (!ok) break;
        for (int mf : forms)
        {
            if (cf == NIMBUS_ACOUSTIC_CONST && mf == NIMBUS_ACOUSTIC_CONST) continue;  // timed above
            auto marching = [](int f) { return f == NIMBUS_ACOUSTIC_MARCH || f == NIMBUS_ACOUSTIC_CMARCH; };
            const int march = (marching(cf) || marching(mf)) ? 16 : saved.march;
            if (!(ok = trial({lanes, cf, mf, march}))) break;
        }
    }
    out->candidates = n;
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    const Candidate& keep = status == NIMBUS_OK ? chosen : saved;
    e->lane_target = keep.lanes;
    e->acoustic_form = keep.form;
    e->momentum_form = keep.momentum;
    e->march_len = keep.march;
    e->dirty = true;
    NB_TRY(rebuild_table(e));
    launch_image(e, 0, backup);  // every run back to its state before tuning
    e->scan_pending = false;     // the state changed
    NB_CUDA(ctx, cudaFreeAsync(backup, e->stream));
    NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
    NB_TRY(status);
    out->lanes = e->lane_target;
    out->acoustic_form = e->acoustic_form;
    out->momentum_form = e->momentum_form;
    out->march = e->march_len;
    out->ms_per_step = best;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_member_substeps(nimbus_engine* e, int member_id, int* n_substeps)
{
    if (!e || !n_substeps) return NIMBUS_ERR_INVALID_ARGUMENT;
    MemberSlot* s = find_slot(e, member_id);
    if (!s) return fail(e->ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    *n_substeps = s->m.n_substeps;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_synchronize(nimbus_engine* e)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    nimbus_cuda_context* ctx = e->ctx;
    NB_CUDA(ctx, cudaStreamSynchronize(e->stream));
    NB_TRY(sync_table_to_host(e));
    unsigned any = 0;
    for (auto& s : e->slots)
    {
        unsigned f = 0;
        NB_CUDA(ctx, cudaMemcpy(&f, s.m.status, sizeof(unsigned), cudaMemcpyDeviceToHost));
        any |= f;
    }
    if (any & kStatusInvalidEos)
    {
        // A refused projection keeps that member's pressure buffer: read the
        // true pointers back.
        e->mirror_exact = false;
        e->table_current = false;
        NB_TRY(sync_table_to_host(e));
    }
    if (any & kStatusNonfiniteMassFlux) return fail(ctx, NIMBUS_ERR_NONFINITE, "a member's retained mass flux went non-finite");
    if (any & kStatusNonfiniteTransport) return fail(ctx, NIMBUS_ERR_NONFINITE, "a member's transported scalar went non-finite");
    if (any & kStatusInvalidEos) return fail(ctx, NIMBUS_ERR_NONFINITE, "a member's EOS projection was refused");
    if (any & kStatusStagingTimeout) return fail(ctx, NIMBUS_ERR_CUDA, "a bulk-staged tile's copies did not complete");
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_member_status(nimbus_engine* e, int member_id, unsigned* flags)
{
    if (!e || !flags) return NIMBUS_ERR_INVALID_ARGUMENT;
    MemberSlot* s = find_slot(e, member_id);
    if (!s) return fail(e->ctx, NIMBUS_ERR_INVALID_ARGUMENT, "unknown member id");
    NB_CUDA(e->ctx, cudaStreamSynchronize(e->stream));
    NB_TRY(sync_table_to_host(e));
    NB_CUDA(e->ctx, cudaMemcpy(flags, s->m.status, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_set_graph(nimbus_engine* e, int enable)
{
    if (!e) return NIMBUS_ERR_INVALID_ARGUMENT;
    e->use_graph = enable != 0;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_set_lanes(nimbus_engine* e, int lanes)
{
    if (!e || lanes < 1) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (lanes != e->lane_target)
    {
        NB_TRY(sync_table_to_host(e));
        e->lane_target = lanes;
        e->dirty = true;
    }
    return NIMBUS_OK;
}

int nimbus_cuda_engine_lanes(const nimbus_engine* e) { return e ? static_cast<int>(e->lanes.size()) : 0; }

nimbus_status nimbus_cuda_engine_set_pass_forms(nimbus_engine* e, int continuity_form, int momentum_form)
{
    auto valid = [](int f) { return f >= NIMBUS_ACOUSTIC_TABLE && f <= NIMBUS_ACOUSTIC_CMARCH; };
    if (!e || !valid(continuity_form) || !valid(momentum_form)) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (continuity_form != e->acoustic_form || momentum_form != e->momentum_form)
    {
        NB_TRY(sync_table_to_host(e));
        e->acoustic_form = continuity_form;
        e->momentum_form = momentum_form;
        e->dirty = true;
    }
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_pass_forms(const nimbus_engine* e, int* continuity_form, int* momentum_form)
{
    if (!e || !continuity_form || !momentum_form) return NIMBUS_ERR_INVALID_ARGUMENT;
    *continuity_form = e->acoustic_form;
    *momentum_form = e->momentum_form;
    return NIMBUS_OK;
}

nimbus_status nimbus_cuda_engine_set_acoustic_form(nimbus_engine* e, int form)
{
    return nimbus_cuda_engine_set_pass_forms(e, form, form);
}

int nimbus_cuda_engine_acoustic_form(const nimbus_engine* e) { return e ? e->acoustic_form : -1; }

nimbus_status nimbus_cuda_engine_set_march(nimbus_engine* e, int planes)
{
    if (!e || planes < 1 || planes > 4096) return NIMBUS_ERR_INVALID_ARGUMENT;
    if (planes != e->march_len)
    {
        NB_TRY(sync_table_to_host(e));
        e->march_len = planes;
        e->dirty = true;
    }
    return NIMBUS_OK;
}

int nimbus_cuda_engine_march(const nimbus_engine* e) { return e ? e->march_len : -1; }

int nimbus_cuda_engine_members(const nimbus_engine* e) { return e ? static_cast<int>(e->slots.size()) : 0; }

int nimbus_cuda_engine_launches_per_step(const nimbus_engine* e) { return e ? e->launches_per_step : 0; }

}  // extern "C"
