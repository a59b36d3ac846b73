// Batched kernels of the member engine: one launch per phase advances that
// phase for every resident member.
//
// Work layout.  Each phase has an item kind (cells, west/east boundary rows,
// south/north rows, columns, KW78 history slots).  A member's items are cut
// into tiles of one block (blockDim.x items) and the members' tiles are laid
// end to end; prefix[kind][m] is the first tile of member m.  A persistent
// grid (a few CTAs per SM) strides over the tiles, so the member of a tile is
// uniform across its block and the per-member parameters are warp-broadcast
// loads from the member table.  Members are kept sorted by substep count
// (descending): at substep s the active members are a prefix of the table and
// the launch covers prefix[kind][active_s] tiles -- a ragged ensemble wastes
// no tiles on members that have finished their loop.
//
// Every item runs the same cell function as the per-operation kernels, with
// the member's pointers and parameters, so a member's arithmetic does not
// depend on the batch it shares.
#pragma once

#include "acoustic_kernels.cuh"
#include "acoustic_split.cuh"
#include "bulk_stage.cuh"
#include "physics_kernels.cuh"
#include "relaxation_kernels.cuh"
#include "slow_kernels.cuh"
#include "transport_kernels.cuh"

namespace nimbus
{

enum ItemKind
{
    kItemCells = 0,
    kItemRowsWE,     // ny*nz west/east boundary rows
    kItemRowsSN,     // nx*nz south/north boundary rows
    kItemColumns,    // nx*ny columns
    kItemHistory,    // (ny + nx)*nz KW78 history slots
    kItemPerimeter,  // 3 nx + 3 (ny - 3) columns the lateral closures write
    kItemMarch,      // rows along x: (j, k) positions in blocks times i-chunks (for_member_rows)
    kItemScan,       // cells in groups of kScanCells (engine_sound_speed_kernel)
    kItemKinds
};

constexpr int kScanCells = 8;  // cells one thread of the acoustic speed scan reads

constexpr int kEngineScalars = 4;  // theta, qv, qc, qr

struct __align__(16) EngineMember
{
    // Prognostic state and the two ping-pong partners (swapped on the device
    // at the end of the loop / after Kessler, see engine_swap_kernel).
    float *u, *v, *w, *rho, *rho_alt, *p, *theta, *qv, *qc, *qr, *qr_alt;
    // Retained transport context and per-step scratch.
    float *rho_begin, *mfx, *mfy, *mfz, *wave;
    float *sf;        // [3][cells] float4 face fluxes (one lane per scalar)
    float *rl;        // [cells] float4 limiter factors
    float *q4;        // [cells] float4 theta, qv, qc, qr before transport (written by the slow predictor)
    float *k1, *xs;   // [cells] float4 {u, v, w, p}: Heun k1 and predictor state
    float *eos;       // EOS candidate pressure
    unsigned* status; // this member's status word (kStatus* bits)
    const double *rho0, *p0, *qv0, *u0, *v0;
    const float2* dp0;
    const float4* eos0;
    FusedParams F;
    BoundaryParams B;
    TransportParams T;  // geometry and flags; the scalar pointers are taken from the fields above
    SlowParams S;
    KesslerParams K;
    double gamma;
    EosSeries eos_series;  // FP32 EOS coefficients binom(gamma, n)
    RelaxTables R;         // end-of-step sponge (all do_* zero: none)
    int close_step;        // end the step with the boundary closure
    int n_substeps;
    int microphysics;
    int march_len;         // i-planes one thread of a marching kernel advances (kItemMarch tiles)
    int march_blocks;      // blocks of blockDim.x (j, k) positions per i-chunk
    int items[kItemKinds];
    long long image_offset;  // first float of this member's block in the engine's state image
};

__device__ __forceinline__ const float* engine_scalar(const EngineMember& M, int s)
{
    return s == 0 ? M.theta : (s == 1 ? M.qv : (s == 2 ? M.qc : M.qr));
}

__device__ __forceinline__ float* engine_scalar_out(const EngineMember& M, int s)
{
    return s == 0 ? M.theta : (s == 1 ? M.qv : (s == 2 ? M.qc : M.qr));
}

// Items per thread in a tile: a tile is kItemsPerThread * blockDim.x
// consecutive items of one member (one item per thread measured fastest:
// more items per thread cost more registers than the shared member lookup
// saves).
constexpr int kItemsPerThread = 1;

// Calls fn(member, item) for every item of the first tiles of a kind.
template <class Fn>
__device__ __forceinline__ void for_member_items(const EngineMember* __restrict__ table,
                                                 const long long* __restrict__ prefix, long long tiles, int kind,
                                                 Fn&& fn)
{
    int m = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= prefix[m + 1]) ++m;
        const EngineMember& M = table[m];
        const int count = M.items[kind];
        const int base = (int)((t - prefix[m]) * (kItemsPerThread * blockDim.x)) + (int)threadIdx.x;
#pragma unroll
        for (int q = 0; q < kItemsPerThread; ++q)
        {
            const int item = base + q * (int)blockDim.x;
            if (item < count) fn(M, item);
        }
    }
}

// Calls fn(member, i0, i1, j, k, q) for the rows of the first tiles of
// kItemMarch: a member's (j, k) positions q = j nz + k are cut into blocks of
// blockDim.x (a warp reads 32 consecutive floats of a plane) and its x range
// into chunks of march_len planes; tile = chunk * march_blocks + block.  The
// thread of position q advances the cells (i0 .. i1-1, j, k) of its row.
template <class Fn>
__device__ __forceinline__ void for_member_rows(const EngineMember* __restrict__ table,
                                                const long long* __restrict__ prefix, long long tiles, Fn&& fn)
{
    int m = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= prefix[m + 1]) ++m;
        const EngineMember& M = table[m];
        const int local = (int)(t - prefix[m]);
        const int chunk = local / M.march_blocks;
        const int q = (local - chunk * M.march_blocks) * (int)blockDim.x + (int)threadIdx.x;
        const Dims d = M.F.d;
        if (q >= d.ny * d.nz) continue;
        int i, j, k;
        decompose(d, q, i, j, k);
        const int i0 = chunk * M.march_len;
        fn(M, i0, min(d.nx, i0 + M.march_len), j, k, q);
    }
}

// ---- Heun slow step -------------------------------------------------------

// Resident CTAs per SM of the slow Heun pair: the FP32 form at 5 (48
// registers; measured 3.14 -> 2.88 ms per ensemble step against 4), the
// reference-precision form at 4 (64 registers; its FP64 arithmetic spills
// heavily at 48).
#ifndef NIMBUS_SLOW_MINB
#define NIMBUS_SLOW_MINB 4
#endif
#ifndef NIMBUS_SLOW_MINB_F32
#define NIMBUS_SLOW_MINB_F32 5
#endif
template <class Policy>
constexpr int slow_min_blocks()
{
    return sizeof(typename Policy::real) == 4 ? NIMBUS_SLOW_MINB_F32 : NIMBUS_SLOW_MINB;
}
template <class Policy>
static __global__ void __launch_bounds__(256, NIMBUS_SLOW_MINB) engine_slow_predict_kernel(const EngineMember* __restrict__ table,
                                                                  const long long* __restrict__ prefix,
                                                                  long long tiles)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        slow_predict_packed<Policy>(M.S, M.u, M.v, M.w, M.rho, M.p, M.qv, M.qc, M.qr, M.rho0, M.qv0, M.u0, M.v0,
                                    reinterpret_cast<float4*>(M.k1), reinterpret_cast<float4*>(M.xs), c);
        // The transported scalars do not change before transport: keep their
        // interleaved copy for the transport kernels.
        reinterpret_cast<float4*>(M.q4)[c] = make_float4(M.theta[c], M.qv[c], M.qc[c], M.qr[c]);
    });
}

template <class Policy>
static __global__ void __launch_bounds__(256, NIMBUS_SLOW_MINB) engine_slow_correct_kernel(const EngineMember* __restrict__ table,
                                                                  const long long* __restrict__ prefix,
                                                                  long long tiles)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        slow_correct_packed<Policy>(M.S, reinterpret_cast<const float4*>(M.xs), M.rho, M.qv, M.qc, M.qr, M.rho0,
                                    M.qv0, M.u0, M.v0, reinterpret_cast<const float4*>(M.k1), M.u, M.v, M.w, M.p, c);
    });
}

// The Heun pair with the members' constants in the constant bank (the
// acoustic passes' reason, below: parameters read from the member table sit
// in registers, and the pair spilled at 64 registers).  Each lane's launch
// gets its members' SlowParams and every buffer that does not rotate as one
// __grid_constant__ parameter; density, pressure and rain, which rotate, are
// read from the table.
struct SlowConst
{
    SlowParams S;
    float *u, *v, *w, *theta, *qv, *qc;
    float4 *k1, *xs, *q4;
    const double *rho0, *qv0, *u0, *v0;
};

constexpr int kSlowConstMembers = 64;

struct SlowLaunch
{
    long long prefix[kSlowConstMembers + 1];  // first cell tile of each member
    SlowConst m[kSlowConstMembers];
};
static_assert(sizeof(SlowLaunch) <= 32000, "a kernel parameter block holds at most 32764 bytes");

template <class Policy>
static __global__ void __launch_bounds__(256, slow_min_blocks<Policy>()) engine_slow_predict_const_kernel(
    const __grid_constant__ SlowLaunch L, const EngineMember* __restrict__ table, long long tiles)
{
    int m = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= L.prefix[m + 1]) ++m;
        const SlowConst& A = L.m[m];
        const int c = (int)((t - L.prefix[m]) * blockDim.x) + (int)threadIdx.x;
        if (c >= A.S.d.cells()) continue;
        const EngineMember& M = table[m];
        slow_predict_packed<Policy>(A.S, A.u, A.v, A.w, M.rho, M.p, A.qv, A.qc, M.qr, A.rho0, A.qv0, A.u0, A.v0, A.k1,
                                    A.xs, c);
        A.q4[c] = make_float4(A.theta[c], A.qv[c], A.qc[c], M.qr[c]);
    }
}

template <class Policy>
static __global__ void __launch_bounds__(256, slow_min_blocks<Policy>()) engine_slow_correct_const_kernel(
    const __grid_constant__ SlowLaunch L, const EngineMember* __restrict__ table, long long tiles)
{
    int m = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= L.prefix[m + 1]) ++m;
        const SlowConst& A = L.m[m];
        const int c = (int)((t - L.prefix[m]) * blockDim.x) + (int)threadIdx.x;
        if (c >= A.S.d.cells()) continue;
        const EngineMember& M = table[m];
        slow_correct_packed<Policy>(A.S, A.xs, M.rho, A.qv, A.qc, M.qr, A.rho0, A.qv0, A.u0, A.v0, A.k1, A.u, A.v,
                                    A.w, M.p, c);
    }
}

// ---- Boundaries and KW78 seed ---------------------------------------------
//
// The density buffer substep s reads (written == false) or writes: substep s
// reads (s even ? rho : rho_alt) and writes the other one.  The boundary
// closure after substep s works on the written buffer; the refresh before the
// loop on the current density.

__device__ __forceinline__ float* engine_density(const EngineMember& M, int s, bool written)
{
    const bool even = (s & 1) == 0;
    return written ? (even ? M.rho_alt : M.rho) : (even ? M.rho : M.rho_alt);
}

static __global__ void __launch_bounds__(256) engine_bc_we_kernel(const EngineMember* __restrict__ table,
                                                           const long long* __restrict__ prefix, long long tiles,
                                                           int s, int refresh)
{
    for_member_items(table, prefix, tiles, kItemRowsWE, [&](const EngineMember& M, int r) {
        if (refresh == 2 && !M.close_step) return;  // the closing refresh only where asked
        BoundaryParams B = M.B;
        if (refresh) B.dt_rad = 0.0f;
        float* rho = refresh ? M.rho : engine_density(M, s, true);
        const int yz = B.d.ny * B.d.nz;
        bc_we_row(B, M.u, M.v, M.w, rho, M.p, M.wave, M.wave + yz, r);
    });
}

static __global__ void __launch_bounds__(256) engine_bc_sn_kernel(const EngineMember* __restrict__ table,
                                                           const long long* __restrict__ prefix, long long tiles,
                                                           int s, int refresh)
{
    for_member_items(table, prefix, tiles, kItemRowsSN, [&](const EngineMember& M, int r) {
        if (refresh == 2 && !M.close_step) return;
        BoundaryParams B = M.B;
        if (refresh) B.dt_rad = 0.0f;
        float* rho = refresh ? M.rho : engine_density(M, s, true);
        const int yz = B.d.ny * B.d.nz, xz = B.d.nx * B.d.nz;
        bc_sn_row(B, M.u, M.v, M.w, rho, M.p, M.wave + 2 * yz, M.wave + 2 * yz + xz, r);
    });
}

// refresh: 1 before the acoustic loop, 2 the closing refresh at the end of the
// step (members with close_step only).
static __global__ void __launch_bounds__(256) engine_bc_vertical_kernel(const EngineMember* __restrict__ table,
                                                                 const long long* __restrict__ prefix,
                                                                 long long tiles, int refresh)
{
    for_member_items(table, prefix, tiles, kItemColumns, [&](const EngineMember& M, int col) {
        if (refresh == 2 && !M.close_step) return;
        bc_vertical_column(M.B, M.u, M.v, M.w, col);
    });
}

// The vertical closure inside the acoustic loop, for the columns the lateral
// closures write (i in {0, nx-2, nx-1} or j in {0, ny-2, ny-1}); the momentum
// kernel closes every other column itself (momentum_cell, fuse_vertical).
// Item q: rows j = 0, ny-2, ny-1 for every i first, then i = 0, nx-2, nx-1
// for j = 1 .. ny-3.
static __global__ void __launch_bounds__(256) engine_bc_vertical_perimeter_kernel(
    const EngineMember* __restrict__ table, const long long* __restrict__ prefix, long long tiles)
{
    for_member_items(table, prefix, tiles, kItemPerimeter, [&](const EngineMember& M, int q) {
        const int nx = M.B.d.nx, ny = M.B.d.ny;
        int i, j;
        if (q < 3 * nx)
        {
            const int row = q / nx;
            i = q - row * nx;
            j = row == 0 ? 0 : ny - 3 + row;
        }
        else
        {
            const int r = q - 3 * nx, side = r % 3;
            j = 1 + r / 3;
            i = side == 0 ? 0 : nx - 3 + side;
        }
        bc_vertical_column(M.B, M.u, M.v, M.w, i * ny + j);
    });
}

static __global__ void __launch_bounds__(256) engine_seed_kernel(const EngineMember* __restrict__ table,
                                                          const long long* __restrict__ prefix, long long tiles)
{
    for_member_items(table, prefix, tiles, kItemHistory, [&](const EngineMember& M, int r) {
        seed_radiation_row(M.B.d, M.u, M.v, M.wave, r);
    });
}

// ---- Acoustic substep (split form, u/v/w in place, rho ping-pong) ---------

template <class Policy>
static __global__ void __launch_bounds__(256, 5) engine_continuity_kernel(const EngineMember* __restrict__ table,
                                                                const long long* __restrict__ prefix,
                                                                long long tiles, int s)
{
    const bool first = s == 0;
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        unsigned flags = 0;
        continuity_eos_cell<Policy>(M.F, engine_density(M, s, false), M.u, M.v, M.w, M.theta, M.rho0, M.eos0,
                                    engine_density(M, s, true), M.p, nullptr, M.mfx, M.mfy, M.mfz, c, flags, first,
                                    first ? M.rho_begin : nullptr);
        if (flags) atomicOr(M.status, flags);
    });
}

template <class Policy>
static __global__ void __launch_bounds__(256) engine_momentum_kernel(const EngineMember* __restrict__ table,
                                                              const long long* __restrict__ prefix, long long tiles,
                                                              int s)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        const int vertical = kFuseVertical | (M.B.bottom == kBottomNoSlip ? kFuseNoSlipBottom : 0) |
                             (M.B.top == kTopOpen ? kFuseOpenTop : 0);
        momentum_cell<Policy>(M.F, engine_density(M, s, true), M.p, M.p0, M.dp0, M.u, M.v, M.w, M.u, M.v, M.w, c,
                              vertical);
    });
}

// The same two passes marching along x (continuity_eos_march, momentum_march):
// one thread per (j, k) row segment of march_len cells.
#ifndef NIMBUS_MARCH_MINB
#define NIMBUS_MARCH_MINB 4
#endif
template <class Policy>
static __global__ void __launch_bounds__(256, NIMBUS_MARCH_MINB) engine_continuity_march_kernel(const EngineMember* __restrict__ table,
                                                                      const long long* __restrict__ prefix,
                                                                      long long tiles, int s)
{
    const bool first = s == 0;
    for_member_rows(table, prefix, tiles, [&](const EngineMember& M, int i0, int i1, int j, int k, int q) {
        unsigned flags = 0;
        continuity_eos_march<Policy>(M.F, engine_density(M, s, false), M.u, M.v, M.w, M.theta, M.rho0, M.eos0,
                                     engine_density(M, s, true), M.p, M.mfx, M.mfy, M.mfz, i0, i1, j, k, q, flags,
                                     first, first ? M.rho_begin : nullptr);
        if (flags) atomicOr(M.status, flags);
    });
}

template <class Policy>
static __global__ void __launch_bounds__(256) engine_momentum_march_kernel(const EngineMember* __restrict__ table,
                                                                    const long long* __restrict__ prefix,
                                                                    long long tiles, int s)
{
    for_member_rows(table, prefix, tiles, [&](const EngineMember& M, int i0, int i1, int j, int k, int q) {
        const int vertical = kFuseVertical | (M.B.bottom == kBottomNoSlip ? kFuseNoSlipBottom : 0) |
                             (M.B.top == kTopOpen ? kFuseOpenTop : 0);
        momentum_march<Policy>(M.F, engine_density(M, s, true), M.p, M.p0, M.dp0, M.u, M.v, M.w, i0, i1, j, k, q,
                               vertical);
    });
}

// ---- Acoustic passes with the members' constants in the constant bank ----
//
// A kernel that reads a member's parameters and pointers from the member
// table holds them in registers (about 50 values for continuity), which caps
// it at 5-6 resident CTAs per SM; the per-operation kernels take the same
// values from the constant bank as instruction operands and run at full
// occupancy with 32 registers.  So each launch of a lane gets its members'
// constants as one kernel parameter (__grid_constant__, the constant bank):
// the parameter blocks and every buffer that does not rotate.  The rotating
// buffers (density ping-pong, pressure) are read from the member table.
struct AcousticConst
{
    FusedParams F;
    float *u, *v, *w, *theta, *mfx, *mfy, *mfz, *rho_begin;
    unsigned* status;
    const double *rho0, *p0;
    const float2* dp0;
    const float4* eos0;
    int vertical;  // kFuse* bits of the momentum pass
    int march_len, march_blocks;  // the marching forms' row tiling (kItemMarch)
};

constexpr int kConstMembers = 64;  // members one launch can carry in its parameter

// The part of the parameter block every member of a launch holds alike (field
// bounds, EOS exponent and coefficients, frame velocity, top condition).  A
// member's own block is indexed by the member, so each value it supplies is an
// indexed constant load per cell; from here the kernel takes them as operands
// at fixed constant-bank offsets.
struct AcousticShared
{
    double gamma, frame_u, frame_v;
    float rho_min, rho_max, p_min, p_max, p_ref_fallback, frame_u_f, frame_v_f;
    int top_open;
    float eos_c[6];
};

inline AcousticShared acoustic_shared_of(const FusedParams& F)
{
    AcousticShared S{};
    S.gamma = F.gamma;
    S.frame_u = F.frame_u;
    S.frame_v = F.frame_v;
    S.rho_min = F.rho_min;
    S.rho_max = F.rho_max;
    S.p_min = F.p_min;
    S.p_max = F.p_max;
    S.p_ref_fallback = F.p_ref_fallback;
    S.frame_u_f = F.frame_u_f;
    S.frame_v_f = F.frame_v_f;
    S.top_open = F.top_open;
    for (int n = 0; n < 6; ++n) S.eos_c[n] = F.eos_c[n];
    return S;
}

// A member's block with the shared values read from S (bitwise equal to its
// own: the launch checks that before choosing a kernel that uses this).
__device__ __forceinline__ FusedParams with_shared(const FusedParams& F, const AcousticShared& S)
{
    FusedParams P = F;
    P.gamma = S.gamma;
    P.frame_u = S.frame_u;
    P.frame_v = S.frame_v;
    P.rho_min = S.rho_min;
    P.rho_max = S.rho_max;
    P.p_min = S.p_min;
    P.p_max = S.p_max;
    P.p_ref_fallback = S.p_ref_fallback;
    P.frame_u_f = S.frame_u_f;
    P.frame_v_f = S.frame_v_f;
    P.top_open = S.top_open;
    for (int n = 0; n < 6; ++n) P.eos_c[n] = S.eos_c[n];
    return P;
}

// Resident CTAs per SM the launch bounds ask for (continuity, momentum):
// measured on the 64-member ensemble, FP32, ms per step: natural register
// counts (48 / 36 registers) 14.41, 6 / 7 CTAs (40 / 36) 13.49, 8 / 8 (32
// registers, spilling) 14.49.
#ifndef NIMBUS_CONST_MINB
#define NIMBUS_CONST_MINB 6
#endif
#ifndef NIMBUS_CONST_MINB_MOM
#define NIMBUS_CONST_MINB_MOM 7
#endif

struct AcousticLaunch
{
    long long prefix[kConstMembers + 1];        // first cell tile of each member
    int prefix32[kConstMembers + 1];            // the same as 32-bit values (a lane's tiles fit)
    long long march_prefix[kConstMembers + 1];  // first row tile of each member (marching forms)
    AcousticConst m[kConstMembers];
    int bulk_sy4;                               // the members' largest nz rounded up to 4 (bulk-staged forms)
    AcousticShared shared;                      // every member's shared values (kernels with kShared)
};
static_assert(sizeof(AcousticLaunch) <= 32000, "a kernel parameter block holds at most 32764 bytes");

// kFirst: the first substep of the step (the retained fluxes are written, not
// accumulated, and the beginning density is kept).
// kShared: every member's shared values equal L.shared (acoustic_shared_of).
// Measured on the 64-member ensemble, FP32: continuity 3.58 -> 3.49 ms per
// step.  (Deriving the member's buffers from one pointer and the arena's field
// stride as well, two indexed loads instead of eight, spilled at the launch
// bound and took 3.78 ms; an inner loop over one member's tiles, so that its
// values could be loaded once per member, kept the loads per cell and took
// 3.58 ms.)
template <class Policy, bool kFirst, bool kShared>
static __global__ void __launch_bounds__(256, NIMBUS_CONST_MINB) engine_continuity_const_kernel(const __grid_constant__ AcousticLaunch L,
                                                                      const EngineMember* __restrict__ table,
                                                                      long long tiles, int s)
{
    constexpr bool first = kFirst;
    const bool even = (s & 1) == 0;
    int m = 0;
    const int ntiles = (int)tiles;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        while (t >= L.prefix32[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const int c = (t - L.prefix32[m]) * (int)blockDim.x + (int)threadIdx.x;
        if (c >= A.F.d.cells()) continue;
        const EngineMember& M = table[m];
        unsigned flags = 0;
        if constexpr (kShared)
        {
            const FusedParams F = with_shared(A.F, L.shared);
            continuity_eos_cell<Policy>(F, even ? M.rho : M.rho_alt, A.u, A.v, A.w, A.theta, A.rho0, A.eos0,
                                        even ? M.rho_alt : M.rho, M.p, nullptr, A.mfx, A.mfy, A.mfz, c, flags, first,
                                        first ? A.rho_begin : nullptr);
        }
        else
            continuity_eos_cell<Policy>(A.F, even ? M.rho : M.rho_alt, A.u, A.v, A.w, A.theta, A.rho0, A.eos0,
                                        even ? M.rho_alt : M.rho, M.p, nullptr, A.mfx, A.mfy, A.mfz, c, flags, first,
                                        first ? A.rho_begin : nullptr);
        if (flags) atomicOr(A.status, flags);
    }
}

template <class Policy>
static __global__ void __launch_bounds__(256, NIMBUS_CONST_MINB_MOM) engine_momentum_const_kernel(const __grid_constant__ AcousticLaunch L,
                                                                    const EngineMember* __restrict__ table,
                                                                    long long tiles, int s)
{
    const bool even = (s & 1) == 0;
    int m = 0;
    const int ntiles = (int)tiles;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        while (t >= L.prefix32[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const int c = (t - L.prefix32[m]) * (int)blockDim.x + (int)threadIdx.x;
        if (c >= A.F.d.cells()) continue;
        const EngineMember& M = table[m];
        momentum_cell<Policy>(A.F, even ? M.rho_alt : M.rho, M.p, A.p0, A.dp0, A.u, A.v, A.w, A.u, A.v, A.w, c,
                              A.vertical);
    }
}

// The marching passes with the members' constants in the constant bank.
#ifndef NIMBUS_CMARCH_MINB
#define NIMBUS_CMARCH_MINB 5
#endif
template <class Fn>
__device__ __forceinline__ void for_const_rows(const AcousticLaunch& L, const EngineMember* __restrict__ table,
                                               long long tiles, Fn&& fn)
{
    int m = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= L.march_prefix[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const int local = (int)(t - L.march_prefix[m]);
        const int chunk = local / A.march_blocks;
        const int q = (local - chunk * A.march_blocks) * (int)blockDim.x + (int)threadIdx.x;
        const Dims d = A.F.d;
        if (q >= d.ny * d.nz) continue;
        int i, j, k;
        decompose(d, q, i, j, k);
        const int i0 = chunk * A.march_len;
        fn(A, table[m], i0, min(d.nx, i0 + A.march_len), j, k, q);
    }
}

template <class Policy, bool kFirst>
static __global__ void __launch_bounds__(256, NIMBUS_CMARCH_MINB) engine_continuity_cmarch_kernel(
    const __grid_constant__ AcousticLaunch L, const EngineMember* __restrict__ table, long long tiles, int s)
{
    const bool even = (s & 1) == 0;
    for_const_rows(L, table, tiles, [&](const AcousticConst& A, const EngineMember& M, int i0, int i1, int j, int k,
                                        int q) {
        unsigned flags = 0;
        continuity_eos_march<Policy>(A.F, even ? M.rho : M.rho_alt, A.u, A.v, A.w, A.theta, A.rho0, A.eos0,
                                     even ? M.rho_alt : M.rho, M.p, A.mfx, A.mfy, A.mfz, i0, i1, j, k, q, flags, kFirst,
                                     kFirst ? A.rho_begin : nullptr);
        if (flags) atomicOr(A.status, flags);
    });
}

template <class Policy>
static __global__ void __launch_bounds__(256, NIMBUS_CMARCH_MINB) engine_momentum_cmarch_kernel(
    const __grid_constant__ AcousticLaunch L, const EngineMember* __restrict__ table, long long tiles, int s)
{
    const bool even = (s & 1) == 0;
    for_const_rows(L, table, tiles, [&](const AcousticConst& A, const EngineMember& M, int i0, int i1, int j, int k,
                                        int q) {
        momentum_march<Policy>(A.F, even ? M.rho_alt : M.rho, M.p, A.p0, A.dp0, A.u, A.v, A.w, i0, i1, j, k, q,
                               A.vertical);
    });
}

// The same two passes with two vertically adjacent cells per thread: a CTA
// of half a tile's threads takes cells c and c + 1 (c even) of each tile.  In
// a member whose nz is even the pair lies in one column, so the pair's index,
// neighbour offsets and member constants are formed once and every field's
// values at the pair (and at the pair shifted by +-sx or +-sy) are one 8-byte
// load (continuity_eos_kpair, momentum_kpair); in a member with an odd nz the
// thread advances its two cells one after the other.  Each cell's arithmetic
// is the one-cell form's.  ensemble_64, FP32, one lane: continuity
// 3.49 -> 3.30 ms per step against the one-cell constant-bank form (cells c
// and c + 128 per thread instead: 3.97), momentum 2.38 against 2.33 marching.
#ifndef NIMBUS_PAIR_MINB
#define NIMBUS_PAIR_MINB 8
#endif
#ifndef NIMBUS_PAIR_MINB_MOM
#define NIMBUS_PAIR_MINB_MOM 8
#endif

template <class Policy, bool kFirst, bool kShared>
static __global__ void __launch_bounds__(128, NIMBUS_PAIR_MINB) engine_continuity_pair_kernel(const __grid_constant__ AcousticLaunch L,
                                                                     const EngineMember* __restrict__ table,
                                                                     long long tiles, int s)
{
    const bool even = (s & 1) == 0;
    const int half = (int)blockDim.x;
    int m = 0;
    const int ntiles = (int)tiles;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        while (t >= L.prefix32[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const FusedParams F = kShared ? with_shared(A.F, L.shared) : A.F;
        const int n = F.d.cells();
        const int c0 = (t - L.prefix32[m]) * (2 * half) + 2 * (int)threadIdx.x;
        if (c0 >= n) continue;
        const EngineMember& M = table[m];
        const float* rho = even ? M.rho : M.rho_alt;
        float* rho_out = even ? M.rho_alt : M.rho;
        unsigned flags = 0;
        if ((F.d.nz & 1) == 0)
            continuity_eos_kpair<Policy>(F, rho, A.u, A.v, A.w, A.theta, A.rho0, A.eos0, rho_out, M.p, A.mfx, A.mfy,
                                         A.mfz, c0, flags, kFirst, kFirst ? A.rho_begin : nullptr);
        else
        {
            continuity_eos_cell<Policy>(F, rho, A.u, A.v, A.w, A.theta, A.rho0, A.eos0, rho_out, M.p, nullptr, A.mfx,
                                        A.mfy, A.mfz, c0, flags, kFirst, kFirst ? A.rho_begin : nullptr);
            if (c0 + 1 < n)
                continuity_eos_cell<Policy>(F, rho, A.u, A.v, A.w, A.theta, A.rho0, A.eos0, rho_out, M.p, nullptr,
                                            A.mfx, A.mfy, A.mfz, c0 + 1, flags, kFirst,
                                            kFirst ? A.rho_begin : nullptr);
        }
        if (flags) atomicOr(A.status, flags);
    }
}

template <class Policy>
static __global__ void __launch_bounds__(128, NIMBUS_PAIR_MINB_MOM) engine_momentum_pair_kernel(const __grid_constant__ AcousticLaunch L,
                                                                       const EngineMember* __restrict__ table,
                                                                       long long tiles, int s)
{
    const bool even = (s & 1) == 0;
    const int half = (int)blockDim.x;
    int m = 0;
    const int ntiles = (int)tiles;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x)
    {
        while (t >= L.prefix32[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const Dims d = A.F.d;
        const int n = d.cells();
        const int c0 = (t - L.prefix32[m]) * (2 * half) + 2 * (int)threadIdx.x;
        if (c0 >= n) continue;
        const EngineMember& M = table[m];
        const float* rho = even ? M.rho_alt : M.rho;
        if ((d.nz & 1) == 0)
            momentum_kpair<Policy>(A.F, rho, M.p, A.p0, A.dp0, A.u, A.v, A.w, c0, A.vertical);
        else
        {
            momentum_cell<Policy>(A.F, rho, M.p, A.p0, A.dp0, A.u, A.v, A.w, A.u, A.v, A.w, c0, A.vertical);
            if (c0 + 1 < n)
                momentum_cell<Policy>(A.F, rho, M.p, A.p0, A.dp0, A.u, A.v, A.w, A.u, A.v, A.w, c0 + 1, A.vertical);
        }
    }
}

// The same two passes with each tile's stencil data staged in shared memory
// by bulk copies (bulk_stage.cuh).  A tile is 256 consecutive cells of one
// member (one per thread); its stencils read, per field, the tile itself and
// the tile shifted by the neighbour strides, each a contiguous run of cells,
// so one CTA stages a tile with a handful of bulk copies issued by one thread
// and keeps kBulkStages tiles in flight while it computes.  Each cell's
// arithmetic is the one-cell form's, on the same values.
constexpr int kBulkStages = 4;
constexpr int kBulkTile = 256;
constexpr int kBulkCap = kBulkTile + 8;  // a run of the tile's length widened to 16-byte units
constexpr int kBulkBarrierBytes = 64;
#ifndef NIMBUS_BULK_MINB
#define NIMBUS_BULK_MINB 4
#endif

// Floats of one continuity stage: eleven runs, R0 (rho at -x), R1 (rho at
// the tile, +-1, +-y), R2 (rho at +x), U1 (u at the tile), U0 (u at -x), V (v
// at the tile and -y), W (w at the tile and -1), TH, MX, MY, MZ.
__host__ __device__ constexpr int continuity_stage_floats(int sy4) { return 11 * kBulkCap + 3 * sy4; }
// Floats of one momentum stage: RA, PA (tile, +1, +y), RB, PB (+x), U, V, W.
__host__ __device__ constexpr int momentum_stage_floats(int sy4) { return 7 * kBulkCap + 2 * sy4; }

// Slot offsets of the two stage layouts (floats), the last entry the stage end.
__host__ __device__ constexpr int continuity_slot(int slot, int sy4)
{
    // R0, R1 (+2 sy4), R2, U1, U0, V (+sy4), W, TH, MX, MY, MZ
    return slot * kBulkCap + (slot >= 2 ? 2 * sy4 : 0) + (slot >= 6 ? sy4 : 0);
}
__host__ __device__ constexpr int momentum_slot(int slot, int sy4)
{
    // RA (+sy4), PA (+sy4), RB, PB, U, V, W
    return slot * kBulkCap + (slot >= 1 ? sy4 : 0) + (slot >= 2 ? sy4 : 0);
}
static_assert(continuity_slot(11, 8) == continuity_stage_floats(8) && continuity_slot(11, 64) == continuity_stage_floats(64),
              "continuity stage layout");
static_assert(momentum_slot(7, 8) == momentum_stage_floats(8) && momentum_slot(7, 64) == momentum_stage_floats(64),
              "momentum stage layout");

__device__ __forceinline__ unsigned run_bytes(const CellRun& r) { return r.hi > r.lo ? 4u * (r.hi - r.lo) : 0u; }

__device__ __forceinline__ void stage_run(float* dst, const float* field, const CellRun& r, uint64_t* bar)
{
    if (r.hi > r.lo) bulk_copy_g2s(dst, field + r.lo, run_bytes(r), bar);
}

struct ContinuityRuns
{
    CellRun r0, r1, r2, t, v, w;  // r0 also serves u at -x; t the tile (u, theta, mx, my, mz)
};

__device__ __forceinline__ ContinuityRuns continuity_runs(int c0, int c1, int n, int sx, int sy)
{
    ContinuityRuns R;
    R.r0 = cell_run((long long)c0 - sx, (long long)c1 - sx, n);
    R.r1 = cell_run((long long)c0 - sy, (long long)c1 + sy, n);
    R.r2 = cell_run((long long)c0 + sx, (long long)c1 + sx, n);
    R.t = cell_run(c0, c1, n);
    R.v = cell_run((long long)c0 - sy, c1, n);
    R.w = cell_run((long long)c0 - 1, c1, n);
    return R;
}

struct MomentumRuns
{
    CellRun a, b, t;  // a: tile .. +y (rho, p); b: +x (rho, p); t: the tile (u, v, w)
};

__device__ __forceinline__ MomentumRuns momentum_runs(int c0, int c1, int n, int sx, int sy)
{
    MomentumRuns R;
    R.a = cell_run(c0, (long long)c1 + sy, n);
    R.b = cell_run((long long)c0 + sx, (long long)c1 + sx, n);
    R.t = cell_run(c0, c1, n);
    return R;
}

// Ends a CTA whose stage wait timed out: the member's status gets
// kStatusStagingTimeout and thread 0 waits (bounded) for the copies of the
// stages it issued that are still outstanding before the CTA leaves.
__device__ __forceinline__ void bulk_abandon(uint64_t* bar, unsigned parity_bits, int pending, unsigned* status)
{
    if (threadIdx.x == 0)
    {
        atomicOr(status, kStatusStagingTimeout);
        for (int q = 0; q < kBulkStages; ++q)
            if (pending & (1 << q)) (void)mbar_wait(&bar[q], (parity_bits >> q) & 1u);
    }
    __syncthreads();
}

template <class Policy, bool kFirst>
static __global__ void __launch_bounds__(256, NIMBUS_BULK_MINB) engine_continuity_bulk_kernel(const __grid_constant__ AcousticLaunch L,
                                                                     const EngineMember* __restrict__ table,
                                                                     long long tiles, int s)
{
    extern __shared__ __align__(16) unsigned char bulk_smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(bulk_smem);
    float* stages = reinterpret_cast<float*>(bulk_smem + kBulkBarrierBytes);
    const int sy4 = L.bulk_sy4;
    const int o_r1 = continuity_slot(1, sy4), o_r2 = continuity_slot(2, sy4), o_u1 = continuity_slot(3, sy4),
              o_u0 = continuity_slot(4, sy4), o_v = continuity_slot(5, sy4), o_w = continuity_slot(6, sy4),
              o_th = continuity_slot(7, sy4), o_mx = continuity_slot(8, sy4), o_my = continuity_slot(9, sy4),
              o_mz = continuity_slot(10, sy4);
    const int stage_floats = continuity_stage_floats(sy4);
    const bool even = (s & 1) == 0;
    if (threadIdx.x == 0)
    {
        for (int q = 0; q < kBulkStages; ++q) mbar_init(&bar[q], 1);
        mbar_init_fence();
    }
    __syncthreads();

    int pm = 0;                        // the producer's member cursor
    unsigned parity = 0;               // bit q: the parity of stage q's next phase
    int pending = 0;                   // stages issued and not yet consumed (thread 0's view)
    // Thread 0: stage tile t into stage q.
    auto issue = [&](long long t, int q) {
        while (t >= L.prefix[pm + 1]) ++pm;
        const AcousticConst& A = L.m[pm];
        const Dims d = A.F.d;
        const int n = d.cells();
        const int c0 = (int)((t - L.prefix[pm]) * kBulkTile), c1 = min(c0 + kBulkTile, n);
        const EngineMember& M = table[pm];
        const float* rho = even ? M.rho : M.rho_alt;
        const ContinuityRuns R = continuity_runs(c0, c1, n, d.sx(), d.sy());
        unsigned bytes = 2 * run_bytes(R.r0) + run_bytes(R.r1) + run_bytes(R.r2) + 2 * run_bytes(R.t) +
                         run_bytes(R.v) + run_bytes(R.w);
        if (!kFirst) bytes += 3 * run_bytes(R.t);
        float* S = stages + q * stage_floats;
        mbar_arrive_expect_tx(&bar[q], bytes);
        stage_run(S, rho, R.r0, &bar[q]);
        stage_run(S + o_r1, rho, R.r1, &bar[q]);
        stage_run(S + o_r2, rho, R.r2, &bar[q]);
        stage_run(S + o_u1, A.u, R.t, &bar[q]);
        stage_run(S + o_u0, A.u, R.r0, &bar[q]);
        stage_run(S + o_v, A.v, R.v, &bar[q]);
        stage_run(S + o_w, A.w, R.w, &bar[q]);
        stage_run(S + o_th, A.theta, R.t, &bar[q]);
        if (!kFirst)
        {
            stage_run(S + o_mx, A.mfx, R.t, &bar[q]);
            stage_run(S + o_my, A.mfy, R.t, &bar[q]);
            stage_run(S + o_mz, A.mfz, R.t, &bar[q]);
        }
        pending |= 1 << q;
    };
    const long long stride = gridDim.x;
    if (threadIdx.x == 0)
        for (int q = 0; q < kBulkStages; ++q)
        {
            const long long t = blockIdx.x + q * stride;
            if (t < tiles) issue(t, q);
        }

    int m = 0;
    int it = 0;
    for (long long t = blockIdx.x; t < tiles; t += stride, ++it)
    {
        const int q = it % kBulkStages;
        while (t >= L.prefix[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const bool ok = mbar_wait(&bar[q], (parity >> q) & 1u);
        if (ok)
        {
            const Dims d = A.F.d;
            const int n = d.cells(), sx = d.sx(), sy = d.sy();
            const int c0 = (int)((t - L.prefix[m]) * kBulkTile), c1 = min(c0 + kBulkTile, n);
            const int c = c0 + (int)threadIdx.x;
            if (c < c1)
            {
                const ContinuityRuns R = continuity_runs(c0, c1, n, sx, sy);
                const float* S = stages + q * stage_floats;
                int i, j, k;
                decompose(d, c, i, j, k);
                const bool xlo = i >= 1, xhi = i < d.nx - 1, ylo = j >= 1, yhi = j < d.ny - 1;
                const bool zlo = k > 0, zhi = k + 1 < d.nz;
                const float* r1 = S + o_r1 + (c - R.r1.lo);  // rho at the cell
                ContinuityStencil st;
                st.rho_c = r1[0];
                st.rxp = xhi ? S[o_r2 + (c + sx - R.r2.lo)] : st.rho_c;
                st.rxm = xlo ? S[c - sx - R.r0.lo] : st.rho_c;
                st.ryp = yhi ? r1[sy] : st.rho_c;
                st.rym = ylo ? r1[-sy] : st.rho_c;
                st.rzp = zhi ? r1[1] : st.rho_c;
                st.rzm = zlo ? r1[-1] : st.rho_c;
                const int ct = c - R.t.lo;
                st.uc = S[o_u1 + ct];
                st.uxm = xlo ? S[o_u0 + c - sx - R.r0.lo] : st.uc;
                st.vc = S[o_v + c - R.v.lo];
                st.vym = ylo ? S[o_v + c - sy - R.v.lo] : st.vc;
                st.wc = S[o_w + c - R.w.lo];
                st.wzm = zlo ? S[o_w + c - 1 - R.w.lo] : st.wc;
                st.th = S[o_th + ct];
                st.mx = kFirst ? 0.0f : S[o_mx + ct];
                st.my = kFirst ? 0.0f : S[o_my + ct];
                st.mz = kFirst ? 0.0f : S[o_mz + ct];
                const EngineMember& M = table[m];
                unsigned flags = 0;
                continuity_eos_values<Policy>(A.F, st, i, j, k, c, A.rho0, A.eos0, even ? M.rho_alt : M.rho, M.p,
                                              nullptr, A.mfx, A.mfy, A.mfz, flags, kFirst,
                                              kFirst ? A.rho_begin : nullptr);
                if (flags) atomicOr(A.status, flags);
            }
        }
        // Every thread is done with stage q (and agrees whether its wait
        // completed) before it is refilled.
        if (!__syncthreads_and(ok))
        {
            bulk_abandon(bar, parity, pending, A.status);
            return;
        }
        parity ^= 1u << q;
        if (threadIdx.x == 0)
        {
            pending &= ~(1 << q);
            const long long next = t + kBulkStages * stride;
            if (next < tiles) issue(next, q);
        }
    }
}

template <class Policy>
static __global__ void __launch_bounds__(256, NIMBUS_BULK_MINB) engine_momentum_bulk_kernel(const __grid_constant__ AcousticLaunch L,
                                                                   const EngineMember* __restrict__ table,
                                                                   long long tiles, int s)
{
    extern __shared__ __align__(16) unsigned char bulk_smem[];
    uint64_t* bar = reinterpret_cast<uint64_t*>(bulk_smem);
    float* stages = reinterpret_cast<float*>(bulk_smem + kBulkBarrierBytes);
    const int sy4 = L.bulk_sy4;
    const int o_pa = momentum_slot(1, sy4), o_rb = momentum_slot(2, sy4), o_pb = momentum_slot(3, sy4),
              o_u = momentum_slot(4, sy4), o_v = momentum_slot(5, sy4), o_w = momentum_slot(6, sy4);
    const int stage_floats = momentum_stage_floats(sy4);
    const bool even = (s & 1) == 0;
    if (threadIdx.x == 0)
    {
        for (int q = 0; q < kBulkStages; ++q) mbar_init(&bar[q], 1);
        mbar_init_fence();
    }
    __syncthreads();

    int pm = 0;
    unsigned parity = 0;
    int pending = 0;
    auto issue = [&](long long t, int q) {
        while (t >= L.prefix[pm + 1]) ++pm;
        const AcousticConst& A = L.m[pm];
        const Dims d = A.F.d;
        const int n = d.cells();
        const int c0 = (int)((t - L.prefix[pm]) * kBulkTile), c1 = min(c0 + kBulkTile, n);
        const EngineMember& M = table[pm];
        const float* rho = even ? M.rho_alt : M.rho;
        const MomentumRuns R = momentum_runs(c0, c1, n, d.sx(), d.sy());
        const unsigned bytes = 2 * run_bytes(R.a) + 2 * run_bytes(R.b) + 3 * run_bytes(R.t);
        float* S = stages + q * stage_floats;
        mbar_arrive_expect_tx(&bar[q], bytes);
        stage_run(S, rho, R.a, &bar[q]);
        stage_run(S + o_pa, M.p, R.a, &bar[q]);
        stage_run(S + o_rb, rho, R.b, &bar[q]);
        stage_run(S + o_pb, M.p, R.b, &bar[q]);
        stage_run(S + o_u, A.u, R.t, &bar[q]);
        stage_run(S + o_v, A.v, R.t, &bar[q]);
        stage_run(S + o_w, A.w, R.t, &bar[q]);
        pending |= 1 << q;
    };
    const long long stride = gridDim.x;
    if (threadIdx.x == 0)
        for (int q = 0; q < kBulkStages; ++q)
        {
            const long long t = blockIdx.x + q * stride;
            if (t < tiles) issue(t, q);
        }

    int m = 0;
    int it = 0;
    for (long long t = blockIdx.x; t < tiles; t += stride, ++it)
    {
        const int q = it % kBulkStages;
        while (t >= L.prefix[m + 1]) ++m;
        const AcousticConst& A = L.m[m];
        const bool ok = mbar_wait(&bar[q], (parity >> q) & 1u);
        if (ok)
        {
            const Dims d = A.F.d;
            const int n = d.cells(), sx = d.sx(), sy = d.sy();
            const int c0 = (int)((t - L.prefix[m]) * kBulkTile), c1 = min(c0 + kBulkTile, n);
            const int c = c0 + (int)threadIdx.x;
            if (c < c1)
            {
                const MomentumRuns R = momentum_runs(c0, c1, n, sx, sy);
                const float* S = stages + q * stage_floats;
                int i, j, k;
                decompose(d, c, i, j, k);
                const bool interior = i >= 1 && i < d.nx - 1 && j >= 1 && j < d.ny - 1 && k < d.nz - 1;
                const float* ra = S + (c - R.a.lo);  // rho at the cell
                const float* pa = S + o_pa + (c - R.a.lo);
                MomentumStencil st;
                st.rc = ra[0];
                st.pc = pa[0];
                st.rx = interior ? S[o_rb + (c + sx - R.b.lo)] : st.rc;
                st.px = interior ? S[o_pb + (c + sx - R.b.lo)] : st.pc;
                st.ry = interior ? ra[sy] : st.rc;
                st.py = interior ? pa[sy] : st.pc;
                st.rz = interior ? ra[1] : st.rc;
                st.pz = interior ? pa[1] : st.pc;
                const int ct = c - R.t.lo;
                st.uc = S[o_u + ct];
                st.vc = S[o_v + ct];
                st.wc = S[o_w + ct];
                momentum_values<Policy>(A.F, st, i, j, k, c, A.p0, A.dp0, A.u, A.v, A.w, A.vertical);
            }
        }
        if (!__syncthreads_and(ok))
        {
            bulk_abandon(bar, parity, pending, A.status);
            return;
        }
        parity ^= 1u << q;
        if (threadIdx.x == 0)
        {
            pending &= ~(1 << q);
            const long long next = t + kBulkStages * stride;
            if (next < tiles) issue(next, q);
        }
    }
}

// ---- state image ----------------------------------------------------------
// The engine's state image holds every member's nine prognostic fields back to
// back (u, v, w, rho, p, theta, qv, qc, qr, each items[kItemCells] floats) from
// image + image_offset.  gather = 0 scatters the image into the members'
// current buffers, gather = 1 collects them into it; one coalesced pass over
// all cells of all members either way.
static __global__ void __launch_bounds__(256) engine_image_kernel(const EngineMember* __restrict__ table,
                                                                  const long long* __restrict__ prefix,
                                                                  long long tiles, float* __restrict__ image,
                                                                  int gather)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        const long long n = M.items[kItemCells];
        float* blk = image + M.image_offset + c;
        float* const field[9] = {M.u, M.v, M.w, M.rho, M.p, M.theta, M.qv, M.qc, M.qr};
        float x[9];
        if (gather)
        {
#pragma unroll
            for (int f = 0; f < 9; ++f) x[f] = field[f][c];
#pragma unroll
            for (int f = 0; f < 9; ++f) blk[f * n] = x[f];
        }
        else
        {
#pragma unroll
            for (int f = 0; f < 9; ++f) x[f] = blk[f * n];
#pragma unroll
            for (int f = 0; f < 9; ++f) field[f][c] = x[f];
        }
    });
}

// Pointer rotation after the acoustic loop (rho: with an odd substep count
// the final density sits in the partner) and at the end of the step (qr after
// Kessler; p and the EOS candidate, which publishes the projection).
static __global__ void engine_swap_kernel(EngineMember* table, int members, int which)
{
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= members) return;
    EngineMember& M = table[m];
    if (which == 0)
    {
        if (M.n_substeps & 1)
        {
            float* t = M.rho;
            M.rho = M.rho_alt;
            M.rho_alt = t;
        }
    }
    else
    {
        if (M.microphysics)
        {
            float* t = M.qr;
            M.qr = M.qr_alt;
            M.qr_alt = t;
        }
        if (!(*M.status & kStatusInvalidEos))
        {
            float* t = M.p;
            M.p = M.eos;
            M.eos = t;
        }
    }
}

// ---- Transport (every scalar of a cell in one thread) -----------------------

template <bool kFp32>
// Resident CTAs per SM of the face-flux pass: the FP32 form at 4 (64
// registers; 1.85 -> 1.81 ms per ensemble step), the reference-precision
// form at 2 (its natural 90 registers).
#ifndef NIMBUS_FACES_MINB
#define NIMBUS_FACES_MINB 2
#endif
#ifndef NIMBUS_FACES_MINB_F32
#define NIMBUS_FACES_MINB_F32 4
#endif
static __global__ void __launch_bounds__(256, NIMBUS_FACES_MINB) engine_transport_faces_kernel(const EngineMember* __restrict__ table,
                                                                            const long long* __restrict__ prefix,
                                                                            long long tiles)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        transport_faces_cell4<kFp32>(M.T, reinterpret_cast<const float4*>(M.q4), M.mfx, M.mfy, M.mfz,
                                     reinterpret_cast<float4*>(M.sf), c);
    });
}

template <bool kFp32>
static __global__ void __launch_bounds__(256) engine_transport_limiter_kernel(const EngineMember* __restrict__ table,
                                                                              const long long* __restrict__ prefix,
                                                                              long long tiles)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        transport_limiter_cell4<kFp32>(M.T, reinterpret_cast<const float4*>(M.q4), M.rho_begin,
                                       reinterpret_cast<const float4*>(M.sf), reinterpret_cast<float4*>(M.rl), c);
    });
}

template <bool kFp32>
static __global__ void __launch_bounds__(256) engine_transport_update_kernel(const EngineMember* __restrict__ table,
                                                                             const long long* __restrict__ prefix,
                                                                             long long tiles)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        unsigned flags = 0;
        transport_update_cell4<kFp32>(M.T, reinterpret_cast<const float4*>(M.q4), [&](int s) { return engine_scalar(M, s); },
                                      [&](int s) { return engine_scalar_out(M, s); }, M.rho, M.rho_begin,
                                      reinterpret_cast<const float4*>(M.sf), reinterpret_cast<const float4*>(M.rl), c,
                                      flags);
        if (flags) atomicOr(M.status, flags);
    });
}

// The three transport passes with the members' constants in the constant
// bank: a compact copy of each member's transport parameters and its buffers
// that do not rotate; the end-of-loop density and the rain, which rotate,
// are read from the table.
struct TransportConst
{
    TransportCompact T;
    const float4* q4;
    const float *mfx, *mfy, *mfz, *rho_begin;
    float4 *sf, *rl;
    float *theta, *qv, *qc;
    unsigned* status;
};

constexpr int kTransportConstMembers = 64;

struct TransportLaunch
{
    long long prefix[kTransportConstMembers + 1];
    TransportConst m[kTransportConstMembers];
};
static_assert(sizeof(TransportLaunch) <= 32000, "a kernel parameter block holds at most 32764 bytes");

// Calls fn(A, M, c) for every cell of the first tiles of the launch.
template <class Fn>
__device__ __forceinline__ void for_transport_cells(const TransportLaunch& L, const EngineMember* __restrict__ table,
                                                    long long tiles, Fn&& fn)
{
    int m = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= L.prefix[m + 1]) ++m;
        const TransportConst& A = L.m[m];
        const int c = (int)((t - L.prefix[m]) * blockDim.x) + (int)threadIdx.x;
        if (c >= A.T.d.cells()) continue;
        fn(A, table[m], c);
    }
}

template <bool kFp32>
static __global__ void __launch_bounds__(256, kFp32 ? NIMBUS_FACES_MINB_F32 : NIMBUS_FACES_MINB) engine_transport_faces_const_kernel(
    const __grid_constant__ TransportLaunch L, const EngineMember* __restrict__ table, long long tiles)
{
    for_transport_cells(L, table, tiles, [&](const TransportConst& A, const EngineMember&, int c) {
        transport_faces_cell4<kFp32>(A.T, A.q4, A.mfx, A.mfy, A.mfz, A.sf, c);
    });
}

#ifndef NIMBUS_LIMITER_MINB_F32
#define NIMBUS_LIMITER_MINB_F32 6
#endif
template <bool kFp32>
static __global__ void __launch_bounds__(256, kFp32 ? NIMBUS_LIMITER_MINB_F32 : 3) engine_transport_limiter_const_kernel(
    const __grid_constant__ TransportLaunch L, const EngineMember* __restrict__ table, long long tiles)
{
    for_transport_cells(L, table, tiles, [&](const TransportConst& A, const EngineMember&, int c) {
        transport_limiter_cell4<kFp32>(A.T, A.q4, A.rho_begin, A.sf, A.rl, c);
    });
}

// Resident CTAs per SM of the update pass: the FP32 form at 4 (64
// registers; 0.88 -> 0.83 ms per ensemble step), the reference-precision
// form at 3 (at most 85 registers).
#ifndef NIMBUS_UPDATE_MINB_F32
#define NIMBUS_UPDATE_MINB_F32 4
#endif
template <bool kFp32>
static __global__ void __launch_bounds__(256, kFp32 ? NIMBUS_UPDATE_MINB_F32 : 3) engine_transport_update_const_kernel(
    const __grid_constant__ TransportLaunch L, const EngineMember* __restrict__ table, long long tiles)
{
    for_transport_cells(L, table, tiles, [&](const TransportConst& A, const EngineMember& M, int c) {
        unsigned flags = 0;
        float* const in_place[4] = {A.theta, A.qv, A.qc, M.qr};
        transport_update_cell4<kFp32>(A.T, A.q4, [&](int s) { return (const float*)in_place[s]; },
                                      [&](int s) { return in_place[s]; }, M.rho, A.rho_begin, A.sf, A.rl, c, flags);
        if (flags) atomicOr(A.status, flags);
    });
}

// ---- Acoustic speed scan before a large step --------------------------------
// Per member the largest (gamma p) / rho of its cells, as ordered double bits
// into c2[row] (row = the member's table row in this launch), for the
// substep count the reference re-derives before every large step
// (src/numerics/runtime.cpp:346-401,854-880).  The member of a tile is
// block-uniform, so a block keeps a running maximum while it walks one
// member's tiles and publishes it with one atomicMax when it moves on.
// One thread reads kScanCells cells (kItemScan tiles), which keeps the
// per-tile member lookup off the scan's critical path.
static __global__ void __launch_bounds__(256) engine_sound_speed_kernel(const EngineMember* __restrict__ table,
                                                                        const long long* __restrict__ prefix,
                                                                        long long tiles, unsigned long long* c2)
{
    int m = 0, held = -1;
    unsigned long long best = 0;
    for (long long t = blockIdx.x; t < tiles; t += gridDim.x)
    {
        while (t >= prefix[m + 1]) ++m;
        if (m != held)
        {
            if (held >= 0)
            {
                const unsigned long long b = block_max_u64(best);
                if (threadIdx.x == 0 && b) atomicMax(c2 + held, b);
            }
            held = m;
            best = 0;
        }
        const EngineMember& M = table[m];
        const int c0 = (int)((t - prefix[m]) * blockDim.x * kScanCells) + (int)threadIdx.x;
        unsigned flags = 0;
#pragma unroll
        for (int q = 0; q < kScanCells; ++q)
        {
            const int c = c0 + q * (int)blockDim.x;
            if (c < M.items[kItemCells]) best = max(best, sound_speed_sq_bits(M.gamma, M.p[c], M.rho[c], flags));
        }
        if (flags) atomicOr(M.status, flags);
    }
    if (held >= 0)
    {
        const unsigned long long b = block_max_u64(best);
        if (threadIdx.x == 0 && b) atomicMax(c2 + held, b);
    }
}

// ---- Kessler and EOS --------------------------------------------------------

// The Kessler step and the EOS re-projection in one pass: the candidate
// pressure is formed from the applied state while it is still in registers
// and written to the member's candidate buffer; engine_swap_kernel publishes
// it by exchanging p and the candidate unless the projection was refused.
// Resident CTAs per SM of the Kessler + EOS pass: the FP32 form at 5 (48
// registers; 1.03 -> 0.99 ms per ensemble step), the reference-precision
// form at 4.
#ifndef NIMBUS_MICRO_MINB_F32
#define NIMBUS_MICRO_MINB_F32 5
#endif
template <bool kFp32>
static __global__ void __launch_bounds__(256, kFp32 ? NIMBUS_MICRO_MINB_F32 : 4) engine_microphysics_eos_kernel(const EngineMember* __restrict__ table,
                                                                             const long long* __restrict__ prefix,
                                                                             long long tiles)
{
    for_member_items(table, prefix, tiles, kItemCells, [&](const EngineMember& M, int c) {
        unsigned flags = 0;
        float4 s;
        const float po = M.p[c];
        if (M.microphysics)
        {
            if constexpr (kFp32)
                kessler_cell_f32<true>(M.K, M.theta, M.qv, M.qc, M.qr, M.p, M.rho, M.qr_alt, nullptr, nullptr,
                                       nullptr, nullptr, c, &s);
            else
                kessler_cell<true>(M.K, M.theta, M.qv, M.qc, M.qr, M.p, M.rho, M.qr_alt, nullptr, nullptr, nullptr,
                                   nullptr, c, &s);
        }
        else
            s = make_float4(M.theta[c], M.qv[c], M.qc[c], M.qr[c]);
        float p_new;
        bool ok;
        if constexpr (kFp32)
            ok = eos_candidate_value_f32(M.K.d, c, c % M.K.d.nz, M.rho[c], s.x, M.eos0, M.eos_series, M.gamma, true,
                                         po, s.y, s.z, s.w, p_new, flags);
        else
            ok = eos_candidate_value(M.K.d, c, M.rho[c], s.x, M.gamma, true, po, s.y, s.z, s.w, p_new, flags);
        if (ok) M.eos[c] = p_new;
        if (flags) atomicOr(M.status, flags);
        // The end-of-step sponge after the EOS projection (dynamics.cpp:7323-7340).
        if (M.R.do_upper | M.R.do_w_only | M.R.do_lateral)
        {
            int i, j, k;
            decompose(M.K.d, c, i, j, k);
            float uu = M.u[c], vv = M.v[c], ww = M.w[c], th = s.x;
            if (relax_cell(M.R, M.K.d.nx, M.K.d.ny, i, j, k, uu, vv, ww, th))
            {
                M.u[c] = uu;
                M.v[c] = vv;
                M.w[c] = ww;
                M.theta[c] = th;
            }
        }
    });
}

}  // namespace nimbus
