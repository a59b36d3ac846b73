/*
 * nimbus_cuda.h -- C-ABI of the B200 (sm_100a) CUDA backend for the Nimbus
 * dynamical-core hot path: the Klemp-Wilhelmson split-explicit acoustic
 * substep loop and the conservative WENO5 scalar transport on the flat
 * Cartesian Arakawa C-grid.
 *
 * Plain pointers and sizes only.  Every field is row-major [nx][ny][nz] float
 * (k fastest, index (i*ny + j)*nz + k): u on x-faces i+1/2, v on y-faces
 * j+1/2, w on z-faces k+1/2, scalars at cell centres.  Base-state columns are
 * FP64, as the reference CPU solver holds them.
 *
 * Memory: each argument block names where its field pointers live.
 *   NIMBUS_MEMORY_HOST    host arrays; the call stages them through the
 *                         context's device workspace and returns after the
 *                         results are back in the host arrays (the reference's
 *                         "fence-confirmed" dispatch contract).  A refused or
 *                         failed call leaves every host array untouched.
 *   NIMBUS_MEMORY_DEVICE  device pointers; the call enqueues on `stream` (a
 *                         cudaStream_t, NULL = the context's stream) and returns
 *                         without synchronising.
 *
 * Errors: every entry point returns a nimbus_status; nimbus_cuda_last_error()
 * gives the message of the last failure on that context.  No exception or
 * C++ type crosses this boundary.  A context is used by one host thread at a
 * time.
 */
#ifndef NIMBUS_CUDA_H
#define NIMBUS_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NIMBUS_CUDA_ABI_VERSION 1

typedef enum nimbus_status
{
    NIMBUS_OK = 0,
    NIMBUS_ERR_INVALID_ARGUMENT = 1, /* dispatch refused before any mutation */
    NIMBUS_ERR_CUDA = 2,             /* a CUDA runtime call failed */
    NIMBUS_ERR_OUT_OF_MEMORY = 3,    /* device allocation or admission failed */
    NIMBUS_ERR_NONFINITE = 4,        /* a produced value was non-finite; outputs not published */
    NIMBUS_ERR_UNSUPPORTED = 5,      /* valid request outside this backend's contract */
    NIMBUS_ERR_NO_DEVICE = 6,        /* no usable sm_100 device */
    NIMBUS_ERR_TOO_LARGE = 7,        /* grid exceeds a fixed capacity (see NIMBUS_STATIC_SCRATCH_CELLS) */
    NIMBUS_ERR_IO = 8                /* a history file could not be written */
} nimbus_status;

typedef enum nimbus_memory
{
    NIMBUS_MEMORY_HOST = 0,
    NIMBUS_MEMORY_DEVICE = 1
} nimbus_memory;

/* Lateral boundary codes: tmv::init::config::LateralBC (include/init/config/config_v1.hpp:40-48). */
enum
{
    NIMBUS_BC_PERIODIC = 0,
    NIMBUS_BC_RADIATIVE = 1,
    NIMBUS_BC_RIGID = 2,
    NIMBUS_BC_RIGID_SLIP = 3,
    NIMBUS_BC_ZERO_GRADIENT = 4
};
/* Bottom: BottomBC {RigidNoSlip, RigidSlip}; top: TopBC {Rigid, RigidWithSponge, Open}. */
enum
{
    NIMBUS_BOTTOM_NO_SLIP = 0,
    NIMBUS_BOTTOM_SLIP = 1
};
enum
{
    NIMBUS_TOP_RIGID = 0,
    NIMBUS_TOP_SPONGE = 1,
    NIMBUS_TOP_OPEN = 2
};

typedef struct nimbus_cuda_context nimbus_cuda_context;

/* Context lifecycle.  Replaces ComputeBackend::initialize / shutdown
 * (include/compute/backend_interface.hpp:19-60) for the CUDA backend: binds a
 * device, creates a stream, and owns the staging workspace.  Fails with
 * NIMBUS_ERR_NO_DEVICE when no sm_100 device is present -- there is no CPU
 * fallback. */
nimbus_status nimbus_cuda_create(int device, nimbus_cuda_context** out);
void nimbus_cuda_destroy(nimbus_cuda_context* ctx);
const char* nimbus_cuda_last_error(const nimbus_cuda_context* ctx);
int nimbus_cuda_abi_version(void);
/* Kernels this context launched so far (all entry points); the analogue of
 * ComputeBackend::successful_kernel_dispatch_count (backend_interface.hpp:55-60). */
uint64_t nimbus_cuda_kernel_launches(const nimbus_cuda_context* ctx);
/* The context's stream, as a cudaStream_t. */
void* nimbus_cuda_stream(const nimbus_cuda_context* ctx);
/* The context's device: its name, SM count, compute capability and memory
 * (total, and free now); what ComputeBackend::populate_hardware_info and
 * memory_properties report (backend_interface.hpp:39-44). */
typedef struct nimbus_device_info
{
    char name[256];
    int sm_count;
    int cc_major, cc_minor;
    unsigned long long total_bytes;
    unsigned long long free_bytes;
} nimbus_device_info;
nimbus_status nimbus_cuda_device_info(nimbus_cuda_context* ctx, nimbus_device_info* out);
/* Waits for all work on the context's stream, then reads and clears the
 * device status word that NIMBUS_MEMORY_DEVICE calls accumulate: returns
 * NIMBUS_ERR_NONFINITE if any enqueued call produced a non-finite retained
 * mass flux or transported scalar since the last check. */
nimbus_status nimbus_cuda_synchronize(nimbus_cuda_context* ctx);

/* Arithmetic of the hot-path kernels on this context.
 *   NIMBUS_PRECISION_REFERENCE (default): FP64 interior arithmetic over FP32
 *     storage in the reference CPU solver's operation order -- bit-identical
 *     results to the reference.
 *   NIMBUS_PRECISION_FP32: FP32 arithmetic throughout (stencils, WENO5 in
 *     paired f32x2 instructions, Kessler), with the FP64 base state entering
 *     as per-level FP32 hi+lo pairs: the hydrostatic pressure differences and
 *     the compensated EOS p = p0 (1 + d)^gamma; the retained mass-flux sums
 *     are single-rounding FMAs.  Errors against the FP64 oracle are stated,
 *     not zero. */
enum
{
    NIMBUS_PRECISION_REFERENCE = 0,
    NIMBUS_PRECISION_FP32 = 1
};
nimbus_status nimbus_cuda_set_precision(nimbus_cuda_context* ctx, int precision);

/* Form of the acoustic substep kernels.
 *   NIMBUS_SUBSTEP_AUTO  (default) the form the autotuner chose for the grid
 *                        shape and precision, else SPLIT.
 *   NIMBUS_SUBSTEP_FUSED one launch per substep: 2.5-D i-marching strips with
 *                        cp.async-staged shared-memory planes (64 B/cell).
 *   NIMBUS_SUBSTEP_SPLIT two launches per substep (continuity+EOS, momentum),
 *                        one thread per cell (84 B/cell, fewer instructions).
 * Every form gives identical results in reference precision. */
enum
{
    NIMBUS_SUBSTEP_AUTO = 0,
    NIMBUS_SUBSTEP_FUSED = 1,
    NIMBUS_SUBSTEP_SPLIT = 2
};
nimbus_status nimbus_cuda_set_substep_form(nimbus_cuda_context* ctx, int form);
/* Autotuner: times each substep form on an nx*ny*nz scratch state (a few
 * substeps each, CUDA events, after a warm-up) in the context's current
 * precision and records the fastest for NIMBUS_SUBSTEP_AUTO launches of that
 * shape.  Synchronous; allocates scratch.  *chosen_form (may be NULL)
 * receives the choice and *ms_per_substep (may be NULL) its time. */
nimbus_status nimbus_cuda_autotune_substep(nimbus_cuda_context* ctx, int nx, int ny, int nz, int* chosen_form,
                                           double* ms_per_substep);

/* Kernel families for per-launch device timing. */
enum
{
    NIMBUS_KERNEL_ACOUSTIC_SUBSTEP = 0,   /* continuity + EOS (+ retained mass flux) */
    NIMBUS_KERNEL_ACOUSTIC_MOMENTUM = 1,
    NIMBUS_KERNEL_ACOUSTIC_BOUNDARY = 2,  /* the three face-closure kernels of one substep */
    NIMBUS_KERNEL_TRANSPORT_FACES = 3,
    NIMBUS_KERNEL_TRANSPORT_LIMITER = 4,
    NIMBUS_KERNEL_TRANSPORT_UPDATE = 5,
    NIMBUS_KERNEL_SLOW = 6,               /* slow tendencies (k1+predictor, k2+apply) */
    NIMBUS_KERNEL_MICROPHYSICS = 7,       /* Kessler, the EOS re-projection, the end-of-step sponge and the
                                             engine's acoustic speed scan */
    NIMBUS_KERNEL_OUTPUT = 8,             /* cell-centre velocities for output */
    NIMBUS_KERNEL_SGS = 9,                /* Smagorinsky closure, SGS apply and stability */
    NIMBUS_KERNEL_FAMILIES = 10
};
/* When enabled, every launch is bracketed by CUDA events on its own stream
 * and nimbus_cuda_kernel_timing() returns, per family, the launch count and
 * the summed device time since timing was enabled (it synchronises).  Timing
 * adds two event records per launch; leave it off for throughput runs. */
nimbus_status nimbus_cuda_set_kernel_timing(nimbus_cuda_context* ctx, int enable);
nimbus_status nimbus_cuda_kernel_timing(nimbus_cuda_context* ctx, int family, uint64_t* launches, double* total_ms);

/*
 * One fused acoustic substep, in place on (u, v, w, rho, p).
 * Replaces DynamicsComputeKernels::dispatch_acoustic_substep_fused_cartesian_cgrid
 * (include/compute/dispatch/dynamics.hpp:220-277,686; CPU semantics
 * src/compute/cpu/acoustic_cgrid_fast.cpp:12-219): flux-form continuity on
 * 1<=i<=nx-2, 1<=j<=ny-2, all k; rho forward Euler with fallback and clamp;
 * p = p00 (rho R_d theta / p00)^gamma with clamp; then u,v,w forward Euler
 * from the new pressure gradient (k<=nz-2) with clamps.  Interior arithmetic
 * is FP64 over FP32 storage, the reference's own sequence.
 * drho_scratch is optional (NULL = not written); when given it receives the
 * stored FP32 continuity tendency.  Requires nx>=3, ny>=3, nz>=2, base_len>=nz.
 */
typedef struct nimbus_acoustic_fused_args
{
    float* u;
    float* v;
    float* w;
    float* rho;
    float* p;
    const float* theta;
    const double* rho0_base; /* FP64 [base_len] */
    const double* p0_base;   /* FP64 [base_len] */
    int base_len;
    int nx, ny, nz;
    double dx, dy, dz;
    double dt_small;
    double gamma;            /* cp / (cp - R_d) */
    float rho_min, rho_max;
    float p_min, p_max;
    float p_ref_fallback;
    float wind_clamp_h, wind_clamp_v;
    float* drho_scratch;
    int memory;              /* nimbus_memory */
    void* stream;            /* cudaStream_t for NIMBUS_MEMORY_DEVICE, NULL = context stream */
} nimbus_acoustic_fused_args;

nimbus_status nimbus_cuda_acoustic_fused(nimbus_cuda_context* ctx, const nimbus_acoustic_fused_args* a);

/*
 * The fused acoustic substep for callers that cannot allocate device memory.
 * This entry point has no counterpart in the reference.
 *
 * Who needs it: a host that has already committed its whole HBM budget (for
 * example runs admitted by free device memory, whose state is sized up front
 * and must not grow), or a latency-sensitive stepping loop that cannot afford
 * the implicit device-wide synchronisation of cudaMalloc/cudaFree.  Every
 * other entry point may grow the context workspace; this one allocates
 * nothing and needs no context.
 *
 * It always computes in reference precision (FP64 interior arithmetic on
 * FP32 storage): its results equal nimbus_cuda_acoustic_fused's for a context
 * in NIMBUS_PRECISION_REFERENCE, bit for bit; the FP32 form is not offered
 * here.  Requirements:
 *   - memory == NIMBUS_MEMORY_DEVICE: every field pointer is device memory on
 *     the current device; the substep is enqueued on `stream` (NULL = the
 *     default stream) and the call returns without synchronising;
 *   - nx*ny*nz <= NIMBUS_STATIC_SCRATCH_CELLS, else NIMBUS_ERR_TOO_LARGE.
 * Scratch: the new density is staged in one file-scope device array of
 * NIMBUS_STATIC_SCRATCH_CELLS floats (16 MiB) that every GPU which loads the
 * library holds until the process exits.  The first call on a device resolves
 * that array's device address (with the device current), so make the first
 * call on each device before any stream capture.  Every call shares the one
 * array: calls that overlap on the GPU (different streams, or different host
 * threads on the same device) race and must be serialised by the caller.
 * Each call overwrites the whole scratch range it reads, so no clearing is
 * needed between calls.
 * Errors: an error left by earlier work of the process is cleared, not
 * reported; NIMBUS_ERR_CUDA from a launch means nothing was enqueued after
 * it; if the final copy of the new density fails, p, u, v and w are already
 * advanced while rho still holds its old values.
 */
#define NIMBUS_STATIC_SCRATCH_CELLS 4194304
nimbus_status nimbus_cuda_acoustic_fused_static_scratch(const nimbus_acoustic_fused_args* a);

/*
 * All n_substeps acoustic substeps of one large step in one submission, with
 * the boundary closure after every substep and the time-averaged face mass
 * flux exported.  Replaces
 * DynamicsComputeKernels::dispatch_acoustic_substeps_batched_cartesian_cgrid
 * (include/compute/dispatch/dynamics.hpp:279-326,726; contract
 * include/compute/acoustic_cgrid_dispatch_contract.hpp:114-156) and follows
 * the CPU loop order of SplitExplicitScheme::step_split_acoustic
 * (src/numerics/time_stepping/schemes/split_explicit/split_explicit.cpp:174-260):
 *   per substep: mass_flux += weight * rho_face * (velocity - frame) from the
 *   pre-substep state (advection_cartesian.cpp:610-870, unfused FP64 add);
 *   fused substep; boundary closure W, E, S, N, vertical with the KW78
 *   radiation integrated over dt_small
 *   (boundary_conditions_cartesian_cgrid.cpp:884-1187).
 * wave_history (in) / wave_history_output (out): KW78 face memory, layout
 *   u_west[ny*nz], u_east[ny*nz], v_south[nx*nz], v_north[nx*nz]
 *   (2*(nx+ny)*nz floats).  wave_history NULL seeds it from the current faces
 *   (seed_acoustic_radiation, :798-822).  The two may be the same array.
 * density_begin: optional; receives rho at loop start (the scalar-paired
 *   density of CartesianCGridTransportContext::capture_density_begin).
 * mass_flux_*: accumulated into (callers zero them at the start of a large
 *   step, as CartesianCGridTransportContext::begin does).
 * Requires nx>=4, ny>=4, nz>=2, 1<=n_substeps<=4096.
 */
typedef struct nimbus_acoustic_batched_args
{
    float* u;
    float* v;
    float* w;
    float* rho;
    float* p;
    const float* theta;
    const double* rho0_base;
    const double* p0_base;
    int base_len;
    int nx, ny, nz;
    double dx, dy, dz;
    double dt_small;
    int n_substeps;
    double gamma;
    float rho_min, rho_max;
    float p_min, p_max;
    float p_ref_fallback;
    float wind_clamp_h, wind_clamp_v;
    int bc_west, bc_east, bc_south, bc_north, bc_bottom, bc_top;
    float* mass_flux_x;
    float* mass_flux_y;
    float* mass_flux_z;
    int accumulate_mass_flux;
    double mass_flux_weight;  /* dt_small / dt_large */
    float frame_velocity_u_ms, frame_velocity_v_ms;
    const float* wave_history;
    float* wave_history_output;
    float* density_begin;
    int memory;
    void* stream;
} nimbus_acoustic_batched_args;

nimbus_status nimbus_cuda_acoustic_batched(nimbus_cuda_context* ctx, const nimbus_acoustic_batched_args* a);

/*
 * Conservative flux-form transport of n_scalars scalars against the retained
 * time-averaged face mass fluxes.  Replaces
 * AdvectionComputeKernels::dispatch_advect_scalars_conservative_cartesian_cgrid
 * (include/compute/dispatch/advection.hpp:154-230; CPU semantics
 * advect_scalar_conservative_3d_cartesian_impl, advection_cartesian.cpp:1652-2640):
 * face value by WENO5-JS where the 5-point stencil fits, else the MC-limited
 * slope (weno5_face.hpp:43-86, advection_cartesian.cpp:1943-2172);
 * positive-definite donor limiting for flagged scalars (:2174-2240);
 * phi_new = (rho_begin phi - dt div SF) / max(rho_end, rho_floor) on
 * 1<=i<=nx-2, 1<=j<=ny-2, all k (:2465-2640).  q_in[s] may equal q_out[s]
 * (in place).  At most 16 scalars.
 */
typedef struct nimbus_scalar_transport_args
{
    const float* const* q_in;
    float* const* q_out;
    const int* positive_definite;
    int n_scalars;
    int nx, ny, nz;
    double dx, dy, dz;
    double dt;
    const float* rho_end;
    const float* rho_begin;
    const float* mass_flux_x;
    const float* mass_flux_y;
    const float* mass_flux_z;
    int weno;                 /* 1 = WENO5 (production), 0 = MC everywhere */
    int top_open;             /* C-grid open top owns the k=nz-1 boundary face */
    float rho_floor;          /* 0.05 (density_min_kgm3) */
    int memory;
    void* stream;
} nimbus_scalar_transport_args;

nimbus_status nimbus_cuda_scalar_transport(nimbus_cuda_context* ctx, const nimbus_scalar_transport_args* a);

/*
 * Slow (advective) tendencies of the C-grid KW scheme and the Heun slow step.
 *
 * nimbus_cuda_slow_tendencies evaluates the operator once: it replaces
 * DynamicsComputeKernels::dispatch_cartesian_cgrid_slow_tendencies
 * (include/compute/dispatch/dynamics.hpp:374-420) with CPU semantics
 * CartesianCGrid3DScheme::compute_slow_tendencies (cartesian_cgrid_3d.cpp:724-1416)
 * on the stationary flat branch: du, dv, dw on 1<=i<=nx-2, 1<=j<=ny-2,
 * 0<=k<=nz-2 (fd5/fd3/fd1 upwind-biased advection, f-plane Coriolis on the
 * perturbation wind, buoyancy with vapour and hydrometeor loading on w) and
 * dp = -u.grad p on 1<=k<=nz-2; zero elsewhere.  u, v, w, p are inputs and
 * du_dt .. dp_dt are required outputs.
 *
 * nimbus_cuda_slow_step advances u, v, w, p in place by one Heun slow step
 * with dt_large: k1 = L(x), x* = x + dt k1, k2 = L(x*), x += dt*0.5f(k2+k1)
 * (prepare_slow_rk2_tendencies, dynamics.cpp:5123-5292, then
 * apply_slow_tendencies, dynamics.cpp:1955-2092).  du_dt .. dp_dt are
 * optional and receive the averaged tendency.
 *
 * qv/qc/qr may be NULL (dry, or no loading); qi, qs, qg, qh are taken as zero.
 */
typedef struct nimbus_slow_args
{
    float* u;
    float* v;
    float* w;
    float* p;
    const float* rho;
    const float* qv;
    const float* qc;
    const float* qr;
    const double* rho0_base;
    const double* qv0_base;  /* may be NULL when qv is NULL */
    const double* u0_base;   /* environment wind for the Coriolis terms; NULL = 0 */
    const double* v0_base;
    int base_len;
    int nx, ny, nz;
    double dx, dy, dz;
    double dt_large;
    double gravity;          /* 9.81 */
    double coriolis_f;
    float frame_velocity_u_ms, frame_velocity_v_ms;
    float* du_dt;
    float* dv_dt;
    float* dw_dt;
    float* dp_dt;
    int memory;
    void* stream;
} nimbus_slow_args;

nimbus_status nimbus_cuda_slow_tendencies(nimbus_cuda_context* ctx, const nimbus_slow_args* a);

/*
 * The slow tendencies applied over the large step.  Replaces
 * DynamicsComputeKernels::dispatch_slow_apply (include/compute/dispatch/
 * dynamics.hpp:328-352,760) with the CPU semantics of apply_slow_tendencies_cpu
 * (src/core/orchestration/dynamics/dynamics.cpp:1955-2095): u and v take
 * their tendency plus the boundary-layer one (du_dt_pbl, dv_dt_pbl; NULL =
 * zero), w and p their own; with sanitize a non-finite tendency counts as
 * zero; each field becomes x + t dt formed in FP64 and rounded once.
 */
typedef struct nimbus_slow_apply_args
{
    float* u;
    float* v;
    float* w;
    float* p;
    const float* du_dt;
    const float* dv_dt;
    const float* dw_dt;
    const float* dp_dt;
    const float* du_dt_pbl;  /* may be NULL */
    const float* dv_dt_pbl;  /* may be NULL */
    int nx, ny, nz;
    double dt_large;
    int sanitize;            /* the runtime's primary-state repairs */
    int memory;
    void* stream;
} nimbus_slow_apply_args;

nimbus_status nimbus_cuda_slow_apply(nimbus_cuda_context* ctx, const nimbus_slow_apply_args* a);

/*
 * The slow-tendency operator of the reference's device route
 * (CartesianCGrid3DScheme::compute_slow_tendencies, cartesian_cgrid_3d.cpp:835-925,
 * when the backend supports DynamicsKernelOp::CartesianCgridSlowTendencies):
 * FP32 fields and spacings, FP32 base profiles (rho0 of at least nz levels;
 * qv0 when has_moisture; u0/v0 used when wind0_base_len >= nz, else zero),
 * the host-summed hydrometeor loading, f at grid y = 0 and the beta-plane
 * df/dy.  Every output is written (zero where the scheme does not act;
 * drho_dt zero); the three advection outputs come together or not at all.
 * FP32 arithmetic, the reference's device operator
 * (vulkan/shaders/compute/dynamics/cartesian_cgrid_slow_tendencies.comp).
 * Mirrors CartesianCgridSlowTendenciesDispatch (include/compute/dispatch/dynamics.hpp:374-420).
 */
typedef struct nimbus_cgrid_slow_tendencies_args
{
    const float* u;
    const float* v;
    const float* w;
    const float* rho;
    const float* p;
    const float* rho0_base;
    int rho0_base_len;
    const float* qv0_base;
    int qv0_base_len;
    const float* u0_base;
    const float* v0_base;
    int wind0_base_len;
    const float* qv;
    const float* loading;
    float* du_dt;
    float* dv_dt;
    float* dw_dt;
    float* drho_dt;          /* optional */
    float* dp_dt;
    int nx, ny, nz;
    float dx, dy, dz, g, coriolis_f;
    int has_moisture, has_loading;
    float* du_advection_dt;  /* optional, all three or none */
    float* dv_advection_dt;
    float* dw_advection_dt;
    float frame_velocity_u, frame_velocity_v, coriolis_beta;
    int memory;
    void* stream;
} nimbus_cgrid_slow_tendencies_args;

nimbus_status nimbus_cuda_cgrid_slow_tendencies(nimbus_cuda_context* ctx, const nimbus_cgrid_slow_tendencies_args* a);
nimbus_status nimbus_cuda_slow_step(nimbus_cuda_context* ctx, const nimbus_slow_args* a);

/*
 * Kessler warm-rain microphysics.
 * nimbus_cuda_kessler_tendencies replaces the Kessler MicrophysicsComputeKernels
 * dispatches (include/compute/dispatch/microphysics.hpp) with CPU semantics
 * KesslerScheme::compute_tendencies (src/microphysics/schemes/kessler/kessler.cpp:103-520):
 * coupled saturation adjustment, autoconversion (qc0 1e-3, 1e-3 /s),
 * accretion (2.2), rain evaporation and rain sedimentation over the cell
 * domain [i0,i1)x[j0,j1)x[k0,k1); dtheta/dqv/dqc/dqr are required outputs
 * (zero outside the domain).
 * nimbus_cuda_kessler_step also applies them with dt over the domain: water
 * species as clamp(q + dt dq, 0, 0.05) (bounded_water_value,
 * microphysics_step.cpp:503-532), theta as theta + dt dtheta; the tendency
 * outputs are optional there.
 */
typedef struct nimbus_kessler_args
{
    float* theta;
    float* qv;
    float* qc;
    float* qr;
    const float* p;
    const float* rho;
    int nx, ny, nz;
    double dz;
    double dt;
    int domain[6];           /* i0, i1, j0, j1, k0, k1; the C-grid uses {1, nx-1, 1, ny-1, 0, nz} */
    float* dtheta_dt;
    float* dqv_dt;
    float* dqc_dt;
    float* dqr_dt;
    int memory;
    void* stream;
} nimbus_kessler_args;

nimbus_status nimbus_cuda_kessler_tendencies(nimbus_cuda_context* ctx, const nimbus_kessler_args* a);
nimbus_status nimbus_cuda_kessler_step(nimbus_cuda_context* ctx, const nimbus_kessler_args* a);

/*
 * The Kessler operators of the reference's device route
 * (KesslerScheme::compute_tendencies, kessler.cpp:152-300, when the active
 * backend supports MicrophysicsKernelOp::KesslerPointwise): the host runs the
 * saturation adjustment, the pointwise operator takes the adjusted
 * temperature, qv and qc and writes the warm-rain tendencies (production and
 * rain evaporation; dtheta_dt is the temperature tendency before the theta
 * conversion) over the whole grid, zero outside the cell domain; the
 * sedimentation operator adds the rain fallout to dqr_dt in place.  FP32
 * arithmetic, the reference's device operator
 * (vulkan/shaders/compute/microphysics/kessler_pointwise.comp,
 * kessler_sedimentation.comp).  Mirror KesslerPointwiseDispatch and
 * KesslerSedimentationDispatch (include/compute/dispatch/microphysics.hpp:436-492);
 * the inert qg/qh slots are dropped (dqg_dt/dqh_dt, when given, are written
 * zero).
 */
typedef struct nimbus_kessler_pointwise_args
{
    const float* temperature;
    const float* p;
    const float* qv;
    const float* qc;
    const float* qr;
    const float* rho_d;
    float* dtheta_dt;
    float* dqv_dt;
    float* dqc_dt;
    float* dqr_dt;
    float* dqg_dt;           /* optional */
    float* dqh_dt;           /* optional */
    int nx, ny, nz;
    int i_begin, i_end, j_begin, j_end, k_begin, k_end;
    float qc0, c_auto, c_accr, evaporation_efficiency, lv_cp, t0, dt_step;
    int memory;
    void* stream;
} nimbus_kessler_pointwise_args;

typedef struct nimbus_kessler_sedimentation_args
{
    const float* qr;
    const float* rho_d;              /* optional: density-corrected fall speeds and receiver weights */
    const float* layer_thickness_m;  /* optional: per-cell layer thickness instead of dz */
    float* dqr_dt;                   /* read and updated in place */
    int nx, ny, nz;
    int i_begin, i_end, j_begin, j_end, k_begin, k_end;
    float dz, vt_max_rain, vt_cap, dt_step;
    int memory;
    void* stream;
} nimbus_kessler_sedimentation_args;

nimbus_status nimbus_cuda_kessler_pointwise(nimbus_cuda_context* ctx, const nimbus_kessler_pointwise_args* a);
nimbus_status nimbus_cuda_kessler_sedimentation(nimbus_cuda_context* ctx,
                                                const nimbus_kessler_sedimentation_args* a);

/*
 * EOS pressure re-projection after transport and microphysics
 * (tmv::dynamics_eos::apply_pressure_projection, eos_apply.cpp:50-200):
 * p = clamp(float(p00 (rho R_d theta / p00)^gamma), 1000, 2e5) in FP64 for
 * every cell.  qv/qc/qr are optional (all or none); given, the state counts as
 * complete and the attributed cells (the one-cell lateral ring dropped where
 * the extent is >= 3) are also checked as the reference's energy attribution
 * checks them.  The energy report itself is not formed.  An invalid cell
 * refuses the whole projection and p keeps its old values: host memory returns
 * NIMBUS_ERR_NONFINITE; device memory reports it at nimbus_cuda_synchronize.
 */
typedef struct nimbus_eos_args
{
    float* p;
    const float* rho;
    const float* theta;
    const float* qv;
    const float* qc;
    const float* qr;
    int nx, ny, nz;
    double gamma;
    int memory;
    void* stream;
    /* Optional FP64 base pressure per level (nz; host or device as `memory`).
     * Under NIMBUS_PRECISION_FP32 the projection is then evaluated around it
     * in the compensated FP32 form of the acoustic substeps (within about
     * half an FP32 ulp of the FP64 value); NULL keeps the FP64 evaluation. */
    const double* p0_base;
} nimbus_eos_args;

nimbus_status nimbus_cuda_eos_projection(nimbus_cuda_context* ctx, const nimbus_eos_args* a);

/*
 * Acoustic substep count before a large step.  The reference re-derives it
 * before every large step from the live state: choose_runtime_timestep
 * (src/numerics/runtime.cpp:712-880) samples c_max = max sqrt(gamma p / rho)
 * over every cell (the flat Cartesian CFL scan, runtime.cpp:346-401) and the
 * base columns (:854-870), and SplitExplicitScheme::resolve_substep_count
 * (src/numerics/time_stepping/schemes/split_explicit/split_explicit.cpp:67-170)
 * turns it into N = max(requested, ceil(dt c_max / (0.5 min(dx,dy,dz))) + 1, 2).
 *
 * nimbus_cuda_max_sound_speed scans p and rho (host or device memory as
 * `memory`) on the device and returns c_max in *max_sound_speed after waiting
 * for the scan; base columns (host memory, length nz) may be NULL.  A
 * non-finite or non-positive pressure or density: NIMBUS_ERR_NONFINITE
 * (where the reference throws).
 * nimbus_cuda_resolve_substep_count: the count, or -1 where the reference
 * throws (dt, c_max or spacing non-finite or non-positive; unrepresentable N).
 */
typedef struct nimbus_sound_speed_args
{
    const float* p;
    const float* rho;
    int nx, ny, nz;
    const double* p0_base;    /* host, nz values, or NULL */
    const double* rho0_base;  /* host, nz values, or NULL */
    int memory;
    void* stream;
    double max_sound_speed;   /* out */
} nimbus_sound_speed_args;

nimbus_status nimbus_cuda_max_sound_speed(nimbus_cuda_context* ctx, nimbus_sound_speed_args* a);
int nimbus_cuda_resolve_substep_count(double dt_large, double max_sound_speed, double min_spacing, int requested);

/*
 * End-of-step sponge (state relaxation) on a flat C-grid level: the upper
 * Rayleigh sponge, the w-only lid absorber and the lateral band, in that
 * order, relaxing u, v, w toward (u_ref, v_ref, 0) and theta toward
 * theta_ref (rho and p are not relaxed).  Replaces apply_rayleigh_damping +
 * apply_lateral_damping (src/core/infra/rayleigh_damping.cpp:720-1119,
 * 1194-1476) as dynamics.cpp:7323-7340 calls them after the EOS projection,
 * and the fused device dispatch dispatch_state_relaxation_cartesian_backend
 * (src/compute/dispatch/dynamics.cpp:432-470).  Profiles are the reference
 * runtime's FP64 per-level values (host memory): alpha / upper_w_alpha are
 * the upper sponge's rates at scalar and w levels (a level takes part when
 * either is > 0; upper_w_alpha applies to w when staggered), w_only_alpha the
 * lid absorber's (levels with a rate > 0), lateral_alpha the band's rate by
 * distance from the nearest lateral face.  A factor is -expm1(-alpha dt)
 * (implicit_mode: alpha dt / (1 + alpha dt)); a cell adds factor * (ref -
 * old) formed in FP64, rounded to FP32, in FP32: the reference's results bit
 * for bit.  Invalid rates or dt where the reference would evaluate them:
 * NIMBUS_ERR_INVALID_ARGUMENT, nothing changed.
 */
typedef struct nimbus_state_relaxation_args
{
    float* u;
    float* v;
    float* w;
    float* theta;
    int nx, ny, nz;
    const double* alpha;          /* [nz] upper sponge, scalar levels */
    const double* upper_w_alpha;  /* [nz] upper sponge, w levels */
    const double* w_only_alpha;   /* [nz] w-only lid absorber */
    const double* u_ref;          /* [nz] */
    const double* v_ref;          /* [nz] */
    const double* theta_ref;      /* [nz] theta0 base profile */
    int lateral_width;            /* cells from each lateral face */
    const double* lateral_alpha;  /* [lateral_width] */
    int do_upper, do_w_only, do_lateral;
    int staggered;                /* 1: w takes upper_w_alpha (C-grid) */
    int implicit_mode;
    double dt;
    int memory;
    void* stream;
} nimbus_state_relaxation_args;

nimbus_status nimbus_cuda_state_relaxation(nimbus_cuda_context* ctx, const nimbus_state_relaxation_args* a);

/*
 * Acoustic boundary closure on its own: CartesianCGridBCScheme::apply_acoustic
 * (boundary_conditions_cartesian_cgrid.cpp:141-236) with the lateral faces in
 * the order W, E, S, N and then the vertical closure.  dt_small == 0 only
 * refreshes the ghosts (the closure the split stepper runs before seeding the
 * KW78 history, dynamics.cpp:5384-5396); dt_small > 0 also integrates the
 * radiative faces against wave_history (2*(nx+ny)*nz floats, the layout of
 * nimbus_acoustic_batched_args).  Device memory only.
 */
typedef struct nimbus_boundary_args
{
    float *u, *v, *w, *rho, *p;
    float* wave_history;     /* required when dt_small > 0 and a face is radiative */
    int nx, ny, nz;
    double dx, dy;
    double dt_small;
    int bc_west, bc_east, bc_south, bc_north, bc_bottom, bc_top;
    float frame_velocity_u_ms, frame_velocity_v_ms;
    void* stream;
} nimbus_boundary_args;

nimbus_status nimbus_cuda_acoustic_boundaries(nimbus_cuda_context* ctx, const nimbus_boundary_args* a);

/*
 * Smagorinsky SGS closure on a flat C-grid (stability correction "none"),
 * the operations of TurbulenceComputeKernels
 * (include/compute/dispatch/turbulence.hpp:100-195,200-285) with the CPU
 * solver's arithmetic: FP64 over FP32 storage in the reference's order, so
 * every output is bit-identical to SmagorinskyScheme::compute and
 * apply_sgs_tendencies_cpu.  The flat filter width is formed per level on
 * the host (sqrt(dx dy) or cbrt(dx dy dz_k), the C library's functions, as
 * compute_filter_width calls them, eddy_viscosity.cpp:1414-1468).
 *
 * On a context in NIMBUS_PRECISION_FP32 the closure (coefficients and
 * tendencies) computes in FP32 instead: within 1e-6 relative of the FP64
 * result; the apply and the stability limit stay FP64.
 *
 * nimbus_cuda_smagorinsky_fused replaces dispatch_smagorinsky_fused: eddy
 * coefficients of every cell (nu = Cs^2 Delta^2 |S| capped at nu_t_max;
 * K_theta = nu / Pr_t, K_q = nu / Sc_t capped at K_max), then the
 * live-density stress divergence for u, v, w and the flux-form diffusion of
 * theta and qv (zero flux at the ground and lid; a lateral face that is
 * neither periodic nor open reflects).  nu_t / K_theta / K_q may be NULL
 * (kept in device scratch); dqvdt_sgs is zero-filled when qv is NULL.  A
 * state outside the reference's contract (u, v, w finite; theta, rho finite
 * and positive; qv finite and non-negative) or a non-finite coefficient:
 * NIMBUS_ERR_INVALID_ARGUMENT with host outputs untouched (host memory), or
 * reported by nimbus_cuda_synchronize (device memory).
 */
typedef struct nimbus_smagorinsky_args
{
    const float *u, *v, *w, *theta, *qv, *rho;  /* [nx][ny][nz]; qv may be NULL */
    const double* dz;          /* [nz] cell thickness (host memory, FP64) */
    int nx, ny, nz;            /* >= 3, 3, 2 */
    int filter_mode;           /* 0 cubic root of the cell volume, 1 sqrt(dx dy) */
    int use_horizontal, use_vertical;  /* mode: both "3d", one of them horizontal_only / vertical_only */
    int periodic_x, periodic_y;
    int open_lateral[4];       /* W, E, S, N: radiative or zero-gradient face */
    int open_top;              /* open lid (stability only) */
    double dx, dy, Cs, Pr_t, Sc_t, nu_t_max, K_max;
    float *nu_t, *K_theta, *K_q;  /* outputs, may be NULL */
    float *dudt_sgs, *dvdt_sgs, *dwdt_sgs, *dthetadt_sgs, *dqvdt_sgs;  /* outputs (inputs of the stability call) */
    int memory;
    void* stream;
} nimbus_smagorinsky_args;

nimbus_status nimbus_cuda_smagorinsky_fused(nimbus_cuda_context* ctx, const nimbus_smagorinsky_args* a);

/*
 * SGS tendency application, replacing dispatch_sgs_apply (SgsApplyDispatch,
 * turbulence.hpp:62-98) with the CPU semantics of apply_sgs_tendencies_cpu
 * (src/core/orchestration/dynamics/sgs_apply.cpp:436-956, without the energy
 * ledger): every cell, x += dt dx/dt formed in FP64, rounded to FP32 and
 * clamped (u, v to +-wind_h_max, w to +-wind_v_max, theta to [theta_min,
 * theta_max], qv to [0, qv_max]).  sanitize = primary_state_repairs_enabled:
 * non-finite tendencies count as zero, a non-finite sum falls back (winds and
 * qv to 0, theta to its old value, else theta0_base[k], else
 * theta_reference), tke stays non-negative.  qv and tke (with dtkedt and
 * dtkedt_pbl) may be NULL.  dt must be finite and positive.
 */
typedef struct nimbus_sgs_apply_args
{
    float *u, *v, *w, *theta, *qv, *tke;
    const float *dudt, *dvdt, *dwdt, *dthetadt, *dqvdt, *dtkedt, *dtkedt_pbl;
    const double* theta0_base;  /* [nz] host memory, may be NULL */
    int nx, ny, nz;
    double dt;
    int sanitize;
    double theta_reference;     /* 300 K in the reference (theta0) */
    float theta_min, theta_max, qv_max, wind_h_max, wind_v_max;  /* 200, 700, 0.05, 180, 120 */
    int memory;
    void* stream;
} nimbus_sgs_apply_args;

nimbus_status nimbus_cuda_sgs_apply(nimbus_cuda_context* ctx, const nimbus_sgs_apply_args* a);

/*
 * Explicit stability limit of the realized SGS tendencies
 * (compute_sgs_explicit_stability, sgs_apply.cpp:1483-1973) with the
 * reference's deterministic reductions (each x-slab summed serially in j-k
 * order, slabs merged in increasing i with its compensated sum): the same
 * binary64 results.  Reads the state and the five rates of `a`.  Lateral
 * faces must be periodic or closed and the lid closed to shear stress (an
 * open one needs the realized boundary-power term): NIMBUS_ERR_UNSUPPORTED
 * otherwise.  NIMBUS_ERR_INVALID_ARGUMENT for a state the reference rejects,
 * NIMBUS_ERR_NONFINITE for a non-dissipative tendency or no positive limit.
 * Synchronous.
 */
typedef struct nimbus_sgs_stability
{
    double maximum_timestep_s;
    double momentum_energy_timestep_s;
    double theta_monotonic_timestep_s;
    double qv_monotonic_timestep_s;
    double momentum_irreversible_dissipation_w;
} nimbus_sgs_stability;

nimbus_status nimbus_cuda_sgs_stability(nimbus_cuda_context* ctx, const nimbus_smagorinsky_args* a,
                                        nimbus_sgs_stability* out);

/*
 * The explicit SGS integration of one large step (dynamics.cpp:7159-7217):
 * until dt is covered, refresh the closure from the live state
 * (nimbus_cuda_smagorinsky_fused), bound the substep by the stability limit
 * and dt_sgs, and apply it (nimbus_cuda_sgs_apply).  Device memory; u, v, w,
 * theta, qv updated in place; the rate and coefficient pointers of `closure`
 * may be NULL (device scratch).  One host synchronisation per substep (the
 * limit decides its length).  time_s: the model time at the start (enters
 * the reference's progress floor).  substeps / stability_limit_s (may be
 * NULL) receive the substep count and the smallest limit seen.
 */
typedef struct nimbus_sgs_step_args
{
    nimbus_smagorinsky_args closure;  /* memory must be NIMBUS_MEMORY_DEVICE */
    const double* theta0_base;        /* [nz] host memory, may be NULL */
    double dt, dt_sgs, time_s;
    int sanitize;
} nimbus_sgs_step_args;

nimbus_status nimbus_cuda_sgs_step(nimbus_cuda_context* ctx, const nimbus_sgs_step_args* a, int* substeps,
                                   double* stability_limit_s);

/*
 * Cell-centre velocities for output.  Replaces interpolate_u_face_to_center,
 * interpolate_v_face_to_center and both interpolate_w_face_to_center forms
 * (src/core/output/stagger_interpolation.cpp), which the reference runs
 * before every history or live export of a C-grid level
 * (headless_runtime.cpp:2577-2601).  Centre i of u is 0.5f * (face i-1 +
 * face i) and cell 0 keeps face 0; v likewise in j; centre k of w is
 * 0.5f * (face k-1 + face k) for k > 0 and 0.5 * (ground_w + face 0) in FP64,
 * rounded once, for k = 0: bit-identical to the reference.  A NULL output
 * skips that component (its input may then be NULL too).  ground_w: the
 * terrain lower-face velocity of each column ([nx][ny] FP64, host memory),
 * NULL on flat ground (0).  Refused with NIMBUS_ERR_INVALID_ARGUMENT, nothing
 * written: a non-finite ground_w value (the reference's invalid_argument), an
 * output overlapping an input or another output.  Zero cells: nothing to do.
 */
typedef struct nimbus_cell_centre_args
{
    const float* u;           /* face fields [nx][ny][nz] */
    const float* v;
    const float* w;
    float* u_centre;          /* [nx][ny][nz]; NULL: skipped */
    float* v_centre;
    float* w_centre;
    const double* ground_w;   /* [nx][ny], host memory; NULL: flat ground */
    int nx, ny, nz;
    int memory;
    void* stream;
} nimbus_cell_centre_args;

nimbus_status nimbus_cuda_cell_centre_velocity(nimbus_cuda_context* ctx, const nimbus_cell_centre_args* a);

/* History fields, in the order of the reference's core volume bindings
 * (core_field_binding_array, headless_runtime.cpp:588-600). */
enum
{
    NIMBUS_HISTORY_U = 1u << 0,
    NIMBUS_HISTORY_V = 1u << 1,
    NIMBUS_HISTORY_W = 1u << 2,
    NIMBUS_HISTORY_RHO = 1u << 3,
    NIMBUS_HISTORY_P = 1u << 4,
    NIMBUS_HISTORY_THETA = 1u << 5,
    NIMBUS_HISTORY_QV = 1u << 6,
    NIMBUS_HISTORY_QC = 1u << 7,
    NIMBUS_HISTORY_QR = 1u << 8,
    NIMBUS_HISTORY_CORE = 0x1ffu
};

/*
 * One history frame of a resident level, fed from device memory: the
 * selected fields with u, v, w cell-centred (as above, on flat ground unless
 * ground_w is given), copied to host_image in the order of the bits, each
 * nx*ny*nz floats -- the payloads the reference's export writes
 * (write_or_snapshot_core_volume_fields, include/core/output/core_volume_writer.hpp:26-64).
 * Enqueued on `stream` (NULL: the context's): one centring launch into device
 * staging, one device-to-host copy for the staged velocities and one per
 * scalar field; the image
 * is complete once the stream is synchronised.  host_image should be pinned
 * (cudaHostAlloc) for the copies to run at bus rate and overlap later work.
 * A field whose bit is set must be non-NULL.
 */
typedef struct nimbus_history_args
{
    const float *u, *v, *w, *rho, *p, *theta, *qv, *qc, *qr;  /* device memory */
    unsigned fields;          /* NIMBUS_HISTORY_* bits */
    const double* ground_w;   /* [nx][ny], host memory; NULL: flat ground */
    int nx, ny, nz;
    float* host_image;
    void* stream;
} nimbus_history_args;

nimbus_status nimbus_cuda_history_snapshot(nimbus_cuda_context* ctx, const nimbus_history_args* a);

/* Host-side npy writers, byte for byte those of the reference
 * (src/core/output/npy_writer.cpp): NPY 1.0, header dict
 * "{'descr': '<f4', 'fortran_order': False, 'shape': (d0, d1, d2), }" padded
 * with spaces to a 16-byte boundary, C-order float32 payload.
 * nimbus_npy_write_3d replaces npy::write_3d (npy_writer.cpp:143-156):
 * NIMBUS_ERR_INVALID_ARGUMENT for a NULL pointer or a dimension <= 0,
 * NIMBUS_ERR_IO when the file cannot be written.  nimbus_history_write writes
 * the fields of one history image as <step_dir>/<name>.npy (u, v, w, rho, p,
 * theta, qv, qc, qr), the reference's synchronous npy export
 * (core_volume_writer.hpp:60-63); the directory must exist. */
nimbus_status nimbus_npy_write_3d(const float* data, int dim0, int dim1, int dim2, const char* path);
nimbus_status nimbus_history_write(const float* host_image, unsigned fields, int nx, int ny, int nz,
                                   const char* step_dir);

/*
 * Member engine: many runs (ensemble members, served requests) resident in
 * HBM and advanced together, each large step of every member in one batched
 * launch per phase.  No counterpart in the reference, which advances one run
 * per process; each member's arithmetic is exactly that of the per-operation
 * entry points above (same kernels, same order), so a member's result does
 * not depend on which other members share the launch.
 *
 * One large step of a member (the order of step_dynamics_new,
 * dynamics.cpp:5123-7317, for the phases this backend owns):
 *   Heun slow step; boundary refresh and KW78 seed; n_substeps acoustic
 *   substeps (retained mass flux, continuity + EOS, momentum, boundaries);
 *   conservative WENO5 transport of theta, qv, qc, qr; Kessler tendencies and
 *   their application (microphysics == 1); EOS pressure re-projection.
 * Several engines may share one context, and each may be driven from its own
 * host thread (one thread per engine at a time): an engine's step waits only
 * for its own acoustic speed scans.
 * Members may differ in grid, spacing, dt and substep count.  With Kessler
 * on, dt must not exceed 0.8 dz / (20 m/s), the bound under which the
 * reference runs the microphysics in one call instead of subcycling it.
 */
typedef struct nimbus_engine nimbus_engine;

/* Optional end-of-step sponge of an engine member: the profiles and switches
 * of nimbus_state_relaxation_args (FP64, host memory, copied at admission),
 * applied with the member's dt after the EOS projection, as
 * dynamics.cpp:7323-7340 applies it. */
typedef struct nimbus_sponge_desc
{
    const double* alpha;
    const double* upper_w_alpha;
    const double* w_only_alpha;
    const double* u_ref;
    const double* v_ref;
    const double* theta_ref;
    int lateral_width;
    const double* lateral_alpha;
    int do_upper, do_w_only, do_lateral;
    int staggered;
    int implicit_mode;
} nimbus_sponge_desc;

typedef struct nimbus_member_desc
{
    int nx, ny, nz;
    double dx, dy, dz;
    double dt;               /* large step */
    int n_substeps;          /* acoustic substeps per large step, >= 1 */
    int bc[6];               /* west, east, south, north, bottom, top */
    double coriolis_f;
    float frame_velocity_u_ms, frame_velocity_v_ms;
    int microphysics;        /* 0 none, 1 Kessler */
    /* FP64 base profiles of length nz in host memory (copied at admission) */
    const double* rho0_base;
    const double* p0_base;
    const double* qv0_base;
    const double* u0_base;   /* may be null: zero */
    const double* v0_base;   /* may be null: zero */
    const nimbus_sponge_desc* sponge;  /* may be null: no end-of-step sponge */
    int final_closure;       /* 1: end the step with the boundary closure
                                apply_full_attributed (= apply_acoustic(0) on u, v,
                                w, rho, p; dynamics.cpp:7415, after the sponge) */
    int resolve_substeps;    /* 1: re-derive the substep count before every large
                                step from the live state, as the reference does
                                (choose_runtime_timestep, src/numerics/runtime.cpp:
                                846-880, then SplitExplicitScheme::resolve_substep_count,
                                split_explicit.cpp:67-170): N = max(n_substeps,
                                ceil(dt c_max / (0.5 min(dx, dy, dz))) + 1, 2) with
                                c_max = max sqrt(gamma p / rho) over the member's cells
                                and base columns; n_substeps is then the requested
                                minimum (0: the rule alone).  0: n_substeps every step. */
} nimbus_member_desc;

/* Host arrays [nx][ny][nz] of one member's prognostic state. */
typedef struct nimbus_member_state
{
    float *u, *v, *w, *rho, *p, *theta, *qv, *qc, *qr;
} nimbus_member_state;

nimbus_status nimbus_cuda_engine_create(nimbus_cuda_context* ctx, nimbus_engine** out);
void nimbus_cuda_engine_destroy(nimbus_engine* e);
/* Device bytes one member of this shape holds while resident. */
size_t nimbus_cuda_engine_member_bytes(const nimbus_member_desc* desc);
/* Admits a member with its initial state when its footprint plus
 * reserve_bytes fits the free HBM (cudaMemGetInfo's free bytes plus what the
 * default memory pool holds unused); otherwise returns
 * NIMBUS_ERR_OUT_OF_MEMORY and changes nothing.  Does not wait for enqueued
 * steps: the arena is allocated and the state copied in stream order on the
 * engine's stream (pageable arrays are staged before the call returns, pinned
 * ones must stay untouched until the member's first step has run). */
nimbus_status nimbus_cuda_engine_admit(nimbus_engine* e, const nimbus_member_desc* desc,
                                       const nimbus_member_state* initial, size_t reserve_bytes, int* member_id);
/* Frees a member's device memory in stream order, after the enqueued steps
 * and copies that use it (does not wait). */
nimbus_status nimbus_cuda_engine_retire(nimbus_engine* e, int member_id);
/* Copies a member's current state to host arrays (waits for enqueued steps). */
nimbus_status nimbus_cuda_engine_read(nimbus_engine* e, int member_id, const nimbus_member_state* out);
/* Replaces a member's state with host arrays (waits for enqueued steps). */
nimbus_status nimbus_cuda_engine_write(nimbus_engine* e, int member_id, const nimbus_member_state* in);
/* The same copies enqueued on the engine's stream without waiting, ordered
 * with its steps: host arrays should be pinned and must stay untouched until
 * nimbus_cuda_engine_synchronize.  Several engines (each with its own stream)
 * overlap one engine's copies with another's steps. */
nimbus_status nimbus_cuda_engine_write_async(nimbus_engine* e, int member_id, const nimbus_member_state* in);
nimbus_status nimbus_cuda_engine_read_async(nimbus_engine* e, int member_id, const nimbus_member_state* out);
/* The engine's own CUDA stream (cudaStream_t), on which its steps run. */
void* nimbus_cuda_engine_stream(const nimbus_engine* e);
/* The state image: every member's nine prognostic fields in one block, members
 * in admission order, each member's fields in nimbus_member_state order (u, v,
 * w, rho, p, theta, qv, qc, qr), each nx*ny*nz floats.  Moving it costs one
 * host<->device copy per direction plus one device pass that scatters it into
 * (or gathers it from) the members' current buffers, where the per-member
 * copies above cost nine each: many small copies in both directions at once
 * run well below the bus rate, one large copy each way runs at it.
 * image_bytes: the image size (0 for an empty engine); image_offset: a
 * member's byte offset in it ((size_t)-1 for an unknown id). */
size_t nimbus_cuda_engine_image_bytes(const nimbus_engine* e);
size_t nimbus_cuda_engine_image_offset(const nimbus_engine* e, int member_id);
/* Enqueue the image copies on the engine's stream, ordered with its steps
 * (host memory should be pinned and stay untouched until synchronize). */
nimbus_status nimbus_cuda_engine_upload_image_async(nimbus_engine* e, const void* host_image);
nimbus_status nimbus_cuda_engine_download_image_async(nimbus_engine* e, void* host_image);
/* One history frame of a member (flat ground), enqueued on the engine's
 * stream after its enqueued steps: the nimbus_cuda_history_snapshot image of
 * the member's current state (fields as NIMBUS_HISTORY_* bits, nx*ny*nz floats
 * each).  host_image should be pinned and is complete after
 * nimbus_cuda_engine_synchronize. */
nimbus_status nimbus_cuda_engine_history_async(nimbus_engine* e, int member_id, unsigned fields, void* host_image);
/* Lanes: the members are split into up to `lanes` size-balanced groups whose
 * launches run on parallel streams (branches of the one step graph), so one
 * group's kernels fill the SMs another's launch tails leave idle.  Results do
 * not depend on the lane count.  Default 4; takes effect at the next step.
 * nimbus_cuda_engine_lanes: the lanes the current table uses. */
nimbus_status nimbus_cuda_engine_set_lanes(nimbus_engine* e, int lanes);
int nimbus_cuda_engine_lanes(const nimbus_engine* e);
/* Kernel form of the acoustic substep's continuity and momentum passes (the
 * bulk of a step).  Results do not depend on it; it takes effect at the next
 * step.
 *   NIMBUS_ACOUSTIC_TABLE  one thread per cell, each member's parameters and
 *                          buffers read from the member table in HBM;
 *   NIMBUS_ACOUSTIC_CONST  one thread per cell, each lane's members' constants
 *                          passed as one kernel parameter (the constant bank),
 *                          only the rotating buffers read from the table
 *                          (the continuity pass's default; lanes of more than
 *                          64 members fall back to the table form);
 *   NIMBUS_ACOUSTIC_MARCH  one thread advances nimbus_cuda_engine_set_march
 *                          consecutive cells of a row along x (default 16),
 *                          neighbour data of the previous cell carried over in
 *                          registers (the momentum pass's default);
 *   NIMBUS_ACOUSTIC_PAIR   the constant-bank form with two vertically
 *                          adjacent cells per thread (in members with an even
 *                          nz the pair's values are one 8-byte load per field
 *                          and neighbour; both cells' loads are issued before
 *                          either's arithmetic);
 *   NIMBUS_ACOUSTIC_BULK   the constant-bank form with each 256-cell tile's
 *                          stencil data staged in shared memory by bulk
 *                          copies (cp.async.bulk on an mbarrier, four tiles in
 *                          flight per CTA); a staged copy that does not
 *                          complete sets member status bit 32 and the step
 *                          fails with NIMBUS_ERR_CUDA at synchronisation;
 *   NIMBUS_ACOUSTIC_CMARCH the marching form with the constant-bank
 *                          parameters.
 * nimbus_cuda_engine_set_acoustic_form sets both passes; set_pass_forms sets
 * each; nimbus_cuda_engine_acoustic_form reports the continuity pass's. */
enum
{
    NIMBUS_ACOUSTIC_TABLE = 0,
    NIMBUS_ACOUSTIC_CONST = 1,
    NIMBUS_ACOUSTIC_MARCH = 2,
    NIMBUS_ACOUSTIC_PAIR = 3,
    NIMBUS_ACOUSTIC_BULK = 4,
    NIMBUS_ACOUSTIC_CMARCH = 5
};
nimbus_status nimbus_cuda_engine_set_acoustic_form(nimbus_engine* e, int form);
int nimbus_cuda_engine_acoustic_form(const nimbus_engine* e);
nimbus_status nimbus_cuda_engine_set_pass_forms(nimbus_engine* e, int continuity_form, int momentum_form);
nimbus_status nimbus_cuda_engine_pass_forms(const nimbus_engine* e, int* continuity_form, int* momentum_form);
nimbus_status nimbus_cuda_engine_set_march(nimbus_engine* e, int planes);
int nimbus_cuda_engine_march(const nimbus_engine* e);

/* The engine autotuner (no counterpart in the reference).  Times candidate
 * launch configurations on the resident members themselves, `steps` timed
 * steps each after one warm-up step, keeps the fastest and reports every
 * candidate's time: first the lane count {1, 2, 4, 6, 8} (at most the member
 * count) with the constant-bank form, then, at the fastest lane count, every
 * pair of pass forms (continuity x momentum, each of constant bank, member
 * table, marching 16 planes, two cells per thread, bulk-staged tiles,
 * constant-bank marching).  The members' states are
 * saved on the device before and restored after, so the runs are where they
 * were (status words and substep counts may reflect the tuning steps).
 * Waits for the device. */
#define NIMBUS_TUNING_CANDIDATES 48
typedef struct nimbus_engine_tuning
{
    int lanes, acoustic_form, march;  /* the chosen configuration (now set); acoustic_form: continuity */
    int momentum_form;
    double ms_per_step;               /* its time */
    int candidates;
    int candidate_lanes[NIMBUS_TUNING_CANDIDATES];
    int candidate_form[NIMBUS_TUNING_CANDIDATES];
    int candidate_momentum_form[NIMBUS_TUNING_CANDIDATES];
    int candidate_march[NIMBUS_TUNING_CANDIDATES];
    double candidate_ms[NIMBUS_TUNING_CANDIDATES];
} nimbus_engine_tuning;

nimbus_status nimbus_cuda_engine_autotune(nimbus_engine* e, int steps, nimbus_engine_tuning* out);
/* Enqueues n_steps large steps of every resident member on the engine's
 * stream: replayed from a CUDA graph when graphs are on (the default), the
 * graph rebuilt after admissions, retirements, a precision change or a
 * changed substep count.  With resolve_substeps members, each step first
 * scans every member's acoustic speed on the device and waits for the
 * per-member maxima (a few bytes) before enqueuing the step, since the
 * step's launches depend on the counts. */
nimbus_status nimbus_cuda_engine_step(nimbus_engine* e, int n_steps);
/* Waits for the enqueued steps; NIMBUS_ERR_NONFINITE when a retained mass
 * flux or transported scalar went non-finite or the EOS projection refused. */
nimbus_status nimbus_cuda_engine_synchronize(nimbus_engine* e);
/* A member's status bits (1 non-finite mass flux, 2 non-finite transported
 * scalar, 4 EOS projection refused, 16 a pressure or density failed the
 * acoustic speed scan); waits for enqueued steps. */
nimbus_status nimbus_cuda_engine_member_status(nimbus_engine* e, int member_id, unsigned* flags);
/* The same status bits copied into pinned host memory in stream order (after
 * the enqueued steps), without waiting: read them once the stream has passed
 * that point (an event recorded after the call, or a synchronisation). */
nimbus_status nimbus_cuda_engine_member_status_async(nimbus_engine* e, int member_id, unsigned* host_flags);
/* How often the engine instantiated its step graphs and how often it updated
 * an instantiated graph in place (an admission or retirement that keeps the
 * graphs' shape). */
nimbus_status nimbus_cuda_engine_graph_builds(const nimbus_engine* e, uint64_t* instantiations, uint64_t* updates);
/* The acoustic substep count of a member's last enqueued (or, before any,
 * its first) large step. */
nimbus_status nimbus_cuda_engine_member_substeps(nimbus_engine* e, int member_id, int* n_substeps);
nimbus_status nimbus_cuda_engine_set_graph(nimbus_engine* e, int enable);
int nimbus_cuda_engine_members(const nimbus_engine* e);
/* Kernel launches one large step enqueues (batched over all members). */
int nimbus_cuda_engine_launches_per_step(const nimbus_engine* e);

#ifdef __cplusplus
}
#endif

#endif /* NIMBUS_CUDA_H */
