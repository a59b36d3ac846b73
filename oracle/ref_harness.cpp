// Test infrastructure, not product code.
//
// A thin extern "C" harness around the reference Nimbus CPU solver, linked
// from the reference's own sources (oracle/ref.mk builds them, unmodified,
// into oracle/_ref/libnimbus_ref.a).  It lets the Python tests and the CPU
// baseline of bench.py drive the reference's real kernels on arrays that the
// CUDA path also receives:
//
//   ref_acoustic_fused      CpuComputeBackend::dispatch_acoustic_substep_fused_cartesian_cgrid
//                           (src/compute/cpu/acoustic_cgrid.cpp:50, fast path
//                           src/compute/cpu/acoustic_cgrid_fast.cpp:12-219)
//   ref_acoustic_loop       the production per-substep order of
//                           SplitExplicitScheme::step_split_acoustic
//                           (src/numerics/time_stepping/schemes/split_explicit/split_explicit.cpp:174-260):
//                           seed KW78 radiation, then N x {retained mass-flux accumulate
//                           (advection_cartesian.cpp:610-870, Host precision, as
//                           dynamics.cpp:4545-4557 calls it), fused substep, apply_acoustic(dt_s)
//                           (boundary_conditions_cartesian_cgrid.cpp:141,884-1187)}
//   ref_slow_tendencies     CartesianCGrid3DScheme::compute_slow_tendencies
//                           (src/dynamics/schemes/klemp_wilhelmson_split/cartesian_cgrid_3d.cpp:724-1416)
//                           on a stationary flat level with moisture and Kessler loading
//   ref_backend_slow_tendencies  the same on the scheme's device route through a
//                           loaded backend (cartesian_cgrid_3d.cpp:835-925)
//   ref_kessler_tendencies  KesslerScheme::compute_tendencies
//                           (src/microphysics/schemes/kessler/kessler.cpp:103-520)
//   ref_backend_kessler_tendencies  the same scheme on its device route through a
//                           loaded backend (kessler.cpp:152-300: the Kessler pointwise
//                           and sedimentation dispatches)
//   ref_acoustic_boundaries CartesianCGridBCScheme::apply_acoustic
//                           (boundary_conditions_cartesian_cgrid.cpp:141-236)
//   ref_eos_projection      tmv::dynamics_eos::apply_pressure_projection
//                           (src/core/orchestration/dynamics/eos_apply.cpp:50-200)
//   ref_state_relaxation    apply_rayleigh_damping then apply_lateral_damping
//                           (src/core/infra/rayleigh_damping.cpp:720-1119,1194-1476),
//                           the end-of-step sponge of dynamics.cpp:7323-7340, with
//                           the per-level profiles its runtime built
//   ref_cell_centre         interpolate_u/v/w_face_to_center
//                           (src/core/output/stagger_interpolation.cpp), the C-grid
//                           output staging of the history and live export
//                           (headless_runtime.cpp:2577-2601)
//   ref_npy_write_3d        npy::write_3d (src/core/output/npy_writer.cpp:143-156)
//   ref_smagorinsky         SmagorinskyScheme::compute on the flat C-grid CPU path
//                           (src/turbulence/schemes/smagorinsky/smagorinsky.cpp:96-440:
//                           eddy coefficients, then compute_momentum_diffusion_tendencies
//                           and compute_scalar_diffusion_tendencies,
//                           src/turbulence/base/eddy_viscosity.cpp:1532-2090)
//   ref_sgs_apply           apply_admitted_sgs_substep, CPU path
//                           (src/core/orchestration/dynamics/sgs_apply.cpp:436-956,1975-2029)
//   ref_sgs_stability       compute_sgs_explicit_stability (sgs_apply.cpp:1483-1973)
//   ref_backend_acoustic_fused, ref_backend_acoustic_batched, ref_backend_smagorinsky
//                           the same reference calls with a ComputeBackend loaded
//                           from a shared library (the CUDA backend's adapter,
//                           nimbus_cuda_create_compute_backend): the reference's own
//                           dispatch structs and, for the closure, its own
//                           SmagorinskyScheme::compute routing to the backend
//                           through dispatch_smagorinsky_fused_backend
//   ref_backend_scalar_transport  the same transport through the reference's bridge
//                           dispatch_advect_scalars_conservative_cartesian_cgrid_backend
//                           (src/compute/dispatch/advection.cpp:95-150) to a loaded backend
//   ref_resolve_substep_count, ref_max_sound_speed  SplitExplicitScheme::resolve_substep_count
//                           and the acoustic speed choose_runtime_timestep samples
//   ref_scalar_transport    advect_scalars_conservative_3d_cartesian
//                           (advection_cartesian.cpp:3532) on a retained context whose
//                           face mass fluxes and beginning density are supplied
//                           (CartesianCGridTransportContext::record_external_accumulation).
//
// Nothing here re-implements the physics; every number comes from the
// reference objects.  Errors are reported as a negative return code and a
// message retrievable with ref_last_error().
#include "compute/backend_interface.hpp"
#include "compute/compute_backend_factory.hpp"
#include "compute/dispatch/dynamics.hpp"
#include "boundary_conditions/factory.hpp"
#include "boundary_conditions/boundary_conditions_base.hpp"
#include "core/field/field3d.hpp"
#include "core/field/field_bounds.hpp"
#include "core/runtime/simulation_state.hpp"
#include "core/runtime/runtime_config.hpp"
#include "dynamics/dynamics_base.hpp"
#include "numerics/advection/advection_cartesian.hpp"
#include "dynamics/schemes/klemp_wilhelmson_split/cartesian_cgrid_3d.hpp"
#include "microphysics/schemes/kessler/kessler.hpp"
#include "dynamics/eos_pressure.hpp"
#include "core/infra/rayleigh_damping.hpp"
#include "core/output/npy_writer.hpp"
#include "core/output/stagger_interpolation.hpp"
#include "core/orchestration/dynamics/sgs_apply.hpp"
#include "core/orchestration/dynamics/sgs_apply_internal.hpp"
#include "compute/backend_runtime.hpp"
#include "diagnostics/deterministic_reduction.hpp"
#include "turbulence/schemes/smagorinsky/smagorinsky.hpp"
#include "numerics/runtime.hpp"
#include "compute/bridge/advection.hpp"
#include "compute/bridge/dynamics.hpp"
#include "dynamics/coriolis.hpp"
#include "numerics/time_stepping/schemes/split_explicit/split_explicit.hpp"

#include <dlfcn.h>

#include <algorithm>
#include <cstring>
#include <exception>
#include <memory>
#include <string>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace
{
thread_local std::string g_error;

int fail(const char* what)
{
    g_error = what;
    return -1;
}

void to_field(Field3D& f, const float* src, int nx, int ny, int nz)
{
    f.resize(nx, ny, nz, 0.0f);
    std::memcpy(f.data(), src, sizeof(float) * static_cast<std::size_t>(nx) * ny * nz);
}

void from_field(float* dst, const Field3D& f)
{
    std::memcpy(dst, const_cast<Field3D&>(f).data(), sizeof(float) * f.size());
}

// A compute backend: the reference's CPU backend, or one created by the
// factory symbol of a shared library (loaded once, never unloaded).
std::unique_ptr<ComputeBackend> load_backend(const char* library)
{
    if (!library) return create_cpu_compute_backend();
    void* handle = dlopen(library, RTLD_NOW | RTLD_LOCAL);
    if (!handle) throw std::runtime_error(std::string("dlopen: ") + dlerror());
    using Factory = ComputeBackend* (*)();
    auto make = reinterpret_cast<Factory>(dlsym(handle, "nimbus_cuda_create_compute_backend"));
    if (!make) throw std::runtime_error("library has no nimbus_cuda_create_compute_backend");
    return std::unique_ptr<ComputeBackend>(make());
}

using tmv::init::config::BottomBC;
using tmv::init::config::LateralBC;
using tmv::init::config::TopBC;

// A self-contained level for one call: grid, fields, base profiles and the
// boundary-condition configuration, viewed exactly as the solver views its own.
struct Level
{
    SimulationStorageState storage;
    SimulationStateView view;

    static SimulationStorageState& configured(SimulationStorageState& s, int nx, int ny, int nz,
                                              double dx, double dy, double dz)
    {
        s.configuration.stagger_type = StaggerType::CGrid;
        s.grid.geometry.initialize(nx, ny, nz, dx, dz, dy, CoordinateSystem::Cartesian, StaggerType::CGrid);
        return s;
    }

    Level(int nx, int ny, int nz, double dx, double dy, double dz, double dt)
        : storage(GridStorageState(nx, ny, nz, dx, dz, dt, dy)),
          view(make_simulation_state_view(configured(storage, nx, ny, nz, dx, dy, dz)))
    {
    }

    void set_bcs(int west, int east, int south, int north, int bottom, int top)
    {
        auto& c = storage.configuration;
        c.lateral_bc_west = static_cast<LateralBC>(west);
        c.lateral_bc_east = static_cast<LateralBC>(east);
        c.lateral_bc_south = static_cast<LateralBC>(south);
        c.lateral_bc_north = static_cast<LateralBC>(north);
        c.bottom_bc = static_cast<BottomBC>(bottom);
        c.top_bc = static_cast<TopBC>(top);
    }
};

AcousticSubstepFusedCartesianCgridDispatch make_fused(Level& L, const double* rho0, const double* p0b,
                                                      double dt_small, float* drho_scratch)
{
    auto& f = L.storage.fields;
    AcousticSubstepFusedCartesianCgridDispatch d;
    d.u = f.u.data();
    d.v = f.v.data();
    d.w = f.w.data();
    d.rho = f.rho.data();
    d.p = f.p.data();
    d.theta_data = f.theta.data();
    d.base_len = L.storage.grid.nz;
    d.nx = L.storage.grid.nr;
    d.ny = L.storage.grid.nth;
    d.nz = L.storage.grid.nz;
    d.gamma_val = static_cast<float>(dynamics_constants::gamma);
    d.rho_min = density_min_kgm3;
    d.rho_max = density_max_kgm3;
    d.p_min = pressure_min_pa;
    d.p_max = pressure_max_pa;
    d.p_ref_fallback = static_cast<float>(p0);
    d.wind_clamp_h = wind_horizontal_abs_max_ms;
    d.wind_clamp_v = wind_vertical_abs_max_ms;
    d.rho0_base_host = rho0;
    d.p0_base_host = p0b;
    d.dx_host = L.storage.grid.dx;
    d.dy_host = L.storage.grid.dy;
    d.dz_host = L.storage.grid.dz;
    d.dt_small_host = dt_small;
    d.gamma_host = dynamics_constants::gamma;
    d.drho_scratch = drho_scratch;
    return d;
}
} // namespace

extern "C" {

const char* ref_last_error(void) { return g_error.c_str(); }

int ref_set_threads(int n)
{
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

// One fused acoustic substep on host arrays, in place, through `library`'s
// backend (null: the reference's CPU backend).
int ref_backend_acoustic_fused(const char* library, float* u, float* v, float* w, float* rho, float* p,
                               const float* theta, const double* rho0, const double* p0b, int nx, int ny, int nz,
                               double dx, double dy, double dz, double dt_small, float* drho_scratch)
{
    try
    {
        auto backend = load_backend(library);
        std::string err;
        if (!backend->initialize(err)) return fail(err.c_str());
        AcousticSubstepFusedCartesianCgridDispatch d;
        d.u = u; d.v = v; d.w = w; d.rho = rho; d.p = p; d.theta_data = theta;
        d.base_len = nz; d.nx = nx; d.ny = ny; d.nz = nz;
        d.gamma_val = static_cast<float>(dynamics_constants::gamma);
        d.rho_min = density_min_kgm3; d.rho_max = density_max_kgm3;
        d.p_min = pressure_min_pa; d.p_max = pressure_max_pa;
        d.p_ref_fallback = static_cast<float>(p0);
        d.wind_clamp_h = wind_horizontal_abs_max_ms; d.wind_clamp_v = wind_vertical_abs_max_ms;
        d.rho0_base_host = rho0; d.p0_base_host = p0b;
        d.dx_host = dx; d.dy_host = dy; d.dz_host = dz; d.dt_small_host = dt_small;
        d.gamma_host = dynamics_constants::gamma;
        d.drho_scratch = drho_scratch;
        if (!backend->dynamics_kernels()->dispatch_acoustic_substep_fused_cartesian_cgrid(d))
            return fail("the backend refused the fused acoustic dispatch");
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// The whole acoustic loop of a large step through `library`'s backend as the
// reference's accelerator route hands it over: an
// AcousticSubstepsBatchedCartesianCgridDispatch with FP32 base profiles,
// spacings and dt_small (narrowed here from the FP64 inputs), the strict
// contract's KW78 history in and out and the mass-flux weight 1/n.
int ref_backend_acoustic_batched(const char* library, float* u, float* v, float* w, float* rho, float* p,
                                 const float* theta, const double* rho0, const double* p0b, int nx, int ny, int nz,
                                 double dx, double dy, double dz, double dt_small, int n_substeps, const int* bc,
                                 float* mfx, float* mfy, float* mfz, const float* wave_in, float* wave_out)
{
    try
    {
        auto backend = load_backend(library);
        std::string err;
        if (!backend->initialize(err)) return fail(err.c_str());
        std::vector<float> r0(rho0, rho0 + nz), pb(p0b, p0b + nz);
        AcousticSubstepsBatchedCartesianCgridDispatch d;
        d.u = u; d.v = v; d.w = w; d.rho = rho; d.p = p; d.theta_data = theta;
        d.rho0_base_data = r0.data(); d.p0_base_data = pb.data(); d.base_len = nz;
        d.nx = nx; d.ny = ny; d.nz = nz;
        d.dx = static_cast<float>(dx); d.dy = static_cast<float>(dy); d.dz = static_cast<float>(dz);
        d.gamma_val = static_cast<float>(dynamics_constants::gamma);
        d.dt_small = static_cast<float>(dt_small); d.n_substeps = n_substeps;
        d.rho_min = density_min_kgm3; d.rho_max = density_max_kgm3;
        d.p_min = pressure_min_pa; d.p_max = pressure_max_pa;
        d.p_ref_fallback = static_cast<float>(p0);
        d.wind_clamp_h = wind_horizontal_abs_max_ms; d.wind_clamp_v = wind_vertical_abs_max_ms;
        d.bc_west = bc[0]; d.bc_east = bc[1]; d.bc_south = bc[2]; d.bc_north = bc[3];
        d.bc_bottom = bc[4]; d.bc_top = bc[5];
        d.mass_flux_x = mfx; d.mass_flux_y = mfy; d.mass_flux_z = mfz;
        d.accumulate_mass_flux = true;
        d.mass_flux_weight = 1.0 / n_substeps;
        d.wave_history = wave_in;
        d.wave_history_output = wave_out;
        if (!backend->dynamics_kernels() ||
            !backend->dynamics_kernels()->supports(DynamicsKernelOp::AcousticSubstepsBatchedCartesianCgrid))
            return fail("the backend does not offer the batched acoustic loop");
        if (!backend->dynamics_kernels()->dispatch_acoustic_substeps_batched_cartesian_cgrid(d))
            return fail("the backend refused the batched acoustic dispatch");
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// The reference CPU backend's fused substep (see ref_backend_acoustic_fused).
int ref_acoustic_fused(float* u, float* v, float* w, float* rho, float* p, const float* theta,
                       const double* rho0, const double* p0b, int nx, int ny, int nz,
                       double dx, double dy, double dz, double dt_small, float* drho_scratch)
{
    return ref_backend_acoustic_fused(nullptr, u, v, w, rho, p, theta, rho0, p0b, nx, ny, nz, dx, dy, dz, dt_small,
                                      drho_scratch);
}

// The boundary closure alone: CartesianCGridBCScheme::apply_acoustic(dt_small)
// on u, v, w, rho, p in place (dt_small == 0 refreshes the ghosts, the call
// seed_acoustic_radiation's caller makes before seeding).
int ref_acoustic_boundaries(float* u, float* v, float* w, float* rho, float* p, int nx, int ny, int nz, double dx,
                            double dy, double dz, double dt_small, int bc_west, int bc_east, int bc_south,
                            int bc_north, int bc_bottom, int bc_top)
{
    try
    {
        Level L(nx, ny, nz, dx, dy, dz, 1.0);
        L.set_bcs(bc_west, bc_east, bc_south, bc_north, bc_bottom, bc_top);
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.rho, rho, nx, ny, nz);
        to_field(f.p, p, nx, ny, nz);
        auto bc = tmv::create_cartesian_cgrid_bc_scheme(L.view);
        bc->apply_acoustic(dt_small);
        from_field(u, f.u);
        from_field(v, f.v);
        from_field(w, f.w);
        from_field(rho, f.rho);
        from_field(p, f.p);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// The acoustic substep loop of one large step, in place, exporting the
// time-averaged face mass fluxes, the beginning density and the KW78
// radiation history (layout: u_west[ny*nz], u_east[ny*nz], v_south[nx*nz],
// v_north[nx*nz]).  wave_in may be null: the loop then seeds from the
// post-slow faces, which is what seed_acoustic_radiation does every step.
int ref_acoustic_loop(float* u, float* v, float* w, float* rho, float* p, const float* theta,
                      const double* rho0, const double* p0b, int nx, int ny, int nz,
                      double dx, double dy, double dz, double dt_large, int n_substeps,
                      int bc_west, int bc_east, int bc_south, int bc_north, int bc_bottom, int bc_top,
                      float* mfx, float* mfy, float* mfz, float* rho_begin, float* wave_out)
{
    try
    {
        if (n_substeps < 1) return fail("n_substeps must be >= 1");
        Level L(nx, ny, nz, dx, dy, dz, dt_large);
        L.set_bcs(bc_west, bc_east, bc_south, bc_north, bc_bottom, bc_top);
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.rho, rho, nx, ny, nz);
        to_field(f.p, p, nx, ny, nz);
        to_field(f.theta, theta, nx, ny, nz);
        Field3D scratch(nx, ny, nz, 0.0f);

        auto backend = create_cpu_compute_backend();
        std::string err;
        if (!backend->initialize(err)) return fail(err.c_str());
        auto bc = tmv::create_cartesian_cgrid_bc_scheme(L.view);
        tmv::CartesianCGridTransportContext ctx;
        ctx.begin(L.view, nx, ny, nz, dt_large);

        const double dt_small = dt_large / n_substeps;
        bc->seed_acoustic_radiation();
        for (int n = 0; n < n_substeps; ++n)
        {
            ctx.accumulate(L.view, f.rho, f.u, f.v, f.w, dt_small);
            auto d = make_fused(L, rho0, p0b, dt_small, scratch.data());
            if (!backend->dynamics_kernels()->dispatch_acoustic_substep_fused_cartesian_cgrid(d))
                return fail("the backend refused the fused acoustic dispatch");
            bc->apply_acoustic(dt_small);
        }
        ctx.complete(L.view);

        from_field(u, f.u);
        from_field(v, f.v);
        from_field(w, f.w);
        from_field(rho, f.rho);
        from_field(p, f.p);
        if (mfx) from_field(mfx, ctx.mass_flux_x);
        if (mfy) from_field(mfy, ctx.mass_flux_y);
        if (mfz) from_field(mfz, ctx.mass_flux_z);
        if (rho_begin) from_field(rho_begin, ctx.density_begin);
        if (wave_out)
        {
            const auto& s = *L.view.boundary_condition_runtime;
            const std::size_t yz = std::size_t(ny) * nz, xz = std::size_t(nx) * nz;
            std::memcpy(wave_out, s.radiative_u_west.data(), yz * sizeof(float));
            std::memcpy(wave_out + yz, s.radiative_u_east.data(), yz * sizeof(float));
            std::memcpy(wave_out + 2 * yz, s.radiative_v_south.data(), xz * sizeof(float));
            std::memcpy(wave_out + 2 * yz + xz, s.radiative_v_north.data(), xz * sizeof(float));
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// Conservative WENO5 (or MC) transport of n scalars, in place, against the
// supplied retained face mass fluxes.  rho_end is the density the dynamics
// retained; rho_begin the density paired with the scalars at step start.
int ref_scalar_transport(float** q, const int* positive_definite, int n_scalars,
                         const float* u, const float* v, const float* w, const float* rho_end,
                         const float* rho_begin, const float* mfx, const float* mfy, const float* mfz,
                         int nx, int ny, int nz, double dx, double dy, double dz, double dt,
                         int weno, int top_open)
{
    try
    {
        if (n_scalars < 0 || n_scalars > 16) return fail("n_scalars out of range");
        Level L(nx, ny, nz, dx, dy, dz, dt);
        L.set_bcs(4, 4, 4, 4, 1, top_open ? 2 : 0);
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.rho, rho_end, nx, ny, nz);
        tmv::CartesianCGridTransportContext ctx;
        ctx.begin(L.view, nx, ny, nz, dt);
        Field3D begin_density;
        to_field(begin_density, rho_begin, nx, ny, nz);
        ctx.capture_density_begin(begin_density);
        std::memcpy(ctx.mass_flux_x.data(), mfx, sizeof(float) * f.u.size());
        std::memcpy(ctx.mass_flux_y.data(), mfy, sizeof(float) * f.u.size());
        std::memcpy(ctx.mass_flux_z.data(), mfz, sizeof(float) * f.u.size());
        ctx.record_external_accumulation(dt, 1);
        ctx.complete(L.view);

        std::unique_ptr<Field3D[]> fields(new Field3D[n_scalars > 0 ? n_scalars : 1]);
        tmv::CartesianScalarTransport scalars[16]{};
        for (int s = 0; s < n_scalars; ++s)
        {
            to_field(fields[s], q[s], nx, ny, nz);
            scalars[s].field = &fields[s];
            scalars[s].kappa = 0.0;
            scalars[s].positive_definite = positive_definite[s] != 0;
        }
        tmv::advect_scalars_conservative_3d_cartesian(
            L.view, scalars, static_cast<std::size_t>(n_scalars), dt, &ctx,
            weno ? tmv::CartesianFaceReconstruction::WENO5 : tmv::CartesianFaceReconstruction::MonotonicCentered);
        for (int s = 0; s < n_scalars; ++s)
            from_field(q[s], fields[s]);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// Kessler warm-rain tendencies (dtheta, dqv, dqc, dqr) over the cell domain
// {i0, i1, j0, j1, k0, k1} with uniform vertical spacing dz: the scheme's CPU
// route, or (library given) its device route through that library's
// ComputeBackend (kessler.cpp:152-300: the pointwise and sedimentation
// dispatches, the scheme throwing rather than falling back).
int ref_backend_kessler_tendencies(const char* library, const float* theta, const float* p, const float* rho,
                                   const float* qv, const float* qc, const float* qr, int nx, int ny, int nz,
                                   double dz, double dt, const int* domain, float* dth, float* dqv, float* dqc,
                                   float* dqr)
{
    try
    {
        ComputeBackendRuntimeState runtime;
        if (library)
        {
            runtime.backend = load_backend(library);
            std::string err;
            if (!runtime.backend->initialize(err)) return fail(err.c_str());
            runtime.active_kind = ComputeBackendKind::Vulkan;  // any accelerator kind
            runtime.requested_kind = runtime.active_kind;
        }
        Field3D fth, fp, frho, fqv, fqc, fqr;
        to_field(fth, theta, nx, ny, nz);
        to_field(fp, p, nx, ny, nz);
        to_field(frho, rho, nx, ny, nz);
        to_field(fqv, qv, nx, ny, nz);
        to_field(fqc, qc, nx, ny, nz);
        to_field(fqr, qr, nx, ny, nz);
        Field3D zero(nx, ny, nz, 0.0f);
        Field3D o_th, o_qv, o_qc, o_qr, o_qi, o_qs, o_qg, o_qh;
        tmv::KesslerScheme scheme;
        scheme.set_vertical_spacing_m(dz);
        PhysicalCellDomain d;
        d.i_begin = domain[0]; d.i_end = domain[1];
        d.j_begin = domain[2]; d.j_end = domain[3];
        d.k_begin = domain[4]; d.k_end = domain[5];
        scheme.set_physical_cell_domain(nx, ny, nz, d);
        if (library)
        {
            scheme.bind_execution_owners(runtime, nullptr);
            scheme.set_require_native_dispatch(true);
        }
        scheme.compute_tendencies(fp, fth, frho, fqv, fqc, fqr, zero, zero, zero, zero, dt, o_th, o_qv, o_qc, o_qr,
                                  o_qi, o_qs, o_qg, o_qh);
        from_field(dth, o_th);
        from_field(dqv, o_qv);
        from_field(dqc, o_qc);
        from_field(dqr, o_qr);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

int ref_kessler_tendencies(const float* theta, const float* p, const float* rho, const float* qv, const float* qc,
                           const float* qr, int nx, int ny, int nz, double dz, double dt, const int* domain,
                           float* dth, float* dqv, float* dqc, float* dqr)
{
    return ref_backend_kessler_tendencies(nullptr, theta, p, rho, qv, qc, qr, nx, ny, nz, dz, dt, domain, dth, dqv,
                                          dqc, dqr);
}

// EOS pressure re-projection on a level whose p is replaced in place.  With
// qv/qc/qr given the state is complete (ice and TKE zero) and the reference's
// moist energy attribution and its extra rejection checks run too.  Returns 0
// when p was published, 1 when the reference refused the state (p untouched).
int ref_eos_projection(const float* rho, const float* theta, float* p, const float* qv, const float* qc,
                       const float* qr, int nx, int ny, int nz, double dx, double dy, double dz)
{
    try
    {
        Level L(nx, ny, nz, dx, dy, dz, 1.0);
        auto& f = L.storage.fields;
        for (Field3D* z : {&f.u, &f.v, &f.w}) z->resize(nx, ny, nz, 0.0f);
        to_field(f.rho, rho, nx, ny, nz);
        to_field(f.theta, theta, nx, ny, nz);
        to_field(f.p, p, nx, ny, nz);
        if (qv)
        {
            to_field(f.qv, qv, nx, ny, nz);
            to_field(f.qc, qc, nx, ny, nz);
            to_field(f.qr, qr, nx, ny, nz);
            for (Field3D* z : {&f.qi, &f.qs, &f.qg, &f.qh, &f.tke}) z->resize(nx, ny, nz, 0.0f);
        }
        try
        {
            tmv::dynamics_eos::apply_pressure_projection(L.view);
        }
        catch (const std::runtime_error& e)
        {
            g_error = e.what();
            return 1;
        }
        from_field(p, f.p);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// Slow tendencies (du, dv, dw at faces; dp at centres) of the reference's
// C-grid scheme.  qv/qc/qr may be null (dry / no loading); base profiles are
// FP64 columns of length nz.
// The slow tendencies on the CPU route, or (library given) on the scheme's
// device route through that library's ComputeBackend
// (cartesian_cgrid_3d.cpp:835-925, dispatch_cartesian_cgrid_slow_tendencies);
// beta != 0 sets a beta-plane Coriolis profile (f at grid y = 0, df/dy).
int ref_backend_slow_tendencies(const char* library, const float* u, const float* v, const float* w,
                                const float* rho, const float* p, const float* theta, const float* qv,
                                const float* qc, const float* qr, const double* rho0, const double* p0b,
                                const double* qv0, const double* u0, const double* v0, const double* theta0, int nx,
                                int ny, int nz, double dx, double dy, double dz, double coriolis_f, double beta,
                                float* du, float* dv, float* dw, float* dp)
{
    try
    {
        ComputeBackendRuntimeState runtime;
        if (library)
        {
            runtime.backend = load_backend(library);
            std::string err;
            if (!runtime.backend->initialize(err)) return fail(err.c_str());
            runtime.active_kind = ComputeBackendKind::Vulkan;  // any accelerator kind
            runtime.requested_kind = runtime.active_kind;
        }
        Level L(nx, ny, nz, dx, dy, dz, 1.0);
        if (library) L.view.compute_runtime = &runtime;
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.rho, rho, nx, ny, nz);
        to_field(f.p, p, nx, ny, nz);
        to_field(f.theta, theta, nx, ny, nz);
        if (qv) to_field(f.qv, qv, nx, ny, nz);
        if (qc)
        {
            to_field(f.qc, qc, nx, ny, nz);
            to_field(f.qr, qr, nx, ny, nz);
            for (Field3D* z : {&f.qi, &f.qs, &f.qg, &f.qh}) z->resize(nx, ny, nz, 0.0f);
        }
        auto& b = L.storage.base;
        b.rho0.assign(rho0, rho0 + nz);
        b.p0.assign(p0b, p0b + nz);
        if (qv0) b.qv0.assign(qv0, qv0 + nz);
        if (u0) b.u0.assign(u0, u0 + nz);
        if (v0) b.v0.assign(v0, v0 + nz);
        if (theta0) b.theta0.assign(theta0, theta0 + nz);
        L.storage.coriolis_f = coriolis_f;
        tmv::CartesianCGrid3DScheme scheme(L.view);
        if (beta != 0.0) scheme.set_coriolis_profile(tmv::CartesianCoriolisProfile{coriolis_f, beta});
        Field3D fdu(nx, ny, nz, 0.0f), fdv(nx, ny, nz, 0.0f), fdw(nx, ny, nz, 0.0f), fdr(nx, ny, nz, 0.0f),
            fdp(nx, ny, nz, 0.0f);
        scheme.compute_slow_tendencies(f.u, f.v, f.w, f.rho, f.p, f.theta, 1.0, fdu, fdv, fdw, fdr, fdp, nullptr);
        if (library && runtime.backend->successful_dispatch_count() == 0)
            return fail("the scheme did not take its device route");
        from_field(du, fdu);
        from_field(dv, fdv);
        from_field(dw, fdw);
        from_field(dp, fdp);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

int ref_slow_tendencies(const float* u, const float* v, const float* w, const float* rho, const float* p,
                        const float* theta, const float* qv, const float* qc, const float* qr, const double* rho0,
                        const double* p0b, const double* qv0, const double* u0, const double* v0,
                        const double* theta0, int nx, int ny, int nz, double dx, double dy, double dz,
                        double coriolis_f, float* du, float* dv, float* dw, float* dp)
{
    return ref_backend_slow_tendencies(nullptr, u, v, w, rho, p, theta, qv, qc, qr, rho0, p0b, qv0, u0, v0, theta0,
                                       nx, ny, nz, dx, dy, dz, coriolis_f, 0.0, du, dv, dw, dp);
}

// The end-of-step sponge on a flat C-grid level: the upper Rayleigh sponge
// (and the w-only lid absorber when w_only_cells > 0), then the lateral
// sponge of lateral_width cells, exactly as dynamics.cpp calls them.  u, v,
// w, theta are relaxed in place; theta0 is the base profile (nz).  The
// reference's own per-level profiles are returned: alpha, upper_w_alpha,
// w_only_alpha, u_ref, v_ref (nz each) and lateral_alpha (lateral_width).
int ref_state_relaxation(float* u, float* v, float* w, float* theta, const double* theta0, int nx, int ny, int nz,
                         double dx, double dy, double dz, double dt, double z_damp, double alpha_max,
                         int w_only_cells, double w_only_alpha_max, int lateral_width, double lateral_alpha_max,
                         int implicit_mode, const double* wind /* u_sfc v_sfc u_1km v_1km u_6km v_6km */,
                         double* alpha, double* upper_w_alpha, double* w_only_alpha, double* u_ref, double* v_ref,
                         double* lateral_alpha)
{
    try
    {
        Level L(nx, ny, nz, dx, dy, dz, dt);
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.theta, theta, nx, ny, nz);
        L.storage.base.theta0.assign(theta0, theta0 + nz);
        auto& c = L.storage.configuration;
        c.damping_enabled = true;
        c.damping_z_d = z_damp;
        c.damping_alpha = alpha_max;
        c.w_only_top_sponge = w_only_cells > 0;
        c.w_only_depth_cells = w_only_cells;
        c.w_only_alpha_max = w_only_alpha_max;
        c.lateral_sponge_enabled = lateral_width > 0;
        c.lateral_sponge_width = lateral_width;
        c.lateral_sponge_alpha = lateral_alpha_max;
        c.damping_mode = implicit_mode ? tmv::init::config::DampingMode::Implicit
                                       : tmv::init::config::DampingMode::Explicit;
        c.wind_profile = WindProfile{wind[0], wind[1], wind[2], wind[3], wind[4], wind[5]};
        RayleighDampingRuntimeState runtime;
        L.view.rayleigh_runtime = &runtime;
        apply_rayleigh_damping(L.view, dt);
        apply_lateral_damping(L.view, dt);
        from_field(u, f.u);
        from_field(v, f.v);
        from_field(w, f.w);
        from_field(theta, f.theta);
        for (int k = 0; k < nz; ++k)
        {
            alpha[k] = runtime.alpha[k];
            upper_w_alpha[k] = runtime.upper_w_alpha[k];
            w_only_alpha[k] = runtime.w_only_alpha[k];
            u_ref[k] = runtime.u_ref[k];
            v_ref[k] = runtime.v_ref[k];
        }
        for (int d = 0; d < lateral_width && d < static_cast<int>(runtime.lateral_alpha.size()); ++d)
            lateral_alpha[d] = runtime.lateral_alpha[d];
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// Cell-centre velocities of face fields u, v, w ([nx][ny][nz] each); a null
// output skips that component; ground_w (nx*ny, may be null) is the terrain
// lower-face w the reference's terrain form takes.
int ref_cell_centre(const float* u, const float* v, const float* w, float* uc, float* vc, float* wc,
                    const double* ground_w, int nx, int ny, int nz)
{
    try
    {
        Field3D face, centre;
        if (uc)
        {
            to_field(face, u, nx, ny, nz);
            interpolate_u_face_to_center(face, centre);
            from_field(uc, centre);
        }
        if (vc)
        {
            to_field(face, v, nx, ny, nz);
            interpolate_v_face_to_center(face, centre);
            from_field(vc, centre);
        }
        if (wc)
        {
            to_field(face, w, nx, ny, nz);
            if (ground_w)
                interpolate_w_face_to_center(
                    face, centre, std::vector<double>(ground_w, ground_w + static_cast<std::size_t>(nx) * ny));
            else
                interpolate_w_face_to_center(face, centre);
            from_field(wc, centre);
        }
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// npy::write_3d of a float32 array; 0 on success.
int ref_npy_write_3d(const float* data, int dim0, int dim1, int dim2, const char* path)
{
    return npy::write_3d(data, dim0, dim1, dim2, std::string(path)) ? 0 : fail("npy::write_3d failed");
}

namespace
{
const char* const kSgsModes[3] = {"3d", "horizontal_only", "vertical_only"};
}

// The Smagorinsky producer on host arrays: mode 0 3d, 1 horizontal_only,
// 2 vertical_only; filter 0 cubic_root, 1 dx; open: W, E, S, N.  qv may be
// null.  Outputs: the coefficients (from the scheme's diagnostics) and the
// five tendencies.
int ref_backend_smagorinsky(const char* library, const float* u, const float* v, const float* w,
                            const float* theta, const float* qv, const float* rho, const double* dz, int nx, int ny,
                            int nz, double dx, double dy, int mode, int filter, int periodic_x, int periodic_y,
                            const int* open, double Cs, double Pr_t, double Sc_t, double nu_max, double K_max,
                            float* nu_t, float* K_theta, float* K_q, float* dudt, float* dvdt, float* dwdt,
                            float* dthdt, float* dqvdt)
{
    try
    {
        // With a library, the scheme sees it as the level's active backend and
        // takes its native path (smagorinsky.cpp:170-176,276-318).
        ComputeBackendRuntimeState runtime;
        if (library)
        {
            runtime.backend = load_backend(library);
            std::string err;
            if (!runtime.backend->initialize(err)) return fail(err.c_str());
            runtime.active_kind = ComputeBackendKind::Vulkan;  // any accelerator kind
            runtime.requested_kind = runtime.active_kind;
        }
        Field3D fu, fv, fw, fth, fqv, frho;
        to_field(fu, u, nx, ny, nz);
        to_field(fv, v, nx, ny, nz);
        to_field(fw, w, nx, ny, nz);
        to_field(fth, theta, nx, ny, nz);
        to_field(frho, rho, nx, ny, nz);
        if (qv) to_field(fqv, qv, nx, ny, nz);
        std::vector<double> rho0(static_cast<std::size_t>(nz), 1.0);
        TurbulenceStateView sv;
        sv.u = &fu;
        sv.v = &fv;
        sv.w = &fw;
        sv.theta = &fth;
        sv.rho = &frho;
        sv.qv = qv ? &fqv : nullptr;
        sv.rho0 = &rho0;
        sv.c_grid = true;
        sv.NR = nx;
        sv.NTH = ny;
        sv.NZ = nz;
        sv.periodic_x = periodic_x != 0;
        sv.periodic_y = periodic_y != 0;
        sv.open_lateral = {open[0] != 0, open[1] != 0, open[2] != 0, open[3] != 0};
        if (library)
        {
            sv.compute_runtime = &runtime;
            sv.require_native_dispatch = true;  // the scheme throws rather than fall back to its CPU path
        }
        GridMetrics g;
        g.dx = dx;
        g.dy = dy;
        g.dz.assign(dz, dz + nz);
        TurbulenceConfig cfg;
        cfg.mode = kSgsModes[mode];
        cfg.filter_width = filter ? "dx" : "cubic_root";
        cfg.Cs = Cs;
        cfg.Pr_t = Pr_t;
        cfg.Sc_t = Sc_t;
        cfg.nu_t_max = nu_max;
        cfg.K_max = K_max;
        SmagorinskyScheme scheme;
        scheme.initialize(cfg);
        TurbulenceTendencies t;
        TurbulenceDiagnostics d;
        scheme.compute(cfg, g, sv, t, &d);
        from_field(nu_t, d.nu_t);
        from_field(K_theta, d.K_theta);
        from_field(K_q, d.K_q);
        from_field(dudt, t.dudt_sgs);
        from_field(dvdt, t.dvdt_sgs);
        from_field(dwdt, t.dwdt_sgs);
        from_field(dthdt, t.dthetadt_sgs);
        if (qv)
            from_field(dqvdt, t.dqvdt_sgs);
        else
            std::memset(dqvdt, 0, sizeof(float) * static_cast<std::size_t>(nx) * ny * nz);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// SmagorinskyScheme::compute on the reference's CPU path.
int ref_smagorinsky(const float* u, const float* v, const float* w, const float* theta, const float* qv,
                    const float* rho, const double* dz, int nx, int ny, int nz, double dx, double dy, int mode,
                    int filter, int periodic_x, int periodic_y, const int* open, double Cs, double Pr_t, double Sc_t,
                    double nu_max, double K_max, float* nu_t, float* K_theta, float* K_q, float* dudt, float* dvdt,
                    float* dwdt, float* dthdt, float* dqvdt)
{
    return ref_backend_smagorinsky(nullptr, u, v, w, theta, qv, rho, dz, nx, ny, nz, dx, dy, mode, filter, periodic_x,
                                   periodic_y, open, Cs, Pr_t, Sc_t, nu_max, K_max, nu_t, K_theta, K_q, dudt, dvdt,
                                   dwdt, dthdt, dqvdt);
}

namespace
{
// A level with the turbulence and compute runtimes the SGS apply and
// stability code expect (CPU kind, no scheme: no work ledger).
struct SgsLevel
{
    Level L;
    ComputeBackendRuntimeState compute;
    tmv::TurbulenceRuntimeState turbulence;
    TurbulenceTendencies tend;
    SgsLevel(int nx, int ny, int nz, double dx, double dy, double dz, double dt) : L(nx, ny, nz, dx, dy, dz, dt)
    {
        L.view.compute_runtime = &compute;
        L.view.turbulence_runtime = &turbulence;
    }
    void load(const float* const rates[6], int nx, int ny, int nz)
    {
        Field3D* out[6] = {&tend.dudt_sgs, &tend.dvdt_sgs, &tend.dwdt_sgs, &tend.dthetadt_sgs, &tend.dqvdt_sgs,
                           &tend.dtkedt_sgs};
        for (int f = 0; f < 6; ++f)
        {
            if (rates[f])
                to_field(*out[f], rates[f], nx, ny, nz);
            else
                out[f]->resize(nx, ny, nz, 0.0f);
        }
    }
};
}  // namespace

// apply_admitted_sgs_substep on host arrays in place (u, v, w, theta, qv; qv
// may be null, which leaves the level without moisture); repairs sets the
// writer repair policy for the call.
int ref_sgs_apply(float* u, float* v, float* w, float* theta, float* qv, const float* dudt, const float* dvdt,
                  const float* dwdt, const float* dthdt, const float* dqvdt, const double* theta0, int nx, int ny,
                  int nz, double dt, int repairs)
{
    const bool saved = primary_state_repairs_enabled;
    try
    {
        SgsLevel S(nx, ny, nz, 1000.0, 1000.0, 500.0, dt);
        auto& f = S.L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.theta, theta, nx, ny, nz);
        if (qv)
            to_field(f.qv, qv, nx, ny, nz);
        else
            f.qv = Field3D();
        f.tke = Field3D();
        if (theta0) S.L.storage.base.theta0.assign(theta0, theta0 + nz);
        const float* rates[6] = {dudt, dvdt, dwdt, dthdt, dqvdt, nullptr};
        S.load(rates, nx, ny, nz);
        set_primary_state_repairs_enabled(repairs != 0);
        apply_admitted_sgs_substep(S.L.view, dt, S.tend);
        set_primary_state_repairs_enabled(saved);
        from_field(u, f.u);
        from_field(v, f.v);
        from_field(w, f.w);
        from_field(theta, f.theta);
        if (qv) from_field(qv, f.qv);
        return 0;
    }
    catch (const std::exception& e)
    {
        set_primary_state_repairs_enabled(saved);
        return fail(e.what());
    }
}

// compute_sgs_explicit_stability with the reference's deterministic
// (thread-count independent) reductions.  bc: W, E, S, N, bottom, top codes.
// out: maximum, momentum-energy, theta-monotonic and qv-monotonic timesteps,
// then the irreversible dissipation power.
int ref_sgs_stability(const float* u, const float* v, const float* w, const float* theta, const float* qv,
                      const float* rho, const float* dudt, const float* dvdt, const float* dwdt, const float* dthdt,
                      const float* dqvdt, int nx, int ny, int nz, double dx, double dy, double dz, const int* bc,
                      int mode, double* out)
{
    const bool saved = tmv::diagnostics::deterministic_reductions_enabled();
    try
    {
        SgsLevel S(nx, ny, nz, dx, dy, dz, 1.0);
        S.L.set_bcs(bc[0], bc[1], bc[2], bc[3], bc[4], bc[5]);
        S.turbulence.config.mode = kSgsModes[mode];
        auto& f = S.L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.theta, theta, nx, ny, nz);
        to_field(f.rho, rho, nx, ny, nz);
        if (qv)
            to_field(f.qv, qv, nx, ny, nz);
        else
            f.qv = Field3D();
        f.tke = Field3D();
        const float* rates[6] = {dudt, dvdt, dwdt, dthdt, dqvdt, nullptr};
        S.load(rates, nx, ny, nz);
        tmv::diagnostics::set_deterministic_reductions(true);
        const SgsExplicitStability r = compute_sgs_explicit_stability(S.L.view, S.tend);
        tmv::diagnostics::set_deterministic_reductions(saved);
        out[0] = r.maximum_timestep_s;
        out[1] = r.momentum_energy_timestep_s;
        out[2] = r.theta_monotonic_timestep_s;
        out[3] = r.qv_monotonic_timestep_s;
        out[4] = r.momentum_irreversible_dissipation_w;
        return 0;
    }
    catch (const std::exception& e)
    {
        tmv::diagnostics::set_deterministic_reductions(saved);
        return fail(e.what());
    }
}

// Conservative transport of n_scalars scalars routed through the reference's
// own bridge dispatch_advect_scalars_conservative_cartesian_cgrid_backend
// (src/compute/dispatch/advection.cpp:95-150) to the backend `library` holds
// (NULL: the reference's CPU backend), with the arguments
// advect_thermodynamics_impl passes (advection_batch.cpp:832-886): inverse
// spacings divided in FP64 and rounded once, the retained context's face
// mass fluxes and beginning density, the host fields, zero kappas, the FP64
// dt and the level's state view.  Returns 1 when the backend declined.
int ref_backend_scalar_transport(const char* library, float** q, const int* positive_definite, int n_scalars,
                                 const float* u, const float* v, const float* w, const float* rho_end,
                                 const float* rho_begin, const float* mfx, const float* mfy, const float* mfz,
                                 int nx, int ny, int nz, double dx, double dy, double dz, double dt, int weno,
                                 int top_open)
{
    try
    {
        if (n_scalars < 0 || n_scalars > 16) return fail("n_scalars out of range");
        ComputeBackendRuntimeState runtime;
        runtime.backend = load_backend(library);
        std::string err;
        if (!runtime.backend->initialize(err)) return fail(err.c_str());
        Level L(nx, ny, nz, dx, dy, dz, dt);
        L.set_bcs(4, 4, 4, 4, 1, top_open ? 2 : 0);
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.rho, rho_end, nx, ny, nz);
        tmv::CartesianCGridTransportContext ctx;
        ctx.begin(L.view, nx, ny, nz, dt);
        Field3D begin_density;
        to_field(begin_density, rho_begin, nx, ny, nz);
        ctx.capture_density_begin(begin_density);
        std::memcpy(ctx.mass_flux_x.data(), mfx, sizeof(float) * f.u.size());
        std::memcpy(ctx.mass_flux_y.data(), mfy, sizeof(float) * f.u.size());
        std::memcpy(ctx.mass_flux_z.data(), mfz, sizeof(float) * f.u.size());
        ctx.record_external_accumulation(dt, 1);
        ctx.complete(L.view);

        std::unique_ptr<Field3D[]> fields(new Field3D[n_scalars > 0 ? n_scalars : 1]);
        Field3D* field_ptrs[16] = {};
        const float* q_in[16] = {};
        float* q_out[16] = {};
        float dt_kappas[16] = {};
        double kappas[16] = {};
        for (int s = 0; s < n_scalars; ++s)
        {
            to_field(fields[s], q[s], nx, ny, nz);
            field_ptrs[s] = &fields[s];
            q_in[s] = fields[s].data();
            q_out[s] = fields[s].data();
        }
        const bool done = dispatch_advect_scalars_conservative_cartesian_cgrid_backend(
            runtime, f.u.data(), f.v.data(), f.w.data(), f.rho.data(), q_in, q_out, dt_kappas, positive_definite,
            n_scalars, nx, ny, nz, static_cast<float>(1.0 / dx), static_cast<float>(1.0 / dy),
            static_cast<float>(1.0 / dz), static_cast<float>(1.0 / (dx * dx)), static_cast<float>(1.0 / (dy * dy)),
            static_cast<float>(1.0 / (dz * dz)), static_cast<float>(dt), density_min_kgm3,
            ctx.density_begin.data(), ctx.mass_flux_x.data(), ctx.mass_flux_y.data(), ctx.mass_flux_z.data(), true,
            field_ptrs, kappas, &ctx, dt, nullptr, nullptr, nullptr, 0.0f, 0.0f, &L.view, nullptr, weno != 0);
        if (!done) return 1;
        for (int s = 0; s < n_scalars; ++s)
            from_field(q[s], fields[s]);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// A completion observer that keeps the committed fields the backend hands it.
struct ObservedCommit
{
    std::vector<float>* out = nullptr;
    std::size_t n = 0;
    int calls = 0;
};

void observe_commit(void* context, const float* a, const float* b, const float* c, const float* d)
{
    auto* o = static_cast<ObservedCommit*>(context);
    const float* committed[4] = {a, b, c, d};
    for (int f = 0; f < 4; ++f) std::copy(committed[f], committed[f] + o->n, o->out[f].begin());
    ++o->calls;
}

// The slow tendencies applied through the reference's bridge
// dispatch_slow_apply_backend (src/compute/dispatch/dynamics.cpp:489-513) to
// the backend `library` holds (NULL: the CPU backend), with the arguments
// dynamics.cpp:2346-2364 passes; observed != 0 adds a completion observer
// whose committed fields are written to out_*.  Returns 1 when declined.
int ref_backend_slow_apply(const char* library, float* u, float* v, float* w, float* p, const float* du,
                           const float* dv, const float* dw, const float* dp, const float* du_pbl,
                           const float* dv_pbl, int nx, int ny, int nz, float dt, int sanitize, int observed,
                           float* out_u, float* out_v, float* out_w, float* out_p, int* observer_calls)
{
    try
    {
        ComputeBackendRuntimeState runtime;
        runtime.backend = load_backend(library);
        std::string err;
        if (!runtime.backend->initialize(err)) return fail(err.c_str());
        const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
        std::vector<float> kept[4];
        for (auto& k : kept) k.assign(n, 0.0f);
        ObservedCommit obs;
        obs.out = kept;
        obs.n = n;
        const bool done = dispatch_slow_apply_backend(runtime, u, v, w, p, du, dv, dw, dp, du_pbl, dv_pbl, nx, ny, nz,
                                                      dt, observed ? &observe_commit : nullptr,
                                                      observed ? &obs : nullptr, sanitize != 0);
        if (!done) return 1;
        float* outs[4] = {out_u, out_v, out_w, out_p};
        for (int f = 0; f < 4; ++f)
            if (outs[f]) std::copy(kept[f].begin(), kept[f].end(), outs[f]);
        *observer_calls = obs.calls;
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// The end-of-step sponge through the reference's bridge
// dispatch_state_relaxation_cartesian_backend (src/compute/dispatch/dynamics.cpp:
// 440-470) with a packed FP32 profile block laid out as dynamics.cpp:538-567
// builds it (rows of nz: upper alpha, w-only alpha, u_ref, v_ref, theta0,
// lateral alpha by distance, upper-w alpha) and a completion observer, as
// try_state_relaxation_gpu calls it.  Returns 1 when declined.
int ref_backend_state_relaxation(const char* library, float* u, float* v, float* w, float* theta,
                                 const float* profiles, int nx, int ny, int nz, int lateral_width, int do_upper,
                                 int do_w_only, int do_lateral, float dt, int* observer_calls)
{
    try
    {
        ComputeBackendRuntimeState runtime;
        runtime.backend = load_backend(library);
        std::string err;
        if (!runtime.backend->initialize(err)) return fail(err.c_str());
        const std::size_t n = static_cast<std::size_t>(nx) * ny * nz;
        std::vector<float> kept[4];
        for (auto& k : kept) k.assign(n, 0.0f);
        ObservedCommit obs;
        obs.out = kept;
        obs.n = n;
        const bool done = dispatch_state_relaxation_cartesian_backend(
            runtime, u, v, w, theta, profiles, 7 * nz, nx, ny, nz, lateral_width, do_upper != 0, do_w_only != 0,
            do_lateral != 0, dt, &observe_commit, &obs);
        if (!done) return 1;
        *observer_calls = obs.calls;
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// SplitExplicitScheme::resolve_substep_count
// (src/numerics/time_stepping/schemes/split_explicit/split_explicit.cpp:67-170)
// with the runtime's sampled sound speed and diagnosed minimum spacing.
int ref_resolve_substep_count(double dt_large, double max_acoustic_speed, double min_spacing, int requested,
                              int* out)
{
    try
    {
        tmv::SplitExplicitScheme scheme;
        TimeSteppingConfig cfg;
        cfg.split_acoustic = true;
        cfg.n_acoustic_substeps = requested;
        cfg.max_acoustic_speed_ms = max_acoustic_speed;
        cfg.min_acoustic_spacing_m = min_spacing;
        *out = scheme.resolve_substep_count(cfg, dt_large);
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

// The acoustic speed and spacing choose_runtime_timestep
// (src/numerics/runtime.cpp:712-880) hands the split-explicit scheme before a
// large step: the Cartesian CFL scan's max sqrt(gamma p / rho) over the state
// (runtime.cpp:346-401), raised to the base columns' (runtime.cpp:854-870),
// and min(dx, dy, dz).
int ref_max_sound_speed(const float* u, const float* v, const float* w, const float* rho, const float* p, int nx,
                        int ny, int nz, double dx, double dy, double dz, double dt, const double* rho0,
                        const double* p0, double* out)
{
    try
    {
        Level L(nx, ny, nz, dx, dy, dz, dt);
        auto& f = L.storage.fields;
        to_field(f.u, u, nx, ny, nz);
        to_field(f.v, v, nx, ny, nz);
        to_field(f.w, w, nx, ny, nz);
        to_field(f.rho, rho, nx, ny, nz);
        to_field(f.p, p, nx, ny, nz);
        L.storage.base.rho0.assign(rho0, rho0 + nz);
        L.storage.base.p0.assign(p0, p0 + nz);
        auto& metrics = tmv::require_level_runtime(L.view.process_grid_metrics, "grid metrics");
        metrics.dx = dx;
        metrics.dy = dy;
        metrics.dz.assign(static_cast<std::size_t>(nz), dz);
        auto& ts = tmv::require_level_runtime(L.view.time_stepping_runtime, "time_stepping_runtime");
        ts.config.split_acoustic = true;
        (void)choose_runtime_timestep(L.view);
        out[0] = ts.config.max_acoustic_speed_ms;
        out[1] = ts.config.min_acoustic_spacing_m;
        return 0;
    }
    catch (const std::exception& e)
    {
        return fail(e.what());
    }
}

} // extern "C"
