// The CUDA backend as a ComputeBackend of the reference solver: the class a
// maintainer registers beside CpuComputeBackend (src/compute/compute_backend.cpp:76-88,
// include/compute/backend_types.hpp:27-32 gain a Cuda kind).  It implements
// the reference's own interfaces (include/compute/backend_interface.hpp,
// include/compute/dispatch/dynamics.hpp, include/compute/dispatch/turbulence.hpp)
// and forwards each dispatch struct to the C-ABI in include/nimbus_cuda.h;
// nothing here computes.  Built against the reference's headers only (every
// virtual it overrides is declared inline there), linked to libnimbus_cuda.so.
//
// Dispatches follow the reference's contract: false leaves host fields
// untouched and the caller decides between its CPU path and an error
// (dynamics.cpp:4453,4604).
//   AcousticSubstepFusedCartesianCgrid  the dispatch carries the CPU solver's
//       FP64 profiles and spacings (rho0_base_host, dx_host, ...): the result
//       is the CPU backend's, bit for bit.
//   AcousticSubstepsBatchedCartesianCgrid  the whole acoustic loop of a large
//       step (split_explicit.cpp's GPU route); this dispatch carries only FP32
//       base profiles, spacings and dt_small, which are widened to FP64, so the
//       result is the C-ABI's on those widened values (and differs from the
//       CPU loop by that FP32 narrowing of its inputs, as the reference's own
//       accelerator backends do).  A dispatch that turns the state repairs
//       off is declined; one that accumulates mass flux without a weight
//       (the runtime's generic route) adds each substep's flux with 1/N, as
//       the reference's device backends do.
//   Smagorinsky (dispatch_smagorinsky_fused)  the bridge passes FP32 copies of
//       dz, dx, dy and the closure constants (src/compute/dispatch/turbulence.cpp:87-146);
//       they are widened to FP64, so the result equals the CPU scheme's
//       exactly when those values are FP32-representable (dz = 250 m, Cs =
//       0.25, ...), and differs by their FP32 rounding otherwise.
//   SgsApply  the same widening of dt_step and the bounds; a dispatch that
//       asks for a completion observer is declined (false).
//   ConservativeCartesianCgridTransport  the coupled WENO5/MC transport of the
//       retained acoustic context (advection_batch.cpp's route): FP64 spacings
//       from the level's state view and dt_step_host, so the result is the CPU
//       backend's bit for bit; see the dispatch for what it declines.
//   CartesianCgridSlowTendencies  the scheme's device route for the slow
//       tendencies (cartesian_cgrid_3d.cpp:835-925), FP32 as the reference's
//       device operator computes it: within the reference's own stencil
//       parity tier of the CPU route.
//   KesslerPointwise / KesslerSedimentation  the two operators of
//       KesslerScheme's device route (kessler.cpp:152-300), FP32 as the
//       reference's device operators compute them; the scheme's result then
//       matches its CPU route within FP32 rounding (the routes book the
//       saturation adjustment in a different order and the CPU one computes
//       in FP64).
#include "compute/backend_interface.hpp"
#include "core/infra/hardware_info.hpp"
#include "compute/dispatch/advection.hpp"
#include "compute/dispatch/dynamics.hpp"
#include "compute/dispatch/microphysics.hpp"
#include "compute/dispatch/turbulence.hpp"
#include "core/runtime/runtime_config.hpp"
#include "core/runtime/simulation_state.hpp"

#include "../../include/nimbus_cuda.h"

#include <algorithm>
#include <cstdint>
#include <string>
#include <vector>

namespace
{

class NimbusCudaComputeBackend final : public ComputeBackend,
                                       public AdvectionComputeKernels,
                                       public DynamicsComputeKernels,
                                       public MicrophysicsComputeKernels,
                                       public TurbulenceComputeKernels
{
public:
    ~NimbusCudaComputeBackend() override { shutdown(); }

    std::string name() const override { return "cuda"; }

    // The configured device (device_index < 0: the first one).
    void configure(const ComputeBackendConfig& config) override { device_ = config.device_index > 0 ? config.device_index : 0; }

    bool initialize(std::string& error) override
    {
        if (ctx_) return true;
        if (nimbus_cuda_create(device_, &ctx_) != NIMBUS_OK)
        {
            ctx_ = nullptr;
            error = "no sm_100 CUDA device (the CUDA backend has no CPU fallback)";
            return false;
        }
        nimbus_cuda_set_precision(ctx_, NIMBUS_PRECISION_REFERENCE);
        return true;
    }

    void shutdown() override
    {
        if (ctx_) nimbus_cuda_destroy(ctx_);
        ctx_ = nullptr;
    }

    std::uint64_t successful_dispatch_count() const override { return dispatches_; }

    void populate_hardware_info(HardwareInfo& info) const override
    {
        nimbus_device_info d{};
        if (!ctx_ || nimbus_cuda_device_info(ctx_, &d) != NIMBUS_OK) return;
        info.gpu_available = true;
        info.gpu_device_name = d.name;
    }

    // Device-separated HBM, its whole size addressable by one buffer; the
    // free bytes are a live estimate.  Dispatches stage through a
    // per-context workspace sized by the largest call.
    ComputeMemoryProperties memory_properties() const override
    {
        ComputeMemoryProperties m{};
        nimbus_device_info d{};
        if (!ctx_ || nimbus_cuda_device_info(ctx_, &d) != NIMBUS_OK) return m;
        m.accelerator = true;
        m.unified_host_device_memory = false;
        m.device_local_heap_bytes = d.total_bytes;
        m.max_storage_buffer_bytes = d.total_bytes;
        m.device_budget_is_live = true;
        m.device_available_budget_bytes = d.free_bytes;
        return m;
    }

    AdvectionComputeKernels* advection_kernels() override { return ctx_ ? this : nullptr; }
    const AdvectionComputeKernels* advection_kernels() const override { return ctx_ ? this : nullptr; }
    DynamicsComputeKernels* dynamics_kernels() override { return ctx_ ? this : nullptr; }
    const DynamicsComputeKernels* dynamics_kernels() const override { return ctx_ ? this : nullptr; }
    MicrophysicsComputeKernels* microphysics_kernels() override { return ctx_ ? this : nullptr; }
    const MicrophysicsComputeKernels* microphysics_kernels() const override { return ctx_ ? this : nullptr; }
    TurbulenceComputeKernels* turbulence_kernels() override { return ctx_ ? this : nullptr; }
    const TurbulenceComputeKernels* turbulence_kernels() const override { return ctx_ ? this : nullptr; }

    bool supports(AdvectionKernelOp op) const override
    {
        return op == AdvectionKernelOp::ConservativeCartesianCgridTransport;
    }

    bool supports_supplied_cartesian_cgrid_mass_flux() const override { return true; }

    // The coupled transport of the retained acoustic context: the face mass
    // fluxes and beginning density the split continuity solve accumulated.
    // The raw ABI carries FP32 inverse spacings and dt; the level's state
    // view (execution_state) and dt_step_host carry the FP64 values the CPU
    // backend uses, and its configuration the open-top flag, so the result is
    // the CPU backend's bit for bit.  Declined (false, nothing written): no
    // state view, the instantaneous-flux mode, a positive-support
    // reconstruction, non-zero kappas, terrain, a collocated grid, or any
    // requested boundary / energy report or interface-flux register (this
    // backend produces none, and a non-null report must be produced or the
    // dispatch refused).
    bool dispatch_advect_scalars_conservative_cartesian_cgrid(
        const ConservativeCartesianCgridTransportDispatch& d) override
    {
        if (!ctx_ || d.n_scalars < 0 || d.n_scalars > 16) return false;
        if (d.n_scalars == 0) return true;
        if (!d.use_supplied_mass_flux || !d.density_begin || !d.mass_flux_x || !d.mass_flux_y || !d.mass_flux_z)
            return false;
        if (!d.q_in || !d.q_out || !d.positive_definite || !d.rho_data || d.preserve_positive_support) return false;
        const SimulationStateView* es = d.execution_state;
        if (!es || !es->configuration || es->configuration->stagger_type != StaggerType::CGrid) return false;
        if (es->process_grid_metrics && es->process_grid_metrics->terrain_metrics_active) return false;
        for (int s = 0; s < d.n_scalars; ++s)
        {
            if (d.dt_kappas && d.dt_kappas[s] != 0.0f) return false;
            if (d.host_kappas && d.host_kappas[s] != 0.0) return false;
            if (d.host_boundary_reports && d.host_boundary_reports[s]) return false;
            if (d.host_energy_reports && d.host_energy_reports[s]) return false;
            if (d.host_energy_kinds && d.host_energy_kinds[s] != tmv::ScalarMoistEnergyKind::None) return false;
            if (d.host_interface_registers && d.host_interface_registers[s]) return false;
        }
        nimbus_scalar_transport_args a{};
        a.q_in = d.q_in;
        a.q_out = d.q_out;
        a.positive_definite = d.positive_definite;
        a.n_scalars = d.n_scalars;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.dx = es->grid.dr;
        a.dy = es->grid.dtheta;
        a.dz = es->grid.dz;
        a.dt = d.dt_step_host > 0.0 ? d.dt_step_host : static_cast<double>(d.dt_step);
        a.rho_end = d.rho_data;
        a.rho_begin = d.density_begin;
        a.mass_flux_x = d.mass_flux_x;
        a.mass_flux_y = d.mass_flux_y;
        a.mass_flux_z = d.mass_flux_z;
        a.weno = d.weno ? 1 : 0;
        a.top_open = es->configuration->top_bc == tmv::init::config::TopBC::Open ? 1 : 0;
        a.rho_floor = d.rho_floor;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_scalar_transport(ctx_, &a));
    }

    bool supports(MicrophysicsKernelOp op) const override
    {
        return op == MicrophysicsKernelOp::KesslerPointwise || op == MicrophysicsKernelOp::KesslerSedimentation;
    }

    bool dispatch_kessler_pointwise(const KesslerPointwiseDispatch& d) override
    {
        if (!ctx_) return false;
        nimbus_kessler_pointwise_args a{};
        a.temperature = d.temperature_data;
        a.p = d.p_data;
        a.qv = d.qv_data;
        a.qc = d.qc_data;
        a.qr = d.qr_data;
        a.rho_d = d.rho_d_data;
        a.dtheta_dt = d.dtheta_dt_data;
        a.dqv_dt = d.dqv_dt_data;
        a.dqc_dt = d.dqc_dt_data;
        a.dqr_dt = d.dqr_dt_data;
        a.dqg_dt = d.dqg_dt_data;
        a.dqh_dt = d.dqh_dt_data;
        a.nx = d.nr;
        a.ny = d.nth;
        a.nz = d.nz;
        a.i_begin = d.i_begin;
        a.i_end = d.i_end;
        a.j_begin = d.j_begin;
        a.j_end = d.j_end;
        a.k_begin = d.k_begin;
        a.k_end = d.k_end;
        a.qc0 = d.qc0;
        a.c_auto = d.c_auto;
        a.c_accr = d.c_accr;
        a.evaporation_efficiency = d.evaporation_efficiency;
        a.lv_cp = d.Lv_cp;
        a.t0 = d.T0;
        a.dt_step = d.dt_step;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_kessler_pointwise(ctx_, &a));
    }

    bool dispatch_kessler_sedimentation(const KesslerSedimentationDispatch& d) override
    {
        if (!ctx_) return false;
        nimbus_kessler_sedimentation_args a{};
        a.qr = d.qr_data;
        a.rho_d = d.rho_d_data;
        a.layer_thickness_m = d.layer_thickness_m;
        a.dqr_dt = d.dqr_dt_data;
        a.nx = d.nr;
        a.ny = d.nth;
        a.nz = d.nz;
        a.i_begin = d.i_begin;
        a.i_end = d.i_end;
        a.j_begin = d.j_begin;
        a.j_end = d.j_end;
        a.k_begin = d.k_begin;
        a.k_end = d.k_end;
        a.dz = d.dz_val;
        a.vt_max_rain = d.Vt_max_rain;
        a.vt_cap = d.vt_cap;
        a.dt_step = d.dt_step;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_kessler_sedimentation(ctx_, &a));
    }

    bool supports(DynamicsKernelOp op) const override
    {
        return op == DynamicsKernelOp::AcousticSubstepFusedCartesianCgrid ||
               op == DynamicsKernelOp::AcousticSubstepsBatchedCartesianCgrid ||
               op == DynamicsKernelOp::SlowApply || op == DynamicsKernelOp::StateRelaxationCartesian ||
               op == DynamicsKernelOp::CartesianCgridSlowTendencies;
    }

    // The scheme's device route for the slow tendencies (FP32 operator; the
    // residency hint is moot: every dispatch uploads what it is given).
    bool dispatch_cartesian_cgrid_slow_tendencies(const CartesianCgridSlowTendenciesDispatch& d) override
    {
        if (!ctx_) return false;
        nimbus_cgrid_slow_tendencies_args a{};
        a.u = d.u_data;
        a.v = d.v_data;
        a.w = d.w_data;
        a.rho = d.rho_data;
        a.p = d.p_data;
        a.rho0_base = d.rho0_base_data;
        a.rho0_base_len = d.rho0_base_len;
        a.qv0_base = d.qv0_base_data;
        a.qv0_base_len = d.qv0_base_len;
        a.u0_base = d.u0_base_data;
        a.v0_base = d.v0_base_data;
        a.wind0_base_len = d.wind0_base_len;
        a.qv = d.qv_data;
        a.loading = d.loading_data;
        a.du_dt = d.du_dt_data;
        a.dv_dt = d.dv_dt_data;
        a.dw_dt = d.dw_dt_data;
        a.drho_dt = d.drho_dt_data;
        a.dp_dt = d.dp_dt_data;
        a.nx = d.nr;
        a.ny = d.nth;
        a.nz = d.nz;
        a.dx = d.dx;
        a.dy = d.dy;
        a.dz = d.dz;
        a.g = d.g;
        a.coriolis_f = d.coriolis_f_val;
        a.has_moisture = d.has_moisture ? 1 : 0;
        a.has_loading = d.has_loading ? 1 : 0;
        a.du_advection_dt = d.du_advection_dt_data;
        a.dv_advection_dt = d.dv_advection_dt_data;
        a.dw_advection_dt = d.dw_advection_dt_data;
        a.frame_velocity_u = d.frame_velocity_u_ms;
        a.frame_velocity_v = d.frame_velocity_v_ms;
        a.coriolis_beta = d.coriolis_beta;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_cgrid_slow_tendencies(ctx_, &a));
    }

    // apply_slow_tendencies_cpu's arithmetic on the dispatched fields (the
    // FP32 dt_large widened to FP64: the CPU's result bit for bit when dt is
    // FP32-representable, as 1.5, 3 or 6 s are).  With a completion
    // observer, the committed fields are handed to it before the host fields
    // change, as the contract asks.
    bool dispatch_slow_apply(const SlowApplyDispatch& d) override
    {
        if (!ctx_ || !d.u || !d.v || !d.w || !d.p_data || !d.du_dt || !d.dv_dt || !d.dw_dt || !d.dp_dt) return false;
        const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
        std::vector<float> fields;
        float* out[4] = {d.u, d.v, d.w, d.p_data};
        if (d.completed_observer)
        {
            fields.resize(4 * n);
            for (int f = 0; f < 4; ++f)
            {
                std::copy(out[f], out[f] + n, fields.begin() + f * n);
                out[f] = fields.data() + f * n;
            }
        }
        nimbus_slow_apply_args a{};
        a.u = out[0];
        a.v = out[1];
        a.w = out[2];
        a.p = out[3];
        a.du_dt = d.du_dt;
        a.dv_dt = d.dv_dt;
        a.dw_dt = d.dw_dt;
        a.dp_dt = d.dp_dt;
        a.du_dt_pbl = d.du_dt_pbl;
        a.dv_dt_pbl = d.dv_dt_pbl;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.dt_large = static_cast<double>(d.dt_large);
        a.sanitize = d.sanitize ? 1 : 0;
        a.memory = NIMBUS_MEMORY_HOST;
        if (!count(nimbus_cuda_slow_apply(ctx_, &a))) return false;
        if (d.completed_observer)
        {
            d.completed_observer(d.completed_observer_context, out[0], out[1], out[2], out[3]);
            std::copy(out[0], out[0] + n, d.u);
            std::copy(out[1], out[1] + n, d.v);
            std::copy(out[2], out[2] + n, d.w);
            std::copy(out[3], out[3] + n, d.p_data);
        }
        return true;
    }

    // The end-of-step sponge from the dispatch's packed FP32 profile block
    // (rows of nz: upper alpha, w-only alpha, u_ref, v_ref, theta0, lateral
    // alpha by distance, stagger-aware upper-w alpha; dynamics.cpp:538-567),
    // widened to FP64, with the exact exponential factor and C-grid
    // staggering the compact device ABI implies (the caller keeps the
    // implicit mode on its CPU writer, dynamics.cpp:478-485).  The result is
    // the C-ABI's on those widened profiles; it differs from the CPU writer by
    // their FP32 rounding, as the reference's accelerator backends do.
    bool dispatch_state_relaxation_cartesian(const StateRelaxationDispatch& d) override
    {
        if (!ctx_ || !d.u || !d.v || !d.w || !d.theta_data || !d.profiles) return false;
        const int nz = d.nz;
        if (d.profiles_len < 7 * nz || d.lateral_width < 0 || d.lateral_width > nz) return false;
        std::vector<double> rows(static_cast<size_t>(7 * nz));
        for (int r = 0; r < 7 * nz; ++r) rows[static_cast<size_t>(r)] = static_cast<double>(d.profiles[r]);
        const size_t n = static_cast<size_t>(d.nx) * d.ny * nz;
        std::vector<float> fields;
        float* out[4] = {d.u, d.v, d.w, d.theta_data};
        if (d.completed_observer)
        {
            fields.resize(4 * n);
            for (int f = 0; f < 4; ++f)
            {
                std::copy(out[f], out[f] + n, fields.begin() + f * n);
                out[f] = fields.data() + f * n;
            }
        }
        nimbus_state_relaxation_args a{};
        a.u = out[0];
        a.v = out[1];
        a.w = out[2];
        a.theta = out[3];
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = nz;
        a.alpha = rows.data();
        a.w_only_alpha = rows.data() + nz;
        a.u_ref = rows.data() + 2 * nz;
        a.v_ref = rows.data() + 3 * nz;
        a.theta_ref = rows.data() + 4 * nz;
        a.lateral_alpha = rows.data() + 5 * nz;
        a.upper_w_alpha = rows.data() + 6 * nz;
        a.lateral_width = d.lateral_width;
        a.do_upper = d.do_upper ? 1 : 0;
        a.do_w_only = d.do_w_only ? 1 : 0;
        a.do_lateral = d.do_lateral ? 1 : 0;
        a.staggered = 1;
        a.implicit_mode = 0;
        a.dt = static_cast<double>(d.dt_step);
        a.memory = NIMBUS_MEMORY_HOST;
        if (!count(nimbus_cuda_state_relaxation(ctx_, &a))) return false;
        if (d.completed_observer)
        {
            d.completed_observer(d.completed_observer_context, out[0], out[1], out[2], out[3]);
            for (int f = 0; f < 4; ++f)
            {
                float* dst = f == 0 ? d.u : f == 1 ? d.v : f == 2 ? d.w : d.theta_data;
                std::copy(out[f], out[f] + n, dst);
            }
        }
        return true;
    }

    // Residency: every dispatch uploads the host fields it is given and
    // writes its results back before returning, and no device copy outlives
    // a dispatch, so there is nothing to keep or invalidate between them.
    void begin_resident_step() override {}
    void select_residency_scope(ComputeResidencyScope) noexcept override {}
    void invalidate_residency_scope(ComputeResidencyScope) noexcept override {}
    void invalidate_resident_field(const char*) noexcept override {}
    void invalidate_all_resident_fields() noexcept override {}

    bool supports_batched_cartesian_cgrid_mass_flux_export() const override { return true; }

    bool supports(TurbulenceKernelOp op) const override
    {
        return op == TurbulenceKernelOp::Smagorinsky || op == TurbulenceKernelOp::SgsApply;
    }

    bool dispatch_acoustic_substep_fused_cartesian_cgrid(const AcousticSubstepFusedCartesianCgridDispatch& d) override
    {
        if (!ctx_ || !d.rho0_base_host || !d.p0_base_host) return false;
        nimbus_acoustic_fused_args a{};
        a.u = d.u;
        a.v = d.v;
        a.w = d.w;
        a.rho = d.rho;
        a.p = d.p;
        a.theta = d.theta_data;
        a.rho0_base = d.rho0_base_host;
        a.p0_base = d.p0_base_host;
        a.base_len = d.base_len;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.dx = d.dx_host;
        a.dy = d.dy_host;
        a.dz = d.dz_host;
        a.dt_small = d.dt_small_host;
        a.gamma = d.gamma_host;
        a.rho_min = d.rho_min;
        a.rho_max = d.rho_max;
        a.p_min = d.p_min;
        a.p_max = d.p_max;
        a.p_ref_fallback = d.p_ref_fallback;
        a.wind_clamp_h = d.wind_clamp_h;
        a.wind_clamp_v = d.wind_clamp_v;
        a.drho_scratch = d.drho_scratch;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_acoustic_fused(ctx_, &a));
    }

    bool dispatch_acoustic_substeps_batched_cartesian_cgrid(const AcousticSubstepsBatchedCartesianCgridDispatch& d) override
    {
        if (!ctx_ || !d.rho0_base_data || !d.p0_base_data || d.nz < 1 || d.base_len < d.nz || !d.repair_primary_state)
            return false;
        // The generic (repaired) route passes no weight: each substep's flux
        // then enters with 1/N, as the reference's device backends take it
        // (the loop's substeps split the large step evenly).
        if (d.accumulate_mass_flux && !(d.mass_flux_weight > 0.0) && d.mass_flux_weight != 0.0) return false;
        if (d.accumulate_mass_flux && d.n_substeps < 1) return false;
        const double flux_weight = d.mass_flux_weight > 0.0 ? d.mass_flux_weight : 1.0 / d.n_substeps;
        std::vector<double> rho0(d.rho0_base_data, d.rho0_base_data + d.nz);
        std::vector<double> p0(d.p0_base_data, d.p0_base_data + d.nz);
        std::vector<float> wave_out;
        float* wave_output = d.wave_history_output;
        if (!wave_output)
        {
            wave_out.assign(2 * (static_cast<size_t>(d.nx) + d.ny) * d.nz, 0.0f);
            wave_output = wave_out.data();
        }
        nimbus_acoustic_batched_args a{};
        a.u = d.u;
        a.v = d.v;
        a.w = d.w;
        a.rho = d.rho;
        a.p = d.p;
        a.theta = d.theta_data;
        a.rho0_base = rho0.data();
        a.p0_base = p0.data();
        a.base_len = d.nz;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.dx = d.dx;
        a.dy = d.dy;
        a.dz = d.dz;
        a.dt_small = d.dt_small;
        a.n_substeps = d.n_substeps;
        a.gamma = d.gamma_val;
        a.rho_min = d.rho_min;
        a.rho_max = d.rho_max;
        a.p_min = d.p_min;
        a.p_max = d.p_max;
        a.p_ref_fallback = d.p_ref_fallback;
        a.wind_clamp_h = d.wind_clamp_h;
        a.wind_clamp_v = d.wind_clamp_v;
        a.bc_west = d.bc_west;
        a.bc_east = d.bc_east;
        a.bc_south = d.bc_south;
        a.bc_north = d.bc_north;
        a.bc_bottom = d.bc_bottom;
        a.bc_top = d.bc_top;
        a.mass_flux_x = d.mass_flux_x;
        a.mass_flux_y = d.mass_flux_y;
        a.mass_flux_z = d.mass_flux_z;
        a.accumulate_mass_flux = d.accumulate_mass_flux;
        a.mass_flux_weight = flux_weight;
        a.frame_velocity_u_ms = d.frame_velocity_u_ms;
        a.frame_velocity_v_ms = d.frame_velocity_v_ms;
        a.wave_history = d.wave_history;
        a.wave_history_output = wave_output;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_acoustic_batched(ctx_, &a));
    }

    bool dispatch_smagorinsky_fused(const SmagorinskyFusedDispatch& d) override
    {
        if (!ctx_ || !d.dz_prof || d.prof_len < d.nz) return false;
        std::vector<double> dz(static_cast<size_t>(d.nz));
        for (int k = 0; k < d.nz; ++k) dz[k] = static_cast<double>(d.dz_prof[k]);
        // The scheme sizes its coefficient fields only when it wants them back.
        std::vector<float> scratch;
        const size_t n = static_cast<size_t>(d.nx) * d.ny * d.nz;
        const bool coefficients = d.download_coefficients && d.nu_t && d.K_theta && d.K_q;
        nimbus_smagorinsky_args a{};
        a.u = d.u_data;
        a.v = d.v_data;
        a.w = d.w_data;
        a.theta = d.theta_data;
        a.qv = d.has_qv ? d.qv_data : nullptr;
        a.rho = d.rho;
        a.dz = dz.data();
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.filter_mode = d.filter_mode;
        a.use_horizontal = d.use_horizontal;
        a.use_vertical = d.use_vertical;
        a.periodic_x = d.periodic_x;
        a.periodic_y = d.periodic_y;
        for (int f = 0; f < 4; ++f) a.open_lateral[f] = d.open_lateral[f];
        a.dx = d.dx_val;
        a.dy = d.dy_val;
        a.Cs = d.Cs;
        a.Pr_t = d.Pr_t;
        a.Sc_t = d.Sc_t;
        a.nu_t_max = d.nu_t_max;
        a.K_max = d.K_max;
        a.nu_t = coefficients ? d.nu_t : nullptr;
        a.K_theta = coefficients ? d.K_theta : nullptr;
        a.K_q = coefficients ? d.K_q : nullptr;
        a.dudt_sgs = d.dudt_sgs;
        a.dvdt_sgs = d.dvdt_sgs;
        a.dwdt_sgs = d.dwdt_sgs;
        a.dthetadt_sgs = d.dthetadt_sgs;
        if (!d.has_qv && d.dqvdt_sgs)
        {
            scratch.assign(n, 0.0f);  // the reference leaves dqvdt untouched without qv
            a.dqvdt_sgs = scratch.data();
        }
        else
        {
            a.dqvdt_sgs = d.dqvdt_sgs;
        }
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_smagorinsky_fused(ctx_, &a));
    }

    bool dispatch_sgs_apply(const SgsApplyDispatch& d) override
    {
        if (!ctx_ || d.completed_observer || d.collocated) return false;
        nimbus_sgs_apply_args a{};
        a.u = d.u;
        a.v = d.v;
        a.w = d.w;
        a.theta = d.theta_data;
        a.qv = d.has_qv ? d.qv_data : nullptr;
        a.tke = d.has_tke ? d.tke_data : nullptr;
        a.dudt = d.dudt;
        a.dvdt = d.dvdt;
        a.dwdt = d.dwdt;
        a.dthetadt = d.dthetadt;
        a.dqvdt = d.dqvdt;
        a.dtkedt = d.dtkedt;
        a.dtkedt_pbl = d.dtkedt_pbl;
        a.nx = d.nx;
        a.ny = d.ny;
        a.nz = d.nz;
        a.dt = d.dt_step;
        a.sanitize = d.sanitize;
        a.theta_reference = d.theta_fallback;
        a.theta_min = d.theta_min;
        a.theta_max = d.theta_max;
        a.qv_max = d.qv_max_val;
        a.wind_h_max = d.wind_h_max;
        a.wind_v_max = d.wind_v_max;
        a.memory = NIMBUS_MEMORY_HOST;
        return count(nimbus_cuda_sgs_apply(ctx_, &a));
    }

private:
    bool count(nimbus_status s)
    {
        if (s != NIMBUS_OK) return false;
        ++dispatches_;
        return true;
    }

    nimbus_cuda_context* ctx_ = nullptr;
    int device_ = 0;
    std::uint64_t dispatches_ = 0;
};

}  // namespace

// Factory hooks: the maintainer's create_compute_backend(ComputeBackendKind::Cuda)
// returns nimbus_cuda_create_compute_backend(); a plugin loader can dlopen
// this library and resolve the same symbol.
extern "C" ComputeBackend* nimbus_cuda_create_compute_backend() { return new NimbusCudaComputeBackend(); }

extern "C" void nimbus_cuda_destroy_compute_backend(ComputeBackend* backend) { delete backend; }
