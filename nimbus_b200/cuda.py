"""ctypes binding of the C-ABI in include/nimbus_cuda.h.

This is the Python stub a maintainer would bind the backend with; the names
and argument blocks mirror the reference's dispatch structs
(include/compute/dispatch/dynamics.hpp, include/compute/dispatch/advection.hpp)
and ``CudaComputeBackend`` mirrors ``ComputeBackend`` /
``DynamicsComputeKernels`` / ``AdvectionComputeKernels``
(include/compute/backend_interface.hpp).  Dispatches return ``bool`` as the
reference's do; ``last_error`` holds the reason for a ``False``.

There is no fallback: if the shared library is missing or no sm_100 device is
present, construction raises.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from pathlib import Path
from typing import Optional, Sequence

import numpy as np

from . import initial

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libnimbus_cuda.so"

NIMBUS_OK = 0
NIMBUS_ERR_INVALID_ARGUMENT = 1
NIMBUS_ERR_OUT_OF_MEMORY = 3
NIMBUS_ERR_NONFINITE = 4
NIMBUS_ERR_IO = 8
STATUS_NAMES = {
    0: "NIMBUS_OK",
    1: "NIMBUS_ERR_INVALID_ARGUMENT",
    2: "NIMBUS_ERR_CUDA",
    3: "NIMBUS_ERR_OUT_OF_MEMORY",
    4: "NIMBUS_ERR_NONFINITE",
    5: "NIMBUS_ERR_UNSUPPORTED",
    6: "NIMBUS_ERR_NO_DEVICE",
    7: "NIMBUS_ERR_TOO_LARGE",
    8: "NIMBUS_ERR_IO",
}
MEMORY_HOST, MEMORY_DEVICE = 0, 1

_fp = ctypes.POINTER(ctypes.c_float)
_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


class AcousticFusedArgs(ctypes.Structure):
    _fields_ = [
        ("u", _fp), ("v", _fp), ("w", _fp), ("rho", _fp), ("p", _fp), ("theta", _fp),
        ("rho0_base", _dp), ("p0_base", _dp), ("base_len", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("dt_small", ctypes.c_double), ("gamma", ctypes.c_double),
        ("rho_min", ctypes.c_float), ("rho_max", ctypes.c_float),
        ("p_min", ctypes.c_float), ("p_max", ctypes.c_float), ("p_ref_fallback", ctypes.c_float),
        ("wind_clamp_h", ctypes.c_float), ("wind_clamp_v", ctypes.c_float),
        ("drho_scratch", _fp), ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class AcousticBatchedArgs(ctypes.Structure):
    _fields_ = [
        ("u", _fp), ("v", _fp), ("w", _fp), ("rho", _fp), ("p", _fp), ("theta", _fp),
        ("rho0_base", _dp), ("p0_base", _dp), ("base_len", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
        ("dt_small", ctypes.c_double), ("n_substeps", ctypes.c_int), ("gamma", ctypes.c_double),
        ("rho_min", ctypes.c_float), ("rho_max", ctypes.c_float),
        ("p_min", ctypes.c_float), ("p_max", ctypes.c_float), ("p_ref_fallback", ctypes.c_float),
        ("wind_clamp_h", ctypes.c_float), ("wind_clamp_v", ctypes.c_float),
        ("bc_west", ctypes.c_int), ("bc_east", ctypes.c_int), ("bc_south", ctypes.c_int),
        ("bc_north", ctypes.c_int), ("bc_bottom", ctypes.c_int), ("bc_top", ctypes.c_int),
        ("mass_flux_x", _fp), ("mass_flux_y", _fp), ("mass_flux_z", _fp),
        ("accumulate_mass_flux", ctypes.c_int), ("mass_flux_weight", ctypes.c_double),
        ("frame_velocity_u_ms", ctypes.c_float), ("frame_velocity_v_ms", ctypes.c_float),
        ("wave_history", _fp), ("wave_history_output", _fp), ("density_begin", _fp),
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class ScalarTransportArgs(ctypes.Structure):
    _fields_ = [
        ("q_in", ctypes.POINTER(_fp)), ("q_out", ctypes.POINTER(_fp)), ("positive_definite", _ip),
        ("n_scalars", ctypes.c_int), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("rho_end", _fp), ("rho_begin", _fp), ("mass_flux_x", _fp), ("mass_flux_y", _fp),
        ("mass_flux_z", _fp), ("weno", ctypes.c_int), ("top_open", ctypes.c_int),
        ("rho_floor", ctypes.c_float), ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class SlowArgs(ctypes.Structure):
    _fields_ = [
        ("u", _fp), ("v", _fp), ("w", _fp), ("p", _fp), ("rho", _fp), ("qv", _fp), ("qc", _fp), ("qr", _fp),
        ("rho0_base", _dp), ("qv0_base", _dp), ("u0_base", _dp), ("v0_base", _dp), ("base_len", ctypes.c_int),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt_large", ctypes.c_double),
        ("gravity", ctypes.c_double), ("coriolis_f", ctypes.c_double),
        ("frame_velocity_u_ms", ctypes.c_float), ("frame_velocity_v_ms", ctypes.c_float),
        ("du_dt", _fp), ("dv_dt", _fp), ("dw_dt", _fp), ("dp_dt", _fp),
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class KesslerArgs(ctypes.Structure):
    _fields_ = [
        ("theta", _fp), ("qv", _fp), ("qc", _fp), ("qr", _fp), ("p", _fp), ("rho", _fp),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dz", ctypes.c_double), ("dt", ctypes.c_double), ("domain", ctypes.c_int * 6),
        ("dtheta_dt", _fp), ("dqv_dt", _fp), ("dqc_dt", _fp), ("dqr_dt", _fp),
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class EosArgs(ctypes.Structure):
    _fields_ = [
        ("p", _fp), ("rho", _fp), ("theta", _fp), ("qv", _fp), ("qc", _fp), ("qr", _fp),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("gamma", ctypes.c_double),
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p), ("p0_base", _dp),
    ]


class StateRelaxationArgs(ctypes.Structure):
    _fields_ = [
        ("u", _fp), ("v", _fp), ("w", _fp), ("theta", _fp),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("alpha", _dp), ("upper_w_alpha", _dp), ("w_only_alpha", _dp), ("u_ref", _dp), ("v_ref", _dp),
        ("theta_ref", _dp), ("lateral_width", ctypes.c_int), ("lateral_alpha", _dp),
        ("do_upper", ctypes.c_int), ("do_w_only", ctypes.c_int), ("do_lateral", ctypes.c_int),
        ("staggered", ctypes.c_int), ("implicit_mode", ctypes.c_int), ("dt", ctypes.c_double),
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class BoundaryArgs(ctypes.Structure):
    _fields_ = [
        ("u", _fp), ("v", _fp), ("w", _fp), ("rho", _fp), ("p", _fp), ("wave_history", _fp),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dt_small", ctypes.c_double),
        ("bc_west", ctypes.c_int), ("bc_east", ctypes.c_int), ("bc_south", ctypes.c_int), ("bc_north", ctypes.c_int),
        ("bc_bottom", ctypes.c_int), ("bc_top", ctypes.c_int),
        ("frame_velocity_u_ms", ctypes.c_float), ("frame_velocity_v_ms", ctypes.c_float),
        ("stream", ctypes.c_void_p),
    ]


class SpongeDesc(ctypes.Structure):
    _fields_ = [
        ("alpha", _dp), ("upper_w_alpha", _dp), ("w_only_alpha", _dp), ("u_ref", _dp), ("v_ref", _dp),
        ("theta_ref", _dp), ("lateral_width", ctypes.c_int), ("lateral_alpha", _dp),
        ("do_upper", ctypes.c_int), ("do_w_only", ctypes.c_int), ("do_lateral", ctypes.c_int),
        ("staggered", ctypes.c_int), ("implicit_mode", ctypes.c_int),
    ]


class MemberDesc(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double), ("dt", ctypes.c_double),
        ("n_substeps", ctypes.c_int), ("bc", ctypes.c_int * 6), ("coriolis_f", ctypes.c_double),
        ("frame_velocity_u_ms", ctypes.c_float), ("frame_velocity_v_ms", ctypes.c_float),
        ("microphysics", ctypes.c_int),
        ("rho0_base", _dp), ("p0_base", _dp), ("qv0_base", _dp), ("u0_base", _dp), ("v0_base", _dp),
        ("sponge", ctypes.POINTER(SpongeDesc)), ("final_closure", ctypes.c_int),
        ("resolve_substeps", ctypes.c_int),
    ]


class SlowApplyArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("u", "v", "w", "p", "du_dt", "dv_dt", "dw_dt", "dp_dt", "du_dt_pbl", "dv_dt_pbl")],
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("dt_large", ctypes.c_double),
        ("sanitize", ctypes.c_int), ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class KesslerPointwiseArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("temperature", "p", "qv", "qc", "qr", "rho_d", "dtheta_dt", "dqv_dt", "dqc_dt", "dqr_dt",
                             "dqg_dt", "dqh_dt")],
        *[(k, ctypes.c_int) for k in ("nx", "ny", "nz", "i_begin", "i_end", "j_begin", "j_end", "k_begin", "k_end")],
        *[(k, ctypes.c_float) for k in ("qc0", "c_auto", "c_accr", "evaporation_efficiency", "lv_cp", "t0",
                                        "dt_step")],
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class KesslerSedimentationArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("qr", "rho_d", "layer_thickness_m", "dqr_dt")],
        *[(k, ctypes.c_int) for k in ("nx", "ny", "nz", "i_begin", "i_end", "j_begin", "j_end", "k_begin", "k_end")],
        *[(k, ctypes.c_float) for k in ("dz", "vt_max_rain", "vt_cap", "dt_step")],
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class CgridSlowTendenciesArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("u", "v", "w", "rho", "p", "rho0_base")], ("rho0_base_len", ctypes.c_int),
        ("qv0_base", _fp), ("qv0_base_len", ctypes.c_int), ("u0_base", _fp), ("v0_base", _fp),
        ("wind0_base_len", ctypes.c_int),
        *[(k, _fp) for k in ("qv", "loading", "du_dt", "dv_dt", "dw_dt", "drho_dt", "dp_dt")],
        *[(k, ctypes.c_int) for k in ("nx", "ny", "nz")],
        *[(k, ctypes.c_float) for k in ("dx", "dy", "dz", "g", "coriolis_f")],
        ("has_moisture", ctypes.c_int), ("has_loading", ctypes.c_int),
        *[(k, _fp) for k in ("du_advection_dt", "dv_advection_dt", "dw_advection_dt")],
        *[(k, ctypes.c_float) for k in ("frame_velocity_u", "frame_velocity_v", "coriolis_beta")],
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class DeviceInfo(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 256), ("sm_count", ctypes.c_int), ("cc_major", ctypes.c_int),
                ("cc_minor", ctypes.c_int), ("total_bytes", ctypes.c_ulonglong), ("free_bytes", ctypes.c_ulonglong)]


TUNING_CANDIDATES = 48


class EngineTuning(ctypes.Structure):
    _fields_ = [
        ("lanes", ctypes.c_int), ("acoustic_form", ctypes.c_int), ("march", ctypes.c_int),
        ("momentum_form", ctypes.c_int), ("ms_per_step", ctypes.c_double), ("candidates", ctypes.c_int),
        ("candidate_lanes", ctypes.c_int * TUNING_CANDIDATES), ("candidate_form", ctypes.c_int * TUNING_CANDIDATES),
        ("candidate_momentum_form", ctypes.c_int * TUNING_CANDIDATES),
        ("candidate_march", ctypes.c_int * TUNING_CANDIDATES),
        ("candidate_ms", ctypes.c_double * TUNING_CANDIDATES),
    ]


class SoundSpeedArgs(ctypes.Structure):
    _fields_ = [
        ("p", _fp), ("rho", _fp), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("p0_base", _dp), ("rho0_base", _dp), ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
        ("max_sound_speed", ctypes.c_double),
    ]


class SmagorinskyArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("u", "v", "w", "theta", "qv", "rho")], ("dz", _dp),
        ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int), ("filter_mode", ctypes.c_int),
        ("use_horizontal", ctypes.c_int), ("use_vertical", ctypes.c_int), ("periodic_x", ctypes.c_int),
        ("periodic_y", ctypes.c_int), ("open_lateral", ctypes.c_int * 4), ("open_top", ctypes.c_int),
        *[(k, ctypes.c_double) for k in ("dx", "dy", "Cs", "Pr_t", "Sc_t", "nu_t_max", "K_max")],
        *[(k, _fp) for k in ("nu_t", "K_theta", "K_q", "dudt_sgs", "dvdt_sgs", "dwdt_sgs", "dthetadt_sgs",
                             "dqvdt_sgs")],
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class SgsApplyArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("u", "v", "w", "theta", "qv", "tke", "dudt", "dvdt", "dwdt", "dthetadt", "dqvdt",
                             "dtkedt", "dtkedt_pbl")],
        ("theta0_base", _dp), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("dt", ctypes.c_double), ("sanitize", ctypes.c_int), ("theta_reference", ctypes.c_double),
        *[(k, ctypes.c_float) for k in ("theta_min", "theta_max", "qv_max", "wind_h_max", "wind_v_max")],
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class SgsStability(ctypes.Structure):
    _fields_ = [(k, ctypes.c_double) for k in ("maximum_timestep_s", "momentum_energy_timestep_s",
                                               "theta_monotonic_timestep_s", "qv_monotonic_timestep_s",
                                               "momentum_irreversible_dissipation_w")]


class SgsStepArgs(ctypes.Structure):
    _fields_ = [("closure", SmagorinskyArgs), ("theta0_base", _dp), ("dt", ctypes.c_double),
                ("dt_sgs", ctypes.c_double), ("time_s", ctypes.c_double), ("sanitize", ctypes.c_int)]


class CellCentreArgs(ctypes.Structure):
    _fields_ = [
        ("u", _fp), ("v", _fp), ("w", _fp), ("u_centre", _fp), ("v_centre", _fp), ("w_centre", _fp),
        ("ground_w", _dp), ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
        ("memory", ctypes.c_int), ("stream", ctypes.c_void_p),
    ]


class HistoryArgs(ctypes.Structure):
    _fields_ = [
        *[(k, _fp) for k in ("u", "v", "w", "rho", "p", "theta", "qv", "qc", "qr")],
        ("fields", ctypes.c_uint), ("ground_w", _dp), ("nx", ctypes.c_int), ("ny", ctypes.c_int),
        ("nz", ctypes.c_int), ("host_image", _fp), ("stream", ctypes.c_void_p),
    ]


class MemberState(ctypes.Structure):
    _fields_ = [(k, _fp) for k in ("u", "v", "w", "rho", "p", "theta", "qv", "qc", "qr")]


EXPORTED_SYMBOLS = (
    "nimbus_cuda_abi_version", "nimbus_cuda_create", "nimbus_cuda_destroy", "nimbus_cuda_last_error",
    "nimbus_cuda_kernel_launches", "nimbus_cuda_stream", "nimbus_cuda_synchronize",
    "nimbus_cuda_acoustic_fused", "nimbus_cuda_acoustic_batched", "nimbus_cuda_scalar_transport",
    "nimbus_cuda_set_kernel_timing", "nimbus_cuda_kernel_timing",
    "nimbus_cuda_acoustic_fused_static_scratch", "nimbus_cuda_set_precision",
    "nimbus_cuda_set_substep_form", "nimbus_cuda_autotune_substep",
    "nimbus_cuda_slow_tendencies", "nimbus_cuda_slow_step",
    "nimbus_cuda_kessler_tendencies", "nimbus_cuda_kessler_step", "nimbus_cuda_eos_projection",
    "nimbus_cuda_acoustic_boundaries", "nimbus_cuda_state_relaxation",
    "nimbus_cuda_smagorinsky_fused", "nimbus_cuda_sgs_apply", "nimbus_cuda_sgs_stability", "nimbus_cuda_sgs_step",
    "nimbus_cuda_cell_centre_velocity", "nimbus_cuda_history_snapshot", "nimbus_npy_write_3d",
    "nimbus_history_write", "nimbus_cuda_engine_history_async",
    "nimbus_cuda_engine_create", "nimbus_cuda_engine_destroy", "nimbus_cuda_engine_member_bytes",
    "nimbus_cuda_engine_admit", "nimbus_cuda_engine_retire", "nimbus_cuda_engine_read", "nimbus_cuda_engine_write", "nimbus_cuda_engine_step",
    "nimbus_cuda_engine_read_async", "nimbus_cuda_engine_write_async", "nimbus_cuda_engine_stream",
    "nimbus_cuda_engine_image_bytes", "nimbus_cuda_engine_image_offset",
    "nimbus_cuda_engine_upload_image_async", "nimbus_cuda_engine_download_image_async",
    "nimbus_cuda_engine_set_lanes", "nimbus_cuda_engine_lanes",
    "nimbus_cuda_engine_synchronize", "nimbus_cuda_engine_member_status", "nimbus_cuda_engine_set_graph",
    "nimbus_cuda_engine_members", "nimbus_cuda_engine_launches_per_step", "nimbus_cuda_engine_member_substeps",
    "nimbus_cuda_max_sound_speed", "nimbus_cuda_resolve_substep_count",
    "nimbus_cuda_engine_set_march", "nimbus_cuda_engine_march", "nimbus_cuda_engine_set_acoustic_form",
    "nimbus_cuda_engine_acoustic_form", "nimbus_cuda_engine_member_status_async", "nimbus_cuda_engine_graph_builds",
    "nimbus_cuda_engine_set_pass_forms", "nimbus_cuda_engine_pass_forms",
    "nimbus_cuda_engine_autotune", "nimbus_cuda_slow_apply", "nimbus_cuda_kessler_pointwise",
    "nimbus_cuda_kessler_sedimentation", "nimbus_cuda_cgrid_slow_tendencies", "nimbus_cuda_device_info",
)
ACOUSTIC_FORM_NAMES = {0: "member-table", 1: "constant-bank", 2: "marching", 3: "constant-bank, two cells per thread",
                       4: "bulk-staged tiles", 5: "constant-bank marching"}
ACOUSTIC_TABLE, ACOUSTIC_CONST, ACOUSTIC_MARCH, ACOUSTIC_PAIR, ACOUSTIC_BULK, ACOUSTIC_CMARCH = 0, 1, 2, 3, 4, 5
SUBSTEP_AUTO, SUBSTEP_FUSED, SUBSTEP_SPLIT = 0, 1, 2
PRECISION_REFERENCE, PRECISION_FP32 = 0, 1
STATIC_SCRATCH_CELLS = 4194304  # NIMBUS_STATIC_SCRATCH_CELLS
KERNEL_FAMILIES = ("acoustic_substep", "acoustic_momentum", "acoustic_boundary", "transport_faces",
                   "transport_limiter", "transport_update", "slow", "microphysics", "output", "sgs")
# History fields (NIMBUS_HISTORY_* bit order): the reference's core volume
# bindings, headless_runtime.cpp:588-600.
HISTORY_FIELDS = ("u", "v", "w", "rho", "p", "theta", "qv", "qc", "qr")
HISTORY_CORE = (1 << len(HISTORY_FIELDS)) - 1


def history_mask(names) -> int:
    """NIMBUS_HISTORY_* bits of field names (any order)."""
    mask = 0
    for name in names:
        mask |= 1 << HISTORY_FIELDS.index(name)
    return mask


def history_names(mask: int) -> tuple:
    """Field names of a NIMBUS_HISTORY_* mask, in image order."""
    return tuple(k for i, k in enumerate(HISTORY_FIELDS) if mask >> i & 1)


def load_library(path: Path = LIB_PATH) -> ctypes.CDLL:
    """Load the backend library; raise if it is missing (no fallback path)."""
    if not path.exists():
        raise RuntimeError(f"CUDA backend library {path} is missing; run __graft_entry__.build()")
    lib = ctypes.CDLL(str(path))
    lib.nimbus_cuda_create.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_void_p)]
    lib.nimbus_cuda_destroy.argtypes = [ctypes.c_void_p]
    lib.nimbus_cuda_last_error.argtypes = [ctypes.c_void_p]
    lib.nimbus_cuda_last_error.restype = ctypes.c_char_p
    lib.nimbus_cuda_kernel_launches.argtypes = [ctypes.c_void_p]
    lib.nimbus_cuda_kernel_launches.restype = ctypes.c_uint64
    lib.nimbus_cuda_stream.argtypes = [ctypes.c_void_p]
    lib.nimbus_cuda_stream.restype = ctypes.c_void_p
    lib.nimbus_cuda_synchronize.argtypes = [ctypes.c_void_p]
    lib.nimbus_cuda_acoustic_fused.argtypes = [ctypes.c_void_p, ctypes.POINTER(AcousticFusedArgs)]
    lib.nimbus_cuda_acoustic_batched.argtypes = [ctypes.c_void_p, ctypes.POINTER(AcousticBatchedArgs)]
    lib.nimbus_cuda_scalar_transport.argtypes = [ctypes.c_void_p, ctypes.POINTER(ScalarTransportArgs)]
    lib.nimbus_cuda_set_precision.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.nimbus_cuda_set_substep_form.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.nimbus_cuda_autotune_substep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                                 ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_double)]
    lib.nimbus_cuda_acoustic_fused_static_scratch.argtypes = [ctypes.POINTER(AcousticFusedArgs)]
    lib.nimbus_cuda_slow_tendencies.argtypes = [ctypes.c_void_p, ctypes.POINTER(SlowArgs)]
    lib.nimbus_cuda_slow_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(SlowArgs)]
    lib.nimbus_cuda_kessler_tendencies.argtypes = [ctypes.c_void_p, ctypes.POINTER(KesslerArgs)]
    lib.nimbus_cuda_kessler_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(KesslerArgs)]
    lib.nimbus_cuda_eos_projection.argtypes = [ctypes.c_void_p, ctypes.POINTER(EosArgs)]
    lib.nimbus_cuda_acoustic_boundaries.argtypes = [ctypes.c_void_p, ctypes.POINTER(BoundaryArgs)]
    lib.nimbus_cuda_state_relaxation.argtypes = [ctypes.c_void_p, ctypes.POINTER(StateRelaxationArgs)]
    lib.nimbus_cuda_smagorinsky_fused.argtypes = [ctypes.c_void_p, ctypes.POINTER(SmagorinskyArgs)]
    lib.nimbus_cuda_sgs_apply.argtypes = [ctypes.c_void_p, ctypes.POINTER(SgsApplyArgs)]
    lib.nimbus_cuda_sgs_stability.argtypes = [ctypes.c_void_p, ctypes.POINTER(SmagorinskyArgs),
                                              ctypes.POINTER(SgsStability)]
    lib.nimbus_cuda_sgs_step.argtypes = [ctypes.c_void_p, ctypes.POINTER(SgsStepArgs), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_double)]
    lib.nimbus_cuda_cell_centre_velocity.argtypes = [ctypes.c_void_p, ctypes.POINTER(CellCentreArgs)]
    lib.nimbus_cuda_history_snapshot.argtypes = [ctypes.c_void_p, ctypes.POINTER(HistoryArgs)]
    lib.nimbus_npy_write_3d.argtypes = [_fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p]
    lib.nimbus_history_write.argtypes = [_fp, ctypes.c_uint, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                         ctypes.c_char_p]
    vp = ctypes.c_void_p
    lib.nimbus_cuda_engine_history_async.argtypes = [vp, ctypes.c_int, ctypes.c_uint, vp]
    lib.nimbus_cuda_engine_create.argtypes = [vp, ctypes.POINTER(vp)]
    lib.nimbus_cuda_engine_destroy.argtypes = [vp]
    lib.nimbus_cuda_engine_destroy.restype = None
    lib.nimbus_cuda_engine_member_bytes.argtypes = [ctypes.POINTER(MemberDesc)]
    lib.nimbus_cuda_engine_member_bytes.restype = ctypes.c_size_t
    lib.nimbus_cuda_engine_admit.argtypes = [vp, ctypes.POINTER(MemberDesc), ctypes.POINTER(MemberState),
                                             ctypes.c_size_t, ctypes.POINTER(ctypes.c_int)]
    lib.nimbus_cuda_engine_retire.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_read.argtypes = [vp, ctypes.c_int, ctypes.POINTER(MemberState)]
    lib.nimbus_cuda_engine_write.argtypes = [vp, ctypes.c_int, ctypes.POINTER(MemberState)]
    lib.nimbus_cuda_engine_write_async.argtypes = [vp, ctypes.c_int, ctypes.POINTER(MemberState)]
    lib.nimbus_cuda_engine_read_async.argtypes = [vp, ctypes.c_int, ctypes.POINTER(MemberState)]
    lib.nimbus_cuda_engine_stream.argtypes = [vp]
    lib.nimbus_cuda_engine_stream.restype = vp
    lib.nimbus_cuda_engine_image_bytes.argtypes = [vp]
    lib.nimbus_cuda_engine_image_bytes.restype = ctypes.c_size_t
    lib.nimbus_cuda_engine_image_offset.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_image_offset.restype = ctypes.c_size_t
    lib.nimbus_cuda_engine_upload_image_async.argtypes = [vp, vp]
    lib.nimbus_cuda_engine_download_image_async.argtypes = [vp, vp]
    lib.nimbus_cuda_engine_set_lanes.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_lanes.argtypes = [vp]
    lib.nimbus_cuda_engine_step.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_synchronize.argtypes = [vp]
    lib.nimbus_cuda_engine_member_status.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_uint)]
    lib.nimbus_cuda_engine_set_graph.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_members.argtypes = [vp]
    lib.nimbus_cuda_engine_launches_per_step.argtypes = [vp]
    lib.nimbus_cuda_engine_member_substeps.argtypes = [vp, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
    lib.nimbus_cuda_engine_set_march.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_march.argtypes = [vp]
    lib.nimbus_cuda_engine_set_acoustic_form.argtypes = [vp, ctypes.c_int]
    lib.nimbus_cuda_engine_member_status_async.argtypes = [vp, ctypes.c_int, ctypes.c_void_p]
    lib.nimbus_cuda_engine_autotune.argtypes = [vp, ctypes.c_int, ctypes.POINTER(EngineTuning)]
    lib.nimbus_cuda_slow_apply.argtypes = [vp, ctypes.POINTER(SlowApplyArgs)]
    lib.nimbus_cuda_kessler_pointwise.argtypes = [vp, ctypes.POINTER(KesslerPointwiseArgs)]
    lib.nimbus_cuda_kessler_sedimentation.argtypes = [vp, ctypes.POINTER(KesslerSedimentationArgs)]
    lib.nimbus_cuda_cgrid_slow_tendencies.argtypes = [vp, ctypes.POINTER(CgridSlowTendenciesArgs)]
    lib.nimbus_cuda_device_info.argtypes = [vp, ctypes.POINTER(DeviceInfo)]
    lib.nimbus_cuda_engine_graph_builds.argtypes = [vp, ctypes.POINTER(ctypes.c_uint64),
                                                    ctypes.POINTER(ctypes.c_uint64)]
    lib.nimbus_cuda_engine_acoustic_form.argtypes = [vp]
    lib.nimbus_cuda_engine_set_pass_forms.argtypes = [vp, ctypes.c_int, ctypes.c_int]
    lib.nimbus_cuda_engine_pass_forms.argtypes = [vp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
    lib.nimbus_cuda_max_sound_speed.argtypes = [vp, ctypes.POINTER(SoundSpeedArgs)]
    lib.nimbus_cuda_resolve_substep_count.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                                      ctypes.c_int]
    lib.nimbus_cuda_set_kernel_timing.argtypes = [ctypes.c_void_p, ctypes.c_int]
    lib.nimbus_cuda_kernel_timing.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_uint64),
                                              ctypes.POINTER(ctypes.c_double)]
    return lib


def _f(a) -> "ctypes._Pointer":
    """float* of a host float32 array, or of a device tensor (int address)."""
    if a is None:
        return None
    if isinstance(a, int):
        return ctypes.cast(ctypes.c_void_p(a), _fp)
    if hasattr(a, "data_ptr"):
        assert a.dtype.__str__() == "torch.float32" and a.is_contiguous()
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _fp)
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"], (a.dtype, a.flags)
    return a.ctypes.data_as(_fp)


def _d(a):
    if a is None:
        return None
    if hasattr(a, "data_ptr"):
        assert a.dtype.__str__() == "torch.float64" and a.is_contiguous()
        return ctypes.cast(ctypes.c_void_p(a.data_ptr()), _dp)
    assert a.dtype == np.float64 and a.flags["C_CONTIGUOUS"], "base profiles must be contiguous float64"
    return a.ctypes.data_as(_dp)


class NimbusCudaError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Context:
    """Owns one nimbus_cuda_context (device, stream, staging workspace)."""

    def __init__(self, device: int = 0, lib: Optional[ctypes.CDLL] = None):
        self.lib = lib or load_library()
        handle = ctypes.c_void_p()
        rc = self.lib.nimbus_cuda_create(int(device), ctypes.byref(handle))
        if rc != NIMBUS_OK:
            raise NimbusCudaError(rc, "could not create a CUDA context on an sm_100 device")
        self.handle = handle
        self.device = device

    def close(self):
        if getattr(self, "handle", None):
            self.lib.nimbus_cuda_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def last_error(self) -> str:
        return self.lib.nimbus_cuda_last_error(self.handle).decode()

    @property
    def kernel_launches(self) -> int:
        return int(self.lib.nimbus_cuda_kernel_launches(self.handle))

    @property
    def stream(self) -> int:
        return int(self.lib.nimbus_cuda_stream(self.handle) or 0)

    def check(self, rc: int):
        if rc != NIMBUS_OK:
            raise NimbusCudaError(rc, self.last_error)

    def synchronize(self):
        self.check(self.lib.nimbus_cuda_synchronize(self.handle))

    def set_precision(self, precision: int):
        self.check(self.lib.nimbus_cuda_set_precision(self.handle, int(precision)))

    def set_substep_form(self, form: int):
        self.check(self.lib.nimbus_cuda_set_substep_form(self.handle, int(form)))

    def autotune_substep(self, nx: int, ny: int, nz: int):
        """(chosen form, ms per substep) for this shape in the current precision."""
        form = ctypes.c_int()
        ms = ctypes.c_double()
        self.check(self.lib.nimbus_cuda_autotune_substep(self.handle, nx, ny, nz, ctypes.byref(form), ctypes.byref(ms)))
        return int(form.value), float(ms.value)

    def set_kernel_timing(self, enable: bool):
        self.check(self.lib.nimbus_cuda_set_kernel_timing(self.handle, int(enable)))

    def kernel_timing(self) -> dict:
        """{family: (launches, total_ms)} since timing was enabled."""
        out = {}
        for f, name in enumerate(KERNEL_FAMILIES):
            n = ctypes.c_uint64()
            ms = ctypes.c_double()
            self.check(self.lib.nimbus_cuda_kernel_timing(self.handle, f, ctypes.byref(n), ctypes.byref(ms)))
            out[name] = (int(n.value), float(ms.value))
        return out

    # -- raw entry points -------------------------------------------------
    def acoustic_fused(self, args: AcousticFusedArgs) -> int:
        return self.lib.nimbus_cuda_acoustic_fused(self.handle, ctypes.byref(args))

    def acoustic_batched(self, args: AcousticBatchedArgs) -> int:
        return self.lib.nimbus_cuda_acoustic_batched(self.handle, ctypes.byref(args))

    def scalar_transport(self, args: ScalarTransportArgs) -> int:
        return self.lib.nimbus_cuda_scalar_transport(self.handle, ctypes.byref(args))

    def slow_tendencies(self, args: SlowArgs) -> int:
        return self.lib.nimbus_cuda_slow_tendencies(self.handle, ctypes.byref(args))

    def slow_step(self, args: SlowArgs) -> int:
        return self.lib.nimbus_cuda_slow_step(self.handle, ctypes.byref(args))

    def kessler_tendencies(self, args: KesslerArgs) -> int:
        return self.lib.nimbus_cuda_kessler_tendencies(self.handle, ctypes.byref(args))

    def kessler_step(self, args: KesslerArgs) -> int:
        return self.lib.nimbus_cuda_kessler_step(self.handle, ctypes.byref(args))

    def eos_projection(self, args: EosArgs) -> int:
        return self.lib.nimbus_cuda_eos_projection(self.handle, ctypes.byref(args))

    def max_sound_speed(self, p, rho, shape, base=None, stream=None) -> float:
        """Largest sqrt(gamma p / rho) over the fields (host float32 arrays or
        device tensors) and, with `base`, its p0/rho0 columns; waits for it."""
        a = SoundSpeedArgs()
        a.p, a.rho = _f(p), _f(rho)
        a.nx, a.ny, a.nz = (int(x) for x in shape)
        keep = None
        if base is not None:
            keep = (np.ascontiguousarray(base["p0"], np.float64), np.ascontiguousarray(base["rho0"], np.float64))
            a.p0_base, a.rho0_base = _d(keep[0]), _d(keep[1])
        a.memory = MEMORY_DEVICE if hasattr(p, "data_ptr") else MEMORY_HOST
        a.stream = stream
        self.check(self.lib.nimbus_cuda_max_sound_speed(self.handle, ctypes.byref(a)))
        return a.max_sound_speed

    def slow_apply(self, u, v, w, p, du, dv, dw, dp, dt, du_pbl=None, dv_pbl=None, sanitize=True) -> None:
        """apply_slow_tendencies_cpu on host float32 arrays (in place) or device tensors."""
        a = SlowApplyArgs()
        a._keep = (u, v, w, p, du, dv, dw, dp, du_pbl, dv_pbl)
        for name, x in zip(("u", "v", "w", "p", "du_dt", "dv_dt", "dw_dt", "dp_dt", "du_dt_pbl", "dv_dt_pbl"),
                           a._keep):
            setattr(a, name, _f(x))
        a.nx, a.ny, a.nz = (int(x) for x in u.shape)
        a.dt_large = float(dt)
        a.sanitize = int(bool(sanitize))
        a.memory = MEMORY_DEVICE if hasattr(u, "data_ptr") else MEMORY_HOST
        self.check(self.lib.nimbus_cuda_slow_apply(self.handle, ctypes.byref(a)))

    def kessler_pointwise(self, T, p, qv, qc, qr, rho_d, outs, domain, qc0=1.0e-3, c_auto=1.0e-3, c_accr=2.2,
                          evaporation_efficiency=1.0, lv_cp=2.5e6 / 1004.0, t0=273.15, dt=3.0) -> None:
        """The device route's Kessler pointwise operator: outs = (dtheta, dqv,
        dqc, dqr[, dqg, dqh]) written over the whole grid (host float32 arrays
        or device tensors)."""
        a = KesslerPointwiseArgs()
        outs = list(outs) + [None] * (6 - len(outs))
        a._keep = (T, p, qv, qc, qr, rho_d, outs)
        for name, x in zip(("temperature", "p", "qv", "qc", "qr", "rho_d"), (T, p, qv, qc, qr, rho_d)):
            setattr(a, name, _f(x))
        for name, x in zip(("dtheta_dt", "dqv_dt", "dqc_dt", "dqr_dt", "dqg_dt", "dqh_dt"), outs):
            setattr(a, name, _f(x) if x is not None else None)
        a.nx, a.ny, a.nz = (int(x) for x in T.shape)
        a.i_begin, a.i_end, a.j_begin, a.j_end, a.k_begin, a.k_end = (int(x) for x in domain)
        a.qc0, a.c_auto, a.c_accr = qc0, c_auto, c_accr
        a.evaporation_efficiency, a.lv_cp, a.t0, a.dt_step = evaporation_efficiency, lv_cp, t0, dt
        a.memory = MEMORY_DEVICE if hasattr(T, "data_ptr") else MEMORY_HOST
        self.check(self.lib.nimbus_cuda_kessler_pointwise(self.handle, ctypes.byref(a)))

    def kessler_sedimentation(self, qr, dqr, domain, dz, vt_max=20.0, vt_cap=3.4028234663852886e38, rho_d=None,
                              layers=None, dt=3.0) -> None:
        """The device route's Kessler sedimentation operator: the rain fallout
        added to dqr in place."""
        a = KesslerSedimentationArgs()
        a._keep = (qr, dqr, rho_d, layers)
        a.qr, a.dqr_dt = _f(qr), _f(dqr)
        a.rho_d = _f(rho_d) if rho_d is not None else None
        a.layer_thickness_m = _f(layers) if layers is not None else None
        a.nx, a.ny, a.nz = (int(x) for x in qr.shape)
        a.i_begin, a.i_end, a.j_begin, a.j_end, a.k_begin, a.k_end = (int(x) for x in domain)
        a.dz, a.vt_max_rain, a.vt_cap, a.dt_step = dz, vt_max, vt_cap, dt
        a.memory = MEMORY_DEVICE if hasattr(qr, "data_ptr") else MEMORY_HOST
        self.check(self.lib.nimbus_cuda_kessler_sedimentation(self.handle, ctypes.byref(a)))

    def cgrid_slow_tendencies(self, st, profiles, outs, grid, g=9.81, coriolis_f=0.0, beta=0.0, loading=None,
                              advection=None, frame=(0.0, 0.0)) -> None:
        """The device route's slow-tendency operator.  st: u, v, w, rho, p
        (and qv for moisture); profiles: FP32 rho0 (and qv0, u0, v0); outs:
        du, dv, dw, drho (or None), dp; advection: three outputs or None.
        Host float32 arrays or device tensors."""
        a = CgridSlowTendenciesArgs()
        a._keep = (dict(st), dict(profiles), list(outs), loading, advection)
        for k in ("u", "v", "w", "rho", "p"):
            setattr(a, k, _f(st[k]))
        nz = int(st["u"].shape[2])
        a.rho0_base, a.rho0_base_len = _f(profiles["rho0"]), int(profiles["rho0"].shape[0])
        moist = st.get("qv") is not None and profiles.get("qv0") is not None
        if moist:
            a.qv, a.qv0_base, a.qv0_base_len = _f(st["qv"]), _f(profiles["qv0"]), int(profiles["qv0"].shape[0])
        if profiles.get("u0") is not None:
            a.u0_base, a.v0_base = _f(profiles["u0"]), _f(profiles["v0"])
            a.wind0_base_len = int(profiles["u0"].shape[0])
        if loading is not None:
            a.loading = _f(loading)
        for name, x in zip(("du_dt", "dv_dt", "dw_dt", "drho_dt", "dp_dt"), outs):
            setattr(a, name, _f(x) if x is not None else None)
        if advection is not None:
            a.du_advection_dt, a.dv_advection_dt, a.dw_advection_dt = (_f(x) for x in advection)
        a.nx, a.ny, a.nz = (int(x) for x in st["u"].shape)
        a.dx, a.dy, a.dz = (float(x) for x in grid)
        a.g, a.coriolis_f, a.coriolis_beta = g, coriolis_f, beta
        a.has_moisture, a.has_loading = int(moist), int(loading is not None)
        a.frame_velocity_u, a.frame_velocity_v = frame
        a.memory = MEMORY_DEVICE if hasattr(st["u"], "data_ptr") else MEMORY_HOST
        assert nz >= 2
        self.check(self.lib.nimbus_cuda_cgrid_slow_tendencies(self.handle, ctypes.byref(a)))

    def device_info(self) -> dict:
        """Name, SM count, compute capability and memory of the context's device."""
        d = DeviceInfo()
        self.check(self.lib.nimbus_cuda_device_info(self.handle, ctypes.byref(d)))
        return {"name": d.name.decode(), "sm_count": d.sm_count, "cc": (d.cc_major, d.cc_minor),
                "total_bytes": d.total_bytes, "free_bytes": d.free_bytes}

    def resolve_substep_count(self, dt, c_max, min_spacing, requested=0) -> int:
        """The reference's substep-count rule (split_explicit.cpp:67-170)."""
        n = int(self.lib.nimbus_cuda_resolve_substep_count(float(dt), float(c_max), float(min_spacing),
                                                             int(requested)))
        if n < 1:
            raise ValueError("split-explicit acoustic CFL cannot be resolved")
        return n

    def acoustic_boundaries(self, args: BoundaryArgs) -> int:
        return self.lib.nimbus_cuda_acoustic_boundaries(self.handle, ctypes.byref(args))

    def smagorinsky_fused(self, args: SmagorinskyArgs) -> int:
        return self.lib.nimbus_cuda_smagorinsky_fused(self.handle, ctypes.byref(args))

    def sgs_apply(self, args: SgsApplyArgs) -> int:
        return self.lib.nimbus_cuda_sgs_apply(self.handle, ctypes.byref(args))

    def sgs_stability(self, args: SmagorinskyArgs) -> dict:
        """The stability limits of args' state and rates; raises on refusal."""
        out = SgsStability()
        self.check(self.lib.nimbus_cuda_sgs_stability(self.handle, ctypes.byref(args), ctypes.byref(out)))
        return {"maximum": out.maximum_timestep_s, "momentum_energy": out.momentum_energy_timestep_s,
                "theta_monotonic": out.theta_monotonic_timestep_s, "qv_monotonic": out.qv_monotonic_timestep_s,
                "dissipation_w": out.momentum_irreversible_dissipation_w}

    def sgs_step(self, args: SgsStepArgs) -> tuple:
        """(substeps, smallest stability limit) of one explicit SGS integration."""
        count = ctypes.c_int(0)
        limit = ctypes.c_double(0.0)
        self.check(self.lib.nimbus_cuda_sgs_step(self.handle, ctypes.byref(args), ctypes.byref(count),
                                                 ctypes.byref(limit)))
        return count.value, limit.value

    def cell_centre_velocity(self, args: CellCentreArgs) -> int:
        return self.lib.nimbus_cuda_cell_centre_velocity(self.handle, ctypes.byref(args))

    def history_snapshot(self, args: HistoryArgs) -> int:
        return self.lib.nimbus_cuda_history_snapshot(self.handle, ctypes.byref(args))

    def state_relaxation(self, args: StateRelaxationArgs) -> int:
        return self.lib.nimbus_cuda_state_relaxation(self.handle, ctypes.byref(args))


def clamp_defaults() -> dict:
    """The reference's dispatch constants (dynamics.cpp:4560-4586, field_bounds.hpp)."""
    return dict(gamma=initial.GAMMA, rho_min=initial.RHO_MIN, rho_max=initial.RHO_MAX, p_min=initial.P_MIN,
                p_max=initial.P_MAX, p_ref_fallback=100000.0, wind_clamp_h=initial.WIND_H,
                wind_clamp_v=initial.WIND_V)


def fused_args(st, rho0, p0, dt_small, grid, drho=None, memory=MEMORY_HOST, stream=None) -> AcousticFusedArgs:
    nx, ny, nz = (st["u"].shape if hasattr(st["u"], "shape") else st["shape"])
    a = AcousticFusedArgs()
    a.u, a.v, a.w, a.rho, a.p, a.theta = (_f(st[k]) for k in ("u", "v", "w", "rho", "p", "theta"))
    a.rho0_base, a.p0_base = _d(rho0), _d(p0)
    a._keep = (dict(st), rho0, p0, drho)  # the block holds raw pointers: keep every array alive
    a.base_len = nz
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dx, a.dy, a.dz = grid
    a.dt_small = dt_small
    for key, val in clamp_defaults().items():
        setattr(a, key, val)
    a.drho_scratch = _f(drho)
    a.memory = memory
    a.stream = stream
    return a


def batched_args(st, rho0, p0, dt_small, n_substeps, grid, bc, mfx, mfy, mfz, weight, wave_in, wave_out,
                 density_begin=None, frame=(0.0, 0.0), memory=MEMORY_HOST, stream=None) -> AcousticBatchedArgs:
    nx, ny, nz = st["u"].shape
    a = AcousticBatchedArgs()
    a._keep = (dict(st), rho0, p0, mfx, mfy, mfz, wave_in, wave_out, density_begin)
    a.u, a.v, a.w, a.rho, a.p, a.theta = (_f(st[k]) for k in ("u", "v", "w", "rho", "p", "theta"))
    a.rho0_base, a.p0_base = _d(rho0), _d(p0)
    a.base_len = nz
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dx, a.dy, a.dz = grid
    a.dt_small = dt_small
    a.n_substeps = n_substeps
    for key, val in clamp_defaults().items():
        setattr(a, key, val)
    a.bc_west, a.bc_east, a.bc_south, a.bc_north, a.bc_bottom, a.bc_top = (int(x) for x in bc)
    a.mass_flux_x, a.mass_flux_y, a.mass_flux_z = _f(mfx), _f(mfy), _f(mfz)
    a.accumulate_mass_flux = 1 if mfx is not None else 0
    a.mass_flux_weight = weight
    a.frame_velocity_u_ms, a.frame_velocity_v_ms = frame
    a.wave_history = _f(wave_in)
    a.wave_history_output = _f(wave_out)
    a.density_begin = _f(density_begin)
    a.memory = memory
    a.stream = stream
    return a


def transport_args(q_in: Sequence, q_out: Sequence, pd: Sequence[int], rho_end, rho_begin, mfx, mfy, mfz, dt,
                   grid, weno=True, top_open=False, memory=MEMORY_HOST, stream=None) -> ScalarTransportArgs:
    n = len(q_in)
    nx, ny, nz = rho_end.shape
    a = ScalarTransportArgs()
    qi = (_fp * max(n, 1))(*[_f(q) for q in q_in])
    qo = (_fp * max(n, 1))(*[_f(q) for q in q_out])
    flags = (ctypes.c_int * max(n, 1))(*[int(x) for x in pd])
    a._keep = (qi, qo, flags, list(q_in), list(q_out), rho_end, rho_begin, mfx, mfy, mfz)
    a.q_in, a.q_out, a.positive_definite = qi, qo, flags
    a.n_scalars = n
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dx, a.dy, a.dz = grid
    a.dt = dt
    a.rho_end, a.rho_begin = _f(rho_end), _f(rho_begin)
    a.mass_flux_x, a.mass_flux_y, a.mass_flux_z = _f(mfx), _f(mfy), _f(mfz)
    a.weno = int(weno)
    a.top_open = int(top_open)
    a.rho_floor = initial.RHO_MIN
    a.memory = memory
    a.stream = stream
    return a


def slow_args(st, base, grid, dt_large=0.0, coriolis_f=0.0, moist=True, outputs=None, frame=(0.0, 0.0),
              memory=MEMORY_HOST, stream=None) -> SlowArgs:
    """Argument block for nimbus_cuda_slow_tendencies / nimbus_cuda_slow_step.
    `outputs` is (du, dv, dw, dp) or None."""
    nx, ny, nz = st["u"].shape
    a = SlowArgs()
    qv = st.get("qv") if moist else None
    qc = st.get("qc") if moist else None
    qr = st.get("qr") if moist else None
    outs = outputs or (None, None, None, None)
    a._keep = (dict(st), base["rho0"], base.get("qv0"), base.get("u0"), base.get("v0"), outs)
    a.u, a.v, a.w, a.p, a.rho = (_f(st[k]) for k in ("u", "v", "w", "p", "rho"))
    a.qv, a.qc, a.qr = _f(qv), _f(qc), _f(qr)
    a.rho0_base = _d(base["rho0"])
    a.qv0_base = _d(base["qv0"]) if moist else None
    a.u0_base, a.v0_base = _d(base["u0"]), _d(base["v0"])
    a.base_len = nz
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dx, a.dy, a.dz = grid
    a.dt_large = dt_large
    a.gravity = initial.G
    a.coriolis_f = coriolis_f
    a.frame_velocity_u_ms, a.frame_velocity_v_ms = frame
    a.du_dt, a.dv_dt, a.dw_dt, a.dp_dt = (_f(o) for o in outs)
    a.memory = memory
    a.stream = stream
    return a


def cgrid_cell_domain(nx: int, ny: int, nz: int) -> tuple:
    """Physical cell domain of the C-grid microphysics step: the lateral
    ghost ring is excluded, every level is kept (microphysics_step.cpp:86-96)."""
    return (1, nx - 1, 1, ny - 1, 0, nz)


def kessler_args(st, dz, dt, domain=None, outputs=None, memory=MEMORY_HOST, stream=None) -> KesslerArgs:
    """Argument block for nimbus_cuda_kessler_tendencies / _step.  `st` holds
    theta, qv, qc, qr, p, rho; `outputs` is (dtheta, dqv, dqc, dqr) or None."""
    nx, ny, nz = st["theta"].shape
    a = KesslerArgs()
    outs = outputs or (None, None, None, None)
    a._keep = (dict(st), outs)
    a.theta, a.qv, a.qc, a.qr, a.p, a.rho = (_f(st[k]) for k in ("theta", "qv", "qc", "qr", "p", "rho"))
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dz, a.dt = dz, dt
    a.domain[:] = [int(x) for x in (domain or cgrid_cell_domain(nx, ny, nz))]
    a.dtheta_dt, a.dqv_dt, a.dqc_dt, a.dqr_dt = (_f(o) for o in outs)
    a.memory = memory
    a.stream = stream
    return a


def state_relaxation_args(fields, profiles, dt, memory=MEMORY_HOST, stream=None) -> StateRelaxationArgs:
    """Argument block for nimbus_cuda_state_relaxation on fields' u, v, w,
    theta with a nimbus_b200.sponge.SpongeProfiles."""
    P = profiles
    d = lambda x: np.ascontiguousarray(x, dtype=np.float64)  # noqa: E731
    prof = [d(P.alpha), d(P.upper_w_alpha), d(P.w_only_alpha), d(P.u_ref), d(P.v_ref), d(P.theta_ref)]
    lateral = d(P.lateral_alpha) if len(P.lateral_alpha) else None
    a = StateRelaxationArgs()
    a._keep = (fields, prof, lateral)
    a.u, a.v, a.w, a.theta = (_f(fields[k]) for k in ("u", "v", "w", "theta"))
    a.nx, a.ny, a.nz = tuple(fields["u"].shape)
    a.alpha, a.upper_w_alpha, a.w_only_alpha, a.u_ref, a.v_ref, a.theta_ref = (_d(x) for x in prof)
    a.lateral_width = len(P.lateral_alpha)
    a.lateral_alpha = _d(lateral)
    a.do_upper, a.do_w_only, a.do_lateral = int(P.do_upper), int(P.do_w_only), int(P.do_lateral)
    a.staggered, a.implicit_mode = int(P.staggered), int(P.implicit_mode)
    a.dt = float(dt)
    a.memory = memory
    a.stream = stream
    return a


SGS_RATES = ("dudt", "dvdt", "dwdt", "dthdt", "dqvdt")


def _empty_like(x):
    return np.empty_like(x) if isinstance(x, np.ndarray) else x.new_empty(x.shape)


def smagorinsky_args(st, dz, grid, sgs, outputs=None, rates=None, memory=MEMORY_HOST, stream=None,
                     open_top=False) -> SmagorinskyArgs:
    """Argument block for nimbus_cuda_smagorinsky_fused / _sgs_stability on st's
    u, v, w, theta, rho and optional qv with a nimbus_b200.sgs.SgsConfig.
    outputs: {nu_t, K_theta, K_q, dudt, dvdt, dwdt, dthdt, dqvdt} arrays or
    tensors (default: new ones like u); rates: the five rates for the
    stability call instead."""
    u = st["u"]
    qv = st.get("qv")
    if outputs is None:
        outputs = {k: _empty_like(u) for k in ("nu_t", "K_theta", "K_q", *SGS_RATES)}
    if rates is not None:
        outputs = {**outputs, **rates}
    dzh = np.ascontiguousarray(dz, dtype=np.float64)
    a = SmagorinskyArgs()
    a._keep = (st, dzh, outputs)
    a.outputs = outputs
    for k in ("u", "v", "w", "theta", "rho"):
        setattr(a, k, _f(st[k]))
    a.qv = _f(qv)
    a.dz = _d(dzh)
    a.nx, a.ny, a.nz = tuple(u.shape)
    a.filter_mode = 1 if sgs.filter_width == "dx" else 0
    a.use_horizontal, a.use_vertical = int(sgs.use_horizontal), int(sgs.use_vertical)
    a.periodic_x, a.periodic_y = int(sgs.periodic_x), int(sgs.periodic_y)
    for f in range(4):
        a.open_lateral[f] = int(bool(sgs.open_lateral[f]))
    a.open_top = int(bool(open_top))
    a.dx, a.dy = float(grid[0]), float(grid[1])
    a.Cs, a.Pr_t, a.Sc_t, a.nu_t_max, a.K_max = (float(x) for x in (sgs.Cs, sgs.Pr_t, sgs.Sc_t, sgs.nu_t_max,
                                                                    sgs.K_max))
    a.nu_t, a.K_theta, a.K_q = (_f(outputs.get(k)) for k in ("nu_t", "K_theta", "K_q"))
    a.dudt_sgs, a.dvdt_sgs, a.dwdt_sgs, a.dthetadt_sgs, a.dqvdt_sgs = (_f(outputs.get(k)) for k in SGS_RATES)
    a.memory = memory
    a.stream = stream
    return a


def sgs_apply_args(st, rates, dt, theta0=None, sanitize=True, memory=MEMORY_HOST, stream=None) -> SgsApplyArgs:
    """Argument block for nimbus_cuda_sgs_apply on st's u, v, w, theta and
    optional qv with the reference's clamp bounds."""
    t0 = None if theta0 is None else np.ascontiguousarray(theta0, dtype=np.float64)
    a = SgsApplyArgs()
    a._keep = (st, rates, t0)
    for k in ("u", "v", "w", "theta"):
        setattr(a, k, _f(st[k]))
    a.qv = _f(st.get("qv"))
    a.dudt, a.dvdt, a.dwdt, a.dthetadt = (_f(rates[k]) for k in ("dudt", "dvdt", "dwdt", "dthdt"))
    a.dqvdt = _f(rates.get("dqvdt")) if st.get("qv") is not None else None
    a.theta0_base = _d(t0)
    a.nx, a.ny, a.nz = tuple(st["u"].shape)
    a.dt = float(dt)
    a.sanitize = int(bool(sanitize))
    a.theta_reference = 300.0
    a.theta_min, a.theta_max, a.qv_max, a.wind_h_max, a.wind_v_max = 200.0, 700.0, 0.05, 180.0, 120.0
    a.memory = memory
    a.stream = stream
    return a


def sgs_step_args(st, dz, grid, sgs, dt, theta0=None, time_s=0.0, sanitize=True, stream=None,
                  open_top=False) -> SgsStepArgs:
    """Argument block for nimbus_cuda_sgs_step on device tensors (scratch for
    the coefficients and rates comes from the context)."""
    closure = smagorinsky_args(st, dz, grid, sgs, outputs={}, memory=MEMORY_DEVICE, stream=stream,
                               open_top=open_top)
    t0 = None if theta0 is None else np.ascontiguousarray(theta0, dtype=np.float64)
    a = SgsStepArgs()
    a._keep = (closure, t0)
    a.closure = closure
    a.theta0_base = _d(t0)
    a.dt, a.dt_sgs, a.time_s = float(dt), float(sgs.dt_sgs), float(time_s)
    a.sanitize = int(bool(sanitize))
    return a


def cell_centre_args(u=None, v=None, w=None, outputs=None, ground_w=None, memory=MEMORY_HOST,
                     stream=None) -> CellCentreArgs:
    """Argument block for nimbus_cuda_cell_centre_velocity.  outputs: (uc, vc,
    wc) arrays or tensors, None entries skipped; by default one array (host) or
    tensor (device) per given face field."""
    faces = (u, v, w)
    face = next(x for x in faces if x is not None)
    if outputs is None:
        outputs = tuple(None if x is None else (np.empty_like(x) if isinstance(x, np.ndarray) else x.new_empty(x.shape))
                        for x in faces)
    g = None if ground_w is None else np.ascontiguousarray(ground_w, dtype=np.float64)
    a = CellCentreArgs()
    a._keep = (faces, outputs, g)
    a.outputs = outputs
    a.u, a.v, a.w = (_f(x) for x in faces)
    a.u_centre, a.v_centre, a.w_centre = (_f(x) for x in outputs)
    a.ground_w = _d(g)
    a.nx, a.ny, a.nz = tuple(face.shape)
    a.memory = memory
    a.stream = stream
    return a


def history_args(fields: dict, mask: int, host_image, shape, ground_w=None, stream=None) -> HistoryArgs:
    """Argument block for nimbus_cuda_history_snapshot: fields maps names to
    device tensors (or addresses); host_image a C-contiguous float32 array of
    at least popcount(mask) * cells floats (pinned for overlap)."""
    g = None if ground_w is None else np.ascontiguousarray(ground_w, dtype=np.float64)
    a = HistoryArgs()
    a._keep = (fields, host_image, g)
    for k in HISTORY_FIELDS:
        setattr(a, k, _f(fields.get(k)))
    a.fields = int(mask)
    a.ground_w = _d(g)
    a.nx, a.ny, a.nz = (int(x) for x in shape)
    a.host_image = _f(host_image)
    a.stream = stream
    return a


def npy_write_3d(data: np.ndarray, path, lib: Optional[ctypes.CDLL] = None) -> int:
    """nimbus_npy_write_3d of a C-contiguous float32 [d0][d1][d2] array; the
    status code."""
    lib = lib or load_library()
    a = np.ascontiguousarray(data, dtype=np.float32)
    d = tuple(a.shape) if a.ndim == 3 else (0, 0, 0)
    return lib.nimbus_npy_write_3d(a.ctypes.data_as(_fp), *[int(x) for x in d], str(path).encode())


def history_write(image: np.ndarray, mask: int, shape, step_dir, lib: Optional[ctypes.CDLL] = None) -> int:
    """nimbus_history_write: <step_dir>/<name>.npy for each field of mask
    from a history image; the status code."""
    lib = lib or load_library()
    assert image.dtype == np.float32 and image.flags["C_CONTIGUOUS"]
    return lib.nimbus_history_write(image.ctypes.data_as(_fp), int(mask), *[int(x) for x in shape],
                                    str(step_dir).encode())


def eos_args(p, rho, theta, qv=None, qc=None, qr=None, memory=MEMORY_HOST, stream=None, p0=None) -> EosArgs:
    """Argument block for nimbus_cuda_eos_projection over every cell; qv/qc/qr
    (all or none) add the moist-state checks; p0 (FP64 per level) lets the
    FP32 form evaluate around the base pressure."""
    a = EosArgs()
    a._keep = (p, rho, theta, qv, qc, qr, p0)
    a.p0_base = _d(p0) if p0 is not None else None
    a.p, a.rho, a.theta = _f(p), _f(rho), _f(theta)
    a.qv, a.qc, a.qr = _f(qv), _f(qc), _f(qr)
    a.nx, a.ny, a.nz = tuple(p.shape)
    a.gamma = initial.GAMMA
    a.memory = memory
    a.stream = stream
    return a


def boundary_args(st, grid, bc, dt_small=0.0, wave=None, frame=(0.0, 0.0), stream=None) -> BoundaryArgs:
    """Argument block for nimbus_cuda_acoustic_boundaries (device tensors)."""
    nx, ny, nz = tuple(st["u"].shape)
    a = BoundaryArgs()
    a._keep = (dict(st), wave)
    a.u, a.v, a.w, a.rho, a.p = (_f(st[k]) for k in ("u", "v", "w", "rho", "p"))
    a.wave_history = _f(wave)
    a.nx, a.ny, a.nz = nx, ny, nz
    a.dx, a.dy = grid[0], grid[1]
    a.dt_small = dt_small
    a.bc_west, a.bc_east, a.bc_south, a.bc_north, a.bc_bottom, a.bc_top = (int(x) for x in bc)
    a.frame_velocity_u_ms, a.frame_velocity_v_ms = frame
    a.stream = stream
    return a


MEMBER_FIELDS = ("u", "v", "w", "rho", "p", "theta", "qv", "qc", "qr")


def sponge_desc(profiles) -> SpongeDesc:
    """nimbus_sponge_desc from a nimbus_b200.sponge.SpongeProfiles."""
    P = profiles
    d = lambda x: np.ascontiguousarray(x, dtype=np.float64)  # noqa: E731
    prof = [d(P.alpha), d(P.upper_w_alpha), d(P.w_only_alpha), d(P.u_ref), d(P.v_ref), d(P.theta_ref)]
    lateral = d(P.lateral_alpha) if len(P.lateral_alpha) else None
    s = SpongeDesc()
    s._keep = (prof, lateral)
    s.alpha, s.upper_w_alpha, s.w_only_alpha, s.u_ref, s.v_ref, s.theta_ref = (_d(x) for x in prof)
    s.lateral_width = len(P.lateral_alpha)
    s.lateral_alpha = _d(lateral)
    s.do_upper, s.do_w_only, s.do_lateral = int(P.do_upper), int(P.do_w_only), int(P.do_lateral)
    s.staggered, s.implicit_mode = int(P.staggered), int(P.implicit_mode)
    return s


def member_desc(shape, grid, dt, n_substeps, bc, base, coriolis_f=0.0, frame=(0.0, 0.0),
                microphysics=1, sponge=None, final_closure=False, resolve_substeps=False) -> MemberDesc:
    """Descriptor of one engine member; `base` holds the FP64 profiles
    rho0, p0, qv0 (and optionally u0, v0); `sponge` (SpongeProfiles) adds the
    end-of-step sponge, `final_closure` the closing boundary refresh.  With
    resolve_substeps the substep count is re-derived from the state before
    every large step and n_substeps is the requested minimum (0: none)."""
    d = MemberDesc()
    d.nx, d.ny, d.nz = (int(x) for x in shape)
    d.dx, d.dy, d.dz = grid
    d.dt = dt
    d.n_substeps = int(n_substeps)
    d.bc[:] = [int(x) for x in bc]
    d.coriolis_f = coriolis_f
    d.frame_velocity_u_ms, d.frame_velocity_v_ms = frame
    d.microphysics = int(microphysics)
    prof = {k: np.ascontiguousarray(base[k], dtype=np.float64) for k in ("rho0", "p0", "qv0", "u0", "v0")
            if base.get(k) is not None}
    d._keep = prof
    d.rho0_base, d.p0_base, d.qv0_base = _d(prof["rho0"]), _d(prof["p0"]), _d(prof["qv0"])
    d.u0_base = _d(prof["u0"]) if "u0" in prof else None
    d.v0_base = _d(prof["v0"]) if "v0" in prof else None
    if sponge is not None:
        sd = sponge_desc(sponge)
        d._sponge = sd
        d.sponge = ctypes.pointer(sd)
    d.final_closure = int(bool(final_closure))
    d.resolve_substeps = int(bool(resolve_substeps))
    return d


def member_state(st) -> MemberState:
    s = MemberState()
    s._keep = {k: np.ascontiguousarray(st[k], dtype=np.float32) for k in MEMBER_FIELDS}
    for k in MEMBER_FIELDS:
        setattr(s, k, _f(s._keep[k]))
    return s


class Engine:
    """Resident members advanced together (nimbus_cuda_engine_*): one
    batched launch per phase of the large step, replayed from a CUDA graph."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        self.lib = ctx.lib
        h = ctypes.c_void_p()
        ctx.check(self.lib.nimbus_cuda_engine_create(ctx.handle, ctypes.byref(h)))
        self.handle = h.value
        self.shapes = {}

    def close(self):
        if self.handle:
            self.lib.nimbus_cuda_engine_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def member_bytes(self, desc: MemberDesc) -> int:
        return int(self.lib.nimbus_cuda_engine_member_bytes(ctypes.byref(desc)))

    def admit(self, desc: MemberDesc, state, reserve_bytes: int = 0) -> int:
        """Admit a member with its initial state; raises NimbusCudaError
        (OUT_OF_MEMORY) when it does not fit the free HBM."""
        mid = ctypes.c_int(0)
        st = member_state(state)
        self.ctx.check(self.lib.nimbus_cuda_engine_admit(self.handle, ctypes.byref(desc), ctypes.byref(st),
                                                         int(reserve_bytes), ctypes.byref(mid)))
        self.shapes[mid.value] = (desc.nx, desc.ny, desc.nz)
        return mid.value

    def try_admit(self, desc: MemberDesc, state, reserve_bytes: int = 0) -> Optional[int]:
        """Admission that returns None instead of raising when HBM is full."""
        mid = ctypes.c_int(0)
        st = member_state(state)
        rc = self.lib.nimbus_cuda_engine_admit(self.handle, ctypes.byref(desc), ctypes.byref(st),
                                               int(reserve_bytes), ctypes.byref(mid))
        if rc == NIMBUS_ERR_OUT_OF_MEMORY:
            return None
        self.ctx.check(rc)
        self.shapes[mid.value] = (desc.nx, desc.ny, desc.nz)
        return mid.value

    def member_status_async(self, member_id: int, host_flags) -> None:
        """Enqueue the copy of a member's status word into host_flags (a pinned
        uint32 array of one element), in stream order."""
        self.ctx.check(self.lib.nimbus_cuda_engine_member_status_async(self.handle, int(member_id),
                                                                      ctypes.c_void_p(host_flags.ctypes.data)))

    def autotune(self, steps: int = 3) -> dict:
        """Time the lane count, then the continuity x momentum kernel forms,
        on the resident members (states restored afterwards), keep the
        fastest; returns the choice and every candidate's ms per step."""
        t = EngineTuning()
        self.ctx.check(self.lib.nimbus_cuda_engine_autotune(self.handle, int(steps), ctypes.byref(t)))
        cands = [{"lanes": t.candidate_lanes[i], "continuity": ACOUSTIC_FORM_NAMES[t.candidate_form[i]],
                  "momentum": ACOUSTIC_FORM_NAMES[t.candidate_momentum_form[i]],
                  "march": t.candidate_march[i], "ms_per_step": round(t.candidate_ms[i], 4)}
                 for i in range(t.candidates)]
        return {"lanes": t.lanes, "continuity_form": ACOUSTIC_FORM_NAMES[t.acoustic_form],
                "momentum_form": ACOUSTIC_FORM_NAMES[t.momentum_form], "march": t.march,
                "ms_per_step": round(t.ms_per_step, 4), "steps_per_candidate": int(steps), "candidates": cands}

    def graph_builds(self) -> tuple:
        """(instantiations, in-place updates) of the step graphs so far."""
        a, b = ctypes.c_uint64(), ctypes.c_uint64()
        self.ctx.check(self.lib.nimbus_cuda_engine_graph_builds(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def member_substeps(self, member_id: int) -> int:
        """Substep count of the member's last enqueued (or first) large step."""
        n = ctypes.c_int(0)
        self.ctx.check(self.lib.nimbus_cuda_engine_member_substeps(self.handle, int(member_id), ctypes.byref(n)))
        return n.value

    def retire(self, member_id: int):
        self.ctx.check(self.lib.nimbus_cuda_engine_retire(self.handle, int(member_id)))
        self.shapes.pop(member_id, None)

    def read(self, member_id: int) -> dict:
        shape = self.shapes[member_id]
        out = {k: np.empty(shape, np.float32) for k in MEMBER_FIELDS}
        self.ctx.check(self.lib.nimbus_cuda_engine_read(self.handle, int(member_id), ctypes.byref(member_state(out))))
        return out

    def read_into(self, member_id: int, out: dict):
        st = MemberState()
        for k in MEMBER_FIELDS:
            setattr(st, k, _f(out[k]))
        self.ctx.check(self.lib.nimbus_cuda_engine_read(self.handle, int(member_id), ctypes.byref(st)))

    def write(self, member_id: int, state: dict):
        """Replace a member's state from host arrays (pinned arrays copy fastest)."""
        st = MemberState()
        for k in MEMBER_FIELDS:
            a = state[k]
            assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"] and a.shape == self.shapes[member_id], k
            setattr(st, k, _f(a))
        self.ctx.check(self.lib.nimbus_cuda_engine_write(self.handle, int(member_id), ctypes.byref(st)))

    def _state_of(self, member_id: int, arrays: dict) -> MemberState:
        st = MemberState()
        for k in MEMBER_FIELDS:
            a = arrays[k]
            assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"] and a.shape == self.shapes[member_id], k
            setattr(st, k, _f(a))
        return st

    def write_async(self, member_id: int, state: dict):
        """Enqueue the state upload on the engine's stream (pinned arrays; keep
        them alive and unchanged until synchronize)."""
        self.ctx.check(self.lib.nimbus_cuda_engine_write_async(self.handle, int(member_id),
                                                               ctypes.byref(self._state_of(member_id, state))))

    def read_async(self, member_id: int, out: dict):
        """Enqueue the state download on the engine's stream into `out`."""
        self.ctx.check(self.lib.nimbus_cuda_engine_read_async(self.handle, int(member_id),
                                                              ctypes.byref(self._state_of(member_id, out))))

    @property
    def stream(self) -> int:
        return int(self.lib.nimbus_cuda_engine_stream(self.handle) or 0)

    def set_lanes(self, lanes: int):
        """Split the members over up to `lanes` parallel streams (default 4)."""
        self.ctx.check(self.lib.nimbus_cuda_engine_set_lanes(self.handle, int(lanes)))

    @property
    def lanes(self) -> int:
        return int(self.lib.nimbus_cuda_engine_lanes(self.handle))

    def set_acoustic_form(self, form: int):
        """ACOUSTIC_TABLE / _CONST / _MARCH / _PAIR / _BULK kernels for the
        continuity and momentum passes; results do not depend on it."""
        self.ctx.check(self.lib.nimbus_cuda_engine_set_acoustic_form(self.handle, int(form)))

    @property
    def acoustic_form(self) -> int:
        return int(self.lib.nimbus_cuda_engine_acoustic_form(self.handle))

    def set_pass_forms(self, continuity: int, momentum: int):
        """Kernel form of each acoustic pass."""
        self.ctx.check(self.lib.nimbus_cuda_engine_set_pass_forms(self.handle, int(continuity), int(momentum)))

    @property
    def pass_forms(self) -> tuple:
        a, b = ctypes.c_int(), ctypes.c_int()
        self.ctx.check(self.lib.nimbus_cuda_engine_pass_forms(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def set_march(self, planes: int):
        """Cells one thread of the marching acoustic passes advances along x."""
        self.ctx.check(self.lib.nimbus_cuda_engine_set_march(self.handle, int(planes)))

    @property
    def march(self) -> int:
        return int(self.lib.nimbus_cuda_engine_march(self.handle))

    def image_bytes(self) -> int:
        """Size of the state image (all members' nine fields in one block)."""
        return int(self.lib.nimbus_cuda_engine_image_bytes(self.handle))

    def image_offset(self, member_id: int) -> int:
        off = int(self.lib.nimbus_cuda_engine_image_offset(self.handle, int(member_id)))
        if off == ctypes.c_size_t(-1).value:
            raise KeyError(member_id)
        return off

    def image_views(self, image: np.ndarray) -> dict:
        """{member id: {field: array view}} into a host image of image_bytes()
        bytes (any dtype, C-contiguous)."""
        flat = image.reshape(-1).view(np.uint8)
        assert flat.nbytes >= self.image_bytes()
        views = {}
        for mid, shape in self.shapes.items():
            n = shape[0] * shape[1] * shape[2]
            blk = flat[self.image_offset(mid):].view(np.float32)[:9 * n] if n else flat[:0].view(np.float32)
            views[mid] = {k: blk[i * n:(i + 1) * n].reshape(shape) for i, k in enumerate(MEMBER_FIELDS)}
        return views

    def upload_image_async(self, image: np.ndarray):
        """Enqueue the whole state image upload on the engine's stream (pinned
        memory; keep it alive and unchanged until synchronize)."""
        assert image.flags["C_CONTIGUOUS"] and image.nbytes >= self.image_bytes()
        self.ctx.check(self.lib.nimbus_cuda_engine_upload_image_async(self.handle, image.ctypes.data))

    def download_image_async(self, image: np.ndarray):
        assert image.flags["C_CONTIGUOUS"] and image.nbytes >= self.image_bytes()
        self.ctx.check(self.lib.nimbus_cuda_engine_download_image_async(self.handle, image.ctypes.data))

    def history_async(self, member_id: int, mask: int, image: np.ndarray):
        """Enqueue a history frame of the member (cell-centred u, v, w and the
        scalars of mask, image order) into a pinned float32 image on the
        engine's stream; complete after synchronize."""
        shape = self.shapes.get(member_id, (0, 0, 0))  # an unknown id is the library's to refuse
        assert image.dtype == np.float32 and image.flags["C_CONTIGUOUS"]
        assert image.size >= bin(mask).count("1") * shape[0] * shape[1] * shape[2]
        self.ctx.check(self.lib.nimbus_cuda_engine_history_async(self.handle, int(member_id), int(mask),
                                                                 image.ctypes.data))

    def step(self, n: int = 1):
        self.ctx.check(self.lib.nimbus_cuda_engine_step(self.handle, int(n)))

    def synchronize(self):
        self.ctx.check(self.lib.nimbus_cuda_engine_synchronize(self.handle))

    def member_status(self, member_id: int) -> int:
        f = ctypes.c_uint(0)
        self.ctx.check(self.lib.nimbus_cuda_engine_member_status(self.handle, int(member_id), ctypes.byref(f)))
        return f.value

    def set_graph(self, enable: bool):
        self.ctx.check(self.lib.nimbus_cuda_engine_set_graph(self.handle, int(bool(enable))))

    @property
    def members(self) -> int:
        return int(self.lib.nimbus_cuda_engine_members(self.handle))

    @property
    def launches_per_step(self) -> int:
        return int(self.lib.nimbus_cuda_engine_launches_per_step(self.handle))


class CudaComputeBackend:
    """Mirror of the reference's ComputeBackend for the CUDA backend: name(),
    initialize(), shutdown(), supports(), successful_kernel_dispatch_count()
    and the three hot-path dispatches.  Dispatches take host numpy arrays and
    return ``True`` on success, ``False`` when refused (``last_error`` says why),
    leaving the arrays untouched on refusal -- the reference's contract."""

    SUPPORTED = ("AcousticSubstepFusedCartesianCgrid", "AcousticSubstepsBatchedCartesianCgrid",
                 "ConservativeCartesianCgridTransport")

    def __init__(self, device: int = 0):
        self.device = device
        self.ctx: Optional[Context] = None
        self.last_error = ""

    def name(self) -> str:
        return "cuda"

    def initialize(self) -> bool:
        try:
            self.ctx = Context(self.device)
            return True
        except Exception as exc:  # the reference reports initialize failures as (false, error)
            self.last_error = str(exc)
            return False

    def shutdown(self):
        if self.ctx:
            self.ctx.close()
            self.ctx = None

    def supports(self, op: str) -> bool:
        return op in self.SUPPORTED

    def supports_supplied_cartesian_cgrid_mass_flux(self) -> bool:
        return True

    def supports_batched_cartesian_cgrid_mass_flux_export(self) -> bool:
        return True

    def successful_kernel_dispatch_count(self) -> int:
        return self.ctx.kernel_launches if self.ctx else 0

    def _run(self, fn, args) -> bool:
        rc = fn(args)
        if rc != NIMBUS_OK:
            self.last_error = f"{STATUS_NAMES.get(rc, rc)}: {self.ctx.last_error}"
            return False
        return True

    def dispatch_acoustic_substep_fused_cartesian_cgrid(self, st, rho0, p0, dt_small, grid, drho=None) -> bool:
        return self._run(self.ctx.acoustic_fused, fused_args(st, rho0, p0, dt_small, grid, drho))

    def dispatch_acoustic_substeps_batched_cartesian_cgrid(self, st, rho0, p0, dt_small, n_substeps, grid, bc,
                                                           mfx, mfy, mfz, weight, wave_in, wave_out,
                                                           density_begin=None, frame=(0.0, 0.0)) -> bool:
        return self._run(self.ctx.acoustic_batched,
                         batched_args(st, rho0, p0, dt_small, n_substeps, grid, bc, mfx, mfy, mfz, weight,
                                      wave_in, wave_out, density_begin, frame))

    def dispatch_advect_scalars_conservative_cartesian_cgrid(self, q_in, q_out, pd, rho_end, rho_begin, mfx, mfy,
                                                             mfz, dt, grid, weno=True, top_open=False) -> bool:
        return self._run(self.ctx.scalar_transport,
                         transport_args(q_in, q_out, pd, rho_end, rho_begin, mfx, mfy, mfz, dt, grid, weno,
                                        top_open))
