"""The end-of-step sponge (state relaxation) of a flat C-grid level: its
configuration and the per-level profiles it relaxes with.

The reference builds these profiles once per level in its Rayleigh runtime
(``ensure_initialized`` and ``ensure_lateral_initialized``,
src/core/infra/rayleigh_damping.cpp:403-509 and 1148-1192) and hands them,
packed, to its GPU dispatch (``dispatch_state_relaxation_cartesian_backend``,
src/compute/dispatch/dynamics.cpp:432-470).  ``build_profiles`` forms the same
FP64 values with the same formulas (``math.sin`` is the C library's ``sin``,
as ``std::sin`` is in the reference); ``nimbus_cuda_state_relaxation`` takes
them.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class SpongeConfig:
    """The run-configuration fields of the sponge (runtime_config.hpp:112-122,
    wind_profile.hpp): damping height z_damp (m, <= 0: 70 % of the model
    top), upper sponge rate alpha_max (1/s), w-only lid absorber depth (cells)
    and rate, lateral band width (cells) and rate, implicit (alpha dt / (1 +
    alpha dt)) or explicit (1 - exp(-alpha dt)) relaxation, and the
    environmental hodograph (u, v at the surface, 1 km and 6 km)."""
    z_damp: float = -1.0
    alpha_max: float = 0.05
    w_only_cells: int = 8
    w_only_alpha_max: float = 0.20
    lateral_width: int = 20
    lateral_alpha_max: float = 0.05
    implicit_mode: int = 0
    wind: tuple = (0.0, 0.0, 0.0, 0.0, 0.0, 0.0)


@dataclass
class SpongeProfiles:
    """Per-level rates and references of one level's sponge (FP64)."""
    alpha: np.ndarray
    upper_w_alpha: np.ndarray
    w_only_alpha: np.ndarray
    u_ref: np.ndarray
    v_ref: np.ndarray
    theta_ref: np.ndarray
    lateral_alpha: np.ndarray
    do_upper: int = 1
    do_w_only: int = 1
    do_lateral: int = 1
    staggered: int = 1
    implicit_mode: int = 0
    extra: dict = field(default_factory=dict)


def wind_at(wind, z: float):
    """compute_wind_profile (src/core/runtime/nimbus_sim.cpp:87-110): linear
    between the surface, 1 km and 6 km winds, constant above."""
    u_sfc, v_sfc, u_1, v_1, u_6, v_6 = wind
    if z <= 1000.0:
        frac = (z - 0.0) / (1000.0 - 0.0)
        return u_sfc + frac * (u_1 - u_sfc), v_sfc + frac * (v_1 - v_sfc)
    if z <= 6000.0:
        frac = (z - 1000.0) / (6000.0 - 1000.0)
        return u_1 + frac * (u_6 - u_1), v_1 + frac * (v_6 - v_1)
    return u_6, v_6


def build_profiles(config: SpongeConfig, nz: int, dz: float, theta0, staggered: bool = True) -> SpongeProfiles:
    """The profiles the reference's runtime builds for a flat level of nz
    layers of thickness dz: scalar levels at (k + 0.5) dz, w levels at
    (k + 1) dz, model top nz dz."""
    pi_half = 3.14159265358979323846 * 0.5
    z_top = float(nz) * dz
    z_damp = config.z_damp if config.z_damp > 0.0 else z_top * (1.0 - 0.3)
    depth = z_top - z_damp

    def alpha_at(h):
        if depth <= 0.0 or h <= z_damp:
            return 0.0
        frac = min(1.0, (h - z_damp) / depth)
        s = math.sin(pi_half * frac)
        return config.alpha_max * s * s

    alpha = np.zeros(nz)
    upper_w = np.zeros(nz)
    u_ref = np.zeros(nz)
    v_ref = np.zeros(nz)
    for k in range(nz):
        z = (float(k) + 0.5) * dz
        u_ref[k], v_ref[k] = wind_at(config.wind, z)
        alpha[k] = alpha_at(z)
        upper_w[k] = alpha_at(float(k + 1) * dz if staggered else z)
    w_only = np.zeros(nz)
    depth_cells = min(max(config.w_only_cells, 0), nz)
    wmax = max(config.w_only_alpha_max, 0.0)
    if depth_cells > 0 and wmax > 0.0:
        for d in range(depth_cells):
            frac = 1.0 - float(d) / float(depth_cells - 1) if depth_cells > 1 else 1.0
            s = math.sin(pi_half * frac)
            w_only[nz - 1 - d] = wmax * s * s
    width = config.lateral_width if config.lateral_alpha_max > 0.0 else 0
    lateral = np.zeros(max(width, 0))
    for d in range(width):
        s = math.sin(pi_half * (1.0 - float(d) / float(width)))
        lateral[d] = config.lateral_alpha_max * s * s
    return SpongeProfiles(alpha=alpha, upper_w_alpha=upper_w, w_only_alpha=w_only, u_ref=u_ref, v_ref=v_ref,
                          theta_ref=np.ascontiguousarray(theta0, dtype=np.float64), lateral_alpha=lateral,
                          do_upper=1, do_w_only=int(config.w_only_cells > 0), do_lateral=int(width > 0),
                          staggered=int(staggered), implicit_mode=int(config.implicit_mode))
