"""The Smagorinsky SGS closure of a flat C-grid level: its configuration and
the per-level filter widths the device kernels take.

The reference configures the closure with TurbulenceConfig
(include/turbulence/turbulence_base.hpp:47-64) and derives the lateral
topology from the run's boundary conditions (bind_flow_execution,
include/core/runtime/simulation_state.hpp:459-478): an axis is periodic when
either of its faces is, and a face is open when it is radiative or
zero-gradient.  The flat filter width depends on the level only
(compute_filter_width, src/turbulence/base/eddy_viscosity.cpp:1414-1468); the
library forms it on the host with the C library's sqrt / cbrt, the functions
the reference calls.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

BC_PERIODIC, BC_RADIATIVE, BC_ZERO_GRADIENT = 0, 1, 4
FILTER_CUBIC_ROOT, FILTER_DX = 0, 1


@dataclass
class SgsConfig:
    """Closure constants (defaults: turbulence_base.hpp:36-64), the stress
    directions (mode "3d" = both, "horizontal_only", "vertical_only"), the
    lateral topology and the explicit SGS interval dt_sgs."""
    Cs: float = 0.18
    Pr_t: float = 1.0 / 3.0
    Sc_t: float = 1.0 / 3.0
    nu_t_max: float = 1000.0
    K_max: float = 1000.0
    filter_width: str = "cubic_root"
    use_horizontal: bool = True
    use_vertical: bool = True
    periodic_x: bool = False
    periodic_y: bool = False
    open_lateral: tuple = (True, True, True, True)  # W, E, S, N
    dt_sgs: float = 1.0
    extra: dict = field(default_factory=dict)

    @classmethod
    def from_bc(cls, bc, **kw):
        """Topology from lateral boundary codes (W, E, S, N, ...)."""
        w, e, s, n = bc[:4]
        return cls(periodic_x=BC_PERIODIC in (w, e), periodic_y=BC_PERIODIC in (s, n),
                   open_lateral=tuple(b in (BC_RADIATIVE, BC_ZERO_GRADIENT) for b in (w, e, s, n)), **kw)

    @property
    def mode(self) -> str:
        return {(True, True): "3d", (True, False): "horizontal_only", (False, True): "vertical_only"}[
            (bool(self.use_horizontal), bool(self.use_vertical))]


def filter_widths(config: SgsConfig, dx: float, dy: float, dz) -> np.ndarray:
    """Delta per level: sqrt(dx dy) ("dx") or cbrt(dx dy dz_k) ("cubic_root")."""
    if config.filter_width == "dx":
        return np.full(len(dz), math.sqrt(dx * dy))
    if config.filter_width == "cubic_root":
        return np.array([math.cbrt(dx * dy * float(d)) for d in dz])
    raise ValueError(f"unsupported filter width {config.filter_width!r}")
