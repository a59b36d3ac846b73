"""Synthetic supercell initial states for the hot-path workloads.

The reference reads soundings from configuration or files; the workloads here
are generated analytically, once on the host, and the very same arrays are fed
to the CUDA path and to the CPU oracles:

* Weisman-Klemp (1982) analytic sounding: theta(z) = theta_sfc + (theta_tr -
  theta_sfc) (z/z_tr)^(5/4) below the tropopause, isothermal above; relative
  humidity 1 - 0.75 (z/z_tr)^(5/4) (0.25 above) with vapour capped at 14 g/kg.
* Hydrostatic base state integrated in FP64 with the model's dry EOS,
  p = p00 (rho R_d theta / p00)^gamma (cartesian_cgrid_3d.hpp, acoustic_cgrid_fast.cpp:140).
* Quarter-circle hodograph of total shear U_s over 0-5 km, constant above.
* Warm bubble: theta' = A cos^2(pi r / 2) for r = sqrt((x/r_h)^2 + ((z-z_c)/r_z)^2) < 1.
* Seeded uniform theta' noise below 1 km from a counter-based SplitMix64 hash
  of (seed, member, i, j, k), so any subset of cells can be regenerated
  identically on any host.

Layout is the reference's: [nx][ny][nz] float32, k fastest; u on x-faces
i+1/2, v on y-faces j+1/2, w on z-faces k+1/2.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

G = 9.81
R_D = 287.0
R_V = 461.5
CP = 1004.0
P00 = 100000.0
GAMMA = CP / (CP - R_D)
EPS_RV = R_D / R_V

# Reference clamp bounds (include/core/field/field_bounds.hpp:12-17).
RHO_MIN, RHO_MAX = 0.05, 2.0
P_MIN, P_MAX = 1000.0, 200000.0
WIND_H, WIND_V = 180.0, 120.0

# Boundary codes (include/init/config/config_v1.hpp:40-67).
PERIODIC, RADIATIVE, RIGID, RIGID_SLIP, ZERO_GRADIENT = 0, 1, 2, 3, 4
BOTTOM_NO_SLIP, BOTTOM_SLIP = 0, 1
TOP_RIGID, TOP_SPONGE, TOP_OPEN = 0, 1, 2


@dataclass
class Case:
    """One run: grid, timestep and initial-condition parameters."""

    nx: int
    ny: int
    nz: int
    dx: float
    dy: float
    dz: float
    dt: float
    substeps: int = 0            # requested minimum; 0 = the CFL rule alone
    theta_sfc: float = 300.0
    theta_tr: float = 343.0
    z_tr: float = 12000.0
    t_tr: float = 213.0
    qv_cap: float = 0.014
    shear_us: float = 25.0
    shear_depth: float = 5000.0
    bubble_amp: float = 3.0
    bubble_rh: float = 10000.0
    bubble_rz: float = 1400.0
    bubble_zc: float = 1400.0
    noise_amp: float = 0.0
    noise_depth: float = 1000.0
    seed: int = 0
    member: int = 0
    bc: tuple = (RADIATIVE, RADIATIVE, RADIATIVE, RADIATIVE, BOTTOM_SLIP, TOP_RIGID)

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape(self):
        return (self.nx, self.ny, self.nz)


def splitmix64_uniform(seed: int, member: int, i, j, k) -> np.ndarray:
    """Uniform [0,1) from SplitMix64 of a (seed, member, i, j, k) counter."""
    with np.errstate(over="ignore"):
        x = (np.uint64(seed & 0xFFFFFFFF) << np.uint64(32)) ^ np.uint64(member & 0xFFFFFFFF)
        x = x * np.uint64(0x9E3779B97F4A7C15)
        x = x ^ (np.asarray(i, np.uint64) << np.uint64(42)) ^ (np.asarray(j, np.uint64) << np.uint64(21)) \
            ^ np.asarray(k, np.uint64)
        z = x + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return (z >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def sounding(case: Case):
    """Base-state columns at scalar levels: theta0, qv0, u0, v0, p0, rho0 (FP64)."""
    nz, dz = case.nz, case.dz
    z = (np.arange(nz) + 0.5) * dz
    theta = np.where(
        z <= case.z_tr,
        case.theta_sfc + (case.theta_tr - case.theta_sfc) * (z / case.z_tr) ** 1.25,
        case.theta_tr * np.exp(G * (z - case.z_tr) / (CP * case.t_tr)),
    )
    rh = np.where(z <= case.z_tr, 1.0 - 0.75 * (z / case.z_tr) ** 1.25, 0.25)
    # Dry hydrostatic Exner integrated level to level in FP64 (midpoint theta).
    exner = np.empty(nz)
    exner[0] = 1.0 - G * z[0] / (CP * theta[0])
    for k in range(1, nz):
        exner[k] = exner[k - 1] - G * dz / (CP * 0.5 * (theta[k] + theta[k - 1]))
    p0 = P00 * exner ** (CP / R_D)
    # Invert the model EOS so that the base state is in exact EOS balance.
    rho0 = (p0 / P00) ** (1.0 / GAMMA) * P00 / (R_D * theta)
    temp = theta * exner
    es = 611.2 * np.exp(17.67 * (temp - 273.15) / (temp - 29.65))
    qvs = EPS_RV * es / np.maximum(p0 - es, 1.0)
    qv = np.minimum(rh * qvs, case.qv_cap)
    phi = 0.5 * math.pi * np.minimum(z / case.shear_depth, 1.0)
    # Quarter circle of radius U_s/2, translated so the depth-mean is small.
    u0 = 0.5 * case.shear_us * (1.0 - np.cos(phi)) * 2.0 - 0.5 * case.shear_us
    v0 = 0.5 * case.shear_us * np.sin(phi) * 2.0 - 0.25 * case.shear_us
    return dict(z=z, theta0=theta, qv0=qv, u0=u0, v0=v0, p0=p0, rho0=rho0)


def initial_state(case: Case):
    """Prognostic fields (float32) and FP64 base profiles for one case."""
    nx, ny, nz = case.shape
    base = sounding(case)
    i = np.arange(nx)[:, None, None]
    j = np.arange(ny)[None, :, None]
    k = np.arange(nz)[None, None, :]
    x = (i - 0.5 * (nx - 1)) * case.dx
    y = (j - 0.5 * (ny - 1)) * case.dy
    z = base["z"][None, None, :]
    r = np.sqrt((x / case.bubble_rh) ** 2 + (y / case.bubble_rh) ** 2 + ((z - case.bubble_zc) / case.bubble_rz) ** 2)
    dtheta = np.where(r < 1.0, case.bubble_amp * np.cos(0.5 * math.pi * r) ** 2, 0.0)
    if case.noise_amp > 0.0:
        ii, jj, kk = np.broadcast_arrays(i, j, k)
        rnd = splitmix64_uniform(case.seed, case.member, ii, jj, kk)
        dtheta = dtheta + np.where(z < case.noise_depth, case.noise_amp * (2.0 * rnd - 1.0), 0.0)
    theta = base["theta0"][None, None, :] + dtheta
    p = np.broadcast_to(base["p0"][None, None, :], (nx, ny, nz))
    rho = (p / P00) ** (1.0 / GAMMA) * P00 / (R_D * theta)
    shape = (nx, ny, nz)
    u0 = base["u0"][None, None, :]
    v0 = base["v0"][None, None, :]
    qv = np.broadcast_to(base["qv0"][None, None, :], shape)
    st = {
        "u": np.ascontiguousarray(np.broadcast_to(u0, shape), np.float32),
        "v": np.ascontiguousarray(np.broadcast_to(v0, shape), np.float32),
        "w": np.zeros(shape, np.float32),
        "rho": np.ascontiguousarray(rho, np.float32),
        "p": np.ascontiguousarray(p, np.float32),
        "theta": np.ascontiguousarray(theta, np.float32),
        "qv": np.ascontiguousarray(qv, np.float32),
        "qc": np.zeros(shape, np.float32),
        "qr": np.zeros(shape, np.float32),
    }
    return st, base


def max_sound_speed(p: np.ndarray, rho: np.ndarray, base) -> float:
    """Largest sqrt(gamma p / rho) over the state and the base columns (the
    acoustic speed choose_runtime_timestep samples before every large step,
    src/numerics/runtime.cpp:346-401,854-870), each product formed as
    (gamma * p) / rho in FP64; the maximum is taken before the (monotone,
    correctly rounded) square root, which gives the same value."""
    c_state = float(np.sqrt(np.max(GAMMA * p.astype(np.float64) / rho.astype(np.float64))))
    c_base = float(np.sqrt(np.max(GAMMA * np.asarray(base["p0"], np.float64) / np.asarray(base["rho0"], np.float64))))
    return max(c_state, c_base)


def resolve_substep_count(dt_large: float, c_max: float, dx: float, dy: float, dz: float,
                          requested: int = 0) -> int:
    """N = max(requested, ceil(dt c_max / (0.5 min(dx,dy,dz))) + 1, 2):
    SplitExplicitScheme::resolve_substep_count (split_explicit.cpp:67-170)."""
    if not (dt_large > 0.0 and math.isfinite(dt_large)):
        raise ValueError("split-explicit stepping requires a positive finite large timestep")
    if not (c_max > 0.0 and math.isfinite(c_max)):
        raise ValueError("split-explicit acoustic CFL needs a positive maximum sound speed")
    dx_min = min(dx, dy, dz)
    required = max(int(math.ceil(dt_large * c_max / (0.5 * dx_min))) + 1, 2)
    return max(requested, required) if requested > 0 else required


def perturbed_state(case: Case, amplitude: float = 1.0, seed: int = 1):
    """Initial state plus seeded velocity/pressure perturbations: a stressed
    input for single-kernel parity tests (every branch of the stencils fires)."""
    st, base = initial_state(case)
    rng = np.random.default_rng(seed)
    shape = case.shape
    for key, scale in (("u", 2.0), ("v", 2.0), ("w", 1.0)):
        st[key] = (st[key] + amplitude * scale * rng.uniform(-1, 1, shape)).astype(np.float32)
    st["p"] = (st["p"] * (1.0 + amplitude * 2e-4 * rng.uniform(-1, 1, shape))).astype(np.float32)
    st["qc"] = np.where(rng.uniform(0, 1, shape) < 0.3, amplitude * 1e-3 * rng.uniform(0, 1, shape), 0).astype(np.float32)
    st["qr"] = np.where(rng.uniform(0, 1, shape) < 0.2, amplitude * 5e-4 * rng.uniform(0, 1, shape), 0).astype(np.float32)
    return st, base


def cloudy_state(case: Case, seed: int = 1):
    """perturbed_state with vapour scattered +/-30 % around the sounding and
    cloud and rain in half of the cells: saturation adjustment, warm rain,
    evaporation and sedimentation all act somewhere in the grid."""
    st, base = perturbed_state(case, amplitude=1.0, seed=seed)
    rng = np.random.default_rng(seed)
    shape = case.shape
    st["qv"] = (st["qv"] * (1.0 + 0.3 * rng.uniform(-1, 1, shape))).astype(np.float32)
    st["qc"] = np.where(rng.uniform(0, 1, shape) < 0.5, 2e-3 * rng.uniform(0, 1, shape), 0).astype(np.float32)
    st["qr"] = np.where(rng.uniform(0, 1, shape) < 0.5, 3e-3 * rng.uniform(0, 1, shape), 0).astype(np.float32)
    return st, base


def benchmark_case(name: str) -> Case:
    """Named workloads (grid, dt, acoustic substeps)."""
    if name == "supercell_1km_64x64x40":
        return Case(64, 64, 40, 1000.0, 1000.0, 500.0, 6.0, substeps=6)
    if name == "supercell_250m_256x256x80":
        return Case(256, 256, 80, 250.0, 250.0, 250.0, 1.5, substeps=8, noise_amp=0.1, seed=2,
                    bubble_rh=2500.0, bubble_rz=350.0, bubble_zc=350.0)
    if name == "supercell_100m_512x512x128":
        return Case(512, 512, 128, 100.0, 100.0, 150.0, 0.6, substeps=10, noise_amp=0.1, seed=3,
                    bubble_rh=1000.0, bubble_rz=140.0, bubble_zc=140.0)
    raise KeyError(name)
