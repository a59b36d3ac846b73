"""Test infrastructure: ctypes access to the two CPU oracles of the hot path.

* ``Restatement("f32" | "f64")`` -- the C restatement in ``nimbus_oracle.c``
  (FP32 storage mirroring the reference CPU solver, or FP64 storage for the
  error statement).
* ``ReferenceHarness`` -- the reference Nimbus CPU solver itself, built from
  its own sources by ``oracle/ref.mk`` and driven through ``ref_harness.cpp``.

Only tests, the smoke check and bench.py's CPU-baseline leg use this package,
and only as the checker.  Nothing in ``nimbus_b200`` imports it.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
BUILD = ROOT / "_build"
REF = ROOT / "_ref"

_F = ctypes.POINTER(ctypes.c_float)
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


def _fp(a):
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    if a.dtype == np.float32:
        return _ptr(a, ctypes.c_float)
    if a.dtype == np.float64:
        return _ptr(a, ctypes.c_double)
    raise TypeError(a.dtype)


def _bcs(bc):
    arr = (ctypes.c_int * 6)(*[int(x) for x in bc])
    return arr


class Restatement:
    """The C restatement, compiled with FP32 ("f32") or FP64 ("f64") storage."""

    def __init__(self, precision: str = "f32"):
        assert precision in ("f32", "f64")
        self.precision = precision
        self.dtype = np.float32 if precision == "f32" else np.float64
        path = BUILD / f"liboracle_{precision}.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -f oracle/oracle.mk`")
        self.lib = ctypes.CDLL(str(path))
        self.lib.oracle_weno5_face.restype = ctypes.c_double
        self.lib.oracle_weno5_face.argtypes = [ctypes.c_double] * 5
        self.lib.oracle_mc_slope.restype = ctypes.c_double
        self.lib.oracle_mc_slope.argtypes = [ctypes.c_double] * 3
        self.lib.oracle_gamma.restype = ctypes.c_double
        assert self.lib.oracle_real_bytes() == np.dtype(self.dtype).itemsize

    def _chk(self, *arrs):
        for a in arrs:
            if a is not None:
                assert a.dtype == self.dtype and a.flags["C_CONTIGUOUS"], (a.dtype, self.dtype)

    def weno5_face(self, a, b, c, d, e):
        return self.lib.oracle_weno5_face(a, b, c, d, e)

    def mc_slope(self, qm, q0, qp):
        return self.lib.oracle_mc_slope(qm, q0, qp)

    def acoustic_fused(self, st, rho0, p0, dt_small, grid, drho=None):
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        self._chk(u, v, w, rho, p, th, drho)
        nx, ny, nz = u.shape
        self.lib.oracle_acoustic_fused(
            nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _fp(rho0), _fp(p0),
            ctypes.c_double(dt_small), _fp(drho) if drho is not None else None)

    def acoustic_loop(self, st, rho0, p0, dt_large, n_substeps, grid, bc, frame=(0.0, 0.0)):
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        self._chk(u, v, w, rho, p, th)
        nx, ny, nz = u.shape
        out = {k: np.zeros_like(u) for k in ("mfx", "mfy", "mfz", "rho_begin")}
        out["wave"] = np.zeros(2 * (nx + ny) * nz, self.dtype)
        rc = self.lib.oracle_acoustic_loop(
            nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _fp(rho0), _fp(p0),
            ctypes.c_double(dt_large), int(n_substeps), _bcs(bc), ctypes.c_double(frame[0]),
            ctypes.c_double(frame[1]), _fp(out["mfx"]), _fp(out["mfy"]), _fp(out["mfz"]),
            _fp(out["rho_begin"]), _fp(out["wave"]))
        if rc != 0:
            raise FloatingPointError("oracle mass-flux accumulation produced a non-finite flux")
        return out

    def slow_tendencies(self, st, base, grid, coriolis_f=0.0, moist=True, frame=(0.0, 0.0)):
        """(du, dv, dw, dp) of the slow operator at the given state."""
        u, v, w, rho, p = (st[k] for k in ("u", "v", "w", "rho", "p"))
        qv, qc, qr = _slow_inputs(st, base, moist)
        self._chk(u, v, w, rho, p, qv, qc, qr)
        nx, ny, nz = u.shape
        out = [np.zeros_like(u) for _ in range(4)]
        self.lib.oracle_slow_tendencies(
            nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _opt(qv), _opt(qc), _opt(qr), _fp(base["rho0"]),
            _fp(base["qv0"]) if moist else None, _fp(base["u0"]), _fp(base["v0"]), ctypes.c_double(coriolis_f),
            ctypes.c_double(frame[0]), ctypes.c_double(frame[1]), *[_fp(o) for o in out])
        return out

    def slow_rk2_step(self, st, base, grid, dt, coriolis_f=0.0, moist=True, frame=(0.0, 0.0)):
        """Heun slow step applied in place to u, v, w, p."""
        u, v, w, rho, p = (st[k] for k in ("u", "v", "w", "rho", "p"))
        qv, qc, qr = _slow_inputs(st, base, moist)
        self._chk(u, v, w, rho, p, qv, qc, qr)
        nx, ny, nz = u.shape
        rc = self.lib.oracle_slow_rk2_step(
            nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _opt(qv), _opt(qc), _opt(qr), _fp(base["rho0"]),
            _fp(base["qv0"]) if moist else None, _fp(base["u0"]), _fp(base["v0"]), ctypes.c_double(coriolis_f),
            ctypes.c_double(frame[0]), ctypes.c_double(frame[1]), ctypes.c_double(dt))
        if rc != 0:
            raise MemoryError("oracle slow-step scratch allocation failed")

    def acoustic_batched(self, st, rho0, p0, dt_small, n_substeps, grid, bc, backend, wave_in=None):
        """The acoustic loop as one AcousticSubstepsBatchedCartesianCgridDispatch
        (FP32 profiles, spacings and dt_small) through the ComputeBackend of
        the shared library at `backend`, in place; returns the mass fluxes and
        the KW78 history."""
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        nx, ny, nz = u.shape
        out = {k: np.zeros_like(u) for k in ("mfx", "mfy", "mfz")}
        out["wave"] = np.zeros(2 * (nx + ny) * nz, np.float32)
        bcs = (ctypes.c_int * 6)(*[int(x) for x in bc])
        self._rc(self.lib.ref_backend_acoustic_batched(
            str(backend).encode(), _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _fp(rho0), _fp(p0), nx, ny,
            nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            ctypes.c_double(dt_small), int(n_substeps), bcs, _fp(out["mfx"]), _fp(out["mfy"]), _fp(out["mfz"]),
            _opt(wave_in), _fp(out["wave"])))
        return out

    def kessler_tendencies(self, st, dz, dt, domain):
        th, p, rho, qv, qc, qr = (st[k] for k in ("theta", "p", "rho", "qv", "qc", "qr"))
        self._chk(th, p, rho, qv, qc, qr)
        nx, ny, nz = th.shape
        out = [np.zeros_like(th) for _ in range(4)]
        dom = (ctypes.c_int * 6)(*[int(x) for x in domain])
        self.lib.oracle_kessler_tendencies(nx, ny, nz, ctypes.c_double(dz), ctypes.c_double(dt), _fp(th), _fp(p),
                                           _fp(rho), _fp(qv), _fp(qc), _fp(qr), dom, *[_fp(o) for o in out])
        return out

    def kessler_step(self, st, dz, dt, domain):
        """Kessler tendencies, then their application in place (theta, qv, qc, qr)."""
        dth, dqv, dqc, dqr = self.kessler_tendencies(st, dz, dt, domain)
        nx, ny, nz = st["theta"].shape
        dom = (ctypes.c_int * 6)(*[int(x) for x in domain])
        self.lib.oracle_kessler_apply(nx, ny, nz, ctypes.c_double(dt), dom, _fp(st["theta"]), _fp(st["qv"]),
                                      _fp(st["qc"]), _fp(st["qr"]), _fp(dth), _fp(dqv), _fp(dqc), _fp(dqr))
        return dth, dqv, dqc, dqr

    def acoustic_boundaries(self, st, grid, bc, dt_small=0.0, wave=None, frame=(0.0, 0.0)):
        """apply_acoustic(dt_small) on u, v, w, rho, p in place (dt_small == 0:
        refresh only, no wave history needed)."""
        u, v, w, rho, p = (st[k] for k in ("u", "v", "w", "rho", "p"))
        self._chk(u, v, w, rho, p)
        nx, ny, nz = u.shape
        if wave is None:
            wave = np.zeros(2 * (nx + ny) * nz, self.dtype)
        self.lib.oracle_acoustic_bcs(nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), _fp(u), _fp(v),
                                     _fp(w), _fp(rho), _fp(p), _fp(wave), ctypes.c_double(dt_small), _bcs(bc),
                                     ctypes.c_double(frame[0]), ctypes.c_double(frame[1]))

    def large_step(self, st, base, grid, dt, n_substeps, bc, coriolis_f=0.0, microphysics=True, sponge=None,
                   final_closure=False, sgs=None, time_s=0.0):
        """One large step of the hot path in the reference's order
        (dynamics.cpp:5123-7317): Heun slow step, boundary refresh, the
        acoustic loop (KW78 seed, N substeps with retained mass flux),
        conservative WENO5 transport of theta, qv, qc, qr, the Kessler step
        over the C-grid cell domain and the EOS re-projection.  In place on
        the state dict; raises when the EOS projection refuses the state.
        sgs (a nimbus_b200.sgs.SgsConfig) adds the explicit Smagorinsky
        integration between the Kessler step and the EOS projection, as the
        reference orders them; time_s is the model time at the step start."""
        self.slow_rk2_step(st, base, grid, dt, coriolis_f=coriolis_f)
        self.acoustic_boundaries(st, grid, bc, 0.0)
        loop = self.acoustic_loop(st, base["rho0"], base["p0"], dt, n_substeps, grid, bc)
        qs = [st["theta"], st["qv"], st["qc"], st["qr"]]
        self.scalar_transport(qs, [0, 1, 1, 1], st["rho"], loop["rho_begin"], loop["mfx"], loop["mfy"], loop["mfz"],
                              dt, grid, weno=True, top_open=bc[5] == 2)
        nx, ny, nz = st["u"].shape
        if microphysics:
            self.kessler_step(st, grid[2], dt, (1, nx - 1, 1, ny - 1, 0, nz))
        if sgs is not None:  # the explicit SGS integration (dynamics.cpp:7151-7250)
            self.sgs_step(st, np.full(nz, grid[2]), grid, sgs, dt, theta0=base["theta0"], time_s=time_s)
        if not self.eos_projection(st["p"], st["rho"], st["theta"], st["qv"], st["qc"], st["qr"]):
            raise FloatingPointError("EOS pressure projection rejected an invalid physical state")
        if sponge is not None:
            self.state_relaxation(st, sponge, dt)
        if final_closure:  # apply_full_attributed (dynamics.cpp:7415) = apply_acoustic(0)
            self.acoustic_boundaries(st, grid, bc, 0.0)
        return loop

    def max_sound_speed(self, st, base):
        """Largest sqrt(gamma p / rho) over the state and the base columns
        (runtime.cpp:346-401, 854-870); raises on a non-finite or
        non-positive pressure or density, where the reference throws."""
        self._chk(st["p"], st["rho"])
        nx, ny, nz = st["p"].shape
        out = ctypes.c_double(0.0)
        p0 = np.ascontiguousarray(base["p0"], np.float64)
        rho0 = np.ascontiguousarray(base["rho0"], np.float64)
        if self.lib.oracle_max_sound_speed(nx, ny, nz, _fp(st["p"]), _fp(st["rho"]), _fp(p0), _fp(rho0),
                                           ctypes.byref(out)) != 0:
            raise ValueError("CFL scan requires finite wind and positive finite pressure/density")
        return out.value

    def resolve_substeps(self, dt, c_max, min_spacing, requested=0):
        """split_explicit.cpp:67-170 with a positive diagnosed spacing."""
        self.lib.oracle_resolve_substeps.argtypes = [ctypes.c_double, ctypes.c_double, ctypes.c_double, ctypes.c_int]
        n = self.lib.oracle_resolve_substeps(dt, c_max, min_spacing, int(requested))
        if n < 1:
            raise ValueError("split-explicit acoustic CFL cannot be resolved")
        return n

    def substeps(self, st, base, grid, dt, requested=0):
        """The substep count the reference uses for a large step from this state."""
        return self.resolve_substeps(dt, self.max_sound_speed(st, base), min(grid), requested)

    def run(self, st, base, grid, dt, steps, bc, requested=0, **kw):
        """`steps` large steps in place, the substep count re-derived from the
        state before each one as the reference does; returns the counts."""
        counts = []
        for _ in range(steps):
            n = self.substeps(st, base, grid, dt, requested)
            counts.append(n)
            self.large_step(st, base, grid, dt, n, bc, **kw)
        return counts

    def eos_projection(self, p, rho, theta, qv=None, qc=None, qr=None):
        """EOS pressure re-projection in place; returns False (p untouched)
        when the state is refused.  qv/qc/qr (all or none) add the moist-state
        checks of the attributed domain."""
        self._chk(p, rho, theta, qv, qc, qr)
        nx, ny, nz = p.shape
        return self.lib.oracle_eos_projection(nx, ny, nz, _fp(rho), _fp(theta), _fp(p), _opt(qv), _opt(qc),
                                              _opt(qr)) == 0

    def state_relaxation(self, st, profiles, dt):
        """The end-of-step sponge on st's u, v, w, theta in place
        (oracle_state_relaxation); profiles as nimbus_b200.sponge.SpongeProfiles."""
        u, v, w, th = (st[k] for k in ("u", "v", "w", "theta"))
        self._chk(u, v, w, th)
        nx, ny, nz = u.shape
        P = profiles
        d = lambda a: np.ascontiguousarray(a, dtype=np.float64)  # noqa: E731
        arrs = [d(P.theta_ref), d(P.alpha), d(P.upper_w_alpha), d(P.w_only_alpha), d(P.u_ref), d(P.v_ref)]
        lat = d(P.lateral_alpha) if len(P.lateral_alpha) else np.zeros(1)
        rc = self.lib.oracle_state_relaxation(
            nx, ny, nz, _fp(u), _fp(v), _fp(w), _fp(th), *[_fp(a) for a in arrs], int(len(P.lateral_alpha)), _fp(lat),
            int(P.do_upper), int(P.do_w_only), int(P.do_lateral), int(P.staggered), int(P.implicit_mode),
            ctypes.c_double(dt))
        if rc != 0:
            raise ValueError("state relaxation: invalid alpha or dt")

    def cell_centre(self, u, v, w, ground_w=None):
        """Cell-centre u, v, w of face fields (oracle_cell_centre); a None
        input skips that component (its output is None).  ground_w: the
        terrain lower-face w per column ([nx][ny] FP64) or None (flat)."""
        face = next(a for a in (u, v, w) if a is not None)
        self._chk(*[a for a in (u, v, w) if a is not None])
        nx, ny, nz = face.shape
        outs = [None if a is None else np.empty_like(a) for a in (u, v, w)]
        g = None if ground_w is None else np.ascontiguousarray(ground_w, dtype=np.float64)
        rc = self.lib.oracle_cell_centre(nx, ny, nz, *[_opt(a) for a in (u, v, w)], *[_opt(o) for o in outs],
                                         _opt(g))
        if rc != 0:
            raise ValueError("terrain lower-boundary velocity must contain only finite values")
        return tuple(outs)

    def smagorinsky(self, st, dz, grid, sgs):
        """The Smagorinsky producer (oracle_smagorinsky) on st's u, v, w,
        theta, rho and optional qv; dz: FP64 cell thickness per level; sgs: a
        nimbus_b200.sgs.SgsConfig.  Returns {nu_t, K_theta, K_q, dudt, dvdt,
        dwdt, dthdt, dqvdt}; raises ValueError where the reference throws."""
        u = st["u"]
        qv = st.get("qv")
        self._chk(u, st["v"], st["w"], st["theta"], st["rho"], qv)
        nx, ny, nz = u.shape
        dz = np.ascontiguousarray(dz, dtype=np.float64)
        delta = np.array([sgs_filter_width(sgs.filter_width, grid[0], grid[1], float(dz[k])) for k in range(nz)])
        out = {k: np.empty_like(u) for k in SGS_OUTPUTS}
        opened = (ctypes.c_int * 4)(*[int(x) for x in sgs.open_lateral])
        rc = self.lib.oracle_smagorinsky(
            nx, ny, nz, _fp(u), _fp(st["v"]), _fp(st["w"]), _fp(st["theta"]), _opt(qv), _fp(st["rho"]), _fp(dz),
            _fp(delta), ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), int(sgs.use_horizontal),
            int(sgs.use_vertical), int(sgs.periodic_x), int(sgs.periodic_y), opened, ctypes.c_double(sgs.Cs),
            ctypes.c_double(sgs.Pr_t), ctypes.c_double(sgs.Sc_t), ctypes.c_double(sgs.nu_t_max),
            ctypes.c_double(sgs.K_max), *[_fp(out[k]) for k in SGS_OUTPUTS])
        if rc == -2:
            raise ValueError("turbulence field violates its finite physical domain")
        if rc != 0:
            raise ValueError("Smagorinsky coefficient is not finite")
        return out

    def sgs_apply(self, st, rates, dt, theta0=None, repairs=True, theta_ref=300.0):
        """Forward-Euler SGS application in place on st's u, v, w, theta and
        optional qv (oracle_sgs_apply); rates as smagorinsky() returns."""
        u = st["u"]
        qv = st.get("qv")
        nx, ny, nz = u.shape
        t0 = None if theta0 is None else np.ascontiguousarray(theta0, dtype=np.float64)
        self.lib.oracle_sgs_apply(
            nx, ny, nz, _fp(u), _fp(st["v"]), _fp(st["w"]), _fp(st["theta"]), _opt(qv), None,
            _fp(rates["dudt"]), _fp(rates["dvdt"]), _fp(rates["dwdt"]), _fp(rates["dthdt"]),
            _opt(rates["dqvdt"] if qv is not None else None), None, None, _opt(t0), ctypes.c_double(dt),
            int(bool(repairs)), ctypes.c_double(theta_ref), ctypes.c_float(200.0), ctypes.c_float(700.0),
            ctypes.c_float(0.05), ctypes.c_float(180.0), ctypes.c_float(120.0))

    def sgs_stability(self, st, rates, grid, dz, sgs):
        """oracle_sgs_stability (periodic or closed lateral faces only): the
        same dict as ReferenceHarness.sgs_stability."""
        u = st["u"]
        qv = st.get("qv")
        nx, ny, nz = u.shape
        out = np.zeros(5)
        rc = self.lib.oracle_sgs_stability(
            nx, ny, nz, _fp(u), _fp(st["v"]), _fp(st["w"]), _fp(st["theta"]), _opt(qv), _fp(st["rho"]),
            _fp(rates["dudt"]), _fp(rates["dvdt"]), _fp(rates["dwdt"]), _fp(rates["dthdt"]),
            _opt(rates["dqvdt"] if qv is not None else None), ctypes.c_double(grid[0]), ctypes.c_double(grid[1]),
            _fp(np.ascontiguousarray(dz, dtype=np.float64)), int(sgs.periodic_x), int(sgs.periodic_y), _fp(out))
        if rc == -2:
            raise ValueError("SGS stability evaluation requires a finite, positive state")
        if rc != 0:
            raise ValueError("realized SGS tendency has no positive stable timestep")
        return dict(zip(("maximum", "momentum_energy", "theta_monotonic", "qv_monotonic", "dissipation_w"), out))

    def sgs_step(self, st, dz, grid, sgs, dt, theta0=None, time_s=0.0, repairs=True):
        """The explicit SGS integration of one large step in place
        (dynamics.cpp:7159-7217): refresh the closure, bound the substep by
        the stability limit and dt_sgs, apply; returns (substeps, smallest
        limit)."""
        import sys
        eps = sys.float_info.epsilon
        floor_s = 64.0 * eps * max(1.0, dt, abs(time_s))
        advanced, seen, count = 0.0, float("inf"), 0
        while advanced < dt:
            rates = self.smagorinsky(st, dz, grid, sgs)
            limit = self.sgs_stability(st, rates, grid, dz, sgs)["maximum"]
            seen = min(seen, limit)
            sub = min(dt - advanced, sgs.dt_sgs, limit)
            count += 1
            if not np.isfinite(sub) or sub <= floor_s:
                raise ValueError("SGS explicit integration cannot make stable progress")
            self.sgs_apply(st, rates, sub, theta0=theta0, repairs=repairs)
            advanced += sub
            if dt - advanced <= floor_s:
                advanced = dt
        return count, seen

    def scalar_transport(self, qs, pd, rho_end, rho_begin, mfx, mfy, mfz, dt, grid, weno=True, top_open=False):
        self._chk(rho_end, rho_begin, mfx, mfy, mfz, *qs)
        nx, ny, nz = rho_end.shape
        n = len(qs)
        ctype = ctypes.c_float if self.dtype == np.float32 else ctypes.c_double
        arr = (ctypes.POINTER(ctype) * max(n, 1))(*[_ptr(q, ctype) for q in qs])
        flags = (ctypes.c_int * max(n, 1))(*[int(x) for x in pd])
        rc = self.lib.oracle_scalar_transport(
            nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            arr, flags, n, _fp(rho_end), _fp(rho_begin), _fp(mfx), _fp(mfy), _fp(mfz),
            ctypes.c_double(dt), int(weno), int(top_open))
        if rc != 0:
            raise MemoryError("oracle transport scratch allocation failed")


def _opt(a):
    return None if a is None else _fp(a)


SGS_OUTPUTS = ("nu_t", "K_theta", "K_q", "dudt", "dvdt", "dwdt", "dthdt", "dqvdt")
SGS_MODES = {(1, 1): 0, (1, 0): 1, (0, 1): 2}


def sgs_filter_width(kind: str, dx: float, dy: float, dz: float) -> float:
    """compute_filter_width (src/turbulence/base/eddy_viscosity.cpp:1414-1468),
    flat grid: sqrt(dx dy) for "dx", cbrt(dx dy dz) for "cubic_root"
    (math.sqrt / math.cbrt are the C library's, as in the reference)."""
    import math
    if kind == "dx":
        return math.sqrt(dx * dy)
    if kind == "cubic_root":
        return math.cbrt(dx * dy * dz)
    raise ValueError(kind)


def npy_header(shape, descr: str = "<f4") -> bytes:
    """The header npy::write_3d / write_2d write (src/core/output/npy_writer.cpp:27-118):
    magic, version 1.0, a little-endian uint16 header length, the dict
    "{'descr': '<f4', 'fortran_order': False, 'shape': (a, b, c), }" padded
    with spaces so that the preamble, dict and newline end on a 16-byte
    boundary."""
    dims = ", ".join(str(int(x)) for x in shape) + ("," if len(shape) == 1 else "")
    head = "{'descr': '" + descr + "', 'fortran_order': False, 'shape': (" + dims + "), }"
    pad = (16 - (10 + len(head) + 1) % 16) % 16
    body = (head + " " * pad + "\n").encode("ascii")
    return b"\x93NUMPY\x01\x00" + len(body).to_bytes(2, "little") + body


def npy_bytes(data) -> bytes:
    """The whole file the reference's writer produces for a float32 (or
    float64) array: npy_header, then the C-order little-endian payload."""
    a = np.ascontiguousarray(data)
    descr = {np.dtype(np.float32): "<f4", np.dtype(np.float64): "<f8"}[a.dtype]
    return npy_header(a.shape, descr) + a.astype(a.dtype.newbyteorder("<")).tobytes()


def _slow_inputs(st, base, moist=True):
    qv = st.get("qv") if moist else None
    qc = st.get("qc") if moist else None
    qr = st.get("qr") if moist else None
    return qv, qc, qr


class ReferenceHarness:
    """The reference CPU solver's own objects behind ``ref_harness.cpp``."""

    def __init__(self, threads: int | None = None):
        path = REF / "libnimbus_ref_harness.so"
        if not path.exists():
            raise FileNotFoundError(f"{path} missing: run `make -f oracle/ref.mk all harness`")
        self.lib = ctypes.CDLL(str(path))
        self.lib.ref_last_error.restype = ctypes.c_char_p
        self.threads = self.lib.ref_set_threads(int(threads or 0))

    def set_threads(self, n):
        self.threads = self.lib.ref_set_threads(int(n))
        return self.threads

    def _rc(self, rc):
        if rc != 0:
            raise RuntimeError(self.lib.ref_last_error().decode())

    def acoustic_fused(self, st, rho0, p0, dt_small, grid, drho=None, backend=None):
        """One fused substep through a ComputeBackend: the reference's CPU
        backend, or the one a shared library's nimbus_cuda_create_compute_backend
        makes (backend: its path)."""
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        nx, ny, nz = u.shape
        scratch = drho if drho is not None else np.zeros_like(u)
        lib_path = None if backend is None else str(backend).encode()
        self._rc(self.lib.ref_backend_acoustic_fused(
            lib_path, _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _fp(rho0), _fp(p0), nx, ny, nz,
            ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            ctypes.c_double(dt_small), _fp(scratch)))

    def acoustic_loop(self, st, rho0, p0, dt_large, n_substeps, grid, bc):
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        nx, ny, nz = u.shape
        out = {k: np.zeros_like(u) for k in ("mfx", "mfy", "mfz", "rho_begin")}
        out["wave"] = np.zeros(2 * (nx + ny) * nz, np.float32)
        self._rc(self.lib.ref_acoustic_loop(
            _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _fp(rho0), _fp(p0), nx, ny, nz,
            ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            ctypes.c_double(dt_large), int(n_substeps), *[int(x) for x in bc],
            _fp(out["mfx"]), _fp(out["mfy"]), _fp(out["mfz"]), _fp(out["rho_begin"]), _fp(out["wave"])))
        return out

    def acoustic_batched(self, st, rho0, p0, dt_small, n_substeps, grid, bc, backend, wave_in=None):
        """The acoustic loop as one AcousticSubstepsBatchedCartesianCgridDispatch
        (FP32 profiles, spacings and dt_small) through the ComputeBackend of
        the shared library at `backend`, in place; returns the mass fluxes and
        the KW78 history."""
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        nx, ny, nz = u.shape
        out = {k: np.zeros_like(u) for k in ("mfx", "mfy", "mfz")}
        out["wave"] = np.zeros(2 * (nx + ny) * nz, np.float32)
        bcs = (ctypes.c_int * 6)(*[int(x) for x in bc])
        self._rc(self.lib.ref_backend_acoustic_batched(
            str(backend).encode(), _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _fp(rho0), _fp(p0), nx, ny,
            nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]),
            ctypes.c_double(dt_small), int(n_substeps), bcs, _fp(out["mfx"]), _fp(out["mfy"]), _fp(out["mfz"]),
            _opt(wave_in), _fp(out["wave"])))
        return out

    def kessler_tendencies(self, st, dz, dt, domain, backend=None):
        """KesslerScheme::compute_tendencies: the CPU route, or (backend: a
        shared library's path) the device route through that library's
        ComputeBackend (the pointwise and sedimentation dispatches)."""
        th, p, rho, qv, qc, qr = (st[k] for k in ("theta", "p", "rho", "qv", "qc", "qr"))
        nx, ny, nz = th.shape
        out = [np.zeros_like(th) for _ in range(4)]
        dom = (ctypes.c_int * 6)(*[int(x) for x in domain])
        lib = str(backend).encode() if backend is not None else None
        self._rc(self.lib.ref_backend_kessler_tendencies(lib, _fp(th), _fp(p), _fp(rho), _fp(qv), _fp(qc), _fp(qr),
                                                         nx, ny, nz, ctypes.c_double(dz), ctypes.c_double(dt), dom,
                                                         *[_fp(o) for o in out]))
        return out

    def acoustic_boundaries(self, st, grid, bc, dt_small=0.0):
        """apply_acoustic(dt_small) on u, v, w, rho, p in place."""
        u, v, w, rho, p = (st[k] for k in ("u", "v", "w", "rho", "p"))
        nx, ny, nz = u.shape
        self._rc(self.lib.ref_acoustic_boundaries(_fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), nx, ny, nz,
                                                  ctypes.c_double(grid[0]), ctypes.c_double(grid[1]),
                                                  ctypes.c_double(grid[2]), ctypes.c_double(dt_small),
                                                  *[int(x) for x in bc]))

    def eos_projection(self, p, rho, theta, grid, qv=None, qc=None, qr=None):
        """apply_pressure_projection on p in place; False when refused."""
        nx, ny, nz = p.shape
        rc = self.lib.ref_eos_projection(_fp(rho), _fp(theta), _fp(p), _opt(qv), _opt(qc), _opt(qr), nx, ny, nz,
                                         ctypes.c_double(grid[0]), ctypes.c_double(grid[1]),
                                         ctypes.c_double(grid[2]))
        if rc < 0:
            self._rc(rc)
        return rc == 0

    def state_relaxation(self, st, theta0, grid, dt, config):
        """apply_rayleigh_damping then apply_lateral_damping on st's u, v, w,
        theta in place, configured from a nimbus_b200.sponge.SpongeConfig;
        returns the reference runtime's own profiles
        (alpha, upper_w_alpha, w_only_alpha, u_ref, v_ref, lateral_alpha)."""
        u, v, w, th = (st[k] for k in ("u", "v", "w", "theta"))
        nx, ny, nz = u.shape
        c = config
        out = [np.zeros(nz) for _ in range(5)] + [np.zeros(max(c.lateral_width, 1))]
        wind = (ctypes.c_double * 6)(*[float(x) for x in c.wind])
        self._rc(self.lib.ref_state_relaxation(
            _fp(u), _fp(v), _fp(w), _fp(th), _fp(np.ascontiguousarray(theta0, dtype=np.float64)), nx, ny, nz,
            ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]), ctypes.c_double(dt),
            ctypes.c_double(c.z_damp), ctypes.c_double(c.alpha_max), int(c.w_only_cells),
            ctypes.c_double(c.w_only_alpha_max), int(c.lateral_width), ctypes.c_double(c.lateral_alpha_max),
            int(c.implicit_mode), wind, *[_fp(o) for o in out]))
        names = ("alpha", "upper_w_alpha", "w_only_alpha", "u_ref", "v_ref", "lateral_alpha")
        prof = dict(zip(names, out))
        prof["lateral_alpha"] = prof["lateral_alpha"][:c.lateral_width]
        return prof

    def cell_centre(self, u, v, w, ground_w=None):
        """interpolate_u/v/w_face_to_center on face fields; a None input
        skips that component.  A non-finite ground_w raises (the reference's
        invalid_argument)."""
        face = next(a for a in (u, v, w) if a is not None)
        nx, ny, nz = face.shape
        outs = [None if a is None else np.empty_like(a) for a in (u, v, w)]
        g = None if ground_w is None else np.ascontiguousarray(ground_w, dtype=np.float64)
        self._rc(self.lib.ref_cell_centre(*[_opt(a) for a in (u, v, w)], *[_opt(o) for o in outs], _opt(g),
                                          nx, ny, nz))
        return tuple(outs)

    def npy_write_3d(self, data, path):
        """npy::write_3d of a float32 [d0][d1][d2] array to path."""
        a = np.ascontiguousarray(data, dtype=np.float32)
        self._rc(self.lib.ref_npy_write_3d(_fp(a), *[int(x) for x in a.shape], str(path).encode()))

    def smagorinsky(self, st, dz, grid, sgs, backend=None):
        """SmagorinskyScheme::compute on the flat C-grid: the CPU path, or
        (backend: a shared library's path) the scheme's native path through
        that library's ComputeBackend.  Same outputs as Restatement.smagorinsky."""
        u = st["u"]
        qv = st.get("qv")
        nx, ny, nz = u.shape
        out = {k: np.empty_like(u) for k in SGS_OUTPUTS}
        opened = (ctypes.c_int * 4)(*[int(x) for x in sgs.open_lateral])
        lib_path = None if backend is None else str(backend).encode()
        self._rc(self.lib.ref_backend_smagorinsky(
            lib_path, _fp(u), _fp(st["v"]), _fp(st["w"]), _fp(st["theta"]), _opt(qv), _fp(st["rho"]),
            _fp(np.ascontiguousarray(dz, dtype=np.float64)), nx, ny, nz, ctypes.c_double(grid[0]),
            ctypes.c_double(grid[1]), SGS_MODES[(int(sgs.use_horizontal), int(sgs.use_vertical))],
            int(sgs.filter_width == "dx"), int(sgs.periodic_x), int(sgs.periodic_y), opened,
            ctypes.c_double(sgs.Cs), ctypes.c_double(sgs.Pr_t), ctypes.c_double(sgs.Sc_t),
            ctypes.c_double(sgs.nu_t_max), ctypes.c_double(sgs.K_max), *[_fp(out[k]) for k in SGS_OUTPUTS]))
        return out

    def sgs_apply(self, st, rates, dt, theta0=None, repairs=True):
        """apply_admitted_sgs_substep (CPU path) in place on st's u, v, w,
        theta and optional qv."""
        u = st["u"]
        qv = st.get("qv")
        nx, ny, nz = u.shape
        t0 = None if theta0 is None else np.ascontiguousarray(theta0, dtype=np.float64)
        self._rc(self.lib.ref_sgs_apply(
            _fp(u), _fp(st["v"]), _fp(st["w"]), _fp(st["theta"]), _opt(qv), _fp(rates["dudt"]),
            _fp(rates["dvdt"]), _fp(rates["dwdt"]), _fp(rates["dthdt"]),
            _opt(rates["dqvdt"] if qv is not None else None), _opt(t0), nx, ny, nz, ctypes.c_double(dt),
            int(bool(repairs))))

    def sgs_stability(self, st, rates, grid, bc, sgs):
        """compute_sgs_explicit_stability with deterministic reductions:
        {maximum, momentum_energy, theta_monotonic, qv_monotonic,
        dissipation_w}."""
        u = st["u"]
        qv = st.get("qv")
        nx, ny, nz = u.shape
        out = np.zeros(5)
        bcs = (ctypes.c_int * 6)(*[int(x) for x in bc])
        self._rc(self.lib.ref_sgs_stability(
            _fp(u), _fp(st["v"]), _fp(st["w"]), _fp(st["theta"]), _opt(qv), _fp(st["rho"]), _fp(rates["dudt"]),
            _fp(rates["dvdt"]), _fp(rates["dwdt"]), _fp(rates["dthdt"]),
            _opt(rates["dqvdt"] if qv is not None else None), nx, ny, nz, ctypes.c_double(grid[0]),
            ctypes.c_double(grid[1]), ctypes.c_double(grid[2]), bcs,
            SGS_MODES[(int(sgs.use_horizontal), int(sgs.use_vertical))], _fp(out)))
        return dict(zip(("maximum", "momentum_energy", "theta_monotonic", "qv_monotonic", "dissipation_w"), out))

    def large_step(self, st, base, grid, dt, n_substeps, bc, coriolis_f=0.0):
        """One large step of the hot path from the reference's own objects:
        slow tendencies (k1, k2), boundary refresh, acoustic loop, transport,
        Kessler tendencies and the EOS projection are the reference's calls;
        the pointwise Heun combination and the microphysics commit between
        them are written out here with the reference's rounding
        (dynamics.cpp:1955-2408, microphysics_step.cpp:3026-3245)."""
        f32, f64 = np.float32, np.float64

        def apply(x, t):
            t64 = np.where(np.isfinite(t), t, 0).astype(f64)
            return (x.astype(f64) + t64 * dt).astype(f32)

        keys = ("u", "v", "w", "p")
        k1 = self.slow_tendencies(st, base, grid, coriolis_f)
        star = dict(st)
        for key, t in zip(keys, k1):
            star[key] = apply(st[key], t)
        k2 = self.slow_tendencies(star, base, grid, coriolis_f)
        for key, a, b in zip(keys, k1, k2):
            st[key][...] = apply(st[key], f32(0.5) * (b + a))
        self.acoustic_boundaries(st, grid, bc, 0.0)
        loop = self.acoustic_loop(st, base["rho0"], base["p0"], dt, n_substeps, grid, bc)
        qs = [st["theta"], st["qv"], st["qc"], st["qr"]]
        self.scalar_transport(qs, [0, 1, 1, 1], st["u"], st["v"], st["w"], st["rho"], loop["rho_begin"],
                              loop["mfx"], loop["mfy"], loop["mfz"], dt, grid, top_open=bc[5] == 2)
        nx, ny, nz = st["u"].shape
        dth, dqv, dqc, dqr = self.kessler_tendencies(st, grid[2], dt, (1, nx - 1, 1, ny - 1, 0, nz))
        sl = (slice(1, nx - 1), slice(1, ny - 1), slice(None))
        with np.errstate(invalid="ignore", over="ignore"):
            for key, d in (("qv", dqv), ("qc", dqc), ("qr", dqr)):
                q = st[key][sl]
                raw = (q.astype(f64) + np.where(np.isfinite(d[sl]), d[sl], 0).astype(f64) * dt).astype(f32)
                st[key][sl] = np.where(np.isfinite(raw), np.clip(raw, f32(0), f32(0.05)), f32(0))
            told = st["theta"][sl].astype(f64)
            total = np.where(np.isfinite(dth[sl]), dth[sl], 0).astype(f64) * dt
            total = np.where(np.isfinite(total), total, 0.0)
            tn = told + np.clip(total, -50.0, 50.0)
            tn = np.where(np.isfinite(tn), tn, np.where(np.isfinite(told), told, 300.0))
            stored = tn.astype(f32)
            st["theta"][sl] = np.where(np.isfinite(stored), np.clip(stored, f32(200), f32(700)), f32(300))
        if not self.eos_projection(st["p"], st["rho"], st["theta"], grid, st["qv"], st["qc"], st["qr"]):
            raise FloatingPointError("EOS pressure projection rejected an invalid physical state")
        return loop

    def max_sound_speed(self, st, base, grid, dt):
        """(c_max, min spacing) that choose_runtime_timestep (runtime.cpp:712-880)
        hands the split-explicit scheme for this state."""
        nx, ny, nz = st["p"].shape
        out = np.zeros(2, np.float64)
        self._rc(self.lib.ref_max_sound_speed(
            _fp(st["u"]), _fp(st["v"]), _fp(st["w"]), _fp(st["rho"]), _fp(st["p"]), nx, ny, nz,
            ctypes.c_double(grid[0]), ctypes.c_double(grid[1]), ctypes.c_double(grid[2]), ctypes.c_double(dt),
            _fp(np.ascontiguousarray(base["rho0"], np.float64)), _fp(np.ascontiguousarray(base["p0"], np.float64)),
            _fp(out)))
        return float(out[0]), float(out[1])

    def resolve_substep_count(self, dt, c_max, min_spacing, requested=0):
        """SplitExplicitScheme::resolve_substep_count (split_explicit.cpp:67-170)."""
        n = ctypes.c_int(0)
        self._rc(self.lib.ref_resolve_substep_count(ctypes.c_double(dt), ctypes.c_double(c_max),
                                                    ctypes.c_double(min_spacing), int(requested), ctypes.byref(n)))
        return n.value

    def substeps(self, st, base, grid, dt, requested=0):
        c, spacing = self.max_sound_speed(st, base, grid, dt)
        return self.resolve_substep_count(dt, c, spacing, requested)

    def run(self, st, base, grid, dt, steps, bc, requested=0, coriolis_f=0.0):
        """`steps` large steps in place with the substep count re-derived
        before each one; returns the counts."""
        counts = []
        for _ in range(steps):
            n = self.substeps(st, base, grid, dt, requested)
            counts.append(n)
            self.large_step(st, base, grid, dt, n, bc, coriolis_f=coriolis_f)
        return counts

    def slow_tendencies(self, st, base, grid, coriolis_f=0.0, moist=True, beta=0.0, backend=None):
        """CartesianCGrid3DScheme::compute_slow_tendencies: the CPU route, or
        (backend: a shared library's path) the scheme's device route through
        that library's ComputeBackend.  Returns du, dv, dw, dp."""
        u, v, w, rho, p, th = (st[k] for k in ("u", "v", "w", "rho", "p", "theta"))
        qv, qc, qr = _slow_inputs(st, base, moist)
        nx, ny, nz = u.shape
        out = [np.zeros_like(u) for _ in range(4)]
        lib = str(backend).encode() if backend is not None else None
        self._rc(self.lib.ref_backend_slow_tendencies(
            lib, _fp(u), _fp(v), _fp(w), _fp(rho), _fp(p), _fp(th), _opt(qv), _opt(qc), _opt(qr), _fp(base["rho0"]),
            _fp(base["p0"]), _fp(base["qv0"]) if moist else None, _fp(base["u0"]), _fp(base["v0"]),
            _fp(base["theta0"]), nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]),
            ctypes.c_double(grid[2]), ctypes.c_double(coriolis_f), ctypes.c_double(beta), *[_fp(o) for o in out]))
        return out

    def scalar_transport(self, qs, pd, u, v, w, rho_end, rho_begin, mfx, mfy, mfz, dt, grid,
                         weno=True, top_open=False):
        nx, ny, nz = rho_end.shape
        n = len(qs)
        arr = (_F * max(n, 1))(*[_ptr(q, ctypes.c_float) for q in qs])
        flags = (ctypes.c_int * max(n, 1))(*[int(x) for x in pd])
        self._rc(self.lib.ref_scalar_transport(
            arr, flags, n, _fp(u), _fp(v), _fp(w), _fp(rho_end), _fp(rho_begin), _fp(mfx), _fp(mfy),
            _fp(mfz), nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]),
            ctypes.c_double(grid[2]), ctypes.c_double(dt), int(weno), int(top_open)))


    def bridge_scalar_transport(self, qs, pd, u, v, w, rho_end, rho_begin, mfx, mfy, mfz, dt, grid,
                                weno=True, top_open=False, backend=None):
        """The transport through the reference's bridge
        dispatch_advect_scalars_conservative_cartesian_cgrid_backend to the
        CPU backend (backend=None) or a shared library's ComputeBackend, with
        the arguments advection_batch.cpp passes; in place.  Returns False when
        the backend declined the dispatch (fields untouched)."""
        nx, ny, nz = rho_end.shape
        n = len(qs)
        arr = (_F * max(n, 1))(*[_ptr(q, ctypes.c_float) for q in qs])
        flags = (ctypes.c_int * max(n, 1))(*[int(x) for x in pd])
        lib = str(backend).encode() if backend is not None else None
        rc = self.lib.ref_backend_scalar_transport(
            lib, arr, flags, n, _fp(u), _fp(v), _fp(w), _fp(rho_end), _fp(rho_begin), _fp(mfx), _fp(mfy),
            _fp(mfz), nx, ny, nz, ctypes.c_double(grid[0]), ctypes.c_double(grid[1]),
            ctypes.c_double(grid[2]), ctypes.c_double(dt), int(weno), int(top_open))
        if rc == 1:
            return False
        self._rc(rc)
        return True


    def bridge_slow_apply(self, st, tend, dt, pbl=None, sanitize=True, observed=False, backend=None):
        """apply through the reference's bridge dispatch_slow_apply_backend to
        `backend` (a shared library; None: the CPU backend, which declines it);
        in place on st's u, v, w, p.  Returns (False, None) when declined,
        else (True, the committed fields the observer saw or None)."""
        u, v, w, p = (st[k] for k in ("u", "v", "w", "p"))
        nx, ny, nz = u.shape
        outs = [np.zeros_like(u) for _ in range(4)] if observed else [None] * 4
        calls = ctypes.c_int(0)
        lib = str(backend).encode() if backend is not None else None
        du_pbl, dv_pbl = (pbl if pbl is not None else (None, None))
        rc = self.lib.ref_backend_slow_apply(
            lib, _fp(u), _fp(v), _fp(w), _fp(p), *[_fp(t) for t in tend], _opt(du_pbl), _opt(dv_pbl), nx, ny, nz,
            ctypes.c_float(dt), int(sanitize), int(observed), *[_opt(o) for o in outs], ctypes.byref(calls))
        if rc == 1:
            return False, None
        self._rc(rc)
        return True, (dict(zip("uvwp", outs)) if observed else None, calls.value)

    def bridge_state_relaxation(self, st, profiles_block, lateral_width, flags, dt, backend=None):
        """the sponge through dispatch_state_relaxation_cartesian_backend with a
        packed FP32 profile block (7 rows of nz) and a completion observer;
        in place.  Returns False when declined, else the observer's call count."""
        u, v, w, th = (st[k] for k in ("u", "v", "w", "theta"))
        nx, ny, nz = u.shape
        calls = ctypes.c_int(0)
        lib = str(backend).encode() if backend is not None else None
        rc = self.lib.ref_backend_state_relaxation(
            lib, _fp(u), _fp(v), _fp(w), _fp(th), _fp(np.ascontiguousarray(profiles_block, np.float32)), nx, ny, nz,
            int(lateral_width), *[int(bool(x)) for x in flags], ctypes.c_float(dt), ctypes.byref(calls))
        if rc == 1:
            return False
        self._rc(rc)
        return calls.value


def reference_available() -> bool:
    return (REF / "libnimbus_ref_harness.so").exists()


def restatement_available() -> bool:
    return (BUILD / "liboracle_f32.so").exists() and (BUILD / "liboracle_f64.so").exists()
