"""Generates the golden fixtures in tests/golden/ from the reference Nimbus CPU
solver itself (its own sources, built by oracle/ref.mk and driven through
oracle/ref_harness.cpp).

    make -f oracle/ref.mk -j8 all harness
    python tests/golden/make_golden.py

Each fixture is one .npz holding the seeded inputs and the reference's
outputs for a small grid, so the parity tests can pin the oracle restatement
and the CUDA path without the reference tree present.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))

from nimbus_b200.initial import Case, cloudy_state, perturbed_state  # noqa: E402
from oracle import ReferenceHarness  # noqa: E402

GRID = (1000.0, 1000.0, 500.0)

# (name, lateral W,E,S,N, bottom, top)
BC_SETS = {
    "radiative_slip_rigidlid": (1, 1, 1, 1, 1, 0),
    "periodic_noslip_open": (0, 0, 0, 0, 0, 2),
    "mixed_walls_sponge": (2, 3, 4, 1, 1, 1),
}


def close_walls(st, bc):
    """Zero-time wall closure so a rigid wall starts impermeable (the solver
    applies its boundary conditions before the first step)."""
    u, v = st["u"], st["v"]
    if bc[0] in (2, 3):
        u[0] = 0.0
    if bc[1] in (2, 3):
        u[-2] = 0.0
        u[-1] = 0.0
    if bc[2] in (2, 3):
        v[:, 0] = 0.0
    if bc[3] in (2, 3):
        v[:, -2] = 0.0
        v[:, -1] = 0.0


def main():
    ref = ReferenceHarness(threads=1)
    case = Case(14, 12, 9, *GRID, 6.0, seed=5)
    st, base = perturbed_state(case, seed=11)

    # 1. One fused substep.
    inp = {k: v.copy() for k, v in st.items()}
    out = {k: v.copy() for k, v in st.items()}
    drho = np.zeros(case.shape, np.float32)
    ref.acoustic_fused(out, base["rho0"], base["p0"], 0.6, GRID, drho)
    np.savez_compressed(HERE / "fused_substep.npz", grid=np.array(GRID), dt_small=0.6, rho0=base["rho0"],
                        p0=base["p0"], **{f"in_{k}": v for k, v in inp.items()},
                        **{f"out_{k}": out[k] for k in ("u", "v", "w", "rho", "p")}, out_drho=drho)

    # 2. Acoustic loop + 3. transport, per boundary set.
    for name, bc in BC_SETS.items():
        st2 = {k: v.copy() for k, v in st.items()}
        close_walls(st2, bc)
        inp = {k: v.copy() for k, v in st2.items()}
        n_sub, dt_large = 7, 6.0
        loop = ref.acoustic_loop(st2, base["rho0"], base["p0"], dt_large, n_sub, GRID, bc)
        top_open = bc[5] == 2
        scalars = {}
        for weno in (1, 0):
            qs = [st2["theta"].copy(), st2["qv"].copy(), st2["qc"].copy(), st2["qr"].copy()]
            ref.scalar_transport(qs, [0, 1, 1, 1], st2["u"], st2["v"], st2["w"], st2["rho"], loop["rho_begin"],
                                 loop["mfx"], loop["mfy"], loop["mfz"], dt_large, GRID, weno=bool(weno),
                                 top_open=top_open)
            for key, q in zip(("theta", "qv", "qc", "qr"), qs):
                scalars[f"tr{'weno' if weno else 'mc'}_{key}"] = q
        np.savez_compressed(
            HERE / f"loop_{name}.npz", grid=np.array(GRID), dt_large=dt_large, n_substeps=n_sub, bc=np.array(bc),
            rho0=base["rho0"], p0=base["p0"], **{f"in_{k}": v for k, v in inp.items()},
            **{f"out_{k}": st2[k] for k in ("u", "v", "w", "rho", "p")},
            **{f"out_{k}": v for k, v in loop.items()}, **scalars)
        print("wrote", name)

    # 4. Slow tendencies of the reference's C-grid scheme (moist, with Coriolis).
    sc = Case(17, 14, 12, 800.0, 700.0, 400.0, 4.0, seed=6)
    ss, sb = perturbed_state(sc, seed=12)
    outs = ref.slow_tendencies(ss, sb, (800.0, 700.0, 400.0), coriolis_f=1e-4, moist=True)
    dry = ref.slow_tendencies(ss, sb, (800.0, 700.0, 400.0), coriolis_f=0.0, moist=False)
    np.savez_compressed(HERE / "slow_tendencies.npz", grid=np.array((800.0, 700.0, 400.0)), coriolis_f=1e-4,
                        **{f"in_{k}": v for k, v in ss.items()}, **{f"base_{k}": v for k, v in sb.items()},
                        **{f"out_{k}": o for k, o in zip(("du", "dv", "dw", "dp"), outs)},
                        **{f"dry_{k}": o for k, o in zip(("du", "dv", "dw", "dp"), dry)})
    print("wrote slow_tendencies")

    # 5. Kessler tendencies on a cloudy state (C-grid cell domain and the full
    #    grid), and the EOS re-projection of that state, dry and moist.
    kc = Case(15, 13, 20, 1000.0, 1000.0, 500.0, 6.0, seed=3)
    ks, _ = cloudy_state(kc, seed=3)
    kdom = {"cgrid": (1, 14, 1, 12, 0, 20), "full": (0, 15, 0, 13, 0, 20)}
    kout = {}
    for name, dom in kdom.items():
        for key, o in zip(("dtheta", "dqv", "dqc", "dqr"), ref.kessler_tendencies(ks, 500.0, 6.0, dom)):
            kout[f"{name}_{key}"] = o
    p_dry, p_moist = ks["p"].copy(), ks["p"].copy()
    assert ref.eos_projection(p_dry, ks["rho"], ks["theta"], (kc.dx, kc.dy, kc.dz))
    assert ref.eos_projection(p_moist, ks["rho"], ks["theta"], (kc.dx, kc.dy, kc.dz), ks["qv"], ks["qc"], ks["qr"])
    np.savez_compressed(HERE / "kessler_eos.npz", dz=500.0, dt=6.0, grid=np.array((kc.dx, kc.dy, kc.dz)),
                        **{f"dom_{k}": np.array(v) for k, v in kdom.items()},
                        **{f"in_{k}": ks[k] for k in ("theta", "qv", "qc", "qr", "p", "rho")}, **kout,
                        eos_p_dry=p_dry, eos_p_moist=p_moist)
    print("wrote kessler_eos")


# The end-of-step sponge: two configurations on one seeded level, each with
# the reference runtime's own profiles and the relaxed fields.
SPONGE_CONFIGS = {
    "explicit": dict(z_damp=-1.0, alpha_max=0.05, w_only_cells=4, w_only_alpha_max=0.2, lateral_width=5,
                     lateral_alpha_max=0.08, implicit_mode=0, wind=(2.0, -1.0, 8.0, 3.0, 15.0, 7.0)),
    "implicit": dict(z_damp=2500.0, alpha_max=0.1, w_only_cells=0, w_only_alpha_max=0.0, lateral_width=3,
                     lateral_alpha_max=0.3, implicit_mode=1, wind=(0.5, 1.0, 4.0, -2.0, 9.0, 3.0)),
}


def make_state_relaxation():
    from nimbus_b200.sponge import SpongeConfig

    ref = ReferenceHarness()
    case = Case(18, 15, 12, 500.0, 600.0, 400.0, 6.0, seed=21)
    st, base = cloudy_state(case, seed=21)
    out = {"grid": np.array((case.dx, case.dy, case.dz)), "dt": 6.0, "theta0": base["theta0"],
           **{f"in_{k}": st[k] for k in ("u", "v", "w", "theta")}}
    for name, kw in SPONGE_CONFIGS.items():
        fields = {k: st[k].copy() for k in ("u", "v", "w", "theta")}
        prof = ref.state_relaxation(fields, base["theta0"], (case.dx, case.dy, case.dz), 6.0, SpongeConfig(**kw))
        for k, v in kw.items():
            out[f"{name}_cfg_{k}"] = np.array(v)
        for k, v in prof.items():
            out[f"{name}_prof_{k}"] = v
        for k, v in fields.items():
            out[f"{name}_out_{k}"] = v
    np.savez_compressed(HERE / "state_relaxation.npz", **out)
    print("wrote state_relaxation")


# Output: cell-centre velocities on grids whose nz takes every run width of
# the device kernel (4, 2, 1) plus a single cell, flat and with a terrain
# lower-face velocity; and one npy file written by the reference's writer.
OUTPUT_SHAPES = ((6, 5, 8), (9, 7, 6), (5, 4, 7), (1, 1, 1), (1, 6, 3), (4, 1, 5))


def make_output():
    ref = ReferenceHarness()
    rng = np.random.default_rng(61)
    out = {}
    for n, shape in enumerate(OUTPUT_SHAPES):
        faces = [(rng.standard_normal(shape) * 12.0).astype(np.float32) for _ in range(3)]
        ground = rng.standard_normal(shape[:2]) * 2.5
        flat = ref.cell_centre(*faces)
        terrain = ref.cell_centre(None, None, faces[2], ground)
        for k, a in zip("uvw", faces):
            out[f"s{n}_{k}"] = a
        for k, a in zip("uvw", flat):
            out[f"s{n}_{k}c"] = a
        out[f"s{n}_ground"] = ground
        out[f"s{n}_wc_terrain"] = terrain[2]
    data = (rng.standard_normal((3, 4, 5)) * 100.0).astype(np.float32)
    out["npy_data"] = data
    np.savez_compressed(HERE / "cell_centre.npz", **out)
    ref.npy_write_3d(data, HERE / "npy_write_3d.npy")
    print("wrote cell_centre, npy_write_3d")


# Smagorinsky SGS: one seeded level with strong wind noise, four closure
# configurations (bc W, E, S, N, bottom, top; keyword overrides), each with
# the reference's coefficients and tendencies, one applied SGS substep and,
# where the lateral faces are periodic or closed, its stability limits.
SGS_CASES = {
    "closed_3d_cubic": ((2, 2, 2, 2, 1, 0), {}),
    "periodic_3d_dx": ((0, 0, 0, 0, 1, 0), {"filter_width": "dx"}),
    "open_horizontal": ((1, 1, 4, 1, 1, 0), {"use_vertical": False, "Cs": 0.2}),
    "mixed_vertical": ((0, 0, 2, 3, 1, 0), {"use_horizontal": False, "nu_t_max": 50.0, "K_max": 40.0}),
}
SGS_SHAPE = (12, 11, 8)
SGS_GRID = (500.0, 600.0, 400.0)


def sgs_state(seed=41):
    case = Case(*SGS_SHAPE, *SGS_GRID, 3.0, seed=seed)
    st, base = cloudy_state(case, seed=seed)
    rng = np.random.default_rng(seed)
    for k in "uvw":
        st[k] = (st[k] + rng.standard_normal(SGS_SHAPE).astype(np.float32) * 3.0).astype(np.float32)
    return st, base


def make_sgs():
    from nimbus_b200.sgs import SgsConfig

    ref = ReferenceHarness()
    st, base = sgs_state()
    dz = np.full(SGS_SHAPE[2], SGS_GRID[2])
    out = {"grid": np.array(SGS_GRID), "dz": dz, "theta0": base["theta0"],
           **{f"in_{k}": st[k] for k in ("u", "v", "w", "theta", "qv", "rho")}}
    for name, (bc, kw) in SGS_CASES.items():
        cfg = SgsConfig.from_bc(bc, **kw)
        rates = ref.smagorinsky(st, dz, SGS_GRID, cfg)
        for k, v in rates.items():
            out[f"{name}_{k}"] = v
        applied = {k: st[k].copy() for k in ("u", "v", "w", "theta", "qv")}
        ref.sgs_apply(applied, rates, 2.5, theta0=base["theta0"])
        for k, v in applied.items():
            out[f"{name}_applied_{k}"] = v
        if not any(cfg.open_lateral):
            stab = ref.sgs_stability({**st}, rates, SGS_GRID, bc, cfg)
            out[f"{name}_stability"] = np.array([stab[k] for k in ("maximum", "momentum_energy", "theta_monotonic",
                                                                    "qv_monotonic", "dissipation_w")])
    np.savez_compressed(HERE / "smagorinsky.npz", **out)
    print("wrote smagorinsky")


if __name__ == "__main__":
    # `make_golden.py state_relaxation` (or `output`, `sgs`) writes only that fixture.
    if sys.argv[1:] == ["state_relaxation"]:
        make_state_relaxation()
    elif sys.argv[1:] == ["output"]:
        make_output()
    elif sys.argv[1:] == ["sgs"]:
        make_sgs()
    else:
        main()
        make_state_relaxation()
        make_output()
        make_sgs()
