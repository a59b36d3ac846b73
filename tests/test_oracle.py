"""The oracle restatement pinned to the reference: known-answer tests of the
WENO5 face (tests/numerics/test_weno5_reconstruction.cpp), the committed golden
fixtures produced by the reference CPU solver itself (tests/golden/), and --
where the reference was built here -- live seeded comparisons against the
reference objects (oracle/_ref).  All bit-exact."""
import glob
import math

import numpy as np
import pytest

import oracle
from nimbus_b200.initial import Case, cloudy_state, perturbed_state
from tests.golden.make_golden import BC_SETS, close_walls

pytestmark = pytest.mark.skipif(not oracle.restatement_available(),
                                reason="oracle restatement not built (make -f oracle/oracle.mk)")

GOLDEN = sorted(glob.glob("tests/golden/loop_*.npz"))


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


@pytest.fixture(scope="module")
def o64():
    return oracle.Restatement("f64")


def _jiang_shu(a, b, c, d, e):
    """Independent Jiang-Shu restatement (test_weno5_reconstruction.cpp:25-45)."""
    eps = 1.0e-6 * max(a * a, b * b, c * c, d * d, e * e) + 1.0e-40
    p0 = (2.0 * a - 7.0 * b + 11.0 * c) / 6.0
    p1 = (-1.0 * b + 5.0 * c + 2.0 * d) / 6.0
    p2 = (2.0 * c + 5.0 * d - 1.0 * e) / 6.0
    b0 = 13 / 12 * (a - 2 * b + c) ** 2 + 0.25 * (a - 4 * b + 3 * c) ** 2
    b1 = 13 / 12 * (b - 2 * c + d) ** 2 + 0.25 * (b - d) ** 2
    b2 = 13 / 12 * (c - 2 * d + e) ** 2 + 0.25 * (3 * c - 4 * d + e) ** 2
    a0, a1, a2 = 0.1 / (eps + b0) ** 2, 0.6 / (eps + b1) ** 2, 0.3 / (eps + b2) ** 2
    return (a0 * p0 + a1 * p1 + a2 * p2) / (a0 + a1 + a2)


def test_weno5_free_stream(o32):
    for v in (2.5, -3.0, 0.0):
        assert abs(o32.weno5_face(v, v, v, v, v) - v) <= 1e-13


def test_weno5_linear_exact(o32):
    assert o32.weno5_face(1, 2, 3, 4, 5) == pytest.approx(3.5, abs=1e-12)
    assert o32.weno5_face(3, 5, 7, 9, 11) == pytest.approx(8.0, abs=1e-12)
    assert o32.weno5_face(10, 8, 6, 4, 2) == pytest.approx(5.0, abs=1e-12)


def test_weno5_quadratic_exact(o32):
    t = 1.0 / 12.0
    assert o32.weno5_face(0 + t, 1 + t, 4 + t, 9 + t, 16 + t) == pytest.approx(6.25, abs=1e-9)


def test_weno5_coefficient_lock(o32):
    for q in ([1.0, 0.5, 2.0, 1.5, 3.0], [0.2, 1.7, 1.1, 2.9, 0.4], [-1.0, 2.0, -0.5, 3.0, 1.0],
              [7.3, 7.1, 6.4, 2.0, 9.9]):
        assert o32.weno5_face(*q) == pytest.approx(_jiang_shu(*q), rel=0, abs=1e-12)


def test_weno5_scale_invariant(o32):
    q = [1.0, 0.5, 2.0, 1.5, 3.0]
    base = o32.weno5_face(*q)
    for s in (1e3, 1e-3, 1e-6):
        assert o32.weno5_face(*[s * x for x in q]) == pytest.approx(s * base, rel=1e-9)


def test_weno5_eno_at_jump(o32):
    up = o32.weno5_face(5, 5, 5, 9, 9)
    assert up == pytest.approx(5.0, abs=1e-2) and 5.0 - 1e-9 <= up <= 9.0 + 1e-9
    assert o32.weno5_face(9, 9, 9, 5, 5) == pytest.approx(9.0, abs=1e-2)


def test_weno5_nonfinite_fallback(o32):
    nan, inf = math.nan, math.inf
    assert o32.weno5_face(nan, 1, 2, 3, 4) == pytest.approx(2.0)
    assert o32.weno5_face(1, 2, 3, 4, inf) == pytest.approx(3.0)
    assert o32.weno5_face(nan, nan, 5, nan, nan) == pytest.approx(5.0)


def test_mc_slope_extremum_and_limits(o32):
    assert o32.mc_slope(1.0, 2.0, 1.0) == 0.0            # extremum: zero slope
    assert o32.mc_slope(0.0, 1.0, 2.0) == pytest.approx(1.0)
    assert o32.mc_slope(0.0, 1.0, 1.1) == pytest.approx(0.2)   # limited by 2*right


def _state(g, prefix="in_"):
    return {k[len(prefix):]: g[k].copy() for k in g.files if k.startswith(prefix)}


def test_golden_fused_substep(o32):
    g = np.load("tests/golden/fused_substep.npz")
    st = _state(g)
    drho = np.zeros_like(st["u"])
    o32.acoustic_fused(st, g["rho0"], g["p0"], float(g["dt_small"]), tuple(g["grid"]), drho)
    for k in ("u", "v", "w", "rho", "p"):
        np.testing.assert_array_equal(st[k], g["out_" + k], err_msg=k)
    np.testing.assert_array_equal(drho, g["out_drho"])


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.split("/")[-1])
def test_golden_acoustic_loop_and_transport(o32, path):
    g = np.load(path)
    st = _state(g)
    bc = tuple(int(x) for x in g["bc"])
    dt = float(g["dt_large"])
    out = o32.acoustic_loop(st, g["rho0"], g["p0"], dt, int(g["n_substeps"]), tuple(g["grid"]), bc)
    for k in ("u", "v", "w", "rho", "p"):
        np.testing.assert_array_equal(st[k], g["out_" + k], err_msg=k)
    for k in ("mfx", "mfy", "mfz", "rho_begin", "wave"):
        np.testing.assert_array_equal(out[k], g["out_" + k], err_msg=k)
    src = _state(g)
    for tag, weno in (("weno", True), ("mc", False)):
        qs = [src[k].copy() for k in ("theta", "qv", "qc", "qr")]
        o32.scalar_transport(qs, [0, 1, 1, 1], g["out_rho"], g["out_rho_begin"], g["out_mfx"], g["out_mfy"],
                             g["out_mfz"], dt, tuple(g["grid"]), weno=weno, top_open=bc[5] == 2)
        for key, q in zip(("theta", "qv", "qc", "qr"), qs):
            np.testing.assert_array_equal(q, g[f"tr{tag}_{key}"], err_msg=f"{tag} {key}")


def test_fp64_oracle_tracks_fp32(o32, o64):
    """The FP64-storage oracle differs from the FP32 one only by storage rounding."""
    g = np.load(GOLDEN[0])
    st32 = _state(g)
    st64 = {k: v.astype(np.float64) for k, v in st32.items()}
    bc = tuple(int(x) for x in g["bc"])
    o32.acoustic_loop(st32, g["rho0"], g["p0"], 6.0, 7, tuple(g["grid"]), bc)
    o64.acoustic_loop(st64, g["rho0"], g["p0"], 6.0, 7, tuple(g["grid"]), bc)
    for k in ("u", "v", "w", "rho", "p"):
        a, b = st32[k].astype(np.float64), st64[k]
        rel = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
        assert rel < 1e-5, (k, rel)


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("bc_name", list(BC_SETS))
@pytest.mark.parametrize("seed", [21, 22])
def test_live_reference_pin(o32, bc_name, seed):
    ref = oracle.ReferenceHarness()
    bc = BC_SETS[bc_name]
    case = Case(18, 15, 11, 800.0, 900.0, 400.0, 4.0, seed=seed)
    st, base = perturbed_state(case, seed=seed)
    close_walls(st, bc)
    a = {k: v.copy() for k, v in st.items()}
    b = {k: v.copy() for k, v in st.items()}
    ra = ref.acoustic_loop(a, base["rho0"], base["p0"], 4.0, 9, (800.0, 900.0, 400.0), bc)
    rb = o32.acoustic_loop(b, base["rho0"], base["p0"], 4.0, 9, (800.0, 900.0, 400.0), bc)
    for k in ("u", "v", "w", "rho", "p"):
        np.testing.assert_array_equal(a[k], b[k], err_msg=k)
    for k in ra:
        np.testing.assert_array_equal(ra[k], rb[k], err_msg=k)
    qa = [a["theta"].copy(), a["qv"].copy(), a["qc"].copy(), a["qr"].copy()]
    qb = [q.copy() for q in qa]
    ref.scalar_transport(qa, [0, 1, 1, 1], a["u"], a["v"], a["w"], a["rho"], ra["rho_begin"], ra["mfx"], ra["mfy"],
                         ra["mfz"], 4.0, (800.0, 900.0, 400.0), top_open=bc[5] == 2)
    o32.scalar_transport(qb, [0, 1, 1, 1], a["rho"], ra["rho_begin"], ra["mfx"], ra["mfy"], ra["mfz"], 4.0,
                         (800.0, 900.0, 400.0), top_open=bc[5] == 2)
    for x, y in zip(qa, qb):
        np.testing.assert_array_equal(x, y)


def _slow_case(g):
    st = {k[3:]: g[k].copy() for k in g.files if k.startswith("in_")}
    base = {k[5:]: g[k] for k in g.files if k.startswith("base_")}
    return st, base


def test_golden_slow_tendencies(o32):
    g = np.load("tests/golden/slow_tendencies.npz")
    st, base = _slow_case(g)
    grid = tuple(g["grid"])
    got = o32.slow_tendencies(st, base, grid, coriolis_f=float(g["coriolis_f"]), moist=True)
    for key, arr in zip(("du", "dv", "dw", "dp"), got):
        np.testing.assert_array_equal(arr, g["out_" + key], err_msg=key)
    dry = o32.slow_tendencies(st, base, grid, coriolis_f=0.0, moist=False)
    for key, arr in zip(("du", "dv", "dw", "dp"), dry):
        np.testing.assert_array_equal(arr, g["dry_" + key], err_msg="dry " + key)


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed", [31, 32])
def test_live_reference_pin_slow(o32, seed):
    ref = oracle.ReferenceHarness()
    case = Case(19, 16, 13, 600.0, 650.0, 350.0, 3.0, seed=seed)
    st, base = perturbed_state(case, seed=seed)
    for cor, moist in ((1.2e-4, True), (0.0, False)):
        a = ref.slow_tendencies(st, base, (600.0, 650.0, 350.0), cor, moist)
        b = o32.slow_tendencies(st, base, (600.0, 650.0, 350.0), cor, moist)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


def test_heun_step_is_average_of_two_evaluations(o32):
    """The composition, checked on the CPU: one Heun step equals applying
    0.5f*(k1 + k2) with k2 taken at the predictor state."""
    g = np.load("tests/golden/slow_tendencies.npz")
    st, base = _slow_case(g)
    grid = tuple(g["grid"])
    dt = 2.0
    a = {k: v.copy() for k, v in st.items()}
    o32.slow_rk2_step(a, base, grid, dt, coriolis_f=1e-4)
    k1 = o32.slow_tendencies(st, base, grid, 1e-4)
    star = {k: v.copy() for k, v in st.items()}
    for key, t in zip(("u", "v", "w", "p"), k1):
        star[key] = (star[key].astype(np.float64) + t.astype(np.float64) * dt).astype(np.float32)
    k2 = o32.slow_tendencies(star, base, grid, 1e-4)
    for key, t1, t2 in zip(("u", "v", "w", "p"), k1, k2):
        avg = np.float32(0.5) * (t2 + t1)
        want = (st[key].astype(np.float64) + avg.astype(np.float64) * dt).astype(np.float32)
        np.testing.assert_array_equal(a[key], want, err_msg=key)


def _kessler_case(g):
    return {k[3:]: g[k].copy() for k in g.files if k.startswith("in_")}


@pytest.mark.parametrize("dom", ["cgrid", "full"])
def test_golden_kessler_tendencies(o32, dom):
    g = np.load("tests/golden/kessler_eos.npz")
    st = _kessler_case(g)
    got = o32.kessler_tendencies(st, float(g["dz"]), float(g["dt"]), tuple(g["dom_" + dom]))
    for key, arr in zip(("dtheta", "dqv", "dqc", "dqr"), got):
        np.testing.assert_array_equal(arr, g[f"{dom}_{key}"], err_msg=key)
    # every process acted somewhere: condensation and evaporation both present,
    # rain gained (autoconversion/accretion) and lost (evaporation/fall-out)
    dqv = g[f"{dom}_dqv"]
    dqr = g[f"{dom}_dqr"]
    assert (dqv > 0).any() and (dqv < 0).any() and (dqr > 0).any() and (dqr < 0).any()


def test_golden_eos_projection(o32):
    g = np.load("tests/golden/kessler_eos.npz")
    st = _kessler_case(g)
    p = st["p"].copy()
    assert o32.eos_projection(p, st["rho"], st["theta"])
    np.testing.assert_array_equal(p, g["eos_p_dry"])
    p = st["p"].copy()
    assert o32.eos_projection(p, st["rho"], st["theta"], st["qv"], st["qc"], st["qr"])
    np.testing.assert_array_equal(p, g["eos_p_moist"])


# (field, cell, value, refused when dry, refused when moist): invalid density or
# temperature refuses everywhere; bad water or old pressure only inside the
# attributed domain of a complete moist state (eos_apply.cpp:89-158).
EOS_CASES = [
    ("rho", (3, 3, 3), -1.0, True, True),
    ("theta", (0, 0, 0), np.nan, True, True),
    ("theta", (2, 2, 2), 3e38, True, True),
    ("qv", (3, 3, 3), -1e-6, False, True),
    ("qv", (0, 3, 3), -1e-6, False, False),
    ("qc", (2, 2, 0), -1e-3, False, True),
    ("qr", (1, 1, 1), np.inf, False, True),
    ("p", (4, 4, 4), 0.0, False, True),
    ("p", (8, 3, 3), np.nan, False, False),
]


@pytest.mark.parametrize("field,cell,value,dry_refused,moist_refused", EOS_CASES)
def test_eos_refusal_rules(o32, field, cell, value, dry_refused, moist_refused):
    case = Case(9, 7, 6, 1000.0, 1000.0, 500.0, 6.0, seed=1)
    st, _ = cloudy_state(case, seed=3)
    st[field][cell] = value
    for moist, refused in ((False, dry_refused), (True, moist_refused)):
        p = st["p"].copy()
        q = (st["qv"], st["qc"], st["qr"]) if moist else (None, None, None)
        ok = o32.eos_projection(p, st["rho"], st["theta"], *q)
        assert ok == (not refused), (field, moist)
        if refused:
            np.testing.assert_array_equal(p.view(np.uint32), st["p"].view(np.uint32))


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed", [1, 2])
def test_live_reference_pin_kessler(o32, seed):
    ref = oracle.ReferenceHarness()
    case = Case(15, 13, 20, 1000.0, 1000.0, 500.0, 6.0, seed=seed)
    st, _ = cloudy_state(case, seed=seed)
    for dom in ((1, 14, 1, 12, 0, 20), (2, 9, 0, 13, 3, 17)):
        a = ref.kessler_tendencies(st, 500.0, 6.0, dom)
        b = o32.kessler_tendencies(st, 500.0, 6.0, dom)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("field,cell,value,dry_refused,moist_refused", EOS_CASES)
def test_live_reference_pin_eos(o32, field, cell, value, dry_refused, moist_refused):
    ref = oracle.ReferenceHarness()
    case = Case(9, 7, 6, 1000.0, 1000.0, 500.0, 6.0, seed=1)
    st, _ = cloudy_state(case, seed=3)
    st[field][cell] = value
    for moist in (False, True):
        q = (st["qv"], st["qc"], st["qr"]) if moist else (None, None, None)
        a, b = st["p"].copy(), st["p"].copy()
        ra = ref.eos_projection(a, st["rho"], st["theta"], (1000.0, 1000.0, 500.0), *q)
        rb = o32.eos_projection(b, st["rho"], st["theta"], *q)
        assert ra == rb
        np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("bc_name", list(BC_SETS))
def test_live_reference_pin_boundary_refresh(o32, bc_name):
    """apply_acoustic(0): the ghost refresh before the KW78 seed."""
    ref = oracle.ReferenceHarness()
    case = Case(13, 11, 8, 1000.0, 1000.0, 500.0, 6.0, seed=4)
    st, _ = perturbed_state(case, seed=21)
    close_walls(st, BC_SETS[bc_name])
    a = {k: st[k].copy() for k in ("u", "v", "w", "rho", "p")}
    b = {k: st[k].copy() for k in ("u", "v", "w", "rho", "p")}
    ref.acoustic_boundaries(a, (1000.0, 1000.0, 500.0), BC_SETS[bc_name], 0.0)
    o32.acoustic_boundaries(b, (1000.0, 1000.0, 500.0), BC_SETS[bc_name], 0.0)
    for k in a:
        np.testing.assert_array_equal(a[k].view(np.uint32), b[k].view(np.uint32), err_msg=k)
    assert any(not np.array_equal(a[k], st[k]) for k in a)  # the refresh did something


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("bc_name", list(BC_SETS))
def test_live_reference_pin_large_step(o32, bc_name):
    """The oracle's whole large step against the same step assembled from the
    reference's own objects, two steps, every prognostic field bit for bit."""
    from nimbus_b200.initial import cloudy_state
    ref = oracle.ReferenceHarness()
    case = Case(17, 15, 13, 800.0, 700.0, 400.0, 4.0, seed=8)
    st, base = cloudy_state(case, seed=8)
    close_walls(st, BC_SETS[bc_name])
    a = {k: v.copy() for k, v in st.items()}
    b = {k: v.copy() for k, v in st.items()}
    grid = (800.0, 700.0, 400.0)
    for _ in range(2):
        ref.large_step(a, base, grid, 4.0, 5, BC_SETS[bc_name], coriolis_f=1e-4)
        o32.large_step(b, base, grid, 4.0, 5, BC_SETS[bc_name], coriolis_f=1e-4)
    for k in ("u", "v", "w", "rho", "p", "theta", "qv", "qc", "qr"):
        np.testing.assert_array_equal(a[k].view(np.uint32), b[k].view(np.uint32), err_msg=k)


# ---- End-of-step sponge (state relaxation) ------------------------------------
def _sponge_config(g, name):
    from nimbus_b200.sponge import SpongeConfig

    kw = {k[len(name) + 5:]: g[k] for k in g.files if k.startswith(f"{name}_cfg_")}
    kw = {k: (tuple(float(x) for x in v) if k == "wind" else v.item()) for k, v in kw.items()}
    return SpongeConfig(**kw)


@pytest.mark.parametrize("name", ["explicit", "implicit"])
def test_golden_state_relaxation(o32, name):
    """The profile builder reproduces the reference runtime's profiles, and the
    restatement the reference's relaxed fields, bit for bit (fixture from the
    reference's own apply_rayleigh_damping + apply_lateral_damping)."""
    from nimbus_b200.sponge import build_profiles

    g = np.load("tests/golden/state_relaxation.npz")
    cfg = _sponge_config(g, name)
    nz = g["in_u"].shape[2]
    P = build_profiles(cfg, nz, float(g["grid"][2]), g["theta0"])
    for k in ("alpha", "upper_w_alpha", "w_only_alpha", "u_ref", "v_ref", "lateral_alpha"):
        want = g[f"{name}_prof_{k}"]
        got = getattr(P, k)
        assert got.shape == want.shape and np.array_equal(got.view(np.uint64), want.view(np.uint64)), k
    st = {k: g[f"in_{k}"].copy() for k in ("u", "v", "w", "theta")}
    o32.state_relaxation(st, P, float(g["dt"]))
    for k in st:
        want = g[f"{name}_out_{k}"]
        assert np.count_nonzero(st[k].view(np.uint32) != want.view(np.uint32)) == 0, k
        assert np.count_nonzero(want != g[f"in_{k}"]) > 0, k  # the sponge acted on every field


@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed", [31, 32, 33])
def test_live_reference_pin_state_relaxation(o32, seed):
    """Seeded configurations (explicit and implicit, with and without the lid
    absorber and the lateral band, default and set damping heights) against
    the reference objects: profiles and fields bit-exact."""
    from nimbus_b200.sponge import SpongeConfig, build_profiles

    rng = np.random.default_rng(seed)
    cfg = SpongeConfig(z_damp=float(rng.choice([-1.0, 1800.0])), alpha_max=float(rng.uniform(0.01, 0.2)),
                       w_only_cells=int(rng.integers(0, 6)), w_only_alpha_max=float(rng.uniform(0.05, 0.5)),
                       lateral_width=int(rng.integers(0, 9)), lateral_alpha_max=float(rng.uniform(0.0, 0.4)),
                       implicit_mode=int(rng.integers(0, 2)), wind=tuple(rng.uniform(-10, 20, 6)))
    case = Case(int(rng.integers(5, 20)), int(rng.integers(5, 20)), int(rng.integers(4, 16)), 500.0, 700.0,
                350.0, 4.0, seed=seed)
    st, base = cloudy_state(case, seed=seed)
    ref_fields = {k: st[k].copy() for k in ("u", "v", "w", "theta")}
    prof = oracle.ReferenceHarness().state_relaxation(ref_fields, base["theta0"], (case.dx, case.dy, case.dz), 4.0,
                                                      cfg)
    P = build_profiles(cfg, case.nz, case.dz, base["theta0"])
    for k, want in prof.items():
        assert np.array_equal(getattr(P, k).view(np.uint64), want.view(np.uint64)), k
    mine = {k: st[k].copy() for k in ref_fields}
    o32.state_relaxation(mine, P, 4.0)
    for k in mine:
        assert np.count_nonzero(mine[k].view(np.uint32) != ref_fields[k].view(np.uint32)) == 0, k


def test_state_relaxation_rejects_invalid_rates(o32):
    from nimbus_b200.sponge import SpongeConfig, build_profiles

    case = Case(8, 8, 6, 500.0, 500.0, 400.0, 3.0, seed=2)
    st, base = cloudy_state(case, seed=2)
    P = build_profiles(SpongeConfig(z_damp=100.0), case.nz, case.dz, base["theta0"])
    P.alpha[3] = -1.0
    with pytest.raises(ValueError):
        o32.state_relaxation({k: st[k].copy() for k in ("u", "v", "w", "theta")}, P, 3.0)
    P = build_profiles(SpongeConfig(), case.nz, case.dz, base["theta0"])
    with pytest.raises(ValueError):
        o32.state_relaxation({k: st[k].copy() for k in ("u", "v", "w", "theta")}, P, 0.0)


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
def test_transport_bridge_route_equals_the_direct_call(o32):
    """The reference's transport bridge with its CPU backend (the route a
    device backend replaces) gives the direct call's bits: the harness's route
    arguments are the ones advection_batch.cpp passes."""
    ref = oracle.ReferenceHarness()
    bc = BC_SETS["periodic_noslip_open"]
    case = Case(18, 15, 11, 800.0, 900.0, 400.0, 4.0, seed=23)
    st, base = perturbed_state(case, seed=23)
    close_walls(st, bc)
    a = {k: v.copy() for k, v in st.items()}
    loop = o32.acoustic_loop(a, base["rho0"], base["p0"], 4.0, 9, (800.0, 900.0, 400.0), bc)
    args = (a["u"], a["v"], a["w"], a["rho"], loop["rho_begin"], loop["mfx"], loop["mfy"], loop["mfz"], 4.0,
            (800.0, 900.0, 400.0))
    qa = [a[k].copy() for k in ("theta", "qv", "qc", "qr")]
    qb = [q.copy() for q in qa]
    ref.scalar_transport(qa, [0, 1, 1, 1], *args, top_open=True)
    assert ref.bridge_scalar_transport(qb, [0, 1, 1, 1], *args, top_open=True)
    for x, y in zip(qa, qb):
        np.testing.assert_array_equal(x.view(np.uint32), y.view(np.uint32))


def test_kessler_device_restatement_fp32_floor():
    """The device-route Kessler operators' FP64 statement against an FP32
    evaluation of the same sequence (numpy, IEEE single): the FP32 floor the
    CUDA operators' tolerances are set above (6e-6 of each field's scale for
    the pointwise operator, 3e-7 for the fallout)."""
    from oracle.kessler_device import kessler_pointwise, kessler_sedimentation
    from tests.test_kessler_dispatch_gpu import PARAMS, VT_CAP, kessler_inputs

    st = kessler_inputs((24, 20, 30), 1)
    dom = (1, 23, 1, 19, 0, 30)
    args = [PARAMS[k] for k in ("qc0", "c_auto", "c_accr", "evaporation_efficiency", "lv_cp", "t0", "dt")]
    ins = [st[k] for k in ("T", "p", "qv", "qc", "qr", "rho")]
    f64 = kessler_pointwise(*ins, dom, *args)
    f32 = kessler_pointwise(*ins, dom, *args, dtype=np.float32)
    for a, b in zip(f64, f32):
        assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max()
    s64 = kessler_sedimentation(st["qr"], f64[3], dom, 400.0, 20.0, VT_CAP, rho_d=st["rho"])
    s32 = kessler_sedimentation(st["qr"], f64[3].astype(np.float32), dom, 400.0, 20.0, VT_CAP, rho_d=st["rho"],
                                dtype=np.float32)
    assert np.abs(s64 - s32).max() <= 1e-6 * np.abs(s64).max()
