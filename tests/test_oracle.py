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
from nimbus_b200.initial import Case, perturbed_state
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
