"""Smagorinsky SGS path on the CPU: the oracle restatement pinned to the
reference (golden fixture written by SmagorinskyScheme::compute,
apply_admitted_sgs_substep and compute_sgs_explicit_stability, and live
through the harness where it is built), plus the host-side configuration.
Every comparison is bit for bit."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from nimbus_b200.sgs import SgsConfig, filter_widths
from tests.golden.make_golden import SGS_CASES, SGS_GRID, SGS_SHAPE, sgs_state

GOLDEN = Path(__file__).resolve().parent / "golden" / "smagorinsky.npz"
STABILITY_KEYS = ("maximum", "momentum_energy", "theta_monotonic", "qv_monotonic", "dissipation_w")


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def state_of(g):
    return {k: g[f"in_{k}"].copy() for k in ("u", "v", "w", "theta", "qv", "rho")}


@pytest.mark.parametrize("name", list(SGS_CASES))
def test_golden_closure(o32, golden, name):
    bc, kw = SGS_CASES[name]
    got = o32.smagorinsky(state_of(golden), golden["dz"], SGS_GRID, SgsConfig.from_bc(bc, **kw))
    for k, v in got.items():
        assert np.array_equal(bits(v), bits(golden[f"{name}_{k}"])), k


@pytest.mark.parametrize("name", list(SGS_CASES))
def test_golden_apply(o32, golden, name):
    st = state_of(golden)
    rates = {k: golden[f"{name}_{k}"] for k in ("dudt", "dvdt", "dwdt", "dthdt", "dqvdt")}
    o32.sgs_apply(st, rates, 2.5, theta0=golden["theta0"])
    for k in ("u", "v", "w", "theta", "qv"):
        assert np.array_equal(bits(st[k]), bits(golden[f"{name}_applied_{k}"])), k


@pytest.mark.parametrize("name", [n for n, (bc, _) in SGS_CASES.items() if not any(b in (1, 4) for b in bc[:4])])
def test_golden_stability(o32, golden, name):
    bc, kw = SGS_CASES[name]
    st = state_of(golden)
    rates = {k: golden[f"{name}_{k}"] for k in ("dudt", "dvdt", "dwdt", "dthdt", "dqvdt")}
    got = o32.sgs_stability(st, rates, SGS_GRID, golden["dz"], SgsConfig.from_bc(bc, **kw))
    assert [got[k] for k in STABILITY_KEYS] == list(golden[f"{name}_stability"])


def test_config_topology():
    c = SgsConfig.from_bc((0, 1, 4, 2, 1, 0))
    assert c.periodic_x and not c.periodic_y
    assert c.open_lateral == (False, True, True, False)
    assert SgsConfig(use_vertical=False).mode == "horizontal_only"
    dz = np.array([100.0, 250.0])
    assert np.array_equal(filter_widths(SgsConfig(filter_width="dx"), 500.0, 600.0, dz), np.full(2, np.sqrt(3e5)))
    assert filter_widths(SgsConfig(), 500.0, 600.0, dz)[1] == np.cbrt(500.0 * 600.0 * 250.0)


def test_refusals(o32, golden):
    """A non-positive theta or a non-finite wind is refused (the reference's
    invalid_argument)."""
    st = state_of(golden)
    st["theta"][3, 4, 2] = 0.0
    with pytest.raises(ValueError, match="finite physical domain"):
        o32.smagorinsky(st, golden["dz"], SGS_GRID, SgsConfig())
    st = state_of(golden)
    st["u"][1, 1, 1] = np.nan
    with pytest.raises(ValueError, match="finite physical domain"):
        o32.smagorinsky(st, golden["dz"], SGS_GRID, SgsConfig())


def test_sgs_step_substeps_follow_dt_sgs(o32, golden):
    """dt = 2.5 s with dt_sgs = 1 s: three substeps (1, 1, 0.5 s), each
    refreshing the closure from the live state."""
    st = state_of(golden)
    count, limit = o32.sgs_step(st, golden["dz"], SGS_GRID, SgsConfig.from_bc((2, 2, 2, 2, 1, 0)), 2.5,
                                theta0=golden["theta0"])
    assert count == 3 and limit > 1.0


@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("seed", [51, 52])
@pytest.mark.parametrize("name", list(SGS_CASES))
def test_live_reference_pin(o32, name, seed):
    ref = oracle.ReferenceHarness(threads=3)
    bc, kw = SGS_CASES[name]
    cfg = SgsConfig.from_bc(bc, **kw)
    st, base = sgs_state(seed)
    dz = np.linspace(300.0, 500.0, SGS_SHAPE[2])  # stretched levels
    a = o32.smagorinsky(st, dz, SGS_GRID, cfg)
    b = ref.smagorinsky(st, dz, SGS_GRID, cfg)
    for k in a:
        assert np.array_equal(bits(a[k]), bits(b[k])), k
    x = {k: st[k].copy() for k in ("u", "v", "w", "theta", "qv")}
    y = {k: st[k].copy() for k in ("u", "v", "w", "theta", "qv")}
    a["dudt"].flat[17] = np.inf  # the repairs treat it as zero in both
    o32.sgs_apply(x, a, 1.7, theta0=base["theta0"])
    ref.sgs_apply(y, a, 1.7, theta0=base["theta0"])
    for k in x:
        assert np.array_equal(bits(x[k]), bits(y[k])), k
    if not any(cfg.open_lateral):
        dzu = np.full(SGS_SHAPE[2], SGS_GRID[2])
        r = o32.smagorinsky(st, dzu, SGS_GRID, cfg)
        assert o32.sgs_stability(st, r, SGS_GRID, dzu, cfg) == ref.sgs_stability(st, r, SGS_GRID, bc, cfg)
