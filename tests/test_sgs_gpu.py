"""Smagorinsky SGS path on the device against the reference, bit for bit:
the fused closure (host and device memory), the SGS apply, the stability
limit and the substepped SGS integration of a large step."""
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from nimbus_b200 import cuda
from nimbus_b200.initial import Case, cloudy_state
from nimbus_b200.sgs import SgsConfig
from tests.golden.make_golden import SGS_CASES, SGS_GRID, SGS_SHAPE, sgs_state

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "smagorinsky.npz"
RATES = ("dudt", "dvdt", "dwdt", "dthdt", "dqvdt")
STABILITY_KEYS = ("maximum", "momentum_energy", "theta_monotonic", "qv_monotonic", "dissipation_w")


@pytest.fixture(scope="module")
def ctx():
    c = cuda.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


@pytest.fixture(scope="module")
def golden():
    return np.load(GOLDEN)


def assert_bitwise(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    bad = np.count_nonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad == 0, f"{what}: {bad}/{a.size} values differ"


def state_of(g):
    return {k: g[f"in_{k}"].copy() for k in ("u", "v", "w", "theta", "qv", "rho")}


def on_device(st):
    return {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in st.items()}


@pytest.mark.parametrize("name", list(SGS_CASES))
def test_closure_golden_host(ctx, golden, name):
    bc, kw = SGS_CASES[name]
    args = cuda.smagorinsky_args(state_of(golden), golden["dz"], SGS_GRID, SgsConfig.from_bc(bc, **kw))
    ctx.check(ctx.smagorinsky_fused(args))
    for k, v in args.outputs.items():
        assert_bitwise(v, golden[f"{name}_{k}"], k)


@pytest.mark.parametrize("name", list(SGS_CASES))
def test_apply_golden_host(ctx, golden, name):
    st = state_of(golden)
    rates = {k: golden[f"{name}_{k}"] for k in RATES}
    ctx.check(ctx.sgs_apply(cuda.sgs_apply_args(st, rates, 2.5, theta0=golden["theta0"])))
    for k in ("u", "v", "w", "theta", "qv"):
        assert_bitwise(st[k], golden[f"{name}_applied_{k}"], k)


@pytest.mark.parametrize("name", [n for n, (bc, _) in SGS_CASES.items() if not any(b in (1, 4) for b in bc[:4])])
def test_stability_golden_host(ctx, golden, name):
    bc, kw = SGS_CASES[name]
    rates = {k: golden[f"{name}_{k}"] for k in RATES}
    got = ctx.sgs_stability(cuda.smagorinsky_args(state_of(golden), golden["dz"], SGS_GRID,
                                                  SgsConfig.from_bc(bc, **kw), rates=rates))
    assert [got[k] for k in STABILITY_KEYS] == list(golden[f"{name}_stability"])


# Larger seeded levels on the device against the oracle: every mode, both
# filters, periodic / closed / open faces, stretched levels, no moisture.
DEVICE_CASES = [
    ((48, 40, 24), (2, 2, 2, 2, 1, 0), {}, "uniform"),
    ((37, 29, 17), (0, 0, 0, 0, 1, 0), {"filter_width": "dx"}, "stretched"),
    ((40, 33, 20), (1, 1, 4, 1, 1, 0), {"use_vertical": False}, "uniform"),
    ((31, 44, 15), (0, 0, 2, 3, 1, 0), {"use_horizontal": False, "nu_t_max": 30.0, "K_max": 25.0}, "stretched"),
    ((3, 3, 2), (2, 3, 2, 3, 1, 0), {}, "uniform"),
]


def _case(shape, seed):
    case = Case(*shape, *SGS_GRID, 3.0, seed=seed)
    st, base = cloudy_state(case, seed=seed)
    rng = np.random.default_rng(seed)
    for k in "uvw":
        st[k] = (st[k] + rng.standard_normal(shape).astype(np.float32) * 4.0).astype(np.float32)
    return st, base


def _dz(nz, kind):
    return np.full(nz, SGS_GRID[2]) if kind == "uniform" else np.linspace(250.0, 550.0, nz)


@pytest.mark.parametrize("moist", [True, False])
@pytest.mark.parametrize("shape,bc,kw,dzkind", DEVICE_CASES, ids=[str(c[0]) for c in DEVICE_CASES])
def test_closure_device_vs_oracle(ctx, o32, shape, bc, kw, dzkind, moist):
    st, _ = _case(shape, sum(shape))
    if not moist:
        st.pop("qv")
    dz = _dz(shape[2], dzkind)
    cfg = SgsConfig.from_bc(bc, **kw)
    dev = on_device({k: st[k] for k in ("u", "v", "w", "theta", "rho") + (("qv",) if moist else ())})
    args = cuda.smagorinsky_args(dev, dz, SGS_GRID, cfg, memory=cuda.MEMORY_DEVICE)
    ctx.check(ctx.smagorinsky_fused(args))
    ctx.synchronize()
    want = o32.smagorinsky(st, dz, SGS_GRID, cfg)
    for k, v in args.outputs.items():
        assert_bitwise(v.cpu().numpy(), want[k], k)


@pytest.mark.parametrize("sanitize", [True, False])
def test_apply_device_vs_oracle(ctx, o32, sanitize):
    st, base = _case((40, 36, 20), 9)
    rates = o32.smagorinsky(st, _dz(20, "uniform"), SGS_GRID, SgsConfig())
    rates["dudt"].flat[11] = np.nan
    rates["dthdt"].flat[13] = np.inf
    rates["dvdt"].flat[17] = 3e6  # clamps
    dev = on_device({k: st[k] for k in ("u", "v", "w", "theta", "qv")})
    drates = on_device(rates)
    ctx.check(ctx.sgs_apply(cuda.sgs_apply_args(dev, drates, 1.3, theta0=base["theta0"], sanitize=sanitize,
                                                memory=cuda.MEMORY_DEVICE)))
    ctx.synchronize()
    want = {k: st[k].copy() for k in ("u", "v", "w", "theta", "qv")}
    o32.sgs_apply(want, rates, 1.3, theta0=base["theta0"], repairs=sanitize)
    for k in want:
        assert_bitwise(dev[k].cpu().numpy(), want[k], k)


CLOSED_CASES = [c for c in DEVICE_CASES if not any(b in (1, 4) for b in c[1][:4])]


@pytest.mark.parametrize("shape,bc,kw,dzkind", CLOSED_CASES, ids=[str(c[0]) for c in CLOSED_CASES])
def test_stability_device_vs_oracle(ctx, o32, shape, bc, kw, dzkind):
    st, _ = _case(shape, 3 + sum(shape))
    dz = _dz(shape[2], dzkind)
    cfg = SgsConfig.from_bc(bc, **kw)
    rates = o32.smagorinsky(st, dz, SGS_GRID, cfg)
    want = o32.sgs_stability(st, rates, SGS_GRID, dz, cfg)
    dev = on_device({k: st[k] for k in ("u", "v", "w", "theta", "rho", "qv")})
    got = ctx.sgs_stability(cuda.smagorinsky_args(dev, dz, SGS_GRID, cfg, rates=on_device(rates),
                                                  memory=cuda.MEMORY_DEVICE))
    assert got == want


@pytest.mark.parametrize("dt,dt_sgs", [(2.5, 1.0), (3.0, 5.0)])
def test_sgs_step_vs_oracle(ctx, o32, dt, dt_sgs):
    """The substepped SGS integration on the device equals the oracle's loop
    of pinned parts (closure, stability, apply), substep for substep."""
    st, base = _case((44, 38, 22), 21)
    dz = _dz(22, "stretched")
    cfg = SgsConfig.from_bc((2, 3, 0, 0, 1, 0), dt_sgs=dt_sgs)
    dev = on_device({k: st[k] for k in ("u", "v", "w", "theta", "rho", "qv")})
    count, limit = ctx.sgs_step(cuda.sgs_step_args(dev, dz, SGS_GRID, cfg, dt, theta0=base["theta0"], time_s=600.0))
    want = {k: st[k].copy() for k in ("u", "v", "w", "theta", "qv", "rho")}
    w_count, w_limit = o32.sgs_step(want, dz, SGS_GRID, cfg, dt, theta0=base["theta0"], time_s=600.0)
    assert (count, limit) == (w_count, w_limit)
    for k in ("u", "v", "w", "theta", "qv"):
        assert_bitwise(dev[k].cpu().numpy(), want[k], k)


def test_refusals(ctx, golden):
    """The reference's invalid states are refused with host outputs untouched;
    open stress boundaries are outside the stability contract."""
    st = state_of(golden)
    st["rho"][2, 2, 2] = -1.0
    outputs = {k: np.full(SGS_SHAPE, 7.0, np.float32) for k in ("nu_t", "K_theta", "K_q", *RATES)}
    args = cuda.smagorinsky_args(st, golden["dz"], SGS_GRID, SgsConfig(), outputs=outputs)
    assert ctx.smagorinsky_fused(args) == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    assert all(np.all(v == 7.0) for v in outputs.values())
    bad_cfg = SgsConfig(Pr_t=0.0)
    assert ctx.smagorinsky_fused(cuda.smagorinsky_args(state_of(golden), golden["dz"], SGS_GRID, bad_cfg)) == \
        cuda.NIMBUS_ERR_INVALID_ARGUMENT
    rates = {k: golden[f"closed_3d_cubic_{k}"] for k in RATES}
    with pytest.raises(cuda.NimbusCudaError) as e:
        ctx.sgs_stability(cuda.smagorinsky_args(state_of(golden), golden["dz"], SGS_GRID,
                                                SgsConfig.from_bc((1, 1, 1, 1, 1, 0)), rates=rates))
    assert e.value.status == 5  # NIMBUS_ERR_UNSUPPORTED
    st = state_of(golden)
    assert ctx.sgs_apply(cuda.sgs_apply_args(st, rates, 0.0)) == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    dev = on_device(state_of(golden))
    dev["theta"][1, 1, 1] = float("nan")
    args = cuda.smagorinsky_args(dev, golden["dz"], SGS_GRID, SgsConfig(), memory=cuda.MEMORY_DEVICE)
    ctx.check(ctx.smagorinsky_fused(args))
    with pytest.raises(cuda.NimbusCudaError, match="SGS closure"):
        ctx.synchronize()


def test_full_level(ctx, o32):
    """A 320x320x64 level (26 MB per field, 14 fields read or written: more
    than L2) bit for bit; the closure's ncu capture uses this case."""
    st, _ = _case((320, 320, 64), 77)
    dz = _dz(64, "uniform")
    cfg = SgsConfig.from_bc((2, 2, 2, 2, 1, 0))
    dev = on_device({k: st[k] for k in ("u", "v", "w", "theta", "rho", "qv")})
    args = cuda.smagorinsky_args(dev, dz, SGS_GRID, cfg, memory=cuda.MEMORY_DEVICE)
    for _ in range(2):
        ctx.check(ctx.smagorinsky_fused(args))
    ctx.synchronize()
    want = o32.smagorinsky(st, dz, SGS_GRID, cfg)
    for k, v in args.outputs.items():
        assert_bitwise(v.cpu().numpy(), want[k], k)


@pytest.mark.parametrize("bc,dt_sgs", [((2, 2, 2, 2, 1, 0), 1.0), ((0, 0, 2, 3, 0, 0), 4.0)])
def test_resident_run_with_sgs_matches_oracle(ctx, o32, bc, dt_sgs):
    """Two large steps of the plain path with the Smagorinsky integration
    between the Kessler step and the EOS projection, against the oracle's
    large step with the same closure: bit for bit."""
    from nimbus_b200.run import PROGNOSTIC, ResidentRun

    case = Case(24, 20, 16, 1000.0, 1000.0, 500.0, 3.0, seed=12, bc=bc, substeps=6)
    st, base = cloudy_state(case, seed=12)
    cfg = SgsConfig.from_bc(bc, dt_sgs=dt_sgs)
    run = ResidentRun(ctx, case, {k: v.copy() for k, v in st.items()}, base, precision=cuda.PRECISION_REFERENCE,
                      autotune=False, sgs=cfg)
    want = {k: v.copy() for k, v in st.items()}
    for step in range(2):
        run.step()
        o32.large_step(want, base, (case.dx, case.dy, case.dz), case.dt, run.n_substeps, case.bc, sgs=cfg,
                       time_s=step * case.dt)
    got = run.download()
    for k in PROGNOSTIC:
        assert_bitwise(got[k], want[k], k)
    assert run.sgs_substeps == 2 * int(np.ceil(case.dt / dt_sgs))


@pytest.mark.parametrize("shape,bc,kw,dzkind", DEVICE_CASES[:4], ids=[str(c[0]) for c in DEVICE_CASES[:4]])
def test_fp32_closure_error_against_fp64(shape, bc, kw, dzkind):
    """The FP32 form of the closure (an FP32-precision context) against the
    FP64 oracle on the same FP32 inputs: every output within 1e-6 relative L2
    and 1e-6 of its largest magnitude (measured: at most 2.8e-7 and 4.2e-7),
    where the reference-precision closure's error is only its final FP32
    rounding (about 3e-8)."""
    o64 = oracle.Restatement("f64")
    st, _ = _case(shape, sum(shape))
    dz = _dz(shape[2], dzkind)
    cfg = SgsConfig.from_bc(bc, **kw)
    c32 = cuda.Context(0)
    c32.set_precision(cuda.PRECISION_FP32)
    dev = on_device({k: st[k] for k in ("u", "v", "w", "theta", "rho", "qv")})
    args = cuda.smagorinsky_args(dev, dz, SGS_GRID, cfg, memory=cuda.MEMORY_DEVICE)
    c32.check(c32.smagorinsky_fused(args))
    c32.synchronize()
    ref = o64.smagorinsky({k: v.astype(np.float64) for k, v in st.items()}, dz, SGS_GRID, cfg)
    for k, v in args.outputs.items():
        got = v.cpu().numpy().astype(np.float64)
        norm = np.linalg.norm(ref[k])
        if norm == 0.0:
            assert np.all(got == 0.0), k
            continue
        assert np.linalg.norm(got - ref[k]) / norm <= 1e-6, k
        assert np.abs(got - ref[k]).max() <= 1e-6 * np.abs(ref[k]).max(), k
    c32.close()
