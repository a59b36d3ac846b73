"""The CUDA backend behind the reference's own C++ interface: the adapter
library (nimbus_b200/reference_backend/nimbus_compute_backend.cpp) loaded as a
ComputeBackend by the reference-linked harness, driven with the reference's
dispatch structs and, for the Smagorinsky closure, by the reference's own
SmagorinskyScheme::compute taking its native-backend path.  The results must
equal the reference's CPU backend / CPU path bit for bit, except for the
operators the reference defines in FP32 on its device route (Kessler, the
slow tendencies), which must agree with its CPU route within the
reference's own parity tiers."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from nimbus_b200.initial import Case, cloudy_state, perturbed_state
from nimbus_b200.sgs import SgsConfig
from tests.golden.make_golden import close_walls

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.reference_available(),
                                                   reason="reference harness not built")]

ADAPTER = Path(__file__).resolve().parents[1] / "nimbus_b200" / "lib" / "libnimbus_reference_backend.so"


# The reference's own GPU-vs-CPU parity tiers (src/compute/parity_comparison.cpp:115-123,
# include/compute/parity_types.hpp:12-22): |gpu - cpu| <= abs + rel |cpu| as
# (rel, abs); its runtime checks the slow-tendency kernel against the CPU
# route with the stencil tier (cartesian_cgrid_3d.cpp:983-998).
STENCIL_TIER = (1e-4, 5e-5)
MICROPHYSICS_TIER = (1e-4, 1e-7)
MICROPHYSICS_HEATING_TIER = (1e-4, 6e-4)


def assert_tier(got, want, tier, what):
    rel, abs_ = tier
    bad = np.abs(got.astype(np.float64) - want) > abs_ + rel * np.abs(want.astype(np.float64))
    assert not bad.any(), (f"{what}: {np.count_nonzero(bad)} cells outside the tier, max |diff| "
                           f"{np.abs(got.astype(np.float64) - want).max():.3e}")


@pytest.fixture(scope="module")
def ref():
    if not ADAPTER.exists():
        pytest.fail(f"{ADAPTER} missing: build it with python -m nimbus_b200.build where the reference headers are")
    return oracle.ReferenceHarness(threads=4)


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


@pytest.mark.parametrize("seed", [3, 4])
def test_fused_substep_through_the_reference_interface(ref, seed):
    """AcousticSubstepFusedCartesianCgridDispatch through the reference's CPU
    backend and through the CUDA backend's adapter: identical fields and
    continuity tendency."""
    case = Case(33, 27, 19, 1000.0, 1000.0, 500.0, 6.0, seed=seed)
    st, base = perturbed_state(case, seed=seed)
    a = {k: v.copy() for k, v in st.items()}
    b = {k: v.copy() for k, v in st.items()}
    da = np.zeros(case.shape, np.float32)
    db = np.zeros(case.shape, np.float32)
    for _ in range(3):
        ref.acoustic_fused(a, base["rho0"], base["p0"], 0.6, (case.dx, case.dy, case.dz), da)
        ref.acoustic_fused(b, base["rho0"], base["p0"], 0.6, (case.dx, case.dy, case.dz), db, backend=ADAPTER)
    for k in ("u", "v", "w", "rho", "p"):
        assert np.array_equal(bits(a[k]), bits(b[k])), k
    assert np.array_equal(bits(da), bits(db))


@pytest.mark.parametrize("bc,kw", [((2, 2, 2, 2, 1, 0), {}), ((0, 0, 1, 4, 1, 0), {"filter_width": "dx"}),
                                   ((1, 1, 1, 1, 1, 0), {"use_vertical": False})])
def test_smagorinsky_scheme_takes_the_cuda_backend(ref, bc, kw):
    """SmagorinskyScheme::compute with the adapter as the level's backend (its
    native path: dispatch_smagorinsky_fused_backend) against the same call on
    the CPU path.  The bridge hands the backend FP32 copies of the closure
    constants and spacings; with FP32-representable values the two paths agree
    bit for bit."""
    case = Case(30, 26, 18, 500.0, 625.0, 250.0, 3.0, seed=9)
    st, _ = cloudy_state(case, seed=9)
    rng = np.random.default_rng(9)
    for k in "uvw":
        st[k] = (st[k] + rng.standard_normal(case.shape).astype(np.float32) * 2.0).astype(np.float32)
    cfg = SgsConfig.from_bc(bc, Cs=0.25, Pr_t=0.5, Sc_t=0.5, nu_t_max=512.0, K_max=1024.0, **kw)
    dz = np.full(case.nz, case.dz)
    grid = (case.dx, case.dy, case.dz)
    cpu = ref.smagorinsky(st, dz, grid, cfg)
    gpu = ref.smagorinsky(st, dz, grid, cfg, backend=ADAPTER)
    for k in cpu:
        assert np.array_equal(bits(cpu[k]), bits(gpu[k])), k


@pytest.mark.parametrize("bc", [(1, 1, 1, 1, 1, 0), (0, 0, 2, 3, 0, 2)])
def test_batched_loop_through_the_reference_interface(ref, bc):
    """AcousticSubstepsBatchedCartesianCgridDispatch (the reference's
    accelerator route for the acoustic loop) through the adapter.  The
    dispatch carries FP32 profiles, spacings and dt_small: the adapter's
    result equals the C-ABI loop given those values widened to FP64, bit for
    bit, and the reference's CPU loop within the FP32 narrowing of its inputs."""
    from nimbus_b200 import cuda

    case = Case(36, 30, 20, 1000.0, 1000.0, 500.0, 6.0, seed=5, bc=bc)
    st, base = perturbed_state(case, seed=5)
    close_walls(st, bc)  # rigid walls start impermeable, as the solver's initial closure leaves them
    n, dt = 6, 6.0
    grid = (case.dx, case.dy, case.dz)
    got = {k: v.copy() for k, v in st.items()}
    out = ref.acoustic_batched(got, base["rho0"], base["p0"], dt / n, n, grid, bc, ADAPTER)
    # The same loop through the C-ABI on the widened FP32 inputs.
    ctx = cuda.Context(0)
    want = {k: v.copy() for k, v in st.items()}
    widen = lambda x: np.asarray(x, np.float32).astype(np.float64)  # noqa: E731
    mf = [np.zeros(case.shape, np.float32) for _ in range(3)]
    wave = np.zeros(2 * (case.nx + case.ny) * case.nz, np.float32)
    args = cuda.batched_args(want, widen(base["rho0"]), widen(base["p0"]), float(np.float32(dt / n)), n,
                             tuple(float(np.float32(g)) for g in grid), bc, *mf, 1.0 / n, None, wave)
    args.gamma = float(np.float32(args.gamma))
    ctx.check(ctx.acoustic_batched(args))
    ctx.close()
    for k in ("u", "v", "w", "rho", "p"):
        assert np.array_equal(bits(got[k]), bits(want[k])), k
    for k, m in zip(("mfx", "mfy", "mfz"), mf):
        assert np.array_equal(bits(out[k]), bits(m)), k
    assert np.array_equal(bits(out["wave"]), bits(wave))
    # Against the reference's CPU loop on the FP64 inputs.
    cpu = {k: v.copy() for k, v in st.items()}
    ref.acoustic_loop(cpu, base["rho0"], base["p0"], dt, n, grid, bc)
    for k in ("u", "v", "w", "rho", "p"):
        a, b = got[k].astype(np.float64), cpu[k].astype(np.float64)
        scale = max(np.abs(b).max(), 1e-30)
        assert np.abs(a - b).max() <= 1e-4 * scale, (k, np.abs(a - b).max(), scale)


@pytest.mark.parametrize("bc_name", ["radiative_slip_rigidlid", "periodic_noslip_open", "mixed_walls_sponge"])
@pytest.mark.parametrize("weno", [True, False], ids=["weno5", "mc"])
def test_transport_through_the_reference_bridge(ref, bc_name, weno):
    """The coupled scalar transport through the reference's own bridge
    (dispatch_advect_scalars_conservative_cartesian_cgrid_backend) with the
    arguments advect_thermodynamics_impl passes: the CUDA backend's adapter
    against the reference's CPU backend on the same retained fluxes, and both
    against the direct CPU call.  Bit for bit."""
    from tests.golden.make_golden import BC_SETS
    bc = BC_SETS[bc_name]
    o32 = oracle.Restatement("f32")
    case = Case(29, 23, 17, 800.0, 900.0, 400.0, 4.0, seed=21)
    st, base = cloudy_state(case, seed=21)
    close_walls(st, bc)
    grid = (case.dx, case.dy, case.dz)
    a = {k: v.copy() for k, v in st.items()}
    loop = o32.acoustic_loop(a, base["rho0"], base["p0"], 4.0, 9, grid, bc)
    args = (a["u"], a["v"], a["w"], a["rho"], loop["rho_begin"], loop["mfx"], loop["mfy"], loop["mfz"], 4.0, grid)
    names = ("theta", "qv", "qc", "qr")
    direct = [a[k].copy() for k in names]
    cpu = [a[k].copy() for k in names]
    cuda_route = [a[k].copy() for k in names]
    ref.scalar_transport(direct, [0, 1, 1, 1], *args, weno=weno, top_open=bc[5] == 2)
    assert ref.bridge_scalar_transport(cpu, [0, 1, 1, 1], *args, weno=weno, top_open=bc[5] == 2)
    assert ref.bridge_scalar_transport(cuda_route, [0, 1, 1, 1], *args, weno=weno, top_open=bc[5] == 2,
                                       backend=ADAPTER)
    for k, x, y, z in zip(names, direct, cpu, cuda_route):
        assert np.array_equal(bits(x), bits(y)), k
        assert np.array_equal(bits(y), bits(z)), k


@pytest.mark.parametrize("sanitize,observed,pbl", [(True, False, True), (True, True, False), (False, True, True)])
def test_slow_apply_through_the_reference_bridge(ref, sanitize, observed, pbl):
    """dispatch_slow_apply_backend (the accelerator route of the slow apply;
    the reference's CPU backend declines it) with the CUDA backend's adapter:
    apply_slow_tendencies_cpu's arithmetic bit for bit (dt FP32-representable),
    boundary-layer tendencies added, non-finite tendencies zeroed under the
    repairs, and the committed fields handed to the completion observer
    before the host fields change."""
    rng = np.random.default_rng(5)
    shape = (23, 17, 11)
    st = {k: rng.uniform(-30, 30, shape).astype(np.float32) for k in "uvw"}
    st["p"] = rng.uniform(5e4, 1e5, shape).astype(np.float32)
    tend = [rng.uniform(-1, 1, shape).astype(np.float32) for _ in range(3)] + \
        [rng.uniform(-20, 20, shape).astype(np.float32)]
    tend[0][1, 2, 3] = np.nan
    tend[3][4, 4, 4] = np.inf
    tend[1][0, 0, 0] = -0.0
    st["v"][0, 0, 0] = -0.0
    pbl_fields = (rng.uniform(-0.1, 0.1, shape).astype(np.float32),
                  rng.uniform(-0.1, 0.1, shape).astype(np.float32)) if pbl else None
    dt = 3.0
    f64 = np.float64
    want = {}
    for k, t, extra in (("u", tend[0], pbl_fields[0] if pbl else None), ("v", tend[1], pbl_fields[1] if pbl else None),
                        ("w", tend[2], None), ("p", tend[3], None)):
        ts = t.astype(f64) + (extra.astype(f64) if extra is not None else 0.0)
        if sanitize:
            ts = np.where(np.isfinite(ts), ts, 0.0)
        with np.errstate(invalid="ignore"):
            want[k] = (st[k].astype(f64) + ts * dt).astype(np.float32)
    cpu = {k: v.copy() for k, v in st.items()}
    assert ref.bridge_slow_apply(cpu, tend, dt, pbl_fields, sanitize) == (False, None)
    for k in st:
        assert np.array_equal(bits(cpu[k]), bits(st[k])), "a declined dispatch leaves the fields untouched"
    got = {k: v.copy() for k, v in st.items()}
    ok, extra = ref.bridge_slow_apply(got, tend, dt, pbl_fields, sanitize, observed=observed, backend=ADAPTER)
    assert ok
    for k in st:
        assert np.array_equal(bits(got[k]), bits(want[k])), k
    if observed:
        committed, calls = extra
        assert calls == 1
        for k in st:
            assert np.array_equal(bits(committed[k]), bits(want[k])), k


def test_state_relaxation_through_the_reference_bridge(ref):
    """dispatch_state_relaxation_cartesian_backend with the profile block
    try_state_relaxation_gpu packs (FP32 rows) and its completion observer:
    the adapter equals the C-ABI on the widened FP32 profiles bit for bit, and
    the reference's CPU sponge (FP64 profiles) within that narrowing."""
    from nimbus_b200 import cuda
    from nimbus_b200.sponge import SpongeConfig, SpongeProfiles

    cfg = SpongeConfig(z_damp=-1.0, alpha_max=0.05, w_only_cells=6, w_only_alpha_max=0.2, lateral_width=7,
                       lateral_alpha_max=0.05, implicit_mode=0, wind=(2.0, 1.0, 8.0, 4.0, 20.0, 10.0))
    case = Case(30, 26, 24, 500.0, 600.0, 400.0, 3.0, seed=6)
    st, base = cloudy_state(case, seed=6)
    fields = {k: st[k].copy() for k in ("u", "v", "w", "theta")}
    cpu = {k: v.copy() for k, v in fields.items()}
    prof = ref.state_relaxation(cpu, base["theta0"], (case.dx, case.dy, case.dz), case.dt, cfg)
    nz = case.nz
    block = np.zeros((7, nz), np.float32)
    block[0], block[1] = prof["alpha"], prof["w_only_alpha"]
    block[2], block[3] = prof["u_ref"], prof["v_ref"]
    block[4] = base["theta0"]
    block[5, :cfg.lateral_width] = prof["lateral_alpha"]
    block[6] = prof["upper_w_alpha"]
    flags = (1, 1, 1)
    got = {k: v.copy() for k, v in fields.items()}
    calls = ref.bridge_state_relaxation(got, block, cfg.lateral_width, flags, np.float32(case.dt), backend=ADAPTER)
    assert calls == 1
    wide = block.astype(np.float64)
    P = SpongeProfiles(alpha=wide[0], upper_w_alpha=wide[6], w_only_alpha=wide[1], u_ref=wide[2], v_ref=wide[3],
                       theta_ref=wide[4], lateral_alpha=wide[5, :cfg.lateral_width].copy(), staggered=1,
                       implicit_mode=0)
    ctx = cuda.Context(0)
    mine = {k: v.copy() for k, v in fields.items()}
    ctx.check(ctx.state_relaxation(cuda.state_relaxation_args(mine, P, float(np.float32(case.dt)))))
    ctx.close()
    for k in fields:
        assert np.array_equal(bits(got[k]), bits(mine[k])), k
        scale = np.abs(cpu[k]).max() + 1e-30
        assert np.abs(got[k].astype(np.float64) - cpu[k]).max() / scale < 1e-5, k


def test_kessler_scheme_takes_the_cuda_backend(ref):
    """KesslerScheme::compute_tendencies with the adapter as its backend: the
    scheme's device route (host saturation adjustment, then the adapter's
    dispatch_kessler_pointwise and dispatch_kessler_sedimentation, the scheme
    refusing to fall back) against the same call on its CPU route.  The
    reference defines these operators in FP32 and books the adjustment in a
    different order on that route, so the routes agree within FP32 rounding:
    here within 1e-4 of each field's largest magnitude."""
    from tests.test_kessler_dispatch_gpu import kessler_inputs

    raw = kessler_inputs((22, 19, 30), 9)
    # theta from temperature (the scheme takes theta and converts it back).
    theta = (raw["T"].astype(np.float64) * (1.0e5 / raw["p"].astype(np.float64)) ** (287.04 / 1004.0))
    st = {"theta": np.ascontiguousarray(theta, np.float32), "p": raw["p"], "rho": raw["rho"], "qv": raw["qv"],
          "qc": raw["qc"], "qr": raw["qr"]}
    nx, ny, nz = st["p"].shape
    domain = (1, nx - 1, 1, ny - 1, 0, nz)
    cpu = ref.kessler_tendencies(st, 400.0, 3.0, domain)
    dev = ref.kessler_tendencies(st, 400.0, 3.0, domain, backend=ADAPTER)
    for name, a, b in zip(("dtheta", "dqv", "dqc", "dqr"), cpu, dev):
        scale = float(np.abs(a).max())
        err = float(np.abs(a.astype(np.float64) - b).max())
        assert scale > 0 and err <= 1e-4 * scale, f"{name}: {err:.3e} against {scale:.3e}"
        # The reference's own microphysics parity tiers (parity_comparison.cpp:119-122).
        assert_tier(b, a, MICROPHYSICS_HEATING_TIER if name == "dtheta" else MICROPHYSICS_TIER, name)


def _slow_level(seed, wind=True):
    case = Case(30, 26, 22, 800.0, 700.0, 400.0, 3.0, seed=seed, noise_amp=0.3)
    st, base = cloudy_state(case, seed=seed + 1)
    if not wind:
        base = dict(base, u0=np.zeros_like(base["u0"]), v0=np.zeros_like(base["v0"]))
    return case, st, base


@pytest.mark.parametrize("moist,cor,beta", [(True, 1e-4, 0.0), (False, 0.0, 0.0), (True, 1e-4, 2e-11)],
                         ids=["moist-f", "dry", "beta-plane"])
def test_slow_tendencies_scheme_takes_the_cuda_backend(ref, moist, cor, beta):
    """CartesianCGrid3DScheme::compute_slow_tendencies with the adapter as the
    level's backend takes its device route (dispatch_cartesian_cgrid_slow_tendencies:
    FP32 profiles, the host-summed hydrometeor loading) and agrees with its
    CPU route within the reference's stencil tier over the whole field."""
    case, st, base = _slow_level(21)
    grid = (case.dx, case.dy, case.dz)
    cpu = ref.slow_tendencies(st, base, grid, coriolis_f=cor, moist=moist, beta=beta)
    dev = ref.slow_tendencies(st, base, grid, coriolis_f=cor, moist=moist, beta=beta, backend=ADAPTER)
    for name, a, b in zip(("du", "dv", "dw", "dp"), cpu, dev):
        assert np.abs(a).max() > 0, name
        assert_tier(b, a, STENCIL_TIER, name)


@pytest.mark.parametrize("memory", ["host", "device"])
def test_slow_tendency_operator_through_the_c_abi(ref, memory):
    """nimbus_cuda_cgrid_slow_tendencies called directly with the dispatch's
    inputs (FP32 profiles, loading = qc + qr), host or device memory, with the
    advection components: the stencil tier against the CPU route, drho zero,
    and du = advection + Coriolis exactly as the components say."""
    import torch

    from nimbus_b200 import cuda

    case, st, base = _slow_level(31)
    grid = (case.dx, case.dy, case.dz)
    cpu = ref.slow_tendencies(st, base, grid, coriolis_f=1e-4, moist=True)
    prof = {k: np.ascontiguousarray(base[k], np.float32) for k in ("rho0", "qv0", "u0", "v0")}
    load = np.ascontiguousarray(st["qc"] + st["qr"], np.float32)
    fields = {k: st[k] for k in ("u", "v", "w", "rho", "p", "qv")}
    outs = [np.full_like(st["u"], np.nan) for _ in range(5)]
    adv = [np.full_like(st["u"], np.nan) for _ in range(3)]
    ctx = cuda.Context(0)
    try:
        if memory == "device":
            d = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
            dfields = {k: d(v) for k, v in fields.items()}
            dprof = {k: d(v) for k, v in prof.items()}
            douts, dadv = [d(a) for a in outs], [d(a) for a in adv]
            ctx.cgrid_slow_tendencies(dfields, dprof, douts, grid, coriolis_f=1e-4, loading=d(load), advection=dadv)
            ctx.synchronize()
            outs, adv = [a.cpu().numpy() for a in douts], [a.cpu().numpy() for a in dadv]
        else:
            ctx.cgrid_slow_tendencies(fields, prof, outs, grid, coriolis_f=1e-4, loading=load, advection=adv)
    finally:
        ctx.close()
    du, dv, dw, drho, dp = outs
    for name, a, b in zip(("du", "dv", "dw", "dp"), cpu, (du, dv, dw, dp)):
        assert_tier(b, a, STENCIL_TIER, name)
    assert np.all(drho == 0.0)
    assert np.all(np.isfinite(adv[0])) and np.abs(adv[2]).max() > 0
