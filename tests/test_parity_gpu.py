"""CUDA path against the reference, bit for bit.

The golden fixtures were produced by the reference CPU solver itself
(tests/golden/make_golden.py); the CUDA kernels run in reference precision
(FP64 interior arithmetic over FP32 storage, no contracted FMA), so every
stored value must be identical -- the tolerance is zero ULP.  Larger seeded
cases compare against the oracle restatement, itself pinned bit-exact to the
reference (tests/test_oracle.py)."""
import glob

import numpy as np
import pytest

import oracle
from nimbus_b200 import cuda
from nimbus_b200.initial import Case, cloudy_state, initial_state, perturbed_state
from tests.golden.make_golden import BC_SETS, close_walls

pytestmark = pytest.mark.gpu

GOLDEN = sorted(glob.glob("tests/golden/loop_*.npz"))


@pytest.fixture(scope="module", params=[cuda.SUBSTEP_FUSED, cuda.SUBSTEP_SPLIT], ids=["fused", "split"])
def ctx(request):
    """A reference-precision context, once per substep form: every form must
    reproduce the reference bit for bit."""
    c = cuda.Context(0)
    c.set_precision(cuda.PRECISION_REFERENCE)
    c.set_substep_form(request.param)
    yield c
    c.close()


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


def _state(g, prefix="in_"):
    return {k[len(prefix):]: g[k].copy() for k in g.files if k.startswith(prefix)}


def assert_bitwise(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    bad = np.count_nonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad == 0, f"{what}: {bad}/{a.size} values differ, max |diff| {np.abs(a - b).max():.3e}"


def run_loop(ctx, st, rho0, p0, dt, n, grid, bc, wave_in=None):
    shape = st["u"].shape
    mf = [np.zeros(shape, np.float32) for _ in range(3)]
    rb = np.zeros(shape, np.float32)
    wave = np.zeros(2 * (shape[0] + shape[1]) * shape[2], np.float32)
    ctx.check(ctx.acoustic_batched(cuda.batched_args(st, rho0, p0, dt / n, n, grid, bc, *mf, (dt / n) / dt, wave_in,
                                                     wave, rb)))
    return dict(mfx=mf[0], mfy=mf[1], mfz=mf[2], rho_begin=rb, wave=wave)


def test_fused_substep_matches_reference(ctx):
    g = np.load("tests/golden/fused_substep.npz")
    st = _state(g)
    drho = np.zeros_like(st["u"])
    ctx.check(ctx.acoustic_fused(cuda.fused_args(st, g["rho0"], g["p0"], float(g["dt_small"]), tuple(g["grid"]),
                                                 drho)))
    for k in ("u", "v", "w", "rho", "p"):
        assert_bitwise(st[k], g["out_" + k], k)
    assert_bitwise(drho, g["out_drho"], "drho")


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.split("/")[-1])
def test_acoustic_loop_and_transport_match_reference(ctx, path):
    g = np.load(path)
    st = _state(g)
    bc = tuple(int(x) for x in g["bc"])
    dt, n = float(g["dt_large"]), int(g["n_substeps"])
    out = run_loop(ctx, st, g["rho0"], g["p0"], dt, n, tuple(g["grid"]), bc)
    for k in ("u", "v", "w", "rho", "p"):
        assert_bitwise(st[k], g["out_" + k], k)
    for k in ("mfx", "mfy", "mfz", "rho_begin", "wave"):
        assert_bitwise(out[k], g["out_" + k], k)
    src = _state(g)
    for tag, weno in (("weno", 1), ("mc", 0)):
        qi = [src[k].copy() for k in ("theta", "qv", "qc", "qr")]
        qo = [np.zeros_like(q) for q in qi]
        ctx.check(ctx.scalar_transport(cuda.transport_args(
            qi, qo, [0, 1, 1, 1], g["out_rho"], g["out_rho_begin"], g["out_mfx"], g["out_mfy"], g["out_mfz"], dt,
            tuple(g["grid"]), weno=weno, top_open=bc[5] == 2)))
        for key, q in zip(("theta", "qv", "qc", "qr"), qo):
            assert_bitwise(q, g[f"tr{tag}_{key}"], f"{tag} {key}")


@pytest.mark.parametrize("bc_name", list(BC_SETS))
def test_seeded_loop_vs_oracle_ragged_grid(ctx, o32, bc_name):
    """Odd, non-power-of-two extents and a carried-in wave history."""
    bc = BC_SETS[bc_name]
    grid = (700.0, 650.0, 330.0)
    case = Case(37, 29, 23, *grid, 5.0, seed=7)
    st, base = perturbed_state(case, seed=8)
    close_walls(st, bc)
    gpu = {k: v.copy() for k, v in st.items()}
    cpu = {k: v.copy() for k, v in st.items()}
    out = run_loop(ctx, gpu, base["rho0"], base["p0"], 5.0, 11, grid, bc)
    ref = o32.acoustic_loop(cpu, base["rho0"], base["p0"], 5.0, 11, grid, bc)
    for k in ("u", "v", "w", "rho", "p"):
        assert_bitwise(gpu[k], cpu[k], k)
    for k in out:
        assert_bitwise(out[k], ref[k], k)
    # second large step continues from the carried KW78 history
    wave_in = out["wave"].copy()
    out2 = run_loop(ctx, gpu, base["rho0"], base["p0"], 5.0, 11, grid, bc, wave_in=wave_in)
    assert out2["wave"].shape == wave_in.shape and np.isfinite(out2["wave"]).all()


def test_minimum_grid_and_in_place_transport(ctx, o32):
    """The reference's minimum extents (4x4x2 batched) and in-place scalars."""
    grid = (500.0, 500.0, 250.0)
    case = Case(4, 4, 2, *grid, 2.0)
    st, base = perturbed_state(case, seed=3)
    gpu = {k: v.copy() for k, v in st.items()}
    cpu = {k: v.copy() for k, v in st.items()}
    bc = (1, 1, 1, 1, 1, 0)
    out = run_loop(ctx, gpu, base["rho0"], base["p0"], 2.0, 3, grid, bc)
    ref = o32.acoustic_loop(cpu, base["rho0"], base["p0"], 2.0, 3, grid, bc)
    for k in ("u", "v", "w", "rho", "p"):
        assert_bitwise(gpu[k], cpu[k], k)
    qs = [gpu["theta"].copy(), gpu["qv"].copy()]
    ctx.check(ctx.scalar_transport(cuda.transport_args(qs, qs, [0, 1], gpu["rho"], out["rho_begin"], out["mfx"],
                                                       out["mfy"], out["mfz"], 2.0, grid)))
    qr = [cpu["theta"].copy(), cpu["qv"].copy()]
    o32.scalar_transport(qr, [0, 1], cpu["rho"], ref["rho_begin"], ref["mfx"], ref["mfy"], ref["mfz"], 2.0, grid)
    for a, b in zip(qs, qr):
        assert_bitwise(a, b, "scalar")


def test_hydrostatic_identity(ctx):
    """A resting base state is a fixed point of the substep to within a few ULP
    (the reference's hydrostatic-identity parity case)."""
    case = Case(12, 10, 16, 1000.0, 1000.0, 500.0, 6.0, bubble_amp=0.0)
    st, base = initial_state(case)
    for k in ("u", "v", "w"):
        st[k][:] = 0.0
    before = {k: v.copy() for k, v in st.items()}
    ctx.check(ctx.acoustic_fused(cuda.fused_args(st, base["rho0"], base["p0"], 0.6, (1000.0, 1000.0, 500.0))))
    for k in ("rho", "p"):
        rel = np.abs(st[k].astype(np.float64) - before[k]) / np.abs(before[k])
        assert rel.max() <= 8 * np.finfo(np.float32).eps, (k, rel.max())
    assert np.abs(st["w"]).max() < 1e-3


def test_refused_dispatch_leaves_host_fields_untouched(ctx):
    case = Case(8, 8, 4, 1000.0, 1000.0, 500.0, 6.0)
    st, base = perturbed_state(case)
    before = {k: v.copy() for k, v in st.items()}
    args = cuda.fused_args(st, base["rho0"], base["p0"], -1.0, (1000.0, 1000.0, 500.0))  # dt < 0
    rc = ctx.acoustic_fused(args)
    assert rc == 1 and "dt_small" in ctx.last_error
    args = cuda.fused_args(st, base["rho0"], base["p0"], 0.5, (1000.0, 1000.0, 500.0))
    args.rho_min = 3.0  # rho_min > rho_max
    assert ctx.acoustic_fused(args) == 1
    for k in st:
        assert_bitwise(st[k], before[k], k)


def test_nonfinite_mass_flux_is_reported_not_published(ctx):
    case = Case(8, 8, 4, 1000.0, 1000.0, 500.0, 6.0)
    st, base = perturbed_state(case)
    shape = case.shape
    mf = [np.zeros(shape, np.float32) for _ in range(3)]
    mf[0][3, 3, 1] = np.float32(3.4e38)  # the next weighted add overflows the FP32 store
    st["u"][3, 3, 1] = 150.0
    before = {k: v.copy() for k, v in st.items()}
    wave = np.zeros(2 * (8 + 8) * 4, np.float32)
    args = cuda.batched_args(st, base["rho0"], base["p0"], 0.5, 2, (1000.0, 1000.0, 500.0), (1, 1, 1, 1, 1, 0),
                             *mf, 1e36, None, wave)
    rc = ctx.acoustic_batched(args)
    assert rc == 4, ctx.last_error   # NIMBUS_ERR_NONFINITE
    for k in st:
        assert_bitwise(st[k], before[k], k)


def _slow_case(g):
    st = {k[3:]: g[k].copy() for k in g.files if k.startswith("in_")}
    base = {k[5:]: g[k] for k in g.files if k.startswith("base_")}
    return st, base


def test_slow_tendencies_match_reference(ctx):
    g = np.load("tests/golden/slow_tendencies.npz")
    st, base = _slow_case(g)
    grid = tuple(g["grid"])
    for moist, cor, prefix in ((True, float(g["coriolis_f"]), "out_"), (False, 0.0, "dry_")):
        outs = tuple(np.zeros_like(st["u"]) for _ in range(4))
        ctx.check(ctx.slow_tendencies(cuda.slow_args(st, base, grid, coriolis_f=cor, moist=moist, outputs=outs)))
        for key, arr in zip(("du", "dv", "dw", "dp"), outs):
            assert_bitwise(arr, g[prefix + key], prefix + key)


def test_slow_heun_step_matches_oracle(ctx, o32):
    case = Case(23, 19, 17, 500.0, 550.0, 300.0, 3.0, seed=13)
    st, base = perturbed_state(case, seed=14)
    gpu = {k: v.copy() for k, v in st.items()}
    cpu = {k: v.copy() for k, v in st.items()}
    outs = tuple(np.zeros_like(st["u"]) for _ in range(4))
    ctx.check(ctx.slow_step(cuda.slow_args(gpu, base, (500.0, 550.0, 300.0), dt_large=3.0, coriolis_f=1e-4,
                                           outputs=outs)))
    o32.slow_rk2_step(cpu, base, (500.0, 550.0, 300.0), 3.0, coriolis_f=1e-4)
    for k in ("u", "v", "w", "p"):
        assert_bitwise(gpu[k], cpu[k], k)


@pytest.mark.parametrize("dom", ["cgrid", "full"])
def test_kessler_tendencies_match_reference(ctx, dom):
    g = np.load("tests/golden/kessler_eos.npz")
    st = _state(g)
    outs = tuple(np.zeros_like(st["theta"]) for _ in range(4))
    ctx.check(ctx.kessler_tendencies(cuda.kessler_args(st, float(g["dz"]), float(g["dt"]), tuple(g["dom_" + dom]),
                                                       outputs=outs)))
    for key, arr in zip(("dtheta", "dqv", "dqc", "dqr"), outs):
        assert_bitwise(arr, g[f"{dom}_{key}"], key)


def test_kessler_step_matches_oracle(ctx, o32):
    case = Case(33, 27, 31, 700.0, 800.0, 350.0, 4.0, seed=21)
    st, _ = cloudy_state(case, seed=21)
    gpu = {k: v.copy() for k, v in st.items()}
    cpu = {k: v.copy() for k, v in st.items()}
    outs = tuple(np.zeros_like(st["theta"]) for _ in range(4))
    ctx.check(ctx.kessler_step(cuda.kessler_args(gpu, 350.0, 4.0, outputs=outs)))
    want = o32.kessler_step(cpu, 350.0, 4.0, cuda.cgrid_cell_domain(*case.shape))
    for key, a, b in zip(("dtheta", "dqv", "dqc", "dqr"), outs, want):
        assert_bitwise(a, b, key)
    for k in ("theta", "qv", "qc", "qr"):
        assert_bitwise(gpu[k], cpu[k], k)
    # the step form without tendency outputs gives the same state
    again = {k: v.copy() for k, v in st.items()}
    ctx.check(ctx.kessler_step(cuda.kessler_args(again, 350.0, 4.0)))
    for k in ("theta", "qv", "qc", "qr"):
        assert_bitwise(again[k], cpu[k], k)


def test_eos_projection_matches_reference(ctx):
    g = np.load("tests/golden/kessler_eos.npz")
    st = _state(g)
    p = st["p"].copy()
    ctx.check(ctx.eos_projection(cuda.eos_args(p, st["rho"], st["theta"])))
    assert_bitwise(p, g["eos_p_dry"], "dry")
    p = st["p"].copy()
    ctx.check(ctx.eos_projection(cuda.eos_args(p, st["rho"], st["theta"], st["qv"], st["qc"], st["qr"])))
    assert_bitwise(p, g["eos_p_moist"], "moist")


# (field, cell, value, refused when dry, refused when moist), as pinned against
# the reference in tests/test_oracle.py.
EOS_CASES = [
    ("rho", (3, 3, 3), -1.0, True, True),
    ("theta", (0, 0, 0), np.nan, True, True),
    ("qv", (3, 3, 3), -1e-6, False, True),
    ("qv", (0, 3, 3), -1e-6, False, False),
    ("qc", (2, 2, 0), -1e-3, False, True),
    ("p", (4, 4, 4), 0.0, False, True),
]


@pytest.mark.parametrize("field,cell,value,dry_refused,moist_refused", EOS_CASES)
def test_eos_refusal_matches_oracle(ctx, o32, field, cell, value, dry_refused, moist_refused):
    case = Case(9, 7, 6, 1000.0, 1000.0, 500.0, 6.0, seed=1)
    st, _ = cloudy_state(case, seed=3)
    st[field][cell] = value
    for moist, refused in ((False, dry_refused), (True, moist_refused)):
        q = (st["qv"], st["qc"], st["qr"]) if moist else (None, None, None)
        gpu, cpu = st["p"].copy(), st["p"].copy()
        rc = ctx.eos_projection(cuda.eos_args(gpu, st["rho"], st["theta"], *q))
        assert o32.eos_projection(cpu, st["rho"], st["theta"], *q) == (not refused)
        assert rc == (4 if refused else 0), ctx.last_error
        assert_bitwise(gpu, cpu, f"{field} moist={moist}")


def test_eos_device_refusal_keeps_pressure(ctx):
    """Device memory: a refused projection publishes nothing and the refusal
    surfaces at synchronize."""
    import torch
    case = Case(12, 10, 8, 1000.0, 1000.0, 500.0, 6.0, seed=1)
    st, _ = cloudy_state(case, seed=4)
    st["rho"][5, 5, 5] = np.nan
    dev = {k: torch.from_numpy(st[k]).cuda() for k in ("p", "rho", "theta")}
    torch.cuda.synchronize()
    args = cuda.eos_args(dev["p"], dev["rho"], dev["theta"], memory=cuda.MEMORY_DEVICE, stream=ctx.stream)
    ctx.check(ctx.eos_projection(args))
    assert ctx.lib.nimbus_cuda_synchronize(ctx.handle) == 4
    assert_bitwise(dev["p"].cpu().numpy(), st["p"], "p")
    # a clean state publishes afterwards
    st["rho"][5, 5, 5] = 1.0
    dev["rho"].copy_(torch.from_numpy(st["rho"]))
    torch.cuda.synchronize()
    ctx.check(ctx.eos_projection(args))
    ctx.synchronize()
    want = st["p"].copy()
    oracle.Restatement("f32").eos_projection(want, st["rho"], st["theta"])
    assert_bitwise(dev["p"].cpu().numpy(), want, "p")


@pytest.fixture(scope="module")
def ctx32():
    c = cuda.Context(0)
    c.set_precision(cuda.PRECISION_FP32)
    yield c
    c.close()


def _fp32_transport(ctx32, g, scale=1.0):
    st = _state(g)
    grid = tuple(g["grid"])
    qs = [st[k] * np.float32(scale) for k in ("theta", "qv", "qc", "qr")]
    ctx32.check(ctx32.scalar_transport(cuda.transport_args(
        qs, qs, [0, 1, 1, 1], g["out_rho"], g["out_rho_begin"], g["out_mfx"], g["out_mfy"], g["out_mfz"],
        float(g["dt_large"]), grid, weno=True, top_open=int(g["bc"][5]) == 2)))
    return qs


def _rel(a, b):
    return float(np.linalg.norm((a.astype(np.float64) - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def _fp64_transport(g, scale=1.0):
    o64 = oracle.Restatement("f64")
    st = _state(g)
    ref = [st[k].astype(np.float64) * scale for k in ("theta", "qv", "qc", "qr")]
    f64 = lambda k: g[k].astype(np.float64)  # noqa: E731
    o64.scalar_transport(ref, [0, 1, 1, 1], f64("out_rho"), f64("out_rho_begin"), f64("out_mfx"), f64("out_mfy"),
                         f64("out_mfz"), float(g["dt_large"]), tuple(g["grid"]), weno=True,
                         top_open=int(g["bc"][5]) == 2)
    return ref


@pytest.mark.parametrize("path", GOLDEN, ids=lambda p: p.split("/")[-1])
def test_fp32_transport_tracks_fp64(ctx32, path):
    """The FP32 form's WENO5 transport against the FP64 oracle on the same
    retained fluxes: relative L2 within 1e-5 per scalar."""
    g = np.load(path)
    got = _fp32_transport(ctx32, g)
    ref = _fp64_transport(g)
    for name, a, b in zip(("theta", "qv", "qc", "qr"), got, ref):
        assert _rel(a, b) <= 1e-5, (name, _rel(a, b))
        if name != "theta":
            assert (a >= -1e-12).all(), name  # positive definite


def test_fp32_paired_faces_equal_single_faces(ctx32):
    """The FP32 faces evaluate scalars two at a time in paired f32x2
    instructions; a scalar gets the same bits whether it is paired (either
    lane) or evaluated alone."""
    g = np.load(GOLDEN[0])
    st = _state(g)
    grid = tuple(g["grid"])

    def run(names):
        qs = [st[k].copy() for k in names]
        ctx32.check(ctx32.scalar_transport(cuda.transport_args(
            qs, qs, [1] * len(qs), g["out_rho"], g["out_rho_begin"], g["out_mfx"], g["out_mfy"], g["out_mfz"],
            float(g["dt_large"]), grid, weno=True, top_open=int(g["bc"][5]) == 2)))
        return dict(zip(names, qs))

    runs = [run(("qv", "qc", "qr")), run(("qr", "qv", "qc")), run(("qc", "qr", "qv"))]
    for k in ("qv", "qc", "qr"):
        alone = run((k,))[k]
        for r in runs:
            assert np.array_equal(r[k].view(np.uint32), alone.view(np.uint32)), k


@pytest.mark.parametrize("scale", [1e-30, 1e-10, 1e10, 1e30])
def test_fp32_transport_across_scales(ctx32, scale):
    """Fields scaled anywhere from 1e-30 to 1e30 stay finite and track the
    FP64 oracle at the same scale (the FP32 form normalises each stencil by
    its magnitude; below the 1e-20 floor both forms fall back to the linear
    weights, as eps = 1e-6 max^2 + 1e-40 makes the reference do)."""
    g = np.load(GOLDEN[0])
    got = _fp32_transport(ctx32, g, scale)
    ref = _fp64_transport(g, scale)
    for a, b in zip(got, ref):
        assert np.isfinite(a).all()
        assert _rel(a, b) <= 1e-5


# ---- End-of-step sponge (state relaxation) ------------------------------------
@pytest.fixture(scope="module")
def rctx():
    c = cuda.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("name", ["explicit", "implicit"])
def test_state_relaxation_matches_reference(rctx, name):
    """nimbus_cuda_state_relaxation on host arrays against the reference's own
    apply_rayleigh_damping + apply_lateral_damping (golden fixture): 0 ULP."""
    from nimbus_b200.sponge import build_profiles
    from tests.test_oracle import _sponge_config

    g = np.load("tests/golden/state_relaxation.npz")
    P = build_profiles(_sponge_config(g, name), g["in_u"].shape[2], float(g["grid"][2]), g["theta0"])
    st = {k: g[f"in_{k}"].copy() for k in ("u", "v", "w", "theta")}
    rctx.check(rctx.state_relaxation(cuda.state_relaxation_args(st, P, float(g["dt"]))))
    for k in st:
        want = g[f"{name}_out_{k}"]
        assert np.count_nonzero(st[k].view(np.uint32) != want.view(np.uint32)) == 0, k


@pytest.mark.parametrize("seed", [41, 42, 43, 44])
def test_state_relaxation_device_memory_matches_oracle(rctx, o32, seed):
    """Device arrays, seeded configurations (lid absorber and lateral band on or
    off, explicit or implicit, unstaggered w): equal to the restatement, which
    the reference pins."""
    import torch

    from nimbus_b200.sponge import SpongeConfig, build_profiles

    rng = np.random.default_rng(seed)
    cfg = SpongeConfig(z_damp=float(rng.choice([-1.0, 1500.0])), alpha_max=float(rng.uniform(0.01, 0.3)),
                       w_only_cells=int(rng.integers(0, 7)), w_only_alpha_max=float(rng.uniform(0.05, 0.5)),
                       lateral_width=int(rng.integers(0, 12)), lateral_alpha_max=float(rng.uniform(0.0, 0.5)),
                       implicit_mode=int(rng.integers(0, 2)), wind=tuple(rng.uniform(-10, 20, 6)))
    case = Case(int(rng.integers(4, 40)), int(rng.integers(4, 40)), int(rng.integers(2, 30)), 500.0, 600.0, 300.0,
                4.0, seed=seed)
    st, base = cloudy_state(case, seed=seed)
    P = build_profiles(cfg, case.nz, case.dz, base["theta0"], staggered=bool(seed % 2))
    want = {k: st[k].copy() for k in ("u", "v", "w", "theta")}
    o32.state_relaxation(want, P, 4.0)
    dev = {k: torch.from_numpy(st[k].copy()).cuda() for k in want}
    rctx.check(rctx.state_relaxation(cuda.state_relaxation_args(dev, P, 4.0, memory=cuda.MEMORY_DEVICE)))
    rctx.synchronize()
    for k in want:
        got = dev[k].cpu().numpy()
        assert np.count_nonzero(got.view(np.uint32) != want[k].view(np.uint32)) == 0, k


def test_state_relaxation_refuses_invalid_rates(rctx):
    from nimbus_b200.sponge import SpongeConfig, build_profiles

    case = Case(10, 9, 8, 500.0, 500.0, 400.0, 3.0, seed=5)
    st, base = cloudy_state(case, seed=5)
    P = build_profiles(SpongeConfig(z_damp=200.0), case.nz, case.dz, base["theta0"])
    P.alpha[2] = float("nan")
    fields = {k: st[k].copy() for k in ("u", "v", "w", "theta")}
    rc = rctx.state_relaxation(cuda.state_relaxation_args(fields, P, 3.0))
    assert rc == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    for k in fields:
        assert np.array_equal(fields[k], st[k]), k


def test_device_info_reports_the_b200(ctx):
    """nimbus_cuda_device_info: what the adapter's populate_hardware_info and
    memory_properties report to the reference runtime."""
    info = ctx.device_info()
    assert info["cc"][0] == 10 and info["sm_count"] > 0 and info["name"]
    assert 0 < info["free_bytes"] <= info["total_bytes"]
