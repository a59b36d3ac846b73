"""The whole large step on the device, bit for bit against the oracle, and the
member engine against the per-operation path.

Reference precision: the plain path (one C-ABI call per operation) and the
engine (batched launches under a CUDA graph) must both reproduce the oracle's
composition of the pinned rows -- Heun slow step, boundary refresh, KW78 seed,
acoustic loop, WENO5 transport, Kessler, EOS -- with zero ULP.  FP32 form:
a member's result is identical alone and in any mix (no cross-member
arithmetic), and identical to the plain FP32 path (same kernels)."""
import numpy as np
import pytest

import oracle
from nimbus_b200 import cuda
from nimbus_b200.initial import Case, cloudy_state
from nimbus_b200.run import PROGNOSTIC, EngineRun, HostPipeline, ResidentRun

pytestmark = pytest.mark.gpu

BCS = {
    "radiative": (1, 1, 1, 1, 1, 0),
    "periodic_open": (0, 0, 0, 0, 0, 2),
    "walls_sponge": (2, 3, 4, 1, 1, 1),
}


def assert_bitwise(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    bad = np.count_nonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad == 0, f"{what}: {bad}/{a.size} values differ, max |diff| {np.abs(a - b).max():.3e}"


@pytest.fixture(scope="module")
def ctx():
    c = cuda.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


def _case(shape, bc, seed, dt=4.0, grid=(700.0, 800.0, 350.0)):
    return Case(*shape, *grid, dt, seed=seed, bc=bc)


def _state(case, seed):
    st, base = cloudy_state(case, seed=seed)
    if case.bc[0] in (2, 3):
        st["u"][0] = 0.0
    if case.bc[1] in (2, 3):
        st["u"][-2:] = 0.0
    if case.bc[2] in (2, 3):
        st["v"][:, 0] = 0.0
    if case.bc[3] in (2, 3):
        st["v"][:, -2:] = 0.0
    return st, base


def _oracle_steps(o32, case, st, base, n_sub, steps, coriolis_f):
    ref = {k: v.copy() for k, v in st.items()}
    for _ in range(steps):
        o32.large_step(ref, base, (case.dx, case.dy, case.dz), case.dt, n_sub, case.bc, coriolis_f=coriolis_f)
    return ref


@pytest.mark.parametrize("bc_name", list(BCS))
def test_plain_large_step_matches_oracle(ctx, o32, bc_name):
    case = _case((21, 17, 15), BCS[bc_name], seed=3)
    st, base = _state(case, 3)
    run = ResidentRun(ctx, case, {k: v.copy() for k, v in st.items()}, base,
                      precision=cuda.PRECISION_REFERENCE, autotune=False, coriolis_f=1e-4)
    ctx.set_substep_form(cuda.SUBSTEP_SPLIT)
    for _ in range(2):
        run.step()
    got = run.download()
    ctx.set_substep_form(cuda.SUBSTEP_AUTO)
    want = _oracle_steps(o32, case, st, base, run.n_substeps, 2, 1e-4)
    for k in PROGNOSTIC:
        assert_bitwise(got[k], want[k], f"{bc_name} {k}")


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "eager"])
def test_engine_ragged_members_match_oracle(ctx, o32, graph):
    """Three members of different shapes, spacings, dt and substep counts in
    one engine, three large steps: each equals the oracle run alone."""
    specs = [((19, 16, 13), BCS["radiative"], 4.0, 5), ((24, 14, 17), BCS["walls_sponge"], 3.0, 7),
             ((12, 22, 9), BCS["periodic_open"], 5.0, 4)]
    run = EngineRun(ctx, precision=cuda.PRECISION_REFERENCE, graph=graph)
    members = []
    for i, (shape, bc, dt, n_sub) in enumerate(specs):
        case = _case(shape, bc, seed=10 + i, dt=dt)
        st, base = _state(case, 10 + i)
        mid = run.admit(case, st, base, coriolis_f=1e-4, n_substeps=n_sub)
        members.append((mid, case, st, base, n_sub))
    run.step(3)
    run.engine.synchronize()
    for mid, case, st, base, n_sub in members:
        got = run.read(mid)
        want = _oracle_steps(o32, case, st, base, n_sub, 3, 1e-4)
        for k in PROGNOSTIC:
            assert_bitwise(got[k], want[k], f"member {mid} {k}")
    run.close()


def test_engine_member_alone_equals_member_in_mix(ctx):
    """FP32 form: the result of a member does not depend on its batch mates,
    on admissions and retirements between steps, or on the graph."""
    case = _case((26, 21, 18), BCS["radiative"], seed=40, dt=3.0)
    st, base = _state(case, 40)
    alone = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    a = alone.admit(case, st, base)
    alone.step(4)
    want = alone.read(a)
    alone.close()

    mix = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    others = []
    for i, shape in enumerate([(40, 33, 25), (9, 11, 6)]):
        c2 = _case(shape, BCS["periodic_open"], seed=50 + i, dt=2.5)
        s2, b2 = _state(c2, 50 + i)
        others.append(mix.admit(c2, s2, b2))
    m = mix.admit(case, st, base)
    mix.step(1)
    mix.engine.retire(others[0])          # a batch mate leaves
    mix.step(2)
    c3 = _case((30, 12, 20), BCS["walls_sponge"], seed=60, dt=3.5)
    s3, b3 = _state(c3, 60)
    mix.admit(c3, s3, b3)                 # another arrives
    mix.step(1)
    got = mix.read(m)
    mix.close()
    for k in PROGNOSTIC:
        assert_bitwise(got[k], want[k], k)


@pytest.mark.parametrize("precision", [cuda.PRECISION_FP32, cuda.PRECISION_REFERENCE], ids=["fp32", "reference"])
def test_continuity_kernel_with_and_without_launch_shared_values(ctx, precision):
    """A launch whose members all hold the same bounds, EOS coefficients,
    frame velocity and top condition reads those from the launch-wide block;
    one lane that mixes a rigid and an open top reads them per member.  A
    member's result is the same either way."""
    case = _case((26, 21, 18), BCS["radiative"], seed=41, dt=3.0)
    st, base = _state(case, 41)
    alone = EngineRun(ctx, precision=precision, lanes=1)
    a = alone.admit(case, st, base)
    alone.step(3)
    want = alone.read(a)
    alone.close()

    mix = EngineRun(ctx, precision=precision, lanes=1)
    mate = _case((30, 24, 20), BCS["periodic_open"], seed=42, dt=3.0)
    s2, b2 = _state(mate, 42)
    mix.admit(mate, s2, b2)
    m = mix.admit(case, st, base)
    mix.step(3)
    got = mix.read(m)
    mix.close()
    for k in PROGNOSTIC:
        assert_bitwise(got[k], want[k], k)


def test_recurring_graph_topology_is_updated_not_instantiated(ctx):
    """A batch that returns to a lane and substep layout it had before reuses
    that layout's instantiated step graphs (updated in place), and the
    members' results do not depend on which instantiation ran them."""
    cases = [_case((24, 20, 16), BCS["radiative"], seed=70 + i, dt=3.0) for i in range(2)]
    states = [_state(c, 70 + i) for i, c in enumerate(cases)]
    mate = _case((36, 30, 22), BCS["periodic_open"], seed=80, dt=2.0)
    mate_st, mate_base = _state(mate, 80)

    def run_cycle(cycles):
        run = EngineRun(ctx, precision=cuda.PRECISION_FP32, lanes=2)
        ids = [run.admit(c, s, b, n_substeps=4) for c, (s, b) in zip(cases, states)]
        run.step(1)
        builds = []
        for _ in range(cycles):
            m = run.admit(mate, mate_st, mate_base, n_substeps=6)
            run.step(1)
            run.engine.retire(m)
            run.step(1)
            builds.append(run.engine.graph_builds())
        out = [run.read(i) for i in ids]
        run.close()
        return out, builds

    got, builds = run_cycle(3)
    # every later cycle finds both layouts among the kept instantiations
    assert builds[2][0] == builds[0][0], builds
    assert builds[2][1] > builds[0][1], builds
    alone = EngineRun(ctx, precision=cuda.PRECISION_FP32, lanes=2)
    ids = [alone.admit(c, s, b, n_substeps=4) for c, (s, b) in zip(cases, states)]
    alone.step(7)
    want = [alone.read(i) for i in ids]
    alone.close()
    for g, w in zip(got, want):
        for k in PROGNOSTIC:
            assert_bitwise(g[k], w[k], k)


def test_engine_matches_plain_fp32_path(ctx):
    case = _case((23, 19, 16), BCS["radiative"], seed=70, dt=3.0)
    st, base = _state(case, 70)
    plain = ResidentRun(ctx, case, {k: v.copy() for k, v in st.items()}, base, precision=cuda.PRECISION_FP32,
                        autotune=False)
    ctx.set_substep_form(cuda.SUBSTEP_SPLIT)
    for _ in range(2):
        plain.step()
    got_plain = plain.download()
    ctx.set_substep_form(cuda.SUBSTEP_AUTO)
    run = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    mid = run.admit(case, st, base)
    run.step(2)
    got = run.read(mid)
    run.close()
    for k in PROGNOSTIC:
        assert_bitwise(got[k], got_plain[k], k)


def test_admission_refuses_beyond_free_memory(ctx):
    case = _case((10, 10, 8), BCS["radiative"], seed=1)
    st, base = _state(case, 1)
    run = EngineRun(ctx)
    desc = cuda.member_desc(case.shape, (case.dx, case.dy, case.dz), case.dt, 4, case.bc, base)
    assert run.engine.member_bytes(desc) > 40 * case.cells
    assert run.engine.try_admit(desc, st, reserve_bytes=1 << 50) is None
    assert run.engine.members == 0
    mid = run.engine.admit(desc, st)
    assert run.engine.members == 1
    run.engine.retire(mid)
    assert run.engine.members == 0
    run.step(1)  # an empty engine steps as a no-op
    # a dt the reference would subcycle the microphysics for is refused
    fast = cuda.member_desc(case.shape, (case.dx, case.dy, case.dz), 0.8 * case.dz / 20.0 + 1.0, 4, case.bc, base)
    with pytest.raises(cuda.NimbusCudaError):
        run.engine.admit(fast, st)
    run.close()


def test_boundary_refresh_matches_oracle(ctx, o32):
    import torch
    case = _case((14, 12, 9), BCS["walls_sponge"], seed=5)
    st, _ = _state(case, 5)
    dev = {k: torch.from_numpy(st[k].copy()).cuda() for k in ("u", "v", "w", "rho", "p")}
    torch.cuda.synchronize()
    ctx.check(ctx.acoustic_boundaries(cuda.boundary_args(dev, (case.dx, case.dy), case.bc, 0.0, stream=ctx.stream)))
    ctx.synchronize()
    want = {k: st[k].copy() for k in ("u", "v", "w", "rho", "p")}
    o32.acoustic_boundaries(want, (case.dx, case.dy, case.dz), case.bc, 0.0)
    for k in want:
        assert_bitwise(dev[k].cpu().numpy(), want[k], k)


def test_engine_reports_a_refused_member_only(ctx):
    """A member whose EOS projection is refused keeps its pressure and is
    flagged; its batch mate is unaffected."""
    good_case = _case((12, 11, 9), BCS["radiative"], seed=80)
    gs, gb = _state(good_case, 80)
    bad_case = _case((10, 13, 8), BCS["radiative"], seed=81)
    bs, bb = _state(bad_case, 81)
    bs["theta"][0, 5, 3] = -5.0   # a ghost-ring temperature nothing repairs; the EOS refuses it
    run = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    g = run.admit(good_case, gs, gb)
    b = run.admit(bad_case, bs, bb)
    run.step(1)
    with pytest.raises(cuda.NimbusCudaError):
        run.engine.synchronize()
    assert run.engine.member_status(b) & 4
    assert run.engine.member_status(g) == 0
    alone = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    a = alone.admit(good_case, gs, gb)
    alone.step(1)
    want = alone.read(a)
    got = run.read(g)
    for k in PROGNOSTIC:
        assert_bitwise(got[k], want[k], k)
    run.close()
    alone.close()


def test_host_pipeline_equals_resident_engine(ctx):
    """Async host copies on several engine streams: uploading each state,
    stepping and reading back every step gives the states the resident engine
    reaches.  Odd and even substep counts and the Kessler step exercise the
    rotated density, rain and pressure buffers the host side tracks."""
    cases, prepared = [], []
    for i, (shape, dt) in enumerate([((20, 17, 14), 3.0), ((12, 15, 10), 2.0), ((16, 16, 12), 3.5),
                                     ((9, 14, 8), 2.5), ((18, 10, 11), 3.0)]):
        c = _case(shape, BCS["radiative"] if i % 2 else BCS["periodic_open"], seed=90 + i, dt=dt)
        cases.append(c)
        prepared.append(_state(c, 90 + i))
    pipe = HostPipeline(ctx, cases, prepared, groups=3)
    for _ in range(3):
        pipe.step()
    order = sorted(range(len(cases)), key=lambda i: -cases[i].cells)
    by_case = {idx: pipe.host[r][2] for r, idx in enumerate(order)}
    pipe.close()
    for i, (c, (st, base)) in enumerate(zip(cases, prepared)):
        alone = EngineRun(ctx, precision=cuda.PRECISION_FP32)
        mid = alone.admit(c, st, base)
        alone.step(3)
        want = alone.read(mid)
        alone.close()
        for k in PROGNOSTIC:
            assert_bitwise(by_case[i][k], want[k], f"run {i} {k}")


def test_state_image_round_trip(ctx):
    """The state image holds each member's fields at its offset, in admission
    order: a download right after admission returns the initial states, and an
    uploaded image replaces them (retirements close the gaps)."""
    run = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    states = {}
    for i, shape in enumerate([(11, 9, 7), (6, 13, 5), (8, 8, 9)]):
        c = _case(shape, BCS["radiative"], seed=100 + i)
        st, base = _state(c, 100 + i)
        states[run.admit(c, st, base)] = st
    first = next(iter(states))
    run.engine.retire(first)
    states.pop(first)
    eng = run.engine
    want_bytes = sum(9 * 4 * st["u"].size for st in states.values())
    assert eng.image_bytes() == want_bytes
    img = np.zeros(want_bytes // 4, np.float32)
    eng.download_image_async(img)
    eng.synchronize()
    views = eng.image_views(img)
    for mid, st in states.items():
        for k in PROGNOSTIC:
            assert_bitwise(views[mid][k], st[k], f"{mid} {k}")
    for mid in states:
        for k in PROGNOSTIC:
            views[mid][k][...] = views[mid][k] * np.float32(1.0 + 1e-3)
    eng.upload_image_async(img)
    eng.synchronize()
    for mid in states:
        got = eng.read(mid)
        for k in PROGNOSTIC:
            assert_bitwise(got[k], views[mid][k], f"{mid} {k} after upload")
    with pytest.raises(KeyError):
        eng.image_offset(first)
    run.close()


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "eager"])
def test_lanes_do_not_change_results(ctx, graph):
    """Members split over parallel lanes (forked streams, one graph) reach the
    states they reach in one lane; lanes above the member count collapse."""
    specs = [((21, 17, 12), 3.0), ((9, 12, 7), 2.0), ((16, 14, 10), 3.5), ((12, 9, 11), 2.5),
             ((19, 10, 9), 3.0), ((7, 7, 6), 4.0)]
    members = []
    for i, (shape, dt) in enumerate(specs):
        c = _case(shape, list(BCS.values())[i % 3], seed=110 + i, dt=dt)
        members.append((c, *_state(c, 110 + i)))
    results = {}
    for lanes in (1, 3, 16):
        run = EngineRun(ctx, precision=cuda.PRECISION_FP32, graph=graph, lanes=lanes)
        ids = [run.admit(c, st, base) for c, st, base in members]
        run.step(2)
        assert run.engine.lanes == min(lanes, len(members))
        results[lanes] = [run.read(m) for m in ids]
        run.close()
    for lanes in (3, 16):
        for i, (got, want) in enumerate(zip(results[lanes], results[1])):
            for k in PROGNOSTIC:
                assert_bitwise(got[k], want[k], f"lanes {lanes} member {i} {k}")


def test_fp32_form_error_against_fp64_is_the_reference_forms(ctx):
    """Several large steps of a cloudy, radiative-boundary run: the FP32 form
    and the reference-precision form (FP32 storage, the reference's own
    arithmetic) both against the FP64 restatement of the same step.  Per
    field, the FP32 form's relative L2 error stays within 1.5x the reference
    form's (plus a 1e-7 floor): reduced-precision arithmetic adds no error
    beyond what FP32 storage already costs."""
    case = _case((28, 26, 20), BCS["radiative"], seed=130, dt=3.0)
    st, base = _state(case, 130)
    n_sub, steps = 6, 12
    o64 = oracle.Restatement("f64")
    ref = {k: v.astype(np.float64) for k, v in st.items()}
    for _ in range(steps):
        o64.large_step(ref, base, (case.dx, case.dy, case.dz), case.dt, n_sub, case.bc)
    theta0 = base["theta0"][None, None, :]
    errors = {}
    for prec in (cuda.PRECISION_FP32, cuda.PRECISION_REFERENCE):
        run = EngineRun(ctx, precision=prec)
        mid = run.admit(case, st, base, n_substeps=n_sub)
        run.step(steps)
        got = run.read(mid)
        run.close()
        err = {}
        for k in ("u", "v", "w", "theta", "qv", "qc", "p", "rho"):
            a, b = got[k].astype(np.float64), ref[k]
            if k == "theta":
                a, b = a - theta0, b - theta0
            den = max(float(np.linalg.norm(b)), 1e-30)
            err[k] = float(np.linalg.norm(a - b)) / den
        errors[prec] = err
    for k, e32 in errors[cuda.PRECISION_FP32].items():
        eref = errors[cuda.PRECISION_REFERENCE][k]
        assert np.isfinite(e32) and e32 <= 1.5 * eref + 1e-7, (k, e32, eref)


def test_engine_minimal_members_match_oracle(ctx, o32):
    """Members at the admission minimum (4x4 columns, 2 levels) and just
    above: the vertical closure that the momentum pass applies to interior
    columns meets nz = 2 (level 0 is also level nz - 2), one interior column
    and a perimeter of all but one column.  Reference precision, bit-exact
    against the oracle run alone; the FP32 form gives each member the same
    bits alone and in the mix."""
    specs = [((4, 4, 2), "radiative"), ((5, 4, 3), "walls_sponge"), ((4, 6, 2), "periodic_open"),
             ((4, 4, 5), "walls_sponge")]
    members = []
    for i, (shape, bc) in enumerate(specs):
        case = _case(shape, BCS[bc], seed=140 + i, dt=3.0)
        members.append((case, *_state(case, 140 + i)))
    run = EngineRun(ctx, precision=cuda.PRECISION_REFERENCE)
    ids = [run.admit(c, st, base, coriolis_f=1e-4, n_substeps=4) for c, st, base in members]
    run.step(3)
    for mid, (case, st, base) in zip(ids, members):
        got = run.read(mid)
        want = _oracle_steps(o32, case, st, base, 4, 3, 1e-4)
        for k in PROGNOSTIC:
            assert_bitwise(got[k], want[k], f"{case.shape} {k}")
    run.close()
    mix = EngineRun(ctx, precision=cuda.PRECISION_FP32, lanes=2)
    ids = [mix.admit(c, st, base, n_substeps=4) for c, st, base in members]
    mix.step(2)
    for mid, (case, st, base) in zip(ids, members):
        alone = EngineRun(ctx, precision=cuda.PRECISION_FP32)
        a = alone.admit(case, st, base, n_substeps=4)
        alone.step(2)
        want = alone.read(a)
        alone.close()
        got = mix.read(mid)
        for k in PROGNOSTIC:
            assert_bitwise(got[k], want[k], f"fp32 {case.shape} {k}")
    mix.close()


def test_empty_engine_steps_and_copies_nothing(ctx):
    eng = cuda.Engine(ctx)
    eng.step(2)
    eng.synchronize()
    assert eng.members == 0 and eng.image_bytes() == 0
    img = np.zeros(4, np.float32)
    eng.upload_image_async(img)
    eng.download_image_async(img)
    eng.synchronize()
    assert eng.lanes == 0 and not img.any()
    eng.close()


def _sponge_profiles(case, base, seed):
    from nimbus_b200.sponge import SpongeConfig, build_profiles

    rng = np.random.default_rng(seed)
    cfg = SpongeConfig(z_damp=float(case.nz * case.dz * rng.uniform(0.3, 0.8)), alpha_max=float(rng.uniform(0.02, 0.2)),
                       w_only_cells=int(rng.integers(0, 4)), w_only_alpha_max=0.3, lateral_width=int(rng.integers(1, 5)),
                       lateral_alpha_max=float(rng.uniform(0.05, 0.3)), implicit_mode=int(seed % 2),
                       wind=tuple(rng.uniform(-8, 15, 6)))
    return build_profiles(cfg, case.nz, case.dz, base["theta0"])


@pytest.mark.parametrize("graph", [True, False], ids=["graph", "eager"])
def test_engine_sponge_matches_oracle(ctx, o32, graph):
    """Members with and without the end-of-step sponge (different
    configurations) and the closing boundary refresh, in every combination:
    each equals the oracle large step followed by the same end of step,
    reference precision, bit-exact."""
    specs = [((17, 14, 12), BCS["radiative"], 3.0, 5, True, True),
             ((13, 19, 10), BCS["walls_sponge"], 4.0, 4, True, False),
             ((11, 12, 9), BCS["periodic_open"], 3.0, 4, False, True),
             ((10, 9, 8), BCS["radiative"], 3.0, 3, False, False)]
    run = EngineRun(ctx, precision=cuda.PRECISION_REFERENCE, graph=graph)
    members = []
    for i, (shape, bc, dt, n_sub, with_sponge, closure) in enumerate(specs):
        case = _case(shape, bc, seed=150 + i, dt=dt)
        st, base = _state(case, 150 + i)
        P = _sponge_profiles(case, base, 150 + i) if with_sponge else None
        mid = run.admit(case, st, base, coriolis_f=1e-4, n_substeps=n_sub, sponge=P, final_closure=closure)
        members.append((mid, case, st, base, n_sub, P, closure))
    run.step(2)
    for mid, case, st, base, n_sub, P, closure in members:
        want = {k: v.copy() for k, v in st.items()}
        for _ in range(2):
            o32.large_step(want, base, (case.dx, case.dy, case.dz), case.dt, n_sub, case.bc, coriolis_f=1e-4,
                           sponge=P, final_closure=closure)
        got = run.read(mid)
        for k in PROGNOSTIC:
            assert_bitwise(got[k], want[k], f"member {mid} {k}")
    run.close()


def test_engine_sponge_fp32_matches_plain(ctx):
    case = _case((20, 16, 14), BCS["radiative"], seed=160, dt=3.0)
    st, base = _state(case, 160)
    P = _sponge_profiles(case, base, 160)
    plain = ResidentRun(ctx, case, {k: v.copy() for k, v in st.items()}, base, precision=cuda.PRECISION_FP32,
                        autotune=False, sponge=P, final_closure=True)
    ctx.set_substep_form(cuda.SUBSTEP_SPLIT)
    for _ in range(2):
        plain.step()
    got_plain = plain.download()
    ctx.set_substep_form(cuda.SUBSTEP_AUTO)
    run = EngineRun(ctx, precision=cuda.PRECISION_FP32)
    mid = run.admit(case, st, base, sponge=P, final_closure=True)
    run.step(2)
    got = run.read(mid)
    run.close()
    for k in PROGNOSTIC:
        assert_bitwise(got[k], got_plain[k], k)
