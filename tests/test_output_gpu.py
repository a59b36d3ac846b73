"""Device-side output against the reference, bit for bit: the cell-centre
kernel (interpolate_*_face_to_center), history frames of a resident run and
of engine members, and the npy files the writer thread produces.

Every comparison is 0 ULP: the kernel forms the reference's FP32 face means
and its FP64 surface mean rounded once."""
from pathlib import Path

import numpy as np
import pytest
import torch

import oracle
from nimbus_b200 import cuda
from nimbus_b200.history import HistoryWriter, frame_dir
from nimbus_b200.initial import Case, cloudy_state
from nimbus_b200.run import EngineRun, ResidentRun
from tests.golden.make_golden import OUTPUT_SHAPES

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def ctx():
    c = cuda.Context(0)
    yield c
    c.close()


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


def assert_bitwise(a, b, what):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    bad = np.count_nonzero(a.view(np.uint32) != b.view(np.uint32))
    assert bad == 0, f"{what}: {bad}/{a.size} values differ"


def faces_of(shape, seed, scale=25.0):
    rng = np.random.default_rng(seed)
    return [(rng.standard_normal(shape) * scale).astype(np.float32) for _ in range(3)]


@pytest.mark.parametrize("n", range(len(OUTPUT_SHAPES)), ids=[str(s) for s in OUTPUT_SHAPES])
def test_cell_centre_golden_host(ctx, n):
    """Host-memory call against the reference's own outputs (golden)."""
    g = np.load(GOLDEN / "cell_centre.npz")
    faces = [g[f"s{n}_{k}"] for k in "uvw"]
    args = cuda.cell_centre_args(*faces)
    ctx.check(ctx.cell_centre_velocity(args))
    for k, a in zip("uvw", args.outputs):
        assert_bitwise(a, g[f"s{n}_{k}c"], k)
    args = cuda.cell_centre_args(None, None, faces[2], ground_w=g[f"s{n}_ground"])
    ctx.check(ctx.cell_centre_velocity(args))
    assert_bitwise(args.outputs[2], g[f"s{n}_wc_terrain"], "w terrain")


# nz covers the run widths 4, 2 and 1; the large case exceeds L2.
@pytest.mark.parametrize("shape", [(64, 48, 40), (33, 17, 50), (20, 30, 41), (1, 1, 1), (1, 70, 9), (70, 1, 12),
                                   (5, 7, 1), (256, 256, 96)])
def test_cell_centre_device_vs_oracle(ctx, o32, shape):
    faces = faces_of(shape, sum(shape))
    ground = np.random.default_rng(3).standard_normal(shape[:2]) * 4.0
    dev = [torch.from_numpy(f).cuda() for f in faces]
    args = cuda.cell_centre_args(*dev, memory=cuda.MEMORY_DEVICE)
    ctx.check(ctx.cell_centre_velocity(args))
    targs = cuda.cell_centre_args(None, None, dev[2], ground_w=ground, memory=cuda.MEMORY_DEVICE)
    ctx.check(ctx.cell_centre_velocity(targs))
    torch.cuda.synchronize()
    ctx.synchronize()
    want = o32.cell_centre(*faces)
    for k, got, ref in zip("uvw", args.outputs, want):
        assert_bitwise(got.cpu().numpy(), ref, k)
    assert_bitwise(targs.outputs[2].cpu().numpy(), o32.cell_centre(None, None, faces[2], ground)[2], "w terrain")


def test_cell_centre_full_level(ctx, o32):
    """A 512x512x80 level (84 MB per field, larger than L2), bit for bit
    against the oracle; also the case the kernel's ncu summary captures."""
    shape = (512, 512, 80)
    faces = faces_of(shape, 80, scale=30.0)
    dev = [torch.from_numpy(f).cuda() for f in faces]
    args = cuda.cell_centre_args(*dev, memory=cuda.MEMORY_DEVICE)
    for _ in range(2):
        ctx.check(ctx.cell_centre_velocity(args))
    ctx.synchronize()
    for k, got, ref in zip("uvw", args.outputs, o32.cell_centre(*faces)):
        assert_bitwise(got.cpu().numpy(), ref, k)


def test_cell_centre_unaligned_and_subsets(ctx, o32):
    """Views one float off a 16-byte boundary take the scalar run; a single
    component leaves the others unwritten."""
    shape = (24, 20, 16)
    n = 24 * 20 * 16
    faces = faces_of(shape, 9)
    buf = torch.zeros(3 * n + 3, dtype=torch.float32, device="cuda")
    dev = []
    for f, a in enumerate(faces):
        view = buf[f * n + 1:(f + 1) * n + 1].view(shape)
        view.copy_(torch.from_numpy(a))
        dev.append(view)
    out = torch.full((n + 1,), -7.0, device="cuda")[1:].view(shape)
    args = cuda.cell_centre_args(None, dev[1], None, outputs=(None, out, None), memory=cuda.MEMORY_DEVICE)
    ctx.check(ctx.cell_centre_velocity(args))
    torch.cuda.synchronize()
    assert_bitwise(out.cpu().numpy(), o32.cell_centre(None, faces[1], None)[1], "v unaligned")


def test_cell_centre_refusals(ctx):
    """A non-finite ground value or an output overlapping an input is refused
    with nothing written; zero cells is a no-op."""
    shape = (6, 5, 4)
    faces = faces_of(shape, 4)
    ground = np.zeros(shape[:2])
    ground[2, 3] = np.nan
    out = np.full(shape, 99.0, np.float32)
    args = cuda.cell_centre_args(None, None, faces[2], outputs=(None, None, out), ground_w=ground)
    assert ctx.cell_centre_velocity(args) == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    assert "finite" in ctx.last_error
    assert np.all(out == 99.0)
    args = cuda.cell_centre_args(faces[0], None, None, outputs=(faces[0], None, None))
    assert ctx.cell_centre_velocity(args) == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    empty = np.zeros((0, 5, 4), np.float32)
    assert ctx.cell_centre_velocity(cuda.cell_centre_args(empty, empty, empty)) == cuda.NIMBUS_OK


def _resident_fields(shape, seed):
    case = Case(*shape, 500.0, 500.0, 20000.0 / shape[2], 3.0, seed=seed)
    st, base = cloudy_state(case, seed=seed)
    return case, st, base


@pytest.mark.parametrize("names", [cuda.HISTORY_FIELDS, ("w", "theta"), ("u", "v"), ("qr",), ("v", "rho", "qc")])
def test_history_snapshot_vs_oracle(ctx, o32, names):
    """The snapshot image holds the selected fields in image order, u, v, w
    centred, the scalars copied unchanged."""
    case, st, _ = _resident_fields((40, 36, 30), 5)
    dev = {k: torch.from_numpy(st[k]).cuda() for k in cuda.HISTORY_FIELDS}
    mask = cuda.history_mask(names)
    img = torch.empty(len(names) * case.cells, dtype=torch.float32).pin_memory().numpy()
    ground = np.random.default_rng(1).standard_normal(case.shape[:2])
    ctx.check(ctx.history_snapshot(cuda.history_args(dev, mask, img, case.shape, ground_w=ground)))
    ctx.synchronize()
    uc, vc, _ = o32.cell_centre(st["u"], st["v"], None)
    centred = {"u": uc, "v": vc, "w": o32.cell_centre(None, None, st["w"], ground)[2]}
    for slot, k in enumerate(cuda.history_names(mask)):
        want = centred[k] if k in "uvw" else st[k]
        assert_bitwise(img[slot * case.cells:(slot + 1) * case.cells].reshape(case.shape), want, k)


def test_history_snapshot_refusals(ctx):
    case, st, _ = _resident_fields((8, 8, 6), 2)
    dev = {k: torch.from_numpy(st[k]).cuda() for k in ("u", "v")}
    img = np.zeros(3 * case.cells, np.float32)
    assert ctx.history_snapshot(cuda.history_args(dev, cuda.history_mask(("u", "w")), img, case.shape)) == \
        cuda.NIMBUS_ERR_INVALID_ARGUMENT
    assert ctx.history_snapshot(cuda.history_args(dev, 1 << 12, img, case.shape)) == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    bad = np.full(case.shape[:2], np.inf)
    assert ctx.history_snapshot(cuda.history_args({"w": torch.zeros(case.shape, device="cuda")},
                                                  cuda.history_mask(("w",)), img, case.shape, ground_w=bad)) == \
        cuda.NIMBUS_ERR_INVALID_ARGUMENT
    assert np.all(img == 0.0)


def test_resident_run_history_files(ctx, o32, tmp_path):
    """Two large steps of a resident run with a frame after each: every npy
    file is, byte for byte, the reference writer's file of the oracle-centred
    state at that step."""
    case = Case(48, 40, 32, 500.0, 500.0, 20000.0 / 32, 3.0, seed=8)
    run = ResidentRun(ctx, case, precision=cuda.PRECISION_REFERENCE, autotune=False)
    writer = HistoryWriter(ctx)
    states = []
    for index in range(2):
        run.step()
        writer.frame(run, index, tmp_path)
        states.append(run.download())
    writer.close()
    assert writer.frames == 2
    for index, st in enumerate(states):
        d = frame_dir(tmp_path, index)
        uc, vc, wc = o32.cell_centre(st["u"], st["v"], st["w"])
        want = {"u": uc, "v": vc, "w": wc, **{k: st[k] for k in cuda.HISTORY_FIELDS[3:]}}
        for k in cuda.HISTORY_FIELDS:
            assert (d / f"{k}.npy").read_bytes() == oracle.npy_bytes(want[k]), (index, k)


def test_engine_history_vs_oracle(ctx, o32, tmp_path):
    """Engine members of different shapes: a frame after a step matches the
    oracle-centred member state; files as the reference writes them."""
    er = EngineRun(ctx, precision=cuda.PRECISION_REFERENCE)
    ids = [er.admit(Case(*s, 500.0, 500.0, 20000.0 / s[2], 3.0, seed=i)) for i, s in
           enumerate(((24, 20, 16), (17, 19, 13), (30, 12, 22)))]
    er.step(1)
    writer = HistoryWriter(ctx, fields=("u", "w", "p", "qv"))
    for mid in ids:
        writer.frame_member(er, mid, 1, tmp_path / f"member_{mid}")
    writer.close()
    for mid in ids:
        st = er.read(mid)
        uc, _, wc = o32.cell_centre(st["u"], None, st["w"])
        d = frame_dir(tmp_path / f"member_{mid}", 1)
        assert sorted(p.name for p in d.iterdir()) == ["p.npy", "qv.npy", "u.npy", "w.npy"]
        for k, want in (("u", uc), ("w", wc), ("p", st["p"]), ("qv", st["qv"])):
            assert (d / f"{k}.npy").read_bytes() == oracle.npy_bytes(want), (mid, k)
    er.close()


def test_engine_history_refusals(ctx):
    er = EngineRun(ctx)
    mid = er.admit(Case(8, 8, 6, 500.0, 500.0, 20000.0 / 6, 3.0, seed=1))
    img = np.zeros(9 * 8 * 8 * 6, np.float32)
    with pytest.raises(cuda.NimbusCudaError):
        er.engine.history_async(mid + 100, cuda.HISTORY_CORE, img)
    with pytest.raises(cuda.NimbusCudaError):
        er.engine.history_async(mid, 1 << 10, img)
    er.close()
