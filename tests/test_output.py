"""Output path on the CPU: the oracle's cell-centre restatement and npy bytes
pinned against the reference (its own unit-test cases, golden fixtures
written by its functions, and the live harness where it is built), and the
library's host-side npy writers, which need no device.

Reference behaviour: src/core/output/stagger_interpolation.cpp,
src/core/output/npy_writer.cpp, tests/core/test_stagger_interpolation.cpp."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from nimbus_b200 import cuda
from tests.golden.make_golden import OUTPUT_SHAPES

GOLDEN = Path(__file__).resolve().parent / "golden"


@pytest.fixture(scope="module")
def o32():
    return oracle.Restatement("f32")


@pytest.fixture(scope="module")
def lib():
    return cuda.load_library()


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def full(shape, value):
    return np.full(shape, value, np.float32)


# --- the reference's own unit-test cases (test_stagger_interpolation.cpp) ---

def test_u_interior_mean_and_west_face(o32):
    """Gate 1: u_face[i] = i + 0.5 -> u_center[i] = i, u_center[0] = 0.5."""
    u = np.broadcast_to((np.arange(8, dtype=np.float32) + 0.5)[:, None, None], (8, 4, 6)).copy()
    uc, _, _ = o32.cell_centre(u, None, None)
    assert np.all(uc[0] == 0.5)
    assert np.array_equal(uc[1:], np.broadcast_to(np.arange(1, 8, dtype=np.float32)[:, None, None], (7, 4, 6)))


def test_v_never_wraps(o32):
    """Gate 2: a north-edge sentinel never reaches the south cell."""
    v = np.broadcast_to(np.arange(8, dtype=np.float32)[None, :, None], (4, 8, 4)).copy()
    v[:, 7, :] = 1000.0
    _, vc, _ = o32.cell_centre(None, v, None)
    assert np.all(vc[:, 0] == 0.0)
    assert np.array_equal(vc[:, 1:7], np.broadcast_to((np.arange(1, 7, dtype=np.float32) - 0.5)[None, :, None],
                                                      (4, 6, 4)))
    assert np.all(vc[:, 7] == np.float32(0.5) * (np.float32(6.0) + np.float32(1000.0)))


def test_w_surface_half_cell(o32):
    """Gate 3: w_face[k] = k + 0.5 -> w_center[k] = k, w_center[0] = 0.25."""
    w = np.broadcast_to((np.arange(8, dtype=np.float32) + 0.5)[None, None, :], (4, 4, 8)).copy()
    _, _, wc = o32.cell_centre(None, None, w)
    assert np.all(wc[..., 0] == 0.25)
    assert np.array_equal(wc[..., 1:], np.broadcast_to(np.arange(1, 8, dtype=np.float32), (4, 4, 7)))


def test_w_terrain_surface(o32):
    """Terrain case: the surface cell averages the lower-face velocity in FP64."""
    nx, ny = 4, 5
    i, j = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    ground = 2.0 + 0.25 * i - 0.1 * j
    w = np.zeros((nx, ny, 3), np.float32)
    w[..., 0] = (6.0 + i + j).astype(np.float32)
    w[..., 1] = 10.0
    w[..., 2] = 14.0
    _, _, wc = o32.cell_centre(None, None, w, ground)
    assert np.array_equal(wc[..., 0], (0.5 * (ground + w[..., 0].astype(np.float64))).astype(np.float32))
    assert np.array_equal(wc[..., 1], np.float32(0.5) * (w[..., 0] + w[..., 1]))
    assert np.all(wc[..., 2] == 12.0)
    bad = ground.copy()
    bad[0, 0] = np.nan
    with pytest.raises(ValueError, match="finite"):
        o32.cell_centre(None, None, w, bad)


def test_constant_and_uniform_fields(o32):
    """Gates 4-5: constant faces give constant centres in the interior and on
    the west/south planes; the surface halves w against the ground face."""
    u, v, w = full((6, 8, 6), 7.5), full((6, 8, 6), -3.25), full((6, 8, 6), 12.0)
    uc, vc, wc = o32.cell_centre(u, v, w)
    assert np.all(uc == 7.5) and np.all(vc == -3.25)
    assert np.all(wc[..., 1:] == 12.0) and np.all(wc[..., 0] == 6.0)


# --- golden fixtures written by the reference's own functions ---

@pytest.mark.parametrize("n", range(len(OUTPUT_SHAPES)), ids=[str(s) for s in OUTPUT_SHAPES])
def test_golden_cell_centre(o32, n):
    g = np.load(GOLDEN / "cell_centre.npz")
    faces = [g[f"s{n}_{k}"] for k in "uvw"]
    got = o32.cell_centre(*faces)
    for k, a in zip("uvw", got):
        assert np.array_equal(bits(a), bits(g[f"s{n}_{k}c"])), k
    _, _, wt = o32.cell_centre(None, None, faces[2], g[f"s{n}_ground"])
    assert np.array_equal(bits(wt), bits(g[f"s{n}_wc_terrain"]))


def test_golden_npy_bytes():
    """The oracle's npy bytes are the reference writer's file, byte for byte."""
    g = np.load(GOLDEN / "cell_centre.npz")
    assert oracle.npy_bytes(g["npy_data"]) == (GOLDEN / "npy_write_3d.npy").read_bytes()


@pytest.mark.parametrize("shape", [(1, 1, 1), (2, 3, 4), (96, 96, 50), (10, 1000, 7), (123, 4567, 89)])
def test_npy_header_alignment(shape):
    """Header padding keeps the payload on a 16-byte boundary for any shape,
    and numpy parses the header."""
    import io
    head = oracle.npy_header(shape)
    n = int.from_bytes(head[8:10], "little")
    assert len(head) == 10 + n and len(head) % 16 == 0 and head.endswith(b"\n")
    assert np.lib.format.read_array_header_1_0(io.BytesIO(head[8:])) == (tuple(shape), False, np.dtype("<f4"))


# --- the library's host-side writers (no device needed) ---

def test_library_npy_write_matches_reference(lib, tmp_path):
    g = np.load(GOLDEN / "cell_centre.npz")
    path = tmp_path / "x.npy"
    assert cuda.npy_write_3d(g["npy_data"], path, lib) == cuda.NIMBUS_OK
    assert path.read_bytes() == (GOLDEN / "npy_write_3d.npy").read_bytes()


@pytest.mark.parametrize("shape", [(1, 1, 1), (7, 5, 3), (32, 33, 17)])
def test_library_npy_write_matches_oracle(lib, tmp_path, shape):
    data = np.random.default_rng(sum(shape)).standard_normal(shape).astype(np.float32)
    assert cuda.npy_write_3d(data, tmp_path / "a.npy", lib) == cuda.NIMBUS_OK
    assert (tmp_path / "a.npy").read_bytes() == oracle.npy_bytes(data)


def test_library_npy_write_refusals(lib, tmp_path):
    """npy::write_3d returns false for an empty dimension or an unopenable
    path; the C-ABI reports INVALID_ARGUMENT and IO."""
    empty = np.zeros((0, 4, 4), np.float32)
    assert cuda.npy_write_3d(empty, tmp_path / "e.npy", lib) == cuda.NIMBUS_ERR_INVALID_ARGUMENT
    assert not (tmp_path / "e.npy").exists()
    ok = np.ones((2, 2, 2), np.float32)
    assert cuda.npy_write_3d(ok, tmp_path / "missing" / "x.npy", lib) == cuda.NIMBUS_ERR_IO


@pytest.mark.parametrize("names", [cuda.HISTORY_FIELDS, ("w",), ("u", "theta", "qr"), ("rho", "p")])
def test_library_history_write(lib, tmp_path, names):
    """nimbus_history_write: one <name>.npy per selected field, in image order."""
    shape = (5, 4, 3)
    n = 60
    mask = cuda.history_mask(names)
    image = np.random.default_rng(len(names)).standard_normal(len(names) * n).astype(np.float32)
    assert cuda.history_write(image, mask, shape, tmp_path, lib) == cuda.NIMBUS_OK
    assert sorted(p.name for p in tmp_path.iterdir()) == sorted(f"{k}.npy" for k in names)
    for slot, k in enumerate(cuda.history_names(mask)):
        assert (tmp_path / f"{k}.npy").read_bytes() == oracle.npy_bytes(image[slot * n:(slot + 1) * n].reshape(shape))
    assert cuda.history_write(image, 1 << 9, shape, tmp_path, lib) == cuda.NIMBUS_ERR_INVALID_ARGUMENT


# --- live pin against the reference's functions ---

@pytest.mark.reference
@pytest.mark.skipif(not oracle.reference_available(), reason="reference harness not built here")
@pytest.mark.parametrize("shape", [(12, 9, 10), (3, 2, 1), (17, 13, 5)])
def test_live_reference_pin_cell_centre(o32, shape):
    ref = oracle.ReferenceHarness(threads=2)
    rng = np.random.default_rng(shape[0])
    faces = [(rng.standard_normal(shape) * 40.0).astype(np.float32) for _ in range(3)]
    faces[0].flat[::7] = np.float32(3.4e38)  # overflowing face sums round the same way
    ground = rng.standard_normal(shape[:2]) * 1e3
    for a, b in zip(o32.cell_centre(*faces), ref.cell_centre(*faces)):
        assert np.array_equal(bits(a), bits(b))
    assert np.array_equal(bits(o32.cell_centre(None, None, faces[2], ground)[2]),
                          bits(ref.cell_centre(None, None, faces[2], ground)[2]))
    bad = ground.copy()
    bad[-1, -1] = np.inf
    with pytest.raises(RuntimeError, match="finite"):
        ref.cell_centre(None, None, faces[2], bad)
