"""The allocation-free fused substep, nimbus_cuda_acoustic_fused_static_scratch.

It exists for callers that cannot allocate device memory: hosts whose HBM
budget is fully committed up front (runs admitted by free device memory) and
stepping loops that cannot take cudaMalloc's implicit device synchronisation.
It stages the new density in a fixed file-scope device array instead of the
context workspace, so this test checks, through the C-ABI, that two
consecutive substeps give exactly what the allocating entry point gives
(0 ULP, the tolerance of every other parity test here), and that a grid
beyond the array's capacity is refused.

This file is collected last on purpose: it must pass both alone in a fresh
process and after every other test.
"""
import ctypes

import numpy as np
import pytest

from nimbus_b200 import cuda
from nimbus_b200.initial import Case, perturbed_state

pytestmark = pytest.mark.gpu

FIELDS = ("u", "v", "w", "rho", "p", "theta")


def _device_state(torch, st):
    return {k: torch.from_numpy(np.ascontiguousarray(st[k])).cuda() for k in FIELDS}


def test_static_scratch_substeps_match_allocating_entry_point():
    import torch

    lib = cuda.load_library()
    case = Case(41, 35, 26, 700.0, 650.0, 330.0, 5.0, seed=9)
    st, base = perturbed_state(case, seed=10)
    rho0 = torch.from_numpy(base["rho0"]).cuda()
    p0 = torch.from_numpy(base["p0"]).cuda()
    grid = (case.dx, case.dy, case.dz)
    dt_small = 0.45

    ctx = cuda.Context(0)
    want = _device_state(torch, st)
    got = _device_state(torch, st)
    drho_want = torch.zeros(case.shape, dtype=torch.float32, device="cuda")
    drho_got = torch.zeros(case.shape, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()

    for _ in range(2):  # two calls in a row: the shared scratch keeps the last call's contents
        a = cuda.fused_args(want, rho0, p0, dt_small, grid, drho_want, memory=cuda.MEMORY_DEVICE)
        ctx.check(ctx.acoustic_fused(a))
        ctx.synchronize()
        b = cuda.fused_args(got, rho0, p0, dt_small, grid, drho_got, memory=cuda.MEMORY_DEVICE, stream=None)
        rc = lib.nimbus_cuda_acoustic_fused_static_scratch(ctypes.byref(b))
        assert rc == 0, cuda.STATUS_NAMES.get(rc, rc)
        torch.cuda.synchronize()
        for k in FIELDS:
            x = want[k].cpu().numpy()
            y = got[k].cpu().numpy()
            assert np.array_equal(x.view(np.uint32), y.view(np.uint32)), k
        assert np.array_equal(drho_want.cpu().numpy().view(np.uint32), drho_got.cpu().numpy().view(np.uint32))
    ctx.close()


def test_static_scratch_at_capacity_matches_allocating_entry_point():
    """A grid of exactly NIMBUS_STATIC_SCRATCH_CELLS cells (256x256x64) is
    accepted, and its grid-stride launch (capped at 16 blocks per SM) gives
    the allocating entry point's bits."""
    import torch

    lib = cuda.load_library()
    case = Case(256, 256, 64, 500.0, 500.0, 300.0, 3.0, seed=4)
    assert case.cells == cuda.STATIC_SCRATCH_CELLS
    st, base = perturbed_state(case, seed=5)
    rho0 = torch.from_numpy(base["rho0"]).cuda()
    p0 = torch.from_numpy(base["p0"]).cuda()
    grid = (case.dx, case.dy, case.dz)
    ctx = cuda.Context(0)
    ctx.set_precision(cuda.PRECISION_REFERENCE)
    want = _device_state(torch, st)
    got = _device_state(torch, st)
    torch.cuda.synchronize()
    for _ in range(2):
        ctx.check(ctx.acoustic_fused(cuda.fused_args(want, rho0, p0, 0.3, grid, memory=cuda.MEMORY_DEVICE)))
        ctx.synchronize()
        b = cuda.fused_args(got, rho0, p0, 0.3, grid, memory=cuda.MEMORY_DEVICE)
        rc = lib.nimbus_cuda_acoustic_fused_static_scratch(ctypes.byref(b))
        assert rc == 0, cuda.STATUS_NAMES.get(rc, rc)
        torch.cuda.synchronize()
    for k in FIELDS:
        assert torch.equal(want[k].view(torch.int32), got[k].view(torch.int32)), k
    ctx.close()


def test_static_scratch_refuses_grids_beyond_capacity():
    import torch

    lib = cuda.load_library()
    case = Case(8, 8, 4, 1000.0, 1000.0, 500.0, 6.0)
    st, base = perturbed_state(case)
    dev = _device_state(torch, st)
    rho0 = torch.from_numpy(np.resize(base["rho0"], 64)).cuda()
    p0 = torch.from_numpy(np.resize(base["p0"], 64)).cuda()
    a = cuda.fused_args(dev, rho0, p0, 0.5, (1000.0, 1000.0, 500.0), memory=cuda.MEMORY_DEVICE)
    # Claim a grid larger than the static array; it is refused before any launch.
    a.nx, a.ny, a.nz, a.base_len = 1024, 1024, 8, 64
    assert 1024 * 1024 * 8 > cuda.STATIC_SCRATCH_CELLS
    assert lib.nimbus_cuda_acoustic_fused_static_scratch(ctypes.byref(a)) == 7  # NIMBUS_ERR_TOO_LARGE
    # One cell beyond the capacity (5 x 397 x 2113 = 4,194,305) is refused too.
    rho0_long = torch.from_numpy(np.resize(base["rho0"], 2113)).cuda()
    p0_long = torch.from_numpy(np.resize(base["p0"], 2113)).cuda()
    c = cuda.fused_args(dev, rho0_long, p0_long, 0.5, (1000.0, 1000.0, 500.0), memory=cuda.MEMORY_DEVICE)
    c.nx, c.ny, c.nz, c.base_len = 5, 397, 2113, 2113
    assert 5 * 397 * 2113 == cuda.STATIC_SCRATCH_CELLS + 1
    assert lib.nimbus_cuda_acoustic_fused_static_scratch(ctypes.byref(c)) == 7
    # Host memory is not accepted either: the entry point never stages.
    host = {k: np.ascontiguousarray(st[k]) for k in FIELDS}
    h = cuda.fused_args(host, base["rho0"], base["p0"], 0.5, (1000.0, 1000.0, 500.0))
    assert lib.nimbus_cuda_acoustic_fused_static_scratch(ctypes.byref(h)) == 1  # NIMBUS_ERR_INVALID_ARGUMENT
