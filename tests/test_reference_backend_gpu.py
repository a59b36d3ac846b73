"""The CUDA backend behind the reference's own C++ interface: the adapter
library (nimbus_b200/reference_backend/nimbus_compute_backend.cpp) loaded as a
ComputeBackend by the reference-linked harness, driven with the reference's
dispatch structs and, for the Smagorinsky closure, by the reference's own
SmagorinskyScheme::compute taking its native-backend path.  The results must
equal the reference's CPU backend / CPU path bit for bit."""
from pathlib import Path

import numpy as np
import pytest

import oracle
from nimbus_b200.initial import Case, cloudy_state, perturbed_state
from nimbus_b200.sgs import SgsConfig

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not oracle.reference_available(),
                                                   reason="reference harness not built")]

ADAPTER = Path(__file__).resolve().parents[1] / "nimbus_b200" / "lib" / "libnimbus_reference_backend.so"


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
