"""The Kessler operators of the reference's device route
(nimbus_cuda_kessler_pointwise / _sedimentation, and the adapter's
dispatch_kessler_pointwise / dispatch_kessler_sedimentation).

The reference defines these operators in FP32 (its device shaders), so parity
is within a tolerance, written here against the scale of each field: the
FP64 restatement (oracle/kessler_device.py) and the reference's own scheme
on its CPU route.  An FP32 evaluation of the same statements sits within
6e-6 of the FP64 one (test_oracle.py::test_kessler_device_restatement_fp32_floor);
the tolerances leave room for CUDA's powf / expf.
"""
import numpy as np
import pytest

from nimbus_b200 import cuda
from oracle.kessler_device import kessler_pointwise, kessler_sedimentation

pytestmark = pytest.mark.gpu

PARAMS = dict(qc0=1.0e-3, c_auto=1.0e-3, c_accr=2.2, evaporation_efficiency=1.0, lv_cp=2.5e6 / 1004.0, t0=273.15,
              dt=3.0)
POINTWISE_TOL = 5e-5      # of max |field| (FP32 operator vs its FP64 statement)
SEDIMENTATION_TOL = 1e-5
VT_CAP = float(np.finfo(np.float32).max)


def kessler_inputs(shape, seed):
    """A moist column state: temperature and pressure of a standard
    atmosphere with noise, vapour from 40% to 105% of saturation, cloud and
    rain in part of the cells (some rain below the fallout threshold)."""
    rng = np.random.default_rng(seed)
    nz = shape[2]
    z = (np.arange(nz) + 0.5) * 400.0
    T = (300.0 - 6.5e-3 * z)[None, None, :] + rng.normal(0, 1.5, shape)
    p = (1.0e5 * np.exp(-z / 8000.0))[None, None, :] * (1 + rng.normal(0, 1e-3, shape))
    tc = T - 273.15
    es = 611.21 * np.exp((18.678 - tc / 234.5) * tc / (257.14 + tc))
    qv = 0.62198 * es / (p - es) * rng.uniform(0.4, 1.05, shape)
    qc = np.where(rng.random(shape) < 0.5, 0.0, rng.uniform(0, 2.5e-3, shape))
    qr = np.where(rng.random(shape) < 0.4, 0.0, rng.uniform(0, 4e-3, shape) ** 1.3)
    qr[rng.random(shape) < 0.05] = 3e-10
    rho = p / (287.0 * T)
    return {k: np.ascontiguousarray(v, np.float32) for k, v in dict(T=T, p=p, qv=qv, qc=qc, qr=qr, rho=rho).items()}


def assert_close(got, want, tol, what):
    scale = float(np.abs(want).max())
    err = float(np.abs(got.astype(np.float64) - want).max())
    assert err <= tol * max(scale, 1e-30), f"{what}: max error {err:.3e} against scale {scale:.3e}"


@pytest.fixture(scope="module")
def ctx():
    c = cuda.Context(0)
    yield c
    c.close()


@pytest.mark.parametrize("memory", ["host", "device"])
def test_kessler_pointwise_matches_its_fp64_statement(ctx, memory):
    import torch

    st = kessler_inputs((26, 21, 30), 3)
    dom = (1, 25, 1, 20, 0, 30)
    want = kessler_pointwise(st["T"], st["p"], st["qv"], st["qc"], st["qr"], st["rho"], dom, PARAMS["qc0"],
                             PARAMS["c_auto"], PARAMS["c_accr"], PARAMS["evaporation_efficiency"], PARAMS["lv_cp"],
                             PARAMS["t0"], PARAMS["dt"])
    ins = [st[k] for k in ("T", "p", "qv", "qc", "qr", "rho")]
    outs = [np.full_like(st["T"], np.nan) for _ in range(6)]
    if memory == "device":
        ins = [torch.from_numpy(a).cuda() for a in ins]
        douts = [torch.from_numpy(a).cuda() for a in outs]
        ctx.kessler_pointwise(*ins, douts, dom, **PARAMS)
        ctx.synchronize()
        outs = [d.cpu().numpy() for d in douts]
    else:
        ctx.kessler_pointwise(*ins, outs, dom, **PARAMS)
    inside = np.zeros(st["T"].shape, bool)
    inside[1:25, 1:20, :] = True
    for name, got, ref in zip(("dtheta", "dqv", "dqc", "dqr"), outs, want):
        assert np.all(got[~inside] == 0.0), f"{name} outside the domain"
        assert_close(got, ref, POINTWISE_TOL, name)
    assert np.all(outs[4] == 0.0) and np.all(outs[5] == 0.0)
    assert np.count_nonzero(want[1]) > 100, "evaporation should act in part of the cells"


@pytest.mark.parametrize("variant", ["uniform", "density", "layers"])
@pytest.mark.parametrize("memory", ["host", "device"])
def test_kessler_sedimentation_matches_its_fp64_statement(ctx, memory, variant):
    import torch

    st = kessler_inputs((20, 17, 33), 5)
    dom = (1, 19, 1, 16, 2, 31)
    rng = np.random.default_rng(6)
    dqr0 = np.ascontiguousarray(rng.normal(0, 1e-6, st["qr"].shape), np.float32)
    rho = st["rho"] if variant != "uniform" else None
    layers = (np.ascontiguousarray(rng.uniform(300, 500, st["qr"].shape), np.float32) if variant == "layers"
              else None)
    want = kessler_sedimentation(st["qr"], dqr0, dom, 400.0, 20.0, VT_CAP, rho_d=rho, layers=layers)
    got = dqr0.copy()
    if memory == "device":
        dev = lambda a: torch.from_numpy(a).cuda() if a is not None else None
        g = dev(got)
        ctx.kessler_sedimentation(dev(st["qr"]), g, dom, 400.0, 20.0, VT_CAP, rho_d=dev(rho), layers=dev(layers))
        ctx.synchronize()
        got = g.cpu().numpy()
    else:
        ctx.kessler_sedimentation(st["qr"], got, dom, 400.0, 20.0, VT_CAP, rho_d=rho, layers=layers)
    inside = np.zeros(got.shape, bool)
    inside[1:19, 1:16, 2:31] = True
    assert np.array_equal(got[~inside].view(np.uint32), dqr0[~inside].view(np.uint32)), "outside the domain"
    assert_close(got - dqr0, want - dqr0, SEDIMENTATION_TOL, f"fallout ({variant})")


def test_kessler_operators_refuse_bad_domains(ctx):
    st = kessler_inputs((6, 5, 4), 1)
    outs = [np.zeros_like(st["T"]) for _ in range(4)]
    with pytest.raises(cuda.NimbusCudaError):
        ctx.kessler_pointwise(st["T"], st["p"], st["qv"], st["qc"], st["qr"], st["rho"], outs, (0, 7, 0, 5, 0, 4))
    with pytest.raises(cuda.NimbusCudaError):
        ctx.kessler_sedimentation(st["qr"], outs[0], (0, 6, 0, 5, 0, 4), 0.0)
