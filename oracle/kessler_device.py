"""Test infrastructure: numpy restatement of the two Kessler operators of the
reference's device route (the checker for nimbus_cuda_kessler_pointwise and
nimbus_cuda_kessler_sedimentation).

KesslerScheme::compute_tendencies (src/microphysics/schemes/kessler/kessler.cpp:152-300)
hands the adjusted temperature, qv and qc to dispatch_kessler_pointwise and
then calls dispatch_kessler_sedimentation; the reference's device operators
behind them are vulkan/shaders/compute/microphysics/kessler_pointwise.comp
(lines 55-172) and kessler_sedimentation.comp (lines 44-117).  The functions
here follow those statements; with ``dtype=np.float64`` they are the FP64
statement the FP32 CUDA kernels are checked against (within a tolerance
written in the tests), with ``np.float32`` an FP32 evaluation of the same
sequence.  Parity of these operators is anchored on the reference's CPU route
of the whole scheme too (ReferenceHarness.kessler_tendencies with and
without a backend).
"""
from __future__ import annotations

import numpy as np


def _domain_mask(shape, domain):
    i0, i1, j0, j1, k0, k1 = domain
    m = np.zeros(shape, bool)
    m[i0:i1, j0:j1, k0:k1] = True
    return m


def kessler_pointwise(T, p, qv, qc, qr, rho, domain, qc0, c_auto, c_accr, eff, lv_cp, t0, dt, dtype=np.float64):
    """(dtheta, dqv, dqc, dqr): warm-rain production and rain evaporation
    (kessler_pointwise.comp:111-163), zero outside the cell domain (:97-108).
    dtheta is the temperature tendency before the theta conversion."""
    f = lambda a: np.asarray(a, dtype=dtype)
    T, p, qv, qc, qr, rho = (f(a) for a in (T, p, qv, qc, qr, rho))
    one, zero = dtype(1), dtype(0)
    qc0, c_auto, c_accr, eff, lv_cp, t0, dt = (dtype(x) for x in (qc0, c_auto, c_accr, eff, lv_cp, t0, dt))
    with np.errstate(all="ignore"):
        # production (:115-128)
        prod_on = (dt > 0) & (qc > 0)
        factor = one / (one + c_accr * dt * np.power(np.maximum(qr, zero), dtype(0.875)))
        amount = qc * (one - factor) + factor * c_auto * dt * np.maximum(qc - qc0, zero)
        amount = np.minimum(np.maximum(amount, zero), qc)
        production = np.where(prod_on, amount / dt if dt > 0 else zero, zero)
        dqc = -production
        dqr = production.copy()
        # evaporation (:131-163); saturation mixing ratio (:55-69)
        tc = T - t0
        es = dtype(611.21) * np.exp((dtype(18.678) - tc / dtype(234.5)) * tc / (dtype(257.14) + tc))
        qvsat = np.minimum(np.maximum(dtype(0.62198) * es / np.maximum(p - es, one), zero), dtype(0.2))
        avail = qr + production * dt
        rcgs = dtype(1.0e-3) * rho
        content = rcgs * np.maximum(avail, zero)
        vent = (dtype(1.6) + dtype(124.9) * np.power(content, dtype(0.2046))) * np.power(content, dtype(0.525))
        resist = dtype(2.55e8) / (p * qvsat) + dtype(5.4e5)
        raw = eff * (vent / resist) * ((qvsat - qv) / (rcgs * qvsat))
        gamma = lv_cp * (dtype(2.5e6) / dtype(461.5)) * qvsat / np.maximum(T * T, one)
        bound = (qvsat - qv) / (one + gamma)
        evap = np.minimum(np.maximum(raw, zero), np.minimum(bound / dt, avail / dt))
        evap_on = ((qr > 0) | (production > 0)) & (qvsat > 0) & (qv < qvsat) & (rho > 0) & (p > 0)
        evap = np.where(evap_on, evap, zero)
    dqv = evap
    dqr = dqr - evap
    dth = -(lv_cp * evap)
    inside = _domain_mask(T.shape, domain)
    return tuple(np.where(inside, a, zero) for a in (dth, dqv, dqc, dqr))


def kessler_sedimentation(qr, dqr, domain, dz, vt_max, vt_cap, rho_d=None, layers=None, dtype=np.float64):
    """dqr with the rain fallout added (kessler_sedimentation.comp:71-116):
    per column, level k loses Vt q / donor_dz and level k-1 gains
    w Vt q / receiver_dz, in the column's k order; the lowest domain level is
    a sink."""
    qr = np.asarray(qr, dtype=dtype)
    out = np.array(dqr, dtype=dtype, copy=True)
    i0, i1, j0, j1, k0, k1 = domain
    for k in range(k0, k1):
        q = np.maximum(qr[i0:i1, j0:j1, k], dtype(0))
        donor = np.full(q.shape, dtype(dz)) if layers is None else np.asarray(layers[i0:i1, j0:j1, k], dtype)
        receiver = donor if (layers is None or k == k0) else np.asarray(layers[i0:i1, j0:j1, k - 1], dtype)
        if rho_d is None:
            fall, weight, rho_air = dtype(1), dtype(1), dtype(1.2)
        else:
            rk = np.asarray(rho_d[i0:i1, j0:j1, k], dtype)
            rkm = rk if k == k0 else np.asarray(rho_d[i0:i1, j0:j1, k - 1], dtype)
            fall, weight, rho_air = np.sqrt(dtype(1.2) / rk), rk / rkm, rk
        with np.errstate(all="ignore"):
            vt = dtype(36.34) * np.power(dtype(1.0e-3) * rho_air * q, dtype(0.1346))
            vt = np.minimum(np.minimum(vt * fall, dtype(vt_max)), dtype(vt_cap))
            flux = vt * q
        on = q > dtype(1.0e-9)
        out[i0:i1, j0:j1, k] = np.where(on, out[i0:i1, j0:j1, k] - flux / donor, out[i0:i1, j0:j1, k])
        if k > k0:
            out[i0:i1, j0:j1, k - 1] = np.where(on, out[i0:i1, j0:j1, k - 1] + weight * flux / receiver,
                                                out[i0:i1, j0:j1, k - 1])
    return out
