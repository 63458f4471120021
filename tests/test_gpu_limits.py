"""Analytic limits on the GPU kernels (the formulas and their derivation are
in tests/limits.py): the Fuchs-Sondheimer in-plane MFP of a fully diffuse
film and the Casimir MFP of a ballistic wire with fully diffuse walls, from
the reference's effective MFP Lambda_eff(L) = 0.75 L <T> (src/RTMCphon.f90:
2418-2451) with diffuse walls re-emitting by Lambert's law (:2332-2380).
These pin the persistent FP32 kernel and the plain FP64 kernel to numbers
that do not come from the oracle."""
import math

import numpy as np
import pytest

import limits
from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu


def _wire(L, w, h, py, pz):
    m = synth.nanowire(length=L, width=w, height=h, p_side=0.0)
    m.cellspec = (1.0, 1.0, py, py, pz, pz)
    return m


def _flux_T(model, lam, np_, precision, seed=7, nangle=11):
    gb = A.GeomBuf(model)
    spec = synth.spectrum(1, seed=0)
    with A.Handle(gb.view, spec) as h:
        t, _ = h.transmission(lam, nangle, np_, seed=seed, precision=precision)
        st = h.stats()
    assert st["lost"] == 0
    return limits.flux_transmission(t[0, 0, :], np_, nangle)


@pytest.mark.parametrize("kn,precision,np_", [(0.5, A.PREC_FP32, 400000), (1.0, A.PREC_FP32, 400000),
                                              (2.0, A.PREC_FP32, 400000), (1.0, A.PREC_FP64, 60000)])
def test_fuchs_sondheimer_film(kn, precision, np_):
    """In-plane MFP of a film 40 nm thick with fully diffuse walls (specular
    side walls: an infinite film) at Knudsen number kn, two-length estimate
    at L = 10 and 20 max(Lambda, d), against the Fuchs-Sondheimer integral:
    within 3 standard errors plus 0.5% (what is left of the bath term at
    these lengths, and the Simpson bias at Nangle = 11, 5.5e-5)."""
    d = 40.0
    lam = kn * d
    L1, L2 = 10 * max(lam, d), 20 * max(lam, d)
    T1, v1 = _flux_T(_wire(L1, 40.0, d, 1.0, 0.0), lam, np_, precision)
    T2, v2 = _flux_T(_wire(L2, 40.0, d, 1.0, 0.0), lam, np_, precision, seed=8)
    est, se = limits.two_length_mfp(L1, T1, v1, L2, T2, v2)
    want = lam * limits.fuchs_sondheimer(kn)
    assert abs(est - want) < 3 * se + 0.005 * want, (est, want, se)


def test_casimir_wire():
    """Ballistic square wire (side a = 20 nm, fully diffuse walls, no
    intrinsic scattering) at lengths 20a ... 640a.  Lambda_eff(L) rises with
    L and stays below the Casimir length 1.114954 a, and a weighted fit of
    1/<T(L)> = 3 L / (4 Lambda_C) + alpha ln(L/a) + beta + gamma a/L (the bath
    term of a ballistic wire grows like ln L, tests/limits.py) puts Lambda_C
    within 3 standard errors plus 2.5% of it: the bath term's form beyond
    these orders is not derived, and the approach is slow (measured: 0.96 a
    at 20a, 1.08 a at 640a; the fit gives 1.09 a)."""
    a = 20.0
    ks = np.array([20, 40, 80, 160, 320, 640], float)
    ys, ws, leff = [], [], []
    for k in ks:
        T, v = _flux_T(_wire(k * a, a, a, 0.0, 0.0), 1.0e10, 2000000 if k <= 160 else 1000000, A.PREC_FP32,
                       seed=int(k))
        ys.append(1.0 / T)
        ws.append(T ** 4 / v)  # 1 / var(1/T)
        leff.append(0.75 * k * T)  # Lambda_eff / a
    want = limits.casimir_square(1.0)
    leff = np.array(leff)
    assert np.all(np.diff(leff) > 0) and np.all(leff < want), leff
    y, w = np.array(ys), np.array(ws)
    X = np.column_stack([0.75 * ks, np.log(ks), np.ones_like(ks), 1.0 / ks])  # lengths in units of a
    cov = np.linalg.inv(X.T @ (w[:, None] * X))
    p = cov @ X.T @ (w * y)
    lam = 1.0 / p[0]
    se = math.sqrt(cov[0, 0]) / p[0] ** 2
    assert abs(lam - want) < 3 * se + 0.025 * want, (lam, se, want, leff)
