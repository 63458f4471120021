"""Pins of the CPU oracle (no GPU): published Philox4x32-10 known-answer
vectors, accuracy of its log / sincos against libm, and analytic limits that
the reference's formulas imply (src/RTMCphon.f90:2418-2451, 1544-1841)."""
import math

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth


# Random123 kat_vectors, philox4x32 with 10 rounds: (ctr, key) -> out
PHILOX_KAT = [
    ((0, 0, 0, 0), (0, 0), (0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8)),
    ((0xFFFFFFFF,) * 4, (0xFFFFFFFF,) * 2, (0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD)),
    ((0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344), (0xA4093822, 0x299F31D0),
     (0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1)),
]


@pytest.mark.parametrize("ctr,key,want", PHILOX_KAT)
def test_philox_known_answers(orc, ctr, key, want):
    assert tuple(orc.philox(ctr, key)) == want


def test_log_matches_libm(orc):
    rng = np.random.default_rng(1)
    xs = np.concatenate([rng.uniform(0, 1, 20000), np.exp(-rng.uniform(0, 700, 2000)),
                         [1.0, 0.5, 2.0 ** -52, 1 - 2.0 ** -52, 0.7071067811865476]])
    xs = xs[xs > 0]
    got = np.array([orc.olog(float(x)) for x in xs])
    ref = np.log(xs)
    err = np.abs(got - ref) / np.maximum(np.abs(ref), 1e-300)
    assert np.all((np.abs(got - ref) <= 4e-16) | (err <= 4e-16))


def test_sincos_matches_libm(orc):
    rng = np.random.default_rng(2)
    us = np.concatenate([rng.uniform(0, 1, 20000), np.arange(0, 1, 1 / 64)])
    s, c = zip(*(orc.osincos2pi(float(u)) for u in us))
    assert np.max(np.abs(np.array(s) - np.sin(2 * np.pi * us))) < 1e-15
    assert np.max(np.abs(np.array(c) - np.cos(2 * np.pi * us))) < 1e-15


def _simpson_unit(nangle):
    """(dtheta/3) * sum_a c_a sin cos over a < nangle-1 (T = 1 there, 0 at pi/2)."""
    th = np.array([ia / (nangle - 1) * (math.pi / 2) for ia in range(nangle)])
    c = np.zeros(nangle)
    for ia in range(1, nangle - 1, 2):
        c[ia - 1] += 1
        c[ia] += 4
        c[ia + 1] += 1
    w = c * np.sin(th) * np.cos(th)
    w[-1] = 0.0
    return (th[1] - th[0]) / 3 * w.sum()


def test_ballistic_specular_duct_is_three_quarters_length(orc):
    """T = 1 for every angle in a specular duct without intrinsic scattering,
    so the effective MFP is 0.75 * Lx times Simpson's value of 2*int sin cos."""
    m = synth.nanowire(length=500.0, width=50.0, height=50.0, p_side=1.0)
    spec = synth.spectrum(8, seed=3)
    o = orc.Oracle(model=m, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_MATTHIESSEN, nangle=11, np_=64, seed=5)
    cnt, lost, res = o.counts(run)
    assert lost.sum() == 0
    assert np.all(cnt == 64)
    k = o.kappa(run, cnt)
    t = k["transmit"].reshape(11, -1)
    assert np.all(t[:-1] == 1.0) and np.all(t[-1] == 0.0)
    # Matthiessen with SEMFP = 0.75 Lx * 2 * simpson
    semfp = 1.5 * 500.0 * _simpson_unit(11)
    assert abs(semfp - 0.75 * 500.0) / (0.75 * 500.0) < 2e-4   # Simpson bias at Nangle = 11
    mfp = spec.mfp_nm(300.0) * 1e-9
    expect = 1.0 / (1.0 / mfp + 1.0 / (semfp * 1e-9)) * 1e9
    np.testing.assert_allclose(k["emfp_nm"], expect, rtol=1e-12)


def test_diffusive_limit(orc):
    """Lambda << L in a specular duct: Lambda_eff -> Lambda * L / (L + 2 z0 Lambda),
    z0 = 0.7104 the Milne extrapolation length."""
    L, lam = 400.0, 8.0
    m = synth.nanowire(length=L, width=40.0, height=40.0, p_side=1.0)
    spec = synth.spectrum(1, seed=0)
    o = orc.Oracle(model=m, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_GRID, nangle=11, np_=20000, seed=11, mfp_grid=[lam])
    cnt, lost, res = o.counts(run)
    k = o.kappa(run, cnt)
    th = np.array([ia / 10 * math.pi / 2 for ia in range(11)])
    c = np.array([1, 4, 2, 4, 2, 4, 2, 4, 2, 4, 1], float)
    t = k["transmit"].reshape(11, -1)[:, 0]
    s = 1.5 * L * (math.pi / 20) / 3
    semfp = s * np.sum(c * np.sin(th) * np.cos(th) * t)
    sigma = s * math.sqrt(np.sum((c * np.sin(th) * np.cos(th)) ** 2 * t * (1 - t) / 20000))
    expect = lam * L / (L + 2 * 0.7104 * lam)
    assert abs(semfp - expect) < 3 * sigma + 0.01 * expect, (semfp, expect, sigma)


def test_lost_phonons_counted_with_quirk(orc):
    """A flight cap of 1 loses every phonon that needs a second flight; with
    the reference quirk a lost phonon counts as transmitted (RT:1701, 1833)."""
    m = synth.nanowire(length=500.0, width=50.0, height=50.0, p_side=0.0)
    spec = synth.spectrum(2, seed=1)
    o = orc.Oracle(model=m, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_MATTHIESSEN, nangle=5, np_=200, seed=5)
    c0, l0, r0 = o.counts(run, max_flights=1)
    c1, l1, r1 = o.counts(run, max_flights=1, ref_quirks=1)
    assert r0["capped"] > 0 and r0["lost"] == r0["capped"]
    np.testing.assert_array_equal(c1, c0 + l0)


def _film_model(L, d, width=40.0):
    """A film of thickness d (diffuse z walls) along x, infinite in-plane:
    specular y walls, which mirror a film without inclusions exactly."""
    m = synth.nanowire(length=L, width=width, height=d, p_side=0.0)
    m.cellspec = (1.0, 1.0, 1.0, 1.0, 0.0, 0.0)
    return m


def _oracle_flux_T(orc, model, lam, np_, nangle=11, seed=5):
    import limits
    spec = synth.spectrum(1, seed=0)
    o = orc.Oracle(model=model, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_GRID, nangle=nangle, np_=np_, seed=seed, mfp_grid=[lam])
    cnt, lost, _ = o.counts(run)
    assert lost.sum() == 0
    return limits.flux_transmission(cnt[: nangle - 1] / np_, np_, nangle)


@pytest.mark.parametrize("kn", [0.5, 2.0])
def test_fuchs_sondheimer_film_limit(orc, kn):
    """In-plane MFP of a fully diffuse film (thickness d = 40 nm, gray MFP
    Kn * d) from the two-length estimate at L = 10 and 20 max(Lambda, d)
    against the Fuchs-Sondheimer integral, within 3 standard errors plus 1%
    for what is left of the contact term at these lengths and the Simpson
    bias at Nangle = 11 (5.5e-5)."""
    import limits
    d = 40.0
    lam = kn * d
    L1, L2 = 10 * max(lam, d), 20 * max(lam, d)
    T1, v1 = _oracle_flux_T(orc, _film_model(L1, d), lam, 30000)
    T2, v2 = _oracle_flux_T(orc, _film_model(L2, d), lam, 30000)
    est, se = limits.two_length_mfp(L1, T1, v1, L2, T2, v2)
    want = lam * limits.fuchs_sondheimer(kn)
    assert abs(est - want) < 3 * se + 0.01 * want, (est, want, se)


def test_casimir_closed_form_equals_its_integral():
    """The closed form of the square wire's Casimir MFP equals the defining
    integral 3/(8A) int dA int dphi s(r, phi) evaluated by quadrature."""
    import limits
    assert abs(limits.casimir_square(1.0) - limits.casimir_numeric(1.0, 1.0, 400)) < 2e-5
    assert abs(limits.casimir_square(1.0) - 1.114954) < 1e-6
