"""Analytic limits of the effective MFP, shared by the oracle and GPU tests.

P-TRANS's effective MFP for a structure of length L between two black heat
baths is Lambda_eff(L) = 0.75 L <T>, <T> = 2 int_0^{pi/2} T(theta) sin cos
dtheta (src/RTMCphon.f90:2418-2451), the flux-weighted transmission.  Deep
in the diffusive regime the baths add an L-independent resistance:
1/<T(L)> = 3 L / (4 Lambda) + c, so two lengths give the structure's own MFP
without the contact term:

    Lambda = (L2 - L1) / (L2 / Lambda_eff(L2) - L1 / Lambda_eff(L1)).

Fuchs-Sondheimer (film of thickness d with fully diffuse walls, infinite
in-plane, gray MFP Lambda, Kn = Lambda / d), in-plane:

    Lambda_FS / Lambda = 1 - (3 Kn / 2) int_1^inf (t^-3 - t^-5)(1 - e^{-t/Kn}) dt,

from the Boltzmann equation with diffuse (equilibrium) re-emission at both
walls: a phonon moving at polar cosine mu to the wall normal carries the
bulk deviation times 1 - exp(-z / (Lambda mu)), averaged over the thickness.

Casimir (ballistic, square cross-section of side a, fully diffuse walls,
infinitely long): the walls re-emit at the local temperature of a uniform
gradient, so a ray through a cross-section point r in direction Omega carries
the temperature difference over its back-length to the wall,
l = s(r, phi) / sin(theta_x), and

    Lambda_C = 3 / (4 pi A) int_A dA int dOmega l cos^2 theta_x
             = 3 / (8 A) int_A dA int_0^{2 pi} s(r, phi) dphi
             = (3/2) [ln(1 + sqrt 2) - (sqrt 2 - 1) / 3] a = 1.114955 a

(for a circle of diameter d the same formula gives the classic Lambda = d).
A wall-to-wall flight's axial displacement z has a tail P(|z| > Z) ~ Z^-3, so
the bath resistance of a ballistic wire does not settle to a constant: the
extrapolation length grows like ln L, and 1/<T(L)> = 3 L / (4 Lambda_C) +
alpha ln(L / a) + beta.  The two-length estimate then carries a correction
of order ln(L2/L1) / L1; it is removed by fitting alpha and beta with
Lambda_C over several lengths.
"""
import math

import numpy as np


def simpson_weights(nangle):
    """w_a with <T> = sum_a w_a T_a over a < nangle - 1 (T = 0 at pi/2), the
    reference's composite Simpson rule over theta_a = a / (nangle-1) * pi/2."""
    th = np.array([ia / (nangle - 1) * (math.pi / 2) for ia in range(nangle)])
    c = np.zeros(nangle)
    for ia in range(1, nangle - 1, 2):
        c[ia - 1] += 1
        c[ia] += 4
        c[ia + 1] += 1
    w = 2.0 * (th[1] - th[0]) / 3.0 * c * np.sin(th) * np.cos(th)
    return w[:-1]


def flux_transmission(t_angle, np_, nangle):
    """<T> and its binomial variance from per-angle transmissions."""
    w = simpson_weights(nangle)
    t = np.asarray(t_angle, float)[: nangle - 1]
    return float(np.sum(w * t)), float(np.sum(w * w * t * (1.0 - t)) / np_)


def two_length_mfp(L1, T1, v1, L2, T2, v2):
    """Lambda from <T> at two lengths, and its standard error."""
    D = 1.0 / T2 - 1.0 / T1
    lam = 0.75 * (L2 - L1) / D
    g = 0.75 * (L2 - L1) / (D * D)
    se = g * math.sqrt(v2 / T2 ** 4 + v1 / T1 ** 4)
    return lam, se


def fuchs_sondheimer(kn):
    """Lambda_FS / Lambda for a fully diffuse film (in-plane), by quadrature of
    the mu-form, 1 - (3/2) Kn int_0^1 (1 - mu^2) mu (1 - e^{-1/(Kn mu)}) dmu."""
    from scipy import integrate
    f = lambda mu: (1.0 - mu * mu) * mu * (-math.expm1(-1.0 / (kn * mu))) if mu > 0 else 0.0
    val, _ = integrate.quad(f, 0.0, 1.0, limit=200, epsabs=1e-13, epsrel=1e-12)
    return 1.0 - 1.5 * kn * val


def casimir_square(a):
    """Casimir MFP of an infinitely long wire of square cross-section a x a."""
    return 1.5 * (math.log(1.0 + math.sqrt(2.0)) - (math.sqrt(2.0) - 1.0) / 3.0) * a


def casimir_numeric(wx, wy, n=400):
    """The same Casimir integral, 3/(8A) int dA int dphi s(r, phi), by
    quadrature for a wx x wy rectangle (an independent check of the closed
    form): for a direction phi the inner integral over the area is
    int chord(w)^2 / 2 dw over the chords parallel to phi."""
    tot = 0.0
    phis = (np.arange(n) + 0.5) * (2.0 * math.pi / n)
    for phi in phis:
        c, s = abs(math.cos(phi)), abs(math.sin(phi))
        # chords of a rectangle along (c, s): projected width and chord lengths
        ws = np.linspace(0.0, wx * s + wy * c, 4001)
        wm = 0.5 * (ws[1:] + ws[:-1])
        # chord length at transverse offset w, by clipping the line
        # {w-offset} against the rectangle: min of the two slab lengths
        lx = wx / c if c > 1e-15 else np.inf
        ly = wy / s if s > 1e-15 else np.inf
        full = min(lx, ly)
        ramp1 = wm / (c * s) if c * s > 1e-15 else np.full_like(wm, np.inf)
        ramp2 = (ws[-1] - wm) / (c * s) if c * s > 1e-15 else np.full_like(wm, np.inf)
        chord = np.minimum(full, np.minimum(ramp1, ramp2))
        tot += np.sum(chord * chord / 2.0) * (ws[1] - ws[0])
    tot *= 2.0 * math.pi / n
    return 3.0 / (8.0 * wx * wy) * tot
