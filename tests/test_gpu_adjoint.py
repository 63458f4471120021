"""Adjoint (score-function) derivatives of kappa against central finite
differences with common random numbers (CRN): the same seeds, so the two
kappa evaluations share every trajectory until a specular decision u <= p
flips.  Finite differences are taken with the GPU FP32 kernel and with the
CPU FP64 oracle (the reference algorithm); agreement is required within
3.5 combined standard errors, the errors coming from independent seeds."""
import math

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu


def _film(p_hole=0.5):
    return synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=4,
                                 p_hole=p_hole, t_hole=0.0, p_z=0.3)


def _with_spec(geom_np, records, delta):
    d = {k: (np.array(v) if isinstance(v, np.ndarray) else v) for k, v in geom_np.items()}
    d["specularity"] = geom_np["specularity"].copy()
    d["specularity"][records] += delta
    return d


def _mean_se(x):
    x = np.asarray(x, float)
    return x.mean(), x.std(ddof=1) / math.sqrt(len(x))


def test_adjoint_specularity_matches_finite_differences(orc):
    model = _film()
    spec = synth.spectrum(24, seed=3, mfp_lo=20e-9, mfp_hi=2e-6)
    gb = A.GeomBuf(model)
    g = gb.numpy()
    holes = np.where(g["shape"] == A.SHAPE_CYLINDER)[0]
    delta = 0.05
    seeds = [11, 12, 13, 14, 15, 16]
    np_ = 3000
    adj, fd = [], []
    gp = A.numpy_to_geometry(_with_spec(g, holes, +delta))
    gm = A.numpy_to_geometry(_with_spec(g, holes, -delta))
    with A.Handle(gb.view, spec) as h0, A.Handle(gp, spec) as hp, A.Handle(gm, spec) as hm:
        for sd in seeds:
            run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=np_, seed=sd)
            a = h0.adjoint(run)
            assert a["mismatched"] == 0
            assert a["replayed"] > 0
            adj.append(np.nansum(a["dk_dp"][holes]))
            fd.append((hp.kappa(run)["kappa"] - hm.kappa(run)["kappa"]) / (2 * delta))
    ma, sa = _mean_se(adj)
    mf, sf = _mean_se(fd)
    assert abs(ma - mf) < 3.5 * math.hypot(sa, sf), (ma, sa, mf, sf)
    assert abs(ma) > 3 * sa  # a resolved, non-zero derivative

    # the reference-side finite difference: CPU FP64 oracle with CRN
    from oracle import oracle as O
    op = O.Oracle(geometry=A.numpy_to_geometry(_with_spec(g, holes, +delta)), spectrum=spec)
    om = O.Oracle(geometry=A.numpy_to_geometry(_with_spec(g, holes, -delta)), spectrum=spec)
    ofd = []
    for sd in seeds[:4]:
        run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=1500, seed=sd)
        cp, _, _ = op.counts(run)
        cm, _, _ = om.counts(run)
        ofd.append((op.kappa(run, cp)["kappa"] - om.kappa(run, cm)["kappa"]) / (2 * delta))
    mo, so = _mean_se(ofd)
    assert abs(ma - mo) < 3.5 * math.hypot(sa, so), (ma, sa, mo, so)


def test_adjoint_scale_matches_finite_differences():
    model = _film()
    spec = synth.spectrum(24, seed=5, mfp_lo=10e-9, mfp_hi=1e-6)
    gb = A.GeomBuf(model)
    delta = 0.05
    adj, fd = [], []
    with A.Handle(gb.view, spec) as h:
        for sd in [21, 22, 23, 24, 25, 26]:
            kw = dict(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=3000, seed=sd)
            a = h.adjoint(A.make_run(**kw))
            assert a["mismatched"] == 0
            adj.append(a["dk_dscale"])
            kp = h.kappa(A.make_run(scatter_scale=1 + delta, **kw))["kappa"]
            km = h.kappa(A.make_run(scatter_scale=1 - delta, **kw))["kappa"]
            fd.append((kp - km) / (2 * delta))
    ma, sa = _mean_se(adj)
    mf, sf = _mean_se(fd)
    assert ma < 0  # stronger intrinsic scattering lowers kappa
    assert abs(ma - mf) < 3.5 * math.hypot(sa, sf), (ma, sa, mf, sf)


def test_matthiessen_scale_derivative_is_analytic():
    """With the Matthiessen rule the transport is ballistic and the scale only
    enters EMFP = 1/(s/MFP + 1/SEMFP): with common random numbers the finite
    difference equals the analytic term."""
    model = _film()
    spec = synth.spectrum(16, seed=6)
    gb = A.GeomBuf(model)
    d = 1e-4
    with A.Handle(gb.view, spec) as h:
        kw = dict(kind_mfp=A.MFP_MATTHIESSEN, nangle=9, np_=500, seed=3)
        a = h.adjoint(A.make_run(**kw))
        kp = h.kappa(A.make_run(scatter_scale=1 + d, **kw))["kappa"]
        km = h.kappa(A.make_run(scatter_scale=1 - d, **kw))["kappa"]
    assert a["dk_dscale"] == pytest.approx((kp - km) / (2 * d), rel=1e-4)


def test_adjoint_replays_exactly_the_transmitted_samples():
    model = _film()
    spec = synth.spectrum(12, seed=7)
    gb = A.GeomBuf(model)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=700, seed=9)
    with A.Handle(gb.view, spec) as h:
        a = h.adjoint(run)
        k = h.kappa(run, want_counts=True)
    assert a["replayed"] == int(k["counts"].sum())
    assert a["mismatched"] == 0
    assert a["kappa"] == pytest.approx(k["kappa"], rel=1e-12)
    # records never hit (brick interiors of void holes, x faces) have zero derivative
    g = gb.numpy()
    bricks = np.where((g["shape"] == A.SHAPE_CYLINDER) & (g["grain_inside"] != g["igrain_fill"]))[0]
    assert np.all(a["dk_dp"][bricks] == 0.0)
    assert np.isnan(a["dk_dp"][0]) or a["dk_dp"][0] == 0.0



def test_adjoint_capped_cylinders_matches_finite_differences():
    """dkappa/dp of random-axis capped cylinders (the C3 extension) against
    the GPU finite difference with common random numbers."""
    model = synth.spheres_cylinders_box(n_spheres=6, n_cylinders=8, l=300.0, seed=5, r_sphere=(15.0, 35.0),
                                        r_cylinder=25.0, length=(80.0, 200.0), trans=0.0, p_wall=0.2,
                                        per_surface_p=False)
    model.surf_spec = np.full(len(model.grain_shape), 0.5)
    spec = synth.spectrum(16, seed=8, mfp_lo=20e-9, mfp_hi=2e-6)
    gb = A.GeomBuf(model)
    g = gb.numpy()
    caps = np.where(g["shape"] == A.SHAPE_CAPPED)[0]
    delta = 0.05
    gp = A.numpy_to_geometry(_with_spec(g, caps, +delta))
    gm = A.numpy_to_geometry(_with_spec(g, caps, -delta))
    adj, fd = [], []
    with A.Handle(gb.view, spec) as h0, A.Handle(gp, spec) as hp, A.Handle(gm, spec) as hm:
        for sd in [21, 22, 23, 24, 25, 26]:
            run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=3000, seed=sd)
            a = h0.adjoint(run)
            assert a["mismatched"] == 0
            adj.append(np.nansum(a["dk_dp"][caps]))
            fd.append((hp.kappa(run)["kappa"] - hm.kappa(run)["kappa"]) / (2 * delta))
    ma, sa = _mean_se(adj)
    mf, sf = _mean_se(fd)
    assert abs(ma - mf) < 3.5 * math.hypot(sa, sf), (ma, sa, mf, sf)
    assert abs(ma) > 3 * sa


def test_adjoint_with_a_blob_past_the_default_shared_memory():
    """A staged geometry blob of tens of KB plus the adjoint kernels' static
    shared memory (accumulators, cooperative rows) passes the 48 KB a launch
    gets without opting in: both passes still launch, replay every
    transmitted sample and reproduce the forward kappa."""
    model = synth.spheres_cylinders_box(n_spheres=150, n_cylinders=30, l=1000.0, seed=2,
                                        r_sphere=(15.0, 40.0), r_cylinder=15.0, length=(60.0, 160.0))
    spec = synth.spectrum(10, seed=3, mfp_lo=2e-9, mfp_hi=1e-6)
    gb = A.GeomBuf(model)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=200, seed=4)
    with A.Handle(gb.view, spec) as h:
        a = h.adjoint(run)
        k = h.kappa(run, want_counts=True)
    assert a["replayed"] == int(k["counts"].sum()) > 0
    assert a["mismatched"] == 0
    assert a["kappa"] == pytest.approx(k["kappa"], rel=1e-12)
    assert np.all(np.isfinite(a["dk_dp"][~np.isnan(a["dk_dp"])]))


def _c3_like():
    """Spheres and random-axis capped cylinders as voids in a 200 nm box, each
    surface with its own specularity p ~ U(0, 1) (the C3 configuration, small)."""
    return synth.spheres_cylinders_box(n_spheres=4, n_cylinders=3, l=200.0, seed=7, r_sphere=(25.0, 40.0),
                                       r_cylinder=20.0, length=(60.0, 120.0), trans=0.0, p_wall=0.0,
                                       per_surface_p=True)


def test_adjoint_per_surface_matches_central_differences(orc):
    """Every surface's d kappa / d p_k (C3-like structure) against central
    finite differences with Delta = 1e-3 and common random numbers: the two
    kappa runs share every trajectory until a decision u <= p_k flips.  Means
    and standard errors over 10 seeds; every derivative resolved at 3 sigma
    agrees with its finite difference within 3 combined standard errors, and
    the sum of squared z over all surfaces stays below the 0.999 quantile of
    chi-square.  The oracle's own finite difference (FP64, the reference
    algorithm, 4 seeds) agrees the same way."""
    from scipy import stats
    model = _c3_like()
    spec = synth.spectrum(12, seed=4, mfp_lo=50e-9, mfp_hi=2e-6)
    gb = A.GeomBuf(model)
    g = gb.numpy()
    recs = np.where(((g["shape"] == A.SHAPE_SPHERE) | (g["shape"] == A.SHAPE_CAPPED)) &
                    (g["grain_inside"] == g["igrain_fill"]))[0]
    p = g["specularity"][recs]
    assert len(recs) == 7 and np.all((p > 2e-3) & (p < 1 - 2e-3))
    delta = 1e-3
    seeds = list(range(31, 41))
    kw = dict(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=20000)
    adj = np.zeros((len(seeds), len(recs)))
    fd = np.zeros_like(adj)
    with A.Handle(gb.view, spec) as h0:
        for i, sd in enumerate(seeds):
            a = h0.adjoint(A.make_run(seed=sd, **kw))
            assert a["mismatched"] == 0
            adj[i] = a["dk_dp"][recs]
    for j, k in enumerate(recs):
        gp = A.numpy_to_geometry(_with_spec(g, [k], +delta))
        gm = A.numpy_to_geometry(_with_spec(g, [k], -delta))
        with A.Handle(gp, spec) as hp, A.Handle(gm, spec) as hm:
            for i, sd in enumerate(seeds):
                run = A.make_run(seed=sd, **kw)
                fd[i, j] = (hp.kappa(run)["kappa"] - hm.kappa(run)["kappa"]) / (2 * delta)
    ma, sa = adj.mean(0), adj.std(0, ddof=1) / math.sqrt(len(seeds))
    mf, sf = fd.mean(0), fd.std(0, ddof=1) / math.sqrt(len(seeds))
    z = (ma - mf) / np.hypot(sa, sf)
    resolved = np.abs(ma) > 3 * sa
    table = "\n".join(f"rec {k:3d} p={pk:.3f} adj {a:+.4e} +- {e:.1e}  fd {f:+.4e} +- {s:.1e}  z {zz:+.2f}"
                      for k, pk, a, e, f, s, zz in zip(recs, p, ma, sa, mf, sf, z))
    assert resolved.sum() >= 3, table
    assert np.all(np.abs(z[resolved]) < 3.0), table
    assert np.sum(z * z) < stats.chi2.ppf(0.999, len(recs)), table

    # the reference algorithm's finite difference: the CPU FP64 oracle with CRN
    from oracle import oracle as O
    ofd = np.zeros((4, len(recs)))
    for j, k in enumerate(recs):
        op = O.Oracle(geometry=A.numpy_to_geometry(_with_spec(g, [k], +delta)), spectrum=spec)
        om = O.Oracle(geometry=A.numpy_to_geometry(_with_spec(g, [k], -delta)), spectrum=spec)
        for i, sd in enumerate(seeds[:4]):
            run = A.make_run(seed=sd, **kw)
            cp, _, _ = op.counts(run)
            cm, _, _ = om.counts(run)
            ofd[i, j] = (op.kappa(run, cp)["kappa"] - om.kappa(run, cm)["kappa"]) / (2 * delta)
    mo, so = ofd.mean(0), ofd.std(0, ddof=1) / 2.0
    zo = (ma - mo) / np.hypot(sa, so)
    assert np.all(np.abs(zo[resolved]) < 3.0), (zo, table)
