"""GPU parity of the CUDA path against the CPU FP64 oracle, through the C ABI.

- The plain FP64 kernel replays the oracle bit for bit: same exit side, same
  number of free flights and the same final position for every particle, and
  identical transmitted counts per task (integer tallies: exact).
- The persistent FP32 kernel draws the same kind of trajectories with FP32
  geometry; its per-task and per-mode transmissions and kappa agree with the
  oracle within the combined binomial confidence interval (|z| bounds written
  in each test).
- The device FP64 reduction gives the host assembly's kappa to 1e-12.
"""
import math

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu


def _tbc_gamma(tbc=3.0e8):
    """gamma of a TBC entry (GammaDeterm on the host) for a fixed material."""
    st, g = A.gamma_from_tbc(synth.spectrum(200, seed=0), 300.0, tbc)
    assert st == 0
    return g


def geometries():
    spheres = synth.spheres_in_box(l=200.0, centres=((70, 90, 100), (140, 110, 90)), radii=(35, 40),
                                   t=0.5, p=0.3, p_wall=0.2)
    brick = synth.brick_box(t=0.5, p=0.2, p_wall=0.1)
    return {
        "nanowire_diffuse": synth.nanowire(length=300.0, width=60.0, height=50.0, p_side=0.0),
        "nanowire_mixed": synth.nanowire(length=300.0, width=60.0, height=50.0, p_side=0.6),
        "film_periodic": synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, seed=2),
        "film_mirror_transmit": synth.film_with_holes(seed=3, periodic_y=False, p_hole=0.3, t_hole=0.4, p_z=0.5),
        "spheres": synth.spheres_in_box(l=200.0, centres=((70, 90, 100), (140, 110, 90)), radii=(35, 40),
                                        t=0.5, p=0.3, p_wall=0.2),
        "brick_quads": synth.brick_box(t=0.5, p=0.3, p_wall=0.1),
        "brick_tris": synth.brick_box(t=0.7, p=0.0, p_wall=0.5, triangles=True),
        "lattice_tris": synth.cube_lattice(n=3, l=300.0, fill=0.5, trans=0.3, spec=0.2, p_wall=0.3),
        "voronoi": synth.voronoi_box(6, box=(300.0, 200.0, 200.0), seed=4, trans=0.5, spec=0.1,
                                     p_wall=0.2),
        "capped": synth.spheres_cylinders_box(n_spheres=4, n_cylinders=5, l=300.0, seed=3,
                                              r_sphere=(15.0, 35.0), r_cylinder=20.0, length=(50.0, 150.0),
                                              trans=0.3, p_wall=0.2),
        # Gamma / TBC interfaces: per-mode threshold (one material) and random
        # threshold (two materials), src/RTMCphon.f90:1417-1424, 2391-2402
        "spheres_gamma": synth.with_interface(spheres, A.TRANS_GAMMA, 0.8, spec=0.3),
        "spheres_gamma_2mat": synth.with_interface(spheres, A.TRANS_GAMMA, 0.8, spec=0.3, two_materials=True),
        "brick_tbc": synth.with_interface(brick, A.TRANS_TBC, _tbc_gamma(), spec=0.2),
        "brick_tbc_2mat": synth.with_interface(brick, A.TRANS_TBC, _tbc_gamma(), spec=0.2, two_materials=True),
    }


def setup(name, nmode=6, seed=1):
    m = geometries()[name]
    spec = synth.spectrum(nmode, seed=seed, mfp_lo=5e-9, mfp_hi=2e-6)
    gb = A.GeomBuf(m)
    return m, spec, gb


@pytest.mark.parametrize("name", list(geometries()))
def test_fp64_replay_is_bit_exact(orc, name):
    m, spec, gb = setup(name)
    o = orc.Oracle(model=m, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=64, seed=12345, stream=3,
                     precision=A.PREC_FP64)
    with A.Handle(gb.view, spec) as h:
        for task in (0, 5, 13, 20, 35):
            es_g, fl_g, fp_g = h.replay_task(run, task)
            es_o, fl_o, fp_o = o.replay(run, task)
            np.testing.assert_array_equal(es_g, es_o)
            np.testing.assert_array_equal(fl_g, fl_o)
            np.testing.assert_array_equal(fp_g, fp_o)


@pytest.mark.parametrize("name", ["nanowire_diffuse", "film_periodic", "spheres", "brick_tris",
                                  "spheres_gamma", "brick_tbc_2mat"])
def test_fp64_counts_equal_oracle(orc, name):
    m, spec, gb = setup(name, nmode=10)
    o = orc.Oracle(model=m, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=200, seed=7, precision=A.PREC_FP64,
                     nbins=4, bin_omega=(0.0, float(spec.omega.max())))
    cnt_o, lost_o, res_o = o.counts(run)
    ko = o.kappa(run, cnt_o)
    with A.Handle(gb.view, spec) as h:
        kg = h.kappa(run, want_counts=True, want_transmit=True)
    np.testing.assert_array_equal(kg["counts"], cnt_o)
    assert kg["flights"] == res_o["flights"]
    assert kg["lost"] == res_o["lost"]
    assert kg["kappa"] == pytest.approx(ko["kappa"], rel=1e-12)
    np.testing.assert_allclose(kg["emfp_nm"], ko["emfp_nm"], rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(kg["bin_T"], ko["bin_T"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(kg["transmit"], ko["transmit"], rtol=0, atol=0)


def test_transmission_function_layout_and_ranks(orc):
    """ptg_transmission fills transmit(nb,nk,nangle) with count/np per rank,
    transmit(:,:,nangle) = 0; summing the ranks gives the single-rank result
    (the reference's MPI_Allreduce, src/RTMCphon.f90:1584-1590)."""
    m, spec, gb = setup("film_mirror_transmit", nmode=5)
    o = orc.Oracle(model=m, spectrum=spec)
    run = A.make_run(kind_mfp=A.MFP_GRID, nangle=7, np_=150, seed=99, mfp_grid=[40.0])
    cnt_o, _, _ = o.counts(run)
    with A.Handle(gb.view, spec) as h:
        t1, e1 = h.transmission(40.0, 7, 150, seed=99, precision=A.PREC_FP64)
        t_r0, _ = h.transmission(40.0, 7, 150, rank=0, nranks=2, seed=99, precision=A.PREC_FP64)
        t_r1, _ = h.transmission(40.0, 7, 150, rank=1, nranks=2, seed=99, precision=A.PREC_FP64)
    ref = (cnt_o / 150.0).reshape(6, 5)  # (angle, mode) with nbranch = 1
    np.testing.assert_array_equal(t1[0, :, :6].T, ref)
    assert np.all(t1[:, :, 6] == 0.0)
    np.testing.assert_allclose(t_r0 + t_r1, t1, rtol=0, atol=1e-15)
    np.testing.assert_allclose(e1, np.sqrt(t1 * (1 - t1) / 150.0))


def _z(c1, c2, n):
    p1, p2 = c1 / n, c2 / n
    var = (p1 * (1 - p1) + p2 * (1 - p2)) / n
    return (p1 - p2) / np.sqrt(np.maximum(var, 0.5 / n / n))


@pytest.mark.parametrize("name", ["nanowire_diffuse", "film_periodic", "film_mirror_transmit", "spheres",
                                  "brick_quads", "brick_tris", "spheres_gamma", "spheres_gamma_2mat",
                                  "brick_tbc", "brick_tbc_2mat"])
def test_fp32_statistical_parity(orc, name):
    """Per-mode transmission sums and kappa of the FP32 kernel vs the oracle:
    every |z| < 5 and the kappa difference within 4 combined standard errors."""
    m, spec, gb = setup(name, nmode=24, seed=5)
    o = orc.Oracle(model=m, spectrum=spec)
    np_ = 2000
    run64 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=np_, seed=1, nbins=4,
                       bin_omega=(0.0, float(spec.omega.max())))
    cnt_o, lost_o, _ = o.counts(run64)
    ko = o.kappa(run64, cnt_o)
    run32 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=np_, seed=2, nbins=4,
                       bin_omega=(0.0, float(spec.omega.max())), precision=A.PREC_FP32)
    with A.Handle(gb.view, spec) as h:
        kg = h.kappa(run32, want_counts=True)
    assert kg["lost"] <= max(2, 1e-4 * kg["samples"])
    z = _z(kg["counts"].astype(float), cnt_o.astype(float), np_)
    assert np.max(np.abs(z)) < 5.0, np.max(np.abs(z))
    se = np.hypot(kg["kappa_stderr"], ko["kappa_stderr"])
    assert abs(kg["kappa"] - ko["kappa"]) < 4 * se + 1e-12 * abs(ko["kappa"]), (kg["kappa"], ko["kappa"], se)
    seb = np.hypot(kg["bin_T_stderr"], ko["bin_T_stderr"])
    assert np.all(np.abs(kg["bin_T"] - ko["bin_T"]) < 4 * seb + 1e-12)


def test_device_reduction_matches_host_assembly():
    m, spec, gb = setup("film_periodic", nmode=30)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=300, seed=4, nbins=6,
                     bin_omega=(0.0, float(spec.omega.max())))
    with A.Handle(gb.view, spec) as h:
        kg = h.kappa(run, want_counts=True)
    kh = A.kappa_from_counts(gb.view, spec, run, kg["counts"])
    assert kg["kappa"] == pytest.approx(kh["kappa"], rel=1e-12)
    assert kg["kappa_stderr"] == pytest.approx(kh["kappa_stderr"], rel=1e-10)
    np.testing.assert_allclose(kg["bin_T"], kh["bin_T"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(kg["emfp_nm"], kh["emfp_nm"], rtol=1e-12)


@pytest.mark.parametrize("prec", [A.PREC_FP32, A.PREC_FP64])
def test_ballistic_specular_duct_transmits_everything(prec):
    m = synth.nanowire(length=500.0, width=50.0, height=50.0, p_side=1.0)
    spec = synth.spectrum(4, seed=0)
    gb = A.GeomBuf(m)
    run = A.make_run(kind_mfp=A.MFP_MATTHIESSEN, nangle=11, np_=500, seed=3, precision=prec)
    with A.Handle(gb.view, spec) as h:
        k = h.kappa(run, want_counts=True)
    assert np.all(k["counts"] == 500)
    assert k["lost"] == 0


@pytest.mark.parametrize("prec", [A.PREC_FP32, A.PREC_FP64])
def test_lost_phonons_with_flight_cap(orc, prec):
    m, spec, gb = setup("nanowire_diffuse", nmode=3)
    run = A.make_run(kind_mfp=A.MFP_MATTHIESSEN, nangle=5, np_=300, seed=5, precision=prec)
    with A.Handle(gb.view, spec, max_flights=1) as h:
        a = h.kappa(run, want_counts=True)
        sa = h.stats()
    with A.Handle(gb.view, spec, max_flights=1, ref_quirks=1) as h:
        b = h.kappa(run, want_counts=True)
    assert sa["capped"] > 0 and a["lost"] == sa["capped"]
    assert int(b["counts"].sum()) == int(a["counts"].sum()) + a["lost"]
    with A.Handle(gb.view, spec, max_flights=1, lost_limit=1e-3) as h:
        with pytest.raises(A.PtgError) as e:
            h.kappa(run)
        assert e.value.status == A.PTG_ERR_LOST


def test_rank_partition_is_exact_fp32():
    """Counts of two FP32 ranks sum to the single-rank counts exactly: every
    trajectory depends only on its Philox counter."""
    m, spec, gb = setup("film_periodic", nmode=8)
    kw = dict(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=301, seed=8, precision=A.PREC_FP32)
    with A.Handle(gb.view, spec) as h:
        full = h.kappa(A.make_run(**kw), want_counts=True)["counts"]
        r0 = h.kappa(A.make_run(rank=0, nranks=2, **kw), want_counts=True)["counts"]
        r1 = h.kappa(A.make_run(rank=1, nranks=2, **kw), want_counts=True)["counts"]
        again = h.kappa(A.make_run(**kw), want_counts=True)["counts"]
    np.testing.assert_array_equal(r0 + r1, full)
    np.testing.assert_array_equal(again, full)


@pytest.mark.parametrize("name", ["film_periodic", "film_mirror_transmit", "spheres", "brick_tris",
                                  "nanowire_mixed", "capped", "lattice_tris"])
@pytest.mark.parametrize("cap", [0, 40])
def test_cooperative_tail_takes_the_same_trajectories(name, cap):
    """The tail phase (a warp of cooperating lanes per diffusive phonon once
    the queue is dry: handed over at once with coop_lanes = 32, or when a
    warp holds at most 8 or 1 live phonons) and the one-lane path to the end
    (tune_flags bit 1) give identical per-task counts, lost counts and
    flight totals: a flight advances the position with the same rounding on
    every path, so the trajectory depends only on its Philox counter.  The
    tail phase takes its surface events inside the rounds, orders its list
    by expected walk, and in a BVH grain (lattice_tris: 324 triangles) tests
    flights against its warp's local list of the nearest triangles.  With
    the fast path off (tune_flags bit 0) no safe ball or grain ball is ever
    computed and every flight takes the full test, so the variants without
    it also show that the tests the balls skip could not have hit."""
    m = geometries()[name]
    spec = synth.spectrum(12, seed=5, mfp_lo=1e-9, mfp_hi=3e-8)
    gb = A.GeomBuf(m)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=257, seed=21, precision=A.PREC_FP32)
    out = {}
    for key, opts in (("lane", dict(tune_flags=2)), ("coop8", dict(coop_lanes=8)),
                      ("tail", dict()), ("coop_nofast", dict(tune_flags=1)),
                      ("coop1", dict(coop_lanes=1)), ("lane_nofast", dict(tune_flags=3))):
        with A.Handle(gb.view, spec, max_flights=cap, **opts) as h:
            k = h.kappa(run, want_counts=True)
            out[key] = (k["counts"], k["lost"], h.stats())
    base_counts, base_lost, base_st = out["lane"]
    assert base_st["coop_rounds"] == 0
    for key in ("coop8", "tail", "coop_nofast", "coop1", "lane_nofast"):
        counts, lost, st = out[key]
        np.testing.assert_array_equal(counts, base_counts, err_msg=key)
        assert lost == base_lost, key
        assert st["flights"] == base_st["flights"], key
        assert st["max_traj_flights"] == base_st["max_traj_flights"], key
    for key in ("tail", "coop8", "coop1"):
        assert out[key][2]["coop_rounds"] > 0 and out[key][2]["coop_flights"] > 0, key
    if cap:
        assert base_lost > 0



def _many_spheres(n=40, l=400.0, seed=0):
    rng = np.random.default_rng(seed)
    c, r = [], []
    while len(c) < n:
        rr = rng.uniform(8.0, 20.0)
        p = rng.uniform(rr + 5.0, l - rr - 5.0, 3)
        if all(np.linalg.norm(p - q) > rr + s + 2.0 for q, s in zip(c, r)):
            c.append(p)
            r.append(rr)
    return synth.spheres_in_box(l=l, centres=[tuple(x) for x in c], radii=r, t=0.4, p=0.3, p_wall=0.2)


@pytest.mark.parametrize("name", ["lattice", "spheres", "holes", "capped"])
def test_bvh_and_linear_scan_take_the_same_trajectories(name):
    """A grain with more than 32 candidates gets a BVH; its nearest hit is the
    linear scan's (nearest raw distance, ties to the lower surface index) and
    the BVH-pruned safe ball does not change the trajectory, so counts,
    lost counts and flight totals are identical for every leaf size and with
    no BVH at all (bvh_leaf = -1)."""
    m = {"lattice": lambda: synth.cube_lattice(n=4, l=400.0, fill=0.5, trans=0.3, spec=0.2, p_wall=0.3),
         "spheres": _many_spheres,
         "holes": lambda: synth.film_with_holes(lx=600.0, ly=600.0, lz=100.0, nholes=40, radius=20.0,
                                                seed=5, p_hole=0.3, t_hole=0.2),
         "capped": lambda: synth.spheres_cylinders_box(n_spheres=12, n_cylinders=30, l=600.0, seed=6,
                                                       r_sphere=(10.0, 30.0), r_cylinder=15.0,
                                                       length=(40.0, 120.0), trans=0.3, p_wall=0.2)}[name]()
    spec = synth.spectrum(10, seed=7, mfp_lo=2e-9, mfp_hi=1e-6)
    gb = A.GeomBuf(m)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=203, seed=3, precision=A.PREC_FP32)
    ref = None
    for leaf in (-1, 1, 4, 8):
        with A.Handle(gb.view, spec, bvh_leaf=leaf) as h:
            k = h.kappa(run, want_counts=True)
            st = h.stats()
        cur = (k["counts"], k["lost"], st["flights"], st["max_traj_flights"])
        if ref is None:
            ref = cur
            continue
        np.testing.assert_array_equal(cur[0], ref[0], err_msg=f"leaf {leaf}")
        assert cur[1:] == ref[1:], leaf


def test_autotune_keeps_results_and_caches(tmp_path):
    """ptg_autotune leaves valid options on the handle, every option it tries
    gives the same counts (trajectories depend only on Philox counters), and
    the Python cache reapplies the stored options without timing."""
    m = synth.cube_lattice(n=4, l=400.0, fill=0.5, trans=0.3, spec=0.2, p_wall=0.3)
    spec = synth.spectrum(10, seed=9, mfp_lo=2e-9, mfp_hi=1e-6)
    gb = A.GeomBuf(m)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=101, seed=4, precision=A.PREC_FP32)
    cache = str(tmp_path / "tune.json")
    with A.Handle(gb.view, spec) as h:
        base = h.kappa(run, want_counts=True)["counts"]
        res = h.autotune(run, reps=1, cache=cache, key="lattice4")
        o = h.options()
        assert not res["cached"] and res["kernel_ms"] > 0
        assert o["block_size"] in (0, 128, 256) and o["bvh_leaf"] in (0, 1, 2, 4, 8, 16)
        np.testing.assert_array_equal(h.kappa(run, want_counts=True)["counts"], base)
        with pytest.raises(A.PtgError) as e:
            h.set_options(block_size=100)
        assert e.value.status == A.PTG_ERR_INVALID
    with A.Handle(gb.view, spec) as h:
        again = h.autotune(run, cache=cache, key="lattice4")
        assert again["cached"] and h.options() == o
        np.testing.assert_array_equal(h.kappa(run, want_counts=True)["counts"], base)


@pytest.mark.parametrize("lam", [2.0, 8.0])
def test_fp32_diffusive_limit_is_milne(lam):
    """Lambda << L in a specular duct (an infinite slab): the persistent FP32
    kernel, with its safe-ball fast path and cooperative tail doing most
    flights, gives Lambda_eff = Lambda L / (L + 2 z0 Lambda), z0 = 0.7104 the
    Milne extrapolation length (the reference's Simpson rule applied to the
    computed transmissions), within 3 sigma + 1 %."""
    L = 400.0
    m = synth.nanowire(length=L, width=40.0, height=40.0, p_side=1.0)
    spec = synth.spectrum(1, seed=0)
    gb = A.GeomBuf(m)
    npart = 40000
    run = A.make_run(kind_mfp=A.MFP_GRID, nangle=11, np_=npart, seed=13, mfp_grid=[lam],
                     precision=A.PREC_FP32)
    with A.Handle(gb.view, spec) as h:
        k = h.kappa(run, want_transmit=True)
        st = h.stats()
    if lam < 4.0:  # below a tenth of the smallest box side: fast path and cooperative tail
        assert st["coop_rounds"] > 0 and st["safe_balls"] > 0
    th = np.array([ia / 10 * math.pi / 2 for ia in range(11)])
    c = np.array([1, 4, 2, 4, 2, 4, 2, 4, 2, 4, 1], float)
    t = np.asarray(k["transmit"]).reshape(11, -1)[:, 0]
    s = 1.5 * L * (math.pi / 20) / 3
    semfp = s * np.sum(c * np.sin(th) * np.cos(th) * t)
    sigma = s * math.sqrt(np.sum((c * np.sin(th) * np.cos(th)) ** 2 * t * (1 - t) / npart))
    expect = lam * L / (L + 2 * 0.7104 * lam)
    assert abs(semfp - expect) < 3 * sigma + 0.01 * expect, (semfp, expect, sigma)


def test_headline_thin_film_matches_the_oracle(orc):
    """The bench workload's structure and full spectrum (thin film 300 x 300 x
    145 nm, 3 void holes r = 50 nm, y periodic, diffuse walls; 2000 modes with
    MFPs from 1 nm to 10 um, 64 frequency bins) at 20 particles per (mode,
    angle): the FP32 kernel's kappa within 3 combined standard errors of the
    FP64 oracle's (independent seeds) and every populated bin's transmission
    within 4."""
    model = synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=0,
                                  periodic_y=True, p_hole=0.0, t_hole=0.0, p_z=0.0)
    spec = synth.spectrum(2000, seed=0)
    bins = dict(temperature=300.0, nbins=64, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))
    run64 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=20, seed=777, **bins)
    run32 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=11, np_=20, seed=12345, precision=A.PREC_FP32,
                       **bins)
    o = orc.Oracle(model=model, spectrum=spec)
    cnt_o, _, _ = o.counts(run64)
    ko = o.kappa(run64, cnt_o)
    gb = A.GeomBuf(model)
    with A.Handle(gb.view, spec) as h:
        kg = h.kappa(run32)
        st = h.stats()
    assert st["lost"] <= 1e-5 * st["samples"]
    se = math.hypot(kg["kappa_stderr"], ko["kappa_stderr"])
    z = (kg["kappa"] - ko["kappa"]) / se
    assert abs(z) < 3.0, (kg["kappa"], ko["kappa"], se)
    seb = np.hypot(kg["bin_T_stderr"], ko["bin_T_stderr"])
    live = seb > 0
    assert live.sum() >= 60
    zb = (kg["bin_T"][live] - ko["bin_T"][live]) / seb[live]
    assert np.max(np.abs(zb)) < 4.0, np.max(np.abs(zb))


def test_triangulated_polycrystal_matches_its_polygon_form(orc):
    """A Voronoi polycrystal (grain boundaries T = 0.5, p = 0, diffuse walls)
    given as polygons and as a triangle mesh of the same facets (4^2 triangles
    per fan triangle, a BVH in every grain) is the same structure: the FP32
    kappa of the mesh form agrees with the oracle's polygon run within 4
    combined standard errors, and every per-task |z| < 5."""
    kw = dict(box=(300.0, 250.0, 250.0), seed=5, trans=0.5, spec=0.0, p_wall=0.0)
    poly = synth.voronoi_box(5, **kw)
    mesh = synth.voronoi_box(5, tri_levels=2, **kw)
    spec = synth.spectrum(12, seed=9, mfp_lo=10e-9, mfp_hi=2e-6)
    np_ = 1500
    run64 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=np_, seed=3)
    run32 = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=np_, seed=4, precision=A.PREC_FP32)
    o = orc.Oracle(model=poly, spectrum=spec)
    cnt_o, _, _ = o.counts(run64)
    ko = o.kappa(run64, cnt_o)
    gb = A.GeomBuf(mesh)
    with A.Handle(gb.view, spec) as h:
        kg = h.kappa(run32, want_counts=True)
        st = h.stats()
    assert st["box_tests"] > 0  # the grains' BVHs were walked
    z = _z(kg["counts"].astype(float), cnt_o.astype(float), np_)
    assert np.max(np.abs(z)) < 5.0
    se = np.hypot(kg["kappa_stderr"], ko["kappa_stderr"])
    assert abs(kg["kappa"] - ko["kappa"]) < 4 * se, (kg["kappa"], ko["kappa"], se)
