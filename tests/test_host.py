"""Host-side checks of the product library that need no GPU: the C ABI loads
and exports every entry point of include/ptrans_gpu.h, the host geometry
builder equals the oracle's restatement of setupBoxGrain / setupFillGrain /
setupSurfaceGeometry bit for bit, the host FP64 kappa assembly equals the
oracle's effectiveMFP + fileoutput, the input readers round-trip, and a
missing device is reported as an error status."""
import os
import re

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ptrans_gpu.h")


def header_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"\b(ptg_[a-z_0-9]+)\s*\(", txt)))


def test_library_exports_every_header_function():
    import ctypes
    lib = ctypes.CDLL(A.LIB_PATH)
    names = header_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing
    assert set(names) == set(A.SIGNATURES), set(names) ^ set(A.SIGNATURES)


def test_strerror_for_every_status():
    lib = A.load_library()
    for st in range(0, 9):
        assert lib.ptg_strerror(st)
    assert lib.ptg_strerror(0) == b"ok"


def models():
    return {
        "nanowire": synth.nanowire(length=400.0, width=60.0, height=80.0, p_side=0.3),
        "film": synth.film_with_holes(seed=4),
        "film_mirror": synth.film_with_holes(seed=5, periodic_y=False, p_hole=0.4, t_hole=0.2),
        "spheres": synth.spheres_in_box(centres=((60, 70, 80), (140, 130, 120)), radii=(30, 45), t=0.3, p=0.5),
        "brick_quads": synth.brick_box(t=0.5, p=0.25),
        "brick_tris": synth.brick_box(t=0.5, p=0.25, triangles=True),
        "fluct": _with(synth.brick_box(t=0.5, p=0.5), specfluc=0.2, fluct_seed=77),
    }


def _with(m, **kw):
    for k, v in kw.items():
        setattr(m, k, v)
    return m


@pytest.mark.parametrize("name", list(models()))
def test_geometry_builder_matches_oracle(orc, name):
    m = models()[name]
    prod = A.GeomBuf(m).numpy()
    ref = orc.Oracle(model=m).geometry()
    for k, v in ref.items():
        np.testing.assert_array_equal(np.asarray(prod[k]), np.asarray(v), err_msg=k)


def test_geometry_rejects_bad_input():
    m = synth.brick_box()
    m.facet_vertex = m.facet_vertex.copy()
    m.facet_vertex[:9] = 0.0  # first facet collapses to a point
    with pytest.raises(A.PtgError) as e:
        A.GeomBuf(m)
    assert e.value.status == A.PTG_ERR_INVALID
    m2 = synth.film_with_holes(seed=1)
    m2.face_kind = (A.FACE_PERIODIC, A.FACE_PERIODIC, 0, 0, 0, 0)
    with pytest.raises(A.PtgError):
        A.GeomBuf(m2)
    m3 = synth.nanowire()
    m3.grain_shape = np.zeros(0, np.int32)
    with pytest.raises(A.PtgError):
        A.GeomBuf(m3)


@pytest.mark.parametrize("kind", [A.MFP_PER_MODE, A.MFP_MATTHIESSEN, A.MFP_GRID])
def test_host_kappa_assembly_matches_oracle(orc, kind):
    m = synth.film_with_holes(seed=2)
    spec = synth.spectrum(40, seed=9)
    gb = A.GeomBuf(m)
    o = orc.Oracle(model=m, spectrum=spec)
    grid = np.geomspace(2.0, 5000.0, 6) if kind == A.MFP_GRID else None
    run = A.make_run(kind_mfp=kind, nangle=7, np_=30, seed=3, nbins=8,
                     bin_omega=(0.0, float(spec.omega.max())), mfp_grid=grid)
    cnt, lost, _ = o.counts(run)
    ref = o.kappa(run, cnt)
    got = A.kappa_from_counts(gb.view, spec, run, cnt)
    assert got["kappa"] == pytest.approx(ref["kappa"], rel=1e-12)
    assert got["kappa_stderr"] == pytest.approx(ref["kappa_stderr"], rel=1e-9)
    np.testing.assert_allclose(got["emfp_nm"], ref["emfp_nm"], rtol=1e-12)
    np.testing.assert_allclose(got["bin_T"], ref["bin_T"], rtol=1e-12, atol=1e-15)
    np.testing.assert_allclose(got["bin_T_stderr"], ref["bin_T_stderr"], rtol=1e-9, atol=1e-15)


def test_create_without_device_reports_status():
    from conftest import gpu_available
    if gpu_available():
        pytest.skip("a device is present")
    m = synth.nanowire()
    spec = synth.spectrum(4, seed=0)
    gb = A.GeomBuf(m)
    with pytest.raises(A.PtgError) as e:
        A.Handle(gb.view, spec)
    assert e.value.status == A.PTG_ERR_NO_DEVICE


def test_mcp_round_trip(tmp_path):
    for m in (synth.film_with_holes(seed=8, periodic_y=False), synth.nanowire(), synth.brick_box(triangles=True),
              synth.spheres_in_box()):
        p = str(tmp_path / "x.mcp")
        synth.write_mcp(m, p, np_=123, nangle=9, mean_free_path="1 1000 5 log")
        back, info = A.mcp_load(p)
        assert info["np"] == 123 and info["nangle"] == 9 and info["kind_mfp"] == A.MFP_GRID
        np.testing.assert_allclose(info["mfp_grid"], np.geomspace(1, 1000, 5), rtol=1e-12)
        g1 = A.GeomBuf(m).numpy()
        g2 = A.GeomBuf(back).numpy()
        for k in g1:
            np.testing.assert_allclose(np.asarray(g2[k], float), np.asarray(g1[k], float), rtol=1e-8,
                                       atol=1e-8, err_msg=k)


def test_anphon_round_trip(tmp_path):
    s = synth.spectrum(50, seed=4)
    p = str(tmp_path / "Si.anphon")
    A.anphon_write(p, s)
    b = A.anphon_load(p)
    np.testing.assert_allclose(b.omega, s.omega, rtol=1e-14)
    np.testing.assert_array_equal(b.tau, s.tau)
    np.testing.assert_array_equal(b.vel, s.vel)
    assert b.nbranch == 1 and b.rtemp == s.rtemp and b.vol == s.vol


REF_EXAMPLES = "/root/reference/Examples"


@pytest.mark.skipif(not os.path.isdir(REF_EXAMPLES), reason="reference examples not mounted")
def test_reference_examples_parse():
    """Counts from the shipped .mcp inputs (tests/golden/examples_summary.json
    holds the same figures for machines without the reference)."""
    import json
    want = json.load(open(os.path.join(ROOT, "tests", "golden", "examples_summary.json")))
    for name, w in want.items():
        m, info = A.mcp_load(os.path.join(REF_EXAMPLES, name))
        assert m.ngrain == w["ngrain"], name
        assert int(m.grain_nfacet.sum()) == w["nsurf"], name
        assert list(m.box) == w["box"], name
        assert info["np"] == w["np"] and info["nangle"] == w["nangle"], name
        g = A.GeomBuf(m).numpy()
        assert g["nsurf"] == w["built_nsurf"], name
        assert int(g["internal"].sum()) == w["built_internal"], name
