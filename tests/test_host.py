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
        "voronoi": synth.voronoi_box(7, box=(300.0, 200.0, 250.0), seed=2, trans=0.5, spec=0.2),
        "lattice": synth.cube_lattice(n=3, l=300.0, fill=0.4, trans=0.2, spec=0.1),
        "capped": synth.spheres_cylinders_box(n_spheres=5, n_cylinders=6, l=400.0, seed=2,
                                              r_sphere=(15.0, 40.0), r_cylinder=20.0, length=(60.0, 200.0),
                                              trans=0.3),
        "voronoi_mesh": synth.voronoi_box(4, box=(300.0, 200.0, 250.0), seed=3, trans=0.5, spec=0.2,
                                          tri_levels=1),
        "gamma_2mat": synth.with_interface(synth.brick_box(t=0.5, p=0.25), A.TRANS_GAMMA, 1.2, spec=0.3,
                                           two_materials=True),
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


# the reference's Examples/ folder, where a checkout of it is at hand
REF_EXAMPLES = os.environ.get("PTRANS_REFERENCE_EXAMPLES", "")


@pytest.mark.skipif(not REF_EXAMPLES or not os.path.isdir(REF_EXAMPLES),
                    reason="PTRANS_REFERENCE_EXAMPLES does not name the reference's Examples folder")
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



@pytest.mark.parametrize("seed", range(4))
def test_voronoi_cells_tile_the_box(seed):
    """The generated Voronoi cells are closed, outward-oriented polyhedra that
    tile the box (volumes by the divergence theorem sum to the box volume),
    every internal facet i->j has its twin j->i of equal area, and box facets
    lie exactly on a box plane (so the builder marks them non-internal)."""
    box = (400.0, 300.0, 200.0)
    m = synth.voronoi_box(9, box=box, seed=seed)
    v = m.facet_vertex.reshape(-1, 3)
    k = f = 0
    vols, area = [], {}
    for g, nf in enumerate(m.grain_nfacet):
        vol = 0.0
        for _ in range(nf):
            nv = m.facet_nvertex[f]
            P = v[k:k + nv]
            k += nv
            a = 0.5 * sum(np.cross(P[i], P[(i + 1) % nv]) for i in range(nv))
            vol += float(np.dot(P[0], a)) / 3.0
            to = int(m.surf_grain_to[f])
            if to == 0:
                assert any(np.all(P[:, d] == 0.0) or np.all(P[:, d] == box[d]) for d in range(3))
            else:
                area[(g + 1, to)] = float(np.linalg.norm(a))
            f += 1
        assert vol > 0.0
        vols.append(vol)
    assert abs(sum(vols) - np.prod(box)) < 1e-9 * np.prod(box)
    for (a, b), x in area.items():
        assert abs(area[(b, a)] - x) < 1e-9 * max(x, 1.0)


def test_struct_layouts_agree_with_the_header(tmp_path):
    """Every ctypes mirror in abi.py has the C struct's size and field
    offsets (a C program compiled against include/ptrans_gpu.h prints them),
    and the Fortran ptg_options type lists the header's fields in order."""
    import ctypes
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    pairs = {"ptg_model": A.PtgModel, "ptg_spectrum": A.PtgSpectrum, "ptg_geometry": A.PtgGeometry,
             "ptg_options": A.PtgOptions, "ptg_run": A.PtgRun, "ptg_kappa_out": A.PtgKappaOut,
             "ptg_stats": A.PtgStats, "ptg_adjoint_out": A.PtgAdjointOut,
             "ptg_batch_item": A.PtgBatchItem, "ptg_batch_out": A.PtgBatchOut}
    lines = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void) {"]
    expect = []
    for cname, cls in pairs.items():
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expect.append(ctypes.sizeof(cls))
        for fname, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append(getattr(cls, fname).offset)
    lines.append("  return 0; }")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run([cc, "-std=c99", "-o", str(exe), str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got == expect
    txt = open(HEADER).read()
    body = txt[txt.index("typedef struct ptg_options {"):txt.index("} ptg_options;")]
    c_fields = re.findall(r"\b(?:int32_t|int64_t|double)\s+(\w+)\s*;", body)
    f90 = open(os.path.join(ROOT, "p-trans_b200", "fortran", "ptrans_gpu.f90")).read()
    ftype = f90[f90.index("type, bind(C), public :: ptg_options"):f90.index("end type ptg_options")]
    f_fields = []
    for line in ftype.splitlines()[1:]:
        if "::" in line:
            f_fields += [x.split("=")[0].strip() for x in line.split("::")[1].split(",")]
    assert f_fields == c_fields
    assert [n for n, _ in A.PtgOptions._fields_] == c_fields


@pytest.mark.parametrize("kind,v,w,d,text", [
    ("E", 1.0, 15, 6, "   0.100000E+01"),
    ("E", -1234.5, 15, 6, "  -0.123450E+04"),
    ("E", 0.0, 15, 6, "   0.000000E+00"),
    ("E", 9.9999996, 15, 6, "   0.100000E+02"),
    ("E", 3.0e-9, 15, 6, "   0.300000E-08"),
    ("E", 1.0e-120, 20, 10, "    0.1000000000-119"),
    ("E", 6.2831853e13, 20, 10, "    0.6283185300E+14"),
    ("F", 10.302305849, 20, 10, "       10.3023058490"),
    ("F", 0.5, 20, 10, "        0.5000000000"),
    ("F", 300.0, 0, 6, "300.000000"),
    ("I", 500, 6, 0, "   500"),
    ("I", 20000, 3, 0, "***"),
    ("I", 7, 5, 0, "    7"),
])
def test_fortran_edit_descriptors(kind, v, w, d, text):
    """The writer renders I, F and E descriptors as gfortran does: E with a
    0.d mantissa and a 2-digit exponent (3 digits without the E), F with its
    leading zero, asterisks when the field is too narrow."""
    assert A.fortran_format(kind, v, w, d) == text


def _two_branch_spectrum(nk=40, seed=3, ties=True):
    rng = np.random.default_rng(seed)
    nb = 2
    f = rng.uniform(0.5, 15.0, nb * nk)
    if ties:
        f[5] = f[7]          # equal frequencies in one branch (m = ib + nb*ik: both branch 1)
        f[2] = f[3]          # and across branches
    v = np.exp(rng.normal(np.log(4000.0), 0.5, nb * nk))
    mfp = np.exp(rng.uniform(np.log(2e-9), np.log(2e-6), nb * nk))
    return A.Spectrum(omega=f * synth.THZ, tau=mfp / v * 1e12, vel=v, weight=np.ones(nb * nk), nbranch=nb,
                      rtemp=300.0, vol=4e-29, mfp=mfp)


@pytest.mark.parametrize("kind", ["per_mode", "matthiessen", "grid"])
def test_writers_match_the_oracle_restatement(orc, tmp_path, kind):
    """ptg_write_outputs writes the same bytes as the oracle's restatement of
    fileoutput for the same counts: sorted records with tied effective MFPs
    (zero counts) and tied frequencies, two branches, every MFP rule."""
    m = synth.film_with_holes(lx=200.0, ly=200.0, lz=100.0, nholes=2, radius=30.0, seed=1)
    spec = _two_branch_spectrum()
    kw = {"per_mode": dict(kind_mfp=A.MFP_PER_MODE),
          "matthiessen": dict(kind_mfp=A.MFP_MATTHIESSEN),
          "grid": dict(kind_mfp=A.MFP_GRID, mfp_grid=[5.0, 50.0, 500.0])}[kind]
    run = A.make_run(nangle=7, np_=6, seed=11, precision=A.PREC_FP64, temperature=300.0, **kw)
    o = orc.Oracle(model=m, spectrum=spec)
    counts, _, _ = o.counts(run)
    gb = A.GeomBuf(m)
    (tmp_path / "a").mkdir()
    (tmp_path / "b").mkdir()
    A.write_outputs(str(tmp_path / "a" / "structure.mcp"), gb.view, spec, run, counts)
    o.write_outputs(str(tmp_path / "b" / "structure.mcp"), run, counts)
    for name in ("thermalproperty.out", "effectiveMFP.out", "phononconductivity.out"):
        a = (tmp_path / "a" / name).read_bytes()
        b = (tmp_path / "b" / name).read_bytes()
        assert a == b, name
    em = (tmp_path / "a" / "effectiveMFP.out").read_text().splitlines()
    assert len(em) == 6 + spec.nmode
    effs = [float(line[25:40]) for line in em[6:]]
    assert effs == sorted(effs)
    if kind == "per_mode":
        assert effs.count(0.0) >= 2   # zero counts: tied keys, the exchange-sort path
    pc = (tmp_path / "a" / "phononconductivity.out").read_text().splitlines()
    assert pc[1] == "# Nb = " + A.fortran_format("I", len(set(spec.omega)) - 1, 6)


@pytest.mark.parametrize("tbc_mw", [50.0, 300.0, 2000.0])
def test_gamma_from_tbc_matches_oracle_and_target(orc, tbc_mw):
    """ptg_gamma_from_tbc equals the oracle's GammaDeterm restatement bit for
    bit, and the gamma it returns reproduces the conductance: with
    T = 1/(gamma w/w_max + 1), G_T / (1 - G_T / G_1) = TBC (Newton's stop at
    |step| <= 1e-6 in gamma)."""
    spec = _two_branch_spectrum(nk=60, seed=8, ties=False)
    T = 300.0
    tbc = tbc_mw * 1e6
    st, g = A.gamma_from_tbc(spec, T, tbc)
    ost, og = orc.Oracle(model=synth.nanowire(), spectrum=spec).gamma_from_tbc(T, tbc)
    assert st == ost == 0 and g == og and g > 0
    hbar, kB = 1.054571e-34, 1.3806503e-23
    x = hbar * spec.omega / (kB * T)
    C = kB * ((x / 2) / np.sinh(x / 2)) ** 2
    nq = int(spec.weight.sum() / spec.nbranch)
    base = spec.weight * C * spec.vel / 2 / spec.vol / nq
    G1 = base.sum()
    GT = (base / (g * spec.omega / spec.omega.max() + 1)).sum()
    assert abs(GT / (1 - GT / G1) - tbc) < 1e-5 * tbc
