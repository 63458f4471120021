"""Host-side failure paths, each made on the host (no device involved):
malformed .mcp and .anphon inputs return PTG_ERR_IO, non-finite or
degenerate geometry returns PTG_ERR_INVALID, and an injected allocation
failure (ptg_debug_fail_allocations) returns PTG_ERR_NOMEM from the
geometry builder and the file loaders, at the first allocation and in the
middle of a build, with the library working normally afterwards.  The
reference reports the same kinds of failure through its loaders' status
argument (src/RTMCphon.f90:293-419, 661-733)."""
import dataclasses
import os

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth


def _mcp(tmp_path, name="ok.mcp", **kw):
    p = str(tmp_path / name)
    synth.write_mcp(synth.film_with_holes(seed=1, periodic_y=False), p, **kw)
    return p


@pytest.mark.parametrize("cut", ["truncated", "no_grains", "bad_number", "empty"])
def test_malformed_mcp_is_an_io_error(tmp_path, cut):
    good = open(_mcp(tmp_path)).read().splitlines()
    if cut == "truncated":
        lines = good[: len(good) // 2]
    elif cut == "no_grains":
        lines = [l for l in good if not l.startswith("Ng")]
    elif cut == "bad_number":
        i = next(i for i, l in enumerate(good) if l.startswith("LXcell"))
        lines = good[:i + 1] + ["\tnot-a-number"] + good[i + 2:]
    else:
        lines = []
    p = str(tmp_path / f"{cut}.mcp")
    open(p, "w").write("\n".join(lines) + "\n")
    with pytest.raises(A.PtgError) as e:
        A.mcp_load(p)
    assert e.value.status in (A.PTG_ERR_IO, A.PTG_ERR_INVALID)
    A.mcp_load(_mcp(tmp_path))  # a good file still loads


def test_missing_file_is_an_io_error(tmp_path):
    with pytest.raises(A.PtgError) as e:
        A.mcp_load(str(tmp_path / "absent.mcp"))
    assert e.value.status == A.PTG_ERR_IO
    with pytest.raises(A.PtgError) as e:
        A.anphon_load(str(tmp_path / "absent.anphon"))
    assert e.value.status == A.PTG_ERR_IO


@pytest.mark.parametrize("cut", ["short", "bad_value", "huge_count"])
def test_malformed_anphon_is_an_io_error(tmp_path, cut):
    p = str(tmp_path / "Si.anphon")
    A.anphon_write(p, synth.spectrum(10, seed=1))
    lines = open(p).read().splitlines()
    if cut == "short":
        lines = lines[:-3]
    elif cut == "bad_value":
        t = lines[8].split()
        t[3] = "x"
        lines[8] = " ".join(t)
    else:
        # a mode count far beyond the file: the loader must fail, not allocate it all
        t = lines[4].split()
        t[4] = "4000000000"
        lines[4] = " ".join(t)
    q = str(tmp_path / f"{cut}.anphon")
    open(q, "w").write("\n".join(lines) + "\n")
    with pytest.raises(A.PtgError) as e:
        A.anphon_load(q)
    assert e.value.status in (A.PTG_ERR_IO, A.PTG_ERR_NOMEM)


def test_non_finite_or_degenerate_geometry_is_invalid():
    base = synth.brick_box(t=0.5, p=0.2)
    v = base.facet_vertex.copy()
    v[4] = np.nan
    bad = {
        "nan_vertex": dataclasses.replace(base, facet_vertex=v),
        "inf_box": dataclasses.replace(base, box=(200.0, np.inf, 200.0)),
        "zero_box": dataclasses.replace(base, box=(200.0, 0.0, 200.0)),
        "nan_sphere": synth.spheres_in_box(centres=((np.nan, 100.0, 100.0),), radii=(40.0,)),
        "unknown_material": dataclasses.replace(base, grain_material=np.array([3], np.int32)),
    }
    for name, m in bad.items():
        with pytest.raises(A.PtgError) as e:
            A.GeomBuf(m)
        assert e.value.status == A.PTG_ERR_INVALID, name


def test_injected_allocation_failure_returns_nomem(tmp_path):
    m = synth.voronoi_box(5, box=(300.0, 200.0, 200.0), seed=2, trans=0.5)
    for after in (0, 1, 3):
        with A.fail_allocations(after):
            with pytest.raises(A.PtgError) as e:
                A.GeomBuf(m)
        assert e.value.status == A.PTG_ERR_NOMEM, after
    p = _mcp(tmp_path)
    with A.fail_allocations(0):
        with pytest.raises(A.PtgError) as e:
            A.mcp_load(p)
        assert e.value.status == A.PTG_ERR_NOMEM
    # injection off: the same calls succeed and give the same geometry
    g1 = A.GeomBuf(m).numpy()
    g2 = A.GeomBuf(m).numpy()
    assert g1["nsurf"] == g2["nsurf"] > 0
    np.testing.assert_array_equal(g1["vertex"], g2["vertex"])
    A.mcp_load(p)


def test_reserved_option_is_refused_before_any_device_work():
    lib = A.load_library()
    gb = A.GeomBuf(synth.nanowire())
    spec = synth.spectrum(4, seed=1)
    o = A.PtgOptions()
    o.reserved = 7
    import ctypes as C
    h = C.c_void_p()
    cs = spec.to_c()
    assert lib.ptg_create(C.byref(gb.view), C.byref(cs), C.byref(o), C.byref(h)) == A.PTG_ERR_INVALID
    assert not h.value
