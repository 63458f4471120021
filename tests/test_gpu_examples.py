"""The reference's own example structures end to end on the GPU.

tests/golden/examples_models.json holds Examples/01-05 as parsed by
ptg_mcp_load (src/RTMCphon.f90:252-1251; the generating script is
tests/golden/make_examples_models.py).  The reference's material database is
not shipped with it, so a seeded synthetic Si.anphon stands in for
Materials/Si.anphon: it is written with ptg_anphon_write and read back with
ptg_anphon_load (src/RTMCphon.f90:661-733).  Each structure then runs with
the example's own Np, Nangle and MFP settings through ptg_create and
ptg_kappa on the plain FP64 kernel, and
  - the transmitted counts equal the oracle's exactly,
  - kappa and the effective MFPs equal the oracle's to 1e-12,
  - the three result files of ptg_write_outputs are byte-identical to the
    oracle's restatement of fileoutput (src/RTMCphon.f90:2601-2881),
and the persistent FP32 kernel's kappa agrees within 4 combined standard
errors.
"""
import json
import math
import os

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURE = os.path.join(HERE, "golden", "examples_models.json")


def _examples():
    if not os.path.exists(FIXTURE):
        return {}
    return json.load(open(FIXTURE))


def _model(rec):
    fields = {k: v for k, v in rec.items() if k != "info"}
    for k in ("box", "cellspec", "face_kind", "scope"):
        fields[k] = tuple(fields[k])
    return A.Model(**fields)


def _run(info, precision, seed):
    kind = info["kind_mfp"]
    grid = info["mfp_grid"] if kind == A.MFP_GRID else None
    return A.make_run(kind_mfp=kind, nangle=info["nangle"], np_=info["np"], seed=seed, precision=precision,
                      mfp_grid=grid, nbins=8, bin_omega=(0.0, 15.0 * 2 * math.pi * 1e12))


@pytest.mark.skipif(not os.path.exists(FIXTURE), reason="example fixture missing")
@pytest.mark.parametrize("name", sorted(_examples()))
def test_reference_example_end_to_end(orc, name, tmp_path):
    rec = _examples()[name]
    info = rec["info"]
    model = _model(rec)
    mat = tmp_path / "Materials"
    mat.mkdir()
    apath = str(mat / f"{info['material1']}.anphon")
    A.anphon_write(apath, synth.spectrum(16, seed=3))
    spec = A.anphon_load(apath)
    gb = A.GeomBuf(model)
    o = orc.Oracle(model=model, spectrum=spec)
    run64 = _run(info, A.PREC_FP64, seed=2024)
    cnt_o, lost_o, res_o = o.counts(run64)
    ko = o.kappa(run64, cnt_o)
    with A.Handle(gb.view, spec) as h:
        kg = h.kappa(run64, want_counts=True)
        run32 = _run(info, A.PREC_FP32, seed=99)
        k32 = h.kappa(run32)
    np.testing.assert_array_equal(kg["counts"], cnt_o)
    assert kg["flights"] == res_o["flights"] and kg["lost"] == res_o["lost"]
    assert kg["kappa"] == pytest.approx(ko["kappa"], rel=1e-12)
    np.testing.assert_allclose(kg["emfp_nm"], ko["emfp_nm"], rtol=1e-12, atol=1e-12)
    se = math.hypot(k32["kappa_stderr"], ko["kappa_stderr"])
    assert abs(k32["kappa"] - ko["kappa"]) < 4 * se + 1e-12 * abs(ko["kappa"])
    # fileoutput's three files from the GPU counts vs the oracle's restatement
    ours, theirs = tmp_path / "ours", tmp_path / "oracle"
    ours.mkdir()
    theirs.mkdir()
    A.write_outputs(str(ours / name), gb.view, spec, run64, kg["counts"])
    o.write_outputs(str(theirs / name), run64, cnt_o)
    files = sorted(os.listdir(theirs))
    assert files == sorted(os.listdir(ours)) and len(files) == 3
    for f in files:
        assert (ours / f).read_bytes() == (theirs / f).read_bytes(), f
