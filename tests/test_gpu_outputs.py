"""GPU checks of the output paths: the trace replay (ptg_trace /
ptg_write_trace) re-generates exactly the trajectories of the forward run,
and the result files come from the device counts."""
import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu


def test_trace_replays_the_forward_trajectories(tmp_path):
    """Tracing every sample of a run gives the forward run's flight total and
    per-task transmitted counts exactly (the forward run takes its flights on
    the fast, cooperative and full paths, the trace on the full path only);
    traces start on x = 0 and end on the exit face."""
    m = synth.film_with_holes(lx=200.0, ly=150.0, lz=80.0, nholes=2, radius=25.0, seed=3,
                              p_hole=0.2, t_hole=0.0, p_z=0.4)
    spec = synth.spectrum(4, seed=2, mfp_lo=3e-9, mfp_hi=3e-7)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=50, seed=17, precision=A.PREC_FP32)
    ntask = 4 * 4
    gb = A.GeomBuf(m)
    with A.Handle(gb.view, spec) as h:
        fwd = h.kappa(run, want_counts=True)
        st = h.stats()
        tr = h.trace(run, np.arange(ntask * 50))
        h.write_trace(run, 7, str(tmp_path / "trace.out"))
    assert sum(len(p) - 1 for p, _ in tr) == st["flights"]
    counts = np.zeros(ntask, np.uint64)
    for s, (p, e) in enumerate(tr):
        if e == 2:
            counts[s // 50] += 1
        assert p[0, 0] == 0.0
        eps = 200.0 / 2 ** 20 * 4
        assert np.all(p[:, 0] >= -eps) and np.all(p[:, 0] <= 200.0 + eps)
        assert np.all(p[:, 2] >= -eps) and np.all(p[:, 2] <= 80.0 + eps)
        if e == 2:
            assert abs(p[-1, 0] - 200.0) <= eps
        elif e == 1:
            assert abs(p[-1, 0]) <= eps
    np.testing.assert_array_equal(counts, fwd["counts"])
    lines = (tmp_path / "trace.out").read_text().split("\n")
    assert lines[0] == "# Datatype = trace"
    assert lines[1] == "# particle_trace =        7"
    interval = ntask * 50 // 7
    assert lines[2] == f"# interval_trace = {interval:8d}"
    recs = [ln for ln in lines[4:] if ln.strip()]
    assert len(recs) == sum(len(tr[k * interval][0]) for k in range(7))
    first = np.array(recs[0].split(), dtype=np.float32)
    np.testing.assert_array_equal(first, tr[0][0][0])


def test_result_files_from_device_counts(tmp_path):
    """ptg_write_outputs on the counts of a device run writes the three files
    with one record per mode, kappa equal to ptg_kappa's to the printed
    digits."""
    m = synth.nanowire(length=300.0, width=60.0, height=50.0, p_side=0.3)
    spec = synth.spectrum(30, seed=4, mfp_lo=5e-9, mfp_hi=2e-6)
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=5, np_=400, seed=5, precision=A.PREC_FP32)
    gb = A.GeomBuf(m)
    with A.Handle(gb.view, spec) as h:
        k = h.kappa(run, want_counts=True)
    A.write_outputs(str(tmp_path / "wire.mcp"), gb.view, spec, run, k["counts"])
    tp = (tmp_path / "thermalproperty.out").read_text().splitlines()
    assert tp[0] == "# Datatype = thermalproperty"
    kap = float(tp[3].split("=")[1])
    assert abs(kap - k["kappa"]) <= 1e-9 * abs(k["kappa"]) + 1e-10
    em = (tmp_path / "effectiveMFP.out").read_text().splitlines()
    assert len(em) == 6 + 30
