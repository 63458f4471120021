"""Batched screening (ptg_batch_*): several structures in one persistent launch
replayed as a CUDA graph.  Each geometry must get exactly the counts of its
own ptg_kappa run with the same particles, seed and stream (integer tallies:
exact), and the same kappa (1e-12); replaying the graph gives the same
result again."""
import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu


def test_batch_equals_individual_runs():
    models, _ = synth.film_batch(n=6, seed=3, n_modes=40, nangle=9)
    nps = [17, 300, 5, 120, 64, 1]
    seeds = [1, 2, 3, 4, 5, 6]
    streams = [0, 7, 0, 3, 11, 2]
    spec = synth.spectrum(40, seed=1)
    bins = (0.0, float(spec.omega.max()))
    bufs = [A.GeomBuf(m) for m in models]
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=1, nbins=8, bin_omega=bins)
    with A.Batch([b.view for b in bufs], nps, seeds, streams, spec, run) as bt:
        r1 = bt.run(want_counts=True)
        r2 = bt.run(want_counts=True)
    np.testing.assert_array_equal(r1["counts"], r2["counts"])
    np.testing.assert_array_equal(r1["kappa"], r2["kappa"])
    for g in range(len(models)):
        single = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=9, np_=nps[g], seed=seeds[g],
                            stream=streams[g], nbins=8, bin_omega=bins)
        with A.Handle(bufs[g].view, spec) as h:
            k = h.kappa(single, want_counts=True)
        np.testing.assert_array_equal(r1["counts"][g], k["counts"])
        assert r1["kappa"][g] == pytest.approx(k["kappa"], rel=1e-12)
        assert r1["kappa_stderr"][g] == pytest.approx(k["kappa_stderr"], rel=1e-10)
        np.testing.assert_allclose(r1["bin_T"][g], k["bin_T"], rtol=1e-12, atol=1e-15)
    assert r1["samples"] == sum(nps) * 40 * 8
    assert r1["lost"] == 0


def test_batch_adjoint_equals_individual_adjoints():
    """ptg_batch_adjoint gives every geometry what ptg_adjoint gives for its
    own run: the same kappa (the same counts), the same replayed samples, the
    same specularity derivatives up to the order of the FP64 sums (the scores
    of the same samples, added in another order), and the scale derivative up
    to the FP32 summation order of the samples' path lengths."""
    import dataclasses
    models, _ = synth.film_batch(n=4, seed=5, n_modes=12, nangle=7)
    models = [dataclasses.replace(m, tt_spec=np.array([0.4, 0.0]), cellspec=(1.0, 1.0, 1.0, 1.0, 0.5, 0.3))
              for m in models]
    nps = [200, 50, 400, 10]
    seeds = [11, 12, 13, 14]
    streams = [0, 3, 1, 0]
    spec = synth.spectrum(12, seed=2)
    bins = (0.0, float(spec.omega.max()))
    bufs = [A.GeomBuf(m) for m in models]
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=1, nbins=4, bin_omega=bins, precision=A.PREC_FP32)
    with A.Batch([b.view for b in bufs], nps, seeds, streams, spec, run) as bt:
        ba = bt.adjoint()
        fwd = bt.run()
    assert ba["mismatched"] == 0
    # the same counts; host (adjoint) and device (forward) FP64 assembly differ in rounding only
    np.testing.assert_allclose(ba["kappa"], fwd["kappa"], rtol=1e-12)
    replayed = 0
    for g in range(len(models)):
        single = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=nps[g], seed=seeds[g], stream=streams[g],
                            nbins=4, bin_omega=bins, precision=A.PREC_FP32)
        with A.Handle(bufs[g].view, spec) as h:
            sa = h.adjoint(single)
        replayed += sa["replayed"]
        assert ba["kappa"][g] == pytest.approx(sa["kappa"], rel=1e-12)
        assert ba["kappa_stderr"][g] == pytest.approx(sa["kappa_stderr"], rel=1e-10)
        got, want, se = ba["dk_dp"][g], sa["dk_dp"], sa["dk_dp_stderr"]
        np.testing.assert_array_equal(np.isnan(got), np.isnan(want))
        ok = ~np.isnan(want)
        assert ok.sum() >= 3
        assert np.all(np.abs(got[ok] - want[ok]) <= 1e-6 * se[ok] + 1e-12 * np.abs(want[ok]))
        np.testing.assert_allclose(ba["dk_dp_stderr"][g][ok], se[ok], rtol=1e-6)
        # the scale score sums each sample's FP32 path length, in another order
        # where the single run's tail phase adds a round's flights by warp shuffles
        assert abs(ba["dk_dscale"][g] - sa["dk_dscale"]) <= 1e-3 * sa["dk_dscale_stderr"] + 1e-5 * abs(sa["dk_dscale"])
    assert ba["replayed"] == replayed
