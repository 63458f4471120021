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
