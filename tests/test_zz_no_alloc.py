"""ptg_transmission_noalloc: the FP32 transmission function for hosts that
cannot allocate memory while they run (device memory reserved up front by
another framework, or a service that must keep a fixed footprint).

The entry point keeps the kernel's scratch in a fixed static device array, so
its result must equal ptg_transmission's (FP32 path, integer tallies: exact)
on consecutive calls, which also shows that each call clears the shared array
it reuses.  This file is collected last so that a failure here leaves every
other test already run; it also passes on its own in a fresh process.
"""
import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu


def _handle():
    model = synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=6)
    spec = synth.spectrum(40, seed=2)
    gb = A.GeomBuf(model)
    return gb, spec, A.Handle(gb.view, spec)


def test_noalloc_matches_transmission_on_consecutive_calls():
    gb, spec, h = _handle()
    with h:
        cases = [(25.0, 11, 400, 0, 1, 17), (3.0, 7, 333, 1, 2, 99)]
        for mfp, nangle, np_, rank, nranks, seed in cases:
            want, _ = h.transmission(mfp, nangle, np_, rank=rank, nranks=nranks, seed=seed,
                                     precision=A.PREC_FP32)
            got1 = h.transmission_noalloc(mfp, nangle, np_, rank=rank, nranks=nranks, seed=seed)
            got2 = h.transmission_noalloc(mfp, nangle, np_, rank=rank, nranks=nranks, seed=seed)
            np.testing.assert_array_equal(got1, want)
            np.testing.assert_array_equal(got2, want)
            assert np.all(want[:, :, -1] == 0.0) and want[:, :, :-1].sum() > 0


def test_noalloc_rejects_runs_beyond_its_fixed_scratch():
    spec = synth.spectrum(A.NOALLOC_MAX_TASKS // 10 + 1, seed=1)
    gb = A.GeomBuf(synth.nanowire())
    with A.Handle(gb.view, spec) as h:
        with pytest.raises(A.PtgError) as e:
            h.transmission_noalloc(10.0, 11, 10)
        assert e.value.status == A.PTG_ERR_INVALID
