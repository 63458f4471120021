"""ptg_transmission_noalloc: the FP32 transmission function for hosts that
cannot allocate memory while they run (device memory reserved up front by
another framework, or a service that must keep a fixed footprint).

The entry point keeps the kernel's scratch in a fixed static device array, so
its result must equal ptg_transmission's (FP32 path, integer tallies: exact)
on consecutive calls, which also shows that each call clears the shared array
it reuses.  This file is collected last so that a failure here leaves every
other test already run; it also passes on its own in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu

# phonons the static tail-phase list holds (noalloc.cu kMaxTail)
NOALLOC_TAIL_CAP = 65536


def _handle(**opts):
    model = synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=6)
    spec = synth.spectrum(40, seed=2)
    gb = A.GeomBuf(model)
    return gb, spec, A.Handle(gb.view, spec, **opts)


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


def test_noalloc_tail_list_overflow_keeps_every_phonon():
    """A strongly diffusive run (MFP 2 nm in a 145 nm film) with every lane
    refilled at once keeps more phonons alive when the work queue runs dry than
    the fixed 65536-phonon tail list holds.  The list admits exactly its
    capacity, the rest stay in the drain phase, and no phonon is lost from the
    counts: the result equals ptg_transmission's (whose list has a slot per
    lane) bit for bit, on two calls in a row."""
    model = synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=6)
    spec = synth.spectrum(1, seed=2)
    gb = A.GeomBuf(model)
    with A.Handle(gb.view, spec, regen_threshold=1) as h:
        args = (2.0, 11, 24000)
        want, _ = h.transmission(*args, seed=5, precision=A.PREC_FP32)
        sw = h.stats()
        assert sw["tail_refused"] == 0
        for _ in range(2):
            got = h.transmission_noalloc(*args, seed=5)
            st = h.stats()
            assert st["tail_refused"] > 0, st
            assert st["tail_phonons"] == NOALLOC_TAIL_CAP, st
            assert st["samples"] == sw["samples"] == 10 * 24000
            assert st["flights"] == sw["flights"]
            np.testing.assert_array_equal(got, want)


def test_noalloc_applies_the_lost_phonon_limit():
    """A flight cap of 2 loses most phonons of a diffusive run; with a lost
    limit of 1% both entry points return PTG_ERR_LOST."""
    gb, spec, h = _handle(max_flights=2, lost_limit=0.01)
    with h:
        for call in (lambda: h.transmission(3.0, 5, 64, seed=1, precision=A.PREC_FP32),
                     lambda: h.transmission_noalloc(3.0, 5, 64, seed=1)):
            with pytest.raises(A.PtgError) as e:
                call()
            assert e.value.status == A.PTG_ERR_LOST


def test_noalloc_timeout_returns_no_counts():
    """On PTG_ERR_TIMEOUT the no-alloc entry leaves zeros in the caller's
    array, never raw count bits."""
    gb, spec, h = _handle(tune_flags=4)  # tune_flags bit 2: staging copy not issued (test only)
    with h:
        t = np.full(spec.nmode * 7, np.nan)
        st = h.lib.ptg_transmission_noalloc(h.h, 20.0, 7, 300, 0, 1, 3, t.ctypes.data_as(C.POINTER(C.c_double)))
        assert st == A.PTG_ERR_TIMEOUT
        assert np.all(t == 0.0)
        h.set_options(tune_flags=0)
        got = h.transmission_noalloc(20.0, 7, 300, seed=3)
        want, _ = h.transmission(20.0, 7, 300, seed=3, precision=A.PREC_FP32)
        np.testing.assert_array_equal(got, want)


def test_noalloc_rejects_runs_beyond_its_fixed_scratch():
    spec = synth.spectrum(A.NOALLOC_MAX_TASKS // 10 + 1, seed=1)
    gb = A.GeomBuf(synth.nanowire())
    with A.Handle(gb.view, spec) as h:
        with pytest.raises(A.PtgError) as e:
            h.transmission_noalloc(10.0, 11, 10)
        assert e.value.status == A.PTG_ERR_INVALID
