"""Error paths of the GPU transport, made without any device fault.

The persistent FP32 kernel stages a small geometry blob into shared memory
with one bulk copy and waits for it on an mbarrier with a bounded wait.  The
test-only option tune_flags bit 2 sets the barrier up without issuing the
copy, so the wait must run out with nothing in flight: the call returns
PTG_ERR_TIMEOUT, and the same handle then computes the right result once the
option is cleared (the context stays usable).  Invalid options are refused
with PTG_ERR_INVALID and leave the handle usable.
"""
import numpy as np
import pytest

from ptrans_b200 import abi as A
from ptrans_b200 import synth

pytestmark = pytest.mark.gpu

STAGE_TEST = 4  # tune_flags bit 2


def _film():
    model = synth.film_with_holes(lx=300.0, ly=300.0, lz=145.0, nholes=3, radius=50.0, seed=1)
    return A.GeomBuf(model), synth.spectrum(8, seed=1)


def test_staging_wait_runs_out_and_the_handle_recovers():
    gb, spec = _film()
    with A.Handle(gb.view, spec) as ref:
        want, _ = ref.transmission(20.0, 7, 300, seed=3, precision=A.PREC_FP32)
    with A.Handle(gb.view, spec, tune_flags=STAGE_TEST) as h:
        for _ in range(2):
            with pytest.raises(A.PtgError) as e:
                h.transmission(20.0, 7, 300, seed=3, precision=A.PREC_FP32)
            assert e.value.status == A.PTG_ERR_TIMEOUT
        h.set_options(tune_flags=0)
        got, _ = h.transmission(20.0, 7, 300, seed=3, precision=A.PREC_FP32)
        np.testing.assert_array_equal(got, want)
        # the FP64 kernel stages nothing: the option does not touch it
        h.set_options(tune_flags=STAGE_TEST)
        t64, _ = h.transmission(20.0, 7, 300, seed=3, precision=A.PREC_FP64)
        assert t64.sum() > 0


def test_reserved_option_and_bad_block_size_are_rejected():
    gb, spec = _film()
    with A.Handle(gb.view, spec) as h:
        for bad in ({"reserved": 1}, {"block_size": 48}):
            with pytest.raises(A.PtgError) as e:
                h.set_options(**bad)
            assert e.value.status == A.PTG_ERR_INVALID
        t, _ = h.transmission(20.0, 5, 50, seed=1, precision=A.PREC_FP32)
        assert t.shape == (1, spec.nmode, 5)


def test_injected_device_allocation_failures_return_nomem():
    """ptg_debug_fail_allocations makes the library's device-buffer requests
    fail on the host side (cudaMalloc is never called): handle creation and a
    first kappa run (whose tallies and tables are allocated then) return
    PTG_ERR_NOMEM, and after injection is off the same handle computes the
    same result as a fresh one."""
    gb, spec = _film()
    run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=200, seed=4, precision=A.PREC_FP32)
    with A.Handle(gb.view, spec) as ref:
        want = ref.kappa(run, want_counts=True)
    for after in (0, 2):
        with A.fail_allocations(after):
            with pytest.raises(A.PtgError) as e:
                A.Handle(gb.view, spec)
        assert e.value.status == A.PTG_ERR_NOMEM
    with A.Handle(gb.view, spec) as h:
        with A.fail_allocations(0):
            with pytest.raises(A.PtgError) as e:
                h.kappa(run)
            assert e.value.status == A.PTG_ERR_NOMEM
        got = h.kappa(run, want_counts=True)
    np.testing.assert_array_equal(got["counts"], want["counts"])
    assert got["kappa"] == want["kappa"]
