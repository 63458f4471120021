"""The bounds-checked build (libptrans_b200_check.so, FP32 kernels compiled
with -DPT_CHECK): every geometry-blob index the kernels read and every live
phonon's state are checked, failures are counted without trapping.  The same
transports (film, two-material Gamma spheres, a triangulated Voronoi
polycrystal with BVHs, capped cylinders, a cube lattice; forward, tail phase
and adjoint replay) run with the regular and with the checked build, each in
a process of its own: no check fails, and the checked build computes the same
counts and flights as the regular one."""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _run(lib=None):
    env = dict(os.environ)
    env.pop("PTRANS_B200_LIB", None)
    if lib:
        env["PTRANS_B200_LIB"] = lib
    p = subprocess.run([sys.executable, os.path.join(HERE, "checked_run.py")], capture_output=True, text=True,
                       env=env, timeout=900)
    assert p.returncode == 0, p.stderr[-3000:]
    return json.loads(p.stdout.strip().splitlines()[-1])


def test_checked_build_finds_no_violation_and_matches_the_regular_build():
    from ptrans_b200 import abi as A
    assert os.path.exists(A.CHECK_LIB_PATH)
    regular = _run()
    checked = _run(A.CHECK_LIB_PATH)
    assert regular.pop("check") == {"status": A.PTG_ERR_UNSUPPORTED}
    rep = checked.pop("check")
    assert rep["violations"] == 0, rep
    for name in regular:
        assert checked[name]["counts"] == regular[name]["counts"], name
        assert checked[name]["flights"] == regular[name]["flights"], name
        assert checked[name]["mismatched"] == 0 and regular[name]["mismatched"] == 0
