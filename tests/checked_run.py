"""Runs representative transports with whatever library PTRANS_B200_LIB names
and prints one JSON line: per case the transmitted counts' checksum, the
flights, and (for a bounds-checked build) ptg_check_report.  Used by
tests/test_gpu_checked.py, once with the regular and once with the checked
build, in processes of their own."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import conftest  # noqa: E402,F401  (loads the package as ptrans_b200)
from ptrans_b200 import abi as A  # noqa: E402
from ptrans_b200 import synth  # noqa: E402


def cases():
    return {
        "film": synth.film_with_holes(seed=2),
        "spheres_gamma": synth.with_interface(
            synth.spheres_in_box(l=200.0, centres=((70, 90, 100), (140, 110, 90)), radii=(35, 40), t=0.5, p=0.3,
                                 p_wall=0.2), A.TRANS_GAMMA, 0.8, spec=0.3, two_materials=True),
        "voronoi_mesh": synth.voronoi_box(5, box=(300.0, 250.0, 250.0), seed=5, trans=0.5, tri_levels=2),
        "capped": synth.spheres_cylinders_box(n_spheres=4, n_cylinders=5, l=300.0, seed=3, r_sphere=(15.0, 35.0),
                                              r_cylinder=20.0, length=(50.0, 150.0), trans=0.3, p_wall=0.2),
        "lattice": synth.cube_lattice(n=4, l=300.0, fill=0.5, trans=0.3, spec=0.2, p_wall=0.3),
    }


def main():
    out = {}
    spec = synth.spectrum(8, seed=1, mfp_lo=2e-9, mfp_hi=2e-6)
    for name, m in cases().items():
        gb = A.GeomBuf(m)
        with A.Handle(gb.view, spec) as h:
            run = A.make_run(kind_mfp=A.MFP_PER_MODE, nangle=7, np_=400, seed=5, precision=A.PREC_FP32)
            k = h.kappa(run, want_counts=True)
            st = h.stats()
            a = h.adjoint(run)
        out[name] = {"counts": int(np.sum(k["counts"] * np.arange(1, k["counts"].size + 1, dtype=np.uint64))),
                     "flights": int(st["flights"]), "tail_phonons": int(st["tail_phonons"]),
                     "replayed": int(a["replayed"]), "mismatched": int(a["mismatched"])}
    try:
        out["check"] = A.check_report()
    except A.PtgError as e:
        out["check"] = {"status": e.status}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
