"""Writes tests/golden/examples_models.json: the structures of the reference's
Examples/*.mcp as parsed by ptg_mcp_load, as plain numbers (the ptg_model
arrays and the run parameters Np, Nangle, MFP mode and grid, material name).

The GPU test tests/test_gpu_examples.py runs these structures end to end on
machines without the reference.  Run where a checkout of the reference is at
hand, after building the library:
    python tests/golden/make_examples_models.py <P-TRANS checkout>/Examples

The parse itself is pinned by tests/test_host.py::test_reference_examples_parse
(counts from an independent text scan, tests/golden/examples_summary.json).
"""
import glob
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


def main(examples):
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import conftest  # noqa: F401  (loads the package as ptrans_b200)
    from ptrans_b200 import abi as A
    out = {}
    for path in sorted(glob.glob(os.path.join(examples, "*.mcp"))):
        m, info = A.mcp_load(path)
        rec = {k: (v.tolist() if hasattr(v, "tolist") else (list(v) if isinstance(v, tuple) else v))
               for k, v in vars(m).items() if v is not None}
        rec["info"] = {k: (v.tolist() if hasattr(v, "tolist") else v) for k, v in info.items()}
        out[os.path.basename(path)] = rec
    dst = os.path.join(HERE, "examples_models.json")
    with open(dst, "w") as f:
        json.dump(out, f, indent=0, sort_keys=True)
    print(f"wrote {dst}: {len(out)} structures")


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_examples_models.py <P-TRANS checkout>/Examples")
    main(sys.argv[1])
