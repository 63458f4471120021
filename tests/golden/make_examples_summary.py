"""Writes tests/golden/examples_summary.json from the reference's Examples/*.mcp.

Run where a checkout of the reference is at hand:
    python tests/golden/make_examples_summary.py <P-TRANS checkout>/Examples

The figures are counted by plain text scanning, independently of the C++
reader under test: grains (the "Ng" value), model surfaces (material_to
lines), the box (L?cell * N?cell), Np, Nangle (91 when absent,
src/RTMCphon.f90:471), and the built surface counts implied by
setupBoxGrain / setupFillGrain (6 box faces + model surfaces + one fill copy
per internal brick surface) with the incident / internal rules of
src/RTMCphon.f90:1202-1246.
"""
import json
import os
import sys


def scan(path):
    lines = open(path).read().splitlines()
    toks = [l.split() for l in lines]

    def after(key):
        for i, t in enumerate(toks):
            if t and t[0] == key:
                return toks[i + 1]
        return None

    n = [int(after(k)[0]) for k in ("NXcell", "NYcell", "NZcell")]
    L = [float(after(k)[0]) for k in ("LXcell", "LYcell", "LZcell")]
    box = [L[i] * n[i] for i in range(3)]
    ng = int(after("Ng")[0])
    shape = after("Shape")[0]
    na = after("Nangle")
    nangle = int(na[0]) if na else 91
    np_ = int(after("Np")[0])
    nsurf = sum(1 for t in toks if t and t[0] == "material_to")
    # polygons: collect vertex lists per facet in order
    facets = []
    i = 0
    while i < len(toks):
        t = toks[i]
        if t and t[0] == "Nv":
            nv = int(toks[i + 1][0])
            vs = []
            for k in range(nv):
                vs.append([float(x) for x in toks[i + 3 + 2 * k][:3]])
            facets.append(vs)
            i += 2 + 2 * nv
            continue
        i += 1
    quadric = nsurf - len(facets)
    internal_model = quadric
    for vs in facets:
        out = False
        for d in range(3):
            if all(v[d] <= 0.0 for v in vs) or all(v[d] >= box[d] for v in vs):
                out = True
        internal_model += 0 if out else 1
    built = 6 + nsurf + (internal_model if shape == "bricks" else 0)
    built_internal = 6 + internal_model + (internal_model if shape == "bricks" else 0)
    return {"ngrain": ng, "nsurf": nsurf, "box": box, "np": np_, "nangle": nangle,
            "built_nsurf": built, "built_internal": built_internal}


def main(d):
    out = {}
    for name in sorted(os.listdir(d)):
        if name.endswith(".mcp"):
            out[name] = scan(os.path.join(d, name))
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "examples_summary.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(json.dumps(out, indent=1))


if __name__ == "__main__":
    if len(sys.argv) < 2:
        sys.exit("usage: make_examples_summary.py <P-TRANS checkout>/Examples")
    main(sys.argv[1])
