"""Seeded synthetic inputs: phonon spectra and structures.

The reference reads a bulk mode table (Materials/<name>.anphon) and a .mcp
structure written by its GUI; neither ships with it.  These generators make
inputs of the same form from a seed:
  - ``spectrum``: N modes, one branch, weight 1; f ~ U(0, fmax) THz,
    v ~ LogNormal(median 4 km/s, sigma 0.5), bulk MFP ~ LogUniform(1 nm, 10 um),
    tau = MFP / v; the heat capacity follows from omega and T in the kappa sum
    (src/RTMCphon.f90:2693-2704).  RTemp equals T so the tau rescale of
    fileoutput (:2647) is the identity.
  - ``nanowire``: one Voronoi grain whose six facets lie on the box
    (Examples/01_square_nanowire.mcp layout), side walls by CellSpecularity.
  - ``film_with_holes``: bricks with through-thickness z-cylinders
    (Examples/02_thinfilm_3holes.mcp layout), holes as voids (T = 0).
  - ``write_mcp``: the .mcp text layout the reference's loaders read.
Random draws use numpy's PCG64 seeded with the given seed.
"""
from __future__ import annotations

import math
from typing import Optional

import numpy as np

from .abi import (FACE_PERIODIC, GRAIN_BRICKS, GRAIN_VORONOI, MATERIAL_BOUNDARY, MATERIAL_INTERNAL, SHAPE_CAPPED,
                  SHAPE_CYLINDER, SHAPE_POLYGON, SHAPE_SPHERE, TRANS_VALUE, Model, Spectrum)

THZ = 2.0 * math.pi * 1.0e12


def spectrum(n_modes: int, seed: int = 0, temperature: float = 300.0, fmax_thz: float = 15.0,
             v_median: float = 4000.0, v_sigma: float = 0.5, mfp_lo: float = 1e-9,
             mfp_hi: float = 1e-5, vol: float = 4.0e-29) -> Spectrum:
    rng = np.random.default_rng(seed)
    f = rng.uniform(0.0, fmax_thz, n_modes)
    v = np.exp(rng.normal(math.log(v_median), v_sigma, n_modes))
    mfp = np.exp(rng.uniform(math.log(mfp_lo), math.log(mfp_hi), n_modes))
    tau_ps = mfp / v * 1e12
    return Spectrum(omega=f * THZ, tau=tau_ps, vel=v, weight=np.ones(n_modes), nbranch=1,
                    rtemp=temperature, vol=vol, mfp=mfp)


def _box_faces(x0, x1, y0, y1, z0, z1):
    """Six quads of an axis-aligned box, counter-clockwise seen from outside."""
    return [
        [(x0, y0, z0), (x0, y0, z1), (x0, y1, z1), (x0, y1, z0)],  # x-
        [(x1, y0, z0), (x1, y1, z0), (x1, y1, z1), (x1, y0, z1)],  # x+
        [(x0, y0, z0), (x1, y0, z0), (x1, y0, z1), (x0, y0, z1)],  # y-
        [(x1, y1, z0), (x0, y1, z0), (x0, y1, z1), (x1, y1, z1)],  # y+
        [(x0, y0, z0), (x0, y1, z0), (x1, y1, z0), (x1, y0, z0)],  # z-
        [(x0, y1, z1), (x0, y0, z1), (x1, y0, z1), (x1, y1, z1)],  # z+
    ]


def _table(trans: float, spec: float, kind: int = TRANS_VALUE):
    # param%X(nt2+1, nt1) with nt1 = nt2 = 1: entry (1,1) then the boundary row
    return (np.array([kind, TRANS_VALUE], np.int32), np.array([trans, 0.0]), np.array([spec, 0.0]))


def nanowire(length: float = 1000.0, width: float = 100.0, height: float = 100.0,
             p_side: float = 0.0, trans: float = 0.5, spec: float = 0.0) -> Model:
    """Square nanowire: one Voronoi grain on the box, side walls with specularity p_side."""
    faces = _box_faces(0, length, 0, width, 0, height)
    kind, tt, ts = _table(trans, spec)
    return Model(
        box=(length, width, height), kind_grain=GRAIN_VORONOI,
        grain_shape=[SHAPE_POLYGON], grain_generatrix=[0.5 * length, 0.5 * width, 0.5 * height],
        grain_diameter=[0.0], grain_material=[1], grain_nfacet=[6],
        facet_nvertex=[4] * 6, facet_vertex=np.array(faces, dtype=np.float64).ravel(),
        surf_material_to=[MATERIAL_BOUNDARY] * 6, surf_grain_to=[0] * 6,
        cellspec=(1.0, 1.0, p_side, p_side, p_side, p_side), tt_kind=kind, tt_trans=tt, tt_spec=ts)


def hole_centres(n: int, lx: float, ly: float, r: float, seed: int, gap: float = 2.0,
                 margin: float = 2.0) -> np.ndarray:
    """n non-overlapping disc centres of radius r inside [0,lx] x [0,ly],
    at least r + margin from every edge (rejection sampling)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(200000):
        if len(out) == n:
            break
        c = rng.uniform([r + margin, r + margin], [lx - r - margin, ly - r - margin])
        if all(np.hypot(*(c - o)) >= 2 * r + gap for o in out):
            out.append(c)
    if len(out) != n:
        raise ValueError("could not place the holes")
    return np.array(out)


def film_with_holes(lx: float = 300.0, ly: float = 300.0, lz: float = 145.0, nholes: int = 3,
                    radius: float = 50.0, seed: int = 0, periodic_y: bool = True,
                    p_hole: float = 0.0, t_hole: float = 0.0, p_z: float = 0.0,
                    centres: Optional[np.ndarray] = None) -> Model:
    """Thin film (x transport, z thickness) pierced by z-cylinders.

    The holes are brick grains whose wall transmits with t_hole (0: voids) and
    reflects with specularity p_hole; z walls have specularity p_z; y walls
    are periodic (extension) or specular mirrors (the reference's option)."""
    if centres is None:
        centres = hole_centres(nholes, lx, ly, radius, seed)
    n = len(centres)
    gen = np.column_stack([centres, np.full(n, 0.5 * lz)])
    kind, tt, ts = _table(t_hole, p_hole)
    return Model(
        box=(lx, ly, lz), kind_grain=GRAIN_BRICKS, grain_shape=[SHAPE_CYLINDER] * n,
        grain_generatrix=gen.ravel(), grain_diameter=[2 * radius] * n, grain_material=[1] * n,
        grain_nfacet=[1] * n, facet_nvertex=[], facet_vertex=[],
        surf_material_to=[MATERIAL_INTERNAL] * n, surf_grain_to=[0] * n,
        cellspec=(1.0, 1.0, 1.0, 1.0, p_z, p_z),
        face_kind=(0, 0, FACE_PERIODIC, FACE_PERIODIC, 0, 0) if periodic_y else (0,) * 6,
        tt_kind=kind, tt_trans=tt, tt_spec=ts)


def spheres_in_box(l: float = 200.0, centres=((100.0, 100.0, 100.0),), radii=(40.0,),
                   p: float = 0.0, t: float = 0.0, p_wall: float = 0.0) -> Model:
    """Bricks of spheres in a box (for sphere intersection checks)."""
    n = len(radii)
    kind, tt, ts = _table(t, p)
    return Model(
        box=(l, l, l), kind_grain=GRAIN_BRICKS, grain_shape=[SHAPE_SPHERE] * n,
        grain_generatrix=np.array(centres, np.float64).ravel(), grain_diameter=[2 * r for r in radii],
        grain_material=[1] * n, grain_nfacet=[1] * n, facet_nvertex=[], facet_vertex=[],
        surf_material_to=[MATERIAL_INTERNAL] * n, surf_grain_to=[0] * n,
        cellspec=(1.0, 1.0, p_wall, p_wall, p_wall, p_wall), tt_kind=kind, tt_trans=tt, tt_spec=ts)


def brick_box(l: float = 200.0, lo=(60.0, 60.0, 60.0), hi=(140.0, 140.0, 140.0), p: float = 0.0,
              t: float = 0.5, p_wall: float = 0.0, triangles: bool = False) -> Model:
    """One polygon brick (a box, as quads or as 12 triangles) in a box."""
    faces = _box_faces(lo[0], hi[0], lo[1], hi[1], lo[2], hi[2])
    if triangles:
        tri = []
        for f in faces:
            tri.append([f[0], f[1], f[2]])
            tri.append([f[0], f[2], f[3]])
        faces = tri
    nv = [len(f) for f in faces]
    kind, tt, ts = _table(t, p)
    gen = [(lo[d] + hi[d]) * 0.5 for d in range(3)]
    return Model(
        box=(l, l, l), kind_grain=GRAIN_BRICKS, grain_shape=[SHAPE_POLYGON], grain_generatrix=gen,
        grain_diameter=[0.0], grain_material=[1], grain_nfacet=[len(faces)], facet_nvertex=nv,
        facet_vertex=np.array([v for f in faces for v in f], np.float64).ravel(),
        surf_material_to=[MATERIAL_INTERNAL] * len(faces), surf_grain_to=[0] * len(faces),
        cellspec=(1.0, 1.0, p_wall, p_wall, p_wall, p_wall), tt_kind=kind, tt_trans=tt, tt_spec=ts)


def with_interface(model: Model, kind: int, param: float, spec: float = 0.0,
                   two_materials: bool = False) -> Model:
    """The model with every internal interface of the given transmission kind
    (the Nt table, src/RTMCphon.f90:749-890, 1402-1429): TRANS_VALUE with
    param = T, or TRANS_GAMMA / TRANS_TBC with param = gamma (a TBC entry is
    solved to gamma on the host first: abi.gamma_from_tbc).  With one material
    the kernels draw against T(omega) = 1/(gamma omega/omega_max + 1); with two
    (the inclusions of material 2 in a matrix of material 1) the threshold is
    random, t11 + u (1 - t11), t11 = 1/(gamma + 1) (src/RTMCphon.f90:2391-2402)."""
    import dataclasses
    if not two_materials:
        kind_t, tt, ts = _table(param, spec, kind)
        return dataclasses.replace(model, tt_kind=kind_t, tt_trans=tt, tt_spec=ts, nmaterial=1, nt1=1, nt2=1)
    # param%X(nt2+1, nt1), nt1 = nt2 = 2: rows 1..2 are materials, row 3 the boundary
    kind_t = np.full(6, kind, np.int32)
    tt = np.full(6, float(param))
    ts = np.full(6, float(spec))
    for i1 in (1, 2):
        k = 2 + 3 * (i1 - 1)
        kind_t[k], tt[k], ts[k] = TRANS_VALUE, 0.0, 0.0
    return dataclasses.replace(model, tt_kind=kind_t, tt_trans=tt, tt_spec=ts, nmaterial=2, nt1=2, nt2=2,
                               grain_material=np.full(model.ngrain, 2, np.int32))


def write_mcp(model: Model, path: str, np_: int = 100, nangle: int = 11,
              mean_free_path: Optional[str] = None, material: str = "Si", trace: int = 1000):
    """Writes the model as a .mcp file in the reference's layout."""
    w = []
    a = w.append
    a("# sample")
    for k, v in (("NXcell", 1), ("NYcell", 1), ("NZcell", 1)):
        a(k)
        a(f"\t{v}")
    for k, v in zip(("LXcell", "LYcell", "LZcell"), model.box):
        a(k)
        a(f"\t{v:.9e} # nm")
    a("")
    a("## Raytracing")
    a("CellSpecularity")
    a("\t" + " ".join(f"{x:.6f}" for x in model.cellspec))
    a("FluctuationSpecularity")
    a(f"\t{model.specfluc:.6f}")
    a("temp # Temperature")
    a(f"\t{model.temperature:.6f}")
    a("Np # number of incident phonons")
    a(f"\t{np_}")
    a("Nangle # number of incident angles")
    a(f"\t{nangle}")
    a("ScopeY # Y region of phonon emission")
    a(f"\t{model.scope[0]:.6f}")
    a("ScopeZ #")
    a(f"\t{model.scope[1]:.6f}")
    if mean_free_path is not None:
        a("MeanFreePath # list of mean free path")
        a(f"\t{mean_free_path}")
    a("Trace # number of phonon for output trace")
    a(f"\t{trace}")
    a("")
    a("# materials")
    a("Nm # number of materials")
    a("\t1")
    a("material contents")
    a(f"\t{material}")
    a("\t\t100.000000")
    a("")
    a("# truns functions")
    a("Nt")
    a("\t1 1")
    a("materials")
    names = {1: "Value", 2: "Gamma", 3: "TBC"}
    a(f"\t{material} {material} mode {names[int(model.tt_kind[0])]} Specular")
    a(f"\t\t{model.tt_trans[0]:.6f} {model.tt_spec[0]:.6f}")
    a("")
    a("# grains")
    a("Shape # shape of grains")
    a("\tvoronoi" if model.kind_grain == GRAIN_VORONOI else "\tbricks")
    a("Ng Ngx Ngy Ngz # number of grains")
    a(f"\t{model.ngrain} {model.ngrain} 1 1")
    fpos = vpos = spos = 0
    for g in range(model.ngrain):
        a(f"## grain No.{g + 1}")
        a("  generator")
        gx, gy, gz = model.grain_generatrix[3 * g:3 * g + 3]
        a(f"\t{gx:+.9f} {gy:+.9f} {gz:+.9f}")
        sh = int(model.grain_shape[g])
        d = float(model.grain_diameter[g])
        if model.kind_grain == GRAIN_VORONOI:
            a("  length")
            a("\t+25.000000 +25.000000 +25.000000")
        elif sh == SHAPE_SPHERE:
            a("  sphere")
            a(f"\t{d:+.9f} {d:+.9f} {d:+.9f}")
        elif sh == SHAPE_CYLINDER:
            a("  cylinder")
            a(f"\t{d:+.9f} {d:+.9f} {model.box[2]:+.9f}")
        else:
            a("  box")
            a("\t+0.000000 +0.000000 +0.000000")
        a("  material")
        a(f"\t{material}")
        nsurf = int(model.grain_nfacet[g]) if (sh == SHAPE_POLYGON or model.kind_grain == GRAIN_VORONOI) else 1
        if sh == SHAPE_POLYGON or model.kind_grain == GRAIN_VORONOI:
            a(f"# facets of grain No.{g + 1}")
            a("  Nf # number of facets")
            a(f"\t{nsurf}")
        for s in range(nsurf):
            if sh == SHAPE_POLYGON or model.kind_grain == GRAIN_VORONOI:
                nv = int(model.facet_nvertex[fpos])
                fpos += 1
                a(f"#  facet No.{s + 1}")
                a("  Nv # number of vertex")
                a(f"\t\t{nv}")
                for k in range(nv):
                    x, y, z = model.facet_vertex[3 * (vpos + k):3 * (vpos + k) + 3]
                    a(f"\tvertex {k + 1}")
                    a(f"\t\t{x:+.9f} {y:+.9f} {z:+.9f}")
                vpos += nv
            mto = int(model.surf_material_to[spos])
            mname = "Internal" if mto == MATERIAL_INTERNAL else ("Boundary" if mto < 0 else material)
            a(f"  material_to = {mname}")
            a(f"  grain_to = {int(model.surf_grain_to[spos])}")
            spos += 1
    with open(path, "w") as f:
        f.write("\n".join(w) + "\n")


def film_batch(n: int = 256, seed: int = 0, n_modes: int = 2000, nangle: int = 11,
               samples_lo: float = 1e5, samples_hi: float = 1e7):
    """Screening set: n periodic films, one through-thickness hole per cell.

    hole radius ~ U(10, 60) nm, period ~ U(100, 400) nm (cell x = y = period,
    radius kept below period/2 - 5 nm), thickness ~ U(50, 300) nm, samples per
    film log-uniform in [samples_lo, samples_hi] (rounded to particles per
    (mode, angle) task).  Returns (models, particles per task)."""
    rng = np.random.default_rng(seed)
    models, nps = [], []
    for _ in range(n):
        period = rng.uniform(100.0, 400.0)
        radius = min(rng.uniform(10.0, 60.0), period / 2 - 5.0)
        thick = rng.uniform(50.0, 300.0)
        m = film_with_holes(lx=period, ly=period, lz=thick, nholes=1, radius=radius,
                            centres=np.array([[period / 2, period / 2]]), periodic_y=True)
        samples = math.exp(rng.uniform(math.log(samples_lo), math.log(samples_hi)))
        nps.append(max(1, int(round(samples / (n_modes * (nangle - 1))))))
        models.append(m)
    return models, nps


def _clip_cell(faces, labels, nrm, c, label, tol):
    """Clips a convex polyhedron (outward vertex loops `faces` with `labels`)
    to the half-space nrm . x <= c; the cut face gets `label`."""
    out_f, out_l, cut = [], [], []
    for f, lab in zip(faces, labels):
        d = [float(np.dot(nrm, v)) - c for v in f]
        if max(d) <= tol:
            out_f.append(f)
            out_l.append(lab)
            continue
        if min(d) >= -tol:
            for v, dv in zip(f, d):
                if abs(dv) <= tol:
                    cut.append(v)
            continue
        loop = []
        n = len(f)
        for i in range(n):
            a, b = f[i], f[(i + 1) % n]
            da, db = d[i], d[(i + 1) % n]
            if da <= tol:
                loop.append(a)
                if abs(da) <= tol:
                    cut.append(a)
            if (da < -tol and db > tol) or (da > tol and db < -tol):
                p = a + (b - a) * (da / (da - db))
                loop.append(p)
                cut.append(p)
        if len(loop) >= 3:
            out_f.append(loop)
            out_l.append(lab)
    # cap polygon: the cut points, counter-clockwise seen along +nrm
    pts = []
    for p in cut:
        if not any(np.linalg.norm(p - q) <= 10 * tol for q in pts):
            pts.append(p)
    if len(pts) >= 3:
        ctr = np.mean(pts, axis=0)
        u = pts[0] - ctr
        u = u / np.linalg.norm(u)
        w = np.cross(nrm, u)
        ang = [math.atan2(float(np.dot(p - ctr, w)), float(np.dot(p - ctr, u))) for p in pts]
        out_f.append([pts[i] for i in np.argsort(ang)])
        out_l.append(label)
    return out_f, out_l


def _triangulate(poly, levels):
    """A convex polygon (vertex loop) as triangles: a fan about the vertex
    mean, each fan triangle split `levels` times into four by its edge
    midpoints, every triangle keeping the polygon's orientation.  The two
    cells sharing a facet hold its vertex loop in opposite orders, and both
    get the same triangles (reversed)."""
    c = np.mean(poly, axis=0)
    tris = [(c, poly[i], poly[(i + 1) % len(poly)]) for i in range(len(poly))]
    for _ in range(levels):
        nxt = []
        for a, b, d in tris:
            ab, bd, da = 0.5 * (a + b), 0.5 * (b + d), 0.5 * (d + a)
            nxt += [(a, ab, da), (ab, b, bd), (da, bd, d), (ab, bd, da)]
        tris = nxt
    return [list(t) for t in tris]


def voronoi_box(n_grains: int = 5, box=(1000.0, 1000.0, 1000.0), seed: int = 0, trans: float = 0.5,
                spec: float = 0.0, p_wall: float = 0.0, generators=None, tri_levels: int = -1) -> Model:
    """Voronoi polycrystal in the box: seeded generators (uniform in the inner
    90% of the box), every cell the box clipped by the bisector planes of the
    other generators.  Facets on the box are Boundary facets (grain_to 0, the
    box's CellSpecularity applies), facets between cells carry material 1 and
    the neighbour's grain id, with the (1,1) transmission-table entry
    (T = trans, p = spec) as in Examples/04_voronoi_5grain.mcp.  With
    tri_levels >= 0 every facet is given as a triangle mesh instead (a fan
    refined tri_levels times, 4^levels triangles per fan triangle), as a
    grain exported from a mesher or an STL file would be."""
    L = np.asarray(box, np.float64)
    rng = np.random.default_rng(seed)
    gens = (np.asarray(generators, np.float64) if generators is not None
            else L * (0.05 + 0.9 * rng.random((n_grains, 3))))
    n = len(gens)
    tol = 1e-9 * float(L.max())
    faces0 = [[np.array(v, np.float64) for v in f] for f in _box_faces(0, L[0], 0, L[1], 0, L[2])]
    nfacet, nv, verts, mto, gto = [], [], [], [], []
    for i in range(n):
        faces, labels = list(faces0), [-1] * 6
        for j in range(n):
            if j == i:
                continue
            nrm = gens[j] - gens[i]
            nrm = nrm / np.linalg.norm(nrm)
            c = float(np.dot(nrm, 0.5 * (gens[i] + gens[j])))
            faces, labels = _clip_cell(faces, labels, nrm, c, j, tol)
        kept = 0
        for f, lab in zip(faces, labels):
            fv = []
            for v in f:
                v = v.copy()
                for d in range(3):  # exact box coordinates on box facets
                    if abs(v[d]) <= tol:
                        v[d] = 0.0
                    elif abs(v[d] - L[d]) <= tol:
                        v[d] = L[d]
                fv.append(v)
            pieces = [fv] if tri_levels < 0 else _triangulate(fv, tri_levels)
            for pc in pieces:
                nv.append(len(pc))
                verts.extend(pc)
                mto.append(MATERIAL_BOUNDARY if lab < 0 else 1)
                gto.append(0 if lab < 0 else lab + 1)
                kept += 1
        nfacet.append(kept)
    kind, tt, ts = _table(trans, spec)
    return Model(
        box=tuple(float(x) for x in L), kind_grain=GRAIN_VORONOI, grain_shape=[SHAPE_POLYGON] * n,
        grain_generatrix=gens.ravel(), grain_diameter=[0.0] * n, grain_material=[1] * n,
        grain_nfacet=nfacet, facet_nvertex=nv, facet_vertex=np.array(verts, np.float64).ravel(),
        surf_material_to=mto, surf_grain_to=gto,
        cellspec=(1.0, 1.0, p_wall, p_wall, p_wall, p_wall), tt_kind=kind, tt_trans=tt, tt_spec=ts)


def cube_lattice(n: int = 16, l: float = 1000.0, fill: float = 0.5, trans: float = 0.0,
                 spec: float = 0.0, p_wall: float = 0.0, triangles: bool = True) -> Model:
    """Simple-cubic lattice of n^3 cubic inclusions (bricks) in an l^3 box:
    pitch l/n, cube side fill * pitch, every cube face as two triangles
    (12 per cube: n = 16 gives 49152 triangles) or as one quad.  The matrix
    (fill grain) sees every inclusion facet, the case a BVH is for."""
    pitch = l / n
    a = 0.5 * fill * pitch
    faces_all, nf, gens = [], [], []
    for ix in range(n):
        for iy in range(n):
            for iz in range(n):
                cx, cy, cz = (ix + 0.5) * pitch, (iy + 0.5) * pitch, (iz + 0.5) * pitch
                faces = _box_faces(cx - a, cx + a, cy - a, cy + a, cz - a, cz + a)
                if triangles:
                    tri = []
                    for f in faces:
                        tri.append([f[0], f[1], f[2]])
                        tri.append([f[0], f[2], f[3]])
                    faces = tri
                faces_all.extend(faces)
                nf.append(len(faces))
                gens.append((cx, cy, cz))
    ng = len(nf)
    kind, tt, ts = _table(trans, spec)
    return Model(
        box=(l, l, l), kind_grain=GRAIN_BRICKS, grain_shape=[SHAPE_POLYGON] * ng,
        grain_generatrix=np.array(gens).ravel(), grain_diameter=[0.0] * ng, grain_material=[1] * ng,
        grain_nfacet=nf, facet_nvertex=[len(f) for f in faces_all],
        facet_vertex=np.array([v for f in faces_all for v in f], np.float64).ravel(),
        surf_material_to=[MATERIAL_INTERNAL] * len(faces_all), surf_grain_to=[0] * len(faces_all),
        cellspec=(1.0, 1.0, p_wall, p_wall, p_wall, p_wall), tt_kind=kind, tt_trans=tt, tt_spec=ts)


def spheres_cylinders_box(n_spheres: int = 64, n_cylinders: int = 16, l: float = 1000.0, seed: int = 0,
                          r_sphere=(20.0, 80.0), r_cylinder: float = 30.0, length=(100.0, 400.0),
                          trans: float = 0.0, p_wall: float = 0.0, per_surface_p: bool = True,
                          gap: float = 2.0) -> Model:
    """Spheres (radius ~ U(r_sphere)) and capped cylinders of random axis
    (radius r_cylinder, length ~ U(length)) in an l^3 box, placed by
    rejection so that no two objects' bounding spheres come closer than gap
    and every object stays inside the box.  Inclusions transmit with
    `trans`; with per_surface_p every surface gets its own specularity
    p ~ U(0, 1) (the model's per-surface override), else p = 0."""
    rng = np.random.default_rng(seed)
    placed = []   # (centre, bounding radius)
    shapes, gens, diam, axes = [], [], [], []

    def fits(c, rb, ext):
        if np.any(c - ext <= gap) or np.any(c + ext >= l - gap):
            return False
        return all(np.linalg.norm(c - q) > rb + rq + gap for q, rq in placed)

    for _ in range(n_cylinders):
        for _attempt in range(100000):
            u = rng.normal(size=3)
            a = u / np.linalg.norm(u)
            ln = rng.uniform(*length)
            c = rng.uniform(0.0, l, 3)
            ext = 0.5 * ln * np.abs(a) + r_cylinder * np.sqrt(np.maximum(0.0, 1.0 - a * a))
            rb = math.hypot(r_cylinder, 0.5 * ln)
            if fits(c, rb, ext):
                placed.append((c, rb))
                shapes.append(SHAPE_CAPPED)
                gens.append(c)
                diam.append(2.0 * r_cylinder)
                axes.append(a * ln)
                break
        else:
            raise RuntimeError("could not place a cylinder")
    for _ in range(n_spheres):
        for _attempt in range(100000):
            r = rng.uniform(*r_sphere)
            c = rng.uniform(0.0, l, 3)
            if fits(c, r, np.full(3, r)):
                placed.append((c, r))
                shapes.append(SHAPE_SPHERE)
                gens.append(c)
                diam.append(2.0 * r)
                axes.append(np.zeros(3))
                break
        else:
            raise RuntimeError("could not place a sphere")
    n = len(shapes)
    kind, tt, ts = _table(trans, 0.0)
    spec = rng.uniform(0.0, 1.0, n) if per_surface_p else None
    return Model(
        box=(l, l, l), kind_grain=GRAIN_BRICKS, grain_shape=shapes, grain_generatrix=np.array(gens).ravel(),
        grain_diameter=diam, grain_material=[1] * n, grain_nfacet=[1] * n, facet_nvertex=[], facet_vertex=[],
        surf_material_to=[MATERIAL_INTERNAL] * n, surf_grain_to=[0] * n,
        cellspec=(1.0, 1.0, p_wall, p_wall, p_wall, p_wall), tt_kind=kind, tt_trans=tt, tt_spec=ts,
        surf_spec=spec, grain_axis=np.array(axes).ravel())
