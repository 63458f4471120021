"""ctypes binding of include/ptrans_gpu.h (libptrans_b200.so).

This is the Python host mirror of the drop-in seam: the same entry points a
Fortran host binds with ISO_C_BINDING (p-trans_b200/fortran/ptrans_gpu.f90), with the
reference's argument meaning (``RayTrace``'s parameters, ``TransmissionFunction``
filling ``transmit(nbranch,nkpoint,nangle)``, src/RTMCphon.f90:1544-1604) and
its error behaviour (a non-zero status raises ``PtgError``).

The library must be built (``make -C p-trans_b200``); loading fails loudly
otherwise, there is no Python fallback for any transport computation.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# PTRANS_B200_LIB selects another build of the library, e.g. the
# bounds-checked libptrans_b200_check.so
LIB_PATH = os.environ.get("PTRANS_B200_LIB") or os.path.join(HERE, "libptrans_b200.so")
CHECK_LIB_PATH = os.path.join(HERE, "libptrans_b200_check.so")

# ---- constants (include/ptrans_gpu.h) --------------------------------------
PTG_OK = 0
PTG_ERR_INVALID = 1
PTG_ERR_CUDA = 2
PTG_ERR_NO_DEVICE = 3
PTG_ERR_TIMEOUT = 4
PTG_ERR_LOST = 5
PTG_ERR_NOMEM = 6
PTG_ERR_IO = 7
PTG_ERR_UNSUPPORTED = 8

SHAPE_POLYGON, SHAPE_SPHERE, SHAPE_CYLINDER, SHAPE_CAPPED = 1, 2, 3, 4
TRANS_VALUE, TRANS_GAMMA, TRANS_TBC = 1, 2, 3
MFP_MATTHIESSEN, MFP_GRID, MFP_PER_MODE = 1, 2, 3
GRAIN_VORONOI, GRAIN_BRICKS = 1, 2
FACE_REFERENCE, FACE_PERIODIC = 0, 1
PREC_FP32, PREC_FP64 = 0, 1
MATERIAL_INTERNAL, MATERIAL_BOUNDARY = 0, -1

I32P = C.POINTER(C.c_int32)
F64P = C.POINTER(C.c_double)
U64P = C.POINTER(C.c_uint64)
U32P = C.POINTER(C.c_uint32)


class PtgModel(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("cellspec", C.c_double * 6), ("face_kind", C.c_int32 * 6),
        ("specfluc", C.c_double), ("scope", C.c_double * 2), ("temperature", C.c_double),
        ("kind_grain", C.c_int32), ("nmaterial", C.c_int32), ("nt1", C.c_int32), ("nt2", C.c_int32),
        ("tt_kind", I32P), ("tt_trans", F64P), ("tt_spec", F64P), ("ngrain", C.c_int32),
        ("grain_shape", I32P), ("grain_generatrix", F64P), ("grain_diameter", F64P),
        ("grain_material", I32P), ("grain_nfacet", I32P), ("facet_nvertex", I32P),
        ("facet_vertex", F64P), ("surf_material_to", I32P), ("surf_grain_to", I32P),
        ("surf_spec", F64P), ("fluct_seed", C.c_uint64), ("grain_axis", F64P),
    ]


class PtgSpectrum(C.Structure):
    _fields_ = [
        ("nbranch", C.c_int32), ("nkpoint", C.c_int32), ("rtemp", C.c_double), ("vol", C.c_double),
        ("omega", F64P), ("tau", F64P), ("vel", F64P), ("mfp", F64P), ("weight", F64P),
    ]


class PtgGeometry(C.Structure):
    _fields_ = [
        ("box", C.c_double * 3), ("scope", C.c_double * 2), ("face_kind", C.c_int32 * 6),
        ("kind_grain", C.c_int32), ("ngrain", C.c_int32), ("igrain_fill", C.c_int32),
        ("nmaterial", C.c_int32), ("ngrain_total", C.c_int32), ("nsurf", C.c_int32),
        ("nvertex_total", C.c_int32), ("grain_begin", I32P), ("grain_incident", I32P),
        ("grain_generatrix", F64P), ("shape", I32P), ("nvertex", I32P), ("vertex_begin", I32P),
        ("vertex", F64P), ("normal", F64P), ("tangent", F64P), ("center", F64P), ("radius", F64P),
        ("kind_trans", I32P), ("specularity", F64P), ("trans_param", F64P),
        ("grain_inside", I32P), ("grain_outside", I32P), ("internal", I32P), ("incident", I32P),
        ("material1", I32P), ("material2", I32P),
    ]


class PtgOptions(C.Structure):
    _fields_ = [
        ("device", C.c_int32), ("block_size", C.c_int32), ("blocks_per_sm", C.c_int32),
        ("regen_threshold", C.c_int32), ("ref_quirks", C.c_int32), ("bvh_leaf", C.c_int32),
        ("max_flights", C.c_int64), ("lost_limit", C.c_double), ("chunk", C.c_int64),
        ("tune_flags", C.c_int32), ("fast_steps", C.c_int32), ("coop_lanes", C.c_int32),
        ("reserved", C.c_int32),
    ]


class PtgRun(C.Structure):
    _fields_ = [
        ("kind_mfp", C.c_int32), ("nangle", C.c_int32), ("np", C.c_int64), ("nmfp", C.c_int32),
        ("mfp_grid_nm", F64P), ("seed", C.c_uint64), ("stream", C.c_int32), ("rank", C.c_int32),
        ("nranks", C.c_int32), ("precision", C.c_int32), ("temperature", C.c_double),
        ("nbins", C.c_int32), ("bin_omega_min", C.c_double), ("bin_omega_max", C.c_double),
        ("scatter_scale", C.c_double),
    ]


class PtgKappaOut(C.Structure):
    _fields_ = [
        ("kappa", C.c_double), ("kappa_stderr", C.c_double), ("bin_T", F64P),
        ("bin_T_stderr", F64P), ("emfp_nm", F64P), ("transmit", F64P), ("counts", U64P),
        ("flights", C.c_uint64), ("lost", C.c_uint64), ("samples", C.c_uint64),
        ("kernel_ms", C.c_double),
    ]


class PtgStats(C.Structure):
    _fields_ = [
        ("flights", C.c_uint64), ("lost", C.c_uint64), ("samples", C.c_uint64),
        ("capped", C.c_uint64), ("kernel_ms", C.c_double), ("reduce_ms", C.c_double),
        ("launches", C.c_int32), ("grid", C.c_int32), ("block", C.c_int32),
        ("h2d_bytes", C.c_uint64), ("d2h_bytes", C.c_uint64),
        ("max_traj_flights", C.c_uint64), ("drain_ms", C.c_double), ("tail_ms", C.c_double),
        ("full_flights", C.c_uint64), ("safe_balls", C.c_uint64),
        ("coop_rounds", C.c_uint64), ("coop_flights", C.c_uint64),
        ("box_tests", C.c_uint64), ("surface_tests", C.c_uint64),
        ("drain_kernel_ms", C.c_double), ("tail_kernel_ms", C.c_double),
        ("tail_phonons", C.c_uint64), ("tail_flights", C.c_uint64),
        ("tail_refused", C.c_uint64),
    ]


class PtgAdjointOut(C.Structure):
    _fields_ = [
        ("kappa", C.c_double), ("kappa_stderr", C.c_double), ("dk_dp", F64P), ("dk_dp_stderr", F64P),
        ("dk_dscale", C.c_double), ("dk_dscale_stderr", C.c_double), ("flights", C.c_uint64),
        ("replayed", C.c_uint64), ("mismatched", C.c_uint64), ("kernel_ms", C.c_double),
    ]


class PtgBatchItem(C.Structure):
    _fields_ = [("geom", C.POINTER(PtgGeometry)), ("np", C.c_int64), ("seed", C.c_uint64),
                ("stream", C.c_int32)]


class PtgBatchOut(C.Structure):
    _fields_ = [("kappa", F64P), ("kappa_stderr", F64P), ("bin_T", F64P), ("bin_T_stderr", F64P),
                ("counts", U64P), ("flights", C.c_uint64), ("lost", C.c_uint64),
                ("samples", C.c_uint64), ("graph_ms", C.c_double)]


class PtgBatchAdjointOut(C.Structure):
    _fields_ = [("kappa", F64P), ("kappa_stderr", F64P), ("dk_dp", F64P), ("dk_dp_stderr", F64P),
                ("dk_dscale", F64P), ("dk_dscale_stderr", F64P), ("flights", C.c_uint64),
                ("replayed", C.c_uint64), ("mismatched", C.c_uint64), ("kernel_ms", C.c_double)]


class PtgError(RuntimeError):
    def __init__(self, status: int, what: str = ""):
        self.status = status
        msg = STATUS_TEXT.get(status, "unknown status")
        super().__init__(f"{what}: status {status} ({msg})" if what else f"status {status} ({msg})")


STATUS_TEXT = {
    PTG_OK: "ok", PTG_ERR_INVALID: "invalid argument or inconsistent input",
    PTG_ERR_CUDA: "CUDA runtime error", PTG_ERR_NO_DEVICE: "no usable sm_100 CUDA device",
    PTG_ERR_TIMEOUT: "a bounded device wait timed out",
    PTG_ERR_LOST: "lost-phonon fraction above the limit", PTG_ERR_NOMEM: "out of memory",
    PTG_ERR_IO: "file missing or malformed", PTG_ERR_UNSUPPORTED: "unsupported combination",
}

# every entry point of include/ptrans_gpu.h with its ctypes signature
SIGNATURES = {
    "ptg_geometry_build": (C.c_int, [C.POINTER(PtgModel), C.POINTER(PtgSpectrum), C.POINTER(C.c_void_p)]),
    "ptg_geombuf_view": (C.POINTER(PtgGeometry), [C.c_void_p]),
    "ptg_geombuf_free": (None, [C.c_void_p]),
    "ptg_mcp_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "ptg_mcpbuf_model": (C.POINTER(PtgModel), [C.c_void_p]),
    "ptg_mcpbuf_info": (C.c_int, [C.c_void_p, C.POINTER(C.c_int64), I32P, I32P, I32P, F64P, I32P,
                                  C.c_char_p, C.c_int32]),
    "ptg_mcpbuf_free": (None, [C.c_void_p]),
    "ptg_anphon_load": (C.c_int, [C.c_char_p, C.POINTER(C.c_void_p)]),
    "ptg_anphonbuf_spectrum": (C.POINTER(PtgSpectrum), [C.c_void_p]),
    "ptg_anphonbuf_free": (None, [C.c_void_p]),
    "ptg_anphon_write": (C.c_int, [C.c_char_p, C.POINTER(PtgSpectrum)]),
    "ptg_create": (C.c_int, [C.POINTER(PtgGeometry), C.POINTER(PtgSpectrum), C.POINTER(PtgOptions),
                             C.POINTER(C.c_void_p)]),
    "ptg_set_spectrum": (C.c_int, [C.c_void_p, C.POINTER(PtgSpectrum)]),
    "ptg_destroy": (None, [C.c_void_p]),
    "ptg_strerror": (C.c_char_p, [C.c_int]),
    "ptg_transmission": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.c_int64, C.c_int32,
                                   C.c_int32, C.c_uint64, C.c_int32, F64P, F64P]),
    "ptg_kappa": (C.c_int, [C.c_void_p, C.POINTER(PtgRun), C.POINTER(PtgKappaOut)]),
    "ptg_kappa_from_counts": (C.c_int, [C.POINTER(PtgGeometry), C.POINTER(PtgSpectrum),
                                        C.POINTER(PtgRun), U64P, C.POINTER(PtgKappaOut)]),
    "ptg_last_stats": (C.c_int, [C.c_void_p, C.POINTER(PtgStats)]),
    "ptg_check_report": (C.c_int, [C.c_int32, C.POINTER(C.c_int64), C.POINTER(C.c_int32),
                                   C.POINTER(C.c_int32), C.c_int32]),
    "ptg_debug_fail_allocations": (C.c_int, [C.c_int64]),
    "ptg_write_outputs": (C.c_int, [C.c_char_p, C.POINTER(PtgGeometry), C.POINTER(PtgSpectrum),
                                    C.POINTER(PtgRun), U64P]),
    "ptg_gamma_from_tbc": (C.c_int, [C.POINTER(PtgSpectrum), C.c_double, C.c_double, F64P]),
    "ptg_fortran_format": (C.c_int, [C.c_int32, C.c_double, C.c_int32, C.c_int32, C.c_char_p,
                                     C.c_int32]),
    "ptg_trace": (C.c_int, [C.c_void_p, C.POINTER(PtgRun), C.c_int64, U64P, C.c_int64, C.POINTER(C.c_float),
                            C.POINTER(C.c_int64), I32P]),
    "ptg_write_trace": (C.c_int, [C.c_void_p, C.POINTER(PtgRun), C.c_int32, C.c_char_p]),
    "ptg_get_options": (C.c_int, [C.c_void_p, C.POINTER(PtgOptions)]),
    "ptg_set_options": (C.c_int, [C.c_void_p, C.POINTER(PtgOptions)]),
    "ptg_autotune": (C.c_int, [C.c_void_p, C.POINTER(PtgRun), C.c_int32, C.POINTER(PtgOptions),
                               F64P]),
    "ptg_replay_task": (C.c_int, [C.c_void_p, C.POINTER(PtgRun), C.c_int64, I32P, U32P, F64P]),
    "ptg_adjoint": (C.c_int, [C.c_void_p, C.POINTER(PtgRun), C.POINTER(PtgAdjointOut)]),
    "ptg_batch_create": (C.c_int, [C.POINTER(PtgBatchItem), C.c_int32, C.POINTER(PtgSpectrum),
                                   C.POINTER(PtgRun), C.POINTER(PtgOptions), C.POINTER(C.c_void_p)]),
    "ptg_batch_run": (C.c_int, [C.c_void_p, C.POINTER(PtgBatchOut)]),
    "ptg_batch_adjoint": (C.c_int, [C.c_void_p, C.POINTER(PtgBatchAdjointOut)]),
    "ptg_batch_destroy": (None, [C.c_void_p]),
    "ptg_transmission_noalloc": (C.c_int, [C.c_void_p, C.c_double, C.c_int32, C.c_int64, C.c_int32,
                                           C.c_int32, C.c_uint64, F64P]),
}
NOALLOC_MAX_TASKS = 16384

_LIB = None


def load_library(path: Optional[str] = None):
    """Loads libptrans_b200.so; raises if it has not been built."""
    global _LIB
    if _LIB is not None and path is None:
        return _LIB
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(f"{p} is missing: build it with `make -C p-trans_b200` "
                           "(the transport has no Python or CPU fallback)")
    lib = C.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _LIB = lib
    return lib


def _check(st: int, what: str):
    if st != PTG_OK:
        raise PtgError(st, what)


def _ptr(a: Optional[np.ndarray], ctype):
    if a is None:
        return C.cast(None, C.POINTER(ctype))
    return a.ctypes.data_as(C.POINTER(ctype))


# ---- Python-side model and spectrum ----------------------------------------

@dataclass
class Model:
    """Raw structure description (the content of a .mcp file)."""
    box: tuple
    kind_grain: int
    grain_shape: np.ndarray
    grain_generatrix: np.ndarray
    grain_diameter: np.ndarray
    grain_material: np.ndarray
    grain_nfacet: np.ndarray
    facet_nvertex: np.ndarray
    facet_vertex: np.ndarray
    surf_material_to: np.ndarray
    surf_grain_to: np.ndarray
    cellspec: tuple = (1.0, 1.0, 1.0, 1.0, 1.0, 1.0)
    face_kind: tuple = (0, 0, 0, 0, 0, 0)
    specfluc: float = 0.0
    scope: tuple = (1.0, 1.0)
    temperature: float = 300.0
    nmaterial: int = 1
    tt_kind: np.ndarray = field(default_factory=lambda: np.array([TRANS_VALUE, TRANS_VALUE], np.int32))
    tt_trans: np.ndarray = field(default_factory=lambda: np.zeros(2))
    tt_spec: np.ndarray = field(default_factory=lambda: np.zeros(2))
    nt1: int = 1
    nt2: int = 1
    surf_spec: Optional[np.ndarray] = None
    fluct_seed: int = 0
    grain_axis: Optional[np.ndarray] = None

    def __post_init__(self):
        i32 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.int32).ravel())
        f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
        self.grain_shape = i32(self.grain_shape)
        self.grain_generatrix = f64(self.grain_generatrix)
        self.grain_diameter = f64(self.grain_diameter)
        self.grain_material = i32(self.grain_material)
        self.grain_nfacet = i32(self.grain_nfacet)
        self.facet_nvertex = i32(self.facet_nvertex) if len(self.facet_nvertex) else np.zeros(1, np.int32)
        self.facet_vertex = f64(self.facet_vertex) if len(self.facet_vertex) else np.zeros(3)
        self.surf_material_to = i32(self.surf_material_to)
        self.surf_grain_to = i32(self.surf_grain_to)
        self.tt_kind = i32(self.tt_kind)
        self.tt_trans = f64(self.tt_trans)
        self.tt_spec = f64(self.tt_spec)
        if self.surf_spec is not None:
            self.surf_spec = f64(self.surf_spec)
        if self.grain_axis is not None:
            self.grain_axis = f64(self.grain_axis)

    @property
    def ngrain(self) -> int:
        return int(self.grain_shape.size)

    def to_c(self) -> PtgModel:
        m = PtgModel()
        m.box[:] = list(self.box)
        m.cellspec[:] = list(self.cellspec)
        m.face_kind[:] = list(self.face_kind)
        m.specfluc = self.specfluc
        m.scope[:] = list(self.scope)
        m.temperature = self.temperature
        m.kind_grain = self.kind_grain
        m.nmaterial = self.nmaterial
        m.nt1, m.nt2 = self.nt1, self.nt2
        m.tt_kind = _ptr(self.tt_kind, C.c_int32)
        m.tt_trans = _ptr(self.tt_trans, C.c_double)
        m.tt_spec = _ptr(self.tt_spec, C.c_double)
        m.ngrain = self.ngrain
        m.grain_shape = _ptr(self.grain_shape, C.c_int32)
        m.grain_generatrix = _ptr(self.grain_generatrix, C.c_double)
        m.grain_diameter = _ptr(self.grain_diameter, C.c_double)
        m.grain_material = _ptr(self.grain_material, C.c_int32)
        m.grain_nfacet = _ptr(self.grain_nfacet, C.c_int32)
        m.facet_nvertex = _ptr(self.facet_nvertex, C.c_int32)
        m.facet_vertex = _ptr(self.facet_vertex, C.c_double)
        m.surf_material_to = _ptr(self.surf_material_to, C.c_int32)
        m.surf_grain_to = _ptr(self.surf_grain_to, C.c_int32)
        m.surf_spec = _ptr(self.surf_spec, C.c_double)
        m.fluct_seed = self.fluct_seed
        m.grain_axis = _ptr(self.grain_axis, C.c_double)
        m._keep = self  # arrays stay alive with the struct
        return m


@dataclass
class Spectrum:
    """Per-mode bulk data as held after loadAnphon (omega in rad/s, tau in ps)."""
    omega: np.ndarray
    tau: np.ndarray
    vel: np.ndarray
    weight: np.ndarray
    nbranch: int = 1
    rtemp: float = 300.0
    vol: float = 4.0e-29
    mfp: Optional[np.ndarray] = None

    def __post_init__(self):
        f64 = lambda a: np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
        self.omega, self.tau, self.vel, self.weight = map(f64, (self.omega, self.tau, self.vel, self.weight))
        self.mfp = f64(self.mfp) if self.mfp is not None else self.tau * self.vel * 1e-12

    @property
    def nmode(self) -> int:
        return int(self.omega.size)

    @property
    def nkpoint(self) -> int:
        return self.nmode // self.nbranch

    def to_c(self) -> PtgSpectrum:
        s = PtgSpectrum()
        s.nbranch, s.nkpoint = self.nbranch, self.nkpoint
        s.rtemp, s.vol = self.rtemp, self.vol
        s.omega = _ptr(self.omega, C.c_double)
        s.tau = _ptr(self.tau, C.c_double)
        s.vel = _ptr(self.vel, C.c_double)
        s.mfp = _ptr(self.mfp, C.c_double)
        s.weight = _ptr(self.weight, C.c_double)
        s._keep = self
        return s

    def mfp_nm(self, temperature: float) -> np.ndarray:
        """Bulk MFP in nm after the tau rescale of fileoutput (src/RTMCphon.f90:2645-2650)."""
        return self.tau * 1e-12 * (self.rtemp / temperature) * self.vel * 1e9


GEOM_FIELDS_I = ["shape", "nvertex", "vertex_begin", "kind_trans", "grain_inside", "grain_outside",
                 "internal", "incident", "material1", "material2"]
GEOM_FIELDS_F = [("normal", 3), ("tangent", 9), ("center", 3), ("radius", 1), ("specularity", 1),
                 ("trans_param", 1)]


def geometry_to_numpy(g: PtgGeometry) -> dict:
    """Copies a ptg_geometry into numpy arrays (for comparisons)."""
    ns, ngt, nvt = g.nsurf, g.ngrain_total, g.nvertex_total
    out = {
        "box": np.array(g.box[:]), "scope": np.array(g.scope[:]), "face_kind": np.array(g.face_kind[:]),
        "kind_grain": g.kind_grain, "ngrain": g.ngrain, "igrain_fill": g.igrain_fill,
        "nmaterial": g.nmaterial, "ngrain_total": ngt, "nsurf": ns, "nvertex_total": nvt,
        "grain_begin": np.ctypeslib.as_array(g.grain_begin, (ngt + 1,)).copy(),
        "grain_incident": np.ctypeslib.as_array(g.grain_incident, (ngt,)).copy(),
        "grain_generatrix": np.ctypeslib.as_array(g.grain_generatrix, (3 * ngt,)).copy(),
        "vertex": np.ctypeslib.as_array(g.vertex, (3 * nvt,)).copy() if nvt else np.zeros(0),
    }
    for f in GEOM_FIELDS_I:
        out[f] = np.ctypeslib.as_array(getattr(g, f), (ns,)).copy()
    for f, k in GEOM_FIELDS_F:
        out[f] = np.ctypeslib.as_array(getattr(g, f), (k * ns,)).copy()
    return out


def numpy_to_geometry(d: dict) -> PtgGeometry:
    """Builds a ptg_geometry over numpy arrays (kept alive by the struct)."""
    g = PtgGeometry()
    keep = {}
    g.box[:] = list(d["box"])
    g.scope[:] = list(d["scope"])
    g.face_kind[:] = [int(x) for x in d["face_kind"]]
    for k in ("kind_grain", "ngrain", "igrain_fill", "nmaterial", "ngrain_total", "nsurf", "nvertex_total"):
        setattr(g, k, int(d[k]))
    for k in ["grain_begin", "grain_incident"] + GEOM_FIELDS_I:
        a = np.ascontiguousarray(d[k], dtype=np.int32)
        keep[k] = a
        setattr(g, k, _ptr(a, C.c_int32))
    for k in ["grain_generatrix", "vertex"] + [f for f, _ in GEOM_FIELDS_F]:
        a = np.ascontiguousarray(d[k], dtype=np.float64)
        if a.size == 0:
            a = np.zeros(1)
        keep[k] = a
        setattr(g, k, _ptr(a, C.c_double))
    g._keep = keep
    return g


class GeomBuf:
    """Owning wrapper of ptg_geometry_build's result."""

    def __init__(self, model: Model, spectrum: Optional[Spectrum] = None):
        self.lib = load_library()
        self._m = model.to_c()
        self._s = spectrum.to_c() if spectrum is not None else None
        h = C.c_void_p()
        st = self.lib.ptg_geometry_build(C.byref(self._m), C.byref(self._s) if self._s else None,
                                         C.byref(h))
        _check(st, "ptg_geometry_build")
        self.h = h

    @property
    def view(self) -> PtgGeometry:
        return self.lib.ptg_geombuf_view(self.h).contents

    def numpy(self) -> dict:
        return geometry_to_numpy(self.view)

    def close(self):
        if self.h:
            self.lib.ptg_geombuf_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def make_run(kind_mfp=MFP_PER_MODE, nangle=11, np_=100, seed=0, stream=0, rank=0, nranks=1,
             precision=PREC_FP32, temperature=300.0, nbins=0, bin_omega=(0.0, 1.0),
             mfp_grid=None, scatter_scale=1.0) -> PtgRun:
    r = PtgRun()
    r.kind_mfp, r.nangle, r.np = kind_mfp, nangle, np_
    if mfp_grid is not None:
        g = np.ascontiguousarray(mfp_grid, dtype=np.float64)
        r.nmfp = g.size
        r.mfp_grid_nm = _ptr(g, C.c_double)
        r._keep = g
    else:
        r.nmfp = 0
        r.mfp_grid_nm = _ptr(None, C.c_double)
    r.seed, r.stream, r.rank, r.nranks = seed, stream, rank, nranks
    r.precision, r.temperature = precision, temperature
    r.nbins = nbins
    r.bin_omega_min, r.bin_omega_max = bin_omega
    r.scatter_scale = scatter_scale
    return r


def ntask_of(nmode: int, run: PtgRun) -> int:
    ns = run.nmfp if run.kind_mfp == MFP_GRID else 1
    return nmode * ns * (run.nangle - 1)


class Handle:
    """A device handle (ptg_create ... ptg_destroy)."""

    def __init__(self, geometry: PtgGeometry, spectrum: Spectrum, device=0, **opts):
        self.lib = load_library()
        o = PtgOptions()
        o.device = device
        for k, v in opts.items():
            setattr(o, k, v)
        self._spec = spectrum
        self._cs = spectrum.to_c()
        self._geom = geometry
        h = C.c_void_p()
        st = self.lib.ptg_create(C.byref(geometry), C.byref(self._cs), C.byref(o), C.byref(h))
        _check(st, "ptg_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.ptg_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def transmission(self, mfp_nm, nangle, np_, rank=0, nranks=1, seed=0, precision=PREC_FP32):
        nb, nk = self._spec.nbranch, self._spec.nkpoint
        t = np.zeros(nb * nk * nangle)
        e = np.zeros_like(t)
        st = self.lib.ptg_transmission(self.h, mfp_nm, nangle, np_, rank, nranks, seed, precision,
                                       _ptr(t, C.c_double), _ptr(e, C.c_double))
        _check(st, "ptg_transmission")
        return t.reshape(nangle, nk, nb).transpose(2, 1, 0), e.reshape(nangle, nk, nb).transpose(2, 1, 0)

    def transmission_noalloc(self, mfp_nm, nangle, np_, rank=0, nranks=1, seed=0):
        """ptg_transmission_noalloc: the FP32 transmission function without any
        allocation by the call (scratch in a fixed static device array)."""
        nb, nk = self._spec.nbranch, self._spec.nkpoint
        t = np.zeros(nb * nk * nangle)
        st = self.lib.ptg_transmission_noalloc(self.h, mfp_nm, nangle, np_, rank, nranks, seed,
                                               _ptr(t, C.c_double))
        _check(st, "ptg_transmission_noalloc")
        return t.reshape(nangle, nk, nb).transpose(2, 1, 0)

    def kappa(self, run: PtgRun, want_transmit=False, want_counts=False) -> dict:
        nm = self._spec.nmode
        ns = run.nmfp if run.kind_mfp == MFP_GRID else 1
        out = PtgKappaOut()
        bt = np.zeros(max(run.nbins, 1))
        be = np.zeros_like(bt)
        em = np.zeros(nm)
        tr = np.zeros(nm * ns * run.nangle) if want_transmit else None
        cn = np.zeros(ntask_of(nm, run), np.uint64) if want_counts else None
        out.bin_T, out.bin_T_stderr, out.emfp_nm = _ptr(bt, C.c_double), _ptr(be, C.c_double), _ptr(em, C.c_double)
        out.transmit = _ptr(tr, C.c_double)
        out.counts = _ptr(cn, C.c_uint64)
        st = self.lib.ptg_kappa(self.h, C.byref(run), C.byref(out))
        _check(st, "ptg_kappa")
        return {"kappa": out.kappa, "kappa_stderr": out.kappa_stderr, "bin_T": bt[: run.nbins],
                "bin_T_stderr": be[: run.nbins], "emfp_nm": em, "transmit": tr, "counts": cn,
                "flights": out.flights, "lost": out.lost, "samples": out.samples,
                "kernel_ms": out.kernel_ms}

    def adjoint(self, run: PtgRun) -> dict:
        """ptg_adjoint: kappa and its path-reweighting derivatives with respect
        to every surface record's specularity and the intrinsic-rate scale."""
        ns = self._geom.nsurf
        out = PtgAdjointOut()
        d = np.zeros(ns)
        e = np.zeros(ns)
        out.dk_dp, out.dk_dp_stderr = _ptr(d, C.c_double), _ptr(e, C.c_double)
        _check(self.lib.ptg_adjoint(self.h, C.byref(run), C.byref(out)), "ptg_adjoint")
        return {"kappa": out.kappa, "kappa_stderr": out.kappa_stderr, "dk_dp": d, "dk_dp_stderr": e,
                "dk_dscale": out.dk_dscale, "dk_dscale_stderr": out.dk_dscale_stderr,
                "flights": out.flights, "replayed": out.replayed, "mismatched": out.mismatched,
                "kernel_ms": out.kernel_ms}

    def stats(self) -> dict:
        s = PtgStats()
        _check(self.lib.ptg_last_stats(self.h, C.byref(s)), "ptg_last_stats")
        return {k: getattr(s, k) for k, _ in PtgStats._fields_}

    def trace(self, run: PtgRun, samples) -> list:
        """ptg_trace: per sample (positions [npos, 3] float32, exit side)."""
        smp = np.ascontiguousarray(samples, dtype=np.uint64)
        n = smp.size
        npos = np.zeros(n, np.int64)
        ends = np.zeros(n, np.int32)
        _check(self.lib.ptg_trace(self.h, C.byref(run), n, _ptr(smp, C.c_uint64), 0, None,
                                  _ptr(npos, C.c_int64), _ptr(ends, C.c_int32)), "ptg_trace")
        tot = int(npos.sum())
        pos = np.zeros(3 * max(tot, 1), np.float32)
        _check(self.lib.ptg_trace(self.h, C.byref(run), n, _ptr(smp, C.c_uint64), tot, _ptr(pos, C.c_float),
                                  _ptr(npos, C.c_int64), _ptr(ends, C.c_int32)), "ptg_trace")
        out, k = [], 0
        for i in range(n):
            out.append((pos[3 * k:3 * (k + npos[i])].reshape(-1, 3), int(ends[i])))
            k += int(npos[i])
        return out

    def write_trace(self, run: PtgRun, particle_trace: int, path: str) -> None:
        _check(self.lib.ptg_write_trace(self.h, C.byref(run), particle_trace, path.encode()), "ptg_write_trace")

    def options(self) -> dict:
        o = PtgOptions()
        _check(self.lib.ptg_get_options(self.h, C.byref(o)), "ptg_get_options")
        return {k: getattr(o, k) for k, _ in PtgOptions._fields_}

    def set_options(self, **kw):
        o = PtgOptions()
        _check(self.lib.ptg_get_options(self.h, C.byref(o)), "ptg_get_options")
        for k, v in kw.items():
            setattr(o, k, v)
        _check(self.lib.ptg_set_options(self.h, C.byref(o)), "ptg_set_options")

    def autotune(self, run: PtgRun, reps: int = 2, cache: Optional[str] = None, key: str = "") -> dict:
        """ptg_autotune; with `cache` (a JSON file) the options found for `key`
        are stored there and reused (applied without timing) on later calls."""
        import json
        if cache and key and os.path.exists(cache):
            data = json.load(open(cache))
            if key in data:
                self.set_options(**data[key]["options"])
                return dict(data[key], cached=True)
        o = PtgOptions()
        ms = C.c_double(0.0)
        _check(self.lib.ptg_autotune(self.h, C.byref(run), reps, C.byref(o), C.byref(ms)), "ptg_autotune")
        res = {"options": {k: getattr(o, k) for k, _ in PtgOptions._fields_}, "kernel_ms": ms.value,
               "cached": False}
        if cache and key:
            data = json.load(open(cache)) if os.path.exists(cache) else {}
            data[key] = {"options": res["options"], "kernel_ms": res["kernel_ms"]}
            with open(cache, "w") as f:
                json.dump(data, f, indent=1, sort_keys=True)
        return res

    def replay_task(self, run: PtgRun, task: int):
        npl = len(range(run.rank, run.np, run.nranks))
        es = np.zeros(npl, np.int32)
        fl = np.zeros(npl, np.uint32)
        fp = np.zeros(3 * npl)
        st = self.lib.ptg_replay_task(self.h, C.byref(run), task, _ptr(es, C.c_int32),
                                      _ptr(fl, C.c_uint32), _ptr(fp, C.c_double))
        _check(st, "ptg_replay_task")
        return es, fl, fp.reshape(npl, 3)


class Batch:
    """ptg_batch_*: many geometries in one persistent launch replayed as a CUDA graph."""

    def __init__(self, geometries, nps, seeds, streams, spectrum: Spectrum, run: PtgRun, device=0, **opts):
        self.lib = load_library()
        n = len(geometries)
        self._geoms = list(geometries)
        items = (PtgBatchItem * n)()
        for i, g in enumerate(self._geoms):
            items[i].geom = C.pointer(g)
            items[i].np, items[i].seed, items[i].stream = int(nps[i]), int(seeds[i]), int(streams[i])
        self._items = items
        self.n = n
        self.nbins = run.nbins
        self.ntask = ntask_of(spectrum.nmode, run)
        self._cs = spectrum.to_c()
        self._run = run
        o = PtgOptions()
        o.device = device
        for k, v in opts.items():
            setattr(o, k, v)
        h = C.c_void_p()
        _check(self.lib.ptg_batch_create(items, n, C.byref(self._cs), C.byref(run), C.byref(o), C.byref(h)),
               "ptg_batch_create")
        self.h = h

    def run(self, want_counts=False) -> dict:
        out = PtgBatchOut()
        k = np.zeros(self.n)
        ke = np.zeros(self.n)
        bt = np.zeros(max(1, self.n * self.nbins))
        be = np.zeros_like(bt)
        cn = np.zeros(self.n * self.ntask, np.uint64) if want_counts else None
        out.kappa, out.kappa_stderr = _ptr(k, C.c_double), _ptr(ke, C.c_double)
        out.bin_T, out.bin_T_stderr = _ptr(bt, C.c_double), _ptr(be, C.c_double)
        out.counts = _ptr(cn, C.c_uint64)
        _check(self.lib.ptg_batch_run(self.h, C.byref(out)), "ptg_batch_run")
        return {"kappa": k, "kappa_stderr": ke, "bin_T": bt[: self.n * self.nbins].reshape(self.n, self.nbins),
                "bin_T_stderr": be[: self.n * self.nbins].reshape(self.n, self.nbins),
                "counts": None if cn is None else cn.reshape(self.n, self.ntask),
                "flights": out.flights, "lost": out.lost, "samples": out.samples, "graph_ms": out.graph_ms}

    def adjoint(self) -> dict:
        """ptg_batch_adjoint: every geometry's kappa, d kappa / d p of its
        surface records (a list of arrays, one per geometry) and d kappa / d
        scale, from one batched listing pass and one batched replay."""
        ns = [int(g.nsurf) for g in self._geoms]
        tot = max(1, sum(ns))
        k, ke = np.zeros(self.n), np.zeros(self.n)
        dp, dpe = np.zeros(tot), np.zeros(tot)
        ds, dse = np.zeros(self.n), np.zeros(self.n)
        out = PtgBatchAdjointOut()
        out.kappa, out.kappa_stderr = _ptr(k, C.c_double), _ptr(ke, C.c_double)
        out.dk_dp, out.dk_dp_stderr = _ptr(dp, C.c_double), _ptr(dpe, C.c_double)
        out.dk_dscale, out.dk_dscale_stderr = _ptr(ds, C.c_double), _ptr(dse, C.c_double)
        _check(self.lib.ptg_batch_adjoint(self.h, C.byref(out)), "ptg_batch_adjoint")
        off = np.concatenate([[0], np.cumsum(ns)])
        return {"kappa": k, "kappa_stderr": ke,
                "dk_dp": [dp[off[g]:off[g + 1]] for g in range(self.n)],
                "dk_dp_stderr": [dpe[off[g]:off[g + 1]] for g in range(self.n)],
                "dk_dscale": ds, "dk_dscale_stderr": dse, "flights": out.flights,
                "replayed": out.replayed, "mismatched": out.mismatched, "kernel_ms": out.kernel_ms}

    def close(self):
        if getattr(self, "h", None):
            self.lib.ptg_batch_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class fail_allocations:
    """Context manager of ptg_debug_fail_allocations: inside it the library's
    allocations after the first `after` fail (a test hook)."""

    def __init__(self, after: int):
        self.after = after

    def __enter__(self):
        load_library().ptg_debug_fail_allocations(self.after)
        return self

    def __exit__(self, *a):
        load_library().ptg_debug_fail_allocations(-1)


def check_report(device: int = 0, reset: bool = False) -> dict:
    """ptg_check_report of a bounds-checked build (PTRANS_B200_LIB pointing at
    libptrans_b200_check.so): failed checks since the last reset."""
    lib = load_library()
    n, code, idx = C.c_int64(), C.c_int32(), C.c_int32()
    _check(lib.ptg_check_report(device, C.byref(n), C.byref(code), C.byref(idx), 1 if reset else 0),
           "ptg_check_report")
    return {"violations": n.value, "first_code": code.value, "first_index": idx.value}


def kappa_from_counts(geometry: PtgGeometry, spectrum: Spectrum, run: PtgRun, counts: np.ndarray) -> dict:
    """Host FP64 assembly after an all-reduce of the counts (multi-rank callers)."""
    lib = load_library()
    cs = spectrum.to_c()
    out = PtgKappaOut()
    bt = np.zeros(max(run.nbins, 1))
    be = np.zeros_like(bt)
    em = np.zeros(spectrum.nmode)
    out.bin_T, out.bin_T_stderr, out.emfp_nm = _ptr(bt, C.c_double), _ptr(be, C.c_double), _ptr(em, C.c_double)
    out.transmit = _ptr(None, C.c_double)
    out.counts = _ptr(None, C.c_uint64)
    c = np.ascontiguousarray(counts, dtype=np.uint64)
    st = lib.ptg_kappa_from_counts(C.byref(geometry), C.byref(cs), C.byref(run), _ptr(c, C.c_uint64),
                                   C.byref(out))
    _check(st, "ptg_kappa_from_counts")
    return {"kappa": out.kappa, "kappa_stderr": out.kappa_stderr, "bin_T": bt[: run.nbins],
            "bin_T_stderr": be[: run.nbins], "emfp_nm": em}


def write_outputs(geofile: str, geometry: PtgGeometry, spectrum: Spectrum, run: PtgRun,
                  counts: np.ndarray) -> None:
    """ptg_write_outputs: thermalproperty.out, effectiveMFP.out and
    phononconductivity.out in the directory of geofile."""
    lib = load_library()
    cs = spectrum.to_c()
    c = np.ascontiguousarray(counts, dtype=np.uint64)
    _check(lib.ptg_write_outputs(geofile.encode(), C.byref(geometry), C.byref(cs), C.byref(run),
                                 _ptr(c, C.c_uint64)), "ptg_write_outputs")


def gamma_from_tbc(material: Spectrum, temperature: float, tbc: float):
    """ptg_gamma_from_tbc: (status, gamma) for a conductance tbc [W m^-2 K^-1]."""
    lib = load_library()
    cs = material.to_c()
    g = C.c_double(0.0)
    st = lib.ptg_gamma_from_tbc(C.byref(cs), temperature, tbc, C.byref(g))
    return st, g.value


def fortran_format(kind: str, v: float, w: int, d: int = 0) -> str:
    """The writer's rendering of an I / F / E edit descriptor."""
    lib = load_library()
    buf = C.create_string_buffer(256)
    k = {"I": 0, "F": 1, "E": 2}[kind]
    _check(lib.ptg_fortran_format(k, float(v), w, d, buf, 256), "ptg_fortran_format")
    return buf.value.decode()


def mcp_load(path: str):
    """Parses a .mcp file; returns (model PtgModel copy as dict-like Model, info dict)."""
    lib = load_library()
    h = C.c_void_p()
    _check(lib.ptg_mcp_load(path.encode(), C.byref(h)), f"ptg_mcp_load({path})")
    try:
        m = lib.ptg_mcpbuf_model(h).contents
        np_ = C.c_int64()
        na, km, nm, pt = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        name = C.create_string_buffer(64)
        lib.ptg_mcpbuf_info(h, C.byref(np_), C.byref(na), C.byref(km), C.byref(nm), None, C.byref(pt), name, 64)
        grid = np.zeros(max(nm.value, 1))
        lib.ptg_mcpbuf_info(h, None, None, None, None, _ptr(grid, C.c_double), None, None, 0)
        ng = m.ngrain

        def arr(ptr, n, dtype):
            if n <= 0 or not ptr:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(ptr, (n,)).copy()

        shapes = arr(m.grain_shape, ng, np.int32)
        nfacet = arr(m.grain_nfacet, ng, np.int32)
        npoly = int(sum(nfacet[i] for i in range(ng) if shapes[i] == SHAPE_POLYGON))
        nvert = arr(m.facet_nvertex, npoly, np.int32)
        nsm = int(nfacet.sum())
        tsz = (m.nt2 + 1) * m.nt1
        model = Model(
            box=tuple(m.box), kind_grain=m.kind_grain, grain_shape=shapes,
            grain_generatrix=arr(m.grain_generatrix, 3 * ng, np.float64),
            grain_diameter=arr(m.grain_diameter, ng, np.float64),
            grain_material=arr(m.grain_material, ng, np.int32),
            grain_nfacet=nfacet, facet_nvertex=nvert,
            facet_vertex=arr(m.facet_vertex, 3 * int(nvert.sum()), np.float64),
            surf_material_to=arr(m.surf_material_to, nsm, np.int32),
            surf_grain_to=arr(m.surf_grain_to, nsm, np.int32),
            cellspec=tuple(m.cellspec), face_kind=tuple(m.face_kind), specfluc=m.specfluc,
            scope=tuple(m.scope), temperature=m.temperature, nmaterial=m.nmaterial,
            tt_kind=arr(m.tt_kind, tsz, np.int32), tt_trans=arr(m.tt_trans, tsz, np.float64),
            tt_spec=arr(m.tt_spec, tsz, np.float64), nt1=m.nt1, nt2=m.nt2)
        info = {"np": np_.value, "nangle": na.value, "kind_mfp": km.value,
                "mfp_grid": grid[: nm.value].copy(), "particle_trace": pt.value,
                "material1": name.value.decode()}
        return model, info
    finally:
        lib.ptg_mcpbuf_free(h)


def anphon_write(path: str, spectrum: Spectrum):
    lib = load_library()
    cs = spectrum.to_c()
    _check(lib.ptg_anphon_write(path.encode(), C.byref(cs)), "ptg_anphon_write")


def anphon_load(path: str) -> Spectrum:
    lib = load_library()
    h = C.c_void_p()
    _check(lib.ptg_anphon_load(path.encode(), C.byref(h)), f"ptg_anphon_load({path})")
    try:
        s = lib.ptg_anphonbuf_spectrum(h).contents
        n = s.nbranch * s.nkpoint
        a = lambda p: np.ctypeslib.as_array(p, (n,)).copy()
        return Spectrum(omega=a(s.omega), tau=a(s.tau), vel=a(s.vel), weight=a(s.weight),
                        nbranch=s.nbranch, rtemp=s.rtemp, vol=s.vol, mfp=a(s.mfp))
    finally:
        lib.ptg_anphonbuf_free(h)
