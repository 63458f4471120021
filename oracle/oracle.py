"""TEST INFRASTRUCTURE: ctypes binding of the CPU FP64 oracle
(oracle/_build/libptrans_oracle.so, a restatement of src/RTMCphon.f90).

Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline use it, as the
checker; the product never calls it.  PARITY UNPINNED: see ptrans_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "libptrans_oracle.so")

_LIB = None


class OrcResult(C.Structure):
    _fields_ = [("flights", C.c_uint64), ("lost", C.c_uint64), ("capped", C.c_uint64),
                ("samples", C.c_uint64), ("seconds", C.c_double), ("threads", C.c_int32)]


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(LIB_PATH):
        build()
    from ptrans_b200 import abi as A  # struct layouts of the C ABI
    L = C.CDLL(LIB_PATH)
    vp = C.c_void_p
    I32P, F64P, U64P, U32P = A.I32P, A.F64P, A.U64P, A.U32P
    L.orc_build_model.argtypes = [C.POINTER(A.PtgModel), C.POINTER(A.PtgSpectrum), C.POINTER(vp)]
    L.orc_from_geometry.argtypes = [C.POINTER(A.PtgGeometry), C.POINTER(A.PtgSpectrum), C.POINTER(vp)]
    L.orc_free.argtypes = [vp]
    L.orc_free.restype = None
    L.orc_geometry_sizes.argtypes = [vp, I32P, I32P, I32P]
    L.orc_geometry_export.argtypes = [vp] + [I32P, I32P, F64P, I32P, I32P, I32P, F64P, F64P, F64P,
                                             F64P, F64P, I32P, F64P, F64P, I32P, I32P, I32P, I32P,
                                             I32P, I32P]
    L.orc_ntask.argtypes = [vp, C.POINTER(A.PtgRun)]
    L.orc_ntask.restype = C.c_int64
    L.orc_run_counts.argtypes = [vp, C.POINTER(A.PtgRun), C.c_int64, C.c_int32, C.c_int32,
                                 C.POINTER(C.c_int64), C.c_int64, U64P, U64P, C.POINTER(OrcResult)]
    L.orc_replay_task.argtypes = [vp, C.POINTER(A.PtgRun), C.c_int64, C.c_int64, I32P, U32P, F64P]
    L.orc_kappa_from_counts.argtypes = [vp, C.POINTER(A.PtgRun), U64P, C.POINTER(A.PtgKappaOut)]
    L.orc_write_outputs.argtypes = [vp, C.c_char_p, C.POINTER(A.PtgRun), U64P]
    L.orc_gamma_from_tbc.argtypes = [vp, C.c_double, C.c_double, C.POINTER(C.c_double)]
    L.orc_philox.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
    L.orc_philox.restype = None
    L.orc_log.argtypes = [C.c_double]
    L.orc_log.restype = C.c_double
    L.orc_sincos2pi.argtypes = [C.c_double, F64P, F64P]
    L.orc_sincos2pi.restype = None
    _LIB = L
    return L


def _p(a, t):
    if a is None:
        return C.cast(None, C.POINTER(t))
    return a.ctypes.data_as(C.POINTER(t))


class Oracle:
    """An oracle instance over a raw model (its own geometry builder) or over a
    caller-built ptg_geometry."""

    def __init__(self, model=None, spectrum=None, geometry=None):
        self.L = lib()
        self._s = spectrum.to_c() if spectrum is not None else None
        self.spectrum = spectrum
        h = C.c_void_p()
        if geometry is not None:
            st = self.L.orc_from_geometry(C.byref(geometry), C.byref(self._s) if self._s else None, C.byref(h))
        else:
            self._m = model.to_c()
            st = self.L.orc_build_model(C.byref(self._m), C.byref(self._s) if self._s else None, C.byref(h))
        if st != 0:
            raise RuntimeError(f"oracle build failed: status {st}")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.L.orc_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def geometry(self) -> dict:
        ngt, ns, nvt = C.c_int32(), C.c_int32(), C.c_int32()
        self.L.orc_geometry_sizes(self.h, C.byref(ngt), C.byref(ns), C.byref(nvt))
        ngt, ns, nvt = ngt.value, ns.value, nvt.value
        d = {"grain_begin": np.zeros(ngt + 1, np.int32), "grain_incident": np.zeros(ngt, np.int32),
             "grain_generatrix": np.zeros(3 * ngt), "vertex": np.zeros(max(3 * nvt, 1))}
        from ptrans_b200.abi import GEOM_FIELDS_F, GEOM_FIELDS_I
        for f in GEOM_FIELDS_I:
            d[f] = np.zeros(ns, np.int32)
        for f, k in GEOM_FIELDS_F:
            d[f] = np.zeros(k * ns)
        i, f = C.c_int32, C.c_double
        self.L.orc_geometry_export(
            self.h, _p(d["grain_begin"], i), _p(d["grain_incident"], i), _p(d["grain_generatrix"], f),
            _p(d["shape"], i), _p(d["nvertex"], i), _p(d["vertex_begin"], i), _p(d["vertex"], f),
            _p(d["normal"], f), _p(d["tangent"], f), _p(d["center"], f), _p(d["radius"], f),
            _p(d["kind_trans"], i), _p(d["specularity"], f), _p(d["trans_param"], f),
            _p(d["grain_inside"], i), _p(d["grain_outside"], i), _p(d["internal"], i),
            _p(d["incident"], i), _p(d["material1"], i), _p(d["material2"], i))
        d["vertex"] = d["vertex"][: 3 * nvt]
        d["ngrain_total"], d["nsurf"], d["nvertex_total"] = ngt, ns, nvt
        return d

    def ntask(self, run) -> int:
        return int(self.L.orc_ntask(self.h, C.byref(run)))

    def counts(self, run, max_flights=0, ref_quirks=0, threads=0, subset=None):
        nt = self.ntask(run)
        cnt = np.zeros(nt, np.uint64)
        lost = np.zeros(nt, np.uint64)
        res = OrcResult()
        sub = None if subset is None else np.ascontiguousarray(subset, dtype=np.int64)
        st = self.L.orc_run_counts(self.h, C.byref(run), max_flights, ref_quirks, threads,
                                   _p(sub, C.c_int64), 0 if sub is None else sub.size,
                                   _p(cnt, C.c_uint64), _p(lost, C.c_uint64), C.byref(res))
        if st != 0:
            raise RuntimeError(f"oracle run failed: status {st}")
        return cnt, lost, {k: getattr(res, k) for k, _ in OrcResult._fields_}

    def replay(self, run, task, max_flights=0):
        n = len(range(run.rank, run.np, run.nranks))
        es = np.zeros(n, np.int32)
        fl = np.zeros(n, np.uint32)
        fp = np.zeros(3 * n)
        st = self.L.orc_replay_task(self.h, C.byref(run), task, max_flights, _p(es, C.c_int32),
                                    _p(fl, C.c_uint32), _p(fp, C.c_double))
        if st != 0:
            raise RuntimeError(f"oracle replay failed: status {st}")
        return es, fl, fp.reshape(n, 3)

    def gamma_from_tbc(self, temperature, tbc):
        """GammaDeterm: (status, gamma)."""
        g = C.c_double(0.0)
        st = self.L.orc_gamma_from_tbc(self.h, temperature, tbc, C.byref(g))
        return st, g.value

    def write_outputs(self, geofile, run, counts):
        """fileoutput's three files next to geofile."""
        c = np.ascontiguousarray(counts, dtype=np.uint64)
        st = self.L.orc_write_outputs(self.h, geofile.encode(), C.byref(run), _p(c, C.c_uint64))
        if st != 0:
            raise RuntimeError(f"orc_write_outputs: status {st}")

    def kappa(self, run, counts):
        from ptrans_b200 import abi as A
        out = A.PtgKappaOut()
        nm = self.spectrum.nmode
        ns = run.nmfp if run.kind_mfp == A.MFP_GRID else 1
        bt = np.zeros(max(run.nbins, 1))
        be = np.zeros_like(bt)
        em = np.zeros(nm)
        tr = np.zeros(nm * ns * run.nangle)
        out.bin_T, out.bin_T_stderr = _p(bt, C.c_double), _p(be, C.c_double)
        out.emfp_nm, out.transmit = _p(em, C.c_double), _p(tr, C.c_double)
        out.counts = _p(None, C.c_uint64)
        c = np.ascontiguousarray(counts, dtype=np.uint64)
        st = self.L.orc_kappa_from_counts(self.h, C.byref(run), _p(c, C.c_uint64), C.byref(out))
        if st != 0:
            raise RuntimeError(f"oracle kappa failed: status {st}")
        return {"kappa": out.kappa, "kappa_stderr": out.kappa_stderr, "bin_T": bt[: run.nbins],
                "bin_T_stderr": be[: run.nbins], "emfp_nm": em, "transmit": tr}


def philox(ctr, key):
    L = lib()
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    L.orc_philox(c, k, o)
    return list(o)


def olog(x: float) -> float:
    return lib().orc_log(x)


def osincos2pi(u: float):
    s, c = C.c_double(), C.c_double()
    lib().orc_sincos2pi(u, C.byref(s), C.byref(c))
    return s.value, c.value
