"""TEST INFRASTRUCTURE — ctypes wrapper of the CPU FP64 oracle (oracle.c).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module,
and only as the checker or the timed CPU baseline.  The product never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from src_b200.cabi import MeshMarshal, MpgDiag, MpgGcrStats, RunParams

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liboracle.so")
_lib = None


def build() -> str:
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB) or os.path.getmtime(_LIB) < os.path.getmtime(os.path.join(_HERE, "oracle.c")):
            build()
        L = C.CDLL(_LIB)
        vp, dp, ip = C.c_void_p, C.POINTER(C.c_double), C.c_int
        L.orc_create.restype = vp
        L.orc_create.argtypes = [vp, vp]
        L.orc_destroy.argtypes = [vp]
        L.orc_field.restype = dp
        L.orc_field.argtypes = [vp, ip]
        L.orc_npoin.restype = ip
        L.orc_npoin.argtypes = [vp]
        L.orc_derivative.argtypes = [vp, dp, dp, ip]
        L.orc_bcv.argtypes = [vp, dp, dp, dp, C.c_double]
        L.orc_laplc.argtypes = [vp, dp, dp, ip]
        L.orc_prfr.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, ip]
        L.orc_div.argtypes = [vp, dp, dp, dp, dp, ip, vp]
        L.orc_precon.argtypes = [vp, dp, dp, dp, ip, ip]
        L.orc_gcrk.argtypes = [vp, dp, dp, dp, dp, dp, dp, dp, ip, vp]
        L.orc_mpdatamper.argtypes = [vp, dp, ip]
        L.orc_mpdatam.argtypes = [vp, dp, ip]
        L.orc_courant.argtypes = [vp, ip, vp]
        L.orc_stats.argtypes = [vp, vp]
        L.orc_setup.argtypes = [vp, vp]
        L.orc_step.argtypes = [vp, vp]
        L.orc_velprd.argtypes = [vp]
        L.orc_get_gcr_stats.argtypes = [vp, vp]
        L.orc_beta.restype = C.c_double
        L.orc_beta.argtypes = [vp]
        L.orc_line_solve.argtypes = [vp, dp, dp, ip]
        L.orc_set_reduction.argtypes = [vp, ip]
        L.orc_set_ref_bugs.argtypes = [vp, ip]
        L.orc_wide_entries.argtypes = [vp, ip, dp, dp, dp]
        L.orc_wide_solve.argtypes = [vp, dp, dp, ip]
        L.orc_wide_factors.argtypes = [vp, ip, dp, dp, dp]
        L.orc_set_coarse.argtypes = [vp, ip, vp, C.POINTER(C.c_int)]
        L.orc_mg_restrict.argtypes = [vp, dp, dp, ip]
        L.orc_mg_prolong.argtypes = [vp, dp, dp, ip]
        L.orc_level_npoin.restype = ip
        L.orc_level_npoin.argtypes = [vp, ip]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """The reference restated on the CPU; fields addressed by the product's field ids."""

    def __init__(self, params: RunParams, refmesh, gpu_order: bool = False, ref_bugs: bool = True):
        self.params = params
        self.mm = MeshMarshal(refmesh)
        self._cp = params.to_c()
        self.L = lib()
        self.h = self.L.orc_create(C.byref(self._cp), C.byref(self.mm.c))
        if not self.h:
            raise ValueError("oracle rejected the parameters (isfera/mg_flag/nscal/lord)")
        self.n = refmesh.npoin
        if gpu_order:
            self.L.orc_set_reduction(self.h, 1)
        if not ref_bugs:
            self.L.orc_set_ref_bugs(self.h, 0)

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            self.L.orc_destroy(h)
            self.h = None

    def set_coarse(self, level: int, refmesh, match=None) -> None:
        """Attach the coarse (1) or coarsest (2) mesh of the V-cycle (mg_flag = 1), with its match
        array (coarse node -> node of the next finer mesh, 0-based) or None to match by
        coordinates as the reference does."""
        mm = MeshMarshal(refmesh)
        m = None
        if match is not None:
            keep = np.ascontiguousarray(match, np.int32)
            m = keep.ctypes.data_as(C.POINTER(C.c_int))
        if self.L.orc_set_coarse(self.h, level, C.byref(mm.c), m) != 0:
            raise ValueError("oracle rejected the coarse level")

    def mg_restrict(self, s, flg):
        out = np.zeros(self.L.orc_level_npoin(self.h, flg))
        self.L.orc_mg_restrict(self.h, _p(np.ascontiguousarray(s, np.float64)), _p(out), flg)
        return out

    def mg_prolong(self, sc, flg):
        out = np.zeros(self.L.orc_level_npoin(self.h, flg - 1))
        self.L.orc_mg_prolong(self.h, _p(np.ascontiguousarray(sc, np.float64)), _p(out), flg)
        return out

    # ---- fields
    def field(self, fid: int) -> np.ndarray:
        """A numpy view of oracle field `fid` (writes go to the oracle)."""
        ptr = self.L.orc_field(self.h, fid)
        if not ptr:
            raise KeyError(fid)
        return np.ctypeslib.as_array(ptr, shape=(self.n,))

    def set(self, fid: int, v) -> None:
        self.field(fid)[:] = v

    def get(self, fid: int) -> np.ndarray:
        return self.field(fid).copy()

    # ---- subroutines on numpy arrays
    def derivative(self, unk, idx):
        out = np.zeros(self.n)
        self.L.orc_derivative(self.h, _p(np.ascontiguousarray(unk, np.float64)), _p(out), idx)
        return out

    def laplc(self, p, impfl):
        out = np.zeros(self.n)
        self.L.orc_laplc(self.h, _p(np.ascontiguousarray(p, np.float64)), _p(out), impfl)
        return out

    def prfr(self, p, us, vs, ws, impfl):
        uo, vo, wo = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        a = [np.ascontiguousarray(x, np.float64) for x in (p, us, vs, ws)]
        self.L.orc_prfr(self.h, *[_p(x) for x in a], _p(uo), _p(vo), _p(wo), impfl)
        return uo, vo, wo

    def div(self, u, v, w, iflg):
        rhs = np.zeros(self.n)
        a = [np.ascontiguousarray(x, np.float64) for x in (u, v, w)]
        d = MpgDiag()
        self.L.orc_div(self.h, *[_p(x) for x in a], _p(rhs), iflg, C.byref(d))
        return rhs, d

    def bcv(self, u, v, w, flag):
        a = [np.array(x, np.float64) for x in (u, v, w)]
        self.L.orc_bcv(self.h, *[_p(x) for x in a], flag)
        return a

    def precon(self, rhs, iprc, impfl):
        p, r = np.zeros(self.n), np.zeros(self.n)
        self.L.orc_precon(self.h, _p(np.ascontiguousarray(rhs, np.float64)), _p(p), _p(r), iprc, impfl)
        return p

    def line_solve(self, rhs, impfl):
        z = np.zeros(self.n)
        self.L.orc_line_solve(self.h, _p(np.ascontiguousarray(rhs, np.float64)), _p(z), impfl)
        return z

    def wide_entries(self, impfl):
        lo, dg, hi = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self.L.orc_wide_entries(self.h, impfl, _p(lo), _p(dg), _p(hi))
        return lo, dg, hi

    def wide_factors(self, impfl):
        a, m, cp = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        self.L.orc_wide_factors(self.h, impfl, _p(a), _p(m), _p(cp))
        return a, m, cp

    def wide_solve(self, rhs, impfl):
        z = np.zeros(self.n)
        self.L.orc_wide_solve(self.h, _p(np.ascontiguousarray(rhs, np.float64)), _p(z), impfl)
        return z

    def gcrk(self, p, u1, v1, w1, impfl):
        p = np.array(p, np.float64)
        u2, v2, w2 = np.zeros(self.n), np.zeros(self.n), np.zeros(self.n)
        a = [np.ascontiguousarray(x, np.float64) for x in (u1, v1, w1)]
        st = MpgGcrStats()
        self.L.orc_gcrk(self.h, _p(p), *[_p(x) for x in a], _p(u2), _p(v2), _p(w2), impfl, C.byref(st))
        return p, (u2, v2, w2), st

    def mpdatamper(self, unk, iflag):
        u = np.array(unk, np.float64)
        self.L.orc_mpdatamper(self.h, _p(u), iflag)
        return u

    def mpdatam(self, unk, iflag):
        u = np.array(unk, np.float64)
        self.L.orc_mpdatam(self.h, _p(u), iflag)
        return u

    # ---- driver
    def velprd(self) -> None:
        self.L.orc_velprd(self.h)

    def setup(self) -> MpgDiag:
        d = MpgDiag()
        self.L.orc_setup(self.h, C.byref(d))
        return d

    def step(self) -> MpgDiag:
        d = MpgDiag()
        self.L.orc_step(self.h, C.byref(d))
        return d

    def courant(self, iflag=1) -> MpgDiag:
        d = MpgDiag()
        self.L.orc_courant(self.h, iflag, C.byref(d))
        return d

    def stats(self) -> MpgDiag:
        d = MpgDiag()
        self.L.orc_stats(self.h, C.byref(d))
        return d

    def gcr_stats(self) -> MpgGcrStats:
        st = MpgGcrStats()
        self.L.orc_get_gcr_stats(self.h, C.byref(st))
        return st

    def beta(self) -> float:
        return self.L.orc_beta(self.h)
