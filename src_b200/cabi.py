"""ctypes mirrors of the C ABI structs in include/mpgcr.h and helpers to marshal meshes.

The structs follow the three configuration layers of the reference: ``inputinc.d``
(lippsLFroude_implgwopks3D_unstr3.f:2293-2321), ``input_mg_v3.d`` (ref.f:2265-2276) and the
constants hard-coded in ``mpsolver`` (ref.f:108-138).
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os

import numpy as np

from .mesh import RefMesh


class MpgParams(C.Structure):
    _fields_ = [
        ("ntime", C.c_int32), ("istst", C.c_int32), ("isfera", C.c_int32), ("iper", C.c_int32),
        ("cfl", C.c_double), ("delt", C.c_double),
        ("p0inf", C.c_double), ("u0inf", C.c_double), ("v0inf", C.c_double), ("w0inf", C.c_double),
        ("ielast", C.c_int32), ("eps0", C.c_double), ("itr", C.c_int32), ("lord", C.c_int32),
        ("irl", C.c_int32),
        ("dxabl", C.c_double), ("dxabr", C.c_double), ("dyabd", C.c_double),
        ("dyabu", C.c_double), ("dzabd", C.c_double), ("dzabu", C.c_double),
        ("towxl", C.c_double), ("towxr", C.c_double), ("towyd", C.c_double),
        ("towyu", C.c_double), ("towzd", C.c_double), ("towzu", C.c_double),
        ("mg_flag", C.c_int32), ("sm_flag1", C.c_int32), ("omega", C.c_double),
        ("itrp1", C.c_int32), ("itrp2", C.c_int32),
        ("implgw", C.c_int32), ("lipps", C.c_int32),
        ("strat", C.c_double), ("tetbar", C.c_double), ("g", C.c_double),
        ("iprc", C.c_int32), ("nscal", C.c_int32), ("precision", C.c_int32), ("itmn", C.c_int32),
        ("nn_rate", C.c_double), ("itraj", C.c_int32),
        ("itrp_c1", C.c_int32), ("itrp_c2", C.c_int32), ("itrp_cc", C.c_int32), ("mg_bugs", C.c_int32),
    ]


class MpgMeshRef(C.Structure):
    _fields_ = [
        ("npoin", C.c_int32), ("nedge", C.c_int32), ("nbface", C.c_int32), ("nboun", C.c_int32),
        ("npoinx", C.c_int32), ("nedgex", C.c_int32), ("nfacesx", C.c_int32),
        ("coord", C.POINTER(C.c_double)), ("vol", C.POINTER(C.c_double)),
        ("iedge", C.POINTER(C.c_int32)), ("sn", C.POINTER(C.c_double)),
        ("kbface", C.POINTER(C.c_int32)), ("sb", C.POINTER(C.c_double)),
        ("ibpoin", C.POINTER(C.c_int32)), ("sbb", C.POINTER(C.c_double)),
        ("anp", C.POINTER(C.c_double)),
        ("ncoin", C.c_int32), ("ncoin2", C.c_int32), ("ncoin4", C.c_int32), ("ldcoin", C.c_int32),
        ("icoin", C.POINTER(C.c_int32)), ("icoin2", C.POINTER(C.c_int32)),
        ("icoin4", C.POINTER(C.c_int32)),
    ]


class MpgGcrStats(C.Structure):
    _fields_ = [
        ("niter", C.c_int32), ("nitsm", C.c_int32), ("icount", C.c_int32), ("status", C.c_int32),
        ("eer", C.c_double), ("eem", C.c_double), ("dvmx", C.c_double), ("rl2", C.c_double),
        ("fallbacks", C.c_int32), ("pad", C.c_int32), ("rate", C.c_double),
    ]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "pad"}


class MpgDiag(C.Structure):
    _fields_ = [
        ("divmx", C.c_double), ("divmn", C.c_double), ("divav", C.c_double), ("divsd", C.c_double),
        ("crnmx", C.c_double), ("crnmn", C.c_double), ("crnav", C.c_double), ("crnsd", C.c_double),
        ("icrnmx", C.c_int32), ("niter", C.c_int32), ("nitav", C.c_int32), ("niter1", C.c_int32),
        ("eer", C.c_double), ("eem", C.c_double),
        ("stats", C.c_double * 16), ("mass", C.c_double * 8),
        ("smin", C.c_double * 4), ("smax", C.c_double * 4),
        ("rate1", C.c_double), ("fallbacks", C.c_int32), ("pad", C.c_int32),
    ]

    def as_dict(self):
        d = {}
        for k, _ in self._fields_:
            if k == "pad":
                continue
            v = getattr(self, k)
            d[k] = list(v) if not isinstance(v, (int, float)) else v
        return d


class MpgKtime(C.Structure):
    _fields_ = [("name", C.c_char * 24), ("launches", C.c_int64), ("total_ms", C.c_double)]


class MpgInfo(C.Structure):
    _fields_ = [
        ("npoin", C.c_int64), ("nedge", C.c_int64), ("ncol", C.c_int64), ("nedge2d", C.c_int64),
        ("nlev", C.c_int32), ("precision", C.c_int32), ("device_bytes", C.c_int64),
    ]


# field ids (include/mpgcr.h)
F_UNK, F_UNK1, F_UUU, F_UUU0, F_FRC, F_UNKDASH = 0, 16, 20, 23, 26, 30
F_PRPOT, F_RHS, F_COUR, F_ALPHA, F_COEFW, F_RH0, F_TH0, F_THE, F_DTHEDZ, F_D1 = range(33, 43)
F_UUU1 = 43
F_WORK = 48
F_COUNT = 56

GCR_STATUS = {0: "converged", 1: "stalled", 2: "maxit", 3: "nan", 4: "fallback"}


@dataclasses.dataclass
class RunParams:
    """Run parameters, named as in the reference input files and mpsolver constants."""

    ntime: int = 100
    istst: int = 2
    isfera: int = 0
    iper: int = 2
    cfl: float = 0.5
    delt: float = 10.0
    p0inf: float = 0.0
    u0inf: float = 10.0
    v0inf: float = 0.0
    w0inf: float = 0.0
    ielast: int = 0
    eps0: float = 1e-8
    itr: int = 100
    lord: int = 3
    irl: int = 1
    dxabl: float = 0.0
    dxabr: float = 0.0
    dyabd: float = 0.0
    dyabu: float = 0.0
    dzabd: float = 0.0
    dzabu: float = 5000.0
    towxl: float = 0.0
    towxr: float = 0.0
    towyd: float = 0.0
    towyu: float = 0.0
    towzd: float = 0.0
    towzu: float = 300.0
    mg_flag: int = 0
    sm_flag1: int = 1
    omega: float = 1.0
    itrp1: int = 1
    itrp2: int = 0
    implgw: int = 1
    lipps: int = 1
    strat: float = 0.01 ** 2 / 9.80616
    tetbar: float = 300.0
    g: float = 9.80616
    iprc: int = 2
    nscal: int = 0
    precision: int = 0
    itmn: int = 3
    nn_rate: float = 0.0
    itraj: int = 0
    itrp_c1: int = 1
    itrp_c2: int = 1
    itrp_cc: int = 2
    mg_bugs: int = 1

    def to_c(self) -> MpgParams:
        p = MpgParams()
        for k, _ in MpgParams._fields_:
            setattr(p, k, getattr(self, k))
        return p

    def write_input_files(self, directory: str) -> None:
        """Write inputinc.d, input_mg_v3.d and inputre.d in the layout `input` reads."""
        with open(os.path.join(directory, "inputinc.d"), "w") as f:
            f.write("ntime nrkstage istst mrestart isfera iper\n")
            f.write(f"{self.ntime} 2 {self.istst} 0 {self.isfera} {self.iper}\n")
            f.write("cfl delt adapt relax\n")
            f.write(f"{self.cfl} {self.delt} 0. 0.\n")
            f.write("p0inf u0inf v0inf w0inf Re\n")
            f.write(f"{self.p0inf} {self.u0inf} {self.v0inf} {self.w0inf} 0.\n")
            f.write("elliptic solver\n")
            f.write("ielast eps0 itr lord\n")
            f.write(f"{self.ielast} {self.eps0:.6e} {self.itr} {self.lord}\n")
            f.write("itrp betap\n")
            f.write("1 0.\n")
            f.write("irl\n")
            f.write(f"{self.irl}\n")
            if self.irl == 1:
                f.write("dxabl dxabr dyabd dyabu dzabd dzabu\n")
                f.write(f"{self.dxabl} {self.dxabr} {self.dyabd} {self.dyabu} {self.dzabd} {self.dzabu}\n")
                f.write("towxl towxr towyd towyu towzd towzu\n")
                f.write(f"{self.towxl} {self.towxr} {self.towyd} {self.towyu} {self.towzd} {self.towzu}\n")
        with open(os.path.join(directory, "input_mg_v3.d"), "w") as f:
            f.write("mg_flag\n")
            f.write(f"{self.mg_flag}\n")
            f.write("smoothing\n")
            f.write("sm_flag1 sm_flag2\n")
            f.write(f"{self.sm_flag1} 0\n")
            f.write("omega\n")
            f.write(f"{self.omega}\n")
            f.write("sweeps\n")
            f.write("itrp1 itrp2 itrp_c1 itrp_c2 itrp_cc\n")
            f.write(f"{self.itrp1} {self.itrp2} {self.itrp_c1} {self.itrp_c2} {self.itrp_cc}\n")
            f.write("match_flag\n")
            f.write("1\n")
        with open(os.path.join(directory, "inputre.d"), "w") as f:
            f.write("nrstart\n0\nntimet\n0\nirestart nre\n0 0\n")


class MeshMarshal:
    """Holds Fortran-layout (column-major, 1-based) copies of a RefMesh and the C struct."""

    def __init__(self, rm: RefMesh):
        self.rm = rm
        n, ne, nb, nbo = rm.npoin, rm.nedge, rm.nbface, rm.nboun
        nf = max(nb, nbo, 1)
        self.coord = np.ascontiguousarray(rm.coord.T)              # (3, npoin)
        self.vol = np.ascontiguousarray(rm.vol)
        self.iedge = np.ascontiguousarray((rm.iedge.astype(np.int32) + 1).T)
        self.sn = np.ascontiguousarray(rm.sn.T)
        self.kbface = np.zeros((2, nf), np.int32)
        self.kbface[:, :nb] = (rm.kbface.astype(np.int32) + 1).T
        self.sb = np.zeros((3, nf))
        self.sb[:, :nb] = rm.sb.T
        self.ibpoin = np.zeros((2, nf), np.int32)
        self.ibpoin[0, :nbo] = rm.ibpoin[:, 0] + 1
        self.ibpoin[1, :nbo] = rm.ibpoin[:, 1]
        self.sbb = np.zeros((3, nf))
        self.sbb[:, :nbo] = rm.sbb.T
        self.anp = np.zeros((3, nf))
        self.anp[:, :nbo] = rm.anp.T
        nc, nc2, nc4 = rm.icoin.shape[0], rm.icoin2.shape[0], rm.icoin4.shape[0]
        ldc = max(2 * nf, nc, 1)
        self.icoin = np.zeros((2, ldc), np.int32)
        self.icoin[:, :nc] = (rm.icoin + 1).T
        nf2 = max(nf, nc2, nc4)
        self.icoin2 = np.zeros((2, nf2), np.int32)
        self.icoin2[:, :nc2] = (rm.icoin2 + 1).T
        self.icoin4 = np.zeros((4, nf2), np.int32)
        self.icoin4[:, :nc4] = (rm.icoin4 + 1).T
        if nf2 != nf:
            raise ValueError("periodic lists longer than the boundary arrays are not supported")
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int32)
        m = MpgMeshRef()
        m.npoin, m.nedge, m.nbface, m.nboun = n, ne, nb, nbo
        m.npoinx, m.nedgex, m.nfacesx = n, ne, nf
        m.coord = self.coord.ctypes.data_as(dp)
        m.vol = self.vol.ctypes.data_as(dp)
        m.iedge = self.iedge.ctypes.data_as(ip)
        m.sn = self.sn.ctypes.data_as(dp)
        m.kbface = self.kbface.ctypes.data_as(ip)
        m.sb = self.sb.ctypes.data_as(dp)
        m.ibpoin = self.ibpoin.ctypes.data_as(ip)
        m.sbb = self.sbb.ctypes.data_as(dp)
        m.anp = self.anp.ctypes.data_as(dp)
        m.ncoin, m.ncoin2, m.ncoin4, m.ldcoin = nc, nc2, nc4, ldc
        m.icoin = self.icoin.ctypes.data_as(ip)
        m.icoin2 = self.icoin2.ctypes.data_as(ip)
        m.icoin4 = self.icoin4.ctypes.data_as(ip)
        self.c = m
