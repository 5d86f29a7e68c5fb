"""Python host side of the C ABI (include/mpgcr.h): one `Solver` per GPU-resident run.

Method names and argument meaning follow the reference subroutines of
lippsLFroude_implgwopks3D_unstr3.f: ``gcrk`` (ref.f:1776), ``prfr`` (ref.f:1536),
``laplc`` (ref.f:1288), ``div`` (ref.f:2096), ``derivative`` (ref.f:3943), ``precon``
(ref.f:482), ``bcv`` (ref.f:1583), ``mpdatamper`` (ref.f:3617), ``mpdatam`` (ref.f:3029), ``courant`` (ref.f:1974),
``stats`` (ref.f:2847), and the driver ``mpsolver`` split into ``setup`` (ref.f:99-273) and
``step`` (one DO ITIME pass, ref.f:285-463).  Arrays passed in or out are in the reference
node order.  The CUDA library must be built (``__graft_entry__.build()``); there is no CPU
fallback — a missing library raises.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import cabi
from .cabi import MeshMarshal, MpgDiag, MpgGcrStats, MpgInfo, RunParams

_HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(_HERE, "libmpgcr.so")
_lib = None

EXPORTS = [
    "mpg_create", "mpg_destroy", "mpg_last_error", "mpg_get_info", "mpg_set_field", "mpg_get_field",
    "mpg_derivative", "mpg_bcv", "mpg_laplc", "mpg_prfr", "mpg_div", "mpg_precon", "mpg_gcrk",
    "mpg_mpdatamper", "mpg_mpdatam", "mpg_courant", "mpg_stats", "mpg_setup", "mpg_step", "mpg_half_forcing",
    "mpg_explicit_forcing", "mpg_post_solve", "mpg_extrapolate", "mpg_get_gcr_stats",
    "mpg_synchronize", "mpg_analyze_mesh", "mpg_analyze_wide", "mpg_get_stream", "mpg_kernel_timing", "mpg_kernel_times",
    "mpg_laplc_noalloc", "mpg_learned_init", "mpg_learned_set_params", "mpg_learned_get_params",
    "mpg_learned_forward", "mpg_learned_grad", "mpg_learned_train_pair", "mpg_learned_harvest",
    "mpg_learned_train_records", "mpg_learned_loss", "mpg_laplc_adjoint", "mpg_restart_write",
    "mpg_restart_read", "mpg_velprd", "mpg_selftest_wait", "mpg_write_output", "mpg_set_coarse",
]
NPARAM = 9505


class MpgError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"mpgcr error {code}: {msg}")
        self.code = code


def lib():
    """Load libmpgcr.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIBPATH):
            raise RuntimeError(f"CUDA library {LIBPATH} not built; run __graft_entry__.build()")
        L = C.CDLL(LIBPATH)
        vp, ip, dp = C.c_void_p, C.c_int, C.c_double
        L.mpg_last_error.restype = C.c_char_p
        L.mpg_create.argtypes = [vp, vp, ip, C.POINTER(vp)]
        L.mpg_destroy.argtypes = [vp]
        L.mpg_get_info.argtypes = [vp, vp]
        L.mpg_set_field.argtypes = [vp, ip, vp]
        L.mpg_get_field.argtypes = [vp, ip, vp]
        L.mpg_derivative.argtypes = [vp, ip, ip, ip]
        L.mpg_bcv.argtypes = [vp, ip, ip, ip, dp]
        L.mpg_laplc.argtypes = [vp, ip, ip, ip]
        L.mpg_laplc_adjoint.argtypes = [vp, ip, ip, ip]
        L.mpg_prfr.argtypes = [vp] + [ip] * 8
        L.mpg_div.argtypes = [vp, ip, ip, ip, ip, ip, vp]
        L.mpg_precon.argtypes = [vp, ip, ip, ip, ip, ip]
        L.mpg_gcrk.argtypes = [vp] + [ip] * 8 + [vp]
        L.mpg_mpdatamper.argtypes = [vp, ip, ip]
        L.mpg_mpdatam.argtypes = [vp, ip, ip]
        L.mpg_courant.argtypes = [vp, ip, vp]
        L.mpg_stats.argtypes = [vp, vp]
        L.mpg_setup.argtypes = [vp, vp]
        L.mpg_step.argtypes = [vp, vp]
        for nm in ("mpg_half_forcing", "mpg_extrapolate", "mpg_synchronize"):
            getattr(L, nm).argtypes = [vp]
        for nm in ("mpg_explicit_forcing", "mpg_post_solve"):
            getattr(L, nm).argtypes = [vp, ip]
        L.mpg_get_gcr_stats.argtypes = [vp, vp]
        L.mpg_analyze_mesh.argtypes = [vp, vp]
        L.mpg_analyze_wide.argtypes = [vp, vp, ip, vp, vp, vp]
        L.mpg_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.mpg_kernel_timing.argtypes = [vp, ip]
        L.mpg_kernel_times.argtypes = [vp, vp, ip, C.POINTER(C.c_int)]
        L.mpg_laplc_noalloc.argtypes = [vp, vp, vp, ip]
        fp = C.POINTER(C.c_float)
        L.mpg_learned_init.argtypes = [vp, ip]
        L.mpg_learned_set_params.argtypes = [vp, fp, ip]
        L.mpg_learned_get_params.argtypes = [vp, fp, ip]
        L.mpg_learned_forward.argtypes = [vp, ip, ip]
        L.mpg_learned_grad.argtypes = [vp, ip, ip, fp, C.POINTER(C.c_double)]
        L.mpg_learned_train_pair.argtypes = [vp, ip, ip, C.c_float, C.POINTER(C.c_double)]
        L.mpg_learned_harvest.argtypes = [vp, ip, ip]
        L.mpg_learned_train_records.argtypes = [vp, ip, C.c_float, C.POINTER(C.c_double), C.POINTER(C.c_int)]
        L.mpg_learned_loss.argtypes = [vp, ip]
        L.mpg_restart_write.argtypes = [vp, C.c_char_p, ip, ip]
        L.mpg_velprd.argtypes = [vp]
        L.mpg_set_coarse.argtypes = [vp, ip, vp, vp]
        L.mpg_write_output.argtypes = [vp, C.c_char_p, vp, ip]
        L.mpg_selftest_wait.argtypes = [vp, ip, ip, C.POINTER(C.c_int)]
        L.mpg_restart_read.argtypes = [vp, C.c_char_p, ip, C.POINTER(C.c_int)]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise MpgError(rc, lib().mpg_last_error().decode())


def reference_restart_name(ntime: int) -> str:
    """File name Restart_Out_old gives step `ntime`: 'Rstart_Out' // i9 // '.d' (ref.f:4794-4796)."""
    return "Rstart_Out%9d.d" % ntime


def analyze_mesh(refmesh) -> dict:
    """Prism-column analysis of a mesh on the host (no GPU needed)."""
    mm = MeshMarshal(refmesh)
    i = MpgInfo()
    _check(lib().mpg_analyze_mesh(C.byref(mm.c), C.byref(i)))
    d = {k: getattr(i, k) for k, _ in MpgInfo._fields_}
    d["bitwise_order"] = bool(d.pop("precision"))
    d.pop("device_bytes")
    return d


def analyze_wide(params: RunParams, refmesh, impfl: int):
    """Host-side factorisation of laplc's column blocks used by iprc = 4, per reference node:
    (a = A[k][k-2], inverse pivot, c') on the node's parity chain (no GPU needed)."""
    mm = MeshMarshal(refmesh)
    cp = params.to_c()
    n = refmesh.npoin
    a, m, c = np.zeros(n), np.zeros(n), np.zeros(n)
    dp = C.POINTER(C.c_double)
    _check(lib().mpg_analyze_wide(C.byref(cp), C.byref(mm.c), impfl, a.ctypes.data_as(dp),
                                  m.ctypes.data_as(dp), c.ctypes.data_as(dp)))
    return a, m, c


class Solver:
    """A run on one GPU: mesh uploaded once, fields resident, reference subroutines as methods."""

    def __init__(self, params: RunParams, refmesh, device: int = 0):
        self.params = params
        self.n = refmesh.npoin
        self._mm = MeshMarshal(refmesh)
        self._cp = params.to_c()
        self.L = lib()
        h = C.c_void_p()
        _check(self.L.mpg_create(C.byref(self._cp), C.byref(self._mm.c), device, C.byref(h)))
        self.h = h
        self._mm = None          # the library keeps its own copy

    def close(self):
        if getattr(self, "h", None):
            self.L.mpg_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_coarse(self, level: int, refmesh, match=None) -> None:
        """mg_flag = 1: attach the coarse (1) or coarsest (2) mesh of precon's V-cycle, with its
        match array (0-based: coarse node -> node of the next finer mesh) or None to match by
        coordinates as the reference does."""
        mm = MeshMarshal(refmesh)
        m = None
        if match is not None:
            m = np.ascontiguousarray(np.asarray(match) + 1, np.int32)
        _check(self.L.mpg_set_coarse(self.h, level, C.byref(mm.c), m.ctypes.data if m is not None else None))

    # ---------------------------------------------------------------- fields
    def set(self, fid: int, values) -> None:
        a = np.ascontiguousarray(np.broadcast_to(np.asarray(values, np.float64), (self.n,)))
        _check(self.L.mpg_set_field(self.h, fid, a.ctypes.data))

    def get(self, fid: int, out: np.ndarray = None) -> np.ndarray:
        """Field `fid` in reference node order, into `out` when given (a C-contiguous float64
        array of npoin values; pass pinned host memory for a full-bandwidth copy)."""
        if out is None:
            out = np.empty(self.n)
        elif out.dtype != np.float64 or out.shape != (self.n,) or not out.flags["C_CONTIGUOUS"]:
            raise ValueError("out must be a C-contiguous float64 array of npoin values")
        _check(self.L.mpg_get_field(self.h, fid, out.ctypes.data))
        return out

    def info(self) -> dict:
        i = MpgInfo()
        _check(self.L.mpg_get_info(self.h, C.byref(i)))
        return {k: getattr(i, k) for k, _ in MpgInfo._fields_}

    # ---------------------------------------------------------------- subroutines (field ids)
    def derivative(self, unk: int, out: int, idx: int) -> None:
        _check(self.L.mpg_derivative(self.h, unk, out, idx))

    def bcv(self, u: int, v: int, w: int, flag: float) -> None:
        _check(self.L.mpg_bcv(self.h, u, v, w, flag))

    def laplc(self, press: int, alap: int, impfl: int) -> None:
        _check(self.L.mpg_laplc(self.h, press, alap, impfl))

    def laplc_adjoint(self, y: int, out: int, impfl: int) -> None:
        """Adjoint of laplc in the vol*rh0-weighted inner product."""
        _check(self.L.mpg_laplc_adjoint(self.h, y, out, impfl))

    def prfr(self, press, ustr, vstr, wstr, uout, vout, wout, impfl) -> None:
        _check(self.L.mpg_prfr(self.h, press, ustr, vstr, wstr, uout, vout, wout, impfl))

    def div(self, ua, va, wa, rhs, iflg) -> MpgDiag:
        d = MpgDiag()
        _check(self.L.mpg_div(self.h, ua, va, wa, rhs, iflg, C.byref(d)))
        return d

    def precon(self, rhs, p, r, iprc, impfl) -> None:
        _check(self.L.mpg_precon(self.h, rhs, p, r, iprc, impfl))

    def gcrk(self, p, u1, v1, w1, u2, v2, w2, impfl) -> MpgGcrStats:
        st = MpgGcrStats()
        _check(self.L.mpg_gcrk(self.h, p, u1, v1, w1, u2, v2, w2, impfl, C.byref(st)))
        return st

    def mpdatamper(self, unk: int, iflag: int) -> None:
        _check(self.L.mpg_mpdatamper(self.h, unk, iflag))

    def mpdatam(self, unk: int, iflag: int) -> None:
        """Open-boundary MPDATA (ref.f:3029-3311), for ``iper = 0``."""
        _check(self.L.mpg_mpdatam(self.h, unk, iflag))

    def courant(self, iflag: int = 1) -> MpgDiag:
        d = MpgDiag()
        _check(self.L.mpg_courant(self.h, iflag, C.byref(d)))
        return d

    def stats(self) -> MpgDiag:
        d = MpgDiag()
        _check(self.L.mpg_stats(self.h, C.byref(d)))
        return d

    def gcr_stats(self) -> MpgGcrStats:
        st = MpgGcrStats()
        _check(self.L.mpg_get_gcr_stats(self.h, C.byref(st)))
        return st

    # ---------------------------------------------------------------- driver
    def setup(self) -> MpgDiag:
        d = MpgDiag()
        _check(self.L.mpg_setup(self.h, C.byref(d)))
        return d

    def step(self, diag: bool = True) -> MpgDiag:
        d = MpgDiag()
        _check(self.L.mpg_step(self.h, C.byref(d) if diag else None))
        return d

    def velprd(self) -> None:
        """velprd (ref.f:4448): trajectory prediction of the advective velocity (itraj = 1 path)."""
        _check(self.L.mpg_velprd(self.h))

    def synchronize(self) -> None:
        _check(self.L.mpg_synchronize(self.h))

    # ---------------------------------------------------------------- restart files
    def restart_write(self, path: str, fmt: int = 0, ntime: int = 0) -> None:
        """Restart_Out_old (fmt 0: the reference's F14.6 text layout) or the lossless binary form (1)."""
        _check(self.L.mpg_restart_write(self.h, os.fsencode(path), fmt, ntime))

    def restart_read(self, path: str, fmt: int = 0) -> int:
        """Restart_In_old (fmt 0) or the binary form (1); returns the step number stored in the file."""
        nt = C.c_int()
        _check(self.L.mpg_restart_read(self.h, os.fsencode(path), fmt, C.byref(nt)))
        return nt.value

    def write_output(self, path: str, coord) -> None:
        """output(unk) (ref.f:2771): the r.d field file; coord is the mesh's (npoin, 3) coordinates."""
        cf = np.ascontiguousarray(np.asarray(coord, np.float64).T)     # coord(npoinx, 3), column-major
        _check(self.L.mpg_write_output(self.h, os.fsencode(path), cf.ctypes.data, cf.shape[1]))

    # ---------------------------------------------------------------- learned preconditioner
    def learned_init(self, seed: int = 0) -> None:
        _check(self.L.mpg_learned_init(self.h, seed))

    def learned_params(self) -> np.ndarray:
        out = np.empty(NPARAM, np.float32)
        _check(self.L.mpg_learned_get_params(self.h, out.ctypes.data_as(C.POINTER(C.c_float)), NPARAM))
        return out

    def learned_set_params(self, prm) -> None:
        a = np.ascontiguousarray(prm, np.float32)
        _check(self.L.mpg_learned_set_params(self.h, a.ctypes.data_as(C.POINTER(C.c_float)), a.size))

    def learned_forward(self, r: int, q: int) -> None:
        _check(self.L.mpg_learned_forward(self.h, r, q))

    def learned_grad(self, r: int, t: int):
        g = np.empty(NPARAM, np.float32)
        loss = C.c_double()
        _check(self.L.mpg_learned_grad(self.h, r, t, g.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loss)))
        return g, loss.value

    def learned_train_pair(self, r: int, t: int, lr: float) -> float:
        loss = C.c_double()
        _check(self.L.mpg_learned_train_pair(self.h, r, t, lr, C.byref(loss)))
        return loss.value

    def selftest_wait(self, arrive: bool, spins: int) -> bool:
        """Run the bounded-wait self-test; True when the wait completed, False when it gave up."""
        done = C.c_int()
        _check(self.L.mpg_selftest_wait(self.h, 1 if arrive else 0, spins, C.byref(done)))
        return bool(done.value)

    def learned_loss(self, mode: int) -> None:
        """0: residual norm ||A q - r||_W (default), 1: regression on the scaled error."""
        _check(self.L.mpg_learned_loss(self.h, mode))

    def learned_harvest(self, every: int, max_records: int) -> None:
        _check(self.L.mpg_learned_harvest(self.h, every, max_records))

    def learned_train_records(self, epochs: int, lr: float):
        loss, n = C.c_double(), C.c_int()
        _check(self.L.mpg_learned_train_records(self.h, epochs, lr, C.byref(loss), C.byref(n)))
        return loss.value, n.value

    # ---------------------------------------------------------------- instrumentation
    def stream(self) -> int:
        """cudaStream_t of the handle, as an integer (for torch.cuda.ExternalStream)."""
        p = C.c_void_p()
        _check(self.L.mpg_get_stream(self.h, C.byref(p)))
        return p.value or 0

    def kernel_timing(self, enable: bool) -> None:
        _check(self.L.mpg_kernel_timing(self.h, 1 if enable else 0))

    def kernel_times(self) -> dict:
        """{class: (launches, total_ms)} from CUDA events around each launch."""
        from .cabi import MpgKtime
        arr = (MpgKtime * 32)()
        n = C.c_int()
        _check(self.L.mpg_kernel_times(self.h, arr, 32, C.byref(n)))
        return {arr[i].name.decode(): (arr[i].launches, arr[i].total_ms) for i in range(min(n.value, 32))}


# convenience re-exports of the field ids
F_UNK, F_UNK1, F_UUU, F_UUU0, F_FRC, F_UNKDASH = (cabi.F_UNK, cabi.F_UNK1, cabi.F_UUU, cabi.F_UUU0,
                                                 cabi.F_FRC, cabi.F_UNKDASH)
F_PRPOT, F_RHS, F_COUR, F_ALPHA, F_COEFW, F_RH0 = (cabi.F_PRPOT, cabi.F_RHS, cabi.F_COUR, cabi.F_ALPHA,
                                                   cabi.F_COEFW, cabi.F_RH0)
F_WORK = cabi.F_WORK
