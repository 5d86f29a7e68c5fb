"""Restart files: the reference's Restart_Out_old / Restart_In_old text layout (F14.6, lossy) and
the lossless binary form, written and read through the C ABI."""
import os

import numpy as np
import pytest

from src_b200.api import MpgError, Solver, reference_restart_name
from src_b200.cabi import (F_COEFW, F_COUR, F_FRC, F_PRPOT, F_RHS, F_UNK, F_UNK1, F_UNKDASH, F_UUU,
                           F_UUU0, RunParams)

pytestmark = pytest.mark.gpu

STATE = ([F_UNK + k for k in range(5)] + [F_UNK1 + k for k in range(4)] + [F_UUU + k for k in range(3)] +
         [F_UUU0 + k for k in range(3)] + [F_FRC + k for k in range(4)] + [F_UNKDASH + k for k in range(3)] +
         [F_PRPOT, F_RHS, F_COUR])


def _params():
    return RunParams(delt=10.0, nscal=1)


def _started(rm, steps):
    s = Solver(_params(), rm)
    s.setup()
    x, y, z = rm.coord.T
    s.set(F_UNK + 4, np.exp(-((x - x.mean()) ** 2 + (y - y.mean()) ** 2) / 2e8))
    for _ in range(steps):
        s.step()
    return s


def test_binary_restart_continues_bit_for_bit(small_mesh, tmp_path):
    _, rm = small_mesh
    path = str(tmp_path / "state.bin")
    with _started(rm, 3) as a:
        a.restart_write(path, 1, ntime=3)
        ref = [a.step() for _ in range(2)]
        want = {f: a.get(f) for f in STATE}
        st_a = a.gcr_stats()
    with Solver(_params(), rm) as b:
        assert b.restart_read(path, 1) == 3
        got = [b.step() for _ in range(2)]
        for f in STATE:
            assert np.array_equal(b.get(f), want[f]), f
        st_b = b.gcr_stats()
    assert (st_a.nitsm, st_a.icount) == (st_b.nitsm, st_b.icount)
    for d1, d2 in zip(ref, got):
        assert d1.as_dict() == d2.as_dict()


def test_text_restart_reference_layout(small_mesh, tmp_path):
    _, rm = small_mesh
    n = rm.npoin
    path = str(tmp_path / reference_restart_name(3))
    assert os.path.basename(path) == "Rstart_Out        3.d"
    with _started(rm, 3) as a:
        a.restart_write(path, 0, ntime=3)
        fields = {f: a.get(f) for f in (F_UUU, F_UUU + 1, F_UUU + 2, F_UNKDASH, F_UNKDASH + 1, F_UNKDASH + 2,
                                        F_UNK, F_UNK + 1, F_UNK + 2, F_UNK + 3, F_FRC, F_FRC + 1, F_FRC + 2,
                                        F_FRC + 3, F_PRPOT, F_RHS, F_COUR, F_COEFW)}
        st = a.gcr_stats()
    lines = open(path).read().split("\n")
    assert lines[-1] == ""
    lines = lines[:-1]
    assert len(lines) == 6 * n + 2
    assert all(len(l) == 42 for l in lines[:3 * n]) and all(len(l) == 56 for l in lines[3 * n:6 * n])
    assert [int(v) for v in lines[6 * n].split()] == [st.nitsm, st.icount]
    assert int(lines[6 * n + 1]) == 3
    # uuu1 (the velocity predictor's array, unused with itraj = 0) is written as zeros
    assert all(float(l[i:i + 14]) == 0.0 for l in lines[n:2 * n] for i in (0, 14, 28))
    # field values: the F14.6 rendering of the device values
    blocks = [(0, [F_UUU, F_UUU + 1, F_UUU + 2]), (2, [F_UNKDASH, F_UNKDASH + 1, F_UNKDASH + 2]),
              (3, [F_UNK, F_UNK + 1, F_UNK + 2, F_UNK + 3]), (4, [F_FRC, F_FRC + 1, F_FRC + 2, F_FRC + 3]),
              (5, [F_PRPOT, F_RHS, F_COUR, F_COEFW])]
    for b, fids in blocks:
        for j, f in enumerate(fids):
            col = [lines[b * n + ip][14 * j:14 * j + 14] for ip in range(n)]
            assert col == ["%14.6f" % v for v in fields[f]], f
    # reading restores the rounded values and the counters
    with Solver(_params(), rm) as b:
        assert b.restart_read(path, 0) == 3
        for f, v in fields.items():
            assert np.array_equal(b.get(f), np.array([float("%14.6f" % x) for x in v])), f
        st_b = b.gcr_stats()
        assert (st_b.nitsm, st_b.icount) == (st.nitsm, st.icount)
        b.step()                              # a run continues from the text restart


def test_restart_errors(small_mesh, tmp_path):
    _, rm = small_mesh
    with Solver(_params(), rm) as s:
        with pytest.raises(MpgError):
            s.restart_read(str(tmp_path / "missing.d"), 0)
        bad = tmp_path / "bad.bin"
        bad.write_bytes(b"not a restart file")
        with pytest.raises(MpgError):
            s.restart_read(str(bad), 1)
        short = tmp_path / "short.d"
        short.write_text("      1.000000      2.000000\n")
        with pytest.raises(MpgError):
            s.restart_read(str(short), 0)
        with pytest.raises(MpgError):
            s.restart_write(str(tmp_path / "x"), 7)


def test_output_file_reference_layout(small_mesh, tmp_path):
    """output(unk) (ref.f:2771-2806): header, then one line per node in format (1x,i7,8e12.4)."""
    _, rm = small_mesh
    path = str(tmp_path / "r.d")
    with _started(rm, 2) as s:
        s.write_output(path, rm.coord)
        u = [s.get(F_UNK + k) for k in range(4)]
    lines = open(path).read().split("\n")[:-1]
    n = rm.npoin
    assert float(lines[0]) == 1.0 and int(lines[1]) == n
    assert lines[2] == "point X Y Z u v w temp Velocity"
    assert len(lines) == n + 3 and all(len(l) == 104 for l in lines[3:])

    def e4(x):                                  # the value an E12.4 field denotes
        return float("%.3E" % x)

    vv = np.sqrt(u[0] ** 2 + u[1] ** 2 + u[2] ** 2)
    for ip in (0, 1, n // 2, n - 1):
        l = lines[3 + ip]
        assert int(l[:8]) == ip + 1
        f = [l[8 + 12 * i:20 + 12 * i] for i in range(8)]
        assert all(x.strip()[0] in "-0" and "E" in x for x in f), f
        want = [rm.coord[ip, 0] / 1e3, rm.coord[ip, 1] / 1e3, rm.coord[ip, 2] / 1e3,
                u[0][ip], u[1][ip], u[2][ip], u[3][ip], vv[ip]]
        assert [float(x) for x in f] == [e4(x) for x in want]
