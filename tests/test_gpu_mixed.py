"""Mixed-precision runs (MPG_PREC_MIXED): FP32 face vectors, MPDATA face fluxes and
intermediates, FP32 GCR directions and operator; FP64 pressure, residual, inner products,
coefficients, stopping test, column Thomas solves and mass sums.  Each result is compared with
the FP64 oracle."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200.api import Solver
from src_b200.cabi import F_UNK, RunParams

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_mixed_against_fp64_oracle(c1_mesh):
    cm, rm = c1_mesh
    x, y, z = rm.coord.T
    g = np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
    o = Oracle(RunParams(delt=10.0, nscal=1), rm)
    o.setup()
    o.set(F_UNK + 4, g)
    with Solver(RunParams(delt=10.0, nscal=1, precision=1), rm) as s:
        s.setup()
        s.set(F_UNK + 4, g)
        m0 = s.stats().mass[4]
        for _ in range(5):
            do = o.step()
            d = s.step()
            assert s.gcr_stats().status == 0
        assert rel(s.get(F_UNK), o.get(F_UNK)) <= 1e-6              # u, dominated by U = 10 m/s
        for k in (1, 2, 3):                                          # v, w, theta' (small fields)
            assert rel(s.get(F_UNK + k), o.get(F_UNK + k)) <= 1e-4, k
        assert rel(s.get(F_UNK + 4), o.get(F_UNK + 4)) <= 1e-6      # passive scalar
        assert d.smin[0] >= 0.0                                      # sign preserved
        # FP32 face fluxes, FP64 node updates: conserved to FP64 round-off
        assert abs(d.mass[4] - m0) <= 1e-12 * m0
        assert abs(d.niter1 - do.niter1) <= 2
