"""The 512x512x81 workload (21.2M nodes) on the GPU, checked through properties that do not depend
on size, since the CPU oracle needs minutes per step there:

* the passive scalar's mass sum(vol*rh0*psi) is conserved by MPDATA's antisymmetric face fluxes,
  to round-off;
* MPDATA with the nonoscillatory option keeps the positive scalar non-negative and within its
  initial maximum;
* every pressure solve stops on the reference's test max|r| <= eps0/dt;
* the mixed-precision path stays within the stated tolerance of the FP64 path and conserves the
  scalar's mass to FP64 round-off as well;
* laplc is W-self-adjoint for impfl = 0 (<A u, v>_W = <u, A v>_W) and its adjoint entry point
  satisfies the adjoint identity for impfl = 1;
* results are run-to-run deterministic (bit-identical) at this size as well.
"""
import numpy as np
import pytest

from src_b200 import mesh
from src_b200.api import Solver
from src_b200.cabi import F_RH0, F_UNK, F_WORK, RunParams

pytestmark = pytest.mark.gpu

NX, LEV, DT = 512, 81, 6.0


@pytest.fixture(scope="module")
def big_mesh():
    return mesh.generate(NX, L=LEV, seed=0, h0=400.0).to_reference()


def _params(precision=0):
    return RunParams(delt=DT, lord=3, nscal=1, eps0=1e-8, itr=200, iprc=2, itrp1=1, lipps=1,
                     strat=0.01 ** 2 / 9.80616, precision=precision)


def _scalar(rm):
    x, y, z = rm.coord.T
    return np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))


def _run(rm, precision, steps):
    s = Solver(_params(precision), rm)
    s.setup()
    s.set(F_UNK + 4, _scalar(rm))
    diags = [s.step() for _ in range(steps)]
    return s, diags


def test_fullsize_conservation_sign_and_stopping(big_mesh):
    rm = big_mesh
    s, diags = _run(rm, 0, 3)
    with s:
        w = rm.vol * s.get(F_RH0)
        psi0 = _scalar(rm)
        m0 = np.sum(w * psi0)
        psi = s.get(F_UNK + 4)
        assert abs(np.sum(w * psi) - m0) <= 1e-11 * m0
        assert abs(diags[-1].mass[4] - m0) <= 1e-11 * m0
        assert psi.min() >= 0.0 and psi.max() <= psi0.max()
        st = s.gcr_stats()
        assert st.status == 0 and st.dvmx <= s.params.eps0 / s.params.delt
        for d in diags:
            assert d.niter1 > 0 and d.smin[0] >= 0.0


def test_fullsize_mixed_precision_within_tolerance(big_mesh):
    rm = big_mesh
    a, _ = _run(rm, 0, 2)
    b, db = _run(rm, 1, 2)
    with a, b:
        for k, tol in ((0, 1e-6), (1, 1e-3), (2, 1e-3), (3, 1e-3)):
            x, y = b.get(F_UNK + k), a.get(F_UNK + k)
            assert np.linalg.norm(x - y) / np.linalg.norm(y) < tol, k
        # FP32 face fluxes with FP64 node updates: the scalar's mass to FP64 round-off
        w = rm.vol * b.get(F_RH0)
        m0 = np.sum(w * _scalar(rm))
        assert abs(db[-1].mass[4] - m0) <= 1e-11 * m0


def test_fullsize_laplc_adjoint_and_determinism(big_mesh):
    rm = big_mesh
    rng = np.random.default_rng(11)
    u, v = rng.standard_normal(rm.npoin), rng.standard_normal(rm.npoin)
    with Solver(_params(0), rm) as s:
        s.setup()
        w = rm.vol * s.get(F_RH0)
        s.set(F_WORK, u)
        s.set(F_WORK + 1, v)
        for impfl in (0, 1):
            s.laplc(F_WORK, F_WORK + 2, impfl)
            au = s.get(F_WORK + 2)
            s.laplc(F_WORK, F_WORK + 2, impfl)
            assert np.array_equal(s.get(F_WORK + 2), au)          # run-to-run bit-identical
            s.laplc_adjoint(F_WORK + 1, F_WORK + 3, impfl)
            atv = s.get(F_WORK + 3)
            scale = np.sqrt(np.sum(w * au * au) * np.sum(w * v * v))
            assert abs(np.sum(w * au * v) - np.sum(w * u * atv)) <= 1e-11 * scale
            if impfl == 0:
                s.laplc(F_WORK + 1, F_WORK + 4, 0)
                av = s.get(F_WORK + 4)
                assert np.linalg.norm(atv - av) <= 1e-10 * np.linalg.norm(av)
