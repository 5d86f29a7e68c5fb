"""laplc's column blocks as the line preconditioner (iprc = 4) on the GPU, through the C ABI,
against the oracle's restatement (`orc_wide_solve`, `orc_precon`, `orc_gcrk`).

laplc's gradient uses face averages (p_n + p_j)/2, so in a column it couples level k with k and
k +- 2 only: its column block is tridiagonal on the even and on the odd levels.  `k_wide_solve`
runs the stride-2 Thomas recurrences in FP64 with the host's factorisation, in the oracle's
order of operations, so the solve, precon with one and two sweeps, gcrk and whole time steps
agree bit for bit (the last two with the oracle replaying the GPU's reduction order).  Covered:
the torus (iper = 2) on two meshes and the open channel (iper = 0), impfl 0 and 1.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200.api import MpgError, Solver
from src_b200.cabi import F_UNK, F_UNK1, F_WORK, RunParams

pytestmark = pytest.mark.gpu

W0, W1, W2, W3, W4, W5, W6 = range(F_WORK, F_WORK + 7)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def params(case, **kw):
    base = dict(delt=10.0, nscal=1, iprc=4)
    if case == "open":
        base.update(iper=0, v0inf=1.5, w0inf=0.25)
    base.update(kw)
    return RunParams(**base)


@pytest.fixture(scope="module", params=["small", "c1", "open"])
def case(request, small_mesh, c1_mesh, open_mesh):
    cm, rm = {"small": small_mesh, "c1": c1_mesh, "open": open_mesh}[request.param]
    return request.param, rm


@pytest.mark.parametrize("impfl", [0, 1])
def test_wide_solve_bitwise(case, impfl):
    name, rm = case
    P = params(name)
    o = Oracle(P, rm)
    o.setup()                    # rh0 and coefw, which the column blocks depend on
    r = np.random.default_rng(31).standard_normal(rm.npoin)
    with Solver(P, rm) as s:
        s.set(W0, r)
        s.precon(W0, W1, W2, 4, impfl)
        assert np.array_equal(s.get(W1), o.wide_solve(r, impfl))


@pytest.mark.parametrize("itrp1", [1, 2])
@pytest.mark.parametrize("impfl", [0, 1])
def test_precon_wide_bitwise(case, itrp1, impfl):
    name, rm = case
    P = params(name, itrp1=itrp1)
    o = Oracle(P, rm)
    o.setup()
    r = np.random.default_rng(32).standard_normal(rm.npoin)
    with Solver(P, rm) as s:
        s.setup()
        s.set(W0, r)
        s.precon(W0, W1, W2, 4, impfl)
        assert np.array_equal(s.get(W1), o.precon(r, 4, impfl))


def test_gcrk_wide_bitwise(case):
    name, rm = case
    P = params(name)
    o = Oracle(P, rm, gpu_order=True)
    o.setup()
    with Solver(P, rm) as s:
        s.setup()
        x, y, z = rm.coord.T
        bump = np.exp(-((x - 40e3) ** 2 + (y - 70e3) ** 2) / 15e3 ** 2 - (z - 6e3) ** 2 / 3e3 ** 2)
        u1 = [o.get(F_UNK1 + k) + (0.5, -0.3, 0.2)[k] * bump for k in range(3)]
        for k in range(3):
            s.set(W1 + k, u1[k])
        s.set(W0, 0.0)
        st = s.gcrk(W0, W1, W2, W3, W4, W5, W6, 1)
        p, (u2, v2, w2), sto = o.gcrk(np.zeros(rm.npoin), u1[0], u1[1], u1[2], 1)
        assert st.status == sto.status and st.niter == sto.niter
        assert np.array_equal(s.get(W0), p)
        for k, ref in enumerate((u2, v2, w2)):
            assert np.array_equal(s.get(W4 + k), ref)
        assert st.eer == sto.eer and st.eem == sto.eem and st.rl2 == sto.rl2


def test_steps_wide_bitwise(case):
    """Set-up and 3 time steps with iprc = 4, every field and diagnostic bit for bit."""
    name, rm = case
    P = params(name)
    o = Oracle(P, rm, gpu_order=True)
    with Solver(P, rm) as s:
        a, b = s.setup().as_dict(), o.setup().as_dict()
        assert a == b
        x, y, z = rm.coord.T
        g = np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
        s.set(F_UNK + 4, g)
        o.set(F_UNK + 4, g)
        for _ in range(3):
            d, do = s.step().as_dict(), o.step().as_dict()
            assert d == do
        for k in range(5):
            assert np.array_equal(s.get(F_UNK + k), o.get(F_UNK + k)), k


def test_wide_mixed_against_fp64_oracle(c1_mesh):
    """Mixed precision with the column blocks: FP32 operator and directions, FP64 Thomas solves,
    inner products and stopping test; 3 steps within the mixed path's tolerances of the FP64
    oracle with the same preconditioner."""
    cm, rm = c1_mesh
    o = Oracle(params("c1"), rm)
    o.setup()
    with Solver(params("c1", precision=1), rm) as s:
        s.setup()
        for _ in range(3):
            do = o.step()
            d = s.step()
            assert s.gcr_stats().status == 0
        assert rel(s.get(F_UNK), o.get(F_UNK)) <= 1e-6
        for k in (1, 2, 3):
            assert rel(s.get(F_UNK + k), o.get(F_UNK + k)) <= 1e-4, k
        assert abs(d.niter1 - do.niter1) <= 2


def test_wide_needs_its_factors(small_mesh):
    """A handle created for another preconditioner has no column-block factors: iprc = 4 at
    call time is an argument error, not a silent fallback."""
    cm, rm = small_mesh
    with Solver(RunParams(delt=10.0, iprc=2), rm) as s:
        with pytest.raises(MpgError) as e:
            s.precon(W0, W1, W2, 4, 1)
        assert e.value.code == 1
