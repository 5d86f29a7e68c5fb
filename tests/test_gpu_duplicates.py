"""The reference's own periodic input form on the GPU, through the C ABI, against the oracle:
duplicate nodes on opposite sides (icoin pairs, icoin2 pairs, icoin4 corner quadruples), each copy
with its part of the dual cell, every edge sum completed over the copy group in cyclicr's order
(ref.f:4377-4446) and the copies' volumes summed at set-up (ref.f:99-103).  mpdatamper takes the
FCT bounds over the periodic lists with the reference's corner minima (ref.f:3821-3867) and sums
the in/out fluxes over the copies (ref.f:3897-3902).  Operators agree bit for bit; gcrk and whole
steps do with the oracle replaying the GPU's reduction order."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200 import mesh
from src_b200.api import MpgError, Solver
from src_b200.cabi import F_UNK, F_UNK1, F_UUU, F_WORK, RunParams

pytestmark = pytest.mark.gpu

W0, W1, W2, W3, W4, W5, W6 = range(F_WORK, F_WORK + 7)


@pytest.fixture(scope="module", params=[(8, 9), (24, 21)])
def dup(request):
    nx, L = request.param
    rm = mesh.generate(nx, L=L, seed=2, duplicates=True).to_reference()
    P = RunParams(delt=10.0, nscal=1)
    o = Oracle(P, rm, gpu_order=True)
    o.setup()
    s = Solver(P, rm)
    s.setup()
    yield rm, o, s
    s.close()


def test_operators_bitwise(dup):
    rm, o, s = dup
    rng = np.random.default_rng(51)
    a = [rng.standard_normal(rm.npoin) for _ in range(4)]
    s.set(W0, a[0])
    for idx in (1, 2, 3):
        s.derivative(W0, W1, idx)
        assert np.array_equal(s.get(W1), o.derivative(a[0], idx)), idx
    for impfl in (0, 1):
        s.set(W0, a[0])
        s.laplc(W0, W1, impfl)
        assert np.array_equal(s.get(W1), o.laplc(a[0], impfl)), impfl
        for k in range(4):
            s.set(W0 + k, a[k])
        s.prfr(W0, W1, W2, W3, W4, W5, W6, impfl)
        ref = o.prfr(a[0], a[1], a[2], a[3], impfl)
        for k in range(3):
            assert np.array_equal(s.get(W4 + k), ref[k]), (impfl, k)
    for iflg in (-1, 1):
        for k in range(3):
            s.set(W0 + k, a[k])
        s.div(W0, W1, W2, W3, iflg)
        assert np.array_equal(s.get(W3), o.div(a[0], a[1], a[2], iflg)[0]), iflg


@pytest.mark.parametrize("iprc", [1, 2])
def test_precon_bitwise(dup, iprc):
    rm, o, s = dup
    r = np.random.default_rng(52).standard_normal(rm.npoin)
    s.set(W0, r)
    s.precon(W0, W1, W2, iprc, 1)
    assert np.array_equal(s.get(W1), o.precon(r, iprc, 1))


@pytest.mark.parametrize("iflag", [1, 2, 3, 4, 5])
def test_mpdatamper_bitwise(dup, iflag):
    rm, o, s = dup
    for k in range(3):
        s.set(F_UUU + k, o.get(F_UUU + k))
    psi = np.random.default_rng(53 + iflag).uniform(0.5, 1.5, rm.npoin)
    s.set(W0, psi)
    s.mpdatamper(W0, iflag)
    assert np.array_equal(s.get(W0), o.mpdatamper(psi, iflag))


def test_gcrk_and_steps_bitwise(dup):
    rm, _, _ = dup
    P = RunParams(delt=10.0, nscal=1)
    o = Oracle(P, rm, gpu_order=True)
    with Solver(P, rm) as s:
        assert s.setup().as_dict() == o.setup().as_dict()
        x, y, z = rm.coord.T
        g = np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
        s.set(F_UNK + 4, g)
        o.set(F_UNK + 4, g)
        for _ in range(3):
            assert s.step().as_dict() == o.step().as_dict()
        for k in range(5):
            assert np.array_equal(s.get(F_UNK + k), o.get(F_UNK + k)), k
        bump = np.exp(-((x - 40e3) ** 2 + (y - 70e3) ** 2) / 15e3 ** 2 - (z - 6e3) ** 2 / 3e3 ** 2)
        u1 = [o.get(F_UNK1 + k) + (0.5, -0.3, 0.2)[k] * bump for k in range(3)]
        for k in range(3):
            s.set(W1 + k, u1[k])
        s.set(W0, 0.0)
        st = s.gcrk(W0, W1, W2, W3, W4, W5, W6, 1)
        p, _, sto = o.gcrk(np.zeros(rm.npoin), u1[0], u1[1], u1[2], 1)
        assert (st.status, st.niter) == (sto.status, sto.niter)
        assert np.array_equal(s.get(W0), p)


def test_mixed_precision_duplicate_form(dup):
    """FP32 operator, directions and MPDATA fluxes on the duplicate form, against the FP64 oracle;
    the scalar stays non-negative.  On these small meshes the pressure solve stops at the
    iteration limit (8x8x9) or just under eps0, so where it stops moves the small fields: the
    FP64 oracle's own v, w, theta' change by up to 7e-4 when eps0 goes from 1e-8 to 1e-9.  The
    bound for each small field is therefore three times that change (at least 1e-4).  The scalar
    starts as a periodic bump, equal on the copies of every seam node.
    (The sum of vol*rh0*psi over all nodes is not an invariant of this form: every copy carries
    its group's summed volume and edge sums, so the FP64 reference does not conserve it either.)"""
    rm, _, _ = dup
    # a periodic bump: both copies of a seam node start with the same value, as the duplicate form
    # requires (a bump by plain coordinates gives the x = 0 and x = Lx copies different values, and
    # then the FP64 reference's scalar goes negative at the seam as well)
    x, y, z = rm.coord.T
    Lx, Ly = x.max() - x.min(), y.max() - y.min()
    dx = np.abs(x - 30e3)
    dy = np.abs(y - 60e3)
    dx, dy = np.minimum(dx, Lx - dx), np.minimum(dy, Ly - dy)
    g = np.exp(-(dx ** 2 + dy ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
    ref = {}
    for eps0 in (1e-8, 1e-9):
        o = Oracle(RunParams(delt=10.0, nscal=1, eps0=eps0), rm)
        o.setup()
        o.set(F_UNK + 4, g)
        for _ in range(3):
            o.step()
        ref[eps0] = [o.get(F_UNK + k) for k in range(5)]
    rel = lambda a, b: np.linalg.norm(a - b) / np.linalg.norm(b)
    with Solver(RunParams(delt=10.0, nscal=1, precision=1), rm) as s:
        s.setup()
        s.set(F_UNK + 4, g)
        for _ in range(3):
            d = s.step()
        assert rel(s.get(F_UNK), ref[1e-8][0]) <= 3e-6
        for k in (1, 2, 3):
            tol = max(1e-4, 3.0 * rel(ref[1e-9][k], ref[1e-8][k]))
            assert rel(s.get(F_UNK + k), ref[1e-8][k]) <= tol, (k, tol)
        assert rel(s.get(F_UNK + 4), ref[1e-8][4]) <= 1e-6
        assert d.smin[0] >= 0.0


def test_unsupported_with_copy_lists():
    rm = mesh.generate(8, L=9, seed=2, duplicates=True).to_reference()
    for iprc in (3, 4):
        with pytest.raises(MpgError) as e:
            Solver(RunParams(delt=10.0, iprc=iprc), rm)
        assert e.value.code == 5
    with Solver(RunParams(delt=10.0), rm) as s:
        with pytest.raises(MpgError) as e:
            s.laplc_adjoint(W0, W1, 1)
        assert e.value.code == 5
