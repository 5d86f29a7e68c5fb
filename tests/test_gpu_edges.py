"""Edge shapes of the column layout on the GPU, through the C ABI, against the oracle: a single
level (no vertical faces), two and three levels (the level-pair kernels' odd and even ends), the
largest supported column (128 levels, one line-solve warp holding it whole), and a column count
that is not a multiple of 32 (partial line-solve warps).  Operators bit for bit, then a set-up
solve and three whole steps bit for bit with the oracle replaying the GPU's reduction order; more
than 128 levels is refused at creation."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200 import mesh
from src_b200.api import MpgError, Solver
from src_b200.cabi import F_UNK, F_UUU, F_WORK, RunParams

pytestmark = pytest.mark.gpu

W0, W1, W2, W3, W4, W5, W6 = range(F_WORK, F_WORK + 7)
SHAPES = [(9, 1), (5, 2), (7, 3), (4, 128), (33, 5)]


@pytest.fixture(scope="module", params=SHAPES, ids=[f"{nx}x{nx}x{L}" for nx, L in SHAPES])
def edge(request):
    nx, L = request.param
    rm = mesh.generate(nx, L=L, seed=4, h0=300.0).to_reference()
    P = RunParams(delt=10.0, nscal=1)
    o = Oracle(P, rm, gpu_order=True)
    s = Solver(P, rm)
    assert s.setup().as_dict() == o.setup().as_dict()
    yield rm, o, s
    s.close()


def test_operators_bitwise(edge):
    rm, o, s = edge
    rng = np.random.default_rng(11)
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
def test_precon_bitwise(edge, iprc):
    rm, o, s = edge
    r = np.random.default_rng(12).standard_normal(rm.npoin)
    s.set(W0, r)
    s.precon(W0, W1, W2, iprc, 1)
    assert np.array_equal(s.get(W1), o.precon(r, iprc, 1))


def test_mpdatamper_bitwise(edge):
    rm, o, s = edge
    for k in range(3):
        s.set(F_UUU + k, o.get(F_UUU + k))
    psi = np.random.default_rng(13).uniform(0.5, 1.5, rm.npoin)
    for iflag in (1, 4, 5):
        s.set(W0, psi)
        s.mpdatamper(W0, iflag)
        assert np.array_equal(s.get(W0), o.mpdatamper(psi, iflag)), iflag


def test_steps_bitwise(edge):
    rm, _, _ = edge
    P = RunParams(delt=10.0, nscal=1)
    o = Oracle(P, rm, gpu_order=True)
    x, y, z = rm.coord.T
    g = np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
    with Solver(P, rm) as s:
        assert s.setup().as_dict() == o.setup().as_dict()
        s.set(F_UNK + 4, g)
        o.set(F_UNK + 4, g)
        for _ in range(3):
            assert s.step().as_dict() == o.step().as_dict()
        for k in range(5):
            assert np.array_equal(s.get(F_UNK + k), o.get(F_UNK + k)), k


def test_more_than_128_levels_refused():
    rm = mesh.generate(3, L=129, seed=4).to_reference()
    with pytest.raises(MpgError) as e:
        Solver(RunParams(delt=10.0), rm)
    assert "128 levels" in str(e.value)
