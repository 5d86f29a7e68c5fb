"""The single-launch laplc (k_lap_fused, chosen with MPG_LAPLC_FUSED=1 at creation): gradient and
divergence items taken by ticket, each divergence item waiting for the gradient items it reads.
Each node's arithmetic is the two-launch form's, so laplc is bit-identical to the oracle, and
gcrk and whole steps are bit-identical to a solver using the two launches, in FP64 and in mixed
precision, on the periodic torus and the open channel."""
import os

import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200.api import Solver
from src_b200.cabi import F_UNK, F_WORK, RunParams

pytestmark = pytest.mark.gpu

W0, W1 = F_WORK, F_WORK + 1


def fused_solver(P, rm):
    os.environ["MPG_LAPLC_FUSED"] = "1"
    try:
        return Solver(P, rm)
    finally:
        del os.environ["MPG_LAPLC_FUSED"]


@pytest.fixture(scope="module", params=["torus", "channel"])
def meshes(request, c1_mesh, open_mesh):
    if request.param == "torus":
        return c1_mesh[1], RunParams(delt=10.0)
    return open_mesh[1], RunParams(delt=10.0, iper=0, v0inf=1.5, w0inf=0.25)


@pytest.mark.parametrize("impfl", [0, 1])
def test_fused_laplc_bitwise(meshes, impfl):
    rm, P = meshes
    o = Oracle(P, rm)
    o.setup()
    rng = np.random.default_rng(7 + impfl)
    with fused_solver(P, rm) as s:
        s.setup()
        for _ in range(3):                       # the ticket counter and epochs carry over launches
            p = rng.standard_normal(rm.npoin)
            s.set(W0, p)
            s.laplc(W0, W1, impfl)
            assert np.array_equal(s.get(W1), o.laplc(p, impfl))


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_steps_match_two_launches(c1_mesh, precision):
    _, rm = c1_mesh
    P = RunParams(delt=10.0, nscal=1, precision=precision)
    x, y, z = rm.coord.T
    g = np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
    with fused_solver(P, rm) as a, Solver(P, rm) as b:
        assert a.setup().as_dict() == b.setup().as_dict()
        a.set(F_UNK + 4, g)
        b.set(F_UNK + 4, g)
        for _ in range(3):
            assert a.step().as_dict() == b.step().as_dict()
        for k in range(5):
            assert np.array_equal(a.get(F_UNK + k), b.get(F_UNK + k)), k
