"""precon's multigrid V-cycle (mg_flag = 1, ref.f:618-748) on the GPU, through the C ABI, against
the oracle: the coarser meshes attached with mpg_set_coarse run laplc_c / laplc_cc as laplc on
their own meshes, the transfers (restriction_unstr, prolongation_unstr, ref.f:757-951) follow the
reference's summation order per node, so precon, gcrk and whole steps agree bit for bit (gcrk and
steps with the oracle replaying the GPU's reduction order), with the reference's indexing
(mg_bugs = 1) and corrected (mg_bugs = 0), for each smoother (sm_flag1 = 1, 2, 3)."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200 import mesh
from src_b200.api import MpgError, Solver
from src_b200.cabi import F_UNK, F_UNK1, F_WORK, RunParams

pytestmark = pytest.mark.gpu

W0, W1, W2, W3, W4, W5, W6 = range(F_WORK, F_WORK + 7)


@pytest.fixture(scope="module")
def levels():
    cm = mesh.generate(16, L=9, seed=3)
    c1 = mesh.coarsen(cm)
    c2 = mesh.coarsen(c1)
    return (cm, c1, c2), [m.to_reference() for m in (cm, c1, c2)]


def pair(levels, gpu_order=False, by_coordinates=False, **kw):
    (cm, c1, c2), (rm, r1, r2) = levels
    P = RunParams(**{**dict(delt=10.0, mg_flag=1, iprc=1, itrp2=1, itr=4), **kw})
    o = Oracle(P, rm, gpu_order=gpu_order)
    s = Solver(P, rm)
    m1, m2 = mesh.coarse_match(cm, c1), mesh.coarse_match(c1, c2)
    for x in (o, s):
        x.set_coarse(1, r1, None if by_coordinates else m1)
        x.set_coarse(2, r2, m2)
    return o, s


@pytest.mark.parametrize("bugs", [1, 0])
@pytest.mark.parametrize("sm", [1, 2, 3])
@pytest.mark.parametrize("impfl", [0, 1])
def test_precon_vcycle_bitwise(levels, bugs, sm, impfl):
    o, s = pair(levels, mg_bugs=bugs, sm_flag1=sm, by_coordinates=(sm == 2))
    o.setup()
    s.setup()
    r = np.random.default_rng(41).standard_normal(s.n)
    s.set(W0, r)
    s.precon(W0, W1, W2, 1, impfl)
    assert np.array_equal(s.get(W1), o.precon(r, 1, impfl))
    s.close()


@pytest.mark.parametrize("bugs", [1, 0])
def test_gcrk_and_steps_vcycle_bitwise(levels, bugs):
    o, s = pair(levels, gpu_order=True, mg_bugs=bugs)
    a, b = s.setup().as_dict(), o.setup().as_dict()
    assert a == b
    for _ in range(2):
        assert s.step().as_dict() == o.step().as_dict()
    for k in range(4):
        assert np.array_equal(s.get(F_UNK + k), o.get(F_UNK + k)), k
    st = s.gcr_stats()
    assert st.status == o.gcr_stats().status and st.niter == o.gcr_stats().niter
    s.close()


def test_vcycle_needs_both_levels(levels):
    (cm, c1, c2), (rm, r1, r2) = levels
    with Solver(RunParams(delt=10.0, mg_flag=1, iprc=1), rm) as s:
        s.set(W0, 1.0)
        with pytest.raises(MpgError) as e:
            s.precon(W0, W1, W2, 1, 1)
        assert e.value.code == 1
        with pytest.raises(MpgError) as e:
            s.set_coarse(2, r2)                           # level 1 first
        assert e.value.code == 1
    with Solver(RunParams(delt=10.0), rm) as s:
        with pytest.raises(MpgError) as e:
            s.set_coarse(1, r1)                           # handle made without mg_flag
        assert e.value.code == 1
