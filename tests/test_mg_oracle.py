"""The multigrid V-cycle of precon (mg_flag = 1, ref.f:618-748) in the oracle, on the CPU: the
generator's coarser meshes, the match maps, the transfers (restriction_unstr, prolongation_unstr,
ref.f:757-951) with the reference's indexing (mg_bugs = 1) and corrected (mg_bugs = 0), and the
library's host-side acceptance of the levels."""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200 import mesh
from src_b200.cabi import RunParams


@pytest.fixture(scope="module")
def levels():
    cm = mesh.generate(16, L=9, seed=3)
    c1 = mesh.coarsen(cm)
    c2 = mesh.coarsen(c1)
    return (cm, c1, c2), [m.to_reference() for m in (cm, c1, c2)]


def make(levels, bugs, **kw):
    (cm, c1, c2), (rm, r1, r2) = levels
    P = RunParams(delt=10.0, mg_flag=1, iprc=1, mg_bugs=bugs, **kw)
    o = Oracle(P, rm)
    o.set_coarse(1, r1)                                   # matched by coordinates
    o.set_coarse(2, r2, mesh.coarse_match(c1, c2))        # the match2 array
    return o


def test_coarse_meshes_sit_on_fine_nodes(levels):
    (cm, c1, c2), (rm, r1, r2) = levels
    assert (c1.ncol, c2.ncol) == (cm.ncol // 4, cm.ncol // 16) and c1.L == c2.L == cm.L
    m1 = mesh.coarse_match(cm, c1)
    assert np.array_equal(r1.coord, rm.coord[m1])
    assert np.abs(mesh.closure_residual(r1)).max() < 1e-6 * np.abs(r1.sbb).max()


@pytest.mark.parametrize("bugs", [1, 0])
def test_prolongation_of_a_constant(levels, bugs):
    """The reference's own check (ref.f:563-582, dormant): a constant prolongated from the
    coarsest mesh to the coarse one and on to the fine one stays that constant."""
    (cm, c1, c2), (rm, r1, r2) = levels
    o = make(levels, bugs)
    e1 = o.mg_prolong(np.ones(r2.npoin), 2)
    e0 = o.mg_prolong(e1, 1)
    assert np.all(e1 == 1.0) and np.all(e0 == 1.0)


@pytest.mark.parametrize("bugs", [1, 0])
def test_restriction_of_a_constant(levels, bugs):
    (cm, c1, c2), (rm, r1, r2) = levels
    o = make(levels, bugs)
    assert np.allclose(o.mg_restrict(np.full(rm.npoin, 3.0), 1), 3.0, rtol=0, atol=1e-15)


def test_corrected_transfers_follow_the_neighbour_lists(levels):
    """mg_bugs = 0: restriction averages (s_ip + s_j)/2 over the matched node's true neighbours,
    prolongation fills every fine node; with the reference's loop-counter indexing the
    restriction reads nodes 1..count instead."""
    (cm, c1, c2), (rm, r1, r2) = levels
    rng = np.random.default_rng(4)
    s = rng.standard_normal(rm.npoin)
    m1 = mesh.coarse_match(cm, c1)
    nb = [[] for _ in range(rm.npoin)]
    for a, b in rm.iedge:
        nb[a].append(b)
        nb[b].append(a)
    want0 = np.array([np.mean([(s[ip] + s[j]) / 2 for j in nb[ip]]) for ip in m1])
    want1 = np.array([np.mean([(s[ip] + s[j]) / 2 for j in range(len(nb[ip]))]) for ip in m1])
    assert np.allclose(make(levels, 0).mg_restrict(s, 1), want0, rtol=1e-14, atol=1e-14)
    assert np.allclose(make(levels, 1).mg_restrict(s, 1), want1, rtol=1e-14, atol=1e-14)
    e = make(levels, 0).mg_prolong(rng.standard_normal(r1.npoin) + 5.0, 1)
    assert np.all(e != 0.0)


def test_vcycle_runs_and_its_gcr_records(levels):
    """The V-cycle as the reference builds it (wide-stencil laplc rediscretised on the coarser
    meshes, pointwise Jacobi smoothing) slows GCR down on these meshes: the set-up solve stops at
    itr restart cycles, where the plain reference smoother converges."""
    (cm, c1, c2), (rm, r1, r2) = levels
    for bugs in (1, 0):
        o = make(levels, bugs, itr=20)
        o.setup()
        assert o.gcr_stats().niter == 60
    plain = Oracle(RunParams(delt=10.0, iprc=1, itr=100), rm)
    plain.setup()
    assert plain.gcr_stats().status == 0 and plain.gcr_stats().niter < 150


def test_library_accepts_the_levels_on_the_host(levels):
    """mg_flag = 1 needs iprc = 1 in FP64; other combinations are refused when the handle is made."""
    from src_b200.api import lib
    import ctypes as C
    from src_b200.cabi import MeshMarshal
    (cm, c1, c2), (rm, r1, r2) = levels
    L = lib()
    for P, code in ((RunParams(mg_flag=1, iprc=2), 5), (RunParams(mg_flag=1, iprc=1, precision=1), 5),
                    (RunParams(mg_flag=2, iprc=1), 1)):
        mm = MeshMarshal(rm)
        h = C.c_void_p()
        cp = P.to_c()
        assert L.mpg_create(C.byref(cp), C.byref(mm.c), 0, C.byref(h)) == code
