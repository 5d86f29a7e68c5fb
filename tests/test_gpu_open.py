"""Open channel (iper = 0) on the GPU, through the C ABI, against the oracle.

The channel has inflow (type 7) at x = 0, outflow (type 8) at x = Lx and walls (types 5, 6) at
y = 0 and y = Ly, so every iper = 0 branch of the reference runs: the derivative's boundary
closure (ref.f:4007-4014), bcv's wall projections and prescribed u (ref.f:1613-1641), courant's
boundary terms (ref.f:2049-2069) and mpdatam's inflow/outflow closure (ref.f:3143-3169).
Per-node sums follow the reference's order, so operators agree bit for bit; with the oracle
replaying the GPU's reduction order so do set-up and whole steps.
"""
import numpy as np
import pytest

from oracle.oracle import Oracle
from src_b200.api import MpgError, Solver
from src_b200.cabi import F_COUR, F_UNK, F_UNK1, F_UUU, F_WORK, RunParams

pytestmark = pytest.mark.gpu

W0, W1, W2, W3, W4, W5, W6 = range(F_WORK, F_WORK + 7)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def same_diag(d, do):
    a, b = d.as_dict(), do.as_dict()
    for k in a:
        assert a[k] == b[k], (k, a[k], b[k])


@pytest.fixture(scope="module")
def chan(open_mesh):
    cm, rm = open_mesh
    P = RunParams(delt=10.0, iper=0, nscal=1, v0inf=1.5, w0inf=0.25)
    o = Oracle(P, rm, gpu_order=True)
    o.setup()
    s = Solver(P, rm)
    s.setup()
    yield rm, o, s
    s.close()


def test_operators_bitwise(chan):
    rm, o, s = chan
    rng = np.random.default_rng(21)
    a = [rng.standard_normal(rm.npoin) for _ in range(4)]
    s.set(W0, a[0])
    for idx in (1, 2, 3):
        s.derivative(W0, W1, idx)
        assert np.array_equal(s.get(W1), o.derivative(a[0], idx)), idx
    for impfl in (0, 1):
        s.laplc(W0, W1, impfl)
        assert np.array_equal(s.get(W1), o.laplc(a[0], impfl)), impfl
        for k in range(4):
            s.set(W0 + k, a[k])
        s.prfr(W0, W1, W2, W3, W4, W5, W6, impfl)
        ref = o.prfr(a[0], a[1], a[2], a[3], impfl)
        for k in range(3):
            assert np.array_equal(s.get(W4 + k), ref[k]), (impfl, k)
    for k in range(3):
        s.set(W0 + k, a[k])
    s.div(W0, W1, W2, W3, -1)
    assert np.array_equal(s.get(W3), o.div(a[0], a[1], a[2], -1)[0])
    s.bcv(W0, W1, W2, 1.0)
    ref = o.bcv(a[0], a[1], a[2], 1.0)
    for k in range(3):
        assert np.array_equal(s.get(W0 + k), ref[k]), k


def test_courant_bitwise(chan):
    rm, o, s = chan
    for k in range(3):
        s.set(F_UUU + k, o.get(F_UUU + k))
    d, dref = s.courant(1), o.courant(1)
    assert np.array_equal(s.get(F_COUR), o.get(F_COUR))
    assert d.crnmx == dref.crnmx and d.icrnmx == dref.icrnmx


@pytest.mark.parametrize("iflag", [1, 2, 3, 4, 5])
def test_mpdatam_bitwise(chan, iflag):
    rm, o, s = chan
    for k in range(3):
        s.set(F_UUU + k, o.get(F_UUU + k))
    psi = np.random.default_rng(22 + iflag).uniform(0.5, 1.5, rm.npoin)
    s.set(W0, psi)
    s.mpdatam(W0, iflag)
    assert np.array_equal(s.get(W0), o.mpdatam(psi, iflag))


def test_gcrk_bitwise(chan):
    rm, o, s = chan
    x, y, z = rm.coord.T
    bump = np.exp(-((x - 40e3) ** 2 + (y - 70e3) ** 2) / 15e3 ** 2 - (z - 6e3) ** 2 / 3e3 ** 2)
    u1 = [o.get(F_UNK1 + k) + (0.5, -0.3, 0.2)[k] * bump for k in range(3)]
    for k in range(3):
        s.set(W1 + k, u1[k])
    s.set(W0, 0.0)
    st = s.gcrk(W0, W1, W2, W3, W4, W5, W6, 1)
    p, (u2, v2, w2), sto = o.gcrk(np.zeros(rm.npoin), u1[0], u1[1], u1[2], 1)
    assert st.status == sto.status == 0 and st.niter == sto.niter
    assert np.array_equal(s.get(W0), p)
    for k, ref in enumerate((u2, v2, w2)):
        assert np.array_equal(s.get(W4 + k), ref)


def _pair(rm, gpu_order, **kw):
    P = RunParams(delt=10.0, iper=0, nscal=1, **kw)
    o = Oracle(P, rm, gpu_order=gpu_order)
    s = Solver(P, rm)
    x, y, z = rm.coord.T
    g = np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))
    return o, s, g


def test_steps_bitwise(open_mesh):
    """Set-up and 20 steps of the channel: every field, diagnostic and iteration count equal."""
    _, rm = open_mesh
    o, s, g = _pair(rm, True)
    with s:
        same_diag(s.setup(), o.setup())
        o.set(F_UNK + 4, g)
        s.set(F_UNK + 4, g)
        for _ in range(20):
            d, do = s.step(), o.step()
            same_diag(d, do)
        for k in range(5):
            assert np.array_equal(s.get(F_UNK + k), o.get(F_UNK + k)), k
        assert d.smin[0] >= 0.0


def test_one_step_reference_order(open_mesh):
    """Against the oracle's sequential sums.  The channel's pressure problem converges slowly
    (the set-up's potential-flow solve from p = 0 takes about 300 iterations), so the two
    summation orders follow different GCR paths and the results agree to what the stopping test
    allows, not to round-off: measured after one step, 1.5e-9 (u), 6.1e-7 (v), 2.6e-8 (w),
    2.9e-8 (theta').  The GPU equals the oracle in its own reduction order bit for bit
    (test_steps_bitwise), so these are properties of the case, not of the kernels."""
    _, rm = open_mesh
    o, s, g = _pair(rm, False)
    with s:
        o.setup()
        s.setup()
        o.step()
        s.step()
        assert rel(s.get(F_UNK), o.get(F_UNK)) <= 1e-8
        for k in range(1, 4):
            assert rel(s.get(F_UNK + k), o.get(F_UNK + k)) <= 1e-5, k


def test_mixed_precision_channel(open_mesh):
    """Mixed precision on the channel (FP32 fluxes, operator and MPDATA intermediates, FP64
    stopping test): one step stays close to the FP64 oracle and its solves converge."""
    _, rm = open_mesh
    o, _, g = _pair(rm, False)
    with Solver(RunParams(delt=10.0, iper=0, nscal=1, precision=1), rm) as s:
        o.setup()
        s.setup()
        o.step()
        s.step()
        assert rel(s.get(F_UNK), o.get(F_UNK)) <= 1e-5
        for k in range(1, 4):
            assert rel(s.get(F_UNK + k), o.get(F_UNK + k)) <= 1e-2, k
        assert s.gcr_stats().status == 0


def test_wrong_variant_is_an_argument_error(chan, small_mesh):
    rm, o, s = chan
    with pytest.raises(MpgError) as e:
        s.mpdatamper(W0, 1)
    assert e.value.code == 1
    with Solver(RunParams(delt=10.0), small_mesh[1]) as s2:
        with pytest.raises(MpgError) as e:
            s2.mpdatam(W0, 1)
        assert e.value.code == 1
