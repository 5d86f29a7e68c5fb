"""Learned preconditioner (iprc = 3) on the GPU: network forward and gradient against the CPU
reference of the network, training, convergence of the learned solve, and the fallback to the
plain vertical-line preconditioner."""
import numpy as np
import pytest

from tests import learned_ref as nr

pytestmark = pytest.mark.gpu

W0, W1, W2, W3, W4 = 48, 49, 50, 51, 52     # MPG_F_WORK slots


def _solver(rm, **kw):
    from src_b200.api import Solver
    from src_b200.cabi import RunParams
    return Solver(RunParams(**kw), rm)


def _geo(s, rm):
    from src_b200.cabi import F_COEFW, F_RH0
    return nr.Geometry(rm, s.get(F_RH0), rm.vol, s.get(F_COEFW), s.params.delt)


def _pair(s, rm, seed):
    """A residual r (smooth + noise), the line solve z = M^{-1} r and a target t near z."""
    rng = np.random.default_rng(seed)
    x, y, z = rm.coord.T
    r = np.sin(2 * np.pi * x / x.max()) * np.cos(z / 3000.0) + 0.3 * rng.standard_normal(rm.npoin)
    s.set(W0, r)
    s.precon(W0, W2, W3, 2, 1)
    zz = s.get(W2)
    t = zz + 0.5 * np.roll(zz, 7)
    return r, zz, t


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def test_untrained_network_is_plain_preconditioner(small_mesh):
    _, rm = small_mesh
    with _solver(rm) as s:
        s.setup()
        s.learned_init(0)
        r, z, _ = _pair(s, rm, 1)
        s.learned_forward(W0, W1)
        assert np.array_equal(s.get(W1), z)       # zero output layer: q = z exactly


def test_forward_matches_cpu_reference(small_mesh):
    _, rm = small_mesh
    prm = nr.init_params(seed=3, out_scale=0.3)
    with _solver(rm) as s:
        s.setup()
        s.learned_set_params(prm)
        assert np.array_equal(s.learned_params(), prm)
        r, z, _ = _pair(s, rm, 2)
        s.learned_forward(W0, W1)
        q = s.get(W1)
        geo = _geo(s, rm)
    fw = nr.forward(prm, r, z, geo, rnd=True)
    sig = np.abs(r).max()
    y_gpu = (q - z) * geo.bdiag.astype(np.float64) / sig
    # BF16 activations: occasional one-ulp flips between GPU and CPU rounding points
    assert _rel(y_gpu, fw["y"]) < 2e-2
    fw64 = nr.forward(prm, r, z, geo, rnd=False)
    assert _rel(y_gpu, fw64["y"]) < 5e-2


def test_gradient_matches_cpu_reference(small_mesh):
    """Error loss: regression of the network output on the scaled error of the pair."""
    _, rm = small_mesh
    prm = nr.init_params(seed=4, out_scale=0.3)
    with _solver(rm) as s:
        s.setup()
        s.learned_set_params(prm)
        s.learned_loss(1)
        r, z, t = _pair(s, rm, 3)
        s.set(W4, t)
        g, loss = s.learned_grad(W0, W4)
        g2, loss2 = s.learned_grad(W0, W4)
        geo = _geo(s, rm)
    assert np.array_equal(g, g2) and loss == loss2          # deterministic reductions
    fw = nr.forward(prm, r, z, geo, rnd=True)
    lref, gref = nr.backward(prm, fw, t, z, geo, rnd=True)
    assert loss == pytest.approx(lref, rel=2e-2)
    for name, (a, b) in _segments().items():
        ga, gb = g[a:b].astype(np.float64), gref[a:b]
        cos = ga @ gb / (np.linalg.norm(ga) * np.linalg.norm(gb))
        assert cos > 0.995, (name, cos)
        assert _rel(ga, gb) < 0.1, (name, _rel(ga, gb))


def _segments():
    segs = {"in": (nr.OFF_WIN, nr.OFF_L0), "out": (nr.OFF_WOUT, nr.NPARAM)}
    for l in range(nr.NL):
        segs[f"layer{l}"] = (nr.OFF_L0 + l * nr.LSTRIDE, nr.OFF_L0 + (l + 1) * nr.LSTRIDE)
    return segs


def test_residual_loss_gradient_matches_cpu_reference(small_mesh):
    """Residual loss 0.5*min_a ||r - a A q||_W^2/||r||_W^2: the loss from the GPU's own q, and the
    gradient against the CPU network reference driven by dL/dy = (a/||r||_W^2) (A^T W e) s/|b|
    with e = a A q - r and A^T W e from the adjoint entry point (checked against the assembled
    transpose in test_gpu_parity.py)."""
    from src_b200.cabi import F_RH0
    _, rm = small_mesh
    prm = nr.init_params(seed=6, out_scale=0.3)
    with _solver(rm) as s:
        s.setup()
        s.learned_set_params(prm)
        r, z, _ = _pair(s, rm, 5)
        g, loss = s.learned_grad(W0, W4)
        g2, loss2 = s.learned_grad(W0, W4)
        s.learned_forward(W0, W1)
        s.laplc(W1, W2, 1)
        a = s.get(W2)
        w = rm.vol * s.get(F_RH0)
        alpha = np.sum(w * a * r) / np.sum(w * a * a)
        e = alpha * a - r
        s.set(W3, e)
        s.laplc_adjoint(W3, W2, 1)
        atwe = w * s.get(W2)
        geo = _geo(s, rm)
    assert np.array_equal(g, g2) and loss == loss2
    swr = np.sum(w * r * r)
    assert loss == pytest.approx(0.5 * np.sum(w * e * e) / swr, rel=1e-6)
    fw = nr.forward(prm, r, z, geo, rnd=True)
    dy = alpha * atwe / swr * fw["s"] / geo.bdiag.astype(np.float64)
    _, gref = nr.backward(prm, fw, None, z, geo, rnd=True, dy=dy)
    for name, (a, b) in _segments().items():
        ga, gb = g[a:b].astype(np.float64), gref[a:b]
        cos = ga @ gb / (np.linalg.norm(ga) * np.linalg.norm(gb))
        assert cos > 0.995, (name, cos)
        assert _rel(ga, gb) < 0.1, (name, _rel(ga, gb))


def test_training_reduces_loss(small_mesh):
    _, rm = small_mesh
    with _solver(rm) as s:
        s.setup()
        s.learned_init(1)
        s.learned_loss(1)
        _, _, t = _pair(s, rm, 4)
        s.set(W4, t)
        losses = [s.learned_train_pair(W0, W4, 3e-3) for _ in range(60)]
    assert losses[-1] < 0.5 * losses[0], losses[::10]


def test_training_reduces_residual_loss(small_mesh):
    _, rm = small_mesh
    with _solver(rm) as s:
        s.setup()
        s.learned_init(1)
        _pair(s, rm, 4)
        losses = [s.learned_train_pair(W0, W4, 3e-3) for _ in range(60)]
    assert losses[-1] < 0.8 * losses[0], losses[::10]


def test_harvest_and_learned_solve(small_mesh):
    """Plain solves record (r, A^{-1} r) pairs; training on them lowers the loss; the learned
    solve converges to the same tolerance as the plain one."""
    from src_b200.cabi import F_UNK
    from src_b200.learned import compare, train
    from src_b200.cabi import RunParams
    _, rm = small_mesh
    P = RunParams(itr=200)
    w, hist, _ = train(rm, P, steps=4, every=2, max_records=32, epochs=4, lr=2e-3)
    assert all(h["pairs"] > 0 for h in hist)
    assert hist[-1]["loss"] < hist[0]["loss"]
    res = compare(rm, P, w, steps=3, warm=1)
    assert res["learned"]["iters_per_step"] > 0
    # both solves stop on the same criterion: the velocities agree to the solver tolerance
    du = np.abs(res["learned"]["u"] - res["plain"]["u"]).max()
    assert du < 1e-4 * max(np.abs(res["plain"]["u"]).max(), 1.0), du


def test_trained_network_gain_over_plain(small_mesh):
    """What the trained network gains over the method without it, on the 12x12x9 mesh: trained on
    4 steps of its own plain solves (4 epochs, residual loss), with the plain solves' measured
    contraction as the hand-over threshold, it cuts the first-solve GCR iterations of the next
    steps (measured on a B200: 124, 28, 29 against 142, 120, 84).  Training and inference are
    deterministic, so the comparison is reproducible.  Every learned solve still meets the same
    stopping test; on the 21.2M-node workload the network does not pay for its cost."""
    from src_b200.learned import compare, train
    from src_b200.cabi import RunParams
    _, rm = small_mesh
    P = RunParams(itr=200)
    w, hist, rate = train(rm, P, steps=4, every=2, max_records=48, epochs=4, lr=2e-3)
    assert hist[-1]["loss"] < hist[0]["loss"]
    res = compare(rm, RunParams(**{**P.__dict__, "nn_rate": rate}), w, steps=3, warm=1)
    plain, learned = res["plain"]["first_solve_iters"], res["learned"]["first_solve_iters"]
    assert sum(learned) < 0.8 * sum(plain), (learned, plain)
    du = np.abs(res["learned"]["u"] - res["plain"]["u"]).max()
    assert du < 1e-3, du


def test_nonfinite_network_falls_back_to_plain(small_mesh):
    """Non-finite network output: gcrk switches to the plain preconditioner before using it, so
    the step equals the plain step bit for bit and the fallback is counted."""
    from src_b200.cabi import F_UNK
    _, rm = small_mesh
    prm = nr.init_params(seed=5)
    prm[nr.OFF_BOUT] = np.nan
    with _solver(rm, iprc=2) as a, _solver(rm, iprc=3) as b:
        b.learned_set_params(prm)
        a.setup()
        b.setup()
        for _ in range(2):
            a.step()
            b.step()
            assert b.gcr_stats().fallbacks >= 1
        for f in range(F_UNK, F_UNK + 4):
            assert np.array_equal(a.get(f), b.get(f))


def test_slow_network_falls_back_and_converges(small_mesh):
    """A network that contracts the residual more slowly than nn_rate per iteration is replaced
    by the plain preconditioner mid-solve; the solve still meets the same stopping test."""
    from src_b200.cabi import F_UNK
    _, rm = small_mesh
    prm = nr.init_params(seed=7, out_scale=3.0)
    with _solver(rm, iprc=2) as a, _solver(rm, iprc=3, nn_rate=0.3) as b:
        b.learned_set_params(prm)
        a.setup()
        b.setup()
        eps = b.params.eps0 / b.params.delt
        for _ in range(2):
            a.step()
            db = b.step()
            assert db.fallbacks >= 1
            st = b.gcr_stats()
            assert st.status == 0 and st.dvmx <= eps
        # both runs stop on the same max-norm test; they took different paths to it, so the
        # fields agree to what that tolerance allows (the flow speed is 10 m/s)
        for f in range(F_UNK, F_UNK + 4):
            ga, gb = a.get(f), b.get(f)
            assert np.abs(ga - gb).max() < 1e-3 * 10.0


def test_bounded_wait_gives_up_and_device_stays_usable(small_mesh):
    """The tensor-core kernels' mbarrier waits are bounded: a wait whose arrival never comes (a
    flag nothing sets) gives up after its poll limit and reports it, and the device keeps working."""
    import time
    from src_b200.cabi import F_WORK
    _, rm = small_mesh
    with _solver(rm) as s:
        s.setup()
        assert s.selftest_wait(True, 1000) is True
        t0 = time.time()
        assert s.selftest_wait(False, 2000) is False
        assert time.time() - t0 < 30.0
        s.set(F_WORK, np.ones(rm.npoin))
        s.laplc(F_WORK, F_WORK + 1, 1)                # the context is still usable
        assert np.all(np.isfinite(s.get(F_WORK + 1)))
        s.step()
        from src_b200.api import MpgError
        with pytest.raises(MpgError):
            s.selftest_wait(False, 0)


def test_learned_requires_parameters(small_mesh):
    from src_b200.api import MpgError
    _, rm = small_mesh
    with _solver(rm, iprc=3) as s:
        with pytest.raises(MpgError):
            s.setup()
            s.step()
        with pytest.raises(MpgError):
            s.learned_set_params(np.zeros(10, np.float32))
