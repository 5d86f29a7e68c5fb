"""CPU checks of the network reference used by the learned-preconditioner GPU tests."""
import numpy as np
import pytest

from tests import learned_ref as nr


def _geometry(small_mesh, seed=0):
    _, rm = small_mesh
    rng = np.random.default_rng(seed)
    z = rm.coord[:, 2]
    rh0 = np.exp(-z / 9000.0) * (1.0 + 0.01 * rng.standard_normal(rm.npoin))
    coefw = np.ones(rm.npoin)
    return nr.Geometry(rm, rh0, rm.vol, coefw, 10.0), rng


def test_bf16_rounding_matches_torch():
    import torch
    x = np.random.default_rng(1).standard_normal(10000).astype(np.float32) * 37.0
    ref = torch.tensor(x).to(torch.bfloat16).float().numpy()
    assert np.array_equal(nr.bf16(x), ref)


def test_parameter_layout():
    assert nr.NPARAM == 9505
    Win, bin_, Ws, bs, wout, bout = nr.unpack(np.arange(nr.NPARAM, dtype=np.float64))
    assert Win.shape == (32, 4) and Ws[2].shape == (32, 96) and wout[-1] == nr.NPARAM - 2 and bout == nr.NPARAM - 1


def test_geometry_sane(small_mesh):
    geo, _ = _geometry(small_mesh)
    n = geo.n
    assert geo.bdiag.shape == (n,) and np.all(geo.bdiag > 0)
    assert np.all(geo.iDh > 0) and np.all(geo.iDv > 0)
    # aggregation of a constant field vanishes
    a = geo.aggregate(np.ones((n, 32)), "h")
    assert np.abs(a).max() < 1e-12


def test_backward_matches_autograd(small_mesh):
    geo, rng = _geometry(small_mesh)
    n = geo.n
    prm = nr.init_params(seed=2, out_scale=0.3)
    r = rng.standard_normal(n)
    z = r / geo.bdiag
    t = z + 0.1 * rng.standard_normal(n) / geo.bdiag
    fw = nr.forward(prm, r, z, geo, rnd=False)
    loss, g = nr.backward(prm, fw, t, z, geo, rnd=False)
    tl, tg = nr.torch_loss(prm, r, z, t, geo)
    assert loss == pytest.approx(tl, rel=1e-10)
    segs = [(nr.OFF_WIN, nr.OFF_L0)] + [(nr.OFF_L0 + l * nr.LSTRIDE, nr.OFF_L0 + (l + 1) * nr.LSTRIDE)
                                        for l in range(nr.NL)] + [(nr.OFF_WOUT, nr.NPARAM)]
    for a, b in segs:
        err = np.linalg.norm(g[a:b] - tg[a:b]) / max(np.linalg.norm(tg[a:b]), 1e-30)
        assert err < 1e-5, (a, b, err)


def test_bf16_forward_close_to_fp64(small_mesh):
    geo, rng = _geometry(small_mesh, seed=4)
    prm = nr.init_params(seed=5, out_scale=0.3)
    r = rng.standard_normal(geo.n)
    z = r / geo.bdiag
    y64 = nr.forward(prm, r, z, geo, rnd=False)["y"]
    y16 = nr.forward(prm, r, z, geo, rnd=True)["y"]
    assert np.linalg.norm(y16 - y64) / np.linalg.norm(y64) < 3e-2
