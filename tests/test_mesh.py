"""Generator properties: torus Delaunay counts, closed dual cells, positive volumes, file round trip."""
import numpy as np

from src_b200 import mesh


def test_counts_and_degree(small_mesh):
    cm, rm = small_mesh
    assert cm.tri.shape[0] == 2 * cm.ncol
    assert cm.edges2d.shape[0] == 3 * cm.ncol
    assert rm.npoin == cm.ncol * cm.L
    assert rm.nedge == 3 * cm.ncol * cm.L + cm.ncol * (cm.L - 1)
    assert rm.nboun == 2 * cm.ncol


def test_dual_cells_close(small_mesh):
    cm, rm = small_mesh
    res = mesh.closure_residual(rm, include_boundary=True)
    scale = np.abs(rm.sn).max()
    assert np.abs(res).max() <= 1e-12 * scale


def test_interior_closure_without_boundary(small_mesh):
    cm, rm = small_mesh
    res = mesh.closure_residual(rm, include_boundary=False)
    scale = np.abs(rm.sn).max()
    k = rm.iedge  # noqa: F841
    lev = np.arange(rm.npoin) % cm.L
    interior = (lev > 0) & (lev < cm.L - 1)
    assert np.abs(res[interior]).max() <= 1e-12 * scale
    # at the top/bottom the open face equals the boundary face vector
    bot = np.arange(cm.ncol) * cm.L
    assert np.allclose(res[bot], cm.A, rtol=1e-12, atol=1e-12 * scale)


def test_volumes(small_mesh):
    cm, rm = small_mesh
    assert rm.vol.min() > 0
    # total volume = Lx*Ly*H - integral of the (piecewise linear) terrain
    assert np.isclose(cm.W.sum() * cm.H, rm.vol.sum(), rtol=1e-12)
    assert rm.vol.sum() < cm.Lx * cm.Ly * cm.H
    assert np.isclose(cm.A[:, 2].sum(), cm.Lx * cm.Ly, rtol=1e-12)


def test_flat_mesh_has_no_slopes():
    cm = mesh.generate(8, L=5, seed=0, h0=0.0)
    assert np.abs(cm.A[:, :2]).max() == 0.0
    rm = cm.to_reference()
    lev = np.arange(rm.npoin) % cm.L
    assert np.allclose(rm.coord[lev == 0, 2], 0.0)


def test_seeded(small_mesh):
    cm, _ = small_mesh
    cm2 = mesh.generate(12, L=9, seed=3)
    assert np.array_equal(cm.xy, cm2.xy) and np.array_equal(cm.T, cm2.T)
    cm3 = mesh.generate(12, L=9, seed=4)
    assert not np.array_equal(cm.xy, cm3.xy)


def test_stretched_levels():
    z = mesh.level_set(64, 20e3, stretch_dz0=0.117)
    assert np.isclose(z[-1], 20e3) and np.all(np.diff(z) > 0)
    assert np.diff(z)[0] < 0.2


def test_mesh3d_round_trip(tmp_path, small_mesh):
    _, rm = small_mesh
    p = tmp_path / "mesh3d.d"
    mesh.write_mesh3d(str(p), rm)
    back = mesh.read_mesh3d(str(p))
    assert back.npoin == rm.npoin and back.nedge == rm.nedge and back.nboun == rm.nboun
    assert np.array_equal(back.iedge, rm.iedge)
    assert np.array_equal(back.ibpoin, rm.ibpoin)
    assert np.array_equal(back.coord, rm.coord) and np.array_equal(back.sn, rm.sn)
    assert np.array_equal(back.vol, rm.vol) and np.array_equal(back.anp, rm.anp)


def test_reference_input_files(tmp_path, small_mesh):
    from src_b200.cabi import RunParams
    _, rm = small_mesh
    mesh.write_reference_inputs(str(tmp_path), rm, RunParams())
    for name in ("mesh3d.d", "mesh3d_c.d", "mesh3d_cc.d", "inputinc.d", "input_mg_v3.d", "inputre.d",
                 "match1.d", "match2.d"):
        assert (tmp_path / name).exists()
    lines = (tmp_path / "inputinc.d").read_text().splitlines()
    assert lines[1].split()[5] == "2"   # iper


def test_open_channel_counts_and_closure(open_mesh):
    """Open channel: a triangulated rectangle has 3V - 3 - V_b edges; every dual cell closes with
    its lateral side faces, which point along the side's outward normal."""
    cm, rm = open_mesh
    nbv = np.unique(cm.bcol).shape[0]
    assert nbv == 2 * (cm.nx + cm.ny) - 4
    assert cm.edges2d.shape[0] == 3 * cm.ncol - 3 - nbv
    assert cm.tri.shape[0] == 2 * cm.ncol - 2 - nbv
    res = mesh.closure_residual(rm, include_boundary=True)
    assert np.abs(res).max() <= 1e-12 * np.abs(rm.sn).max()
    lat = rm.ibpoin[:, 1] != 11
    assert rm.ibpoin.shape[0] == 2 * cm.ncol + cm.bcol.shape[0] * cm.L
    n = rm.sbb[lat] / np.linalg.norm(rm.sbb[lat], axis=1)[:, None]
    assert np.allclose(n, rm.anp[lat], atol=1e-12)
    assert sorted(np.unique(rm.ibpoin[lat, 1]).tolist()) == [5, 6, 7, 8]
    # corner columns sit on two sides
    assert np.bincount(cm.bcol).max() == 2 and np.sum(np.bincount(cm.bcol) == 2) == 4
    assert np.isclose(cm.W.sum() * cm.H, rm.vol.sum(), rtol=1e-12)


def test_open_channel_files(tmp_path, open_mesh):
    """The channel writes and reads back in the reference's iper = 0 layout (no periodic lists),
    and the control file carries iper = 0."""
    from src_b200.cabi import RunParams
    _, rm = open_mesh
    mesh.write_reference_inputs(str(tmp_path), rm, RunParams(iper=0))
    back = mesh.read_mesh3d(str(tmp_path / "mesh3d.d"), iper=0)
    assert back.nboun == rm.nboun
    assert np.array_equal(back.ibpoin, rm.ibpoin) and np.array_equal(back.sbb, rm.sbb)
    assert np.array_equal(back.iedge, rm.iedge) and np.array_equal(back.sn, rm.sn)
    lines = (tmp_path / "inputinc.d").read_text().splitlines()
    assert lines[1].split()[5] == "0"
