"""The C-ABI library loads, exports every entry point the header declares, its structs match
the ctypes mirrors, and the host-only mesh analysis accepts column meshes and rejects others.
No GPU is used."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

from src_b200 import api, cabi, mesh

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "mpgcr.h")


def declared_functions():
    txt = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|const char \*)\s*(mpg_\w+)\s*\(", txt, re.M)))


def test_library_exports_header():
    L = api.lib()
    names = declared_functions()
    assert len(names) >= 25
    for nm in names:
        assert hasattr(L, nm), nm
    assert set(names) == set(api.EXPORTS)


def test_struct_layout_matches_header(tmp_path):
    src = tmp_path / "sz.c"
    src.write_text('#include "mpgcr.h"\n#include <stdio.h>\n#include <stddef.h>\n'
                   'int main(void){printf("%zu %zu %zu %zu %zu %zu\\n", sizeof(mpg_params), sizeof(mpg_mesh_ref),'
                   ' sizeof(mpg_gcr_stats), sizeof(mpg_diag), sizeof(mpg_info), offsetof(mpg_params, itmn));return 0;}\n')
    exe = tmp_path / "sz"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = [int(x) for x in subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split()]
    assert out == [C.sizeof(cabi.MpgParams), C.sizeof(cabi.MpgMeshRef), C.sizeof(cabi.MpgGcrStats),
                   C.sizeof(cabi.MpgDiag), C.sizeof(cabi.MpgInfo), cabi.MpgParams.itmn.offset]


def test_analyze_column_mesh(small_mesh):
    cm, rm = small_mesh
    info = api.analyze_mesh(rm)
    assert info["ncol"] == cm.ncol and info["nlev"] == cm.L
    assert info["nedge2d"] == 3 * cm.ncol and info["npoin"] == rm.npoin
    assert info["bitwise_order"]


def test_analyze_open_channel(open_mesh):
    """The iper = 0 channel (lateral boundary points at every level) is a column mesh too, and
    its per-node sums keep the reference's edge order."""
    cm, rm = open_mesh
    info = api.analyze_mesh(rm)
    assert info["ncol"] == cm.ncol and info["nlev"] == cm.L
    assert info["nedge2d"] == cm.edges2d.shape[0] and info["bitwise_order"]


def test_analyze_permuted_mesh(small_mesh):
    """Node and edge numbering are free: a shuffled mesh is still recognised."""
    cm, rm = small_mesh
    rng = np.random.default_rng(0)
    perm = rng.permutation(rm.npoin)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(rm.npoin)
    eperm = rng.permutation(rm.nedge)
    rm2 = mesh.RefMesh(**{**rm.__dict__})
    rm2.coord = rm.coord[inv]
    rm2.vol = rm.vol[inv]
    rm2.iedge = perm[rm.iedge[eperm]].astype(np.int32)
    rm2.sn = rm.sn[eperm]
    rm2.ibpoin = rm.ibpoin.copy()
    rm2.ibpoin[:, 0] = perm[rm.ibpoin[:, 0]]
    info = api.analyze_mesh(rm2)
    assert info["ncol"] == cm.ncol and info["nlev"] == cm.L


def test_analyze_rejects_non_column_mesh(small_mesh):
    cm, rm = small_mesh
    bad = mesh.RefMesh(**{**rm.__dict__})
    bad.iedge = rm.iedge.copy()
    bad.iedge[0, 1] = (bad.iedge[0, 1] // cm.L) * cm.L + (bad.iedge[0, 0] % cm.L + 2) % cm.L
    with pytest.raises(api.MpgError) as e:
        api.analyze_mesh(bad)
    assert e.value.code == 3
    bad2 = mesh.RefMesh(**{**rm.__dict__})
    bad2.iedge = rm.iedge.copy()
    bad2.iedge[5, 0] = rm.npoin + 7
    with pytest.raises(api.MpgError) as e:
        api.analyze_mesh(bad2)
    assert e.value.code == 3


def test_analyze_periodic_duplicate_form():
    """The reference's duplicate-node periodic form (icoin/icoin2/icoin4 copy lists) is accepted;
    a node named in two copy groups is not."""
    m = mesh.generate(6, L=5, seed=2, duplicates=True)
    rm = m.to_reference()
    info = api.analyze_mesh(rm)
    assert info["ncol"] == 49 and info["nlev"] == 5
    bad = mesh.RefMesh(**{**rm.__dict__})
    bad.icoin2 = rm.icoin2.copy()
    bad.icoin2[0, 0] = rm.icoin[0, 0]
    with pytest.raises(api.MpgError) as e:
        api.analyze_mesh(bad)
    assert e.value.code == 5


def test_params_round_trip():
    p = cabi.RunParams(lord=5, eps0=1e-9, nscal=2)
    c = p.to_c()
    assert c.lord == 5 and c.eps0 == 1e-9 and c.nscal == 2 and c.iprc == 2
