"""Golden fixtures (tests/golden/): reference-format input decks and the oracle's results on them.

The decks are what the reference program reads (mesh3d.d and the control files); the fixtures
hold the oracle's fields after set-up and 3 steps in the reference's own configuration (iprc = 1,
lord = 9, lipps = 0, strat = 1e-5, sequential sums), made by tests/golden/make_golden.py.  The
reference itself could not be run (no Fortran compiler), so these pin the oracle: it must keep
reproducing them bit for bit from the committed decks, and the library's host side must accept
the decks as they are.
"""
import os

import numpy as np
import pytest

from src_b200 import api, mesh
from tests.golden import make_golden as mg

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("case", list(mg.CASES))
def test_oracle_reproduces_golden(case):
    P = mg.params(case)
    rm = mesh.read_mesh3d(os.path.join(HERE, case, "mesh3d.d"), P.iper)
    fields, diags = mg.run_oracle(rm, P)
    want = np.load(os.path.join(HERE, f"{case}_oracle.npz"))
    assert np.array_equal(fields, want["fields"])
    assert np.array_equal(diags, want["diags"])
    # every solve converged within itr restart cycles: set-up, then lord*(itmn-1) = 18 per step
    assert diags[0, 0] < P.itr * P.lord and np.all(diags[1:, 0] == 18)


@pytest.mark.parametrize("case", list(mg.CASES))
def test_deck_is_reference_input(case):
    P = mg.params(case)
    d = os.path.join(HERE, case)
    lines = open(os.path.join(d, "inputinc.d")).read().splitlines()
    assert lines[1].split()[5] == str(P.iper) and lines[1].split()[0] == str(mg.NSTEPS)
    rm = mesh.read_mesh3d(os.path.join(d, "mesh3d.d"), P.iper)
    info = api.analyze_mesh(rm)
    assert info["npoin"] == rm.npoin == 180 and info["nlev"] == 5 and info["bitwise_order"]
