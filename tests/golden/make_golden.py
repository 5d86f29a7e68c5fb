"""Generate the golden fixtures in this directory (test infrastructure).

Two small decks in the input layout of the reference program lippsLFroude_implgwopks3D_unstr3.f
(`input`, ref.f:2172-2679): a doubly periodic torus mesh (iper = 2) and an open channel
(iper = 0), each 6x6 columns x 5 levels.  For each deck this writes

* ``<case>/mesh3d.d``, ``inputinc.d``, ``input_mg_v3.d``, ``inputre.d``: what the reference reads
  (its multigrid files ``mesh3d_c.d``, ``mesh3d_cc.d``, ``match1.d``, ``match2.d`` are unused with
  mg_flag = 0; ``--full-deck DIR`` writes them too, as copies of the fine mesh and identity maps);
* ``<case>_oracle.npz``: the CPU oracle's fields after set-up and after each of 3 time steps, and
  the per-step diagnostics, in the configuration the unmodified reference runs with this deck:
  the reference smoother (iprc = 1, ref.f:1811), lord = 9 (a compile-time constant, ref.f:1782),
  lipps = 0 and strat = 1e-5 (hard-coded, ref.f:133-134), sequential FP64 sums.

No Fortran compiler exists where this was made, so the reference itself has not been run on these
decks; the fixtures pin the oracle (against regressions here, and against the reference for
anyone who runs ``gfortran -O2 -fdefault-real-8 -fdefault-double-8`` on it in a deck directory).

Run from the repository root: ``python tests/golden/make_golden.py``.
"""
import argparse
import os
import shutil
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.oracle import Oracle                     # noqa: E402
from src_b200 import mesh                            # noqa: E402
from src_b200.cabi import F_PRPOT, F_UNK, F_UUU, RunParams   # noqa: E402

NSTEPS = 3
CASES = {"periodic": dict(periodic=True), "channel": dict(periodic=False)}


def params(case: str) -> RunParams:
    return RunParams(ntime=NSTEPS, delt=10.0, iper=2 if CASES[case]["periodic"] else 0, iprc=1, lord=9,
                     lipps=0, strat=1e-5)


def build(case: str):
    cm = mesh.generate(6, L=5, seed=2, **CASES[case])
    rm = cm.to_reference()
    assert cm.max_degree() <= 10             # neigh_list(npoinx,10) of the reference (ref.f:783)
    return rm


def run_oracle(rm, P):
    o = Oracle(P, rm)
    snaps, diags = [], []
    fids = [F_UNK + k for k in range(4)] + [F_UUU + k for k in range(3)] + [F_PRPOT]
    d = o.setup()
    for s in range(NSTEPS + 1):
        if s:
            d = o.step()
        snaps.append(np.stack([o.get(f) for f in fids]))
        dd = d.as_dict()
        diags.append([dd["niter"], dd["divmx"], dd["divmn"], dd["crnmx"]] + list(dd["stats"]))
    return np.stack(snaps), np.array(diags, dtype=np.float64)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--full-deck", default=None, help="also write a complete reference deck here")
    a = ap.parse_args()
    for case in CASES:
        rm, P = build(case), params(case)
        d = os.path.join(HERE, case)
        os.makedirs(d, exist_ok=True)
        mesh.write_mesh3d(os.path.join(d, "mesh3d.d"), rm, P.iper)
        P.write_input_files(d)
        fields, diags = run_oracle(mesh.read_mesh3d(os.path.join(d, "mesh3d.d"), P.iper), P)
        np.savez_compressed(os.path.join(HERE, f"{case}_oracle.npz"), fields=fields, diags=diags)
        if a.full_deck:
            full = os.path.join(a.full_deck, case)
            os.makedirs(full, exist_ok=True)
            mesh.write_reference_inputs(full, rm, P)
            shutil.copy(os.path.join(d, "mesh3d.d"), full)
        print(case, rm.npoin, "nodes", fields.shape)


if __name__ == "__main__":
    main()
