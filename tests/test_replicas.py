"""The N-GPU path of bench.py is N independent replicas: the only exchange is the maximum of the
per-rank device times.  Checked with two gloo ranks on the CPU (127.0.0.1 rendezvous)."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, q):
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    import datetime
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench
        ms = [120.0, 150.0][rank]
        m = bench.max_over_ranks(ms, device="cpu")
        # each replica advances its own state: the oracle on its own copy of the mesh
        import numpy as np
        from oracle.oracle import Oracle
        from src_b200 import mesh
        from src_b200.cabi import F_UNK, RunParams
        rm = mesh.generate(6, L=5, seed=1).to_reference()
        o = Oracle(RunParams(delt=10.0), rm)
        o.setup()
        o.step()
        u = o.get(F_UNK)
        q.put((rank, m, bench.whole_job_rate(world, 10, m / 1000.0), float(np.sum(u * u))))
    finally:
        dist.destroy_process_group()


def test_two_replicas_take_the_max_time():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert [r[1] for r in res] == [150.0, 150.0]                 # both ranks see the slowest time
    assert res[0][2] == res[1][2] == pytest.approx(2 * 10 / 0.150)
    assert res[0][3] == res[1][3]                                 # identical independent replicas


def test_single_rank_is_identity():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.max_over_ranks(42.0) == 42.0
    assert bench.whole_job_rate(1, 10, 2.0) == 5.0


def test_reference_arm_sums_replicas():
    """`bench.py --impl reference` runs one serial oracle replica per requested host thread and
    reports their summed throughput on the workload's metric, with the core count; the config
    says that the value is modelled from components timed on a sample mesh."""
    import json
    import subprocess
    out = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "1", "--warmup", "3", "--ref-replicas", "2", "--ref-sample", "fp64_48x48x41"],
                         capture_output=True, text=True, timeout=600, check=True).stdout
    line = json.loads(out.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["cores"] == 2 and line["e2e"]["value"] == line["value"]
    assert "fp64_48x48x41" in line["config"]["cpu_sample"] and line["per_node_extrapolation"]["value"] > 0


def test_step_model_adds_the_components():
    """The per-work model: fields x MPDATA + two solves' fixed parts + iterations + diagnostics,
    scaled by the node ratio."""
    sys.path.insert(0, ROOT)
    import bench
    t = dict(mpdata_field=1.0, prfr=0.1, div=0.2, precon=0.3, laplc=0.4, iteration=0.5, diagnostics=0.6)
    assert bench.modelled_step_seconds(t, 100, 5, 4.0) == pytest.approx(4.0 * (5 + 2 * 1.1 + 50 + 0.6))


def test_bench_workloads():
    """The headline workload keeps the compact line (iprc = 2, GCR(3), N = 0.01); the stiff case
    (1024x1024x64, lowest dx/dz about 1e3, N = 0.02, GCR(5)) uses laplc's column blocks."""
    sys.path.insert(0, ROOT)
    import bench
    P = bench.build_params("fp64_512x512x81")
    assert (P.iprc, P.lord, P.strat, P.delt) == (2, 3, 0.01 ** 2 / 9.80616, 6.0)
    S = bench.build_params("stiff_1024x1024x64")
    assert (S.iprc, S.lord, S.strat) == (4, 5, 0.02 ** 2 / 9.80616)
    from src_b200 import mesh
    z = mesh.level_set(64, 20e3, stretch_dz0=bench.WORKLOAD_EXTRA["stiff_1024x1024x64"]["stretch_dz0"])
    assert 900 < (120e3 / 1024) / (z[1] - z[0]) < 1100
