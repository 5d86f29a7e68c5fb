#!/usr/bin/env python
"""Time steps of the anelastic MPDATA + GCR solver on B200 (one JSON line on rank 0).

Workload (default): the 21.2M-node plain FP64 case — 512x512 jittered columns on a doubly
periodic 120 km square, Delaunay-triangulated with median-dual cells, 81 terrain-following
levels over 20 km above a 400 m Witch-of-Agnesi hill (half-width 10 km), N = 0.01 1/s,
U = 10 m/s, anelastic reference state; dt = 6 s, MPDATA iord=2 with the nonoscillatory option,
GCR(3) to max|r|*dt <= 1e-8 with the vertical-line preconditioner, plus one passive positive
scalar (3D Gaussian, peak 1, sigma 5 km).  Synthetic, seeded inputs.

A step is one pass of mpsolver's DO ITIME loop: 5 MPDATA fields, two (gcrk + prfr) pressure
solves, the node loops and the per-step diagnostics.  `value` is steps/s over all GPUs with the
state resident in HBM; `e2e` is the same through the C ABI from pinned host state (upload,
K steps with the per-step diagnostics read back, download).  `--impl reference` times the CPU
restatement of the reference (the oracle; no Fortran compiler exists on these machines), one
serial replica per host thread, throughput summed.

Multi-GPU: the path does not shard (a single mesh per GPU), so N GPUs run N independent
replicas; the timed region is bracketed by barriers and the max over ranks is taken.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "steps/s & ms/pressure-solve: learned+mixed vs plain FP64 GCR, 1 B200, resid≤1e-8"
WORKLOADS = {
    # name: (nx, levels, dt, h0, lord, nscal)
    "fp64_512x512x81": (512, 81, 6.0, 400.0, 3, 1),
    "fp64_48x48x41": (48, 41, 10.0, 400.0, 3, 0),
    "fp64_256x256x81": (256, 81, 6.0, 400.0, 3, 1),
}
# the stiff large case: levels stretched so the lowest aspect ratio dx/dz is about 1e3 (dx = 117 m,
# lowest dz = 0.117 m), N = 0.02 1/s, GCR(5).  The compact vertical line stalls on such cells, so
# its plain method uses laplc's column blocks (iprc = 4).  Run on request only (--workload).
WORKLOADS["stiff_1024x1024x64"] = (1024, 64, 6.0, 800.0, 5, 0)
WORKLOAD_EXTRA = {"stiff_1024x1024x64": dict(stretch_dz0=0.117, N=0.02, iprc=4)}
DEFAULT = "fp64_512x512x81"
CPU_SAMPLE = "fp64_48x48x41"
L2_BYTES = 126 * 2 ** 20


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("LOCAL_RANK", 0)), int(os.environ.get("WORLD_SIZE", 1))


def max_over_ranks(x, device="cuda"):
    """The largest of a per-rank value over all ranks (the value itself on one rank).  The N-GPU
    run is N independent replicas, so this maximum of the device times is the only exchange."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(world, steps, seconds):
    """Steps per second of the whole job: every replica runs `steps` steps in at most `seconds`."""
    return world * steps / seconds


def build_params(name, precision=0):
    from src_b200.cabi import RunParams
    nx, L, dt, h0, lord, nscal = WORKLOADS[name]
    ex = WORKLOAD_EXTRA.get(name, {})
    return RunParams(delt=dt, lord=lord, nscal=nscal, eps0=1e-8, itr=200, iprc=ex.get("iprc", 2), itrp1=1,
                     lipps=1, strat=ex.get("N", 0.01) ** 2 / 9.80616, precision=precision)


def build_mesh(name):
    from src_b200 import mesh
    nx, L, dt, h0, lord, nscal = WORKLOADS[name]
    cm = mesh.generate(nx, L=L, seed=0, h0=h0, stretch_dz0=WORKLOAD_EXTRA.get(name, {}).get("stretch_dz0"))
    return cm, cm.to_reference()


def gaussian_scalar(rm):
    x, y, z = rm.coord[:, 0], rm.coord[:, 1], rm.coord[:, 2]
    return np.exp(-((x - 30e3) ** 2 + (y - 60e3) ** 2 + (z - 5e3) ** 2) / (2 * 5e3 ** 2))


def algorithmic_bytes(cls, N, Eh, Ev):
    """FP64 bytes each launch must move: every distinct array element read once, written once.

    N nodes, Eh horizontal faces (2D edges x levels), Ev vertical faces; a face vector is 3
    doubles.  The per-column adjacency lists (a few ints per column) are not counted."""
    E = Eh + Ev
    table = {
        "lap_grad": 56 * N + 24 * E,      # p, vol, rh0, coefw in; S; Fx, Fy, Fz out
        "lap_div": 48 * N + 24 * E,       # Fx, Fy, Fz, vol, rh0 in; S; alap out
        "laplc": 40 * N + 24 * E,         # both halves in one launch: p, vol, rh0, coefw in; S; alap out
        "prfr": 72 * N + 24 * E,          # p, u*, v*, w*, vol, coefw in; S; u, v, w out
        "div": 48 * N + 24 * E,           # u, v, w, vol, rh0 in; S; rhs out
        "line_solve": 40 * N,             # rhs, a, m, c' in; p out
        "aun": 24 * N + 32 * E,           # uuu in; S in; aun out
        "mp_donor": 32 * N + 8 * E,       # psi, vol, rh0 in; aun; psi1 out
        "mp_grad_bounds": 48 * N + 24 * E,  # psi1 in; S; 3 gradients, max, min out
        "mp_anti": 72 * N + 16 * E,       # psi1, grad x3, vol, rh0, uuu x3; aun in, A out
        "mp_cpcn": 56 * N + 8 * E,        # A; psi1, mx, mn, vol, rh0 in; cp, cn out
        "mp_pass2": 48 * N + 8 * E,       # A; psi1, cp, cn, vol, rh0 in; psi out
        "courant": 40 * N + 24 * E,       # uuu, rh0, vol in; S; cour out
    }
    return table.get(cls)


def rule_bytes(cls, N, Eh, Ev, b=8):
    """Algorithmic bytes per launch by the workload's counting rule for the reference's
    operators, b bytes per value: a gradient G or divergence D moves (8+3b)E + 6bN, laplc G + D, prfr
    (8+3b)E + 9bN, the line solve 5bN.  The 8 bytes per face are the reference's two int32 edge
    indices, which the column layout does not read (it derives neighbours from a per-column
    adjacency list), so for the edge kernels these bytes exceed what the kernel must move;
    `algorithmic_bytes` gives the latter."""
    E = Eh + Ev
    table = {
        "lap_grad": (8 + 3 * b) * E + 6 * b * N,
        "lap_div": (8 + 3 * b) * E + 6 * b * N,
        "laplc": 2 * ((8 + 3 * b) * E + 6 * b * N),     # laplc = G + D
        "div": (8 + 3 * b) * E + 6 * b * N,
        "prfr": (8 + 3 * b) * E + 9 * b * N,
        "line_solve": 5 * b * N,
    }
    return table.get(cls)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        try:
            os.remove(self.path)
        except OSError:
            pass
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": reasons,
                "samples": len(rows)}


def learned_weights(name, rm, device):
    """Weights of the learned preconditioner: the committed training run when present (trained by
    `python -m src_b200.learned` on the 256x256x81 family), else a short training on this
    workload's own plain solves (untimed).  Returns (params, description)."""
    from src_b200 import learned
    if os.path.exists(learned.WEIGHTS):
        w, _ = learned.load_weights()
        return w, os.path.relpath(learned.WEIGHTS, ROOT)
    w, hist, rate = learned.train(rm, build_params(name), steps=3, every=4, max_records=48, epochs=2,
                                  device=device)
    return w, "trained here on 3 plain steps of this workload"


def network_ms(P, rm, weights, device):
    """Device time of one application of the learned correction (network kernels only; the line
    solve it corrects is part of every plain iteration too), on this workload's mesh."""
    from src_b200.api import Solver
    from src_b200.cabi import F_WORK
    P = build_params_copy(P, iprc=3)
    with Solver(P, rm, device=device) as s:
        s.learned_set_params(weights)
        s.set(F_WORK, np.random.default_rng(0).standard_normal(rm.npoin))
        s.learned_forward(F_WORK, F_WORK + 1)
        s.synchronize()
        s.kernel_timing(True)
        for _ in range(3):
            s.learned_forward(F_WORK, F_WORK + 1)
        s.synchronize()
        n, ms = s.kernel_times().get("learned", (1, 0.0))
        s.kernel_timing(False)
    return ms / max(n, 1)


def build_params_copy(P, **kw):
    from src_b200.cabi import RunParams
    return RunParams(**{**P.__dict__, **kw})


CPU_WORK_SAMPLE = "fp64_256x256x81"
# GCR iterations per time step (the two pressure solves together) of a workload, as measured by
# the FP64 GPU path of this bench, which runs the oracle's algorithm step for step (bit for bit
# with the oracle replaying the GPU's summation order).  The CPU legs use it to turn per-iteration
# costs into a per-step cost, because a single full-size step of the serial restatement takes
# about 25 minutes (5 MPDATA fields and ~240 GCR iterations over 21.2M nodes).  The b200 arm's
# cpu_baseline uses the count its own run measured instead.
GCR_ITERS_PER_STEP = {"fp64_512x512x81": 226.4, "fp64_256x256x81": 165.0, "fp64_48x48x41": 130.0}


def cpu_sample(steps, warmup):
    """Oracle (CPU restatement, 1 thread) full steps of the 48x48x41 workload: seconds per step and
    the sample's node count (the per-node extrapolation)."""
    from oracle.oracle import Oracle
    cm, rm = build_mesh(CPU_SAMPLE)
    o = Oracle(build_params(CPU_SAMPLE), rm)
    o.setup()
    for _ in range(warmup):
        o.step()
    t0 = time.perf_counter()
    for _ in range(steps):
        o.step()
    dt = (time.perf_counter() - t0) / steps
    return dt, rm.npoin


def work_oracle(sample):
    """An oracle on the sample workload whose GCR solves stop after one restart cycle (itr = 1),
    set up, for timing the components of a step.  Returns (oracle, reference mesh)."""
    from oracle.oracle import Oracle
    from src_b200.cabi import F_UNK
    cm, rm = build_mesh(sample)
    P = build_params(sample)
    P.itr = 1
    o = Oracle(P, rm)
    o.setup()
    if P.nscal:
        o.set(F_UNK + 4, gaussian_scalar(rm))
    return o, rm


def work_sample(o):
    """Seconds of one call of each component of a time step, on the oracle's mesh:
    one MPDATA field, prfr, div(-1), the line preconditioner, laplc, a gcrk capped at one restart
    cycle (from which the cost of one GCR iteration follows) and the per-step diagnostics."""
    from src_b200.cabi import F_PRPOT, F_UNK, F_UNK1
    T = time.perf_counter
    t = {}
    a = T(); o.mpdatamper(o.get(F_UNK + 1), 2); t["mpdata_field"] = T() - a
    p, u = o.get(F_PRPOT), [o.get(F_UNK1 + k) for k in range(3)]
    a = T(); uo = o.prfr(p, *u, 1); t["prfr"] = T() - a
    a = T(); r, _ = o.div(*uo, -1); t["div"] = T() - a
    a = T(); q = o.precon(r, 2, 1); t["precon"] = T() - a
    a = T(); o.laplc(q, 1); t["laplc"] = T() - a
    a = T(); _, _, st = o.gcrk(p, *u, 1); t["gcrk_capped"] = T() - a
    t["gcrk_capped_iterations"] = int(st.niter)
    t["iteration"] = max(t["gcrk_capped"] - t["prfr"] - t["div"] - t["precon"] - t["laplc"], 0.0) / max(st.niter, 1)
    a = T(); o.div(*uo, 1); o.courant(1); o.stats(); t["diagnostics"] = T() - a
    return t


def modelled_step_seconds(t, iters_per_step, nfields, scale):
    """Seconds of one full time step from component times `t` (work_sample) measured on a mesh
    `scale` times smaller: nfields MPDATA fields; two pressure solves, each prfr + div + precon +
    laplc before its iterations and the caller's prfr after it; iters_per_step GCR iterations; the
    diagnostics.  Every component is a fixed number of passes over the nodes, so its cost scales
    with the node count once the fields exceed the CPU caches (the 256x256x81 sample holds 42 MB
    per field)."""
    solve_fixed = t["prfr"] + t["div"] + t["precon"] + t["laplc"] + t["prfr"]
    return scale * (nfields * t["mpdata_field"] + 2 * solve_fixed + iters_per_step * t["iteration"] +
                    t["diagnostics"])


_BARRIER = None


def _replica_init(barrier):
    global _BARRIER
    _BARRIER = barrier


def _replica_sample(args):
    """One serial oracle replica: real steps of the 48x48x41 mesh (the per-node extrapolation),
    then component samples of the sample workload (the per-work model); every replica waits for
    the others before each timed part."""
    steps, warmup, sample = args
    from oracle.oracle import Oracle
    cm, rm = build_mesh(CPU_SAMPLE)
    o = Oracle(build_params(CPU_SAMPLE), rm)
    o.setup()
    o.step()
    _BARRIER.wait()
    t0 = time.perf_counter()
    for _ in range(2):
        o.step()
    per_node = ((time.perf_counter() - t0) / 2, rm.npoin)
    del o
    ow, rmw = work_oracle(sample)
    for _ in range(warmup):
        work_sample(ow)
    _BARRIER.wait()
    samples = [work_sample(ow) for _ in range(steps)]
    return per_node, samples, rmw.npoin


REF_MAX_REPLICAS = 64          # bounds the reference arm's memory
REF_REPLICA_BYTES = 4 << 30    # one replica: the 256x256x81 sample oracle (~2.8 GB) and its mesh


def host_threads():
    """Host threads this process may use: its CPU affinity, lowered to a cgroup CPU quota."""
    try:
        n = len(os.sched_getaffinity(0))
    except AttributeError:
        n = os.cpu_count() or 1
    for path in ("/sys/fs/cgroup/cpu.max", "/sys/fs/cgroup/cpu/cpu.cfs_quota_us"):
        try:
            f = open(path).read().split()
            if path.endswith("cpu.max") and f[0] != "max":
                n = min(n, max(1, int(int(f[0]) / int(f[1]))))
            elif path.endswith("quota_us") and int(f[0]) > 0:
                period = int(open("/sys/fs/cgroup/cpu/cpu.cfs_period_us").read())
                n = min(n, max(1, int(f[0]) // period))
        except (OSError, ValueError, IndexError):
            pass
    return n


def reference_replicas(requested=0):
    """Replicas for the reference arm: one per usable host thread (or as requested), at most
    REF_MAX_REPLICAS and at most what half of the available memory holds at REF_REPLICA_BYTES each."""
    n = host_threads() if requested <= 0 else min(requested, host_threads())
    try:
        for ln in open("/proc/meminfo"):
            if ln.startswith("MemAvailable:"):
                n = min(n, max(1, int(ln.split()[1]) * 1024 // 2 // REF_REPLICA_BYTES))
    except OSError:
        pass
    return max(1, min(n, REF_MAX_REPLICAS))


def run_reference(args):
    """The reference's path on the host cores.  The reference is serial Fortran (no compiler for
    it here), so its restatement runs as one independent replica per usable host thread (at most
    REF_MAX_REPLICAS, and as many as memory allows), started together in spawned processes, and
    the throughput of all replicas is summed.

    A full step of the 21.2M-node workload takes the serial restatement about 25 minutes, so each
    replica times the components of a step on a sample mesh instead (work_sample: one MPDATA field,
    one GCR iteration, the fixed parts of a solve, the diagnostics) and `value` is the step they
    add up to at full size (modelled_step_seconds) with the workload's GCR iteration count.  The
    per-node extrapolation of real 48x48x41 steps, which needs half as many iterations per solve
    and keeps its fields in cache, is reported beside it."""
    rank, _, world = dist_env()
    if rank != 0:
        return
    import multiprocessing as mp
    name, sample = DEFAULT, args.ref_sample
    nx, L = WORKLOADS[name][0], WORKLOADS[name][1]
    n_work = nx * nx * L
    nfields = 4 + WORKLOADS[name][5]
    iters = GCR_ITERS_PER_STEP[name]
    nrep = reference_replicas(args.ref_replicas)
    ctx = mp.get_context("spawn")
    barrier = ctx.Barrier(nrep)
    with ctx.Pool(nrep, initializer=_replica_init, initargs=(barrier,)) as pool:
        res = pool.map(_replica_sample, [(args.steps, args.warmup, sample)] * nrep)
    per_node = sum(n / sec for (sec, n), _, _ in res) / n_work
    step_s = []                      # modelled full-size step time of each replica, per sample step
    for _, samples, n_s in res:
        step_s.append([modelled_step_seconds(t, iters, nfields, n_work / n_s) for t in samples])
    value = sum(1.0 / float(np.mean(x)) for x in step_s)
    t0 = {k: float(np.median([s[k] for _, ss, _ in res for s in ss])) for k in res[0][1][0]}
    n_s = res[0][2]
    sample_txt = (f"{nrep} concurrent serial oracle replicas; each timed {args.steps} samples (after {args.warmup} "
                  f"untimed) of the components of one step on the {sample} mesh ({n_s} nodes, GCR solves capped "
                  f"at one restart cycle): median s per call mpdata_field {t0['mpdata_field']:.3f}, prfr "
                  f"{t0['prfr']:.3f}, div {t0['div']:.3f}, precon {t0['precon']:.3f}, laplc {t0['laplc']:.3f}, "
                  f"GCR iteration {t0['iteration']:.3f}, diagnostics {t0['diagnostics']:.3f}; a step of the "
                  f"{n_work}-node workload = {nfields} fields + 2 solves of {iters:g} GCR iterations in all, "
                  f"scaled by nodes x{n_work / n_s:.2f}: {float(np.mean(step_s[0])):.0f} s per replica")
    cfg = workload_config(name)
    cfg["cpu_sample"] = (f"components of a step timed on the {sample} mesh and modelled at full size "
                         f"({iters:g} GCR iterations per step, the count the FP64 GPU path measures on this "
                         f"workload); not a run of the full workload")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 / value,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": "steps/s", "cores": nrep, "kind": "port", "sample": sample_txt},
            "per_node_extrapolation": {
                "value": per_node, "unit": "steps/s",
                "sample": f"{nrep} replicas x 2 real steps of the 48x48x41 mesh ({res[0][0][1]} nodes, "
                          f"about half the GCR iterations per solve), node-steps/s summed and divided by {n_work}"},
            "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def workload_config(name, iprc=None):
    nx, L, dt, h0, lord, nscal = WORKLOADS[name]
    if iprc is None:
        iprc = WORKLOAD_EXTRA.get(name, {}).get("iprc", 2)
    return {"workload": f"plain FP64 MPDATA+GCR step, {nx}x{nx} jittered periodic columns x {L} levels "
                        f"({nx * nx * L} nodes), Agnesi hill h0={h0:g} m, dt={dt:g} s",
            "nodes": nx * nx * L, "edges": 3 * nx * nx * L + nx * nx * (L - 1), "levels": L, "dt_s": dt,
            "gcr": f"GCR({lord}) to max|r|*dt<=1e-8, " + (
                "laplc's column blocks as the line preconditioner" if iprc == 4
                else "vertical-line preconditioner" if iprc == 2 else f"preconditioner iprc={iprc}"),
            **({"levels_stretched_lowest_dz_m": WORKLOAD_EXTRA[name]["stretch_dz0"],
                "N_per_s": WORKLOAD_EXTRA[name]["N"]} if name in WORKLOAD_EXTRA else {}),
            "mpdata": "iord=2 + nonoscillatory (FCT)", "passive_scalars": nscal,
            "l2": "inputs larger than L2 (each FP64 node field is 8*nodes bytes > 126 MB)"}


def report_mixed_errors(args):
    """The mixed-precision path against the FP64 path on the same workload, run side by side for
    max(--error-steps) steps: relative L2 of u, v, w, theta' and pi' (prpot) at each requested
    step, the GCR iterations of both, and the passive scalar's minimum, maximum and mass on the
    FP64 path (sign, bounds and conservation).  The FP64 path agrees bit for bit with the oracle
    replaying the GPU's summation order, so it stands for the FP64 oracle at a size the CPU
    restatement cannot run in reasonable time.  Prints one JSON object."""
    from src_b200.api import Solver
    from src_b200.cabi import F_PRPOT, F_UNK
    name = args.workload
    want = sorted({int(x) for x in args.error_steps.split(",") if x.strip()})
    cm, rm = build_mesh(name)
    runs = {}
    for tag, prec in (("fp64", 0), ("mixed", 1)):
        s = Solver(build_params(name, precision=prec), rm, device=0)
        s.setup()
        if s.params.nscal:
            s.set(F_UNK + 4, gaussian_scalar(rm))
        runs[tag] = s
    s64, smx = runs["fp64"], runs["mixed"]
    m0 = s64.stats().mass[4] if s64.params.nscal else None
    rows = []
    for step in range(1, want[-1] + 1):
        d64, dmx = s64.step(), smx.step()
        if step in want:
            err = {}
            for k, nm in enumerate(("u", "v", "w", "theta")):
                a, b = smx.get(F_UNK + k), s64.get(F_UNK + k)
                err[nm] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            a, b = smx.get(F_PRPOT), s64.get(F_PRPOT)
            a, b = a - a.mean(), b - b.mean()          # pi' up to the constant of the periodic solve
            err["pi"] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            row = {"step": step, "rel_l2_mixed_vs_fp64": err,
                   "gcr_iters_fp64": [d64.niter1, d64.niter], "gcr_iters_mixed": [dmx.niter1, dmx.niter],
                   "divmx_fp64": d64.divmx, "divmx_mixed": dmx.divmx}
            if m0 is not None:
                row.update({"scalar_min_fp64": d64.smin[0], "scalar_max_fp64": d64.smax[0],
                            "scalar_mass_rel_change_fp64": (d64.mass[4] - m0) / m0,
                            "scalar_min_mixed": dmx.smin[0], "scalar_mass_rel_change_mixed": (dmx.mass[4] - m0) / m0})
            rows.append(row)
            print(json.dumps(row), file=sys.stderr, flush=True)
    for s in runs.values():
        s.close()
    print(json.dumps({"report": "mixed_vs_fp64", "config": workload_config(name), "rows": rows}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--ref-replicas", type=int, default=0,
                    help="--impl reference: oracle replicas (default: one per host thread)")
    ap.add_argument("--ref-sample", default=CPU_WORK_SAMPLE, choices=sorted(WORKLOADS),
                    help="--impl reference and the CPU baseline: mesh on which the step's components are timed")
    ap.add_argument("--workload", default=DEFAULT, choices=sorted(WORKLOADS))
    ap.add_argument("--iprc", type=int, default=None, choices=[1, 2, 4],
                    help="preconditioner of the plain path (default: the workload's own)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-variants", action="store_true", help="skip the mixed-precision variant")
    ap.add_argument("--error-steps", default="",
                    help="report mode: mixed vs FP64 errors at these steps (e.g. 1,50,200) instead of timing")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
        return
    if args.error_steps:
        report_mixed_errors(args)
        return

    import torch
    rank, local, world = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    from src_b200.api import Solver
    from src_b200.cabi import F_UNK, F_UUU, F_UUU0, F_FRC, F_UNKDASH, F_PRPOT, MpgDiag

    name = args.workload
    cm, rm = build_mesh(name)
    P = build_params(name)
    if args.iprc is not None:
        P.iprc = args.iprc
    s = Solver(P, rm, device=local)
    info = s.info()
    d0 = s.setup()
    if P.nscal:
        s.set(F_UNK + 4, gaussian_scalar(rm))
    stream = torch.cuda.ExternalStream(s.stream())
    for _ in range(args.warmup):
        s.step()
    s.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()

    # ---------------- timed region: K steps, state resident in HBM
    sampler = ClockSampler(local)
    barrier()
    torch.cuda.synchronize()
    s.kernel_timing(True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler.start()
    torch.cuda.nvtx.range_push("timed_steps")       # lets a profiler capture just this region
    e0.record(stream)
    iters, diags = [], []
    for _ in range(args.steps):
        d = s.step()
        iters.append((d.niter1, d.niter))
        diags.append(d)
    e1.record(stream)
    torch.cuda.nvtx.range_pop()
    e1.synchronize()
    clocks = sampler.stop()
    torch.cuda.synchronize()
    barrier()
    ms = e0.elapsed_time(e1)
    kt = s.kernel_times()
    s.kernel_timing(False)
    ref_fields = None
    if not args.no_variants:
        ref_fields = {k: s.get(F_UNK + k) for k in range(4)}
        ref_fields["pi"] = s.get(F_PRPOT) - s.get(F_PRPOT).mean()
    rates = [d.rate1 for d in diags if d.rate1 > 0]
    plain_rate = float(np.exp(np.mean(np.log(rates)))) if rates else 0.0
    ms_max = max_over_ranks(ms)
    value = whole_job_rate(world, args.steps, ms_max / 1000.0)

    # ---------------- per-kernel roofline
    N, L, NC, NE2 = info["npoin"], info["nlev"], info["ncol"], info["nedge2d"]
    Eh, Ev = NE2 * L, NC * (L - 1)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    kernels = {}
    for cls, (nl, tot) in kt.items():
        ent = {"launches": nl, "total_ms": round(tot, 3), "avg_us": round(1000 * tot / nl, 2)}
        ab = algorithmic_bytes(cls, N, Eh, Ev)
        if ab:
            gbs = ab / (tot / nl / 1000.0) / 1e9
            ent.update({"bytes_per_launch": ab, "gbs": round(gbs, 1), "frac": round(gbs / hbm, 3)})
        rb = rule_bytes(cls, N, Eh, Ev)
        if rb:
            gr = rb / (tot / nl / 1000.0) / 1e9
            ent.update({"rule_bytes_per_launch": rb, "rule_gbs": round(gr, 1), "rule_frac": round(gr / hbm, 3)})
        kernels[cls] = ent
    real = {k: v for k, v in kernels.items() if k != "pressure_solve"}
    dom = max((k for k in real if "gbs" in real[k]), key=lambda k: real[k]["total_ms"])
    launches = int(sum(v["launches"] for v in real.values()))
    solve = kernels.get("pressure_solve", {"launches": 0, "total_ms": 0.0})
    ms_solve = solve["total_ms"] / max(solve["launches"], 1)
    # achieved/frac by the counting rule of the reference's operators (edge indices included);
    # *_own: by the bytes the column layout must move (no edge index arrays), a stricter figure
    rd = real[dom].get("rule_gbs", real[dom]["gbs"])
    roof = {"kernel": dom, "bound": "hbm", "achieved": rd, "peak": hbm, "unit": "GB/s",
            "frac": round(rd / hbm, 3), "peak_source": peak_src, "traffic": None,
            "bytes_per_launch": real[dom].get("rule_bytes_per_launch", real[dom]["bytes_per_launch"]),
            "achieved_own": real[dom]["gbs"], "frac_own": real[dom]["frac"],
            "own_bytes_per_launch": real[dom]["bytes_per_launch"]}
    tr_path = os.path.join(ROOT, "profiles", "traffic.txt")     # ncu figures, see that file
    if os.path.exists(tr_path):
        for ln in open(tr_path):
            f = ln.split()
            if len(f) == 3 and not ln.startswith("#") and f[0] == name and f[1] == dom:
                roof["traffic"] = int(f[2])
                roof["traffic_source"] = "ncu dram bytes of the 256x256x81 case scaled by units" \
                    if name != "fp64_256x256x81" else "ncu dram bytes"

    # ---------------- end to end through the C ABI from pinned host state
    e2e = None
    if not args.no_e2e:
        fids = [F_UNK + k for k in range(4 + P.nscal)] + [F_UUU + k for k in range(3)] + \
               [F_UUU0 + k for k in range(3)] + [F_FRC + k for k in range(4)] + \
               [F_UNKDASH + k for k in range(3)] + [F_PRPOT]
        host = {f: torch.empty(rm.npoin, dtype=torch.float64, pin_memory=True).numpy() for f in fids}
        for f in fids:
            host[f][:] = s.get(f)
        barrier()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for f in fids:
            s.set(f, host[f])
        for _ in range(args.steps):
            s.step()
        for f in fids:
            s.get(f, out=host[f])
        t1 = time.perf_counter()
        sec = max_over_ranks(t1 - t0)
        state = len(fids) * 8 * rm.npoin
        import ctypes
        e2e = {"value": whole_job_rate(world, args.steps, sec), "unit": "steps/s",
               "h2d_bytes_per_step": state // args.steps,
               "d2h_bytes_per_step": (state + args.steps * ctypes.sizeof(MpgDiag)) // args.steps,
               "path": "mpg_set_field x%d from pinned host arrays, %d x mpg_step (per-step diagnostics "
                       "read back), mpg_get_field x%d into the same pinned arrays" % (len(fids), args.steps, len(fids))}

    s.close()

    # ---------------- variants on the same workload (reported beside the headline FP64 path)
    variants = {}
    if not args.no_variants:
        base = P.iprc
        plan = (("mixed", 1, 2), ("learned_mixed", 1, 3)) if base == 2 else (("mixed", 1, base),)
        for vname, prec, iprc in plan:
            Pv = build_params(name, precision=prec)
            Pv.iprc = iprc
            weights_src = None
            if iprc == 3:
                # The network is kept while it contracts the residual at least as fast per unit
                # of time as the plain preconditioner: per iteration it must beat the plain
                # solves' contraction on this workload raised to the cost of a learned iteration
                # in plain iterations (one network application timed here, the plain iteration
                # from the mixed-precision run above).
                weights, weights_src = learned_weights(name, rm, local)
                t_nn = network_ms(build_params(name, precision=prec), rm, weights, local)
                mv = variants.get("mixed")
                t_iter = mv["ms_per_pressure_solve"] / max(mv["gcr_iters_per_solve"], 1.0) if mv else t_nn
                cost = 1.0 + t_nn / max(t_iter, 1e-9)
                Pv.nn_rate = plain_rate ** cost
            sv = Solver(Pv, rm, device=local)
            if iprc == 3:
                sv.learned_set_params(weights)
            sv.setup()
            if Pv.nscal:
                sv.set(F_UNK + 4, gaussian_scalar(rm))
            for _ in range(args.warmup):
                sv.step()
            sv.synchronize()
            stream_v = torch.cuda.ExternalStream(sv.stream())
            barrier()
            torch.cuda.synchronize()
            sv.kernel_timing(True)
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream_v)
            vit, vfb, vrate = [], 0, []
            for _ in range(args.steps):
                dv = sv.step()
                vit.append((dv.niter1, dv.niter))
                vfb += dv.fallbacks
                vrate.append(dv.rate1)
            a1.record(stream_v)
            a1.synchronize()
            barrier()
            vms = max_over_ranks(a0.elapsed_time(a1))
            vkt = sv.kernel_times()
            vsolve = vkt.get("pressure_solve", (1, 0.0))
            err = {}
            for k, nm in enumerate(("u", "v", "w", "theta")):
                a, b = sv.get(F_UNK + k), ref_fields[k]
                err[nm] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
            a = sv.get(F_PRPOT)
            err["pi"] = float(np.linalg.norm(a - a.mean() - ref_fields["pi"]) / max(np.linalg.norm(ref_fields["pi"]), 1e-300))
            variants[vname] = {
                "value": whole_job_rate(world, args.steps, vms / 1000.0), "unit": "steps/s",
                "ms_per_step": vms / args.steps,
                "ms_per_pressure_solve": round(vsolve[1] / max(vsolve[0], 1), 3),
                "gcr_iters_per_solve": round(float(np.mean([a for p in vit for a in p])), 2),
                "gcr_iters_first_solve": round(float(np.mean([p[0] for p in vit])), 2),
                "gcr_rate_first_solve": round(float(np.exp(np.mean(np.log([x for x in vrate if x > 0] or [1.0])))), 5),
                "speedup_vs_fp64": round(whole_job_rate(world, args.steps, vms / 1000.0) / value, 3),
                "rel_l2_vs_fp64": err,
                "kernels_ms": {k: round(v[1], 2) for k, v in vkt.items()},
                "precision": "FP32 face vectors, MPDATA fluxes, GCR directions and operator; "
                             "FP64 p, r, inner products, coefficients, stopping test, Thomas solves, mass sums"}
            if iprc == 3:
                variants[vname].update({"fallbacks": vfb, "nn_rate": Pv.nn_rate, "weights": weights_src,
                                        "ms_per_network_application": round(t_nn, 3),
                                        "learned_iteration_cost_in_plain_iterations": round(cost, 2),
                                        "network": "3 message-passing layers x 32 channels, BF16 tcgen05 "
                                                   "forward, corrects the vertical-line preconditioner"})
            sv.close()

        # the learned correction on a hill it was not trained on: the 256x256x81 family's held-out
        # seed, plain mixed vs learned + mixed with the committed weights (fallback threshold = the
        # training run's plain contraction, so the network is kept while it contracts faster per
        # iteration); guarded like the variants below
        if base == 2:
            try:
                from src_b200 import learned, mesh as _mesh
                from src_b200.cabi import RunParams
                w_h, rate_h = learned.load_weights()
                sd = learned.HELDOUT_SEED
                rm_h = _mesh.generate(256, L=81, seed=sd, h0=learned.seed_h0(sd)).to_reference()
                P_h = RunParams(delt=6.0, lord=3, eps0=1e-8, itr=200, itrp1=1, lipps=1, strat=0.01 ** 2 / 9.80616,
                                nn_rate=rate_h, precision=1)
                res = learned.compare(rm_h, P_h, w_h, steps=3, warm=1, device=local)
                variants["learned_heldout_256x256x81"] = {
                    "mesh": f"256x256x81, seed {sd} (not trained on), h0 = {learned.seed_h0(sd):.1f} m",
                    "precision": "mixed, both paths",
                    "first_solve_iters_plain": res["plain"]["first_solve_iters"],
                    "first_solve_iters_learned": res["learned"]["first_solve_iters"],
                    "ms_per_step_plain": round(res["plain"]["ms_per_step"], 2),
                    "ms_per_step_learned": round(res["learned"]["ms_per_step"], 2),
                    "fallbacks": res["learned"]["fallbacks"], "nn_rate": rate_h,
                    "timing": "host wall clock around 3 synchronised steps after 1 warm-up"}
            except Exception as exc:                      # reported, not fatal
                variants["learned_heldout_256x256x81"] = {"error": f"{type(exc).__name__}: {exc}"[:300]}

        # laplc's own column blocks as the line preconditioner (iprc = 4), FP64 and mixed.  Run
        # last and guarded: a failure here is reported in the line instead of ending the run.
        for vname, prec in ((("column_blocks_fp64", 0), ("column_blocks_mixed", 1)) if base == 2 else ()):
            try:
                Pv = build_params(name, precision=prec)
                Pv.iprc = 4
                sv = Solver(Pv, rm, device=local)
                try:
                    sv.setup()
                    if Pv.nscal:
                        sv.set(F_UNK + 4, gaussian_scalar(rm))
                    for _ in range(args.warmup):
                        sv.step()
                    sv.synchronize()
                    stream_v = torch.cuda.ExternalStream(sv.stream())
                    barrier()
                    torch.cuda.synchronize()
                    sv.kernel_timing(True)
                    a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a0.record(stream_v)
                    vit = []
                    for _ in range(args.steps):
                        dv = sv.step()
                        vit.append((dv.niter1, dv.niter))
                    a1.record(stream_v)
                    a1.synchronize()
                    barrier()
                    vms = max_over_ranks(a0.elapsed_time(a1))
                    vkt = sv.kernel_times()
                    vsolve = vkt.get("pressure_solve", (1, 0.0))
                    err = {}
                    for k, nm in enumerate(("u", "v", "w", "theta")):
                        a, b = sv.get(F_UNK + k), ref_fields[k]
                        err[nm] = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
                    a = sv.get(F_PRPOT)
                    err["pi"] = float(np.linalg.norm(a - a.mean() - ref_fields["pi"]) /
                                      max(np.linalg.norm(ref_fields["pi"]), 1e-300))
                    vval = whole_job_rate(world, args.steps, vms / 1000.0)
                    variants[vname] = {
                        "value": vval, "unit": "steps/s", "ms_per_step": vms / args.steps,
                        "ms_per_pressure_solve": round(vsolve[1] / max(vsolve[0], 1), 3),
                        "gcr_iters_per_solve": round(float(np.mean([a for p in vit for a in p])), 2),
                        "gcr_iters_first_solve": round(float(np.mean([p[0] for p in vit])), 2),
                        "speedup_vs_fp64": round(vval / value, 3),
                        "rel_l2_vs_fp64": err,
                        "kernels_ms": {k: round(v[1], 2) for k, v in vkt.items()},
                        "preconditioner": "laplc's column blocks (tridiagonal on even and odd levels), "
                                          "stride-2 Thomas in FP64",
                        "precision": "FP64" if prec == 0 else
                                     "FP32 face vectors, MPDATA fluxes, GCR directions and operator; "
                                     "FP64 p, r, inner products, coefficients, stopping test, Thomas solves"}
                finally:
                    sv.close()
            except Exception as exc:                      # reported, not fatal
                variants[vname] = {"error": f"{type(exc).__name__}: {exc}"[:300]}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # per-work model: components of a step timed on the sample mesh (1 thread), combined with
        # this run's own GCR iteration count and field count at the workload's node count
        ow, rmw = work_oracle(args.ref_sample)
        work_sample(ow)                                   # untimed: first touch of the arrays
        t = work_sample(ow)
        del ow
        iters_step = float(np.mean([a + b for a, b in iters]))
        nfields = 4 + P.nscal
        step_s = modelled_step_seconds(t, iters_step, nfields, N / rmw.npoin)
        sec, n_sample = cpu_sample(2, 1)
        cpu = {"value": 1.0 / step_s, "unit": "steps/s", "cores": 1, "kind": "port",
               "sample": f"oracle components of one step timed once on the {args.ref_sample} mesh ({rmw.npoin} "
                         f"nodes): mpdata_field {t['mpdata_field']:.3f} s, GCR iteration {t['iteration']:.3f} s, "
                         f"prfr {t['prfr']:.3f}, div {t['div']:.3f}, precon {t['precon']:.3f}, laplc "
                         f"{t['laplc']:.3f}, diagnostics {t['diagnostics']:.3f}; modelled at {N} nodes with this "
                         f"run's {iters_step:.1f} GCR iterations per step and {nfields} fields: {step_s:.0f} s/step",
               "per_node_extrapolation": {
                   "value": (1.0 / sec) * n_sample / N, "unit": "steps/s",
                   "sample": f"2 oracle steps of the 48x48x41 mesh ({n_sample} nodes, dt=10 s), {sec:.3f} s/step, "
                             f"per-node cost scaled to {N} nodes"}}

    if rank == 0:
        last = diags[-1]
        line = {"metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": workload_config(name, P.iprc),
                "ms_per_pressure_solve": round(ms_solve, 3),
                "gcr_iters_per_solve": round(float(np.mean([a for p in iters for a in p])), 2),
                "gcr_iters_first_solve": round(float(np.mean([p[0] for p in iters])), 2),
                "gcr_rate_first_solve": round(plain_rate, 5),
                "roofline": roof, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "kernels": kernels, "variants": variants,
                "diag_last_step": {"divmx": last.divmx, "crnmx": last.crnmx,
                                   "scalar_min": last.smin[0] if P.nscal else None,
                                   "mass_scalar": last.mass[4] if P.nscal else None},
                "setup_gcr_iters": d0.niter}
        print(json.dumps(line), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
