#!/usr/bin/env python
"""Benchmark of the GMRES + FMM Laplace BVP solve (BEM-MEL boundary-value problem).

Metric: BVP solves/s at <= 1e-8 relative error against the FP64 oracle (one step = one
complete BVP solve: set-up of geometry, octree, interaction lists, near-field quadrature and
rigid-mode diagonal, then GMRES) on the 60k-node synthetic tank (2.0 x 1.0 x 0.5 m,
h = 2/185 m, free-surface z-noise sigma = 0.2 h, p = 10, theta = 0.25, <= 30 elements per
leaf).  The FP64 oracle is the FP64 GPU solve of the same tank at relative residual 1e-12.
The solver tolerance of the timed solves is the loosest of 1e-9 .. 1e-12 at which the mixed
solve lands within half the gate; the FP64 GPU path is timed at the same tolerance, and the
line reports both paths' solves/s, their errors against the oracle and the ratio.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --batch P --workers W [--config tank_15k]   # serving mode, one GPU

Multi-GPU: independent BVPs per rank (replicas, weak scaling, no collective on the data
path); time is the max over ranks.  `--impl reference` times the reference algorithm on the
host cores: the oracle's CPU restatement of the reference path on the same tank, each step
one whole operator of a mat-vec (the compiled reference cannot hold this workload's per-pair
M2L term cache, ~400 GB); solves/s from the measured set-up and mat-vec with the reference
algorithm's iteration count (modeled, see REFERENCE_ITERATIONS).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

CONFIGS = {
    "tank_60k": dict(tank=dict(length=2.0, width=1.0, depth=0.5, h=2.0 / 185, noise=0.2, seed=1), p=10, rel_tol=1e-8),
    "tank_2800": dict(tank=dict(length=2.0, width=1.0, depth=0.5, h=0.05, noise=0.0, seed=1), p=8, rel_tol=1e-10),
    # a quarter of tank_60k (same tank, h doubled): small enough for full ncu captures
    "tank_15k": dict(tank=dict(length=2.0, width=1.0, depth=0.5, h=2.0 / 92, noise=0.2, seed=1), p=10, rel_tol=1e-8),
    # tank_60k at expansion order 12 (two 128-row tiles per tensor-core table)
    "tank_60k_p12": dict(tank=dict(length=2.0, width=1.0, depth=0.5, h=2.0 / 185, noise=0.2, seed=1), p=12, rel_tol=1e-8),
    # the large-tank size class: 10 x 4 x 1 m, ~500k points, p = 12 (a plain box, no cylinder)
    "tank_500k": dict(tank=dict(length=10.0, width=4.0, depth=1.0, h=0.0147, noise=0.2, seed=1), p=12, rel_tol=1e-8),
}
GATE = 1e-8                  # max |x - x_ref| / max |x_ref| against the FP64 oracle
ORACLE_REL_TOL = 1e-12       # relative residual of the FP64 oracle solve
TOL_LADDER = (1e-9, 1e-10, 1e-11, 1e-12)
# GMRES iterations of the unpreconditioned reference algorithm (the reference's default,
# preconditioner NONE) on each workload, by relative tolerance: the same Krylov iteration on the
# same operator, counted by the FP64 GPU path with `bench.py --count-reference-iterations`.
# They turn the CPU baseline's measured set-up and mat-vec into a (modeled) solve time.
# tank_60k at 1e-11: 713 iterations (`bench.py --count-reference-iterations --tol 1e-11`, B200);
# tank_2800 at 1e-10: 384.
REFERENCE_ITERATIONS = {"tank_60k": {1e-11: 713}, "tank_2800": {1e-10: 384}}


def reference_iterations(config, tol):
    """(iterations, how): the counted value at this tolerance, else the count at the nearest
    counted tolerance scaled by the ratio of the digits to gain (GMRES on this operator
    converges at a steady rate)."""
    tab = REFERENCE_ITERATIONS.get(config, {})
    if tol in tab:
        return tab[tol], f"counted at relative tolerance {tol:g}"
    if not tab:
        return None, "not counted"
    t0 = min(tab, key=lambda k: abs(math.log10(k) - math.log10(tol)))
    n = int(round(tab[t0] * math.log10(tol) / math.log10(t0)))
    return n, f"{tab[t0]} counted at {t0:g}, scaled by the digits to gain to {tol:g}"


def make_problem(cfg, rank):
    from bem_for_nonlinear_waves_b200 import build_dofs, known_values, make_tank, point_normals
    tk = dict(cfg["tank"])
    noise = tk.pop("noise")
    tk.pop("seed")
    t = make_tank(noise_sigma=noise * tk["h"], seed=replica_seed(cfg, rank), **tk)
    d = build_dofs(t.X, t.tri, t.face_dirichlet)
    kv = known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))
    return t, d, kv


def workload_config(name, cfg, t, n_dof):
    """The `config` object of both arms: the workload alone (no run-time choices), so the two
    lines describe the same thing."""
    return {"workload": name, "n_points": int(t.n_points), "n_faces": int(t.n_faces), "n_dof": int(n_dof), "p": cfg["p"],
            "theta": 0.25, "leaf_max": 30,
            "accuracy": f"max|x - x_ref| / max|x_ref| <= {GATE:g}; x_ref = FP64 GPU solve at relative residual {ORACLE_REL_TOL:g}",
            "inputs": "synthetic seeded tank; working set larger than L2 (near-field weights)"}


def physical_cores():
    """Physical cores among the CPUs this process may run on (distinct (package, core) ids)."""
    try:
        cpus = sorted(os.sched_getaffinity(0))
    except AttributeError:
        cpus = list(range(os.cpu_count() or 1))
    ids = set()
    for c in cpus:
        base = f"/sys/devices/system/cpu/cpu{c}/topology/"
        try:
            ids.add((open(base + "physical_package_id").read().strip(), open(base + "core_id").read().strip()))
        except OSError:
            ids.add(("?", str(c)))
    return len(ids), len(cpus)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i].lower() == "active"})
        loaded = [s for s in sm if s > 0.5 * max(sm)] if sm else []
        return {"sm_mhz": statistics.median(loaded) if loaded else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", local))
    return rank, world, local


def allreduce_max(vals, world, device="cuda"):
    """Max over ranks (the per-rank times of independent replicas)."""
    if world == 1:
        return list(vals)
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_seed(cfg, rank):
    """Each rank solves its own seeded tank of the same size (weak scaling)."""
    return cfg["tank"]["seed"] + rank


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


PORT_STAGES = ("p2m", "m2m", "m2l", "l2l", "near", "l2p")


def port_context(cfg, t, d):
    """The oracle (CPU restatement of the reference path, all host threads) set up on the whole
    tank: tree, lists and the near-field quadrature of every point, each timed whole."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    w0 = time.perf_counter()
    o = O.Oracle(t.X, t.tri, t.face_dirichlet, d, p=cfg["p"])
    setup_wall = time.perf_counter() - w0
    st = o.setup_times()
    return o, dict(st, setup_s=st["tree_lists"] + st["near_setup"], setup_wall_s=setup_wall)


def port_solve_model(setup_s, matvec_s, iters):
    """Modeled solve time of the reference algorithm from measured parts: set-up + (iterations +
    1 right-hand side + 1 rigid-mode diagonal) mat-vecs."""
    return setup_s + (iters + 2) * matvec_s


def cpu_port_baseline(args, cfg, t, d, tol):
    """Bounded CPU sample on the same tank: the oracle's whole set-up and one whole mat-vec (every
    stage over the whole problem, measured), with the reference algorithm's iteration count."""
    o, su = port_context(cfg, t, d)
    stages = {k: o.time_stage(k) for k in PORT_STAGES}
    mv = sum(stages.values())
    iters, how = reference_iterations(args.config, tol)
    res = {"matvecs_per_s": 1.0 / mv, "matvec_s": mv, "stages_s": {k: round(v, 4) for k, v in stages.items()},
           "setup_s": su["setup_s"], "threads": su["threads"], "iterations": iters, "iterations_how": how}
    if iters:
        res["solves_per_s_modeled"] = 1.0 / port_solve_model(su["setup_s"], mv, iters)
    del o
    return res


def cpu_reference_config1(args, local):
    """The compiled, unmodified reference (oracle/_ref/bem_ref_p8) solving the 2,802-point
    configuration (p = 8, relative tolerance 1e-10) on the host cores, timed by its own
    time_setup / time_solve (BEM_BVP::solve(), bem/BEM_solveBVP.hpp:618-629), next to this GPU
    path on the same tank and tolerance."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refrun
    if not refrun.available(8):
        return None
    from bem_for_nonlinear_waves_b200 import BEM_BVP
    cfg = CONFIGS["tank_2800"]
    t, d, kv = make_problem(cfg, 0)
    gpu = {}
    for prec in ("fp64", "mixed"):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=cfg["p"], solver_tol=cfg["rel_tol"], tol_relative=True,
                    solver_max_iter=4000, preconditioner=args.precond, dofs=d, device=local, precision=prec)
        b.setup()
        b.solve(kv)  # warm
        w0 = time.perf_counter()
        b.setup()
        b.solve(kv)
        gpu[prec] = {"solves_per_s": 1.0 / b.stats.time_device_s, "e2e_solves_per_s": 1.0 / (time.perf_counter() - w0),
                     "gmres_iterations": int(b.stats.iterations), "ans": b.ans.copy()}
        abs_tol = float(b.stats.tol_abs)
        del b
    phys, ncpu = physical_cores()
    w0 = time.perf_counter()
    R = refrun.run(8, t, tol=abs_tol, max_iter=4000, threads=ncpu, timeout=900)
    wall = time.perf_counter() - w0
    solve_s = R["time_setup"] + R["time_solve"]
    # the reference's DOF order -> ours
    keys = {(int(a), int(b)): i for i, (a, b) in enumerate(zip(d["dof_point"], d["dof_face"]))}
    perm = np.array([keys[(int(a), int(b))] for a, b in zip(R["dof_point"], R["dof_face"])])
    ref = np.zeros(len(perm))
    ref[perm] = R["ans"]
    out = {"value": 1.0 / solve_s, "unit": "solves/s", "cores": phys, "threads": ncpu, "kind": "reference",
           "sample": (f"one whole solve of the 2,802-point tank (h = 0.05, p = 8, relative tolerance 1e-10 = absolute "
                      f"{abs_tol:.3e}) by the compiled, unmodified reference (oracle/_ref/bem_ref_p8), timed by its own "
                      f"time_setup + time_solve; a different, smaller workload than the headline"),
           "time_setup_s": R["time_setup"], "time_solve_s": R["time_solve"], "wall_s": wall, "gmres_iterations": R["gmres_iter"],
           "gpu_same_config": {}}
    for prec, g in gpu.items():
        err = float(np.abs(g["ans"] - ref).max() / np.abs(ref).max())
        out["gpu_same_config"][prec] = {k: v for k, v in g.items() if k != "ans"}
        out["gpu_same_config"][prec].update({"max_rel_diff_vs_reference": err, "device_ratio": g["solves_per_s"] * solve_s,
                                             "e2e_ratio": g["e2e_solves_per_s"] * solve_s})
    return out


def run_reference(args, cfg):
    """The reference arm: the oracle's CPU restatement of the reference algorithm on the same tank,
    all host threads.  Set-up (tree, lists, near quadrature of every point) once, measured whole;
    then each step runs ONE whole stage of the mat-vec (P2M, M2M, M2L, L2L, near sums, L2P in
    turn) over the whole problem.  ms_per_step is the measured step time; value = 1 / (set-up +
    (iterations + 2) x mat-vec) with the mat-vec the sum of the stages' median times and the
    iteration count of the reference algorithm on this workload (modeled: REFERENCE_ITERATIONS)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    from bem_for_nonlinear_waves_b200.tank import make_tank  # mesh generator only
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    tk = dict(cfg["tank"])
    noise = tk.pop("noise")
    seed = tk.pop("seed")
    t = make_tank(noise_sigma=noise * tk["h"], seed=seed, **tk)
    d = O.build_dofs(t.X, t.tri, t.face_dirichlet)
    o, su = port_context(cfg, t, d)
    samples = {k: [] for k in PORT_STAGES}
    timed = 0.0
    for k in range(args.warmup + args.steps):
        stage = PORT_STAGES[k % len(PORT_STAGES)]
        w0 = time.perf_counter()
        o.time_stage(stage)
        dt = time.perf_counter() - w0
        samples[stage].append(dt)
        if k >= args.warmup:
            timed += dt
    for stage in PORT_STAGES:  # fewer than six steps in all: time the missing stages once more
        if not samples[stage]:
            w0 = time.perf_counter()
            o.time_stage(stage)
            samples[stage].append(time.perf_counter() - w0)
    med = {k: statistics.median(v) for k, v in samples.items()}
    mv = sum(med.values())
    tol = args.tol or 1e-11
    iters, how = reference_iterations(args.config, tol)
    iters = iters or args.ref_iters
    value = 1.0 / port_solve_model(su["setup_s"], mv, iters)
    phys, ncpu = physical_cores()
    line = {"impl": "reference", "metric": "bvp_solves_per_s", "value": value, "unit": "solves/s", "n_gpus": 0,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * timed / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config(args.config, cfg, t, d["dof_point"].shape[0]),
            "matvecs_per_s": 1.0 / mv, "matvec_stage_s": {k: round(v, 4) for k, v in med.items()},
            "setup_s": su["setup_s"], "tolerance": tol, "reference_iterations": iters, "reference_iterations_how": how,
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": phys, "threads": su["threads"], "kind": "port",
                             "sample": ("oracle CPU restatement of the reference algorithm on the same tank; set-up measured whole "
                                        "once; each step one whole mat-vec stage (P2M, M2M, M2L, L2L, near sums, L2P in turn) "
                                        f"over the whole tank; solves/s modeled as 1 / (set-up + ({iters} iterations + 2) x "
                                        "mat-vec)")},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def load_traffic(kernel, workload):
    """dram bytes per launch of a kernel from a committed ncu summary (profiles/), else None."""
    path = os.path.join(ROOT, "profiles", f"{kernel}_{workload}.txt")
    if not os.path.exists(path):
        return None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch:"):
            return float(line.split(":")[1])
    return None


def load_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        try:
            return json.load(open(path)), "measured"
        except ValueError:
            pass
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def mixed_problems(n, seed, floating_box=True):
    """The batch workload: tanks of mixed sizes drawn from one seed -- length U[1, 4], width 1,
    depth U[0.3, 1.0], h chosen so the point count is log-uniform in [2k, 80k], amplitude
    U[0.005, 0.05], wavelength U[0.5, 2] -- each with a floating box 0.3 x 0.3 m, draft 0.2 m, at a
    random x (centred in y, snapped to the grid), its faces Neumann with the rigid-body velocity of
    seeded 6-DOF velocities U, Omega in U[-0.1, 0.1]^3."""
    from bem_for_nonlinear_waves_b200 import build_dofs, known_values, make_tank, point_normals
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L, W, D = rng.uniform(1, 4), 1.0, rng.uniform(0.3, 1.0)
        pts = math.exp(rng.uniform(math.log(2e3), math.log(8e4)))
        h = math.sqrt(2 * (L * W + L * D + W * D) / pts)
        amp, wl = rng.uniform(0.005, 0.05), rng.uniform(0.5, 2.0)
        xb = rng.uniform(0.3, L - 0.3)
        U, Om = rng.uniform(-0.1, 0.1, 3), rng.uniform(-0.1, 0.1, 3)
        fb = (xb, W / 2, 0.3, 0.3, 0.2, U, Om) if floating_box else None
        t = make_tank(L, W, D, h, amplitude=amp, wavelength=wl, floating_box=fb)
        d = build_dofs(t.X, t.tri, t.face_dirichlet)
        out.append((t, d, known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))))
    return out


def run_batch(args, cfg, local):
    """Batch mode.  `--mixed-sizes`: the 96-tank batch workload (mixed_problems: 2k-80k points,
    floating box, p = 8).  Every problem is first solved by the FP64 GPU path at relative residual
    1e-12 (its oracle, not timed); then, at the accuracy gate's tolerance, (a) the batch through a
    BatchSolver of `--workers W` mixed-precision contexts, all submitted at once or with seeded
    Poisson arrivals (`--arrival-rate`), with per-problem latency from submission to result, and
    (b) the same problems one after another through the plain FP64 GPU path; both solutions are
    checked against the oracle.  Without `--mixed-sizes`: `--batch P` seeded tanks of the
    workload's size."""
    from bem_for_nonlinear_waves_b200 import BEM_BVP, BatchSolver
    if args.mixed_sizes:
        probs = mixed_problems(args.batch, 2024)
        cfg = dict(cfg, p=8)
        workload = "mixed_2k_80k_floating_box_p8"
    else:
        probs = [make_problem(cfg, 1000 + i) for i in range(args.batch)]
        workload = args.config
    tol = args.tol or 1e-11
    base = dict(expansion_order=cfg["p"], tol_relative=True, solver_max_iter=args.max_iter, preconditioner=args.precond,
                poly_degree=args.poly_degree, device=local)
    # oracles: the FP64 GPU solve of each problem at relative residual 1e-12
    refs = []
    for t, d, kv in probs:
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, solver_tol=ORACLE_REL_TOL, precision="fp64", **dict(base, solver_max_iter=4000))
        b.solve(kv)
        refs.append(b.ans.copy())
        del b

    def err(ans, ref):
        return float(np.abs(ans - ref).max() / np.abs(ref).max())

    # (b) plain FP64 GPU path, one after another (one warm solve first)
    b = BEM_BVP(probs[0][0].X, probs[0][0].tri, probs[0][0].face_dirichlet, dofs=probs[0][1], solver_tol=tol, precision="fp64", **base)
    b.solve(probs[0][2])
    del b
    seq_lat, seq_err = [], []
    w0 = time.perf_counter()
    for (t, d, kv), ref in zip(probs, refs):
        b = BEM_BVP(t.X, t.tri, t.face_dirichlet, dofs=d, solver_tol=tol, precision="fp64", **base)
        s0 = time.perf_counter()
        b.solve(kv)
        seq_lat.append(time.perf_counter() - s0)
        seq_err.append(err(b.ans, ref))
        del b
    seq_s = time.perf_counter() - w0
    # (a) the batched mixed-precision solver
    bs = BatchSolver(args.workers, solver_tol=tol, precision=args.precision, tc_deterministic=bool(args.tc_deterministic), **base)
    for tk in [bs.submit(t.X, t.tri, t.face_dirichlet, kv, dofs=d) for t, d, kv in probs[:args.workers]]:
        bs.result(tk)  # every worker context warm
    with ClockSampler(local) as clk:
        w0 = time.perf_counter()
        sub, lat = {}, {}

        def reap():
            for tk in sub:
                if tk not in lat and bs.done(tk):
                    lat[tk] = time.perf_counter() - sub[tk]

        gaps = np.random.default_rng(77).exponential(1.0 / args.arrival_rate, len(probs)) if args.arrival_rate > 0 else None
        t_next = w0
        order = []
        for i, (t, d, kv) in enumerate(probs):
            if gaps is not None:
                t_next += gaps[i]
                while time.perf_counter() < t_next:
                    reap()
                    time.sleep(0.0002)
            tk = bs.submit(t.X, t.tri, t.face_dirichlet, kv, dofs=d)
            sub[tk] = time.perf_counter()
            order.append(tk)
        while len(lat) < len(sub):
            reap()
            time.sleep(0.0005)
        batch_s = time.perf_counter() - w0
    b_err, conv = [], True
    for tk, (t, d, kv), ref in zip(order, probs, refs):
        phi, phin, st = bs.result(tk)
        conv = conv and bool(st.converged)
        b_err.append(err(np.where(d["dof_kind"] == 0, phin, phi), ref))
    bs.close()
    lats = sorted(lat.values())
    pct = lambda v, q: float(np.percentile(np.asarray(v), q))  # noqa: E731
    value = len(probs) / batch_s
    seq_v = len(probs) / seq_s
    line = {"metric": "bvp_solves_per_s", "value": value, "unit": "solves/s", "n_gpus": 1, "mode": "batch",
            "higher_is_better": True, "dtype": "f64/f16x3-tc" if args.precision == "mixed" else "f64", "data": "synthetic",
            "config": {"workload": workload, "problems": len(probs), "points": [int(p[0].n_points) for p in probs],
                       "workers": args.workers, "precision": args.precision, "preconditioner": args.precond, "rel_tol": tol,
                       "arrivals": f"poisson {args.arrival_rate}/s" if args.arrival_rate > 0 else "all at once"},
            "latency_s": {"p50": pct(lats, 50), "p99": pct(lats, 99), "max": lats[-1]},
            "accuracy": {"gate": GATE, "max_rel_err_batch": max(b_err), "max_rel_err_fp64": max(seq_err),
                         "within_gate": bool(max(b_err) <= GATE and max(seq_err) <= GATE), "converged": conv},
            "fp64_gpu_sequential": {"solves_per_s": seq_v, "latency_p50_s": pct(seq_lat, 50), "latency_p99_s": pct(seq_lat, 99)},
            "speedup_vs_fp64_gpu": value / seq_v,
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def chain_problems(n, seed, median=15000, sigma=0.75, lo=3000, hi=200000):
    """The serving workload's tanks: as mixed_problems (floating box), with point counts
    lognormal around `median` (sigma in log space), clipped to [lo, hi]."""
    from bem_for_nonlinear_waves_b200 import build_dofs, known_values, make_tank, point_normals
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        L, W, D = rng.uniform(1, 4), 1.0, rng.uniform(0.3, 1.0)
        pts = float(np.clip(median * math.exp(rng.normal(0.0, sigma)), lo, hi))
        h = math.sqrt(2 * (L * W + L * D + W * D) / pts)
        amp, wl = rng.uniform(0.005, 0.05), rng.uniform(0.5, 2.0)
        xb = rng.uniform(0.3, L - 0.3)
        U, Om = rng.uniform(-0.1, 0.1, 3), rng.uniform(-0.1, 0.1, 3)
        t = make_tank(L, W, D, h, amplitude=amp, wavelength=wl, floating_box=(xb, W / 2, 0.3, 0.3, 0.2, U, Om))
        d = build_dofs(t.X, t.tri, t.face_dirichlet)
        out.append((t, d, known_values(t, d["dof_point"], d["dof_face"], d["dof_kind"], point_normals(t))))
    return out


def run_serve(args, local):
    """Serving mode: `--serve-chains R` requests, each a whole RK4 time-stepping chain of
    `--chain-steps` steps (4 BVPs per step, the MEL update between them) on a tank of the serving
    workload (chain_problems), arriving as a seeded Poisson stream of `--arrival-rate` requests/s,
    served by a BatchSolver of `--workers` contexts with admission by device memory (150 GB, or
    90 % of the free memory if less).  Run for the mixed-precision and the plain FP64 solver;
    reports request latency p50/p99 (arrival to result) and BVP solves/s."""
    import torch
    from bem_for_nonlinear_waves_b200 import BatchSolver
    probs = chain_problems(args.serve_chains, 4242)
    free = torch.cuda.mem_get_info(local)[0]
    budget = int(min(150e9, 0.9 * free))
    tol = args.tol or 1e-11
    out = {}
    for prec in ("mixed", "fp64"):
        bs = BatchSolver(args.workers, expansion_order=8, solver_tol=tol, tol_relative=True, solver_max_iter=args.max_iter,
                         preconditioner=args.precond, device=local, precision=prec)
        bs.set_budget(budget)
        t0, d0, k0 = probs[0]  # every worker context warm
        for tk in [bs.submit(t0.X, t0.tri, t0.face_dirichlet, k0, dofs=d0) for _ in range(args.workers)]:
            bs.result(tk)
        gaps = np.random.default_rng(99).exponential(1.0 / args.arrival_rate, len(probs))
        sub, lat, order = {}, {}, []
        with ClockSampler(local) as clk:
            w0 = time.perf_counter()
            t_next = w0
            for i, (t, d, kv) in enumerate(probs):
                t_next += gaps[i]
                while time.perf_counter() < t_next:
                    time.sleep(0.0002)
                tk = bs.submit_chain(t.X, t.tri, t.face_dirichlet, kv, n_steps=args.chain_steps, dt=1e-3, dofs=d)
                sub[tk] = time.perf_counter()
                order.append(tk)
            while len(lat) < len(sub):
                for tk in order:
                    if tk not in lat and bs.done(tk):
                        lat[tk] = time.perf_counter() - sub[tk]
                time.sleep(0.001)
            wall = time.perf_counter() - w0
        iters, conv = 0, True
        for tk in order:
            _, _, st = bs.result_chain(tk)
            iters += st.iterations
            conv = conv and bool(st.converged)
        stats = bs.stats()
        bs.close()
        solves = len(probs) * args.chain_steps * 4
        lats = sorted(lat.values())
        out[prec] = {"solves_per_s": solves / wall, "requests_per_s": len(probs) / wall,
                     "latency_s": {"p50": float(np.percentile(lats, 50)), "p99": float(np.percentile(lats, 99)), "max": lats[-1]},
                     "gmres_iterations_per_solve": iters / solves, "converged": conv, "admission": stats, "clocks": clk.summary()}
    line = {"metric": "bvp_solves_per_s", "value": out["mixed"]["solves_per_s"], "unit": "solves/s", "n_gpus": 1, "mode": "serve",
            "higher_is_better": True, "dtype": "f64/f16x3-tc", "data": "synthetic",
            "config": {"workload": "rk4_chains_lognormal_15k_floating_box_p8", "requests": len(probs), "chain_steps": args.chain_steps,
                       "bvps_per_request": 4 * args.chain_steps, "points": [int(p[0].n_points) for p in probs],
                       "arrivals": f"poisson {args.arrival_rate}/s", "workers": args.workers, "hbm_budget_bytes": budget,
                       "rel_tol": tol},
            "mixed": out["mixed"], "fp64": out["fp64"],
            "speedup_vs_fp64_gpu": out["mixed"]["solves_per_s"] / out["fp64"]["solves_per_s"]}
    print(json.dumps(line), flush=True)
    return 0


def time_solves(bvp, kv, steps, clk=None):
    """`steps` x (set-up + solve) through the public API, host arrays in and out: device time
    (CUDA events around the device work), wall time, and the per-step detail."""
    dev_s = e2e_s = plan_s = upload_s = 0.0
    launches = h2d = d2h = iters = mv = mv_lo = 0
    converged = True
    detail = []
    for _ in range(steps):
        w0 = time.perf_counter()
        bvp.setup()
        w1 = time.perf_counter()
        bvp.solve(kv)
        w2 = time.perf_counter()
        e2e_s += w2 - w0
        st = bvp.stats
        ph = bvp.setup_phases()
        detail.append({"setup_wall_ms": round(1e3 * (w1 - w0), 2), "solve_wall_ms": round(1e3 * (w2 - w1), 2),
                       "device_ms": round(1e3 * st.time_device_s, 3), "setup_device_ms": round(1e3 * st.time_setup_device_s, 3),
                       "gmres_iterations": int(st.iterations),
                       "setup_parts_ms": {k: round(1e3 * v, 2) for k, v in ph.items() if isinstance(v, float)}})
        dev_s += st.time_device_s
        plan_s += st.time_plan_s
        upload_s += st.time_upload_s
        launches += st.kernel_launches
        h2d += st.h2d_bytes
        d2h += st.d2h_bytes
        iters += st.iterations
        mv += st.matvecs
        mv_lo += st.matvecs_lo
        converged = converged and bool(st.converged)
    return dict(dev_s=dev_s, e2e_s=e2e_s, plan_s=plan_s, upload_s=upload_s, launches=launches, h2d=h2d, d2h=d2h, iters=iters,
                matvecs=mv, matvecs_lo=mv_lo, converged=converged, detail=detail)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="tank_60k", choices=list(CONFIGS))
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--precond", default="near_block", choices=["near_block", "jacobi", "none", "near_poly"])
    ap.add_argument("--poly-degree", type=int, default=8, help="degree of the near_poly preconditioner")
    ap.add_argument("--overlap-near", type=int, default=1, help="1: near field of the mixed A.x on a second stream (0: after the FMM passes)")
    ap.add_argument("--max-iter", type=int, default=1500)
    ap.add_argument("--refine-rtol", type=float, default=0.0, help="mixed: inner-cycle relative tolerance (0: library default)")
    ap.add_argument("--tc-deterministic", type=int, default=0,
                    help="mixed: 1 = tensor-core M2L partials summed in a fixed order (bit-reproducible), 0 = fused L2 reduction")
    ap.add_argument("--tol", type=float, default=0.0,
                    help="relative tolerance of the timed solves (0: the loosest of 1e-9..1e-12 within half the accuracy gate)")
    ap.add_argument("--ref-iters", type=int, default=1000)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the batch, re-solve and RK4 measurements")
    ap.add_argument("--count-reference-iterations", action="store_true",
                    help="count the unpreconditioned FP64 GMRES iterations at --tol (the reference algorithm) and exit")
    ap.add_argument("--batch", type=int, default=0, help="serving mode: number of problems (one GPU)")
    ap.add_argument("--workers", type=int, default=2)
    ap.add_argument("--mixed-sizes", action="store_true", help="serving mode over tanks of 2k-80k points (p = 8)")
    ap.add_argument("--arrival-rate", type=float, default=0.0, help="serving mode: Poisson arrivals per second (0: all at once)")
    ap.add_argument("--serve-chains", type=int, default=0, help="serving mode: number of RK4-chain requests (one GPU)")
    ap.add_argument("--chain-steps", type=int, default=20, help="serving mode: RK4 steps per chain request")
    args = ap.parse_args()
    cfg = CONFIGS[args.config]
    if args.impl == "reference":
        return run_reference(args, cfg)
    if args.serve_chains > 0:
        if args.arrival_rate <= 0:
            args.arrival_rate = 200.0
        return run_serve(args, int(os.environ.get("LOCAL_RANK", "0")))
    if args.batch > 0:
        return run_batch(args, cfg, int(os.environ.get("LOCAL_RANK", "0")))

    rank, world, local = dist_init()
    from bem_for_nonlinear_waves_b200 import BEM_BVP
    from bem_for_nonlinear_waves_b200 import _lib
    t, d, kv = make_problem(cfg, rank)
    mixed = args.precision == "mixed"

    def make(prec, tol, precond=None, max_iter=None):
        return BEM_BVP(t.X, t.tri, t.face_dirichlet, expansion_order=cfg["p"], solver_tol=tol, tol_relative=True,
                       solver_max_iter=max_iter or args.max_iter, preconditioner=precond or args.precond, poly_degree=args.poly_degree,
                       overlap_near=args.overlap_near, dofs=d, device=local, precision=prec, refine_rtol=args.refine_rtol,
                       tc_deterministic=bool(args.tc_deterministic))

    if args.count_reference_iterations:
        tol = args.tol or cfg["rel_tol"]
        b = make("fp64", tol, precond="none", max_iter=6000)
        b.solve(kv)
        print(json.dumps({"workload": args.config, "rel_tol": tol, "reference_iterations": int(b.stats.iterations),
                          "converged": bool(b.stats.converged)}), flush=True)
        return 0

    # the FP64 oracle: the FP64 GPU solve of the same tank at relative residual 1e-12 (not timed)
    b_ref = make("fp64", ORACLE_REL_TOL, max_iter=4000)
    b_ref.solve(kv)
    x_ref = b_ref.ans.copy()
    oracle_info = {"rel_tol": ORACLE_REL_TOL, "gmres_iterations": int(b_ref.stats.iterations), "converged": bool(b_ref.stats.converged)}
    del b_ref

    def rel_err(x):
        return float(np.abs(x - x_ref).max() / np.abs(x_ref).max())

    # the timed tolerance: the loosest of the ladder whose solve lands within half the gate
    ladder = []
    if args.tol > 0:
        tol = args.tol
    else:
        tol = TOL_LADDER[-1]
        for cand in TOL_LADDER:
            b = make(args.precision, cand)
            b.solve(kv)
            e = rel_err(b.ans)
            ladder.append({"rel_tol": cand, "max_rel_err": e, "gmres_iterations": int(b.stats.iterations)})
            del b
            if e <= 0.5 * GATE:
                tol = cand
                break

    bvp = make(args.precision, tol)
    for _ in range(args.warmup):
        bvp.setup()
        bvp.solve(kv)
    prof = bvp.profile_matvec(repeats=5, mixed=mixed)
    prof64 = bvp.profile_matvec(repeats=5) if mixed else prof
    tree = bvp.tree_stats()
    fp64_peak = _lib.load().bem_gpu_fp64_peak_tflops(local)

    barrier(world)
    import torch
    # the timed steps are the profiled range of a profiler run with --profile-from-start off
    # (no effect otherwise)
    torch.cuda.profiler.start()
    with ClockSampler(local) as clk:
        r = time_solves(bvp, kv, args.steps)
    torch.cuda.profiler.stop()
    barrier(world)
    dev_max, e2e_max = allreduce_max([r["dev_s"], r["e2e_s"]], world)
    ans = bvp.ans.copy()
    err_max = rel_err(ans)
    err_l2 = float(np.linalg.norm(ans - x_ref) / np.linalg.norm(x_ref))

    # the plain FP64 GPU path on the same tank at the same tolerance, timed the same way
    fp64 = None
    if mixed:
        b64 = make("fp64", tol)
        for _ in range(max(1, min(args.warmup, 2))):
            b64.setup()
            b64.solve(kv)
        barrier(world)
        r64 = time_solves(b64, kv, args.steps)
        barrier(world)
        dev64, e2e64 = allreduce_max([r64["dev_s"], r64["e2e_s"]], world)
        e64 = rel_err(b64.ans)
        fp64 = {"solves_per_s": world * args.steps / dev64, "e2e_solves_per_s": world * args.steps / e2e64,
                "gmres_iterations": r64["iters"] / args.steps, "matvec_ms": prof64["total"], "max_rel_err": e64,
                "within_gate": bool(e64 <= GATE)}
        del b64

    value = world * args.steps / dev_max
    accuracy = {"gate": GATE, "rel_tol": tol, "max_rel_err": err_max, "l2_rel_err": err_l2, "within_gate": bool(err_max <= GATE),
                "oracle": oracle_info, "tolerance_search": ladder or "fixed by --tol"}
    if fp64:
        accuracy["speedup_vs_fp64_gpu"] = value / fp64["solves_per_s"]
        accuracy["e2e_speedup_vs_fp64_gpu"] = (world * args.steps / e2e_max) / fp64["e2e_solves_per_s"]

    extras = {}
    if not args.no_extras:
        extras = measure_extras(args, cfg, t, d, kv, bvp, tol, local)

    peaks, peaks_kind = load_peaks()
    p = cfg["p"]
    nc = (p + 1) * (p + 2) // 2
    m2l_flops = tree["m2l_pairs"] * 2 * nc * (p + 1) ** 2 * 8.0  # the reference's M2L: complex MACs, both densities
    if mixed:
        kp = ((p + 1) ** 2 + 63) // 64 * 64
        t_k = prof["m2l_contract"] * 1e-3
        achieved = m2l_flops / t_k / 1e12
        roof = {"kernel": "k_m2l_tc", "bound": "tensor", "achieved": achieved, "peak": peaks["bf16_tflops"], "unit": "TFLOP/s",
                "frac": achieved / peaks["bf16_tflops"], "traffic": load_traffic("k_m2l_tc", args.config),
                "peak_source": f"{peaks_kind} bf16 dense burst (MEASURED_PEAKS.json bf16_tflops); kernel timed alone",
                "algorithmic_flops_per_launch": m2l_flops,
                "tensor_flops_issued_per_launch": tree["m2l_pairs"] * 128.0 * kp * 2 * 3,
                "kernel_ms": prof["m2l_contract"], "m2l_stage_ms": prof["m2l"]}
        if roof["traffic"]:  # the same launch against HBM: DRAM bytes (ncu) / CUDA-event time
            roof["hbm_gbs_of_traffic"] = roof["traffic"] / t_k / 1e9
            roof["hbm_frac_of_traffic"] = roof["hbm_gbs_of_traffic"] / peaks["hbm_gbs"]
    else:
        t_k = prof["m2l"] * 1e-3
        achieved = m2l_flops / t_k / 1e12
        roof = {"kernel": "k_m2l_grp", "bound": "fp64", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak if fp64_peak > 0 else None, "traffic": load_traffic("k_m2l_grp", args.config),
                "peak_source": "measured FP64 FMA probe on this GPU (MEASURED_PEAKS.json has no FP64 figure)",
                "algorithmic_flops_per_launch": m2l_flops, "kernel_ms": prof["m2l"]}
    near = near_roofline(bvp, tree, prof, peaks, peaks_kind, mixed, args.config)
    phys, ncpu = physical_cores()
    line = {
        "metric": "bvp_solves_per_s", "value": value, "unit": "solves/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dev_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64/f16x3-tc" if mixed else "f64", "data": "synthetic",
        "config": workload_config(args.config, cfg, t, bvp.matrix_size),
        "parallelism": f"replicas{world}",
        "solve": {"precision": args.precision, "preconditioner": args.precond + (f" (degree {args.poly_degree})" if args.precond == "near_poly" else ""),
                  "rel_tol": tol, "gmres_iterations": r["iters"] / args.steps, "matvecs_fp64": r["matvecs"] / args.steps,
                  "matvecs_lowp": r["matvecs_lo"] / args.steps, "converged": r["converged"], "overlap_near": bool(args.overlap_near),
                  "l2": "working set > L2 (near-field weights %.1f GB)" % (tree["nnz"] * 16 / 1e9)},
        "accuracy": accuracy,
        "matvecs_per_s": world * 1e3 / prof["total"],
        "host_setup_s_per_step": {"plan": r["plan_s"] / args.steps, "upload": r["upload_s"] / args.steps},
        "matvec_stage_ms": prof,
        "tc_item_tuning": bvp.tc_tuning() if mixed else None,
        "e2e": {"value": world * args.steps / e2e_max, "unit": "solves/s", "h2d_bytes_per_step": r["h2d"] // args.steps,
                "d2h_bytes_per_step": r["d2h"] // args.steps},
        "gpu_launches": r["launches"],
        "steps_detail": r["detail"],
        "roofline": roof,
        "roofline_near": near,
        "clocks": clk.summary(),
        "host": {"physical_cores": phys, "cpus": ncpu},
    }
    if fp64 is not None:
        line["fp64_gpu"] = fp64
    line.update(extras)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        ref1 = cpu_reference_config1(args, local)
        port = cpu_port_baseline(args, cfg, t, d, tol)
        port_line = {"value": port.get("solves_per_s_modeled"), "unit": "solves/s", "cores": phys, "threads": port["threads"],
                     "kind": "port", "matvecs_per_s": port["matvecs_per_s"], "matvec_stages_s": port["stages_s"],
                     "setup_s": port["setup_s"], "iterations": port["iterations"], "iterations_how": port["iterations_how"],
                     "sample": ("oracle CPU restatement of the reference algorithm on this tank: whole set-up and one whole "
                                "mat-vec measured; solves/s modeled as 1 / (set-up + (iterations + 2) x mat-vec)"),
                     "matvec_ratio_gpu": (1e3 / prof["total"]) / port["matvecs_per_s"]}
        if ref1 is not None:
            line["cpu_baseline"] = ref1
            line["cpu_baseline_port"] = port_line
        else:
            line["cpu_baseline"] = port_line
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


def near_roofline(bvp, tree, prof, peaks, peaks_kind, mixed, workload):
    """The near-field SpMV of A.x against HBM.  Mixed operator: k_near_sums<float> timed alone,
    algorithmic bytes = the stored FP32 weight blocks + the gathered unknowns and their DOF
    indices + the per-target sums written.  FP64 operator: the whole targets stage (near sums,
    then the L2P and rows), with the rows written on top."""
    nb = bvp.near_bytes()
    if mixed:
        alg = nb["weights_fp32"] + nb["x_gather"] + nb["dof_index"] + nb["near_sums"]
        ms, name = prof["near_sums"], "k_near_sums<float>"
    else:
        alg = nb["weights_fp64"] + nb["x_gather"] + nb["dof_index"] + nb["near_sums"] + nb["rows"]
        ms, name = prof["targets"], "k_near_sums<double> + k_target_rows"
    achieved = alg / (ms * 1e-3) / 1e9
    return {"kernel": name, "bound": "hbm", "achieved": achieved,
            "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
            "traffic": load_traffic("k_near_sums", workload), "algorithmic_bytes_per_launch": alg,
            "peak_source": f"{peaks_kind} HBM copy bandwidth (MEASURED_PEAKS.json hbm_gbs)", "kernel_ms": ms,
            "targets_stage_ms": prof["targets"]}


def measure_extras(args, cfg, t, d, kv, bvp, tol, local):
    """Batch API, second right-hand side and one RK4 step of the BEM-MEL loop on the same tank."""
    from bem_for_nonlinear_waves_b200 import BatchSolver, MELStage
    out = {}
    # the same solves through the batch API with two worker contexts: the host set-up of one
    # problem overlaps the device solve of the previous one (host arrays in and out)
    bs = BatchSolver(2, expansion_order=cfg["p"], solver_tol=tol, tol_relative=True, solver_max_iter=args.max_iter,
                     preconditioner=args.precond, poly_degree=args.poly_degree, device=local, precision=args.precision)
    for tk in [bs.submit(t.X, t.tri, t.face_dirichlet, kv, dofs=d) for _ in range(2)]:
        bs.result(tk)
    nb = max(2 * args.steps, 4)
    w0 = time.perf_counter()
    for tk in [bs.submit(t.X, t.tri, t.face_dirichlet, kv, dofs=d) for _ in range(nb)]:
        bs.result(tk)
    out["e2e_batch"] = {"value": nb / (time.perf_counter() - w0), "unit": "solves/s", "workers": 2, "solves": nb,
                        "note": "the same problem submitted nb times through bem_gpu_batch_*; host arrays in and out"}
    bs.close()
    # a second right-hand side on the same set-up (phi_t BVP / next stage with unchanged
    # geometry): the solve alone, host arrays in and out
    kv2 = -0.7 * kv + 0.01 * np.random.default_rng(7).standard_normal(kv.shape)
    w0 = time.perf_counter()
    bvp.solve(kv2)
    out["resolve_same_setup"] = {"wall_ms": 1e3 * (time.perf_counter() - w0), "gmres_iterations": bvp.stats.iterations,
                                 "converged": bool(bvp.stats.converged)}
    # the MEL update after a solve, then one full RK4 step of the BEM-MEL loop: four (set-up +
    # solve + update) at the stage positions with the stage's free-surface phi
    bvp.solve(kv)
    mel = MELStage(t.X, t.tri, t.face_dirichlet, dofs=d, device=local)
    mel.stage(0, 1e-3, t.X, bvp.phi, bvp.phin)
    w0 = time.perf_counter()
    for k in range(4):
        mel.stage(k, 1e-3, t.X, bvp.phi, bvp.phin)
    mel_ms = 1e3 * (time.perf_counter() - w0) / 4
    dirichlet = d["dof_kind"] == 0

    def rk4_step(refresh):
        Xs, known = t.X.copy(), kv.copy()
        w0 = time.perf_counter()
        prev = None
        iters, reused, setup_ms = [], [], []
        for k in range(4):  # the same context, set up again at the stage positions; warm start
            s0 = time.perf_counter()
            if refresh:
                reused.append(int(bvp.refresh(Xs)))
            else:
                bvp.X = np.ascontiguousarray(Xs, np.float64)
                bvp.setup()
            setup_ms.append(round(1e3 * (time.perf_counter() - s0), 2))
            bvp.solve(known, x0=prev)
            prev = bvp.ans.copy()
            iters.append(int(bvp.stats.iterations))
            Xs, pnext, _, _ = mel.stage(k, 1e-3, Xs, bvp.phi, bvp.phin)
            known = known.copy()
            known[dirichlet] = pnext[d["dof_point"][dirichlet]]
        return time.perf_counter() - w0, iters, reused, setup_ms

    full_s, iters_full, _, setup_full = rk4_step(False)
    ref_s, iters_ref, reused_ref, setup_ref = rk4_step(True)
    out["mel_rk4"] = {"mel_stage_wall_ms": mel_ms, "rk4_step_wall_s": ref_s, "dt": 1e-3, "gmres_iterations": iters_ref,
                      "setup_wall_ms": setup_ref, "structure_kept": reused_ref,
                      "full_setup": {"rk4_step_wall_s": full_s, "setup_wall_ms": setup_full, "gmres_iterations": iters_full},
                      "note": "4 x (set-up at the stage positions + solve + MEL update), host arrays in and out; stage set-ups by "
                              "bem_gpu_setup_refresh (tree regrown in the previous root, structure kept when unchanged), "
                              "full_setup: bem_gpu_setup each stage"}
    return out


if __name__ == "__main__":
    sys.exit(main())
