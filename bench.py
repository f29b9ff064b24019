"""Benchmark of the DG residual / time-step path: DOF*RK-stages per second.

Workload (one GPU): 2D shock-bubble on [0,2]x[0,1], 512x256 structured quads, p = 2 (9 nodal DOF per
field, 5 fields), Rusanov flux, m2 limiter, SSP-RK3 with the CFL step (CFL 0.3), plain FP64.
Synthetic seeded initial state (Mach-1.5 shock hitting a gamma=1.67 bubble; no dataset involved).
A "step" is one SSP-RK3 step = 3 stages (residual + stage update + limiter each) plus the
device-side CFL step.  DOF = N_E * N_s * N_F = 5,898,240.

  value      whole-job DOF*stages/s with the state resident in HBM, device time (CUDA events on the
             library stream) summed over exactly K steps; L2 is flushed before every timed step
  e2e        the same metric through the C ABI with host buffers, wall clock: every step copies the
             state from pinned host memory, advances one step and reads the state back, in the
             host-resident time loop dgb_advance_host (a step's download and the next step's upload
             overlap, chunk by chunk); per_step_calls: the same steps as dgb_set_state + dgb_advance
             + dgb_get_state per step
  roofline   the fused residual kernel: algorithmic HBM bytes per launch (21.33 B per DOF and stage
             on average for SSP-RK3) / its average device time from a profiled pass of the same steps
  cpu_baseline  the reference CPU build (oracle/_ref, compiled from the reference sources) on a
             bounded sample of the same workload, one process on one core
  forms      plain FP64, mixed and mixed + learned indicator at equal L1 error (same protocol)
  mass_fraction  the workload with one passive mass fraction (6 fields): time per step
  gamma_model  the workload grid with Roe + hrl in both gamma models (GAMNCON, GAMCONS): time per step
  slab_local  the workload split into y-slabs with ghost rows, all in this process on one GPU
             (dg_b200.slab, LocalTransport): time per step against the whole grid, and the owned
             rows' distance from it
  tube_1d    the 1D two-fluid shock tube (1000 elements, p=2, Roe, RK4, CFL 0.4, 2000 steps): device
             time, distance from the reference's own run, the reference CPU build's time
  learned_deploy  the learned indicator on a 1024x1024 four-quadrant problem: FP64 / mixed / mixed +
             gated limiter, time per step and L1 density distance from the FP64 full-limiter run
  mixed_p3   the 2048x1024 p=3 Roe shock-bubble: FP64 and mixed throughput, per-field L1 / Linf of
             the mixed form against the FP64 run and the conserved totals after 300 steps
  ensemble   the batched ensemble (256 independent cases of uneven sizes, dgb_batch): aggregate
             DOF*stages/s against the same cases advanced one after another, autotuned tiling,
             per-case completion times for a common end time

--impl reference runs the reference CPU implementation (oracle/_ref) on the host cores: one process
per core, each advancing its own copy of the workload; a bench step there is one SSP-RK3 stage
(a bounded sample: a full step of this workload takes seconds on one core).

Multi-GPU (torchrun): every rank advances its own replica of the workload (weak scaling, no data-path
collective); the timed region is bracketed by barriers and the max over ranks is taken.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "DOF·RK-stages/sec: plain FP64 vs mixed+learned-limiter form at equal L1 error"
UNIT = "DOF*stages/s"
NX, NY, ORDER = 512, 256, 2
DOMAIN = (0.0, 2.0, 0.0, 1.0)
BC = ("reflective", "transmissive", "reflective", "transmissive")  # bottom, right, top, left
CFL = 0.3
SEED = 7
STAGES_PER_STEP = 3
BYTES_PER_DOF_STAGE = (16.0 + 24.0 + 24.0) / 3.0  # SSP-RK3 Shu-Osher, fully fused stages
# the learned indicator scores every IND_EVERY-th step: a discontinuity moves at most CFL/(2p+1) =
# 0.06 of an element per step here, so the band (flagged cells and their face neighbours) of one
# scoring covers it for half of the 16 steps it could
IND_EVERY = 8


def config(extra=None):
    c = {"workload": "2D shock-bubble 512x256 quads, p=2, Rusanov, m2l limiter, SSP-RK3, CFL 0.3",
         "form": "plain FP64", "n_elem": NX * NY, "order": ORDER, "dof": NX * NY * (ORDER + 1) ** 2 * 5,
         "scheme": "SSP-RK3 (3 stages/step)", "l2": "flushed (256 MiB write) before every timed step",
         "parallelism": "replicas"}
    if extra:
        c.update(extra)
    return c


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.tmp = None

    def __enter__(self):
        try:
            self.tmp = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.tmp, stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if self.proc is None or self.tmp is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.tmp.flush()
        rows = []
        for line in Path(self.tmp.name).read_text().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.tmp.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def build_problem(nx=NX, ny=NY):
    import dg_b200 as dgb
    x0, x1, y0, y1 = DOMAIN
    prob = dgb.Problem.structured(2, ORDER, nx, ny, x0, x1, y0, y1, BC, flux="rusanov", limiter="m2l", cfl=CFL)
    U0 = prob.init_state("shock_bubble", seed=SEED)
    return prob, U0


def cpu_baseline(U0_limited: np.ndarray, steps: int = 2):
    """Reference CPU build, one process on one core, `steps` SSP-RK3 steps of the workload."""
    from oracle.ref_run import RefCase, available
    if not available(2, "rusanov"):
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "oracle/_ref binaries not built on this host"}
    x0, x1, y0, y1 = DOMAIN
    case = RefCase(2, ORDER, NX, NY, x0, x1, y0, y1, BC, "rusanov", "m2l")
    case.write_deck(cfl=CFL)
    out, log = case.run("rk3", U0_limited, dt=0.0, nsteps=steps, timeout=1800)
    wall = float(log.split("DGREF_WALL_S")[1].split()[0])
    dof = NX * NY * (ORDER + 1) ** 2 * 5
    return {"value": dof * STAGES_PER_STEP * steps / wall, "unit": UNIT, "cores": 1, "kind": "reference",
            "sample": f"{steps} SSP-RK3 steps ({steps * STAGES_PER_STEP} stages) of the full 512x256 workload, "
                      f"reference residual/Lsolver/m2l limiter/DtFromCFL, 1 process, {wall:.2f} s"}


def run_reference(args):
    """--impl reference: the reference CPU implementation on all host cores (one process per core).

    This process loads nothing of this package: the mesh file and the seeded initial state come
    from oracle/workload.py (pure Python, bit-identical to the library's writer and initial state),
    the initial limiting and the time stepping from the reference binary oracle/_ref/dgref_2d_rus
    (the reference sources compiled by oracle/build_ref.py)."""
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    from oracle.ref_run import RefCase, available
    from oracle.workload import shock_bubble
    if not available(2, "rusanov"):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref reference binaries are not built"}))
        return 0
    x0, x1, y0, y1 = DOMAIN
    Uraw = shock_bubble(ORDER, NX, NY, x0, x1, y0, y1, seed=SEED)
    first = RefCase(2, ORDER, NX, NY, x0, x1, y0, y1, BC, "rusanov", "m2l")
    first.write_deck(cfl=CFL)
    U0 = first.limit(Uraw)  # the reference limits the initial condition when CFL > 0 (rk.cc:108-114)
    ncores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count()
    total = args.warmup + args.steps  # bench steps; one reference bench step = one SSP-RK3 stage
    rk_steps = (total + STAGES_PER_STEP - 1) // STAGES_PER_STEP
    procs, cases = [], []
    for k in range(ncores):
        case = RefCase(2, ORDER, NX, NY, x0, x1, y0, y1, BC, "rusanov", "m2l")
        case.write_deck(cfl=CFL)
        np.ascontiguousarray(U0).tofile(case.workdir / "in.bin")
        exe = str(ROOT / "oracle" / "_ref" / "dgref_2d_rus")
        cmd = [exe, "-d", "deck.inp", "--cmd", "rk3", "--dt", "0", "--nsteps", str(rk_steps), "--in", "in.bin",
               "--out", "out.bin"]
        if hasattr(os, "sched_setaffinity"):
            cpus = sorted(os.sched_getaffinity(0))
            cmd = ["taskset", "-c", str(cpus[k % len(cpus)])] + cmd
        env = dict(os.environ, OPENBLAS_NUM_THREADS="1", OMP_NUM_THREADS="1")
        procs.append(subprocess.Popen(cmd, cwd=case.workdir, stdout=subprocess.PIPE, stderr=subprocess.PIPE,
                                      text=True, env=env))
        cases.append(case)
    per_proc = []
    for p in procs:
        out, err = p.communicate(timeout=3600)
        if p.returncode != 0:
            print(json.dumps({"impl": "reference", "unavailable": f"reference run failed: {err[-200:]}"}))
            return 0
        marks = [float(l.split()[3]) for l in out.splitlines() if l.startswith("DGREF_STAGE_S")]
        stages = [marks[0]] + [marks[i] - marks[i - 1] for i in range(1, len(marks))]
        per_proc.append(stages)
    timed = [max(pp[args.warmup + k] for pp in per_proc) for k in range(args.steps)]
    t = sum(timed)
    dof = NX * NY * (ORDER + 1) ** 2 * 5
    value = ncores * dof * args.steps / t
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference", "config": config(),
            "reference_step": (f"one bench step = one SSP-RK3 stage of the workload in each of {ncores} "
                               f"independent processes (one per core); the metric counts stages, so the rate "
                               f"compares with the GPU arm's, whose bench step is a whole 3-stage step"),
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": ncores, "kind": "reference",
                             "sample": f"each of {ncores} processes (one per core) advances its own copy of the "
                                       f"workload; one bench step = one SSP-RK3 stage (reference residual, "
                                       f"Lsolver, update, m2l limiter; the CFL step in stage 1); stage time = "
                                       f"max over processes"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def max_over_ranks(value: float, ws: int, device: str) -> float:
    """Max of a per-rank time over all ranks (identity on one rank); every rank must call it."""
    if ws <= 1:
        return value
    import torch
    import torch.distributed as dist
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(ws: int, dof: int, steps: int, t_max_s: float) -> float:
    """DOF*stages/s of all replicas together: every rank advances its own copy of the workload."""
    return ws * dof * STAGES_PER_STEP * steps / t_max_s


def time_steps(dgb, solver, steps, warmup, flush):
    """Device time (ms) and launches of `steps` SSP-RK3 steps, L2 flushed before each one."""
    import torch
    for _ in range(warmup):
        solver.advance(1, 0.0, scheme=dgb.SSPRK3)
    torch.cuda.synchronize()
    dev_ms, launches = 0.0, 0
    for _ in range(steps):
        flush.fill_(1.0)
        torch.cuda.synchronize()
        solver.advance(1, 0.0, scheme=dgb.SSPRK3)
        ms, n = solver.last_timing()
        dev_ms += ms
        launches += n
    torch.cuda.synchronize()
    return dev_ms, launches


def kernel_breakdown(dgb, solver, steps=2 * IND_EVERY):
    """Device time per step of each kernel class (residual, limiter, learned-indicator scoring, CFL
    step) from a separate profiled pass of `steps` CFL steps: eager launches, each class bracketed by
    CUDA events (adds launch gaps; the timed figures are graph replays)."""
    solver.set_profiling(True)
    solver.advance(steps, 0.0, scheme=dgb.SSPRK3)
    out = {k: solver.kernel_timing(k)[0] / steps for k in ("residual", "limiter", "indicator", "dt")}
    solver.set_profiling(False)
    return out


def cell_means(prob, U, field=0):
    """Cell averages of one field: sum_i w_i U_i with w_i = sum_g phi_w[g, i] / |reference element|."""
    i = prob.info
    w = prob.array("phi_w").reshape(i.n_s, i.n_g).sum(axis=1) / 4.0
    return U.reshape(i.n_elem, i.n_fields, i.n_s)[:, field, :] @ w


def compare_forms(dgb, U0_coarse, dev, steps, warmup, flush, acc_steps=200):
    """The forms of the solver on the benchmark workload: throughput of plain FP64, mixed and
    mixed + learned indicator (same timing protocol as the headline), and their L1 density error
    after `acc_steps` fixed steps against a 2x-refined plain FP64 solution (1024 x 512, half the
    step) projected on the 512 x 256 cells."""
    from dg_b200 import learned as L
    params, meta = L.load()
    prob, _ = build_problem()
    out = {}
    solvers = {}
    for name, form, learned in (("fp64", "fp64", False), ("mixed", "mixed", False), ("mixed_learned", "mixed", True)):
        s = dgb.DGSolver(prob, device=dev)
        s.set_form(form)
        if learned:
            L.set_indicator(s, params, 0.2, every=IND_EVERY)
        s.set_state(U0_coarse)
        ms, n = time_steps(dgb, s, steps, warmup, flush)
        dof = prob.info.n_elem * prob.info.n_s * prob.info.n_fields
        out[name] = {"value": dof * STAGES_PER_STEP * steps / (ms / 1e3), "ms_per_step": ms / steps,
                     "gpu_launches_per_step": n / steps, "kernel_ms_per_step": kernel_breakdown(dgb, s)}
        solvers[name] = s
    base = out["fp64"]["value"]
    for k in out:
        out[k]["speedup_vs_fp64"] = out[k]["value"] / base
    # accuracy at a fixed step
    ref = solvers["fp64"]
    dt = 0.8 * ref.dt_from_cfl(U0_coarse)
    finals = {}
    for name, s in solvers.items():
        s.set_state(U0_coarse)
        try:
            s.advance(acc_steps, dt, scheme=dgb.SSPRK3)
            finals[name] = s.get_state()
        except dgb.DGBError as e:
            finals[name] = None
            out[name]["failed"] = str(e)
    if finals.get("mixed_learned") is not None:
        sc, cnt = L.scores(solvers["mixed_learned"], finals["mixed_learned"])
        out["mixed_learned"]["flagged_fraction_final"] = cnt / prob.info.n_elem
    for s in solvers.values():
        s.close()
    fprob, fU0 = build_problem(2 * NX, 2 * NY)
    fs = dgb.DGSolver(fprob, device=dev)
    fs.set_state(fs.limit(fU0))
    fs.advance(2 * acc_steps, 0.5 * dt, scheme=dgb.SSPRK3)
    fine = cell_means(fprob, fs.get_state()).reshape(2 * NY, 2 * NX)
    fs.close()
    truth = 0.25 * (fine[0::2, 0::2] + fine[1::2, 0::2] + fine[0::2, 1::2] + fine[1::2, 1::2]).reshape(-1)
    for name, U in finals.items():
        if U is None:
            continue
        err = float(np.abs(cell_means(prob, U) - truth).sum() / np.abs(truth).sum())
        out[name]["l1_density_error_vs_refined_fp64"] = err
    if "l1_density_error_vs_refined_fp64" in out["fp64"]:
        e0 = out["fp64"]["l1_density_error_vs_refined_fp64"]
        for k in out:
            if "l1_density_error_vs_refined_fp64" in out[k]:
                out[k]["l1_error_ratio_vs_fp64"] = out[k]["l1_density_error_vs_refined_fp64"] / e0
    if finals.get("fp64") is not None:
        i = prob.info
        for k in ("mixed", "mixed_learned"):
            if finals.get(k) is None:
                continue
            A = finals[k].reshape(i.n_elem, i.n_fields, i.n_s)
            B = finals["fp64"].reshape(i.n_elem, i.n_fields, i.n_s)
            mom = max(np.abs(B[:, 1]).sum(), np.abs(B[:, 2]).sum())
            out[k]["per_field_rel_l1_vs_fp64"] = [
                float(np.abs(A[:, f] - B[:, f]).sum() / (mom if f in (1, 2) else np.abs(B[:, f]).sum()))
                for f in range(i.n_fields)]
    out["protocol"] = (f"{steps} timed SSP-RK3 steps each (L2 flushed); accuracy: {acc_steps} steps of dt = 0.8 x "
                       f"the initial CFL step, truth = plain FP64 on 1024x512 with dt/2, cell-averaged onto "
                       f"512x256; learned threshold 0.2, scored every {IND_EVERY} steps, network {meta.get('samples')} "
                       f"samples, held-out recall {meta.get('held_out', {}).get('0.2', {}).get('recall')}")
    return out


ENSEMBLE_SEED = 11
ENSEMBLE_T_END = 1e-4


def ensemble_cases(dgb, seed=ENSEMBLE_SEED):
    """The batched-ensemble workload: 192 1D two-fluid Riemann problems on [0,1] with element counts
    log-uniform in [200, 20000] and p uniform in {1, 2, 3}, and 64 2D four-quadrant Riemann problems
    on the unit square with square meshes of side log-uniform in [64, 512] (rounded to a multiple
    of 32), p = 2; all Rusanov, m2l, CFL 0.3, FP64, transmissive boundaries; seeded left/right and
    quadrant states (rho, p ~ U[0.1, 2], u, v ~ U[-1, 1], gamma in {1.4, 1.67})."""
    rng = np.random.default_rng(seed)
    cases = []
    for k in range(192):
        ne = int(round(np.exp(rng.uniform(np.log(200), np.log(20000)))))
        p = int(rng.integers(1, 4))
        prob = dgb.Problem.structured(1, p, ne, 1, 0.0, 1.0, bc=("transmissive",) * 2, flux="rusanov",
                                      limiter="m2l", cfl=CFL)
        cases.append((prob, prob.init_state("riemann", seed=1000 + k)))
    for k in range(64):
        n = int(32 * round(np.exp(rng.uniform(np.log(64), np.log(512))) / 32))
        prob = dgb.Problem.structured(2, 2, n, n, 0.0, 1.0, 0.0, 1.0, bc=("transmissive",) * 4, flux="rusanov",
                                      limiter="m2l", cfl=CFL)
        cases.append((prob, prob.init_state("quadrants", seed=2000 + k)))
    return cases


def ensemble(dgb, dev, steps, warmup):
    """Batched ensemble: all cases in one dgb_batch (a persistent launch per element class and
    operator, one CUDA graph per step), autotuned; against the same cases advanced one after another
    with dgb_advance.  Device time (CUDA events) over `steps` steps, each case with its own CFL
    step; then every case run to t = ENSEMBLE_T_END for the per-case completion times."""
    t0 = time.perf_counter()
    cases = ensemble_cases(dgb)
    setup_s = time.perf_counter() - t0
    solvers, starts = [], []
    for prob, U0 in cases:
        s = dgb.DGSolver(prob, device=dev)
        U = s.limit(U0)  # the reference limits the initial condition (rk.cc:108-114)
        s.set_state(U)
        solvers.append(s)
        starts.append(U)
    dof = np.array([p.info.n_elem * p.info.n_s * p.info.n_fields for p, _ in cases], dtype=np.float64)
    b = dgb.DGBatch(solvers)
    classes = b.autotune(5)
    b.advance(warmup)
    b.advance(steps)
    ms, launches = b.last_timing()
    _, case_steps, _ = b.case_stats()
    value = float((dof * case_steps).sum() * STAGES_PER_STEP / (ms / 1e3))
    # completion time of every case for a common end time
    for s, U in zip(solvers, starts):
        s.set_state(U)
    n_end = b.advance(100000, ENSEMBLE_T_END)
    end_ms, _ = b.last_timing()
    t_case, st_case, wall = b.case_stats()
    b.close()
    # the same cases one after another, each through its own context and graph
    seq_ms = 0.0
    for s, U in zip(solvers, starts):
        s.set_state(U)
        s.advance(warmup, 0.0, scheme=dgb.SSPRK3)
        s.advance(steps, 0.0, scheme=dgb.SSPRK3)
        seq_ms += s.last_timing()[0]
    for s in solvers:
        s.close()
    seq_value = float(dof.sum() * steps * STAGES_PER_STEP / (seq_ms / 1e3))
    w = np.sort(wall[wall >= 0])
    return {"workload": "192 1D Riemann (N_E log-uniform 200..20000, p 1-3) + 64 2D quadrants (64^2..512^2, p=2), "
                        "Rusanov, m2l, SSP-RK3, CFL 0.3 per case, FP64",
            "cases": len(cases), "dof_total": int(dof.sum()), "dof_1d": int(dof[:192].sum()),
            "dof_2d": int(dof[192:].sum()), "steps": steps,
            "value": value, "unit": UNIT, "ms_per_step": ms / steps, "gpu_launches_per_step": launches / max(steps, 1),
            "one_after_another": {"value": seq_value, "ms_per_step": seq_ms / steps},
            "speedup_vs_one_after_another": value / seq_value,
            "hbm_algorithmic_gbs": value * BYTES_PER_DOF_STAGE / 1e9,
            "classes": classes,
            "to_t_end": {"t_end": ENSEMBLE_T_END, "graph_steps": n_end, "ms": end_ms,
                         "case_steps_min_median_max": [int(st_case.min()), float(np.median(st_case)), int(st_case.max())],
                         "case_wall_ms_min_median_max": [float(w[0]), float(np.median(w)), float(w[-1])] if w.size else None,
                         "all_at_t_end": bool(np.all(t_case == ENSEMBLE_T_END))},
            "host_setup_s": setup_s}


TUBE_FIXTURE = ROOT / "tests" / "golden" / "run_d1_tube_p2_roe_m2l_1000.npz"


def tube_1d(dgb, dev, with_reference=True):
    """The 1D two-fluid shock tube: 1000 elements on [0, 1], p = 2, Roe, m2l, RK4 with the CFL step
    (CFL 0.4), transmissive ends, seeded +-1e-3 density noise, 2000 steps from the limited initial
    state.  Device time of the 2000 steps (one dgb_advance call, CUDA graph replays), the relative L1
    density distance from the reference's own 2000-step run (committed fixture), and the reference
    CPU build's wall time for the same 2000 steps (one process, one core)."""
    d = np.load(TUBE_FIXTURE)
    c = json.loads(str(d["meta"]))
    prob = dgb.Problem.structured(1, c["order"], c["nx"], 1, 0.0, 1.0, bc=("transmissive",) * 2, flux=c["flux"],
                                  limiter=c["limiter"], cfl=c["cfl"])
    info = prob.info
    dof = info.n_elem * info.n_s * info.n_fields
    s = dgb.DGSolver(prob, device=dev)
    s.set_state(d["U0"])
    s.advance(20, 0.0, scheme=dgb.RK4)  # warm-up (graph capture)
    s.set_state(d["U0"])
    t = s.advance(2000, 0.0, scheme=dgb.RK4)
    ms, launches = s.last_timing()
    U = s.get_state()
    s.close()
    A = U.reshape(info.n_elem, info.n_fields, info.n_s)[:, 0]
    B = d["U2000"].reshape(info.n_elem, info.n_fields, info.n_s)[:, 0]
    out = {"workload": "1D two-fluid shock tube, 1000 elements, p=2, Roe, m2l, RK4, CFL 0.4, 2000 steps",
           "dof": dof, "value": dof * 4 * 2000 / (ms / 1e3), "unit": UNIT, "ms_total": ms,
           "us_per_step": 1e3 * ms / 2000, "gpu_launches_per_step": launches / 2000, "time_reached": t,
           "rel_l1_density_vs_reference_run": float(np.abs(A - B).sum() / np.abs(B).sum())}
    if with_reference:
        from oracle.ref_run import RefCase, available
        if available(1, "roe"):
            case = RefCase(1, c["order"], c["nx"], 1, 0.0, 1.0, 0.0, 1.0, ("transmissive",) * 4, c["flux"],
                           c["limiter"])
            case.write_deck(cfl=c["cfl"])
            _, log = case.run("rk4n", d["U0"], dt=0.0, nsteps=2000, timeout=600)
            wall = float(log.split("DGREF_WALL_S")[1].split()[0])
            out["reference_cpu"] = {"value": dof * 4 * 2000 / wall, "unit": UNIT, "cores": 1, "kind": "reference",
                                    "wall_s": wall, "sample": "the same 2000 RK4 steps, reference step body, 1 process"}
            out["speedup_vs_reference_cpu"] = out["value"] / out["reference_cpu"]["value"]
    return out


DEPLOY_N, DEPLOY_STEPS, DEPLOY_SEED = 1024, 100, 4097


def learned_deploy(dgb, dev, timed=20, warmup=3, steps=DEPLOY_STEPS):
    """The learned indicator on its deployment problem: a seeded four-quadrant Riemann problem on
    1024 x 1024 quads, p = 2, Rusanov, m2l, SSP-RK3, CFL 0.3 (states as in the training set, a
    problem outside it).  Plain FP64 with the full limiter, mixed with the full limiter and mixed
    with the indicator-gated limiter (threshold 0.2, band of face neighbours, scored every
    IND_EVERY steps): device time per step, and after `steps` fixed steps the L1 density distance of each
    run from the plain FP64 full-limiter run (the judge) and the flagged / band fractions."""
    from dg_b200 import learned as L
    params, _ = L.load()
    prob = dgb.Problem.structured(2, 2, DEPLOY_N, DEPLOY_N, 0.0, 1.0, 0.0, 1.0, bc=("transmissive",) * 4,
                                  flux="rusanov", limiter="m2l", cfl=CFL)
    info = prob.info
    dof = info.n_elem * info.n_s * info.n_fields
    out = {"workload": "2D four-quadrant Riemann problem 1024x1024 quads, p=2, Rusanov, m2l, SSP-RK3, CFL 0.3",
           "dof": dof}
    U0, dt, finals = None, None, {}
    for name, form, learned in (("fp64", "fp64", False), ("mixed", "mixed", False), ("mixed_learned", "mixed", True)):
        s = dgb.DGSolver(prob, device=dev)
        s.set_form(form)
        if U0 is None:
            U0 = s.limit(prob.init_state("quadrants", seed=DEPLOY_SEED))
            dt = 0.8 * s.dt_from_cfl(U0)
        if learned:
            L.set_indicator(s, params, 0.2, every=IND_EVERY)
        s.set_state(U0)
        s.advance(warmup, 0.0, scheme=dgb.SSPRK3)
        s.advance(timed, 0.0, scheme=dgb.SSPRK3)
        ms, n = s.last_timing()
        out[name] = {"value": dof * STAGES_PER_STEP * timed / (ms / 1e3), "ms_per_step": ms / timed,
                     "gpu_launches_per_step": n / timed, "kernel_ms_per_step": kernel_breakdown(dgb, s)}
        s.set_state(U0)
        s.advance(steps, dt, scheme=dgb.SSPRK3)
        finals[name] = s.get_state()
        if learned:
            sc, cnt = L.scores(s, finals[name])
            out[name]["flagged_fraction_final"] = cnt / info.n_elem
        s.close()
    base = out["fp64"]["value"]
    rho = {k: v.reshape(info.n_elem, info.n_fields, info.n_s)[:, 0] for k, v in finals.items()}
    for k in out:
        if isinstance(out[k], dict) and "value" in out[k]:
            out[k]["speedup_vs_fp64"] = out[k]["value"] / base
            out[k]["l1_density_vs_fp64_full_limiter"] = float(np.abs(rho[k] - rho["fp64"]).sum() / np.abs(rho["fp64"]).sum())
    out["protocol"] = f"{timed} timed CFL steps after {warmup}; accuracy after {steps} steps of dt = 0.8 x the initial CFL step"
    return out


def mass_fraction(dgb, dev, base_ms, steps=20, warmup=3):
    """The benchmark workload with one passive mass fraction marking the bubble (rho Y = rho inside;
    6 fields): device time per step against the plain workload's (same protocol, L2 flushed by
    the 47 MB+ state being read once per stage; no extra flush here), and the Y total carried."""
    x0, x1, y0, y1 = DOMAIN
    prob = dgb.Problem.structured(2, ORDER, NX, NY, x0, x1, y0, y1, BC, flux="rusanov", limiter="m2l", cfl=CFL,
                                  n_mass=1)
    info = prob.info
    dof = info.n_elem * info.n_s * info.n_fields
    s = dgb.DGSolver(prob, device=dev)
    s.set_state(s.limit(prob.init_state("shock_bubble", seed=SEED)))
    c0 = s.conservation()
    s.advance(warmup, 0.0, scheme=dgb.SSPRK3)
    s.advance(steps, 0.0, scheme=dgb.SSPRK3)
    ms, _ = s.last_timing()
    c1 = s.conservation()
    s.close()
    return {"workload": "2D shock-bubble 512x256, p=2, Rusanov, m2l, SSP-RK3, CFL 0.3, one mass fraction (6 fields)",
            "dof": dof, "value": dof * STAGES_PER_STEP * steps / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / steps, "ms_per_step_without": base_ms,
            "rhoY_total_start_end": [float(c0[5]), float(c1[5])]}


def slab_local(dgb, dev, steps=10, warmup=3):
    """The benchmark workload as 2 and 4 y-slabs (2 ghost rows a side), every slab a context in
    this process on one GPU, ghost rows refreshed before every stage by device copies ordered by
    events between the slabs' streams, the CFL wave speed max-reduced over the slabs on the device.
    Wall time per step (the per-step status check synchronises the host), against the whole grid's
    device time per step, and the max distance of the owned rows from the whole grid after the same
    steps."""
    import time
    import torch
    from dg_b200 import slab as S
    x0, x1, y0, y1 = DOMAIN
    out = {"workload": "2D shock-bubble 512x256, p=2, Rusanov, m2l, SSP-RK3, CFL 0.3"}
    prob = dgb.Problem.structured(2, ORDER, NX, NY, x0, x1, y0, y1, BC, flux="rusanov", limiter="m2l", cfl=CFL)
    whole = dgb.DGSolver(prob, device=dev)
    U0 = whole.limit(prob.init_state("shock_bubble", seed=SEED))
    whole.set_state(U0)
    whole.advance(warmup, 0.0, scheme=dgb.SSPRK3)
    whole.advance(steps, 0.0, scheme=dgb.SSPRK3)
    ms, _ = whole.last_timing()
    ref = whole.get_state()
    whole.close()
    out["whole_ms_per_step"] = ms / steps
    for ns, captured in ((2, True), (4, True), (2, False)):
        dec = S.Decomposition(ORDER, NX, NY, ns, x0, x1, y0, y1, BC, flux="rusanov", limiter="m2l", cfl=CFL)
        run = S.SlabRun(dec, range(ns), S.LocalTransport(captured=captured), device=dev)
        try:
            run.set_global_state(U0)
            run.advance(warmup, 0.0, scheme=dgb.SSPRK3)
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            run.advance(steps, 0.0, scheme=dgb.SSPRK3)
            torch.cuda.synchronize(dev)
            wall = (time.perf_counter() - t0) * 1e3 / steps
            got = run.global_state()
        finally:
            run.close()
        out[f"slabs_{ns}" + ("" if captured else "_eager")] = {
            "rows": [r1 - r0 for r0, r1 in dec.ranges], "ms_per_step_wall": wall,
            "step": "one captured graph per step (dgb_slabs_advance_local)" if captured
            else "phase-level step driven from Python, eager launches",
            "max_abs_diff_vs_whole": float(np.abs(got - ref).max())}
    return out


def free_port() -> int:
    import socket
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_slab(args, dgb, ws, rank, dev):
    """--slab: one grid over all ranks.  The shock-bubble grid is 512 x (256 * ranks) elements on
    [0, 2] x [0, ranks] (weak scaling: every rank owns the element count of the 512 x 256 workload),
    split into one y-slab per rank with 2 ghost rows a side (dg_b200.slab.DistTransport): the ghost
    rows cross between neighbour ranks by NCCL send/receive on the context's stream before every
    stage, the CFL wave speed is MAX-all-reduced on the device, and the step's status once per step.
    One rank runs the same code in a single-rank group.  Device time per step: CUDA events on the
    slab's stream from the step's first to its last launch, summed over the timed steps, max over
    ranks."""
    import torch
    import torch.distributed as dist
    from dg_b200 import slab as S
    if not dist.is_initialized():
        dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{free_port()}", rank=0, world_size=1,
                                timeout=__import__("datetime").timedelta(seconds=120))
    x0, x1, y0, y1 = DOMAIN
    nyg = NY * ws
    dec = S.Decomposition(ORDER, NX, nyg, ws, x0, x1, y0, y1 * ws, BC, flux="rusanov", limiter="m2l", cfl=CFL)
    gprob = dec.global_problem()
    g = dgb.DGSolver(gprob, device=dev)  # the initial limiting of the whole grid (rk.cc:108-114)
    U0 = g.limit(gprob.init_state("shock_bubble", seed=SEED))
    g.close()
    run = S.SlabRun(dec, [rank], S.DistTransport(), device=dev)
    (slab,) = run.slabs
    run.set_global_state(U0)
    dof = gprob.info.n_elem * gprob.info.n_s * gprob.info.n_fields
    run.advance(max(args.warmup, 3), 0.0, scheme=dgb.SSPRK3)
    torch.cuda.synchronize(dev)
    dist.barrier()
    dev_ms, launches = 0.0, 0
    with Clocks(dev) as clk:
        for _ in range(args.steps):
            run.advance(1, 0.0, scheme=dgb.SSPRK3)
            ms, n = slab.solver.last_timing()
            dev_ms += ms
            launches += n
        torch.cuda.synchronize(dev)
    dist.barrier()
    clocks = clk.summary()
    t_s = max_over_ranks(dev_ms / 1e3, ws, f"cuda:{dev}")
    value = dof * STAGES_PER_STEP * args.steps / t_s
    # end to end: every step the rank's slab from host memory, one step, its owned rows back
    e2e_steps = max(args.e2e_steps, 1)
    n_slab = slab.problem.state_size
    n_owned = slab.owned().size
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        run.set_global_state(U0)
        run.advance(1, 0.0, scheme=dgb.SSPRK3)
        slab.owned()
    e2e_s = max_over_ranks(time.perf_counter() - t0, ws, f"cuda:{dev}")
    run.close()
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": 1e3 * t_s / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": config({"workload": f"2D shock-bubble {NX}x{nyg} quads on [0,2]x[0,{ws}] as {ws} y-slabs "
                                              f"(2 ghost rows a side), p=2, Rusanov, m2l, SSP-RK3, CFL 0.3",
                                  "n_elem": gprob.info.n_elem, "dof": dof,
                                  "parallelism": f"slab{ws}: one y-slab per rank, ghost rows by NCCL send/recv "
                                                 f"before every stage, wave speed MAX all-reduce per step",
                                  "l2": "not flushed (state per rank 48 MB, streamed 3x per step)"}),
                "e2e": {"value": dof * STAGES_PER_STEP * e2e_steps / e2e_s, "unit": UNIT,
                        "h2d_bytes_per_step": ws * n_slab * 8, "d2h_bytes_per_step": ws * n_owned * 8,
                        "steps": e2e_steps},
                "clocks": clocks, "gpu_launches": launches,
                "slab_rows": [r1 - r0 for r0, r1 in dec.ranges]}
        print(json.dumps(line))
    dist.barrier()
    dist.destroy_process_group()
    return 0


def gamma_models(dgb, dev, steps=20, warmup=3):
    """The benchmark grid (512 x 256, p=2, SSP-RK3, CFL 0.3) with Roe and hrl in both gamma models:
    GAMNCON (1/(gamma-1) with its non-conservative source) and GAMCONS (rho/(gamma-1) transported
    conservatively; the reference's M2limiting stops for it, hence hrl for both).  Device time per
    step and the total of the gamma-model field at the start and the end (conserved for GAMCONS up
    to the open x boundaries)."""
    x0, x1, y0, y1 = DOMAIN
    out = {"workload": "2D shock-bubble 512x256, p=2, Roe, hrl, SSP-RK3, CFL 0.3"}
    for gm in ("gamncon", "gamcons"):
        prob = dgb.Problem.structured(2, ORDER, NX, NY, x0, x1, y0, y1, BC, flux="roe", limiter="hrl", cfl=CFL,
                                      gamma_model=gm)
        info = prob.info
        dof = info.n_elem * info.n_s * info.n_fields
        s = dgb.DGSolver(prob, device=dev)
        s.set_state(s.limit(prob.init_state("shock_bubble", seed=SEED)))
        c0 = s.conservation()
        s.advance(warmup, 0.0, scheme=dgb.SSPRK3)
        s.advance(steps, 0.0, scheme=dgb.SSPRK3)
        ms, _ = s.last_timing()
        c1 = s.conservation()
        s.close()
        out[gm] = {"value": dof * STAGES_PER_STEP * steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / steps,
                   "gamma_field_total_start_end": [float(c0[4]), float(c1[4])]}
    return out


P3_NX, P3_NY, P3_STEPS = 2048, 1024, 300


def mixed_p3(dgb, dev, steps=P3_STEPS, timed=10):
    """The p=3 configuration: shock-bubble on 2048 x 1024 quads, p = 3, Roe, m2l, SSP-RK3, CFL 0.3.
    Throughput of the plain FP64 and the mixed form (same protocol as the headline, without the L2
    flush: the 2.7 GB state is 21x the L2), then both advanced `steps` CFL steps from the same
    state: per-field relative L1 and Linf error of the mixed form against the FP64 run, and the
    conserved totals (domain integrals of the five fields) of both at the start and the end."""
    prob = dgb.Problem.structured(2, 3, P3_NX, P3_NY, *DOMAIN, bc=BC, flux="roe", limiter="m2l", cfl=CFL)
    info = prob.info
    dof = info.n_elem * info.n_s * info.n_fields
    U0 = None
    out = {"workload": "2D shock-bubble 2048x1024 quads, p=3, Roe, m2l, SSP-RK3, CFL 0.3", "dof": dof}
    finals, totals = {}, {}
    for form in ("fp64", "mixed"):
        s = dgb.DGSolver(prob, device=dev)
        s.set_form(form)
        if U0 is None:
            U0 = s.limit(prob.init_state("shock_bubble", seed=SEED))
        s.set_state(U0)
        s.advance(3, 0.0, scheme=dgb.SSPRK3)
        s.advance(timed, 0.0, scheme=dgb.SSPRK3)
        ms, _ = s.last_timing()
        out[form] = {"value": dof * STAGES_PER_STEP * timed / (ms / 1e3), "ms_per_step": ms / timed}
        s.set_state(U0)
        c0 = s.conservation()
        try:
            t = s.advance(steps, 0.0, scheme=dgb.SSPRK3)
            finals[form] = s.get_state()
            totals[form] = (c0, s.conservation())
            out[form]["time_after_steps"] = t
        except dgb.DGBError as e:
            out[form]["failed"] = str(e)
        s.close()
    out["speedup_mixed_vs_fp64"] = out["mixed"]["value"] / out["fp64"]["value"]
    if len(finals) == 2:
        A = finals["mixed"].reshape(info.n_elem, info.n_fields, info.n_s)
        B = finals["fp64"].reshape(info.n_elem, info.n_fields, info.n_s)
        names = ("rho", "rho_u", "rho_v", "E", "alpha")
        l1, li = {}, {}
        for f, nm in enumerate(names):
            sc1 = np.abs(B[:, f]).sum() if f not in (1, 2) else max(np.abs(B[:, 1]).sum(), np.abs(B[:, 2]).sum())
            sci = np.abs(B[:, f]).max() if f not in (1, 2) else max(np.abs(B[:, 1]).max(), np.abs(B[:, 2]).max())
            l1[nm] = float(np.abs(A[:, f] - B[:, f]).sum() / sc1)
            li[nm] = float(np.abs(A[:, f] - B[:, f]).max() / sci)
        c0, r1 = totals["fp64"]
        _, m1 = totals["mixed"]
        scale = np.abs(c0).copy()
        scale[1:3] = np.abs(c0).max()
        out["after_steps"] = steps
        out["rel_l1_mixed_vs_fp64"] = l1
        out["rel_linf_mixed_vs_fp64"] = li
        out["conserved_totals"] = {"start": c0.tolist(), "fp64_end": r1.tolist(), "mixed_end": m1.tolist(),
                                   "mixed_minus_fp64_rel": ((m1 - r1) / scale).tolist(),
                                   "note": "totals change through the open (transmissive) x boundaries in both forms"}
    return out


PROFILE_CASES = ("p2step", "p2mixed", "p2learned", "deploylearned", "p3fp64", "p3mixed", "batch", "indicator")


def profile_case(dgb, dev, name):
    """A small run of one kernel family for an ncu capture (inputs larger than L2, a few launches,
    no timing): p2step -- 3 SSP-RK3 steps of the benchmark workload's problem at 1024 x 512 (p=2,
    Rusanov, m2l, FP64; 189 MB per state array); p2mixed -- the same in the mixed form; p2learned --
    9 steps of the 512 x 256 workload in the mixed form with the learned-indicator-gated limiter
    (scored every IND_EVERY steps); deploylearned -- the same 9 steps on the learned indicator's 1024^2
    four-quadrant deployment problem; p3fp64 / p3mixed -- 2 SSP-RK3 steps of the 1024 x 512 p=3 Roe shock-bubble in the
    FP64 / mixed form; batch -- 2 batched steps of 8 2D quadrant problems (256^2, p=2) and 8 1D
    Riemann problems (5000 elements, p=2); indicator -- 3 scorings of the 1024 x 512 p=2
    shock-bubble (after 10 steps) by the trained network."""
    if name in ("p2learned", "deploylearned"):
        from dg_b200 import learned as L
        if name == "p2learned":
            prob, U0 = build_problem()
        else:
            prob = dgb.Problem.structured(2, 2, DEPLOY_N, DEPLOY_N, 0.0, 1.0, 0.0, 1.0, bc=("transmissive",) * 4,
                                          flux="rusanov", limiter="m2l", cfl=CFL)
            U0 = prob.init_state("quadrants", seed=DEPLOY_SEED)
        s = dgb.DGSolver(prob, device=dev)
        s.set_form("mixed")
        L.set_indicator(s, L.load()[0], 0.2, every=IND_EVERY)
        s.set_state(s.limit(U0))
        s.advance(9, 0.0, scheme=dgb.SSPRK3)
        s.close()
    elif name in ("p2step", "p2mixed"):
        prob, U0 = build_problem(1024, 512)
        s = dgb.DGSolver(prob, device=dev)
        s.set_form("fp64" if name == "p2step" else "mixed")
        s.set_state(s.limit(U0))
        s.advance(3, 0.0, scheme=dgb.SSPRK3)
        s.close()
    elif name in ("p3fp64", "p3mixed"):
        prob = dgb.Problem.structured(2, 3, 1024, 512, *DOMAIN, bc=BC, flux="roe", limiter="m2l", cfl=CFL)
        s = dgb.DGSolver(prob, device=dev)
        s.set_form("fp64" if name == "p3fp64" else "mixed")
        s.set_state(s.limit(prob.init_state("shock_bubble", seed=SEED)))
        s.advance(2, 0.0, scheme=dgb.SSPRK3)
        s.close()
    elif name == "batch":
        solvers = []
        for k in range(8):
            prob = dgb.Problem.structured(2, 2, 256, 256, 0.0, 1.0, 0.0, 1.0, bc=("transmissive",) * 4,
                                          flux="rusanov", limiter="m2l", cfl=CFL)
            s = dgb.DGSolver(prob, device=dev)
            s.set_state(s.limit(prob.init_state("quadrants", seed=300 + k)))
            solvers.append(s)
        for k in range(8):
            prob = dgb.Problem.structured(1, 2, 5000, 1, 0.0, 1.0, bc=("transmissive",) * 2, flux="rusanov",
                                          limiter="m2l", cfl=CFL)
            s = dgb.DGSolver(prob, device=dev)
            s.set_state(s.limit(prob.init_state("riemann", seed=400 + k)))
            solvers.append(s)
        b = dgb.DGBatch(solvers)
        b.advance(2)
        b.close()
        for s in solvers:
            s.close()
    elif name == "indicator":
        from dg_b200 import learned as L
        prob, U0 = build_problem(1024, 512)
        s = dgb.DGSolver(prob, device=dev)
        s.set_state(s.limit(U0))
        s.advance(10, 0.0, scheme=dgb.SSPRK3)
        U = s.get_state()
        L.set_indicator(s, L.load()[0], 0.2, every=IND_EVERY)
        for _ in range(3):
            L.scores(s, U)
        s.close()
    else:
        raise ValueError(name)
    return 0


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=40)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=20)
    ap.add_argument("--nx", type=int, default=NX, help="elements in x (profiling cases; default the workload)")
    ap.add_argument("--ny", type=int, default=NY)
    ap.add_argument("--form", default="fp64", choices=["fp64", "mixed"],
                    help="arithmetic of the residual (fp64: the plain parity form)")
    ap.add_argument("--learned", action="store_true", help="gate the limiter with the learned indicator")
    ap.add_argument("--no-forms", action="store_true", help="skip the mixed / learned form comparison")
    ap.add_argument("--no-ensemble", action="store_true", help="skip the batched-ensemble measurement")
    ap.add_argument("--ensemble-only", action="store_true", help="print only the batched-ensemble measurement")
    ap.add_argument("--no-p3", action="store_true", help="skip the 2048x1024 p=3 FP64 / mixed comparison")
    ap.add_argument("--no-deploy", action="store_true", help="skip the learned indicator's 1024x1024 deployment")
    ap.add_argument("--deploy-only", action="store_true", help="print only the learned indicator's deployment")
    ap.add_argument("--profile-case", choices=PROFILE_CASES, help="run a small case of one kernel family for ncu")
    ap.add_argument("--no-tube", action="store_true", help="skip the 1D shock-tube run")
    ap.add_argument("--tube-only", action="store_true", help="print only the 1D shock-tube run")
    ap.add_argument("--p3-only", action="store_true", help="print only the 2048x1024 p=3 FP64 / mixed comparison")
    ap.add_argument("--slab-only", action="store_true",
                    help="print only the one-GPU slab-mode line (512x256 as 2 and 4 slabs)")
    ap.add_argument("--slab", action="store_true",
                    help="one grid over all ranks as y-slabs with NCCL halo exchange (weak scaling)")
    ap.add_argument("--models-only", action="store_true",
                    help="print only the mass-fraction and gamma-model lines (512x256, p=2)")
    args = ap.parse_args(argv)
    if args.impl == "reference":
        return run_reference(args)
    args.warmup = max(args.warmup, 3)

    import torch
    import torch.distributed as dist
    import dg_b200 as dgb

    ws, rank, local = dist_env()
    if ws > 1:
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    torch.cuda.set_device(local)
    dev = local
    if args.slab:
        return run_slab(args, dgb, ws, rank, dev)

    if args.profile_case:
        return profile_case(dgb, dev, args.profile_case)
    if args.tube_only:
        if rank == 0:
            print(json.dumps({"tube_1d": tube_1d(dgb, dev)}))
        return 0
    if args.deploy_only:
        if rank == 0:
            print(json.dumps({"learned_deploy": learned_deploy(dgb, dev)}))
        return 0
    if args.p3_only:
        if rank == 0:
            print(json.dumps({"mixed_p3": mixed_p3(dgb, dev)}))
        return 0
    if args.slab_only:
        if rank == 0:
            print(json.dumps({"slab_local": slab_local(dgb, dev)}))
        return 0
    if args.models_only:
        if rank == 0:
            print(json.dumps({"mass_fraction": mass_fraction(dgb, dev, None), "gamma_model": gamma_models(dgb, dev)}))
        return 0
    if args.ensemble_only:
        if rank == 0:
            print(json.dumps({"ensemble": ensemble(dgb, dev, min(args.steps, 20), args.warmup)}))
        return 0

    prob, U0 = build_problem(args.nx, args.ny)
    solver = dgb.DGSolver(prob, device=dev)
    solver.set_form(args.form)
    U0 = solver.limit(U0)  # the reference limits the initial condition when CFL > 0 (rk.cc:108-114)
    if args.learned:
        from dg_b200 import learned as L
        L.set_indicator(solver, L.load()[0], 0.2, every=IND_EVERY)
    solver.set_state(U0)
    dof = prob.info.n_elem * prob.info.n_s * prob.info.n_fields

    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=f"cuda:{dev}")
    ev_a = torch.cuda.Event(enable_timing=True)
    ev_b = torch.cuda.Event(enable_timing=True)

    for _ in range(args.warmup):
        solver.advance(1, 0.0, scheme=dgb.SSPRK3)
    torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    launches = 0
    dev_ms = 0.0
    with Clocks(dev) as clk:
        torch.cuda.synchronize()
        for _ in range(args.steps):
            flush.fill_(1.0)  # evict L2 (126 MB) before the step
            torch.cuda.synchronize()
            solver.advance(1, 0.0, scheme=dgb.SSPRK3)
            ms, n = solver.last_timing()  # CUDA events on the library stream around the step
            dev_ms += ms
            launches += n
        torch.cuda.synchronize()
    if ws > 1:
        dist.barrier()
    clocks = clk.summary()
    t_s = max_over_ranks(dev_ms / 1e3, ws, f"cuda:{dev}")
    value = whole_job_rate(ws, dof, args.steps, t_s)

    # per-kernel device time (profiled pass over the same number of steps, same state evolution)
    solver.set_profiling(True)
    solver.advance(args.steps, 0.0, scheme=dgb.SSPRK3)
    res_ms, res_n = solver.kernel_timing("residual")
    lim_ms, lim_n = solver.kernel_timing("limiter")
    dt_ms, dt_n = solver.kernel_timing("dt")
    ind_ms, _ = solver.kernel_timing("indicator")
    solver.set_profiling(False)
    res_avg_s = res_ms / 1e3 / max(res_n, 1)
    achieved_gbs = BYTES_PER_DOF_STAGE * dof / res_avg_s / 1e9
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    traffic, traffic_stages = None, None
    tf = ROOT / "profiles" / "residual2d_tile_p2_512x256_traffic.json"
    if tf.exists():
        tj = json.loads(tf.read_text())
        traffic = tj.get("bytes_per_launch_full_size")
        traffic_stages = {"stage1": tj.get("stage1_bytes_per_launch"), "stage2_3": tj.get("stage23_bytes_per_launch"),
                          "source": tj.get("measured_case")}

    # end to end through the C ABI with pinned host buffers: every step uploads the whole state,
    # advances it and downloads the result
    n_state = prob.state_size
    host = torch.empty(n_state, dtype=torch.float64, pin_memory=True)
    hostv = host.numpy()
    args.e2e_steps = max(args.e2e_steps, 1)
    # (a) the host-resident time loop (dgb_advance_host): one call for all steps, the copies
    # chunked so that a step's download and the next step's upload overlap
    hostv[:] = solver.get_state()
    solver.advance_host(hostv, 1, 0.0, scheme=dgb.SSPRK3)  # untimed: creates the copy streams
    t0 = time.perf_counter()
    solver.advance_host(hostv, args.e2e_steps, 0.0, scheme=dgb.SSPRK3)
    e2e_s = max_over_ranks(time.perf_counter() - t0, ws, f"cuda:{dev}")
    # (b) the same steps one call sequence per step: dgb_set_state, dgb_advance, dgb_get_state
    hostv[:] = solver.get_state()
    t0 = time.perf_counter()
    for _ in range(args.e2e_steps):
        solver.set_state(hostv)  # pinned host -> device, layout conversion
        solver.advance(1, 0.0, scheme=dgb.SSPRK3)
        solver.get_state(out=hostv)  # device -> the same pinned host buffer
    seq_s = max_over_ranks(time.perf_counter() - t0, ws, f"cuda:{dev}")
    e2e = {"value": whole_job_rate(ws, dof, args.e2e_steps, e2e_s), "unit": UNIT,
           "h2d_bytes_per_step": n_state * 8, "d2h_bytes_per_step": n_state * 8,
           "steps": args.e2e_steps,
           "api": "dgb_advance_host: per step the whole state pinned host -> device, one SSP-RK3 step, "
                  "the result device -> the same host buffer; wall clock",
           "per_step_calls": {"value": whole_job_rate(ws, dof, args.e2e_steps, seq_s), "unit": UNIT,
                              "api": "dgb_set_state + dgb_advance(1) + dgb_get_state per step (no copy overlap)"}}

    cpu = None
    if rank == 0 and ws == 1 and not args.no_cpu_baseline and (args.nx, args.ny) == (NX, NY):
        cpu = cpu_baseline(U0)
    forms = None
    if ws == 1 and not args.no_forms and (args.nx, args.ny) == (NX, NY):
        forms = compare_forms(dgb, U0, dev, args.steps, args.warmup, flush)

    ens = None
    if ws == 1 and not args.no_ensemble and (args.nx, args.ny) == (NX, NY):
        ens = ensemble(dgb, dev, min(args.steps, 20), args.warmup)
    p3 = None
    if ws == 1 and not args.no_p3 and (args.nx, args.ny) == (NX, NY):
        p3 = mixed_p3(dgb, dev)
    deploy = None
    if ws == 1 and not args.no_deploy and (args.nx, args.ny) == (NX, NY):
        deploy = learned_deploy(dgb, dev)
    mf = None
    if ws == 1 and not args.no_tube and (args.nx, args.ny) == (NX, NY):
        mf = mass_fraction(dgb, dev, dev_ms / args.steps)
    gms = None
    if ws == 1 and not args.no_tube and (args.nx, args.ny) == (NX, NY):
        gms = gamma_models(dgb, dev)
    slabs = None
    if ws == 1 and not args.no_tube and (args.nx, args.ny) == (NX, NY):
        slabs = slab_local(dgb, dev)
    tube = None
    if ws == 1 and not args.no_tube and (args.nx, args.ny) == (NX, NY):
        tube = tube_1d(dgb, dev, with_reference=rank == 0 and not args.no_cpu_baseline)

    form_cfg = {"form": ("plain FP64" if args.form == "fp64" else
                         "mixed: FP32 contractions/Rusanov flux on FP64 anchors, FP64 pressure, state and update")
                + (f" + learned indicator (threshold 0.2, scored every {IND_EVERY} steps)" if args.learned else "")}
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.form == "fp64" else "f64+f32",
                "data": "synthetic",
                "config": config(form_cfg) if (args.nx, args.ny) == (NX, NY) else config(
                    {"workload": f"profiling case {args.nx}x{args.ny} (not the benchmark workload)",
                     "n_elem": args.nx * args.ny, "dof": dof, **form_cfg}),
                "e2e": e2e,
                "roofline": {"bound": "hbm", "achieved": achieved_gbs, "peak": peak, "unit": "GB/s",
                             "frac": achieved_gbs / peak, "traffic": traffic,
                             "kernel": ("residual2d_tile_kernel<p=2,Rusanov,SSP> (fused residual + stage update)"
                                        if args.form == "fp64" else
                                        "residual2d_tile_mixed_kernel<p=2,Rusanov,SSP> (mixed form)"),
                             "algorithmic_bytes_per_launch": BYTES_PER_DOF_STAGE * dof,
                             "algorithmic_bytes_per_stage": {"stage1": 16.0 * dof, "stage2_3": 24.0 * dof},
                             "traffic_per_stage": traffic_stages,
                             "avg_launch_ms": res_avg_s * 1e3,
                             "avg_launch_ms_source": "CUDA events around each residual launch in a separate profiled "
                                                     "pass of the same number of steps (eager launches)",
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured copy)" if "hbm_gbs" in peaks
                             else "fallback 6650 GB/s (an earlier copy measurement on this pool; MEASURED_PEAKS.json absent)"},
                "kernel_ms_per_step": {"residual": res_ms / args.steps, "limiter": lim_ms / args.steps,
                                       "dt": dt_ms / args.steps,
                                       **({"indicator": ind_ms / args.steps} if args.learned else {}),
                                       "source": "separate profiled pass: eager launches, each kernel class "
                                                 "bracketed by CUDA events (adds launch gaps; the headline "
                                                 "ms_per_step is the captured graph's replay)"},
                "cpu_baseline": cpu, "clocks": clocks, "gpu_launches": launches, "forms": forms,
                "ensemble": ens, "mixed_p3": p3, "learned_deploy": deploy, "tube_1d": tube, "mass_fraction": mf,
                "gamma_model": gms, "slab_local": slabs}
        print(json.dumps(line))
    solver.close()
    if ws > 1:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
