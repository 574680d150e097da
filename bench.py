#!/usr/bin/env python
"""Headline benchmark: batched CTDS SAT solves on B200.

Workload (the at-scale GPU configuration): 64 planted random 3-SAT instances with
N=1000 variables and M=4250 clauses (alpha 4.25, uniform literals, random signs,
clauses violating a hidden assignment redrawn), 256 trajectories per instance,
s(0) ~ U(-1,1), a(0) = 1, FP32 state with a_m held as ln a_m, FP64 error norm and
time, Cash-Karp RK45 with eps = 1e-6, clause check every 50 steps, at most 1e5
steps per trajectory (the reference SatSolver's default maxSteps).  One bench "step"
runs all 16,384 trajectories to their SatResult in one persistent launch.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Metric: solves/s = instances solved per second.  The 256 trajectories of an instance
race from independent random starts and the first solution stops the others
(early exit on device); every reported solution passes the exact clause check.  The
reference's plain method solves an instance with one trajectory per Solve() call,
so its solves/s is Solve() calls that found a solution per second.  RHS
evaluations/s and trajectory-level counts are reported beside it
(--all-trajectories runs every trajectory to its own SatResult instead).  `value` is timed
with CUDA events with the initial states already in HBM; `e2e` goes through the
C ABI from pinned host buffers (H2D of the initial states, D2H of the results and
final states inside the timed region).

--impl reference times the reference AnalogSAT CPU solver (CpuSat<double> +
CpuRungeKutta<double> driven by SatSolver, compiled from the reference's sources)
with all host threads on a fixed sample of the same trajectories (trajectories 0
and 1 of every instance, each run to its own SatResult; the GPU line's
cpu_baseline is the same sample).

Multi-GPU (torchrun, one process per GPU): replicas -- every rank solves its own
64 instances x 256 trajectories (weak scaling, no data-path collective); the time
is the max over ranks.
"""
from __future__ import annotations

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

WORKLOAD = dict(name="planted-3sat-N1000-M4250-x64-inst-x256-traj", instances=64, n=1000,
                m=4250, k=3, traj=256, eps=1e-6, batch=50, maxsteps=100000, tmax=1e8)


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=WORKLOAD["instances"])
    ap.add_argument("--traj", type=int, default=WORKLOAD["traj"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-rhs-bench", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the comparators (FP64, every trajectory, plain GPU path) and the "
                         "other configurations (uneven batch, adjoint, MAXSAT)")
    ap.add_argument("--plain-seconds", type=float, default=20.0,
                    help="per precision: the plain GPU path starts runs while this budget lasts")
    ap.add_argument("--extras-maxsat-seconds", type=float, default=10.0)
    ap.add_argument("--no-autotune", action="store_true",
                    help="keep the default launch shape instead of the autotuned one")
    ap.add_argument("--threads", type=int, default=0,
                    help="force this CTA size for the solver (no autotuning)")
    ap.add_argument("--all-trajectories", action="store_true",
                    help="run every trajectory to its own SatResult (no early exit per instance)")
    ap.add_argument("--workload", default="planted1000",
                    choices=["planted1000", "uneven", "maxsat", "adjoint", "ingest"],
                    help="planted1000: the headline configuration; uneven: 512 planted instances "
                         "N~U{100..5000}, alpha~U(3.8,4.26), 64 trajectories each, one graph-captured "
                         "launch; maxsat: one random 4-SAT N=1e5, M=1e6 instance, 32 trajectories, "
                         "minimise unsat over --maxsat-seconds; adjoint: gradients of V at T=5 for "
                         "1024 random 3-SAT N=200, M=850 instances, FP32 vs FP64; ingest: GPU CNF "
                         "reader on the N=1e5, M=1e6 file and device-generated initial states")
    ap.add_argument("--maxsat-seconds", type=float, default=60.0)
    ap.add_argument("--maxsat-steps", type=int, default=0,
                    help="maxsat workload: stop every trajectory after this many steps (0: budget only)")
    ap.add_argument("--max-steps", type=int, default=WORKLOAD["maxsteps"],
                    help="per-trajectory step cap (profiling runs use a small one)")
    ap.add_argument("--n", type=int, default=0,
                    help="profiling runs: planted instances of this N (M = 4.25 N) instead of "
                         "N=1000; the bench line then names that workload")
    args = ap.parse_args()
    if args.n:
        m = int(round(4.25 * args.n))
        WORKLOAD.update(n=args.n, m=m, name=f"planted-3sat-N{args.n}-M{m}-x{args.instances}-inst-"
                                            f"x{args.traj}-traj")
    return args


def reduce_over_ranks(dist, sums, tmax, device):
    """Sum `sums` and take the max of `tmax` over all ranks (identity without dist).
    The replicas exchange nothing else: this is the only collective of the run."""
    if dist is None:
        return np.asarray(sums, np.float64), float(tmax)
    import torch
    s = torch.tensor(np.asarray(sums, np.float64), device=device)
    t = torch.tensor([float(tmax)], dtype=torch.float64, device=device)
    dist.all_reduce(s)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return s.cpu().numpy(), float(t.item())


def make_workload(rank: int, instances: int, traj: int):
    from analogsat_b200.instances import make_instance, initial_states
    W = WORKLOAD
    probs = []
    for i in range(instances):
        lits, lens, _ = make_instance("planted", W["n"], W["m"], W["k"], seed=2000 + 1000 * rank + i)
        probs.append((lits, lens))
    ics = np.concatenate([initial_states(W["n"], W["m"], traj, seed=10_000 * (rank + 1) + i,
                                         dtype=np.float32) for i in range(instances)])
    pidx = np.repeat(np.arange(instances), traj).astype(np.int32)
    return probs, pidx, ics


class Clocks:
    """nvidia-smi sampling during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        self.skip = 0
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return self
        # wait until the sampler runs, so that the samples kept are the timed region's
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 5.0 and self.p.poll() is None:
            self.f.flush()
            with open(self.f.name) as fh:
                n = sum(1 for _ in fh)
            if n:
                self.skip = n
                break
            time.sleep(0.01)
        return self

    def __exit__(self, *a):
        if self.p:
            # at least one sample from the timed region (or the instant after it)
            t0 = time.perf_counter()
            while time.perf_counter() - t0 < 0.5 and self.p.poll() is None:
                self.f.flush()
                with open(self.f.name) as fh:
                    if sum(1 for _ in fh) > self.skip:
                        break
                time.sleep(0.01)
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for i, line in enumerate(open(self.f.name)):
                parts = [x.strip() for x in line.split(",")]
                if i >= self.skip and len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons, "samples": len(rows)}


# The reference CPU sample: trajectories 0 and 1 of every instance (128 runs for the
# 64-instance workload), the same initial states the GPU solves, each run to its own
# SatResult under the same step cap.  A fixed set of runs, none cut short, so the rate
# does not depend on a time budget (a budget that drops long runs drops exactly the
# heavy tail of slow starts and overstates the rate).
CPU_SAMPLE_PER_INSTANCE = 2


def cpu_sample_units(instances: int, traj: int, per_instance: int = CPU_SAMPLE_PER_INSTANCE):
    """Unit indices of the CPU sample: trajectory j of instance i, j < per_instance, in
    round-robin order over the instances."""
    return np.array([i * traj + j for j in range(min(per_instance, traj)) for i in range(instances)],
                    np.int64)


def cpu_baseline(probs, pidx, ics, units, nthreads=None, maxsteps=None):
    """Reference CPU solver (oracle/_ref: CpuSat<double> + CpuRungeKutta<double> driven by
    SatSolver) on the given units of the workload, all host threads, every run to its own
    SatResult.  The rate is solved runs per second of thread-busy time times the threads:
    the runs' own wall seconds spread over the threads, so threads waiting idle for the
    last run are not charged.  With one start per Solve() (the reference's plain
    method), every solved run is one instance solved."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import Reference
    R = Reference()
    W = WORKLOAD
    ics = ics.reshape(len(pidx), -1)
    used = sorted(set(int(pidx[u]) for u in units))
    remap = {i: k for k, i in enumerate(used)}
    handles = [R.problem(*probs[i]) for i in used]
    units_p = np.array([remap[int(pidx[u])] for u in units], np.int32)
    units_x = [ics[u].astype(np.float64) for u in units]
    r = R.solve_many(handles, units_p, units_x, eps=W["eps"], tmax=W["tmax"],
                     maxsteps=maxsteps or W["maxsteps"], batch=W["batch"], nthreads=nthreads)
    assert int(r["done"].sum()) == len(units), "every run of the sample completes"
    solved = int((r["result"] == 0).sum())
    busy = float(r["busy"].sum()) / r["threads"]
    return dict(value=solved / busy, rhs_per_s=float(r["rhs"].sum()) / busy, wall=r["wall"],
                busy=busy, runs=len(units), solved=solved, threads=r["threads"],
                steps_mean=float(r["steps"].mean()), steps_median=float(np.median(r["steps"])),
                rhs_per_solve=float(r["rhs"].sum()) / max(solved, 1))


def cpu_sample_text(c, instances):
    return (f"{c['runs']} runs = trajectories 0..{c['runs'] // instances - 1} of each of the "
            f"{instances} instances (the GPU's own initial states), each run to its SatResult "
            f"(max_steps {WORKLOAD['maxsteps']}), none cut short: {c['solved']} solved, mean "
            f"{c['steps_mean']:.0f} / median {c['steps_median']:.0f} steps, {c['wall']:.1f} s wall; "
            f"reference CpuSat<double>+CpuRungeKutta<double> via SatSolver, {c['threads']} threads on "
            f"{cpu_name()}; rate = solved runs per second of thread-busy time x threads")


def cpu_name():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    probs, pidx, ics = make_workload(0, args.instances, args.traj)
    units = cpu_sample_units(args.instances, args.traj)
    threads = os.cpu_count() or 1
    for i in range(args.warmup):  # untimed: the first runs of the sample, capped short
        cpu_baseline(probs, pidx, ics, units[:threads], maxsteps=200)
    # the timed steps: the fixed sample dealt over the K steps (run u in step u mod K),
    # run back to back by all host threads; the value is over the whole sample
    order = np.concatenate([units[k::args.steps] for k in range(args.steps)])
    c = cpu_baseline(probs, pidx, ics, order)
    line = {
        "impl": "reference", "metric": "solves/s", "value": c["value"], "unit": "solves/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * c["wall"] / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD["name"], "instances": args.instances,
                   "trajectories_per_instance": args.traj, "N": WORKLOAD["n"], "M": WORKLOAD["m"],
                   "K": WORKLOAD["k"], "eps": WORKLOAD["eps"], "batch": WORKLOAD["batch"],
                   "max_steps": WORKLOAD["maxsteps"], "sample_runs": c["runs"]},
        "rhs_evals_per_s": c["rhs_per_s"],
        "cpu_baseline": {"value": c["value"], "unit": "solves/s", "cores": c["threads"],
                         "kind": "reference", "sample": cpu_sample_text(c, args.instances)},
        "e2e": {"value": c["value"], "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args):
    import torch
    import analogsat_b200 as A

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    W = WORKLOAD
    probs_raw, pidx, ics = make_workload(rank, args.instances, args.traj)
    probs = [A.SatProblem.from_arrays(l, n) for l, n in probs_raw]
    solver = A.SatSolver(probs, precision=A.AS_PREC_F32_LOGA, device=local)
    solver.SetEpsilon(W["eps"])
    solver.SetBatchSize(W["batch"])
    solver.SetMaxSteps(args.max_steps)
    solver.SetMaxTime(W["tmax"])
    solver.SetStopOnFirst(not args.all_trajectories)
    shape = None
    if args.threads:
        shape = {"threads": args.threads, "storage": 0}
        solver.ForceThreads(args.threads)
    elif not args.no_autotune:
        # launch shape (CTA size, storage mode) picked by timing fixed-work solves of
        # this instance size, outside the timed region (analogsat_b200/autotune.py)
        from analogsat_b200 import autotune
        best = autotune.tune(probs[0], A.AS_PREC_F32_LOGA, save=False)
        shape = {"threads": best["threads"], "storage": best["storage"]}
        solver.ForceThreads(shape["threads"])
        solver.SetStorageMode(shape["storage"])
    ics_dev = torch.from_numpy(ics).cuda()
    st = torch.cuda.Stream()
    nm = W["n"] + W["m"]
    B_rhs = 8 * nm + 4 * W["k"] * W["m"]  # algorithmic bytes per RHS evaluation (T_share = 1)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    def device_step():
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        with torch.cuda.stream(st):
            ev[0].record(st)
            solver.SetSatStates(pidx, ics_dev, stream=st.cuda_stream)
            ev[1].record(st)
            solver.SolveAsync(stream=st.cuda_stream)
            ev[2].record(st)
        return ev

    for _ in range(args.warmup):
        device_step()
        st.synchronize()
    r = solver.results()
    verify_solutions(solver, probs_raw, pidx, r, nm)

    barrier()
    totals = dict(solved=0, rhs=0, inst=0, steps_solved=[])
    evs = []
    with Clocks(local) as clk:
        barrier()
        for _ in range(args.steps):
            evs.append(device_step())
            st.synchronize()
            r = solver.results()
            totals["solved"] += int((r["status"] == 0).sum())
            totals["rhs"] += int(r["rhs"].sum())
            totals["inst"] += len(set(pidx[r["status"] == 0]))
            totals["steps_solved"] += list(r["steps"][r["status"] == 0])
        barrier()
    clocks = clk.summary()
    step_ms = [a.elapsed_time(c) for a, _, c in evs]
    kern_ms = [b.elapsed_time(c) for _, b, c in evs]
    t_total = sum(step_ms) / 1e3
    sums, t_max = reduce_over_ranks(dist, [totals["solved"], totals["rhs"], totals["inst"]], t_total,
                                    "cuda")
    solved_all, rhs_all, inst_all = sums

    rhs_line = rhs_kernel_bench(A, probs[0], ics_dev, nm, st) if not args.no_rhs_bench else None

    # end to end through the C ABI from pinned host buffers, two solver instances in a
    # pipeline: while one solves step k, the other receives step k+1's initial states
    # (host-to-device copy on its own stream); every step still copies its inputs in
    # and reads its results out
    e2e = None
    if not args.no_e2e:
        host_in = torch.from_numpy(ics).pin_memory().numpy()
        pair = [solver, A.SatSolver(probs, precision=A.AS_PREC_F32_LOGA, device=local)]
        other = pair[1]
        other.SetEpsilon(W["eps"]); other.SetBatchSize(W["batch"]); other.SetMaxSteps(args.max_steps)
        other.SetMaxTime(W["tmax"]); other.SetStopOnFirst(not args.all_trajectories)
        if shape:
            other.ForceThreads(shape["threads"])
            other.SetStorageMode(shape["storage"])

        def issue(s):
            s.SetSatStates(pidx, host_in)  # asynchronous from pinned memory
            s.SolveAsync()

        for s_ in pair:  # warm-up: captures each solver's graph
            issue(s_)
            s_.Sync()
        barrier()
        t0 = time.perf_counter()
        e_solved, d2h = 0, 0
        issue(pair[0])
        for k in range(args.steps):
            cur = pair[k % 2]
            if k + 1 < args.steps:
                issue(pair[(k + 1) % 2])
            cur.Sync()
            # the step's result: every trajectory's SatResult and counters, and the
            # final state (the satisfying assignment) of every solved trajectory
            r = cur.results()
            won = np.nonzero(r["status"] == 0)[0]
            for u in won:
                cur.GetSatState(int(u), np.float32)
            d2h += len(pidx) * 48 + 4 * nm * len(won)
            e_solved += (len(won) if args.all_trajectories else len(set(pidx[won])))
        barrier()
        t_e = time.perf_counter() - t0
        (e_solved,), t_e = reduce_over_ranks(dist, [e_solved], t_e, "cuda")
        e2e = {"value": e_solved / t_e, "unit": "solves/s", "h2d_bytes_per_step": int(ics.nbytes),
               "d2h_bytes_per_step": int(d2h // args.steps), "seconds": t_e,
               "result_read": "SatResult and counters of every trajectory + final state of each solved one",
               "pipeline": "two solver instances: step k+1's host-to-device copy overlaps step k's solve"}
        del other, pair

    if rank != 0:
        if dist is not None:
            dist.destroy_process_group()
        return

    # comparators and the other configurations (one GPU only: they are reported
    # beside the headline, not scaled)
    extras = {}
    if world == 1 and not args.no_extras:
        extras = bench_extras(args, A, probs, probs_raw, pidx, ics, shape)

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    hbm_peak = float(peaks.get("hbm_gbs", 6650.0))
    kern_s = sum(kern_ms) / 1e3
    achieved = (totals["rhs"] * B_rhs) / kern_s / 1e9
    headline = solved_all if args.all_trajectories else inst_all
    line = {
        "metric": "solves/s", "value": headline / t_max, "unit": "solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": W["name"], "instances_per_gpu": args.instances,
                   "stop_on_first": not args.all_trajectories,
                   "trajectories_per_instance": args.traj, "N": W["n"], "M": W["m"], "K": W["k"],
                   "eps": W["eps"], "batch": W["batch"], "max_steps": W["maxsteps"],
                   "state": "fp32, a in log space, fp64 error norm/time",
                   "l2": "state 344 MB per GPU > 126 MB L2 (no flush needed)",
                   "parallelism": f"replicas x{world}"},
        "rhs_evals_per_s": rhs_all / t_max,
        "instances_solved_per_s": inst_all / t_max,
        "trajectory_solves_per_s": solved_all / t_max,
        "instances_solved_fraction": totals["inst"] / (args.instances * args.steps),
        "median_steps_of_solved_trajectories": float(np.median(totals["steps_solved"]))
        if totals["steps_solved"] else None,
        "mode": "all trajectories to their own result" if args.all_trajectories
        else "first solution per instance stops its other trajectories",
        "gpu_launches": args.steps * len(solver_groups(solver)),
        "launch_shape": dict(solver.launch_shape(), autotuned=shape is not None and not args.threads),
        "roofline": {"bound": "hbm", "kernel": solver.kernel_name(), "achieved": achieved,
                     "peak": hbm_peak, "unit": "GB/s", "frac": achieved / hbm_peak,
                     # ncu dram__bytes_read+write of one solve_kernel_fast launch over 148
                     # trajectories (profiles/solve_kernel_fast_planted3sat_N1000_M4250.md):
                     # 3.29 MB, i.e. 22.3 KB per trajectory, scaled to this launch
                     "traffic": 3.294e6 / 148 * len(pidx),
                     "note": "achieved = RHS evals x 8(N+M)+4KM bytes / kernel time; state, "
                             "stages and contributions stay on chip (shared memory), so DRAM "
                             "traffic is far below the algorithmic bytes"},
        "clocks": clocks,
    }
    if line["roofline"]["kernel"] == "solve_kernel_fast" and W["n"] == 1000:
        # the kernel's actual limit is instruction issue: ncu counts 11.5k warp-instructions
        # per RHS for it on this instance size; the peak is 4 warp-instructions per cycle
        # on each SM at the SM clock sampled during the timed region
        sm_hz = float(clocks.get("sm_mhz") or 1965.0) * 1e6
        wi = 11.5e3 * (totals["rhs"] / kern_s)
        import torch
        peak_wi = 4 * sm_hz * torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
        line["roofline"]["issue"] = {"warp_instructions_per_rhs": 11.5e3, "achieved": wi / 1e9,
                                     "peak": peak_wi / 1e9, "unit": "G warp-instructions/s",
                                     "frac": wi / peak_wi}
    line.update(extras)
    # the metric's own ratios: the batched solver against the plain GPU path
    for name in ("f64", "f32"):
        pg = line.get("plain_gpu_path", {}).get(name, {})
        if pg.get("rhs_evals_per_s"):
            pg["ratio_rhs_evals"] = line["rhs_evals_per_s"] / pg["rhs_evals_per_s"]
            pg["ratio_solves"] = (line["value"] / pg["instances_solved_per_s"]
                                  if pg.get("instances_solved_per_s") else None)
    if e2e:
        line["e2e"] = e2e
    if rhs_line:
        rhs_line["peak"] = hbm_peak
        rhs_line["frac"] = rhs_line["achieved"] / hbm_peak
        line["rhs_roofline"] = rhs_line
    if world == 1 and not args.no_cpu_baseline:
        try:
            c = cpu_baseline(probs_raw, pidx, ics, cpu_sample_units(args.instances, args.traj))
            line["cpu_baseline"] = {
                "value": c["value"], "unit": "solves/s", "cores": c["threads"], "kind": "reference",
                "rhs_evals_per_s": c["rhs_per_s"], "rhs_per_solve": c["rhs_per_solve"],
                "sample": cpu_sample_text(c, args.instances)}
        except Exception as e:  # the checker library may be absent on a foreign box
            line["cpu_baseline"] = {"value": None, "unit": "solves/s", "cores": 0,
                                    "kind": "reference", "sample": f"unavailable: {e}"}
    print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def timed_solves(A, probs, pidx, X, precision, stop_on_first, steps, shape=None, max_steps=None):
    """Our solver on the given trajectories of the headline instances: `steps` timed
    solves after one warm-up, each from the same initial states (copied in on the
    device before the timing), CUDA events around SolveAsync on its stream."""
    import torch
    W = WORKLOAD
    s = A.SatSolver(probs, precision=precision)
    s.SetEpsilon(W["eps"]); s.SetBatchSize(W["batch"]); s.SetMaxSteps(max_steps or W["maxsteps"])
    s.SetMaxTime(W["tmax"])
    s.SetStopOnFirst(stop_on_first)
    if shape and precision == A.AS_PREC_F32_LOGA:
        s.ForceThreads(shape["threads"])
        s.SetStorageMode(shape["storage"])
    Xd = torch.from_numpy(np.ascontiguousarray(X)).cuda()
    st = torch.cuda.Stream()
    ms, solved, inst, rhs, steps_solved = 0.0, 0, 0, 0, []
    for k in range(steps + 1):
        s.SetSatStates(pidx, Xd, stream=st.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        s.SolveAsync(stream=st.cuda_stream)
        e1.record(st)
        st.synchronize()
        if k == 0:
            continue  # warm-up: launch groups and graph
        r = s.results()
        ms += e0.elapsed_time(e1)
        solved += int((r["status"] == 0).sum())
        inst += len(set(pidx[r["status"] == 0]))
        rhs += int(r["rhs"].sum())
        steps_solved += list(r["steps"][r["status"] == 0])
    sec = ms / 1e3
    out = {"seconds": sec, "steps": steps, "trajectories": int(len(pidx)),
           "instances_solved_per_s": inst / sec, "trajectory_solves_per_s": solved / sec,
           "instances_solved_fraction": inst / (steps * len(set(pidx.tolist()))),
           "rhs_evals_per_s": rhs / sec,
           "median_steps_of_solved_trajectories": float(np.median(steps_solved)) if steps_solved else None,
           "launch_shape": s.launch_shape()}
    del s, Xd
    return out


def plain_gpu_path(probs_raw, pidx, ics, units, precision, budget):
    """The reference's own CUDA path, the "plain GPU path": CudaSat1<T> + CudaRungeKutta<T>
    driven by SatSolver, one instance and one trajectory per Solve() in sequence, as the
    reference frontend runs it (Frontend/src/cnf_runner.cpp:28-127), built for sm_100a
    from the reference sources (oracle/_ref/libanalogsat_refcuda.so).  Runs the given
    units in order, starting new ones while the budget lasts; every started run goes to
    its own SatResult."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    from oracle import RefCuda
    W = WORKLOAD
    X = ics.reshape(len(pidx), -1)
    R = RefCuda()
    r = R.solve_many(probs_raw, pidx[units], [X[u].astype(np.float64) for u in units], precision=precision,
                     eps=W["eps"], tmax=W["tmax"], maxsteps=W["maxsteps"], batch=W["batch"], wall_budget=budget)
    d = int(r["done"])
    solved = int((r["result"][:d] == 0).sum())
    return {"instances_solved_per_s": solved / r["wall"], "rhs_evals_per_s": float(r["rhs"][:d].sum()) / r["wall"],
            "runs": d, "solved": solved, "seconds": r["wall"],
            "mean_steps": float(r["steps"][:d].mean()) if d else None,
            "sample": f"trajectory 0 of instances 0, 1, 2, ... of the headline workload (its initial states), "
                      f"started while a {budget:.0f} s budget lasted, each run to its SatResult"}


def bench_extras(args, A, probs, probs_raw, pidx, ics, shape):
    """Comparators of the headline and the other configurations, as extra keys."""
    out = {}
    W = WORKLOAD
    nm = W["n"] + W["m"]

    def guarded(key, fn):
        try:
            out[key] = fn()
        except Exception as e:  # one failed extra must not lose the headline line
            out[key] = {"error": f"{type(e).__name__}: {e}"}

    # FP64 on the headline workload (global-storage mode: an FP64 trajectory of this
    # size does not fit one SM's shared memory)
    guarded("f64", lambda: dict(timed_solves(A, probs, pidx, ics.astype(np.float64), A.AS_PREC_F64, True, 2),
                                mode="first solution per instance stops its other trajectories"))
    # every trajectory to its own SatResult (the like-for-like with the reference's
    # one start per Solve()): trajectories 0..7 of every instance
    units = cpu_sample_units(args.instances, args.traj, 8)
    guarded("all_trajectories", lambda: dict(
        timed_solves(A, probs, pidx[units], ics.reshape(-1, nm)[units], A.AS_PREC_F32_LOGA, False, 2, shape),
        mode="trajectories 0..7 of every instance, each to its own SatResult"))
    # restarts: the same workload with every start capped at 1,000 steps (a start that
    # has not solved by then ends with SAT_MAXITER_REACHED and the queue deals the next
    # start of some instance).  Single starts have a heavy-tailed step count (median 450,
    # mean 11.8k over the reference's own runs), so capped restarts cut the expected
    # work per solved instance; the headline keeps the reference's 1e5-step default.
    guarded("capped_starts", lambda: dict(
        timed_solves(A, probs, pidx, ics, A.AS_PREC_F32_LOGA, True, 3, shape, max_steps=1000),
        max_steps_per_start=1000, mode="first solution per instance stops its other trajectories"))
    # the plain GPU path in both precisions, on the first trajectories of the workload
    plain_units = cpu_sample_units(args.instances, args.traj, 2)
    for name, prec in (("f64", 1), ("f32", 0)):
        guarded(f"plain_{name}", lambda prec=prec: plain_gpu_path(probs_raw, pidx, ics, plain_units, prec,
                                                                    args.plain_seconds))
    plain = {"kernel_path": "reference CudaSat1<T> + CudaRungeKutta<T> via SatSolver, sm_100a"}
    for name in ("f64", "f32"):
        plain[name] = out.pop(f"plain_{name}")
    out["plain_gpu_path"] = plain
    # the other configurations
    guarded("uneven", lambda: bench_uneven(2, WORKLOAD["maxsteps"]))
    guarded("adjoint", bench_adjoint)
    guarded("maxsat", lambda: bench_maxsat(args.extras_maxsat_seconds))
    return out


def rhs_kernel_bench(A, problem, ics_dev, nm, st, reps=10):
    """Standalone batched RHS (ISat::GetDerivatives) over every trajectory's state,
    state in HBM (16,384 x 5,250 FP32 = 344 MB in, 344 MB out per launch)."""
    import torch
    x = ics_dev.view(-1, nm)
    out = torch.empty_like(x)
    B = x.shape[0]
    W = WORKLOAD
    with torch.cuda.stream(st):
        for _ in range(3):
            A.get_derivatives(problem, x, out=out, logspace=False, stream=st.cuda_stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(reps):
            A.get_derivatives(problem, x, out=out, logspace=False, stream=st.cuda_stream)
        e1.record(st)
    st.synchronize()
    ms = e0.elapsed_time(e1) / reps
    # algorithmic bytes: state in + derivative out, and the instance's literal stream once
    # per launch (T_share = all B states of the launch)
    bytes_per_launch = B * 8 * nm + 4 * W["k"] * W["m"]
    # traffic: ncu dram__bytes_read + dram__bytes_write of one launch of this exact
    # configuration (profiles/rhs_pair_kernel_16384_states_N1000_M4250.md)
    kernel = "rhs_pair_kernel" if x.dtype == torch.float32 else "rhs_batch_kernel"
    return {"bound": "hbm", "kernel": kernel, "states_per_launch": B,
            "ms_per_launch": ms, "achieved": bytes_per_launch / (ms / 1e3) / 1e9, "unit": "GB/s",
            "bytes_per_launch": bytes_per_launch,
            "traffic": 640.34e6 if B == 16384 else None}


def solver_groups(solver):
    return [0]  # one launch shape: all 64 instances share N, M, K


def verify_solutions(solver, probs_raw, pidx, r, nm):
    """Exact clause check of every reported solution (on the host, warm-up only)."""
    from analogsat_b200.instances import is_satisfied
    X = solver.GetSatStates(np.float32).reshape(len(pidx), nm)
    n = WORKLOAD["n"]
    bad = 0
    for u in np.nonzero(r["status"] == 0)[0][:512]:
        lits, lens = probs_raw[pidx[u]]
        bad += not is_satisfied(lits, lens, X[u, :n] > 0)
    if bad:
        raise SystemExit(f"{bad} reported solutions failed the exact clause check")


def run_uneven(args):
    print(json.dumps(bench_uneven(args.steps, args.max_steps)), flush=True)


def bench_uneven(steps: int, max_steps: int):
    """512 planted 3-SAT instances of uneven size, 64 trajectories each, first solution per
    instance stops the rest; the whole batch is one graph-captured solve call (shared-
    memory launch group for instances that fit one SM, global-storage group for the rest)."""
    import torch
    import analogsat_b200 as A
    from analogsat_b200.instances import make_instance, initial_states
    rng = np.random.default_rng(3000)
    P, T = 512, 64
    ns = rng.integers(100, 5001, size=P)
    alphas = rng.uniform(3.8, 4.26, size=P)
    raw, sizes = [], []
    t0 = time.perf_counter()
    for i in range(P):
        n = int(ns[i]); m = int(np.floor(alphas[i] * n))
        lits, lens, _ = make_instance("planted", n, m, 3, seed=3000 + i)
        raw.append((lits, lens)); sizes.append((n, m))
    probs = [A.SatProblem.from_arrays(l, c) for l, c in raw]
    s = A.SatSolver(probs)
    s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(max_steps); s.SetMaxTime(1e8)
    s.SetStopOnFirst(True)
    pidx = np.repeat(np.arange(P), T).astype(np.int32)
    X = np.concatenate([initial_states(n, m, T, seed=40_000 + i, dtype=np.float32)
                        for i, (n, m) in enumerate(sizes)], axis=None)
    setup = time.perf_counter() - t0
    s.SetSatStates(pidx, X)
    s.Solve()  # warm-up: builds launch groups, captures the graph
    shape = s.launch_shape()
    walls, solved, rhs = [], 0, 0
    for _ in range(steps):
        s.SetSatStates(pidx, X)
        torch.cuda.synchronize()
        t1 = time.perf_counter()
        s.Solve()
        walls.append(time.perf_counter() - t1)
        r = s.results()
        solved += len(set(pidx[r["status"] == 0]))
        rhs += int(r["rhs"].sum())
    wall = sum(walls)
    small = sum(1 for p in probs if p.layout_stats()["compact"] and p.n <= 1200)
    return {"workload": "uneven-planted-3sat-512-inst-N100-5000-x64-traj", "instances": P,
            "trajectories_per_instance": T, "solves/s": solved / wall,
            "instances_solved_fraction": solved / (P * steps),
            "rhs_evals_per_s": rhs / wall, "ms_per_solve_call": 1000 * wall / steps, "steps": steps,
            "setup_s": setup, "last_group_launch_shape": shape, "instances_N_le_1200": small,
            "timing": "wall clock around each Solve() (states set before, outside the timing)"}


def run_maxsat(args):
    print(json.dumps(bench_maxsat(args.maxsat_seconds, args.maxsat_steps)), flush=True)


def bench_maxsat(seconds: float, max_steps: int = 0):
    """One random 4-SAT instance N=1e5, M=1e6 (alpha 10, unsatisfiable w.h.p.), 32
    trajectories, minimise the unsat-clause count within a wall-clock budget; the best
    assignment of every trajectory is kept on device and re-counted exactly here."""
    import analogsat_b200 as A
    from analogsat_b200.instances import make_instance, initial_states
    n, m, k, T = 100_000, 1_000_000, 4, 32
    lits, lens, _ = make_instance("fast", n, m, k, seed=5000)
    p = A.SatProblem.from_arrays(lits, lens)
    s = A.SatSolver([p])
    steps = max_steps if max_steps > 0 else 10 ** 9
    s.SetEpsilon(1e-6); s.SetBatchSize(min(10, steps)); s.SetMaxSteps(steps); s.SetMaxTime(1e30)
    s.SetTrackBest(True)
    s.SetWallBudget(seconds)
    X = initial_states(n, m, T, seed=50_000, dtype=np.float32)
    s.SetSatStates(np.zeros(T, np.int32), X)
    t0 = time.perf_counter()
    s.Solve()
    wall = time.perf_counter() - t0
    r = s.results()
    c = lits.reshape(-1, k)
    v = np.abs(c) - 1
    exact = []
    for t in range(T):
        best = s.GetBestAssignment(t)
        exact.append(int((~np.where(c > 0, best[v], ~best[v]).any(axis=1)).sum()))
    assert exact == list(r["min_violations"]), "device min-unsat disagrees with the host recount"
    rhs_s = float(r["rhs"].sum()) / wall
    try:
        hbm_peak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))).get("hbm_gbs", 6650.0))
    except OSError:
        hbm_peak = 6650.0
    # streamed mode, eight trajectories per lane group: the literal words are read once
    # per group and RHS, so B_rhs = 8(N+M) + 4KM/8 per trajectory and RHS
    b_rhs = 8 * (n + m) + 4 * k * m / 8
    return {"workload": "maxsat-random-4sat-N1e5-M1e6-x32-traj", "wall_s": wall,
                      "budget_s": seconds, "min_unsat": int(min(exact)),
                      "median_min_unsat": float(np.median(exact)), "steps_median": float(np.median(r["steps"])),
                      "rhs_evals_per_s": rhs_s,
                      "roofline": {"bound": "hbm", "achieved": rhs_s * b_rhs / 1e9, "peak": hbm_peak,
                                   "unit": "GB/s", "frac": rhs_s * b_rhs / 1e9 / hbm_peak,
                                   "note": "achieved = RHS/s x B_rhs (T_share 8); the stage vectors of the "
                                           "clause weights and the contribution intermediate are extra HBM "
                                           "traffic B_rhs leaves out (~12 GB per pass of 192 RHS, "
                                           "profiles/stream_kernels_maxsat_N1e5_M1e6.md)"},
                      "launch_shape": s.launch_shape()}


def run_adjoint(args):
    print(json.dumps(bench_adjoint()), flush=True)


def bench_adjoint():
    """Gradients of V = sum w a K^2 at T=5 w.r.t. s(0), a(0) and per-clause weights for
    1024 random 3-SAT instances (N=200, M=850), FP32 and FP64; reports gradients per
    second, the FP32-vs-FP64 relative error, and one descent step on a(0) lowering V."""
    import analogsat_b200 as A
    from analogsat_b200.instances import make_instance, initial_states
    P, n, m = 1024, 200, 850
    raw = [make_instance("random", n, m, 3, seed=6000 + i)[:2] for i in range(P)]
    probs = [A.SatProblem.from_arrays(l, c) for l, c in raw]
    X = np.concatenate([initial_states(n, m, 1, seed=60_000 + i) for i in range(P)])
    w = np.random.default_rng(6).uniform(0.5, 1.5, size=P * m)
    out = {}
    for prec, dt in ((A.AS_PREC_F32_LOGA, np.float32), (A.AS_PREC_F64, np.float64)):
        s = A.SatSolver(probs, precision=prec)
        s.SetEpsilon(1e-6)
        s.SetSatStates(np.arange(P, dtype=np.int32), X.astype(dt))
        s.Adjoint(5.0, weights=w)  # warm-up
        t0 = time.perf_counter()
        g = s.Adjoint(5.0, weights=w)
        out[prec] = (time.perf_counter() - t0, g, s)
    t32, g32, s32 = out[A.AS_PREC_F32_LOGA]
    t64, g64, s64 = out[A.AS_PREC_F64]
    rel = lambda a, b: float(np.linalg.norm(a - b) / np.linalg.norm(b))
    # one projected descent step on a(0) (clause weights' initial values) with FP64 gradients
    Xr = X.reshape(P, n + m)
    ga = g64["grad_x0"].reshape(P, n + m)[:, n:]
    step = 0.5 / np.maximum(np.abs(ga).max(axis=1, keepdims=True), 1e-30)
    X2 = Xr.copy()
    X2[:, n:] = np.maximum(Xr[:, n:] - step * ga, 1e-3)
    s64.SetSatStates(np.arange(P, dtype=np.int32), X2)
    g2 = s64.Adjoint(5.0, weights=w)
    return {"workload": "adjoint-random-3sat-N200-M850-x1024-T5",
                      "fp32_s": t32, "fp64_s": t64, "gradients_per_s_fp32": P / t32,
                      "gradients_per_s_fp64": P / t64, "median_steps": float(np.median(g64["nsteps"])),
                      "fp32_vs_fp64_rel_err_grad_x0": rel(g32["grad_x0"], g64["grad_x0"]),
                      "fp32_vs_fp64_rel_err_grad_w": rel(g32["grad_w"], g64["grad_w"]),
                      "fp32_vs_fp64_rel_err_loss": rel(g32["loss"], g64["loss"]),
                      "mean_loss_before_a0_step": float(g64["loss"].mean()),
                      "mean_loss_after_a0_step": float(g2["loss"].mean()),
                      "timing": "wall clock around one as_solver_adjoint call after a warm-up call"}


def run_ingest(args):
    """Device-side ingest at the large-instance size.  CNF: the random 4-SAT instance
    N=1e5, M=1e6 as a DIMACS file (about 27 MB) read by the host reader, by the
    reference's CnfReader (CPU baseline, when built) and by the GPU tokeniser; wall
    time of each complete read (file to host clause arrays).  Initial states: the FP32
    batch of 64 x 256 trajectories of N=1000, M=4250 (86M values, 344 MB) generated in
    HBM, against numpy's generator plus the host-to-device copy."""
    import shutil
    import analogsat_b200 as A
    from analogsat_b200.instances import make_instance, initial_states

    def best_of(fn, reps):
        t = []
        for _ in range(max(1, reps)):
            t0 = time.perf_counter()
            fn()
            t.append(time.perf_counter() - t0)
        return min(t)

    lits, lens, _ = make_instance("fast", 100_000, 1_000_000, 4, seed=5000)
    d = tempfile.mkdtemp()
    try:
        f = os.path.join(d, "random-4sat-N1e5-M1e6.cnf")
        A.SatProblem.from_arrays(lits, lens).write_cnf(f)
        size = os.path.getsize(f)
        q = A.SatProblem.read_cnf(f, device=0)  # warm-up, and the exactness check
        ql, qn = q.GetAllClauses()
        assert np.array_equal(ql, lits) and np.array_equal(qn, lens)
        dev = best_of(lambda: A.SatProblem.read_cnf(f, device=0), args.steps)
        host = best_of(lambda: A.SatProblem.read_cnf(f), 2)
        ref = None
        if os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libanalogsat_ref.so")):
            sys.path.insert(0, os.path.join(ROOT, "oracle"))
            from oracle import Reference
            R = Reference()
            ref = best_of(lambda: R.read_cnf(f), 1)
    finally:
        shutil.rmtree(d, ignore_errors=True)
    n, m, T = 1000, 4250, 64 * 256
    pl, pn, _ = make_instance("planted", n, m, 3, seed=2000)
    s = A.SatSolver([A.SatProblem.from_arrays(pl, pn)], precision=0)
    pidx = np.zeros(T, np.int32)
    s.SetRandomInitialState(pidx, seed=1)  # warm-up (allocates the state buffer)
    ic_dev = best_of(lambda: s.SetRandomInitialState(pidx, seed=1), args.steps)

    def host_path():
        s.SetSatStates(pidx, initial_states(n, m, T, seed=1, dtype=np.float32))
    ic_host = best_of(host_path, 2)
    vals = T * (n + m)
    print(json.dumps({"workload": "ingest-cnf-random-4sat-N1e5-M1e6-and-states-64x256-N1000-M4250",
                      "cnf_bytes": size, "cnf_read_s": {"device": dev, "host": host, "reference": ref},
                      "cnf_device_GB_per_s": size / dev / 1e9,
                      "states": {"values": vals, "bytes_fp32": 4 * vals, "device_s": ic_dev,
                                 "numpy_plus_h2d_s": ic_host,
                                 "device_GB_per_s": 4 * vals / ic_dev / 1e9},
                      "note": "wall time per complete call through the C ABI, best of the repeats; "
                              "kernel shares in profiles/ingest_kernels_cnf_N1e5_M1e6.md"}), flush=True)


def main():
    args = parse_args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "uneven":
        run_uneven(args)
    elif args.workload == "maxsat":
        run_maxsat(args)
    elif args.workload == "adjoint":
        run_adjoint(args)
    elif args.workload == "ingest":
        run_ingest(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
