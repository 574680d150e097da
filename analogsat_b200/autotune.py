"""Project-written launch-shape autotuner for the persistent solver.

For an instance-size bucket (N and M rounded to powers of two, K, precision) it times
short fixed-length solves (a fixed number of accepted steps, all trajectories run to
the step cap, so every candidate does the same work) for a set of CTA sizes and both
storage modes the instance admits, keeps the fastest, and caches the choice in a JSON
file keyed by the bucket.  `apply(solver, problem)` sets the cached shape on a solver.

Timing uses CUDA events on the solver's launch stream; candidates that fail to launch
(e.g. a CTA size too small for the shared-memory footprint) are skipped.
"""
from __future__ import annotations

import json
import os
import time

import numpy as np

from . import AS_PREC_F32_LOGA, AnalogSatError, SatProblem, SatSolver
from .instances import initial_states

CACHE = os.environ.get("ANALOGSAT_B200_TUNE_CACHE",
                       os.path.join(os.path.expanduser("~"), ".cache", "analogsat_b200_tune.json"))
CANDIDATE_THREADS = (128, 256, 384, 512, 640, 768, 864, 1024)


def bucket(problem: SatProblem, precision: int) -> str:
    n, m, k = problem.n, problem.m, problem.k
    return f"p{precision}-k{k}-n{1 << max(0, (n - 1).bit_length())}-m{1 << max(0, (m - 1).bit_length())}"


def _load() -> dict:
    try:
        with open(CACHE) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _store(table: dict) -> None:
    os.makedirs(os.path.dirname(CACHE), exist_ok=True)
    tmp = CACHE + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, CACHE)


def time_shape(problem: SatProblem, precision: int, threads: int, storage: int, trajectories: int,
               steps: int, seed: int = 0) -> float:
    """Seconds for `trajectories` trajectories x `steps` accepted steps (no early exit)."""
    import torch
    s = SatSolver([problem], precision=precision)
    s.SetEpsilon(1e-6)
    s.SetBatchSize(steps)
    s.SetMaxSteps(steps)
    s.SetMaxTime(1e30)
    s.ForceThreads(threads)
    s.SetStorageMode(storage)
    dt = np.float32 if precision == AS_PREC_F32_LOGA else np.float64
    x = initial_states(problem.n, problem.m, trajectories, seed=seed, dtype=dt)
    pidx = np.zeros(trajectories, np.int32)
    st = torch.cuda.Stream()
    xd = torch.from_numpy(x).cuda()
    s.SetSatStates(pidx, xd, stream=st.cuda_stream)
    s.SolveAsync(stream=st.cuda_stream)  # warm-up (first launch sets kernel attributes)
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.SetSatStates(pidx, xd, stream=st.cuda_stream)
    with torch.cuda.stream(st):
        e0.record(st)
        s.SolveAsync(stream=st.cuda_stream)
        e1.record(st)
    st.synchronize()
    return e0.elapsed_time(e1) / 1e3


def tune(problem: SatProblem, precision: int = AS_PREC_F32_LOGA, trajectories: int | None = None,
         steps: int = 100, candidates=CANDIDATE_THREADS, save: bool = True) -> dict:
    """Time every candidate shape for this problem's bucket; cache and return the best."""
    from . import load
    sms = load().as_device_sm_count(-1)
    trajectories = trajectories or 2 * max(sms, 1)
    results = []
    for storage in (1, 2):
        for threads in candidates:
            try:
                t = time_shape(problem, precision, threads, storage, trajectories, steps)
            except AnalogSatError:
                continue
            results.append({"threads": threads, "storage": storage, "seconds": t})
    if not results:
        raise AnalogSatError(-4, "no launch shape could run this problem")
    best = min(results, key=lambda r: r["seconds"])
    entry = {"threads": best["threads"], "storage": best["storage"], "seconds": best["seconds"],
             "trajectories": trajectories, "steps": steps, "candidates": results,
             "when": time.strftime("%Y-%m-%dT%H:%M:%S")}
    if save:
        table = _load()
        table[bucket(problem, precision)] = entry
        _store(table)
    return entry


def lookup(problem: SatProblem, precision: int = AS_PREC_F32_LOGA) -> dict | None:
    return _load().get(bucket(problem, precision))


def apply(solver: SatSolver, problem: SatProblem) -> bool:
    """Set the cached best shape for `problem` on `solver`; False if the bucket is untuned."""
    e = lookup(problem, solver.precision)
    if not e:
        return False
    solver.ForceThreads(e["threads"])
    solver.SetStorageMode(e["storage"])
    return True
