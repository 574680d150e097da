"""Correctness beyond the short horizon, where trajectories are chaotic and only
answers and statistics can be compared (fixtures written by the reference itself,
tests/golden/make_golden_stats.py):

* MiniSat cross-check: 64 random 3-SAT instances N=60, M=256 near the threshold, made
  by the reference's RandomSatMaker, about half UNSAT by the reference's MiniSat.  The
  GPU solver (FP32 log-space and FP64, 64 starts per instance) must never report a
  solution of an UNSAT instance, every solution it reports must pass the exact clause
  check, and it must solve at least 95% of the SAT instances within 20,000 steps.
* Solve statistics against the reference CPU solver: the headline workload's
  instances (planted 3-SAT N=1000, M=4250), trajectories 0..3 of each (256 runs, the
  same initial states), every run to its own SatResult.  FP32 log-space on the GPU vs
  the reference CpuSat<double>: solved fractions within 0.03, median steps to the
  result within a factor 1.25, and the two step-count samples not distinguishable by
  a two-sample Kolmogorov-Smirnov test at the 0.1% level.  FP64 on the GPU: the same
  SatResult for every run whose step count equals the reference's (its trajectory
  stayed bit-identical), and that holds for at least half of the runs.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _minisat():
    return dict(np.load(os.path.join(HERE, "golden", "minisat_3sat.npz")))


@pytest.mark.parametrize("precision", [0, 1])
def test_gpu_answers_agree_with_minisat(precision):
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import initial_states, is_satisfied
    d = _minisat()
    n, m, k = (int(v) for v in d["nmk"])
    P, T = len(d["verdict"]), 64
    lens = np.full(m, k, np.int32)
    lits = [d["literals"][i].astype(np.int32) for i in range(P)]
    s = SatSolver([SatProblem.from_arrays(l, lens) for l in lits], precision=precision)
    s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(20000); s.SetMaxTime(1e8)
    s.SetStopOnFirst(True)
    dt = np.float32 if precision == 0 else np.float64
    pidx = np.repeat(np.arange(P), T).astype(np.int32)
    X = np.concatenate([initial_states(n, m, T, seed=900 + i, dtype=dt) for i in range(P)])
    s.SetSatStates(pidx, X)
    s.Solve()
    r = s.results()
    Y = s.GetSatStates(dt).reshape(P * T, n + m)
    solved = np.zeros(P, bool)
    for u in np.nonzero(r["status"] == 0)[0]:
        i = pidx[u]
        assert d["verdict"][i] == 10, f"solution reported for MiniSat-UNSAT instance {i}"
        assert is_satisfied(lits[i], lens, Y[u, :n] > 0)
        solved[i] = True
    sat = d["verdict"] == 10
    assert 0 < sat.sum() < P
    assert solved[sat].mean() >= 0.95, solved[sat].mean()
    # UNSAT instances run every start to the step limit
    unsat_units = ~sat[pidx]
    assert (r["status"][unsat_units] == 4).all()


def _reference_runs():
    return dict(np.load(os.path.join(HERE, "golden", "reference_runs_planted1000.npz")))


def _gpu_runs(precision):
    import bench
    from analogsat_b200 import SatProblem, SatSolver
    W = bench.WORKLOAD
    ref = _reference_runs()
    probs, pidx, ics = bench.make_workload(0, W["instances"], W["traj"])
    units = ref["units"]
    nm = W["n"] + W["m"]
    X = ics.reshape(-1, nm)[units]
    s = SatSolver([SatProblem.from_arrays(*p) for p in probs], precision=precision)
    s.SetEpsilon(W["eps"]); s.SetBatchSize(W["batch"]); s.SetMaxSteps(W["maxsteps"]); s.SetMaxTime(W["tmax"])
    s.SetSatStates(pidx[units], X if precision == 0 else X.astype(np.float64))
    s.Solve()
    return ref, s.results()


def test_f32_solve_statistics_match_reference_cpu():
    from scipy.stats import ks_2samp
    ref, r = _gpu_runs(0)
    f_ref = (ref["result"] == 0).mean()
    f_gpu = (r["status"] == 0).mean()
    med_ref = float(np.median(ref["steps"]))
    med_gpu = float(np.median(r["steps"]))
    ks = ks_2samp(ref["steps"], r["steps"])
    print(f"solved {f_gpu:.3f} vs reference {f_ref:.3f}; median steps {med_gpu:.0f} vs {med_ref:.0f}; "
          f"mean {r['steps'].mean():.0f} vs {ref['steps'].mean():.0f}; KS D={ks.statistic:.3f} p={ks.pvalue:.3g}")
    assert abs(f_gpu - f_ref) <= 0.03
    assert 1 / 1.25 <= med_gpu / med_ref <= 1.25
    assert ks.pvalue > 1e-3


def test_f64_runs_follow_reference_cpu():
    ref, r = _gpu_runs(1)
    same = r["steps"] == ref["steps"]
    print(f"FP64: {same.sum()} of {len(same)} runs take the reference's step count")
    assert same.mean() >= 0.5
    assert np.array_equal(r["status"][same], ref["result"][same].astype(np.int32))
