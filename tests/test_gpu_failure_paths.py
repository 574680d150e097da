"""Failure paths of the solver, every fault injected on the host (no device fault):

* initial states holding NaN or infinite spins or clause weights, all-zero weights
  and negative weights, whose dynamics blow up in finite time so that the step size
  underflows (SAT_UNDERFLOW, AnalogSAT/cpu_sat/CpuRungeKutta.cpp:246-248, reported by
  SatSolver.h:322): the FP64 solver reproduces the reference's SatResult and counters
  (through the oracle, which tests/test_oracle.py pins to the reference itself on
  exactly these inputs);
* the smallest epsilon SetEpsilon accepts (1e-16: same SatResult and steps as the
  reference, the RHS count within 1%, since decisions at the rounding floor follow
  the last bit of pow()) and the out-of-range ones it rejects
  (CpuRungeKutta.cpp:127-131);
* wall-clock budgets: 0 is "no budget", a budget that runs out before the first
  check interrupts every trajectory (SAT_ODE_INTERRUPTED), negative budgets and
  other bad parameters are refused with AS_ERR_BAD_INPUT.
"""
import numpy as np
import pytest

from test_oracle import FAILURE_CASES, failure_ic

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


def _solver(golden, precision, eps=1e-6, maxsteps=20000, batch=50, tmax=1e8):
    from analogsat_b200 import SatProblem, SatSolver
    p = SatProblem.from_arrays(golden["p50/literals"], golden["p50/lengths"])
    s = SatSolver([p], precision=precision)
    s.SetEpsilon(eps); s.SetBatchSize(batch); s.SetMaxSteps(maxsteps); s.SetMaxTime(tmax)
    return s


@pytest.mark.parametrize("case", sorted(FAILURE_CASES))
def test_failure_ics_f64_follow_reference(oracle, golden, case):
    from analogsat_b200 import AS_PREC_F64
    x = failure_ic(golden, case)
    s = _solver(golden, AS_PREC_F64)
    s.SetSatStates([0], x[None, :])
    s.Solve()
    r = s.results()
    o = oracle.solve(oracle.problem(golden["p50/literals"], golden["p50/lengths"]), x, eps=1e-6,
                     maxsteps=20000, batch=50, tmax=1e8)
    assert r["status"][0] == o["result"], (case, r["status"][0], o["result"])
    for k, ok in (("steps", "steps"), ("rhs", "rhs"), ("attempts", "attempts"),
                  ("violations", "violations")):
        assert r[k][0] == o[ok], (case, k, r[k][0], o[ok])
    assert abs(r["time"][0] - o["time"]) <= 1e-9 * abs(o["time"])
    if case == "negative_weights":
        assert r["status"][0] == 1  # SAT_UNDERFLOW


@pytest.mark.parametrize("case", ["nan_spin", "inf_spin", "nan_weight", "zero_weights"])
def test_failure_ics_f32_defined_status(oracle, golden, case):
    """FP32 with log-space weights: NaN error ratios are skipped by the max norm as in
    the reference, so these end with the same SatResult as the FP64 run (negative
    weights have no logarithm: the FP32 solver requires a >= 0)."""
    from analogsat_b200 import AS_PREC_F32_LOGA, AS_PREC_F64
    x = failure_ic(golden, case)
    out = {}
    for prec, dt in ((AS_PREC_F32_LOGA, np.float32), (AS_PREC_F64, np.float64)):
        s = _solver(golden, prec)
        s.SetSatStates([0], x[None, :].astype(dt))
        s.Solve()
        out[prec] = s.results()
    assert out[AS_PREC_F32_LOGA]["status"][0] == out[AS_PREC_F64]["status"][0]
    assert out[AS_PREC_F32_LOGA]["violations"][0] == out[AS_PREC_F64]["violations"][0]


def test_smallest_epsilon_follows_reference_and_bad_parameters_are_refused(oracle, golden):
    from analogsat_b200 import AS_PREC_F64, AnalogSatError
    from analogsat_b200._abi import AS_ERR_BAD_INPUT
    ic = golden["p50/solve_ics"][0]
    s = _solver(golden, AS_PREC_F64, eps=1e-16)
    s.SetSatStates([0], ic[None, :])
    s.Solve()
    r = s.results()
    o = oracle.solve(oracle.problem(golden["p50/literals"], golden["p50/lengths"]), ic, eps=1e-16,
                     maxsteps=20000, batch=50, tmax=1e8)
    # at the rounding floor an error ratio sits within an ulp of eps, so a last-bit
    # difference of the controller's pow() (CUDA's against glibc's) can flip a few
    # accept/reject decisions: same SatResult and steps, RHS count within 1%
    assert (r["status"][0], r["steps"][0]) == (o["result"], o["steps"])
    assert abs(int(r["rhs"][0]) - o["rhs"]) <= 0.01 * o["rhs"]
    for bad in (lambda: s.SetEpsilon(9e-17), lambda: s.SetEpsilon(1.5), lambda: s.SetEpsilon(float("nan")),
                lambda: s.SetMaxSteps(0), lambda: s.SetBatchSize(0), lambda: s.SetMaxTime(0.0),
                lambda: s.SetWallBudget(-1.0), lambda: s.SetWallBudget(float("nan"))):
        with pytest.raises(AnalogSatError) as e:
            bad()
        assert e.value.code == AS_ERR_BAD_INPUT


def test_wall_budgets(golden):
    from analogsat_b200 import AS_PREC_F32_LOGA, SatResult
    ics = golden["p1000/solve_ics"][:4].astype(np.float32)
    from analogsat_b200 import SatProblem, SatSolver
    p = SatProblem.from_arrays(golden["p1000/literals"], golden["p1000/lengths"])

    def run(budget):
        s = SatSolver([p], precision=AS_PREC_F32_LOGA)
        s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(400); s.SetMaxTime(1e8)
        s.SetWallBudget(budget)
        s.SetSatStates(np.zeros(len(ics), np.int32), ics)
        s.Solve()
        return s.results()

    free = run(0.0)  # 0: no budget, every trajectory runs to its own result
    assert set(free["status"]) <= {SatResult.SAT_SOLUTION_FOUND, SatResult.SAT_MAXITER_REACHED}
    assert free["steps"].min() > 0
    cut = run(1e-9)  # over before the first check: every trajectory interrupted
    assert (cut["status"] == SatResult.SAT_ODE_INTERRUPTED).all(), cut["status"]
    assert (cut["steps"] == 0).all()
