"""Generate the statistical fixtures by running the REFERENCE code (compiled from the
reference's own sources into oracle/_ref/libanalogsat_ref.so by oracle/Makefile):

* minisat_3sat.npz -- 64 random 3-SAT instances N=60, M=256 (alpha 4.27, near the
  satisfiability threshold, so about half are UNSAT) made by the reference's
  RandomSatMaker (seeds 70000..70063), with MiniSat's verdict for each (10 SAT,
  20 UNSAT) and, for the SAT ones, MiniSat's model.
* reference_runs_planted1000.npz -- the reference solver (CpuSat<double> +
  CpuRungeKutta<double> driven by SatSolver, eps 1e-6, batch 50, max steps 1e5) run
  to its SatResult from trajectories 0..3 of each of the 64 instances of the
  headline workload (planted 3-SAT N=1000, M=4250, bench.make_workload), the initial
  states cast from FP32 as the GPU receives them: SatResult, accepted steps and RHS
  count of every run.

Run where the reference tree is present:  python tests/golden/make_golden_stats.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, ROOT)
from oracle import Reference, build  # noqa: E402

MINISAT_N, MINISAT_M, MINISAT_COUNT, MINISAT_SEED0 = 60, 256, 64, 70000
RUNS_PER_INSTANCE = 4


def make_minisat(R):
    lits, verdict, model = [], [], []
    for i in range(MINISAT_COUNT):
        p = R.make("random", MINISAT_SEED0 + i, MINISAT_N, MINISAT_M, 3)
        l, n = p.export()
        assert (n == 3).all() and p.n == MINISAT_N
        code, sol = R.minisat(p)
        assert code in (10, 20), code
        lits.append(l)
        verdict.append(code)
        model.append(sol if code == 10 else np.zeros(MINISAT_N, np.int32))
    np.savez_compressed(os.path.join(HERE, "minisat_3sat.npz"),
                        literals=np.stack(lits).astype(np.int8), verdict=np.array(verdict, np.int8),
                        model=np.stack(model).astype(np.int8),
                        nmk=np.array([MINISAT_N, MINISAT_M, 3], np.int32))
    print("minisat: SAT", int((np.array(verdict) == 10).sum()), "UNSAT", int((np.array(verdict) == 20).sum()))


def make_runs(R):
    import bench
    W = bench.WORKLOAD
    probs, pidx, ics = bench.make_workload(0, W["instances"], W["traj"])
    units = bench.cpu_sample_units(W["instances"], W["traj"], RUNS_PER_INSTANCE)
    nm = W["n"] + W["m"]
    X = ics.reshape(-1, nm)
    handles = [R.problem(*p) for p in probs]
    r = R.solve_many(handles, pidx[units], [X[u].astype(np.float64) for u in units], eps=W["eps"],
                     tmax=W["tmax"], maxsteps=W["maxsteps"], batch=W["batch"])
    assert int(r["done"].sum()) == len(units)
    np.savez_compressed(os.path.join(HERE, "reference_runs_planted1000.npz"), units=units.astype(np.int32),
                        result=r["result"].astype(np.int8), steps=r["steps"].astype(np.int32),
                        rhs=r["rhs"].astype(np.int32))
    print("runs: solved", int((r["result"] == 0).sum()), "of", len(units), "median steps",
          float(np.median(r["steps"])))


def main():
    build()
    R = Reference()
    make_minisat(R)
    if "--minisat-only" not in sys.argv:
        make_runs(R)


if __name__ == "__main__":
    main()
