"""Against the plain GPU path: the reference's own CUDA solver (CudaSat1 +
CudaRungeKutta, FP64 as its frontend instantiates it, one instance and one trajectory
per SatSolver::Solve) built for sm_100a from the reference sources.

Correctness: on the same instance and initial state its FP64 result equals our FP64
solver's (SatResult and accepted steps).  Throughput: instances solved per second on
planted 3-SAT N=1000, M=4250 -- the reference one trajectory per instance in
sequence, ours 256 racing trajectories per instance in one persistent launch; the
north-star target is >= 10x.  Measured numbers are printed (pytest -s) and, when
ANALOGSAT_PLAIN_GPU_JSON is set, written there as JSON.
"""
import json
import os
import time

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    from oracle import RefCuda, REFCUDA_SO
    if not os.path.exists(REFCUDA_SO):
        pytest.skip("reference CUDA comparator not built")
    return RefCuda()


def test_plain_gpu_path_agrees(refcuda, golden):
    from analogsat_b200 import SatProblem, SatSolver, AS_PREC_F64
    lits, lens = golden["p50/literals"], golden["p50/lengths"]
    ic = golden["p50/solve_ics"][0]
    r = refcuda.solve_many([(lits, lens)], [0], [ic], precision=1, eps=1e-6, maxsteps=200000, batch=50)
    assert r["done"] == 1
    assert r["result"][0] == golden["p50/solve_result"][0]
    s = SatSolver([SatProblem.from_arrays(lits, lens)], precision=AS_PREC_F64)
    s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(200000); s.SetMaxTime(1e8)
    s.SetSatStates([0], ic[None, :])
    s.Solve()
    ours = s.results()
    assert ours["status"][0] == r["result"][0]
    assert ours["steps"][0] == r["steps"][0]


def test_batched_vs_plain_gpu_path_instances_per_second(refcuda):
    from analogsat_b200 import SatProblem, SatSolver
    from analogsat_b200.instances import make_instance, initial_states
    n, m, P, T = 1000, 4250, 16, 256
    raw = [make_instance("planted", n, m, 3, seed=2000 + i)[:2] for i in range(P)]
    ics = [initial_states(n, m, 1, seed=10_000 + i)[0] for i in range(P)]
    plain = refcuda.solve_many(raw, np.arange(P), ics, precision=1, eps=1e-6, maxsteps=100000,
                               batch=50, wall_budget=20.0)
    done = plain["done"]
    assert done >= 1
    plain_rate = int((plain["result"][:done] == 0).sum()) / plain["wall"]

    s = SatSolver([SatProblem.from_arrays(l, c) for l, c in raw])
    s.SetEpsilon(1e-6); s.SetBatchSize(50); s.SetMaxSteps(100000); s.SetMaxTime(1e8)
    s.SetStopOnFirst(True)
    pidx = np.repeat(np.arange(P), T).astype(np.int32)
    X = np.concatenate([initial_states(n, m, T, seed=20_000 + i, dtype=np.float32) for i in range(P)])
    s.SetSatStates(pidx, X)
    s.Solve()  # warm-up
    s.SetSatStates(pidx, X)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s.Solve()
    wall = time.perf_counter() - t0
    r = s.results()
    solved = len(set(pidx[r["status"] == 0]))
    ours_rate = solved / wall
    report = {"plain_gpu_path_instances_per_s": plain_rate, "plain_instances_run": int(done),
              "plain_wall_s": plain["wall"], "plain_mean_steps": float(plain["steps"][:done].mean()),
              "batched_instances_per_s": ours_rate, "batched_wall_s": wall,
              "speedup": ours_rate / plain_rate if plain_rate > 0 else None}
    print(json.dumps(report))
    out = os.environ.get("ANALOGSAT_PLAIN_GPU_JSON")
    if out:
        with open(out, "w") as f:
            json.dump(report, f)
    assert solved == P
    assert ours_rate >= 10.0 * plain_rate
