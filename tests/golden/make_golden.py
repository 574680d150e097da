"""Generate tests/golden/golden.npz (+ p50.cnf) by running the REFERENCE AnalogSAT
CPU solver and MiniSat, compiled from the reference's own sources into
oracle/_ref/libanalogsat_ref.so (oracle/Makefile).

Run in a container that has the reference tree:  python tests/golden/make_golden.py
(and `--models` for golden_models.npz, the tanh and bias variants).
Every array below is an output of the reference code itself (its makers, CpuSat,
CpuRungeKutta, SatSolver, CnfWriter and MiniSat), so the committed fixtures pin both
our C restatement (oracle/ctds_oracle.c) and the CUDA path to the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
from oracle import Reference, build  # noqa: E402


def ics(n, m, count, seed, a0=1.0):
    g = np.random.default_rng(seed)
    s = g.uniform(-1.0, 1.0, size=(count, n))
    return np.concatenate([s, np.full((count, m), a0)], axis=1)


def main():
    build()
    R = Reference()
    out = {}

    def put_problem(tag, p):
        lits, lens = p.export()
        out[f"{tag}/literals"] = lits
        out[f"{tag}/lengths"] = lens
        out[f"{tag}/nmk"] = np.array([p.n, p.m, p.k], np.int32)
        if p.planted is not None:
            out[f"{tag}/planted"] = p.planted.astype(np.int8)

    def put_rhs(tag, p, states):
        out[f"{tag}/rhs_states"] = states
        out[f"{tag}/rhs_f64"] = np.stack([R.rhs(p, x) for x in states])
        out[f"{tag}/rhs_f32"] = np.stack([R.rhs(p, x.astype(np.float32), np.float32) for x in states])
        out[f"{tag}/viol"] = np.array([R.violations(p, x) for x in states], np.int32)

    def put_traj(tag, p, ic, eps, nsteps):
        tr = R.steps(p, ic, eps, nsteps)
        out[f"{tag}/traj_ic"] = ic
        out[f"{tag}/traj_eps"] = np.array([eps])
        out[f"{tag}/traj_time"] = tr["time"]
        out[f"{tag}/traj_h"] = tr["h"]
        out[f"{tag}/traj_rhs"] = tr["rhs"]
        out[f"{tag}/traj_attempts"] = tr["attempts"]
        out[f"{tag}/traj_final"] = tr["states"][-1]
        out[f"{tag}/traj_mid"] = tr["states"][len(tr["states"]) // 2]

    def put_solve(tag, p, states, eps=1e-6, batch=50, maxsteps=200000, tmax=1e8):
        res = [R.solve(p, x, eps=eps, tmax=tmax, maxsteps=maxsteps, batch=batch) for x in states]
        out[f"{tag}/solve_ics"] = states
        out[f"{tag}/solve_params"] = np.array([eps, batch, maxsteps, tmax])
        out[f"{tag}/solve_result"] = np.array([r["result"] for r in res], np.int32)
        out[f"{tag}/solve_steps"] = np.array([r["steps"] for r in res], np.int32)
        out[f"{tag}/solve_rhs"] = np.array([r["rhs"] for r in res], np.int32)
        out[f"{tag}/solve_time"] = np.array([r["time"] for r in res])
        out[f"{tag}/solve_viol"] = np.array([r["violations"] for r in res], np.int32)
        out[f"{tag}/solve_final"] = np.stack([r["state"] for r in res])

    # 1. planted 3-SAT N=50, M=210 (PlantedSatMaker seed 12345)
    p50 = R.make("planted", 12345, 50, 210, 3)
    put_problem("p50", p50)
    st = ics(50, 210, 4, 1)
    put_rhs("p50", p50, st)
    put_traj("p50", p50, st[0], 1e-6, 100)
    put_solve("p50", p50, st)
    out["p50/minisat"] = np.array([R.minisat(p50)[0]], np.int32)
    R.write_cnf(p50, os.path.join(HERE, "p50.cnf"))

    # 2. hand-made mixed clause lengths: unit, 2-, 3- and 5-literal clauses, an unused
    #    variable (7), a repeated variable inside one clause, N not a multiple of 32
    clauses = [[1], [-2, 3], [4, -5, 6], [-1, 2, -3, 4, 5], [8, -9], [10, 11, -12], [-13],
               [14, 15, 16, -17, 18], [2, -2, 19], [20, -19, -18], [3, 6, 9], [-4, -8, 12, 16],
               [5, 10, 15, 20], [-20, -10]]
    lits = np.array([l for c in clauses for l in c], np.int32)
    lens = np.array([len(c) for c in clauses], np.int32)
    mix = R.problem(lits, lens)
    put_problem("mix", mix)
    put_rhs("mix", mix, ics(mix.n, mix.m, 3, 2, a0=1.3))
    put_traj("mix", mix, ics(mix.n, mix.m, 1, 3)[0], 1e-6, 60)

    # 3. random 4-SAT N=40, M=380 (RandomSatMaker seed 777)
    r4 = R.make("random", 777, 40, 380, 4)
    put_problem("r4", r4)
    put_rhs("r4", r4, ics(40, 380, 2, 4, a0=2.0))
    put_traj("r4", r4, ics(40, 380, 1, 5)[0], 1e-6, 80)

    # 4. clause length 12 (the reference's generic k > 10 path) via FastSatMaker
    k12 = R.make("fast", 99, 30, 20, 12)
    put_problem("k12", k12)
    put_rhs("k12", k12, ics(30, 20, 2, 6))

    # 5. the CPU-runnable configuration: first RandomSatMaker seed (1001, 1002, ...) whose
    #    N=50, M=210 3-SAT instance MiniSat certifies SAT; 16 trajectories, FP64, eps 1e-6
    for seed in range(1001, 1100):
        c1 = R.make("random", seed, 50, 210, 3)
        code, sol = R.minisat(c1)
        if code == 10:
            break
    put_problem("cfg1", c1)
    out["cfg1/seed"] = np.array([seed], np.int64)
    out["cfg1/minisat_solution"] = sol.astype(np.int8)
    put_solve("cfg1", c1, ics(50, 210, 16, 7))

    # 6. planted N=200, M=850 (the differentiation configuration's shape)
    p200 = R.make("planted", 4000, 200, 850, 3)
    put_problem("p200", p200)
    put_rhs("p200", p200, ics(200, 850, 2, 8))
    put_traj("p200", p200, ics(200, 850, 1, 9)[0], 1e-6, 100)

    # 7. planted N=1000, M=4250 (the at-scale GPU configuration's shape)
    p1000 = R.make("planted", 2000, 1000, 4250, 3)
    put_problem("p1000", p1000)
    put_rhs("p1000", p1000, ics(1000, 4250, 2, 10))
    put_traj("p1000", p1000, ics(1000, 4250, 1, 11)[0], 1e-6, 40)
    put_solve("p1000", p1000, ics(1000, 4250, 2, 12))

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", len(out), "arrays")


MODELS = {"tanh": (1, 1.1, 0.0), "tanh_q2_b3": (1, 2.0, 3.0), "bias20": (0, 1.1, 20.0)}


def models():
    """tests/golden/golden_models.npz: the reference's CTDS variants -- CpuSatTanh
    (Set_Q) and the bias term (ISat::Set_B) -- on the problems and states of
    golden.npz: FP64 RHS vectors and 30 single steps of CpuRungeKutta<double>."""
    build()
    R = Reference()
    g = np.load(os.path.join(HERE, "golden.npz"))
    out = {}
    for tag in ("p50", "mix", "k12", "r4", "p200"):
        p = R.problem(g[f"{tag}/literals"], g[f"{tag}/lengths"])
        for name, (tanh, q, b) in MODELS.items():
            R.set_model(tanh, q, b)
            out[f"{tag}/{name}/rhs_f64"] = np.stack([R.rhs(p, x) for x in g[f"{tag}/rhs_states"]])
            if f"{tag}/traj_ic" in g.files:
                tr = R.steps(p, g[f"{tag}/traj_ic"], 1e-6, 30)
                out[f"{tag}/{name}/traj_time"] = tr["time"]
                out[f"{tag}/{name}/traj_h"] = tr["h"]
                out[f"{tag}/{name}/traj_rhs"] = tr["rhs"]
                out[f"{tag}/{name}/traj_final"] = tr["states"][-1]
        R.set_model()
    np.savez_compressed(os.path.join(HERE, "golden_models.npz"), **out)
    print("wrote", len(out), "arrays")


if __name__ == "__main__":
    if "--models" in sys.argv:
        models()
    else:
        main()
