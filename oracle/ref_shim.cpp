// TEST INFRASTRUCTURE ONLY -- not part of the product.
//
// A C-ABI shim over the reference AnalogSAT CPU solver (compiled from the
// reference's own sources by oracle/Makefile into oracle/_ref/).  Tests, the
// golden-fixture generator and bench.py's CPU-baseline / reference arm call it
// through ctypes.  Nothing under analogsat_b200/ links or loads it.
//
// Every entry point drives the reference's public C++ API exactly as its own
// frontend does (Frontend/src/cnf_runner.cpp:129-217 SolveOnCpu):
//   CpuSatSolver<T>(new CpuSat<T>(), new CpuRungeKutta<T>()), SetEpsilon,
//   SetProblem, SetMaxTime/SetMaxSteps/SetBatchSize, SetSatState, Solve.
// Initial conditions are injected through SatSolver::SetSatState
// (AnalogSAT/solver/SatSolver.h:183-192) in the public [s_1..s_N, a_1..a_M]
// order (AnalogSAT/solver/ISatState.h:72-127).

#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <memory>
#include <stdexcept>
#include <thread>
#include <vector>

#include "../problem/SatProblem.h"
#include "../problem/RandomSatMaker.h"
#include "../problem/PlantedSatMaker.h"
#include "../problem/FastSatMaker.h"
#include "../io/CnfReader.h"
#include "../io/CnfWriter.h"
#include "../cpu_sat/CpuSat.h"
#include "../cpu_sat/CpuSatTanh.h"
#include "../cpu_sat/CpuRungeKutta.h"
#include "../solver/SatSolver.h"
#include "minisat.h"

using namespace analogsat;

namespace {

struct MemCnf : public Minisat::MemoryCNF {
    std::vector<int> content;
    size_t pos = 0;
    explicit MemCnf(const SatProblem& p) {
        content.push_back(p.Get_N());
        content.push_back(p.Get_M());
        for (int j = 0; j < p.Get_M(); j++) {
            const int* lits = p.GetLiterals() + p.GetClauseStart(j);
            for (int i = 0; i < p.GetClauseLength(j); i++) content.push_back(lits[i]);
            content.push_back(0);
        }
    }
    bool Finished() override { return pos >= content.size(); }
    int NextInt() override { return content[pos++]; }
};

// CTDS variant used by every entry point below (set by ref_set_model): CpuSat or
// CpuSatTanh (with Set_Q), and ISat::Set_B.
struct Model {
    int tanh = 0;
    double q = 1.1, b = 0.0;
};
Model g_model;

template <typename T>
ISat<T, CpuODEState<T>>* make_sat() {
    if (g_model.tanh) {
        CpuSatTanh<T>* s = new CpuSatTanh<T>();
        s->Set_Q((T)g_model.q);
        s->Set_B((T)g_model.b);
        return s;
    }
    CpuSat<T>* s = new CpuSat<T>();
    s->Set_B((T)g_model.b);
    return s;
}

template <typename T>
struct RefSolver {
    CpuSatSolver<T> solver;
    CpuRungeKutta<T>* rk;
    RefSolver(const SatProblem& p, T eps)
        : solver(make_sat<T>(), rk = new CpuRungeKutta<T>()) {
        rk->SetEpsilon(eps);
        solver.SetProblem(p);
    }
};

template <typename T>
int rhs_impl(void* handle, const T* state_pub, T* dxdt_pub) {
    try {
        const SatProblem& p = *static_cast<SatProblem*>(handle);
        std::unique_ptr<ISat<T, CpuODEState<T>>> sat(make_sat<T>());
        sat->SetProblem(p);
        std::unique_ptr<ISatState<T, CpuODEState<T>>> x(sat->MakeState());
        std::unique_ptr<ISatState<T, CpuODEState<T>>> d(sat->MakeState());
        const int nm = p.Get_N() + p.Get_M();
        std::vector<T> v(state_pub, state_pub + nm);
        x->CopyFrom(v);
        sat->GetDerivatives(*d, *x, (T)0);
        std::vector<T> out;
        d->CopyTo(out);
        std::memcpy(dxdt_pub, out.data(), sizeof(T) * nm);
        return 0;
    } catch (...) {
        return -1;
    }
}

template <typename T>
int violations_impl(void* handle, const T* state_pub) {
    try {
        const SatProblem& p = *static_cast<SatProblem*>(handle);
        CpuSat<T> sat;
        sat.SetProblem(p);
        std::vector<T> v(state_pub, state_pub + p.Get_N() + p.Get_M());
        return sat.GetClauseViolationCount(v);
    } catch (...) {
        return -1;
    }
}

// nsteps single-step Step() calls; record after each accepted step.
template <typename T>
int steps_impl(void* handle, const T* ic, T eps, int nsteps, double* times, double* hs,
               int* rhs, int* attempts, T* states) {
    try {
        const SatProblem& p = *static_cast<SatProblem*>(handle);
        const int nm = p.Get_N() + p.Get_M();
        std::shared_ptr<ISat<T, CpuODEState<T>>> sat(make_sat<T>());
        sat->SetProblem(p);
        CpuRungeKutta<T> rk;
        rk.SetEpsilon(eps);
        rk.Configure(sat);
        std::unique_ptr<ISatState<T, CpuODEState<T>>> a(sat->MakeState());
        std::unique_ptr<ISatState<T, CpuODEState<T>>> b(sat->MakeState());
        std::vector<T> v(ic, ic + nm);
        a->CopyFrom(v);
        for (int s = 0; s < nsteps; s++) {
            if (!rk.Step(*a, *b, 1)) return s;  // underflow: number of completed steps
            times[s] = (double)rk.GetTime();
            hs[s] = (double)rk.GetLastStepSize();
            rhs[s] = rk.GetRHSCount();
            attempts[s] = rk.GetAttemptCount();
            std::vector<T> out;
            a->CopyTo(out);
            std::memcpy(states + (size_t)s * nm, out.data(), sizeof(T) * nm);
        }
        return nsteps;
    } catch (...) {
        return -1;
    }
}

template <typename T>
int solve_impl(void* handle, const T* ic, T eps, T tmax, int maxsteps, int batch, T* final_state,
               double* out_time, int* out_steps, int* out_rhs, int* out_viol, double* out_wall,
               const std::chrono::steady_clock::time_point* deadline = nullptr) {
    try {
        const SatProblem& p = *static_cast<SatProblem*>(handle);
        const int nm = p.Get_N() + p.Get_M();
        RefSolver<T> rs(p, eps);
        rs.solver.SetMaxTime(tmax);
        rs.solver.SetMaxSteps(maxsteps);
        rs.solver.SetBatchSize(batch);
        if (deadline) {  // the reference's own per-batch callback stops the run (SAT_ODE_INTERRUPTED)
            const auto d = *deadline;
            rs.solver.SetCallback([d](SatSolver<T, CpuODEState<T>>&) { return std::chrono::steady_clock::now() < d; });
        }
        std::vector<T> v(ic, ic + nm);
        rs.solver.SetSatState(v);
        SatResult r = rs.solver.Solve();
        std::vector<T> out;
        rs.solver.GetSatState().CopyTo(out);
        if (final_state) std::memcpy(final_state, out.data(), sizeof(T) * nm);
        if (out_time) *out_time = (double)rs.solver.GetElapsedTime();
        if (out_steps) *out_steps = rs.solver.GetStepCount();
        if (out_rhs) *out_rhs = rs.solver.GetRhsCount();
        if (out_viol) *out_viol = rs.solver.GetLastClauseViolationCount();
        if (out_wall) *out_wall = rs.solver.GetElapsedWallTime();
        return (int)r;
    } catch (...) {
        return -1;
    }
}

}  // namespace

extern "C" {

void* refp_from_arrays(const int* lits, const int* lens, int m) {
    int total = 0;
    for (int j = 0; j < m; j++) total += lens[j];
    std::vector<int> l(lits, lits + total), n(lens, lens + m);
    SatProblem* p = new SatProblem();
    p->AddClauses(l, n);
    return p;
}

// kind: 0 RandomSatMaker, 1 PlantedSatMaker, 2 FastSatMaker.
void* refp_make(int kind, unsigned long seed, int n, int m, int k, int* planted) {
    SatProblem* p = new SatProblem();
    if (kind == 0) {
        RandomSatMaker mk(seed);
        mk.Set_N(n); mk.Set_M(m); mk.Set_K(k);
        mk.MakeSatProblem(*p);
    } else if (kind == 1) {
        PlantedSatMaker mk(seed);
        mk.Set_N(n); mk.Set_M(m); mk.Set_K(k);
        mk.MakeSatProblem(*p);
        if (planted) {
            std::vector<bool> sol = mk.GetPlantedSolution();
            for (int i = 0; i < n; i++) planted[i] = sol[i] ? 1 : 0;
        }
    } else {
        FastSatMaker mk(seed);
        mk.Set_N(n); mk.Set_M(m); mk.Set_K(k);
        mk.MakeSatProblem(*p);
    }
    return p;
}

void refp_info(void* h, int* n, int* m, int* k) {
    SatProblem* p = static_cast<SatProblem*>(h);
    *n = p->Get_N(); *m = p->Get_M(); *k = p->Get_K();
}

int refp_nlits(void* h) {
    SatProblem* p = static_cast<SatProblem*>(h);
    int t = 0;
    for (int j = 0; j < p->Get_M(); j++) t += p->GetClauseLength(j);
    return t;
}

void refp_export(void* h, int* lits, int* lens) {
    SatProblem* p = static_cast<SatProblem*>(h);
    int o = 0;
    for (int j = 0; j < p->Get_M(); j++) {
        const int* c = p->GetLiterals() + p->GetClauseStart(j);
        lens[j] = p->GetClauseLength(j);
        for (int i = 0; i < lens[j]; i++) lits[o++] = c[i];
    }
}

int refp_write_cnf(void* h, const char* path) {
    CnfWriter w(path);
    return w.Write(*static_cast<SatProblem*>(h)) ? 0 : -1;
}

void* refp_read_cnf(const char* path, char* msg, int msglen) {
    CnfReader r(path);
    SatProblem* p = new SatProblem();
    bool ok = r.Read(*p);
    if (msg && msglen > 0) {
        std::strncpy(msg, r.GetMessage(), msglen - 1);
        msg[msglen - 1] = 0;
    }
    if (!ok) { delete p; return nullptr; }
    return p;
}

void refp_free(void* h) { delete static_cast<SatProblem*>(h); }

// CTDS variant of the following calls: tanh = 1 builds CpuSatTanh (slope q) instead
// of CpuSat; b is passed to ISat::Set_B.  Not thread-safe against running solves.
void ref_set_model(int tanh, double q, double b) {
    g_model.tanh = tanh;
    g_model.q = q;
    g_model.b = b;
}

int ref_rhs_d(void* h, const double* x, double* d) { return rhs_impl<double>(h, x, d); }
int ref_rhs_f(void* h, const float* x, float* d) { return rhs_impl<float>(h, x, d); }
int ref_violations_d(void* h, const double* x) { return violations_impl<double>(h, x); }
int ref_violations_f(void* h, const float* x) { return violations_impl<float>(h, x); }

int ref_steps_d(void* h, const double* ic, double eps, int nsteps, double* times, double* hs,
                int* rhs, int* att, double* states) {
    return steps_impl<double>(h, ic, eps, nsteps, times, hs, rhs, att, states);
}
int ref_steps_f(void* h, const float* ic, float eps, int nsteps, double* times, double* hs,
                int* rhs, int* att, float* states) {
    return steps_impl<float>(h, ic, eps, nsteps, times, hs, rhs, att, states);
}

int ref_solve_d(void* h, const double* ic, double eps, double tmax, int maxsteps, int batch,
                double* fin, double* t, int* steps, int* rhs, int* viol, double* wall) {
    return solve_impl<double>(h, ic, eps, tmax, maxsteps, batch, fin, t, steps, rhs, viol, wall);
}
int ref_solve_f(void* h, const float* ic, float eps, float tmax, int maxsteps, int batch,
                float* fin, double* t, int* steps, int* rhs, int* viol, double* wall) {
    return solve_impl<float>(h, ic, eps, tmax, maxsteps, batch, fin, t, steps, rhs, viol, wall);
}

// Many independent FP64 solves spread over `nthreads` host threads (the reference
// solver is single-threaded; every thread owns its own CpuSatSolver).  Unit u
// solves problems[prob_idx[u]] from ics[ic_off[u] ...].  Threads stop taking new
// units once `wall_budget` seconds have passed, and a unit still running at twice
// the budget is interrupted through the solver's callback and left out (done[u] = 0);
// done[u] = 1 marks units run to their own result, busy[u] their wall seconds.
// Returns the number of units completed and the elapsed wall seconds in *wall.
int ref_solve_many_d(void** problems, const int* prob_idx, const double* ics,
                     const long long* ic_off, int nunits, int nthreads, double eps, double tmax,
                     int maxsteps, int batch, double wall_budget, int* results, int* steps,
                     int* rhs, double* times, int* done, double* busy, double* wall) {
    std::atomic<int> next(0);
    std::atomic<int> completed(0);
    auto t0 = std::chrono::steady_clock::now();
    const auto hard = t0 + std::chrono::duration_cast<std::chrono::steady_clock::duration>(
                               std::chrono::duration<double>(2.0 * wall_budget));
    auto worker = [&]() {
        while (true) {
            double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (wall_budget > 0 && el >= wall_budget) break;
            int u = next.fetch_add(1);
            if (u >= nunits) break;
            double tm = 0; int st = 0, rc = 0, vi = 0; double w = 0;
            const auto u0 = std::chrono::steady_clock::now();
            const int r = solve_impl<double>(problems[prob_idx[u]], ics + ic_off[u], eps, tmax, maxsteps,
                                             batch, nullptr, &tm, &st, &rc, &vi, &w,
                                             wall_budget > 0 ? &hard : nullptr);
            if (wall_budget > 0 && r == SAT_ODE_INTERRUPTED) continue;  // cut at the hard deadline
            if (busy) busy[u] = std::chrono::duration<double>(std::chrono::steady_clock::now() - u0).count();
            results[u] = r;
            steps[u] = st; rhs[u] = rc; times[u] = tm; done[u] = 1;
            completed.fetch_add(1);
        }
    };
    std::vector<std::thread> th;
    for (int i = 0; i < nthreads; i++) th.emplace_back(worker);
    for (auto& t : th) t.join();
    *wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return completed.load();
}

// MiniSat 2.2 (the reference's modified copy) on an in-memory CNF.
// Returns 10 = SAT, 20 = UNSAT, 0 = indeterminate; solution[i] = 1 if var i+1 is TRUE.
int ref_minisat(void* h, int* solution) {
    SatProblem* p = static_cast<SatProblem*>(h);
    MemCnf cnf(*p);
    Minisat::Results r = Minisat::SolveWithMinisat(cnf);
    if (std::strncmp(r.answer, "SATISFIABLE", 11) == 0) {
        if (solution) {
            for (int i = 0; i < p->Get_N(); i++) solution[i] = 0;
            for (int lit : r.solution) {
                int v = lit < 0 ? -lit : lit;
                if (v >= 1 && v <= p->Get_N()) solution[v - 1] = lit > 0 ? 1 : 0;
            }
        }
        return 10;
    }
    if (std::strncmp(r.answer, "UNSATISFIABLE", 13) == 0) return 20;
    return 0;
}

}  // extern "C"
