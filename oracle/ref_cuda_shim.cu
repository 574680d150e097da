// TEST INFRASTRUCTURE ONLY -- not part of the product.
//
// C-ABI shim over the reference AnalogSAT CUDA path ("plain GPU path": CudaSat1 +
// CudaRungeKutta driven by SatSolver, one instance and one trajectory per solver,
// exactly as the reference frontend runs it, Frontend/src/cnf_runner.cpp:28-127),
// compiled for sm_100a from the reference's own sources by oracle/Makefile into
// oracle/_ref/.  Only tests load it, to time the comparator the batched solver is
// measured against.
#include <chrono>
#include <cstring>
#include <vector>

#include "../solver/SatSolver.h"
#include "../problem/SatProblem.h"
#include "../cuda_sat/CudaSat1.h"
#include "../cuda_sat/CudaRungeKutta.h"

using namespace analogsat;

template <typename T>
static int solve_one(const int* lits, const int* lens, int m, const double* ic, double eps, double tmax,
                     int maxsteps, int batch, int* steps, int* rhs, double* time) {
    SatProblem p;
    int total = 0;
    for (int j = 0; j < m; j++) total += lens[j];
    p.AddClauses(std::vector<int>(lits, lits + total), std::vector<int>(lens, lens + m));
    CudaRungeKutta<T>* rk = new CudaRungeKutta<T>();
    rk->SetEpsilon((T)eps);
    CudaSatSolver<T> solver(new CudaSat1<T>(), rk);
    solver.SetProblem(p);
    solver.SetMaxTime((T)tmax);
    solver.SetMaxSteps(maxsteps);
    solver.SetBatchSize(batch);
    const int nm = p.Get_N() + p.Get_M();
    solver.SetSatState(std::vector<T>(ic, ic + nm));
    SatResult r = solver.Solve();
    *steps = solver.GetStepCount();
    *rhs = solver.GetRhsCount();
    *time = (double)solver.GetElapsedTime();
    return (int)r;
}

extern "C" {

// Solves units one after another (unit u: problem prob[u] given by its literal arrays,
// initial state ics + ic_off[u]) until `wall_budget` seconds have passed; returns the
// number of units run and their results; *wall = elapsed seconds.
int refcuda_solve_many(int precision, int nprob, const int* const* lits, const int* const* lens,
                       const int* ms, int nunits, const int* prob, const double* ics,
                       const long long* ic_off, double eps, double tmax, int maxsteps, int batch,
                       double wall_budget, int* results, int* steps, int* rhs, double* times,
                       double* wall) {
    auto t0 = std::chrono::steady_clock::now();
    int done = 0;
    try {
        for (int u = 0; u < nunits; u++) {
            double el = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
            if (wall_budget > 0 && el >= wall_budget) break;
            const int p = prob[u];
            if (precision == 1)
                results[u] = solve_one<double>(lits[p], lens[p], ms[p], ics + ic_off[u], eps, tmax, maxsteps,
                                               batch, steps + u, rhs + u, times + u);
            else
                results[u] = solve_one<float>(lits[p], lens[p], ms[p], ics + ic_off[u], eps, tmax, maxsteps,
                                              batch, steps + u, rhs + u, times + u);
            done++;
        }
    } catch (...) {
        *wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return -1;
    }
    *wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    (void)nprob;
    return done;
}

}  // extern "C"
