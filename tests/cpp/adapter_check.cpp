// Exercises include/analogsat_b200.hpp the way a reference frontend drives
// CudaSatSolver<double> (Frontend/src/cnf_runner.cpp:28-127).
//   adapter_check host <dir>            -- problem, CNF IO and error behaviour (no GPU)
//   adapter_check gpu <cnf> <ic-file>   -- one solve per precision; prints
//                                          "<prec> <result> <steps> <rhs> <time> <viol>"
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "analogsat_b200.hpp"

using namespace analogsat_b200;

static int host_checks(const std::string& dir) {
    SatProblem p;
    p.AddClauses(std::vector<std::vector<int>>{{1, -2, 3}, {-1, 4}, {2, 0, -4}, {}});
    if (p.Get_N() != 4 || p.Get_M() != 3 || p.Get_K() != 3) return 1;
    const std::string f = dir + "/adapter.cnf";
    p.WriteCnf(f);
    SatProblem q = SatProblem::ReadCnf(f);
    std::vector<int> l1, n1, l2, n2;
    p.GetAllClauses(l1, n1);
    q.GetAllClauses(l2, n2);
    if (l1 != l2 || n1 != n2) return 2;
    SatSolver<double> s;
    try {
        s.SetSatState({0.0});
        return 3;
    } catch (const Error& e) {
        if (e.code() != AS_ERR_NO_PROBLEM) return 4;
    }
    try {
        s.SetMaxSteps(0);
        return 5;
    } catch (const Error& e) {
        if (e.code() != AS_ERR_BAD_INPUT) return 6;
    }
    try {
        SatProblem::ReadCnf(dir + "/does-not-exist.cnf");
        return 7;
    } catch (const Error& e) {
        if (e.code() != AS_ERR_IO) return 8;
    }
    std::puts("host ok");
    return 0;
}

template <typename T>
static void solve_one(const SatProblem& p, const std::vector<double>& ic, const char* tag) {
    SatSolver<T> s;
    s.SetProblem(p);
    s.SetMaxTime((T)1e8);
    s.SetMaxSteps(200000);
    s.SetBatchSize(50);
    s.SetEpsilon(1e-6);
    s.SetSatState(std::vector<T>(ic.begin(), ic.end()));
    const SatResult r = s.Solve();
    std::vector<T> x;
    s.GetSatState().CopyTo(x);
    std::printf("%s %d %d %d %.17g %d %zu\n", tag, (int)r, s.GetStepCount(), s.GetRhsCount(),
                (double)s.GetElapsedTime(), s.GetLastClauseViolationCount(), x.size());
}

int main(int argc, char** argv) {
    if (argc >= 3 && std::string(argv[1]) == "host") return host_checks(argv[2]);
    if (argc >= 4 && std::string(argv[1]) == "gpu") {
        SatProblem p = SatProblem::ReadCnf(argv[2]);
        std::ifstream in(argv[3]);
        std::vector<double> ic;
        double v;
        while (in >> v) ic.push_back(v);
        solve_one<double>(p, ic, "f64");
        solve_one<float>(p, ic, "f32");
        // the GPU CNF reader gives the same problem; device-generated initial state
        SatProblem q = SatProblem::ReadCnf(argv[2], 0);
        std::printf("cnf_device %d %d %d\n", q.Get_N(), q.Get_M(), q.Get_K());
        SatSolver<double> s;
        s.SetProblem(q);
        s.SetRandomInitialState(42);
        std::vector<double> x;
        s.GetSatState().CopyTo(x);
        std::printf("rand %zu %.17g %.17g %.17g\n", x.size(), x[0], x[q.Get_N() - 1], x.back());
        return 0;
    }
    std::fprintf(stderr, "usage: adapter_check host <dir> | gpu <cnf> <ic>\n");
    return 64;
}
