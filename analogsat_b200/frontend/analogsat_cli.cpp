// analogsat-b200 -- command-line frontend over the C ABI, with the reference frontend's
// commands, options and output files (Frontend/src/main.cpp:255-440):
//
//   run        solve one CNF file (Frontend/src/cnf_runner.cpp:247-305): the result
//              file <resultfolder>/<name>.out is MiniSat-compatible ("SAT"/"INDET" and
//              the assignment), the per-batch progress line becomes one summary line
//              because the batch loop runs on the device.
//   speedtest  iteration performance over a series of problem sizes N = round(10 2^p)
//              (bench_runner.cpp:79-116): the CNF samples of each N are loaded from the
//              problem folder (cycled to at most 200 runs, as the reference does) and
//              run as ONE batched solve, one trajectory per run, bounded by -timeout;
//              every run appends the reference's perf line to perf_K<k>_a<a>_N<N>.dat
//              and the command prints RHS evaluations per second per N.
//   bench      solve a series of random K-SAT samples (bench_runner.cpp:51-72, 395-460):
//              a sample's CNF is loaded from the problem folder or made (K distinct
//              variables per clause, random signs, no repeated clause, as RandomSatMaker)
//              and written there once solved (a solution certifies SAT; the reference
//              asks MiniSat instead), perf lines as above.
//
// Differences from the reference frontend, by design: one process drives the GPU only
// (no -nogpu / -minisat); the samples of one N run together in one persistent launch;
// -float selects the FP32 solver with log-space clause weights (default FP64, whose
// right-hand side is bit-identical to the reference's); -trajectories T races T random
// starts per problem (the first solution stops the others).  Perf lines carry the wall
// and CPU seconds of the whole batched call.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <random>
#include <set>
#include <string>
#include <sys/stat.h>
#include <vector>

#include "analogsat_b200.hpp"

using namespace analogsat_b200;

namespace {

struct Config {
    std::string command, cnf_file, result_folder = ".", problem_folder = "problems";
    int device = 0, k = 3, batch = 50, sample_start = 0, sample_end = 100, trajectories = 1;
    long long stepmax = 50000000;
    double bias = 0.0, tmax = 1e8, timeout = 3600.0, eps = 1e-6, alpha = 4.25;
    double nstart = 1.0, nend = 5.0, nstep = 0.5;
    bool tanh = false, fp32 = false, rerun = false, force_save_cnf = false;
    unsigned long long seed = 1;
};

[[noreturn]] void usage_error(const std::string& msg) {
    std::fprintf(stderr, "Error: %s\n", msg.c_str());
    std::exit(2);
}

Config parse(int argc, char** argv) {
    Config c;
    if (argc < 2) usage_error("usage: analogsat-b200 run|speedtest|bench [-option value]");
    c.command = argv[1];
    if (c.command != "run" && c.command != "speedtest" && c.command != "bench")
        usage_error("analogsat command not understood: " + c.command);
    for (int i = 2; i < argc; i++) {
        const std::string o = argv[i];
        auto val = [&]() -> std::string {
            if (i + 1 >= argc) usage_error("option " + o + " needs a value");
            return argv[++i];
        };
        if (o == "-problem") c.cnf_file = val();
        else if (o == "-resultfolder") c.result_folder = val();
        else if (o == "-problemfolder") c.problem_folder = val();
        else if (o == "-usegpu") c.device = std::atoi(val().c_str());
        else if (o == "-tanh") c.tanh = true;
        else if (o == "-bias") c.bias = std::atof(val().c_str());
        else if (o == "-tmax") c.tmax = std::atof(val().c_str());
        else if (o == "-stepmax" || o == "-stempax") c.stepmax = std::atoll(val().c_str());
        else if (o == "-timeout") c.timeout = std::atof(val().c_str());
        else if (o == "-eps") c.eps = std::atof(val().c_str());
        else if (o == "-batch") c.batch = std::atoi(val().c_str());
        else if (o == "-k") c.k = std::atoi(val().c_str());
        else if (o == "-alpha") c.alpha = std::atof(val().c_str());
        else if (o == "-nstart") c.nstart = std::atof(val().c_str());
        else if (o == "-nend") c.nend = std::atof(val().c_str());
        else if (o == "-nstep") c.nstep = std::atof(val().c_str());
        else if (o == "-samplestart") c.sample_start = std::atoi(val().c_str());
        else if (o == "-sampleend") c.sample_end = std::atoi(val().c_str());
        else if (o == "-rerun") c.rerun = true;
        else if (o == "-force_save_cnf") c.force_save_cnf = true;
        else if (o == "-float") c.fp32 = true;
        else if (o == "-trajectories") c.trajectories = std::atoi(val().c_str());
        else if (o == "-seed") c.seed = std::strtoull(val().c_str(), nullptr, 10);
        else if (o == "-version") (void)val();  // one B200 solver: the reference's 1/2/3 choice is moot
        else if (o == "-nogpu" || o == "-minisat") usage_error(o + ": this frontend drives the GPU solver only");
        else usage_error("unknown option " + o);
    }
    // the reference's option ranges (Frontend/src/main.cpp:277-292)
    if (!(c.eps >= 1e-16 && c.eps <= 1.0)) usage_error("-eps out of range");
    if (c.batch < 1) usage_error("-batch must be positive");
    if (c.trajectories < 1) usage_error("-trajectories must be positive");
    if (c.stepmax < 1) usage_error("-stepmax must be positive");
    if (c.bias < 0) usage_error("-bias must be >= 0");
    if (c.sample_start < 0 || c.sample_end > 10000 || c.sample_start >= c.sample_end)
        usage_error("sample range out of bounds");
    return c;
}

bool exists(const std::string& p) {
    struct stat st;
    return ::stat(p.c_str(), &st) == 0;
}
void ensure_dir(const std::string& p) {
    std::string cur;
    for (size_t i = 0; i <= p.size(); i++) {
        if (i == p.size() || p[i] == '/') {
            if (!cur.empty() && !exists(cur)) ::mkdir(cur.c_str(), 0755);
        }
        if (i < p.size()) cur += p[i];
    }
}
std::string stem(const std::string& path) {
    std::string f = path.substr(path.find_last_of('/') == std::string::npos ? 0 : path.find_last_of('/') + 1);
    const size_t dot = f.find_last_of('.');
    return dot == std::string::npos ? f : f.substr(0, dot);
}

// bench_runner.cpp:38-48: N = round(10 * 2^p) for p = nstart, nstart + nstep, ... <= nend
std::vector<int> n_values(const Config& c) {
    std::vector<int> ns;
    for (double p = c.nstart; p < c.nend + 1e-3; p += c.nstep) ns.push_back((int)std::lround(10.0 * std::pow(2.0, p)));
    return ns;
}

template <typename T>
void configure(SatBatchSolver<T>& s, const Config& c) {
    s.SetMaxTime(c.tmax);
    s.SetMaxSteps((int)std::min<long long>(c.stepmax, 2147483647ll));
    s.SetBatchSize(c.batch);
    s.SetEpsilon(c.eps);
    s.SetWallBudget(c.timeout);
}

SatProblem model(SatProblem p, const Config& c) {
    p.SetTanh(c.tanh);
    p.Set_B(c.bias);
    return p;
}

std::string solver_name(const Config& c) {
    return std::string("analogsatb200") + (c.fp32 ? "f32" : "f64") + (c.tanh ? "tanh" : "orig");
}

// ---- run ------------------------------------------------------------------
template <typename T>
int run_cnf(const Config& c) {
    if (c.cnf_file.empty()) usage_error("run needs -problem <file.cnf>");
    ensure_dir(c.result_folder);
    SatProblem problem = model(SatProblem::ReadCnf(c.cnf_file), c);
    SatBatchSolver<T> s({&problem}, c.device);
    configure(s, c);
    s.SetStopOnFirst(true);
    std::vector<int32_t> idx(c.trajectories, 0);
    s.SetRandomInitialState(idx, c.seed);
    const std::vector<SatResult> r = s.Solve();
    int best = 0;
    for (int t = 0; t < (int)r.size(); t++)
        if (r[t] == SAT_SOLUTION_FOUND) { best = t; break; }
    long long rhs = 0;
    for (int t = 0; t < (int)r.size(); t++) rhs += s.GetRhsCount(t);
    std::printf("  %d\t%5.4lf\t%e\t%d\t%d\n", s.GetStepCount(best), s.GetElapsedTime(best), s.GetLastStepSize(best),
                s.GetLastClauseViolationCount(best), s.GetMinClauseViolationCount(best));
    std::printf("Performance: %f RK steps/sec\n", (double)rhs / 6.0 / s.GetElapsedWallTime());
    std::printf("%s\n", GetSatResultMessage(r[best]));
    s.WriteResult(best, c.result_folder + "/" + stem(c.cnf_file) + ".out");
    return 0;
}

// ---- random K-SAT samples (RandomSatMaker's distribution, our own stream) ----------
SatProblem make_random(int n, int m, int k, unsigned long long seed) {
    std::mt19937_64 rng(seed);
    std::uniform_int_distribution<int> var(1, n);
    std::set<std::vector<int>> seen;
    std::vector<int> lits, lens;
    while ((int)lens.size() < m) {
        std::vector<int> v;
        while ((int)v.size() < k) {
            const int x = var(rng);
            if (std::find(v.begin(), v.end(), x) == v.end()) v.push_back(x);
        }
        std::sort(v.begin(), v.end());
        for (int& x : v) x = (rng() & 1) ? x : -x;
        if (!seen.insert(v).second) continue;
        lits.insert(lits.end(), v.begin(), v.end());
        lens.push_back(k);
    }
    SatProblem p;
    p.AddClauses(lits, lens);
    return p;
}

struct Sample {
    std::string name, path;
};

// problem folder layout of the reference (bench_runner.cpp:405-420): <folder>/<k>a<100 alpha>/N<N>/p%04d.cnf
Sample sample_of(const Config& c, int n, int s) {
    char cls[64], name[128];
    std::snprintf(cls, sizeof cls, "%da%d", c.k, (int)(c.alpha * 100));
    std::snprintf(name, sizeof name, "%s/N%d/p%04d.cnf", cls, n, s);
    return {name, c.problem_folder + "/" + name};
}
std::string perf_file(const Config& c, int n) {
    char f[128];
    std::snprintf(f, sizeof f, "/perf_K%d_a%d_N%d.dat", c.k, (int)(c.alpha * 100), n);
    return c.result_folder + f;
}

// One batched solve over a list of (problem, sample name) runs, one trajectory each;
// appends the perf lines; returns (runs, solved, rhs, wall).
template <typename T>
void solve_runs(const Config& c, int n, const std::vector<SatProblem>& probs, const std::vector<std::string>& names,
                const std::vector<int>& run_problem, std::vector<SatResult>* out, long long* rhs, double* wall,
                std::vector<std::vector<T>>* states) {
    std::vector<const SatProblem*> ptr;
    for (const auto& p : probs) ptr.push_back(&p);
    SatBatchSolver<T> s(ptr, c.device);
    configure(s, c);
    std::vector<int32_t> idx(run_problem.begin(), run_problem.end());
    s.SetRandomInitialState(idx, c.seed + (unsigned long long)n * 1000003ull);
    *out = s.Solve();
    *wall = s.GetElapsedWallTime();
    *rhs = 0;
    for (size_t t = 0; t < idx.size(); t++) {
        *rhs += s.GetRhsCount((int)t);
        s.AppendPerf((int)t, perf_file(c, n), names[idx[t]], solver_name(c));
        if (states) states->push_back(s.GetSatState((int)t));
    }
}

template <typename T>
int speedtest(const Config& c) {
    ensure_dir(c.result_folder);
    for (int n : n_values(c)) {
        std::vector<SatProblem> probs;
        std::vector<std::string> names;
        for (int s = 0; s < 10000; s++) {
            const Sample sm = sample_of(c, n, s);
            if (!exists(sm.path)) break;
            probs.push_back(model(SatProblem::ReadCnf(sm.path), c));
            names.push_back(sm.name);
        }
        if (probs.empty()) throw Error(AS_ERR_IO, "no cnf samples exist with the given configuration");
        // the reference cycles through the samples until 5 s of solving or 200 runs; one
        // batched call takes the 200 runs at once
        const int runs = 200;
        std::vector<int> rp(runs);
        for (int r = 0; r < runs; r++) rp[r] = r % (int)probs.size();
        std::vector<SatResult> res;
        long long rhs = 0;
        double wall = 0.0;
        solve_runs<T>(c, n, probs, names, rp, &res, &rhs, &wall, nullptr);
        const long long solved = std::count(res.begin(), res.end(), SAT_SOLUTION_FOUND);
        std::printf("N=%d\truns=%d\tsolved=%lld\twall=%.4f s\tRHS evals/s=%.6g\n", n, runs, solved, wall,
                    (double)rhs / wall);
    }
    return 0;
}

template <typename T>
int bench(const Config& c) {
    ensure_dir(c.result_folder);
    for (int n : n_values(c)) {
        const int m = (int)(c.alpha * n);
        std::vector<SatProblem> probs;
        std::vector<std::string> names;
        std::vector<bool> made;
        for (int s = c.sample_start; s < c.sample_end; s++) {
            const Sample sm = sample_of(c, n, s);
            if (exists(sm.path)) {
                probs.push_back(model(SatProblem::ReadCnf(sm.path), c));
                made.push_back(false);
            } else {
                const unsigned long long seed = c.seed ^ ((unsigned long long)c.k << 48) ^
                                                ((unsigned long long)(c.alpha * 100) << 32) ^
                                                ((unsigned long long)n << 14) ^ (unsigned long long)s;
                probs.push_back(model(make_random(n, m, c.k, seed), c));
                made.push_back(true);
            }
            names.push_back(sm.name);
        }
        std::vector<int> rp(probs.size());
        for (size_t i = 0; i < rp.size(); i++) rp[i] = (int)i;
        std::vector<SatResult> res;
        long long rhs = 0;
        double wall = 0.0;
        solve_runs<T>(c, n, probs, names, rp, &res, &rhs, &wall, nullptr);
        int solved = 0;
        for (size_t i = 0; i < res.size(); i++) {
            const bool ok = res[i] == SAT_SOLUTION_FOUND;
            solved += ok;
            if (made[i] && (ok || c.force_save_cnf)) {
                const Sample sm = sample_of(c, n, c.sample_start + (int)i);
                ensure_dir(sm.path.substr(0, sm.path.find_last_of('/')));
                probs[i].WriteCnf(sm.path);
            }
        }
        std::printf("N=%d\tM=%d\tsamples=%zu\tsolved=%d\twall=%.4f s\tRHS evals/s=%.6g\n", n, m, probs.size(),
                    solved, wall, (double)rhs / wall);
    }
    return 0;
}

template <typename T>
int dispatch(const Config& c) {
    if (c.command == "run") return run_cnf<T>(c);
    if (c.command == "speedtest") return speedtest<T>(c);
    return bench<T>(c);
}

}  // namespace

int main(int argc, char** argv) {
    const Config c = parse(argc, argv);
    try {
        const int r = c.fp32 ? dispatch<float>(c) : dispatch<double>(c);
        std::printf("All done.\n");
        return r;
    } catch (const std::exception& e) {
        std::printf("Error: %s\n", e.what());
        return 1;
    }
}
