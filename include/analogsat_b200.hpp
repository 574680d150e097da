// analogsat_b200.hpp -- header-only C++ adapter over the C ABI (analogsat_b200.h).
//
// Mirrors the reference library's C++ API (AnalogSAT/solver/SatSolver.h,
// AnalogSAT/problem/SatProblem.h, AnalogSAT/io/CnfReader.h, CnfWriter.h) so that
// frontend code written against `CudaSatSolver<double>` / `CpuSatSolver<double>` swaps
// to the B200 solver with the same call sequence:
//
//     analogsat_b200::SatProblem problem;
//     problem.AddClauses(literals, lengths);            // or SatProblem::ReadCnf(path)
//     analogsat_b200::SatSolver<float> solver;          // <double>: FP64, bit-exact RHS
//     solver.SetProblem(problem);
//     solver.SetMaxTime(tmax); solver.SetMaxSteps(steps); solver.SetBatchSize(batch);
//     solver.SetEpsilon(eps);                           // CpuRungeKutta::SetEpsilon
//     solver.SetSatState(initial_state);                // public order [s_1..s_N, a_1..a_M]
//     analogsat_b200::SatResult r = solver.Solve();
//     std::vector<float> x; solver.GetSatState().CopyTo(x);
//
// Differences, by design: the whole integration loop runs on the device, so the
// per-batch callback is replaced by a wall-clock budget (SetWallBudget) and
// first-solution early exit across trajectories (SetStopOnFirst); many trajectories
// and instances are solved in one call with SetSatStates / SatBatchSolver.
// Errors throw analogsat_b200::Error (a std::runtime_error carrying the AS_ERR code),
// as the reference throws invalid_argument / runtime_error.
#pragma once

#include <chrono>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "analogsat_b200.h"

namespace analogsat_b200 {

// AnalogSAT/solver/SatResult.h:24-32
enum SatResult {
    SAT_SOLUTION_FOUND = AS_SAT_SOLUTION_FOUND,
    SAT_UNDERFLOW = AS_SAT_UNDERFLOW,
    SAT_ODE_INTERRUPTED = AS_SAT_ODE_INTERRUPTED,
    SAT_MAXTIME_REACHED = AS_SAT_MAXTIME_REACHED,
    SAT_MAXITER_REACHED = AS_SAT_MAXITER_REACHED,
    SAT_UNKNOWN = AS_SAT_UNKNOWN
};

// AnalogSAT/solver/SatResult.cpp:21-33
inline const char* GetSatResultMessage(SatResult r) {
    switch (r) {
        case SAT_SOLUTION_FOUND: return "solution found";
        case SAT_UNDERFLOW: return "underflow";
        case SAT_ODE_INTERRUPTED: return "user interrupt";
        case SAT_MAXTIME_REACHED: return "maximum time reached";
        case SAT_MAXITER_REACHED: return "maximum steps reached";
        default: return "unknown result";
    }
}

class Error : public std::runtime_error {
public:
    Error(int32_t code, const std::string& msg) : std::runtime_error(msg), code_(code) {}
    int32_t code() const { return code_; }

private:
    int32_t code_;
};

inline void check(int32_t code) {
    if (code < 0) {
        char buf[1024];
        as_last_error(buf, sizeof(buf));
        throw Error(code, buf);
    }
}

// analogsat::SatProblem (AnalogSAT/problem/SatProblem.h:26-63)
class SatProblem {
public:
    SatProblem() = default;

    // SatProblem::AddClauses(literals, lengths) (SatProblem.cpp:64-95).  Appends.
    void AddClauses(const std::vector<int>& literals, const std::vector<int>& lengths) {
        lits_.insert(lits_.end(), literals.begin(), literals.end());
        lens_.insert(lens_.end(), lengths.begin(), lengths.end());
        rebuild();
    }
    // SatProblem::AddClause (SatProblem.cpp:38-62)
    void AddClause(const std::vector<int>& clause) { AddClauses(clause, {(int)clause.size()}); }
    // SatProblem::AddClauses(vector<vector<int>>) (SatProblem.cpp:97-103)
    void AddClauses(const std::vector<std::vector<int>>& clauses) {
        for (const auto& c : clauses) {
            lits_.insert(lits_.end(), c.begin(), c.end());
            lens_.push_back((int)c.size());
        }
        rebuild();
    }
    // SatProblem::Clear
    void Clear() { lits_.clear(); lens_.clear(); h_.reset(); }

    // CnfReader::Read (AnalogSAT/io/CnfReader.cpp:48-141); with device >= 0 the clause
    // body is tokenised on that GPU (as_problem_read_cnf_device, same results).
    static SatProblem ReadCnf(const std::string& path, int device = -1) {
        as_problem* h = nullptr;
        char msg[256];
        check(device >= 0 ? as_problem_read_cnf_device(path.c_str(), device, &h, msg, sizeof(msg))
                          : as_problem_read_cnf(path.c_str(), &h, msg, sizeof(msg)));
        SatProblem p;
        p.h_.reset(h, as_problem_free);
        const int32_t nl = as_problem_num_literals(h);
        int32_t n, m, k;
        check(as_problem_get_nmk(h, &n, &m, &k));
        p.lits_.resize(nl);
        p.lens_.resize(m);
        if (m > 0) check(as_problem_get_clauses(h, p.lits_.data(), p.lens_.data()));
        return p;
    }
    // CnfWriter::Write (AnalogSAT/io/CnfWriter.cpp:49-74)
    void WriteCnf(const std::string& path) const { check(as_problem_write_cnf(handle(), path.c_str())); }

    int Get_N() const { return nmk(0); }
    int Get_M() const { return nmk(1); }
    int Get_K() const { return nmk(2); }

    // The CTDS variant, which the reference chooses by class (CpuSat / CpuSatTanh with
    // Set_Q, AnalogSAT/cpu_sat/CpuSatTanh.h:92) and ISat::Set_B (AnalogSAT/solver/
    // ISat.h:50-53).  Solvers take the variant when SetProblem is called.
    void SetTanh(bool on, double q = 1.1) {
        tanh_ = on;
        q_ = q;
        if (h_) apply_model();
    }
    void Set_B(double b) {
        b_ = b;
        if (h_) apply_model();
    }
    double Get_B() const { return b_; }

    // SatProblem::GetAllClauses (SatProblem.cpp:104-110)
    void GetAllClauses(std::vector<int>& literals, std::vector<int>& lengths) const {
        const int32_t nl = as_problem_num_literals(handle());
        literals.resize(nl);
        lengths.resize(Get_M());
        if (!lengths.empty()) check(as_problem_get_clauses(handle(), literals.data(), lengths.data()));
    }

    as_problem* handle() const {
        if (!h_) const_cast<SatProblem*>(this)->rebuild();
        return h_.get();
    }

private:
    std::vector<int32_t> lits_, lens_;
    std::shared_ptr<as_problem> h_;
    bool tanh_ = false;
    double q_ = 1.1, b_ = 0.0;

    void rebuild() {
        as_problem* h = nullptr;
        check(as_problem_create(lits_.data(), lens_.data(), (int32_t)lens_.size(), &h));
        h_.reset(h, as_problem_free);
        apply_model();
    }
    void apply_model() {
        check(as_problem_set_model(h_.get(), tanh_ ? AS_MODEL_TANH : AS_MODEL_CTDS, q_));
        check(as_problem_set_bias(h_.get(), b_));
    }
    int nmk(int i) const {
        int32_t v[3];
        check(as_problem_get_nmk(handle(), &v[0], &v[1], &v[2]));
        return v[i];
    }
};

// Public state copy helper mirroring ISatState::CopyTo (AnalogSAT/solver/ISatState.h:72-94).
template <typename TFloat>
class SatStateView {
public:
    explicit SatStateView(std::vector<TFloat> v) : v_(std::move(v)) {}
    void CopyTo(std::vector<TFloat>& target) const { target = v_; }
    void CopyBooleanTo(std::vector<bool>& target, int n) const {
        target.resize(n);
        for (int i = 0; i < n; i++) target[i] = v_[i] > 0;
    }

private:
    std::vector<TFloat> v_;
};

// Batched solver over several instances x trajectories: the C ABI's as_solver.
template <typename TFloat>
class SatBatchSolver {
    static_assert(std::is_same<TFloat, float>::value || std::is_same<TFloat, double>::value,
                  "TFloat must be float (FP32, log-space weights) or double (FP64)");

public:
    static constexpr int32_t kPrecision = std::is_same<TFloat, float>::value ? AS_PREC_F32_LOGA : AS_PREC_F64;

    explicit SatBatchSolver(const std::vector<const SatProblem*>& problems, int device = -1) {
        std::vector<const as_problem*> hs;
        for (auto* p : problems) {
            hs.push_back(p->handle());
            nm_.push_back(p->Get_N() + p->Get_M());
            n_.push_back(p->Get_N());
        }
        as_solver* s = nullptr;
        check(as_solver_create(hs.data(), (int32_t)hs.size(), kPrecision, device, &s));
        s_.reset(s, as_solver_free);
    }

    void SetMaxTime(double t) { check(as_solver_set_max_time(s_.get(), t)); }
    void SetMaxSteps(int n) { check(as_solver_set_max_steps(s_.get(), n)); }
    void SetBatchSize(int n) { check(as_solver_set_batch_size(s_.get(), n)); }
    void SetEpsilon(double e) { check(as_solver_set_epsilon(s_.get(), e)); }
    void SetWallBudget(double seconds) { check(as_solver_set_wall_budget(s_.get(), seconds)); }
    void SetStopOnFirst(bool f) { check(as_solver_set_stop_on_first(s_.get(), f ? 1 : 0)); }
    void SetTrackBest(bool f) { check(as_solver_set_track_best(s_.get(), f ? 1 : 0)); }

    // Trajectory t solves problem_index[t] from states[t] (public order).
    void SetSatStates(const std::vector<int32_t>& problem_index, const std::vector<std::vector<TFloat>>& states) {
        if (problem_index.size() != states.size())
            throw Error(AS_ERR_BAD_INPUT, "one initial state per trajectory");
        std::vector<TFloat> flat;
        for (size_t t = 0; t < states.size(); t++) {
            if ((int)states[t].size() < nm_.at(problem_index[t]))
                throw Error(AS_ERR_BAD_INPUT, "source vector is too short");  // ISatState::CopyFrom
            flat.insert(flat.end(), states[t].begin(), states[t].begin() + nm_[problem_index[t]]);
        }
        if (kPrecision == AS_PREC_F64)
            check(as_solver_set_states_f64(s_.get(), problem_index.data(), (int32_t)problem_index.size(),
                                           reinterpret_cast<const double*>(flat.data())));
        else
            check(as_solver_set_states_f32(s_.get(), problem_index.data(), (int32_t)problem_index.size(),
                                           reinterpret_cast<const float*>(flat.data())));
        index_ = problem_index;
    }

    // SatSolver::SetRandomInitialState (SatSolver.h:195-201) for every trajectory, generated
    // on the device from Philox4x64-10 keyed by seed (as_solver_set_random_states).
    void SetRandomInitialState(const std::vector<int32_t>& problem_index, uint64_t seed,
                               int32_t distribution = AS_IC_REFERENCE, double a0 = 1.0) {
        check(as_solver_set_random_states(s_.get(), problem_index.data(), (int32_t)problem_index.size(), seed,
                                          distribution, a0));
        index_ = problem_index;
    }

    // Runs every trajectory to its SatResult; returns them in trajectory order.
    std::vector<SatResult> Solve() {
        const auto t0 = std::chrono::steady_clock::now();
        check(as_solver_solve(s_.get()));
        wall_ = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        return results();
    }
    // Asynchronous form: enqueues the solve on `stream` (a cudaStream_t; null: the
    // solver's own stream); Sync() waits for it and returns the SatResults.
    void SolveAsync(void* stream = nullptr) { check(as_solver_solve_async(s_.get(), stream)); }
    std::vector<SatResult> Sync() {
        check(as_solver_sync(s_.get()));
        return results();
    }

    // Launch shape (no reference counterpart): CTA size, storage mode (0 automatic,
    // 1 shared memory, 2 global storage, 3 streamed).
    void ForceThreads(int threads) { check(as_solver_force_threads(s_.get(), threads)); }
    void SetStorageMode(int mode) { check(as_solver_set_storage_mode(s_.get(), mode)); }

    // MAXSAT runs (SetTrackBest(true)): the Boolean assignment with the fewest unsat
    // clauses seen by trajectory traj; element i is variable i + 1.
    std::vector<bool> GetBestAssignment(int traj) const {
        if (traj < 0 || traj >= (int)index_.size()) throw Error(AS_ERR_BAD_INPUT, "trajectory index out of range");
        const int n = n_[index_[traj]];
        std::vector<uint32_t> bits((n + 31) / 32);
        check(as_solver_get_best_assignment(s_.get(), traj, bits.data()));
        std::vector<bool> a(n);
        for (int i = 0; i < n; i++) a[i] = (bits[i >> 5] >> (i & 31)) & 1u;
        return a;
    }

    // The reference frontend's outputs: the MiniSat-compatible result file
    // (cnf_runner.cpp:280-304) and the tab-separated perf line (bench_runner.cpp:331-343).
    void WriteResult(int traj, const std::string& path) const {
        check(as_solver_write_result(s_.get(), traj, path.c_str()));
    }
    void AppendPerf(int traj, const std::string& path, const std::string& sample,
                    const std::string& solver_name) const {
        check(as_solver_append_perf(s_.get(), traj, path.c_str(), sample.c_str(), solver_name.c_str()));
    }

    std::vector<TFloat> GetSatState(int traj) const {
        if (traj < 0 || traj >= (int)index_.size()) throw Error(AS_ERR_BAD_INPUT, "trajectory index out of range");
        std::vector<TFloat> x(nm_[index_[traj]]);
        if (kPrecision == AS_PREC_F64)
            check(as_solver_get_state_f64(s_.get(), traj, reinterpret_cast<double*>(x.data())));
        else
            check(as_solver_get_state_f32(s_.get(), traj, reinterpret_cast<float*>(x.data())));
        return x;
    }

    int GetStepCount(int traj) const { return steps_.at(traj); }
    int GetRhsCount(int traj) const { return rhs_.at(traj); }
    double GetElapsedTime(int traj) const { return time_.at(traj); }
    double GetLastStepSize(int traj) const { return hdid_.at(traj); }
    int GetLastClauseViolationCount(int traj) const { return viol_.at(traj); }
    int GetMinClauseViolationCount(int traj) const { return minv_.at(traj); }
    double GetElapsedWallTime() const { return wall_; }
    as_solver* handle() const { return s_.get(); }

private:
    std::shared_ptr<as_solver> s_;
    std::vector<int> nm_, n_;
    std::vector<int32_t> index_;
    std::vector<int32_t> status_, steps_, rhs_, att_, viol_, minv_;
    std::vector<double> time_, hdid_;
    double wall_ = 0.0;

    size_t total() const {
        size_t t = 0;
        for (auto i : index_) t += nm_[i];
        return t;
    }
    std::vector<SatResult> results() {
        fetch();
        std::vector<SatResult> r(status_.size());
        for (size_t i = 0; i < r.size(); i++) r[i] = (SatResult)status_[i];
        return r;
    }
    void fetch() {
        const size_t n = index_.size();
        status_.resize(n); steps_.resize(n); rhs_.resize(n); att_.resize(n);
        viol_.resize(n); minv_.resize(n); time_.resize(n); hdid_.resize(n);
        check(as_solver_get_results(s_.get(), status_.data(), time_.data(), steps_.data(), rhs_.data(),
                                    att_.data(), viol_.data(), minv_.data(), hdid_.data()));
    }
};

// analogsat::SatSolver<TFloat, TState> for one problem and one trajectory
// (SatSolver.h:41-356): same method names and defaults (maxTime 100, maxSteps 1e5,
// batchSize 20; integrator eps 1e-4).
template <typename TFloat>
class SatSolver {
public:
    explicit SatSolver(int device = -1) : device_(device) {}

    // SatSolver::SetProblem (SatSolver.h:207-218)
    void SetProblem(const SatProblem& problem) {
        problem_ = problem;
        batch_.reset(new SatBatchSolver<TFloat>({&problem_}, device_));
        batch_->SetMaxTime(maxTime_);
        batch_->SetMaxSteps(maxSteps_);
        batch_->SetBatchSize(batchSize_);
        batch_->SetEpsilon(eps_);
        state_.assign(problem.Get_N() + problem.Get_M(), TFloat(0));
    }

    void SetMaxTime(TFloat t) {
        if (!(t > 0)) throw Error(AS_ERR_BAD_INPUT, "Max time must be positive");
        maxTime_ = t;
        if (batch_) batch_->SetMaxTime(t);
    }
    TFloat GetMaxTime() const { return maxTime_; }
    void SetMaxSteps(int n) {
        if (n < 1) throw Error(AS_ERR_BAD_INPUT, "Max iterations must be positive");
        maxSteps_ = n;
        if (batch_) batch_->SetMaxSteps(n);
    }
    int GetMaxSteps() const { return maxSteps_; }
    void SetBatchSize(int n) {
        if (n < 1) throw Error(AS_ERR_BAD_INPUT, "Batch size must be positive");
        batchSize_ = n;
        if (batch_) batch_->SetBatchSize(n);
    }
    int GetBatchSize() const { return batchSize_; }
    // CpuRungeKutta::SetEpsilon (CpuRungeKutta.cpp:126-131)
    void SetEpsilon(double e) {
        if (!(e >= 1e-16 && e <= 1.0)) throw Error(AS_ERR_BAD_INPUT, "epsilon must be between 1e-16 and 1");
        eps_ = e;
        if (batch_) batch_->SetEpsilon(e);
    }
    void SetWallBudget(double seconds) { need().SetWallBudget(seconds); }

    // SatSolver::SetSatState(vector) (SatSolver.h:183-192)
    void SetSatState(const std::vector<TFloat>& state) {
        need();
        if (state.size() < state_.size()) throw Error(AS_ERR_BAD_INPUT, "source vector is too short");
        state_.assign(state.begin(), state.begin() + state_.size());
    }

    // SatSolver::Solve (SatSolver.h:162-165)
    SatResult Solve() {
        need().SetSatStates({0}, {state_});
        const SatResult r = batch_->Solve()[0];
        state_ = batch_->GetSatState(0);
        return r;
    }

    // SatSolver::SetRandomInitialState (SatSolver.h:195-201): the reference's transform
    // (s = 2u - 1, a = u + 1) of Philox uniforms keyed by seed, drawn on the device.
    void SetRandomInitialState(uint64_t seed) {
        need().SetRandomInitialState({0}, seed, AS_IC_REFERENCE);
        state_ = batch_->GetSatState(0);
    }

    SatStateView<TFloat> GetSatState() const { return SatStateView<TFloat>(state_); }
    int GetStepCount() const { return batch_ ? batch_->GetStepCount(0) : 0; }
    int GetRhsCount() const { return batch_ ? batch_->GetRhsCount(0) : 0; }
    TFloat GetElapsedTime() const { return batch_ ? (TFloat)batch_->GetElapsedTime(0) : TFloat(0); }
    TFloat GetLastStepSize() const { return batch_ ? (TFloat)batch_->GetLastStepSize(0) : TFloat(0); }
    int GetLastClauseViolationCount() const { return batch_ ? batch_->GetLastClauseViolationCount(0) : 0; }
    double GetElapsedWallTime() const { return batch_ ? batch_->GetElapsedWallTime() : 0.0; }

private:
    int device_;
    SatProblem problem_;
    std::unique_ptr<SatBatchSolver<TFloat>> batch_;
    std::vector<TFloat> state_;
    TFloat maxTime_ = TFloat(100);
    int maxSteps_ = 100000;
    int batchSize_ = 20;
    double eps_ = 1e-4;

    SatBatchSolver<TFloat>& need() {
        if (!batch_) throw Error(AS_ERR_NO_PROBLEM, "SAT problem has not been set");
        return *batch_;
    }
};

}  // namespace analogsat_b200
