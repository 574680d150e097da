/* TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * Plain-C FP64 restatement of the AnalogSAT CTDS hot path, used as the checker
 * for the CUDA path.  Only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline load it.  It is pinned against the reference solver itself
 * (oracle/_ref, built from the reference's sources) by tests/test_oracle.py
 * and by the golden fixtures in tests/golden/.
 *
 * Public state layout (AnalogSAT/solver/ISatState.h:72-127): [s_1..s_N, a_1..a_M].
 * With `logspace` set, the a-block of every state/derivative vector holds
 * u_m = ln a_m and du_m/dt = K_m^2 instead.
 */
#ifndef CTDS_ORACLE_H
#define CTDS_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_problem orc_problem;

/* SatProblem::AddClauses semantics (AnalogSAT/problem/SatProblem.cpp:64-95). */
orc_problem* orc_problem_new(const int* lits, const int* lens, int m);
void orc_problem_free(orc_problem* p);
/* CTDS variant: tanh_model = 1 restates CpuSatTanh (slope q), b the bias coefficient
 * (ISat::Set_B); default CpuSat with b = 0. */
void orc_problem_set_model(orc_problem* p, int tanh_model, double q, double b);
void orc_problem_info(const orc_problem* p, int* n, int* m, int* k);

/* CpuSat::GetDerivatives (AnalogSAT/cpu_sat/CpuSat.cpp:65-94, 199-241). */
void orc_rhs(const orc_problem* p, const double* x, double* dxdt, int logspace);

/* CpuSat::GetClauseViolationCount (AnalogSAT/cpu_sat/CpuSat.cpp:136-173); spins = N values. */
int orc_violations(const orc_problem* p, const double* spins);

/* nsteps calls of CpuRungeKutta::Step(old,new,1) (AnalogSAT/cpu_sat/CpuRungeKutta.cpp:66-100,
 * 181-267).  ic holds the public state with a in linear space (converted internally when
 * logspace).  Records after each accepted step: time, hdid, cumulative RHS count, cumulative
 * attempts and the public state (a in linear space).  Returns steps completed (< nsteps on
 * step-size underflow). */
int orc_steps(const orc_problem* p, const double* ic, double eps, int nsteps, int logspace,
              double* times, double* hs, int* rhs, int* attempts, double* states);

/* SatSolver::DoSolve without callback (AnalogSAT/solver/SatSolver.h:273-355).
 * Returns the SatResult code (0 found, 1 underflow, 3 max time, 4 max steps). */
int orc_solve(const orc_problem* p, const double* ic, double eps, double tmax, int maxsteps,
              int batch, int logspace, double* final_state, double* out_time, int* out_steps,
              int* out_rhs, int* out_attempts, int* out_viol);

/* Same integrator, final step clamped to end exactly at t_end; returns steps taken. */
int orc_integrate_to(const orc_problem* p, const double* ic, double eps, double t_end,
                     int logspace, int maxsteps, double* out_state, double* out_time);

/* Potential V = sum_m w_m a_m K_m^2 of a public state (a linear). */
double orc_potential(const orc_problem* p, const double* x, const double* w);

/* Differentiation (weighted ODE, see ctds_oracle.c): record the accepted step sizes of
 * an adaptive run to t_end, evaluate L = V(x(T)) through that frozen step sequence,
 * and its discrete adjoint (gradients w.r.t. x0 = [s(0), a(0)] and w). */
int orc_record_steps(const orc_problem* p, const double* ic, double eps, double t_end, int maxsteps,
                     double* hs);
double orc_fixed_loss(const orc_problem* p, const double* x0, const double* w, const double* hs, int nsteps,
                      double* x_final);
double orc_adjoint(const orc_problem* p, const double* x0, const double* w, const double* hs, int nsteps,
                   double* g_x0, double* g_w);

#ifdef __cplusplus
}
#endif
#endif
