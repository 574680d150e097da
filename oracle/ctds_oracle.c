/* TEST INFRASTRUCTURE ONLY -- not part of the product.
 *
 * FP64 C restatement of the AnalogSAT CTDS hot path (the checker the CUDA path
 * is compared with).  Each function cites the reference code it restates; the
 * arithmetic follows the reference's expression order so that, compiled
 * without FMA contraction (-ffp-contract=off), the RHS and RK45 stage values
 * are bit-identical to the reference CpuSat<double> / CpuRungeKutta<double>.
 * tests/test_oracle.py pins that against the reference itself.
 */
#include "ctds_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

struct orc_problem {
    int n, m, k;
    int* C;      /* clause-major [m][k], signed 1-based literals, 0 = padding
                    (AnalogSAT/cpu_sat/CpuSat.cpp:353-377, GetC at 385-388) */
    double knorm; /* 2^-k with k the MAX clause length (CpuSat.cpp:355) */
    int tanh;     /* CpuSatTanh instead of CpuSat (AnalogSAT/cpu_sat/CpuSatTanh.cpp) */
    double q;     /* its slope (CpuSatTanh.cpp:40 default 1.1) */
    double b;     /* bias coefficient, ISat::Set_B (0 = off) */
};

void orc_problem_set_model(orc_problem* p, int tanh_model, double q, double b) {
    p->tanh = tanh_model;
    p->q = q;
    p->b = b;
}

/* SatProblem::AddClauses (AnalogSAT/problem/SatProblem.cpp:64-95): zero literals are
 * filtered, empty clauses dropped, N = max |literal|, K = max clause length. */
orc_problem* orc_problem_new(const int* lits, const int* lens, int m_in) {
    orc_problem* p = (orc_problem*)calloc(1, sizeof(orc_problem));
    int total = 0, j, i, off = 0, mm = 0;
    for (j = 0; j < m_in; j++) {
        int len1 = 0;
        for (i = 0; i < lens[j]; i++) {
            int l = lits[total + i];
            if (l == 0) continue;
            if (abs(l) > p->n) p->n = abs(l);
            len1++;
        }
        if (len1 > 0) { mm++; if (len1 > p->k) p->k = len1; }
        total += lens[j];
    }
    p->m = mm;
    p->C = (int*)calloc((size_t)(mm > 0 ? mm : 1) * (size_t)(p->k > 0 ? p->k : 1), sizeof(int));
    total = 0;
    for (j = 0; j < m_in; j++) {
        int q = 0;
        for (i = 0; i < lens[j]; i++) {
            int l = lits[total + i];
            if (l != 0) p->C[(size_t)off * p->k + q++] = l;
        }
        if (q > 0) off++;
        total += lens[j];
    }
    p->knorm = pow(2.0, -(double)p->k);
    p->q = 1.1;
    return p;
}

void orc_problem_free(orc_problem* p) {
    if (!p) return;
    free(p->C);
    free(p);
}

void orc_problem_info(const orc_problem* p, int* n, int* m, int* k) {
    *n = p->n; *m = p->m; *k = p->k;
}

/* CpuSat::GetDerivatives -> CalculateAllEx<K> (AnalogSAT/cpu_sat/CpuSat.cpp:199-241) with
 * CpuKmiWrapper / CpuProdWrapper (AnalogSAT/cpu_sat/cpu_helper.h:21-126) for K <= 10, and
 * the generic CalculateAll (CpuSat.cpp:291-349) for K > 10.  Internal state has the
 * reference's constant FALSE slot x[0] = -1 in front (CpuSatStateImpl.h:94-99). */
static void rhs_internal(const orc_problem* p, const double* x, double* rhs, int logspace) {
    const int n = p->n, m = p->m, k = p->k;
    const double knorm = p->knorm;
    double f[64];
    int idx[64];
    int j, q, l;
    double sum = 0.0;
    memset(rhs, 0, sizeof(double) * (size_t)(n + m + 1));
    for (j = 0; j < m; j++) {
        double km = knorm, am, r;
        const int* c = p->C + (size_t)j * k;
        for (q = 0; q < k; q++) idx[q] = c[q];
        for (q = 0; q < k; q++) {
            double s = idx[q] != 0 ? x[abs(idx[q])] : -1.0;
            f[q] = idx[q] < 0 ? 1.0 + s : 1.0 - s;
            km *= f[q];
        }
        if (logspace) {
            am = exp(x[n + 1 + j]);
            rhs[n + 1 + j] = km * km;
        } else {
            am = x[n + 1 + j];
            rhs[n + 1 + j] = am * km * km;
        }
        sum += am;
        if (p->tanh) {
            /* CpuSatTanh::CalculateAllEx<K> / KmiFuncTanh (CpuSatTanh.cpp:203-244,
             * cpu_helper.h:115-125) for K <= 10, CalculateAll (CpuSatTanh.cpp:250-297) */
            if (k <= 10) {
                r = knorm * am;
                for (q = 0; q < k; q++) {
                    double prod = 1.0, rr;
                    int first = 1;
                    if (idx[q] == 0) break;
                    for (l = 0; l < k; l++) {
                        if (l == q) continue;
                        if (first) { prod = f[l]; first = 0; } else prod = prod * f[l];
                    }
                    rr = r * (prod < 0 ? -prod : prod) * tanh(p->q * f[q]);
                    rr *= idx[q] < 0 ? -1.0 : 1.0;
                    rhs[abs(idx[q])] += rr;
                }
            } else {
                for (q = 0; q < k; q++) {
                    double temp = 1.0, sign = idx[q] < 0 ? -1.0 : 1.0;
                    for (l = 0; l < k; l++) temp *= (l == q) ? 1.0 : f[l];
                    rhs[abs(idx[q])] += knorm * am * fabs(temp) * sign * tanh(p->q * f[q]);
                }
            }
            continue;
        }
        if (k <= 10) {
            r = km * knorm * am;
            for (q = 0; q < k; q++) {
                double prod = 1.0, rr;
                int first = 1;
                if (idx[q] == 0) break;
                for (l = 0; l < k; l++) {
                    if (l == q) continue;
                    if (first) { prod = f[l]; first = 0; } else prod = prod * f[l];
                }
                rr = r * prod;
                rr *= idx[q] < 0 ? -2.0 : 2.0;
                rhs[abs(idx[q])] += rr;
            }
        } else {
            for (q = 0; q < k; q++) {
                double temp = km, sign = idx[q] < 0 ? -1.0 : 1.0;
                for (l = 0; l < k; l++) temp *= (l == q) ? 1.0 : f[l];
                rhs[abs(idx[q])] += 2.0 * temp * knorm * am * sign;
            }
        }
    }
    {
        /* the bias term (CpuSat.cpp:228-238: only when b knorm^2 > 0; CpuSatTanh.cpp:
         * 233-238 and 298-302: always) */
        const double bb = p->b * knorm * knorm;
        if (bb > 0.0 || p->tanh) {
            const double a = sum / m, alpha = (double)m / (double)n;
            int i;
            for (i = 1; i < n + 1; i++)
                rhs[i] += a * alpha * bb * 1.570796326794897 * sin(x[i] * 3.141592653589793);
        }
    }
    rhs[0] = 0.0;
}

static void to_internal(const orc_problem* p, const double* pub, double* x, int logspace_in) {
    x[0] = -1.0;
    memcpy(x + 1, pub, sizeof(double) * (size_t)(p->n + p->m));
    (void)logspace_in;
}

void orc_rhs(const orc_problem* p, const double* xpub, double* dpub, int logspace) {
    size_t sz = (size_t)(p->n + p->m + 1);
    double* x = (double*)malloc(sizeof(double) * sz);
    double* d = (double*)malloc(sizeof(double) * sz);
    to_internal(p, xpub, x, logspace);
    rhs_internal(p, x, d, logspace);
    memcpy(dpub, d + 1, sizeof(double) * (sz - 1));
    free(x);
    free(d);
}

/* CpuSat::CalculateClauses (AnalogSAT/cpu_sat/CpuSat.cpp:136-164): a literal is TRUE when
 * the spin is > 0 (positive literal) or <= 0 (negative literal); padding is FALSE. */
int orc_violations(const orc_problem* p, const double* spins) {
    int j, q, count = 0;
    for (j = 0; j < p->m; j++) {
        int clause = 0;
        for (q = 0; q < p->k; q++) {
            int item = p->C[(size_t)j * p->k + q];
            int index = item < 0 ? -item : item;
            int lit = index == 0 ? 0 : (spins[index - 1] > 0.0);
            if (item < 0) lit = !lit;
            clause |= lit;
            if (clause) break;
        }
        count += clause ? 0 : 1;
    }
    return count;
}

/* Cash-Karp tableau and NR controller constants (AnalogSAT/cpu_sat/CpuRungeKutta.h:72-112). */
static const double TINY = 1e-20, SAFETY = 0.9, PGROW = -0.2, PSHRNK = -0.25, ERRCON = 1.89e-4,
                    HFACTOR = 0.1;
#define B21 0.2
#define B31 (3.0 / 40.0)
#define B32 (9.0 / 40.0)
#define B41 0.3
#define B42 (-0.9)
#define B43 1.2
#define B51 (-11.0 / 54.0)
#define B52 2.5
#define B53 (-70.0 / 27.0)
#define B54 (35.0 / 27.0)
#define B61 (1631.0 / 55296.0)
#define B62 (175.0 / 512.0)
#define B63 (575.0 / 13824.0)
#define B64 (44275.0 / 110592.0)
#define B65 (253.0 / 4096.0)
#define C1 (37.0 / 378.0)
#define C3 (250.0 / 621.0)
#define C4 (125.0 / 594.0)
#define C6 (512.0 / 1771.0)
#define DC5 (-277.0 / 14336.0)

typedef struct {
    const orc_problem* p;
    int logspace;
    size_t nn; /* N + M + 1 */
    double *dxdt, *xscal, *temp, *xerr, *ak2, *ak3, *ak4, *ak5, *ak6, *xnew;
    double time, hnext, hdid, eps;
    int steps, attempts, rhscount;
} rk_t;

static void rk_init(rk_t* rk, const orc_problem* p, double eps, int logspace) {
    size_t nn = (size_t)(p->n + p->m + 1);
    rk->p = p;
    rk->logspace = logspace;
    rk->nn = nn;
    rk->dxdt = (double*)calloc(nn * 10, sizeof(double));
    rk->xscal = rk->dxdt + nn;
    rk->temp = rk->xscal + nn;
    rk->xerr = rk->temp + nn;
    rk->ak2 = rk->xerr + nn;
    rk->ak3 = rk->ak2 + nn;
    rk->ak4 = rk->ak3 + nn;
    rk->ak5 = rk->ak4 + nn;
    rk->ak6 = rk->ak5 + nn;
    rk->xnew = rk->ak6 + nn;
    /* CpuRungeKutta::Reset (CpuRungeKutta.cpp:168-177) */
    rk->hnext = 1e-9;
    rk->hdid = 0.0;
    rk->time = 0.0;
    rk->steps = rk->attempts = rk->rhscount = 0;
    rk->eps = eps;
}

static void rk_free(rk_t* rk) { free(rk->dxdt); }

/* CpuRungeKutta::rkck (CpuRungeKutta.cpp:181-215) */
static void rkck(rk_t* rk, const double* x, double h) {
    const size_t n = rk->nn;
    const double dc1 = C1 - 2825.0 / 27648.0, dc3 = C3 - 18575.0 / 48384.0,
                 dc4 = C4 - 13525.0 / 55296.0, dc6 = C6 - 0.25;
    double *d = rk->dxdt, *t = rk->temp, *k2 = rk->ak2, *k3 = rk->ak3, *k4 = rk->ak4,
           *k5 = rk->ak5, *k6 = rk->ak6;
    size_t i;
    for (i = 0; i < n; i++) t[i] = x[i] + B21 * h * d[i];
    rhs_internal(rk->p, t, k2, rk->logspace); rk->rhscount++;
    for (i = 0; i < n; i++) t[i] = x[i] + h * (B31 * d[i] + B32 * k2[i]);
    rhs_internal(rk->p, t, k3, rk->logspace); rk->rhscount++;
    for (i = 0; i < n; i++) t[i] = x[i] + h * (B41 * d[i] + B42 * k2[i] + B43 * k3[i]);
    rhs_internal(rk->p, t, k4, rk->logspace); rk->rhscount++;
    for (i = 0; i < n; i++) t[i] = x[i] + h * (B51 * d[i] + B52 * k2[i] + B53 * k3[i] + B54 * k4[i]);
    rhs_internal(rk->p, t, k5, rk->logspace); rk->rhscount++;
    for (i = 0; i < n; i++)
        t[i] = x[i] + h * (B61 * d[i] + B62 * k2[i] + B63 * k3[i] + B64 * k4[i] + B65 * k5[i]);
    rhs_internal(rk->p, t, k6, rk->logspace); rk->rhscount++;
    for (i = 0; i < n; i++) rk->xnew[i] = x[i] + h * (C1 * d[i] + C3 * k3[i] + C4 * k4[i] + C6 * k6[i]);
    for (i = 0; i < n; i++)
        rk->xerr[i] = h * (dc1 * d[i] + dc3 * k3[i] + dc4 * k4[i] + DC5 * k5[i] + dc6 * k6[i]);
}

/* CpuRungeKutta::Step with count = 1 (CpuRungeKutta.cpp:66-100) and rkqs (218-267).
 * In log space the a-block scale is 1 + |h du/dt| (the reference's |a| + |h da/dt| divided
 * by a), so the controller measures the same relative error of a. */
static int rk_step(rk_t* rk, double* x) {
    const orc_problem* p = rk->p;
    const size_t n = rk->nn;
    const size_t abeg = (size_t)p->n + 1;
    double h, ermax = 0.0;
    size_t i;
    rhs_internal(p, x, rk->dxdt, rk->logspace);
    rk->rhscount++;
    for (i = 0; i < n; i++) {
        double xa = (rk->logspace && i >= abeg) ? 1.0 : fabs(x[i]);
        rk->xscal[i] = xa + fabs(rk->dxdt[i] * rk->hnext) + TINY;
    }
    h = rk->hnext;
    for (;;) {
        rkck(rk, x, h);
        rk->attempts++;
        ermax = 0.0;
        for (i = 0; i < n; i++) ermax = fmax(ermax, fabs(rk->xerr[i] / rk->xscal[i]));
        ermax /= rk->eps;
        if (ermax <= 1.0) break;
        {
            double htemp = SAFETY * h * pow(ermax, PSHRNK);
            h = h >= 0.0 ? fmax(htemp, HFACTOR * h) : fmin(htemp, HFACTOR * h);
            if (rk->time + h == rk->time) return 0;
        }
    }
    if (ermax > ERRCON) rk->hnext = SAFETY * h * pow(ermax, PGROW);
    else rk->hnext = 5.0 * h;
    rk->hdid = h;
    rk->time += h;
    rk->steps++;
    memcpy(x, rk->xnew, sizeof(double) * n);
    return 1;
}

static void load_ic(const orc_problem* p, const double* ic, double* x, int logspace) {
    int j;
    x[0] = -1.0;
    memcpy(x + 1, ic, sizeof(double) * (size_t)(p->n + p->m));
    if (logspace)
        for (j = 0; j < p->m; j++) x[p->n + 1 + j] = log(x[p->n + 1 + j]);
}

static void store_pub(const orc_problem* p, const double* x, double* out, int logspace) {
    int j;
    memcpy(out, x + 1, sizeof(double) * (size_t)(p->n + p->m));
    if (logspace)
        for (j = 0; j < p->m; j++) out[p->n + j] = exp(out[p->n + j]);
}

int orc_steps(const orc_problem* p, const double* ic, double eps, int nsteps, int logspace,
              double* times, double* hs, int* rhs, int* attempts, double* states) {
    rk_t rk;
    int s;
    double* x = (double*)malloc(sizeof(double) * (size_t)(p->n + p->m + 1));
    rk_init(&rk, p, eps, logspace);
    load_ic(p, ic, x, logspace);
    for (s = 0; s < nsteps; s++) {
        if (!rk_step(&rk, x)) break;
        times[s] = rk.time;
        hs[s] = rk.hdid;
        rhs[s] = rk.rhscount;
        attempts[s] = rk.attempts;
        store_pub(p, x, states + (size_t)s * (size_t)(p->n + p->m), logspace);
    }
    rk_free(&rk);
    free(x);
    return s;
}

/* SatSolver::DoSolve, no-callback branch (AnalogSAT/solver/SatSolver.h:273-355). */
int orc_solve(const orc_problem* p, const double* ic, double eps, double tmax, int maxsteps,
              int batch, int logspace, double* final_state, double* out_time, int* out_steps,
              int* out_rhs, int* out_attempts, int* out_viol) {
    rk_t rk;
    int result = 5; /* SAT_UNKNOWN */
    int steps = 0, viol = -1, b;
    double time = 0.0;
    double* x = (double*)malloc(sizeof(double) * (size_t)(p->n + p->m + 1));
    rk_init(&rk, p, eps, logspace);
    load_ic(p, ic, x, logspace);
    while (time < tmax && steps < maxsteps) {
        int before = rk.steps, ok = 1;
        for (b = 0; b < batch; b++)
            if (!rk_step(&rk, x)) { ok = 0; break; }
        if (!ok) { result = 1; break; }
        steps += rk.steps - before;
        time = rk.time;
        viol = orc_violations(p, x + 1);
        if (viol == 0) { result = 0; break; }
    }
    if (result == 5) {
        if (time >= tmax) result = 3;
        else if (steps >= maxsteps) result = 4;
    }
    if (final_state) store_pub(p, x, final_state, logspace);
    if (out_time) *out_time = rk.time;
    if (out_steps) *out_steps = steps;
    if (out_rhs) *out_rhs = rk.rhscount;
    if (out_attempts) *out_attempts = rk.attempts;
    if (out_viol) *out_viol = viol;
    rk_free(&rk);
    free(x);
    return result;
}

/* Dense-output reference: the same controller, but the last step is clamped so the
 * integration ends at t_end (used to compare runs whose step sequences differ). */
int orc_integrate_to(const orc_problem* p, const double* ic, double eps, double t_end,
                     int logspace, int maxsteps, double* out_state, double* out_time) {
    rk_t rk;
    int s = 0;
    double* x = (double*)malloc(sizeof(double) * (size_t)(p->n + p->m + 1));
    rk_init(&rk, p, eps, logspace);
    load_ic(p, ic, x, logspace);
    while (rk.time < t_end && s < maxsteps) {
        if (rk.time + rk.hnext > t_end) rk.hnext = t_end - rk.time;
        if (!rk_step(&rk, x)) break;
        s++;
    }
    store_pub(p, x, out_state, logspace);
    *out_time = rk.time;
    rk_free(&rk);
    free(x);
    return s;
}

double orc_potential(const orc_problem* p, const double* x, const double* w) {
    int j, q;
    double v = 0.0;
    for (j = 0; j < p->m; j++) {
        double km = p->knorm;
        for (q = 0; q < p->k; q++) {
            int idx = p->C[(size_t)j * p->k + q];
            double s = idx != 0 ? x[abs(idx) - 1] : -1.0;
            km *= idx < 0 ? 1.0 + s : 1.0 - s;
        }
        v += (w ? w[j] : 1.0) * x[p->n + j] * km * km;
    }
    return v;
}

/* ------------------------------------------------------------------------------------
 * Differentiation (no reference counterpart: the reference has no gradients).
 * Weighted CTDS: a_m -> w_m a_m in the potential and in the spin equation,
 *   ds_i = sum_m 2 w_m a_m c_mi K_mi K_m,   da_m = a_m K_m^2,
 *   L    = V(x(T)) = sum_m w_m a_m(T) K_m(s(T))^2      (w = 1 is the reference ODE).
 * The adaptive controller runs once (forward, last step clamped to end at T) and its
 * accepted step sizes are then frozen: L is a smooth function of (s(0), a(0), w)
 * through the fixed-step Cash-Karp map, and the discrete adjoint below is its exact
 * gradient (checked against central finite differences in tests/test_oracle.py).
 * State vectors here are public-layout [s_1..s_N, a_1..a_M], a linear.
 * ------------------------------------------------------------------------------------ */

static void clause_vals(const orc_problem* p, const double* x, int j, double* f, int* v, double* c) {
    int q;
    for (q = 0; q < p->k; q++) {
        int idx = p->C[(size_t)j * p->k + q];
        if (idx == 0) { f[q] = 2.0; v[q] = -1; c[q] = 1.0; continue; }
        v[q] = abs(idx) - 1;
        c[q] = idx < 0 ? -1.0 : 1.0;
        f[q] = 1.0 - c[q] * x[v[q]];
    }
}

static double prod_except(const double* f, int k, int a, int b) {
    double r = 1.0;
    int l;
    for (l = 0; l < k; l++)
        if (l != a && l != b) r *= f[l];
    return r;
}

/* f(x; w) */
static void wrhs(const orc_problem* p, const double* x, const double* w, double* d) {
    const int n = p->n, m = p->m, k = p->k;
    double f[64], c[64];
    int v[64], j, q;
    memset(d, 0, sizeof(double) * (size_t)(n + m));
    for (j = 0; j < m; j++) {
        double K, a = x[n + j], wj = w ? w[j] : 1.0;
        clause_vals(p, x, j, f, v, c);
        K = p->knorm * prod_except(f, k, -1, -1);
        d[n + j] = a * K * K;
        for (q = 0; q < k; q++)
            if (v[q] >= 0) d[v[q]] += 2.0 * wj * a * c[q] * (p->knorm * prod_except(f, k, q, -1)) * K;
    }
}

/* J(x)^T u and the w-gradient contribution g_w += (df/dw)^T u. */
static void wvjp(const orc_problem* p, const double* x, const double* w, const double* u, double* out,
                 double* gw) {
    const int n = p->n, m = p->m, k = p->k;
    double f[64], c[64], Kq[64];
    int v[64], j, q, r;
    memset(out, 0, sizeof(double) * (size_t)(n + m));
    for (j = 0; j < m; j++) {
        const double a = x[n + j], wj = w ? w[j] : 1.0, ua = u[n + j];
        double K, S = 0.0;
        clause_vals(p, x, j, f, v, c);
        K = p->knorm * prod_except(f, k, -1, -1);
        for (q = 0; q < k; q++) Kq[q] = p->knorm * prod_except(f, k, q, -1);
        for (q = 0; q < k; q++)
            if (v[q] >= 0) S += u[v[q]] * c[q] * Kq[q];
        /* d/da_m: sum_q u_q 2 w c_q K_q K + ua K^2 ;  d/dw_m: sum_q u_q 2 a c_q K_q K */
        out[n + j] = 2.0 * wj * S * K + ua * K * K;
        if (gw) gw[j] += 2.0 * a * S * K;
        /* d/ds_r: -2 c_r [ w a sum_q u_q c_q (K_qr K [q!=r] + K_q K_r) + ua a K K_r ] */
        for (r = 0; r < k; r++) {
            double t = 0.0;
            if (v[r] < 0) continue;
            for (q = 0; q < k; q++) {
                double term;
                if (v[q] < 0) continue;
                term = Kq[q] * Kq[r];
                if (q != r) term += p->knorm * prod_except(f, k, q, r) * K;
                t += u[v[q]] * c[q] * term;
            }
            out[v[r]] += -2.0 * c[r] * (wj * a * t + ua * a * K * Kq[r]);
        }
    }
}

static double wpotential(const orc_problem* p, const double* x, const double* w) {
    return orc_potential(p, x, w);
}

static const double CK_B[7][6] = {
    {0}, {0}, {B21}, {B31, B32}, {B41, B42, B43}, {B51, B52, B53, B54}, {B61, B62, B63, B64, B65}};
static const double CK_C[7] = {0, C1, 0.0, C3, C4, 0.0, C6};

/* One fixed-step Cash-Karp step: x <- x + h sum c_j k_j (k's kept in K[1..6]). */
static void ck_fixed(const orc_problem* p, double* x, const double* w, double h, double* K[7], double* y) {
    const size_t E = (size_t)(p->n + p->m);
    int s, l;
    size_t i;
    for (s = 1; s <= 6; s++) {
        for (i = 0; i < E; i++) {
            double acc = 0.0;
            for (l = 1; l < s; l++) acc += CK_B[s][l - 1] * K[l][i];
            y[i] = x[i] + h * acc;
        }
        wrhs(p, y, w, K[s]);
    }
    for (i = 0; i < E; i++) {
        double acc = 0.0;
        for (s = 1; s <= 6; s++) acc += CK_C[s] * K[s][i];
        x[i] += h * acc;
    }
}

/* Forward adaptive run to t_end (last step clamped), recording accepted step sizes.
 * Returns the number of steps (or -1 if more than maxsteps). */
int orc_record_steps(const orc_problem* p, const double* ic, double eps, double t_end, int maxsteps,
                     double* hs) {
    rk_t rk;
    int s = 0;
    double* x = (double*)malloc(sizeof(double) * (size_t)(p->n + p->m + 1));
    rk_init(&rk, p, eps, 0);
    load_ic(p, ic, x, 0);
    while (rk.time < t_end) {
        if (s >= maxsteps) { s = -1; break; }
        if (rk.time + rk.hnext > t_end) rk.hnext = t_end - rk.time;
        if (!rk_step(&rk, x)) { s = -1; break; }
        hs[s++] = rk.hdid;
    }
    rk_free(&rk);
    free(x);
    return s;
}

/* L(x0, w) through the fixed step sequence hs[0..nsteps). */
double orc_fixed_loss(const orc_problem* p, const double* x0, const double* w, const double* hs, int nsteps,
                      double* x_final) {
    const size_t E = (size_t)(p->n + p->m);
    double *x = (double*)malloc(sizeof(double) * E * 8), *K[7], *y, L;
    int s;
    for (s = 1; s <= 6; s++) K[s] = x + E * (size_t)s;
    y = x + E * 7;
    memcpy(x, x0, sizeof(double) * E);
    for (s = 0; s < nsteps; s++) ck_fixed(p, x, w, hs[s], K, y);
    L = wpotential(p, x, w);
    if (x_final) memcpy(x_final, x, sizeof(double) * E);
    free(x);
    return L;
}

/* Discrete adjoint of orc_fixed_loss: g_x0 = dL/dx0 (public layout), g_w = dL/dw. */
double orc_adjoint(const orc_problem* p, const double* x0, const double* w, const double* hs, int nsteps,
                   double* g_x0, double* g_w) {
    const size_t E = (size_t)(p->n + p->m);
    const int n = p->n, m = p->m;
    double *ck = (double*)malloc(sizeof(double) * E * (size_t)(nsteps + 1));
    double *buf = (double*)malloc(sizeof(double) * E * 20), *K[7], *sig[7], *y, *lam, *rho, *tmp, L;
    int s, j, i2, l;
    size_t i;
    for (s = 1; s <= 6; s++) K[s] = buf + E * (size_t)(s - 1);
    for (s = 1; s <= 6; s++) sig[s] = buf + E * (size_t)(5 + s);
    y = buf + E * 12; lam = buf + E * 13; rho = buf + E * 14; tmp = buf + E * 15;
    /* forward with checkpoints */
    memcpy(ck, x0, sizeof(double) * E);
    for (s = 0; s < nsteps; s++) {
        memcpy(ck + E * (size_t)(s + 1), ck + E * (size_t)s, sizeof(double) * E);
        ck_fixed(p, ck + E * (size_t)(s + 1), w, hs[s], K, y);
    }
    {
        const double* xT = ck + E * (size_t)nsteps;
        L = wpotential(p, xT, w);
        /* dL/dx(T): spins -ds (weighted RHS), weights w K^2; dL/dw = a K^2 */
        wrhs(p, xT, w, tmp);
        for (i = 0; i < (size_t)n; i++) lam[i] = -tmp[i];
        for (j = 0; j < m; j++) {
            const double a = xT[n + j];
            const double Kk2 = a > 0 ? tmp[n + j] / a : 0.0; /* K^2 = (a K^2) / a */
            double f[64], c[64], KK;
            int v[64];
            clause_vals(p, xT, j, f, v, c);
            KK = p->knorm * prod_except(f, p->k, -1, -1);
            (void)Kk2;
            lam[n + j] = (w ? w[j] : 1.0) * KK * KK;
            if (g_w) g_w[j] = a * KK * KK;
        }
    }
    /* backward over steps */
    for (s = nsteps - 1; s >= 0; s--) {
        const double h = hs[s];
        const double* xs = ck + E * (size_t)s;
        /* recompute stage derivatives k1..k5 */
        for (j = 1; j <= 5; j++) {
            for (i = 0; i < E; i++) {
                double acc = 0.0;
                for (l = 1; l < j; l++) acc += CK_B[j][l - 1] * K[l][i];
                y[i] = xs[i] + h * acc;
            }
            wrhs(p, y, w, K[j]);
        }
        for (j = 6; j >= 1; j--) {
            for (i = 0; i < E; i++) {
                double acc = CK_C[j] * lam[i];
                for (i2 = j + 1; i2 <= 6; i2++) acc += CK_B[i2][j - 1] * sig[i2][i];
                rho[i] = h * acc;
            }
            for (i = 0; i < E; i++) {
                double acc = 0.0;
                for (l = 1; l < j; l++) acc += CK_B[j][l - 1] * K[l][i];
                y[i] = xs[i] + h * acc;
            }
            wvjp(p, y, w, rho, sig[j], g_w);
        }
        for (i = 0; i < E; i++)
            lam[i] += sig[1][i] + sig[2][i] + sig[3][i] + sig[4][i] + sig[5][i] + sig[6][i];
    }
    memcpy(g_x0, lam, sizeof(double) * E);
    free(ck);
    free(buf);
    return L;
}
