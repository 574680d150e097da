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
};

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
