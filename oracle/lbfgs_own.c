/*
 * oracle/lbfgs_own.c -- an FP64 L-BFGS behind the libLBFGS 1.10 API used by
 * the reference `clib/pyCNCS/ncs.c` (ncs.c:416, :443, :539-561).
 * TEST INFRASTRUCTURE ONLY (CPU oracle); never on the shipped CUDA path.
 *
 * Algorithm, restated from the published sources rather than from libLBFGS's
 * (absent) source code:
 *  - Limited-memory BFGS with the two-loop recursion of J. Nocedal,
 *    "Updating quasi-Newton matrices with limited storage", Math. Comp. 35
 *    (1980), initial inverse Hessian (s'y / y'y) I from the newest pair.
 *  - Default line search: Moré & Thuente, "Line search algorithms with
 *    guaranteed sufficient decrease", ACM TOMS 20(3):286-307 (1994) -- the
 *    safeguarded cubic/quadratic interval update of their Section 4 and the
 *    two-stage (modified function / original function) driver, enforcing the
 *    strong Wolfe conditions with ftol and gtol.
 *  - Backtracking line searches (Armijo / Wolfe / strong Wolfe) as documented
 *    in lbfgs.h:158-189 (step x 0.5 on failed decrease, x 2.1 on failed
 *    curvature).
 *  - Defaults and stopping rule exactly as documented in lbfgs.h:198-358:
 *    m = 6, epsilon = 1e-5 on ||g|| / max(1, ||x||), unlimited iterations,
 *    max_linesearch = 20, min_step = 1e-20, max_step = 1e20, ftol = 1e-4,
 *    wolfe = 0.9, gtol = 0.9, xtol = 1e-16.
 *  - The first step length is 1/||g|| along -g, later iterations try 1.
 *  - Trial points are written into the caller's x before the callback runs;
 *    ncs.c relies on this because its evaluator reads its own copy of x
 *    (ncs.c:335-364 uses ncs_sr->u, the array passed to lbfgs at :554-557).
 *  - On a failed line search the previous point and gradient are restored.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "lbfgs_api.h"

/* ---- oracle overrides and statistics ---------------------------------- */

static int g_ovr_max_iterations = 0;
static double g_ovr_epsilon = -1.0;
static int g_ovr_m = 0;
static int g_ovr_linesearch = -1;

static __thread long t_calls, t_iterations, t_evaluations, t_failures;
static __thread int t_last_status, t_last_iterations;

void ncs_oracle_set_overrides(int max_iterations, double epsilon, int m, int linesearch) {
    g_ovr_max_iterations = max_iterations < 0 ? 0 : max_iterations;
    g_ovr_epsilon = epsilon;
    g_ovr_m = m;
    g_ovr_linesearch = linesearch;
}

void ncs_oracle_reset_stats(void) {
    t_calls = t_iterations = t_evaluations = t_failures = 0;
    t_last_status = 0;
    t_last_iterations = 0;
}

void ncs_oracle_get_stats(long *calls, long *iterations, long *evaluations, long *failures,
                          int *last_status, int *last_iterations) {
    if (calls) *calls = t_calls;
    if (iterations) *iterations = t_iterations;
    if (evaluations) *evaluations = t_evaluations;
    if (failures) *failures = t_failures;
    if (last_status) *last_status = t_last_status;
    if (last_iterations) *last_iterations = t_last_iterations;
}

/* ---- small vector helpers --------------------------------------------- */

static double dot(const double *a, const double *b, int n) {
    double s = 0.0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

static double max3(double a, double b, double c) {
    double m = a > b ? a : b;
    return m > c ? m : c;
}

void lbfgs_parameter_init(lbfgs_parameter_t *p) {
    p->m = 6;
    p->epsilon = 1e-5;
    p->past = 0;
    p->delta = 1e-5;
    p->max_iterations = 0;
    p->linesearch = LBFGS_LINESEARCH_DEFAULT;
    p->max_linesearch = 20;
    p->min_step = 1e-20;
    p->max_step = 1e20;
    p->ftol = 1e-4;
    p->wolfe = 0.9;
    p->gtol = 0.9;
    p->xtol = 1e-16;
    p->orthantwise_c = 0.0;
    p->orthantwise_start = 0;
    p->orthantwise_end = -1;
    /* oracle overrides (see lbfgs_api.h) */
    if (g_ovr_max_iterations > 0) p->max_iterations = g_ovr_max_iterations;
    if (g_ovr_epsilon >= 0.0) p->epsilon = g_ovr_epsilon;
    if (g_ovr_m > 0) p->m = g_ovr_m;
    if (g_ovr_linesearch >= 0) p->linesearch = g_ovr_linesearch;
}

lbfgsfloatval_t *lbfgs_malloc(int n) {
    void *ptr = NULL;
    if (n <= 0) n = 1;
    if (posix_memalign(&ptr, 16, sizeof(lbfgsfloatval_t) * (size_t)n) != 0) return NULL;
    return (lbfgsfloatval_t *)ptr;
}

void lbfgs_free(lbfgsfloatval_t *x) { free(x); }

typedef struct {
    int n;
    void *instance;
    lbfgs_evaluate_t eval;
} eval_ctx;

/* ---- Moré–Thuente interval update (their Section 4) -------------------- */

/*
 * Given the interval end points (lo, flo, dlo) = best step so far and
 * (hi, fhi, dhi) = the other end, and a trial (t, ft, dt), compute the next
 * trial step in *t and update the interval.  `bracketed` becomes 1 once the
 * minimiser is known to lie between lo and hi.  Returns 0 or an error code.
 */
static int mt_update(double *lo, double *flo, double *dlo,
                     double *hi, double *fhi, double *dhi,
                     double *t, double ft, double dt,
                     int *bracketed, double tmin, double tmax) {
    double cub, quad, next, theta, s, gam, p, q, r;
    int clamp_to_interval = 0;
    double sign_change = dt * (*dlo / fabs(*dlo));

    if (*bracketed) {
        double a = *lo < *hi ? *lo : *hi, b = *lo < *hi ? *hi : *lo;
        if (*t <= a || *t >= b) return LBFGSERR_OUTOFINTERVAL;
        if (*dlo * (*t - *lo) >= 0.0) return LBFGSERR_INCREASEGRADIENT;
        if (tmax < tmin) return LBFGSERR_INCORRECT_TMINMAX;
    }

    if (ft > *flo) {
        /* Case 1: the trial has a higher value; the minimiser is bracketed.
           Take the cubic step if it is closer to lo than the quadratic one,
           else their midpoint. */
        clamp_to_interval = 1;
        theta = 3.0 * (*flo - ft) / (*t - *lo) + *dlo + dt;
        s = max3(fabs(theta), fabs(*dlo), fabs(dt));
        gam = s * sqrt((theta / s) * (theta / s) - (*dlo / s) * (dt / s));
        if (*t < *lo) gam = -gam;
        p = (gam - *dlo) + theta;
        q = ((gam - *dlo) + gam) + dt;
        r = p / q;
        cub = *lo + r * (*t - *lo);
        quad = *lo + ((*dlo / ((*flo - ft) / (*t - *lo) + *dlo)) / 2.0) * (*t - *lo);
        if (fabs(cub - *lo) < fabs(quad - *lo))
            next = cub;
        else
            next = cub + (quad - cub) / 2.0;
        *bracketed = 1;
    } else if (sign_change < 0.0) {
        /* Case 2: lower value, derivatives of opposite sign; bracketed.
           Take whichever of the cubic and secant steps is farther from t. */
        theta = 3.0 * (*flo - ft) / (*t - *lo) + *dlo + dt;
        s = max3(fabs(theta), fabs(*dlo), fabs(dt));
        gam = s * sqrt((theta / s) * (theta / s) - (*dlo / s) * (dt / s));
        if (*t > *lo) gam = -gam;
        p = (gam - dt) + theta;
        q = ((gam - dt) + gam) + *dlo;
        r = p / q;
        cub = *t + r * (*lo - *t);
        quad = *t + (dt / (dt - *dlo)) * (*lo - *t);
        next = fabs(cub - *t) > fabs(quad - *t) ? cub : quad;
        *bracketed = 1;
    } else if (fabs(dt) < fabs(*dlo)) {
        /* Case 3: lower value, same-sign derivatives, |derivative| shrinks.
           The cubic step is used only if it tends to infinity in the
           direction of the step or its minimum lies beyond t. */
        clamp_to_interval = 1;
        theta = 3.0 * (*flo - ft) / (*t - *lo) + *dlo + dt;
        s = max3(fabs(theta), fabs(*dlo), fabs(dt));
        {
            double disc = (theta / s) * (theta / s) - (*dlo / s) * (dt / s);
            gam = s * sqrt(disc > 0.0 ? disc : 0.0);
        }
        if (*t > *lo) gam = -gam;
        p = (gam - dt) + theta;
        q = (gam + (*dlo - dt)) + gam;
        r = p / q;
        if (r < 0.0 && gam != 0.0)
            cub = *t + r * (*lo - *t);
        else if (*t > *lo)
            cub = tmax;
        else
            cub = tmin;
        quad = *t + (dt / (dt - *dlo)) * (*lo - *t);
        if (*bracketed)
            next = fabs(*t - cub) < fabs(*t - quad) ? cub : quad;
        else
            next = fabs(*t - cub) > fabs(*t - quad) ? cub : quad;
    } else {
        /* Case 4: lower value, same-sign derivatives, |derivative| does not
           shrink.  Use the cubic through t and hi if bracketed, else extend
           to the step bound. */
        if (*bracketed) {
            theta = 3.0 * (ft - *fhi) / (*hi - *t) + *dhi + dt;
            s = max3(fabs(theta), fabs(*dhi), fabs(dt));
            gam = s * sqrt((theta / s) * (theta / s) - (*dhi / s) * (dt / s));
            if (*t > *hi) gam = -gam;
            p = (gam - dt) + theta;
            q = ((gam - dt) + gam) + *dhi;
            r = p / q;
            next = *t + r * (*hi - *t);
        } else {
            next = *t > *lo ? tmax : tmin;
        }
    }

    /* Update the interval of uncertainty. */
    if (ft > *flo) {
        *hi = *t; *fhi = ft; *dhi = dt;
    } else {
        if (sign_change < 0.0) { *hi = *lo; *fhi = *flo; *dhi = *dlo; }
        *lo = *t; *flo = ft; *dlo = dt;
    }

    /* Safeguard the new step. */
    if (next > tmax) next = tmax;
    if (next < tmin) next = tmin;
    *t = next;
    if (*bracketed && clamp_to_interval) {
        double lim = *lo + 0.66 * (*hi - *lo);
        if (*hi > *lo) {
            if (lim < *t) *t = lim;
        } else {
            if (lim > *t) *t = lim;
        }
    }
    return 0;
}

/* x = xp + t d; f = eval(x); returns f and fills g. */
static double eval_at(eval_ctx *ec, double *x, const double *xp, const double *d, double t,
                      double *g) {
    for (int i = 0; i < ec->n; i++) x[i] = xp[i] + t * d[i];
    t_evaluations++;
    return ec->eval(ec->instance, x, g, ec->n, t);
}

/* Moré–Thuente driver.  Returns the number of evaluations (>0) or an error. */
static int ls_more_thuente(eval_ctx *ec, double *x, double *f, double *g, const double *d,
                           double *stp, const double *xp, const lbfgs_parameter_t *prm) {
    int n = ec->n, count = 0, bracketed = 0, stage1 = 1, info = 0;
    double dg0, f0, suff, width, width_prev, tmin, tmax;
    double lo = 0.0, flo, dlo, hi = 0.0, fhi, dhi;

    if (*stp <= 0.0) return LBFGSERR_INVALIDPARAMETERS;
    dg0 = dot(g, d, n);
    if (dg0 > 0.0) return LBFGSERR_INCREASEGRADIENT;
    f0 = *f;
    suff = prm->ftol * dg0;
    width = prm->max_step - prm->min_step;
    width_prev = 2.0 * width;
    flo = fhi = f0;
    dlo = dhi = dg0;

    for (;;) {
        double dg, fthresh;
        if (bracketed) {
            tmin = lo < hi ? lo : hi;
            tmax = lo < hi ? hi : lo;
        } else {
            tmin = lo;
            tmax = *stp + 4.0 * (*stp - lo);
        }
        if (*stp < prm->min_step) *stp = prm->min_step;
        if (*stp > prm->max_step) *stp = prm->max_step;
        /* On an imminent abnormal exit fall back to the best step so far. */
        if ((bracketed && (*stp <= tmin || *stp >= tmax || prm->max_linesearch <= count + 1 ||
                           info != 0)) ||
            (bracketed && tmax - tmin <= prm->xtol * tmax))
            *stp = lo;

        *f = eval_at(ec, x, xp, d, *stp, g);
        dg = dot(g, d, n);
        fthresh = f0 + *stp * suff;
        ++count;

        if (bracketed && (*stp <= tmin || *stp >= tmax || info != 0))
            return LBFGSERR_ROUNDING_ERROR;
        if (*stp == prm->max_step && *f <= fthresh && dg <= suff) return LBFGSERR_MAXIMUMSTEP;
        if (*stp == prm->min_step && (*f > fthresh || dg >= suff)) return LBFGSERR_MINIMUMSTEP;
        if (bracketed && tmax - tmin <= prm->xtol * tmax) return LBFGSERR_WIDTHTOOSMALL;
        if (count >= prm->max_linesearch) return LBFGSERR_MAXIMUMLINESEARCH;
        /* strong Wolfe conditions */
        if (*f <= fthresh && fabs(dg) <= prm->gtol * (-dg0)) return count;

        if (stage1 && *f <= fthresh && dg >= (prm->ftol < prm->gtol ? prm->ftol : prm->gtol) * dg0)
            stage1 = 0;

        if (stage1 && *f > fthresh && *f <= flo) {
            /* first stage: work on the modified function f(t) - t*suff */
            double fm = *f - *stp * suff, dgm = dg - suff;
            double flom = flo - lo * suff, fhim = fhi - hi * suff;
            double dlom = dlo - suff, dhim = dhi - suff;
            info = mt_update(&lo, &flom, &dlom, &hi, &fhim, &dhim, stp, fm, dgm, &bracketed, tmin,
                             tmax);
            flo = flom + lo * suff;
            fhi = fhim + hi * suff;
            dlo = dlom + suff;
            dhi = dhim + suff;
        } else {
            info = mt_update(&lo, &flo, &dlo, &hi, &fhi, &dhi, stp, *f, dg, &bracketed, tmin, tmax);
        }

        /* Insist on a sufficient shrink of the bracket; bisect otherwise. */
        if (bracketed) {
            if (fabs(hi - lo) >= 0.66 * width_prev) *stp = lo + 0.5 * (hi - lo);
            width_prev = width;
            width = fabs(hi - lo);
        }
    }
}

/* Backtracking searches of lbfgs.h:158-189. */
static int ls_backtracking(eval_ctx *ec, double *x, double *f, double *g, const double *d,
                           double *stp, const double *xp, const lbfgs_parameter_t *prm) {
    int n = ec->n, count = 0;
    double dg0, f0, suff;
    if (*stp <= 0.0) return LBFGSERR_INVALIDPARAMETERS;
    dg0 = dot(g, d, n);
    if (dg0 > 0.0) return LBFGSERR_INCREASEGRADIENT;
    f0 = *f;
    suff = prm->ftol * dg0;
    for (;;) {
        double dg, factor;
        *f = eval_at(ec, x, xp, d, *stp, g);
        ++count;
        if (*f > f0 + *stp * suff) {
            factor = 0.5;
        } else {
            if (prm->linesearch == LBFGS_LINESEARCH_BACKTRACKING_ARMIJO) return count;
            dg = dot(g, d, n);
            if (dg < prm->wolfe * dg0) {
                factor = 2.1;
            } else {
                if (prm->linesearch == LBFGS_LINESEARCH_BACKTRACKING_WOLFE) return count;
                if (dg > -prm->wolfe * dg0) factor = 0.5;
                else return count;
            }
        }
        if (*stp < prm->min_step) return LBFGSERR_MINIMUMSTEP;
        if (*stp > prm->max_step) return LBFGSERR_MAXIMUMSTEP;
        if (count >= prm->max_linesearch) return LBFGSERR_MAXIMUMLINESEARCH;
        *stp *= factor;
    }
}

static int check_params(int n, const lbfgs_parameter_t *p) {
    if (n <= 0) return LBFGSERR_INVALID_N;
    if (p->epsilon < 0.0) return LBFGSERR_INVALID_EPSILON;
    if (p->past < 0) return LBFGSERR_INVALID_TESTPERIOD;
    if (p->delta < 0.0) return LBFGSERR_INVALID_DELTA;
    if (p->min_step < 0.0) return LBFGSERR_INVALID_MINSTEP;
    if (p->max_step < p->min_step) return LBFGSERR_INVALID_MAXSTEP;
    if (p->ftol < 0.0) return LBFGSERR_INVALID_FTOL;
    if (p->linesearch == LBFGS_LINESEARCH_BACKTRACKING_WOLFE ||
        p->linesearch == LBFGS_LINESEARCH_BACKTRACKING_STRONG_WOLFE) {
        if (p->wolfe <= p->ftol || 1.0 <= p->wolfe) return LBFGSERR_INVALID_WOLFE;
    }
    if (p->gtol < 0.0) return LBFGSERR_INVALID_GTOL;
    if (p->xtol < 0.0) return LBFGSERR_INVALID_XTOL;
    if (p->max_linesearch <= 0) return LBFGSERR_INVALID_MAXLINESEARCH;
    if (p->orthantwise_c != 0.0) return LBFGSERR_INVALID_ORTHANTWISE; /* OWL-QN not needed */
    if (p->linesearch < 0 || p->linesearch > LBFGS_LINESEARCH_BACKTRACKING_STRONG_WOLFE)
        return LBFGSERR_INVALID_LINESEARCH;
    if (p->m <= 0) return LBFGSERR_INVALIDPARAMETERS;
    return 0;
}

int lbfgs(int n, lbfgsfloatval_t *x, lbfgsfloatval_t *ptr_fx, lbfgs_evaluate_t proc_evaluate,
          lbfgs_progress_t proc_progress, void *instance, lbfgs_parameter_t *_param) {
    lbfgs_parameter_t prm;
    int ret, m, k, newest, stored;
    double fx = 0.0, step, xnorm, gnorm;
    double *xp, *g, *gp, *d, *S, *Y, *rho, *alpha, *pf = NULL;
    eval_ctx ec;

    if (_param) prm = *_param; else lbfgs_parameter_init(&prm);
    ret = check_params(n, &prm);
    t_calls++;
    if (ret != 0) {
        t_failures++;
        t_last_status = ret;
        t_last_iterations = 0;
        return ret;
    }
    m = prm.m;
    ec.n = n;
    ec.instance = instance;
    ec.eval = proc_evaluate;

    xp = (double *)calloc((size_t)n, sizeof(double));
    g = (double *)calloc((size_t)n, sizeof(double));
    gp = (double *)calloc((size_t)n, sizeof(double));
    d = (double *)calloc((size_t)n, sizeof(double));
    S = (double *)calloc((size_t)n * m, sizeof(double));
    Y = (double *)calloc((size_t)n * m, sizeof(double));
    rho = (double *)calloc((size_t)m, sizeof(double));
    alpha = (double *)calloc((size_t)m, sizeof(double));
    if (prm.past > 0) pf = (double *)calloc((size_t)prm.past, sizeof(double));
    if (!xp || !g || !gp || !d || !S || !Y || !rho || !alpha || (prm.past > 0 && !pf)) {
        ret = LBFGSERR_OUTOFMEMORY;
        k = 0;
        goto done;
    }

    t_evaluations++;
    fx = proc_evaluate(instance, x, g, n, 0.0);
    if (pf) pf[0] = fx;

    xnorm = sqrt(dot(x, x, n));
    gnorm = sqrt(dot(g, g, n));
    if (xnorm < 1.0) xnorm = 1.0;
    k = 0;
    if (gnorm / xnorm <= prm.epsilon) {
        ret = LBFGS_ALREADY_MINIMIZED;
        goto done;
    }

    for (int i = 0; i < n; i++) d[i] = -g[i];
    step = 1.0 / sqrt(dot(d, d, n));
    newest = -1;
    stored = 0;
    k = 1;

    for (;;) {
        int ls;
        memcpy(xp, x, sizeof(double) * (size_t)n);
        memcpy(gp, g, sizeof(double) * (size_t)n);

        if (prm.linesearch == LBFGS_LINESEARCH_MORETHUENTE)
            ls = ls_more_thuente(&ec, x, &fx, g, d, &step, xp, &prm);
        else
            ls = ls_backtracking(&ec, x, &fx, g, d, &step, xp, &prm);
        if (ls < 0) {
            memcpy(x, xp, sizeof(double) * (size_t)n);
            memcpy(g, gp, sizeof(double) * (size_t)n);
            ret = ls;
            goto done;
        }

        xnorm = sqrt(dot(x, x, n));
        gnorm = sqrt(dot(g, g, n));
        if (proc_progress) {
            ret = proc_progress(instance, x, g, fx, xnorm, gnorm, step, n, k, ls);
            if (ret) goto done;
        }
        if (xnorm < 1.0) xnorm = 1.0;
        if (gnorm / xnorm <= prm.epsilon) {
            ret = LBFGS_SUCCESS;
            break;
        }
        if (pf) {
            if (prm.past <= k) {
                double rate = (pf[k % prm.past] - fx) / fx;
                if (fabs(rate) < prm.delta) {
                    ret = LBFGS_STOP;
                    break;
                }
            }
            pf[k % prm.past] = fx;
        }
        if (prm.max_iterations != 0 && prm.max_iterations < k + 1) {
            ret = LBFGSERR_MAXIMUMITERATION;
            break;
        }

        /* new correction pair into the ring buffer */
        newest = (newest + 1) % m;
        {
            double *s = S + (size_t)newest * n, *y = Y + (size_t)newest * n;
            double ys, yy;
            for (int i = 0; i < n; i++) {
                s[i] = x[i] - xp[i];
                y[i] = g[i] - gp[i];
            }
            ys = dot(y, s, n);
            yy = dot(y, y, n);
            rho[newest] = ys;
            if (stored < m) stored++;
            ++k;

            /* two-loop recursion: d = -H g */
            for (int i = 0; i < n; i++) d[i] = -g[i];
            for (int c = 0, j = newest; c < stored; c++, j = (j + m - 1) % m) {
                alpha[j] = dot(S + (size_t)j * n, d, n) / rho[j];
                const double *yj = Y + (size_t)j * n;
                for (int i = 0; i < n; i++) d[i] -= alpha[j] * yj[i];
            }
            for (int i = 0; i < n; i++) d[i] *= ys / yy;
            for (int c = 0, j = (newest + m - stored + 1) % m; c < stored; c++, j = (j + 1) % m) {
                double beta = dot(Y + (size_t)j * n, d, n) / rho[j];
                const double *sj = S + (size_t)j * n;
                for (int i = 0; i < n; i++) d[i] += (alpha[j] - beta) * sj[i];
            }
        }
        step = 1.0;
    }

done:
    if (ptr_fx) *ptr_fx = fx;
    t_iterations += k > 0 ? k : 0;
    if (ret < 0) t_failures++;
    t_last_status = ret;
    t_last_iterations = k;
    free(xp); free(g); free(gp); free(d); free(S); free(Y); free(rho); free(alpha); free(pf);
    return ret;
}
