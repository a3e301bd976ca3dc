/*
 * oracle/lbfgs_api.h -- the libLBFGS 1.10 C API (64-bit floats) as declared
 * by the reference's vendored header `clib/pyCNCS/lbfgs.h`, which `ncs.c`
 * calls at ncs.c:416, :443, :554-557 and :315.  TEST INFRASTRUCTURE ONLY.
 *
 * libLBFGS (MIT licence, version 1.10 per lbfgs.h:605) is a third-party
 * dependency whose source is not vendored in the reference.  `lbfgs_own.c`
 * restates its published algorithm: Nocedal's two-loop L-BFGS recursion with
 * the Moré–Thuente line search (Moré & Thuente, ACM TOMS 20(3), 1994) as the
 * default, the documented defaults of lbfgs.h:198-358 and the documented
 * stopping rule ||g|| <= epsilon * max(1, ||x||) (lbfgs.h:209-217).
 *
 * The parameter struct layout and the return-code values must be identical to
 * lbfgs.h so that the unmodified reference `ncs.c` links against this
 * implementation; that is the only reason they look alike.
 */
#ifndef NCS_ORACLE_LBFGS_API_H
#define NCS_ORACLE_LBFGS_API_H

#ifdef __cplusplus
extern "C" {
#endif

typedef double lbfgsfloatval_t;

/* Return codes (values fixed by lbfgs.h:67-147). */
enum {
    LBFGS_SUCCESS = 0,
    LBFGS_CONVERGENCE = 0,
    LBFGS_STOP = 1,
    LBFGS_ALREADY_MINIMIZED = 2,
    LBFGSERR_UNKNOWNERROR = -1024,
    LBFGSERR_LOGICERROR = -1023,
    LBFGSERR_OUTOFMEMORY = -1022,
    LBFGSERR_CANCELED = -1021,
    LBFGSERR_INVALID_N = -1020,
    LBFGSERR_INVALID_N_SSE = -1019,
    LBFGSERR_INVALID_X_SSE = -1018,
    LBFGSERR_INVALID_EPSILON = -1017,
    LBFGSERR_INVALID_TESTPERIOD = -1016,
    LBFGSERR_INVALID_DELTA = -1015,
    LBFGSERR_INVALID_LINESEARCH = -1014,
    LBFGSERR_INVALID_MINSTEP = -1013,
    LBFGSERR_INVALID_MAXSTEP = -1012,
    LBFGSERR_INVALID_FTOL = -1011,
    LBFGSERR_INVALID_WOLFE = -1010,
    LBFGSERR_INVALID_GTOL = -1009,
    LBFGSERR_INVALID_XTOL = -1008,
    LBFGSERR_INVALID_MAXLINESEARCH = -1007,
    LBFGSERR_INVALID_ORTHANTWISE = -1006,
    LBFGSERR_INVALID_ORTHANTWISE_START = -1005,
    LBFGSERR_INVALID_ORTHANTWISE_END = -1004,
    LBFGSERR_OUTOFINTERVAL = -1003,
    LBFGSERR_INCORRECT_TMINMAX = -1002,
    LBFGSERR_ROUNDING_ERROR = -1001,
    LBFGSERR_MINIMUMSTEP = -1000,
    LBFGSERR_MAXIMUMSTEP = -999,
    LBFGSERR_MAXIMUMLINESEARCH = -998,
    LBFGSERR_MAXIMUMITERATION = -997,
    LBFGSERR_WIDTHTOOSMALL = -996,
    LBFGSERR_INVALIDPARAMETERS = -995,
    LBFGSERR_INCREASEGRADIENT = -994
};

/* Line searches (lbfgs.h:152-190). */
enum {
    LBFGS_LINESEARCH_DEFAULT = 0,
    LBFGS_LINESEARCH_MORETHUENTE = 0,
    LBFGS_LINESEARCH_BACKTRACKING_ARMIJO = 1,
    LBFGS_LINESEARCH_BACKTRACKING = 2,
    LBFGS_LINESEARCH_BACKTRACKING_WOLFE = 2,
    LBFGS_LINESEARCH_BACKTRACKING_STRONG_WOLFE = 3
};

/* Field order and types as lbfgs.h:198-358. */
typedef struct {
    int m;
    lbfgsfloatval_t epsilon;
    int past;
    lbfgsfloatval_t delta;
    int max_iterations;
    int linesearch;
    int max_linesearch;
    lbfgsfloatval_t min_step;
    lbfgsfloatval_t max_step;
    lbfgsfloatval_t ftol;
    lbfgsfloatval_t wolfe;
    lbfgsfloatval_t gtol;
    lbfgsfloatval_t xtol;
    lbfgsfloatval_t orthantwise_c;
    int orthantwise_start;
    int orthantwise_end;
} lbfgs_parameter_t;

typedef lbfgsfloatval_t (*lbfgs_evaluate_t)(void *instance, const lbfgsfloatval_t *x,
                                            lbfgsfloatval_t *g, const int n,
                                            const lbfgsfloatval_t step);
typedef int (*lbfgs_progress_t)(void *instance, const lbfgsfloatval_t *x,
                                const lbfgsfloatval_t *g, const lbfgsfloatval_t fx,
                                const lbfgsfloatval_t xnorm, const lbfgsfloatval_t gnorm,
                                const lbfgsfloatval_t step, int n, int k, int ls);

int lbfgs(int n, lbfgsfloatval_t *x, lbfgsfloatval_t *ptr_fx, lbfgs_evaluate_t proc_evaluate,
          lbfgs_progress_t proc_progress, void *instance, lbfgs_parameter_t *param);
void lbfgs_parameter_init(lbfgs_parameter_t *param);
lbfgsfloatval_t *lbfgs_malloc(int n);
void lbfgs_free(lbfgsfloatval_t *x);

/*
 * Oracle-only controls (no counterpart in libLBFGS).  The reference calls
 * lbfgs_parameter_init() with no way to change the defaults (ncs.c:442-443),
 * so capped runs (the 15/20-iteration configurations) set process-wide
 * overrides here before calling the unmodified reference.  A value <= 0
 * (epsilon < 0, m <= 0, linesearch < 0) keeps the libLBFGS default;
 * max_iterations = 0 means "no cap" exactly as in libLBFGS.
 */
void ncs_oracle_set_overrides(int max_iterations, double epsilon, int m, int linesearch);
/* Per-thread counters accumulated over lbfgs() calls since the last reset. */
void ncs_oracle_reset_stats(void);
void ncs_oracle_get_stats(long *calls, long *iterations, long *evaluations, long *failures,
                          int *last_status, int *last_iterations);

#ifdef __cplusplus
}
#endif

#endif
