/*
 * oracle/ncs_port.c -- FP64 C restatement of the pyCNCS path
 * (`clib/pyCNCS/ncs.c`).  TEST INFRASTRUCTURE ONLY: the CPU oracle the CUDA
 * path is checked against, and the "port" CPU baseline.  Nothing in the
 * shipped library links or calls it.
 *
 * Every function mirrors one reference function:
 *   ncsp_reduce_noise   <- ncsReduceNoise       ncs.c:41-147
 *   ncsp_loglikelihood  <- ncsSRCalcLogLikelihood ncs.c:185-208
 *   ncsp_ll_gradient    <- ncsSRCalcLLGradient  ncs.c:158-175
 *   ncsp_noise          <- ncsSRCalcNoiseContribution ncs.c:259-299
 *   ncsp_nc_gradient    <- ncsSRCalcNCGradient  ncs.c:220-250
 *   (evaluate)          <- ncsSREvaluate        ncs.c:335-364
 *   ncsp_solve_tile     <- ncsSRNewRegion + ncsSRSetOTFMask + ncsSRSolve
 *                          + ncsSRGetU          ncs.c:459-468, :502-510, :539-561, :375-383
 * It links against the oracle's own FFTW-API shim and libLBFGS-API solver,
 * exactly like the compiled reference does, so the two agree to rounding.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_api.h"
#include "lbfgs_api.h"

typedef struct {
    int r, h;                 /* tile side, r/2+1 */
    double alpha, norm;       /* alpha, 1/r^2 */
    double *data, *gamma, *mask_sq;
    double *u;                /* iterate; also the r2c input */
    double *t1, *t2, *g;      /* scratch; g is the c2r output */
    fftw_complex *u_hat, *g_hat;
    fftw_plan fwd, bwd;
} port_tile;

static port_tile *tile_new(int r) {
    port_tile *t = (port_tile *)calloc(1, sizeof(port_tile));
    size_t n = (size_t)r * r;
    t->r = r;
    t->h = r / 2 + 1;
    t->norm = 1.0 / (double)(r * r);
    t->data = (double *)calloc(n, sizeof(double));
    t->gamma = (double *)calloc(n, sizeof(double));
    t->mask_sq = (double *)calloc(n, sizeof(double));
    t->t1 = (double *)calloc(n, sizeof(double));
    t->t2 = (double *)calloc(n, sizeof(double));
    t->u = lbfgs_malloc((int)n);
    memset(t->u, 0, n * sizeof(double));
    t->g = (double *)fftw_malloc(n * sizeof(double));
    t->u_hat = (fftw_complex *)fftw_malloc((size_t)r * t->h * sizeof(fftw_complex));
    t->g_hat = (fftw_complex *)fftw_malloc((size_t)r * t->h * sizeof(fftw_complex));
    t->fwd = fftw_plan_dft_r2c_2d(r, r, t->u, t->u_hat, FFTW_ESTIMATE);
    t->bwd = fftw_plan_dft_c2r_2d(r, r, t->g_hat, t->g, FFTW_ESTIMATE);
    return t;
}

static void tile_free(port_tile *t) {
    fftw_destroy_plan(t->fwd);
    fftw_destroy_plan(t->bwd);
    free(t->data); free(t->gamma); free(t->mask_sq); free(t->t1); free(t->t2);
    lbfgs_free(t->u);
    fftw_free(t->g); fftw_free(t->u_hat); fftw_free(t->g_hat);
    free(t);
}

/* sum_i u_i - (d_i+g_i) log(max(u_i+g_i, 1e-6))            (ncs.c:185-208) */
double ncsp_loglikelihood(const double *u, const double *data, const double *gamma, int n) {
    double s = 0.0;
    for (int i = 0; i < n; i++) {
        double a = u[i] + gamma[i];
        if (a < 1.0e-6) a = 1.0e-6;
        s += u[i] - (data[i] + gamma[i]) * log(a);
    }
    return s;
}

/* 1 - (d_i+g_i)/max(u_i+g_i, 1e-6)                          (ncs.c:158-175) */
void ncsp_ll_gradient(const double *u, const double *data, const double *gamma, int n,
                      double *grad) {
    for (int i = 0; i < n; i++) {
        double a = u[i] + gamma[i];
        if (a < 1.0e-6) a = 1.0e-6;
        grad[i] = 1.0 - (data[i] + gamma[i]) / a;
    }
}

/* (1/r^2) sum over the full r x r spectrum of |U_k|^2 M_k^2, read from the
   half spectrum by conjugate symmetry                       (ncs.c:259-299) */
static double port_noise(port_tile *t) {
    int r = t->r, h = t->h;
    double s = 0.0;
    fftw_execute(t->fwd);
    for (int i = 0; i < r; i++) {
        for (int j = 0; j < r; j++) {
            int ii = i, jj = j;
            if (j >= h) { ii = (r - i) % r; jj = r - j; }
            const double *z = t->u_hat[ii * h + jj];
            s += (z[0] * z[0] + z[1] * z[1]) * t->mask_sq[i * r + j];
        }
    }
    return s * t->norm;
}

/* (1/r^2) c2r(2 M^2 U) = 2 Q u; needs port_noise() first   (ncs.c:220-250) */
static void port_nc_gradient(port_tile *t, double *grad) {
    int r = t->r, h = t->h;
    for (int i = 0; i < r; i++) {
        for (int j = 0; j < h; j++) {
            double w = 2.0 * t->mask_sq[i * r + j];
            t->g_hat[i * h + j][0] = t->u_hat[i * h + j][0] * w;
            t->g_hat[i * h + j][1] = t->u_hat[i * h + j][1] * w;
        }
    }
    fftw_execute(t->bwd);
    for (int i = 0; i < r * r; i++) grad[i] = t->g[i] * t->norm;
}

/* f = LL + alpha NC, g = g_LL + alpha g_NC                   (ncs.c:335-364) */
static lbfgsfloatval_t port_evaluate(void *inst, const lbfgsfloatval_t *x, lbfgsfloatval_t *g,
                                     const int n, const lbfgsfloatval_t step) {
    port_tile *t = (port_tile *)inst;
    (void)x;
    (void)step;
    double f = ncsp_loglikelihood(t->u, t->data, t->gamma, n);
    f += t->alpha * port_noise(t);
    ncsp_ll_gradient(t->u, t->data, t->gamma, n, t->t1);
    port_nc_gradient(t, t->t2);
    for (int i = 0; i < n; i++) g[i] = t->t1[i] + t->alpha * t->t2[i];
    return f;
}

static int port_solve(port_tile *t, double alpha, double *fx) {
    int n = t->r * t->r;
    double f = 0.0;
    t->alpha = alpha;
    memcpy(t->u, t->data, sizeof(double) * (size_t)n); /* u0 = data (ncs.c:548-551) */
    int ret = lbfgs(n, t->u, &f, port_evaluate, NULL, t, NULL);
    if (fx) *fx = f;
    return ret;
}

/*
 * Solve one r x r tile.  mask_shifted is the fftshifted OTF mask (DC at
 * [0,0]); it is squared here as ncsSRSetOTFMask does.  Returns the libLBFGS
 * status; *fx receives the final cost.
 */
int ncsp_solve_tile(double *u_out, const double *data, const double *gamma,
                    const double *mask_shifted, double alpha, int r, double *fx) {
    if (r <= 0 || (r % 2) != 0) return -1;
    port_tile *t = tile_new(r);
    int n = r * r;
    memcpy(t->data, data, sizeof(double) * (size_t)n);
    memcpy(t->gamma, gamma, sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) t->mask_sq[i] = mask_shifted[i] * mask_shifted[i];
    int ret = port_solve(t, alpha, fx);
    memcpy(u_out, t->u, sizeof(double) * (size_t)n);
    tile_free(t);
    return ret;
}

/* Cost, its two terms and its gradient at u (tests only). */
double ncsp_cost(const double *u, const double *data, const double *gamma,
                 const double *mask_shifted, double alpha, int r, double *grad, double *ll,
                 double *nc) {
    port_tile *t = tile_new(r);
    int n = r * r;
    memcpy(t->data, data, sizeof(double) * (size_t)n);
    memcpy(t->gamma, gamma, sizeof(double) * (size_t)n);
    memcpy(t->u, u, sizeof(double) * (size_t)n);
    for (int i = 0; i < n; i++) t->mask_sq[i] = mask_shifted[i] * mask_shifted[i];
    double l = ncsp_loglikelihood(t->u, t->data, t->gamma, n);
    double q = port_noise(t);
    if (grad) {
        ncsp_ll_gradient(t->u, t->data, t->gamma, n, t->t1);
        port_nc_gradient(t, t->t2);
        for (int i = 0; i < n; i++) grad[i] = t->t1[i] + alpha * t->t2[i];
    }
    if (ll) *ll = l;
    if (nc) *nc = q;
    tile_free(t);
    return l + alpha * q;
}

/*
 * Whole-image NCS (ncs.c:41-147): 1-pixel edge-replicated halo, r x r tiles at
 * stride r-2 whose last tile on each axis is shifted back to end at the edge,
 * interiors copied out in row-major tile order so later tiles overwrite the
 * overlap.  im_x is the slow axis.  Returns 0, or -1 for an odd tile size or
 * an image smaller than the tile interior on an axis (the reference writes
 * out of bounds there).  *n_fail receives the number of tiles whose solver
 * returned non-zero (the reference prints those, ncs.c:116-119).
 */
int ncsp_reduce_noise(double *out, const double *image, const double *gamma,
                      const double *otf_mask_shifted, double alpha, int im_x, int im_y, int r,
                      int *n_fail) {
    int s = r - 2, fails = 0;
    if (r <= 2 || (r % 2) != 0) return -1;
    if (im_x + 2 < r || im_y + 2 < r) return -1;
    port_tile *t = tile_new(r);
    for (int i = 0; i < r * r; i++) t->mask_sq[i] = otf_mask_shifted[i] * otf_mask_shifted[i];

    for (int i = -1; i < im_x + 1; i += s) {
        int bx = (i + r > im_x + 1) ? im_x + 1 - r : i;
        for (int j = -1; j < im_y + 1; j += s) {
            int by = (j + r > im_y + 1) ? im_y + 1 - r : j;
            for (int k = 0; k < r; k++) {
                int xx = k + bx;
                xx = xx < 0 ? 0 : (xx >= im_x ? im_x - 1 : xx);
                for (int l = 0; l < r; l++) {
                    int yy = l + by;
                    yy = yy < 0 ? 0 : (yy >= im_y ? im_y - 1 : yy);
                    t->data[k * r + l] = image[xx * im_y + yy];
                    t->gamma[k * r + l] = gamma[xx * im_y + yy];
                }
            }
            if (port_solve(t, alpha, NULL) != 0) fails++;
            for (int k = 1; k < r - 1; k++)
                for (int l = 1; l < r - 1; l++)
                    out[(k + bx) * im_y + l + by] = t->u[k * r + l];
            if (by == im_y + 1 - r) break;
        }
        if (bx == im_x + 1 - r) break;
    }
    tile_free(t);
    if (n_fail) *n_fail = fails;
    return 0;
}
