/*
 * oracle/fftw_shim.c -- a small FP64 implementation of the FFTW3 entry points
 * used by the reference `clib/pyCNCS/ncs.c` (r2c / c2r 2-D plans, execute,
 * destroy, malloc, free).  TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
 *
 * Semantics follow the FFTW 3 manual for real-data multi-dimensional DFTs:
 *   r2c: out[i*(n1/2+1)+j] = sum_{x,y} in[x*n1+y] * exp(-2 pi i (i x/n0 + j y/n1))
 *   c2r: out[x*n1+y]       = sum_{i, j in 0..n1-1} X[i][j] exp(+2 pi i (...)),
 *        where X is the Hermitian extension of the half spectrum; the
 *        imaginary parts of the self-conjugate columns (j = 0, n1/2) are
 *        ignored.  Neither direction is normalised.
 * The reference only ever uses 16x16 and 10x10 plans (ncs.c:432-439,
 * clib/pyCNCS/test/test_im.py:238).  Power-of-two lengths use an iterative
 * radix-2 transform; other lengths fall back to a direct O(n^2) DFT.
 * Plans own their workspace, so distinct plans may run on distinct threads.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "fftw_api.h"

enum { SHIM_R2C = 1, SHIM_C2R = 2 };

struct fftw_plan_s {
    int kind;
    int n0, n1, h1;          /* h1 = n1/2 + 1 */
    double *rbuf;            /* real array (in for r2c, out for c2r) */
    fftw_complex *cbuf;      /* half spectrum (out for r2c, in for c2r) */
    double *tw0, *tw1;       /* cos/sin tables, 2*n entries each */
    double *work;            /* n0*h1 complex + max(n0,n1) complex scratch */
};

static int is_pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

static double *make_twiddles(int n) {
    double *t = (double *)malloc(sizeof(double) * 2 * (size_t)n);
    for (int k = 0; k < n; k++) {
        double a = 2.0 * M_PI * (double)k / (double)n;
        t[2 * k] = cos(a);
        t[2 * k + 1] = sin(a);
    }
    return t;
}

/* In-place 1-D complex DFT of length n on interleaved (re,im) data.
 * sign = -1 forward, +1 backward.  tw = make_twiddles(n).  scratch >= 2n. */
static void dft1(double *z, int n, int sign, const double *tw, double *scratch) {
    if (n == 1) return;
    if (is_pow2(n)) {
        /* bit reversal permutation */
        for (int i = 1, j = 0; i < n; i++) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double tr = z[2 * i], ti = z[2 * i + 1];
                z[2 * i] = z[2 * j]; z[2 * i + 1] = z[2 * j + 1];
                z[2 * j] = tr; z[2 * j + 1] = ti;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1, step = n / len;
            for (int s = 0; s < n; s += len) {
                for (int k = 0; k < half; k++) {
                    double wr = tw[2 * (k * step)];
                    double wi = sign * tw[2 * (k * step) + 1];
                    double *a = z + 2 * (s + k), *b = z + 2 * (s + k + half);
                    double br = b[0] * wr - b[1] * wi;
                    double bi = b[0] * wi + b[1] * wr;
                    b[0] = a[0] - br; b[1] = a[1] - bi;
                    a[0] += br; a[1] += bi;
                }
            }
        }
    } else {
        for (int k = 0; k < n; k++) {
            double sr = 0.0, si = 0.0;
            for (int x = 0; x < n; x++) {
                int m = (int)(((long)k * x) % n);
                double wr = tw[2 * m], wi = sign * tw[2 * m + 1];
                sr += z[2 * x] * wr - z[2 * x + 1] * wi;
                si += z[2 * x] * wi + z[2 * x + 1] * wr;
            }
            scratch[2 * k] = sr;
            scratch[2 * k + 1] = si;
        }
        memcpy(z, scratch, sizeof(double) * 2 * (size_t)n);
    }
}

static fftw_plan make_plan(int kind, int n0, int n1, double *r, fftw_complex *c) {
    if (n0 <= 0 || n1 <= 0) return NULL;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fftw_plan_s));
    int nmax = n0 > n1 ? n0 : n1;
    p->kind = kind;
    p->n0 = n0;
    p->n1 = n1;
    p->h1 = n1 / 2 + 1;
    p->rbuf = r;
    p->cbuf = c;
    p->tw0 = make_twiddles(n0);
    p->tw1 = make_twiddles(n1);
    p->work = (double *)malloc(sizeof(double) * 2 * ((size_t)n0 * p->h1 + 2 * (size_t)nmax));
    return p;
}

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags) {
    (void)flags;
    return make_plan(SHIM_R2C, n0, n1, in, out);
}

fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags) {
    (void)flags;
    return make_plan(SHIM_C2R, n0, n1, out, in);
}

void fftw_execute(const fftw_plan p) {
    int n0 = p->n0, n1 = p->n1, h1 = p->h1;
    int nmax = n0 > n1 ? n0 : n1;
    double *mid = p->work;                       /* n0 x h1 complex */
    double *line = p->work + 2 * (size_t)n0 * h1; /* nmax complex */
    double *scr = line + 2 * (size_t)nmax;        /* nmax complex */
    if (p->kind == SHIM_R2C) {
        for (int x = 0; x < n0; x++) {
            for (int y = 0; y < n1; y++) {
                line[2 * y] = p->rbuf[x * n1 + y];
                line[2 * y + 1] = 0.0;
            }
            dft1(line, n1, -1, p->tw1, scr);
            memcpy(mid + 2 * (size_t)x * h1, line, sizeof(double) * 2 * (size_t)h1);
        }
        for (int j = 0; j < h1; j++) {
            for (int x = 0; x < n0; x++) {
                line[2 * x] = mid[2 * ((size_t)x * h1 + j)];
                line[2 * x + 1] = mid[2 * ((size_t)x * h1 + j) + 1];
            }
            dft1(line, n0, -1, p->tw0, scr);
            for (int x = 0; x < n0; x++) {
                p->cbuf[x * h1 + j][0] = line[2 * x];
                p->cbuf[x * h1 + j][1] = line[2 * x + 1];
            }
        }
    } else {
        for (int j = 0; j < h1; j++) {
            for (int x = 0; x < n0; x++) {
                line[2 * x] = p->cbuf[x * h1 + j][0];
                line[2 * x + 1] = p->cbuf[x * h1 + j][1];
            }
            dft1(line, n0, +1, p->tw0, scr);
            for (int x = 0; x < n0; x++) {
                mid[2 * ((size_t)x * h1 + j)] = line[2 * x];
                mid[2 * ((size_t)x * h1 + j) + 1] = line[2 * x + 1];
            }
        }
        for (int x = 0; x < n0; x++) {
            for (int j = 0; j < n1; j++) {
                if (j < h1) {
                    line[2 * j] = mid[2 * ((size_t)x * h1 + j)];
                    line[2 * j + 1] = mid[2 * ((size_t)x * h1 + j) + 1];
                } else {
                    line[2 * j] = mid[2 * ((size_t)x * h1 + (n1 - j))];
                    line[2 * j + 1] = -mid[2 * ((size_t)x * h1 + (n1 - j)) + 1];
                }
            }
            /* self-conjugate columns: imaginary parts are ignored */
            line[1] = 0.0;
            if ((n1 & 1) == 0) line[2 * (n1 / 2) + 1] = 0.0;
            dft1(line, n1, +1, p->tw1, scr);
            for (int y = 0; y < n1; y++) p->rbuf[x * n1 + y] = line[2 * y];
        }
    }
}

void fftw_destroy_plan(fftw_plan p) {
    if (!p) return;
    free(p->tw0);
    free(p->tw1);
    free(p->work);
    free(p);
}

void *fftw_malloc(size_t n) {
    void *ptr = NULL;
    if (posix_memalign(&ptr, 64, n ? n : 1) != 0) return NULL;
    return ptr;
}

void fftw_free(void *p) { free(p); }
