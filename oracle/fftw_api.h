/*
 * oracle/fftw_api.h -- the subset of the FFTW3 double-precision C API that the
 * reference solver `clib/pyCNCS/ncs.c` calls (ncs.c:244, :268, :317-322,
 * :433-439).  TEST INFRASTRUCTURE ONLY: this is part of the CPU oracle, never
 * part of the shipped CUDA path.
 *
 * FFTW itself is not installed in this image and its source is not vendored in
 * the reference (only `clib/pyCNCS/fftw3.h` and a Windows DLL, which is not
 * used).  `fftw_shim.c` implements these entry points from FFTW's documented
 * semantics (FFTW 3 manual, "Multi-Dimensional DFTs of Real Data"): an
 * unnormalised forward r2c transform to the n0 x (n1/2+1) half spectrum and an
 * unnormalised c2r inverse of a Hermitian half spectrum.
 *
 * The ABI matches `clib/pyCNCS/fftw3.h` (fftw_plan is an opaque pointer,
 * fftw_complex is double[2]) so the unmodified reference `ncs.c` links
 * against it.
 */
#ifndef NCS_ORACLE_FFTW_API_H
#define NCS_ORACLE_FFTW_API_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct fftw_plan_s *fftw_plan;

#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);

#ifdef __cplusplus
}
#endif

#endif
