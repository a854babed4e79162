/* Type-only FFTW declarations: the reference's public header names these types,
 * but the oracle build compiles none of the FFTW-backed sources, so nothing here
 * is ever called. */
#ifndef ORACLE_STUB_FFTW3_H
#define ORACLE_STUB_FFTW3_H
#include <stdio.h>
typedef struct oracle_stub_fftw_plan_s * fftw_plan;
typedef struct oracle_stub_fftwf_plan_s * fftwf_plan;
typedef int fftw_r2r_kind;
typedef double fftw_complex[2];
typedef float fftwf_complex[2];
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int);
#endif
