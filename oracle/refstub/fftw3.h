/* Declarations of the subset of the FFTW3 single-precision API that the
 * reference's GENERIC vector layer calls (mpifxcorr/src/architecture.h.in:
 * plans at :799-856, execute at :1017-1034). FFTW itself is not part of this
 * build; oracle/refstub/fftwf_shim.c implements these calls with a
 * project-written FFT. */
#ifndef ORACLE_REFSTUB_FFTW3_H
#define ORACLE_REFSTUB_FFTW3_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef float fftwf_complex[2];
typedef double fftw_complex[2];
typedef struct fftwf_plan_s *fftwf_plan;
typedef struct fftw_plan_s *fftw_plan;
#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
fftwf_plan fftwf_plan_dft_1d(int n, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_1d(int n, float *in, fftwf_complex *out, unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_1d(int n, fftwf_complex *in, float *out, unsigned flags);
fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign, unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
#ifdef __cplusplus
}
#endif
#endif
