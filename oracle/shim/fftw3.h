/*
 * fftw3.h -- TEST INFRASTRUCTURE (oracle). A minimal stand-in for the FFTW 3
 * public header, declaring only the entry points the reference's hot-path
 * sources name (NADIA/include/types.h:5-39, NADIA/src/Complex_2D.c++:23-96,
 * 463-523).  The implementations live in fftw_shim.c and run the canonical
 * schedule of canon_fft.h.  FFTW itself is not installed in this image.
 */
#ifndef NADIA_FFTW3_SHIM_H
#define NADIA_FFTW3_SHIM_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#define FFTW_EXHAUSTIVE (1U << 3)

typedef double fftw_complex[2];
typedef float fftwf_complex[2];
typedef struct nadia_shim_plan_d *fftw_plan;
typedef struct nadia_shim_plan_f *fftwf_plan;

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out,
                               unsigned flags);
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out,
                               unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
int fftw_init_threads(void);
void fftw_plan_with_nthreads(int n);

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out,
                             int sign, unsigned flags);
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out,
                                 unsigned flags);
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out,
                                 unsigned flags);
void fftwf_execute(const fftwf_plan p);
void fftwf_destroy_plan(fftwf_plan p);
void *fftwf_malloc(size_t n);
void fftwf_free(void *p);
int fftwf_init_threads(void);
void fftwf_plan_with_nthreads(int n);

/* the FFT thread count for a build that passes it as NUM_THREADS:
   NADIA_REF_FFT_THREADS from the environment, default 1 (not part of FFTW) */
int nadia_shim_env_threads(void);

#ifdef __cplusplus
}
#endif
#endif
