/*
 * fftw_shim.c -- TEST INFRASTRUCTURE (oracle). Implements the FFTW 3 entry
 * points that the reference's hot path calls (NADIA/src/Complex_2D.c++:472-503)
 * on top of the canonical transform in canon_fft.h, so that the unmodified
 * reference sources can be compiled and run here as a CPU oracle and as the
 * timed CPU baseline.  fftw_malloc returns zeroed memory; that neutralises the
 * uninitialised padding rows that Complex_2D::get_padded leaves
 * (NADIA/src/Complex_2D.c++:421-433).  The real-to-complex plans are not used
 * by the phase-retrieval loop and abort if executed.
 */
#include <stdio.h>
#include <stdlib.h>
#include "shim/fftw3.h"
#include "canon_fft.h"

CANON_FFT_DEFINE(d, double)
CANON_FFT_DEFINE(f, float)

struct nadia_shim_plan_d { canon_ctxd *ctx; fftw_complex *in, *out; int nx, ny, fwd, real; };
struct nadia_shim_plan_f { canon_ctxf *ctx; fftwf_complex *in, *out; int nx, ny, fwd, real; };

static void *zalloc(size_t n)
{
    void *p = NULL;
    if (posix_memalign(&p, 64, n ? n : 64) != 0) return NULL;
    memset(p, 0, n);
    return p;
}

fftw_plan fftw_plan_dft_2d(int n0, int n1, fftw_complex *in, fftw_complex *out, int sign,
                           unsigned flags)
{
    (void)flags;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->ctx = canon_ctx_created(n0, n1);
    if (!p->ctx) { fprintf(stderr, "fftw shim: unsupported size %dx%d\n", n0, n1); abort(); }
    p->in = in; p->out = out; p->nx = n0; p->ny = n1; p->fwd = (sign == FFTW_FORWARD);
    return p;
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags)
{
    (void)in; (void)out; (void)flags;
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->nx = n0; p->ny = n1; p->real = 1;
    return p;
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags)
{
    return fftw_plan_dft_r2c_2d(n0, n1, (double *)in, (fftw_complex *)out, flags);
}
void fftw_execute(const fftw_plan p)
{
    if (p->real) { fprintf(stderr, "fftw shim: r2c/c2r not provided\n"); abort(); }
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)p->nx * p->ny);
    canon_fft2d_execd(p->ctx, (canon_cd *)p->out, p->fwd);
}
void fftw_destroy_plan(fftw_plan p) { if (p) { canon_ctx_destroyd(p->ctx); free(p); } }
void *fftw_malloc(size_t n) { return zalloc(n); }
void fftw_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { (void)n; }

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags)
{
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->ctx = canon_ctx_createf(n0, n1);
    if (!p->ctx) { fprintf(stderr, "fftw shim: unsupported size %dx%d\n", n0, n1); abort(); }
    p->in = in; p->out = out; p->nx = n0; p->ny = n1; p->fwd = (sign == FFTW_FORWARD);
    return p;
}
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags)
{
    (void)in; (void)out; (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->nx = n0; p->ny = n1; p->real = 1;
    return p;
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags)
{
    return fftwf_plan_dft_r2c_2d(n0, n1, (float *)in, (fftwf_complex *)out, flags);
}
void fftwf_execute(const fftwf_plan p)
{
    if (p->real) { fprintf(stderr, "fftw shim: r2c/c2r not provided\n"); abort(); }
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftwf_complex) * (size_t)p->nx * p->ny);
    canon_fft2d_execf(p->ctx, (canon_cf *)p->out, p->fwd);
}
void fftwf_destroy_plan(fftwf_plan p) { if (p) { canon_ctx_destroyf(p->ctx); free(p); } }
void *fftwf_malloc(size_t n) { return zalloc(n); }
void fftwf_free(void *p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int n) { (void)n; }
