/*
 * fftw_shim.c -- TEST INFRASTRUCTURE (oracle). Implements the FFTW 3 entry
 * points that the reference's hot path calls (NADIA/src/Complex_2D.c++:472-503)
 * on top of the canonical transform in canon_fft.h, so that the unmodified
 * reference sources can be compiled and run here as a CPU oracle and as the
 * timed CPU baseline.  fftw_malloc returns zeroed memory; that neutralises the
 * uninitialised padding rows that Complex_2D::get_padded leaves
 * (NADIA/src/Complex_2D.c++:421-433).  The real-to-complex plans (used only by
 * the image alignment of PhaseDiverseCDI, NADIA/src/utils.c:1151-1300) go
 * through the same complex transform: r2c keeps columns 0..ny/2 of the
 * transform of (x, 0) in FFTW's n0 x (n1/2+1) layout; c2r extends the half
 * spectrum by Hermitian symmetry, runs the backward transform and keeps the
 * real part (both unnormalised, as FFTW).
 *
 * Threads (the reference's MULTI_THREADED build, Complex_2D.c++:465-467, which
 * calls FFTW_INIT_THREADS and FFTW_PLAN_WITH_NTHREADS(NUM_THREADS) before it
 * plans): complex plans made after fftw[f]_plan_with_nthreads(n), n > 1, split
 * the rows, then the column blocks, of each 2-D transform over n POSIX
 * threads.  Every 1-D transform runs the same canonical arithmetic, so results
 * do not depend on the thread count.  nadia_shim_env_threads() returns
 * NADIA_REF_FFT_THREADS from the environment (default 1); the threaded timing
 * build passes it as NUM_THREADS, so the count is chosen at run time.
 */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include "shim/fftw3.h"
#include "canon_fft.h"

CANON_FFT_DEFINE(d, double)
CANON_FFT_DEFINE(f, float)

static int shim_threads = 1;

int nadia_shim_env_threads(void)
{
    const char *e = getenv("NADIA_REF_FFT_THREADS");
    const int n = e ? atoi(e) : 1;
    return n > 0 ? n : 1;
}

/* real: 0 complex-to-complex, 1 r2c, 2 c2r; nthreads: threads of a complex plan */
struct nadia_shim_plan_d { canon_ctxd *ctx; fftw_complex *in, *out; int nx, ny, fwd, real, nthreads; };
struct nadia_shim_plan_f { canon_ctxf *ctx; fftwf_complex *in, *out; int nx, ny, fwd, real, nthreads; };

/* one thread's share of canon_fft2d_exec: rows [lo, hi) in phase 0, column
 * blocks of 16 starting in [lo, hi) in phase 1, with its own scratch */
#define SHIM_MT_DEFINE(SUF)                                                              \
typedef struct { canon_ctx##SUF *c; canon_c##SUF *a; int fwd, phase, lo, hi; } shim_job##SUF; \
static void *shim_work##SUF(void *arg)                                                  \
{                                                                                       \
    shim_job##SUF *J = (shim_job##SUF *)arg;                                            \
    canon_ctx##SUF *c = J->c;                                                           \
    const int nx = c->nx, ny = c->ny, CB = 16, nmax = nx > ny ? nx : ny;                \
    canon_c##SUF *scratch = (canon_c##SUF *)malloc(sizeof(canon_c##SUF) * (size_t)nmax * 17); \
    canon_c##SUF *blk = scratch + nmax;                                                 \
    if (J->phase == 0) {                                                                \
        for (int i = J->lo; i < J->hi; ++i)                                             \
            canon_fft1d##SUF(J->a + (size_t)i * ny, scratch, ny, c->ry, c->npy, c->Wy, J->fwd); \
    } else {                                                                            \
        for (int j0 = J->lo; j0 < J->hi; j0 += CB) {                                    \
            int nb = (ny - j0) < CB ? (ny - j0) : CB;                                   \
            for (int i = 0; i < nx; ++i)                                                \
                for (int q = 0; q < nb; ++q)                                            \
                    blk[(size_t)q * nx + i] = J->a[(size_t)i * ny + j0 + q];            \
            for (int q = 0; q < nb; ++q)                                                \
                canon_fft1d##SUF(blk + (size_t)q * nx, scratch, nx, c->rx, c->npx, c->Wx, J->fwd); \
            for (int i = 0; i < nx; ++i)                                                \
                for (int q = 0; q < nb; ++q)                                            \
                    J->a[(size_t)i * ny + j0 + q] = blk[(size_t)q * nx + i];            \
        }                                                                               \
    }                                                                                   \
    free(scratch);                                                                      \
    return NULL;                                                                        \
}                                                                                       \
static void shim_exec_mt##SUF(canon_ctx##SUF *c, canon_c##SUF *a, int fwd, int nt)      \
{                                                                                       \
    enum { MAXT = 256 };                                                                \
    pthread_t th[MAXT];                                                                 \
    shim_job##SUF job[MAXT];                                                            \
    if (nt > MAXT) nt = MAXT;                                                           \
    for (int phase = 0; phase < 2; ++phase) {                                           \
        /* rows, or column blocks of 16 (units of 16 columns) */                        \
        const int units = phase == 0 ? c->nx : (c->ny + 15) / 16;                       \
        const int n = nt < units ? nt : units;                                          \
        for (int t = 0; t < n; ++t) {                                                   \
            int lo = (int)((long long)units * t / n), hi = (int)((long long)units * (t + 1) / n); \
            if (phase == 1) { lo *= 16; hi = hi * 16 < c->ny ? hi * 16 : c->ny; }       \
            job[t] = (shim_job##SUF){c, a, fwd, phase, lo, hi};                        \
            if (pthread_create(&th[t], NULL, shim_work##SUF, &job[t]) != 0) {           \
                fprintf(stderr, "fftw shim: pthread_create failed\n");                  \
                abort();                                                                \
            }                                                                           \
        }                                                                               \
        for (int t = 0; t < n; ++t) pthread_join(th[t], NULL);                          \
    }                                                                                   \
}
SHIM_MT_DEFINE(d)
SHIM_MT_DEFINE(f)

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
    p->nthreads = shim_threads;
    return p;
}
static fftw_plan shim_real_pland(int n0, int n1, void *in, void *out, int kind)
{
    fftw_plan p = (fftw_plan)calloc(1, sizeof(*p));
    p->ctx = canon_ctx_created(n0, n1);
    if (!p->ctx) { fprintf(stderr, "fftw shim: unsupported size %dx%d\n", n0, n1); abort(); }
    p->in = (fftw_complex *)in; p->out = (fftw_complex *)out;
    p->nx = n0; p->ny = n1; p->real = kind;
    return p;
}
fftw_plan fftw_plan_dft_r2c_2d(int n0, int n1, double *in, fftw_complex *out, unsigned flags)
{
    (void)flags;
    return shim_real_pland(n0, n1, in, out, 1);
}
fftw_plan fftw_plan_dft_c2r_2d(int n0, int n1, fftw_complex *in, double *out, unsigned flags)
{
    (void)flags;
    return shim_real_pland(n0, n1, in, out, 2);
}

static void shim_real_execd(fftw_plan p)
{
    const int nx = p->nx, ny = p->ny, h = ny / 2 + 1;
    canon_cd *t = (canon_cd *)zalloc(sizeof(canon_cd) * (size_t)nx * ny);
    if (p->real == 1) {
        const double *in = (const double *)p->in;
        double *out = (double *)p->out;
        for (size_t k = 0; k < (size_t)nx * ny; ++k) { t[k].re = in[k]; t[k].im = 0; }
        canon_fft2d_execd(p->ctx, t, 1);
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < h; ++y) {
                out[2 * ((size_t)x * h + y)] = t[(size_t)x * ny + y].re;
                out[2 * ((size_t)x * h + y) + 1] = t[(size_t)x * ny + y].im;
            }
    } else {
        const double *in = (const double *)p->in;
        double *out = (double *)p->out;
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                canon_cd *d = &t[(size_t)x * ny + y];
                if (y < h) {
                    d->re = in[2 * ((size_t)x * h + y)];
                    d->im = in[2 * ((size_t)x * h + y) + 1];
                } else {
                    const size_t k = (size_t)((nx - x) % nx) * h + (ny - y);
                    d->re = in[2 * k];
                    d->im = -in[2 * k + 1];
                }
            }
        canon_fft2d_execd(p->ctx, t, 0);
        for (size_t k = 0; k < (size_t)nx * ny; ++k) out[k] = t[k].re;
    }
    free(t);
}
void fftw_execute(const fftw_plan p)
{
    if (p->real) { shim_real_execd(p); return; }
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftw_complex) * (size_t)p->nx * p->ny);
    if (p->nthreads > 1)
        shim_exec_mtd(p->ctx, (canon_cd *)p->out, p->fwd, p->nthreads);
    else
        canon_fft2d_execd(p->ctx, (canon_cd *)p->out, p->fwd);
}
void fftw_destroy_plan(fftw_plan p) { if (p) { canon_ctx_destroyd(p->ctx); free(p); } }
void *fftw_malloc(size_t n) { return zalloc(n); }
void fftw_free(void *p) { free(p); }
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int n) { shim_threads = n > 1 ? n : 1; }

fftwf_plan fftwf_plan_dft_2d(int n0, int n1, fftwf_complex *in, fftwf_complex *out, int sign,
                             unsigned flags)
{
    (void)flags;
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->ctx = canon_ctx_createf(n0, n1);
    if (!p->ctx) { fprintf(stderr, "fftw shim: unsupported size %dx%d\n", n0, n1); abort(); }
    p->in = in; p->out = out; p->nx = n0; p->ny = n1; p->fwd = (sign == FFTW_FORWARD);
    p->nthreads = shim_threads;
    return p;
}
static fftwf_plan shim_real_planf(int n0, int n1, void *in, void *out, int kind)
{
    fftwf_plan p = (fftwf_plan)calloc(1, sizeof(*p));
    p->ctx = canon_ctx_createf(n0, n1);
    if (!p->ctx) { fprintf(stderr, "fftw shim: unsupported size %dx%d\n", n0, n1); abort(); }
    p->in = (fftwf_complex *)in; p->out = (fftwf_complex *)out;
    p->nx = n0; p->ny = n1; p->real = kind;
    return p;
}
fftwf_plan fftwf_plan_dft_r2c_2d(int n0, int n1, float *in, fftwf_complex *out, unsigned flags)
{
    (void)flags;
    return shim_real_planf(n0, n1, in, out, 1);
}
fftwf_plan fftwf_plan_dft_c2r_2d(int n0, int n1, fftwf_complex *in, float *out, unsigned flags)
{
    (void)flags;
    return shim_real_planf(n0, n1, in, out, 2);
}

static void shim_real_execf(fftwf_plan p)
{
    const int nx = p->nx, ny = p->ny, h = ny / 2 + 1;
    canon_cf *t = (canon_cf *)zalloc(sizeof(canon_cf) * (size_t)nx * ny);
    if (p->real == 1) {
        const float *in = (const float *)p->in;
        float *out = (float *)p->out;
        for (size_t k = 0; k < (size_t)nx * ny; ++k) { t[k].re = in[k]; t[k].im = 0; }
        canon_fft2d_execf(p->ctx, t, 1);
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < h; ++y) {
                out[2 * ((size_t)x * h + y)] = t[(size_t)x * ny + y].re;
                out[2 * ((size_t)x * h + y) + 1] = t[(size_t)x * ny + y].im;
            }
    } else {
        const float *in = (const float *)p->in;
        float *out = (float *)p->out;
        for (int x = 0; x < nx; ++x)
            for (int y = 0; y < ny; ++y) {
                canon_cf *d = &t[(size_t)x * ny + y];
                if (y < h) {
                    d->re = in[2 * ((size_t)x * h + y)];
                    d->im = in[2 * ((size_t)x * h + y) + 1];
                } else {
                    const size_t k = (size_t)((nx - x) % nx) * h + (ny - y);
                    d->re = in[2 * k];
                    d->im = -in[2 * k + 1];
                }
            }
        canon_fft2d_execf(p->ctx, t, 0);
        for (size_t k = 0; k < (size_t)nx * ny; ++k) out[k] = t[k].re;
    }
    free(t);
}
void fftwf_execute(const fftwf_plan p)
{
    if (p->real) { shim_real_execf(p); return; }
    if (p->out != p->in) memcpy(p->out, p->in, sizeof(fftwf_complex) * (size_t)p->nx * p->ny);
    if (p->nthreads > 1)
        shim_exec_mtf(p->ctx, (canon_cf *)p->out, p->fwd, p->nthreads);
    else
        canon_fft2d_execf(p->ctx, (canon_cf *)p->out, p->fwd);
}
void fftwf_destroy_plan(fftwf_plan p) { if (p) { canon_ctx_destroyf(p->ctx); free(p); } }
void *fftwf_malloc(size_t n) { return zalloc(n); }
void fftwf_free(void *p) { free(p); }
int fftwf_init_threads(void) { return 1; }
void fftwf_plan_with_nthreads(int n) { shim_threads = n > 1 ? n : 1; }
