/*
 * canon_fft.h -- TEST INFRASTRUCTURE (oracle). Not part of the product.
 *
 * The canonical 2-D complex DFT used by the CPU oracle and by the FFTW-API
 * shim that lets the unmodified reference sources link without FFTW.
 *
 * The reference computes its FFTs with FFTW 3 (unpinned version; plans made
 * in NADIA/src/Complex_2D.c++:463-484 with FFTW_MEASURE and executed in place
 * by perform_forward_fft / perform_backward_fft, Complex_2D.c++:487-503).
 * FFTW computes the unnormalised DFT
 *     X[k] = sum_n x[n] exp(sign * 2*pi*i * n*k / N),  sign = -1 forward, +1 backward
 * over an nx-by-ny row-major array (element (x,y) at x*ny+y).  FFTW is not
 * available here, so the oracle restates that definition with a fixed
 * schedule, chosen so that the CUDA FP64 path can follow exactly the same
 * sequence of IEEE-754 operations (bitwise-identical results):
 *
 *   - 1-D transforms are Stockham auto-sort passes (Govindaraju et al. 2008
 *     formulation).  Radix plan: 8s first, then the remaining 4 or 2, then the
 *     odd primes in ascending order (canon_plan()).
 *   - Twiddles come from one table per length n:
 *         W[t] = ( cos(2*pi*t/n), -sin(2*pi*t/n) ),  t in [0,n)
 *     computed with libm in double; the backward transform uses conj(W).
 *   - Pass with radix R over span Ns: for j in [0, n/R): k = j mod Ns;
 *     v[r] = in[j + r*n/R]; if k>0, v[r] *= W[k*r*(n/(Ns*R))] (r>=1);
 *     butterfly; out[(j/Ns)*Ns*R + k + r*Ns] = v[r].
 *   - Butterflies: radix 2, 4, 8 written out below; any other (prime) radix
 *     p is the direct sum y[s] = v[0] + sum_{r=1}^{p-1} v[r]*W[((r*s)%p)*(n/p)]
 *     accumulated in increasing r.
 *   - 2-D: all rows (length ny, contiguous) first, then all columns (length nx).
 *   - No fused multiply-add anywhere (compile with -ffp-contract=off).
 *
 * Both a double and a float instantiation are generated from one macro so
 * that the float shim used to time the reference's default single-precision
 * build runs the same algorithm.
 */
#ifndef NADIA_CANON_FFT_H
#define NADIA_CANON_FFT_H

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define CANON_MAX_PASSES 40
#define CANON_MAX_RADIX 1021 /* the largest prime factor supported */

/* Radix plan for length n.  Returns the number of passes, or -1 when n has a
 * prime factor larger than CANON_MAX_RADIX (not supported). */
static int canon_plan(int n, int *radix)
{
    int p = 0;
    if (n < 1) return -1;
    while (n % 8 == 0) { radix[p++] = 8; n /= 8; }
    if (n % 4 == 0) { radix[p++] = 4; n /= 4; }
    if (n % 2 == 0) { radix[p++] = 2; n /= 2; }
    for (int f = 3; n > 1; f += 2) {
        while (n % f == 0) {
            if (f > CANON_MAX_RADIX) return -1;
            radix[p++] = f;
            n /= f;
        }
    }
    return p;
}

#define CANON_FFT_DEFINE(SUF, REAL)                                                 \
typedef struct { REAL re, im; } canon_c##SUF;                                        \
                                                                                     \
static inline canon_c##SUF canon_cmul##SUF(canon_c##SUF a, canon_c##SUF w)           \
{                                                                                    \
    canon_c##SUF r;                                                                  \
    r.re = a.re * w.re - a.im * w.im;                                                \
    r.im = a.re * w.im + a.im * w.re;                                                \
    return r;                                                                        \
}                                                                                    \
                                                                                     \
/* twiddle table W[t] = (cos, -sin)(2 pi t / n), computed in double */             \
static canon_c##SUF *canon_table##SUF(int n)                                         \
{                                                                                    \
    canon_c##SUF *w = (canon_c##SUF *)malloc(sizeof(canon_c##SUF) * (size_t)n);     \
    for (int t = 0; t < n; ++t) {                                                    \
        double ang = (2.0 * M_PI * (double)t) / (double)n;                           \
        w[t].re = (REAL)cos(ang);                                                    \
        w[t].im = (REAL)(-sin(ang));                                                 \
    }                                                                                \
    return w;                                                                        \
}                                                                                    \
                                                                                     \
/* radix-4 butterfly; fwd=1 forward (-i), fwd=0 backward (+i) */                    \
static inline void canon_bf4##SUF(canon_c##SUF *v, int fwd)                         \
{                                                                                    \
    canon_c##SUF a, b, c, d;                                                         \
    a.re = v[0].re + v[2].re; a.im = v[0].im + v[2].im;                              \
    b.re = v[0].re - v[2].re; b.im = v[0].im - v[2].im;                              \
    c.re = v[1].re + v[3].re; c.im = v[1].im + v[3].im;                              \
    d.re = v[1].re - v[3].re; d.im = v[1].im - v[3].im;                              \
    v[0].re = a.re + c.re; v[0].im = a.im + c.im;                                    \
    v[2].re = a.re - c.re; v[2].im = a.im - c.im;                                    \
    if (fwd) {                                                                       \
        v[1].re = b.re + d.im; v[1].im = b.im - d.re;                                \
        v[3].re = b.re - d.im; v[3].im = b.im + d.re;                                \
    } else {                                                                         \
        v[1].re = b.re - d.im; v[1].im = b.im + d.re;                                \
        v[3].re = b.re + d.im; v[3].im = b.im - d.re;                                \
    }                                                                                \
}                                                                                    \
                                                                                     \
/* radix-8 butterfly: radix-2 split, internal twiddles, two radix-4s */             \
static inline void canon_bf8##SUF(canon_c##SUF *v, int fwd)                         \
{                                                                                    \
    const REAL c8 = (REAL)0.70710678118654752440;                                   \
    canon_c##SUF a[4], b[4], t;                                                      \
    for (int r = 0; r < 4; ++r) {                                                    \
        a[r].re = v[r].re + v[r + 4].re; a[r].im = v[r].im + v[r + 4].im;            \
        b[r].re = v[r].re - v[r + 4].re; b[r].im = v[r].im - v[r + 4].im;            \
    }                                                                                \
    if (fwd) {                                                                       \
        t = b[1]; b[1].re = (t.re + t.im) * c8; b[1].im = (t.im - t.re) * c8;        \
        t = b[2]; b[2].re = t.im;               b[2].im = -t.re;                     \
        t = b[3]; b[3].re = (t.im - t.re) * c8; b[3].im = -((t.re + t.im) * c8);     \
    } else {                                                                         \
        t = b[1]; b[1].re = (t.re - t.im) * c8; b[1].im = (t.im + t.re) * c8;        \
        t = b[2]; b[2].re = -t.im;              b[2].im = t.re;                      \
        t = b[3]; b[3].re = -((t.re + t.im) * c8); b[3].im = (t.re - t.im) * c8;     \
    }                                                                                \
    canon_bf4##SUF(a, fwd);                                                          \
    canon_bf4##SUF(b, fwd);                                                          \
    for (int r = 0; r < 4; ++r) { v[2 * r] = a[r]; v[2 * r + 1] = b[r]; }            \
}                                                                                    \
                                                                                     \
/* one Stockham pass of radix R over span Ns on `count` contiguous signals */       \
static void canon_pass##SUF(const canon_c##SUF *src, canon_c##SUF *dst, int n,       \
                            int R, int Ns, const canon_c##SUF *W, int fwd)           \
{                                                                                    \
    canon_c##SUF v[CANON_MAX_RADIX], y[CANON_MAX_RADIX];                             \
    const int m = n / R;                                                             \
    const int tstep = n / (Ns * R);                                                  \
    for (int j = 0; j < m; ++j) {                                                    \
        const int k = j % Ns;                                                        \
        for (int r = 0; r < R; ++r) v[r] = src[j + r * m];                           \
        if (k > 0) {                                                                 \
            for (int r = 1; r < R; ++r) {                                            \
                canon_c##SUF w = W[k * r * tstep];                                   \
                if (!fwd) w.im = -w.im;                                              \
                v[r] = canon_cmul##SUF(v[r], w);                                     \
            }                                                                        \
        }                                                                            \
        if (R == 2) {                                                                \
            canon_c##SUF a = v[0], b = v[1];                                         \
            v[0].re = a.re + b.re; v[0].im = a.im + b.im;                            \
            v[1].re = a.re - b.re; v[1].im = a.im - b.im;                            \
        } else if (R == 4) {                                                         \
            canon_bf4##SUF(v, fwd);                                                  \
        } else if (R == 8) {                                                         \
            canon_bf8##SUF(v, fwd);                                                  \
        } else {                                                                     \
            const int q = n / R;                                                     \
            y[0] = v[0];                                                             \
            for (int r = 1; r < R; ++r) {                                            \
                y[0].re = y[0].re + v[r].re; y[0].im = y[0].im + v[r].im;            \
            }                                                                        \
            for (int s = 1; s < R; ++s) {                                            \
                canon_c##SUF acc = v[0];                                             \
                for (int r = 1; r < R; ++r) {                                        \
                    canon_c##SUF w = W[((r * s) % R) * q];                           \
                    if (!fwd) w.im = -w.im;                                          \
                    canon_c##SUF p = canon_cmul##SUF(v[r], w);                       \
                    acc.re = acc.re + p.re; acc.im = acc.im + p.im;                  \
                }                                                                    \
                y[s] = acc;                                                          \
            }                                                                        \
            for (int r = 0; r < R; ++r) v[r] = y[r];                                 \
        }                                                                            \
        const int base = (j / Ns) * Ns * R + k;                                      \
        for (int r = 0; r < R; ++r) dst[base + r * Ns] = v[r];                       \
    }                                                                                \
}                                                                                    \
                                                                                     \
/* in-place 1-D transform of one contiguous signal; scratch has n elements */       \
static void canon_fft1d##SUF(canon_c##SUF *x, canon_c##SUF *scratch, int n,          \
                             const int *radix, int np, const canon_c##SUF *W,        \
                             int fwd)                                                \
{                                                                                    \
    canon_c##SUF *src = x, *dst = scratch;                                           \
    int Ns = 1;                                                                      \
    for (int p = 0; p < np; ++p) {                                                   \
        canon_pass##SUF(src, dst, n, radix[p], Ns, W, fwd);                          \
        Ns *= radix[p];                                                              \
        canon_c##SUF *t = src; src = dst; dst = t;                                   \
    }                                                                                \
    if (src != x) memcpy(x, src, sizeof(canon_c##SUF) * (size_t)n);                  \
}                                                                                    \
                                                                                     \
/* 2-D context: plans, twiddle tables and scratch for an nx-by-ny array.  */      \
typedef struct {                                                                     \
    int nx, ny, npx, npy;                                                            \
    int rx[CANON_MAX_PASSES], ry[CANON_MAX_PASSES];                                  \
    canon_c##SUF *Wx, *Wy, *scratch, *blk;                                           \
} canon_ctx##SUF;                                                                    \
                                                                                     \
/* Returns NULL when a length has an unsupported prime factor. */                   \
static canon_ctx##SUF *canon_ctx_create##SUF(int nx, int ny)                         \
{                                                                                    \
    canon_ctx##SUF *c = (canon_ctx##SUF *)calloc(1, sizeof(canon_ctx##SUF));         \
    c->nx = nx; c->ny = ny;                                                          \
    c->npx = canon_plan(nx, c->rx);                                                  \
    c->npy = canon_plan(ny, c->ry);                                                  \
    if (c->npx < 0 || c->npy < 0) { free(c); return NULL; }                          \
    c->Wx = canon_table##SUF(nx);                                                    \
    c->Wy = canon_table##SUF(ny);                                                    \
    int nmax = nx > ny ? nx : ny;                                                    \
    c->scratch = (canon_c##SUF *)malloc(sizeof(canon_c##SUF) * (size_t)nmax * 17);   \
    c->blk = c->scratch + nmax;                                                      \
    return c;                                                                        \
}                                                                                    \
                                                                                     \
static void canon_ctx_destroy##SUF(canon_ctx##SUF *c)                                \
{                                                                                    \
    if (!c) return;                                                                  \
    free(c->scratch); free(c->Wx); free(c->Wy); free(c);                             \
}                                                                                    \
                                                                                     \
/* In-place unnormalised 2-D transform: rows first, then columns (gathered  */      \
/* 16 at a time into a contiguous block; the arithmetic is unchanged).      */      \
static void canon_fft2d_exec##SUF(canon_ctx##SUF *c, canon_c##SUF *a, int fwd)       \
{                                                                                    \
    const int nx = c->nx, ny = c->ny, CB = 16;                                       \
    for (int i = 0; i < nx; ++i)                                                     \
        canon_fft1d##SUF(a + (size_t)i * ny, c->scratch, ny, c->ry, c->npy, c->Wy,   \
                         fwd);                                                       \
    for (int j0 = 0; j0 < ny; j0 += CB) {                                            \
        int nb = (ny - j0) < CB ? (ny - j0) : CB;                                    \
        for (int i = 0; i < nx; ++i)                                                 \
            for (int q = 0; q < nb; ++q)                                             \
                c->blk[(size_t)q * nx + i] = a[(size_t)i * ny + j0 + q];             \
        for (int q = 0; q < nb; ++q)                                                 \
            canon_fft1d##SUF(c->blk + (size_t)q * nx, c->scratch, nx, c->rx, c->npx, \
                             c->Wx, fwd);                                            \
        for (int i = 0; i < nx; ++i)                                                 \
            for (int q = 0; q < nb; ++q)                                             \
                a[(size_t)i * ny + j0 + q] = c->blk[(size_t)q * nx + i];             \
    }                                                                                \
}

#endif /* NADIA_CANON_FFT_H */
