// expand_wl_shim.cpp -- a C entry over the drop-in PolyCDI's host-side
// spectrum bookkeeping and expand_wl (include/nadia/PolyCDI.h), so that a
// test can compare them with the reference's PolyCDI::set_spectrum /
// expand_wl / get_intensity without creating a reconstruction (no GPU).
// Arrays are doubles, element (x,y) at x*ny+y, complex interleaved.
#include "PolyCDI.h"

extern "C" int shim_expand_wl(int nx, int ny, const double *spec, int nl, const double *field,
                              int fx, int fy, double *out, int *padding)
{
    Double_2D s(nl, 2);
    for (int i = 0; i < nl; ++i) {
        s.set(i, WL, spec[2 * i]);
        s.set(i, WEIGHT, spec[2 * i + 1]);
    }
    nadia_cxx::PolySpectrum ps;
    ps.set(s, nx, ny);
    padding[0] = ps.paddingx;
    padding[1] = ps.paddingy;
    Complex_2D c(fx, fy);
    for (int i = 0; i < fx; ++i)
        for (int j = 0; j < fy; ++j) {
            c.set_real(i, j, field[2 * ((size_t)i * fy + j)]);
            c.set_imag(i, j, field[2 * ((size_t)i * fy + j) + 1]);
        }
    Double_2D r(nx, ny);
    try {
        nadia_cxx::poly_expand_wl(ps, nx, ny, c, r);
    } catch (const nadia_cxx::Failure &) {
        return 1;
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) out[(size_t)i * ny + j] = r.get(i, j);
    return 0;
}
