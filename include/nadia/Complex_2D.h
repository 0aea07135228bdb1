// Complex_2D.h -- drop-in for the reference's ComplexR_2D<T> / Complex_2D
// (NADIA/include/Complex_2D.h): an nx*ny complex field stored as interleaved
// (re, im) pairs, element (x,y) at x*ny+y.
//
// A field handed to a reconstruction (PlanarCDI, FresnelCDI, PolyCDI) is the
// host mirror of that reconstruction's estimate on the GPU.  After iterate()
// the device holds the newer values; any accessor fetches them first, and a
// field changed on the host is uploaded before the next iteration, so code
// that reads or edits the estimate between iterations (as the reference's
// examples and CDI_reconstruction do) keeps working.
//
// Complex_2D is ComplexR_2D<float> unless DOUBLE_PRECISION is defined
// (Complex_2D.h:511-515 of the reference).
#ifndef NADIA_DROPIN_COMPLEX_2D_H
#define NADIA_DROPIN_COMPLEX_2D_H

#include <cmath>
#include <cstring>
#include <iostream>
#include <vector>

#include "Double_2D.h"
#include "types.h"

template <class T>
class ComplexR_2D {
public:
    ComplexR_2D(int x_size, int y_size) : nx(x_size), ny(y_size), a((size_t)2 * x_size * y_size, T(0)) {}

    ComplexR_2D(const ComplexR_2D &o) : nx(o.nx), ny(o.ny)
    {
        o.fetch();
        a = o.a;
    }

    ComplexR_2D(const Double_2D &d) : nx(d.get_size_x()), ny(d.get_size_y()), a((size_t)2 * nx * ny)
    {
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                a[idx(i, j)] = d.get(i, j);
                a[idx(i, j) + 1] = 0;
            }
    }

    ~ComplexR_2D() {}

    ComplexR_2D &operator=(const ComplexR_2D &o)
    {
        if (this == &o) return *this;
        o.fetch();
        nx = o.nx;
        ny = o.ny;
        a = o.a;
        edited();
        return *this;
    }

    ComplexR_2D &operator=(const Double_2D &d)
    {
        nx = d.get_size_x();
        ny = d.get_size_y();
        a.assign((size_t)2 * nx * ny, T(0));
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) a[idx(i, j)] = d.get(i, j);
        edited();
        return *this;
    }

    // ---- element access (Complex_2D.h:167-305) ----
    void set_value(int x, int y, int type, T value)
    {
        if (x < 0 || x >= nx || y < 0 || y >= ny)
            throw nadia_cxx::Failure(NADIA_ERR_RANGE, "can not set value out of array bounds");
        switch (type) {
        case REAL: set_real(x, y, value); break;
        case IMAG: set_imag(x, y, value); break;
        case MAG: set_mag(x, y, value); break;
        case PHASE: set_phase(x, y, value); break;
        default: throw nadia_cxx::Failure(NADIA_ERR_INVALID, "unknown value type in set_value");
        }
    }
    inline void set_real(int x, int y, T v) { edit()[idx(x, y)] = v; }
    inline void set_imag(int x, int y, T v) { edit()[idx(x, y) + 1] = v; }
    inline void set_mag(int x, int y, T value)
    {
        double mag = get_mag(x, y);
        T *p = &edit()[idx(x, y)];
        if (mag == 0) {
            p[0] = value;
            p[1] = 0;
        } else {
            p[0] *= value / mag;
            p[1] *= value / mag;
        }
    }
    inline void set_phase(int x, int y, T value)
    {
        double mag = get_mag(x, y);
        T *p = &edit()[idx(x, y)];
        p[0] = mag * std::cos(value);
        p[1] = mag * std::sin(value);
    }
    inline T get_real(int x, int y) const { return view()[idx(x, y)]; }
    inline T get_imag(int x, int y) const { return view()[idx(x, y) + 1]; }
    inline T get_mag(int x, int y) const
    {
        const T *p = &view()[idx(x, y)];
        return std::sqrt(p[0] * p[0] + p[1] * p[1]);
    }
    inline T get_phase(int x, int y) const { return std::atan2(get_imag(x, y), get_real(x, y)); }
    T get_value(int x, int y, int type) const
    {
        switch (type) {
        case MAG: return get_mag(x, y);
        case REAL: return get_real(x, y);
        case IMAG: return get_imag(x, y);
        case PHASE: return get_phase(x, y);
        case MAG_SQ: return get_mag(x, y) * get_mag(x, y);
        default: throw nadia_cxx::Failure(NADIA_ERR_INVALID, "unknown value type in get_value");
        }
    }
    int get_size_x() const { return nx; }
    int get_size_y() const { return ny; }

    void get_2d(int type, Double_2D &result) const
    {
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) result.set(i, j, get_value(i, j, type));
    }

    // ---- whole-field operations (Complex_2D.c++:159-353) ----
    void scale(T f)
    {
        for (T &v : edit()) v *= f;
    }
    void add(ComplexR_2D &c2, T sc = 1)
    {
        same_size(c2, "add");
        const std::vector<T> &b = c2.view();
        std::vector<T> &d = edit();
        for (size_t k = 0; k < d.size(); ++k) d[k] += sc * b[k];
    }
    void multiply(ComplexR_2D &c2, T sc = 1)
    {
        same_size(c2, "multiply");
        const std::vector<T> &b = c2.view();
        std::vector<T> &d = edit();
        for (size_t k = 0; k < d.size(); k += 2) {
            T re = b[k] * d[k] - b[k + 1] * d[k + 1];
            T im = b[k] * d[k + 1] + b[k + 1] * d[k];
            d[k] = sc * re;
            d[k + 1] = sc * im;
        }
    }
    void multiply(Double_2D &d2, T sc = 1)
    {
        std::vector<T> &d = edit();
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                d[idx(i, j)] = sc * d2.get(i, j) * d[idx(i, j)];
                d[idx(i, j) + 1] = sc * d2.get(i, j) * d[idx(i, j) + 1];
            }
    }
    T get_norm() const
    {
        T s = 0;
        for (T v : view()) s += v * v;
        return std::sqrt(s);
    }
    ComplexR_2D *clone() const { return new ComplexR_2D(*this); }
    void copy(const ComplexR_2D &c)
    {
        same_size(c, "copy");
        a = c.view();
        edited();
    }
    // quadrant swap, optionally scaled by 1/sqrt(nx*ny) (Complex_2D.c++:318-353)
    void invert(bool scale = false)
    {
        std::vector<T> &d = edit();
        const int mx = nx / 2, my = ny / 2;
        const T s = scale ? T(1.0 / std::sqrt((double)nx * ny)) : T(1);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < my; ++j) {
                int in = i + mx, jn = j + my;
                if (i >= mx) in -= 2 * mx;
                T *p = &d[idx(in, jn)], *q = &d[idx(i, j)];
                T tr = p[0], ti = p[1];
                p[0] = q[0] * s;
                p[1] = q[1] * s;
                q[0] = tr * s;
                q[1] = ti * s;
            }
    }
    void conjugate()
    {
        std::vector<T> &d = edit();
        for (size_t k = 1; k < d.size(); k += 2) d[k] = -d[k];
    }
    void mirror()
    {
        std::vector<T> &d = edit();
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny / 2; ++j) {
                std::swap(d[idx(i, j)], d[idx(i, ny - 1 - j)]);
                std::swap(d[idx(i, j) + 1], d[idx(i, ny - 1 - j) + 1]);
            }
    }
    // unnormalised 2-D DFT on the GPU (Complex_2D.c++:487-503)
    void perform_forward_fft() { fft(1); }
    void perform_backward_fft() { fft(0); }
    void set_fftw_type(int) {}

    ComplexR_2D get_padded(int xa, int ya)
    {
        ComplexR_2D p(nx + 2 * xa, ny + 2 * ya);
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j) {
                p.a[p.idx(i + xa, j + ya)] = get_real(i, j);
                p.a[p.idx(i + xa, j + ya) + 1] = get_imag(i, j);
            }
        return p;
    }
    ComplexR_2D get_unpadded(int xa, int ya)
    {
        ComplexR_2D u(nx - 2 * xa, ny - 2 * ya);
        for (int i = 0; i < u.nx; ++i)
            for (int j = 0; j < u.ny; ++j) {
                u.a[u.idx(i, j)] = get_real(i + xa, j + ya);
                u.a[u.idx(i, j) + 1] = get_imag(i + xa, j + ya);
            }
        return u;
    }

    // interleaved storage (fetches the device copy first)
    const T *data() const { return view().data(); }

private:
    friend class BaseCDI;
    int nx, ny;
    mutable std::vector<T> a;
    mutable nadia_solver *owner = nullptr; // reconstruction whose estimate this mirrors
    mutable bool device_newer = false;     // the GPU holds a newer estimate
    mutable bool host_newer = false;       // edited on the host since the last upload

    inline size_t idx(int x, int y) const { return 2 * ((size_t)x * ny + y); }

    void fetch() const
    {
        if (!device_newer || !owner) return;
        device_newer = false;
        if (sizeof(T) == sizeof(float)) {
            nadia_cxx::check(nadia_get_exit_surface_wave_f32(owner, (float *)a.data()));
        } else {
            nadia_cxx::check(nadia_get_exit_surface_wave(owner, (double *)a.data()));
        }
    }
    const std::vector<T> &view() const
    {
        if (device_newer) fetch();
        return a;
    }
    std::vector<T> &edit()
    {
        if (device_newer) fetch();
        host_newer = true;
        return a;
    }
    void edited() { host_newer = true; }
    void push()
    {
        if (!host_newer || !owner) return;
        host_newer = false;
        if (sizeof(T) == sizeof(float))
            nadia_cxx::check(nadia_set_exit_surface_wave_f32(owner, (const float *)a.data()));
        else
            nadia_cxx::check(nadia_set_exit_surface_wave(owner, (const double *)a.data()));
    }
    void same_size(const ComplexR_2D &c, const char *what) const
    {
        if (c.nx != nx || c.ny != ny)
            throw nadia_cxx::Failure(NADIA_ERR_INVALID,
                                     std::string("in Complex_2D::") + what + ", the dimensions differ");
    }
    void fft(int forward)
    {
        std::vector<T> &d = edit();
        std::vector<double> t(d.begin(), d.end());
        nadia_cxx::check(nadia_fft2d(t.data(), nx, ny, forward));
        for (size_t k = 0; k < d.size(); ++k) d[k] = (T)t[k];
    }
};

#ifndef DOUBLE_PRECISION
typedef ComplexR_2D<float> Complex_2D;
#else
typedef ComplexR_2D<double> Complex_2D;
#endif

#endif
