// io_shim.cpp -- C entry points over the file helpers (io.h) and the
// configuration reader (Config.h), so that a test can drive them from
// Python.  The same source compiles against the drop-in headers
// (include/nadia) and against the reference's own headers (oracle/_ref),
// which is how the tests compare the two byte for byte.  Arrays cross as
// nx*ny doubles with element (x, y) at x*ny + y (complex: interleaved pairs).
#include <cstring>
#include <list>
#include <sstream>
#include <string>

#include "Complex_2D.h"
#include "Config.h"
#include "Double_2D.h"
#include "io.h"

namespace {

void to_2d(Double_2D &d, const double *v, int nx, int ny)
{
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) d.set(i, j, v[(size_t)i * ny + j]);
}

int from_2d(const Double_2D &d, int cap, double *out, int *nx, int *ny)
{
    *nx = d.get_size_x();
    *ny = d.get_size_y();
    if ((long)*nx * *ny > cap) return -1;
    for (int i = 0; i < *nx; ++i)
        for (int j = 0; j < *ny; ++j) out[(size_t)i * *ny + j] = d.get(i, j);
    return 1;
}

int put(const std::string &s, char *out, int cap)
{
    if ((int)s.size() + 1 > cap) return -1;
    std::memcpy(out, s.c_str(), s.size() + 1);
    return 1;
}

} // namespace

extern "C" {

int shim_write_cplx(const char *path, int nx, int ny, const double *v)
{
    Complex_2D c(nx, ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            c.set_real(i, j, v[2 * ((size_t)i * ny + j)]);
            c.set_imag(i, j, v[2 * ((size_t)i * ny + j) + 1]);
        }
    return write_cplx(path, c);
}

int shim_read_cplx(const char *path, int nx, int ny, double *out)
{
    Complex_2D c(nx, ny);
    const int st = read_cplx(path, c);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            out[2 * ((size_t)i * ny + j)] = c.get_real(i, j);
            out[2 * ((size_t)i * ny + j) + 1] = c.get_imag(i, j);
        }
    return st;
}

int shim_write_dbin(const char *path, int nx, int ny, const double *v)
{
    Double_2D d(nx, ny);
    to_2d(d, v, nx, ny);
    return write_dbin(path, d);
}

int shim_read_dbin(const char *path, int nx, int ny, double *out)
{
    Double_2D d;
    const int st = read_dbin(path, nx, ny, d);
    if (st != 1) return st;
    int x, y;
    return from_2d(d, nx * ny, out, &x, &y);
}

int shim_write_ppm(const char *path, int nx, int ny, const double *v, int log_scale, double min,
                   double max)
{
    Double_2D d(nx, ny);
    to_2d(d, v, nx, ny);
    return write_ppm(path, d, log_scale != 0, min, max);
}

int shim_read_ppm(const char *path, int cap, double *out, int *nx, int *ny)
{
    Double_2D d;
    const int st = read_ppm(path, d);
    if (st != 1) return st;
    return from_2d(d, cap, out, nx, ny);
}

int shim_write_spec(const char *path, int nx, int ny, const double *v)
{
    Double_2D d(nx, ny);
    to_2d(d, v, nx, ny);
    return write_spec(path, d);
}

int shim_read_spec(const char *path, int cap, double *out, int *nx, int *ny)
{
    Double_2D d;
    const int st = read_spec(path, d);
    if (st != 1) return st;
    return from_2d(d, cap, out, nx, ny);
}

unsigned shim_scale_value(double min, double max, int pixel_max, double value, int log_scale)
{
    return io_scale_value(min, max, pixel_max, value, log_scale != 0);
}

// kind: 's' getString, 'd' getDouble, 'i' getInt, 'S' getStringList,
// 'I' getIntList; lists are written one entry per line.  Returns the
// reader's status after the call, or -1 when out is too small.
int shim_config(const char *path, const char *key, int kind, char *out, int cap)
{
    Config c(path);
    std::ostringstream s;
    s.precision(17);
    if (kind == 's') s << c.getString(key);
    if (kind == 'd') s << c.getDouble(key);
    if (kind == 'i') s << c.getInt(key);
    if (kind == 'S') {
        std::list<std::string> *l = c.getStringList(key);
        if (l)
            for (const std::string &v : *l) s << v << "\n";
        delete l;
    }
    if (kind == 'I') {
        std::list<int> *l = c.getIntList(key);
        if (l)
            for (int v : *l) s << v << "\n";
        delete l;
    }
    if (put(s.str(), out, cap) < 0) return -1;
    return c.getStatus();
}

// line_tokeniser's fields joined by '|', each followed by it
int shim_tokenise(const char *line, char *out, int cap)
{
    std::vector<std::string> f;
    line_tokeniser(line, &f);
    std::string s;
    for (const std::string &v : f) s += v + "|";
    return put(s, out, cap) < 0 ? -1 : (int)f.size();
}

} // extern "C"
