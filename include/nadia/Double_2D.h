// Double_2D.h -- drop-in for the reference's Real_2D<T> / Double_2D
// (NADIA/include/Double_2D.h): a host array of nx*ny values, element (x,y)
// at x*ny+y, with the accessors and reductions the reconstruction API uses.
// Double_2D is Real_2D<float> unless DOUBLE_PRECISION is defined, as in the
// reference (Double_2D.h:352-356).
#ifndef NADIA_DROPIN_DOUBLE_2D_H
#define NADIA_DROPIN_DOUBLE_2D_H

#include <cmath>
#include <cstring>
#include <vector>

template <class T>
class Real_2D {
public:
    Real_2D() : nx(0), ny(0) {}
    Real_2D(int x_size, int y_size) { allocate_memory(x_size, y_size); }

    void allocate_memory(int x_size, int y_size)
    {
        nx = x_size;
        ny = y_size;
        v.assign((size_t)nx * ny, T(0));
    }

    void copy(const Real_2D<T> &o) { std::memcpy(v.data(), o.v.data(), sizeof(T) * v.size()); }

    inline void set(int x, int y, T value) { v[(size_t)x * ny + y] = value; }

    // out-of-range coordinates read 0 (the reference tests x > nx and y > ny)
    inline T get(int x, int y) const
    {
        if (x < 0 || x >= nx || y < 0 || y >= ny) return 0;
        return v[(size_t)x * ny + y];
    }

    inline int get_size_x() const { return nx; }
    inline int get_size_y() const { return ny; }

    T get_sum() const
    {
        T t = 0;
        for (T a : v) t += a;
        return t;
    }
    T get_abs_sum() const
    {
        T t = 0;
        for (T a : v) t += std::fabs(a);
        return t;
    }
    T get_ave() const { return get_sum() / (T)(nx * ny); }
    T get_max() const
    {
        if (v.empty()) return 0;
        T m = v[0];
        for (T a : v)
            if (a > m) m = a;
        return m;
    }
    T get_min() const
    {
        if (v.empty()) return 0;
        T m = v[0];
        for (T a : v)
            if (a < m) m = a;
        return m;
    }
    void add(const Real_2D<T> &o, double norm = 1.0)
    {
        for (size_t k = 0; k < v.size(); ++k) v[k] += norm * o.v[k];
    }
    void scale(double s)
    {
        for (T &a : v) a *= s;
    }
    void square()
    {
        for (T &a : v) a *= a;
    }
    void sq_root()
    {
        for (T &a : v) a = std::sqrt(a);
    }
    void mirror()
    {
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny / 2; ++j) std::swap(v[(size_t)i * ny + j], v[(size_t)i * ny + ny - 1 - j]);
    }

    // contiguous storage, element (x,y) at x*ny+y
    const T *data() const { return v.data(); }
    T *data() { return v.data(); }

private:
    int nx, ny;
    std::vector<T> v;
};

#ifndef DOUBLE_PRECISION
typedef Real_2D<float> Double_2D;
#else
typedef Real_2D<double> Double_2D;
#endif

#endif
