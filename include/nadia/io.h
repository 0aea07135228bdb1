// io.h -- drop-in for the reference's file helpers (NADIA/include/io.h) that
// need no external library: the raw binary formats .cplx (complex) and .dbin
// (real) -- doubles in column-major order, element (x, y) at y*nx + x --, the
// P2 (ASCII greyscale) .ppm images, and .txt spectra.  TIFF and HDF4 need
// libtiff and libhdf4, which this library does not use: read_tiff,
// read_hdf4 and write_tiff report that and fail.
//
// As in the reference, functions return SUCCESS (1) or FAILURE (0) and print
// why they failed; read_image / write_image dispatch on the file name and,
// on failure, throw nadia_cxx::Failure where the reference exits.
#ifndef NADIA_DROPIN_IO_H
#define NADIA_DROPIN_IO_H

#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "Complex_2D.h"
#include "Double_2D.h"
#include "types.h"

// io_cplx.c: nx*ny interleaved (re, im) doubles, column-major
inline int read_cplx(std::string file_name, Complex_2D &complex)
{
    const int nx = complex.get_size_x(), ny = complex.get_size_y();
    std::vector<double> buf((size_t)2 * nx * ny);
    FILE *f = std::fopen(file_name.c_str(), "rb");
    if (!f) {
        std::cout << "Could not open the file " << file_name << std::endl;
        return FAILURE;
    }
    const size_t got = std::fread(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    if (got != buf.size()) {
        std::cout << "Could not correctly read the file " << file_name
                  << ". Perhaps the dimensions specifies are wrong?" << std::endl;
        return FAILURE;
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            complex.set_real(i, j, buf[2 * ((size_t)j * nx + i)]);
            complex.set_imag(i, j, buf[2 * ((size_t)j * nx + i) + 1]);
        }
    return SUCCESS;
}

inline int write_cplx(std::string file_name, const Complex_2D &complex)
{
    const int nx = complex.get_size_x(), ny = complex.get_size_y();
    std::vector<double> buf((size_t)2 * nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) {
            buf[2 * ((size_t)j * nx + i)] = complex.get_real(i, j);
            buf[2 * ((size_t)j * nx + i) + 1] = complex.get_imag(i, j);
        }
    FILE *f = std::fopen(file_name.c_str(), "w+b");
    if (!f) {
        std::cout << "Could not open the file " << file_name << std::endl;
        return FAILURE;
    }
    std::fwrite(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    return SUCCESS;
}

// io_dbin.c: nx*ny doubles, column-major
inline int read_dbin(std::string file_name, int nx, int ny, Double_2D &data)
{
    std::vector<double> buf((size_t)nx * ny);
    FILE *f = std::fopen(file_name.c_str(), "rb");
    if (!f) {
        std::cout << "Could not open the file " << file_name << "." << std::endl;
        return FAILURE;
    }
    const size_t got = std::fread(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    if (got != buf.size()) {
        std::cout << "Could not correctly read the file" << file_name
                  << ". Perhaps the dimensions specifies are wrong"
                  << " or the format type is not double?" << std::endl;
        return FAILURE;
    }
    if (data.get_size_x() == 0) data.allocate_memory(nx, ny);
    if (data.get_size_x() != nx || data.get_size_y() != ny) {
        std::cout << "The Double_2D object supplied has the wrong dimensions" << std::endl;
        return FAILURE;
    }
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) data.set(i, j, buf[(size_t)j * nx + i]);
    return SUCCESS;
}

inline int write_dbin(std::string file_name, const Double_2D &data)
{
    const int nx = data.get_size_x(), ny = data.get_size_y();
    std::vector<double> buf((size_t)nx * ny);
    for (int i = 0; i < nx; ++i)
        for (int j = 0; j < ny; ++j) buf[(size_t)j * nx + i] = data.get(i, j);
    FILE *f = std::fopen(file_name.c_str(), "w+b");
    if (!f) {
        std::cout << "Could not open the file " << file_name << std::endl;
        return FAILURE;
    }
    std::fwrite(buf.data(), sizeof(double), buf.size(), f);
    std::fclose(f);
    return SUCCESS;
}

// the grey level of a value for an image of pixel_max levels (io.h:88-117)
inline unsigned int io_scale_value(double min, double max, int pixel_max, double value,
                                   bool log_scale)
{
    if (min == max) return max;
    double grad;
    if (log_scale) {
        grad = (double)(pixel_max - 1) / (double)(max - min);
        value = grad * (value - min) + 1;
        min = 0;
        max = log10(pixel_max);
        value = log10(value);
    }
    grad = (double)pixel_max / (double)(max - min);
    value = grad * (value - min);
    if (value < 0) value = min;
    if (value > pixel_max) value = pixel_max;
    return value;
}

// io_ppm.c: 16-bit P2 greyscale, rows of y, scaled between min and max (the
// data's own range when both are 0)
inline int write_ppm(std::string file_name, const Double_2D &data, bool log_scale = false,
                     double min = 0, double max = 0)
{
    const int nx = data.get_size_x(), ny = data.get_size_y();
    const int largest = (int)pow(2.0, 16.0) - 1;
    std::ofstream out(file_name.c_str());
    if (!out.is_open()) {
        std::cout << "Could not open the file " << file_name << "for writing" << std::endl;
        return FAILURE;
    }
    if (min == 0 && max == 0) {
        max = data.get_max();
        min = data.get_min();
    }
    out << "P2" << std::endl;
    out << "#" << file_name << std::endl;
    out << "# original range: " << min << "-" << max << std::endl;
    out << "# log scale? " << log_scale << std::endl;
    out << nx << " " << ny << std::endl;
    out << largest << std::endl;
    for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i)
            out << io_scale_value(min, max, largest, data.get(i, j), log_scale) << " ";
        out << std::endl;
    }
    return SUCCESS;
}

// io.h's line_tokeniser (NADIA/include/io.h:289-299): the tab-separated
// fields of a line appended to *data (a line without tabs is one field)
inline void line_tokeniser(std::string line, std::vector<std::string> *data)
{
    std::string field;
    std::istringstream in(line);
    while (std::getline(in, field, '\t')) data->push_back(field);
}

// a P2 image back into a Double_2D (grey levels as values)
inline int read_ppm(std::string file_name, Double_2D &data)
{
    std::ifstream in(file_name.c_str());
    if (!in.is_open()) {
        std::cout << "Could not open the file " << file_name << std::endl;
        return FAILURE;
    }
    std::vector<std::string> tok;
    std::string line;
    while (std::getline(in, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line = line.substr(0, h);
        std::istringstream ss(line);
        std::string t;
        while (ss >> t) tok.push_back(t);
    }
    if (tok.size() < 4 || tok[0] != "P2") {
        std::cout << "ppm wrong type. Only handling P2 at the moment" << std::endl;
        return FAILURE;
    }
    const int nx = std::atoi(tok[1].c_str()), ny = std::atoi(tok[2].c_str());
    if (nx <= 0 || ny <= 0 || tok.size() != 4 + (size_t)nx * ny) {
        std::cout << "Confused about the ppm dimensions.. exiting." << std::endl;
        return FAILURE;
    }
    if (data.get_size_x() == 0) data.allocate_memory(nx, ny);
    for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i) data.set(i, j, std::atof(tok[4 + (size_t)j * nx + i].c_str()));
    return SUCCESS;
}

// io_spec.c: tab-separated (energy, weight) lines to rows (1/energy, weight)
inline int read_spec(std::string file_name, Double_2D &data)
{
    int n = 0;
    if (nadia_read_spec(file_name.c_str(), nullptr, 0, &n) != NADIA_OK) {
        std::cout << "Could not read the file " << file_name << ": " << nadia_last_error()
                  << std::endl;
        return FAILURE;
    }
    std::vector<double> rows(2 * (size_t)n);
    nadia_cxx::check(nadia_read_spec(file_name.c_str(), rows.data(), n, &n));
    if (n > 100)
        std::cout << "You are using " << n << " number of points"
                  << "which is quite a lot. I usually find ~50 to be a "
                  << "good number." << std::endl;
    if (data.get_size_x() == 0) data.allocate_memory(n, 2);
    for (int i = 0; i < n; ++i) {
        data.set(i, 0, rows[2 * (size_t)i]);
        data.set(i, 1, rows[2 * (size_t)i + 1]);
    }
    return SUCCESS;
}

inline int write_spec(std::string file_name, const Double_2D &data)
{
    std::ofstream out(file_name.c_str());
    if (!out.is_open()) {
        std::cout << "Could not open the file " << file_name << "for writing" << std::endl;
        return FAILURE;
    }
    out << "Energy" << '\t' << "F.Density" << std::endl;
    for (int j = 0; j < data.get_size_y(); ++j) {
        for (int i = 0; i < data.get_size_x(); ++i) out << data.get(i, j) << '\t';
        out << std::endl;
    }
    return SUCCESS;
}

inline int read_tiff(std::string file_name, Double_2D &)
{
    std::cout << "TIFF files need libtiff, which this build does not use: " << file_name << std::endl;
    return FAILURE;
}
inline int write_tiff(std::string file_name, const Double_2D &, bool = false, double = 0,
                      double = 0)
{
    std::cout << "TIFF files need libtiff, which this build does not use: " << file_name << std::endl;
    return FAILURE;
}
inline int read_hdf4(std::string file_name, Double_2D &, const char * = "data")
{
    std::cout << "HDF4 files need libhdf4, which this build does not use: " << file_name << std::endl;
    return FAILURE;
}

// read_image / write_image (io.h:121-185): by extension
inline void read_image(std::string file_name, Double_2D &data, int nx = 0, int ny = 0,
                       const char *data_name = "data")
{
    int status = FAILURE;
    const char *f = file_name.c_str();
    if (std::strstr(f, ".tiff") || std::strstr(f, ".tif")) status = read_tiff(file_name, data);
    if (std::strstr(f, ".ppm")) status = read_ppm(file_name, data);
    if (std::strstr(f, ".txt")) status = read_spec(file_name, data);
    if (std::strstr(f, ".dbin")) {
        if (nx == 0 || ny == 0)
            std::cout << "Please pass the dimensions of the dbin file you"
                      << " wish to read to the read_image method." << std::endl;
        else
            status = read_dbin(file_name, nx, ny, data);
    }
    if (std::strstr(f, ".hdf")) status = read_hdf4(file_name, data, data_name);
    if (status == FAILURE)
        throw nadia_cxx::Failure(NADIA_ERR_INVALID, "failed to read the file: " + file_name);
}

inline void write_image(std::string file_name, Double_2D &data, bool log_scale = false,
                        double min = 0, double max = 0)
{
    int status = FAILURE;
    const char *f = file_name.c_str();
    if (std::strstr(f, ".tiff") || std::strstr(f, ".tif"))
        status = write_tiff(file_name, data, log_scale, min, max);
    if (std::strstr(f, ".ppm")) status = write_ppm(file_name, data, log_scale, min, max);
    if (std::strstr(f, ".txt")) status = write_spec(file_name, data);
    if (std::strstr(f, ".dbin")) status = write_dbin(file_name, data);
    if (status == FAILURE)
        throw nadia_cxx::Failure(NADIA_ERR_INVALID, "failed to write to the file: " + file_name);
}

#endif
