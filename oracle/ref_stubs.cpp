// ref_stubs.cpp -- TEST INFRASTRUCTURE (oracle/_ref only).  Link stand-ins
// for the libraries the reference's tool and file helpers reach but this
// build does not have: libtiff (NADIA/src/io_tiff.c), libhdf4
// (NADIA/src/io_hdf.c) and LAPACK's zhegv (NADIA/src/PartialCDI.c++).  The
// file functions report failure, as the reference does for a file it can
// not read; zhegv is only reached by partially coherent reconstructions,
// which nothing here runs, and aborts if it is.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <string>

#include <Double_2D.h>
#include <io.h>

int read_tiff(std::string file_name, Double_2D &)
{
    std::cout << "libtiff is not linked: " << file_name << std::endl;
    return 0;
}

int write_tiff(std::string file_name, const Double_2D &, bool, double, double)
{
    std::cout << "libtiff is not linked: " << file_name << std::endl;
    return 0;
}

int read_hdf4(std::string file_name, Double_2D &, const char *)
{
    std::cout << "libhdf4 is not linked: " << file_name << std::endl;
    return 0;
}

extern "C" void zhegv_()
{
    std::fprintf(stderr, "LAPACK is not linked (zhegv_)\n");
    std::abort();
}
