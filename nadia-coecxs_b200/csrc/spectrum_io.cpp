// spectrum_io.cpp -- PolyCDI::set_spectrum(string) (NADIA/src/PolyCDI.c++:38-63)
// reading its file with the semantics of read_spec (NADIA/src/io_spec.c:61-133).
#include <cctype>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "solver.h"

namespace nadia {

// Tab-separated lines; tokens accumulate across lines, and the accumulated
// list is dropped whenever its first token does not start with a digit (so
// only leading header lines are discarded).  Pairs (energy, weight) become
// rows (1/energy, weight), each value passing through float.
std::vector<double> read_spec_file(const char *path)
{
    std::ifstream f(path);
    if (!f.is_open()) throw Error(NADIA_ERR_INVALID, std::string("could not open ") + path);
    std::vector<std::string> tok;
    std::string line;
    while (std::getline(f, line)) {
        std::stringstream ss(line);
        std::string t;
        while (std::getline(ss, t, '\t')) tok.push_back(t);
        if (tok.empty())
            throw Error(NADIA_ERR_INVALID, "spectrum file starts with an empty line");
        if (tok[0].empty() || !std::isdigit((unsigned char)tok[0][0])) tok.clear();
    }
    const size_t rows = tok.size() / 2;
    NADIA_REQUIRE(rows >= 1, NADIA_ERR_INVALID, "no spectrum rows in file");
    std::vector<double> out(2 * rows);
    float value = 0;
    for (size_t i = 0, k = 0; i < rows; ++i)
        for (int j = 0; j < 2; ++j, ++k) {
            float v;
            value = (std::sscanf(tok[k].c_str(), "%f", &v) == 1) ? v : 0.0f;
            if (j == 0) value = 1.0 / value;
            out[2 * i + j] = value;
        }
    return out;
}

} // namespace nadia

