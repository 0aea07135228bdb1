// types.h -- constants of the drop-in C++ API (see include/nadia/BaseCDI.h).
// Same names and values as the reference's NADIA/include/types.h:43-61 so that
// code written against the reference compiles unchanged; FFTW itself is not
// needed (its planner flags are accepted and ignored).
#ifndef NADIA_DROPIN_TYPES_H
#define NADIA_DROPIN_TYPES_H

#define FAILURE 0
#define SUCCESS 1

#define REAL 0
#define IMAG 1
#define MAG 2
#define PHASE 3
#define MAG_SQ 4

#ifndef FFTW_MEASURE
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_PATIENT (1U << 5)
#endif

#include <stdexcept>
#include <string>

#include "../nadia_b200.h"

namespace nadia_cxx {

// A failing call of the underlying library.  The reference prints a message
// and exits the process; the drop-in classes throw this instead.
struct Failure : std::runtime_error {
    int code;
    Failure(int c, const std::string &what) : std::runtime_error(what), code(c) {}
};

inline void check(int rc)
{
    if (rc != NADIA_OK) throw Failure(rc, nadia_last_error());
}

} // namespace nadia_cxx

#endif
