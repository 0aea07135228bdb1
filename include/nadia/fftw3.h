// fftw3.h -- for callers of the reference that include <fftw3.h> for its
// planner flags (NADIA/examples/PlanarCDI_example.c:26,
// NADIA/tools/CDI_reconstruction.c:47).  This library does not use FFTW: the
// header only provides the flag constants that set_fftw_type accepts (and
// ignores here), with FFTW's values.  Put the real FFTW include directory
// first if the same program also calls FFTW itself.
#ifndef NADIA_DROPIN_FFTW3_H
#define NADIA_DROPIN_FFTW3_H

#include "types.h"

#ifndef FFTW_EXHAUSTIVE
#define FFTW_EXHAUSTIVE (1U << 3)
#endif

#endif
