/* ORACLE / TEST INFRASTRUCTURE ONLY.
 *
 * Forced-include prelude (g++ -include) for compiling the reference's own
 * PowerGrid/gridding.cpp, griddingSupport.cpp, ftCpu.cpp, fftCPU.cpp and
 * ftCpuWithGrads.cpp in place, unmodified, without Armadillo:
 *   - PGINCLUDES_H is pre-defined so PGIncludes.h (which includes
 *     <armadillo>, PGIncludes.h:26-42) is skipped;
 *   - the few names those four files take from it are supplied here:
 *     arma::uword (also visible unqualified, as griddingSupport.h
 *     expects), MRI_PI with the single-precision build's value
 *     (PGIncludes.h:69), RANGE() as a no-op (Tracer.hpp:19-34 without NVTX),
 *     and griddingTypes.h.
 * OpenACC pragmas are ignored by g++, so the CPU branches are compiled
 * (OPENACC_GPU is undefined: gridding.cpp:514, 529-539).
 */
#ifndef PG_ORACLE_REF_PRELUDE_H
#define PG_ORACLE_REF_PRELUDE_H
#define PGINCLUDES_H
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <string>
#include <algorithm>
namespace arma {
typedef unsigned long long uword;
}
using arma::uword;
#define MRI_PI 3.1415926535897932384626433832795029f
#define RANGE(...)
#include "griddingTypes.h"
#endif
