/* oracle/shim/CImg.h -- TEST INFRASTRUCTURE ONLY (part of the CPU oracle).
 * The reference's 3-D solver headers include <CImg.h> and open its namespace
 * (include/FFT_analysis3D.hpp:7,28) but the 3-D solver sources call nothing in
 * it; this empty stand-in replaces the vendored image library for the oracle
 * build, which keeps X11 out of it. */
#ifndef M3D_CIMG_STUB_H
#define M3D_CIMG_STUB_H
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <cmath>
#include <sys/stat.h>
namespace cimg_library {}
#endif
