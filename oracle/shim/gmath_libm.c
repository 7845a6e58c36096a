/* The project's elementary functions (galic_b200/csrc/gmath.h) under the C
 * library's names, linked into oracle/_ref/libgalic_ref_gmath.so: GALIC's own
 * unmodified C built this way evaluates log, atan2, sin, cos and acos exactly
 * as the CUDA kernels do, so its orbits, grids and merit values can be
 * compared with the GPU's bit for bit.  Test infrastructure only.  The
 * reference objects of that library are compiled with -fno-builtin for these
 * functions (no constant folding, no sin/cos -> sincos fusion) and the
 * library is linked with -Bsymbolic, so every call inside it reaches these
 * definitions. */
#include "../../galic_b200/csrc/gmath.h"

double log(double x) { return gm_log(x); }
double atan2(double y, double x) { return gm_atan2(y, x); }
double sin(double x) { return gm_sin(x); }
double cos(double x) { return gm_cos(x); }
double acos(double x) { return gm_acos(x); }
