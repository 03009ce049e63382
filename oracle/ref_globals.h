/*
 * ref_globals.h - forced include for oracle/ref_harness.cpp (test infrastructure).
 *
 * Provides the compile-time configuration of src/bunnykiller.h:26-78 (DIM 3, RGB spectrum,
 * float Real, MAX_BPT_VERTICES 64, _SIGMA_VISIBILITY_ 1e-5) and defines its include guard,
 * so the reference headers compile with their own triangle/BVH backend instead of the
 * hard-wired _USE_EMBREE_: the ref_render_bvh build of oracle/ref_harness.cpp.
 */
#ifndef _GLOBALS_H_
#define _GLOBALS_H_
/* standard headers some reference headers use without including them */
#include <list>
#include <array>
#include <memory>
#include <limits>
#include <algorithm>
#include <stdexcept>
#define DIM 3
#define SPECTRUM_CHANNELS 3
using Real = float;
#define MAX_BPT_VERTICES 64
#ifdef min
#undef min
#endif
#ifdef max
#undef max
#endif
#ifndef _USE_MATH_DEFINES
#define _USE_MATH_DEFINES
#endif
#define MAX_NB_OBJECTS_LEAF 6
#define _SIGMA_VISIBILITY_ 1e-5
#endif
