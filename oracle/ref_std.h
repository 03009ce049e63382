/*
 * ref_std.h - forced include for the Embree builds of oracle/ref_harness.cpp and
 * oracle/ref_hits.cpp (test infrastructure).  Some reference headers use standard-library
 * names without including their headers (the reference's own build gets them through
 * src/bunnykiller.cpp's include order); this provides them.  The configuration itself is
 * src/bunnykiller.h's, unchanged (_USE_EMBREE_, float Real, _SIGMA_VISIBILITY_ 1e-5).
 */
#include <list>
#include <array>
#include <memory>
#include <limits>
#include <algorithm>
#include <stdexcept>
