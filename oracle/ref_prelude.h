/* Forced-include prelude for compiling the reference's quality headers (dmo/DMOQuality.h and
 * what it includes) unmodified with nvcc on Linux. Test infrastructure only.
 *
 * The headers were written against MSVC, whose standard headers bring <cmath>, <cfloat> and
 * friends in transitively, and they call std::sqrtf, which libstdc++ does not declare. This
 * prelude adds those standard declarations; it changes no line of the reference. */
#pragma once
#include <cmath>
#include <cfloat>
#include <cstdio>
#include <vector>
#include <iostream>
#include <string>
#include <memory>
#include <algorithm>
namespace std { using ::sqrtf; using ::fabsf; using ::cbrtf; }
