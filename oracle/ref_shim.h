/* Force-included before every reference translation unit of the oracle build.
 *
 * The reference defines LinRT::M_PI<T> and LinRT::INFINITY (src/core/core.h:6-11); under glibc
 * with _GNU_SOURCE those names are macros, so the unmodified sources do not compile with g++.
 * Pulling the C headers in first and dropping the two macros lets them build as they are. */
#include <cmath>
#include <math.h>
#include <complex>
#include <atomic>
#include <iostream>
#include <cstdlib>
#include <mutex>
#include <string>
#undef M_PI
#undef INFINITY
