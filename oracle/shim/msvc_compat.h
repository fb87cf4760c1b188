// Test infrastructure (oracle only): force-included when the reference is
// compiled with g++. The reference is an MSVC project, and two things differ
// between MSVC's headers and libstdc++'s:
//  * Code/PathUtils.h:16 calls the MSVC-only localtime_s(tm*, const time_t*);
//    it maps onto POSIX localtime_r with the argument order MSVC uses.
//  * Code/Operator.h (e.g. :140-148, :291-301, :611-643) calls unqualified
//    abs() on doubles inside namespace OLK. MSVC's <cmath>/<stdlib.h> declare
//    the floating-point abs overloads in the global namespace, so those calls
//    take |x|. With libstdc++ and only <cmath> included, the global abs is C's
//    int abs(int), which truncates the distances (metres, < 1) to 0 and
//    silently changes the singular integrals. Including libstdc++'s C++
//    <stdlib.h> wrapper brings std::abs(double) into the global namespace, as
//    MSVC does.
#pragma once
#ifdef __cplusplus
#include <stdlib.h>
#include <math.h>
#include <ctime>
#include <sstream>
#include <iomanip>
#include <map>
#include <array>
#include <unordered_map>
#include <unordered_set>
#include <algorithm>
#include <stdexcept>
inline int localtime_s(std::tm* out, const std::time_t* t) {
  return localtime_r(t, out) ? 0 : 1;
}
#endif
