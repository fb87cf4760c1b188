// Test infrastructure (oracle only): force-included when the reference is
// compiled with g++. The reference is an MSVC project; Code/PathUtils.h:16
// calls the MSVC-only localtime_s(tm*, const time_t*). It maps onto POSIX
// localtime_r with the argument order MSVC uses.
#pragma once
#ifdef __cplusplus
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
