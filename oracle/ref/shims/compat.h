// Force-included when compiling the reference sources with g++ on Linux:
// maps the MSVC-only spellings they use onto GCC/glibc equivalents.
#pragma once
#include <cstdlib>
#include <cmath>
#include <limits>
#include <cstring>
#include <memory>
#include <string>
#define _aligned_malloc(size, align) aligned_alloc((align), (((size) + (align) - 1) / (align)) * (align))
#define _aligned_free(p) free(p)
#define __assume(x) __builtin_unreachable()
#define GYT_ALIGNED(x) alignas(x)
#define GYT_FORCE_INLINE inline
namespace std { using ::atan2f; }
