/*
 * Forced-include header for building the reference's estimator sources
 * (SmallUPBP, written for MSVC 2013) with g++ on Linux.  Test infrastructure
 * only: it is used by oracle/build_ref.py to compile the reference oracle into
 * oracle/_ref/ and is never linked into the product library.
 *
 * It supplies the MSVC-only spellings the reference relies on
 * (__int64, __forceinline, _isnanf, sprintf_s, ...) with their g++ meaning.
 */
#ifndef UPBP_REF_COMPAT_H
#define UPBP_REF_COMPAT_H

#include <cmath>
#include <cstdio>
#include <cstdint>
#include <cstring>
#include <cstdlib>
#include <algorithm>

typedef signed char __int8;
typedef short __int16;
typedef int __int32;
typedef long long __int64;

#ifndef __forceinline
#define __forceinline inline __attribute__((always_inline))
#endif

#define _isnanf(x) std::isnan(x)
#define _finite(x) std::isfinite(x)
#define sprintf_s snprintf
#define sscanf_s sscanf
#define _snprintf snprintf
#define _strdup strdup
#define _stricmp strcasecmp

#endif
