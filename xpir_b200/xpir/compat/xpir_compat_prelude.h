// Force-included (g++ -include) ahead of every XPIR source compiled in this image: XPIR
// was written against older toolchains whose standard headers pulled these in
// transitively; g++ 13 does not.  With these compat headers, XPIR's sources compile
// unchanged without Boost or GMP development headers.
#ifndef XPIR_REF_PRELUDE_H
#define XPIR_REF_PRELUDE_H
#ifdef __cplusplus
#include <cstdint>
#include <cstring>
#include <climits>
#include <cmath>
#include <string>
#include <cassert>
#include <iomanip>
#endif
#include <semaphore.h>  // SEM_VALUE_MAX, used by pir/shared_queue.hpp
#endif
