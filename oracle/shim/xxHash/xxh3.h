/* Build shim for oracle/_ref only: the reference includes "xxHash/xxh3.h" from an
 * empty git submodule.  The xxHash 0.8.x header vendored by pyarrow stands in for
 * it (its include directory is passed on the compiler command line). */
#pragma once
#define XXH_INLINE_ALL
#include "xxhash.h"
