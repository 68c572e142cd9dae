// Internal helpers shared by the library's translation units.
#ifndef FREHD_INTERNAL_H
#define FREHD_INTERNAL_H

#include <cstdarg>
#include <cstdio>

#include "frehd_b200.h"

namespace frehd {

// Record an error message for frehd_last_error() and return `code`.
int fail(int code, const char *fmt, ...);
void clear_error();

}  // namespace frehd

#endif
