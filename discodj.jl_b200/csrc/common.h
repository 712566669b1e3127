// Shared host-side helpers of libdjb200: status codes and the per-thread error text.
#pragma once

#include <cstdarg>
#include <cstdio>
#include <string>

#include "djb200.h"

namespace djb {

void set_error(const char* fmt, ...);
void clear_error();

// Returns `code` after recording the formatted message (use as `return fail(...)`).
int fail(int code, const char* fmt, ...);

}  // namespace djb
