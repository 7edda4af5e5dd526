// Internal declarations shared by the host sources of the native library.
#pragma once
#include <cstdint>

namespace chb {
// Record an error message for chb_last_error() and return `code`.
int set_error(int code, const char* fmt, ...);
void clear_error();
}  // namespace chb
