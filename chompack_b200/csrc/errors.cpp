// Thread-local error text for the C ABI (chb_last_error) and the build tag.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/chompack_b200.h"
#include "internal.h"

namespace chb {
static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }
}  // namespace chb

extern "C" const char* chb_last_error(void) { return chb::g_last_error.c_str(); }

extern "C" const char* chb_version(void) { return "chompack_b200 1.0 (sm_100a, fp64 multifrontal sweeps)"; }
