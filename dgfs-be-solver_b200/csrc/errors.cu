// Thread-local error reporting for the C ABI.
#include <cstdarg>
#include <cstdio>
#include <string>

#include "../../include/dgfs_b200.h"
#include "dgfs_internal.h"

namespace dgfs {

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

}  // namespace dgfs

extern "C" const char* dgfs_last_error(void) { return dgfs::g_last_error.c_str(); }

extern "C" const char* dgfs_version(void) { return "dgfs_b200 0.1.0 (sm_100a)"; }
