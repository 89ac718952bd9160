// Library-internal helpers shared by the host translation units.
#pragma once

namespace dgfs {

// Record a formatted message for dgfs_last_error() and return code.
int set_error(int code, const char* fmt, ...);
void clear_error();

}  // namespace dgfs
