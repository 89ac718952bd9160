// Library-internal helpers shared by the host translation units.
#pragma once

namespace dgfs {

// Record a formatted message for dgfs_last_error() and return code.
int set_error(int code, const char* fmt, ...);
void clear_error();

// Bounded-wait check on the allocation-free path's error flag (vhs_noalloc.cu).
int noalloc_check_wait(unsigned long long limit_ns, void* stream);

}  // namespace dgfs
