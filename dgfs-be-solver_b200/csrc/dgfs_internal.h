// Library-internal helpers shared by the host translation units.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace dgfs {

// A kernel's dynamic shared-memory limit belongs to the device that is
// current when it is set: set it once per device (bit d of `done` records
// device d; devices beyond 63 set it on every call).
template <typename K>
cudaError_t smem_limit_once(K* kern, int bytes, std::atomic<unsigned long long>& done) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
  if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
  e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_release);
  return e;
}

// Record a formatted message for dgfs_last_error() and return code.
int set_error(int code, const char* fmt, ...);
void clear_error();

// Bounded-wait check on the allocation-free path's error flag (vhs_noalloc.cu).
int noalloc_check_wait(unsigned long long limit_ns, void* stream);

}  // namespace dgfs
