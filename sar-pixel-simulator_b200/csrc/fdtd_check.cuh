// fdtd_check.cuh -- the bounds-checked build of the library.
//
// Built with -DFDTD_BOUNDS_CHECK (libfdtd_b200_check.so, build.py
// --bounds-check), every vector and scalar global-memory access of the step
// kernels (vector loads and stores, scalar neighbour loads, the phasor
// accumulators, the asynchronous plane copies) is checked against a device
// table of the library's live allocations, and its alignment against its
// size; shared-memory indices are checked against their arrays at their
// sites. A failed check records the first bad access (address or index,
// size, source line) in a device word and skips the access: a load gives
// zero, a store is dropped. Nothing traps. fdtd_synchronize reports a
// recorded violation as FDTD_ERR_BOUNDS. In the normal build every check is
// the constant true and costs nothing.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace fdtd {

#ifdef FDTD_BOUNDS_CHECK
constexpr int kMaxCheckRanges = 1024;
struct CheckRange {
  unsigned long long lo, hi;   // [lo, hi) of one allocation
};
extern __device__ CheckRange g_check_ranges[kMaxCheckRanges];
extern __device__ int g_check_n;
// [0] bad accesses so far, [1] the first one's address (shared: its index),
// [2] its size in bytes (-1: a shared index), [3] its source line
extern __device__ unsigned long long g_check_bad[4];

__device__ __forceinline__ void check_record(unsigned long long what, long long bytes, int line) {
  if (atomicAdd(&g_check_bad[0], 1ULL) == 0ULL) {
    g_check_bad[1] = what;
    g_check_bad[2] = (unsigned long long)bytes;
    g_check_bad[3] = (unsigned long long)line;
  }
}

static __device__ __noinline__ bool check_global(const void* p, int bytes, int line) {
  const unsigned long long a = (unsigned long long)p;
  const int align = bytes < 16 ? bytes : 16;
  if (a & (unsigned long long)(align - 1)) {
    check_record(a, bytes, line);
    return false;
  }
  const int n = g_check_n;
  for (int k = 0; k < n; ++k)
    if (a >= g_check_ranges[k].lo && a + bytes <= g_check_ranges[k].hi) return true;
  check_record(a, bytes, line);
  return false;
}

__device__ __forceinline__ bool check_shared(long long idx, long long n, int line) {
  if (idx >= 0 && idx < n) return true;
  check_record((unsigned long long)idx, -1, line);
  return false;
}

// p: a global address of `bytes` bytes (shared addresses pass; their
// indices are checked with FDTD_CHECK_SMEM)
#define FDTD_CHECK_PTR(p, bytes) (__isShared(p) || ::fdtd::check_global((p), (bytes), __LINE__))
#define FDTD_CHECK_SMEM(idx, n) ::fdtd::check_shared((long long)(idx), (long long)(n), __LINE__)
#else
#define FDTD_CHECK_PTR(p, bytes) true
#define FDTD_CHECK_SMEM(idx, n) true
#endif

// Checked scalar load and store (plain ones in the normal build).
template <class T>
__device__ __forceinline__ T ldc(const T* p) {
  return FDTD_CHECK_PTR(p, (int)sizeof(T)) ? *p : T(0);
}
template <class T>
__device__ __forceinline__ void stc(T* p, T v) {
  if (FDTD_CHECK_PTR(p, (int)sizeof(T))) *p = v;
}

// Host side (fdtd_check.cu; no-ops in the normal build): allocations enter
// and leave the table; check_take returns the number of bad accesses since
// the last call with the first one's details, and clears them.
bool check_enabled();
int check_register(const void* p, size_t bytes);
void check_unregister(const void* p);
int check_take(unsigned long long* count, unsigned long long* what, long long* bytes, long long* line);

}  // namespace fdtd
