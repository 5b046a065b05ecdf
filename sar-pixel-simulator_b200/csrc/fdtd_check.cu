// fdtd_check.cu -- the device allocation table and the violation word of the
// bounds-checked build (fdtd_check.cuh); no-ops in the normal build.
#include <algorithm>
#include <mutex>
#include <vector>

#include "fdtd_check.cuh"

namespace fdtd {

#ifdef FDTD_BOUNDS_CHECK
__device__ CheckRange g_check_ranges[kMaxCheckRanges];
__device__ int g_check_n;
__device__ unsigned long long g_check_bad[4];

namespace {
std::mutex g_mu;
std::vector<CheckRange> g_host;   // every live allocation of every device

// The table holds the allocations of every device: a copy on the current
// device (the one whose kernels run next).
int push_table() {
  const int n = (int)std::min<size_t>(g_host.size(), kMaxCheckRanges);
  if (n > 0 && cudaMemcpyToSymbol(g_check_ranges, g_host.data(), sizeof(CheckRange) * n) != cudaSuccess)
    return 1;
  return cudaMemcpyToSymbol(g_check_n, &n, sizeof(int)) == cudaSuccess ? 0 : 1;
}
}  // namespace

bool check_enabled() { return true; }

int check_register(const void* p, size_t bytes) {
  std::lock_guard<std::mutex> lock(g_mu);
  const unsigned long long lo = (unsigned long long)p;
  g_host.push_back({lo, lo + bytes});
  if (g_host.size() > (size_t)kMaxCheckRanges) return 1;
  return push_table();
}

void check_unregister(const void* p) {
  std::lock_guard<std::mutex> lock(g_mu);
  const unsigned long long lo = (unsigned long long)p;
  g_host.erase(std::remove_if(g_host.begin(), g_host.end(), [&](const CheckRange& r) { return r.lo == lo; }),
               g_host.end());
  push_table();
}

int check_take(unsigned long long* count, unsigned long long* what, long long* bytes, long long* line) {
  unsigned long long w[4] = {0, 0, 0, 0};
  if (cudaMemcpyFromSymbol(w, g_check_bad, sizeof(w)) != cudaSuccess) return 1;
  *count = w[0];
  *what = w[1];
  *bytes = (long long)w[2];
  *line = (long long)w[3];
  if (w[0]) {
    const unsigned long long z[4] = {0, 0, 0, 0};
    if (cudaMemcpyToSymbol(g_check_bad, z, sizeof(z)) != cudaSuccess) return 1;
  }
  return 0;
}
#else
bool check_enabled() { return false; }
int check_register(const void*, size_t) { return 0; }
void check_unregister(const void*) {}
int check_take(unsigned long long* count, unsigned long long* what, long long* bytes, long long* line) {
  *count = *what = 0;
  *bytes = *line = 0;
  return 0;
}
#endif

}  // namespace fdtd
