// fdtd_selfcheck.cu -- device check of the division by the cell size.
//
// The CPML terms divide by the constant cell size with Markstein's FMA
// correction (div_const, fdtd_common.cuh) instead of an IEEE division. This
// entry point runs both on the device and counts the inputs whose results
// differ in any bit: every one of the 2^32 float bit patterns, or 2^30
// doubles (random significands over the exponents where the correction is
// used, plus the same count of random bit patterns).
#include <cstdint>
#include <cstring>

#include "fdtd_b200.h"
#include "fdtd_launch.h"

namespace fdtd {
namespace {

__device__ __forceinline__ bool same_bits_f(float a, float b) {
  return __float_as_uint(a) == __float_as_uint(b) || (a != a && b != b);
}
__device__ __forceinline__ bool same_bits_d(double a, double b) {
  return __double_as_longlong(a) == __double_as_longlong(b) || (a != a && b != b);
}

__global__ void k_check_div_f(float d, float r, unsigned long long* bad) {
  unsigned long long local = 0;
  const unsigned long long n = 1ULL << 32;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += stride) {
    const float u = __uint_as_float((unsigned)k);
    if (!same_bits_f(div_const(u, d, r), __fdiv_rn(u, d))) ++local;
  }
  if (local) atomicAdd(bad, local);
}

__device__ __forceinline__ unsigned long long mix64(unsigned long long x) {
  x += 0x9e3779b97f4a7c15ULL;
  x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ULL;
  x = (x ^ (x >> 27)) * 0x94d049bb133111ebULL;
  return x ^ (x >> 31);
}

__global__ void k_check_div_d(double d, double r, unsigned long long n, unsigned long long* bad) {
  unsigned long long local = 0;
  const unsigned long long stride = (unsigned long long)gridDim.x * blockDim.x;
  for (unsigned long long k = (unsigned long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += stride) {
    const unsigned long long h = mix64(k);
    // even k: random significand and sign, biased exponent in [123, 1923]
    // (2^-900 .. 2^900); odd k: any bit pattern
    unsigned long long bits = h;
    if (!(k & 1)) {
      const unsigned long long e = 123 + (mix64(h) % 1801);
      bits = (h & 0x800FFFFFFFFFFFFFULL) | (e << 52);
    }
    const double u = __longlong_as_double((long long)bits);
    if (!same_bits_d(div_const(u, d, r), __ddiv_rn(u, d))) ++local;
  }
  if (local) atomicAdd(bad, local);
}

}  // namespace

int report_error(int code, const char* msg);

}  // namespace fdtd

extern "C" int fdtd_check_cell_division(int dtype, double cell_size, int device, int64_t* tested,
                                        int64_t* mismatches) {
  using namespace fdtd;
  if (!tested || !mismatches) return report_error(FDTD_ERR_INVALID, "null argument");
  if (dtype != FDTD_F32 && dtype != FDTD_F64) return report_error(FDTD_ERR_INVALID, "bad dtype");
  if (!(cell_size > 0)) return report_error(FDTD_ERR_INVALID, "cell size must be positive");
  DeviceGuard device_guard;   // the caller's current device is restored on return
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return report_error(FDTD_ERR_CUDA, cudaGetErrorString(e));
  unsigned long long* bad = nullptr;
  if ((e = cudaMalloc(&bad, sizeof(*bad))) != cudaSuccess) return report_error(FDTD_ERR_NOMEM, cudaGetErrorString(e));
  cudaMemset(bad, 0, sizeof(*bad));
  unsigned long long n;
  if (dtype == FDTD_F32) {
    const float d = (float)cell_size;
    const float r = 1.0f / d;   // IEEE division on the host
    n = 1ULL << 32;
    k_check_div_f<<<148 * 16, 256>>>(d, r, bad);
  } else {
    const double r = 1.0 / cell_size;
    n = 1ULL << 30;
    k_check_div_d<<<148 * 16, 256>>>(cell_size, r, n, bad);
  }
  unsigned long long h = 0;
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(&h, bad, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(bad);
  if (e != cudaSuccess) return report_error(FDTD_ERR_CUDA, cudaGetErrorString(e));
  *tested = (int64_t)n;
  *mismatches = (int64_t)h;
  return FDTD_OK;
}
