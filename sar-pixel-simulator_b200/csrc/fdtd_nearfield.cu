// fdtd_nearfield.cu -- Poynting power through the internal phasor planes
// (processresults.py:128-257) on the device, from the simulation's own
// phasor planes.
//
// For each face the time-averaged flux Re(E x conj(H)) . n / 2 of every
// cell is weighted by the separable 2-D Simpson weights of its plane (rows
// by columns; the weights are those scipy.integrate.simpson applies, given
// by the caller) and summed in float64: one block-level shuffle reduction
// per block and face, the block partials summed on the host in block order
// (deterministic). The faces, in output order:
//   0 incident (the incident phasors' plane, normal -z)
//   1, 2 left bottom / top (x plane, normal -x; rows z < size_z_material,
//        then size_z_material <= z < nz_ph - 1)
//   3, 4 right bottom / top (normal +x)
//   5, 6 front bottom / top (y plane, normal -y)
//   7, 8 back bottom / top (normal +y)
//   9 down (z plane, normal -z), 10 up (normal +z)
#include <vector>

#include "fdtd_launch.h"

namespace fdtd {

namespace {

constexpr int kNfThreads = 256;
constexpr int kNfFaces = 11;

template <class T>
struct NearField {
  const T* ph;          // the simulation's phasor planes (complex interleaved)
  long long off[24];    // plane offsets (elements of T)
  const T* inc;         // incident phasors ex, ey, hx, hy: (ny_ph, nx_ph) complex each
  int nx_ph, ny_ph, nz_ph, szm;
  const double* wy;     // Simpson weights: ny_ph
  const double* wx;     // nx_ph
  const double* wzb;    // szm (rows below the material top)
  const double* wzt;    // nz_ph - 1 - szm
  double* partial;      // [face][block]
};

// Re(a conj(b)) and the z, x, y components of Re(E x conj(H)) in float64
__device__ __forceinline__ double re_conj(double ar, double ai, double br, double bi) { return ar * br + ai * bi; }

template <class T>
__device__ __forceinline__ void cplx(const T* p, long long k, double& re, double& im) {
  re = (double)p[2 * k];
  im = (double)p[2 * k + 1];
}

template <class T>
__global__ void __launch_bounds__(kNfThreads) k_near_field(NearField<T> a) {
  const int f = blockIdx.y;
  int rows, cols;
  const double* wr;
  const double* wc;
  int row0 = 0;
  double sign = 1.0;
  int pe1 = 0, pe2 = 0, ph1 = 0, ph2 = 0;   // planes of the two E and two H components
  const T* base = a.ph;
  if (f == 0 || f >= 9) {   // z planes: (ny_ph, nx_ph); E x H* . z = Ex Hy* - Ey Hx*
    rows = a.ny_ph; cols = a.nx_ph; wr = a.wy; wc = a.wx;
    sign = f == 10 ? 1.0 : -1.0;
    const int b = f == 10 ? 4 : 0;   // ex, ey, hx, hy of d (0) / u (4)
    pe1 = b; pe2 = b + 1; ph1 = b + 2; ph2 = b + 3;
  } else {
    const int side = (f - 1) / 2, top = (f - 1) % 2;   // side 0 l, 1 r, 2 f, 3 b
    rows = top ? a.nz_ph - 1 - a.szm : a.szm;
    row0 = top ? a.szm : 0;
    wr = top ? a.wzt : a.wzb;
    const bool xplane = side < 2;
    cols = xplane ? a.ny_ph : a.nx_ph;
    wc = xplane ? a.wy : a.wx;
    sign = (side & 1) ? 1.0 : -1.0;
    const int b = 8 + 4 * side;   // x planes: ey, ez, hy, hz; y planes: ex, ez, hx, hz
    pe1 = b; pe2 = b + 1; ph1 = b + 2; ph2 = b + 3;
  }
  double acc = 0.0;
  const long long n = (long long)rows * cols;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(idx / cols), c = (int)(idx - (long long)r * cols);
    const long long k = (long long)(r + row0) * cols + c;
    double e1r, e1i, e2r, e2i, h1r, h1i, h2r, h2i;
    if (f == 0) {   // incident phasors: four consecutive planes
      const long long pn = (long long)a.ny_ph * a.nx_ph;
      cplx(a.inc, k, e1r, e1i);
      cplx(a.inc, pn + k, e2r, e2i);
      cplx(a.inc, 2 * pn + k, h1r, h1i);
      cplx(a.inc, 3 * pn + k, h2r, h2i);
    } else {
      cplx(base + a.off[pe1], k, e1r, e1i);
      cplx(base + a.off[pe2], k, e2r, e2i);
      cplx(base + a.off[ph1], k, h1r, h1i);
      cplx(base + a.off[ph2], k, h2r, h2i);
    }
    double s;
    if (f == 0 || f >= 9) {
      // z: Ex Hy* - Ey Hx*   (e1 = Ex, e2 = Ey, h1 = Hx, h2 = Hy)
      s = re_conj(e1r, e1i, h2r, h2i) - re_conj(e2r, e2i, h1r, h1i);
    } else if ((f - 1) / 2 < 2) {
      // x: Ey Hz* - Ez Hy*   (e1 = Ey, e2 = Ez, h1 = Hy, h2 = Hz)
      s = re_conj(e1r, e1i, h2r, h2i) - re_conj(e2r, e2i, h1r, h1i);
    } else {
      // y: Ez Hx* - Ex Hz*   (e1 = Ex, e2 = Ez, h1 = Hx, h2 = Hz)
      s = re_conj(e2r, e2i, h1r, h1i) - re_conj(e1r, e1i, h2r, h2i);
    }
    acc += wr[r] * wc[c] * (0.5 * sign * s);
  }
  // block reduction (fixed order within the block)
  __shared__ double red[kNfThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < kNfThreads / 32; ++w) t += red[w];
    a.partial[(long long)f * gridDim.x + blockIdx.x] = t;
  }
}

}  // namespace

template <class T>
int near_field_power_run(const T* ph, const long long* off, const T* inc, int nx_ph, int ny_ph, int nz_ph,
                         int szm, const double* w_dev, double* partial, int blocks, double* out,
                         cudaStream_t st) {
  NearField<T> a;
  a.ph = ph;
  for (int k = 0; k < 24; ++k) a.off[k] = off[k];
  a.inc = inc;
  a.nx_ph = nx_ph; a.ny_ph = ny_ph; a.nz_ph = nz_ph; a.szm = szm;
  a.wy = w_dev;
  a.wx = w_dev + ny_ph;
  a.wzb = w_dev + ny_ph + nx_ph;
  a.wzt = w_dev + ny_ph + nx_ph + szm;
  a.partial = partial;
  k_near_field<T><<<dim3(blocks, kNfFaces, 1), kNfThreads, 0, st>>>(a);
  if (cudaGetLastError() != cudaSuccess) return 1;
  std::vector<double> h((size_t)kNfFaces * blocks);
  if (cudaMemcpyAsync(h.data(), partial, sizeof(double) * h.size(), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return 1;
  for (int f = 0; f < kNfFaces; ++f) {
    double t = 0.0;
    for (int b = 0; b < blocks; ++b) t += h[(size_t)f * blocks + b];
    out[f] = t;
  }
  return 0;
}

template int near_field_power_run<float>(const float*, const long long*, const float*, int, int, int, int,
                                         const double*, double*, int, double*, cudaStream_t);
template int near_field_power_run<double>(const double*, const long long*, const double*, int, int, int, int,
                                          const double*, double*, int, double*, cudaStream_t);

}  // namespace fdtd
