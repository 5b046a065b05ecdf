// fdtd_split.cu -- the split step (H pass, E pass), the phasor pass, the
// step-counter advance and the eps/sigma -> Ca/Cb kernel.
//
// The split step updates the fields in place: the H pass reads E and writes
// H, the E pass reads H and writes E, so no cell is read after another
// thread wrote it within a pass. It moves 80 B per FP32 cell-update against
// the 56 B minimum; the fused pass (fdtd_fused.cu) reaches the minimum.
#include "fdtd_cell.cuh"
#include "fdtd_launch.h"

namespace fdtd {

__global__ void k_advance(int* t, int n) { *t += n; }

template <class T>
__global__ void __launch_bounds__(256) k_h_split(State<T> s, const int* __restrict__ tp, int toff) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= s.nx || y >= s.ny) return;
  const int t = *tp + toff;
  const bool box = in_box(s, z, y, x);
  if (!box && !injects(s, z, t)) return;
  const long long i = (long long)z * s.plane + (long long)y * s.pitch + x;
  ENbr<T> e;
  if (box) {
    e.ex0 = s.iex[i]; e.exz = s.iex[i + s.plane]; e.exy = s.iex[i + s.pitch];
    e.ey0 = s.iey[i]; e.eyz = s.iey[i + s.plane]; e.eyx = s.iey[i + 1];
    e.ez0 = s.iez[i]; e.ezy = s.iez[i + s.pitch]; e.ezx = s.iez[i + 1];
  } else {
    e = ENbr<T>{};
  }
  T hx = s.ihx[i], hy = s.ihy[i], hz = s.ihz[i];
  h_cell(s, e, z, y, x, t, true, hx, hy, hz);
  s.ohx[i] = hx; s.ohy[i] = hy; s.ohz[i] = hz;
}

template <class T>
__global__ void __launch_bounds__(256) k_e_split(State<T> s, const int* __restrict__ tp, int toff) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= s.nx || y >= s.ny) return;
  const int t = *tp + toff;
  const bool box = in_box(s, z, y, x);
  if (!box && !injects(s, z, t)) return;
  const long long i = (long long)z * s.plane + (long long)y * s.pitch + x;
  HNbr<T> h = HNbr<T>{};
  T ca = T(0), cb = T(0);
  if (box) {
    h.hx0 = s.ihx[i]; h.hy0 = s.ihy[i]; h.hz0 = s.ihz[i];
    if (z >= 1) { h.hxz = s.ihx[i - s.plane]; h.hyz = s.ihy[i - s.plane]; }
    if (y >= 1) { h.hxy = s.ihx[i - s.pitch]; h.hzy = s.ihz[i - s.pitch]; }
    if (x >= 1) { h.hyx = s.ihy[i - 1]; h.hzx = s.ihz[i - 1]; }
    ca = s.ca[i]; cb = s.cb[i];
  }
  T ex = s.iex[i], ey = s.iey[i], ez = s.iez[i];
  e_cell(s, h, ca, cb, z, y, x, t, true, ex, ey, ez);
  s.oex[i] = ex; s.oey[i] = ey; s.oez[i] = ez;
}

// ---------------------------------------------------------------------------
// phasors (cpu/field_updates.py:373-461, gpu/field_updates.py:680-906)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void ph_acc(const State<T>& s, int plane, long long k,
                                       double m, double c, double sn) {
  using M = R<T>;
  T* p = s.ph + s.ph_off[plane] + 2 * k;
  if (!s.kahan) {
    // float64 sum of the stored value and the float64 term, rounded to T
    p[0] = M::from_double(__dadd_rn((double)p[0], __dmul_rn(m, c)));
    p[1] = M::from_double(__dadd_rn((double)p[1], __dmul_rn(m, sn)));
  } else {
    T* pc = s.phc + s.ph_off[plane] + 2 * k;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const T term = M::from_double(__dmul_rn(m, j ? sn : c));
      const T yv = M::sub(term, pc[j]);
      const T tv = M::add(p[j], yv);
      pc[j] = M::sub(M::sub(tv, p[j]), yv);
      p[j] = tv;
    }
  }
}

template <class T>
__device__ __forceinline__ double mean2(T a, T b) {
  return 0.5 * (double)R<T>::add(a, b);
}
template <class T>
__device__ __forceinline__ double mean4(T a, T b, T c, T d) {
  using M = R<T>;
  return 0.25 * (double)M::add(M::add(M::add(a, b), c), d);
}

// One thread per phasor cell; blockIdx.y selects the plane pair member
// 0 d, 1 u (z planes), 2 l, 3 r (x planes), 4 f, 5 b (y planes).
template <class T>
__global__ void __launch_bounds__(256) k_phasors(State<T> s, const int* __restrict__ tp, int toff) {
  const int g = blockIdx.y;
  const int m = s.npml;
  int d0, d1;
  if (g < 2) { d0 = s.ny_ph; d1 = s.nx_ph; }
  else if (g < 4) { d0 = s.nz_ph; d1 = s.ny_ph; }
  else { d0 = s.nz_ph; d1 = s.nx_ph; }
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= d0 * d1) return;
  const int a = idx / d1, b = idx - a * d1;
  if (a == 0 || b == 0) return;
  const int t = *tp + toff;
  const double* ph = s.phase + 4 * (long long)t;
  const double cE = ph[0], sE = ph[1], cH = ph[2], sH = ph[3];
  const T* ex = s.oex; const T* ey = s.oey; const T* ez = s.oez;
  const T* hx = s.ohx; const T* hy = s.ohy; const T* hz = s.ohz;
  const long long P = s.plane, W = s.pitch;
  const long long k = (long long)a * d1 + b;
  if (g < 2) {
    const int pz = g == 0 ? m + 1 : s.nz - m - 1;
    const long long i = pz * P + (long long)(m + a) * W + (m + b);
    const int base = g * 4;  // ex, ey, hx, hy
    ph_acc(s, base + 0, k, mean2(ex[i], ex[i - 1]), cE, sE);
    ph_acc(s, base + 1, k, mean2(ey[i], ey[i - W]), cE, sE);
    ph_acc(s, base + 2, k, mean4(hx[i], hx[i - W], hx[i - P], hx[i - P - W]), cH, sH);
    ph_acc(s, base + 3, k, mean4(hy[i], hy[i - 1], hy[i - P], hy[i - P - 1]), cH, sH);
  } else if (g < 4) {
    const int px = g == 2 ? m + 1 : s.nx - m - 1;
    const long long i = (long long)(m + a) * P + (long long)(m + b) * W + px;
    const int base = 8 + (g - 2) * 4;  // ey, ez, hy, hz
    ph_acc(s, base + 0, k, mean2(ey[i], ey[i - W]), cE, sE);
    ph_acc(s, base + 1, k, mean2(ez[i], ez[i - P]), cE, sE);
    ph_acc(s, base + 2, k, mean4(hy[i], hy[i - 1], hy[i - P], hy[i - P - 1]), cH, sH);
    ph_acc(s, base + 3, k, mean4(hz[i], hz[i - 1], hz[i - W], hz[i - W - 1]), cH, sH);
  } else {
    const int py = g == 4 ? m + 1 : s.ny - m - 1;
    const long long i = (long long)(m + a) * P + (long long)py * W + (m + b);
    const int base = 16 + (g - 4) * 4;  // ex, ez, hx, hz
    ph_acc(s, base + 0, k, mean2(ex[i], ex[i - 1]), cE, sE);
    ph_acc(s, base + 1, k, mean2(ez[i], ez[i - P]), cE, sE);
    ph_acc(s, base + 2, k, mean4(hx[i], hx[i - W], hx[i - P], hx[i - P - W]), cH, sH);
    ph_acc(s, base + 3, k, mean4(hz[i], hz[i - W], hz[i - 1], hz[i - W - 1]), cH, sH);
  }
}

// ---------------------------------------------------------------------------
// Ca, Cb from eps_r, sigma (materials/materials.py:23-68). The reference
// evaluates every operation in the array dtype: eps0, dt and dx are first
// rounded to it (numpy scalar promotion), then
//   perm = eps_r * eps0; x = (sigma * dt) / (2 * perm)
//   Ca = (1 - x) / (1 + x);  Cb = (dt / (perm * dx)) / (1 + x)
// Cells at z >= nz_mat are vacuum (eps_r = 1, sigma = 0).
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_eps_sigma(int nx, int ny, int nz, int nz_mat, int pitch,
                            const T* __restrict__ eps, const T* __restrict__ sig,
                            T eps0, T dt, T dx, T* __restrict__ ca, T* __restrict__ cb) {
  using M = R<T>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int z = blockIdx.z;
  if (x >= nx) return;
  T e = T(1), sg = T(0);
  if (z < nz_mat) {
    const long long j = ((long long)z * ny + y) * nx + x;
    e = eps[j];
    sg = sig[j];
  }
  const T perm = M::mul(e, eps0);
  const T xx = M::div(M::mul(sg, dt), M::mul(T(2), perm));
  const T den = M::add(T(1), xx);
  const long long i = ((long long)z * ny + y) * pitch + x;
  ca[i] = M::div(M::sub(T(1), xx), den);
  cb[i] = M::div(M::div(dt, M::mul(perm, dx)), den);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <class T>
void launch_split_step(const State<T>& s, const int* tdev, int toff, cudaStream_t st) {
  const dim3 blk(64, 4, 1);
  const dim3 grd((s.nx + 63) / 64, (s.ny + 3) / 4, s.nz);
  k_h_split<T><<<grd, blk, 0, st>>>(s, tdev, toff);
  k_e_split<T><<<grd, blk, 0, st>>>(s, tdev, toff);
}

template <class T>
void launch_phasors(const State<T>& s, const int* tdev, int toff, cudaStream_t st) {
  int n = s.ny_ph * s.nx_ph;
  n = max(n, s.nz_ph * s.ny_ph);
  n = max(n, s.nz_ph * s.nx_ph);
  const dim3 grd((n + 255) / 256, 6, 1);
  k_phasors<T><<<grd, 256, 0, st>>>(s, tdev, toff);
}

void launch_advance(int* tdev, int n, cudaStream_t st) {
  k_advance<<<1, 1, 0, st>>>(tdev, n);
}

template <class T>
void launch_eps_sigma(int nx, int ny, int nz, int nz_mat, int pitch, const T* eps,
                      const T* sig, T eps0, T dt, T dx, T* ca, T* cb, cudaStream_t st) {
  const dim3 grd((nx + 127) / 128, ny, nz);
  k_eps_sigma<T><<<grd, 128, 0, st>>>(nx, ny, nz, nz_mat, pitch, eps, sig, eps0, dt, dx, ca, cb);
}

template void launch_split_step<float>(const State<float>&, const int*, int, cudaStream_t);
template void launch_split_step<double>(const State<double>&, const int*, int, cudaStream_t);
template void launch_phasors<float>(const State<float>&, const int*, int, cudaStream_t);
template void launch_phasors<double>(const State<double>&, const int*, int, cudaStream_t);
template void launch_eps_sigma<float>(int, int, int, int, int, const float*, const float*, float,
                                      float, float, float*, float*, cudaStream_t);
template void launch_eps_sigma<double>(int, int, int, int, int, const double*, const double*,
                                       double, double, double, double*, double*, cudaStream_t);

}  // namespace fdtd
