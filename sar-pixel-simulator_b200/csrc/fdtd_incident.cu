// fdtd_incident.cu -- the incident beam on the device: the excitation fed
// into the incident simulation, and the per-step kernels of that vacuum run.
//
// Excitation (incidentbeam.py:174-298). For every temporal frequency bin k
// of the pulse spectrum P[k], the tapered wave of Braunisch ("Tapered Wave
// with a Least Squared Error Property", incidentbeam.py:317-433) is
// evaluated on the lateral spatial-frequency grid, weighted by P[k] and
// transformed to space by a 2-D FFT; an inverse FFT along the bins then
// gives the time signal of every lateral cell, normalised to a peak
// magnitude of 10. The reference stores the weighted spectra in the
// simulation's complex type; here every stage is float64 (complex128), and
// only the imaginary parts that the simulation injects are rounded to the
// element type at the end. The FFTs are cuFFT's (a library transform, like
// a library GEMM); the taper, the peak and the extraction are the kernels
// below. The reference's fftshift / ifftshift pairs become index maps: the
// taper writes bin (j, i) at the natural-order frequencies
// (fftfreq(n)[i], fftfreq(n)[j]) the FFT expects, and the extraction reads
// lateral cell (j, i) from (j - ny/2, i - nx/2) mod (ny, nx).
//
// Incident run (cpu/incident_sim.py:67-171): the E pass, the hard source on
// plane feed_in, the H pass (the split passes of the main step, without
// injection), then k_inc_record copies the read-out plane and accumulates the
// incident phasors (cpu/field_updates.py:465-491).
#include <algorithm>
#include <cstdio>
#include <cstring>

#include <cufft.h>

#include "fdtd_b200.h"
#include "fdtd_launch.h"

namespace fdtd {

namespace {

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 rmul(double a, double2 b) { return make_double2(a * b.x, a * b.y); }

// natural-order FFT frequency index of bin i of n (numpy.fft.fftfreq)
__device__ __forceinline__ int fft_index(int i, int n) { return i < (n + 1) / 2 ? i : i - n; }

// One spectrum bin (kt, j, i) of both components, weighted by the pulse
// spectrum. Equation numbers are Braunisch's, as in incidentbeam.py.
__global__ void __launch_bounds__(256) k_inc_taper(IncidentTaper p, const double* __restrict__ kv,
                                                   const double2* __restrict__ pfft,
                                                   double2* __restrict__ sx, double2* __restrict__ sy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, kt = blockIdx.z;
  if (i >= p.nx) return;
  const long long o = ((long long)kt * p.ny + j) * p.nx + i;
  const double k = kv[kt];
  if (k == 0.0) {
    sx[o] = make_double2(0.0, 0.0);
    sy[o] = make_double2(0.0, 0.0);
    return;
  }
  const double two_pi = 6.283185307179586;
  const double kx = two_pi * ((double)fft_index(i, p.nx) * p.dfx);
  const double ky = two_pi * ((double)fft_index(j, p.ny) * p.dfy);
  const double kp = hypot(kx, ky);                                   // Eqn 4
  // Eqn 5, evaluated in complex64 by the reference: the conjugate root
  const float v = __double2float_rn(k * k - kp * kp);
  const double2 kz = v >= 0.0f ? make_double2((double)sqrtf(v), -0.0)
                               : make_double2(0.0, -(double)sqrtf(-v));
  const double kix = (k * p.sin_theta) * p.cos_phi, kiy = (k * p.sin_theta) * p.sin_phi;
  const double kip = hypot(kix, kiy), kiz = sqrt(k * k - kip * kip);
  const double dkx = kx - kix, dky = ky - kiy;
  const double gauss = p.r2_4pi * exp((-p.r2 * (dkx * dkx + dky * dky)) / 4.0);   // Eqn 13
  double hx, hy, vz;                                                  // Eqns 10, 11
  double2 vx, vy;
  if (kp > 0.0) {
    hx = ky / kp;
    hy = -kx / kp;
    const double d = k * kp;
    vx = make_double2(kz.x * kx / d, kz.y * kx / d);
    vy = make_double2(kz.x * ky / d, kz.y * ky / d);
    vz = kp / k;
  } else {
    hx = p.sin_phi;
    hy = -p.cos_phi;
    vx = make_double2(p.cos_phi, 0.0);
    vy = make_double2(p.sin_phi, 0.0);
    vz = 0.0;
  }
  double hix, hiy, vix, viy, viz;                                     // the central plane wave
  if (kip > 0.0) {
    hix = kiy / kip;
    hiy = -kix / kip;
    vix = (kiz * kix) / (k * kip);
    viy = (kiz * kiy) / (k * kip);
    viz = kip / k;
  } else {
    hix = p.sin_phi;
    hiy = -p.cos_phi;
    vix = p.cos_phi;
    viy = p.sin_phi;
    viz = 0.0;
  }
  // Eqns 14-16: polarisation weights
  const double2 eh = cadd(rmul((hix * hx) + (hiy * hy), p.eh), rmul((vix * hx) + (viy * hy), p.ev));
  const double2 ev = cadd(cmul(p.eh, cadd(rmul(hix, vx), rmul(hiy, vy))),
                          cmul(p.ev, cadd(cadd(rmul(vix, vx), rmul(viy, vy)), make_double2(viz * vz, 0.0))));
  // Eqns 8, 1: spectral components, times the pulse spectrum
  const double2 xc = rmul(gauss, cadd(rmul(hx, eh), cmul(ev, vx)));
  const double2 yc = rmul(gauss, cadd(rmul(hy, eh), cmul(ev, vy)));
  const double2 w = pfft[kt];
  sx[o] = cmul(w, xc);
  sy[o] = cmul(w, yc);
}

// Largest magnitude over n complex values of both arrays, as the bit
// pattern of a non-negative double (which orders like the value).
__global__ void __launch_bounds__(256) k_inc_absmax(const double2* __restrict__ a,
                                                    const double2* __restrict__ b, long long n,
                                                    unsigned long long* __restrict__ out) {
  double m = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    m = fmax(m, fmax(hypot(a[i].x, a[i].y), hypot(b[i].x, b[i].y)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  __shared__ double wm[8];
  if ((threadIdx.x & 31) == 0) wm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wm[w]);
    atomicMax(out, (unsigned long long)__double_as_longlong(m));
  }
}

// exc[t, y, x] = Im(signal at lateral cell (y, x)) * 10 / peak, t < nt_pulse.
// The inverse FFT leaves the signal times nt; the peak carries the same
// factor, so the ratio is the reference's normalised value.
template <class T>
__global__ void __launch_bounds__(256) k_inc_extract(const double2* __restrict__ sx,
                                                     const double2* __restrict__ sy, int nx, int ny,
                                                     int pitch, const unsigned long long* __restrict__ peak,
                                                     T* __restrict__ ex, T* __restrict__ ey) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y, t = blockIdx.z;
  if (i >= nx) return;
  const double scale = 10.0 / __longlong_as_double((long long)*peak);
  const int js = (j - ny / 2 + ny) % ny, is = (i - nx / 2 + nx) % nx;
  const long long src = ((long long)t * ny + js) * nx + is;
  const long long dst = ((long long)t * ny + j) * pitch + i;
  ex[dst] = (T)(sx[src].y * scale);
  ey[dst] = (T)(sy[src].y * scale);
}

// Hard source of step t: ex, ey on plane feed_in, y in [1, ny-1),
// x in [0, nx-1), overwritten by the excitation (cpu/incident_sim.py:141-144).
template <class T>
__global__ void __launch_bounds__(256) k_inc_source(T* __restrict__ ex, T* __restrict__ ey,
                                                    const T* __restrict__ sx, const T* __restrict__ sy,
                                                    int nx, int ny, int pitch, long long plane, int feed_in,
                                                    int t) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= nx - 1 || y < 1 || y >= ny - 1) return;
  const long long src = ((long long)t * ny + y) * pitch + x;
  const long long dst = (long long)feed_in * plane + (long long)y * pitch + x;
  ex[dst] = sx[src];
  ey[dst] = sy[src];
}

template <class T>
__device__ __forceinline__ void inc_acc(T* p, double m, double c, double sn) {
  // float64 sum of the stored value and the float64 term, rounded to T
  p[0] = R<T>::from_double(__dadd_rn((double)p[0], __dmul_rn(m, c)));
  p[1] = R<T>::from_double(__dadd_rn((double)p[1], __dmul_rn(m, sn)));
}

// Read-out plane of step t into the recorded planes (all y, x) and the
// incident phasors of cpu/field_updates.py:465-491 at (y, x) in
// [1, ny_ph) x [1, nx_ph): E averaged with phase exp(-i omega (t - 1/2) dt),
// H with exp(-i omega t dt) (phase table columns 2-3 and 0-1).
template <class T>
__global__ void __launch_bounds__(256) k_inc_record(IncidentRecord<T> r, int t) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= r.nx) return;
  const long long P = r.plane, W = r.pitch;
  const long long i = (long long)r.read_out * P + (long long)y * W + x;
  const long long o = ((long long)t * r.ny + y) * W + x;
  r.rex[o] = r.ex[i];
  r.rey[o] = r.ey[i];
  r.rhx[o] = r.hx[i];
  r.rhy[o] = r.hy[i];
  const int a = y - r.npml, b = x - r.npml;
  if (a < 1 || b < 1 || a >= r.ny_ph || b >= r.nx_ph) return;
  const double* ph = r.phase + 4 * (long long)t;
  const double cH = ph[0], sH = ph[1], cE = ph[2], sE = ph[3];
  using M = R<T>;
  const long long k = 2 * ((long long)a * r.nx_ph + b), n = 2 * (long long)r.ny_ph * r.nx_ph;
  inc_acc(r.ph + k, 0.5 * (double)M::add(r.ex[i], r.ex[i - 1]), cE, sE);
  inc_acc(r.ph + n + k, 0.5 * (double)M::add(r.ey[i], r.ey[i - W]), cE, sE);
  inc_acc(r.ph + 2 * n + k,
          0.25 * (double)M::add(M::add(M::add(r.hx[i], r.hx[i - W]), r.hx[i - P]), r.hx[i - P - W]), cH, sH);
  inc_acc(r.ph + 3 * n + k,
          0.25 * (double)M::add(M::add(M::add(r.hy[i], r.hy[i - 1]), r.hy[i - P]), r.hy[i - P - 1]), cH, sH);
}

template <class T>
__global__ void k_fill(T* __restrict__ p, long long n, T v) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = v;
}

const char* cufft_name(cufftResult r) {
  switch (r) {
    case CUFFT_SUCCESS: return "success";
    case CUFFT_INVALID_PLAN: return "invalid plan";
    case CUFFT_ALLOC_FAILED: return "allocation failed";
    case CUFFT_INVALID_VALUE: return "invalid value";
    case CUFFT_INTERNAL_ERROR: return "internal error";
    case CUFFT_EXEC_FAILED: return "exec failed";
    case CUFFT_SETUP_FAILED: return "setup failed";
    case CUFFT_INVALID_SIZE: return "invalid size";
    default: return "error";
  }
}

}  // namespace

template <class T>
int make_incident_excitation(const IncidentTaper& p, const double* k_host, const double* pfft_host,
                             int nt_pulse, int pitch, T* ex, T* ey, double* peak_out, cudaStream_t st) {
  const long long n = (long long)p.nt * p.ny * p.nx;
  char msg[256];
  double2* sx = nullptr;
  double2* sy = nullptr;
  double* kv = nullptr;
  double2* pf = nullptr;
  unsigned long long* peak = nullptr;
  int rc = 0;
  auto cuda_fail = [&](const char* what, cudaError_t e) {
    snprintf(msg, sizeof(msg), "incident excitation: %s: %s", what, cudaGetErrorString(e));
    cudaGetLastError();
    rc = report_error(e == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA, msg);
  };
  auto fft_fail = [&](const char* what, cufftResult r) {
    snprintf(msg, sizeof(msg), "incident excitation: %s: cuFFT %s", what, cufft_name(r));
    rc = report_error(r == CUFFT_ALLOC_FAILED ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA, msg);
  };
  cudaError_t e;
  if ((e = cudaMalloc(&sx, n * sizeof(double2))) != cudaSuccess) cuda_fail("spectrum x", e);
  if (!rc && (e = cudaMalloc(&sy, n * sizeof(double2))) != cudaSuccess) cuda_fail("spectrum y", e);
  if (!rc && (e = cudaMalloc(&kv, p.nt * sizeof(double))) != cudaSuccess) cuda_fail("wavenumbers", e);
  if (!rc && (e = cudaMalloc(&pf, p.nt * sizeof(double2))) != cudaSuccess) cuda_fail("pulse spectrum", e);
  if (!rc && (e = cudaMalloc(&peak, sizeof(unsigned long long))) != cudaSuccess) cuda_fail("peak", e);
  if (!rc && (e = cudaMemcpyAsync(kv, k_host, p.nt * sizeof(double), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    cuda_fail("upload", e);
  if (!rc && (e = cudaMemcpyAsync(pf, pfft_host, p.nt * sizeof(double2), cudaMemcpyHostToDevice, st)) != cudaSuccess)
    cuda_fail("upload", e);
  if (!rc && (e = cudaMemsetAsync(peak, 0, sizeof(unsigned long long), st)) != cudaSuccess) cuda_fail("memset", e);
  if (!rc) {
    k_inc_taper<<<dim3((p.nx + 255) / 256, p.ny, p.nt), 256, 0, st>>>(p, kv, pf, sx, sy);
    if ((e = cudaGetLastError()) != cudaSuccess) cuda_fail("taper", e);
  }
  // Transforms in place, in batches that bound cuFFT's work area: 2-D
  // forward transforms of kBins2d bins at a time, then inverse transforms
  // along the bins (stride ny*nx) of kCells1d lateral cells at a time.
  const int kBins2d = 32, kCells1d = 1 << 16;
  auto run_batches = [&](int rank, int* dims, int* embed, int stride, int dist, int total, int per, int dir,
                         long long step, const char* what) {
    cufftHandle plans[2] = {0, 0};
    bool made[2] = {false, false};
    const int full = std::min(per, total), rest = total % full;
    const int counts[2] = {full, rest};
    for (int k = 0; k < 2 && !rc; ++k) {
      if (counts[k] == 0) continue;
      cufftResult r = cufftPlanMany(&plans[k], rank, dims, embed, stride, dist, embed, stride, dist, CUFFT_Z2Z,
                                    counts[k]);
      if (r != CUFFT_SUCCESS) { fft_fail(what, r); break; }
      made[k] = true;
      if ((r = cufftSetStream(plans[k], st)) != CUFFT_SUCCESS) fft_fail(what, r);
    }
    for (double2* a : {sx, sy}) {
      for (int b = 0; b < total && !rc; b += full) {
        const int k = (total - b < full) ? 1 : 0;
        cufftDoubleComplex* q = (cufftDoubleComplex*)(a + (long long)b * step);
        const cufftResult r = cufftExecZ2Z(plans[k], q, q, dir);
        if (r != CUFFT_SUCCESS) fft_fail(what, r);
      }
    }
    for (int k = 0; k < 2; ++k)
      if (made[k]) cufftDestroy(plans[k]);
  };
  if (!rc) {
    int dims[2] = {p.ny, p.nx};
    run_batches(2, dims, nullptr, 1, 0, p.nt, kBins2d, CUFFT_FORWARD, (long long)p.ny * p.nx, "2-D forward");
  }
  if (!rc) {
    int len[1] = {p.nt};
    run_batches(1, len, len, p.ny * p.nx, 1, p.ny * p.nx, kCells1d, CUFFT_INVERSE, 1, "time inverse");
  }
  if (!rc) {
    k_inc_absmax<<<4 * 148, 256, 0, st>>>(sx, sy, n, peak);
    if (nt_pulse > 0)
      k_inc_extract<T><<<dim3((p.nx + 255) / 256, p.ny, nt_pulse), 256, 0, st>>>(sx, sy, p.nx, p.ny, pitch, peak,
                                                                                 ex, ey);
    if ((e = cudaGetLastError()) != cudaSuccess) cuda_fail("extract", e);
  }
  unsigned long long bits = 0;
  if (!rc && (e = cudaMemcpyAsync(&bits, peak, sizeof(bits), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
    cuda_fail("peak readback", e);
  if (!rc && (e = cudaStreamSynchronize(st)) != cudaSuccess) cuda_fail("excitation", e);
  if (!rc && peak_out) {
    double v;
    memcpy(&v, &bits, sizeof(v));
    *peak_out = v / (double)p.nt;   // the peak of the normalised inverse transform
  }
  cudaStreamSynchronize(st);
  for (void* q : {(void*)sx, (void*)sy, (void*)kv, (void*)pf, (void*)peak})
    if (q) cudaFree(q);
  return rc;
}

template <class T>
void launch_inc_source(T* ex, T* ey, const T* sx, const T* sy, int nx, int ny, int pitch, long long plane,
                       int feed_in, int t, cudaStream_t st) {
  k_inc_source<T><<<dim3((nx + 255) / 256, ny, 1), 256, 0, st>>>(ex, ey, sx, sy, nx, ny, pitch, plane, feed_in, t);
}

template <class T>
void launch_inc_record(const IncidentRecord<T>& r, int t, cudaStream_t st) {
  k_inc_record<T><<<dim3((r.nx + 255) / 256, r.ny, 1), 256, 0, st>>>(r, t);
}

template <class T>
void launch_fill(T* p, long long n, T v, cudaStream_t st) {
  k_fill<T><<<4 * 148, 256, 0, st>>>(p, n, v);
}

template int make_incident_excitation<float>(const IncidentTaper&, const double*, const double*, int, int,
                                             float*, float*, double*, cudaStream_t);
template int make_incident_excitation<double>(const IncidentTaper&, const double*, const double*, int, int,
                                              double*, double*, double*, cudaStream_t);
template void launch_inc_source<float>(float*, float*, const float*, const float*, int, int, int, long long,
                                       int, int, cudaStream_t);
template void launch_inc_source<double>(double*, double*, const double*, const double*, int, int, int,
                                        long long, int, int, cudaStream_t);
template void launch_inc_record<float>(const IncidentRecord<float>&, int, cudaStream_t);
template void launch_inc_record<double>(const IncidentRecord<double>&, int, cudaStream_t);
template void launch_fill<float>(float*, long long, float, cudaStream_t);
template void launch_fill<double>(double*, long long, double, cudaStream_t);

}  // namespace fdtd
