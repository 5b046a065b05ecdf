// near2far.cu -- near-to-far transform of the top phasor plane.
//
// Restates FarFieldTransform (fdtdsarsim/near2far.py:28-156) on the device:
// surface currents J = (-Hy, Hx) and M = (Ey, -Ex) on the plane z = z_val
// are integrated against exp(j k r_hat . r') with composite Simpson weights
// (scipy.integrate.simpson on an odd sample count, x first then y), giving
// the N and L potentials, then E/H theta/phi at radius r.
//
// One thread block per (theta, phi); each thread strides over the plane,
// accumulating the four complex potentials in float64 registers; a
// warp-shuffle + shared-memory tree reduces them. All arithmetic is float64,
// as in the reference (complex128, near2far.py:66-68).
#include <cuda_runtime.h>

#include "fdtd_launch.h"

namespace fdtd {

namespace {

constexpr int kN2fThreads = 256;

__device__ __forceinline__ double simpson_w(int i, int n) {
  if (i == 0 || i == n - 1) return 1.0;
  return (i & 1) ? 4.0 : 2.0;
}

__global__ void __launch_bounds__(kN2fThreads)
k_near2far(const double2* __restrict__ jx, const double2* __restrict__ jy,
           const double2* __restrict__ mx, const double2* __restrict__ my, int nx, int ny,
           double dx, double z_val, double k, const double* __restrict__ thetas,
           const double* __restrict__ phis, int ntheta, int nphi, double r,
           double2* __restrict__ out) {
  const int it = blockIdx.x, ip = blockIdx.y;
  const double th = thetas[it], ph = phis[ip];
  const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
  // x_loc = np.arange(-(nx-1)//2, (nx-1)//2 + 1) * dx  (near2far.py:58-60)
  const int hx = nx / 2, hy = ny / 2;
  // accumulators: N_theta, N_phi, L_theta, L_phi (re, im)
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const int n = nx * ny;
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int y = idx / nx, x = idx - y * nx;
    const double xl = (double)(x - hx) * dx;
    const double yl = (double)(y - hy) * dx;
    // exp_term argument as near2far.py:140-143 evaluates it
    const double arg = k * (((xl * st) * cp + (yl * st) * sp) + z_val * ct);
    double es, ec;
    sincos(arg, &es, &ec);
    const double w = simpson_w(x, nx) * simpson_w(y, ny);
    const double2 Jx = jx[idx], Jy = jy[idx], Mx = mx[idx], My = my[idx];
    // integrands of Taflove 8.33a/b and 8.34a/b before the exponential
    const double ntr = Jx.x * ct * cp + Jy.x * ct * sp, nti = Jx.y * ct * cp + Jy.y * ct * sp;
    const double npr = -Jx.x * sp + Jy.x * cp, npi = -Jx.y * sp + Jy.y * cp;
    const double ltr = Mx.x * ct * cp + My.x * ct * sp, lti = Mx.y * ct * cp + My.y * ct * sp;
    const double lpr = -Mx.x * sp + My.x * cp, lpi = -Mx.y * sp + My.y * cp;
    acc[0] += w * (ntr * ec - nti * es); acc[1] += w * (ntr * es + nti * ec);
    acc[2] += w * (npr * ec - npi * es); acc[3] += w * (npr * es + npi * ec);
    acc[4] += w * (ltr * ec - lti * es); acc[5] += w * (ltr * es + lti * ec);
    acc[6] += w * (lpr * ec - lpi * es); acc[7] += w * (lpr * es + lpi * ec);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_down_sync(0xffffffffu, acc[j], o);
  __shared__ double red[kN2fThreads / 32][8];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (lane == 0)
    for (int j = 0; j < 8; ++j) red[warp][j] = acc[j];
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int w = 0; w < kN2fThreads / 32; ++w)
      for (int j = 0; j < 8; ++j) s[j] += red[w][j];
    const double h = dx / 3.0;  // Simpson factor per axis
    for (int j = 0; j < 8; ++j) s[j] *= h * h;
    const double eta0 = 376.730313668;
    // ff_weight = 1j k exp(-1j k r) / (4 pi r)   (near2far.py:71-72)
    const double c = k / (4.0 * M_PI * r);
    double sr, cr;
    sincos(k * r, &sr, &cr);
    const double2 ffw = make_double2(c * sr, c * cr);  // 1j*c*(cos - j sin)
    const double2 Nt = make_double2(s[0], s[1]), Np = make_double2(s[2], s[3]);
    const double2 Lt = make_double2(s[4], s[5]), Lp = make_double2(s[6], s[7]);
    auto cm = [](double2 a, double2 b) {
      return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    };
    const double2 et = cm(ffw, make_double2(-Lp.x - eta0 * Nt.x, -Lp.y - eta0 * Nt.y));
    const double2 ep = cm(ffw, make_double2(Lt.x - eta0 * Np.x, Lt.y - eta0 * Np.y));
    const double2 ht = cm(ffw, make_double2(Np.x - Lt.x / eta0, Np.y - Lt.y / eta0));
    const double2 hp = cm(ffw, make_double2(-Nt.x - Lp.x / eta0, -Nt.y - Lp.y / eta0));
    const long long plane = (long long)nphi * ntheta;
    const long long o = (long long)ip * ntheta + it;
    out[0 * plane + o] = et;
    out[1 * plane + o] = ep;
    out[2 * plane + o] = ht;
    out[3 * plane + o] = hp;
  }
}

}  // namespace

int near2far_run(const double* jm, int nx, int ny, double dx, double z_val, double k,
                 const double* thetas, int ntheta, const double* phis, int nphi, double r,
                 double* out, cudaStream_t st) {
  const double2* base = reinterpret_cast<const double2*>(jm);
  const long long n = (long long)nx * ny;
  const dim3 grd(ntheta, nphi, 1);
  k_near2far<<<grd, kN2fThreads, 0, st>>>(base, base + n, base + 2 * n, base + 3 * n, nx, ny, dx,
                                          z_val, k, thetas, phis, ntheta, nphi, r,
                                          reinterpret_cast<double2*>(out));
  return cudaGetLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace fdtd

// ---------------------------------------------------------------------------
// Allocation-free variant of fdtd_near2far.
//
// Some callers cannot allocate device memory at the moment they need a far
// field: code running under a memory manager that owns every byte of the
// device (a caching pool or a reserved arena), callers that must not grow
// the footprint of a running job, or contexts where device allocation is
// forbidden or would synchronize the device. fdtd_near2far_noalloc does the
// same work as fdtd_near2far but stages its inputs, angles and results in
// one statically sized device array, kN2fScratchBytes, which every GPU that
// loads this library holds until the process exits. The caller still passes
// host inputs and a host output buffer; nothing is allocated per call.
// ---------------------------------------------------------------------------
#include <cstdio>
#include <mutex>

#include "fdtd_b200.h"

namespace fdtd {

namespace {

// Largest plane (nx_ph * ny_ph cells, complex128 inputs; twice as many for
// complex64) and angle set the static scratch can hold.
constexpr long long kN2fMaxCells = 600000;       // covers a 761 x 761 grid's 741 x 741 plane
constexpr int kN2fMaxTheta = 4096;
constexpr int kN2fMaxPhi = 64;
constexpr int kN2fMaxAngles = 8192;              // nphi * ntheta
constexpr size_t kN2fPlaneBytes = (size_t)4 * kN2fMaxCells * 16;
constexpr size_t kN2fAngleBytes = (size_t)(kN2fMaxTheta + kN2fMaxPhi) * 8;
constexpr size_t kN2fOutBytes = (size_t)kN2fMaxAngles * 4 * 16;
constexpr size_t kN2fScratchBytes = kN2fPlaneBytes + kN2fAngleBytes + kN2fOutBytes;

// Layout: [4 input planes as given][thetas (deg)][phis (deg)][output]
static __device__ __align__(256) unsigned char g_n2f_scratch[kN2fScratchBytes];

std::mutex g_n2f_mutex;
void* g_n2f_addr[64] = {};   // device address of g_n2f_scratch, per device

// Same integration as k_near2far, reading the u-plane phasors as given
// (complex64 or complex128), forming J = (-Hy, Hx), M = (Ey, -Ex) on the fly
// and converting the angles from degrees on the device.
template <class C>
__global__ void __launch_bounds__(kN2fThreads)
k_near2far_raw(unsigned char* __restrict__ scratch, long long plane_bytes, int nx, int ny,
               double dx, double z_val, double k, int ntheta, int nphi, double r) {
  const C* ex_u = reinterpret_cast<const C*>(scratch);
  const long long n = (long long)nx * ny;
  const C* ey_u = ex_u + n;
  const C* hx_u = ey_u + n;
  const C* hy_u = hx_u + n;
  const double* thetas = reinterpret_cast<const double*>(scratch + plane_bytes);
  const double* phis = thetas + ntheta;
  double2* out = reinterpret_cast<double2*>(scratch + plane_bytes + kN2fAngleBytes);
  const int it = blockIdx.x, ip = blockIdx.y;
  const double th = thetas[it] * (M_PI / 180.0), ph = phis[ip] * (M_PI / 180.0);
  const double st = sin(th), ct = cos(th), sp = sin(ph), cp = cos(ph);
  const int hx = nx / 2, hy = ny / 2;
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int idx = threadIdx.x; idx < n; idx += blockDim.x) {
    const int y = idx / nx, x = idx - y * nx;
    const double xl = (double)(x - hx) * dx;
    const double yl = (double)(y - hy) * dx;
    const double arg = k * (((xl * st) * cp + (yl * st) * sp) + z_val * ct);
    double es, ec;
    sincos(arg, &es, &ec);
    const double w = simpson_w(x, nx) * simpson_w(y, ny);
    const double2 Jx = make_double2(-(double)hy_u[idx].x, -(double)hy_u[idx].y);
    const double2 Jy = make_double2((double)hx_u[idx].x, (double)hx_u[idx].y);
    const double2 Mx = make_double2((double)ey_u[idx].x, (double)ey_u[idx].y);
    const double2 My = make_double2(-(double)ex_u[idx].x, -(double)ex_u[idx].y);
    const double ntr = Jx.x * ct * cp + Jy.x * ct * sp, nti = Jx.y * ct * cp + Jy.y * ct * sp;
    const double npr = -Jx.x * sp + Jy.x * cp, npi = -Jx.y * sp + Jy.y * cp;
    const double ltr = Mx.x * ct * cp + My.x * ct * sp, lti = Mx.y * ct * cp + My.y * ct * sp;
    const double lpr = -Mx.x * sp + My.x * cp, lpi = -Mx.y * sp + My.y * cp;
    acc[0] += w * (ntr * ec - nti * es); acc[1] += w * (ntr * es + nti * ec);
    acc[2] += w * (npr * ec - npi * es); acc[3] += w * (npr * es + npi * ec);
    acc[4] += w * (ltr * ec - lti * es); acc[5] += w * (ltr * es + lti * ec);
    acc[6] += w * (lpr * ec - lpi * es); acc[7] += w * (lpr * es + lpi * ec);
  }
#pragma unroll
  for (int j = 0; j < 8; ++j)
    for (int o = 16; o > 0; o >>= 1) acc[j] += __shfl_down_sync(0xffffffffu, acc[j], o);
  __shared__ double red[kN2fThreads / 32][8];
  const int warp = threadIdx.x / 32, lane = threadIdx.x % 32;
  if (lane == 0)
    for (int j = 0; j < 8; ++j) red[warp][j] = acc[j];
  __syncthreads();
  if (threadIdx.x == 0) {
    double s[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    for (int w = 0; w < kN2fThreads / 32; ++w)
      for (int j = 0; j < 8; ++j) s[j] += red[w][j];
    const double h = dx / 3.0;
    for (int j = 0; j < 8; ++j) s[j] *= h * h;
    const double eta0 = 376.730313668;
    const double c = k / (4.0 * M_PI * r);
    double sr, cr;
    sincos(k * r, &sr, &cr);
    const double2 ffw = make_double2(c * sr, c * cr);
    const double2 Nt = make_double2(s[0], s[1]), Np = make_double2(s[2], s[3]);
    const double2 Lt = make_double2(s[4], s[5]), Lp = make_double2(s[6], s[7]);
    auto cm = [](double2 a, double2 b) {
      return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
    };
    const long long plane = (long long)nphi * ntheta;
    const long long o = (long long)ip * ntheta + it;
    out[0 * plane + o] = cm(ffw, make_double2(-Lp.x - eta0 * Nt.x, -Lp.y - eta0 * Nt.y));
    out[1 * plane + o] = cm(ffw, make_double2(Lt.x - eta0 * Np.x, Lt.y - eta0 * Np.y));
    out[2 * plane + o] = cm(ffw, make_double2(Np.x - Lt.x / eta0, Np.y - Lt.y / eta0));
    out[3 * plane + o] = cm(ffw, make_double2(-Nt.x - Lp.x / eta0, -Nt.y - Lp.y / eta0));
  }
}

int n2f_fail(int code, const char* msg) { return report_error(code, msg); }

}  // namespace

}  // namespace fdtd

extern "C" int fdtd_near2far_noalloc(const void* ex_u, const void* ey_u, const void* hx_u,
                                     const void* hy_u, int in_dtype, int nx_ph, int ny_ph,
                                     int nz_ph, double dx, double r, const double* thetas_deg,
                                     int ntheta, const double* phis_deg, int nphi, double freq,
                                     int device, double* out) {
  using namespace fdtd;
  char msg[256];
  if (!ex_u || !ey_u || !hx_u || !hy_u || !thetas_deg || !phis_deg || !out)
    return n2f_fail(FDTD_ERR_INVALID, "null argument");
  if (in_dtype != FDTD_F32 && in_dtype != FDTD_F64)
    return n2f_fail(FDTD_ERR_INVALID, "in_dtype must be FDTD_F32 or FDTD_F64");
  if (nx_ph < 3 || ny_ph < 3 || nx_ph % 2 == 0 || ny_ph % 2 == 0)
    return n2f_fail(FDTD_ERR_INVALID, "Simpson integration needs odd sample counts >= 3");
  if (ntheta < 1 || nphi < 1 || nz_ph < 1) return n2f_fail(FDTD_ERR_INVALID, "empty angle or plane set");
  if (!(freq > 0) || !(dx > 0) || !(r > 0)) return n2f_fail(FDTD_ERR_INVALID, "freq, dx, r must be positive");
  const long long cells = (long long)nx_ph * ny_ph;
  const size_t csz = in_dtype == FDTD_F32 ? 8 : 16;
  const size_t plane_bytes = (size_t)cells * csz;
  if (4 * plane_bytes > kN2fPlaneBytes) {
    snprintf(msg, sizeof(msg),
             "plane of %lld cells exceeds the static scratch (at most %lld cells in complex128, "
             "%lld in complex64); use fdtd_near2far", cells, kN2fMaxCells, 2 * kN2fMaxCells);
    return n2f_fail(FDTD_ERR_INVALID, msg);
  }
  if (ntheta > kN2fMaxTheta || nphi > kN2fMaxPhi || (long long)ntheta * nphi > kN2fMaxAngles) {
    snprintf(msg, sizeof(msg), "angle set %d x %d exceeds the static scratch (theta <= %d, "
             "phi <= %d, product <= %d)", nphi, ntheta, kN2fMaxTheta, kN2fMaxPhi, kN2fMaxAngles);
    return n2f_fail(FDTD_ERR_INVALID, msg);
  }
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return n2f_fail(FDTD_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev || device >= 64) return n2f_fail(FDTD_ERR_INVALID, "device out of range");
  std::lock_guard<std::mutex> lock(g_n2f_mutex);
  DeviceGuard device_guard;   // the caller's current device is restored on return
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return n2f_fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  // set-up, once per device, with that device current: the address of the
  // static scratch on this device (the host-side symbol is not that address)
  if (!g_n2f_addr[device]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_n2f_scratch);
    if (e != cudaSuccess || !p) {
      snprintf(msg, sizeof(msg), "cudaGetSymbolAddress of the near2far scratch: %s",
               cudaGetErrorString(e));
      return n2f_fail(FDTD_ERR_CUDA, msg);
    }
    g_n2f_addr[device] = p;
  }
  unsigned char* base = static_cast<unsigned char*>(g_n2f_addr[device]);
  // every byte the kernel reads is written below and every output it
  // returns is written by the kernel, so no clearing is needed
  const void* planes[4] = {ex_u, ey_u, hx_u, hy_u};
  for (int c = 0; c < 4; ++c) {
    e = cudaMemcpy(base + c * plane_bytes, planes[c], plane_bytes, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) return n2f_fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  }
  unsigned char* ang = base + 4 * plane_bytes;
  if ((e = cudaMemcpy(ang, thetas_deg, (size_t)ntheta * 8, cudaMemcpyHostToDevice)) != cudaSuccess ||
      (e = cudaMemcpy(ang + (size_t)ntheta * 8, phis_deg, (size_t)nphi * 8, cudaMemcpyHostToDevice)) !=
          cudaSuccess)
    return n2f_fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  const double lam = 299792458.0 / freq;
  const double k = 2.0 * M_PI / lam;
  const double z_val = (double)((nz_ph - 1) / 2) * dx;
  const dim3 grd(ntheta, nphi, 1);
  // the kernel finds the angles at 4 * plane_bytes and the output
  // kN2fAngleBytes after them
  if (in_dtype == FDTD_F32)
    k_near2far_raw<float2><<<grd, kN2fThreads>>>(base, (long long)(4 * plane_bytes), nx_ph, ny_ph,
                                                 dx, z_val, k, ntheta, nphi, r);
  else
    k_near2far_raw<double2><<<grd, kN2fThreads>>>(base, (long long)(4 * plane_bytes), nx_ph, ny_ph,
                                                  dx, z_val, k, ntheta, nphi, r);
  if ((e = cudaGetLastError()) != cudaSuccess) return n2f_fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  e = cudaMemcpy(out, ang + kN2fAngleBytes, (size_t)4 * ntheta * nphi * 16, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return n2f_fail(FDTD_ERR_CUDA, cudaGetErrorString(e));
  return FDTD_OK;
}
