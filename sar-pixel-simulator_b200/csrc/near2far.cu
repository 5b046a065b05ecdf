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
