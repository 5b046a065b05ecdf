// fdtd_materials.cu -- material blocks made on the device: layered rough
// surfaces and spherical inclusions, written straight into a simulation's
// eps_r / sigma staging volumes (nz_mat, ny, nx), from which Ca / Cb are
// made on the device as for an uploaded block.
//
// Layers (materials/materials.py:112-164, materials/soilmodels.py:16-195):
// interfaces k = 0 .. n - 1 given as height maps in cells (ny, nx), lowest
// first; a cell (z, y, x) takes the values of the first interface with
// z <= h_k(y, x), and the last values (the medium above every interface,
// normally vacuum) when there is none. Values are rounded to the element
// type as numpy's astype rounds them.
//
// Spheres (materials/bubbles.py:21-199): each (zc, yc, xc, rc, ri) paints
// the cells (rint(zc + dz), rint(yc + dy), rint(xc + dx)) for integer
// |dz|, |dy|, |dx| <= ri with dz^2 + dy^2 + dx^2 < rc^2, rint rounding half
// to even as numpy's rint. Spheres paint the same values, so their order
// and overlaps do not matter. The sphere list is drawn on the host, with
// the reference's random draws and stopping rule (which depend on the
// geometry only).
#include <algorithm>

#include "fdtd_launch.h"

namespace fdtd {

namespace {

template <class T>
__global__ void __launch_bounds__(256) k_fill_layers(T* __restrict__ eps, T* __restrict__ sig, int nx, int ny,
                                                     int nz_mat, int nlayers, const double* __restrict__ h,
                                                     const double* __restrict__ ev, const double* __restrict__ sv) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  if (x >= nx) return;
  const long long col = (long long)y * nx + x;
  const long long plane = (long long)ny * nx;
  for (int z = blockIdx.z; z < nz_mat; z += gridDim.z) {
    int k = 0;
    while (k < nlayers && !((double)z <= h[k * plane + col])) ++k;
    const long long i = (long long)z * plane + col;
    eps[i] = R<T>::from_double(ev[k]);
    sig[i] = R<T>::from_double(sv[k]);
  }
}

// one block per sphere; its threads stride over the (2 ri + 1)^3 offsets
template <class T>
__global__ void __launch_bounds__(256) k_paint_spheres(T* __restrict__ eps, T* __restrict__ sig, int nx, int ny,
                                                       int nz_mat, const double* __restrict__ sp, int n, T e_val,
                                                       T s_val) {
  const int b = blockIdx.x;
  if (b >= n) return;
  const double zc = sp[5 * b], yc = sp[5 * b + 1], xc = sp[5 * b + 2], rc = sp[5 * b + 3];
  const int ri = (int)sp[5 * b + 4];
  const int w = 2 * ri + 1;
  const long long cnt = (long long)w * w * w;
  for (long long o = threadIdx.x; o < cnt; o += blockDim.x) {
    const int dz = (int)(o / ((long long)w * w)) - ri;
    const int dy = (int)((o / w) % w) - ri;
    const int dx = (int)(o % w) - ri;
    if (!((double)(dz * dz + dy * dy + dx * dx) < rc * rc)) continue;
    const int z = (int)rint(zc + dz), y = (int)rint(yc + dy), x = (int)rint(xc + dx);
    if (z < 0 || z >= nz_mat || y < 0 || y >= ny || x < 0 || x >= nx) continue;   // the draws keep them inside
    const long long i = ((long long)z * ny + y) * nx + x;
    eps[i] = e_val;
    sig[i] = s_val;
  }
}

}  // namespace

template <class T>
void launch_fill_layers(T* eps, T* sig, int nx, int ny, int nz_mat, int nlayers, const double* h, const double* ev,
                        const double* sv, cudaStream_t st) {
  const dim3 grd((nx + 255) / 256, ny, (unsigned)std::min(nz_mat, 64));
  k_fill_layers<T><<<grd, 256, 0, st>>>(eps, sig, nx, ny, nz_mat, nlayers, h, ev, sv);
}

template <class T>
void launch_paint_spheres(T* eps, T* sig, int nx, int ny, int nz_mat, const double* sp, int n, double e_val,
                          double s_val, cudaStream_t st) {
  if (n <= 0) return;
  k_paint_spheres<T><<<n, 256, 0, st>>>(eps, sig, nx, ny, nz_mat, sp, n, (T)e_val, (T)s_val);
}

template void launch_fill_layers<float>(float*, float*, int, int, int, int, const double*, const double*,
                                        const double*, cudaStream_t);
template void launch_fill_layers<double>(double*, double*, int, int, int, int, const double*, const double*,
                                         const double*, cudaStream_t);
template void launch_paint_spheres<float>(float*, float*, int, int, int, const double*, int, double, double,
                                          cudaStream_t);
template void launch_paint_spheres<double>(double*, double*, int, int, int, const double*, int, double, double,
                                           cudaStream_t);

}  // namespace fdtd
