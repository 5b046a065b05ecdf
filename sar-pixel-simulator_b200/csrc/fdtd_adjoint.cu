// fdtd_adjoint.cu -- the transposed (adjoint) FDTD step.
//
// The forward step is linear in the fields and the CPML auxiliaries:
//   H' = H - Db curl_E(E) + CPML_H(psi_H'),   psi_H' = bh psi_H + (ch/dx) dE
//   E' = Ca E + Cb curl_H(H') + Cb dx CPML_E(psi_E'),  psi_E' = be psi_E + (ce/dx) dH'
// and the phasors are running sums of plane averages. Reverse-mode
// differentiation of one step is therefore the transposed step run
// backwards in time: the adjoint fields (lambda) of the step's outputs give
// the adjoint fields of its inputs and the step's contribution to
// dJ/dCa = sum_n lambda_E^{n+1} . E^n and dJ/dCb = sum_n lambda_E^{n+1} .
// (curl_H(H^{n+1/2}) + dx psi_E^{n+1}). The transposed curls are the
// backward-difference (for H -> E) and forward-difference (for E -> H)
// stencils of the forward step, with the forward step's index ranges moved
// onto the neighbour that owned the term.
//
// Every kernel is written in gather form (each thread writes only its own
// cell), in the order of the reverse sweep of step n:
//   1. k_adj_phasor_e: lambda_E on the upper phasor plane += dJ/dE^{n+1}
//   2. k_adj_e_to_h:   lambda_H += (E update and E CPML)^T lambda_E
//   3. k_adj_e_own:    gradients; psi_E adjoint; lambda_E = Ca lambda_E
//   4. k_adj_phasor_h: lambda_H on the two planes += dJ/dH^{n+1/2}
//   5. k_adj_h_to_e:   lambda_E += (H update and H CPML)^T lambda_H
//   6. k_adj_h_own:    psi_H adjoint
// Kernel 2 reads lambda_E and the E adjoint auxiliaries of neighbours
// before kernel 3 overwrites them; kernel 5 likewise before kernel 6.
#include "fdtd_launch.h"

namespace fdtd {

namespace {

// index ranges of the forward main updates (cpu/field_updates.py:18-63,
// 198-240)
template <class T>
__device__ __forceinline__ bool re_x(const State<T>& s, int z, int y, int x) {
  return z >= 1 && z < s.nz - 1 && y >= 1 && y < s.ny - 1 && x >= 0 && x < s.nx - 1;
}
template <class T>
__device__ __forceinline__ bool re_y(const State<T>& s, int z, int y, int x) {
  return z >= 1 && z < s.nz - 1 && y >= 0 && y < s.ny - 1 && x >= 1 && x < s.nx - 1;
}
template <class T>
__device__ __forceinline__ bool re_z(const State<T>& s, int z, int y, int x) {
  return z >= 0 && z < s.nz - 1 && y >= 1 && y < s.ny - 1 && x >= 1 && x < s.nx - 1;
}
template <class T>
__device__ __forceinline__ bool rh_x(const State<T>& s, int z, int y, int x) {
  return z >= 0 && z < s.nz - 1 && y >= 0 && y < s.ny - 1 && x >= 1 && x < s.nx - 1;
}
template <class T>
__device__ __forceinline__ bool rh_y(const State<T>& s, int z, int y, int x) {
  return z >= 0 && z < s.nz - 1 && y >= 1 && y < s.ny - 1 && x >= 0 && x < s.nx - 1;
}
template <class T>
__device__ __forceinline__ bool rh_z(const State<T>& s, int z, int y, int x) {
  return z >= 1 && z < s.nz - 1 && y >= 0 && y < s.ny - 1 && x >= 0 && x < s.nx - 1;
}
template <class T>
__device__ __forceinline__ bool box(const State<T>& s, int z, int y, int x) {
  return z >= 0 && y >= 0 && x >= 0 && z < s.nz - 1 && y < s.ny - 1 && x < s.nx - 1;
}

// CPML face membership of a cell: side (0 low, 1 high) and profile index q,
// or false. E faces: 1 <= i < m low, i >= n - m high; H faces: i < m - 1
// low, i >= n - m high (cpu/field_updates.py:66-366); both inside the box.
__device__ __forceinline__ bool e_face(int i, int n, int m, int& side, int& q) {
  if (i >= 1 && i < m) { side = 0; q = i; return true; }
  if (i >= n - m) { side = 1; q = i - (n - m); return true; }
  return false;
}
__device__ __forceinline__ bool h_face(int i, int n, int m, int& side, int& q) {
  if (i >= 0 && i < m - 1) { side = 0; q = i; return true; }
  if (i >= n - m) { side = 1; q = i - (n - m); return true; }
  return false;
}

template <class T>
__device__ __forceinline__ long long idx(const State<T>& s, int z, int y, int x) {
  return ((long long)z * s.ny + y) * s.pitch + x;
}

// psi element of each face layout (z: (m, ny, pitch), x: (nz, ny, m),
// y: (nz, m, pitch))
template <class T>
__device__ __forceinline__ long long kz(const State<T>& s, int q, int y, int x) {
  return ((long long)q * s.ny + y) * s.pitch + x;
}
template <class T>
__device__ __forceinline__ long long kx(const State<T>& s, int z, int y, int q) {
  return ((long long)z * s.ny + y) * s.npml + q;
}
template <class T>
__device__ __forceinline__ long long ky(const State<T>& s, int z, int q, int x) {
  return ((long long)z * s.npml + q) * s.pitch + x;
}

}  // namespace

// ---- 1 / 4: phasor sources -------------------------------------------------
// p(a, b) += avg(F)(a, b) (c + i s) for a in [1, ny_ph), b in [1, nx_ph),
// F sampled around (m + a, m + b) on plane nz - m - 1 (cpu/field_updates.py:
// 373-461, the upper plane). dJ/dF = g_re c + g_im s spread back over the
// averaged samples.
template <class T>
__device__ __forceinline__ double ph_g(const Adj<T>& a, int comp, int ia, int ib, int nyp, int nxp,
                                       double c, double sn) {
  if (ia < 1 || ib < 1 || ia >= nyp || ib >= nxp) return 0.0;
  const long long k = ((long long)comp * nyp + ia) * nxp + ib;
  return a.g_re[k] * c + a.g_im[k] * sn;
}

template <class T>
__global__ void k_adj_phasor_e(const __grid_constant__ State<T> s, Adj<T> a, int t) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= s.nx) return;
  const int m = s.npml, pz = s.nz - m - 1;
  const double* ph = s.phase + 4 * (long long)t;
  const double c = ph[0], sn = ph[1];
  const int ia = y - m, ib = x - m;
  const long long i = idx(s, pz, y, x);
  const double gx = ph_g(a, 0, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 0, ia, ib + 1, s.ny_ph, s.nx_ph, c, sn);
  const double gy = ph_g(a, 1, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 1, ia + 1, ib, s.ny_ph, s.nx_ph, c, sn);
  if (gx != 0.0) a.lex[i] += (T)(0.5 * gx);
  if (gy != 0.0) a.ley[i] += (T)(0.5 * gy);
}

template <class T>
__global__ void k_adj_phasor_h(const __grid_constant__ State<T> s, Adj<T> a, int t) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
  if (x >= s.nx) return;
  const int m = s.npml, pz = s.nz - m - 1;
  const double* ph = s.phase + 4 * (long long)t;
  const double c = ph[2], sn = ph[3];
  const int ia = y - m, ib = x - m;
  const double gx = ph_g(a, 2, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 2, ia + 1, ib, s.ny_ph, s.nx_ph, c, sn);
  const double gy = ph_g(a, 3, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 3, ia, ib + 1, s.ny_ph, s.nx_ph, c, sn);
  if (gx == 0.0 && gy == 0.0) return;
  for (int zz = pz - 1; zz <= pz; ++zz) {
    const long long i = idx(s, zz, y, x);
    a.lhx[i] += (T)(0.25 * gx);
    a.lhy[i] += (T)(0.25 * gy);
  }
}

// ---- 2: lambda_H += (E update + E CPML)^T lambda_E ----------------------------
template <class T>
__global__ void __launch_bounds__(128) k_adj_e_to_h(const __grid_constant__ State<T> s, Adj<T> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= s.nx) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  // F = Cb lambda_E on each component's update range
  auto Fx = [&](int zz, int yy, int xx) -> T {
    if (zz >= nz || yy >= ny || xx >= nx || !re_x(s, zz, yy, xx)) return T(0);
    const long long j = idx(s, zz, yy, xx);
    return s.cb[j] * a.lex[j];
  };
  auto Fy = [&](int zz, int yy, int xx) -> T {
    if (zz >= nz || yy >= ny || xx >= nx || !re_y(s, zz, yy, xx)) return T(0);
    const long long j = idx(s, zz, yy, xx);
    return s.cb[j] * a.ley[j];
  };
  auto Fz = [&](int zz, int yy, int xx) -> T {
    if (zz >= nz || yy >= ny || xx >= nx || !re_z(s, zz, yy, xx)) return T(0);
    const long long j = idx(s, zz, yy, xx);
    return s.cb[j] * a.lez[j];
  };
  const T fx = Fx(z, y, x), fy = Fy(z, y, x), fz = Fz(z, y, x);
  T dhx = (fy - Fy(z + 1, y, x)) - (fz - Fz(z, y + 1, x));
  T dhy = (fz - Fz(z, y, x + 1)) - (fx - Fx(z + 1, y, x));
  T dhz = (fx - Fx(z, y + 1, x)) - (fy - Fy(z, y, x + 1));
  const T rdx = T(1) / s.dx;
  // E-face auxiliaries at (zz, yy, xx): coefficient c/dx times their total
  // adjoint, for the face normal to `axis`, auxiliary slot `slot`
  auto face_term = [&](int axis, int slot, int zz, int yy, int xx) -> T {
    if (zz >= nz || yy >= ny || xx >= nx || !box(s, zz, yy, xx)) return T(0);
    int side, q;
    long long k;
    const T* lp;
    const T* lc;
    T sign;
    if (axis == 0) {
      if (!e_face(zz, nz, m, side, q)) return T(0);
      k = kz(s, q, yy, xx);
      lp = a.lps.z[side][slot];
      lc = slot == 1 ? a.ley : a.lex;
      sign = slot == 1 ? T(1) : T(-1);
    } else if (axis == 1) {
      if (!e_face(xx, nx, m, side, q)) return T(0);
      k = kx(s, zz, yy, q);
      lp = a.lps.x[side][slot];
      lc = slot == 1 ? a.lez : a.ley;
      sign = slot == 1 ? T(1) : T(-1);
    } else {
      if (!e_face(yy, ny, m, side, q)) return T(0);
      k = ky(s, zz, q, xx);
      lp = a.lps.y[side][slot];
      lc = slot == 0 ? a.lex : a.lez;
      sign = slot == 0 ? T(1) : T(-1);
    }
    const long long j = idx(s, zz, yy, xx);
    const T c = s.prof[side ? CE_U : CE_D][q];
    return c * rdx * (lp[k] + sign * s.cb[j] * s.dx * lc[j]);
  };
  // z faces: Eyz uses hx(c) - hx(c - z), Exz uses hy(c) - hy(c - z)
  dhx += face_term(0, 1, z, y, x) - face_term(0, 1, z + 1, y, x);
  dhy += face_term(0, 0, z, y, x) - face_term(0, 0, z + 1, y, x);
  // x faces: Ezx uses hy(c) - hy(c - x), Eyx uses hz(c) - hz(c - x)
  dhy += face_term(1, 1, z, y, x) - face_term(1, 1, z, y, x + 1);
  dhz += face_term(1, 0, z, y, x) - face_term(1, 0, z, y, x + 1);
  // y faces: Exy uses hz(c) - hz(c - y), Ezy uses hx(c) - hx(c - y)
  dhz += face_term(2, 0, z, y, x) - face_term(2, 0, z, y + 1, x);
  dhx += face_term(2, 1, z, y, x) - face_term(2, 1, z, y + 1, x);
  const long long i = idx(s, z, y, x);
  a.lhx[i] += dhx;
  a.lhy[i] += dhy;
  a.lhz[i] += dhz;
}

// ---- 3: gradients, E auxiliaries' adjoint, lambda_E = Ca lambda_E ---------
// s.iex.. hold E^n, s.ihx.. H^{n+1/2}, s.ps the auxiliaries after the step.
template <class T>
__global__ void __launch_bounds__(128) k_adj_e_own(const __grid_constant__ State<T> s, Adj<T> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= s.nx) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  const long long P = s.plane, W = s.pitch;
  const long long i = idx(s, z, y, x);
  const T lx = a.lex[i], ly = a.ley[i], lz = a.lez[i];
  const T cb = s.cb[i], ca = s.ca[i];
  double gca = 0.0, gcb = 0.0;
  const T* hx = s.ihx; const T* hy = s.ihy; const T* hz = s.ihz;
  if (re_x(s, z, y, x)) {
    gca += (double)lx * (double)s.iex[i];
    gcb += (double)lx * (double)((hz[i] - hz[i - W]) - (hy[i] - hy[i - P]));
  }
  if (re_y(s, z, y, x)) {
    gca += (double)ly * (double)s.iey[i];
    gcb += (double)ly * (double)((hx[i] - hx[i - P]) - (hz[i] - hz[i - 1]));
  }
  if (re_z(s, z, y, x)) {
    gca += (double)lz * (double)s.iez[i];
    gcb += (double)lz * (double)((hy[i] - hy[i - 1]) - (hx[i] - hx[i - W]));
  }
  if (box(s, z, y, x)) {
    int side, q;
    if (e_face(z, nz, m, side, q)) {
      const long long k = kz(s, q, y, x);
      const T b = s.prof[side ? BE_U : BE_D][q];
      T* p1 = a.lps.z[side][1];
      T* p0 = a.lps.z[side][0];
      gcb += (double)s.dx * ((double)s.ps.z[side][1][k] * ly - (double)s.ps.z[side][0][k] * lx);
      p1[k] = b * (p1[k] + cb * s.dx * ly);
      p0[k] = b * (p0[k] - cb * s.dx * lx);
    }
    if (e_face(x, nx, m, side, q)) {
      const long long k = kx(s, z, y, q);
      const T b = s.prof[side ? BE_U : BE_D][q];
      T* p1 = a.lps.x[side][1];
      T* p0 = a.lps.x[side][0];
      gcb += (double)s.dx * ((double)s.ps.x[side][1][k] * lz - (double)s.ps.x[side][0][k] * ly);
      p1[k] = b * (p1[k] + cb * s.dx * lz);
      p0[k] = b * (p0[k] - cb * s.dx * ly);
    }
    if (e_face(y, ny, m, side, q)) {
      const long long k = ky(s, z, q, x);
      const T b = s.prof[side ? BE_U : BE_D][q];
      T* p0 = a.lps.y[side][0];
      T* p1 = a.lps.y[side][1];
      gcb += (double)s.dx * ((double)s.ps.y[side][0][k] * lx - (double)s.ps.y[side][1][k] * lz);
      p0[k] = b * (p0[k] + cb * s.dx * lx);
      p1[k] = b * (p1[k] - cb * s.dx * lz);
    }
  }
  if (z < a.nz_grad) {
    a.gca[i] += gca;
    a.gcb[i] += gcb;
  }
  if (re_x(s, z, y, x)) a.lex[i] = ca * lx;
  if (re_y(s, z, y, x)) a.ley[i] = ca * ly;
  if (re_z(s, z, y, x)) a.lez[i] = ca * lz;
}

// ---- 5: lambda_E += (H update + H CPML)^T lambda_H ----------------------------
template <class T>
__global__ void __launch_bounds__(128) k_adj_h_to_e(const __grid_constant__ State<T> s, Adj<T> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= s.nx) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  const T db = s.db;
  auto Gx = [&](int zz, int yy, int xx) -> T {
    if (zz < 0 || yy < 0 || xx < 0 || !rh_x(s, zz, yy, xx)) return T(0);
    return db * a.lhx[idx(s, zz, yy, xx)];
  };
  auto Gy = [&](int zz, int yy, int xx) -> T {
    if (zz < 0 || yy < 0 || xx < 0 || !rh_y(s, zz, yy, xx)) return T(0);
    return db * a.lhy[idx(s, zz, yy, xx)];
  };
  auto Gz = [&](int zz, int yy, int xx) -> T {
    if (zz < 0 || yy < 0 || xx < 0 || !rh_z(s, zz, yy, xx)) return T(0);
    return db * a.lhz[idx(s, zz, yy, xx)];
  };
  const T gx = Gx(z, y, x), gy = Gy(z, y, x), gz = Gz(z, y, x);
  T dex = (gy - Gy(z - 1, y, x)) - (gz - Gz(z, y - 1, x));
  T dey = (gz - Gz(z, y, x - 1)) - (gx - Gx(z - 1, y, x));
  T dez = (gx - Gx(z, y - 1, x)) - (gy - Gy(z, y, x - 1));
  const T rdx = T(1) / s.dx;
  // H-face auxiliaries: their total adjoint times c/dx. slot/comp: z faces
  // 3 Hyz (hy, -) -> ex, 2 Hxz (hx, +) -> ey; x faces 3 Hzx (hz, -) -> ey,
  // 2 Hyx (hy, +) -> ez; y faces 2 Hxy (hx, -) -> ez, 3 Hzy (hz, +) -> ex.
  auto face_term = [&](int axis, int slot, int zz, int yy, int xx) -> T {
    if (!box(s, zz, yy, xx)) return T(0);
    int side, q;
    long long k;
    const T* lp;
    const T* lc;
    T sign;
    if (axis == 0) {
      if (!h_face(zz, nz, m, side, q)) return T(0);
      k = kz(s, q, yy, xx);
      lp = a.lps.z[side][slot];
      lc = slot == 3 ? a.lhy : a.lhx;
      sign = slot == 3 ? T(-1) : T(1);
    } else if (axis == 1) {
      if (!h_face(xx, nx, m, side, q)) return T(0);
      k = kx(s, zz, yy, q);
      lp = a.lps.x[side][slot];
      lc = slot == 3 ? a.lhz : a.lhy;
      sign = slot == 3 ? T(-1) : T(1);
    } else {
      if (!h_face(yy, ny, m, side, q)) return T(0);
      k = ky(s, zz, q, xx);
      lp = a.lps.y[side][slot];
      lc = slot == 2 ? a.lhx : a.lhz;
      sign = slot == 2 ? T(-1) : T(1);
    }
    const T c = s.prof[side ? CH_U : CH_D][q];
    return c * rdx * (lp[k] + sign * s.dtm0 * lc[idx(s, zz, yy, xx)]);
  };
  // the auxiliary at c' uses e(c' + n) - e(c'): e(c) gets +term(c - n) - term(c)
  dex += face_term(0, 3, z - 1, y, x) - face_term(0, 3, z, y, x);
  dey += face_term(0, 2, z - 1, y, x) - face_term(0, 2, z, y, x);
  dey += face_term(1, 3, z, y, x - 1) - face_term(1, 3, z, y, x);
  dez += face_term(1, 2, z, y, x - 1) - face_term(1, 2, z, y, x);
  dez += face_term(2, 2, z, y - 1, x) - face_term(2, 2, z, y, x);
  dex += face_term(2, 3, z, y - 1, x) - face_term(2, 3, z, y, x);
  const long long i = idx(s, z, y, x);
  a.lex[i] += dex;
  a.ley[i] += dey;
  a.lez[i] += dez;
}

// ---- 6: H auxiliaries' adjoint ---------------------------------------------------
template <class T>
__global__ void __launch_bounds__(128) k_adj_h_own(const __grid_constant__ State<T> s, Adj<T> a) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y, z = blockIdx.z;
  if (x >= s.nx || !box(s, z, y, x)) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  const long long i = idx(s, z, y, x);
  const T lhx = a.lhx[i], lhy = a.lhy[i], lhz = a.lhz[i];
  int side, q;
  if (h_face(z, nz, m, side, q)) {
    const long long k = kz(s, q, y, x);
    const T b = s.prof[side ? BH_U : BH_D][q];
    T* p3 = a.lps.z[side][3];
    T* p2 = a.lps.z[side][2];
    p3[k] = b * (p3[k] - s.dtm0 * lhy);
    p2[k] = b * (p2[k] + s.dtm0 * lhx);
  }
  if (h_face(x, nx, m, side, q)) {
    const long long k = kx(s, z, y, q);
    const T b = s.prof[side ? BH_U : BH_D][q];
    T* p3 = a.lps.x[side][3];
    T* p2 = a.lps.x[side][2];
    p3[k] = b * (p3[k] - s.dtm0 * lhz);
    p2[k] = b * (p2[k] + s.dtm0 * lhy);
  }
  if (h_face(y, ny, m, side, q)) {
    const long long k = ky(s, z, q, x);
    const T b = s.prof[side ? BH_U : BH_D][q];
    T* p2 = a.lps.y[side][2];
    T* p3 = a.lps.y[side][3];
    p2[k] = b * (p2[k] - s.dtm0 * lhx);
    p3[k] = b * (p3[k] + s.dtm0 * lhz);
  }
}

template <class T>
void launch_adjoint_step(const State<T>& s, const Adj<T>& a, int t, cudaStream_t st) {
  const dim3 blk(128, 1, 1);
  const dim3 grd((s.nx + 127) / 128, s.ny, s.nz);
  const dim3 gpl((s.nx + 127) / 128, s.ny, 1);
  k_adj_phasor_e<T><<<gpl, blk, 0, st>>>(s, a, t);
  k_adj_e_to_h<T><<<grd, blk, 0, st>>>(s, a);
  k_adj_e_own<T><<<grd, blk, 0, st>>>(s, a);
  k_adj_phasor_h<T><<<gpl, blk, 0, st>>>(s, a, t);
  k_adj_h_to_e<T><<<grd, blk, 0, st>>>(s, a);
  k_adj_h_own<T><<<grd, blk, 0, st>>>(s, a);
}

template void launch_adjoint_step<float>(const State<float>&, const Adj<float>&, int, cudaStream_t);
template void launch_adjoint_step<double>(const State<double>&, const Adj<double>&, int, cudaStream_t);

}  // namespace fdtd
