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
// cell). The reverse sweep of step n is, in order:
//   a. lambda_E on the upper phasor plane += dJ/dE^{n+1}
//   b. lambda_H += (E update and E CPML)^T lambda_E
//   c. gradients; psi_E adjoint; lambda_E = Ca lambda_E
//   d. lambda_H on the two planes += dJ/dH^{n+1/2}
//   e. lambda_E += (H update and H CPML)^T lambda_H
//   f. psi_H adjoint
// b reads lambda_E and the E auxiliaries' adjoint of neighbours before c
// overwrites them; e reads lambda_H and the H auxiliaries' adjoint of
// neighbours before f overwrites them. Two kernels per step do all six:
// k_adj_k1 = f of step n + 1, b, d; k_adj_k2 = c, e, a of step n - 1; only
// the first backward step needs a on its own (k_adj_phasor_e).
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

// phasor E source of step t at cell (z, y, x): (d ex, d ey)
template <class T>
__device__ __forceinline__ void phasor_e_src(const State<T>& s, const Adj<T>& a, int t, int z, int y,
                                             int x, T& dex, T& dey) {
  dex = T(0);
  dey = T(0);
  const int m = s.npml;
  if (z != s.nz - m - 1) return;
  const double* ph = s.phase + 4 * (long long)t;
  const double c = ph[0], sn = ph[1];
  const int ia = y - m, ib = x - m;
  const double gx = ph_g(a, 0, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 0, ia, ib + 1, s.ny_ph, s.nx_ph, c, sn);
  const double gy = ph_g(a, 1, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 1, ia + 1, ib, s.ny_ph, s.nx_ph, c, sn);
  dex = (T)(0.5 * gx);
  dey = (T)(0.5 * gy);
}

// phasor H source of step t at cell (z, y, x): (d hx, d hy), planes pz - 1, pz
template <class T>
__device__ __forceinline__ void phasor_h_src(const State<T>& s, const Adj<T>& a, int t, int z, int y,
                                             int x, T& dhx, T& dhy) {
  dhx = T(0);
  dhy = T(0);
  const int m = s.npml, pz = s.nz - m - 1;
  if (z != pz && z != pz - 1) return;
  const double* ph = s.phase + 4 * (long long)t;
  const double c = ph[2], sn = ph[3];
  const int ia = y - m, ib = x - m;
  const double gx = ph_g(a, 2, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 2, ia + 1, ib, s.ny_ph, s.nx_ph, c, sn);
  const double gy = ph_g(a, 3, ia, ib, s.ny_ph, s.nx_ph, c, sn) + ph_g(a, 3, ia, ib + 1, s.ny_ph, s.nx_ph, c, sn);
  dhx = (T)(0.25 * gx);
  dhy = (T)(0.25 * gy);
}

// standalone E source of the first backward step (the later ones are added
// by k_adj_k2 of the step after them)
template <class T>
__global__ void k_adj_phasor_e(const __grid_constant__ State<T> s, Adj<T> a, int t) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= s.nx || y >= s.ny) return;
  const int z = s.nz - s.npml - 1;
  T dex, dey;
  phasor_e_src(s, a, t, z, y, x, dex, dey);
  const long long i = idx(s, z, y, x);
  if (re_x(s, z, y, x)) a.lex[i] += dex;
  if (re_y(s, z, y, x)) a.ley[i] += dey;
}

// ---- 2: lambda_H += (E update + E CPML)^T lambda_E ----------------------------
template <class T>
__device__ __forceinline__ void e_to_h_terms(const State<T>& s, const Adj<T>& a, int z, int y, int x,
                                             T& out_hx, T& out_hy, T& out_hz) {
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
  out_hx = dhx;
  out_hy = dhy;
  out_hz = dhz;
}

// ---- 3: gradients, E auxiliaries' adjoint, Ca lambda_E --------------------
// s.iex.. hold E^n, s.ihx.. H^{n+1/2}, s.ps the auxiliaries after the step.
// Returns Ca lambda_E of the cell (zero outside the update ranges).
template <class T>
__device__ __forceinline__ void e_own_part(const State<T>& s, const Adj<T>& a, int z, int y, int x,
                                           T& out_x, T& out_y, T& out_z) {
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  const long long P = s.plane, W = s.pitch;
  const long long i = idx(s, z, y, x);
  const T lx = a.lex[i], ly = a.ley[i], lz = a.lez[i];
  const T cb = s.cb[i], ca = s.ca[i];
  double gca = 0.0, gcb = 0.0;
  const T* hx = s.ihx; const T* hy = s.ihy; const T* hz = s.ihz;
  const bool grad = z < a.nz_grad;   // gradients only over the requested planes
  if (grad && re_x(s, z, y, x)) {
    gca += (double)lx * (double)s.iex[i];
    gcb += (double)lx * (double)((hz[i] - hz[i - W]) - (hy[i] - hy[i - P]));
  }
  if (grad && re_y(s, z, y, x)) {
    gca += (double)ly * (double)s.iey[i];
    gcb += (double)ly * (double)((hx[i] - hx[i - P]) - (hz[i] - hz[i - 1]));
  }
  if (grad && re_z(s, z, y, x)) {
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
      if (grad) gcb += (double)s.dx * ((double)s.ps.z[side][1][k] * ly - (double)s.ps.z[side][0][k] * lx);
      p1[k] = b * (p1[k] + cb * s.dx * ly);
      p0[k] = b * (p0[k] - cb * s.dx * lx);
    }
    if (e_face(x, nx, m, side, q)) {
      const long long k = kx(s, z, y, q);
      const T b = s.prof[side ? BE_U : BE_D][q];
      T* p1 = a.lps.x[side][1];
      T* p0 = a.lps.x[side][0];
      if (grad) gcb += (double)s.dx * ((double)s.ps.x[side][1][k] * lz - (double)s.ps.x[side][0][k] * ly);
      p1[k] = b * (p1[k] + cb * s.dx * lz);
      p0[k] = b * (p0[k] - cb * s.dx * ly);
    }
    if (e_face(y, ny, m, side, q)) {
      const long long k = ky(s, z, q, x);
      const T b = s.prof[side ? BE_U : BE_D][q];
      T* p0 = a.lps.y[side][0];
      T* p1 = a.lps.y[side][1];
      if (grad) gcb += (double)s.dx * ((double)s.ps.y[side][0][k] * lx - (double)s.ps.y[side][1][k] * lz);
      p0[k] = b * (p0[k] + cb * s.dx * lx);
      p1[k] = b * (p1[k] - cb * s.dx * lz);
    }
  }
  if (grad) {
    a.gca[i] += gca;
    a.gcb[i] += gcb;
  }
  // A component outside its main-update range is updated in the forward
  // step only by CPML corrections and injection terms that read other such
  // components (the edge sub-systems, e.g. ey, ez, hx on x = 0), or not at
  // all. With an incident beam that vanishes on those edges (as the
  // reference's does) it stays exactly zero, so no parameter reaches J
  // through it, and nothing in range reads it back in the transposed step.
  // Its exact adjoint, fed by the interior's, grows exponentially like the
  // forward sub-system would if driven; it is held at zero instead (here,
  // and by the range tests where adjoints are accumulated), which leaves
  // every gradient unchanged and keeps the sweep finite.
  out_x = re_x(s, z, y, x) ? ca * lx : T(0);
  out_y = re_y(s, z, y, x) ? ca * ly : T(0);
  out_z = re_z(s, z, y, x) ? ca * lz : T(0);
}

// ---- 5: lambda_E += (H update + H CPML)^T lambda_H ----------------------------
template <class T>
__device__ __forceinline__ void h_to_e_terms(const State<T>& s, const Adj<T>& a, int z, int y, int x,
                                             T& out_x, T& out_y, T& out_z) {
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
  out_x = dex;
  out_y = dey;
  out_z = dez;
}

// ---- 6: H auxiliaries' adjoint, from the cell's lambda_H (lhx, lhy, lhz) --
template <class T>
__device__ __forceinline__ void h_own_part(const State<T>& s, const Adj<T>& a, int z, int y, int x,
                                           T lhx, T lhy, T lhz) {
  if (!box(s, z, y, x)) return;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
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

// ---- the two kernels of one backward step ------------------------------------
// K1 (step n): the H auxiliaries' adjoint of step n + 1 (skipped for the
// first backward step), then lambda_H += (E step)^T lambda_E + the H phasor
// source of step n.
template <class T>
__global__ void __launch_bounds__(128) k_adj_k1(const __grid_constant__ State<T> s, Adj<T> a, int t,
                                                int first) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= s.nx || y >= s.ny) return;
  const long long i = idx(s, z, y, x);
  const T lhx = a.lhx[i], lhy = a.lhy[i], lhz = a.lhz[i];
  const int m = s.npml;
  T dhx, dhy, dhz, phx, phy;
  if (z >= m && z < s.nz - m - 1 && y >= m && y < s.ny - m - 1 && x >= m && x < s.nx - m - 1) {
    // the cell and its +x, +y, +z neighbours are away from every CPML face
    // and domain edge: the plain transposed curl
    const long long P = s.plane, W = s.pitch;
    const T fx = s.cb[i] * a.lex[i], fy = s.cb[i] * a.ley[i], fz = s.cb[i] * a.lez[i];
    const T fy_z = s.cb[i + P] * a.ley[i + P], fx_z = s.cb[i + P] * a.lex[i + P];
    const T fz_y = s.cb[i + W] * a.lez[i + W], fx_y = s.cb[i + W] * a.lex[i + W];
    const T fz_x = s.cb[i + 1] * a.lez[i + 1], fy_x = s.cb[i + 1] * a.ley[i + 1];
    dhx = (fy - fy_z) - (fz - fz_y);
    dhy = (fz - fz_x) - (fx - fx_z);
    dhz = (fx - fx_y) - (fy - fy_x);
  } else {
    if (!first) h_own_part(s, a, z, y, x, lhx, lhy, lhz);
    e_to_h_terms(s, a, z, y, x, dhx, dhy, dhz);
  }
  phasor_h_src(s, a, t, z, y, x, phx, phy);
  // components outside their update range keep a zero adjoint (e_own_part)
  a.lhx[i] = rh_x(s, z, y, x) ? lhx + dhx + phx : T(0);
  a.lhy[i] = rh_y(s, z, y, x) ? lhy + dhy + phy : T(0);
  a.lhz[i] = rh_z(s, z, y, x) ? lhz + dhz : T(0);
}

// K2 (step n): gradients and the E auxiliaries' adjoint, then
// lambda_E = Ca lambda_E + (H step)^T lambda_H + the E phasor source of
// step n - 1 (t_prev < 0: none).
template <class T>
__global__ void __launch_bounds__(128) k_adj_k2(const __grid_constant__ State<T> s, Adj<T> a,
                                                int t_prev) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
  const int z = blockIdx.z;
  if (x >= s.nx || y >= s.ny) return;
  const long long i = idx(s, z, y, x);
  const int m = s.npml;
  T ex, ey, ez, dex, dey, dez, pex = T(0), pey = T(0);
  if (z >= m && z < s.nz - m && y >= m && y < s.ny - m && x >= m && x < s.nx - m) {
    // the cell and its -x, -y, -z neighbours are away from every CPML face
    // and domain edge
    const long long P = s.plane, W = s.pitch;
    const T lx = a.lex[i], ly = a.ley[i], lz = a.lez[i];
    if (z < a.nz_grad) {
      const T* hx = s.ihx; const T* hy = s.ihy; const T* hz = s.ihz;
      a.gca[i] += (double)lx * (double)s.iex[i] + (double)ly * (double)s.iey[i] +
                  (double)lz * (double)s.iez[i];
      a.gcb[i] += (double)lx * (double)((hz[i] - hz[i - W]) - (hy[i] - hy[i - P])) +
                  (double)ly * (double)((hx[i] - hx[i - P]) - (hz[i] - hz[i - 1])) +
                  (double)lz * (double)((hy[i] - hy[i - 1]) - (hx[i] - hx[i - W]));
    }
    const T ca = s.ca[i], db = s.db;
    ex = ca * lx;
    ey = ca * ly;
    ez = ca * lz;
    const T gx = db * a.lhx[i], gy = db * a.lhy[i], gz = db * a.lhz[i];
    const T gy_z = db * a.lhy[i - P], gx_z = db * a.lhx[i - P];
    const T gz_y = db * a.lhz[i - W], gx_y = db * a.lhx[i - W];
    const T gz_x = db * a.lhz[i - 1], gy_x = db * a.lhy[i - 1];
    dex = (gy - gy_z) - (gz - gz_y);
    dey = (gz - gz_x) - (gx - gx_z);
    dez = (gx - gx_y) - (gy - gy_x);
  } else {
    e_own_part(s, a, z, y, x, ex, ey, ez);
    h_to_e_terms(s, a, z, y, x, dex, dey, dez);
  }
  if (t_prev >= 0) phasor_e_src(s, a, t_prev, z, y, x, pex, pey);
  a.lex[i] = re_x(s, z, y, x) ? ex + dex + pex : T(0);
  a.ley[i] = re_y(s, z, y, x) ? ey + dey + pey : T(0);
  a.lez[i] = re_z(s, z, y, x) ? ez + dez : T(0);
}

// 32 x 4 cells per block: little x padding on grids a few hundred cells wide
template <class T>
void launch_adjoint_first(const State<T>& s, const Adj<T>& a, int t, cudaStream_t st) {
  k_adj_phasor_e<T><<<dim3((s.nx + 31) / 32, (s.ny + 3) / 4, 1), dim3(32, 4, 1), 0, st>>>(s, a, t);
}

template <class T>
void launch_adjoint_step(const State<T>& s, const Adj<T>& a, int t, bool first, cudaStream_t st) {
  const dim3 grd((s.nx + 31) / 32, (s.ny + 3) / 4, s.nz), blk(32, 4, 1);
  k_adj_k1<T><<<grd, blk, 0, st>>>(s, a, t, first ? 1 : 0);
  k_adj_k2<T><<<grd, blk, 0, st>>>(s, a, t - 1);
}

template void launch_adjoint_first<float>(const State<float>&, const Adj<float>&, int, cudaStream_t);
template void launch_adjoint_first<double>(const State<double>&, const Adj<double>&, int, cudaStream_t);
template void launch_adjoint_step<float>(const State<float>&, const Adj<float>&, int, bool, cudaStream_t);
template void launch_adjoint_step<double>(const State<double>&, const Adj<double>&, int, bool,
                                          cudaStream_t);

}  // namespace fdtd
