// fdtd_cell.cuh -- per-cell H and E updates with CPML and incident injection.
//
// One function computes the complete new value of the three H (or E)
// components of one Yee cell for one half step, in the reference's order:
// main curl update, z-face CPML, x-face CPML, y-face CPML, injection
// (fdtdsarsim/cpu/main_sim.py:140-161; cpu/fdtd_sim.py:29-133).
//
// Index ranges follow the reference kernels exactly
// (cpu/field_updates.py:18-366). Every component shares the box
// z < nz-1, y < ny-1, x < nx-1; inside it
//   Hx main update needs x >= 1, Hy y >= 1, Hz z >= 1   (:198-240)
//   Ex main update needs z,y >= 1, Ey z,x >= 1, Ez y,x >= 1   (:18-63)
// while the CPML corrections cover the whole box slab of their face
// (e.g. cpml_h_down also corrects Hx at x = 0, :243-260). H faces use
// q in [0, npml-1) on both sides; E low faces use q in [1, npml) and E high
// faces q in [0, npml-1) (:66-191). The incident planes are added on the
// whole plane z = tfsf_z, every y and x (cpu/main_sim.py:147-161).
#pragma once

#include "fdtd_common.cuh"

namespace fdtd {

// E at the cell and at its +z, +y, +x neighbours (what the H update reads).
template <class T> struct ENbr {
  T ex0, exz, exy;   // ex, ex(z+1), ex(y+1)
  T ey0, eyz, eyx;   // ey, ey(z+1), ey(x+1)
  T ez0, ezy, ezx;   // ez, ez(y+1), ez(x+1)
};

// H at the cell and at its -z, -y, -x neighbours (what the E update reads).
template <class T> struct HNbr {
  T hx0, hxz, hxy;   // hx, hx(z-1), hx(y-1)
  T hy0, hyz, hyx;   // hy, hy(z-1), hy(x-1)
  T hz0, hzy, hzx;   // hz, hz(y-1), hz(x-1)
};

template <class T>
__device__ __forceinline__ bool in_box(const State<T>& s, int z, int y, int x) {
  return z < s.nz - 1 && y < s.ny - 1 && x < s.nx - 1;
}

template <class T>
__device__ __forceinline__ bool injects(const State<T>& s, int z, int t) {
  return z == s.tfsf_z && t < s.nt_inc;
}

// New H at (z, y, x). hx, hy, hz carry the old values in and the new ones
// out. psi is read from s.ps and, when wpsi, written to s.pd.
template <class T>
__device__ __forceinline__ void h_cell(const State<T>& s, const ENbr<T>& e,
                                       int z, int y, int x, int t, bool wpsi,
                                       T& hx, T& hy, T& hz) {
  using M = R<T>;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  if (in_box(s, z, y, x)) {
    const T dey_z = M::sub(e.eyz, e.ey0);
    const T dez_y = M::sub(e.ezy, e.ez0);
    const T dex_z = M::sub(e.exz, e.ex0);
    const T dez_x = M::sub(e.ezx, e.ez0);
    const T dex_y = M::sub(e.exy, e.ex0);
    const T dey_x = M::sub(e.eyx, e.ey0);
    // Taflove 3.30 (cpu/field_updates.py:198-240)
    if (x >= 1) hx = M::sub(hx, M::mul(s.db, M::sub(dez_y, dey_z)));
    if (y >= 1) hy = M::sub(hy, M::mul(s.db, M::sub(dex_z, dez_x)));
    if (z >= 1) hz = M::sub(hz, M::mul(s.db, M::sub(dey_x, dex_y)));
    // z faces (cpml_h_down/up, cpu/field_updates.py:243-282)
    {
      int side = -1, q = 0;
      if (z < m - 1) { side = 0; q = z; }
      else if (z >= nz - m) { side = 1; q = z - (nz - m); }
      if (side >= 0) {
        const T b = s.prof[side ? BH_U : BH_D][q];
        const T c = s.prof[side ? CH_U : CH_D][q];
        const long long k = ((long long)q * ny + y) * s.pitch + x;
        const T pyz = M::add(M::mul(b, s.ps.z[side][3][k]), div_dx(s, M::mul(c, dex_z)));
        const T pxz = M::add(M::mul(b, s.ps.z[side][2][k]), div_dx(s, M::mul(c, dey_z)));
        if (wpsi) { s.pd.z[side][3][k] = pyz; s.pd.z[side][2][k] = pxz; }
        hy = M::sub(hy, M::mul(s.dtm0, pyz));
        hx = M::add(hx, M::mul(s.dtm0, pxz));
      }
    }
    // x faces (cpml_h_left/right, :285-324)
    {
      int side = -1, q = 0;
      if (x < m - 1) { side = 0; q = x; }
      else if (x >= nx - m) { side = 1; q = x - (nx - m); }
      if (side >= 0) {
        const T b = s.prof[side ? BH_U : BH_D][q];
        const T c = s.prof[side ? CH_U : CH_D][q];
        const long long k = xpsi_index(s, z, y, side, x);
        const T pzx = M::add(M::mul(b, s.ps.x[side][3][k]), div_dx(s, M::mul(c, dey_x)));
        const T pyx = M::add(M::mul(b, s.ps.x[side][2][k]), div_dx(s, M::mul(c, dez_x)));
        if (wpsi) { s.pd.x[side][3][k] = pzx; s.pd.x[side][2][k] = pyx; }
        hz = M::sub(hz, M::mul(s.dtm0, pzx));
        hy = M::add(hy, M::mul(s.dtm0, pyx));
      }
    }
    // y faces (cpml_h_front/back, :327-366)
    {
      int side = -1, q = 0;
      if (y < m - 1) { side = 0; q = y; }
      else if (y >= ny - m) { side = 1; q = y - (ny - m); }
      if (side >= 0) {
        const T b = s.prof[side ? BH_U : BH_D][q];
        const T c = s.prof[side ? CH_U : CH_D][q];
        const long long k = ((long long)z * m + q) * s.pitch + x;
        const T pxy = M::add(M::mul(b, s.ps.y[side][2][k]), div_dx(s, M::mul(c, dez_y)));
        const T pzy = M::add(M::mul(b, s.ps.y[side][3][k]), div_dx(s, M::mul(c, dex_y)));
        if (wpsi) { s.pd.y[side][2][k] = pxy; s.pd.y[side][3][k] = pzy; }
        hx = M::sub(hx, M::mul(s.dtm0, pxy));
        hz = M::add(hz, M::mul(s.dtm0, pzy));
      }
    }
  }
  // E-field injection into H (cpu/main_sim.py:147-150)
  if (injects(s, z, t)) {
    const long long k = ((long long)t * ny + y) * s.pitch + x;
    hx = M::add(hx, M::mul(s.db, s.inc_ey[k]));
    hy = M::sub(hy, M::mul(s.db, s.inc_ex[k]));
  }
}

// New E at (z, y, x) from H^{n+1/2}. ex, ey, ez carry old values in and new
// ones out.
template <class T>
__device__ __forceinline__ void e_cell(const State<T>& s, const HNbr<T>& h,
                                       T ca, T cb, int z, int y, int x, int t,
                                       bool wpsi, T& ex, T& ey, T& ez) {
  using M = R<T>;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  if (in_box(s, z, y, x)) {
    const T dhz_y = M::sub(h.hz0, h.hzy);
    const T dhy_z = M::sub(h.hy0, h.hyz);
    const T dhx_z = M::sub(h.hx0, h.hxz);
    const T dhz_x = M::sub(h.hz0, h.hzx);
    const T dhx_y = M::sub(h.hx0, h.hxy);
    const T dhy_x = M::sub(h.hy0, h.hyx);
    // Taflove 3.29 (cpu/field_updates.py:18-63)
    if (z >= 1 && y >= 1) ex = M::add(M::mul(ex, ca), M::mul(cb, M::sub(dhz_y, dhy_z)));
    if (z >= 1 && x >= 1) ey = M::add(M::mul(ey, ca), M::mul(cb, M::sub(dhx_z, dhz_x)));
    if (y >= 1 && x >= 1) ez = M::add(M::mul(ez, ca), M::mul(cb, M::sub(dhy_x, dhx_y)));
    const T cbdx = M::mul(cb, s.dx);
    // z faces (cpml_e_down/up, :66-105)
    {
      int side = -1, q = 0;
      if (z >= 1 && z < m) { side = 0; q = z; }
      else if (z >= nz - m) { side = 1; q = z - (nz - m); }
      if (side >= 0) {
        const T b = s.prof[side ? BE_U : BE_D][q];
        const T c = s.prof[side ? CE_U : CE_D][q];
        const long long k = ((long long)q * ny + y) * s.pitch + x;
        const T pyz = M::add(M::mul(b, s.ps.z[side][1][k]), div_dx(s, M::mul(c, dhx_z)));
        const T pxz = M::add(M::mul(b, s.ps.z[side][0][k]), div_dx(s, M::mul(c, dhy_z)));
        if (wpsi) { s.pd.z[side][1][k] = pyz; s.pd.z[side][0][k] = pxz; }
        ey = M::add(ey, M::mul(cbdx, pyz));
        ex = M::sub(ex, M::mul(cbdx, pxz));
      }
    }
    // x faces (cpml_e_left/right, :108-148)
    {
      int side = -1, q = 0;
      if (x >= 1 && x < m) { side = 0; q = x; }
      else if (x >= nx - m) { side = 1; q = x - (nx - m); }
      if (side >= 0) {
        const T b = s.prof[side ? BE_U : BE_D][q];
        const T c = s.prof[side ? CE_U : CE_D][q];
        const long long k = xpsi_index(s, z, y, side, x);
        const T pzx = M::add(M::mul(b, s.ps.x[side][1][k]), div_dx(s, M::mul(c, dhy_x)));
        const T pyx = M::add(M::mul(b, s.ps.x[side][0][k]), div_dx(s, M::mul(c, dhz_x)));
        if (wpsi) { s.pd.x[side][1][k] = pzx; s.pd.x[side][0][k] = pyx; }
        ez = M::add(ez, M::mul(cbdx, pzx));
        ey = M::sub(ey, M::mul(cbdx, pyx));
      }
    }
    // y faces (cpml_e_front/back, :151-191)
    {
      int side = -1, q = 0;
      if (y >= 1 && y < m) { side = 0; q = y; }
      else if (y >= ny - m) { side = 1; q = y - (ny - m); }
      if (side >= 0) {
        const T b = s.prof[side ? BE_U : BE_D][q];
        const T c = s.prof[side ? CE_U : CE_D][q];
        const long long k = ((long long)z * m + q) * s.pitch + x;
        const T pxy = M::add(M::mul(b, s.ps.y[side][0][k]), div_dx(s, M::mul(c, dhz_y)));
        const T pzy = M::add(M::mul(b, s.ps.y[side][1][k]), div_dx(s, M::mul(c, dhx_y)));
        if (wpsi) { s.pd.y[side][0][k] = pxy; s.pd.y[side][1][k] = pzy; }
        ex = M::add(ex, M::mul(cbdx, pxy));
        ez = M::sub(ez, M::mul(cbdx, pzy));
      }
    }
  }
  // H-field injection into E (cpu/main_sim.py:158-161)
  if (injects(s, z, t)) {
    const long long k = ((long long)t * ny + y) * s.pitch + x;
    ey = M::add(ey, M::mul(s.dte0dx, s.inc_hx[k]));
    ex = M::sub(ex, M::mul(s.dte0dx, s.inc_hy[k]));
  }
}

}  // namespace fdtd
