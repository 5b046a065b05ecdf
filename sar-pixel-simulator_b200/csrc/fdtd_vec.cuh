// fdtd_vec.cuh -- four-cell vector H and E updates with CPML and injection.
//
// A thread owns four consecutive x cells of one row; the pitch is a multiple
// of 32 elements, so the four cells are one aligned 16-byte (float) or
// 32-byte (double) vector in every (.., pitch)-strided array: fields, Ca/Cb,
// incident planes, and the psi arrays of the z and y faces.
//
// h_vec / e_vec compute the same values as h_cell / e_cell (fdtd_cell.cuh)
// applied to each of the four cells, in the same order of operations:
// main curl update, z-face CPML, x-face CPML, y-face CPML, injection
// (fdtdsarsim/cpu/main_sim.py:140-161, cpu/field_updates.py:18-366). The
// z- and y-face terms and the injection are vector operations (their
// coefficients depend on z or y only, which is uniform over the vector);
// only the x-face terms, whose psi layout is (z, y, npml), run per cell,
// and only in lanes whose vector touches an x face. Cells outside an
// update's index range keep their value, so vectors that straddle the
// domain edge or the padding need no separate path.
#pragma once

#include "fdtd_cell.cuh"
#include "fdtd_check.cuh"

namespace fdtd {

constexpr int kVec = 4;

template <class T>
__device__ __forceinline__ void ld4(T (&d)[kVec], const T* p) {
  if (!FDTD_CHECK_PTR(p, (int)sizeof(T) * kVec)) {   // bounds-checked build only
#pragma unroll
    for (int j = 0; j < kVec; ++j) d[j] = T(0);
    return;
  }
  if constexpr (sizeof(T) == 4) {
    const float4 v = *reinterpret_cast<const float4*>(p);
    d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = v.w;
  } else {
    const double2 a = reinterpret_cast<const double2*>(p)[0];
    const double2 b = reinterpret_cast<const double2*>(p)[1];
    d[0] = a.x; d[1] = a.y; d[2] = b.x; d[3] = b.y;
  }
}

template <class T>
__device__ __forceinline__ void st4(T* p, const T (&d)[kVec]) {
  if (!FDTD_CHECK_PTR(p, (int)sizeof(T) * kVec)) return;   // bounds-checked build only
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(d[0], d[1], d[2], d[3]);
  } else {
    reinterpret_cast<double2*>(p)[0] = make_double2(d[0], d[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(d[2], d[3]);
  }
}

template <class T>
__device__ __forceinline__ void zero4(T (&d)[kVec]) {
#pragma unroll
  for (int j = 0; j < kVec; ++j) d[j] = T(0);
}

template <class T>
__device__ __forceinline__ void copy4(T (&d)[kVec], const T (&a)[kVec]) {
#pragma unroll
  for (int j = 0; j < kVec; ++j) d[j] = a[j];
}

// True when every cell of the vector and every neighbour it reads lies away
// from the CPML faces and the domain edges and plane z does not inject: the
// update is then the plain curl update (Taflove 3.29 / 3.30).
template <class T>
__device__ __forceinline__ bool interior(const State<T>& s, int z, int y, int x0, int t) {
  const int m = s.npml;
  return z >= m && z < s.nz - m && y >= m && y < s.ny - m && x0 >= m && x0 + kVec <= s.nx - m &&
         !injects(s, z, t);
}

// E at the vector and its +z, +y neighbours, and at x0 + kVec (the +x
// neighbour of the last cell).
template <class T> struct EVec {
  T ex[kVec], ey[kVec], ez[kVec];
  T exz[kVec], eyz[kVec];   // E(z+1)
  T exy[kVec], ezy[kVec];   // E(y+1)
  T eyn, ezn;               // ey, ez at x0 + kVec
};

// H^{n+1/2} at the vector and its -z, -y neighbours, and at x0 - 1.
template <class T> struct HVec {
  T hx[kVec], hy[kVec], hz[kVec];
  T hxz[kVec], hyz[kVec];   // H(z-1)
  T hxy[kVec], hzy[kVec];   // H(y-1)
  T hyp, hzp;               // hy, hz at x0 - 1
};

// Plain curl update of H for the four cells (all inside every range).
template <class T>
__device__ __forceinline__ void h_vec_interior(const State<T>& s, const EVec<T>& e,
                                               T (&hx)[kVec], T (&hy)[kVec], T (&hz)[kVec]) {
  using M = R<T>;
#pragma unroll
  for (int j = 0; j < kVec; ++j) {
    const T eyx = j + 1 < kVec ? e.ey[j + 1 < kVec ? j + 1 : j] : e.eyn;
    const T ezx = j + 1 < kVec ? e.ez[j + 1 < kVec ? j + 1 : j] : e.ezn;
    hx[j] = M::sub(hx[j], M::mul(s.db, M::sub(M::sub(e.ezy[j], e.ez[j]), M::sub(e.eyz[j], e.ey[j]))));
    hy[j] = M::sub(hy[j], M::mul(s.db, M::sub(M::sub(e.exz[j], e.ex[j]), M::sub(ezx, e.ez[j]))));
    hz[j] = M::sub(hz[j], M::mul(s.db, M::sub(M::sub(eyx, e.ey[j]), M::sub(e.exy[j], e.ex[j]))));
  }
}

// Plain curl update of E for the four cells.
template <class T>
__device__ __forceinline__ void e_vec_interior(const HVec<T>& h, const T (&ca)[kVec],
                                               const T (&cb)[kVec], T (&ex)[kVec],
                                               T (&ey)[kVec], T (&ez)[kVec]) {
  using M = R<T>;
#pragma unroll
  for (int j = 0; j < kVec; ++j) {
    const T hyx = j > 0 ? h.hy[j > 0 ? j - 1 : 0] : h.hyp;
    const T hzx = j > 0 ? h.hz[j > 0 ? j - 1 : 0] : h.hzp;
    ex[j] = M::add(M::mul(ex[j], ca[j]), M::mul(cb[j], M::sub(M::sub(h.hz[j], h.hzy[j]), M::sub(h.hy[j], h.hyz[j]))));
    ey[j] = M::add(M::mul(ey[j], ca[j]), M::mul(cb[j], M::sub(M::sub(h.hx[j], h.hxz[j]), M::sub(h.hz[j], hzx))));
    ez[j] = M::add(M::mul(ez[j], ca[j]), M::mul(cb[j], M::sub(M::sub(h.hy[j], hyx), M::sub(h.hx[j], h.hxy[j]))));
  }
}

// True when the only boundary term of the vector (for H and for E) is the
// z-face CPML: every cell inside both update ranges in x and y, away from
// the x and y faces, z inside [1, nz - 1) and in an H or E z face, no
// injection. The update is then the plain curl update plus the z-face
// terms, whose coefficients are uniform over the plane.
template <class T>
__device__ __forceinline__ bool zface_only(const State<T>& s, int z, int y, int x0, int t) {
  const int m = s.npml;
  return z >= 1 && z < s.nz - 1 && (z < m || z >= s.nz - m) && y >= m && y < s.ny - m && x0 >= m &&
         x0 + kVec <= s.nx - m && !injects(s, z, t);
}

// H update of a vector for which zface_only holds: the plain update, then
// the z-face terms in h_vec's order (cpml_h_down/up, cpu/field_updates.py:243-282).
// src3, src2: psi_Hyz, psi_Hxz of the vector (a staged copy of the source
// psi, or the source psi itself).
template <class T>
__device__ __forceinline__ void h_vec_zface(const State<T>& s, const EVec<T>& e, int z, int y, int x0,
                                            bool wpsi, const T* src3, const T* src2, T (&hx)[kVec],
                                            T (&hy)[kVec], T (&hz)[kVec]) {
  using M = R<T>;
  const int nz = s.nz, m = s.npml;
  h_vec_interior(s, e, hx, hy, hz);
  if (z < m - 1 || z >= nz - m) {
    const int side = z < m - 1 ? 0 : 1;
    const int q = side ? z - (nz - m) : z;
    const T b = s.prof[side ? BH_U : BH_D][q];
    const T c = s.prof[side ? CH_U : CH_D][q];
    const long long k = ((long long)q * s.ny + y) * s.pitch + x0;
    T p3[kVec], p2[kVec];
    ld4(p3, src3);
    ld4(p2, src2);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      p3[j] = M::add(M::mul(b, p3[j]), div_dx(s, M::mul(c, M::sub(e.exz[j], e.ex[j]))));   // psi_Hyz
      p2[j] = M::add(M::mul(b, p2[j]), div_dx(s, M::mul(c, M::sub(e.eyz[j], e.ey[j]))));   // psi_Hxz
      hy[j] = M::sub(hy[j], M::mul(s.dtm0, p3[j]));
      hx[j] = M::add(hx[j], M::mul(s.dtm0, p2[j]));
    }
    if (wpsi) { st4(s.pd.z[side][3] + k, p3); st4(s.pd.z[side][2] + k, p2); }
  }
}

// E update of a vector for which zface_only holds: the plain update, then
// the z-face terms in e_vec's order (cpml_e_down/up, cpu/field_updates.py:66-105).
// src1, src0: psi_Eyz, psi_Exz of the vector (staged or source).
template <class T>
__device__ __forceinline__ void e_vec_zface(const State<T>& s, const HVec<T>& h, const T (&ca)[kVec],
                                            const T (&cb)[kVec], int z, int y, int x0, const T* src1,
                                            const T* src0, T (&ex)[kVec], T (&ey)[kVec],
                                            T (&ez)[kVec]) {
  using M = R<T>;
  const int nz = s.nz, m = s.npml;
  e_vec_interior(h, ca, cb, ex, ey, ez);
  if (z < m || z >= nz - m) {   // z >= 1 holds (zface_only)
    const int side = z < m ? 0 : 1;
    const int q = side ? z - (nz - m) : z;
    const T b = s.prof[side ? BE_U : BE_D][q];
    const T c = s.prof[side ? CE_U : CE_D][q];
    const long long k = ((long long)q * s.ny + y) * s.pitch + x0;
    T p1[kVec], p0[kVec];
    ld4(p1, src1);
    ld4(p0, src0);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      const T cbdx = M::mul(cb[j], s.dx);
      p1[j] = M::add(M::mul(b, p1[j]), div_dx(s, M::mul(c, M::sub(h.hx[j], h.hxz[j]))));   // psi_Eyz
      p0[j] = M::add(M::mul(b, p0[j]), div_dx(s, M::mul(c, M::sub(h.hy[j], h.hyz[j]))));   // psi_Exz
      ey[j] = M::add(ey[j], M::mul(cbdx, p1[j]));
      ex[j] = M::sub(ex[j], M::mul(cbdx, p0[j]));
    }
    st4(s.pd.z[side][1] + k, p1);
    st4(s.pd.z[side][0] + k, p0);
  }
}

// L2 prefetch of the CPML auxiliaries h_vec (e_vec) will read for the vector
// at (z, y, x0): the same faces and addresses as their loads. Issued before
// the field loads, so that the psi loads, which follow the curl update, hit
// L2 instead of waiting a second DRAM round trip. No value changes.
template <class T>
__device__ __forceinline__ void prefetch_l2(const T* p) {
  asm volatile("prefetch.global.L2 [%0];\n" ::"l"(p));
}

template <class T>
__device__ __forceinline__ void h_psi_prefetch(const State<T>& s, int z, int y, int x0, bool zface = true) {
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  if (!(z < nz - 1 && y < ny - 1)) return;
  if (zface && (z < m - 1 || z >= nz - m)) {
    const int side = z < m - 1 ? 0 : 1;
    const long long k = ((long long)(side ? z - (nz - m) : z) * ny + y) * s.pitch + x0;
    prefetch_l2(s.ps.z[side][3] + k);
    prefetch_l2(s.ps.z[side][2] + k);
  }
  if (x0 <= nx - 2 && (x0 < m - 1 || x0 + kVec - 1 >= nx - m)) {
    const int side = x0 < m - 1 ? 0 : 1;
    const long long k = xpsi_index(s, z, y, side, x0);
    prefetch_l2(s.ps.x[side][3] + k);
    prefetch_l2(s.ps.x[side][2] + k);
  }
  if (y < m - 1 || y >= ny - m) {
    const int side = y < m - 1 ? 0 : 1;
    const long long k = ((long long)z * m + (side ? y - (ny - m) : y)) * s.pitch + x0;
    prefetch_l2(s.ps.y[side][2] + k);
    prefetch_l2(s.ps.y[side][3] + k);
  }
}

template <class T>
__device__ __forceinline__ void e_psi_prefetch(const State<T>& s, int z, int y, int x0, bool zface = true) {
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  if (!(z < nz - 1 && y < ny - 1)) return;
  if (zface && ((z >= 1 && z < m) || z >= nz - m)) {
    const int side = (z >= 1 && z < m) ? 0 : 1;
    const long long k = ((long long)(side ? z - (nz - m) : z) * ny + y) * s.pitch + x0;
    prefetch_l2(s.ps.z[side][1] + k);
    prefetch_l2(s.ps.z[side][0] + k);
  }
  if (x0 <= nx - 2 && (x0 < m || x0 + kVec - 1 >= nx - m)) {
    const int side = x0 < m ? 0 : 1;
    const long long k = xpsi_index(s, z, y, side, x0);
    prefetch_l2(s.ps.x[side][1] + k);
    prefetch_l2(s.ps.x[side][0] + k);
  }
  if ((y >= 1 && y < m) || y >= ny - m) {
    const int side = (y >= 1 && y < m) ? 0 : 1;
    const long long k = ((long long)z * m + (side ? y - (ny - m) : y)) * s.pitch + x0;
    prefetch_l2(s.ps.y[side][0] + k);
    prefetch_l2(s.ps.y[side][1] + k);
  }
}

// Complete H update of the vector at (z, y, x0..x0+3), any position.
// psi is read from s.ps and, when wpsi, written to s.pd.
template <class T>
__device__ __forceinline__ void h_vec(const State<T>& s, const EVec<T>& e, int z, int y, int x0,
                                      int t, bool wpsi, T (&hx)[kVec], T (&hy)[kVec],
                                      T (&hz)[kVec]) {
  using M = R<T>;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  T dey_z[kVec], dez_y[kVec], dex_z[kVec], dez_x[kVec], dex_y[kVec], dey_x[kVec];
  bool inb[kVec];
  const bool zyb = z < nz - 1 && y < ny - 1;
#pragma unroll
  for (int j = 0; j < kVec; ++j) {
    const T eyx = j + 1 < kVec ? e.ey[j + 1 < kVec ? j + 1 : j] : e.eyn;
    const T ezx = j + 1 < kVec ? e.ez[j + 1 < kVec ? j + 1 : j] : e.ezn;
    dey_z[j] = M::sub(e.eyz[j], e.ey[j]);
    dez_y[j] = M::sub(e.ezy[j], e.ez[j]);
    dex_z[j] = M::sub(e.exz[j], e.ex[j]);
    dez_x[j] = M::sub(ezx, e.ez[j]);
    dex_y[j] = M::sub(e.exy[j], e.ex[j]);
    dey_x[j] = M::sub(eyx, e.ey[j]);
    const int x = x0 + j;
    inb[j] = zyb && x < nx - 1;
    // Taflove 3.30 (cpu/field_updates.py:198-240)
    if (inb[j] && x >= 1) hx[j] = M::sub(hx[j], M::mul(s.db, M::sub(dez_y[j], dey_z[j])));
    if (inb[j] && y >= 1) hy[j] = M::sub(hy[j], M::mul(s.db, M::sub(dex_z[j], dez_x[j])));
    if (inb[j] && z >= 1) hz[j] = M::sub(hz[j], M::mul(s.db, M::sub(dey_x[j], dex_y[j])));
  }
  // z faces (cpml_h_down/up, cpu/field_updates.py:243-282)
  if (zyb && (z < m - 1 || z >= nz - m)) {
    const int side = z < m - 1 ? 0 : 1;
    const int q = side ? z - (nz - m) : z;
    const T b = s.prof[side ? BH_U : BH_D][q];
    const T c = s.prof[side ? CH_U : CH_D][q];
    const long long k = ((long long)q * ny + y) * s.pitch + x0;
    T p3[kVec], p2[kVec];
    ld4(p3, s.ps.z[side][3] + k);
    ld4(p2, s.ps.z[side][2] + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      if (!inb[j]) continue;
      p3[j] = M::add(M::mul(b, p3[j]), div_dx(s, M::mul(c, dex_z[j])));   // psi_Hyz
      p2[j] = M::add(M::mul(b, p2[j]), div_dx(s, M::mul(c, dey_z[j])));   // psi_Hxz
      hy[j] = M::sub(hy[j], M::mul(s.dtm0, p3[j]));
      hx[j] = M::add(hx[j], M::mul(s.dtm0, p2[j]));
    }
    if (wpsi) { st4(s.pd.z[side][3] + k, p3); st4(s.pd.z[side][2] + k, p2); }
  }
  // x faces (cpml_h_left/right, :285-324): the vector's psi is one aligned
  // vector of the face's row (xpsi_index); cells outside the face keep
  // their slot. A vector with no cell below nx - 1 has nothing to update.
  if (zyb && x0 <= nx - 2 && (x0 < m - 1 || x0 + kVec - 1 >= nx - m)) {
    const int side = x0 < m - 1 ? 0 : 1;   // no vector reaches both faces (nx >= 2 npml + 3)
    const long long k = xpsi_index(s, z, y, side, x0);
    T p3[kVec], p2[kVec];
    ld4(p3, s.ps.x[side][3] + k);
    ld4(p2, s.ps.x[side][2] + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      const int x = x0 + j;
      if (!inb[j] || !(side ? x >= nx - m : x < m - 1)) continue;
      const int q = side ? x - (nx - m) : x;
      const T b = s.prof[side ? BH_U : BH_D][q];
      const T c = s.prof[side ? CH_U : CH_D][q];
      p3[j] = M::add(M::mul(b, p3[j]), div_dx(s, M::mul(c, dey_x[j])));   // psi_Hzx
      p2[j] = M::add(M::mul(b, p2[j]), div_dx(s, M::mul(c, dez_x[j])));   // psi_Hyx
      hz[j] = M::sub(hz[j], M::mul(s.dtm0, p3[j]));
      hy[j] = M::add(hy[j], M::mul(s.dtm0, p2[j]));
    }
    if (wpsi) { st4(s.pd.x[side][3] + k, p3); st4(s.pd.x[side][2] + k, p2); }
  }
  // y faces (cpml_h_front/back, :327-366)
  if (zyb && (y < m - 1 || y >= ny - m)) {
    const int side = y < m - 1 ? 0 : 1;
    const int q = side ? y - (ny - m) : y;
    const T b = s.prof[side ? BH_U : BH_D][q];
    const T c = s.prof[side ? CH_U : CH_D][q];
    const long long k = ((long long)z * m + q) * s.pitch + x0;
    T p2[kVec], p3[kVec];
    ld4(p2, s.ps.y[side][2] + k);
    ld4(p3, s.ps.y[side][3] + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      if (!inb[j]) continue;
      p2[j] = M::add(M::mul(b, p2[j]), div_dx(s, M::mul(c, dez_y[j])));   // psi_Hxy
      p3[j] = M::add(M::mul(b, p3[j]), div_dx(s, M::mul(c, dex_y[j])));   // psi_Hzy
      hx[j] = M::sub(hx[j], M::mul(s.dtm0, p2[j]));
      hz[j] = M::add(hz[j], M::mul(s.dtm0, p3[j]));
    }
    if (wpsi) { st4(s.pd.y[side][2] + k, p2); st4(s.pd.y[side][3] + k, p3); }
  }
  // E-field injection into H on the whole plane (cpu/main_sim.py:147-150)
  if (injects(s, z, t)) {
    const long long k = ((long long)t * ny + y) * s.pitch + x0;
    T iey[kVec], iex[kVec];
    ld4(iey, s.inc_ey + k);
    ld4(iex, s.inc_ex + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      if (x0 + j >= nx) continue;
      hx[j] = M::add(hx[j], M::mul(s.db, iey[j]));
      hy[j] = M::sub(hy[j], M::mul(s.db, iex[j]));
    }
  }
}

// Complete E update of the vector at (z, y, x0..x0+3) from H^{n+1/2}.
template <class T>
__device__ __forceinline__ void e_vec(const State<T>& s, const HVec<T>& h, const T (&ca)[kVec],
                                      const T (&cb)[kVec], int z, int y, int x0, int t,
                                      bool wpsi, T (&ex)[kVec], T (&ey)[kVec], T (&ez)[kVec]) {
  using M = R<T>;
  const int nx = s.nx, ny = s.ny, nz = s.nz, m = s.npml;
  T dhz_y[kVec], dhy_z[kVec], dhx_z[kVec], dhz_x[kVec], dhx_y[kVec], dhy_x[kVec], cbdx[kVec];
  bool inb[kVec];
  const bool zyb = z < nz - 1 && y < ny - 1;
#pragma unroll
  for (int j = 0; j < kVec; ++j) {
    const T hyx = j > 0 ? h.hy[j > 0 ? j - 1 : 0] : h.hyp;
    const T hzx = j > 0 ? h.hz[j > 0 ? j - 1 : 0] : h.hzp;
    dhz_y[j] = M::sub(h.hz[j], h.hzy[j]);
    dhy_z[j] = M::sub(h.hy[j], h.hyz[j]);
    dhx_z[j] = M::sub(h.hx[j], h.hxz[j]);
    dhz_x[j] = M::sub(h.hz[j], hzx);
    dhx_y[j] = M::sub(h.hx[j], h.hxy[j]);
    dhy_x[j] = M::sub(h.hy[j], hyx);
    const int x = x0 + j;
    inb[j] = zyb && x < nx - 1;
    // Taflove 3.29 (cpu/field_updates.py:18-63)
    if (inb[j] && z >= 1 && y >= 1)
      ex[j] = M::add(M::mul(ex[j], ca[j]), M::mul(cb[j], M::sub(dhz_y[j], dhy_z[j])));
    if (inb[j] && z >= 1 && x >= 1)
      ey[j] = M::add(M::mul(ey[j], ca[j]), M::mul(cb[j], M::sub(dhx_z[j], dhz_x[j])));
    if (inb[j] && y >= 1 && x >= 1)
      ez[j] = M::add(M::mul(ez[j], ca[j]), M::mul(cb[j], M::sub(dhy_x[j], dhx_y[j])));
    cbdx[j] = M::mul(cb[j], s.dx);
  }
  // z faces (cpml_e_down/up, :66-105)
  if (zyb && ((z >= 1 && z < m) || z >= nz - m)) {
    const int side = (z >= 1 && z < m) ? 0 : 1;
    const int q = side ? z - (nz - m) : z;
    const T b = s.prof[side ? BE_U : BE_D][q];
    const T c = s.prof[side ? CE_U : CE_D][q];
    const long long k = ((long long)q * ny + y) * s.pitch + x0;
    T p1[kVec], p0[kVec];
    ld4(p1, s.ps.z[side][1] + k);
    ld4(p0, s.ps.z[side][0] + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      if (!inb[j]) continue;
      p1[j] = M::add(M::mul(b, p1[j]), div_dx(s, M::mul(c, dhx_z[j])));   // psi_Eyz
      p0[j] = M::add(M::mul(b, p0[j]), div_dx(s, M::mul(c, dhy_z[j])));   // psi_Exz
      ey[j] = M::add(ey[j], M::mul(cbdx[j], p1[j]));
      ex[j] = M::sub(ex[j], M::mul(cbdx[j], p0[j]));
    }
    if (wpsi) { st4(s.pd.z[side][1] + k, p1); st4(s.pd.z[side][0] + k, p0); }
  }
  // x faces (cpml_e_left/right, :108-148): one aligned psi vector per
  // face component, as for H
  if (zyb && x0 <= nx - 2 && (x0 < m || x0 + kVec - 1 >= nx - m)) {
    const int side = x0 < m ? 0 : 1;
    const long long k = xpsi_index(s, z, y, side, x0);
    T p1[kVec], p0[kVec];
    ld4(p1, s.ps.x[side][1] + k);
    ld4(p0, s.ps.x[side][0] + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      const int x = x0 + j;
      if (!inb[j] || !(side ? x >= nx - m : (x >= 1 && x < m))) continue;
      const int q = side ? x - (nx - m) : x;
      const T b = s.prof[side ? BE_U : BE_D][q];
      const T c = s.prof[side ? CE_U : CE_D][q];
      p1[j] = M::add(M::mul(b, p1[j]), div_dx(s, M::mul(c, dhy_x[j])));   // psi_Ezx
      p0[j] = M::add(M::mul(b, p0[j]), div_dx(s, M::mul(c, dhz_x[j])));   // psi_Eyx
      ez[j] = M::add(ez[j], M::mul(cbdx[j], p1[j]));
      ey[j] = M::sub(ey[j], M::mul(cbdx[j], p0[j]));
    }
    if (wpsi) { st4(s.pd.x[side][1] + k, p1); st4(s.pd.x[side][0] + k, p0); }
  }
  // y faces (cpml_e_front/back, :151-191)
  if (zyb && ((y >= 1 && y < m) || y >= ny - m)) {
    const int side = (y >= 1 && y < m) ? 0 : 1;
    const int q = side ? y - (ny - m) : y;
    const T b = s.prof[side ? BE_U : BE_D][q];
    const T c = s.prof[side ? CE_U : CE_D][q];
    const long long k = ((long long)z * m + q) * s.pitch + x0;
    T p0[kVec], p1[kVec];
    ld4(p0, s.ps.y[side][0] + k);
    ld4(p1, s.ps.y[side][1] + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      if (!inb[j]) continue;
      p0[j] = M::add(M::mul(b, p0[j]), div_dx(s, M::mul(c, dhz_y[j])));   // psi_Exy
      p1[j] = M::add(M::mul(b, p1[j]), div_dx(s, M::mul(c, dhx_y[j])));   // psi_Ezy
      ex[j] = M::add(ex[j], M::mul(cbdx[j], p0[j]));
      ez[j] = M::sub(ez[j], M::mul(cbdx[j], p1[j]));
    }
    if (wpsi) { st4(s.pd.y[side][0] + k, p0); st4(s.pd.y[side][1] + k, p1); }
  }
  // H-field injection into E on the whole plane (cpu/main_sim.py:158-161)
  if (injects(s, z, t)) {
    const long long k = ((long long)t * ny + y) * s.pitch + x0;
    T ihx[kVec], ihy[kVec];
    ld4(ihx, s.inc_hx + k);
    ld4(ihy, s.inc_hy + k);
#pragma unroll
    for (int j = 0; j < kVec; ++j) {
      if (x0 + j >= nx) continue;
      ey[j] = M::add(ey[j], M::mul(s.dte0dx, ihx[j]));
      ex[j] = M::sub(ex[j], M::mul(s.dte0dx, ihy[j]));
    }
  }
}

}  // namespace fdtd
