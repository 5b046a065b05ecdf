// fdtd_tiles.cuh -- the bodies of the fused step's two z-marching tiles:
// interior_tile, shared by the single-simulation interior kernel
// (fdtd_fused.cu: k_fused_interior) and the batched tile-queue kernel
// (fdtd_batch.cu); march_tile, the body of the shell march (fdtd_march.cu).
//
// interior_tile: a tile of the interior box, the plain curl updates only
// (no CPML face, edge or injection touches it or its recomputed halo).
// march_tile: a tile of a shell box, every boundary term in the march.
// Both read the source field set and write the destination set; the
// descriptions of the marches are in fdtd_fused.cu and fdtd_march.cu.
#pragma once

#include "fdtd_vec.cuh"

namespace fdtd {

constexpr unsigned kFullMask = 0xffffffffu;
constexpr int kLanes = 32;
constexpr int kRowCells = kLanes * kVec;   // x cells of one interior tile row

// One tile of the interior box: tile (bx, by) of the x-y box and z chunk
// bz, by 32 x (TY + 1) threads (lane, row r). sEx, sEz, sHx, sHz: shared
// arrays of (TY + 1) * 128 elements each: E(z) of every thread row (read by
// the row below as its +y neighbour) and H^{n+1/2}(z) (read by the row
// above as its -y neighbour).
template <class T, int TY>
__device__ __forceinline__ void interior_tile(const State<T>& s, const InteriorBox& ib, int lane, int r,
                                              int bx, int by, int bz, T* sEx, T* sEz, T* sHx, T* sHz) {
  using M = R<T>;
  const int x0 = ib.xa + bx * kRowCells + lane * kVec;
  const int y = ib.ya + by * TY + r - 1;   // row 0 is the row below the tile
  int c = bz, k = 0;
  if (c >= ib.chunks0) { c -= ib.chunks0; k = 1; }
  const int z0 = ib.z0[k] + c * ib.zchunk;
  const int z1 = min(ib.z1[k], z0 + ib.zchunk);
  const int zs = z0 - 1;                           // plane below the chunk (interior)
  // Rows from ya - 1 >= 0 up; rows past the grid and lanes past the pitch
  // only feed the shared-memory exchange and the shuffles (as zeros).
  const bool vin = x0 < s.pitch && y < s.ny;
  const bool own = vin && r >= 1 && y < ib.yb && x0 < ib.xb;
  const long long P = s.plane, W = s.pitch;
  long long i = (long long)zs * P + (vin ? (long long)y * W + x0 : 0);
  const int so = lane * kVec;
  // shared indices of this thread (checked build: a bad one skips the
  // thread's shared accesses; the constant true otherwise)
  const bool sm_ok = FDTD_CHECK_SMEM(r * kRowCells + so + kVec - 1, (TY + 1) * kRowCells) &&
                     FDTD_CHECK_SMEM(r * kRowCells + so, (TY + 1) * kRowCells);

  EVec<T> e;
  HVec<T> h;
  T ezz[kVec];   // Ez(z+1)
  if (vin) { ld4(e.ex, s.iex + i); ld4(e.ey, s.iey + i); ld4(e.ez, s.iez + i); }
  else { zero4(e.ex); zero4(e.ey); zero4(e.ez); }
  zero4(h.hxz); zero4(h.hyz);

  for (int z = zs; z < z1; ++z, i += P) {
    const bool work = own && z >= z0;   // this thread updates and stores plane z
    // ---- loads of plane z (z + 1 < nz: the interior ends npml planes below the top)
    if (vin) {
      ld4(e.exz, s.iex + i + P); ld4(e.eyz, s.iey + i + P); ld4(ezz, s.iez + i + P);
      ld4(h.hx, s.ihx + i); ld4(h.hy, s.ihy + i); ld4(h.hz, s.ihz + i);
    } else {
      zero4(e.exz); zero4(e.eyz); zero4(ezz); zero4(h.hx); zero4(h.hy); zero4(h.hz);
    }
    T ca[kVec], cb[kVec];
    if (work) { ld4(ca, s.ca + i); ld4(cb, s.cb + i); }
    else { zero4(ca); zero4(cb); }
    if (r == TY) {   // +y neighbour of the top row lies in the next tile
      if (vin && y + 1 < s.ny) { ld4(e.exy, s.iex + i + W); ld4(e.ezy, s.iez + i + W); }
      else { zero4(e.exy); zero4(e.ezy); }
    }
    T eyr = T(0), ezr = T(0);   // +x neighbour of lane 31 lies in the next tile
    if (lane == kLanes - 1 && vin && x0 + kVec < s.pitch) { eyr = ldc(s.iey + (i + kVec)); ezr = ldc(s.iez + (i + kVec)); }
    // lane 0: the source values that H^{n+1/2} at (z, y, x0 - 1) needs
    // (x0 - 1 >= xa - 1 >= 0; z + 1 and y + 1 lie inside the grid)
    T gx = T(0), gy = T(0), gz = T(0), gxz = T(0), gxy = T(0), ghy = T(0), ghz = T(0);
    if (work && lane == 0) {
      const long long j = i - 1;
      gx = ldc(s.iex + (j)); gy = ldc(s.iey + (j)); gz = ldc(s.iez + (j));
      ghy = ldc(s.ihy + (j)); ghz = ldc(s.ihz + (j));
      gxz = ldc(s.iex + (j + P)); gxy = ldc(s.iex + (j + W));
    }
    // ---- H^{n+1/2}(z) -----------------------------------------------------
    if (sm_ok) { st4(&sEx[r * kRowCells + so], e.ex); st4(&sEz[r * kRowCells + so], e.ez); }
    __syncthreads();
    if (r < TY) {
      if (sm_ok) { ld4(e.exy, &sEx[(r + 1) * kRowCells + so]); ld4(e.ezy, &sEz[(r + 1) * kRowCells + so]); }
      else { zero4(e.exy); zero4(e.ezy); }
    }
    e.eyn = __shfl_down_sync(kFullMask, e.ey[0], 1);
    e.ezn = __shfl_down_sync(kFullMask, e.ez[0], 1);
    if (lane == kLanes - 1) { e.eyn = eyr; e.ezn = ezr; }
    h_vec_interior(s, e, h.hx, h.hy, h.hz);
    if (sm_ok) { st4(&sHx[r * kRowCells + so], h.hx); st4(&sHz[r * kRowCells + so], h.hz); }
    __syncthreads();
    // ---- E^{n+1}(z) ---------------------------------------------------------
    h.hyp = __shfl_up_sync(kFullMask, h.hy[kVec - 1], 1);
    h.hzp = __shfl_up_sync(kFullMask, h.hz[kVec - 1], 1);
    if (work) {
      if (sm_ok) { ld4(h.hxy, &sHx[(r - 1) * kRowCells + so]); ld4(h.hzy, &sHz[(r - 1) * kRowCells + so]); }
      else { zero4(h.hxy); zero4(h.hzy); }
      if (lane == 0) {   // Taflove 3.30 for hy, hz at x0 - 1 (an interior cell)
        h.hyp = M::sub(ghy, M::mul(s.db, M::sub(M::sub(gxz, gx), M::sub(e.ez[0], gz))));
        h.hzp = M::sub(ghz, M::mul(s.db, M::sub(M::sub(e.ey[0], gy), M::sub(gxy, gx))));
      }
      e_vec_interior(h, ca, cb, e.ex, e.ey, e.ez);
      st4(s.ohx + i, h.hx); st4(s.ohy + i, h.hy); st4(s.ohz + i, h.hz);
      st4(s.oex + i, e.ex); st4(s.oey + i, e.ey); st4(s.oez + i, e.ez);
    }
    // ---- next plane: E(z+1) becomes E(z), H^{n+1/2}(z) becomes H(z-1) -----
    copy4(e.ex, e.exz); copy4(e.ey, e.eyz); copy4(e.ez, ezz);
    copy4(h.hxz, h.hx); copy4(h.hyz, h.hy);
  }
}


// One tile of a z-slab or column box (the slab march, fdtd_fused.cu): tile
// (bx, by) of the box's x-y tiling and z chunk bz, by 32 x (TY + 1)
// threads (lane, row r), the step being t. Plain planes take the interior
// march's update; planes in a z face, the domain's edge planes and the
// injection plane take the general one. sEx, sEz, sHx, sHz: shared arrays
// of (TY + 1) * 128 elements each, as interior_tile's.
template <class T, int TY>
__device__ __forceinline__ void slab_tile(const State<T>& s, const InteriorBox& ib, int t, int lane, int r,
                                          int bx, int by, int bz, T* sEx, T* sEz, T* sHx, T* sHz) {
  using M = R<T>;
  const int nz = s.nz, m = s.npml;
  const int x0 = ib.xa + bx * kRowCells + lane * kVec;
  const int y = ib.ya + by * TY + r - 1;
  int c = bz, k = 0;
  if (c >= ib.chunks0) { c -= ib.chunks0; k = 1; }
  const int z0 = ib.z0[k] + c * ib.zchunk;
  const int z1 = min(ib.z1[k], z0 + ib.zchunk);
  const int zs = max(z0 - 1, 0);   // a chunk at plane 0 has nothing below
  const bool vin = x0 < s.pitch && y < s.ny;
  const bool own = vin && r >= 1 && y < ib.yb && x0 < ib.xb;
  const long long P = s.plane, W = s.pitch;
  long long i = (long long)zs * P + (vin ? (long long)y * W + x0 : 0);
  const int so = lane * kVec;

  EVec<T> e;
  HVec<T> h;
  T ezz[kVec];
  if (vin) { ld4(e.ex, s.iex + i); ld4(e.ey, s.iey + i); ld4(e.ez, s.iez + i); }
  else { zero4(e.ex); zero4(e.ey); zero4(e.ez); }
  zero4(h.hxz); zero4(h.hyz);

  for (int z = zs; z < z1; ++z, i += P) {
    const bool work = own && z >= z0;
    if (z >= m && z < nz - m && !(z == s.tfsf_z && t < s.nt_inc)) {
      // a plane with no z face, no domain edge and no injection: the
      // interior march's plain update (the same operations as below, with
      // every plane-dependent term absent)
      if (vin) {
        ld4(e.exz, s.iex + i + P); ld4(e.eyz, s.iey + i + P); ld4(ezz, s.iez + i + P);
        ld4(h.hx, s.ihx + i); ld4(h.hy, s.ihy + i); ld4(h.hz, s.ihz + i);
      } else {
        zero4(e.exz); zero4(e.eyz); zero4(ezz); zero4(h.hx); zero4(h.hy); zero4(h.hz);
      }
      T ca[kVec], cb[kVec];
      if (work) { ld4(ca, s.ca + i); ld4(cb, s.cb + i); }
      else { zero4(ca); zero4(cb); }
      if (r == TY) {
        if (vin && y + 1 < s.ny) { ld4(e.exy, s.iex + i + W); ld4(e.ezy, s.iez + i + W); }
        else { zero4(e.exy); zero4(e.ezy); }
      }
      T eyr = T(0), ezr = T(0);
      if (lane == kLanes - 1 && vin && x0 + kVec < s.pitch) { eyr = ldc(s.iey + (i + kVec)); ezr = ldc(s.iez + (i + kVec)); }
      T gx = T(0), gy = T(0), gz = T(0), gxz = T(0), gxy = T(0), ghy = T(0), ghz = T(0);
      if (work && lane == 0) {
        const long long j = i - 1;
        gx = ldc(s.iex + (j)); gy = ldc(s.iey + (j)); gz = ldc(s.iez + (j));
        ghy = ldc(s.ihy + (j)); ghz = ldc(s.ihz + (j));
        gxz = ldc(s.iex + (j + P)); gxy = ldc(s.iex + (j + W));
      }
      st4(&sEx[r * kRowCells + so], e.ex);
      st4(&sEz[r * kRowCells + so], e.ez);
      __syncthreads();
      if (r < TY) { ld4(e.exy, &sEx[(r + 1) * kRowCells + so]); ld4(e.ezy, &sEz[(r + 1) * kRowCells + so]); }
      e.eyn = __shfl_down_sync(kFullMask, e.ey[0], 1);
      e.ezn = __shfl_down_sync(kFullMask, e.ez[0], 1);
      if (lane == kLanes - 1) { e.eyn = eyr; e.ezn = ezr; }
      h_vec_interior(s, e, h.hx, h.hy, h.hz);
      st4(&sHx[r * kRowCells + so], h.hx);
      st4(&sHz[r * kRowCells + so], h.hz);
      __syncthreads();
      h.hyp = __shfl_up_sync(kFullMask, h.hy[kVec - 1], 1);
      h.hzp = __shfl_up_sync(kFullMask, h.hz[kVec - 1], 1);
      if (work) {
        ld4(h.hxy, &sHx[(r - 1) * kRowCells + so]);
        ld4(h.hzy, &sHz[(r - 1) * kRowCells + so]);
        if (lane == 0) {
          h.hyp = M::sub(ghy, M::mul(s.db, M::sub(M::sub(gxz, gx), M::sub(e.ez[0], gz))));
          h.hzp = M::sub(ghz, M::mul(s.db, M::sub(M::sub(e.ey[0], gy), M::sub(gxy, gx))));
        }
        e_vec_interior(h, ca, cb, e.ex, e.ey, e.ez);
        st4(s.ohx + i, h.hx); st4(s.ohy + i, h.hy); st4(s.ohz + i, h.hz);
        st4(s.oex + i, e.ex); st4(s.oey + i, e.ey); st4(s.oez + i, e.ez);
      }
      copy4(e.ex, e.exz); copy4(e.ey, e.eyz); copy4(e.ez, ezz);
      copy4(h.hxz, h.hx); copy4(h.hyz, h.hy);
      continue;
    }
    const bool top = z + 1 >= nz;   // last plane: nothing above, nothing updated
    // update ranges and CPML faces of plane z (uniform over the plane)
    const bool h_xy = z < nz - 1, h_z = z >= 1 && z < nz - 1;
    const bool e_xy = z >= 1 && z < nz - 1, e_z = z < nz - 1;
    const bool hf = z < nz - 1 && (z < m - 1 || z >= nz - m);
    const bool ef = z < nz - 1 && ((z >= 1 && z < m) || z >= nz - m);
    const int hside = z < m - 1 ? 0 : 1, hq = hside ? z - (nz - m) : z;
    const int eside = z < m ? 0 : 1, eq = eside ? z - (nz - m) : z;
    const bool inj = z == s.tfsf_z && t < s.nt_inc;   // injection plane
    const long long ki = ((long long)t * s.ny + y) * W + x0;   // incident planes (t, y, x)
    if (vin && !top) {
      ld4(e.exz, s.iex + i + P); ld4(e.eyz, s.iey + i + P); ld4(ezz, s.iez + i + P);
    } else {
      zero4(e.exz); zero4(e.eyz); zero4(ezz);
    }
    if (vin) { ld4(h.hx, s.ihx + i); ld4(h.hy, s.ihy + i); ld4(h.hz, s.ihz + i); }
    else { zero4(h.hx); zero4(h.hy); zero4(h.hz); }
    T ca[kVec], cb[kVec];
    if (work) { ld4(ca, s.ca + i); ld4(cb, s.cb + i); }
    else { zero4(ca); zero4(cb); }
    if (r == TY) {
      if (vin && y + 1 < s.ny) { ld4(e.exy, s.iex + i + W); ld4(e.ezy, s.iez + i + W); }
      else { zero4(e.exy); zero4(e.ezy); }
    }
    T eyr = T(0), ezr = T(0);
    if (lane == kLanes - 1 && vin && x0 + kVec < s.pitch) { eyr = ldc(s.iey + (i + kVec)); ezr = ldc(s.iez + (i + kVec)); }
    T gx = T(0), gy = T(0), gz = T(0), gxz = T(0), gxy = T(0), ghy = T(0), ghz = T(0), gpy = T(0), gix = T(0);
    if (work && lane == 0) {
      const long long j = i - 1;
      gx = ldc(s.iex + (j)); gy = ldc(s.iey + (j)); gz = ldc(s.iez + (j));
      ghy = ldc(s.ihy + (j)); ghz = ldc(s.ihz + (j));
      gxz = top ? T(0) : ldc(s.iex + (j + P));
      gxy = ldc(s.iex + (j + W));
      if (hf) gpy = ldc(s.ps.z[hside][3] + (((long long)hq * s.ny + y) * W + x0 - 1));
      if (inj) gix = ldc(s.inc_ex + (ki - 1));
    }
    // ---- H^{n+1/2}(z) -----------------------------------------------------
    st4(&sEx[r * kRowCells + so], e.ex);
    st4(&sEz[r * kRowCells + so], e.ez);
    __syncthreads();
    if (r < TY) { ld4(e.exy, &sEx[(r + 1) * kRowCells + so]); ld4(e.ezy, &sEz[(r + 1) * kRowCells + so]); }
    e.eyn = __shfl_down_sync(kFullMask, e.ey[0], 1);
    e.ezn = __shfl_down_sync(kFullMask, e.ez[0], 1);
    if (lane == kLanes - 1) { e.eyn = eyr; e.ezn = ezr; }
    {
      T hx[kVec], hy[kVec], hz[kVec];
      copy4(hx, h.hx); copy4(hy, h.hy); copy4(hz, h.hz);
      h_vec_interior(s, e, hx, hy, hz);
      if (h_xy) { copy4(h.hx, hx); copy4(h.hy, hy); }
      if (h_z) copy4(h.hz, hz);
    }
    if (hf) {   // z faces: psi_Hyz from dEx/dz, psi_Hxz from dEy/dz
      const long long kq = ((long long)hq * s.ny + y) * W + x0;
      const T b = s.prof[hside ? BH_U : BH_D][hq];
      const T c = s.prof[hside ? CH_U : CH_D][hq];
      T p3[kVec], p2[kVec];
      if (vin) { ld4(p3, s.ps.z[hside][3] + kq); ld4(p2, s.ps.z[hside][2] + kq); }
      else { zero4(p3); zero4(p2); }
#pragma unroll
      for (int j = 0; j < kVec; ++j) {
        p3[j] = M::add(M::mul(b, p3[j]), div_dx(s, M::mul(c, M::sub(e.exz[j], e.ex[j]))));
        p2[j] = M::add(M::mul(b, p2[j]), div_dx(s, M::mul(c, M::sub(e.eyz[j], e.ey[j]))));
        h.hy[j] = M::sub(h.hy[j], M::mul(s.dtm0, p3[j]));
        h.hx[j] = M::add(h.hx[j], M::mul(s.dtm0, p2[j]));
      }
      if (work) { st4(s.pd.z[hside][3] + kq, p3); st4(s.pd.z[hside][2] + kq, p2); }
    }
    if (inj) {   // E-field injection into H (cpu/main_sim.py:147-150)
      T iey[kVec], iex[kVec];
      if (vin) { ld4(iey, s.inc_ey + ki); ld4(iex, s.inc_ex + ki); }
      else { zero4(iey); zero4(iex); }
#pragma unroll
      for (int j = 0; j < kVec; ++j) {
        if (x0 + j >= s.nx) continue;
        h.hx[j] = M::add(h.hx[j], M::mul(s.db, iey[j]));
        h.hy[j] = M::sub(h.hy[j], M::mul(s.db, iex[j]));
      }
    }
    st4(&sHx[r * kRowCells + so], h.hx);
    st4(&sHz[r * kRowCells + so], h.hz);
    __syncthreads();
    // ---- E^{n+1}(z) ---------------------------------------------------------
    h.hyp = __shfl_up_sync(kFullMask, h.hy[kVec - 1], 1);
    h.hzp = __shfl_up_sync(kFullMask, h.hz[kVec - 1], 1);
    if (work) {
      ld4(h.hxy, &sHx[(r - 1) * kRowCells + so]);
      ld4(h.hzy, &sHz[(r - 1) * kRowCells + so]);
      if (lane == 0) {   // hy, hz at x0 - 1, with the z-face term of hy
        T hyp = ghy, hzp = ghz;
        if (h_xy) {
          hyp = M::sub(ghy, M::mul(s.db, M::sub(M::sub(gxz, gx), M::sub(e.ez[0], gz))));
          if (hf) {
            const T b = s.prof[hside ? BH_U : BH_D][hq];
            const T c = s.prof[hside ? CH_U : CH_D][hq];
            const T p3 = M::add(M::mul(b, gpy), div_dx(s, M::mul(c, M::sub(gxz, gx))));
            hyp = M::sub(hyp, M::mul(s.dtm0, p3));
          }
        }
        if (inj) hyp = M::sub(hyp, M::mul(s.db, gix));
        if (h_z) hzp = M::sub(ghz, M::mul(s.db, M::sub(M::sub(e.ey[0], gy), M::sub(gxy, gx))));
        h.hyp = hyp;
        h.hzp = hzp;
      }
      T ex[kVec], ey[kVec], ez[kVec];
      copy4(ex, e.ex); copy4(ey, e.ey); copy4(ez, e.ez);
      e_vec_interior(h, ca, cb, ex, ey, ez);
      T ox[kVec], oy[kVec], oz[kVec];
      copy4(ox, e.ex); copy4(oy, e.ey); copy4(oz, e.ez);
      if (e_xy) { copy4(ox, ex); copy4(oy, ey); }
      if (e_z) copy4(oz, ez);
      if (ef) {   // z faces: psi_Eyz from dHx/dz, psi_Exz from dHy/dz
        const long long kq = ((long long)eq * s.ny + y) * W + x0;
        const T b = s.prof[eside ? BE_U : BE_D][eq];
        const T c = s.prof[eside ? CE_U : CE_D][eq];
        T p1[kVec], p0[kVec];
        ld4(p1, s.ps.z[eside][1] + kq);
        ld4(p0, s.ps.z[eside][0] + kq);
#pragma unroll
        for (int j = 0; j < kVec; ++j) {
          const T cbdx = M::mul(cb[j], s.dx);
          p1[j] = M::add(M::mul(b, p1[j]), div_dx(s, M::mul(c, M::sub(h.hx[j], h.hxz[j]))));
          p0[j] = M::add(M::mul(b, p0[j]), div_dx(s, M::mul(c, M::sub(h.hy[j], h.hyz[j]))));
          oy[j] = M::add(oy[j], M::mul(cbdx, p1[j]));
          ox[j] = M::sub(ox[j], M::mul(cbdx, p0[j]));
        }
        st4(s.pd.z[eside][1] + kq, p1);
        st4(s.pd.z[eside][0] + kq, p0);
      }
      if (inj) {   // H-field injection into E (cpu/main_sim.py:158-161)
        T ihx[kVec], ihy[kVec];
        ld4(ihx, s.inc_hx + ki);
        ld4(ihy, s.inc_hy + ki);
#pragma unroll
        for (int j = 0; j < kVec; ++j) {
          if (x0 + j >= s.nx) continue;
          oy[j] = M::add(oy[j], M::mul(s.dte0dx, ihx[j]));
          ox[j] = M::sub(ox[j], M::mul(s.dte0dx, ihy[j]));
        }
      }
      st4(s.ohx + i, h.hx); st4(s.ohy + i, h.hy); st4(s.ohz + i, h.hz);
      st4(s.oex + i, ox); st4(s.oey + i, oy); st4(s.oez + i, oz);
    }
    copy4(e.ex, e.exz); copy4(e.ey, e.eyz); copy4(e.ez, ezz);
    copy4(h.hxz, h.hx); copy4(h.hyz, h.hy);
  }
}

// Dynamic shared memory of a march tile, in elements of T: the four
// exchange arrays, then two stages of the per-thread staging area. A stage
// holds, per thread, kSlots vectors (E(z+1) x, y, z; H(z) x, y, z; Ca, Cb;
// the z-face psi Hyz, Hxz, Eyz, Exz), then the top row's
// E(y+1) x, z (32 lanes at most) and the last lane's E(x+4) y, z (one pair
// per row).
template <class T>
struct MarchSmem {
  static constexpr int kEx = kMarchThreads * kVec;
  static constexpr int kSlots = 12;
  static constexpr int kMain = kSlots * kMarchThreads * kVec;
  static constexpr int kTop = 2 * 32 * kVec;
  static constexpr int kRight = 2 * (kMarchThreads / 8);
  static constexpr int kStage = (kMain + kTop + kRight + 7) / 8 * 8;   // keeps 32-byte alignment
  static constexpr size_t kBytes = (size_t)(4 * kEx + 2 * kStage) * sizeof(T);
};

// Asynchronous global -> shared copies (cp.async): a 4-element vector
// (16 or 32 bytes) and one element; an invalid copy reads nothing and fills
// zeros (its source is any valid address).
template <class T>
__device__ __forceinline__ void cp_vec(T* dst, const T* src, bool valid) {
  if (valid && !FDTD_CHECK_PTR(src, (int)sizeof(T) * kVec)) valid = false;   // checked build
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
#pragma unroll
  for (int k = 0; k < (int)(sizeof(T) * kVec / 16); ++k)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(sa + 16 * k),
                 "l"(reinterpret_cast<const char*>(src) + 16 * k), "r"(n)
                 : "memory");
}
template <class T>
__device__ __forceinline__ void cp_elem(T* dst, const T* src, bool valid) {
  if (valid && !FDTD_CHECK_PTR(src, (int)sizeof(T))) valid = false;   // checked build
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? (int)sizeof(T) : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(src), "n"((int)sizeof(T)),
               "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// One tile of a march box: tile (bx, by) of the box's x-y tiling and z
// chunk c, by kMarchThreads threads, the step being t. smem: the
// MarchSmem<T> area (exchange arrays, then two stages). The z-face psi is
// staged with the rest of the plane (read from the source psi in the
// bounds-checked build when a shared index fails its check).
template <class T>
__device__ __forceinline__ void march_tile(const State<T>& s, const MarchBox& b, int bx, int by, int c, int t,
                                           T* smem) {
  using SM = MarchSmem<T>;
  // exchange arrays: E(z) of every row (read by the row below as its +y
  // neighbour) and H^{n+1/2}(z) (read by the row above as its -y
  // neighbour), indexed [(row * width + lane) * 4 + j]; then the stages
  T* const sEx = smem;
  T* const sEz = sEx + SM::kEx;
  T* const sHx = sEx + 2 * SM::kEx;
  T* const sHz = sEx + 3 * SM::kEx;
  T* const stage0 = sEx + 4 * SM::kEx;
  const int width = b.width, rows = kMarchThreads / width;
  const int lane = threadIdx.x % width, r = threadIdx.x / width;
  // own vectors start at vector `first_own` of the box; a halo lane 0 sits
  // one vector before
  const int halo = (bx == 0 && b.x0 == 0) ? 0 : 1;
  const int first_own = bx == 0 ? 0 : b.lead + (bx - 1) * (width - 1);
  const int x0 = b.x0 + (first_own + lane - halo) * kVec;
  const int y = b.y0 + by * (rows - 1) + r - 1;   // row 0 is the row below the tile
  const int z0 = b.z0 + c * b.zchunk;
  const int z1 = min(b.z1, z0 + b.zchunk);
  const int zs = max(z0 - 1, 0);                  // the plane below the chunk, if any
  const int ny = s.ny, nz = s.nz, m = s.npml;
  // Rows outside the grid and lanes past the pitch only feed the shared
  // memory exchange and the shuffles (as zeros).
  const bool vin = x0 >= 0 && x0 < s.pitch && y >= 0 && y < ny;
  const bool own = vin && r >= 1 && lane >= halo && y < b.y1 && x0 < b.x1;
  const long long P = s.plane, W = s.pitch;
  const long long base = vin ? (long long)y * W + x0 : 0;
  const int so = threadIdx.x * kVec;
  const int su = so + width * kVec;   // the next row's slot
  const int sd = so - width * kVec;   // the previous row's slot
  const bool top_row = r == rows - 1, last_lane = lane == width - 1;
  // shared indices of this thread (checked build: a bad one skips the
  // thread's shared accesses; the constant true otherwise)
  const bool sm_ok = FDTD_CHECK_SMEM(so + kVec - 1, SM::kEx) &&
                     (top_row || FDTD_CHECK_SMEM(su + kVec - 1, SM::kEx)) && (r == 0 || FDTD_CHECK_SMEM(sd, SM::kEx)) &&
                     FDTD_CHECK_SMEM((SM::kSlots - 1) * SM::kEx + so + kVec - 1, SM::kMain) &&
                     (!top_row || FDTD_CHECK_SMEM(SM::kMain + (32 + lane) * kVec + kVec - 1, SM::kStage)) &&
                     (!last_lane || FDTD_CHECK_SMEM(SM::kMain + SM::kTop + 2 * r + 1, SM::kStage));

  auto slot = [&](int st, int k) { return stage0 + st * SM::kStage + k * SM::kEx + so; };
  auto top = [&](int st, int k) { return stage0 + st * SM::kStage + SM::kMain + (k * 32 + lane) * kVec; };
  auto right = [&](int st) { return stage0 + st * SM::kStage + SM::kMain + SM::kTop + 2 * r; };

  // Stage st <- what plane zz's update reads from global memory.
  auto issue = [&](int zz, int st) {
    if (!sm_ok) return;
    const long long i = (long long)zz * P + base;
    const bool a = vin && zz + 1 < nz;
    cp_vec(slot(st, 0), a ? s.iex + i + P : s.iex, a);
    cp_vec(slot(st, 1), a ? s.iey + i + P : s.iey, a);
    cp_vec(slot(st, 2), a ? s.iez + i + P : s.iez, a);
    cp_vec(slot(st, 3), vin ? s.ihx + i : s.ihx, vin);
    cp_vec(slot(st, 4), vin ? s.ihy + i : s.ihy, vin);
    cp_vec(slot(st, 5), vin ? s.ihz + i : s.ihz, vin);
    const bool w = own && zz >= z0;
    cp_vec(slot(st, 6), w ? s.ca + i : s.ca, w);
    cp_vec(slot(st, 7), w ? s.cb + i : s.cb, w);
    // z-face psi of plane zz (H: q < npml - 1 below, the top npml planes;
    // E: 1 <= q < npml below, the top npml planes)
    const bool hf = vin && (zz < m - 1 || zz >= nz - m);
    const bool ef = vin && ((zz >= 1 && zz < m) || zz >= nz - m);
    const int hsd = zz < m - 1 ? 0 : 1, esd = zz < m ? 0 : 1;
    const long long kh = ((long long)(hsd ? zz - (nz - m) : zz) * ny + y) * W + x0;
    const long long ke = ((long long)(esd ? zz - (nz - m) : zz) * ny + y) * W + x0;
    {
      const T* p0 = s.ps.z[0][0];
      cp_vec(slot(st, 8), hf ? s.ps.z[hsd][3] + kh : p0, hf);
      cp_vec(slot(st, 9), hf ? s.ps.z[hsd][2] + kh : p0, hf);
      cp_vec(slot(st, 10), ef ? s.ps.z[esd][1] + ke : p0, ef);
      cp_vec(slot(st, 11), ef ? s.ps.z[esd][0] + ke : p0, ef);
    }
    if (top_row) {   // +y neighbour of the top row lies in the next tile
      const bool v = vin && y + 1 < ny;
      cp_vec(top(st, 0), v ? s.iex + i + W : s.iex, v);
      cp_vec(top(st, 1), v ? s.iez + i + W : s.iez, v);
    }
    if (last_lane) {   // +x neighbour of the last lane lies in the next tile
      const bool v = vin && x0 + kVec < s.pitch;
      cp_elem(right(st), v ? s.iey + i + kVec : s.iey, v);
      cp_elem(right(st) + 1, v ? s.iez + i + kVec : s.iez, v);
    }
    // the CPML auxiliaries the generic update of plane zz reads from global
    // memory (x and y faces) go to L2 a plane ahead
    if (own && zz >= z0) {
      h_psi_prefetch(s, zz, y, x0, false);
      e_psi_prefetch(s, zz, y, x0, false);
    }
  };

  EVec<T> e;
  HVec<T> h;
  T ezz[kVec];   // Ez(z+1)
  issue(zs, 0);
  cp_commit();
  {
    const long long i = (long long)zs * P + base;
    if (vin) { ld4(e.ex, s.iex + i); ld4(e.ey, s.iey + i); ld4(e.ez, s.iez + i); }
    else { zero4(e.ex); zero4(e.ey); zero4(e.ez); }
  }
  zero4(h.hxz); zero4(h.hyz);

  long long i = (long long)zs * P + base;
  for (int z = zs; z < z1; ++z, i += P) {
    const int st = (z - zs) & 1;
    // the next plane's copies go out before this plane is computed
    if (z + 1 < z1) issue(z + 1, st ^ 1);
    cp_commit();
    cp_wait_prev();
    const bool work = own && z >= z0;   // this thread updates and stores plane z
    T ca[kVec], cb[kVec];
    T eyr = T(0), ezr = T(0);
    if (sm_ok) {
      ld4(e.exz, slot(st, 0)); ld4(e.eyz, slot(st, 1)); ld4(ezz, slot(st, 2));
      ld4(h.hx, slot(st, 3)); ld4(h.hy, slot(st, 4)); ld4(h.hz, slot(st, 5));
      ld4(ca, slot(st, 6)); ld4(cb, slot(st, 7));
      if (top_row) { ld4(e.exy, top(st, 0)); ld4(e.ezy, top(st, 1)); }
      if (last_lane) { eyr = right(st)[0]; ezr = right(st)[1]; }
    } else {
      zero4(e.exz); zero4(e.eyz); zero4(ezz); zero4(h.hx); zero4(h.hy); zero4(h.hz);
      zero4(ca); zero4(cb); zero4(e.exy); zero4(e.ezy);
    }
    // ---- H^{n+1/2}(z) -----------------------------------------------------
    if (sm_ok) { st4(&sEx[so], e.ex); st4(&sEz[so], e.ez); }
    __syncthreads();
    if (!top_row) {
      if (sm_ok) { ld4(e.exy, &sEx[su]); ld4(e.ezy, &sEz[su]); }
      else { zero4(e.exy); zero4(e.ezy); }
    }
    e.eyn = __shfl_down_sync(kFullMask, e.ey[0], 1, width);
    e.ezn = __shfl_down_sync(kFullMask, e.ez[0], 1, width);
    if (last_lane) { e.eyn = eyr; e.ezn = ezr; }
    // warp-uniform paths: every vector of the warp a plain interior vector
    // (for H and for E), or one whose only boundary term is the z face
    const bool plain_h = __all_sync(kFullMask, !vin || interior(s, z, y, x0, t));
    const bool zface_h = !plain_h && __all_sync(kFullMask, !vin || zface_only(s, z, y, x0, t));
    if (vin) {
      if (plain_h) h_vec_interior(s, e, h.hx, h.hy, h.hz);
      else if (zface_h) {
        if (sm_ok) {
          h_vec_zface(s, e, z, y, x0, work, slot(st, 8), slot(st, 9), h.hx, h.hy, h.hz);
        } else {
          const int sd_ = z < m - 1 ? 0 : 1;
          const long long kq = ((long long)(sd_ ? z - (nz - m) : z) * ny + y) * W + x0;
          h_vec_zface(s, e, z, y, x0, work, s.ps.z[sd_][3] + kq, s.ps.z[sd_][2] + kq, h.hx, h.hy, h.hz);
        }
      }
      else h_vec(s, e, z, y, x0, t, work, h.hx, h.hy, h.hz);
    }
    if (sm_ok) { st4(&sHx[so], h.hx); st4(&sHz[so], h.hz); }
    __syncthreads();
    // ---- E^{n+1}(z) ---------------------------------------------------------
    h.hyp = __shfl_up_sync(kFullMask, h.hy[kVec - 1], 1, width);
    h.hzp = __shfl_up_sync(kFullMask, h.hz[kVec - 1], 1, width);
    if (lane == 0) {   // own only at x0 = 0, whose E update reads no x - 1 value
      h.hyp = T(0);
      h.hzp = T(0);
    }
    if (work) {
      if (sm_ok) { ld4(h.hxy, &sHx[sd]); ld4(h.hzy, &sHz[sd]); }
      else { zero4(h.hxy); zero4(h.hzy); }
      if (plain_h) e_vec_interior(h, ca, cb, e.ex, e.ey, e.ez);
      else if (zface_h) {
        if (sm_ok) {
          e_vec_zface(s, h, ca, cb, z, y, x0, slot(st, 10), slot(st, 11), e.ex, e.ey, e.ez);
        } else {
          const int sd_ = z < m ? 0 : 1;
          const long long kq = ((long long)(sd_ ? z - (nz - m) : z) * ny + y) * W + x0;
          e_vec_zface(s, h, ca, cb, z, y, x0, s.ps.z[sd_][1] + kq, s.ps.z[sd_][0] + kq, e.ex, e.ey, e.ez);
        }
      }
      else e_vec(s, h, ca, cb, z, y, x0, t, true, e.ex, e.ey, e.ez);
      st4(s.ohx + i, h.hx); st4(s.ohy + i, h.hy); st4(s.ohz + i, h.hz);
      st4(s.oex + i, e.ex); st4(s.oey + i, e.ey); st4(s.oez + i, e.ez);
    }
    // ---- next plane: E(z+1) becomes E(z), H^{n+1/2}(z) becomes H(z-1) -----
    copy4(e.ex, e.exz); copy4(e.ey, e.eyz); copy4(e.ez, ezz);
    copy4(h.hxz, h.hx); copy4(h.hyz, h.hy);
  }
  cp_wait_prev();   // nothing in flight at exit (the last group is empty)
}


}  // namespace fdtd
