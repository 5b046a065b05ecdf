// fdtd_fused.cu -- the fused step: H^{n+1/2} and E^{n+1} of the whole grid
// from the source field set into the destination set (ping-pong).
//
// Because every cell is written to a set that nothing reads during the
// step, any partition of the grid can be updated by independent kernels,
// each recomputing from the source set the few H^{n+1/2} values it needs
// from a neighbour region. The step uses two regions:
//
//  * the interior box, where no CPML face, domain edge or injection plane
//    touches a cell or the halo it recomputes (about 80 % of the cells at
//    the benchmark sizes): one z-marching pass that reads every field, Ca
//    and Cb once and writes every field once (56 B per FP32 cell-update),
//    with no boundary code at all, so nothing diverges and the kernel needs
//    few registers;
//  * the shell (CPML slabs, the injection planes, the strips beside the
//    interior box): the split H pass over the shell boxes (source E, H ->
//    destination H), then the split E pass (destination H, source E ->
//    destination E). The E pass runs after the interior pass, whose
//    destination H it reads at the shell's inner edge.
//
// Interior kernel. A block owns a tile of 128 x cells (32 lanes x 4 cells)
// by TY rows and a chunk of z planes, and marches up the chunk one plane at
// a time. At plane z a thread holds E(z) of its vector (carried from the
// previous plane), loads E(z+1), H(z), Ca, Cb, and
//   1. computes H^{n+1/2}(z) of its vector; the +x neighbour comes from the
//      next lane by shuffle, the +y neighbour from the next thread row
//      through shared memory, the +z neighbour is E(z+1);
//   2. computes E^{n+1}(z); the -x neighbour comes by shuffle, the -y
//      neighbour through shared memory, the -z neighbour is H^{n+1/2}(z-1)
//      carried in registers.
// Thread row 0 recomputes the row below the tile, lane 0 the column left of
// the tile (one cell per row), and the plane below a chunk is recomputed
// before the chunk. Per-cell values equal the split kernels' (the same
// update formula in the same order of operations).
#include <algorithm>
#include <cstring>

#include "fdtd_launch.h"
#include "fdtd_vec.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kLanes = 32;
constexpr int kRowCells = kLanes * kVec;   // x cells of one tile row

template <class T, int TY>
constexpr int interior_min_blocks() { return sizeof(T) == 4 && TY <= 8 ? 2 : 1; }

template <class T, int TY>
__global__ void __launch_bounds__(kLanes * (TY + 1), interior_min_blocks<T, TY>())
k_fused_interior(const __grid_constant__ State<T> s, InteriorBox ib) {
  using M = R<T>;
  // E(z) of every thread row (read by the row below as its +y neighbour)
  // and H^{n+1/2}(z) (read by the row above as its -y neighbour).
  __shared__ __align__(32) T sEx[TY + 1][kRowCells];
  __shared__ __align__(32) T sEz[TY + 1][kRowCells];
  __shared__ __align__(32) T sHx[TY + 1][kRowCells];
  __shared__ __align__(32) T sHz[TY + 1][kRowCells];

  const int lane = threadIdx.x, r = threadIdx.y;
  const int x0 = ib.xa + blockIdx.x * kRowCells + lane * kVec;
  const int y = ib.ya + blockIdx.y * TY + r - 1;   // row 0 is the row below the tile
  int c = blockIdx.z, k = 0;
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
    if (lane == kLanes - 1 && vin && x0 + kVec < s.pitch) { eyr = s.iey[i + kVec]; ezr = s.iez[i + kVec]; }
    // lane 0: the source values that H^{n+1/2} at (z, y, x0 - 1) needs
    // (x0 - 1 >= xa - 1 >= 0; z + 1 and y + 1 lie inside the grid)
    T gx = T(0), gy = T(0), gz = T(0), gxz = T(0), gxy = T(0), ghy = T(0), ghz = T(0);
    if (work && lane == 0) {
      const long long j = i - 1;
      gx = s.iex[j]; gy = s.iey[j]; gz = s.iez[j];
      ghy = s.ihy[j]; ghz = s.ihz[j];
      gxz = s.iex[j + P]; gxy = s.iex[j + W];
    }
    // ---- H^{n+1/2}(z) -----------------------------------------------------
    st4(&sEx[r][so], e.ex);
    st4(&sEz[r][so], e.ez);
    __syncthreads();
    if (r < TY) { ld4(e.exy, &sEx[r + 1][so]); ld4(e.ezy, &sEz[r + 1][so]); }
    e.eyn = __shfl_down_sync(kFull, e.ey[0], 1);
    e.ezn = __shfl_down_sync(kFull, e.ez[0], 1);
    if (lane == kLanes - 1) { e.eyn = eyr; e.ezn = ezr; }
    h_vec_interior(s, e, h.hx, h.hy, h.hz);
    st4(&sHx[r][so], h.hx);
    st4(&sHz[r][so], h.hz);
    __syncthreads();
    // ---- E^{n+1}(z) ---------------------------------------------------------
    h.hyp = __shfl_up_sync(kFull, h.hy[kVec - 1], 1);
    h.hzp = __shfl_up_sync(kFull, h.hz[kVec - 1], 1);
    if (work) {
      ld4(h.hxy, &sHx[r - 1][so]);
      ld4(h.hzy, &sHz[r - 1][so]);
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

template <class T, int TY>
void launch_interior_ty(const State<T>& s, const InteriorBox& ib, cudaStream_t st) {
  const dim3 blk(kLanes, TY + 1, 1);
  const dim3 grd((ib.xb - ib.xa + kRowCells - 1) / kRowCells, (ib.yb - ib.ya + TY - 1) / TY,
                 ib.chunks);
  k_fused_interior<T, TY><<<grd, blk, 0, st>>>(s, ib);
}

}  // namespace

bool fused_supported_tile(int tile_x, int tile_y, int elem_bytes) {
  if (tile_x != kLanes) return false;
  if (tile_y == 4 || tile_y == 7 || tile_y == 8) return true;
  return elem_bytes == 4 && (tile_y == 15 || tile_y == 16);
}

// The interior box keeps every cell and every recomputed halo cell away
// from the CPML faces (H faces cover q < npml - 1 below and the top npml
// planes; E faces 1 <= q < npml below), from the domain edges and from the
// injection plane tfsf_z (and tfsf_z + 1, whose recomputed plane below would
// be the injection plane).
FusedPlan make_fused_plan(int nx, int ny, int nz, int npml, int tfsf_z, int tile_y, int zchunk) {
  FusedPlan p;
  memset(&p, 0, sizeof(p));
  const int m = npml;
  InteriorBox& ib = p.interior;
  ib.xa = (m + 31) / 32 * 32;
  ib.xb = (nx - m) / kVec * kVec;
  ib.ya = m;
  ib.yb = ny - m;
  // interior z ranges: [m, nz - m) without tfsf_z, tfsf_z + 1
  int zr[2][2] = {{0, 0}, {0, 0}}, nzr = 0;
  const int za = m, zb = nz - m;
  if (tfsf_z >= za && tfsf_z < zb) {
    if (tfsf_z > za) { zr[nzr][0] = za; zr[nzr][1] = tfsf_z; ++nzr; }
    if (tfsf_z + 2 < zb) { zr[nzr][0] = tfsf_z + 2; zr[nzr][1] = zb; ++nzr; }
  } else if (za < zb) {
    zr[0][0] = za; zr[0][1] = zb; nzr = 1;
  }
  p.has_interior = m >= 1 && ib.xa < ib.xb && ib.ya < ib.yb && nzr > 0;
  ShellBoxes& bl = p.shell;
  if (!p.has_interior) {
    add_shell_box(bl, 0, nx, 0, ny, 0, nz);
    return p;
  }
  int planes = 0;
  for (int k = 0; k < nzr; ++k) planes += zr[k][1] - zr[k][0];
  if (zchunk <= 0) {
    // about twelve waves of two resident blocks per SM on 148 SMs (measured
    // on 203 x 761 x 761: chunks of ~50 planes beat ~60 by 6 %), chunks of
    // at least 16 planes (each recomputes the plane below it)
    const long long per_layer = (long long)((ib.xb - ib.xa + kRowCells - 1) / kRowCells) *
                                ((ib.yb - ib.ya + tile_y - 1) / tile_y);
    long long layers = (12LL * 2 * 148 + per_layer - 1) / per_layer;
    layers = std::max(1LL, std::min(layers, (long long)planes / 16));
    zchunk = (int)((planes + layers - 1) / layers);
  }
  ib.zchunk = zchunk;
  ib.nz_ranges = nzr;
  ib.chunks = 0;
  for (int k = 0; k < nzr; ++k) {
    ib.z0[k] = zr[k][0];
    ib.z1[k] = zr[k][1];
    const int ch = (zr[k][1] - zr[k][0] + zchunk - 1) / zchunk;
    if (k == 0) ib.chunks0 = ch;
    ib.chunks += ch;
  }
  // the shell: z planes outside the interior ranges (whole planes), then per
  // interior range the y strips (whole rows) and the x strips
  int zc = 0;
  for (int k = 0; k < nzr; ++k) {
    add_shell_box(bl, 0, nx, 0, ny, zc, ib.z0[k]);
    zc = ib.z1[k];
  }
  add_shell_box(bl, 0, nx, 0, ny, zc, nz);
  for (int k = 0; k < nzr; ++k) {
    add_shell_box(bl, 0, nx, 0, ib.ya, ib.z0[k], ib.z1[k]);
    add_shell_box(bl, 0, nx, ib.yb, ny, ib.z0[k], ib.z1[k]);
    add_shell_box(bl, 0, ib.xa, ib.ya, ib.yb, ib.z0[k], ib.z1[k]);
    add_shell_box(bl, ib.xb, nx, ib.ya, ib.yb, ib.z0[k], ib.z1[k]);
  }
  return p;
}

template <class T>
bool launch_fused_interior(const State<T>& s, const FusedPlan& p, int tile_y, cudaStream_t st) {
  if (!p.has_interior) return true;
  switch (tile_y) {
    case 4: launch_interior_ty<T, 4>(s, p.interior, st); return true;
    case 7: launch_interior_ty<T, 7>(s, p.interior, st); return true;
    case 8: launch_interior_ty<T, 8>(s, p.interior, st); return true;
  }
  if constexpr (sizeof(T) == 4) {
    switch (tile_y) {
      case 15: launch_interior_ty<T, 15>(s, p.interior, st); return true;
      case 16: launch_interior_ty<T, 16>(s, p.interior, st); return true;
    }
  }
  return false;
}

template bool launch_fused_interior<float>(const State<float>&, const FusedPlan&, int, cudaStream_t);
template bool launch_fused_interior<double>(const State<double>&, const FusedPlan&, int, cudaStream_t);

}  // namespace fdtd
