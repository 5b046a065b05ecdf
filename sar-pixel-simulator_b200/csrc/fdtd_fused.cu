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
//  * the z slabs of the same x-y box (the bottom and top npml planes): the
//    same march with the z-face CPML terms, whose coefficients are uniform
//    over a plane (k_fused_slab);
//  * the shell (x and y CPML strips, the injection planes, the domain's
//    edge rows and columns): the split H pass over the shell boxes (source
//    E, H -> destination H), then the split E pass (destination H, source
//    E -> destination E). The E pass runs after the interior and slab
//    passes, whose destination H it reads at the shell's inner edge.
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
#include "fdtd_tiles.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
// z planes per block of the shell march (a box of up to 1.5 times this
// height is one chunk)
constexpr int kMarchZChunk = 48;

template <class T, int TY>
constexpr int interior_min_blocks() { return sizeof(T) == 4 && TY <= 8 ? 2 : 1; }

template <class T, int TY>
__global__ void __launch_bounds__(kLanes * (TY + 1), interior_min_blocks<T, TY>())
k_fused_interior(const __grid_constant__ State<T> s, InteriorBox ib) {
  __shared__ __align__(32) T sEx[(TY + 1) * kRowCells];
  __shared__ __align__(32) T sEz[(TY + 1) * kRowCells];
  __shared__ __align__(32) T sHx[(TY + 1) * kRowCells];
  __shared__ __align__(32) T sHz[(TY + 1) * kRowCells];
  interior_tile<T, TY>(s, ib, threadIdx.x, threadIdx.y, blockIdx.x, blockIdx.y, blockIdx.z, sEx, sEz, sHx, sHz);
}

// The z slabs of the same x-y box (z in [0, npml) and [nz - npml, nz), one
// chunk each), or the whole z extent of the x-y box (the column march), in
// z chunks (blockIdx.z, mapped to the box's z ranges as the interior's),
// marched like the interior. A plane in a z face carries the z-face CPML
// terms, with coefficients uniform over the plane (Taflove 7.x:
// psi_H = bh psi_H + (ch / dx) dE, psi_E = be psi_E + (ce / dx) dH,
// cpu/field_updates.py:66-105, 243-282), applied after the curl update of
// the same component as the split kernels apply them; the injection plane
// (while t < nt_inc) carries the incident terms after them
// (cpu/main_sim.py:147-161); the domain's first and last planes keep the
// components outside their update ranges (cpu/field_updates.py:18-63,
// 198-240). Every term is uniform over a plane, so the march's recomputed
// plane below a chunk gets them too. No x or y face touches the box.
// (four blocks per SM in float32 at 4-row tiles: the interior's 95 registers)
template <class T, int TY>
constexpr int slab_min_blocks() { return sizeof(T) == 4 && TY <= 4 ? 4 : 1; }

template <class T, int TY>
__global__ void __launch_bounds__(kLanes * (TY + 1), slab_min_blocks<T, TY>())
k_fused_slab(const __grid_constant__ State<T> s, InteriorBox ib, const int* __restrict__ tp, int toff) {
  __shared__ __align__(32) T sEx[(TY + 1) * kRowCells];
  __shared__ __align__(32) T sEz[(TY + 1) * kRowCells];
  __shared__ __align__(32) T sHx[(TY + 1) * kRowCells];
  __shared__ __align__(32) T sHz[(TY + 1) * kRowCells];
  slab_tile<T, TY>(s, ib, *tp + toff, threadIdx.x, threadIdx.y, blockIdx.x, blockIdx.y, blockIdx.z, sEx, sEz, sHx,
                   sHz);
}

template <class T, int TY>
void launch_slab_ty(const State<T>& s, const InteriorBox& sb, const int* tdev, int toff, cudaStream_t st) {
  const dim3 blk(kLanes, TY + 1, 1);
  const dim3 grd((sb.xb - sb.xa + kRowCells - 1) / kRowCells, (sb.yb - sb.ya + TY - 1) / TY, sb.chunks);
  k_fused_slab<T, TY><<<grd, blk, 0, st>>>(s, sb, tdev, toff);
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
FusedPlan make_fused_plan(int nx, int ny, int nz, int npml, int tfsf_z, int tile_y, int zchunk,
                          int slab_mode, bool march) {
  FusedPlan p;
  memset(&p, 0, sizeof(p));
  p.march = march ? 1 : 0;
  if (march) slab_mode = 0;
  const bool use_slab = slab_mode == 1;
  const int m = npml;
  InteriorBox& ib = p.interior;
  // rows start on a 128-byte line. Measured against starting at npml + 1
  // rounded up to 4 cells: at 203 x 761 x 761 that was 5 % slower with
  // 48-byte row offsets, and no faster with the arrays' origin shifted to
  // align that column, nor with tiles from column 0 whose lanes left of the
  // box only feed the shuffle (the narrower x strips of the shell took as
  // long); the batched queue's 64-model sweep took 6 % longer with it
  ib.xa = (m + 31) / 32 * 32;
  ib.xb = (nx - m) / kVec * kVec;
  ib.ya = m;
  ib.yb = ny - m;
  // interior z ranges: [m, nz - m) without tfsf_z, tfsf_z + 1
  int zr[2][2] = {{0, 0}, {0, 0}}, nzr = 0;
  const int za = m, zb = nz - m;
  if (tfsf_z >= za - 1 && tfsf_z < zb) {   // also the plane below the first chunk
    if (tfsf_z > za) { zr[nzr][0] = za; zr[nzr][1] = tfsf_z; ++nzr; }
    if (tfsf_z + 2 < zb) { zr[nzr][0] = tfsf_z + 2; zr[nzr][1] = zb; ++nzr; }
  } else if (za < zb) {
    zr[0][0] = za; zr[0][1] = zb; nzr = 1;
  }
  p.has_interior = m >= 1 && ib.xa < ib.xb && ib.ya < ib.yb && nzr > 0;
  ShellBoxes& bl = p.shell;
  if (!p.has_interior) {
    if (march) {
      add_march_box(p.mshell, 0, nx, 0, ny, 0, nz, kMarchZChunk);
      finish_march_boxes(p.mshell);
    } else {
      add_shell_box(bl, 0, nx, 0, ny, 0, nz);
    }
    return p;
  }
  auto add = [&](int x0, int x1, int y0, int y1, int z0, int z1) {
    if (march) add_march_box(p.mshell, x0, x1, y0, y1, z0, z1, kMarchZChunk);
    else add_shell_box(bl, x0, x1, y0, y1, z0, z1);
  };
  auto auto_zchunk = [&](int planes) {
    // about twelve waves of two resident blocks per SM on 148 SMs (measured
    // on 203 x 761 x 761: chunks of ~50 planes beat ~60 by 6 %), chunks of
    // at least 16 planes (each recomputes the plane below it)
    const long long per_layer = (long long)((ib.xb - ib.xa + kRowCells - 1) / kRowCells) *
                                ((ib.yb - ib.ya + tile_y - 1) / tile_y);
    long long layers = (12LL * 2 * 148 + per_layer - 1) / per_layer;
    layers = std::max(1LL, std::min(layers, (long long)planes / 16));
    return (int)((planes + layers - 1) / layers);
  };
  if (slab_mode == 2) {
    // the column march: the interior's x-y box over every z plane (z faces,
    // edges planes and the injection plane in the march); the shell is the
    // y strips (whole rows) and the x strips beside the box, over every z
    InteriorBox& cb = p.slab;
    cb = ib;
    cb.nz_ranges = 1;
    cb.z0[0] = 0;
    cb.z1[0] = nz;
    cb.zchunk = zchunk > 0 ? zchunk : auto_zchunk(nz);
    cb.chunks0 = cb.chunks = (nz + cb.zchunk - 1) / cb.zchunk;
    p.has_slab = 1;
    p.column = 1;
    p.has_interior = 0;
    add(0, nx, 0, ib.ya, 0, nz);
    add(0, nx, ib.yb, ny, 0, nz);
    add(0, ib.xa, ib.ya, ib.yb, 0, nz);
    add(ib.xb, nx, ib.ya, ib.yb, 0, nz);
    return p;
  }
  // with use_slab, the z slabs of the same x-y box (CPML in z only):
  // [0, m) and [nz - m, nz), each unless the injection plane lies in it or
  // is the plane below it (those the split passes sweep as whole planes)
  InteriorBox& sb = p.slab;
  sb = ib;
  sb.nz_ranges = 0;
  const int slab[2][2] = {{0, m}, {nz - m, nz}};
  for (int k = 0; k < 2 && use_slab; ++k) {
    if (tfsf_z >= slab[k][0] - 1 && tfsf_z < slab[k][1]) continue;
    sb.z0[sb.nz_ranges] = slab[k][0];
    sb.z1[sb.nz_ranges] = slab[k][1];
    ++sb.nz_ranges;
  }
  sb.zchunk = m;
  sb.chunks0 = 1;
  sb.chunks = sb.nz_ranges;
  p.has_slab = sb.nz_ranges > 0;
  int planes = 0;
  for (int k = 0; k < nzr; ++k) planes += zr[k][1] - zr[k][0];
  if (zchunk <= 0) zchunk = auto_zchunk(planes);
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
  // the shell: z planes that neither box covers (whole planes), then per
  // covered z range (slabs and interior ranges, in z order) the y strips
  // (whole rows) and the x strips beside the box
  int cz0[4], cz1[4], nc = 0;
  if (sb.nz_ranges > 0 && sb.z0[0] == 0) { cz0[nc] = sb.z0[0]; cz1[nc++] = sb.z1[0]; }
  for (int k = 0; k < nzr; ++k) { cz0[nc] = ib.z0[k]; cz1[nc++] = ib.z1[k]; }
  for (int k = 0; k < sb.nz_ranges; ++k)
    if (sb.z0[k] != 0) { cz0[nc] = sb.z0[k]; cz1[nc++] = sb.z1[k]; }
  int zc = 0;
  for (int k = 0; k < nc; ++k) {
    add(0, nx, 0, ny, zc, cz0[k]);
    zc = cz1[k];
  }
  add(0, nx, 0, ny, zc, nz);
  for (int k = 0; k < nc; ++k) {
    add(0, nx, 0, ib.ya, cz0[k], cz1[k]);
    add(0, nx, ib.yb, ny, cz0[k], cz1[k]);
    add(0, ib.xa, ib.ya, ib.yb, cz0[k], cz1[k]);
    add(ib.xb, nx, ib.ya, ib.yb, cz0[k], cz1[k]);
  }
  if (march) finish_march_boxes(p.mshell);
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

template <class T>
bool launch_fused_slab(const State<T>& s, const FusedPlan& p, int tile_y, const int* tdev, int toff,
                       cudaStream_t st) {
  if (!p.has_slab) return true;
  switch (tile_y) {
    case 4: launch_slab_ty<T, 4>(s, p.slab, tdev, toff, st); return true;
    case 7: launch_slab_ty<T, 7>(s, p.slab, tdev, toff, st); return true;
    case 8: launch_slab_ty<T, 8>(s, p.slab, tdev, toff, st); return true;
  }
  if constexpr (sizeof(T) == 4) {
    switch (tile_y) {
      case 15: launch_slab_ty<T, 15>(s, p.slab, tdev, toff, st); return true;
      case 16: launch_slab_ty<T, 16>(s, p.slab, tdev, toff, st); return true;
    }
  }
  return false;
}

template bool launch_fused_slab<float>(const State<float>&, const FusedPlan&, int, const int*, int, cudaStream_t);
template bool launch_fused_slab<double>(const State<double>&, const FusedPlan&, int, const int*, int,
                                        cudaStream_t);
template bool launch_fused_interior<float>(const State<float>&, const FusedPlan&, int, cudaStream_t);
template bool launch_fused_interior<double>(const State<double>&, const FusedPlan&, int, cudaStream_t);

}  // namespace fdtd
