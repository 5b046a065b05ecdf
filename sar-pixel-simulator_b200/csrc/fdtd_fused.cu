// fdtd_fused.cu -- the fused step: H^{n+1/2} and E^{n+1} of the whole grid
// in one z-marching pass.
//
// The pass reads every field, Ca and Cb once from the source set and
// writes every field once to the destination set (ping-pong), which is the
// 56 B per FP32 cell-update minimum; the split H/E passes move 80 B.
//
// A block owns a tile of 128 x cells (32 lanes x 4 cells) by TY rows and a
// chunk of z planes, and marches up the chunk one plane at a time. At plane
// z a thread holds E(z) of its vector (carried from the previous plane),
// loads E(z+1), H(z), Ca, Cb, and
//   1. computes H^{n+1/2}(z) of its vector; the +x neighbour comes from the
//      next lane by shuffle, the +y neighbour from the next thread row
//      through shared memory, the +z neighbour is E(z+1);
//   2. computes E^{n+1}(z); the -x neighbour comes by shuffle, the -y
//      neighbour through shared memory, the -z neighbour is H^{n+1/2}(z-1)
//      carried in registers.
// H^{n+1/2} values that belong to neighbouring tiles are recomputed from
// the source set rather than exchanged: thread row 0 computes the row below
// the tile, lane 0 the column left of the tile (one cell per row), and the
// first plane of a chunk is preceded by the plane below it. Recomputed cells
// never write psi; every psi element is written once, by its owner, into
// the destination psi set. Per-cell values are the same as the split
// kernels' (the same update functions, the same order of operations).
#include <algorithm>

#include "fdtd_launch.h"
#include "fdtd_vec.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kLanes = 32;
constexpr int kRowCells = kLanes * kVec;   // x cells of one tile row

// Two resident blocks per SM for float tiles up to 8 rows, one otherwise.
template <class T, int TY>
constexpr int fused_min_blocks() { return sizeof(T) == 4 && TY <= 8 ? 2 : 1; }

template <class T, int TY>
__global__ void __launch_bounds__(kLanes * (TY + 1), fused_min_blocks<T, TY>())
k_fused(const __grid_constant__ State<T> s, const int* __restrict__ tp, int toff, int zchunk) {
  // E(z) of every thread row (read by the row below as its +y neighbour)
  // and H^{n+1/2}(z) (read by the row above as its -y neighbour).
  __shared__ __align__(32) T sEx[TY + 1][kRowCells];
  __shared__ __align__(32) T sEz[TY + 1][kRowCells];
  __shared__ __align__(32) T sHx[TY + 1][kRowCells];
  __shared__ __align__(32) T sHz[TY + 1][kRowCells];

  const int lane = threadIdx.x, r = threadIdx.y;
  const int nx = s.nx, ny = s.ny, nz = s.nz;
  const int x0 = blockIdx.x * kRowCells + lane * kVec;
  const int y = blockIdx.y * TY + r - 1;          // row 0 is the row below the tile
  const int z0 = blockIdx.z * zchunk;
  const int z1 = min(nz, z0 + zchunk);
  const int zs = max(z0 - 1, 0);                  // plane below the chunk
  const int t = *tp + toff;
  const bool vin = x0 < s.pitch && y >= 0 && y < ny;
  const bool own = vin && r >= 1;
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
    // ---- loads of plane z ------------------------------------------------
    if (vin && z + 1 < nz) { ld4(e.exz, s.iex + i + P); ld4(e.eyz, s.iey + i + P); ld4(ezz, s.iez + i + P); }
    else { zero4(e.exz); zero4(e.eyz); zero4(ezz); }
    if (vin) { ld4(h.hx, s.ihx + i); ld4(h.hy, s.ihy + i); ld4(h.hz, s.ihz + i); }
    else { zero4(h.hx); zero4(h.hy); zero4(h.hz); }
    T ca[kVec], cb[kVec];
    if (work) { ld4(ca, s.ca + i); ld4(cb, s.cb + i); }
    else { zero4(ca); zero4(cb); }
    if (r == TY) {   // +y neighbour of the top row lies in the next tile
      if (vin && y + 1 < ny) { ld4(e.exy, s.iex + i + W); ld4(e.ezy, s.iez + i + W); }
      else { zero4(e.exy); zero4(e.ezy); }
    }
    T eyr = T(0), ezr = T(0);   // +x neighbour of lane 31 lies in the next tile
    if (lane == kLanes - 1 && vin && x0 + kVec < nx) { eyr = s.iey[i + kVec]; ezr = s.iez[i + kVec]; }
    // lane 0: the source values that H^{n+1/2} at (z, y, x0 - 1) needs
    const bool xh = work && lane == 0 && x0 >= 1;
    T gx = T(0), gy = T(0), gz = T(0), gxz = T(0), gyz = T(0), gxy = T(0), gzy = T(0);
    T ghy = T(0), ghz = T(0);
    if (xh) {
      const long long j = i - 1;
      gx = s.iex[j]; gy = s.iey[j]; gz = s.iez[j];
      ghy = s.ihy[j]; ghz = s.ihz[j];
      if (z + 1 < nz) { gxz = s.iex[j + P]; gyz = s.iey[j + P]; }
      if (y + 1 < ny) { gxy = s.iex[j + W]; gzy = s.iez[j + W]; }
    }
    // ---- H^{n+1/2}(z) -----------------------------------------------------
    st4(&sEx[r][so], e.ex);
    st4(&sEz[r][so], e.ez);
    __syncthreads();
    if (r < TY) { ld4(e.exy, &sEx[r + 1][so]); ld4(e.ezy, &sEz[r + 1][so]); }
    e.eyn = __shfl_down_sync(kFull, e.ey[0], 1);
    e.ezn = __shfl_down_sync(kFull, e.ez[0], 1);
    if (lane == kLanes - 1) { e.eyn = eyr; e.ezn = ezr; }
    const bool fast = interior(s, z, y, x0, t);
    if (vin) {
      if (fast) h_vec_interior(s, e, h.hx, h.hy, h.hz);
      else h_vec(s, e, z, y, x0, t, work, h.hx, h.hy, h.hz);
    }
    st4(&sHx[r][so], h.hx);
    st4(&sHz[r][so], h.hz);
    __syncthreads();
    // ---- E^{n+1}(z) ---------------------------------------------------------
    h.hyp = __shfl_up_sync(kFull, h.hy[kVec - 1], 1);
    h.hzp = __shfl_up_sync(kFull, h.hz[kVec - 1], 1);
    if (work) {
      ld4(h.hxy, &sHx[r - 1][so]);
      ld4(h.hzy, &sHz[r - 1][so]);
      if (lane == 0) {
        T hyl = T(0), hzl = T(0);
        if (xh) {
          ENbr<T> en;
          en.ex0 = gx; en.exz = gxz; en.exy = gxy;
          en.ey0 = gy; en.eyz = gyz; en.eyx = e.ey[0];
          en.ez0 = gz; en.ezy = gzy; en.ezx = e.ez[0];
          T hxl = T(0);
          hyl = ghy; hzl = ghz;
          h_cell(s, en, z, y, x0 - 1, t, false, hxl, hyl, hzl);
        }
        h.hyp = hyl;
        h.hzp = hzl;
      }
      if (fast) e_vec_interior(h, ca, cb, e.ex, e.ey, e.ez);
      else e_vec(s, h, ca, cb, z, y, x0, t, true, e.ex, e.ey, e.ez);
      st4(s.ohx + i, h.hx); st4(s.ohy + i, h.hy); st4(s.ohz + i, h.hz);
      st4(s.oex + i, e.ex); st4(s.oey + i, e.ey); st4(s.oez + i, e.ez);
    }
    // ---- next plane: E(z+1) becomes E(z), H^{n+1/2}(z) becomes H(z-1) -----
    copy4(e.ex, e.exz); copy4(e.ey, e.eyz); copy4(e.ez, ezz);
    copy4(h.hxz, h.hx); copy4(h.hyz, h.hy);
  }
}

template <class T, int TY>
void launch_ty(const State<T>& s, const int* tdev, int toff, int zchunk, cudaStream_t st) {
  const dim3 blk(kLanes, TY + 1, 1);
  const dim3 grd((s.nx + kRowCells - 1) / kRowCells, (s.ny + TY - 1) / TY,
                 (s.nz + zchunk - 1) / zchunk);
  k_fused<T, TY><<<grd, blk, 0, st>>>(s, tdev, toff, zchunk);
}

}  // namespace

// Planes per z chunk when the caller leaves it to the library: enough
// chunks for about eight waves of two resident blocks per SM on 148 SMs,
// each chunk at least 16 planes (one recomputed plane per chunk).
int fused_auto_zchunk(int nx, int ny, int nz, int tile_y) {
  const long long per_layer = (long long)((nx + kRowCells - 1) / kRowCells) * ((ny + tile_y - 1) / tile_y);
  const long long want = 8LL * 2 * 148;
  long long layers = (want + per_layer - 1) / per_layer;
  layers = std::max(1LL, std::min(layers, (long long)nz / 16));
  return (int)((nz + layers - 1) / layers);
}

template <class T>
bool launch_fused_step(const State<T>& s, const int* tdev, int toff, int tile_x, int tile_y,
                       int zchunk, cudaStream_t st) {
  if (tile_x != kLanes) return false;
  if (zchunk <= 0) zchunk = fused_auto_zchunk(s.nx, s.ny, s.nz, tile_y);
  switch (tile_y) {
    case 4: launch_ty<T, 4>(s, tdev, toff, zchunk, st); return true;
    case 7: launch_ty<T, 7>(s, tdev, toff, zchunk, st); return true;
    case 8: launch_ty<T, 8>(s, tdev, toff, zchunk, st); return true;
  }
  // taller tiles: float only (their shared memory exceeds the static limit
  // for double)
  if constexpr (sizeof(T) == 4) {
    switch (tile_y) {
      case 15: launch_ty<T, 15>(s, tdev, toff, zchunk, st); return true;
      case 16: launch_ty<T, 16>(s, tdev, toff, zchunk, st); return true;
    }
  }
  return false;
}

template bool launch_fused_step<float>(const State<float>&, const int*, int, int, int, int, cudaStream_t);
template bool launch_fused_step<double>(const State<double>&, const int*, int, int, int, int, cudaStream_t);

}  // namespace fdtd
