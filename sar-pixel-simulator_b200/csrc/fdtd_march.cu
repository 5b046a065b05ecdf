// fdtd_march.cu -- the general z-marching fused step: H^{n+1/2} and E^{n+1}
// of a list of boxes, read from the source field set and written to the
// destination set, with every CPML face, domain edge and the injection
// plane handled inside the march.
//
// The fused step (fdtd_fused.cu) covers the interior box with a march that
// has no boundary code at all; this kernel covers everything else (the CPML
// z slabs, the x and y strips, the injection planes) in the same one-pass
// form, so the shell no longer needs the split H pass and E pass (80 B per
// cell-update plus psi, and an E pass that has to wait for the interior).
// Both marches read only the source set and write only the destination set,
// so they run side by side.
//
// A block is kMarchThreads threads: `width` lanes of 4 x cells by
// kMarchThreads / width rows (width 32, 16 or 8 per box, whichever pads the
// box least: 8-lane rows keep the narrow x strips dense). It marches up a
// chunk of z planes. At plane z a thread holds E(z) of its vector (carried
// from the previous plane), loads E(z+1) and H(z), and
//   1. computes H^{n+1/2}(z) with the complete per-vector update (h_vec:
//      main update inside its index ranges, z, x and y CPML faces,
//      E-field injection); the +x neighbour comes by shuffle from the next
//      lane, the +y neighbour through shared memory from the next row;
//   2. computes E^{n+1}(z) (e_vec: main update, CPML faces, H-field
//      injection); the -x neighbour by shuffle, the -y neighbour through
//      shared memory, the -z neighbour is H^{n+1/2}(z-1) carried from the
//      previous plane.
// The first row recomputes H of the row below the tile, lane 0 of every row
// H of the vector left of the tile (a halo lane: the same vector update as
// every other lane, so nothing diverges; not in the first tile of a box
// that starts at x = 0, which has no left neighbour), and a chunk starts by
// recomputing the plane below it; recomputed values are never stored, and
// psi is written only for the block's own cells. Warps whose vectors are
// all plain interior vectors take the plain update.
// Per-cell values equal the split passes' bit for bit: the same update
// functions in the same order of operations, fed the same neighbours.
#include <algorithm>
#include <cstring>
#include <mutex>

#include "fdtd_launch.h"
#include "fdtd_vec.cuh"

namespace fdtd {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxDevices = 64;

// Resident blocks per SM the march asks for (registers per thread <=
// 65536 / (160 * n)).
template <class T>
constexpr int march_min_blocks() { return sizeof(T) == 4 ? 3 : 1; }

// Dynamic shared memory of k_march, in elements of T: the four exchange
// arrays, then two stages of the per-thread staging area. A stage holds,
// per thread, kSlots vectors (E(z+1) x, y, z; H(z) x, y, z; Ca, Cb; the
// z-face psi Hyz, Hxz, Eyz, Exz), then the top row's E(y+1) x, z (32 lanes
// at most) and the last lane's E(x+4) y, z (one pair per row).
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
  const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? (int)sizeof(T) : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], %2, %3;\n" ::"r"(sa), "l"(src), "n"((int)sizeof(T)),
               "r"(n)
               : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

__device__ __forceinline__ const MarchBox& find_march_box(const MarchBoxes& mb, int bid) {
  int k = 0;
  while (k + 1 < mb.n && bid >= mb.b[k + 1].first) ++k;
  return mb.b[k];
}

template <class T>
__global__ void __launch_bounds__(kMarchThreads, march_min_blocks<T>())
k_march(const __grid_constant__ State<T> s, const int* __restrict__ tp, int toff,
        const __grid_constant__ MarchBoxes mb) {
  using SM = MarchSmem<T>;
  // exchange arrays: E(z) of every row (read by the row below as its +y
  // neighbour) and H^{n+1/2}(z) (read by the row above as its -y
  // neighbour), indexed [(row * width + lane) * 4 + j]; then the stages
  extern __shared__ __align__(32) unsigned char march_smem[];
  T* const sEx = reinterpret_cast<T*>(march_smem);
  T* const sEz = sEx + SM::kEx;
  T* const sHx = sEx + 2 * SM::kEx;
  T* const sHz = sEx + 3 * SM::kEx;
  T* const stage0 = sEx + 4 * SM::kEx;

  const MarchBox& b = find_march_box(mb, blockIdx.x);
  const int width = b.width, rows = kMarchThreads / width;
  int local = blockIdx.x - b.first;
  const int bx = local % b.gx;
  local /= b.gx;
  const int by = local % b.gy;
  const int c = local / b.gy;
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
  const int t = *tp + toff;
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

  auto slot = [&](int st, int k) { return stage0 + st * SM::kStage + k * SM::kEx + so; };
  auto top = [&](int st, int k) { return stage0 + st * SM::kStage + SM::kMain + (k * 32 + lane) * kVec; };
  auto right = [&](int st) { return stage0 + st * SM::kStage + SM::kMain + SM::kTop + 2 * r; };

  // Stage st <- what plane zz's update reads from global memory.
  auto issue = [&](int zz, int st) {
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
    const T* p0 = s.ps.z[0][0];
    cp_vec(slot(st, 8), hf ? s.ps.z[hsd][3] + kh : p0, hf);
    cp_vec(slot(st, 9), hf ? s.ps.z[hsd][2] + kh : p0, hf);
    cp_vec(slot(st, 10), ef ? s.ps.z[esd][1] + ke : p0, ef);
    cp_vec(slot(st, 11), ef ? s.ps.z[esd][0] + ke : p0, ef);
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
    ld4(e.exz, slot(st, 0)); ld4(e.eyz, slot(st, 1)); ld4(ezz, slot(st, 2));
    ld4(h.hx, slot(st, 3)); ld4(h.hy, slot(st, 4)); ld4(h.hz, slot(st, 5));
    T ca[kVec], cb[kVec];
    ld4(ca, slot(st, 6)); ld4(cb, slot(st, 7));
    if (top_row) { ld4(e.exy, top(st, 0)); ld4(e.ezy, top(st, 1)); }
    T eyr = T(0), ezr = T(0);
    if (last_lane) { eyr = right(st)[0]; ezr = right(st)[1]; }
    // ---- H^{n+1/2}(z) -----------------------------------------------------
    st4(&sEx[so], e.ex);
    st4(&sEz[so], e.ez);
    __syncthreads();
    if (!top_row) { ld4(e.exy, &sEx[su]); ld4(e.ezy, &sEz[su]); }
    e.eyn = __shfl_down_sync(kFull, e.ey[0], 1, width);
    e.ezn = __shfl_down_sync(kFull, e.ez[0], 1, width);
    if (last_lane) { e.eyn = eyr; e.ezn = ezr; }
    // warp-uniform paths: every vector of the warp a plain interior vector
    // (for H and for E), or one whose only boundary term is the z face
    const bool plain_h = __all_sync(kFull, !vin || interior(s, z, y, x0, t));
    const bool zface_h = !plain_h && __all_sync(kFull, !vin || zface_only(s, z, y, x0, t));
    if (vin) {
      if (plain_h) h_vec_interior(s, e, h.hx, h.hy, h.hz);
      else if (zface_h) h_vec_zface(s, e, z, y, x0, work, slot(st, 8), slot(st, 9), h.hx, h.hy, h.hz);
      else h_vec(s, e, z, y, x0, t, work, h.hx, h.hy, h.hz);
    }
    st4(&sHx[so], h.hx);
    st4(&sHz[so], h.hz);
    __syncthreads();
    // ---- E^{n+1}(z) ---------------------------------------------------------
    h.hyp = __shfl_up_sync(kFull, h.hy[kVec - 1], 1, width);
    h.hzp = __shfl_up_sync(kFull, h.hz[kVec - 1], 1, width);
    if (lane == 0) {   // own only at x0 = 0, whose E update reads no x - 1 value
      h.hyp = T(0);
      h.hzp = T(0);
    }
    if (work) {
      ld4(h.hxy, &sHx[sd]);
      ld4(h.hzy, &sHz[sd]);
      if (plain_h) e_vec_interior(h, ca, cb, e.ex, e.ey, e.ez);
      else if (zface_h) e_vec_zface(s, h, ca, cb, z, y, x0, slot(st, 10), slot(st, 11), e.ex, e.ey, e.ez);
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

}  // namespace

void add_march_box(MarchBoxes& mb, int x0, int x1, int y0, int y1, int z0, int z1, int zchunk) {
  if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;
  if (mb.n >= kMaxMarchBoxes) {
    ++mb.dropped;
    return;
  }
  MarchBox& b = mb.b[mb.n++];
  b.x0 = x0; b.x1 = x1; b.y0 = y0; b.y1 = y1; b.z0 = z0; b.z1 = z1;
  // tiles of a row width: `lead` own vectors in the first (the whole row
  // when the box starts at x = 0, else all lanes but the halo lane), then
  // width - 1 per tile
  const int nv = (x1 - x0 + kVec - 1) / kVec;
  auto tiles = [&](int w, int& lead) {
    lead = x0 == 0 ? w : w - 1;
    return nv <= lead ? 1 : 1 + (nv - lead + w - 2) / (w - 1);
  };
  // row width with the fewest threads (ties: the wider rows)
  long long best = -1;
  for (int w : {32, 16, 8}) {
    const int ty = kMarchThreads / w - 1;
    int lead = 0;
    const long long threads = (long long)tiles(w, lead) * ((y1 - y0 + ty - 1) / ty) * kMarchThreads;
    if (best < 0 || threads < best) { best = threads; b.width = w; }
  }
  const int ty = kMarchThreads / b.width - 1;
  b.gx = tiles(b.width, b.lead);
  b.gy = (y1 - y0 + ty - 1) / ty;
  // chunks of about zchunk planes, evenly cut (each recomputes the plane
  // below it)
  const int len = z1 - z0;
  const int zc = std::max(zchunk, 1);
  b.nchunks = std::max(1, (len + zc - 1) / zc);
  b.zchunk = (len + b.nchunks - 1) / b.nchunks;
  b.nchunks = (len + b.zchunk - 1) / b.zchunk;
  b.first = mb.total_blocks;
  mb.total_blocks += b.gx * b.gy * b.nchunks;
}

void finish_march_boxes(MarchBoxes& mb) {
  std::stable_sort(mb.b, mb.b + mb.n, [](const MarchBox& a, const MarchBox& c) { return a.zchunk > c.zchunk; });
  mb.total_blocks = 0;
  for (int k = 0; k < mb.n; ++k) {
    mb.b[k].first = mb.total_blocks;
    mb.total_blocks += mb.b[k].gx * mb.b[k].gy * mb.b[k].nchunks;
  }
}

template <class T>
void launch_march(const State<T>& s, const int* tdev, int toff, const MarchBoxes& mb, cudaStream_t st) {
  if (mb.n == 0 || mb.total_blocks == 0) return;
  // the staging area is above the 48 KB default: allow it once per device
  static std::mutex mu;
  static bool ready[kMaxDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < kMaxDevices) {
    std::lock_guard<std::mutex> lock(mu);
    if (!ready[dev]) {
      cudaFuncSetAttribute(k_march<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MarchSmem<T>::kBytes);
      ready[dev] = true;
    }
  } else {
    cudaFuncSetAttribute(k_march<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)MarchSmem<T>::kBytes);
  }
  k_march<T><<<mb.total_blocks, kMarchThreads, MarchSmem<T>::kBytes, st>>>(s, tdev, toff, mb);
}

template void launch_march<float>(const State<float>&, const int*, int, const MarchBoxes&, cudaStream_t);
template void launch_march<double>(const State<double>&, const int*, int, const MarchBoxes&, cudaStream_t);

}  // namespace fdtd
