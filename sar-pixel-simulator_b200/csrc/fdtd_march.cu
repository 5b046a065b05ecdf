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
#include "fdtd_tiles.cuh"

namespace fdtd {

namespace {

constexpr int kMaxDevices = 64;

// Resident blocks per SM the march asks for (registers per thread <=
// 65536 / (160 * n)).
template <class T>
constexpr int march_min_blocks() { return sizeof(T) == 4 ? 3 : 1; }

__device__ __forceinline__ const MarchBox& find_march_box(const MarchBoxes& mb, int bid) {
  int k = 0;
  while (k + 1 < mb.n && bid >= mb.b[k + 1].first) ++k;
  return mb.b[k];
}

template <class T>
__global__ void __launch_bounds__(kMarchThreads, march_min_blocks<T>())
k_march(const __grid_constant__ State<T> s, const int* __restrict__ tp, int toff,
        const __grid_constant__ MarchBoxes mb) {
  extern __shared__ __align__(32) unsigned char march_smem[];
  const MarchBox& b = find_march_box(mb, blockIdx.x);
  int local = blockIdx.x - b.first;
  const int bx = local % b.gx;
  local /= b.gx;
  const int by = local % b.gy;
  const int c = local / b.gy;
  march_tile<T>(s, b, bx, by, c, *tp + toff, reinterpret_cast<T*>(march_smem));
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
