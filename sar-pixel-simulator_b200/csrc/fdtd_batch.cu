// fdtd_batch.cu -- the batched sweep as one persistent kernel per time step
// that walks a tile queue across every member simulation.
//
// Each member's grid is cut as the fused step cuts it (make_fused_plan with
// the shell marched): tiles of the interior box (the plain z-march,
// interior_tile) and tiles of the shell boxes (the general z-march with
// every CPML face, edge and the injection plane, march_tile). All tiles of
// all members form one list, longest first. The kernel is launched with as
// many blocks as the device holds at once; every block takes the next tile
// index from a device counter (atomicAdd), stages the tile's member State
// in shared memory when the member changes, updates the tile and takes the
// next, until the list is exhausted. Every tile reads only its member's
// source field set and writes only its destination set (the fused step is
// ping-pong), so no block ever waits for another: there is no inter-block
// or inter-step wait in this kernel. Steps follow each other in stream
// order (in captured graphs); the batched phasor pass after each step
// zeroes the counter for the next.
//
// Per-cell values are those of each member's own fused step, bit for bit
// (the same tile bodies, fed the same neighbours).
#include <cstring>

#include "fdtd_launch.h"
#include "fdtd_tiles.cuh"

namespace fdtd {

namespace {

template <class T>
constexpr int queue_min_blocks() { return sizeof(T) == 4 ? 3 : 1; }

template <class T>
__global__ void __launch_bounds__(kMarchThreads, queue_min_blocks<T>())
k_batch_queue(const BatchModel<T>* __restrict__ bm, const QueueMember* __restrict__ qm,
              const QueueTile* __restrict__ tiles, int ntiles, int* __restrict__ counter, int toff) {
  extern __shared__ __align__(32) unsigned char queue_smem[];
  static_assert(sizeof(State<T>) % 8 == 0, "State is copied in 8-byte words");
  __shared__ unsigned long long st_words[sizeof(State<T>) / 8];
  __shared__ int s_tile;
  const State<T>& s = *reinterpret_cast<const State<T>*>(st_words);
  T* const sm = reinterpret_cast<T*>(queue_smem);
  constexpr int kEx = MarchSmem<T, false>::kEx;   // one exchange array; (4 + 1) * 128 elements
  static_assert(kEx == 5 * kRowCells, "the interior tile's exchange arrays are the march's");
  int cached = -1;
  for (;;) {
    if (threadIdx.x == 0) s_tile = atomicAdd(counter, 1);
    __syncthreads();
    const int k = s_tile;
    if (k >= ntiles) break;   // the same k in every thread
    const QueueTile tl = tiles[k];
    if (tl.member != cached) {
      const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&bm[tl.member].s);
      for (int w = threadIdx.x; w < (int)(sizeof(State<T>) / 8); w += blockDim.x) st_words[w] = src[w];
      cached = tl.member;
    }
    __syncthreads();
    if (tl.kind == 0) {
      interior_tile<T, 4>(s, qm[tl.member].ib, threadIdx.x % kLanes, threadIdx.x / kLanes, tl.bx, tl.by, tl.c,
                          sm, sm + kEx, sm + 2 * kEx, sm + 3 * kEx);
    } else {
      march_tile<T, false>(s, qm[tl.member].mb.b[tl.box], tl.bx, tl.by, tl.c, *bm[tl.member].tdev + toff, sm);
    }
    __syncthreads();   // shared memory and s_tile are reused by the next tile
  }
}

}  // namespace

template <class T>
size_t batch_queue_smem() {
  return MarchSmem<T, false>::kBytes;
}

template <class T>
int batch_queue_blocks_per_sm() {
  if (cudaFuncSetAttribute(k_batch_queue<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)batch_queue_smem<T>()) != cudaSuccess)
    return 0;
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_queue<T>, kMarchThreads, batch_queue_smem<T>()) !=
      cudaSuccess)
    return 0;
  return n;
}

template <class T>
void launch_batch_queue(const BatchModel<T>* bm, const QueueMember* qm, const QueueTile* tiles, int ntiles,
                        int* counter, int blocks, int toff, cudaStream_t st) {
  if (ntiles <= 0 || blocks <= 0) return;
  k_batch_queue<T><<<blocks, kMarchThreads, batch_queue_smem<T>(), st>>>(bm, qm, tiles, ntiles, counter, toff);
}

template size_t batch_queue_smem<float>();
template size_t batch_queue_smem<double>();
template int batch_queue_blocks_per_sm<float>();
template int batch_queue_blocks_per_sm<double>();
template void launch_batch_queue<float>(const BatchModel<float>*, const QueueMember*, const QueueTile*, int, int*,
                                        int, int, cudaStream_t);
template void launch_batch_queue<double>(const BatchModel<double>*, const QueueMember*, const QueueTile*, int,
                                         int*, int, int, cudaStream_t);

}  // namespace fdtd
