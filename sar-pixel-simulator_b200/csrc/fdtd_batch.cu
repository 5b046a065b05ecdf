// fdtd_batch.cu -- the batched sweep's interior work as one persistent
// kernel per time step that walks a tile queue across every member
// simulation.
//
// Each member's grid is cut as the fused step cuts it (make_fused_plan):
// the interior box (no CPML face, edge or injection plane) in tiles of the
// plain z-march (interior_tile), the shell in boxes for the batched split
// passes (k_batch_shell, fdtd_split.cu). All interior tiles of all members
// form one list, longest first. The kernel is launched with as many blocks
// as the device holds at once; every block takes the next tile index from
// a device counter (atomicAdd), stages the tile's member State in shared
// memory when the member changes, updates the tile and takes the next,
// until the list is exhausted. Every tile reads only its member's source
// field set and writes only its destination set (the fused step is
// ping-pong), so no block ever waits for another: there is no inter-block
// or inter-step wait in this kernel. Steps follow each other in stream
// order (in captured graphs); the batched phasor pass after each step
// zeroes the counter for the next.
//
// Per-cell values are those of each member's own fused step, bit for bit
// (the same tile body, fed the same neighbours).
#include <cstring>

#include "fdtd_launch.h"
#include "fdtd_tiles.cuh"

namespace fdtd {

namespace {

// four resident blocks per SM in float32 (the interior tile's 95 registers)
template <class T>
constexpr int queue_min_blocks() { return sizeof(T) == 4 ? 4 : 1; }

template <class T>
__global__ void __launch_bounds__(kLanes * 5, queue_min_blocks<T>())
k_batch_queue(const BatchModel<T>* __restrict__ bm, const QueueMember* __restrict__ qm,
              const QueueTile* __restrict__ tiles, int ntiles, int* __restrict__ counter) {
  __shared__ __align__(32) T sEx[5 * kRowCells];
  __shared__ __align__(32) T sEz[5 * kRowCells];
  __shared__ __align__(32) T sHx[5 * kRowCells];
  __shared__ __align__(32) T sHz[5 * kRowCells];
  static_assert(sizeof(State<T>) % 8 == 0, "State is copied in 8-byte words");
  __shared__ unsigned long long st_words[sizeof(State<T>) / 8];
  __shared__ int s_tile;
  const State<T>& s = *reinterpret_cast<const State<T>*>(st_words);
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
    interior_tile<T, 4>(s, qm[tl.member].ib, threadIdx.x % kLanes, threadIdx.x / kLanes, tl.bx, tl.by, tl.c, sEx,
                        sEz, sHx, sHz);
    __syncthreads();   // shared memory and s_tile are reused by the next tile
  }
}

}  // namespace

template <class T>
int batch_queue_blocks_per_sm() {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k_batch_queue<T>, kLanes * 5, 0) != cudaSuccess) return 0;
  return n;
}

template <class T>
void launch_batch_queue(const BatchModel<T>* bm, const QueueMember* qm, const QueueTile* tiles, int ntiles,
                        int* counter, int blocks, cudaStream_t st) {
  if (ntiles <= 0 || blocks <= 0) return;
  k_batch_queue<T><<<blocks, kLanes * 5, 0, st>>>(bm, qm, tiles, ntiles, counter);
}

template int batch_queue_blocks_per_sm<float>();
template int batch_queue_blocks_per_sm<double>();
template void launch_batch_queue<float>(const BatchModel<float>*, const QueueMember*, const QueueTile*, int, int*,
                                        int, cudaStream_t);
template void launch_batch_queue<double>(const BatchModel<double>*, const QueueMember*, const QueueTile*, int,
                                         int*, int, cudaStream_t);

}  // namespace fdtd
