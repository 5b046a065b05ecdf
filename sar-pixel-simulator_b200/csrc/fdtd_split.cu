// fdtd_split.cu -- the split step (H pass, E pass), the phasor pass, the
// step-counter advance and the eps/sigma -> Ca/Cb kernel.
//
// The split step updates the fields in place: the H pass reads E and writes
// H, the E pass reads H and writes E, so no cell is read after another
// thread wrote it within a pass. It moves 80 B per FP32 cell-update
// (H pass 36 B, E pass 44 B) against the 56 B minimum of a fused pass.
// Each thread updates four consecutive x cells with vector loads and
// stores; interior vectors take the plain curl update, the rest (CPML
// faces, domain edges, the injection plane) h_vec / e_vec. The same passes,
// restricted to a list of boxes and run source -> destination, update the
// shell of the fused step (fdtd_fused.cu).
#include <cstring>

#include <algorithm>

#include "fdtd_launch.h"
#include "fdtd_vec.cuh"

namespace fdtd {

__global__ void k_advance(int* t, int n) { *t += n; }

// H pass on one vector: H^{n+1/2} = H^{n-1/2} - Db curl E^n, CPML and
// E-field injection. Reads E and H from the source pointers and writes H
// (and psi_H) to the destination pointers, so it serves both the in-place
// step (source == destination) and the ping-pong shell of the fused step.
// `lane` is the thread's position in a row segment of `width` lanes
// (width * kVec consecutive x cells); every lane of the segment calls this
// (the +x neighbour comes by shuffle), and only lanes with `act` update
// and store their vector.
template <class T>
__device__ __forceinline__ void h_split_vec(const State<T>& s, int t, int z, int y, int x0,
                                            int lane, int width, bool act) {
  const bool vin = x0 < s.pitch && y < s.ny;          // vector inside the row storage
  const long long P = s.plane, W = s.pitch;
  const long long i = (long long)z * P + (long long)y * W + x0;
  const bool plain = interior(s, z, y, x0, t);
  if (act && vin && !plain) h_psi_prefetch(s, z, y, x0);
  EVec<T> e;
  T hx[kVec], hy[kVec], hz[kVec];
  if (vin) {
    ld4(e.ex, s.iex + i); ld4(e.ey, s.iey + i); ld4(e.ez, s.iez + i);
    ld4(hx, s.ihx + i); ld4(hy, s.ihy + i); ld4(hz, s.ihz + i);
  } else {
    zero4(e.ex); zero4(e.ey); zero4(e.ez); zero4(hx); zero4(hy); zero4(hz);
  }
  if (vin && y + 1 < s.ny) { ld4(e.exy, s.iex + i + W); ld4(e.ezy, s.iez + i + W); }
  else { zero4(e.exy); zero4(e.ezy); }
  if (vin && z + 1 < s.nz) { ld4(e.exz, s.iex + i + P); ld4(e.eyz, s.iey + i + P); }
  else { zero4(e.exz); zero4(e.eyz); }
  // x+1 neighbour of the last cell: first cell of the next lane's vector
  e.eyn = __shfl_down_sync(0xffffffffu, e.ey[0], 1, width);
  e.ezn = __shfl_down_sync(0xffffffffu, e.ez[0], 1, width);
  if (lane == width - 1) {
    const bool ok = vin && x0 + kVec < s.nx;
    e.eyn = ok ? ldc(s.iey + (i + kVec)) : T(0);
    e.ezn = ok ? ldc(s.iez + (i + kVec)) : T(0);
  }
  if (!(act && vin)) return;
  if (plain) h_vec_interior(s, e, hx, hy, hz);
  else h_vec(s, e, z, y, x0, t, true, hx, hy, hz);
  st4(s.ohx + i, hx); st4(s.ohy + i, hy); st4(s.ohz + i, hz);
}

// E pass on one vector: E^{n+1} = Ca E^n + Cb curl H^{n+1/2}, CPML and
// H-field injection. Reads H^{n+1/2} and E^n from the source pointers and
// writes E (and psi_E) to the destination pointers.
template <class T>
__device__ __forceinline__ void e_split_vec(const State<T>& s, int t, int z, int y, int x0,
                                            int lane, int width, bool act) {
  const bool vin = x0 < s.pitch && y < s.ny;
  const long long P = s.plane, W = s.pitch;
  const long long i = (long long)z * P + (long long)y * W + x0;
  const bool plain = interior(s, z, y, x0, t);
  if (act && vin && !plain) e_psi_prefetch(s, z, y, x0);
  HVec<T> h;
  T ex[kVec], ey[kVec], ez[kVec], ca[kVec], cb[kVec];
  if (vin) {
    ld4(h.hx, s.ihx + i); ld4(h.hy, s.ihy + i); ld4(h.hz, s.ihz + i);
    ld4(ex, s.iex + i); ld4(ey, s.iey + i); ld4(ez, s.iez + i);
    ld4(ca, s.ca + i); ld4(cb, s.cb + i);
  } else {
    zero4(h.hx); zero4(h.hy); zero4(h.hz); zero4(ex); zero4(ey); zero4(ez); zero4(ca); zero4(cb);
  }
  if (vin && y >= 1) { ld4(h.hxy, s.ihx + i - W); ld4(h.hzy, s.ihz + i - W); }
  else { zero4(h.hxy); zero4(h.hzy); }
  if (vin && z >= 1) { ld4(h.hxz, s.ihx + i - P); ld4(h.hyz, s.ihy + i - P); }
  else { zero4(h.hxz); zero4(h.hyz); }
  // x-1 neighbour of the first cell: last cell of the previous lane's vector
  h.hyp = __shfl_up_sync(0xffffffffu, h.hy[kVec - 1], 1, width);
  h.hzp = __shfl_up_sync(0xffffffffu, h.hz[kVec - 1], 1, width);
  if (lane == 0) {
    const bool ok = vin && x0 >= 1;
    h.hyp = ok ? ldc(s.ihy + (i - 1)) : T(0);
    h.hzp = ok ? ldc(s.ihz + (i - 1)) : T(0);
  }
  if (!(act && vin)) return;
  if (plain) e_vec_interior(h, ca, cb, ex, ey, ez);
  else e_vec(s, h, ca, cb, z, y, x0, t, true, ex, ey, ez);
  st4(s.oex + i, ex); st4(s.oey + i, ey); st4(s.oez + i, ez);
}

// The passes over a list of boxes (the whole grid for the split step, the
// shell of the fused step), bl.planes planes of one box tile per 128-thread block. A box tile is `width` lanes
// (width * kVec x cells) by 128 / width rows.
__device__ __forceinline__ const ShellBox& find_box(const ShellBoxes& bl, int bid) {
  int k = 0;
  while (k + 1 < bl.n && bid >= bl.b[k + 1].first) ++k;
  return bl.b[k];
}

// Resident blocks per SM the split passes ask for (float: register cap 64;
// the passes are latency-bound, so more warps in flight beat a few spills)
template <class T>
constexpr int split_min_blocks() { return sizeof(T) == 4 ? 8 : 1; }

template <class T, bool kH>
__global__ void __launch_bounds__(128, split_min_blocks<T>()) k_shell(State<T> s, const int* __restrict__ tp, int toff,
                                               ShellBoxes bl) {
  const int bid = blockIdx.x;
  const ShellBox& b = find_box(bl, bid);
  int local = bid - b.first;
  const int bx = local % b.gx;
  local /= b.gx;
  const int by = local % b.gy;
  const int za = b.z0 + (local / b.gy) * bl.planes;
  const int zb = min(b.z1, za + bl.planes);
  const int lane = threadIdx.x % b.width, row = threadIdx.x / b.width;
  const int x0 = b.x0 + (bx * b.width + lane) * kVec;
  const int y = b.y0 + by * (128 / b.width) + row;
  const bool act = x0 < b.x1 && y < b.y1;
  const int t = *tp + toff;
  for (int z = za; z < zb; ++z) {   // block-uniform trip count (shuffles inside)
    if (kH) h_split_vec(s, t, z, y, x0, lane, b.width, act);
    else e_split_vec(s, t, z, y, x0, lane, b.width, act);
  }
}

// ---------------------------------------------------------------------------
// phasors (cpu/field_updates.py:373-461, gpu/field_updates.py:680-906)
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void ph_acc(const State<T>& s, int plane, long long k,
                                       double m, double c, double sn) {
  using M = R<T>;
  T* p = s.ph + s.ph_off[plane] + 2 * k;
  if (!s.kahan) {
    // float64 sum of the stored value and the float64 term, rounded to T
    stc(p, M::from_double(__dadd_rn((double)ldc(p), __dmul_rn(m, c))));
    stc(p + 1, M::from_double(__dadd_rn((double)ldc(p + 1), __dmul_rn(m, sn))));
  } else {
    T* pc = s.phc + s.ph_off[plane] + 2 * k;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const T term = M::from_double(__dmul_rn(m, j ? sn : c));
      const T yv = M::sub(term, ldc(pc + j));
      const T pj = ldc(p + j);
      const T tv = M::add(pj, yv);
      stc(pc + j, M::sub(M::sub(tv, pj), yv));
      stc(p + j, tv);
    }
  }
}

template <class T>
__device__ __forceinline__ double mean2(T a, T b) {
  return 0.5 * (double)R<T>::add(a, b);
}
template <class T>
__device__ __forceinline__ double mean4(T a, T b, T c, T d) {
  using M = R<T>;
  return 0.25 * (double)M::add(M::add(M::add(a, b), c), d);
}

// one complex phasor value (re, im) as a single 8-byte (float) or 16-byte
// (double) access: planes start at even element offsets of an aligned base
template <class T>
__device__ __forceinline__ void ld2(T (&d)[2], const T* p) {
  if (!FDTD_CHECK_PTR(p, 2 * (int)sizeof(T))) {   // bounds-checked build only
    d[0] = d[1] = T(0);
    return;
  }
  if constexpr (sizeof(T) == 4) {
    const float2 v = *reinterpret_cast<const float2*>(p);
    d[0] = v.x; d[1] = v.y;
  } else {
    const double2 v = *reinterpret_cast<const double2*>(p);
    d[0] = v.x; d[1] = v.y;
  }
}

template <class T>
__device__ __forceinline__ void st2(T* p, T re, T im) {
  if (!FDTD_CHECK_PTR(p, 2 * (int)sizeof(T))) return;   // bounds-checked build only
  if constexpr (sizeof(T) == 4) *reinterpret_cast<float2*>(p) = make_float2(re, im);
  else *reinterpret_cast<double2*>(p) = make_double2(re, im);
}

// The four components of one phasor cell: base plane `base`, field means
// m[0..3] (E, E, H, H). Every load (the four stored values) is issued before
// any store, so the cell costs one memory round trip rather than four.
template <class T>
__device__ __forceinline__ void ph_acc4(const State<T>& s, int base, long long k, const double (&m)[4],
                                        double cE, double sE, double cH, double sH) {
  using M = R<T>;
  if (s.kahan) {
#pragma unroll
    for (int j = 0; j < 4; ++j) ph_acc(s, base + j, k, m[j], j < 2 ? cE : cH, j < 2 ? sE : sH);
    return;
  }
  T v[4][2];
#pragma unroll
  for (int j = 0; j < 4; ++j) ld2(v[j], s.ph + s.ph_off[base + j] + 2 * k);
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double c = j < 2 ? cE : cH, sn = j < 2 ? sE : sH;
    // float64 sum of the stored value and the float64 term, rounded to T
    st2(s.ph + s.ph_off[base + j] + 2 * k, M::from_double(__dadd_rn((double)v[j][0], __dmul_rn(m[j], c))),
        M::from_double(__dadd_rn((double)v[j][1], __dmul_rn(m[j], sn))));
  }
}

// One phasor cell: plane group g = 0 d, 1 u (z planes), 2 l, 3 r (x
// planes), 4 f, 5 b (y planes); idx runs over the group's plane. The field
// loads of all four components come first, then the phasor update.
template <class T>
__device__ __forceinline__ void phasor_cell(const State<T>& s, int g, int idx, int t) {
  const int m = s.npml;
  int d0, d1;
  if (g < 2) { d0 = s.ny_ph; d1 = s.nx_ph; }
  else if (g < 4) { d0 = s.nz_ph; d1 = s.ny_ph; }
  else { d0 = s.nz_ph; d1 = s.nx_ph; }
  if (idx >= d0 * d1) return;
  const int a = idx / d1, b = idx - a * d1;
  if (a == 0 || b == 0) return;
  const double* ph = s.phase + 4 * (long long)t;
  const double cE = ph[0], sE = ph[1], cH = ph[2], sH = ph[3];
  const T* ex = s.oex; const T* ey = s.oey; const T* ez = s.oez;
  const T* hx = s.ohx; const T* hy = s.ohy; const T* hz = s.ohz;
  const long long P = s.plane, W = s.pitch;
  const long long k = (long long)a * d1 + b;
  double mv[4];
  int base;
  if (g < 2) {
    const int pz = g == 0 ? m + 1 : s.nz - m - 1;
    const long long i = pz * P + (long long)(m + a) * W + (m + b);
    base = g * 4;  // ex, ey, hx, hy
    mv[0] = mean2(ldc(ex + i), ldc(ex + i - 1));
    mv[1] = mean2(ldc(ey + i), ldc(ey + i - W));
    mv[2] = mean4(ldc(hx + i), ldc(hx + i - W), ldc(hx + i - P), ldc(hx + i - P - W));
    mv[3] = mean4(ldc(hy + i), ldc(hy + i - 1), ldc(hy + i - P), ldc(hy + i - P - 1));
  } else if (g < 4) {
    const int px = g == 2 ? m + 1 : s.nx - m - 1;
    const long long i = (long long)(m + a) * P + (long long)(m + b) * W + px;
    base = 8 + (g - 2) * 4;  // ey, ez, hy, hz
    mv[0] = mean2(ldc(ey + i), ldc(ey + i - W));
    mv[1] = mean2(ldc(ez + i), ldc(ez + i - P));
    mv[2] = mean4(ldc(hy + i), ldc(hy + i - 1), ldc(hy + i - P), ldc(hy + i - P - 1));
    mv[3] = mean4(ldc(hz + i), ldc(hz + i - 1), ldc(hz + i - W), ldc(hz + i - W - 1));
  } else {
    const int py = g == 4 ? m + 1 : s.ny - m - 1;
    const long long i = (long long)(m + a) * P + (long long)py * W + (m + b);
    base = 16 + (g - 4) * 4;  // ex, ez, hx, hz
    mv[0] = mean2(ldc(ex + i), ldc(ex + i - 1));
    mv[1] = mean2(ldc(ez + i), ldc(ez + i - P));
    mv[2] = mean4(ldc(hx + i), ldc(hx + i - W), ldc(hx + i - P), ldc(hx + i - P - W));
    mv[3] = mean4(ldc(hz + i), ldc(hz + i - W), ldc(hz + i - 1), ldc(hz + i - W - 1));
  }
  ph_acc4(s, base, k, mv, cE, sE, cH, sH);
}

// One thread per phasor cell; g0 + blockIdx.y selects the plane group.
template <class T>
__global__ void __launch_bounds__(256) k_phasors(State<T> s, const int* __restrict__ tp, int toff, int g0) {
  phasor_cell(s, g0 + (int)blockIdx.y, (int)(blockIdx.x * blockDim.x + threadIdx.x), *tp + toff);
}

// ---------------------------------------------------------------------------
// batched step: the split passes and the phasor pass of many simulations in
// one launch each. Block b belongs to the model m with
// start[m] <= b < start[m + 1]; the model's State lives in device memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ int find_model(const int* __restrict__ start, int n, int bid) {
  int lo = 0, hi = n - 1;   // last m with start[m] <= bid
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (start[mid] <= bid) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

template <class T, bool kH>
__global__ void __launch_bounds__(128, split_min_blocks<T>()) k_batch_split(const BatchModel<T>* __restrict__ bm,
                                                     const int* __restrict__ start, int n, int toff) {
  const int bid = blockIdx.x;
  const int mi = find_model(start, n, bid);
  const BatchModel<T>& b = bm[mi];
  // the member's State, staged once per block in shared memory: the update
  // reads its scalars, pointers and profiles many times per thread
  static_assert(sizeof(State<T>) % 8 == 0, "State is copied in 8-byte words");
  __shared__ unsigned long long st_words[sizeof(State<T>) / 8];
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&b.s);
    for (int k = threadIdx.x; k < (int)(sizeof(State<T>) / 8); k += blockDim.x) st_words[k] = src[k];
  }
  __syncthreads();
  const State<T>& s = *reinterpret_cast<const State<T>*>(st_words);
  int local = bid - start[mi];
  const int bx = local % b.gx;
  local /= b.gx;
  const int by = local % b.gy;
  const int za = (local / b.gy) * kBatchShellPlanes;   // kBatchShellPlanes planes per block
  const int zb = min(s.nz, za + kBatchShellPlanes);
  const int lane = threadIdx.x % b.width, row = threadIdx.x / b.width;
  const int x0 = (bx * b.width + lane) * kVec;
  const int y = by * (128 / b.width) + row;
  const int t = *b.tdev + toff;
  for (int z = za; z < zb; ++z) {   // block-uniform trip count (shuffles inside)
    if (kH) h_split_vec(s, t, z, y, x0, lane, b.width, true);
    else e_split_vec(s, t, z, y, x0, lane, b.width, true);
  }
}

// The shell boxes of every member (BatchShellBox): block b belongs to the
// last box whose first block is <= b and sweeps kBatchShellPlanes planes of
// one box tile (the staged State serves them all). The member's State is
// staged in shared memory; the E pass reads H from the destination set.
template <class T, bool kH>
__global__ void __launch_bounds__(128, split_min_blocks<T>())
k_batch_shell(const BatchModel<T>* __restrict__ bm, const BatchShellBox* __restrict__ boxes, int nboxes, int toff) {
  const int bid = blockIdx.x;
  int lo = 0, hi = nboxes - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (boxes[mid].b.first <= bid) lo = mid;
    else hi = mid - 1;
  }
  const int member = boxes[lo].member;
  const ShellBox b = boxes[lo].b;
  static_assert(sizeof(State<T>) % 8 == 0, "State is copied in 8-byte words");
  __shared__ unsigned long long st_words[sizeof(State<T>) / 8];
  {
    const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&bm[member].s);
    for (int k = threadIdx.x; k < (int)(sizeof(State<T>) / 8); k += blockDim.x) st_words[k] = src[k];
  }
  __syncthreads();
  State<T>& s = *reinterpret_cast<State<T>*>(st_words);
  if (!kH) {
    if (threadIdx.x == 0) { s.ihx = s.ohx; s.ihy = s.ohy; s.ihz = s.ohz; }
    __syncthreads();
  }
  int local = bid - b.first;
  const int bx = local % b.gx;
  local /= b.gx;
  const int by = local % b.gy;
  const int za = b.z0 + (local / b.gy) * kBatchShellPlanes;
  const int zb = min(b.z1, za + kBatchShellPlanes);
  const int lane = threadIdx.x % b.width, row = threadIdx.x / b.width;
  const int x0 = b.x0 + (bx * b.width + lane) * kVec;
  const int y = b.y0 + by * (128 / b.width) + row;
  const bool act = x0 < b.x1 && y < b.y1;
  const int t = *bm[member].tdev + toff;
  for (int z = za; z < zb; ++z) {   // block-uniform trip count (shuffles inside)
    if (kH) h_split_vec(s, t, z, y, x0, lane, b.width, act);
    else e_split_vec(s, t, z, y, x0, lane, b.width, act);
  }
}

template <class T>
__global__ void __launch_bounds__(256) k_batch_phasors(const BatchModel<T>* __restrict__ bm,
                                                       const int* __restrict__ start, int n,
                                                       int toff, int* __restrict__ reset) {
  const int bid = blockIdx.x;
  // the tile counter of the step's tile-queue kernel, which has finished
  // (stream order), starts the next step at zero
  if (reset && bid == 0 && threadIdx.x == 0) *reset = 0;
  const int mi = find_model(start, n, bid);
  const BatchModel<T>& b = bm[mi];
  const int local = bid - start[mi];
  const int per_group = (b.ph_n + 255) / 256;
  const int g = local / per_group;
  const int idx = (local - g * per_group) * 256 + threadIdx.x;
  phasor_cell(b.s, g, idx, *b.tdev + toff);
}

template <class T>
__global__ void k_batch_advance(const BatchModel<T>* __restrict__ bm, int n, int steps) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) *bm[i].tdev += steps;
}

// ---------------------------------------------------------------------------
// Ca, Cb from eps_r, sigma (materials/materials.py:23-68). The reference
// evaluates every operation in the array dtype: eps0, dt and dx are first
// rounded to it (numpy scalar promotion), then
//   perm = eps_r * eps0; x = (sigma * dt) / (2 * perm)
//   Ca = (1 - x) / (1 + x);  Cb = (dt / (perm * dx)) / (1 + x)
// Cells at z >= nz_mat are vacuum (eps_r = 1, sigma = 0).
// ---------------------------------------------------------------------------
template <class T>
__global__ void k_eps_sigma(int nx, int ny, int nz, int nz_mat, int pitch,
                            const T* __restrict__ eps, const T* __restrict__ sig,
                            T eps0, T dt, T dx, T* __restrict__ ca, T* __restrict__ cb) {
  using M = R<T>;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y;
  const int z = blockIdx.z;
  if (x >= nx) return;
  T e = T(1), sg = T(0);
  if (z < nz_mat) {
    const long long j = ((long long)z * ny + y) * nx + x;
    e = eps[j];
    sg = sig[j];
  }
  const T perm = M::mul(e, eps0);
  const T xx = M::div(M::mul(sg, dt), M::mul(T(2), perm));
  const T den = M::add(T(1), xx);
  const long long i = ((long long)z * ny + y) * pitch + x;
  ca[i] = M::div(M::sub(T(1), xx), den);
  cb[i] = M::div(M::div(dt, M::mul(perm, dx)), den);
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
void add_shell_box(ShellBoxes& bl, int x0, int x1, int y0, int y1, int z0, int z1) {
  if (x0 >= x1 || y0 >= y1 || z0 >= z1) return;
  if (bl.n >= kMaxShellBoxes) {
    ++bl.dropped;
    return;
  }
  ShellBox& b = bl.b[bl.n++];
  b.x0 = x0; b.x1 = x1; b.y0 = y0; b.y1 = y1; b.z0 = z0; b.z1 = z1;
  // row width with the least x padding (ties: the wider rows)
  long long best = -1;
  for (int w : {32, 16, 8, 4}) {
    const long long gx = (x1 - x0 + 4 * w - 1) / (4 * w), gy = (y1 - y0 + 128 / w - 1) / (128 / w);
    const long long padded = gx * 4 * w * gy * (128 / w);
    if (best < 0 || padded < best) { best = padded; b.width = w; }
  }
  b.gx = (x1 - x0 + b.width * kVec - 1) / (b.width * kVec);
  b.gy = (y1 - y0 + 128 / b.width - 1) / (128 / b.width);
  b.first = bl.total_blocks;
  bl.total_blocks += b.gx * b.gy * (z1 - z0);
}

template <class T>
void launch_split_step(const State<T>& s, const int* tdev, int toff, cudaStream_t st) {
  ShellBoxes whole;
  memset(&whole, 0, sizeof(whole));
  add_shell_box(whole, 0, s.nx, 0, s.ny, 0, s.nz);
  launch_shell_pass<T>(s, tdev, toff, whole, true, st);
  launch_shell_pass<T>(s, tdev, toff, whole, false, st);
}

template <class T>
void launch_phasors(const State<T>& s, const int* tdev, int toff, cudaStream_t st, int g0, int ng) {
  if (ng <= 0) return;
  int n = s.ny_ph * s.nx_ph;
  n = max(n, s.nz_ph * s.ny_ph);
  n = max(n, s.nz_ph * s.nx_ph);
  const dim3 grd((n + 255) / 256, ng, 1);
  k_phasors<T><<<grd, 256, 0, st>>>(s, tdev, toff, g0);
}

template <class T>
void launch_batch_step(const BatchModel<T>* bm, const int* start, int n, int blocks,
                       const int* start_ph, int blocks_ph, int toff, cudaStream_t st) {
  k_batch_split<T, true><<<blocks, 128, 0, st>>>(bm, start, n, toff);
  k_batch_split<T, false><<<blocks, 128, 0, st>>>(bm, start, n, toff);
  k_batch_phasors<T><<<blocks_ph, 256, 0, st>>>(bm, start_ph, n, toff, nullptr);
}

template <class T>
void launch_batch_phasors(const BatchModel<T>* bm, const int* start_ph, int n, int blocks_ph, int toff,
                          int* reset, cudaStream_t st) {
  k_batch_phasors<T><<<blocks_ph, 256, 0, st>>>(bm, start_ph, n, toff, reset);
}

template <class T>
void launch_batch_shell(const BatchModel<T>* bm, const BatchShellBox* boxes, int nboxes, int blocks, bool h_pass,
                        int toff, cudaStream_t st) {
  if (nboxes <= 0 || blocks <= 0) return;
  if (h_pass) k_batch_shell<T, true><<<blocks, 128, 0, st>>>(bm, boxes, nboxes, toff);
  else k_batch_shell<T, false><<<blocks, 128, 0, st>>>(bm, boxes, nboxes, toff);
}

template <class T>
void launch_batch_advance(const BatchModel<T>* bm, int n, int steps, cudaStream_t st) {
  k_batch_advance<T><<<(n + 127) / 128, 128, 0, st>>>(bm, n, steps);
}

template <class T>
void launch_shell_pass(const State<T>& s, const int* tdev, int toff, const ShellBoxes& bl,
                       bool h_pass, cudaStream_t st) {
  if (bl.n == 0 || bl.total_blocks == 0) return;
  // Several planes per block amortise the block's set-up, but only where
  // one plane per block gives many waves of blocks: 148 SMs hold about
  // 1184 of these blocks at once (8 each). add_shell_box numbered the
  // blocks one plane each; renumber for the choice.
  constexpr int kResident = 148 * 8;
  ShellBoxes p = bl;
  p.planes = bl.total_blocks >= 16 * kResident ? 4 : bl.total_blocks >= 8 * kResident ? 2 : 1;
  p.total_blocks = 0;
  for (int k = 0; k < p.n; ++k) {
    ShellBox& b = p.b[k];
    b.first = p.total_blocks;
    p.total_blocks += b.gx * b.gy * ((b.z1 - b.z0 + p.planes - 1) / p.planes);
  }
  if (h_pass) k_shell<T, true><<<p.total_blocks, 128, 0, st>>>(s, tdev, toff, p);
  else k_shell<T, false><<<p.total_blocks, 128, 0, st>>>(s, tdev, toff, p);
}

void launch_advance(int* tdev, int n, cudaStream_t st) {
  k_advance<<<1, 1, 0, st>>>(tdev, n);
}

// ---------------------------------------------------------------------------
// non-finite check: flags[0] = 1 and flags[1] = step when any of the six
// fields holds a NaN or an infinity (cells, padding included: the padding
// is never written and stays zero). The first detection wins.
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_check_finite(FieldPtrs<T> f, long long vol, int step,
                                                      int* __restrict__ flags) {
  if (*(volatile int*)flags) return;
  bool bad = false;
  for (int c = 0; c < 6; ++c) {
    const T* p = f.p[c];
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < vol;
         i += (long long)gridDim.x * blockDim.x)
      bad |= !isfinite(p[i]);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) {
    if (atomicCAS(flags, 0, 1) == 0) flags[1] = step;
  }
}

template <class T>
void launch_check_finite(const FieldPtrs<T>& f, long long vol, int step, int* flags, cudaStream_t st) {
  k_check_finite<T><<<8 * 148, 256, 0, st>>>(f, vol, step, flags);
}

template void launch_check_finite<float>(const FieldPtrs<float>&, long long, int, int*, cudaStream_t);
template void launch_check_finite<double>(const FieldPtrs<double>&, long long, int, int*, cudaStream_t);

// Packed rows (nx elements each) into pitched rows.
template <class T>
__global__ void __launch_bounds__(256) k_repitch(T* __restrict__ dst, const T* __restrict__ src, int nx,
                                                 long long rows, int pitch) {
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  if (x >= nx) return;
  for (long long r = blockIdx.y; r < rows; r += gridDim.y) dst[r * pitch + x] = src[r * nx + x];
}

template <class T>
void launch_repitch(T* dst, const T* src, int nx, long long rows, int pitch, cudaStream_t st) {
  const dim3 grd((nx + 255) / 256, (unsigned)std::min<long long>(rows, 65535), 1);
  k_repitch<T><<<grd, 256, 0, st>>>(dst, src, nx, rows, pitch);
}

template void launch_repitch<float>(float*, const float*, int, long long, int, cudaStream_t);
template void launch_repitch<double>(double*, const double*, int, long long, int, cudaStream_t);

template <class T>
void launch_eps_sigma(int nx, int ny, int nz, int nz_mat, int pitch, const T* eps,
                      const T* sig, T eps0, T dt, T dx, T* ca, T* cb, cudaStream_t st) {
  const dim3 grd((nx + 127) / 128, ny, nz);
  k_eps_sigma<T><<<grd, 128, 0, st>>>(nx, ny, nz, nz_mat, pitch, eps, sig, eps0, dt, dx, ca, cb);
}

template void launch_split_step<float>(const State<float>&, const int*, int, cudaStream_t);
template void launch_split_step<double>(const State<double>&, const int*, int, cudaStream_t);
template void launch_shell_pass<float>(const State<float>&, const int*, int, const ShellBoxes&,
                                       bool, cudaStream_t);
template void launch_shell_pass<double>(const State<double>&, const int*, int, const ShellBoxes&,
                                        bool, cudaStream_t);
template void launch_batch_step<float>(const BatchModel<float>*, const int*, int, int, const int*,
                                       int, int, cudaStream_t);
template void launch_batch_step<double>(const BatchModel<double>*, const int*, int, int,
                                        const int*, int, int, cudaStream_t);
template void launch_batch_phasors<float>(const BatchModel<float>*, const int*, int, int, int, int*,
                                          cudaStream_t);
template void launch_batch_phasors<double>(const BatchModel<double>*, const int*, int, int, int, int*,
                                           cudaStream_t);
template void launch_batch_shell<float>(const BatchModel<float>*, const BatchShellBox*, int, int, bool, int,
                                       cudaStream_t);
template void launch_batch_shell<double>(const BatchModel<double>*, const BatchShellBox*, int, int, bool, int,
                                        cudaStream_t);
template void launch_batch_advance<float>(const BatchModel<float>*, int, int, cudaStream_t);
template void launch_batch_advance<double>(const BatchModel<double>*, int, int, cudaStream_t);
template void launch_phasors<float>(const State<float>&, const int*, int, cudaStream_t, int, int);
template void launch_phasors<double>(const State<double>&, const int*, int, cudaStream_t, int, int);
template void launch_eps_sigma<float>(int, int, int, int, int, const float*, const float*, float,
                                      float, float, float*, float*, cudaStream_t);
template void launch_eps_sigma<double>(int, int, int, int, int, const double*, const double*,
                                       double, double, double, double*, double*, cudaStream_t);

}  // namespace fdtd
