// fdtd_common.cuh -- shared device-side definitions of the FDTD library.
//
// All field arithmetic goes through R<T>::add/sub/mul/div, which map to the
// round-to-nearest intrinsics. They are never contracted into fused
// multiply-adds, so every update rounds exactly like the reference's numba
// kernels (fdtdsarsim/cpu/field_updates.py), which do not contract either.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace fdtd {

constexpr int kMaxPml = 32;

template <class T> struct R;
template <> struct R<float> {
  static __device__ __forceinline__ float fma(float a, float b, float c) { return __fmaf_rn(a, b, c); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
  static __device__ __forceinline__ float from_double(double a) { return __double2float_rn(a); }
};
template <> struct R<double> {
  static __device__ __forceinline__ double fma(double a, double b, double c) { return __fma_rn(a, b, c); }
  static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
  static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
  static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
  static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
  static __device__ __forceinline__ double from_double(double a) { return a; }
};

// CPML coefficient profiles, indexed [kind][q]. Kinds follow the packing of
// fdtd_set_absorbers: be_d, bh_d, ce_d, ch_d (down/left/front faces) and
// be_u, bh_u, ce_u, ch_u (up/right/back faces).
enum { BE_D = 0, BH_D, CE_D, CH_D, BE_U, BH_U, CE_U, CH_U };

// psi component slots per face.
//   z faces (down/up):    0 Exz, 1 Eyz, 2 Hxz, 3 Hyz   shape (npml, ny, pitch)
//   x faces (left/right): 0 Eyx, 1 Ezx, 2 Hyx, 3 Hzx   shape (nz, ny, xw)
//   y faces (front/back): 0 Exy, 1 Ezy, 2 Hxy, 3 Hzy   shape (nz, npml, pitch)
// An x-face row holds the cells x = xo + p, p < xw, with xo = 0 for the low
// face and xo = (nx - npml) rounded down to a multiple of 4 for the high
// face, xw = npml + 3 rounded up to a multiple of 4: every 4-cell vector
// that touches an x face is one aligned vector of its row (slots of cells
// outside the face are never read).
// Side 0 is the low face (down/left/front), side 1 the high face.
template <class T>
struct Psi {
  T* z[2][4];
  T* x[2][4];
  T* y[2][4];
};

// Everything a step kernel needs, passed by value (lives in the kernel
// parameter bank). Fields are stored (nz, ny, pitch) with pitch >= nx a
// multiple of 32 elements, so rows start 128-byte aligned.
template <class T>
struct State {
  int nx, ny, nz, npml, tfsf_z, nt_inc;
  int pitch;
  int xw, xo1;       // x-face psi rows: width, first x of the high face's row
  long long plane;   // ny * pitch
  T db, dtm0, dte0dx, dx;
  T rdx;   // 1 / dx correctly rounded (host IEEE division)
  T prof[8][kMaxPml];
  // field sets: src is read, dst is written (the same set for the in-place
  // split kernels; ping-pong sets for the fused kernel)
  const T* iex; const T* iey; const T* iez;  // E source
  const T* ihx; const T* ihy; const T* ihz;  // H source
  T* oex; T* oey; T* oez;                    // E destination
  T* ohx; T* ohy; T* ohz;                    // H destination
  const T* ca; const T* cb;
  Psi<T> ps;   // psi source
  Psi<T> pd;   // psi destination
  const T* inc_ex; const T* inc_ey; const T* inc_hx; const T* inc_hy;  // (nt_inc, ny, pitch)
  // phasors: 24 planes, complex interleaved, at offsets ph_off[k]
  T* ph;
  T* phc;    // Kahan compensation (same layout) or nullptr
  long long ph_off[24];
  int nx_ph, ny_ph, nz_ph;
  const double* phase;   // per step: cos_e, sin_e, cos_h, sin_h
  int kahan;
};

// Adjoint state of one simulation (fdtd_adjoint.cu): the adjoint fields,
// the adjoint CPML auxiliaries (same layout as Psi), the gradient
// accumulators with respect to Ca and Cb (float64, planes z < nz_grad), and
// dJ/d(Re p), dJ/d(Im p) of the four upper-plane phasors (ex, ey, hx, hy;
// (ny_ph, nx_ph) each, float64).
template <class T>
struct Adj {
  T* lex; T* ley; T* lez;
  T* lhx; T* lhy; T* lhz;
  Psi<T> lps;
  double* gca;
  double* gcb;
  const double* g_re;
  const double* g_im;
  int nz_grad;
};

// One member of a batched sweep: its State (current field set, in place),
// its step counter, and its tiling: 128-thread blocks of `width` lanes
// (width * 4 x cells) by 128 / width rows, gx x gy of them per plane, each
// block sweeping kBatchShellPlanes planes; ph_n
// cells in its largest phasor plane.
template <class T>
struct BatchModel {
  State<T> s;
  int* tdev;
  int width, gx, gy;
  int ph_n;
};

// A box of the fused step's shell, swept by the split passes:
// [x0, x1) x [y0, y1) x [z0, z1), x0 a multiple of 4. A tile is `width`
// lanes (width * 4 x cells) by 128 / width rows; gx, gy tiles per plane; a
// block sweeps `planes` planes of one tile (the list's choice); `first` is
// the box's first block in the launch.
struct ShellBox {
  int x0, x1, y0, y1, z0, z1;
  int width, gx, gy;
  int first;
};
constexpr int kMaxShellBoxes = 24;
struct ShellBoxes {
  int n, total_blocks;
  int planes;    // z planes per block (0 before launch_shell_pass picks it)
  int dropped;   // boxes that did not fit (a plan with any is rejected)
  ShellBox b[kMaxShellBoxes];
};

// A box of the fused step's shell marched in z by the general kernel
// (fdtd_march.cu): [x0, x1) x [y0, y1) x [z0, z1), x0 a multiple of 4. A
// block is kMarchThreads threads: `width` lanes of 4 x cells by
// kMarchThreads / width rows, the first row recomputing the row below the
// tile. Lane 0 of a tile is a halo lane (recomputes the vector left of the
// tile) except in the first tile of a box that starts at x = 0; `lead` own
// vectors in the first tile, width - 1 in the others; gx, gy tiles per
// plane, z cut into chunks of `zchunk` planes (`nchunks` of them); `first`
// is the box's first block in the launch.
constexpr int kMarchThreads = 160;
struct MarchBox {
  int x0, x1, y0, y1, z0, z1;
  int width, lead, gx, gy;
  int zchunk, nchunks;
  int first;
};
constexpr int kMaxMarchBoxes = 24;
struct MarchBoxes {
  int n, total_blocks;
  int dropped;   // boxes that did not fit (a plan with any is rejected)
  MarchBox b[kMaxMarchBoxes];
};

// The interior box of the fused step: no CPML face, domain edge or
// injection plane touches any of its cells or the halo cells it recomputes.
// x in [xa, xb) (xa a multiple of 32, xb of 4), y in [ya, yb), and up to
// two z ranges [z0[k], z1[k]) cut into chunks of `zchunk` planes.
struct InteriorBox {
  int xa, xb, ya, yb;
  int nz_ranges;
  int z0[2], z1[2];
  int zchunk;
  int chunks0, chunks;   // chunks of the first range, of both ranges
};

// Correctly rounded u / d for d > 0, given r = RN(1/d): Markstein's FMA
// correction (P. W. Markstein, "Computation of elementary functions on the
// IBM RISC System/6000 processor", IBM J. Res. Develop. 34(1), 1990). With
// r within half an ulp of 1/d and q0 = RN(u r) within one ulp of u/d, the
// remainder u - d q0 is exact in one FMA and RN(q0 + r (u - d q0)) is the
// correctly rounded quotient, as long as no step leaves the normal range.
// |u| outside [2^-100, 2^100] (float; [2^-900, 2^900] double) takes the
// IEEE division instead. Used for the CPML terms (c * dE) / dx, whose
// divisor is the constant cell size.
template <class T>
__device__ __forceinline__ T div_const(T u, T d, T r) {
  using M = R<T>;
  const T lo = sizeof(T) == 4 ? T(7.8886090522101181e-31) : T(1.4708983551653345e-271);   // 2^-100, 2^-900
  const T hi = sizeof(T) == 4 ? T(1.2676506002282294e+30) : T(6.7986211919640936e+270);   // 2^100, 2^900
  const T a = u < T(0) ? -u : u;
  if (a >= lo && a <= hi) {
    const T q0 = M::mul(u, r);
    const T rem = M::fma(-q0, d, u);
    return M::fma(rem, r, q0);
  }
  return a == T(0) ? u : M::div(u, d);   // zeros keep their sign; tiny, huge, NaN: IEEE
}

template <class T>
__device__ __forceinline__ T div_dx(const State<T>& s, T u) { return div_const(u, s.dx, s.rdx); }

// Index of cell x of plane z, row y in an x-face psi array of side `side`.
template <class T>
__device__ __forceinline__ long long xpsi_index(const State<T>& s, int z, int y, int side, int x) {
  return ((long long)z * s.ny + y) * s.xw + (x - (side ? s.xo1 : 0));
}

// Row width and high-face origin of the x-face psi arrays (host and device).
__host__ __device__ constexpr int xpsi_width(int npml) { return (npml + 3 + 3) / 4 * 4; }
__host__ __device__ constexpr int xpsi_origin_high(int nx, int npml) { return (nx - npml) / 4 * 4; }

__global__ void k_advance(int* t, int n);

}  // namespace fdtd
