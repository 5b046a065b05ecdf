// fdtd_launch.h -- host-side launchers shared between the kernel files and
// the C-ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include "fdtd_common.cuh"

namespace fdtd {

template <class T>
void launch_split_step(const State<T>& s, const int* tdev, int toff, cudaStream_t st);

template <class T>
void launch_phasors(const State<T>& s, const int* tdev, int toff, cudaStream_t st);

void launch_advance(int* tdev, int n, cudaStream_t st);

template <class T>
void launch_eps_sigma(int nx, int ny, int nz, int nz_mat, int pitch, const T* eps,
                      const T* sig, T eps0, T dt, T dx, T* ca, T* cb, cudaStream_t st);

// Fused z-marching step (fdtd_fused.cu). tile_x is the tile width in
// threads (32: 128 cells), tile_y the rows per tile, zchunk the z planes per
// block (0: automatic). Returns false when the tile shape is not supported.
template <class T>
bool launch_fused_step(const State<T>& s, const int* tdev, int toff, int tile_x,
                       int tile_y, int zchunk, cudaStream_t st);

// Planes per z chunk that launch_fused_step picks for zchunk == 0.
int fused_auto_zchunk(int nx, int ny, int nz, int tile_y);

// Records an error message for fdtd_last_error(); returns code.
int report_error(int code, const char* msg);

// Near-to-far transform (near2far.cu).
int near2far_run(const double* jm /* 4 planes complex128 */, int nx, int ny, double dx,
                 double z_val, double k, const double* thetas, int ntheta,
                 const double* phis, int nphi, double r, double* out, cudaStream_t st);

}  // namespace fdtd
