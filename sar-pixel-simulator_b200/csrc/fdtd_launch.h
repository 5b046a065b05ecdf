// fdtd_launch.h -- host-side launchers shared between the kernel files and
// the C-ABI implementation.
#pragma once

#include <cuda_runtime.h>

#include "fdtd_common.cuh"

namespace fdtd {

// Restores the calling thread's current device when it leaves scope: every
// entry point that makes its simulation's device current leaves the
// caller's device as it found it.
struct DeviceGuard {
  int prev = -1;
  DeviceGuard() {
    if (cudaGetDevice(&prev) != cudaSuccess) {
      prev = -1;
      cudaGetLastError();
    }
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

template <class T>
void launch_split_step(const State<T>& s, const int* tdev, int toff, cudaStream_t st);

// The phasor pass over plane groups g0 .. g0 + ng - 1 (0 d, 1 u, 2 l, 3 r,
// 4 f, 5 b).
template <class T>
void launch_phasors(const State<T>& s, const int* tdev, int toff, cudaStream_t st, int g0 = 0, int ng = 6);

void launch_advance(int* tdev, int n, cudaStream_t st);

// Batched sweep (fdtd_split.cu): one step of every model (H pass, E pass,
// phasors, one launch each); `start` / `start_ph` hold each model's first
// block (n + 1 entries, the last one the total). Then the step counters.
template <class T>
void launch_batch_step(const BatchModel<T>* bm, const int* start, int n, int blocks,
                       const int* start_ph, int blocks_ph, int toff, cudaStream_t st);
template <class T>
void launch_batch_advance(const BatchModel<T>* bm, int n, int steps, cudaStream_t st);
// The phasor pass of every model (one launch); with reset, block 0 first
// zeroes *reset (the tile counter of the tile-queue step).
template <class T>
void launch_batch_phasors(const BatchModel<T>* bm, const int* start_ph, int n, int blocks_ph, int toff,
                          int* reset, cudaStream_t st);

// Batched tile-queue step (fdtd_batch.cu): per member the interior box of
// its fused plan, cut into tiles of the interior march (tile height 4).
struct QueueMember {
  int has_interior;
  InteriorBox ib;
};
// One tile: member, the tile's x and y position in the member's interior
// box and its z chunk.
struct QueueTile {
  int member, bx, by, c;
};
// Resident blocks per SM the tile-queue kernel reaches (0 on error).
template <class T>
int batch_queue_blocks_per_sm();
// The interior tiles of one fused step of every member: `blocks`
// persistent blocks walk the tiles (`ntiles` of them, longest first)
// through the counter, which must be zero at the launch; bm holds each
// member's State of this step (source -> destination set).
template <class T>
void launch_batch_queue(const BatchModel<T>* bm, const QueueMember* qm, const QueueTile* tiles, int ntiles,
                        int* counter, int blocks, cudaStream_t st);

// The shells of every member's fused step as split passes, one launch per
// pass: a box of member `member`, its first block `b.first` counted over
// all boxes of the launch (ascending); a block sweeps kBatchShellPlanes z
// planes of one box tile. The H pass reads each member's source set and
// writes its destination H; the E pass reads the destination H (the
// State's destination pointers) and source E.
constexpr int kBatchShellPlanes = 4;   // also the planes of a k_batch_split block
struct BatchShellBox {
  int member;
  ShellBox b;
};
template <class T>
void launch_batch_shell(const BatchModel<T>* bm, const BatchShellBox* boxes, int nboxes, int blocks, bool h_pass,
                        int toff, cudaStream_t st);

// Packed rows of nx elements into rows of `pitch` elements.
template <class T>
void launch_repitch(T* dst, const T* src, int nx, long long rows, int pitch, cudaStream_t st);

template <class T>
void launch_eps_sigma(int nx, int ny, int nz, int nz_mat, int pitch, const T* eps,
                      const T* sig, T eps0, T dt, T dx, T* ca, T* cb, cudaStream_t st);

// Fused step (fdtd_fused.cu): the interior box in one z-marching pass, the
// shell by the split passes over a box list.
struct FusedPlan {
  int has_interior;
  InteriorBox interior;
  int has_slab;
  InteriorBox slab;   // the z slabs [0, npml), [nz - npml, nz) of the same x-y box, or its column
  int column;         // slab holds the column march (the whole z extent)
  ShellBoxes shell;   // the shell swept by the split passes (shell mode 1)
  int march;          // shell mode 0: the shell is marched by k_march
  MarchBoxes mshell;  // the shell's boxes for k_march (shell mode 0)
};

// Interior box, z slabs and shell boxes of a grid; zchunk 0 picks the z
// chunk. slab 0: no z-slab march; 1: the z slabs of the interior's x-y box
// marched (FDTD_OPT_FUSED_SLAB = 1); 2: the column march, the whole z
// extent of the interior's x-y box in one march (slab box, has_interior 0),
// the shell then only the x and y strips. With march, the shell goes to
// k_march boxes (mshell) and slab is ignored; otherwise to the split
// passes (shell).
FusedPlan make_fused_plan(int nx, int ny, int nz, int npml, int tfsf_z, int tile_y, int zchunk,
                          int slab, bool march = false);

// Appends the box [x0, x1) x [y0, y1) x [z0, z1) to a march box list: the
// row width (32, 16 or 8 lanes) that pads the box least, z chunks of about
// `zchunk` planes.
void add_march_box(MarchBoxes& mb, int x0, int x1, int y0, int y1, int z0, int z1, int zchunk);

// Orders a march box list longest z chunk first (the long blocks start
// first and the short ones fill the tail) and numbers the blocks.
void finish_march_boxes(MarchBoxes& mb);

// Fused step of the march boxes: source set -> destination set, every CPML
// face, domain edge and injection plane handled in the march.
template <class T>
void launch_march(const State<T>& s, const int* tdev, int toff, const MarchBoxes& mb, cudaStream_t st);

// Tile shapes the interior kernel is built for: 32 lanes wide, tile_y rows.
bool fused_supported_tile(int tile_x, int tile_y, int elem_bytes);

// Interior pass and z-slab pass: read the source set, write the
// destination set.
template <class T>
bool launch_fused_interior(const State<T>& s, const FusedPlan& p, int tile_y, cudaStream_t st);
template <class T>
bool launch_fused_slab(const State<T>& s, const FusedPlan& p, int tile_y, const int* tdev, int toff,
                       cudaStream_t st);

// Appends the box [x0, x1) x [y0, y1) x [z0, z1) to a box list, with the
// row width (32, 16, 8 or 4 lanes) that pads x the least.
void add_shell_box(ShellBoxes& bl, int x0, int x1, int y0, int y1, int z0, int z1);

// Split H pass (h_pass) or E pass over the shell boxes, from the State's
// source pointers to its destination pointers.
template <class T>
void launch_shell_pass(const State<T>& s, const int* tdev, int toff, const ShellBoxes& bl,
                       bool h_pass, cudaStream_t st);

// One transposed step (fdtd_adjoint.cu): s holds E^n in its source E
// pointers, H^{n+1/2} in its source H pointers and the CPML auxiliaries
// after the step in ps; t is the step index n; `first` marks the first
// step of the backward sweep (t = size_t - 1), which launch_adjoint_first
// (the E phasor source of that step) must precede.
template <class T>
void launch_adjoint_first(const State<T>& s, const Adj<T>& a, int t, cudaStream_t st);
template <class T>
void launch_adjoint_step(const State<T>& s, const Adj<T>& a, int t, bool first, cudaStream_t st);

// Incident beam (fdtd_incident.cu). The taper of incidentbeam.py:317-433
// for a lateral grid of nx x ny cells and nt pulse bins: dfx = 1 / (nx dx),
// dfy = 1 / (ny dx) (numpy.fft.fftfreq spacing), the incidence angles'
// sines and cosines, r2 = radius^2, r2_4pi = radius^2 / (4 pi), and the
// polarisation weights (Eh, Ev) as complex numbers.
struct IncidentTaper {
  int nx, ny, nt;
  double dfx, dfy;
  double sin_theta, cos_phi, sin_phi;
  double r2, r2_4pi;
  double2 eh, ev;
};

// The excitation of the incident run: the imaginary parts of its first
// nt_pulse time samples into ex, ey ((nt_pulse, ny, pitch), element type T),
// from the pulse bins' wavenumbers and spectrum (host arrays of nt doubles /
// nt complex doubles). peak_out gets the peak magnitude before the
// normalisation to 10. Returns an FDTD status code.
template <class T>
int make_incident_excitation(const IncidentTaper& p, const double* k_host, const double* pfft_host,
                             int nt_pulse, int pitch, T* ex, T* ey, double* peak_out, cudaStream_t st);

// The read-out plane of the incident run and the incident phasors: fields
// of the run (its current set), the recorded planes (nt, ny, pitch), the
// four phasor planes (complex, (ny_ph, nx_ph) each, consecutive) and the
// run's phase table (per step: cos/sin of the t and t - 1/2 angles).
template <class T>
struct IncidentRecord {
  const T* ex; const T* ey; const T* hx; const T* hy;
  T* rex; T* rey; T* rhx; T* rhy;
  T* ph;
  const double* phase;
  int nx, ny, pitch;
  long long plane;
  int npml, read_out, nx_ph, ny_ph;
};

template <class T>
void launch_inc_source(T* ex, T* ey, const T* sx, const T* sy, int nx, int ny, int pitch, long long plane,
                       int feed_in, int t, cudaStream_t st);
template <class T>
void launch_inc_record(const IncidentRecord<T>& r, int t, cudaStream_t st);
template <class T>
void launch_fill(T* p, long long n, T v, cudaStream_t st);

// Non-finite check of one field set (fdtd_split.cu): flags[0] = 1,
// flags[1] = step on the first NaN or infinity in any of the six fields.
template <class T>
struct FieldPtrs {
  const T* p[6];
};
template <class T>
void launch_check_finite(const FieldPtrs<T>& f, long long vol, int step, int* flags, cudaStream_t st);

// Near-field power (fdtd_nearfield.cu): the 11 face powers (incident, left,
// right, front, back bottom/top, down, up) of a simulation's phasor planes
// (ph, plane offsets off) and the incident phasors inc (4 consecutive
// (ny_ph, nx_ph) complex planes, device), with the Simpson weights w_dev
// (ny_ph, nx_ph, szm, nz_ph - 1 - szm values, device) and `blocks` x 11
// float64 partial sums in `partial`. Returns 0 or 1 (CUDA error).
template <class T>
int near_field_power_run(const T* ph, const long long* off, const T* inc, int nx_ph, int ny_ph, int nz_ph,
                         int szm, const double* w_dev, double* partial, int blocks, double* out,
                         cudaStream_t st);

// Material blocks made on the device (fdtd_materials.cu): layers from
// height maps h (nlayers x (ny, nx) cells, device) with values ev, sv
// (nlayers + 1, device), and spheres sp (n x (zc, yc, xc, rc, ri), device),
// into eps / sig volumes (nz_mat, ny, nx).
template <class T>
void launch_fill_layers(T* eps, T* sig, int nx, int ny, int nz_mat, int nlayers, const double* h, const double* ev,
                        const double* sv, cudaStream_t st);
template <class T>
void launch_paint_spheres(T* eps, T* sig, int nx, int ny, int nz_mat, const double* sp, int n, double e_val,
                          double s_val, cudaStream_t st);

// Records an error message for fdtd_last_error(); returns code.
int report_error(int code, const char* msg);

// Near-to-far transform (near2far.cu).
int near2far_run(const double* jm /* 4 planes complex128 */, int nx, int ny, double dx,
                 double z_val, double k, const double* thetas, int ntheta,
                 const double* phis, int nphi, double r, double* out, cudaStream_t st);

}  // namespace fdtd
