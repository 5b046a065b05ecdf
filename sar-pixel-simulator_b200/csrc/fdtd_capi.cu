// fdtd_capi.cu -- the extern "C" boundary of libfdtd_b200.so.
//
// Owns all device memory of a simulation handle, builds the by-value kernel
// state, and schedules the per-step kernels. Errors are reported as status
// codes plus a per-thread message; nothing throws across the boundary.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "fdtd_b200.h"
#include "fdtd_check.cuh"
#include "fdtd_launch.h"

using namespace fdtd;

namespace {

thread_local std::string g_err;

int fail(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return code;
}

#define CK(call)                                                                  \
  do {                                                                            \
    cudaError_t e_ = (call);                                                      \
    if (e_ != cudaSuccess)                                                        \
      return fail(e_ == cudaErrorMemoryAllocation ? FDTD_ERR_NOMEM : FDTD_ERR_CUDA, \
                  "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

}  // namespace

// Lets the other translation units of the library report through
// fdtd_last_error().
int fdtd::report_error(int code, const char* msg) { return fail(code, "%s", msg); }

struct fdtd_sim {
  fdtd_geometry g{};
  int device = 0;
  int batch_refs = 0;                    // batches that hold this simulation as a member
  size_t esz = 4;
  int pitch = 0;
  long long plane = 0, vol = 0;          // elements
  int nx_ph = 0, ny_ph = 0, nz_ph = 0;
  std::vector<DevBuf> bufs;              // every allocation, freed on destroy
  void* fld[2][6] = {};                  // two field sets
  void* ca = nullptr;
  void* cb = nullptr;
  void* psi_base[2] = {};                // two psi sets
  long long psi_elems = 0;
  long long poz[2][4], pox[2][4], poy[2][4];  // offsets within a psi set
  void* inc[4] = {};
  int inc_nt = 0;
  void* ph = nullptr;
  void* phc = nullptr;
  long long ph_off[24];
  long long ph_elems = 0;
  double* phase = nullptr;
  int* tdev = nullptr;
  int* flags = nullptr;                  // non-finite check: found, step
  int64_t t = 0;
  int cur = 0;
  cudaStream_t own = nullptr;
  cudaStream_t stream = nullptr;
  // second stream of the fused step: the shell H pass runs beside the
  // interior pass (fork and join by events)
  cudaStream_t side = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
  // fdtd_run_streamed: copy stream, one event per staging slot, and pinned
  // staging buffers for pageable host planes (created on first use)
  cudaStream_t copy = nullptr;
  cudaEvent_t copy_ev[2] = {nullptr, nullptr};
  void* stage[2] = {nullptr, nullptr};
  // device staging of fdtd_run_streamed: one packed group of planes per
  // slot, re-pitched into the incident buffers on the copy stream
  void* dstage = nullptr;
  size_t dstage_bytes = 0;
  // fdtd_near_field_power: incident phasors, Simpson weights, partial sums
  // (made on first use)
  void* nf_inc = nullptr;
  double* nf_w = nullptr;
  double* nf_part = nullptr;
  // material block staged in packed (eps_r) and packed2 (sigma): its height
  // (-1: none), and scratch for height maps / spheres (grown as needed)
  int mat_nz = -1;
  void* mat_scratch = nullptr;
  size_t mat_scratch_bytes = 0;
  // packed (nz, ny, nx) device copy of a host volume, re-pitched on the
  // device by upload_volume (created on first use)
  void* packed = nullptr;
  void* packed2 = nullptr;               // second one for fdtd_set_materials_eps_sigma
  size_t stage_bytes = 0;
  bool have_abs = false, have_mat = false;
  std::vector<unsigned char> prof;       // 8 * npml values of the element type
  int kernel = FDTD_KERNEL_SPLIT;
  int phasor_mode = FDTD_PHASOR_REFERENCE;
  int tile_x = 32, tile_y = 8;
  int zchunk = 0;
  int slab = 0;                          // FDTD_OPT_FUSED_SLAB
  int shell = FDTD_SHELL_SPLIT;          // FDTD_OPT_SHELL
  FusedPlan plan;
  int plan_ok = 0, plan_tile_y = 0, plan_zchunk = 0, plan_slab = 0, plan_shell = 0;
  int graph_chunk = 0;
  int check_every = 0;
  // captured step chunks (FDTD_OPT_GRAPH_CHUNK), one per starting field set,
  // with the settings they were captured under; absorber uploads bump the
  // epoch (the profiles are captured by value)
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  int gsig[2][9] = {};
  int graph_epoch = 0;
  // gradient (fdtd_grad_*): checkpoints of the forward solve, the segment
  // of recomputed states and the adjoint state; a state is the 6 fields
  // followed by one CPML auxiliary set
  int grad_every = 0, grad_ncp = 0, grad_seg_slots = 0;
  bool grad_forward_done = false;
  void* grad_cp = nullptr;
  void* grad_seg = nullptr;
  void* grad_lam = nullptr;
  void* grad_lpsi = nullptr;
  double* grad_ca = nullptr;
  double* grad_cb = nullptr;
  double* grad_gre = nullptr;
  double* grad_gim = nullptr;
  // per-kernel event timing
  int timing = 0;
  std::vector<cudaEvent_t> ev;   // 3 per timed step: before step, after step, after phasors
  int ev_used = 0;
  double acc_ms[2] = {0, 0};
  int acc_n[2] = {0, 0};
};

// A batched sweep over member simulations (fdtd_batch_*). The members keep
// their own device memory; the batch holds a device table of their States
// and launches one kernel per phase for all of them.
struct fdtd_batch {
  std::vector<fdtd_sim*> sims;
  bool members_counted = false;  // the members' batch_refs include this batch
  int device = 0;
  int dtype = FDTD_F32;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev = nullptr;
  void* d_models = nullptr;   // BatchModel<T>[n]
  int* d_start = nullptr;     // first step-kernel block of each model, n + 1 entries
  int* d_start_ph = nullptr;  // first phasor block of each model, n + 1 entries
  int blocks = 0, blocks_ph = 0;
  std::vector<int> sig;       // each member's current field set when the table was built
  bool table_ok = false;
  int graph_chunk = 64;
  cudaGraphExec_t gexec = nullptr;
  int gexec_chunk = 0;
  int mode = FDTD_BATCH_SPLIT;     // FDTD_OPT_BATCH_MODE
  std::vector<cudaEvent_t> mev;    // one per member: the end of its work in a streams run
  // FDTD_BATCH_QUEUE: per member a State for each step parity (2 n
  // entries: source = current set, then the other), the members' fused
  // plans, the interior tile list, its counter, the shell boxes of the
  // split passes, the phasor blocks and the graph
  void* d_qtab = nullptr;
  QueueMember* d_qm = nullptr;
  QueueTile* d_tiles = nullptr;
  int* d_counter = nullptr;
  int* d_qstart_ph = nullptr;
  BatchShellBox* d_qshell = nullptr;
  int nqshell = 0, qshell_blocks = 0;
  int ntiles = 0, qblocks = 0, qblocks_ph = 0;
  std::vector<int> qsig;
  bool qtable_ok = false;
  cudaGraphExec_t qgexec = nullptr;
  int qgexec_chunk = 0;
};

namespace {

int alloc(fdtd_sim* s, size_t bytes, void** out) {
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FDTD_ERR_NOMEM, "cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
  }
  s->bufs.push_back({p, bytes});
  check_register(p, bytes);   // the bounds-checked build's allocation table
  *out = p;
  return FDTD_OK;
}

// A violation the bounds-checked build recorded since the last look, as
// FDTD_ERR_BOUNDS (FDTD_OK in the normal build).
int take_bounds_violation() {
  unsigned long long n = 0, what = 0;
  long long bytes = 0, line = 0;
  if (check_take(&n, &what, &bytes, &line)) return fail(FDTD_ERR_CUDA, "bounds check word unreadable");
  if (!n) return FDTD_OK;
  if (bytes < 0)
    return fail(FDTD_ERR_BOUNDS, "bounds check: %llu bad accesses; the first: shared index %lld (line %lld)", n,
                (long long)what, line);
  return fail(FDTD_ERR_BOUNDS, "bounds check: %llu bad accesses; the first: %lld bytes at address 0x%llx (line %lld)",
              n, bytes, what, line);
}

void release(fdtd_sim* s, void* p) {
  if (!p) return;
  for (size_t i = 0; i < s->bufs.size(); ++i)
    if (s->bufs[i].p == p) {
      check_unregister(p);
      cudaFree(p);
      s->bufs.erase(s->bufs.begin() + i);
      return;
    }
}

// The handle's two packed volume buffers (made on first use, kept): they
// stage a material block's eps_r (packed) and sigma (packed2).
int stage_buffers(fdtd_sim* s) {
  const size_t vol_bytes = (size_t)s->g.nx * s->g.ny * s->g.nz * s->esz;
  int rc;
  if (!s->packed && (rc = alloc(s, vol_bytes, &s->packed))) return rc;
  if (!s->packed2 && (rc = alloc(s, vol_bytes, &s->packed2))) return rc;
  return FDTD_OK;
}

// Device scratch of at least `bytes` for height maps or sphere lists.
int mat_scratch(fdtd_sim* s, size_t bytes, void** out) {
  if (s->mat_scratch_bytes < bytes) {
    release(s, s->mat_scratch);
    s->mat_scratch = nullptr;
    s->mat_scratch_bytes = 0;
    int rc = alloc(s, bytes, &s->mat_scratch);
    if (rc) return rc;
    s->mat_scratch_bytes = bytes;
  }
  *out = s->mat_scratch;
  return FDTD_OK;
}

// Ca, Cb from the staged eps_r (packed) and sigma (packed2) of the block's
// mat_nz planes, vacuum above (materials/materials.py:23-68).
int materials_from_stage(fdtd_sim* s) {
  const fdtd_geometry& g = s->g;
  const int nz_mat = s->mat_nz;
  const void* de = s->packed;
  const void* ds = s->packed2;
  // eps0 as hard-coded in materials/materials.py:45, rounded to the dtype
  const double eps0 = 8.8541878128e-12;
  if (g.dtype == FDTD_F32)
    launch_eps_sigma<float>(g.nx, g.ny, g.nz, nz_mat, s->pitch, (const float*)de, (const float*)ds,
                            (float)eps0, (float)g.timestep, (float)g.cell_size, (float*)s->ca,
                            (float*)s->cb, s->stream);
  else
    launch_eps_sigma<double>(g.nx, g.ny, g.nz, nz_mat, s->pitch, (const double*)de,
                             (const double*)ds, eps0, g.timestep, g.cell_size, (double*)s->ca,
                             (double*)s->cb, s->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  s->have_mat = true;
  return FDTD_OK;
}


template <class T>
State<T> make_state(const fdtd_sim* s, int src, int dst) {
  State<T> st;
  memset(&st, 0, sizeof(st));
  const fdtd_geometry& g = s->g;
  st.nx = g.nx; st.ny = g.ny; st.nz = g.nz; st.npml = g.npml; st.tfsf_z = g.tfsf_z;
  st.nt_inc = g.nt_inc;
  st.pitch = s->pitch;
  st.xw = xpsi_width(g.npml);
  st.xo1 = xpsi_origin_high(g.nx, g.npml);
  st.plane = s->plane;
  st.db = (T)g.db; st.dtm0 = (T)g.dtm0; st.dte0dx = (T)g.dte0dx;
  st.dx = (T)g.cell_size;
  st.rdx = (T)1 / st.dx;   // IEEE division on the host: correctly rounded
  const T* pr = reinterpret_cast<const T*>(s->prof.data());
  if (!s->prof.empty())
    for (int k = 0; k < 8; ++k)
      for (int q = 0; q < g.npml; ++q) st.prof[k][q] = pr[k * g.npml + q];
  st.iex = (const T*)s->fld[src][0]; st.iey = (const T*)s->fld[src][1]; st.iez = (const T*)s->fld[src][2];
  st.ihx = (const T*)s->fld[src][3]; st.ihy = (const T*)s->fld[src][4]; st.ihz = (const T*)s->fld[src][5];
  st.oex = (T*)s->fld[dst][0]; st.oey = (T*)s->fld[dst][1]; st.oez = (T*)s->fld[dst][2];
  st.ohx = (T*)s->fld[dst][3]; st.ohy = (T*)s->fld[dst][4]; st.ohz = (T*)s->fld[dst][5];
  st.ca = (const T*)s->ca; st.cb = (const T*)s->cb;
  for (int side = 0; side < 2; ++side)
    for (int c = 0; c < 4; ++c) {
      T* bs = (T*)s->psi_base[src];
      T* bd = (T*)s->psi_base[dst];
      st.ps.z[side][c] = bs + s->poz[side][c]; st.pd.z[side][c] = bd + s->poz[side][c];
      st.ps.x[side][c] = bs + s->pox[side][c]; st.pd.x[side][c] = bd + s->pox[side][c];
      st.ps.y[side][c] = bs + s->poy[side][c]; st.pd.y[side][c] = bd + s->poy[side][c];
    }
  st.inc_ex = (const T*)s->inc[0]; st.inc_ey = (const T*)s->inc[1];
  st.inc_hx = (const T*)s->inc[2]; st.inc_hy = (const T*)s->inc[3];
  st.ph = (T*)s->ph;
  st.phc = (T*)s->phc;
  for (int k = 0; k < 24; ++k) st.ph_off[k] = s->ph_off[k];
  st.nx_ph = s->nx_ph; st.ny_ph = s->ny_ph; st.nz_ph = s->nz_ph;
  st.phase = s->phase;
  st.kahan = s->phasor_mode == FDTD_PHASOR_KAHAN ? 1 : 0;
  return st;
}

cudaEvent_t timing_event(fdtd_sim* s) {
  if (s->ev_used >= (int)s->ev.size()) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
    s->ev.push_back(e);
  }
  return s->ev[s->ev_used++];
}

void mark(fdtd_sim* s, cudaEvent_t e) {
  if (e) cudaEventRecord(e, s->stream);
}

int collect_timing(fdtd_sim* s) {
  CK(cudaStreamSynchronize(s->stream));
  for (int i = 0; i + 2 < s->ev_used; i += 3) {
    float a = 0, b = 0;
    CK(cudaEventElapsedTime(&a, s->ev[i], s->ev[i + 1]));
    CK(cudaEventElapsedTime(&b, s->ev[i + 1], s->ev[i + 2]));
    s->acc_ms[0] += a; s->acc_n[0] += 1;
    s->acc_ms[1] += b; s->acc_n[1] += 1;
  }
  s->ev_used = 0;
  return FDTD_OK;
}

// ph_g0, ph_ng: the phasor plane groups each step accumulates (all six by
// default; none with ph_ng = 0; the gradient's forward only the upper plane)
template <class T>
int enqueue_steps(fdtd_sim* s, int n, int ph_g0 = 0, int ph_ng = 6) {
  for (int k = 0; k < n; ++k) {
    if (s->timing && s->ev_used + 3 > 3 * 4096) {
      int rc = collect_timing(s);
      if (rc) return rc;
    }
    cudaEvent_t e0 = s->timing ? timing_event(s) : nullptr;
    cudaEvent_t e1 = s->timing ? timing_event(s) : nullptr;
    cudaEvent_t e2 = s->timing ? timing_event(s) : nullptr;
    mark(s, e0);
    if (s->kernel == FDTD_KERNEL_FUSED) {
      const int nxt = 1 - s->cur;
      if (!fused_supported_tile(s->tile_x, s->tile_y, (int)sizeof(T)))
        return fail(FDTD_ERR_INVALID, "unsupported fused tile %dx%d", s->tile_x, s->tile_y);
      if (!s->plan_ok || s->plan_tile_y != s->tile_y || s->plan_zchunk != s->zchunk ||
          s->plan_slab != s->slab || s->plan_shell != s->shell) {
        const fdtd_geometry& g = s->g;
        s->plan = make_fused_plan(g.nx, g.ny, g.nz, g.npml, g.tfsf_z, s->tile_y, s->zchunk, s->slab,
                                  s->shell == FDTD_SHELL_MARCH);
        s->plan_slab = s->slab;
        s->plan_shell = s->shell;
        if (s->plan.shell.dropped || s->plan.mshell.dropped)
          return fail(FDTD_ERR_INVALID, "fused plan needs more than %d shell boxes", kMaxShellBoxes);
        s->plan_tile_y = s->tile_y;
        s->plan_zchunk = s->zchunk;
        s->plan_ok = 1;
      }
      // interior and shell H pass read the source set only; the shell E
      // pass reads the destination H that both of them wrote
      State<T> st = make_state<T>(s, s->cur, nxt);
      CK(cudaEventRecord(s->fork, s->stream));
      CK(cudaStreamWaitEvent(s->side, s->fork, 0));
      if (s->plan.march) {
        // the shell march and the interior march read the source set only
        // and write disjoint cells of the destination set
        launch_march<T>(st, s->tdev, k, s->plan.mshell, s->side);
        launch_fused_interior<T>(st, s->plan, s->tile_y, s->stream);
        CK(cudaEventRecord(s->join, s->side));
        CK(cudaStreamWaitEvent(s->stream, s->join, 0));
      } else {
        // the shell H pass (and the z slabs' march) beside the interior
        // march, or beside the column march
        if (!s->plan.column) launch_fused_slab<T>(st, s->plan, s->tile_y, s->tdev, k, s->side);
        launch_shell_pass<T>(st, s->tdev, k, s->plan.shell, true, s->side);
        if (s->plan.column) launch_fused_slab<T>(st, s->plan, s->tile_y, s->tdev, k, s->stream);
        launch_fused_interior<T>(st, s->plan, s->tile_y, s->stream);
        CK(cudaEventRecord(s->join, s->side));
        CK(cudaStreamWaitEvent(s->stream, s->join, 0));
        State<T> se = st;
        se.ihx = (const T*)s->fld[nxt][3]; se.ihy = (const T*)s->fld[nxt][4]; se.ihz = (const T*)s->fld[nxt][5];
        launch_shell_pass<T>(se, s->tdev, k, s->plan.shell, false, s->stream);
      }
      s->cur = nxt;
      mark(s, e1);
      State<T> sp = make_state<T>(s, s->cur, s->cur);
      launch_phasors<T>(sp, s->tdev, k, s->stream, ph_g0, ph_ng);
    } else {
      State<T> st = make_state<T>(s, s->cur, s->cur);
      launch_split_step<T>(st, s->tdev, k, s->stream);
      mark(s, e1);
      launch_phasors<T>(st, s->tdev, k, s->stream, ph_g0, ph_ng);
    }
    mark(s, e2);
    const long long done = s->t + k + 1;
    if (s->check_every > 0 && done % s->check_every == 0) {
      FieldPtrs<T> f;
      for (int c = 0; c < 6; ++c) f.p[c] = (const T*)s->fld[s->cur][c];
      launch_check_finite<T>(f, s->vol, (int)done, s->flags, s->stream);
    }
  }
  launch_advance(s->tdev, n, s->stream);
  CK(cudaGetLastError());
  return FDTD_OK;
}

// One chunk of `chunk` steps replayed from a captured graph (captured on
// first use, and again when a setting it depends on changed). The graph
// holds the step kernels with their step offsets, the phasor passes and the
// step-counter advance, so every replay continues from the counter.
template <class T>
int enqueue_graph_chunk(fdtd_sim* s, int chunk) {
  const int start = s->cur;
  const int sig[9] = {chunk,          s->kernel,      s->tile_x,    s->tile_y, s->zchunk,
                      s->phasor_mode, s->graph_epoch, s->slab, s->shell};
  if (!s->gexec[start] || memcmp(sig, s->gsig[start], sizeof(sig)) != 0) {
    if (s->gexec[start]) {
      cudaGraphExecDestroy(s->gexec[start]);
      s->gexec[start] = nullptr;
    }
    CK(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    const int rc = enqueue_steps<T>(s, chunk);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    s->cur = start;   // capturing ran nothing
    if (rc || e != cudaSuccess) {
      if (graph) cudaGraphDestroy(graph);
      cudaGetLastError();
      return rc ? rc : fail(FDTD_ERR_CUDA, "step graph capture: %s", cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&s->gexec[start], graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
      s->gexec[start] = nullptr;
      return fail(FDTD_ERR_CUDA, "step graph instantiation: %s", cudaGetErrorString(ei));
    }
    memcpy(s->gsig[start], sig, sizeof(sig));
  }
  CK(cudaGraphLaunch(s->gexec[start], s->stream));
  if (s->kernel == FDTD_KERNEL_FUSED && (chunk & 1)) s->cur = 1 - start;
  return FDTD_OK;
}

// Steps of fdtd_run: graph chunks when FDTD_OPT_GRAPH_CHUNK is set and
// neither per-kernel timing nor the non-finite check (both tied to the
// absolute step) is on, direct launches otherwise and for the remainder.
template <class T>
int run_steps(fdtd_sim* s, int nsteps) {
  const int chunk = s->graph_chunk;
  if (chunk > 0 && !s->timing && s->check_every == 0) {
    while (nsteps >= chunk) {
      const int rc = enqueue_graph_chunk<T>(s, chunk);
      if (rc) return rc;
      s->t += chunk;
      nsteps -= chunk;
    }
  }
  if (nsteps > 0) {
    const int rc = enqueue_steps<T>(s, nsteps);
    if (rc) return rc;
    s->t += nsteps;
  }
  return FDTD_OK;
}

int check_sim(fdtd_sim* s) {
  if (!s) return fail(FDTD_ERR_INVALID, "null simulation handle");
  cudaError_t e = cudaSetDevice(s->device);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_last_error(char* buf, int len) {
  if (buf && len > 0) {
    strncpy(buf, g_err.c_str(), (size_t)len - 1);
    buf[len - 1] = 0;
  }
  return (int)g_err.size();
}

int fdtd_version(void) { return 100; }

int fdtd_device_count(int* count) {
  if (!count) return fail(FDTD_ERR_INVALID, "null count");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    cudaGetLastError();
    n = 0;
  }
  *count = n;
  return FDTD_OK;
}

int fdtd_device_name(int device, char* name, int len) {
  if (!name || len < 1) return fail(FDTD_ERR_INVALID, "null name buffer");
  name[0] = 0;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev)
    return fail(FDTD_ERR_INVALID, "device %d out of range (%d devices)", device, ndev);
  cudaDeviceProp prop;
  cudaError_t e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "cudaGetDeviceProperties: %s", cudaGetErrorString(e));
  }
  strncpy(name, prop.name, (size_t)len - 1);
  name[len - 1] = 0;
  return FDTD_OK;
}

int fdtd_create(const fdtd_geometry* geom, int device, fdtd_sim** out) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  if (!geom || !out) return fail(FDTD_ERR_INVALID, "null argument");
  *out = nullptr;
  const fdtd_geometry& g = *geom;
  if (g.dtype != FDTD_F32 && g.dtype != FDTD_F64)
    return fail(FDTD_ERR_INVALID, "dtype must be FDTD_F32 or FDTD_F64");
  if (g.npml < 2 || g.npml > kMaxPml)
    return fail(FDTD_ERR_INVALID, "npml %d out of range [2, %d]", g.npml, kMaxPml);
  const int minn = 2 * g.npml + 3;
  if (g.nx < minn || g.ny < minn || g.nz < minn)
    return fail(FDTD_ERR_INVALID, "grid %dx%dx%d too small for npml %d (need >= %d per axis)",
                g.nz, g.ny, g.nx, g.npml, minn);
  if (g.tfsf_z < 0 || g.tfsf_z >= g.nz)
    return fail(FDTD_ERR_INVALID, "tfsf_z %d outside [0, nz=%d)", g.tfsf_z, g.nz);
  if (g.nt < 0 || g.nt_inc < 0)
    return fail(FDTD_ERR_INVALID, "negative step counts");
  if (!(g.cell_size > 0) || !(g.timestep > 0))
    return fail(FDTD_ERR_INVALID, "cell_size and timestep must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev)
    return fail(FDTD_ERR_INVALID, "device %d out of range (%d devices)", device, ndev);
  CK(cudaSetDevice(device));

  fdtd_sim* s = new fdtd_sim();
  s->g = g;
  s->device = device;
  s->esz = g.dtype == FDTD_F32 ? 4 : 8;
  s->pitch = (g.nx + 31) / 32 * 32;
  s->plane = (long long)g.ny * s->pitch;
  s->vol = (long long)g.nz * s->plane;
  s->nx_ph = g.nx - 2 * g.npml;
  s->ny_ph = g.ny - 2 * g.npml;
  s->nz_ph = g.nz - 2 * g.npml;
  int rc = FDTD_OK;
  auto A = [&](size_t bytes, void** p) {
    if (rc == FDTD_OK) rc = alloc(s, bytes, p);
  };
  const size_t fb = (size_t)s->vol * s->esz;
  for (int set = 0; set < 2; ++set)
    for (int c = 0; c < 6; ++c) A(fb, &s->fld[set][c]);
  A(fb, &s->ca);
  A(fb, &s->cb);
  // psi layout within one set: z faces (npml, ny, pitch), x faces
  // (nz, ny, xw), y faces (nz, npml, pitch); 4 components per face side
  long long off = 0;
  const long long zsz = (long long)g.npml * g.ny * s->pitch;
  const long long xsz = (long long)g.nz * g.ny * xpsi_width(g.npml);
  const long long ysz = (long long)g.nz * g.npml * s->pitch;
  auto align32 = [](long long v) { return (v + 31) / 32 * 32; };
  for (int side = 0; side < 2; ++side)
    for (int c = 0; c < 4; ++c) { s->poz[side][c] = off; off += align32(zsz); }
  for (int side = 0; side < 2; ++side)
    for (int c = 0; c < 4; ++c) { s->pox[side][c] = off; off += align32(xsz); }
  for (int side = 0; side < 2; ++side)
    for (int c = 0; c < 4; ++c) { s->poy[side][c] = off; off += align32(ysz); }
  s->psi_elems = off;
  A((size_t)off * s->esz, &s->psi_base[0]);
  A((size_t)off * s->esz, &s->psi_base[1]);
  // phasor planes in the reference's result order
  off = 0;
  for (int k = 0; k < 24; ++k) {
    long long n;
    if (k < 8) n = (long long)s->ny_ph * s->nx_ph;
    else if (k < 16) n = (long long)s->nz_ph * s->ny_ph;
    else n = (long long)s->nz_ph * s->nx_ph;
    s->ph_off[k] = off;
    off += align32(2 * n);
  }
  s->ph_elems = off;
  A((size_t)off * s->esz, &s->ph);
  A((size_t)off * s->esz, &s->phc);
  A((size_t)std::max(g.nt, 1) * 4 * sizeof(double), (void**)&s->phase);
  A(sizeof(int) * 4, (void**)&s->tdev);
  A(sizeof(int) * 2, (void**)&s->flags);
  if (rc != FDTD_OK) {
    fdtd_destroy(s);
    return rc;
  }
  // phase factors per step: the reference evaluates exp(-1j*omega*t*dt) and
  // exp(-1j*omega*(t-0.5)*dt) in complex128 (cpu/field_updates.py:387,395),
  // i.e. cos/sin of (-omega*t)*dt with omega = 2.0*pi*f (cpu/main_sim.py:124)
  {
    std::vector<double> tab((size_t)std::max(g.nt, 1) * 4);
    const double omega = 2.0 * M_PI * g.frequency;
    for (int t = 0; t < g.nt; ++t) {
      volatile double a = -omega * (double)t;
      const double the = a * g.timestep;
      volatile double b = -omega * ((double)t - 0.5);
      const double thh = b * g.timestep;
      tab[4 * t + 0] = std::cos(the);
      tab[4 * t + 1] = std::sin(the);
      tab[4 * t + 2] = std::cos(thh);
      tab[4 * t + 3] = std::sin(thh);
    }
    cudaError_t e = cudaMemcpy(s->phase, tab.data(), tab.size() * sizeof(double),
                               cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      fdtd_destroy(s);
      return fail(FDTD_ERR_CUDA, "phase table upload: %s", cudaGetErrorString(e));
    }
  }
  cudaError_t e = cudaStreamCreateWithFlags(&s->own, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    fdtd_destroy(s);
    return fail(FDTD_ERR_CUDA, "cudaStreamCreate: %s", cudaGetErrorString(e));
  }
  s->stream = s->own;
  if ((e = cudaStreamCreateWithFlags(&s->side, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming)) != cudaSuccess ||
      (e = cudaEventCreateWithFlags(&s->join, cudaEventDisableTiming)) != cudaSuccess) {
    fdtd_destroy(s);
    return fail(FDTD_ERR_CUDA, "stream/event creation: %s", cudaGetErrorString(e));
  }
  rc = fdtd_reset(s);
  if (rc != FDTD_OK) {
    fdtd_destroy(s);
    return rc;
  }
  *out = s;
  return FDTD_OK;
}

int fdtd_destroy(fdtd_sim* s) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  if (!s) return FDTD_OK;
  if (s->batch_refs > 0)
    return fail(FDTD_ERR_STATE, "simulation is a member of %d batch(es): destroy them first",
                s->batch_refs);
  cudaSetDevice(s->device);
  if (s->own) cudaStreamSynchronize(s->own);
  for (auto& b : s->bufs) {
    check_unregister(b.p);
    cudaFree(b.p);
  }
  if (s->side) cudaStreamSynchronize(s->side);
  if (s->copy) cudaStreamSynchronize(s->copy);
  for (int k = 0; k < 2; ++k) {
    if (s->copy_ev[k]) cudaEventDestroy(s->copy_ev[k]);
    if (s->stage[k]) cudaFreeHost(s->stage[k]);
  }
  if (s->copy) cudaStreamDestroy(s->copy);
  for (auto e : s->ev) cudaEventDestroy(e);
  for (int k = 0; k < 2; ++k)
    if (s->gexec[k]) cudaGraphExecDestroy(s->gexec[k]);
  if (s->fork) cudaEventDestroy(s->fork);
  if (s->join) cudaEventDestroy(s->join);
  if (s->side) cudaStreamDestroy(s->side);
  if (s->own) cudaStreamDestroy(s->own);
  delete s;
  cudaGetLastError();
  return FDTD_OK;
}

int fdtd_set_option(fdtd_sim* s, int option, int value) {
  if (!s) return fail(FDTD_ERR_INVALID, "null simulation handle");
  switch (option) {
    case FDTD_OPT_KERNEL:
      if (value != FDTD_KERNEL_SPLIT && value != FDTD_KERNEL_FUSED)
        return fail(FDTD_ERR_INVALID, "unknown kernel %d", value);
      s->kernel = value;
      return FDTD_OK;
    case FDTD_OPT_PHASOR_MODE:
      if (value != FDTD_PHASOR_REFERENCE && value != FDTD_PHASOR_KAHAN)
        return fail(FDTD_ERR_INVALID, "unknown phasor mode %d", value);
      if (s->t != 0 && value != s->phasor_mode)
        return fail(FDTD_ERR_STATE, "phasor mode can only change before the first step");
      s->phasor_mode = value;
      return FDTD_OK;
    case FDTD_OPT_TILE_X:
      if (value < 4 || value > 256 || value % 4) return fail(FDTD_ERR_INVALID, "bad tile_x %d", value);
      s->tile_x = value;
      return FDTD_OK;
    case FDTD_OPT_TILE_Y:
      if (value < 1 || value > 64) return fail(FDTD_ERR_INVALID, "bad tile_y %d", value);
      s->tile_y = value;
      return FDTD_OK;
    case FDTD_OPT_ZCHUNK:
      if (value < 0) return fail(FDTD_ERR_INVALID, "bad z chunk %d", value);
      s->zchunk = value;
      return FDTD_OK;
    case FDTD_OPT_FUSED_SLAB:
      if (value < 0 || value > 2) return fail(FDTD_ERR_INVALID, "FDTD_OPT_FUSED_SLAB %d: 0, 1 or 2", value);
      s->slab = value;
      return FDTD_OK;
    case FDTD_OPT_SHELL:
      if (value != FDTD_SHELL_MARCH && value != FDTD_SHELL_SPLIT)
        return fail(FDTD_ERR_INVALID, "unknown shell mode %d", value);
      s->shell = value;
      return FDTD_OK;
    case FDTD_OPT_GRAPH_CHUNK:
      if (value < 0) return fail(FDTD_ERR_INVALID, "bad graph chunk %d", value);
      s->graph_chunk = value;
      return FDTD_OK;
    case FDTD_OPT_CHECK_EVERY:
      if (value < 0) return fail(FDTD_ERR_INVALID, "bad check period %d", value);
      s->check_every = value;
      return FDTD_OK;
    case FDTD_OPT_TIMING:
      s->timing = value ? 1 : 0;
      return FDTD_OK;
  }
  return fail(FDTD_ERR_INVALID, "unknown option %d", option);
}

int fdtd_get_option(fdtd_sim* s, int option, int* value) {
  if (!s || !value) return fail(FDTD_ERR_INVALID, "null argument");
  switch (option) {
    case FDTD_OPT_KERNEL: *value = s->kernel; return FDTD_OK;
    case FDTD_OPT_PHASOR_MODE: *value = s->phasor_mode; return FDTD_OK;
    case FDTD_OPT_TILE_X: *value = s->tile_x; return FDTD_OK;
    case FDTD_OPT_TILE_Y: *value = s->tile_y; return FDTD_OK;
    case FDTD_OPT_ZCHUNK: *value = s->zchunk; return FDTD_OK;
    case FDTD_OPT_FUSED_SLAB: *value = s->slab; return FDTD_OK;
    case FDTD_OPT_SHELL: *value = s->shell; return FDTD_OK;
    case FDTD_OPT_GRAPH_CHUNK: *value = s->graph_chunk; return FDTD_OK;
    case FDTD_OPT_CHECK_EVERY: *value = s->check_every; return FDTD_OK;
    case FDTD_OPT_TIMING: *value = s->timing; return FDTD_OK;
  }
  return fail(FDTD_ERR_INVALID, "unknown option %d", option);
}

int fdtd_set_absorbers(fdtd_sim* s, const void* profiles) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!profiles) return fail(FDTD_ERR_INVALID, "null profiles");
  const size_t n = 8 * (size_t)s->g.npml * s->esz;
  s->prof.assign((const unsigned char*)profiles, (const unsigned char*)profiles + n);
  s->have_abs = true;
  s->graph_epoch++;
  return FDTD_OK;
}

// A host (nz, ny, nx) volume into a pitched device array: one contiguous
// transfer into a packed device buffer and a re-pitch on the device (a
// pitched host-to-device copy moves one short row at a time: 21.6 GB/s
// against the link's full rate for one contiguous block); the pitched copy
// when the packed buffer cannot be had.
static int upload_volume(fdtd_sim* s, void* dst, const void* src) {
  const size_t w = (size_t)s->g.nx * s->esz;
  const long long rows = (long long)s->g.ny * s->g.nz;
  if (!s->packed && alloc(s, w * rows, &s->packed) != FDTD_OK) s->packed = nullptr;
  s->mat_nz = -1;   // the staging buffer now holds a coefficient volume
  if (s->packed) {
    CK(cudaMemcpyAsync(s->packed, src, w * rows, cudaMemcpyHostToDevice, s->stream));
    if (s->g.dtype == FDTD_F32)
      launch_repitch<float>((float*)dst, (const float*)s->packed, s->g.nx, rows, s->pitch, s->stream);
    else
      launch_repitch<double>((double*)dst, (const double*)s->packed, s->g.nx, rows, s->pitch, s->stream);
    CK(cudaGetLastError());
  } else {
    CK(cudaMemcpy2DAsync(dst, (size_t)s->pitch * s->esz, src, w, w, (size_t)rows, cudaMemcpyHostToDevice,
                         s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_set_materials(fdtd_sim* s, const void* ca, const void* cb) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!ca || !cb) return fail(FDTD_ERR_INVALID, "null Ca/Cb");
  if ((rc = upload_volume(s, s->ca, ca))) return rc;
  if ((rc = upload_volume(s, s->cb, cb))) return rc;
  s->have_mat = true;
  return FDTD_OK;
}

int fdtd_set_materials_eps_sigma(fdtd_sim* s, const void* eps_r, const void* sigma, int nz_mat) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!eps_r || !sigma) return fail(FDTD_ERR_INVALID, "null eps/sigma");
  const fdtd_geometry& g = s->g;
  if (nz_mat < 0 || nz_mat > g.nz) return fail(FDTD_ERR_INVALID, "nz_mat %d outside [0, %d]", nz_mat, g.nz);
  const size_t n = (size_t)nz_mat * g.ny * g.nx;
  if ((rc = stage_buffers(s))) return rc;
  void* de = s->packed;
  void* ds = s->packed2;
  CK(cudaMemcpyAsync(de, eps_r, n * s->esz, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(ds, sigma, n * s->esz, cudaMemcpyHostToDevice, s->stream));
  s->mat_nz = nz_mat;
  return materials_from_stage(s);
}

int fdtd_fill_layers(fdtd_sim* s, int nz_mat, int nlayers, const double* heights, const double* eps_r,
                     const double* sigma) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  const fdtd_geometry& g = s->g;
  if (nz_mat < 0 || nz_mat > g.nz) return fail(FDTD_ERR_INVALID, "nz_mat %d outside [0, %d]", nz_mat, g.nz);
  if (nlayers < 0 || nlayers > 64) return fail(FDTD_ERR_INVALID, "%d layers (0 to 64)", nlayers);
  if ((nlayers > 0 && !heights) || !eps_r || !sigma) return fail(FDTD_ERR_INVALID, "null argument");
  if ((rc = stage_buffers(s))) return rc;
  const size_t plane = (size_t)g.ny * g.nx;
  const size_t hbytes = sizeof(double) * (plane * nlayers + 2 * (nlayers + 1));
  double* d = nullptr;
  if ((rc = mat_scratch(s, hbytes, (void**)&d))) return rc;
  double* dh = d;
  double* dev = d + plane * nlayers;
  double* dsv = dev + nlayers + 1;
  if (nlayers) CK(cudaMemcpyAsync(dh, heights, sizeof(double) * plane * nlayers, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(dev, eps_r, sizeof(double) * (nlayers + 1), cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(dsv, sigma, sizeof(double) * (nlayers + 1), cudaMemcpyHostToDevice, s->stream));
  if (nz_mat > 0) {
    if (g.dtype == FDTD_F32)
      launch_fill_layers<float>((float*)s->packed, (float*)s->packed2, g.nx, g.ny, nz_mat, nlayers, dh, dev, dsv,
                                s->stream);
    else
      launch_fill_layers<double>((double*)s->packed, (double*)s->packed2, g.nx, g.ny, nz_mat, nlayers, dh, dev,
                                 dsv, s->stream);
    CK(cudaGetLastError());
  }
  CK(cudaStreamSynchronize(s->stream));   // the scratch is reused by the next call
  s->mat_nz = nz_mat;
  return take_bounds_violation();
}

int fdtd_paint_spheres(fdtd_sim* s, int n, const double* spheres, double eps_r, double sigma) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (s->mat_nz < 0) return fail(FDTD_ERR_STATE, "no staged material block (fdtd_fill_layers)");
  if (n < 0 || (n > 0 && !spheres)) return fail(FDTD_ERR_INVALID, "bad sphere list");
  if (n == 0) return FDTD_OK;
  const fdtd_geometry& g = s->g;
  for (int k = 0; k < n; ++k) {
    const double ri = spheres[5 * k + 4];
    if (!(ri >= 0 && ri <= 64 && ri == (double)(int)ri))
      return fail(FDTD_ERR_INVALID, "sphere %d: integer radius %g outside [0, 64]", k, ri);
  }
  double* d = nullptr;
  if ((rc = mat_scratch(s, sizeof(double) * 5 * (size_t)n, (void**)&d))) return rc;
  CK(cudaMemcpyAsync(d, spheres, sizeof(double) * 5 * (size_t)n, cudaMemcpyHostToDevice, s->stream));
  if (g.dtype == FDTD_F32)
    launch_paint_spheres<float>((float*)s->packed, (float*)s->packed2, g.nx, g.ny, s->mat_nz, d, n, eps_r, sigma,
                                s->stream);
  else
    launch_paint_spheres<double>((double*)s->packed, (double*)s->packed2, g.nx, g.ny, s->mat_nz, d, n, eps_r,
                                 sigma, s->stream);
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  return take_bounds_violation();
}

int fdtd_set_materials_staged(fdtd_sim* s) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (s->mat_nz < 0) return fail(FDTD_ERR_STATE, "no staged material block (fdtd_fill_layers)");
  return materials_from_stage(s);
}

int fdtd_get_staged_materials(fdtd_sim* s, int nz_mat, void* eps_r, void* sigma) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!eps_r || !sigma) return fail(FDTD_ERR_INVALID, "null argument");
  if (s->mat_nz < 0) return fail(FDTD_ERR_STATE, "no staged material block");
  if (nz_mat != s->mat_nz)
    return fail(FDTD_ERR_INVALID, "staged block has %d planes, not %d", s->mat_nz, nz_mat);
  const size_t n = (size_t)s->mat_nz * s->g.ny * s->g.nx * s->esz;
  CK(cudaMemcpyAsync(eps_r, s->packed, n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaMemcpyAsync(sigma, s->packed2, n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_set_incident(fdtd_sim* s, const void* ex, const void* ey, const void* hx, const void* hy,
                      int nt_inc) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  const fdtd_geometry& g = s->g;
  if (nt_inc != g.nt_inc)
    return fail(FDTD_ERR_INVALID, "incident beam has %d steps, geometry expects %d", nt_inc, g.nt_inc);
  const void* src[4] = {ex, ey, hx, hy};
  for (int c = 0; c < 4; ++c)
    if (!src[c] && nt_inc > 0) return fail(FDTD_ERR_INVALID, "null incident component %d", c);
  const size_t bytes = (size_t)std::max(nt_inc, 1) * s->plane * s->esz;
  for (int c = 0; c < 4; ++c) {
    if (!s->inc[c]) {
      if ((rc = alloc(s, bytes, &s->inc[c]))) return rc;
    }
    if (nt_inc > 0) {
      const size_t w = (size_t)g.nx * s->esz;
      CK(cudaMemcpy2DAsync(s->inc[c], (size_t)s->pitch * s->esz, src[c], w, w,
                           (size_t)g.ny * nt_inc, cudaMemcpyHostToDevice, s->stream));
    }
  }
  CK(cudaStreamSynchronize(s->stream));
  s->inc_nt = nt_inc;
  return FDTD_OK;
}

int fdtd_reset(fdtd_sim* s) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  const size_t fb = (size_t)s->vol * s->esz;
  for (int set = 0; set < 2; ++set)
    for (int c = 0; c < 6; ++c) CK(cudaMemsetAsync(s->fld[set][c], 0, fb, s->stream));
  for (int set = 0; set < 2; ++set)
    CK(cudaMemsetAsync(s->psi_base[set], 0, (size_t)s->psi_elems * s->esz, s->stream));
  CK(cudaMemsetAsync(s->ph, 0, (size_t)s->ph_elems * s->esz, s->stream));
  CK(cudaMemsetAsync(s->phc, 0, (size_t)s->ph_elems * s->esz, s->stream));
  CK(cudaMemsetAsync(s->tdev, 0, sizeof(int) * 4, s->stream));
  CK(cudaMemsetAsync(s->flags, 0, sizeof(int) * 2, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  s->t = 0;
  s->cur = 0;
  return FDTD_OK;
}

int fdtd_run(fdtd_sim* s, int nsteps) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (nsteps < 0) return fail(FDTD_ERR_INVALID, "negative step count");
  if (!s->have_abs) return fail(FDTD_ERR_STATE, "absorbers not set (fdtd_set_absorbers)");
  if (!s->have_mat) return fail(FDTD_ERR_STATE, "materials not set (fdtd_set_materials)");
  if (s->t + nsteps > s->g.nt)
    return fail(FDTD_ERR_INVALID, "step %lld + %d exceeds size_t %d", (long long)s->t, nsteps, s->g.nt);
  if (s->g.nt_inc > 0 && s->t < s->g.nt_inc && s->inc_nt < s->g.nt_inc)
    return fail(FDTD_ERR_STATE, "incident beam not set (fdtd_set_incident)");
  if (nsteps == 0) return FDTD_OK;
  return s->g.dtype == FDTD_F32 ? run_steps<float>(s, nsteps) : run_steps<double>(s, nsteps);
}

int fdtd_run_streamed(fdtd_sim* s, int nsteps, const void* ex, const void* ey, const void* hx,
                      const void* hy) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (nsteps < 0) return fail(FDTD_ERR_INVALID, "negative step count");
  if (!s->have_abs) return fail(FDTD_ERR_STATE, "absorbers not set (fdtd_set_absorbers)");
  if (!s->have_mat) return fail(FDTD_ERR_STATE, "materials not set (fdtd_set_materials)");
  const fdtd_geometry& g = s->g;
  if (s->t + nsteps > g.nt)
    return fail(FDTD_ERR_INVALID, "step %lld + %d exceeds size_t %d", (long long)s->t, nsteps, g.nt);
  const int t0 = (int)s->t, t1 = t0 + nsteps;
  // planes [t0, need) come from the given arrays; earlier ones are not
  // read again
  const int need = std::min(t1, g.nt_inc);
  if (need <= t0) {
    if ((rc = fdtd_run(s, nsteps))) return rc;
    return fdtd_synchronize(s);
  }
  const void* src[4] = {ex, ey, hx, hy};
  for (int c = 0; c < 4; ++c)
    if (!src[c]) return fail(FDTD_ERR_INVALID, "null incident component %d", c);
  const size_t pb = (size_t)s->plane * s->esz;           // one pitched device plane
  const size_t row = (size_t)g.nx * s->esz;
  const size_t hb = row * g.ny;                         // one packed host plane
  for (int c = 0; c < 4; ++c)
    if (!s->inc[c] && (rc = alloc(s, pb * std::max(g.nt_inc, 1), &s->inc[c]))) return rc;
  if (!s->copy) {
    CK(cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking));
    for (int k = 0; k < 2; ++k) CK(cudaEventCreateWithFlags(&s->copy_ev[k], cudaEventDisableTiming));
  }
  // Page-locked host planes are copied straight from the caller's arrays;
  // pageable ones through two pinned staging slots (a host copy into a slot
  // waits for that slot's previous transfer).
  bool pinned = true;
  for (int c = 0; c < 4; ++c) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, src[c]) != cudaSuccess || at.type != cudaMemoryTypeHost) pinned = false;
  }
  cudaGetLastError();
  const int chunk = 16;   // steps whose planes travel in one transfer
  if (!pinned && s->stage_bytes < 4 * hb * chunk) {
    for (int k = 0; k < 2; ++k) {
      if (s->stage[k]) cudaFreeHost(s->stage[k]);
      s->stage[k] = nullptr;
    }
    s->stage_bytes = 0;
    for (int k = 0; k < 2; ++k) CK(cudaHostAlloc(&s->stage[k], 4 * hb * chunk, cudaHostAllocDefault));
    s->stage_bytes = 4 * hb * chunk;
  }
  // Each group's planes cross as one contiguous transfer per component into
  // a device staging slot, then a kernel on the copy stream re-pitches them
  // into the incident buffers (pitched 2-D transfers of short rows ran well
  // below the link's bandwidth). A slot is reused two groups later, after
  // its re-pitch (same stream). Without room for the slots, 2-D transfers.
  const size_t dslot = 4 * hb * chunk;
  if (!s->dstage && alloc(s, 2 * dslot, &s->dstage) == FDTD_OK) s->dstage_bytes = 2 * dslot;
  if (s->dstage && s->dstage_bytes < 2 * dslot) {
    release(s, s->dstage);
    s->dstage = nullptr;
    s->dstage_bytes = 0;
    if (alloc(s, 2 * dslot, &s->dstage) == FDTD_OK) s->dstage_bytes = 2 * dslot;
  }
  cudaGetLastError();
  // the first group is short, so that the stepping starts early
  for (int c0 = t0, slot = 0, grp = std::min(2, chunk); c0 < t1; c0 += grp, slot ^= 1, grp = chunk) {
    const int n = std::min(grp, t1 - c0);
    const int p1 = std::min(c0 + n, need);
    if (p1 > c0) {
      const size_t np = (size_t)(p1 - c0);
      for (int c = 0; c < 4; ++c) {
        const unsigned char* from = static_cast<const unsigned char*>(src[c]) + (size_t)c0 * hb;
        if (!pinned) {
          if (c == 0) CK(cudaEventSynchronize(s->copy_ev[slot]));
          unsigned char* st = static_cast<unsigned char*>(s->stage[slot]) + (size_t)c * hb * chunk;
          memcpy(st, from, np * hb);
          from = st;
        }
        unsigned char* to = static_cast<unsigned char*>(s->inc[c]) + (size_t)c0 * pb;
        if (s->dstage) {
          unsigned char* d = static_cast<unsigned char*>(s->dstage) + slot * dslot + (size_t)c * hb * chunk;
          CK(cudaMemcpyAsync(d, from, np * hb, cudaMemcpyHostToDevice, s->copy));
          if (g.dtype == FDTD_F32)
            launch_repitch<float>((float*)to, (const float*)d, g.nx, (long long)g.ny * np, s->pitch, s->copy);
          else
            launch_repitch<double>((double*)to, (const double*)d, g.nx, (long long)g.ny * np, s->pitch, s->copy);
        } else {
          CK(cudaMemcpy2DAsync(to, (size_t)s->pitch * s->esz, from, row, row, (size_t)g.ny * np,
                               cudaMemcpyHostToDevice, s->copy));
        }
      }
      CK(cudaEventRecord(s->copy_ev[slot], s->copy));
      CK(cudaStreamWaitEvent(s->stream, s->copy_ev[slot], 0));
    }
    rc = g.dtype == FDTD_F32 ? enqueue_steps<float>(s, n) : enqueue_steps<double>(s, n);
    if (rc) return rc;
    s->t += n;
  }
  if (t0 <= s->inc_nt) s->inc_nt = std::max(s->inc_nt, need);
  return fdtd_synchronize(s);
}

int fdtd_synchronize(fdtd_sim* s) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  CK(cudaGetLastError());
  if ((rc = take_bounds_violation())) return rc;
  if (s->check_every > 0) {
    int f[2] = {0, 0};
    CK(cudaMemcpy(f, s->flags, sizeof(f), cudaMemcpyDeviceToHost));
    if (f[0]) return fail(FDTD_ERR_NONFINITE, "non-finite field value found after step %d", f[1]);
  }
  return FDTD_OK;
}

int fdtd_step_index(fdtd_sim* s, int64_t* t) {
  if (!s || !t) return fail(FDTD_ERR_INVALID, "null argument");
  *t = s->t;
  return FDTD_OK;
}

int fdtd_get_stream(fdtd_sim* s, void** stream) {
  if (!s || !stream) return fail(FDTD_ERR_INVALID, "null argument");
  *stream = (void*)s->stream;
  return FDTD_OK;
}

int fdtd_set_stream(fdtd_sim* s, void* stream) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  CK(cudaStreamSynchronize(s->stream));
  s->stream = stream ? (cudaStream_t)stream : s->own;
  return FDTD_OK;
}

int fdtd_get_kernel_time(fdtd_sim* s, int kind, double* total_ms, int* launches) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (kind != FDTD_TIME_STEP && kind != FDTD_TIME_PHASOR)
    return fail(FDTD_ERR_INVALID, "unknown kernel kind %d", kind);
  if ((rc = collect_timing(s))) return rc;
  if (total_ms) *total_ms = s->acc_ms[kind];
  if (launches) *launches = s->acc_n[kind];
  return FDTD_OK;
}

int fdtd_clear_kernel_time(fdtd_sim* s) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if ((rc = collect_timing(s))) return rc;
  s->acc_ms[0] = s->acc_ms[1] = 0;
  s->acc_n[0] = s->acc_n[1] = 0;
  return FDTD_OK;
}

int fdtd_get_phasor(fdtd_sim* s, int plane, void* out) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (plane < 0 || plane >= 24) return fail(FDTD_ERR_INVALID, "phasor plane %d outside [0, 24)", plane);
  if (!out) return fail(FDTD_ERR_INVALID, "null output");
  long long n;
  if (plane < 8) n = (long long)s->ny_ph * s->nx_ph;
  else if (plane < 16) n = (long long)s->nz_ph * s->ny_ph;
  else n = (long long)s->nz_ph * s->nx_ph;
  CK(cudaMemcpyAsync(out, (char*)s->ph + s->ph_off[plane] * s->esz, (size_t)(2 * n) * s->esz,
                     cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_get_phasors(fdtd_sim* s, void* out) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!out) return fail(FDTD_ERR_INVALID, "null output");
  size_t off = 0;
  for (int plane = 0; plane < 24; ++plane) {
    long long n;
    if (plane < 8) n = (long long)s->ny_ph * s->nx_ph;
    else if (plane < 16) n = (long long)s->nz_ph * s->ny_ph;
    else n = (long long)s->nz_ph * s->nx_ph;
    const size_t bytes = (size_t)(2 * n) * s->esz;
    CK(cudaMemcpyAsync(static_cast<unsigned char*>(out) + off, (char*)s->ph + s->ph_off[plane] * s->esz, bytes,
                       cudaMemcpyDeviceToHost, s->stream));
    off += bytes;
  }
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_get_field(fdtd_sim* s, int comp, void* out) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (comp < 0 || comp >= 6) return fail(FDTD_ERR_INVALID, "field component %d outside [0, 6)", comp);
  if (!out) return fail(FDTD_ERR_INVALID, "null output");
  const size_t w = (size_t)s->g.nx * s->esz;
  CK(cudaMemcpy2DAsync(out, w, s->fld[s->cur][comp], (size_t)s->pitch * s->esz, w,
                       (size_t)s->g.ny * s->g.nz, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_set_field(fdtd_sim* s, int comp, const void* in) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (comp < 0 || comp >= 6) return fail(FDTD_ERR_INVALID, "field component %d outside [0, 6)", comp);
  if (!in) return fail(FDTD_ERR_INVALID, "null input");
  return upload_volume(s, s->fld[s->cur][comp], in);
}

}  // extern "C"

extern "C" int fdtd_near2far(const void* ex_u, const void* ey_u, const void* hx_u,
                             const void* hy_u, int in_dtype, int nx_ph, int ny_ph, int nz_ph,
                             double dx, double r, const double* thetas_deg, int ntheta,
                             const double* phis_deg, int nphi, double freq, int device,
                             double* out) {
  if (!ex_u || !ey_u || !hx_u || !hy_u || !thetas_deg || !phis_deg || !out)
    return fail(FDTD_ERR_INVALID, "null argument");
  if (in_dtype != FDTD_F32 && in_dtype != FDTD_F64)
    return fail(FDTD_ERR_INVALID, "in_dtype must be FDTD_F32 or FDTD_F64");
  if (nx_ph < 3 || ny_ph < 3 || nx_ph % 2 == 0 || ny_ph % 2 == 0)
    return fail(FDTD_ERR_INVALID,
                "phasor plane %dx%d: Simpson integration needs odd sample counts >= 3", ny_ph, nx_ph);
  if (ntheta < 1 || nphi < 1 || nz_ph < 1) return fail(FDTD_ERR_INVALID, "empty angle or plane set");
  if (!(freq > 0) || !(dx > 0) || !(r > 0)) return fail(FDTD_ERR_INVALID, "freq, dx, r must be positive");
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
    cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "no CUDA device available");
  }
  if (device < 0 || device >= ndev) return fail(FDTD_ERR_INVALID, "device %d out of range", device);
  DeviceGuard device_guard;   // the caller's current device is restored on return
  CK(cudaSetDevice(device));
  // surface currents in complex128, as near2far.py:64-68 converts them:
  // Jx = -Hy, Jy = Hx, Mx = Ey, My = -Ex   (near2far.py:94-96)
  const size_t n = (size_t)nx_ph * ny_ph;
  std::vector<double> jm(8 * n);
  auto get = [&](const void* p, size_t i, int part) -> double {
    return in_dtype == FDTD_F32 ? (double)((const float*)p)[2 * i + part]
                                : ((const double*)p)[2 * i + part];
  };
  for (size_t i = 0; i < n; ++i) {
    for (int part = 0; part < 2; ++part) {
      jm[2 * (0 * n + i) + part] = -get(hy_u, i, part);
      jm[2 * (1 * n + i) + part] = get(hx_u, i, part);
      jm[2 * (2 * n + i) + part] = get(ey_u, i, part);
      jm[2 * (3 * n + i) + part] = -get(ex_u, i, part);
    }
  }
  std::vector<double> th(ntheta), ph(nphi);
  for (int i = 0; i < ntheta; ++i) th[i] = thetas_deg[i] * (M_PI / 180.0);
  for (int i = 0; i < nphi; ++i) ph[i] = phis_deg[i] * (M_PI / 180.0);
  const double c0 = 299792458.0;
  const double lam = c0 / freq;
  const double k = 2.0 * M_PI / lam;
  const double z_val = (double)((nz_ph - 1) / 2) * dx;
  double *djm = nullptr, *dth = nullptr, *dph = nullptr, *dout = nullptr;
  const size_t out_n = (size_t)8 * nphi * ntheta;
  cudaStream_t st;
  CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
  int rc = FDTD_OK;
  do {
    if (cudaMallocAsync(&djm, jm.size() * sizeof(double), st) != cudaSuccess ||
        cudaMallocAsync(&dth, th.size() * sizeof(double), st) != cudaSuccess ||
        cudaMallocAsync(&dph, ph.size() * sizeof(double), st) != cudaSuccess ||
        cudaMallocAsync(&dout, out_n * sizeof(double), st) != cudaSuccess) {
      rc = fail(FDTD_ERR_NOMEM, "near2far device allocation failed");
      break;
    }
    cudaMemcpyAsync(djm, jm.data(), jm.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dth, th.data(), th.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dph, ph.data(), ph.size() * sizeof(double), cudaMemcpyHostToDevice, st);
    if (near2far_run(djm, nx_ph, ny_ph, dx, z_val, k, dth, ntheta, dph, nphi, r, dout, st)) {
      rc = fail(FDTD_ERR_CUDA, "near2far launch failed: %s", cudaGetErrorString(cudaGetLastError()));
      break;
    }
    cudaMemcpyAsync(out, dout, out_n * sizeof(double), cudaMemcpyDeviceToHost, st);
  } while (0);
  if (djm) cudaFreeAsync(djm, st);
  if (dth) cudaFreeAsync(dth, st);
  if (dph) cudaFreeAsync(dph, st);
  if (dout) cudaFreeAsync(dout, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaStreamDestroy(st);
  if (rc == FDTD_OK && e != cudaSuccess)
    rc = fail(FDTD_ERR_CUDA, "near2far: %s", cudaGetErrorString(e));
  return rc;
}

// ---------------------------------------------------------------------------
// batched sweep
// ---------------------------------------------------------------------------
namespace {

template <class T>
int batch_build_table(fdtd_batch* b) {
  // the batch's earlier steps may still read the table: they finish first
  CK(cudaStreamSynchronize(b->stream));
  const int n = (int)b->sims.size();
  std::vector<BatchModel<T>> tab(n);
  std::vector<int> start(n + 1), start_ph(n + 1);
  long long blk = 0, blk_ph = 0;
  for (int m = 0; m < n; ++m) {
    fdtd_sim* s = b->sims[m];
    BatchModel<T>& bm = tab[m];
    memset(&bm, 0, sizeof(bm));
    bm.s = make_state<T>(s, s->cur, s->cur);
    bm.tdev = s->tdev;
    // row width with the least x padding (ties: the wider rows)
    bm.width = 32;
    long long best = 1LL << 62;
    for (int w : {32, 16, 8}) {
      const long long gx = (s->g.nx + 4 * w - 1) / (4 * w), gy = (s->g.ny + 128 / w - 1) / (128 / w);
      const long long padded = gx * 4 * w * gy * (128 / w);
      if (padded < best) { best = padded; bm.width = w; }
    }
    bm.gx = (s->g.nx + 4 * bm.width - 1) / (4 * bm.width);
    bm.gy = (s->g.ny + 128 / bm.width - 1) / (128 / bm.width);
    bm.ph_n = std::max(s->ny_ph * s->nx_ph, std::max(s->nz_ph * s->ny_ph, s->nz_ph * s->nx_ph));
    start[m] = (int)blk;
    start_ph[m] = (int)blk_ph;
    blk += (long long)bm.gx * bm.gy * ((s->g.nz + kBatchShellPlanes - 1) / kBatchShellPlanes);
    blk_ph += 6LL * ((bm.ph_n + 255) / 256);
    if (blk > INT32_MAX || blk_ph > INT32_MAX) return fail(FDTD_ERR_INVALID, "batch too large");
  }
  start[n] = (int)blk;
  start_ph[n] = (int)blk_ph;
  CK(cudaMemcpy(b->d_models, tab.data(), sizeof(BatchModel<T>) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_start, start.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_start_ph, start_ph.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  b->blocks = (int)blk;
  b->blocks_ph = (int)blk_ph;
  b->sig.resize(n);
  for (int m = 0; m < n; ++m) b->sig[m] = b->sims[m]->cur;
  b->table_ok = true;
  if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
  return FDTD_OK;
}

template <class T>
void batch_enqueue(fdtd_batch* b, int nsteps) {
  const int n = (int)b->sims.size();
  const auto* bm = static_cast<const BatchModel<T>*>(b->d_models);
  for (int k = 0; k < nsteps; ++k)
    launch_batch_step<T>(bm, b->d_start, n, b->blocks, b->d_start_ph, b->blocks_ph, k, b->stream);
  launch_batch_advance<T>(bm, n, nsteps, b->stream);
}

template <class T>
int batch_run(fdtd_batch* b, int nsteps) {
  bool stale = !b->table_ok;
  for (size_t m = 0; m < b->sims.size(); ++m) stale = stale || b->sig[m] != b->sims[m]->cur;
  if (stale) {
    int rc = batch_build_table<T>(b);
    if (rc) return rc;
  }
  // order after the members' own work
  for (fdtd_sim* s : b->sims) {
    CK(cudaEventRecord(b->ev, s->stream));
    CK(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  int left = nsteps;
  const int chunk = b->graph_chunk;
  if (chunk > 0 && left >= chunk) {
    if (!b->gexec || b->gexec_chunk != chunk) {
      if (b->gexec) { cudaGraphExecDestroy(b->gexec); b->gexec = nullptr; }
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      batch_enqueue<T>(b, chunk);
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&b->gexec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        b->gexec = nullptr;
        return fail(FDTD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
      }
      b->gexec_chunk = chunk;
    }
    while (left >= chunk) {
      CK(cudaGraphLaunch(b->gexec, b->stream));
      left -= chunk;
    }
  }
  if (left > 0) batch_enqueue<T>(b, left);
  CK(cudaGetLastError());
  // members' later calls are ordered after the batch
  CK(cudaEventRecord(b->ev, b->stream));
  for (fdtd_sim* s : b->sims) {
    CK(cudaStreamWaitEvent(s->stream, b->ev, 0));
    s->t += nsteps;
  }
  return FDTD_OK;
}

// FDTD_BATCH_QUEUE: the interior tiles of every member's fused step,
// longest first (z chunks of kQueueZChunk planes), for the persistent
// queue; the shell boxes of every member (as the fused plan cuts them) for
// the batched split passes; and per member a State for each parity of the
// step within a run (parity 0 reads the member's current set).
constexpr int kQueueZChunk = 32;

template <class T>
int batch_build_queue(fdtd_batch* b) {
  // the batch's earlier steps may still read the tables: they finish first
  // (the blocking copies below do not wait for a non-blocking stream)
  CK(cudaStreamSynchronize(b->stream));
  const int n = (int)b->sims.size();
  std::vector<BatchModel<T>> tab(2 * (size_t)n);
  std::vector<QueueMember> qm(n);
  std::vector<QueueTile> tiles;
  std::vector<double> cost;
  std::vector<int> start_ph(n + 1);
  std::vector<BatchShellBox> shell;
  long long shell_blocks = 0;
  long long blk_ph = 0;
  for (int m = 0; m < n; ++m) {
    fdtd_sim* s = b->sims[m];
    const fdtd_geometry& g = s->g;
    const int ph_n = std::max(s->ny_ph * s->nx_ph, std::max(s->nz_ph * s->ny_ph, s->nz_ph * s->nx_ph));
    for (int p = 0; p < 2; ++p) {
      const int src = p == 0 ? s->cur : 1 - s->cur;
      BatchModel<T>& bm = tab[(size_t)p * n + m];
      memset(&bm, 0, sizeof(bm));
      bm.s = make_state<T>(s, src, 1 - src);
      bm.tdev = s->tdev;
      bm.ph_n = ph_n;
    }
    const FusedPlan plan = make_fused_plan(g.nx, g.ny, g.nz, g.npml, g.tfsf_z, 4, kQueueZChunk, 0, false);
    if (plan.shell.dropped) return fail(FDTD_ERR_INVALID, "member %d: too many shell boxes", m);
    QueueMember& q = qm[m];
    memset(&q, 0, sizeof(q));
    q.has_interior = plan.has_interior;
    q.ib = plan.interior;
    for (int k = 0; k < plan.shell.n; ++k) {
      BatchShellBox e;
      e.member = m;
      e.b = plan.shell.b[k];
      const long long nb =
          (long long)e.b.gx * e.b.gy * ((e.b.z1 - e.b.z0 + kBatchShellPlanes - 1) / kBatchShellPlanes);
      if (nb <= 0) continue;
      e.b.first = (int)shell_blocks;
      shell_blocks += nb;
      if (shell_blocks > INT32_MAX) return fail(FDTD_ERR_INVALID, "batch too large");
      shell.push_back(e);
    }
    if (plan.has_interior) {
      const InteriorBox& ib = plan.interior;
      const int gx = (ib.xb - ib.xa + 127) / 128, gy = (ib.yb - ib.ya + 3) / 4;
      for (int c = 0; c < ib.chunks; ++c) {
        const int k = c < ib.chunks0 ? 0 : 1, cc = k ? c - ib.chunks0 : c;
        const int z0 = ib.z0[k] + cc * ib.zchunk, z1 = std::min(ib.z1[k], z0 + ib.zchunk);
        for (int by = 0; by < gy; ++by)
          for (int bx = 0; bx < gx; ++bx) {
            tiles.push_back({m, bx, by, c});
            cost.push_back(512.0 * (z1 - z0 + 1));
          }
      }
    }
    start_ph[m] = (int)blk_ph;
    blk_ph += 6LL * ((ph_n + 255) / 256);
    if (tiles.size() > (size_t)INT32_MAX / 2 || blk_ph > INT32_MAX) return fail(FDTD_ERR_INVALID, "batch too large");
  }
  start_ph[n] = (int)blk_ph;
  // longest first: the long tiles start early, the short ones fill the end
  std::vector<int> order(tiles.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return cost[x] > cost[y]; });
  std::vector<QueueTile> sorted(tiles.size());
  for (size_t i = 0; i < order.size(); ++i) sorted[i] = tiles[order[i]];
  const size_t tab_bytes = sizeof(BatchModel<T>) * 2 * (size_t)n;
  if (!b->d_qtab) {
    CK(cudaMalloc(&b->d_qtab, tab_bytes));
    CK(cudaMalloc(&b->d_qm, sizeof(QueueMember) * n));
    CK(cudaMalloc(&b->d_qstart_ph, sizeof(int) * (n + 1)));
    CK(cudaMalloc(&b->d_counter, sizeof(int)));
  }
  if (b->d_tiles && (int)sorted.size() != b->ntiles) {
    cudaFree(b->d_tiles);
    b->d_tiles = nullptr;
  }
  if (!b->d_tiles) CK(cudaMalloc(&b->d_tiles, sizeof(QueueTile) * std::max<size_t>(sorted.size(), 1)));
  if (b->d_qshell && (int)shell.size() != b->nqshell) {
    cudaFree(b->d_qshell);
    b->d_qshell = nullptr;
  }
  if (!b->d_qshell) CK(cudaMalloc(&b->d_qshell, sizeof(BatchShellBox) * std::max<size_t>(shell.size(), 1)));
  if (!shell.empty())
    CK(cudaMemcpy(b->d_qshell, shell.data(), sizeof(BatchShellBox) * shell.size(), cudaMemcpyHostToDevice));
  b->nqshell = (int)shell.size();
  b->qshell_blocks = (int)shell_blocks;
  CK(cudaMemcpy(b->d_qtab, tab.data(), tab_bytes, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_qm, qm.data(), sizeof(QueueMember) * n, cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_tiles, sorted.data(), sizeof(QueueTile) * sorted.size(), cudaMemcpyHostToDevice));
  CK(cudaMemcpy(b->d_qstart_ph, start_ph.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
  CK(cudaMemset(b->d_counter, 0, sizeof(int)));
  b->ntiles = (int)sorted.size();
  b->qblocks_ph = (int)blk_ph;
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device));
  const int per_sm = batch_queue_blocks_per_sm<T>();
  if (per_sm < 1) return fail(FDTD_ERR_CUDA, "tile-queue kernel does not fit on an SM");
  b->qblocks = std::max(1, std::min(b->ntiles, per_sm * sms));
  b->qsig.resize(n);
  for (int m = 0; m < n; ++m) b->qsig[m] = b->sims[m]->cur;
  b->qtable_ok = true;
  if (b->qgexec) { cudaGraphExecDestroy(b->qgexec); b->qgexec = nullptr; }
  return FDTD_OK;
}

template <class T>
void batch_queue_enqueue(fdtd_batch* b, int nsteps) {
  const int n = (int)b->sims.size();
  const auto* tab = static_cast<const BatchModel<T>*>(b->d_qtab);
  for (int k = 0; k < nsteps; ++k) {
    const BatchModel<T>* bm = tab + (size_t)(k & 1) * n;
    // the shells' H pass and the interior tiles read the source sets only
    // (run one after the other: beside each other, with the queue at full
    // or half occupancy, the 64-model sweep took 3 to 10 % longer); the
    // shells' E pass reads the destination H both wrote
    launch_batch_shell<T>(bm, b->d_qshell, b->nqshell, b->qshell_blocks, true, k, b->stream);
    launch_batch_queue<T>(bm, b->d_qm, b->d_tiles, b->ntiles, b->d_counter, b->qblocks, b->stream);
    launch_batch_shell<T>(bm, b->d_qshell, b->nqshell, b->qshell_blocks, false, k, b->stream);
    launch_batch_phasors<T>(bm, b->d_qstart_ph, n, b->qblocks_ph, k, b->d_counter, b->stream);
  }
  launch_batch_advance<T>(tab, n, nsteps, b->stream);
}

template <class T>
int batch_run_queue(fdtd_batch* b, int nsteps) {
  bool stale = !b->qtable_ok;
  for (size_t m = 0; m < b->sims.size(); ++m) stale = stale || b->qsig[m] != b->sims[m]->cur;
  if (stale) {
    int rc = batch_build_queue<T>(b);
    if (rc) return rc;
  }
  for (fdtd_sim* s : b->sims) {
    CK(cudaEventRecord(b->ev, s->stream));
    CK(cudaStreamWaitEvent(b->stream, b->ev, 0));
  }
  int left = nsteps;
  // an even chunk leaves every member on its starting set, so each replay
  // starts at parity 0 again
  const int chunk = b->graph_chunk & ~1;
  if (chunk > 0 && left >= chunk) {
    if (!b->qgexec || b->qgexec_chunk != chunk) {
      if (b->qgexec) { cudaGraphExecDestroy(b->qgexec); b->qgexec = nullptr; }
      cudaGraph_t g = nullptr;
      CK(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
      batch_queue_enqueue<T>(b, chunk);
      cudaError_t e = cudaStreamEndCapture(b->stream, &g);
      if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
      e = cudaGraphInstantiate(&b->qgexec, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        b->qgexec = nullptr;
        return fail(FDTD_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
      }
      b->qgexec_chunk = chunk;
    }
    while (left >= chunk) {
      CK(cudaGraphLaunch(b->qgexec, b->stream));
      left -= chunk;
    }
  }
  if (left > 0) batch_queue_enqueue<T>(b, left);
  CK(cudaGetLastError());
  CK(cudaEventRecord(b->ev, b->stream));
  for (fdtd_sim* s : b->sims) {
    CK(cudaStreamWaitEvent(s->stream, b->ev, 0));
    s->t += nsteps;
    if (nsteps & 1) s->cur = 1 - s->cur;
  }
  return FDTD_OK;
}

// FDTD_BATCH_STREAMS: every member advances by its own step path (its
// kernel choice, its graph chunks) on its own stream, forked from the batch
// stream after the batch's earlier work and joined back into it, so that the
// members' small launches run side by side on the device. Each member's
// results are those of fdtd_run on it alone.
template <class T>
int batch_run_streams(fdtd_batch* b, int nsteps) {
  CK(cudaEventRecord(b->ev, b->stream));
  for (fdtd_sim* s : b->sims) CK(cudaStreamWaitEvent(s->stream, b->ev, 0));
  for (fdtd_sim* s : b->sims) {
    const int rc = run_steps<T>(s, nsteps);
    if (rc) return rc;
  }
  for (size_t m = 0; m < b->sims.size(); ++m) {
    CK(cudaEventRecord(b->mev[m], b->sims[m]->stream));
    CK(cudaStreamWaitEvent(b->stream, b->mev[m], 0));
  }
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_batch_create(fdtd_sim* const* sims, int n, fdtd_batch** out) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  if (!out) return fail(FDTD_ERR_INVALID, "null output handle");
  *out = nullptr;
  if (!sims || n < 1) return fail(FDTD_ERR_INVALID, "a batch needs at least one simulation");
  for (int i = 0; i < n; ++i) {
    if (!sims[i]) return fail(FDTD_ERR_INVALID, "null simulation %d", i);
    if (sims[i]->device != sims[0]->device)
      return fail(FDTD_ERR_INVALID, "simulation %d is on another device", i);
    if (sims[i]->g.dtype != sims[0]->g.dtype)
      return fail(FDTD_ERR_INVALID, "simulation %d has another element type", i);
    for (int j = 0; j < i; ++j)
      if (sims[j] == sims[i]) return fail(FDTD_ERR_INVALID, "simulation %d appears twice", i);
  }
  fdtd_batch* b = new fdtd_batch();
  b->sims.assign(sims, sims + n);
  b->device = sims[0]->device;
  b->dtype = sims[0]->g.dtype;
  cudaError_t e = cudaSetDevice(b->device);
  const size_t msz = b->dtype == FDTD_F32 ? sizeof(BatchModel<float>) : sizeof(BatchModel<double>);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_models, msz * n);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_start, sizeof(int) * (n + 1));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_start_ph, sizeof(int) * (n + 1));
  b->mev.assign(n, nullptr);
  for (int i = 0; i < n && e == cudaSuccess; ++i)
    e = cudaEventCreateWithFlags(&b->mev[i], cudaEventDisableTiming);
  if (e != cudaSuccess) {
    fdtd_batch_destroy(b);
    cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "batch set-up: %s", cudaGetErrorString(e));
  }
  for (fdtd_sim* m : b->sims) ++m->batch_refs;
  b->members_counted = true;
  *out = b;
  return FDTD_OK;
}

int fdtd_batch_destroy(fdtd_batch* b) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  if (!b) return FDTD_OK;
  if (b->members_counted)
    for (fdtd_sim* m : b->sims) --m->batch_refs;
  cudaSetDevice(b->device);
  if (b->stream) cudaStreamSynchronize(b->stream);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->d_models) cudaFree(b->d_models);
  if (b->d_start) cudaFree(b->d_start);
  if (b->d_start_ph) cudaFree(b->d_start_ph);
  if (b->qgexec) cudaGraphExecDestroy(b->qgexec);
  if (b->d_qtab) cudaFree(b->d_qtab);
  if (b->d_qm) cudaFree(b->d_qm);
  if (b->d_tiles) cudaFree(b->d_tiles);
  if (b->d_qshell) cudaFree(b->d_qshell);

  if (b->d_counter) cudaFree(b->d_counter);
  if (b->d_qstart_ph) cudaFree(b->d_qstart_ph);
  if (b->ev) cudaEventDestroy(b->ev);
  for (cudaEvent_t ev : b->mev)
    if (ev) cudaEventDestroy(ev);
  if (b->stream) cudaStreamDestroy(b->stream);
  delete b;
  cudaGetLastError();
  return FDTD_OK;
}

int fdtd_batch_set_option(fdtd_batch* b, int option, int value) {
  if (!b) return fail(FDTD_ERR_INVALID, "null batch handle");
  if (option == FDTD_OPT_BATCH_STREAMS) {
    if (value != 0 && value != 1) return fail(FDTD_ERR_INVALID, "batch streams must be 0 or 1");
    b->mode = value == 1 ? FDTD_BATCH_STREAMS : FDTD_BATCH_SPLIT;
    return FDTD_OK;
  }
  if (option == FDTD_OPT_BATCH_MODE) {
    if (value != FDTD_BATCH_SPLIT && value != FDTD_BATCH_STREAMS && value != FDTD_BATCH_QUEUE)
      return fail(FDTD_ERR_INVALID, "unknown batch mode %d", value);
    b->mode = value;
    return FDTD_OK;
  }
  if (option != FDTD_OPT_GRAPH_CHUNK) return fail(FDTD_ERR_INVALID, "unknown batch option %d", option);
  if (value < 0) return fail(FDTD_ERR_INVALID, "bad graph chunk %d", value);
  b->graph_chunk = value;
  return FDTD_OK;
}

int fdtd_batch_run(fdtd_batch* b, int nsteps) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  if (!b) return fail(FDTD_ERR_INVALID, "null batch handle");
  if (nsteps < 0) return fail(FDTD_ERR_INVALID, "negative step count");
  for (size_t m = 0; m < b->sims.size(); ++m) {
    fdtd_sim* s = b->sims[m];
    if (!s->have_abs) return fail(FDTD_ERR_STATE, "member %zu: absorbers not set", m);
    if (!s->have_mat) return fail(FDTD_ERR_STATE, "member %zu: materials not set", m);
    if (s->t + nsteps > s->g.nt)
      return fail(FDTD_ERR_INVALID, "member %zu: step %lld + %d exceeds size_t %d", m,
                  (long long)s->t, nsteps, s->g.nt);
    if (s->g.nt_inc > 0 && s->t < s->g.nt_inc && s->inc_nt < s->g.nt_inc)
      return fail(FDTD_ERR_STATE, "member %zu: incident beam not set", m);
  }
  if (nsteps == 0) return FDTD_OK;
  cudaError_t e = cudaSetDevice(b->device);
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "cudaSetDevice: %s", cudaGetErrorString(e));
  if (b->mode == FDTD_BATCH_STREAMS)
    return b->dtype == FDTD_F32 ? batch_run_streams<float>(b, nsteps)
                                : batch_run_streams<double>(b, nsteps);
  if (b->mode == FDTD_BATCH_QUEUE)
    return b->dtype == FDTD_F32 ? batch_run_queue<float>(b, nsteps) : batch_run_queue<double>(b, nsteps);
  return b->dtype == FDTD_F32 ? batch_run<float>(b, nsteps) : batch_run<double>(b, nsteps);
}

int fdtd_batch_synchronize(fdtd_batch* b) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  if (!b) return fail(FDTD_ERR_INVALID, "null batch handle");
  CK(cudaSetDevice(b->device));
  CK(cudaStreamSynchronize(b->stream));
  CK(cudaGetLastError());
  return take_bounds_violation();
}

int fdtd_bounds_check_enabled(void) { return check_enabled() ? 1 : 0; }

int fdtd_near_field_power(fdtd_sim* s, const void* inc_phasors, int size_z_material, const double* weights,
                          double* out) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!inc_phasors || !weights || !out) return fail(FDTD_ERR_INVALID, "null argument");
  const int szm = size_z_material;
  if (szm < 1 || szm > s->nz_ph - 2)
    return fail(FDTD_ERR_INVALID, "size_z_material %d outside [1, nz_phasor - 2 = %d]", szm, s->nz_ph - 2);
  const int kBlocks = 296;
  const size_t plane = (size_t)s->ny_ph * s->nx_ph;
  const size_t nw = (size_t)s->ny_ph + s->nx_ph + (size_t)(s->nz_ph - 1);
  if (!s->nf_inc && (rc = alloc(s, 4 * plane * 2 * s->esz, &s->nf_inc))) return rc;
  if (!s->nf_w && (rc = alloc(s, sizeof(double) * (size_t)(s->ny_ph + s->nx_ph + s->nz_ph), (void**)&s->nf_w)))
    return rc;
  if (!s->nf_part && (rc = alloc(s, sizeof(double) * 11 * kBlocks, (void**)&s->nf_part))) return rc;
  CK(cudaMemcpyAsync(s->nf_inc, inc_phasors, 4 * plane * 2 * s->esz, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->nf_w, weights, sizeof(double) * nw, cudaMemcpyHostToDevice, s->stream));
  const int e = s->g.dtype == FDTD_F32
                    ? near_field_power_run<float>((const float*)s->ph, s->ph_off, (const float*)s->nf_inc, s->nx_ph,
                                                  s->ny_ph, s->nz_ph, szm, s->nf_w, s->nf_part, kBlocks, out,
                                                  s->stream)
                    : near_field_power_run<double>((const double*)s->ph, s->ph_off, (const double*)s->nf_inc,
                                                   s->nx_ph, s->ny_ph, s->nz_ph, szm, s->nf_w, s->nf_part, kBlocks,
                                                   out, s->stream);
  if (e) {
    cudaError_t ce = cudaGetLastError();
    return fail(FDTD_ERR_CUDA, "near-field power: %s", cudaGetErrorString(ce));
  }
  return take_bounds_violation();
}

int fdtd_batch_get_stream(fdtd_batch* b, void** stream) {
  if (!b || !stream) return fail(FDTD_ERR_INVALID, "null argument");
  *stream = (void*)b->stream;
  return FDTD_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// gradient of a far-field objective (adjoint sweep with checkpoints)
// ---------------------------------------------------------------------------
namespace {

long long state_elems(const fdtd_sim* s) { return 6 * s->vol + s->psi_elems; }

int save_state(fdtd_sim* s, void* slot) {
  const size_t fb = (size_t)s->vol * s->esz;
  unsigned char* d = static_cast<unsigned char*>(slot);
  for (int c = 0; c < 6; ++c)
    CK(cudaMemcpyAsync(d + c * fb, s->fld[s->cur][c], fb, cudaMemcpyDeviceToDevice, s->stream));
  CK(cudaMemcpyAsync(d + 6 * fb, s->psi_base[s->cur], (size_t)s->psi_elems * s->esz,
                     cudaMemcpyDeviceToDevice, s->stream));
  return FDTD_OK;
}

int restore_state(fdtd_sim* s, const void* slot) {
  const size_t fb = (size_t)s->vol * s->esz;
  const unsigned char* d = static_cast<const unsigned char*>(slot);
  for (int c = 0; c < 6; ++c)
    CK(cudaMemcpyAsync(s->fld[s->cur][c], d + c * fb, fb, cudaMemcpyDeviceToDevice, s->stream));
  CK(cudaMemcpyAsync(s->psi_base[s->cur], d + 6 * fb, (size_t)s->psi_elems * s->esz,
                     cudaMemcpyDeviceToDevice, s->stream));
  return FDTD_OK;
}

int set_step(fdtd_sim* s, int t) {
  CK(cudaStreamSynchronize(s->stream));
  const int h[4] = {t, 0, 0, 0};
  CK(cudaMemcpy(s->tdev, h, sizeof(int), cudaMemcpyHostToDevice));
  s->t = t;
  return FDTD_OK;
}

template <class T>
Psi<T> psi_view(const fdtd_sim* s, T* base) {
  Psi<T> p;
  for (int side = 0; side < 2; ++side)
    for (int c = 0; c < 4; ++c) {
      p.z[side][c] = base + s->poz[side][c];
      p.x[side][c] = base + s->pox[side][c];
      p.y[side][c] = base + s->poy[side][c];
    }
  return p;
}

template <class T>
int grad_backward(fdtd_sim* s, int nz_out, double* out_ca, double* out_cb) {
  const int nt = s->g.nt, every = s->grad_every;
  const long long vol = s->vol, se = state_elems(s);
  T* seg = static_cast<T*>(s->grad_seg);
  T* lam = static_cast<T*>(s->grad_lam);
  Adj<T> a;
  a.lex = lam; a.ley = lam + vol; a.lez = lam + 2 * vol;
  a.lhx = lam + 3 * vol; a.lhy = lam + 4 * vol; a.lhz = lam + 5 * vol;
  a.lps = psi_view<T>(s, static_cast<T*>(s->grad_lpsi));
  a.gca = s->grad_ca;
  a.gcb = s->grad_cb;
  a.g_re = s->grad_gre;
  a.g_im = s->grad_gim;
  a.nz_grad = nz_out;
  ShellBoxes whole;
  memset(&whole, 0, sizeof(whole));
  add_shell_box(whole, 0, s->g.nx, 0, s->g.ny, 0, s->g.nz);
  // Segments are recomputed on the side stream into two alternating slot
  // buffers while the main stream sweeps the previous segment backwards.
  // The recompute reads the step index as toff with a zero counter
  // (tdev[2]), so it needs no counter updates between segments.
  const size_t buf = (size_t)every * se;   // slots 1..every of one buffer
  const int* zero_t = s->tdev + 2;
  cudaEvent_t start = nullptr, rec_done[2] = {nullptr, nullptr}, adj_done[2] = {nullptr, nullptr};
  auto cleanup = [&]() {
    for (cudaEvent_t e : {start, rec_done[0], rec_done[1], adj_done[0], adj_done[1]})
      if (e) cudaEventDestroy(e);
  };
  for (cudaEvent_t* e : {&start, &rec_done[0], &rec_done[1], &adj_done[0], &adj_done[1]})
    if (cudaEventCreateWithFlags(e, cudaEventDisableTiming) != cudaSuccess) {
      cleanup();
      return fail(FDTD_ERR_CUDA, "event creation failed");
    }
  CK(cudaEventRecord(start, s->stream));
  CK(cudaStreamWaitEvent(s->side, start, 0));
  bool first = true;
  for (int idx = 0; idx < s->grad_ncp; ++idx) {
    const int c = s->grad_ncp - 1 - idx, bsel = idx & 1;
    const int z0 = c * every, n = std::min(every, nt - z0);
    T* cp = static_cast<T*>(s->grad_cp) + (size_t)c * se;
    T* base = seg + bsel * buf - se;   // slot j (j >= 1) at base + j * se
    // state j of the segment (step z0 + j): the checkpoint, then the slots
    auto slot = [&](int j) -> T* { return j == 0 ? cp : base + (size_t)j * se; };
    // recompute the segment, state j - 1 -> state j, fields only: the split
    // passes run source -> destination, so nothing is copied
    if (idx >= 2) CK(cudaStreamWaitEvent(s->side, adj_done[bsel], 0));
    for (int j = 1; j <= n; ++j) {
      T* src = slot(j - 1);
      T* dst = slot(j);
      State<T> st = make_state<T>(s, s->cur, s->cur);
      st.iex = src; st.iey = src + vol; st.iez = src + 2 * vol;
      st.ihx = src + 3 * vol; st.ihy = src + 4 * vol; st.ihz = src + 5 * vol;
      st.oex = dst; st.oey = dst + vol; st.oez = dst + 2 * vol;
      st.ohx = dst + 3 * vol; st.ohy = dst + 4 * vol; st.ohz = dst + 5 * vol;
      st.ps = psi_view<T>(s, src + 6 * vol);
      st.pd = psi_view<T>(s, dst + 6 * vol);
      launch_shell_pass<T>(st, zero_t, z0 + j - 1, whole, true, s->side);
      State<T> se2 = st;
      se2.ihx = dst + 3 * vol; se2.ihy = dst + 4 * vol; se2.ihz = dst + 5 * vol;
      launch_shell_pass<T>(se2, zero_t, z0 + j - 1, whole, false, s->side);
    }
    CK(cudaEventRecord(rec_done[bsel], s->side));
    CK(cudaStreamWaitEvent(s->stream, rec_done[bsel], 0));
    for (int j = n - 1; j >= 0; --j) {
      State<T> st = make_state<T>(s, s->cur, s->cur);
      T* sn = slot(j);
      T* sn1 = slot(j + 1);
      st.iex = sn; st.iey = sn + vol; st.iez = sn + 2 * vol;
      st.ihx = sn1 + 3 * vol; st.ihy = sn1 + 4 * vol; st.ihz = sn1 + 5 * vol;
      st.ps = psi_view<T>(s, sn1 + 6 * vol);
      if (first) launch_adjoint_first<T>(st, a, z0 + j, s->stream);
      launch_adjoint_step<T>(st, a, z0 + j, first, s->stream);
      first = false;
    }
    CK(cudaEventRecord(adj_done[bsel], s->stream));
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      cleanup();
      return fail(FDTD_ERR_CUDA, "adjoint sweep: %s", cudaGetErrorString(e));
    }
  }
  cudaError_t e = cudaStreamSynchronize(s->side);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s->stream);
  cleanup();
  if (e != cudaSuccess) return fail(FDTD_ERR_CUDA, "adjoint sweep: %s", cudaGetErrorString(e));
  int rc = set_step(s, nt);   // the fields still hold the forward solve's last state
  if (rc) return rc;
  // the first nz_out planes of the gradients, without the row padding
  const size_t row = (size_t)s->g.nx * sizeof(double);
  const size_t spitch = (size_t)s->pitch * sizeof(double);
  if (out_ca)
    CK(cudaMemcpy2DAsync(out_ca, row, s->grad_ca, spitch, row, (size_t)nz_out * s->g.ny,
                         cudaMemcpyDeviceToHost, s->stream));
  if (out_cb)
    CK(cudaMemcpy2DAsync(out_cb, row, s->grad_cb, spitch, row, (size_t)nz_out * s->g.ny,
                         cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_grad_forward(fdtd_sim* s, int checkpoint_every) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (checkpoint_every < 1) return fail(FDTD_ERR_INVALID, "checkpoint period must be >= 1");
  if (!s->have_abs) return fail(FDTD_ERR_STATE, "absorbers not set (fdtd_set_absorbers)");
  if (!s->have_mat) return fail(FDTD_ERR_STATE, "materials not set (fdtd_set_materials)");
  if (s->g.nt_inc > 0 && s->inc_nt < s->g.nt_inc)
    return fail(FDTD_ERR_STATE, "incident beam not set (fdtd_set_incident)");
  const int nt = s->g.nt;
  const int ncp = (nt + checkpoint_every - 1) / checkpoint_every;
  const size_t sb = (size_t)state_elems(s) * s->esz;
  if (s->grad_cp == nullptr || s->grad_ncp != ncp) {
    release(s, s->grad_cp);
    s->grad_cp = nullptr;
    if ((rc = alloc(s, sb * ncp, &s->grad_cp))) return rc;
  }
  s->grad_every = checkpoint_every;
  s->grad_ncp = ncp;
  s->grad_forward_done = false;
  if ((rc = fdtd_reset(s))) return rc;
  for (int c = 0; c < ncp; ++c) {
    if ((rc = save_state(s, static_cast<unsigned char*>(s->grad_cp) + c * sb))) return rc;
    const int n = std::min(checkpoint_every, nt - c * checkpoint_every);
    // the objective reads the upper plane's phasors only (plane group 1)
    rc = s->g.dtype == FDTD_F32 ? enqueue_steps<float>(s, n, 1, 1) : enqueue_steps<double>(s, n, 1, 1);
    if (rc) return rc;
    s->t += n;
  }
  CK(cudaStreamSynchronize(s->stream));
  s->grad_forward_done = true;
  return FDTD_OK;
}

int fdtd_grad_backward(fdtd_sim* s, const double* dj_dre, const double* dj_dim, int nz_out,
                       double* grad_ca, double* grad_cb) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!dj_dre || !dj_dim) return fail(FDTD_ERR_INVALID, "null phasor gradient");
  if (nz_out < 0 || nz_out > s->g.nz) return fail(FDTD_ERR_INVALID, "bad nz_out %d", nz_out);
  if (!s->grad_forward_done || s->t != s->g.nt)
    return fail(FDTD_ERR_STATE, "run fdtd_grad_forward first (and no steps after it)");
  const size_t sb = (size_t)state_elems(s) * s->esz;
  const int slots = 2 * s->grad_every;   // two buffers of states 1..every
  if (s->grad_seg == nullptr || s->grad_seg_slots != slots) {
    release(s, s->grad_seg);
    s->grad_seg = nullptr;
    if ((rc = alloc(s, sb * slots, &s->grad_seg))) return rc;
    s->grad_seg_slots = slots;
  }
  const size_t fb = (size_t)s->vol * s->esz;
  const size_t gb = (size_t)s->vol * sizeof(double);
  const size_t pb = (size_t)4 * s->ny_ph * s->nx_ph * sizeof(double);
  if (!s->grad_lam) {
    if ((rc = alloc(s, 6 * fb, &s->grad_lam))) return rc;
    if ((rc = alloc(s, (size_t)s->psi_elems * s->esz, &s->grad_lpsi))) return rc;
    if ((rc = alloc(s, gb, (void**)&s->grad_ca))) return rc;
    if ((rc = alloc(s, gb, (void**)&s->grad_cb))) return rc;
    if ((rc = alloc(s, pb, (void**)&s->grad_gre))) return rc;
    if ((rc = alloc(s, pb, (void**)&s->grad_gim))) return rc;
  }
  CK(cudaMemsetAsync(s->grad_lam, 0, 6 * fb, s->stream));
  CK(cudaMemsetAsync(s->grad_lpsi, 0, (size_t)s->psi_elems * s->esz, s->stream));
  CK(cudaMemsetAsync(s->grad_ca, 0, gb, s->stream));
  CK(cudaMemsetAsync(s->grad_cb, 0, gb, s->stream));
  CK(cudaMemcpyAsync(s->grad_gre, dj_dre, pb, cudaMemcpyHostToDevice, s->stream));
  CK(cudaMemcpyAsync(s->grad_gim, dj_dim, pb, cudaMemcpyHostToDevice, s->stream));
  rc = s->g.dtype == FDTD_F32 ? grad_backward<float>(s, nz_out, grad_ca, grad_cb)
                              : grad_backward<double>(s, nz_out, grad_ca, grad_cb);
  s->grad_forward_done = false;
  return rc;
}

}  // extern "C"

// ---------------------------------------------------------------------------
// incident beam: excitation and vacuum run (fdtd_incident_*)
// ---------------------------------------------------------------------------
// The run uses an ordinary simulation handle for its grid: Ca = 1, Cb the
// vacuum's, no TFSF injection (nt_inc = 0), the split passes in place.
struct fdtd_incident {
  fdtd_sim* sim = nullptr;
  int nt_pulse = 0;            // source steps (size_t_pulse, at most nt)
  int feed_in = 0, read_out = 0;
  void* exc[2] = {};           // excitation imaginary parts, (nt_pulse, ny, pitch)
  void* rec[4] = {};           // recorded ex, ey, hx, hy, (nt, ny, pitch)
  void* iph = nullptr;         // incident phasors, 4 x (ny_ph, nx_ph) complex
  bool have_exc = false, ran = false;
};

namespace {

int check_inc(fdtd_incident* b) {
  if (!b || !b->sim) return fail(FDTD_ERR_INVALID, "null incident handle");
  return check_sim(b->sim);
}

template <class T>
int incident_run(fdtd_incident* b) {
  fdtd_sim* s = b->sim;
  const fdtd_geometry& g = s->g;
  int rc = fdtd_reset(s);
  if (rc) return rc;
  const size_t phb = (size_t)8 * s->ny_ph * s->nx_ph * s->esz;
  CK(cudaMemsetAsync(b->iph, 0, phb, s->stream));
  ShellBoxes whole;
  memset(&whole, 0, sizeof(whole));
  add_shell_box(whole, 0, g.nx, 0, g.ny, 0, g.nz);
  const State<T> st = make_state<T>(s, 0, 0);   // split passes in place on set 0
  const int* zero_t = s->tdev + 2;
  IncidentRecord<T> r;
  r.rex = (T*)b->rec[0]; r.rey = (T*)b->rec[1]; r.rhx = (T*)b->rec[2]; r.rhy = (T*)b->rec[3];
  r.ph = (T*)b->iph;
  r.phase = s->phase;
  r.nx = g.nx; r.ny = g.ny; r.pitch = s->pitch; r.plane = s->plane;
  r.npml = g.npml; r.read_out = b->read_out; r.nx_ph = s->nx_ph; r.ny_ph = s->ny_ph;
  auto source = [&](int set, int t) {
    if (t < b->nt_pulse)
      launch_inc_source<T>((T*)s->fld[set][0], (T*)s->fld[set][1], (const T*)b->exc[0], (const T*)b->exc[1],
                           g.nx, g.ny, s->pitch, s->plane, b->feed_in, t, s->stream);
  };
  // E update and E CPML, hard source, H update and H CPML, read-out
  // (cpu/incident_sim.py:134-160)
  launch_shell_pass<T>(st, zero_t, 0, whole, false, s->stream);
  source(0, 0);
  if (s->kernel == FDTD_KERNEL_FUSED) {
    // the fused step of t gives H^{t+1/2} and the next step's E update; the
    // read-out takes E^t from the source set and H^{t+1/2} from the
    // destination set, and the next step's source goes onto the destination
    for (int t = 0; t < g.nt; ++t) {
      const int src = s->cur;
      if ((rc = enqueue_steps<T>(s, 1, 0, 0))) return rc;
      r.ex = (const T*)s->fld[src][0]; r.ey = (const T*)s->fld[src][1];
      r.hx = (const T*)s->fld[s->cur][3]; r.hy = (const T*)s->fld[s->cur][4];
      launch_inc_record<T>(r, t, s->stream);
      source(s->cur, t + 1);
    }
  } else {
    r.ex = st.iex; r.ey = st.iey; r.hx = st.ihx; r.hy = st.ihy;
    for (int t = 0; t < g.nt; ++t) {
      if (t > 0) {
        launch_shell_pass<T>(st, zero_t, t, whole, false, s->stream);
        source(0, t);
      }
      launch_shell_pass<T>(st, zero_t, t, whole, true, s->stream);
      launch_inc_record<T>(r, t, s->stream);
    }
  }
  CK(cudaGetLastError());
  CK(cudaStreamSynchronize(s->stream));
  s->t = g.nt;
  b->ran = true;
  return FDTD_OK;
}

}  // namespace

extern "C" {

int fdtd_incident_create(const fdtd_geometry* geom, int nt_pulse, int device, fdtd_incident** out) {
  if (!geom || !out) return fail(FDTD_ERR_INVALID, "null argument");
  *out = nullptr;
  if (nt_pulse < 0) return fail(FDTD_ERR_INVALID, "negative pulse length");
  if (geom->nt < 1) return fail(FDTD_ERR_INVALID, "incident run needs at least one step");
  fdtd_geometry g = *geom;
  g.nt_inc = 0;            // no TFSF injection in the incident grid
  g.tfsf_z = g.nz / 2;     // unused; any plane inside the grid
  fdtd_incident* b = new fdtd_incident();
  int rc = fdtd_create(&g, device, &b->sim);
  if (rc) {
    delete b;
    return rc;
  }
  fdtd_sim* s = b->sim;
  // no injection plane: the fused step's interior and slab boxes cover every
  // plane of the grid
  s->g.tfsf_z = -2;
  s->kernel = FDTD_KERNEL_FUSED;
  s->tile_x = 32;
  s->tile_y = 4;
  b->nt_pulse = std::min(nt_pulse, g.nt);   // the reference's loop ends at nt
  b->feed_in = g.nz / 2 + 4;                // cpu/incident_sim.py:101-103
  b->read_out = b->feed_in - 4;
  if (b->feed_in >= g.nz - 1) {
    fdtd_incident_destroy(b);
    return fail(FDTD_ERR_INVALID, "incident grid of %d planes too thin for its source plane", g.nz);
  }
  const size_t pb = (size_t)g.ny * s->pitch * s->esz;
  for (int c = 0; c < 2 && !rc; ++c) rc = alloc(s, pb * std::max(b->nt_pulse, 1), &b->exc[c]);
  for (int c = 0; c < 4 && !rc; ++c) rc = alloc(s, pb * g.nt, &b->rec[c]);
  if (!rc) rc = alloc(s, (size_t)8 * s->ny_ph * s->nx_ph * s->esz, &b->iph);
  if (!rc) {
    // vacuum: Ca = 1, Cb = dt / (eps0 dx) (cpu/incident_sim.py:112-116)
    if (g.dtype == FDTD_F32) {
      launch_fill<float>((float*)s->ca, s->vol, 1.0f, s->stream);
      launch_fill<float>((float*)s->cb, s->vol, (float)g.dte0dx, s->stream);
    } else {
      launch_fill<double>((double*)s->ca, s->vol, 1.0, s->stream);
      launch_fill<double>((double*)s->cb, s->vol, g.dte0dx, s->stream);
    }
    cudaError_t e = cudaStreamSynchronize(s->stream);
    if (e != cudaSuccess) rc = fail(FDTD_ERR_CUDA, "vacuum coefficients: %s", cudaGetErrorString(e));
    s->have_mat = true;
  }
  if (rc) {
    fdtd_incident_destroy(b);
    return rc;
  }
  *out = b;
  return FDTD_OK;
}

int fdtd_incident_destroy(fdtd_incident* b) {
  if (!b) return FDTD_OK;
  if (b->sim) fdtd_destroy(b->sim);
  delete b;
  return FDTD_OK;
}

int fdtd_fused_plan_boxes(int nx, int ny, int nz, int npml, int tfsf_z, int tile_y, int zchunk, int mode,
                          int* out, int cap, int* count) {
  if (!out || !count || cap < 0) return fail(FDTD_ERR_INVALID, "null argument");
  if (npml < 2 || npml > kMaxPml || nx < 2 * npml + 3 || ny < 2 * npml + 3 || nz < 2 * npml + 3)
    return fail(FDTD_ERR_INVALID, "grid %dx%dx%d too small for npml %d", nz, ny, nx, npml);
  if (mode < 0 || mode > 3) return fail(FDTD_ERR_INVALID, "unknown plan mode %d", mode);
  const FusedPlan p =
      make_fused_plan(nx, ny, nz, npml, tfsf_z, tile_y, zchunk, mode == 1 ? 1 : mode == 3 ? 2 : 0, mode == 2);
  if (p.shell.dropped || p.mshell.dropped)
    return fail(FDTD_ERR_INVALID, "plan needs more than %d shell boxes", kMaxShellBoxes);
  int n = 0;
  auto put = [&](int kind, int x0, int x1, int y0, int y1, int z0, int z1) {
    if (n < cap) {
      int* r = out + 7 * n;
      r[0] = kind; r[1] = x0; r[2] = x1; r[3] = y0; r[4] = y1; r[5] = z0; r[6] = z1;
    }
    ++n;
  };
  if (p.has_interior)
    for (int k = 0; k < p.interior.nz_ranges; ++k)
      put(0, p.interior.xa, p.interior.xb, p.interior.ya, p.interior.yb, p.interior.z0[k], p.interior.z1[k]);
  if (p.has_slab)
    for (int k = 0; k < p.slab.nz_ranges; ++k)
      put(1, p.slab.xa, p.slab.xb, p.slab.ya, p.slab.yb, p.slab.z0[k], p.slab.z1[k]);
  for (int k = 0; k < p.shell.n; ++k) {
    const ShellBox& b = p.shell.b[k];
    put(2, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1);
  }
  for (int k = 0; k < p.mshell.n; ++k) {
    const MarchBox& b = p.mshell.b[k];
    put(3, b.x0, b.x1, b.y0, b.y1, b.z0, b.z1);
  }
  *count = n;
  return n <= cap ? FDTD_OK : fail(FDTD_ERR_INVALID, "%d boxes, room for %d", n, cap);
}

int fdtd_incident_set_option(fdtd_incident* b, int option, int value) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if (option != FDTD_OPT_KERNEL && option != FDTD_OPT_TILE_Y && option != FDTD_OPT_ZCHUNK &&
      option != FDTD_OPT_FUSED_SLAB)
    return fail(FDTD_ERR_INVALID, "option %d does not apply to an incident run", option);
  return fdtd_set_option(b->sim, option, value);
}

int fdtd_incident_set_absorbers(fdtd_incident* b, const void* profiles) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  return fdtd_set_absorbers(b->sim, profiles);
}

int fdtd_incident_make_excitation(fdtd_incident* b, const double* k_vals, const double* pulse_fft,
                                  int nt_fft, double theta_deg, double phi_deg, int pol,
                                  double gauss_radius, double* peak) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if (!k_vals || !pulse_fft) return fail(FDTD_ERR_INVALID, "null pulse spectrum");
  if (nt_fft < 1 || nt_fft < b->nt_pulse)
    return fail(FDTD_ERR_INVALID, "pulse spectrum of %d bins shorter than the source (%d steps)", nt_fft,
                b->nt_pulse);
  if (nt_fft > 65535) return fail(FDTD_ERR_INVALID, "pulse spectrum of %d bins too long", nt_fft);
  if (!(gauss_radius > 0)) return fail(FDTD_ERR_INVALID, "taper radius must be positive");
  IncidentTaper p;
  switch (pol) {   // (Eh, Ev) of incidentbeam.py:405-419
    case FDTD_POL_HH: p.eh = make_double2(1, 0); p.ev = make_double2(0, 0); break;
    case FDTD_POL_VV: p.eh = make_double2(0, 0); p.ev = make_double2(1, 0); break;
    case FDTD_POL_RHCP: p.eh = make_double2(0, -1); p.ev = make_double2(1, 0); break;
    case FDTD_POL_LHCP: p.eh = make_double2(0, 1); p.ev = make_double2(1, 0); break;
    default: return fail(FDTD_ERR_INVALID, "Invalid polarization value %d", pol);
  }
  fdtd_sim* s = b->sim;
  const fdtd_geometry& g = s->g;
  p.nx = g.nx; p.ny = g.ny; p.nt = nt_fft;
  p.dfx = 1.0 / (g.nx * g.cell_size);   // numpy.fft.fftfreq spacing
  p.dfy = 1.0 / (g.ny * g.cell_size);
  const double th = theta_deg * (M_PI / 180.0), ph = phi_deg * (M_PI / 180.0);
  p.sin_theta = std::sin(th);
  p.cos_phi = std::cos(ph);
  p.sin_phi = std::sin(ph);
  p.r2 = gauss_radius * gauss_radius;
  p.r2_4pi = p.r2 / (4 * M_PI);
  rc = g.dtype == FDTD_F32
           ? make_incident_excitation<float>(p, k_vals, pulse_fft, b->nt_pulse, s->pitch, (float*)b->exc[0],
                                             (float*)b->exc[1], peak, s->stream)
           : make_incident_excitation<double>(p, k_vals, pulse_fft, b->nt_pulse, s->pitch, (double*)b->exc[0],
                                              (double*)b->exc[1], peak, s->stream);
  if (rc) return rc;
  b->have_exc = true;
  return FDTD_OK;
}

int fdtd_incident_set_excitation(fdtd_incident* b, const void* ex_imag, const void* ey_imag) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if ((!ex_imag || !ey_imag) && b->nt_pulse > 0) return fail(FDTD_ERR_INVALID, "null excitation");
  fdtd_sim* s = b->sim;
  const size_t w = (size_t)s->g.nx * s->esz;
  const void* src[2] = {ex_imag, ey_imag};
  for (int c = 0; c < 2 && b->nt_pulse > 0; ++c)
    CK(cudaMemcpy2DAsync(b->exc[c], (size_t)s->pitch * s->esz, src[c], w, w, (size_t)s->g.ny * b->nt_pulse,
                         cudaMemcpyHostToDevice, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  b->have_exc = true;
  return FDTD_OK;
}

int fdtd_incident_get_excitation(fdtd_incident* b, void* ex_imag, void* ey_imag) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if (!b->have_exc) return fail(FDTD_ERR_STATE, "no excitation (fdtd_incident_make_excitation)");
  fdtd_sim* s = b->sim;
  const size_t w = (size_t)s->g.nx * s->esz;
  void* dst[2] = {ex_imag, ey_imag};
  for (int c = 0; c < 2 && b->nt_pulse > 0; ++c)
    if (dst[c])
      CK(cudaMemcpy2DAsync(dst[c], w, b->exc[c], (size_t)s->pitch * s->esz, w, (size_t)s->g.ny * b->nt_pulse,
                           cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_incident_run(fdtd_incident* b) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if (!b->sim->have_abs) return fail(FDTD_ERR_STATE, "absorbers not set (fdtd_incident_set_absorbers)");
  if (!b->have_exc) return fail(FDTD_ERR_STATE, "no excitation (fdtd_incident_make_excitation)");
  return b->sim->g.dtype == FDTD_F32 ? incident_run<float>(b) : incident_run<double>(b);
}

int fdtd_incident_get_planes(fdtd_incident* b, void* ex, void* ey, void* hx, void* hy) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if (!b->ran) return fail(FDTD_ERR_STATE, "incident run not done (fdtd_incident_run)");
  fdtd_sim* s = b->sim;
  const size_t w = (size_t)s->g.nx * s->esz;
  void* dst[4] = {ex, ey, hx, hy};
  for (int c = 0; c < 4; ++c)
    if (dst[c])
      CK(cudaMemcpy2DAsync(dst[c], w, b->rec[c], (size_t)s->pitch * s->esz, w, (size_t)s->g.ny * s->g.nt,
                           cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_incident_get_phasors(fdtd_incident* b, void* ex_ph, void* ey_ph, void* hx_ph, void* hy_ph) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_inc(b);
  if (rc) return rc;
  if (!b->ran) return fail(FDTD_ERR_STATE, "incident run not done (fdtd_incident_run)");
  fdtd_sim* s = b->sim;
  const size_t n = (size_t)2 * s->ny_ph * s->nx_ph * s->esz;
  void* dst[4] = {ex_ph, ey_ph, hx_ph, hy_ph};
  for (int c = 0; c < 4; ++c)
    if (dst[c])
      CK(cudaMemcpyAsync(dst[c], (unsigned char*)b->iph + c * n, n, cudaMemcpyDeviceToHost, s->stream));
  CK(cudaStreamSynchronize(s->stream));
  return FDTD_OK;
}

int fdtd_set_incident_from(fdtd_sim* s, const fdtd_incident* b) {
  DeviceGuard device_guard;   // the caller's current device is restored on return
  int rc = check_sim(s);
  if (rc) return rc;
  if (!b || !b->sim) return fail(FDTD_ERR_INVALID, "null incident handle");
  const fdtd_geometry& g = s->g;
  const fdtd_geometry& gi = b->sim->g;
  if (!b->ran) return fail(FDTD_ERR_STATE, "incident run not done (fdtd_incident_run)");
  if (gi.nx != g.nx || gi.ny != g.ny || gi.dtype != g.dtype || b->sim->device != s->device)
    return fail(FDTD_ERR_INVALID, "incident run of %dx%d (dtype %d, device %d) does not fit %dx%d (dtype %d, "
                "device %d)", gi.ny, gi.nx, gi.dtype, b->sim->device, g.ny, g.nx, g.dtype, s->device);
  if (g.nt_inc > gi.nt)
    return fail(FDTD_ERR_INVALID, "incident run has %d steps, the simulation injects %d", gi.nt, g.nt_inc);
  const size_t bytes = (size_t)std::max(g.nt_inc, 1) * s->plane * s->esz;
  for (int c = 0; c < 4; ++c) {
    if (!s->inc[c] && (rc = alloc(s, bytes, &s->inc[c]))) return rc;
    if (g.nt_inc > 0)
      CK(cudaMemcpyAsync(s->inc[c], b->rec[c], (size_t)g.nt_inc * s->plane * s->esz, cudaMemcpyDeviceToDevice,
                         s->stream));
  }
  CK(cudaStreamSynchronize(s->stream));
  s->inc_nt = g.nt_inc;
  return FDTD_OK;
}

}  // extern "C"
