/*
 * fdtd_b200.h -- C-ABI of the B200-native FDTD time-stepping library
 * (libfdtd_b200.so).
 *
 * This is the drop-in boundary for the time-stepping hot path of
 * wyatt-sfu/sar-pixel-simulator (package `fdtdsarsim`). The reference drives
 * its GPU path from Python through PyCUDA (`fdtdsarsim/gpu/main_sim.py`);
 * each entry point below names the reference interface it replaces.
 *
 * Conventions
 *  - Every function returns an int status (FDTD_OK == 0). On failure the
 *    message is kept per thread and read with fdtd_last_error(). No C++
 *    exception and no device trap crosses this boundary.
 *  - Arrays are C-contiguous, z slowest, x fastest: fields and material
 *    arrays are (nz, ny, nx); incident planes are (nt_inc, ny, nx); phasor
 *    planes are complex (re, im interleaved) of the element type selected by
 *    `dtype` (FDTD_F32 -> float, FDTD_F64 -> double).
 *  - Host pointers are borrowed for the duration of the call only. Device
 *    memory is owned by the handle.
 *  - A handle is not re-entrant: one host thread at a time per handle.
 */
#ifndef FDTD_B200_H
#define FDTD_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define FDTD_OK            0
#define FDTD_ERR_INVALID   1  /* bad argument or size */
#define FDTD_ERR_CUDA      2  /* CUDA runtime error */
#define FDTD_ERR_STATE     3  /* call out of order (e.g. run before set_materials) */
#define FDTD_ERR_NONFINITE 4  /* a NaN/Inf was detected in the fields */
#define FDTD_ERR_NOMEM     5  /* device allocation failed */
#define FDTD_ERR_BOUNDS    6  /* bounds-checked build only: a kernel access left
                                 its allocation or array (it was skipped) */

/* element types */
#define FDTD_F32 0
#define FDTD_F64 1

/* step kernels (fdtd_set_option(FDTD_OPT_KERNEL, ...)) */
#define FDTD_KERNEL_SPLIT 0   /* H pass + E pass + phasor pass per step */
#define FDTD_KERNEL_FUSED 1   /* one z-marching pass per step + phasor pass */

/* phasor accumulation (fdtd_set_option(FDTD_OPT_PHASOR_MODE, ...)) */
#define FDTD_PHASOR_REFERENCE 0 /* float64 add of each term, rounded to the
                                   storage type every step (the reference's
                                   arithmetic, cpu/field_updates.py:385-400) */
#define FDTD_PHASOR_KAHAN     1 /* storage-type accumulator plus a Kahan
                                   compensation term */

/* options */
#define FDTD_OPT_KERNEL       1
#define FDTD_OPT_PHASOR_MODE  2
#define FDTD_OPT_TILE_X       3  /* fused kernel tile width in threads of
                                    4 x cells each; 32 (128 cells) */
#define FDTD_OPT_TILE_Y       4  /* fused kernel tile height in rows:
                                    4, 7, 8 (float, double), 15, 16 (float) */
#define FDTD_OPT_GRAPH_CHUNK  5  /* fdtd_run: steps per captured CUDA graph (0 = no
                                    graph); used while timing and the non-finite
                                    check are off */
#define FDTD_OPT_CHECK_EVERY  6  /* non-finite check period in steps (0 = off) */
#define FDTD_OPT_TIMING       7  /* 1: record CUDA events around every kernel */
#define FDTD_OPT_ZCHUNK       8  /* fused kernel z planes per block (0 = automatic) */
#define FDTD_OPT_FUSED_SLAB   9  /* 1: the fused step marches the CPML z slabs too;
                                    2: the column march, the interior's x-y box
                                    over every z plane (z faces and injection
                                    plane in the march), the split passes then
                                    sweep only the x and y strips (default 0:
                                    the split passes sweep the z slabs) */
#define FDTD_OPT_BATCH_STREAMS 10 /* fdtd_batch_set_option: 1 runs every member's
                                    own step path on its own stream, side by
                                    side; 0 (default) one launch per pass for
                                    all members */
#define FDTD_OPT_SHELL        11 /* how the fused step updates the shell around
                                    its interior box: FDTD_SHELL_* */
#define FDTD_OPT_BATCH_MODE   12 /* fdtd_batch_set_option: FDTD_BATCH_* */

/* batched sweep (fdtd_batch_set_option(FDTD_OPT_BATCH_MODE, ...)) */
#define FDTD_BATCH_SPLIT   0   /* (default) one launch per pass (H, E, phasors)
                                  for all members, in place */
#define FDTD_BATCH_STREAMS 1   /* every member's own step path on its own
                                  stream, side by side */
#define FDTD_BATCH_QUEUE   2   /* every member's fused step: one persistent
                                  launch walks a tile queue over all
                                  interior z-march tiles, one launch per
                                  split pass sweeps all shells, then one
                                  phasor launch */

/* shell of the fused step (fdtd_set_option(FDTD_OPT_SHELL, ...)) */
#define FDTD_SHELL_MARCH 0   /* fused z-marches with the CPML faces, edges and
                                injection in the march, beside the interior
                                march (fewer bytes, lower occupancy) */
#define FDTD_SHELL_SPLIT 1   /* (default) the split H pass beside the
                                interior march, then the split E pass */

/* kernel kinds of fdtd_get_kernel_time */
#define FDTD_TIME_STEP    0   /* the field-update kernel(s) of a step */
#define FDTD_TIME_PHASOR  1   /* the phasor kernel of a step */

/* Geometry and update constants of one simulation.
 * Mirrors fdtdsarsim GeomParams (parameters.py:58-94) plus the scalars the
 * reference's main loop derives from it (cpu/main_sim.py:116-130). The
 * host computes db/dtm0/dte0dx and rounds them to `dtype` exactly as the
 * reference does (np_type(dt / (mu0 * dx)) ...). */
typedef struct fdtd_geometry {
    int32_t nx, ny, nz;      /* size_x, size_y, size_z */
    int32_t npml;            /* size_pml */
    int32_t tfsf_z;          /* injection plane */
    int32_t nt;              /* size_t: total time steps */
    int32_t nt_inc;          /* size_t_inc: steps with incident injection */
    int32_t dtype;           /* FDTD_F32 / FDTD_F64 */
    double cell_size;        /* dx [m] */
    double timestep;         /* dt [s] */
    double frequency;        /* phasor frequency [Hz] */
    double db;               /* dt / (mu0 dx), rounded to dtype */
    double dtm0;             /* dt / mu0, rounded to dtype */
    double dte0dx;           /* dt / (eps0 dx), rounded to dtype */
} fdtd_geometry;

typedef struct fdtd_sim fdtd_sim;

/* Copies the last error message of the calling thread into buf
 * (NUL-terminated, truncated to len). Returns the message length. */
int fdtd_last_error(char *buf, int len);

/* Library version (major*10000 + minor*100 + patch). */
int fdtd_version(void);

/* Number of visible CUDA devices (0 when none). */
int fdtd_device_count(int *count);

/* The device's name (as cudaGetDeviceProperties gives it), NUL-terminated
 * into name[len]; the autotuner's cache key. No reference counterpart. */
int fdtd_device_name(int device, char *name, int len);

/* Creates a simulation on `device`, allocates all device state and zeroes it.
 * Replaces MainSimGpu.__init__ (gpu/main_sim.py:45-72): context creation,
 * _allocate_cuda_arrays (:512-640) and _clear_cuda_arrays (:691-787). */
int fdtd_create(const fdtd_geometry *geom, int device, fdtd_sim **out);

/* Frees every device resource of the handle. Refused (FDTD_ERR_STATE, the
 * handle stays valid) while the simulation is a member of a batch. */
int fdtd_destroy(fdtd_sim *sim);

/* Sets a tuning or behaviour option (FDTD_OPT_*). */
int fdtd_set_option(fdtd_sim *sim, int option, int value);
int fdtd_get_option(fdtd_sim *sim, int option, int *value);

/* Uploads the eight 1-D CPML coefficient profiles, each `npml` values of the
 * element type, packed in this order: be_d, bh_d, ce_d, ch_d (down / left /
 * front faces), be_u, bh_u, ce_u, ch_u (up / right / back faces).
 * Replaces _init_absorber_arrays (gpu/main_sim.py:789-825), which uploads
 * the same profiles tiled into 24 full 3-D arrays (absorbers.py:121-185). */
int fdtd_set_absorbers(fdtd_sim *sim, const void *profiles);

/* Uploads the update coefficient arrays Ca, Cb (nz, ny, nx) from host memory:
 * one contiguous transfer each into a packed device buffer (allocated on the
 * first call and kept: one more volume of device memory), re-pitched on the
 * device. Replaces the Ca/Cb transfer at the top of MainSimGpu._sim_loop
 * (gpu/main_sim.py:200-202). */
int fdtd_set_materials(fdtd_sim *sim, const void *ca, const void *cb);

/* Computes Ca, Cb on the device from relative permittivity and
 * conductivity of the material block (nz_mat, ny, nx), with vacuum stacked
 * above it up to nz, with the arithmetic of compute_material_arrays
 * (materials/materials.py:23-68). */
int fdtd_set_materials_eps_sigma(fdtd_sim *sim, const void *eps_r,
                                 const void *sigma, int nz_mat);

/* Uploads the whole incident beam: four (nt_inc, ny, nx) arrays, kept
 * resident in device memory. Replaces the per-step HDF5 reads and
 * memcpy_htod of ex/ey/hx/hy_inc slices (gpu/main_sim.py:256-264,305-313). */
int fdtd_set_incident(fdtd_sim *sim, const void *ex, const void *ey,
                      const void *hx, const void *hy, int nt_inc);

/* Zeroes fields, CPML auxiliaries and phasors and rewinds the step counter.
 * Replaces _clear_cuda_arrays (gpu/main_sim.py:691-787). */
int fdtd_reset(fdtd_sim *sim);

/* Enqueues `nsteps` time steps on the handle's stream (asynchronous).
 * One step is H update, H CPML, E-field injection, E update, E CPML,
 * H-field injection and the six phasor planes, in the reference's order
 * (gpu/main_sim.py:216-355, cpu/main_sim.py:140-195). */
int fdtd_run(fdtd_sim *sim, int nsteps);

/* Runs `nsteps` time steps while streaming the incident planes of those
 * steps from host memory (four (nt_inc, ny, nx) arrays) on a copy stream,
 * 16 steps' planes per transfer (2 in the first, so that the stepping
 * starts early), overlapped with the time stepping: each
 * group of steps waits only for its own planes. Page-locked arrays are
 * copied directly; pageable ones through two pinned staging buffers.
 * Synchronous. This is the reference's per-step incident transfer
 * (gpu/main_sim.py:256-264,305-313) made asynchronous. */
int fdtd_run_streamed(fdtd_sim *sim, int nsteps, const void *ex,
                      const void *ey, const void *hx, const void *hy);

/* Blocks until all enqueued work of the handle is done; reports deferred
 * CUDA errors and, with FDTD_OPT_CHECK_EVERY = k > 0, FDTD_ERR_NONFINITE
 * when a scan of the six fields after every k-th step found a NaN or an
 * infinity (the message names the first such step; fdtd_reset clears it).
 * The reference has no such check: a diverging run writes NaN phasors. */
int fdtd_synchronize(fdtd_sim *sim);

/* Number of completed (enqueued) steps since the last reset. */
int fdtd_step_index(fdtd_sim *sim, int64_t *t);

/* CUDA stream the handle launches on (cudaStream_t as void*), and a way to
 * make it launch on a caller's stream instead (NULL restores its own). */
int fdtd_get_stream(fdtd_sim *sim, void **stream);
int fdtd_set_stream(fdtd_sim *sim, void *stream);

/* Device time spent in one kernel kind (FDTD_TIME_*) over the steps run
 * since the last clear while FDTD_OPT_TIMING was on, from CUDA events on the
 * handle's stream. Synchronizes. The reference has no counterpart (it only
 * logs wall-clock per model, gpu/main_sim.py:93,112-115). */
int fdtd_get_kernel_time(fdtd_sim *sim, int kind, double *total_ms, int *launches);
int fdtd_clear_kernel_time(fdtd_sim *sim);

/* Copies one of the 24 phasor planes to host memory. `plane` indexes the
 * reference's result order (gpu/main_sim.py:409-418): ex_ph_d, ey_ph_d,
 * hx_ph_d, hy_ph_d, ex_ph_u, ey_ph_u, hx_ph_u, hy_ph_u, ey_ph_l, ez_ph_l,
 * hy_ph_l, hz_ph_l, ey_ph_r, ez_ph_r, hy_ph_r, hz_ph_r, ex_ph_f, ez_ph_f,
 * hx_ph_f, hz_ph_f, ex_ph_b, ez_ph_b, hx_ph_b, hz_ph_b. Shapes: d/u planes
 * (ny-2npml, nx-2npml); l/r (nz-2npml, ny-2npml); f/b (nz-2npml, nx-2npml).
 * Replaces the phasor memcpy_dtoh block (gpu/main_sim.py:357-385). */
int fdtd_get_phasor(fdtd_sim *sim, int plane, void *out);
/* All 24 planes in one call: packed one after the other in that order into
 * `out` (complex of the element type); one synchronisation, and direct
 * transfers when `out` is page-locked. */
int fdtd_get_phasors(fdtd_sim *sim, void *out);

/* Copies a field component (0..5 = ex, ey, ez, hx, hy, hz) of the current
 * state to / from host memory, shape (nz, ny, nx). The reference exposes
 * these as MainSimCpu.ex ... hz after run (cpu/fdtd_sim.py:150-156). */
int fdtd_get_field(fdtd_sim *sim, int comp, void *out);
int fdtd_set_field(fdtd_sim *sim, int comp, const void *in);

/* Near-to-far transform of the top phasor plane on the device.
 * Inputs: the four u-plane phasors (ny_ph, nx_ph) as complex of
 * `in_dtype` (FDTD_F32: complex64, FDTD_F64: complex128); nz is the
 * phasor-plane count in z (sets the plane height). Output: four
 * (nphi, ntheta) complex128 arrays E_theta, E_phi, H_theta, H_phi packed in
 * that order into `out` (2*4*nphi*ntheta doubles).
 * Replaces FarFieldTransform.__call__ (near2far.py:28-112). */
int fdtd_near2far(const void *ex_u, const void *ey_u, const void *hx_u,
                  const void *hy_u, int in_dtype, int nx_ph, int ny_ph,
                  int nz_ph, double dx, double r, const double *thetas_deg,
                  int ntheta, const double *phis_deg, int nphi, double freq,
                  int device, double *out);

/* ---- gradient ---------------------------------------------------------------
 * Reverse-mode derivative of an objective J of the four upper-plane phasors
 * (ex_ph_u, ey_ph_u, hx_ph_u, hy_ph_u) with respect to Ca and Cb of every
 * cell. No counterpart in the reference, which has no gradient.
 * fdtd_grad_forward resets the simulation and runs all size_t steps,
 * keeping the fields and CPML auxiliaries every `checkpoint_every` steps;
 * the caller then reads the phasors, evaluates J and its derivative with
 * respect to the real and imaginary part of each phasor cell, and passes
 * them to fdtd_grad_backward (4 planes each, (ny_ph, nx_ph) float64, in
 * the order above). The backward sweep recomputes each segment of steps
 * from its checkpoint and runs the transposed step backwards through it.
 * Outputs: dJ/dCa and dJ/dCb of the first nz_out planes, (nz_out, ny, nx)
 * float64. The simulation keeps the forward solve's fields and its four
 * upper-plane phasors (the forward accumulates no other phasor plane).
 * Device memory: (size_t / checkpoint_every + 2 checkpoint_every) states of
 * 6 fields and the CPML auxiliaries, plus the adjoint state. */
int fdtd_grad_forward(fdtd_sim *s, int checkpoint_every);
int fdtd_grad_backward(fdtd_sim *s, const double *dj_dre, const double *dj_dim, int nz_out,
                       double *grad_ca, double *grad_cb);

/* ---- batched sweep --------------------------------------------------------
 * Several simulations (uneven grids, one device, one element type) advanced
 * together: every time step runs the H pass, the E pass and the phasor pass
 * of all members in one launch each, and chunks of steps are replayed from
 * a captured CUDA graph. It replaces the loop over material models in
 * run_experiment (experiment.py:61-84), where each model is a separate
 * MainSimGpu.run (gpu/main_sim.py:74-115) and a separate time loop.
 * The members stay ordinary handles: set their absorbers, materials and
 * incident planes, run the batch, then read each member's phasors and
 * fields as usual. Members must outlive the batch (fdtd_destroy refuses a
 * member until its batches are destroyed); a member's own calls are
 * ordered after the batch's work. Each member advances nsteps from its own
 * step index, using its current field set in place (the split step). */
typedef struct fdtd_batch fdtd_batch;

int fdtd_batch_create(fdtd_sim *const *sims, int n, fdtd_batch **out);
int fdtd_batch_destroy(fdtd_batch *b);
/* FDTD_OPT_GRAPH_CHUNK: steps per captured graph (0: no graph; default 64).
 * FDTD_OPT_BATCH_STREAMS = 1: each member advances by its own step path
 * (its FDTD_OPT_KERNEL, its own graph chunks) on its own stream, forked from
 * and joined to the batch stream; results are those of fdtd_run on each
 * member. The all-or-nothing checks of fdtd_batch_run apply in both modes. */
int fdtd_batch_set_option(fdtd_batch *b, int option, int value);
int fdtd_batch_run(fdtd_batch *b, int nsteps);
int fdtd_batch_synchronize(fdtd_batch *b);
int fdtd_batch_get_stream(fdtd_batch *b, void **stream);

/* A material block made on the device instead of uploaded (replaces the
 * host fill of the reference's generators: materials/materials.py:112-164
 * rough_dielectric, materials/soilmodels.py:16-195 one- and two-layer
 * soils, materials/bubbles.py:21-199 bubbles). fdtd_fill_layers stages the
 * block's eps_r and sigma, (nz_mat, ny, nx), from `nlayers` interface height
 * maps in cells ((ny, nx) doubles each, lowest first, host): a cell takes
 * eps_r[k], sigma[k] of the first interface k with z <= height_k(y, x),
 * else eps_r[nlayers], sigma[nlayers] (the medium above: vacuum is 1, 0);
 * values rounded to the element type. fdtd_paint_spheres paints n spheres
 * (zc, yc, xc, rc, ri as doubles each: centre and radius in cells, integer
 * half-width ri <= 64) into the staged block: every cell
 * (rint(zc + dz), rint(yc + dy), rint(xc + dx)), |dz|, |dy|, |dx| <= ri,
 * dz^2 + dy^2 + dx^2 < rc^2, takes eps_r, sigma. fdtd_set_materials_staged
 * makes Ca/Cb from the staged block, as fdtd_set_materials_eps_sigma does
 * from an uploaded one; fdtd_get_staged_materials copies the block back
 * (nz_mat must be the staged block's height).
 * A later fdtd_set_materials discards the staged block. Synchronous. */
int fdtd_fill_layers(fdtd_sim *sim, int nz_mat, int nlayers, const double *heights, const double *eps_r,
                     const double *sigma);
int fdtd_paint_spheres(fdtd_sim *sim, int n, const double *spheres, double eps_r, double sigma);
int fdtd_set_materials_staged(fdtd_sim *sim);
int fdtd_get_staged_materials(fdtd_sim *sim, int nz_mat, void *eps_r, void *sigma);

/* Poynting power through the simulation's internal phasor planes, in
 * float64, from its current phasors on the device. Replaces the near-field
 * half of process_results (processresults.py:128-257), which evaluates it
 * on the host from the result file. inc_phasors: the incident beam's
 * ex, ey, hx, hy phasors, four consecutive (ny_ph, nx_ph) complex planes of
 * the simulation's element type (host). weights: the Simpson weights that
 * scipy.integrate.simpson applies along each axis, ny_ph values (rows of z
 * planes, columns of x planes), nx_ph values (columns of z and y planes),
 * then size_z_material values (side-plane rows below the material top) and
 * nz_ph - 1 - size_z_material values (the rows above, the last phasor row
 * excluded as the reference excludes it). out: 11 powers: incident, left
 * bottom, left top, right bottom, right top, front bottom, front top, back
 * bottom, back top, down, up. The flux of each cell, Re(E x conj(H)) . n / 2,
 * is formed in float64 (the reference forms it in complex64 and integrates
 * in float64), so the powers agree to rounding. Synchronous. */
int fdtd_near_field_power(fdtd_sim *sim, const void *inc_phasors, int size_z_material,
                          const double *weights, double *out);

/* Diagnostic (no counterpart in the reference): 1 in the bounds-checked
 * build of this library (libfdtd_b200_check.so: every global access of the
 * step kernels is checked against the library's live allocations and every
 * shared index against its array; a failed check skips the access and
 * fdtd_synchronize / fdtd_batch_synchronize return FDTD_ERR_BOUNDS), 0 in
 * the normal build. */
int fdtd_bounds_check_enabled(void);

/* Diagnostic (no counterpart in the reference): the CPML terms divide by
 * the cell size with a correctly rounded reciprocal and one FMA correction
 * (Markstein's method) instead of an IEEE division. This runs both on the
 * device for every float bit pattern (FDTD_F32: 2^32 inputs) or for 2^30
 * sampled doubles (FDTD_F64) with divisor `cell_size` rounded to the type,
 * and returns how many inputs gave a result that differs in any bit. */
int fdtd_check_cell_division(int dtype, double cell_size, int device, int64_t *tested,
                             int64_t *mismatches);

/* Diagnostic (no counterpart in the reference): the boxes of the fused
 * step's decomposition of a grid, host computation only (no device use).
 * mode 0: the shell by the split passes (FDTD_SHELL_SPLIT, the default
 * step), 1: the same with the CPML z slabs marched (FDTD_OPT_FUSED_SLAB),
 * 2: the shell marched (FDTD_SHELL_MARCH), 3: the column march
 * (FDTD_OPT_FUSED_SLAB = 2). Rows of 7 ints (kind, x0, x1, y0,
 * y1, z0, z1), kind 0 the interior z-march, 1 the CPML z slabs (mode 3:
 * the column), 2 a shell
 * box swept by the split passes, 3 a shell box of the general march; every
 * cell lies in exactly one box. */
int fdtd_fused_plan_boxes(int nx, int ny, int nz, int npml, int tfsf_z, int tile_y, int zchunk,
                          int mode, int *out, int cap, int *count);

/* fdtd_near2far without any device allocation. This entry point has no
 * counterpart in the reference; it exists for callers that cannot call
 * cudaMalloc when they need a far field: code whose device memory is owned
 * by a pool or arena that must not be bypassed, jobs that must not grow
 * their footprint while running, and contexts where a device allocation is
 * not allowed or would synchronize the device. Arguments, results and
 * errors are those of fdtd_near2far. Instead of allocating, every call
 * stages its inputs, angles and results in one static device array of
 * about 39 MB that every GPU loading this library holds until the process
 * exits. Limits: nx_ph * ny_ph <= 600000 cells for complex128 inputs
 * (1200000 for complex64), ntheta <= 4096, nphi <= 64 and
 * ntheta * nphi <= 8192; larger requests return FDTD_ERR_INVALID with a
 * message naming the limit. The first call on a device looks up the
 * array's device address with that device current and keeps it for the
 * process: after a cudaDeviceReset (or anything else that destroys the
 * device's primary context) the library must be loaded again before this
 * entry point is used. Every call is synchronous: it copies through
 * cudaMemcpy and launches on the legacy default stream, so it waits for the
 * caller's blocking streams, and it cannot be called while a stream is
 * being captured. All calls share the array: calls from one process are
 * serialized by a lock, and work that overlaps a call on the same device
 * through other means races with it. Nothing in the array has to start at
 * zero: each call writes every byte it reads back. The calling thread's
 * current device is the same after the call as before. */
int fdtd_near2far_noalloc(const void *ex_u, const void *ey_u,
                          const void *hx_u, const void *hy_u, int in_dtype,
                          int nx_ph, int ny_ph, int nz_ph, double dx, double r,
                          const double *thetas_deg, int ntheta,
                          const double *phis_deg, int nphi, double freq,
                          int device, double *out);

/* ---- incident beam ----------------------------------------------------------
 * The beam generation of IncidentBeam.setup (incidentbeam.py:41-71): the
 * excitation of create_inc_excitation (incidentbeam.py:206-298, taper_k
 * :301-433) and the vacuum FDTD run of IncidentSimCpu (cpu/incident_sim.py:
 * 22-171), which records ex, ey, hx, hy of its read-out plane at every step
 * (the datasets of the incident file) and the four incident phasors.
 * Geometry: nx, ny, npml, dtype, cell_size, timestep, frequency, db and dtm0
 * as for the main simulation; nz the incident grid's height,
 * int(3 wavelengths / cell_size) (cpu/incident_sim.py:33-37); nt the steps
 * run and recorded (size_t_inc); dte0dx the vacuum's Cb,
 * timestep / (eps0 cell_size) with scipy's eps0 (cpu/incident_sim.py:
 * 104-116); tfsf_z and nt_inc are not used. The hard source overwrites ex,
 * ey on plane nz / 2 + 4 while t < nt_pulse (size_t_pulse) and the read-out
 * plane is nz / 2 (cpu/incident_sim.py:101-103,141-144). */
typedef struct fdtd_incident fdtd_incident;

#define FDTD_POL_HH   0
#define FDTD_POL_VV   1
#define FDTD_POL_RHCP 2
#define FDTD_POL_LHCP 3

int fdtd_incident_create(const fdtd_geometry *geom, int nt_pulse, int device,
                         fdtd_incident **out);
int fdtd_incident_destroy(fdtd_incident *inc);
/* FDTD_OPT_KERNEL (default FDTD_KERNEL_FUSED: the fused step, its source
 * plane written after each step), FDTD_OPT_TILE_Y, FDTD_OPT_ZCHUNK,
 * FDTD_OPT_FUSED_SLAB. */
int fdtd_incident_set_option(fdtd_incident *inc, int option, int value);
/* 8 * npml profiles, packed as for fdtd_set_absorbers (Absorbers(params)
 * of the incident simulation, cpu/fdtd_sim.py:14-23). */
int fdtd_incident_set_absorbers(fdtd_incident *inc, const void *profiles);
/* Computes the excitation on the device (create_inc_excitation): for each of
 * the nt_fft pulse bins, its wavenumber k_vals[i] (2 pi pulse_freqs[i] / c)
 * and its pulse spectrum value pulse_fft[2i], pulse_fft[2i+1] (re, im; the
 * FFT of create_pulse, incidentbeam.py:174-199); incidence angles in
 * degrees, polarisation FDTD_POL_*, taper radius in metres
 * (incidentbeam.py:231-233). The excitation's imaginary parts of the first
 * nt_pulse samples are kept for fdtd_incident_run; `peak` (may be NULL)
 * gets the peak magnitude before the normalisation to 10. */
int fdtd_incident_make_excitation(fdtd_incident *inc, const double *k_vals,
                                  const double *pulse_fft, int nt_fft,
                                  double theta_deg, double phi_deg, int pol,
                                  double gauss_radius, double *peak);
/* The excitation's imaginary parts (np.imag(pulse_ex)[:nt_pulse], and ey),
 * (nt_pulse, ny, nx) of the element type, from / to host memory. */
int fdtd_incident_set_excitation(fdtd_incident *inc, const void *ex_imag,
                                 const void *ey_imag);
int fdtd_incident_get_excitation(fdtd_incident *inc, void *ex_imag, void *ey_imag);
/* Runs all nt steps from zero fields (IncidentSimCpu._sim_loop). */
int fdtd_incident_run(fdtd_incident *inc);
/* The recorded planes, (nt, ny, nx) each (the datasets ex, ey, hx, hy of
 * the incident file), and the incident phasors, complex (ny - 2 npml,
 * nx - 2 npml) each (phasors/{ex,ey,hx,hy}_inc_phasor). */
int fdtd_incident_get_planes(fdtd_incident *inc, void *ex, void *ey, void *hx, void *hy);
int fdtd_incident_get_phasors(fdtd_incident *inc, void *ex_ph, void *ey_ph,
                              void *hx_ph, void *hy_ph);
/* Device-to-device: the first nt_inc recorded planes of an incident run as
 * the incident beam of a main simulation with the same nx, ny, element type
 * and device (replaces writing the incident file and reading it back,
 * cpu/incident_sim.py:140-160 and gpu/main_sim.py:256-264). */
int fdtd_set_incident_from(fdtd_sim *sim, const fdtd_incident *inc);

#ifdef __cplusplus
}
#endif

#endif /* FDTD_B200_H */
