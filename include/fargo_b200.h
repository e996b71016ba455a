/*
 * fargo_b200.h -- C-ABI of the B200 FARGO3D hydro step (libfargo_b200.so).
 *
 * The library advances protoplanetary disks with FARGO3D's hydro time step
 * (main.c:361-448 of the reference): CFL time step, sources (SubStep1/2,
 * viscosity, potential), FARGO transport (van Leer in r / theta, residual van
 * Leer + PPA + integer shift in phi), Stockholm damping and ghost boundaries.
 * Fields live in device memory in the reference's layout (x fastest, then y,
 * then z; NGHY = NGHZ = 3 ghost rows/layers, periodic x without ghosts).
 *
 * Every entry point returns FB_OK (0) or a negative FB_ERR_* code from
 * fb_abi.h; fb_last_error() describes the last failure of the calling thread.
 * The product path has no CPU fallback: without a usable CUDA device every
 * call fails with FB_ERR_CUDA.
 *
 * Reference interfaces replaced (paths inside the reference's src/):
 *   fb_disk_step        one pass of the DT loop body, main.c:366-431, i.e.
 *                       ComputeVmed + cfl + CflFluidsMin + Sources (algogas.c:30)
 *                       + Collisions + Transport (algogas.c:135) +
 *                       StockholmBoundary + FillGhosts, the functions bound by
 *                       ChangeArch (change_arch.c:163-567) to their _gpu flavours
 *   fb_disk_initialize  FillGhosts + init_stockholm (main.c:311-316)
 *   fb_disk_set_state /
 *   fb_disk_get_state   Input_GPU / Output_GPU host<->device transfers of the
 *                       primitive Fields (fresh.c:187-276)
 */
#ifndef FARGO_B200_H
#define FARGO_B200_H

#include <stddef.h>
#include "fb_abi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Run-time parameters of one disk.  Field names follow the reference's .par
 * keys (std/stdpar.par); the layout is stable (append-only). */
typedef struct {
  int nx, ny, nz;              /* Nx, Ny, Nz; nz <= 1 selects a 2D (X,Y) mesh   */
  int spherical;               /* 0: CYLINDRICAL (2D), 1: SPHERICAL (3D)        */
  int log_spacing;             /* Spacing Log                                   */
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double aspectratio, sigmaslope, flaringindex;
  double nu;                   /* Nu (VISCOSITY)                                */
  double alpha; int alpha_visc;/* Alpha (ALPHAVISCOSITY when alpha_visc != 0)   */
  double cfl;                  /* CFL                                           */
  double omegaframe; int frame;/* OmegaFrame, Frame (FB_FRAME_*)                */
  int indirect_term;           /* IndirectTerm                                  */
  double thickness_smoothing, roche_smoothing, mass_taper;
  double damping_zone, tau_damp, killing_bc_colatitude;
  int nplanets;
  double pl_dist[FB_MAXPLANETS], pl_mass[FB_MAXPLANETS];
  int pl_feeldisk[FB_MAXPLANETS], pl_feelothers[FB_MAXPLANETS];
  double eccentricity, inclination;
  int nfluids;                 /* 1: gas; >1: gas + dust with implicit drag      */
  double invstokes[FB_MAXFLUIDS];   /* drag (STOKESNUMBER): [f-1] = 1/St of dust fluid f */
  int stockholm;               /* STOCKHOLM damping                             */
  int adiabatic;               /* ADIABATIC equation of state: the Energy field is
                                  the internal energy e, P = (GAMMA - 1) e; else
                                  ISOTHERMAL (Energy = sound speed).  FP64, 2D
                                  cylindrical, one fluid, one-disk path only     */
  double gamma;                /* GAMMA                                         */
  int dust_diffusion;          /* DUSTDIFFUSION: the dust densities diffuse down
                                  their concentration gradients with the gas's
                                  diffusivity (dust_diffusion_main.c).  FP64, 2D,
                                  nfluids > 1, one-disk path only               */
  int slab_y0;                 /* radial slab of a larger disk (split.c:76-213):  */
  int slab_ny_global;          /* rows [slab_y0, slab_y0 + ny) of a mesh of
                                  slab_ny_global rows spanning [ymin, ymax]; the
                                  boundary templates apply on the mesh's own
                                  edges only.  0: the disk is whole.  One fluid,
                                  FP64, planets that do not feel the disk        */
} fb_params;

typedef struct fb_disk fb_disk;

/* Create a disk on CUDA device `device` with FB_FP64 or FB_FP32 fields. */
int fb_disk_create(const fb_params *p, int precision, int device, fb_disk **out);
int fb_disk_destroy(fb_disk *d);

/* Host <-> device copies of one fluid's state, full stored arrays with ghosts
 * ((Nz+6 or 1) x (Ny+6) x Nx doubles).  Null pointers are skipped; cs only on
 * set (isothermal sound speed, FARGO3D's Energy field). */
int fb_disk_set_state(fb_disk *d, int fluid, const double *rho, const double *vx, const double *vy,
                      const double *vz, const double *cs);
int fb_disk_get_state(fb_disk *d, int fluid, double *rho, double *vx, double *vy, double *vz);
/* The fluid's Energy field (the cs array fb_disk_set_state takes): the
 * internal energy of an adiabatic disk, the sound speed of an isothermal one. */
int fb_disk_get_energy(fb_disk *d, int fluid, double *energy);

int fb_disk_initialize(fb_disk *d);

/* One hydro step: dt = min(CFL dt, what is left of a DT interval of length
 * dt_interval), exactly as main.c:388-395.  *dt_out receives dt. */
int fb_disk_step(fb_disk *d, double dt_interval, double *dt_out);

/* One hydro step in three parts, for a disk split into radial slabs over
 * several GPUs (one slab per process; the reference's MPI run: split.c,
 * comm.c:197-363).  fb_disk_step is the three in a row.
 *   fb_disk_step_begin     ComputeVmed + cfl (main.c:366-388): the slab's CFL
 *                          minimum, to be reduced with MIN over the slabs
 *                          (CflFluidsMin's MPI_Allreduce, cfl_fluids_min.c:14-17)
 *   fb_disk_step_advance   DT clip and planets with the global minimum, then
 *                          Sources (+ SubStep3): V_temp complete on the active
 *                          rows, physical ghosts filled; the caller then
 *                          exchanges the FB_HALO_VTEMP halos (FillGhosts after
 *                          Sources, algogas.c:116-118)
 *   fb_disk_step_transport Transport, NewVelocity, Stockholm and the physical
 *                          ghosts; the caller then exchanges the FB_HALO_STATE
 *                          halos (FillGhosts, main.c:431)
 * Halos: fb_disk_halo copies NGHY = 3 rows of every exchanged field (state:
 * rho, vx, vy[, vz][, energy]; vtemp: rho, vx_temp, vy_temp[, vz_temp][,
 * energy]) between the slab and a contiguous buffer [field][layer][3][Nx] of
 * fb_disk_halo_bytes bytes, device or host memory: side 0 = the inner (lower
 * radius) edge, side 1 = the outer; unpack = 0 packs the slab's first / last
 * three active rows, unpack = 1 writes its three ghost rows.  Synchronous. */
#define FB_HALO_STATE 0
#define FB_HALO_VTEMP 1
int fb_disk_step_begin(fb_disk *d, double *cfl_min);
int fb_disk_step_advance(fb_disk *d, double dt_interval, double cfl_min_global, double *dt_out);
int fb_disk_step_transport(fb_disk *d);
int fb_disk_halo_bytes(fb_disk *d, int which, size_t *bytes);
int fb_disk_halo(fb_disk *d, int which, int side, int unpack, void *buf, int buf_on_host);

/* [0] PhysicalTime [1] OMEGAFRAME [2] last dt [3..6] planet 0 x, y, vx, vy [7] Domega */
int fb_disk_get_scalars(fb_disk *d, double out8[8]);

/* Total mass of one fluid, ComputeMass (LowTasks.c:709-748): the sum over the
 * active cells of rho * Vol(i, j, k), computed on the device in FP64 with
 * compensated (Neumaier) summation, so a change of the total at round-off
 * level stays visible.  Synchronous (the reference returns it to the host
 * too); batch members: call fb_batch_sync first. */
int fb_disk_mass(fb_disk *d, int fluid, double *mass);

/* FARGO3D's output files (output.c): merged field files
 * <dir>/<fluid><field><n>.dat for field = dens, energy (the isothermal sound
 * speed), vx, vy[, vz] -- active cells, raw doubles, x fastest
 * (WriteMerging, output.c:283-315) -- and the restart read of the same files
 * (it replaces the active cells, keeps the ghosts; call fb_disk_initialize
 * after reading a new run's first state).  fluid is FARGO3D's fluid name
 * ("gas", "dust1", ...).  fb_disk_write_planets appends one line per planet
 * to <dir>/planet<k>.dat (WritePlanetFile, output.c:46-75). */
int fb_disk_write_dat(fb_disk *d, int fluid, const char *dir, const char *fluid_name, int n);
int fb_disk_read_dat(fb_disk *d, int fluid, const char *dir, const char *fluid_name, int n);
int fb_disk_write_planets(fb_disk *d, const char *dir, int n);

/* The planetary system and frame rotation (Sys, OMEGAFRAME and the initial
 * OMEGAFRAME0 of main.c:242; psys.c): set
 * replaces the circular orbits built from pl_dist (a running simulation
 * handing over its state), get reads the current one back.  n must equal
 * nplanets. */
int fb_disk_set_planets(fb_disk *d, int n, const double *x, const double *y, const double *z, const double *vx,
                        const double *vy, const double *vz, const double *mass, double omegaframe,
                        double omegaframe0);
int fb_disk_get_planets(fb_disk *d, int n, double *x, double *y, double *z, double *vx, double *vy, double *vz,
                        double *mass, double *omegaframe);

/* Device pointers of one fluid's state (rho, vx, vy, vz, cs) and the element
 * size, for callers that keep their inputs on the device.  FP32 disks hold vx
 * less the fluid's per-ring background (fb_disk_get_background). */
int fb_disk_device_fields(fb_disk *d, int fluid, void *ptrs5[5], size_t *elem_size);

/* FP32 disks store each fluid's azimuthal velocity relative to a per-ring
 * background vbg(j, k): the FP64 ring means of the first vx the caller set.  A
 * float then carries the deviation from the ring's rotation (the planet's wake,
 * the slow viscous drift) instead of the rotation itself, so its rounding is
 * that of the deviation; fb_disk_set_state / get_state convert both ways.  No
 * counterpart in the reference (whose -DFLOAT build stores vx itself in FP32,
 * types_def.h:2-6).  out: (Nz+6 or 1) x (Ny+6) doubles, zero for FP64 disks. */
int fb_disk_get_background(fb_disk *d, int fluid, double *out);

/* Stream the disk's kernels run on (a cudaStream_t). */
void *fb_disk_stream(fb_disk *d);

/* Per-launch device timing of the following steps (CUDA events on the disk's
 * stream).  fb_disk_profile_read returns the number of intervals written:
 * ms[i] is the time of the launch group names[i] in the last profiled step. */
int fb_disk_profile(fb_disk *d, int enable);
int fb_disk_profile_read(fb_disk *d, float *ms, const char **names, int max);

/* ---- many independent disks advanced together (fargo3d_b200/csrc/fb_batch.cu).
 * Each stage of a step is ONE launch over the tiles of all disks; the step's
 * scalar work (time step, planets, frame) runs on the device, one thread per
 * disk, and sequences of steps replay from a captured CUDA graph.  All disks
 * share a precision, a dimensionality and a fluid count.  A disk whose state
 * turns non-finite, or whose time step collapses, is frozen with that status
 * while the others continue.  No counterpart in the reference (one disk per
 * run); each disk's step is the one of fb_disk_step. */
typedef struct fb_batch fb_batch;
int fb_batch_create(const fb_params *ps, int ndisks, int precision, int device, fb_batch **out);
int fb_batch_destroy(fb_batch *b);
/* the disk object of member i: use fb_disk_set_state / fb_disk_get_state on it
 * (call fb_batch_sync first when reading) */
int fb_batch_disk(fb_batch *b, int i, fb_disk **d);
int fb_batch_initialize(fb_batch *b);
/* enqueue nsteps hydro steps of every disk; returns without waiting */
int fb_batch_run(fb_batch *b, int nsteps, double dt_interval);
int fb_batch_sync(fb_batch *b);
int fb_batch_get_scalars(fb_batch *b, int i, double out8[8], int *status);
void *fb_batch_stream(fb_batch *b);
/* one eager step with per-launch-group device timing (see fb_disk_profile_read) */
int fb_batch_profile_step(fb_batch *b, double dt_interval, float *ms, const char **names, int max);

/* Batches with changing membership (no counterpart in the reference).  A
 * batch made with fb_batch_create_slots holds up to `capacity` disks of one
 * precision, dimensionality and fluid count; members join and leave between
 * fb_batch_run calls, and the stage work lists and the captured graph are
 * rebuilt at the next run after a change.  fb_batch_add creates a disk in a
 * free slot (state still to be set through fb_batch_disk + fb_disk_set_state);
 * fb_batch_activate initialises it and lets it step.  With t_end > 0 the disk
 * runs until its physical time reaches t_end (its last step clipped to land
 * on it, as a DT interval of length t_end clips the reference's last step)
 * and is then frozen with FB_DONE; with t_end <= 0 it follows the dt_interval
 * given to fb_batch_run.  fb_batch_remove destroys the slot's disk.
 * fb_batch_poll reads every slot's status (FB_OK, FB_DONE, FB_SLOT_EMPTY,
 * FB_SLOT_RESERVED or the error that froze it), physical time and step count
 * after waiting for the batch's stream; arrays have `capacity` entries. */
int fb_batch_create_slots(int capacity, int precision, int device, int is3d, int nfluids, fb_batch **out);
int fb_batch_add(fb_batch *b, const fb_params *p, double t_end, int *slot);
int fb_batch_activate(fb_batch *b, int slot);
int fb_batch_remove(fb_batch *b, int slot);
int fb_batch_capacity(fb_batch *b);
int fb_batch_poll(fb_batch *b, int *status, double *phys_time, long long *steps);

/* Tile shapes (no counterpart in the reference, whose c2cuda build fixes one
 * block shape per kernel after a sweep, scripts/blocks_function.py):
 * sweep_x_cells = cells per thread of the azimuthal sweep (1, 2, 4, 8 or 16,
 * dividing Nx with at most 256 threads per ring), col_segment = cells per
 * thread of the radial/colatitude sweeps (4, 8 or 16); 0 = the default.  The
 * autotuner (fargo3d_b200/autotune.py) picks them per (Nx, Ny, Nz,
 * precision).  A batch member's choice takes effect at the next run. */
int fb_disk_set_tiles(fb_disk *d, int sweep_x_cells, int col_segment);
/* Failure detection of the azimuthal sweep's staged ring loads (no
 * counterpart in the reference, whose kernels never wait): a CTA polls the
 * copies' completion at most `polls` times (0: the default 2^22; negative:
 * not at all, the wait gives up at once).  A CTA that gives up waits,
 * boundedly again, for its copies to land, writes nothing and flags the
 * disk; fb_disk_step reports FB_ERR_NONFINITE at the next step (the flag is
 * read with that step's CFL minimum), a batch freezes the member.  A batch
 * member takes the value its disk has when it is activated. */
int fb_disk_set_wait_limit(fb_disk *d, long long polls);
int fb_disk_get_tiles(fb_disk *d, int *sweep_x_cells, int *col_segment);
int fb_batch_set_tiles(fb_batch *b, int slot, int sweep_x_cells, int col_segment);
/* Concurrent step chains (1..8; default 4 for FP32 batches, 1 for FP64): the
 * active disks are split into
 * this many groups of about equal cells, each stepped on its own stream, so
 * that the latency-bound launches of one group (the per-disk scalar step,
 * reductions, ghost fills, launch tails) overlap the others' stencil work.
 * Results do not depend on it (each disk's arithmetic is the same). */
int fb_batch_set_chains(fb_batch *b, int chains);
int fb_batch_get_chains(fb_batch *b);
/* Fluid `fluid`'s state of every member in one call (FARGO3D layout, as
 * fb_disk_set_state / fb_disk_get_state): arrays of one host pointer per
 * slot; a NULL array or entry skips that field or slot.  The transfers of all
 * members are queued on the batch's stream and waited for once, so page-
 * locked buffers move back to back by DMA. */
int fb_batch_set_states(fb_batch *b, int fluid, const double *const *rho, const double *const *vx,
                        const double *const *vy, const double *const *vz, const double *const *cs);
int fb_batch_get_states(fb_batch *b, int fluid, double *const *rho, double *const *vx, double *const *vy,
                        double *const *vz);

/* Device bytes: an upper bound of what fb_disk_create requests for these
 * parameters, and what a disk actually requested. */
int fb_params_bytes(const fb_params *p, int precision, size_t *out);
int fb_disk_bytes(fb_disk *d, size_t *out);

/* ---- continuous-batching server (fargo3d_b200/csrc/fb_server.cu; no
 * counterpart in the reference).  Requests (one disk-planet solve each: its
 * parameters, its initial state in host memory and an end time) are queued
 * by fb_server_submit from any thread.  A worker thread admits queued
 * requests in arrival order while their device bytes fit the HBM budget and
 * a slot is free, runs every admitted disk together in chunks of
 * `chunk_steps` steps (one batched launch per stage), and retires each disk
 * when it reaches its end time, copying its final state to host memory.
 * Requests arriving while others run join at the next chunk boundary.  All
 * requests share precision, dimensionality and fluid count (one fluid).
 * Times in info[] are seconds on the server's monotonic clock:
 * [0] submitted [1] admitted [2] finished [3] hydro steps [4] physical time
 * [5] final status [6] device bytes reserved [7] active cells. */
typedef struct fb_server fb_server;
int fb_server_create(int precision, int device, int is3d, size_t hbm_budget, int max_disks, int chunk_steps,
                     fb_server **out);
int fb_server_submit(fb_server *s, const fb_params *p, const double *rho, const double *vx, const double *vy,
                     const double *vz, const double *cs, double t_end, long long *id);
/* request state (FB_REQ_*) */
int fb_server_status(fb_server *s, long long id, int *state);
/* wait up to timeout_s seconds for a request to finish; *state as above */
int fb_server_wait(fb_server *s, long long id, double timeout_s, int *state);
/* copy a finished request's final state and info[8] out and forget it */
int fb_server_fetch(fb_server *s, long long id, double *rho, double *vx, double *vy, double *vz, double info[8]);
/* [0] queued [1] running [2] finished, not fetched [3] device bytes reserved
 * [4] budget [5] chunks run [6] cell-updates done [7] seconds since create */
int fb_server_stats(fb_server *s, double out8[8]);
double fb_server_clock(fb_server *s);
/* tiles (fb_disk_set_tiles) for every later admitted disk of this shape */
int fb_server_set_tiles(fb_server *s, int nx, int ny, int nz, int sweep_x_cells, int col_segment);
int fb_server_destroy(fb_server *s);

/* CFL time step without allocating: for callers that own all device memory
 * and cannot let a library call cudaMalloc (FARGO3D's own GPU build, whose
 * Fields CreateField allocates once; applications on a fixed memory pool).
 * No counterpart in the reference: it computes what ComputeVmed + cfl + cfl_b
 * + CflFluidsMin compute at the start of a step (main.c:366-390), for one FP64
 * fluid whose fields and mesh edges the caller holds in device memory, and
 * writes StepTime to the caller's device double *dt_out on `stream`.  Its
 * scratch is a fixed file-scope device array: meshes with more than
 * FB_NOALLOC_MAX_RINGS rings ((Ny+6) x (Nz+6 or 1)) are rejected with
 * FB_ERR_TOO_LARGE.  The first call on each device looks the array up and must
 * come before any stream capture; calls that overlap on the GPU race.
 * Fields may be pitched as FARGO3D's cudaMallocPitch Fields are (Pitch_gpu /
 * Stride_gpu, allocate.c:169-206): pitch and stride in elements, 0 for a
 * dense [nz+6|1][ny+6][nx] array.  A state with a non-finite limit or a
 * non-positive density yields *dt_out = NaN; a zero limit yields 0 (the
 * reference's null time step). */
#define FB_NOALLOC_MAX_RINGS 65536
typedef struct {
  int nx, ny, nz;              /* active zones; nz <= 1: 2D                      */
  int spherical, alpha_visc;
  const double *rho, *cs, *vx, *vy, *vz;  /* device fields, [nz+6|1][ny+6][pitch] */
  const double *xmin, *ymin, *zmin;       /* device mesh edges (Xmin, Ymin, Zmin) */
  const double *sin_zmed;                 /* device sin(Zmed(k)) (spherical only) */
  double cfl, nu, alpha;
  double mindx;                /* min_i (Xmin[i+1] - Xmin[i])                     */
  double xlen;                 /* XMAX - XMIN                                     */
  int pitch;                   /* elements between rows (Pitch_gpu); 0: nx       */
  long long stride;            /* elements between layers (Stride_gpu); 0: pitch x (ny+6) */
} fb_cfl_static_args;
int fb_cfl_dt_static(const fb_cfl_static_args *args, double *dt_out, void *stream);

const char *fb_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
