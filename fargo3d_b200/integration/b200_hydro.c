/*
 * b200_hydro.c -- the FARGO3D side of the drop-in: compiled INTO a FARGO3D
 * build (list it in setups/<setup>/<setup>.objects, link -lfargo_b200), it
 * hands the hydro step of main.c:361-448 to libfargo_b200 on a B200.
 *
 * It reads what FARGO3D already holds -- the .par variables (var.c globals),
 * the compile-time physics (-DSPHERICAL, -DALPHAVISCOSITY, -DSTOCKHOLM,
 * -DDRAGFORCE/-DSTOKESNUMBER), the Fields of every fluid, the planetary system
 * Sys and OMEGAFRAME -- and keeps them current, so FARGO3D's outputs,
 * monitors and restarts work unchanged:
 *
 *   B200_Attach()         after CondInit, FillGhosts and init_stockholm
 *                         (main.c:311-315): creates the disk and uploads
 *                         every fluid's Density, Vx, Vy[, Vz] and Energy
 *   B200_HydroStep(DT,&dt)  replaces the body of the DT loop (main.c:361-448:
 *                         ComputeVmed ... Sources, Collisions, Transport,
 *                         StockholmBoundary, FillGhosts); returns the dt taken
 *                         with the reference's DT clipping
 *   B200_Sync()           device state -> every fluid's field_cpu, Sys and
 *                         OMEGAFRAME (call before WriteOutputs / monitors)
 *   B200_Detach()
 *
 * A main loop then reads
 *
 *   while (dtemp < DT) { real dt; B200_HydroStep(DT, &dt); dtemp += dt;
 *                        PhysicalTime += dt; Timestepcount++; }
 *   B200_Sync(); MULTIFLUID(WriteOutputs(ALL));
 *
 * Errors follow FARGO3D's contract for its _gpu functions (lowtasks.cu:6-15):
 * the message goes through prs_error and the run stops.
 *
 * Precision: FARGO3D's `real` is double (types_def.h); the disk runs the
 * plain FP64 path (B200_PRECISION=FB_FP32 at compile time selects the FP32
 * transport path instead).
 */
#include <stdio.h>
#include <string.h>

#include "fargo3d.h"
#include "fargo_b200.h"

#ifndef B200_PRECISION
#define B200_PRECISION FB_FP64
#endif
#ifndef B200_DEVICE
#define B200_DEVICE 0
#endif

static fb_disk *b200_disk = NULL;

/* state of the registration through a setup directory (below) */
static int b200_registered = 0;
static int b200_stale[NFLUIDS];        /* the device holds a newer state */
static int b200_dirty[NFLUIDS];        /* host code wrote the state since the last upload */
static int b200_vmed_pending[NFLUIDS]; /* ComputeVmed(Vx) deferred until VxMed is read */
static int b200_in_sync = 0;
static void (*b200_reset_field_host)(Field *) = NULL;

static void b200_check(int rc, const char *what) {
  char msg[512];
  if (rc == FB_OK) return;
  snprintf(msg, sizeof msg, "libfargo_b200: %s failed (%d): %s", what, rc, fb_last_error());
  prs_error(msg);
}

/* fb_params from FARGO3D's run-time and compile-time configuration */
static void b200_params(fb_params *p) {
  int i;
  memset(p, 0, sizeof *p);
  p->nx = NX; p->ny = NY; p->nz = NZ;
#ifdef SPHERICAL
  p->spherical = 1;
#endif
  p->log_spacing = strcmp(SPACING, "Log") == 0 || strcmp(SPACING, "LOG") == 0 || strcmp(SPACING, "log") == 0;
  p->xmin = XMIN; p->xmax = XMAX; p->ymin = YMIN; p->ymax = YMAX; p->zmin = ZMIN; p->zmax = ZMAX;
  p->aspectratio = ASPECTRATIO; p->sigmaslope = SIGMASLOPE; p->flaringindex = FLARINGINDEX;
  p->nu = NU; p->alpha = ALPHA;
#ifdef ALPHAVISCOSITY
  p->alpha_visc = 1;
#endif
  p->cfl = CFL;
  p->omegaframe = OMEGAFRAME;
  p->frame = *FRAME == 'F' ? FB_FRAME_FIXED : (*FRAME == 'C' ? FB_FRAME_COROT : FB_FRAME_GUIDING);
  p->indirect_term = INDIRECTTERM == YES;
  p->thickness_smoothing = THICKNESSSMOOTHING; p->roche_smoothing = ROCHESMOOTHING;
  p->mass_taper = MASSTAPER; p->damping_zone = DAMPINGZONE; p->tau_damp = TAUDAMP;
  p->killing_bc_colatitude = KILLINGBCCOLATITUDE;
  p->nplanets = Sys ? Sys->nb : 0;
  for (i = 0; i < p->nplanets && i < FB_MAXPLANETS; i++) {
    p->pl_dist[i] = sqrt(Sys->x[i] * Sys->x[i] + Sys->y[i] * Sys->y[i] + Sys->z[i] * Sys->z[i]);
    p->pl_mass[i] = Sys->mass[i];
    p->pl_feeldisk[i] = Sys->FeelDisk[i] == YES;
    p->pl_feelothers[i] = Sys->FeelOthers[i] == YES;
  }
  p->eccentricity = ECCENTRICITY; p->inclination = INCLINATION;
  p->nfluids = NFLUIDS;
#ifdef DRAGFORCE
  /* the collision rates ColRate stored (colrate.c): gas row of Alpha */
  for (i = 1; i < NFLUIDS; i++) p->invstokes[i - 1] = Alpha[0 + i * NFLUIDS];
#endif
#ifdef STOCKHOLM
  p->stockholm = 1;
#endif
#ifdef ADIABATIC
  p->adiabatic = 1;
  p->gamma = GAMMA;
#endif
#ifdef DUSTDIFFUSION
  p->dust_diffusion = 1;
#endif
}

void B200_Attach(void) {
  fb_params p;
  int f;
  if (b200_disk) return;
  b200_params(&p);
  b200_check(fb_disk_create(&p, B200_PRECISION, B200_DEVICE, &b200_disk), "fb_disk_create");
  for (f = 0; f < NFLUIDS; f++) {
    Fluid *F = Fluids[f];
    b200_check(fb_disk_set_state(b200_disk, f, F->Density->field_cpu, F->Vx->field_cpu, F->Vy->field_cpu,
#ifdef Z
                                 F->Vz->field_cpu,
#else
                                 NULL,
#endif
                                 F->Energy->field_cpu),
               "fb_disk_set_state");
  }
  if (Sys && Sys->nb > 0)
    b200_check(fb_disk_set_planets(b200_disk, Sys->nb, Sys->x, Sys->y, Sys->z, Sys->vx, Sys->vy, Sys->vz,
                                   Sys->mass, OMEGAFRAME, OMEGAFRAME0),
               "fb_disk_set_planets");
  b200_check(fb_disk_initialize(b200_disk), "fb_disk_initialize");
}

void B200_HydroStep(real DT_interval, real *dt) {
  double d = 0.0;
  if (!b200_disk) B200_Attach();
  b200_check(fb_disk_step(b200_disk, DT_interval, &d), "fb_disk_step");
  if (dt) *dt = d;
}

void B200_Sync(void) {
  int f;
  if (!b200_disk) return;
  for (f = 0; f < NFLUIDS; f++) {
    Fluid *F = Fluids[f];
    b200_check(fb_disk_get_state(b200_disk, f, F->Density->field_cpu, F->Vx->field_cpu, F->Vy->field_cpu,
#ifdef Z
                                 F->Vz->field_cpu
#else
                                 NULL
#endif
                                 ),
               "fb_disk_get_state");
#ifdef ADIABATIC
    b200_check(fb_disk_get_energy(b200_disk, f, F->Energy->field_cpu), "fb_disk_get_energy");
#endif
  }
  if (Sys && Sys->nb > 0) {
    double om;
    b200_check(fb_disk_get_planets(b200_disk, Sys->nb, Sys->x, Sys->y, Sys->z, Sys->vx, Sys->vy, Sys->vz,
                                   Sys->mass, &om),
               "fb_disk_get_planets");
    OMEGAFRAME = om;
  }
  for (f = 0; f < NFLUIDS; f++) b200_stale[f] = 0;
}

void B200_Detach(void) {
  if (b200_disk) fb_disk_destroy(b200_disk);
  b200_disk = NULL;
}

/* ------------------------------------------------------------------------
 * Registration through a setup directory: no edit of main.c.
 *
 * FARGO3D's makefile searches the setup directory first (VPATH,
 * src/makefile:306), so a setup that carries its own copy of a source file
 * replaces the stock one.  The files in fargo3d_b200/integration/setup/ --
 * algogas.c (FillGhosts, Sources, Transport), cfl.c (cfl_cpu),
 * compute_vmed.c (ComputeVmed, ComputeVweight_cpu), dust_diffusion_main.c
 * and fresh.c (INPUT / OUTPUT) -- are written here and route the stock DT
 * loop of main.c:361-448 to the library:
 *
 *   MULTIFLUID(ComputeVmed(Vx))   deferred: the library takes its own means
 *   MULTIFLUID(cfl()); CflFluidsMin()
 *                                 fluid 0: B200_Begin() -> Min[0] (the minimum
 *                                 over every fluid), other fluids 1e30
 *   dt clipping                   main.c's own; the library clips the same way
 *                                 and the two dt must agree
 *   MULTIFLUID(Sources(dt)), Collisions, DustDiffusion_Main
 *                                 fluid 0: B200_Advance(dt); the rest no-ops
 *   MULTIFLUID(Transport(dt)), StockholmBoundary, FillGhosts
 *                                 fluid 0: B200_Transport(); the rest no-ops
 *
 * B200_Begin attaches on its first call (after CondInit, the initial
 * FillGhosts and init_stockholm, or a restart) and rebinds the stage pointers
 * that the loop still calls and that would touch the host fields
 * (StockholmBoundary, _collisions, ComputeTotalDensity, Reset_field on
 * Total_Density) the way ChangeArch binds them (change_arch.c:163-567).
 * The host copies of Density, Vx, Vy, Vz and Energy then follow FARGO3D's
 * own freshness protocol (fresh.c): INPUT(f) in any host code -- outputs,
 * monitors -- copies the fluid back from the device when the device is
 * ahead, OUTPUT(f) on a state field marks it for upload before the next
 * step.  The planetary system and OMEGAFRAME are copied back after every
 * step (host scalars). */


int B200_Attached(void) { return b200_disk != NULL && b200_registered; }

/* the fluid whose state field f is, or -1 */
int B200_StateFluid(const Field *f) {
  int k;
  for (k = 0; k < NFLUIDS; k++) {
    const Fluid *F = Fluids[k];
    if (f == F->Density || f == F->Energy || f == F->Vx || f == F->Vy) return k;
#ifdef Z
    if (f == F->Vz) return k;
#endif
  }
  return -1;
}

/* the fluid whose VxMed f is, or -1 */
int B200_VmedFluid(const Field2D *f) {
  int k;
  for (k = 0; k < NFLUIDS; k++)
    if (f == Fluids[k]->VxMed) return k;
  return -1;
}

static void b200_noop_real(real dt) { (void)dt; }
static void b200_noop_void(void) {}
static void b200_noop_collisions(real dt, int a, int b, int c, int o) {
  (void)dt; (void)a; (void)b; (void)c; (void)o;
}
static void b200_reset_field(Field *f) {
  if (f == Total_Density) return;   /* only the host's total density of the fused step */
  b200_reset_field_host(f);
}

static void b200_register(void) {
  int k;
  StockholmBoundary = b200_noop_real;       /* fused into NewVelocity */
  _collisions = b200_noop_collisions;       /* the drag runs in B200_Advance */
  ComputeTotalDensity = b200_noop_void;     /* the library forms its own */
  b200_reset_field_host = Reset_field;
  Reset_field = b200_reset_field;
  for (k = 0; k < NFLUIDS; k++) b200_stale[k] = b200_dirty[k] = b200_vmed_pending[k] = 0;
  b200_registered = 1;
}

/* device -> host for fluid k (its five state fields), when the device is ahead */
void B200_InputFluid(int k) {
  Fluid *F;
  if (!B200_Attached() || k < 0 || !b200_stale[k] || b200_in_sync) return;
  F = Fluids[k];
  b200_in_sync = 1;
  b200_check(fb_disk_get_state(b200_disk, k, F->Density->field_cpu, F->Vx->field_cpu, F->Vy->field_cpu,
#ifdef Z
                               F->Vz->field_cpu
#else
                               NULL
#endif
                               ),
             "fb_disk_get_state");
  b200_check(fb_disk_get_energy(b200_disk, k, F->Energy->field_cpu), "fb_disk_get_energy");
  b200_stale[k] = 0;
  b200_in_sync = 0;
}

/* host code wrote a state field of fluid k: upload before the next step */
void B200_OutputFluid(int k) {
  if (!B200_Attached() || k < 0 || b200_in_sync) return;
  B200_InputFluid(k);   /* the fields it did not write must be current too */
  b200_dirty[k] = 1;
}

int B200_VmedPending(int k) { return B200_Attached() && k >= 0 && b200_vmed_pending[k]; }
void B200_SetVmedPending(int k, int v) { if (k >= 0) b200_vmed_pending[k] = v; }

/* cfl() of the DT loop, fluid 0: the CFL minimum over every fluid */
real B200_Begin(void) {
  double m = 0.0;
  int k;
  if (!b200_disk) B200_Attach();
  if (!b200_registered) b200_register();
  for (k = 0; k < NFLUIDS; k++) {
    if (!b200_dirty[k]) continue;
    Fluid *F = Fluids[k];
    b200_check(fb_disk_set_state(b200_disk, k, F->Density->field_cpu, F->Vx->field_cpu, F->Vy->field_cpu,
#ifdef Z
                                 F->Vz->field_cpu,
#else
                                 NULL,
#endif
                                 F->Energy->field_cpu),
               "fb_disk_set_state");
    b200_dirty[k] = 0;
  }
  b200_check(fb_disk_step_begin(b200_disk, &m), "fb_disk_step_begin");
  return m;
}

/* Sources(dt) of the DT loop, fluid 0: planets, sources, drag, dust
 * diffusion of every fluid; dt is main.c's clipped step */
void B200_Advance(real dt) {
  double d = 0.0, om;
  int k;
  char msg[160];
  b200_check(fb_disk_step_advance(b200_disk, DT, StepTime, &d), "fb_disk_step_advance");
  if (d != dt) {
    snprintf(msg, sizeof msg, "libfargo_b200: the library's step %.17g differs from main.c's %.17g", d, dt);
    prs_error(msg);
  }
  for (k = 0; k < NFLUIDS; k++) b200_stale[k] = 1;
  if (Sys && Sys->nb > 0) {
    b200_check(fb_disk_get_planets(b200_disk, Sys->nb, Sys->x, Sys->y, Sys->z, Sys->vx, Sys->vy, Sys->vz,
                                   Sys->mass, &om),
               "fb_disk_get_planets");
    OMEGAFRAME = om;
  }
}

/* Transport(dt) of the DT loop, fluid 0: transport, NewVelocity, Stockholm
 * and the ghosts of every fluid */
void B200_Transport(void) {
  int k;
  b200_check(fb_disk_step_transport(b200_disk), "fb_disk_step_transport");
  for (k = 0; k < NFLUIDS; k++) b200_stale[k] = 1;
}
