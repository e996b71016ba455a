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
  }
  if (Sys && Sys->nb > 0) {
    double om;
    b200_check(fb_disk_get_planets(b200_disk, Sys->nb, Sys->x, Sys->y, Sys->z, Sys->vx, Sys->vy, Sys->vz,
                                   Sys->mass, &om),
               "fb_disk_get_planets");
    OMEGAFRAME = om;
  }
}

void B200_Detach(void) {
  if (b200_disk) fb_disk_destroy(b200_disk);
  b200_disk = NULL;
}
