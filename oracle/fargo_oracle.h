/*
 * fargo_oracle.h -- TEST INFRASTRUCTURE ONLY.
 *
 * CPU restatement, in plain C99, of FARGO3D's hydro time step for the two
 * geometries this project covers (2D cylindrical, 3D spherical; isothermal;
 * FARGO orbital advection; constant-nu or alpha viscosity; planets with the
 * indirect term; Stockholm damping; Keplerian ghost boundaries) and of the
 * multifluid implicit drag step.  It exists only so that tests, the smoke
 * check and the CPU leg of the benchmark have something to compare the CUDA
 * path against.  Nothing in the shipped library links or calls it.
 *
 * Parity of this restatement is pinned against the reference's own C
 * kernels, compiled from their sources by oracle/ref/Makefile and driven in
 * main.c order (tests/test_oracle_pin.py, tests/golden/).
 */
#ifndef FARGO_ORACLE_H
#define FARGO_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define FO_NGH 3          /* NGHY = NGHZ = 3 (define.h:57-63) */
#define FO_MAXPLANETS 8
#define FO_MAXFLUIDS 8

enum { FO_FRAME_FIXED = 0, FO_FRAME_COROT = 1, FO_FRAME_GUIDING = 2 };

typedef struct {
  int nx, ny, nz;              /* active zones; nz <= 1 selects the 2D (X,Y) build */
  int spherical;               /* 0: CYLINDRICAL, 1: SPHERICAL (3D only)          */
  int log_spacing;             /* Spacing Log (LowTasks.c:337-341)                */
  double xmin, xmax, ymin, ymax, zmin, zmax;
  double aspectratio, sigmaslope, flaringindex;
  double nu;                   /* VISCOSITY (constant nu)                          */
  double alpha; int alpha_visc;/* ALPHAVISCOSITY when alpha_visc != 0              */
  double cfl;
  double omegaframe; int frame;
  int indirect_term;
  double thickness_smoothing, roche_smoothing, mass_taper;
  double damping_zone, tau_damp, killing_bc_colatitude;
  int nplanets;
  double pl_dist[FO_MAXPLANETS], pl_mass[FO_MAXPLANETS];
  int pl_feeldisk[FO_MAXPLANETS], pl_feelothers[FO_MAXPLANETS];
  double eccentricity, inclination;
  int nfluids;                 /* 1: gas only; >1: gas + dust, implicit drag       */
  double invstokes[FO_MAXFLUIDS]; /* STOKESNUMBER drag: [f-1] = 1/St of dust fluid f */
  int stockholm;               /* STOCKHOLM damping on/off                        */
  int adiabatic;               /* ADIABATIC equation of state (2D cylindrical, gas) */
  double gamma;                /* GAMMA                                            */
  int dust_diffusion;          /* DUSTDIFFUSION (2D cylindrical, dust fluids)       */
  int slab_y0, slab_ny_global; /* the library's radial slabs (unused here: whole disks) */
} fo_params;

typedef struct fo_disk fo_disk;

fo_disk *fo_create(const fo_params *p);
void     fo_destroy(fo_disk *d);

/* Geometry accessors (arrays of the reference sizes: Nx+1, Ny+2*NGHY+1, ...). */
void fo_get_geometry(const fo_disk *d, double *xmin_a, double *ymin_a, double *zmin_a);

/* Full stored arrays (ghosts included), layout l = i + j*Nx + k*Nx*(Ny+6).
 * Fluid f in [0, nfluids). cs is the isothermal sound speed field. */
void fo_set_state(fo_disk *d, int f, const double *rho, const double *vx,
                  const double *vy, const double *vz, const double *cs);
void fo_get_state(const fo_disk *d, int f, double *rho, double *vx, double *vy,
                  double *vz);
/* Boundaries then the Stockholm reference profiles (main.c:311-316). */
void fo_initialize(fo_disk *d);
/* One hydro step with dt = min(CFL dt, dtmax) as main.c:361-448 computes it for
 * a DT interval of length dtmax starting at dtemp = 0.  Returns dt, or -1 on
 * a null time step (cfl_fluids_min.c:18-21). */
double fo_step(fo_disk *d, double dt_interval);
/* Scalars: [0] PhysicalTime, [1] OMEGAFRAME, [2] last dt, [3] planet0 x,
 * [4] planet0 y, [5] planet0 vx, [6] planet0 vy, [7] Domega. */
void fo_get_scalars(const fo_disk *d, double *out8);
/* Total mass of fluid f over the active mesh (compensated sum). */
double fo_mass(const fo_disk *d, int f);
/* the fluid's Energy field: the internal energy of an adiabatic disk, the
 * sound speed of an isothermal one */
void fo_get_energy(const fo_disk *d, int f, double *e);

#ifdef __cplusplus
}
#endif
#endif
