/*
 * ref_glue.c -- drives the reference's own hot-path C sources (compiled from
 * their location in the reference tree by oracle/ref/Makefile) so that the
 * oracle restatement can be pinned against them.  TEST INFRASTRUCTURE ONLY.
 *
 * What is the reference's code: every kernel and driver function called from
 * ref_step() -- Sources, Transport, ComputeVmed, cfl, CflFluidsMin,
 * compute_potential, the planetary system, StockholmBoundary, FillGhosts,
 * boundaries() and all *_cpu kernels.
 * With -DFB_DROPIN the step instead runs through the drop-in binding
 * (fargo3d_b200/integration/b200_hydro.c) on the B200 library, from the same
 * Fields, .par globals and planetary system.  With -DFB_SHADOW the step
 * body stays the stock one and the setup-directory files of
 * fargo3d_b200/integration/setup (algogas.c, cfl.c, compute_vmed.c,
 * dust_diffusion_main.c, fresh.c) replace the reference's, as a FARGO3D setup
 * directory would (VPATH, src/makefile:306).
 * What is written here: what FARGO3D's build generates or its start-up does
 * (main.c, ChangeArch, var.c/param.h, the generated boundary functions from
 * std/boundaries.txt + the setup's .bound file, InitSpace/InitSurfaces,
 * CreateFields), the main.c DT-loop body, and no-op stand-ins for I/O, MPI
 * and timing.  The boundary stand-ins follow scripts/boundparser.py:360-398.
 */
#define __LOCAL
#include "fargo3d.h"
#undef __LOCAL

#include "fargo_oracle.h"

/* ---- stand-ins for functions outside the compiled set ------------------- */
#ifndef FB_SHADOW
/* fresh.c (a CPU build keeps no device copies); with -DFB_SHADOW the
 * setup-directory fresh.c of fargo3d_b200/integration/setup is linked */
void Input_CPU(Field *f, int line, const char *file) { (void)f; (void)line; (void)file; }
void Output_CPU(Field *f, int line, const char *file) { (void)f; (void)line; (void)file; }
void Input2D_CPU(Field2D *f, int line, const char *file) { (void)f; (void)line; (void)file; }
void Output2D_CPU(Field2D *f, int line, const char *file) { (void)f; (void)line; (void)file; }
void Input2DInt_CPU(FieldInt2D *f, int line, const char *file) { (void)f; (void)line; (void)file; }
void Output2DInt_CPU(FieldInt2D *f, int line, const char *file) { (void)f; (void)line; (void)file; }
void Draft(Field *f, int line, const char *file) { (void)f; (void)line; (void)file; }
#endif
void masterprint(const char *t, ...) { (void)t; }
void mastererr(const char *t, ...) { (void)t; }
void prs_exit(int c) { fprintf(stderr, "reference prs_exit(%d)\n", c); exit(c); }
void prs_error(char *s) { fprintf(stderr, "reference error: %s\n", s); exit(1); }
void InitSpecificTime(TimeProcess *t, char *s) { (void)t; (void)s; }
real GiveSpecificTime(TimeProcess t) { (void)t; return 0.0; }
void Write2D(Field2D *f, char *a, char *b, int c) { (void)f; (void)a; (void)b; (void)c; }
boolean Read2D(Field2D *f, char *a, char *b, int c) { (void)f; (void)a; (void)b; (void)c; return TRUE; }
FILE *fopen_prs(char *n, char *m) { return fopen(n, m); }
void CheckMuteY_cpu(void) {}
void CheckMuteZ_cpu(void) {}
static void comm_none(int v) { (void)v; }
/* PrimitiveVariables (LowTasks.c:13-36); only its value is passed to comm. */
#ifdef ADIABATIC
int PrimitiveVariables(void) { return DENS | ENERGY | VX | VY; }
#else
int PrimitiveVariables(void) { return DENS | VX | VY; }
#endif

/* SelectFluid (LowTasks.c:565-593) */
void SelectFluid(int n) {
  Fluidtype = Fluids[n]->Fluidtype;
  Density = Fluids[n]->Density;
  Energy = Fluids[n]->Energy;
  VxMed = Fluids[n]->VxMed;
#ifdef X
  Vx = Fluids[n]->Vx; Vx_temp = Fluids[n]->Vx_temp; Vx_half = Fluids[n]->Vx_half;
#endif
#ifdef Y
  Vy = Fluids[n]->Vy; Vy_temp = Fluids[n]->Vy_temp; Vy_half = Fluids[n]->Vy_half;
#endif
#ifdef Z
  Vz = Fluids[n]->Vz; Vz_temp = Fluids[n]->Vz_temp; Vz_half = Fluids[n]->Vz_half;
#endif
#ifdef STOCKHOLM
  Density0 = Fluids[n]->Density0; Energy0 = Fluids[n]->Energy0;
  Vx0 = Fluids[n]->Vx0; Vy0 = Fluids[n]->Vy0; Vz0 = Fluids[n]->Vz0;
#endif
}

/* ---- boundaries generated from the setup .bound files ------------------- */
#define BND_LOOP_Y(side_body)                                           \
  {                                                                     \
    int i, j, k, nghy = NGHY, ny = Ny;                                  \
    int pitch = Pitch_cpu, stride = Stride_cpu;                         \
    int lgh, lghs, lact, lacts, lacts_null, jgh, jact, size_y = NGHY;   \
    (void)lacts; (void)lghs; (void)lacts_null; (void)size_y;            \
    for (k = 0; k < Nz + 2 * NGHZ; k++)                                 \
      for (j = 0; j < NGHY; j++)                                        \
        for (i = 0; i < Nx + 2 * NGHX; i++) { side_body }               \
  }

/* The adiabatic variant of the fargo setup (written for this oracle: no
 * setup of the reference runs a 2D adiabatic disk) adds
 *   Energy: Ymin: SYMMETRIC  Ymax: SYMMETRIC
 * to setups/fargo/fargo.bound: the ghost energy mirrors the active cell. */
#ifdef ADIABATIC
#define BND_ENERGY_SYMMETRIC Energy->field_cpu[lgh] = Energy->field_cpu[lact];
#else
#define BND_ENERGY_SYMMETRIC
#endif

#ifdef CYLINDRICAL
/* setups/fargo/fargo.bound: KEPLERIAN2DDENS, KEPLERIAN2DVAZIM, ANTISYMMETRIC */
static void bnd_ymin(void) {
  real *density = Density->field_cpu, *vx = Vx->field_cpu, *vy = Vy->field_cpu;
  real sigmaslope = SIGMASLOPE, omegaframe = OMEGAFRAME;
  BND_LOOP_Y(
    lgh = l; lghs = l;
    lact = i + (2 * nghy - j - 1) * pitch + k * stride;
    lacts = i + (2 * nghy - j) * pitch + k * stride;
    lacts_null = i + nghy * pitch + k * stride;
    jgh = j; jact = (2 * nghy - j - 1);
    density[lgh] = density[lact] * pow(Ymed(jact) / Ymed(jgh), sigmaslope);
    vx[lgh] = (vx[lact] + Ymed(jact) * omegaframe) * sqrt(Ymed(jact) / Ymed(jgh)) - Ymed(jgh) * omegaframe;
    BND_ENERGY_SYMMETRIC
    vy[lghs] = -vy[lacts];
    vy[lacts_null] = 0;)
}
static void bnd_ymax(void) {
  real *density = Density->field_cpu, *vx = Vx->field_cpu, *vy = Vy->field_cpu;
  real sigmaslope = SIGMASLOPE, omegaframe = OMEGAFRAME;
  BND_LOOP_Y(
    lgh = i + (ny + nghy + j) * pitch + k * stride;
    lghs = i + (ny + nghy + 1 + j) * pitch + k * stride;
    lact = i + (ny + nghy - 1 - j) * pitch + k * stride;
    lacts = i + (ny + nghy - 1 - j) * pitch + k * stride;
    lacts_null = i + (ny + nghy) * pitch + k * stride;
    jgh = (ny + nghy + j); jact = (ny + nghy - 1 - j);
    density[lgh] = density[lact] * pow(Ymed(jact) / Ymed(jgh), sigmaslope);
    vx[lgh] = (vx[lact] + Ymed(jact) * omegaframe) * sqrt(Ymed(jact) / Ymed(jgh)) - Ymed(jgh) * omegaframe;
    BND_ENERGY_SYMMETRIC
    if (j < size_y - 1) vy[lghs] = -vy[lacts];
    vy[lacts_null] = 0;)
}
#endif

#ifdef SPHERICAL
/* setups/p3disof/p3disof.bound: KEPLERIAN3DSPH*, SYMMETRIC, ANTISYMMETRIC */
static void bnd_ymin(void) {
  real *density = Density->field_cpu, *vx = Vx->field_cpu, *vy = Vy->field_cpu, *vz = Vz->field_cpu;
  real sigmaslope = SIGMASLOPE, omegaframe = OMEGAFRAME, flaringindex = FLARINGINDEX,
       aspectratio = ASPECTRATIO, r0 = R0;
  BND_LOOP_Y(
    lgh = l; lghs = l;
    lact = i + (2 * nghy - j - 1) * pitch + k * stride;
    lacts = i + (2 * nghy - j) * pitch + k * stride;
    lacts_null = i + nghy * pitch + k * stride;
    jgh = j; jact = (2 * nghy - j - 1);
    density[lgh] = density[lact] * pow(Ymed(jact) / Ymed(jgh), sigmaslope + flaringindex + 1.) *
      exp(-pow(cos(Zmed(k)), 2.) / (aspectratio * aspectratio) * (1. - Ymed(jgh) / (.5 * (Ymed(jact) + Ymed(jgh)))) *
          flaringindex * pow(.5 * (Ymed(jgh) + Ymed(jact)) / r0, -2. * flaringindex - 1.));
    vx[lgh] = (vx[lact] + omegaframe * Ymed(jact) * sin(Zmed(k))) * sqrt(Ymed(jact) / Ymed(jgh)) *
      (1. + (2. + sigmaslope - flaringindex) * (Ymed(jact) - Ymed(jgh)) / r0 * flaringindex * aspectratio *
       aspectratio * pow((Ymed(jgh) + Ymed(jact)) / (2. * r0), 2. * flaringindex - 1.)) -
      Ymed(jgh) * omegaframe * sin(Zmed(k));
    vy[lghs] = -vy[lacts];
    vy[lacts_null] = 0;
    vz[lgh] = vz[lact];)
}
static void bnd_ymax(void) {
  real *density = Density->field_cpu, *vx = Vx->field_cpu, *vy = Vy->field_cpu, *vz = Vz->field_cpu;
  real sigmaslope = SIGMASLOPE, omegaframe = OMEGAFRAME, flaringindex = FLARINGINDEX,
       aspectratio = ASPECTRATIO, r0 = R0;
  BND_LOOP_Y(
    lgh = i + (ny + nghy + j) * pitch + k * stride;
    lghs = i + (ny + nghy + 1 + j) * pitch + k * stride;
    lact = i + (ny + nghy - 1 - j) * pitch + k * stride;
    lacts = i + (ny + nghy - 1 - j) * pitch + k * stride;
    lacts_null = i + (ny + nghy) * pitch + k * stride;
    jgh = (ny + nghy + j); jact = (ny + nghy - 1 - j);
    density[lgh] = density[lact] * pow(Ymed(jact) / Ymed(jgh), sigmaslope + flaringindex + 1.) *
      exp(-pow(cos(Zmed(k)), 2.) / (aspectratio * aspectratio) * (1. - Ymed(jgh) / (.5 * (Ymed(jact) + Ymed(jgh)))) *
          flaringindex * pow(.5 * (Ymed(jgh) + Ymed(jact)) / r0, -2. * flaringindex - 1.));
    vx[lgh] = (vx[lact] + omegaframe * Ymed(jact) * sin(Zmed(k))) * sqrt(Ymed(jact) / Ymed(jgh)) *
      (1. + (2. + sigmaslope - flaringindex) * (Ymed(jact) - Ymed(jgh)) / r0 * flaringindex * aspectratio *
       aspectratio * pow((Ymed(jgh) + Ymed(jact)) / (2. * r0), 2. * flaringindex - 1.)) -
      Ymed(jgh) * omegaframe * sin(Zmed(k));
    if (j < size_y - 1) vy[lghs] = -vy[lacts];
    vy[lacts_null] = 0;
    vz[lgh] = vz[lact];)
}
#define BND_LOOP_Z(side_body)                                           \
  {                                                                     \
    int i, j, k, nghz = NGHZ, nz = Nz;                                  \
    int pitch = Pitch_cpu, stride = Stride_cpu;                         \
    int lgh, lghs, lact, lacts, lacts_null, kgh, kact, size_z = NGHZ;   \
    (void)lacts; (void)lghs; (void)lacts_null; (void)size_z; (void)pitch; \
    for (k = 0; k < NGHZ; k++)                                          \
      for (j = 0; j < Ny + 2 * NGHY; j++)                               \
        for (i = 0; i < Nx + 2 * NGHX; i++) { side_body }               \
  }
static void bnd_zmin(void) {
  real *density = Density->field_cpu, *vx = Vx->field_cpu, *vy = Vy->field_cpu, *vz = Vz->field_cpu;
  real sigmaslope = SIGMASLOPE, omegaframe = OMEGAFRAME, flaringindex = FLARINGINDEX,
       aspectratio = ASPECTRATIO, r0 = R0;
  BND_LOOP_Z(
    lgh = l; lghs = l;
    lact = i + j * pitch + (2 * nghz - k - 1) * stride;
    lacts = i + j * pitch + (2 * nghz - k) * stride;
    lacts_null = i + j * pitch + nghz * stride;
    kgh = k; kact = (2 * nghz - k - 1);
    density[lgh] = density[lact] * pow(sin(Zmed(kgh)) / sin(Zmed(kact)),
      flaringindex - 2. - sigmaslope + 1. / (aspectratio * aspectratio) * pow(Ymed(j) / r0, -2. * flaringindex));
    vx[lgh] = (vx[lact] + omegaframe * Ymed(j) * sin(Zmed(kact))) *
      (1. + flaringindex * cos(.5 * (Zmed(kgh) + Zmed(kact))) * (Zmed(kact) - Zmed(kgh))) -
      Ymed(j) * omegaframe * sin(Zmed(kgh));
    vy[lgh] = vy[lact];
    vz[lghs] = -vz[lacts];
    vz[lacts_null] = 0;)
}
static void bnd_zmax(void) {
  real *density = Density->field_cpu, *vx = Vx->field_cpu, *vy = Vy->field_cpu, *vz = Vz->field_cpu;
  real sigmaslope = SIGMASLOPE, omegaframe = OMEGAFRAME, flaringindex = FLARINGINDEX,
       aspectratio = ASPECTRATIO, r0 = R0;
  BND_LOOP_Z(
    lgh = i + j * pitch + (nz + nghz + k) * stride;
    lghs = i + j * pitch + (nz + nghz + 1 + k) * stride;
    lact = i + j * pitch + (nz + nghz - 1 - k) * stride;
    lacts = i + j * pitch + (nz + nghz - 1 - k) * stride;
    lacts_null = i + j * pitch + (nz + nghz) * stride;
    kgh = (nz + nghz + k); kact = (nz + nghz - 1 - k);
    density[lgh] = density[lact] * pow(sin(Zmed(kgh)) / sin(Zmed(kact)),
      flaringindex - 2. - sigmaslope + 1. / (aspectratio * aspectratio) * pow(Ymed(j) / r0, -2. * flaringindex));
    vx[lgh] = (vx[lact] + omegaframe * Ymed(j) * sin(Zmed(kact))) *
      (1. + flaringindex * cos(.5 * (Zmed(kgh) + Zmed(kact))) * (Zmed(kact) - Zmed(kgh))) -
      Ymed(j) * omegaframe * sin(Zmed(kgh));
    vy[lgh] = vy[lact];
    if (k < size_z - 1) vz[lghs] = -vz[lacts];
    vz[lacts_null] = 0;)
}
#endif

/* ---- start-up: InitSpace / InitSurfaces (LowTasks.c:300-563) ------------- */
static void glue_init_space(void) {
  int i, j, k;
  real dx = (XMAX - XMIN) / NX, dy = (YMAX - YMIN) / NY, dz = 0.0;
#ifdef Z
  dz = (ZMAX - ZMIN) / NZ;
#endif
  if (toupper(SPACING[0]) == 'L' && toupper(SPACING[1]) == 'O') {
    dy = (log(YMAX) - log(YMIN)) / NY;
    for (j = 0; j < Ny + 2 * NGHY + 1; j++) Ymin(j) = exp(log(YMIN) + dy * (j - NGHY));
  } else {
    for (j = 0; j < Ny + 2 * NGHY + 1; j++) Ymin(j) = YMIN + dy * (j - NGHY);
  }
  for (k = 0; k < Nz + 2 * NGHZ + 1; k++) {
#ifdef Z
    Zmin(k) = ZMIN + dz * (k - NGHZ);
#else
    Zmin(k) = 0.0;
#endif
  }
  (void)dz;
  for (i = 0; i < Nx + 2 * NGHX + 1; i++) Xmin(i) = XMIN + dx * (i - NGHX);
  for (i = 0; i < Nx + 2 * NGHX; i++) Xmed(i) = 0.5 * (Xmin(i + 1) + Xmin(i));
  for (j = 0; j < Ny + 2 * NGHY; j++) Ymed(j) = 0.5 * (Ymin(j + 1) + Ymin(j));
  for (k = 0; k < Nz + 2 * NGHZ; k++) Zmed(k) = 0.5 * (Zmin(k + 1) + Zmin(k));
  for (i = 1; i < Nx + 2 * NGHX; i++) InvDiffXmed(i) = 1. / (Xmed(i) - Xmed(i - 1));
  InvDiffXmed(0) = 1. / (Xmed(0) - (Xmed(Nx - 1) - (XMAX - XMIN)));
  for (i = 0; i < Nx + 2 * NGHX; i++) Sxi(i) = Xmin(i + 1) - Xmin(i);
  Mindx = Sxi(0);
  for (i = 1; i < Nx + 2 * NGHX; i++)
    if (Sxi(i) < Mindx) Mindx = Sxi(i);
#ifdef CYLINDRICAL
  for (j = 0; j < Ny + 2 * NGHY; j++) {
    Sxj(j) = Ymin(j + 1) - Ymin(j);
    Syj(j) = Ymin(j);
    Szj(j) = 0.5 * (Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j));
    InvVj(j) = 1.0 / Szj(j);
  }
  for (k = 0; k < Nz + 2 * NGHZ; k++) {
#ifdef Z
    Sxk(k) = Zmin(k + 1) - Zmin(k);
#else
    Sxk(k) = 1.0;
#endif
    Syk(k) = Sxk(k);
    Szk(k) = 1.0;
  }
#endif
#ifdef SPHERICAL
  for (j = 0; j < Ny + 2 * NGHY; j++) {
    Sxj(j) = 0.5 * (Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j));
    Syj(j) = Ymin(j) * Ymin(j);
    Szj(j) = 0.5 * (Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j));
    InvVj(j) = 3. / ((Ymin(j + 1) * Ymin(j + 1) * Ymin(j + 1) - Ymin(j) * Ymin(j) * Ymin(j)));
  }
  for (k = 0; k < Nz + 2 * NGHZ; k++) {
    Sxk(k) = Zmin(k + 1) - Zmin(k);
    Syk(k) = cos(Zmin(k)) - cos(Zmin(k + 1));
    Szk(k) = sin(Zmin(k));
  }
#endif
}

/* ChangeArch (change_arch.c:3-160): every pointer on its _cpu flavour. */
static void glue_change_arch(void) {
  ComputePressureFieldIso = ComputePressureFieldIso_cpu;
  SubStep1_x = SubStep1_x_cpu; SubStep1_y = SubStep1_y_cpu; SubStep1_z = SubStep1_z_cpu;
  SubStep2_a = SubStep2_a_cpu; SubStep2_b = SubStep2_b_cpu;
  DivideByRho = DivideByRho_cpu;
  VanLeerX_a = VanLeerX_a_cpu; VanLeerX_b = VanLeerX_b_cpu;
  VanLeerY_a = VanLeerY_a_cpu; VanLeerY_b = VanLeerY_b_cpu;
  VanLeerZ_a = VanLeerZ_a_cpu; VanLeerZ_b = VanLeerZ_b_cpu;
  momenta_x = momenta_x_cpu; momenta_y = momenta_y_cpu; momenta_z = momenta_z_cpu;
  reduction_SUM = reduction_SUM_cpu; reduction_MIN = reduction_MIN_cpu;
  UpdateX = UpdateX_cpu; UpdateY = UpdateY_cpu; UpdateZ = UpdateZ_cpu;
  UpdateDensityX = UpdateDensityX_cpu; UpdateDensityY = UpdateDensityY_cpu; UpdateDensityZ = UpdateDensityZ_cpu;
  NewVelocity_x = NewVelocity_x_cpu; NewVelocity_y = NewVelocity_y_cpu; NewVelocity_z = NewVelocity_z_cpu;
  AdvectSHIFT = AdvectSHIFT_cpu;
  ComputeResidual = ComputeResidual_cpu;
  ComputeVweight = ComputeVweight_cpu;
  Potential = Potential_cpu;
  CorrectVtheta = CorrectVtheta_cpu;
  cfl = cfl_cpu;
  _ComputeForce = _ComputeForce_cpu;
  copy_velocities = copy_velocities_cpu;
  VanLeerX_PPA_a = VanLeerX_PPA_a_cpu; VanLeerX_PPA_b = VanLeerX_PPA_b_cpu;
  VanLeerX_PPA_c = VanLeerX_PPA_c_cpu; VanLeerX_PPA_d = VanLeerX_PPA_d_cpu;
  Reset_field = Reset_field_cpu;
  ComputeTotalDensity = ComputeTotalDensity_cpu;
  StockholmBoundary = StockholmBoundary_cpu;
  visctensor_cyl = visctensor_cyl_cpu; addviscosity_cyl = addviscosity_cyl_cpu;
  visctensor_sph = visctensor_sph_cpu; addviscosity_sph = addviscosity_sph_cpu;
  SetupHook1 = SetupHook1_cpu;
  CheckMuteY = CheckMuteY_cpu; CheckMuteZ = CheckMuteZ_cpu;
#ifdef DRAGFORCE
  _collisions = _collisions_cpu;
#endif
#ifdef ADIABATIC
  ComputePressureFieldAd = ComputePressureFieldAd_cpu;
  SubStep3 = SubStep3_cpu;
#endif
#ifdef DUSTDIFFUSION
  DustDiffusion_Core = DustDiffusion_Core_cpu;
  DustDiffusion_Coefficients = DustDiffusion_Coefficients_cpu;
  copy_field = copy_field_cpu;
#endif
  comm = comm_none;
}

/* ---- driver API used by the tests (same shape as the oracle's) ----------- */
static double g_dtemp = 0.0, g_last_dt = 0.0;
static int g_nfluids = 1;

static void glue_planets(const fo_params *p) {
  /* InitPlanetarySystem (psys.c:141-225) without its file reading. */
  int nb = p->nplanets, i;
  PlanetarySystem *sys = (PlanetarySystem *)calloc(1, sizeof(PlanetarySystem));
  size_t sz = sizeof(real) * (nb + 1);
  sys->x = calloc(1, sz); sys->y = calloc(1, sz); sys->z = calloc(1, sz);
  sys->vx = calloc(1, sz); sys->vy = calloc(1, sz); sys->vz = calloc(1, sz);
  sys->mass = calloc(1, sz); sys->acc = calloc(1, sz);
  sys->FeelDisk = calloc(1, nb + 1); sys->FeelOthers = calloc(1, nb + 1);
  sys->x_cpu = sys->x; sys->y_cpu = sys->y; sys->z_cpu = sys->z; sys->mass_cpu = sys->mass;
  sys->nb = nb;
  for (i = 0; i < nb; i++) {
    real dist = p->pl_dist[i];
    sys->mass[i] = p->pl_mass[i];
    sys->x[i] = (real)dist * (1.0 + ECCENTRICITY);
    sys->y[i] = 0.0; sys->z[i] = 0.0;
    sys->vy[i] = (real)sqrt(G * (MSTAR + sys->mass[i]) / dist) * sqrt((1.0 - ECCENTRICITY) / (1.0 + ECCENTRICITY)) *
                 cos(INCLINATION);
    sys->vx[i] = -0.0000000000 * sys->vy[i];
    sys->vz[i] = sys->vy[i] * sin(INCLINATION) / cos(INCLINATION);
    sys->FeelDisk[i] = p->pl_feeldisk[i] ? YES : NO;
    sys->FeelOthers[i] = p->pl_feelothers[i] ? YES : NO;
  }
  Sys = sys;
  ThereArePlanets = nb > 0 ? YES : NO;
}

int ref_create(const fo_params *p) {
  int f;
  NX = p->nx; NY = p->ny; NZ = p->nz > 1 ? p->nz : 1;
  Nx = NX; Ny = NY; Nz = NZ;
#ifndef Z
  if (p->nz > 1) return -1;
#endif
  XMIN = p->xmin; XMAX = p->xmax; YMIN = p->ymin; YMAX = p->ymax; ZMIN = p->zmin; ZMAX = p->zmax;
  strcpy(SPACING, p->log_spacing ? "Log" : "Lin");
  ASPECTRATIO = p->aspectratio; SIGMASLOPE = p->sigmaslope; FLARINGINDEX = p->flaringindex;
  NU = p->nu; ALPHA = p->alpha; CFL = p->cfl; GAMMA = p->adiabatic ? p->gamma : 1.66666667;
#ifdef ADIABATIC
  if (!p->adiabatic) return -3;
#else
  if (p->adiabatic) return -3;
#endif
#ifdef DUSTDIFFUSION
  if (!p->dust_diffusion) return -4;
#else
  if (p->dust_diffusion) return -4;
#endif
  OMEGAFRAME = p->omegaframe;
  INDIRECTTERM = p->indirect_term ? YES : NO;
  THICKNESSSMOOTHING = p->thickness_smoothing; ROCHESMOOTHING = p->roche_smoothing; MASSTAPER = p->mass_taper;
  DAMPINGZONE = p->damping_zone; TAUDAMP = p->tau_damp; KILLINGBCCOLATITUDE = p->killing_bc_colatitude;
  ECCENTRICITY = p->eccentricity; INCLINATION = p->inclination;
  EXCLUDEHILL = NO; PERIODICY = NO; PERIODICZ = NO;
  RELEASEDATE = 0.0; RELEASERADIUS = 0.0; SEMIMAJORAXIS = 0.0; ORBITALRADIUS = 0.0; PLANETMASS = 0.0;
  strcpy(FRAME, p->frame == FO_FRAME_FIXED ? "F" : (p->frame == FO_FRAME_COROT ? "C" : "G"));
  Corotating = (p->frame != FO_FRAME_FIXED) ? YES : NO;
  GuidingCenter = (p->frame == FO_FRAME_GUIDING) ? YES : NO;
  strcpy(OUTPUTDIR, "./");
  /* split.c for one process: whole mesh, both radial edges are physical */
  Pitch_cpu = Nx + 2 * NGHX;
  Stride_cpu = (Nx + 2 * NGHX) * (Ny + 2 * NGHY);
  Pitch2D = Ny + 2 * NGHY;
  Gridd.bc_left = Gridd.bc_right = Gridd.bc_up = Gridd.bc_down = 1;
  Stride = Stride_cpu;
  /* split.c:157-205 */
  Xmin = calloc(Nx + 2 * NGHX + 1, sizeof(real)); Ymin = calloc(Ny + 2 * NGHY + 1, sizeof(real));
  Zmin = calloc(Nz + 2 * NGHZ + 1, sizeof(real));
  Xmed = calloc(Nx + 2 * NGHX, sizeof(real)); Ymed = calloc(Ny + 2 * NGHY, sizeof(real));
  Zmed = calloc(Nz + 2 * NGHZ, sizeof(real)); InvDiffXmed = calloc(Nx + 2 * NGHX, sizeof(real));
  Sxi = calloc(Nx + 2 * NGHX, sizeof(real));
  Sxj = calloc(Ny + 2 * NGHY, sizeof(real)); Syj = calloc(Ny + 2 * NGHY, sizeof(real));
  Szj = calloc(Ny + 2 * NGHY, sizeof(real)); InvVj = calloc(Ny + 2 * NGHY, sizeof(real));
  Sxk = calloc(Nz + 2 * NGHZ, sizeof(real)); Syk = calloc(Nz + 2 * NGHZ, sizeof(real));
  Szk = calloc(Nz + 2 * NGHZ, sizeof(real));
  Alpha = (real *)calloc(NFLUIDS * NFLUIDS, sizeof(real));
  glue_init_space();
  glue_change_arch();
  /* CreateFields (LowTasks.c:595-640), hydro subset */
  Reduction2D = CreateField2D("Reduction2D", YZ);
  Mpx = CreateField("Moment_Plus_X", 0, 1, 0, 0);
  Mmx = CreateField("Moment_Minus_X", 0, 1, 0, 0);
  Nshift = CreateFieldInt2D("Nshift");
  Mpy = CreateField("Moment_Plus_Y", 0, 0, 1, 0);
  Mmy = CreateField("Moment_Minus_Y", 0, 0, 1, 0);
#ifdef Z
  Mpz = CreateField("Moment_Plus_Z", 0, 0, 0, 1);
  Mmz = CreateField("Moment_Minus_Z", 0, 0, 0, 1);
#endif
  Pot = CreateField("potential", 0, 0, 0, 0);
  Slope = CreateField("Slope", 0, 0, 0, 0);
  DivRho = CreateField("DivRho", 0, 0, 0, 0);
  DensStar = CreateField("DensStar", 0, 0, 0, 0);
  Qs = CreateField("Qs", 0, 0, 0, 0);
  Pressure = CreateField("Pressure", 0, 0, 0, 0);
  Total_Density = CreateField("Total_Density", 0, 0, 0, 0);
  QL = CreateField("QLeft", 0, 0, 0, 0);
  QR = CreateField("QRight", 0, 0, 0, 0);
#ifdef DUSTDIFFUSION
  /* CreateFields (LowTasks.c:649-655): the diffusion coefficients */
  Sdiffyczc = CREATEFIELDALIAS("Sdiffyczc", Mpx, 0);
  Sdiffyfzc = CREATEFIELDALIAS("Sdiffyfzc", Mmx, 0);
#endif
  glue_planets(p);
  /* main.c:240-242 */
  if (Corotating && ThereArePlanets) OMEGAFRAME = GetPsysInfo(FREQUENCY);
  OMEGAFRAME0 = OMEGAFRAME;
  g_nfluids = p->nfluids > 1 ? p->nfluids : 1;
  if (g_nfluids != NFLUIDS) return -2;
  for (f = 0; f < NFLUIDS; f++) {
    Fluids[f] = CreateFluid(f == 0 ? "gas" : "dust", f == 0 ? GAS : DUST);
#ifdef Y
    boundary_ymin[f] = bnd_ymin;
    boundary_ymax[f] = bnd_ymax;
#endif
#ifdef Z
    boundary_zmin[f] = bnd_zmin;
    boundary_zmax[f] = bnd_zmax;
#endif
  }
#ifdef DRAGFORCE
  /* the collision rates of setups/fargo_multifluid/condinit.c:88-94, one per
     dust fluid, with feedback on the gas */
  for (f = 1; f < NFLUIDS; f++) ColRate(p->invstokes[f - 1], 0, f, YES);
#endif
  SelectFluid(0);
  g_dtemp = 0.0;
  return 0;
}

static size_t ncell(void) { return (size_t)(Nx + 2 * NGHX) * (Ny + 2 * NGHY) * (Nz + 2 * NGHZ); }

void ref_set_state(int f, const double *rho, const double *vx, const double *vy, const double *vz,
                   const double *cs) {
  size_t n = sizeof(real) * ncell();
  /* host code announces the Fields it writes (OUTPUT) and reads (INPUT):
   * FARGO3D's freshness protocol, fresh.c */
  OUTPUT(Fluids[f]->Density);
  OUTPUT(Fluids[f]->Vx);
  OUTPUT(Fluids[f]->Vy);
#ifdef Z
  OUTPUT(Fluids[f]->Vz);
#endif
  OUTPUT(Fluids[f]->Energy);
  if (rho) memcpy(Fluids[f]->Density->field_cpu, rho, n);
  if (vx) memcpy(Fluids[f]->Vx->field_cpu, vx, n);
  if (vy) memcpy(Fluids[f]->Vy->field_cpu, vy, n);
#ifdef Z
  if (vz) memcpy(Fluids[f]->Vz->field_cpu, vz, n);
#else
  (void)vz;
#endif
  if (cs) memcpy(Fluids[f]->Energy->field_cpu, cs, n);
}

/* the fluid's Energy field: the internal energy (ADIABATIC) or the sound
 * speed (ISOTHERMAL) */
void ref_get_energy(int f, double *e) {
  INPUT(Fluids[f]->Energy);
  memcpy(e, Fluids[f]->Energy->field_cpu, sizeof(real) * ncell());
}

void ref_get_state(int f, double *rho, double *vx, double *vy, double *vz) {
  size_t n = sizeof(real) * ncell();
  INPUT(Fluids[f]->Density);
  INPUT(Fluids[f]->Vx);
  INPUT(Fluids[f]->Vy);
#ifdef Z
  INPUT(Fluids[f]->Vz);
#endif
  if (rho) memcpy(rho, Fluids[f]->Density->field_cpu, n);
  if (vx) memcpy(vx, Fluids[f]->Vx->field_cpu, n);
  if (vy) memcpy(vy, Fluids[f]->Vy->field_cpu, n);
#ifdef Z
  if (vz) memcpy(vz, Fluids[f]->Vz->field_cpu, n);
#else
  (void)vz;
#endif
}

void ref_initialize(void) {
  /* main.c:297-316 */
  MULTIFLUID(FillGhosts(PrimitiveVariables()));
#ifdef STOCKHOLM
  init_stockholm();
#endif
}

/* One pass of the DT loop body of main.c:361-448. */
#ifdef FB_DROPIN
/* fargo3d_b200/integration/b200_hydro.c: the FARGO3D-side binding of the
 * B200 library, compiled into the reference build in place of the step's body */
void B200_HydroStep(real DT_interval, real *dt);
void B200_Sync(void);
#endif

double ref_step(double DTint) {
  real dt;
#ifdef FB_DROPIN
  B200_HydroStep(DTint, &dt);   /* attaches to the Fields on its first call */
  PhysicalTime += dt;
  Timestepcount++;
  B200_Sync();
  SelectFluid(0);
  g_last_dt = dt;
  return dt;
#endif
  if (g_dtemp >= DTint) g_dtemp = 0.0;
  DT = DTint;
#ifdef X
  MULTIFLUID(ComputeVmed(Vx));
#endif
  MULTIFLUID(cfl());
  CflFluidsMin();
  dt = StepTime;
  g_dtemp += dt;
  if (g_dtemp > DTint) dt = DTint - (g_dtemp - dt);
  Reset_field(Total_Density);
  MULTIFLUID(ComputeTotalDensity());
  MULTIFLUID(Sources(dt));
#ifdef DRAGFORCE
  Collisions(dt, 1);
#endif
#ifdef DUSTDIFFUSION
  DustDiffusion_Main(dt);   /* main.c:417-419 */
#endif
  MULTIFLUID(Transport(dt));
  PhysicalTime += dt;
  Timestepcount++;
#ifdef STOCKHOLM
  MULTIFLUID(StockholmBoundary(dt));
#endif
  MULTIFLUID(FillGhosts(PrimitiveVariables()));
  SelectFluid(0);
  g_last_dt = dt;
  return dt;
}

void ref_get_scalars(double *o) {
  o[0] = PhysicalTime; o[1] = OMEGAFRAME; o[2] = g_last_dt;
  o[3] = Sys->nb ? Sys->x[0] : 0; o[4] = Sys->nb ? Sys->y[0] : 0;
  o[5] = Sys->nb ? Sys->vx[0] : 0; o[6] = Sys->nb ? Sys->vy[0] : 0; o[7] = Domega;
}

/* output.c is compiled in for its merged writer: the writers it can select
 * that the reference build here leaves out, and its monitoring hook, are no-ops here. */
void MakeDir(char *s) { (void)s; }
void Summary(int n) { (void)n; }
void WriteVTK(Field *f, int n) { (void)f; (void)n; }
void WriteVTKMerging(Field *f, int n) { (void)f; (void)n; }

/* Fluid f's output files written by the reference's own writers: the merged
 * field files <outdir>/<fluid><field><n>.dat (WriteMerging, output.c:283-315)
 * of dens, energy, vx, vy[, vz], and, with fluid 0, the next line of every
 * planet<k>.dat (WritePlanetSystemFile, output.c:181-196).  One process:
 * CPU_Master, no offset (split.c with one rank). */
int ref_write_outputs(int f, const char *outdir, int n) {
  if (f < 0 || f >= NFLUIDS) return -1;
  CPU_Master = YES; CPU_Rank = 0; CPU_Number = 1; Y0 = 0; Z0 = 0;
  snprintf(OUTPUTDIR, sizeof OUTPUTDIR, "%s/", outdir);
  WriteMerging(Fluids[f]->Density, n);
  WriteMerging(Fluids[f]->Energy, n);
  WriteMerging(Fluids[f]->Vx, n);
  WriteMerging(Fluids[f]->Vy, n);
#ifdef Z
  WriteMerging(Fluids[f]->Vz, n);
#endif
  if (f == 0) WritePlanetSystemFile(n, NO);
  strcpy(OUTPUTDIR, "./");
  return 0;
}

void ref_get_geometry(double *xa, double *ya, double *za) {
  if (xa) memcpy(xa, Xmin, sizeof(real) * (Nx + 2 * NGHX + 1));
  if (ya) memcpy(ya, Ymin, sizeof(real) * (Ny + 2 * NGHY + 1));
  if (za) memcpy(za, Zmin, sizeof(real) * (Nz + 2 * NGHZ + 1));
}
