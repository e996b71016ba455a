/*
 * cfl.c for a setup whose hydro step runs on a B200 through libfargo_b200
 * (replaces src/cfl.c from the setup directory).  ChangeArch binds cfl to
 * cfl_cpu (change_arch.c:62); the DT loop calls it once per fluid and
 * CflFluidsMin then takes the minimum of Min[] (cfl_fluids_min.c:3-22).
 * The library computes every fluid's CFL limit in one pass, so fluid 0
 * carries the minimum over all fluids and the others stay out of the way.
 */
#include "fargo3d.h"
#include "b200_setup.h"

void cfl_cpu(void) {
  Min[FluidIndex] = FluidIndex == 0 ? B200_Begin() : 1e30;
}
