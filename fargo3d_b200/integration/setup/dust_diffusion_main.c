/*
 * dust_diffusion_main.c for a setup whose hydro step runs on a B200
 * (replaces src/dust_diffusion_main.c from the setup directory).  The
 * library applies the dust diffusion of every dust fluid inside the step's
 * source part (B200_Advance, called from fluid 0's Sources), after the drag,
 * where main.c:417-419 calls DustDiffusion_Main; this call has nothing left
 * to do.
 */
#include "fargo3d.h"
#include "b200_setup.h"

void DustDiffusion_Main(real dt) {
  (void)dt;
  if (Fluids[0]->Fluidtype != GAS) {
    mastererr("ERROR - dust diffusion needs Fluids[0] to be the gas.\n");
    prs_exit(1);
  }
  if (!B200_Attached()) prs_error("DustDiffusion_Main ran before cfl(): the B200 step starts with the CFL condition");
}
