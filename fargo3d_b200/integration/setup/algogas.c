/*
 * algogas.c for a setup whose hydro step runs on a B200 through
 * libfargo_b200 (replaces src/algogas.c from the setup directory).
 *
 * The DT loop of main.c:361-448 calls, per fluid, Sources(dt) and
 * Transport(dt) and, at the end of the step, FillGhosts.  The library
 * advances every fluid at once, so fluid 0's Sources runs the planets, the
 * source terms, the drag and the dust diffusion of every fluid
 * (B200_Advance), fluid 0's Transport runs transport, NewVelocity,
 * Stockholm damping and the ghost fill of every fluid (B200_Transport), and
 * the calls for the other fluids have nothing left to do.  FillGhosts fills
 * the host fields' ghosts as the stock function does (comm, boundaries, the
 * checks of mute dimensions) until the library holds the state -- the
 * initial fill of main.c -- and is a no-op afterwards, when the ghosts live
 * on the device.
 */
#include "fargo3d.h"
#include "b200_setup.h"

TimeProcess t_Comm;
TimeProcess t_Hydro;
TimeProcess t_Mhd;
TimeProcess t_sub1;
TimeProcess t_sub1_x;
TimeProcess t_sub1_y;
TimeProcess t_sub1_z;

#if defined(MHD) || defined(FLOOR) || defined(COLLISIONPREDICTOR) || defined(POLYTROPIC) || defined(STANDARD)
#error "libfargo_b200 runs the hydro step without MHD, FLOOR, COLLISIONPREDICTOR, POLYTROPIC or STANDARD"
#endif

static void b200_attached_or_stop(const char *who) {
  char msg[200];
  if (B200_Attached()) return;
  snprintf(msg, sizeof msg, "%s ran before cfl(): the B200 step starts with the CFL condition", who);
  prs_error(msg);
}

void FillGhosts(int var) {
  if (B200_Attached()) return;
  InitSpecificTime(&t_Comm, "MPI Communications");
  comm(var);
  GiveSpecificTime(t_Comm);
  boundaries();
#ifdef Y
  if (NY == 1) CheckMuteY();
#endif
#ifdef Z
  if (NZ == 1) CheckMuteZ();
#endif
}

void Sources(real dt) {
  b200_attached_or_stop("Sources");
  if (FluidIndex == 0) B200_Advance(dt);
}

void Transport(real dt) {
  (void)dt;
  b200_attached_or_stop("Transport");
  if (FluidIndex == 0) B200_Transport();
  if (ForwardOneStep == YES) prs_exit(EXIT_SUCCESS);
}
