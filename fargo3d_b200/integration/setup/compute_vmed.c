/*
 * compute_vmed.c for a setup whose hydro step runs on a B200 (replaces
 * src/compute_vmed.c from the setup directory).
 *
 * The DT loop's ComputeVmed(Vx) (main.c:366) feeds stages that all run in
 * the library, which forms the ring means itself; while the library holds
 * the state, that call only marks the fluid's VxMed as owed, and the mean
 * is formed on the host when host code reads VxMed (INPUT2D, fresh.c of
 * this folder).  Every other call -- on a host field, or before the library
 * is attached -- computes the mean at once, as the stock function does.
 */
#include "fargo3d.h"
#include "b200_setup.h"

/* Q = V times the width of its cell in x (bound to ComputeVweight) */
void ComputeVweight_cpu(Field *V, Field *Q) {
  int i, j, k;
  INPUT(V);
  OUTPUT(Q);
  for (k = 0; k < Nz + 2 * NGHZ; k++)
    for (j = 0; j < Ny + 2 * NGHY; j++)
      for (i = 0; i < Nx + 2 * NGHX; i++)
        Q->field_cpu[l] = V->field_cpu[l] * (Xmin(i + 1) - Xmin(i));
}

void B200_HostVmed(Field *V, Field2D *out) {
  int j, k;
  ComputeVweight(V, Qs);
  reduction_SUM(Qs, 0, Ny + 2 * NGHY, 0, Nz + 2 * NGHZ);
  INPUT2D(Reduction2D);
  OUTPUT2D(out);
  for (k = 0; k < Nz + 2 * NGHZ; k++)
    for (j = 0; j < Ny + 2 * NGHY; j++)
      out->field_cpu[l2D] = Reduction2D->field_cpu[l2D] / (XMAX - XMIN);
}

void ComputeVmed(Field *V) {
  int f = B200_StateFluid(V);
  if (B200_Attached() && f >= 0 && V == Fluids[f]->Vx && VxMed == Fluids[f]->VxMed) {
    B200_SetVmedPending(f, 1);
    return;
  }
  B200_HostVmed(V, VxMed);
}
