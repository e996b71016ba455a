/*
 * b200_setup.h -- what the setup-directory files of this folder call in
 * b200_hydro.c.  The folder is copied into a FARGO3D setup directory
 * (setups/<setup>/), whose files FARGO3D's makefile finds before the stock
 * ones of src/ (VPATH, src/makefile:306); see b200_hydro.c for the protocol.
 */
#ifndef B200_SETUP_H
#define B200_SETUP_H

int B200_Attached(void);
int B200_StateFluid(const Field *f);
int B200_VmedFluid(const Field2D *f);
void B200_InputFluid(int fluid);
void B200_OutputFluid(int fluid);
int B200_VmedPending(int fluid);
void B200_SetVmedPending(int fluid, int pending);
real B200_Begin(void);
void B200_Advance(real dt);
void B200_Transport(void);
void B200_Sync(void);

/* azimuthal mean of V into out (ComputeVmed's arithmetic: the sum of
 * V dx over the ring over XMAX - XMIN; compute_vmed.c) */
void B200_HostVmed(Field *V, Field2D *out);

#endif
