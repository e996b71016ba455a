/*
 * fresh.c for a setup whose hydro step runs on a B200 through libfargo_b200
 * (replaces src/fresh.c from the setup directory).
 *
 * FARGO3D's host code announces what it reads and writes: INPUT(f) before
 * reading a Field, OUTPUT(f) before writing one (define.h:572-573), and the
 * stock functions here keep a Field's host and device copies coherent for
 * FARGO3D's own GPU build.  With the library the device copy of every
 * fluid's Density, Vx, Vy, Vz and Energy lives in libfargo_b200, so:
 *
 *   INPUT(f) of a state field      copies its fluid back from the B200 when
 *                                  the device is ahead (outputs, monitors)
 *   OUTPUT(f) of a state field     marks its fluid for upload before the
 *                                  next step (restarts, setup hooks)
 *   INPUT2D(VxMed)                 forms a ring mean that ComputeVmed(Vx)
 *                                  deferred (compute_vmed.c of this folder)
 *
 * The storage-ownership checks of the stock INPUT (a Field whose storage was
 * lent to a temporary, CreateFieldAlias) are kept.  FARGO3D's own GPU build
 * is not used together with the library: its _GPU entry points stop the run.
 */
#include "fargo3d.h"
#include "b200_setup.h"

static void b200_no_fargo_gpu(const char *who, int line, const char *file) {
  char msg[300];
  snprintf(msg, sizeof msg, "%s (line %d of %s): FARGO3D's own GPU build is not used with libfargo_b200", who,
           line, file);
  prs_error(msg);
}

static void b200_mark(Field *field, int line, const char *file, boolean host_fresh) {
  int s;
  field->line_origin = line;
  strncpy(field->file_origin, file, MAXLINELENGTH - 1);
  field->fresh_cpu = host_fresh;
  field->fresh_gpu = !host_fresh;
  for (s = 0; s < 4; s++) {
    field->fresh_inside_contour_cpu[s] = field->fresh_outside_contour_cpu[s] = host_fresh;
    field->fresh_inside_contour_gpu[s] = field->fresh_outside_contour_gpu[s] = !host_fresh;
  }
  *(field->owner) = field;
}

void Input_CPU(Field *field, int line, const char *file) {
  if (*(field->owner) != field) {
    if (*(field->owner) == NULL)
      printf("Error! Field %s is read at line %d of %s, but its storage was taken as a temporary at line %d of %s\n",
             field->name, line, file, field->line_origin, field->file_origin);
    else
      printf("Error! Field %s is read at line %d of %s, but its storage holds %s since line %d of %s\n",
             field->name, line, file, (*(field->owner))->name, (*(field->owner))->line_origin,
             (*(field->owner))->file_origin);
    prs_exit(EXIT_FAILURE);
  }
  B200_InputFluid(B200_StateFluid(field));
}

void Output_CPU(Field *field, int line, const char *file) {
  b200_mark(field, line, file, YES);
  B200_OutputFluid(B200_StateFluid(field));
}

void Input2D_CPU(Field2D *field, int line, const char *file) {
  int f = B200_VmedFluid(field);
  (void)line; (void)file;
  if (B200_VmedPending(f)) {
    B200_SetVmedPending(f, 0);
    B200_InputFluid(f);
    B200_HostVmed(Fluids[f]->Vx, field);
  }
}

void Output2D_CPU(Field2D *field, int line, const char *file) {
  (void)line; (void)file;
  B200_SetVmedPending(B200_VmedFluid(field), 0);
  field->fresh_cpu = YES;
  field->fresh_gpu = NO;
}

void Input2DInt_CPU(FieldInt2D *field, int line, const char *file) { (void)field; (void)line; (void)file; }

void Output2DInt_CPU(FieldInt2D *field, int line, const char *file) {
  (void)line; (void)file;
  field->fresh_cpu = YES;
  field->fresh_gpu = NO;
}

void Draft(Field *field, int line, const char *file) {
  *(field->owner) = NULL;
  strncpy(field->file_origin, file, MAXLINELENGTH - 1);
  field->line_origin = line;
}

void Input_GPU(Field *f, int line, const char *file) { (void)f; b200_no_fargo_gpu("Input_GPU", line, file); }
void Output_GPU(Field *f, int line, const char *file) { (void)f; b200_no_fargo_gpu("Output_GPU", line, file); }
void Input2D_GPU(Field2D *f, int line, const char *file) { (void)f; b200_no_fargo_gpu("Input2D_GPU", line, file); }
void Output2D_GPU(Field2D *f, int line, const char *file) { (void)f; b200_no_fargo_gpu("Output2D_GPU", line, file); }
void Input2DInt_GPU(FieldInt2D *f, int line, const char *file) {
  (void)f;
  b200_no_fargo_gpu("Input2DInt_GPU", line, file);
}
void Output2DInt_GPU(FieldInt2D *f, int line, const char *file) {
  (void)f;
  b200_no_fargo_gpu("Output2DInt_GPU", line, file);
}

/* every fluid's host copy made current (the stock functions copy every Field
 * between host and device in FARGO3D's GPU build) */
void send2cpu(void) { B200_Sync(); }
void send2gpu(void) {}
void SynchronizeHD(void) { B200_Sync(); }

void WhereIsField(Field *field) {
  if (field->fresh_cpu) printf("Field %s is fresh on the CPU 0\n", field->name);
  if (B200_StateFluid(field) >= 0 && B200_Attached()) printf("Field %s is held by the B200\n", field->name);
}

void WhereIsFieldInt2D(FieldInt2D *field) {
  if (field->fresh_cpu) printf("Field %s is fresh on the CPU 0\n", field->name);
}

void WhoOwns(Field *field) { printf("Field %s is currently storing %s\n", field->name, (*(field->owner))->name); }

void WhereIsWho(void) {}
