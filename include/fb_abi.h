/*
 * fb_abi.h -- constants shared by the C-ABI header and the device code.
 */
#ifndef FB_ABI_H
#define FB_ABI_H

#define FB_MAXPLANETS 8
#define FB_MAXFLUIDS 8

/* precision of a disk's fields and arithmetic */
#define FB_FP64 0
#define FB_FP32 1

/* frame of reference (std/stdpar.par "Frame": F fixed, C corotating, G guiding centre) */
#define FB_FRAME_FIXED 0
#define FB_FRAME_COROT 1
#define FB_FRAME_GUIDING 2

/* status codes returned by every fb_* entry point */
#define FB_OK 0
#define FB_ERR_ARG -1        /* invalid argument / unsupported configuration */
#define FB_ERR_CUDA -2       /* a CUDA call failed */
#define FB_ERR_NULL_DT -3    /* time step <= SMALLTIME (cfl_fluids_min.c:18-21) */
#define FB_ERR_NONFINITE -4  /* NaN or non-positive density detected */
#define FB_ERR_NOMEM -5      /* device allocation failed */
#define FB_ERR_TOO_LARGE -6  /* request exceeds a fixed capacity */

#endif
