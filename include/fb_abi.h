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

/* per-member states of a batch (fb_batch_poll) */
#define FB_DONE 1            /* reached its end time (fb_batch_add) */
#define FB_SLOT_EMPTY 2      /* no disk in this slot */
#define FB_SLOT_RESERVED 3   /* disk created, not yet activated */

/* request states of a server (fb_server_status) */
#define FB_REQ_QUEUED 0
#define FB_REQ_RUNNING 1
#define FB_REQ_DONE 2
#define FB_REQ_FAILED 3

#endif
