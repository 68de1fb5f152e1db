// Status codes shared by the C-ABI and the kernels (mirrored in
// include/cress_b200.h).
#pragma once

#define CRESS_OK 0
#define CRESS_E_ARG 1          /* bad argument (null pointer, bad size) */
#define CRESS_E_UNSUPPORTED 2  /* option combination not implemented on the GPU */
#define CRESS_E_CUDA 3         /* a CUDA runtime call failed */
#define CRESS_E_NONUNIFORM 4   /* base state not horizontally uniform */
#define CRESS_E_NONFINITE 5    /* NaN/Inf detected in the prognostic state */
#define CRESS_E_TIMEOUT 6      /* a bounded device-side wait gave up */
#define CRESS_E_STATE 7        /* call out of order (e.g. step before base state) */
