/*
 * afd_lms.h - LMS impulse-response estimation on the GPU.
 *
 * Replaces EstimateIr of anc_field_py/ancutil.py:24-37, the reference's
 * identification of an impulse response from a source signal x and a
 * receiver recording d (examples/ie224-noise.py:61,90, dsp.py:48,
 * identification.py:36,54): `epochs` passes of sample-serial LMS with step
 * size mu over the first min(nx, nd) samples, the delay line cleared at the
 * start of each pass and the weights kept, all in FP64. The GPU evaluates
 * the same recursion in blocks of 128 samples (exact up to the order of
 * floating-point additions).
 */
#ifndef AFD_LMS_H
#define AFD_LMS_H

#include <stdint.h>

#include "afd.h"

#ifdef __cplusplus
extern "C" {
#endif

/* w[taps] (host) = the estimate; x, d host arrays. The reference's default
 * is epochs = 16. Returns AFD_OK or AFD_ERR_*. */
int afd_lms_estimate(const double* x, int64_t nx, const double* d, int64_t nd, int32_t taps, double mu,
                     int32_t epochs, int32_t device, double* w);
const char* afd_lms_last_error(void);

#ifdef __cplusplus
}
#endif

#endif
