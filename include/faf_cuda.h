/*
 * faf_cuda.h -- additive GPU entry points of the B200 transform path.
 *
 * Nothing here replaces a reference symbol; everything is new ABI that a
 * GPU-aware caller may use on top of fastandfourier.h:
 *
 *   - streams: faf_cuda_set_stream / faf_cuda_synchronize
 *   - batched execute: many transforms of one plan in one launch
 *
 * Pointers are plain `void *` / `float *` so the header needs no CUDA
 * include; a `void *stream` is a cudaStream_t.
 */
#ifndef FAF_CUDA_H
#define FAF_CUDA_H

#include "fastandfourier.h"

#ifdef __cplusplus
extern "C" {
#endif

/* ---- library / device --------------------------------------------------- */

/* 1 if a CUDA device is usable, 0 otherwise (message in faf_get_error()). */
int faf_cuda_available(void);
/* Name of the plan kind behind t ("c2c", "rader", "bluestein", "r2c", "c2r",
 * "pipeline", "stft", "c2c-4step", ...), or NULL. */
const char *faf_cuda_plan_kind(const faf_transform *t);
/* Number of kernel launches the last execute on this thread made. */
int faf_cuda_last_launches(void);

/* ---- streams ------------------------------------------------------------ */

/* Enqueue this transform's work on `stream` (a cudaStream_t).  With a stream
 * set, faf_execute on device buffers returns without synchronising.  NULL
 * restores the default (legacy stream, synchronous execute). */
int faf_cuda_set_stream(faf_transform *t, void *stream);
void *faf_cuda_get_stream(const faf_transform *t);
int faf_cuda_synchronize(const faf_transform *t);

/* ---- batched execute ------------------------------------------------------ */

/* Run `batch` transforms of plan t.  Transform b reads in->re + b*in_dist
 * (and in->im + b*in_dist) and writes out->re + b*out_dist (...), distances
 * counted in elements of one plane (complex elements for INTERLEAVED).
 * A distance of 0 means "packed": the buffer's own logical length n.
 * in / out describe ONE transform (same validation as faf_execute).
 * Buffers are all device or all host memory; host buffers are copied in and
 * out inside the call. */
int faf_execute_batched(const faf_transform *t, faf_buffer *out, const faf_buffer *in,
                        size_t batch, size_t in_dist, size_t out_dist);

#ifdef __cplusplus
}
#endif

#endif /* FAF_CUDA_H */
