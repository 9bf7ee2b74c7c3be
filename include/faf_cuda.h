/*
 * faf_cuda.h -- additive GPU entry points of the B200 transform path.
 *
 * Nothing here replaces a reference symbol; everything is new ABI that a
 * GPU-aware caller may use on top of fastandfourier.h:
 *
 *   - streams: faf_cuda_set_stream / faf_cuda_synchronize
 *   - batched execute: many transforms of one plan in one launch
 *   - uneven batches: transforms of different lengths in one persistent,
 *     CUDA-graph-captured launch (faf_uneven_*)
 *   - the tensor-core precision form of C2C (FAF_FLAG_TENSOR_CORE)
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

/* ---- flags (bits >= 16: no overlap with the reference's FAF_FLAG_*) ------- */

/* faf_create_fft: run the radix-16 stages of a power-of-two C2C (256 ..
 * 16384 points) as FP16 tensor-core MMAs with hi + lo split operands and FP32
 * accumulation (FP32-level accuracy).  Other sizes ignore the flag. */
#define FAF_FLAG_TENSOR_CORE (1u << 16)

/* ---- library / device --------------------------------------------------- */

/* 1 if a CUDA device is usable, 0 otherwise (message in faf_get_error()). */
int faf_cuda_available(void);
/* Name of the plan kind behind t ("c2c", "rader", "bluestein", "r2c", "c2r",
 * "pipeline", "stft", "c2c-4step", the tensor-core forms "c2c-tc" (radix-16
 * stages) and "c2c-tc64" (64-point DFTs), ...), or NULL. */
const char *faf_cuda_plan_kind(const faf_transform *t);
/* Tensor-core plans: 0 if every MMA wait of this plan's launches so far
 * completed, 1 if one ran out of its bound (the results are then invalid);
 * -1 if t is not a tensor-core plan.  Synchronises the plan's stream. */
int faf_cuda_tc_status(const faf_transform *t);
/* 0 if every bounded wait of this transform's kernels so far completed (the
 * input ring's copy waits, tensor-core MMA waits), 1 if one ran out (the
 * results of that launch are then invalid), -1 on error.  Synchronises the
 * transform's stream. */
int faf_cuda_wait_status(const faf_transform *t);
/* Number of kernel launches the last execute on this thread made. */
int faf_cuda_last_launches(void);

/* ---- streams ------------------------------------------------------------ */

/* Enqueue this transform's work on `stream` (a cudaStream_t).  With a stream
 * set, faf_execute on device buffers returns without synchronising.  NULL
 * restores the default (legacy stream, synchronous execute); to enqueue on
 * the legacy stream without synchronising, pass cudaStreamLegacy. */
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

/* ---- inverse STFT ----------------------------------------------------------- */

/* No counterpart in the reference (its faf_create_inverse of an STFT returns
 * another forward STFT, src/faf_core.c:1122).  cfg: n (even, 5-smooth),
 * win_length (default n), hop_length (default win/4), 0 < hop <= win <= n.
 * faf_execute / faf_execute_batched take HERMITIAN split frames F x (n/2+1)
 * and write a REAL signal of (F - 1) * hop + win samples: each frame's
 * inverse real FFT (1/n scaled) times the same symmetric Hann window as the
 * forward STFT, overlap-added and divided by the summed squared window
 * (0 where that sum is below 1e-10).  Batched signals must be packed. */
faf_transform *faf_cuda_create_istft(const faf_config *cfg);

/* ---- CWT filter bank -------------------------------------------------------- */

/* Replaces the execute of faf_create_cwt (include/fastandfourier.h:774;
 * src/faf_cwt.c:769-847).  The reference builds its bank on the host at
 * create; this transform takes the bank's rows: n_rows rows of n/2+1 real
 * bin weights, psi_stride floats apart (host or device pointer, copied at
 * create), row 0 = the lowpass phi when the bank has one, then the wavelets
 * coarse to fine, as the reference bank stores them (faf_cwt_phi_f32 /
 * faf_cwt_psi_f32).  n even and 5-smooth, n <= 32768.  faf_execute /
 * faf_execute_batched: REAL x[n] -> REAL W[n_rows * n], row r =
 * irfft(rfft(x) * psi_r) with 1/n on the inverse (the reference's NONE norm).
 * The transform's user_aux_n holds n_rows, as the reference's does. */
faf_transform *faf_cuda_create_cwt(size_t n, size_t n_rows, const float *psi,
                                   size_t psi_stride);

/* Replace the execute of faf_create_icwt (include/fastandfourier.h:783;
 * src/faf_cwt.c:849-985).  faf_execute / faf_execute_batched: REAL W[n_rows
 * * n] -> REAL x[n]; batched coefficient sets must be packed.
 *   _dual: x = irfft(sum_r rfft(W_r) * dual_r), DC / Nyquist imaginary parts
 *          zeroed, 1/n on the inverse; dual: the bank's dual rows (the
 *          reference's psi_r / (sum_r psi_r^2 + eps), n/2+1 weights per row,
 *          dual_stride floats apart, host or device pointer).
 *   _l1:   x = (sum over the wavelet rows of W_r * dlog) / C, plus row 0
 *          when has_lowpass; dlog = ln 2 / voices, C the bank report's
 *          admissibility_C (C <= 0 is taken as 1). */
faf_transform *faf_cuda_create_icwt_dual(size_t n, size_t n_rows, const float *dual,
                                         size_t dual_stride);
faf_transform *faf_cuda_create_icwt_l1(size_t n, size_t n_rows, int has_lowpass, double dlog,
                                       double C);

/* ---- uneven batches (one persistent launch) ------------------------------- */

typedef struct faf_uneven faf_uneven;

/* Plan `count` C2C transforms of the given lengths, each a legal
 * faf_create_fft size <= 65536 (5-smooth, codelet or Rader prime).  cfg gives
 * dir / norm / flags (n is ignored); FAF_FLAG_TENSOR_CORE puts the power-of-two
 * lengths 256..16384 on the tensor-core precision form; FAF_FLAG_MEASURE runs the launch-shape
 * autotuner on the plan's own workload.  Layout: split planes, ragged and
 * packed -- transform i starts at element offset sum_{j<i} lengths[j]. */
faf_uneven *faf_uneven_create(const size_t *lengths, size_t count, const faf_config *cfg);
/* All transforms in one persistent launch (CUDA-graph replay while the
 * device pointers stay the same).  Device buffers; synchronous unless a
 * stream was set. */
int faf_uneven_execute(faf_uneven *u, float *out_re, float *out_im, const float *in_re,
                       const float *in_im);
/* Reference GPU method: one batched launch per run of equal lengths. */
int faf_uneven_execute_plain(faf_uneven *u, float *out_re, float *out_im, const float *in_re,
                             const float *in_im);
int faf_uneven_set_stream(faf_uneven *u, void *stream);
size_t faf_uneven_total(const faf_uneven *u); /* total complex elements */
void faf_uneven_destroy(faf_uneven *u);

/* ---- allocation-free four-step C2C ----------------------------------------- */

/* No counterpart in the reference.  Runs `batch` packed C2C transforms of
 * plan t (a C2C plan longer than 16384 points, i.e. the four-step path, up to
 * 65536) on device buffers without allocating any memory.  It is meant for
 * callers that must not allocate while they run: a real-time callback that
 * cannot wait inside the driver's allocator, or a program whose device memory
 * is fully reserved by another allocator so that a cudaMalloc would fail.
 * The four-step scratch is a fixed 16 MiB array per GPU, held until process
 * exit.  Creating a four-step C2C plan on a GPU places that array there (it
 * loads the array's module, and the kernels' modules, which CUDA's default
 * lazy module loading would otherwise do at the first call) and looks up its
 * device address, so plan creation is where the allocation happens and the
 * calls allocate nothing.  Power-of-two lengths run in chunks of
 * 16 MiB / (8 n) transforms on the regular two-pass kernels; other lengths
 * run one transform per CTA on at most 16 MiB / (8 n) CTAs.  A length whose
 * per-transform scratch would exceed the array, host buffers and other plan
 * kinds are rejected with an error.  All calls on a GPU share that array:
 * launches that overlap on the GPU race and must be serialised by the caller.
 * Stream and synchronisation rules are those of faf_execute. */
int faf_cuda_execute_c2c_noalloc(const faf_transform *t, float *out_re, float *out_im,
                                 const float *in_re, const float *in_im, size_t batch);

#ifdef __cplusplus
}
#endif

#endif /* FAF_CUDA_H */
