/*
 * chirp.h -- the Chirp entry points of the B200 transform path.
 *
 * Restates the reference's Chirp API (reference include/chirp.h) for the
 * forms that emit transforms on this path: standalone (fft)/(ifft)/(rfft)/
 * (irfft) and the fused pipeline
 *     (pipeline (rfft :size N [:norm ..]) OP... (irfft))
 * with OP one of conj, (mul-spectrum), (bandpass :lo A :hi B),
 * (spectral NAME).  chirp_compile returns the same faf_transform * shape as
 * the reference (type FAF_TRANSFORM_PIPELINE, inner = forward R2C,
 * inner_inv = inverse, code[] = FAF_CALL_BUILTIN ops with the reserved
 * CHIRP_OP_* codes in a0).
 *
 * Built-in ops run inside the fused GPU kernel.  A host (spectral NAME)
 * callback cannot run on the device: such a pipeline executes as R2C kernel
 * -> host callback -> C2R kernel (a host round trip), unless NAME was
 * registered as a device op with chirp_register_spectral_device().
 */
#ifndef CHIRP_H
#define CHIRP_H

#include "fastandfourier.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    CHIRP_KIND_UNARY = 0,
    CHIRP_KIND_OTHER = 1,
    CHIRP_KIND_COMPLEX,
    CHIRP_KIND_VECTOR,
    CHIRP_KIND_SPECTRAL,        /* void(re, im, n_bins, ctx) split-plane */
    CHIRP_KIND_HERMITIAN        /* SPECTRAL, then DC/Nyquist imag forced to 0 */
} chirp_kind;

typedef void (*chirp_spectral_fn)(float *re, float *im, size_t n_bins, void *ctx);
typedef void (*chirp_spectral_fn_f64)(double *re, double *im, size_t n_bins, void *ctx);

/* Reserved CALL_BUILTIN.a0 values (reference include/chirp.h:36-38). */
#define CHIRP_OP_CONJ 0x7ffffffdu
#define CHIRP_OP_MUL 0x7ffffffeu
#define CHIRP_OP_BANDPASS 0x7fffffffu

/* Register a host split-plane spectral callback; returns its index >= 0. */
int chirp_register_spectral(const char *name, chirp_spectral_fn fn, void *ctx);
int chirp_register_spectral_ex(const char *name, chirp_spectral_fn f32,
                               chirp_spectral_fn_f64 f64, void *ctx);
int chirp_builtin_kind(int idx);
void *chirp_builtin_ctx(int idx);
const char *chirp_builtin_name(int idx);
int chirp_count(void);

/* Device spectral ops.  No counterpart in the reference, whose
 * (spectral NAME) always calls a host function.  A name registered here runs
 * inside the fused GPU pipeline kernel, with no host round trip; if the same
 * pipeline also holds a host callback, every op of it runs on the host, this
 * one included.  Registering a name replaces an earlier host or device
 * registration of that name; returns its index >= 0, or -1. */
typedef enum {
    CHIRP_DEVICE_GAIN = 0,     /* every bin times p0 (real) */
    CHIRP_DEVICE_PHASE = 1,    /* every bin times exp(i p0), p0 in radians */
    CHIRP_DEVICE_DELAY = 2,    /* bin k times exp(-2 pi i k p0 / n): circular delay by
                                  p0 samples (n = the pipeline's length) */
    CHIRP_DEVICE_LOWPASS = 3,  /* bins k > p0 set to 0 */
    CHIRP_DEVICE_HIGHPASS = 4  /* bins k < p0 set to 0 */
} chirp_device_op;
int chirp_register_spectral_device(const char *name, chirp_device_op op, double p0);

/* Bind the auxiliary spectrum "H" (also "mul-spectrum" / "kernel") used by
 * (mul-spectrum).  re/im may be host or device memory, caller-owned, and
 * must outlive execution; host memory is read at every execute. */
int chirp_bind(faf_transform *t, const char *name, void *re, void *im, size_t n_bins);

/* Apply one CALL_BUILTIN / reserved op to host split-plane bins. */
void chirp_apply_split_f32(const faf_transform *t, uint32_t a0, uint32_t a1, uint32_t a2,
                           float *re, float *im, size_t n);

/* Reset the registry (device op registrations included). */
void chirp_cleanup(void);

/* Compile a Chirp S-expression to a transform (NULL + faf_get_error()). */
faf_transform *chirp_compile(const char *source);

#ifdef __cplusplus
}
#endif

#endif /* CHIRP_H */
