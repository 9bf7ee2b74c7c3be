/*
 * fastandfourier.h -- public C API of the B200 transform path.
 *
 * This header restates, declaration for declaration, the part of the
 * FastAndFourier public API (reference: include/fastandfourier.h) that the
 * batched split-plane transform path uses, so that code written against the
 * reference compiles and links unchanged against libfaf_b200.so:
 *
 *   - every enum keeps the reference's numeric values (they are stored in
 *     faf_config / faf_transform, whose field layout is part of the ABI);
 *   - faf_config and faf_transform keep every reference field at the same
 *     offset; faf_transform gains ONE trailing field, `device_plan`, which
 *     owns all GPU state and is released by faf_destroy_transform;
 *   - FAF_BACKEND_CUDA (= 3) is the one new enum value.  AUTO resolves to
 *     CUDA in this library.  VM and JIT name the reference's CPU engines,
 *     which this library does not contain: creating with them fails.
 *
 * Additive GPU entry points (batched execute, streams, uneven batches,
 * serving, tensor-core form) are declared in faf_cuda.h.
 */
#ifndef FASTANDFOURIER_H
#define FASTANDFOURIER_H

#ifdef __cplusplus
extern "C" {
#endif

#include <stdbool.h>
#include <stddef.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef FAF_RESTRICT
#if defined(__cplusplus)
#define FAF_RESTRICT __restrict__
#else
#define FAF_RESTRICT restrict
#endif
#endif

/* Version of the reference API this header is compatible with
 * (reference include/fastandfourier.h:45-48). */
#define FASTANDFOURIER_VERSION_MAJOR 1
#define FASTANDFOURIER_VERSION_MINOR 2
#define FASTANDFOURIER_VERSION_PATCH 0
#define FASTANDFOURIER_VERSION_STRING "1.2.0"

#define FAF_ALIGN 64

/* ---- enums (reference include/fastandfourier.h:116-304) ---------------- */

typedef enum {
    FAF_PREC_FP8 = 0,
    FAF_PREC_FP16 = 1,
    FAF_PREC_BF16 = 2,
    FAF_PREC_FP32 = 3,
    FAF_PREC_FP64 = 4,
    FAF_PREC_INT8 = 5,
    FAF_PREC_INT16 = 6,
    FAF_PREC_INT32 = 7
} faf_precision;

typedef enum {
    FAF_TRANSFORM_FFT,          /* 0 */
    FAF_TRANSFORM_IFFT,         /* 1 */
    FAF_TRANSFORM_RFFT,         /* 2 */
    FAF_TRANSFORM_IRFFT,        /* 3 */
    FAF_TRANSFORM_DCT_I,
    FAF_TRANSFORM_DCT_II,
    FAF_TRANSFORM_DCT_III,
    FAF_TRANSFORM_DCT_IV,
    FAF_TRANSFORM_DST_I,
    FAF_TRANSFORM_DST_II,
    FAF_TRANSFORM_DST_III,
    FAF_TRANSFORM_DST_IV,
    FAF_TRANSFORM_STFT,         /* 12 */
    FAF_TRANSFORM_MDCT,
    FAF_TRANSFORM_IMDCT,
    FAF_TRANSFORM_HAAR,
    FAF_TRANSFORM_DAUBECHIES4,
    FAF_TRANSFORM_CDF53,
    FAF_TRANSFORM_CDF97,
    FAF_TRANSFORM_SYM4,
    FAF_TRANSFORM_PIPELINE,     /* 20 */
    FAF_TRANSFORM_CWT,
    FAF_TRANSFORM_ICWT
} faf_transform_type;

/* Wavelet-side enums are kept only because faf_config embeds them. */
typedef enum {
    FAF_WAVELET_HAAR = 0,
    FAF_WAVELET_D4,
    FAF_WAVELET_CDF53,
    FAF_WAVELET_CDF97,
    FAF_WAVELET_SYM4,
    FAF_WAVELET_COUNT
} faf_wavelet_family;

typedef enum {
    FAF_CONV_UNSPEC = 0,
    FAF_CONV_HAAR_ORTHO,
    FAF_CONV_HAAR_LAZY,
    FAF_CONV_HAAR_MEAN,
    FAF_CONV_D4_ORTHO,
    FAF_CONV_SYM4_ORTHO,
    FAF_CONV_CDF53_INT,
    FAF_CONV_CDF53_ENERGY,
    FAF_CONV_CDF97_JPEG,
    FAF_CONV_CDF97_ORTHO,
    FAF_CONV_CUSTOM_PR,
    FAF_CONV_ANALYSIS_ONLY
} faf_wavelet_convention;

typedef enum {
    FAF_DWT_BACKEND_AUTO = 0,
    FAF_DWT_BACKEND_LIFT = 1,
    FAF_DWT_BACKEND_FIR = 2
} faf_dwt_backend;

/* Buffer / spectrum layout. */
typedef enum {
    FAF_LAYOUT_DEFAULT = 0,     /* type-specific default */
    FAF_LAYOUT_SPLIT,           /* re[n], im[n]: native for C2C */
    FAF_LAYOUT_HERMITIAN,       /* R2C spectrum, n/2+1 split-plane bins */
    FAF_LAYOUT_REAL,            /* float[n] */
    FAF_LAYOUT_INTERLEAVED      /* complex float[2n] */
} faf_layout;

/* Scaling. NONE: forward unscaled, inverse 1/n (NumPy). ORTHO: 1/sqrt(n)
 * both ways. FORWARD: 1/n on the forward transform only. */
typedef enum {
    FAF_NORM_DEFAULT = 0,
    FAF_NORM_NONE,
    FAF_NORM_ORTHO,
    FAF_NORM_FORWARD,
    FAF_NORM_LAZY,
    FAF_NORM_JPEG2000
} faf_norm;

typedef enum {
    FAF_DIR_FORWARD = 0,
    FAF_DIR_INVERSE
} faf_direction;

typedef enum {
    FAF_BACKEND_AUTO = 0,       /* this library: CUDA */
    FAF_BACKEND_VM,             /* reference CPU interpreter: not in this library */
    FAF_BACKEND_JIT,            /* reference CPU JIT: not in this library */
    FAF_BACKEND_CUDA = 3        /* B200 kernels (new) */
} faf_backend;

/* ---- config and buffers (reference :372-404) -------------------------- */

typedef struct faf_config {
    size_t n;                   /* transform length (real length for R2C) */
    faf_precision precision;    /* FP32 (the GPU path is FP32) */
    faf_layout layout;
    faf_norm norm;
    faf_direction dir;
    faf_backend backend;
    uint32_t flags;

    faf_wavelet_family family;  /* DWT only; ignored */
    size_t levels;
    faf_wavelet_convention conv;
    faf_dwt_backend dwt_backend;
    int dct_type;
    size_t hop_length;          /* STFT */
    size_t win_length;          /* STFT */
} faf_config;

typedef struct faf_buffer {
    void *re;                   /* host or device pointer */
    void *im;                   /* NULL for REAL */
    size_t n;                   /* logical length (n, or n/2+1 bins) */
    faf_layout layout;
} faf_buffer;

/* ---- IR types kept for struct layout (reference :409-470) -------------- */

typedef enum {
    FAF_NOP = 0,
    FAF_LOAD,
    FAF_STORE,
    FAF_LOAD_CONST,
    FAF_BFLY2,
    FAF_BFLY4,
    FAF_BFLY8,
    FAF_TWIDDLE_MUL,
    FAF_TWIDDLE_MUL_CONJ,
    FAF_FMA,
    FAF_FMUL,
    FAF_FADD,
    FAF_FSUB,
    FAF_BARRIER,
    FAF_FFT_STAGE,
    FAF_DCT_STAGE,
    FAF_DST_STAGE,
    FAF_LIFT_PRED,
    FAF_LIFT_UPD,
    FAF_LIFT_SCALE,
    FAF_DOWN2,
    FAF_UP2,
    FAF_POLY_FIR,
    FAF_POLY_IIR,
    FAF_PERMUTE,
    FAF_SHUFFLE,
    FAF_BLEND,
    FAF_REDUCE_SUM,
    FAF_REDUCE_MAX,
    FAF_REDUCE_MIN,
    FAF_CALL_BUILTIN,           /* 30: pipeline spectral op */
    FAF_BITREV,
    FAF_DWT_STAGE,
    FAF_THRESHOLD,
    FAF_END = 255
} faf_opcode;

typedef struct {
    uint32_t packed;            /* [opcode:8][flags:8][reserved:16] */
    uint32_t a0;
    uint32_t a1;
    uint32_t a2;
} faf_inst;

typedef struct {
    void *handle;
    void *kernel_fn;
    void *native_code;
    char *so_path;
    char *c_path;
} faf_jit_cache;

/* ---- transform object (reference :475-506, plus device_plan) ----------- */

typedef struct faf_transform {
    size_t n;
    size_t n_inst;              /* pipeline: number of spectral ops in code */
    faf_inst *code;             /* pipeline: CALL_BUILTIN ops */
    void *twiddles[8];          /* host tables (unused by the GPU path) */
    size_t twiddle_sizes[8];
    faf_precision precision;
    faf_transform_type type;
    uint32_t flags;
    faf_jit_cache *jit_cache;   /* always NULL here: no CPU JIT */
    size_t hop_length;
    size_t win_length;
    size_t levels;
    faf_wavelet_family family;
    faf_config cfg;             /* resolved create-time configuration */
    void *scratch;              /* host staging (pinned) for host buffers */
    size_t scratch_size;
    int (*execute_func)(const struct faf_transform *t, void *out_re, void *out_im,
                        const void *in_re, const void *in_im);
    struct faf_transform *inner;     /* R2C / pipeline forward part */
    struct faf_transform *inner_inv; /* pipeline inverse part */
    void *user_aux;             /* bound spectrum re[] (mul-spectrum) */
    void *user_aux_im;          /* bound spectrum im[] */
    size_t user_aux_n;          /* bound spectrum length (bins) */
    const float *custom_h;
    const float *custom_g;
    const float *custom_ht;
    const float *custom_gt;
    int custom_len_hg;
    int custom_len_syn;
    void *device_plan;          /* NEW: GPU plan, owned by the transform */
} faf_transform;

/* Transform flags stored in faf_transform.flags / faf_config.flags. */
#define FAF_FLAG_INVERSE 0x0001u
#define FAF_FLAG_REAL 0x0008u
#define FAF_FLAG_JIT_INPLACE 0x0100u
#define FAF_FLAG_JIT_SIMD 0x0200u
#define FAF_FLAG_JIT_SPLIT_PLANE 0x0400u
/* Opt-in Bluestein for sizes that are not 5-smooth / codelet / Rader. */
#define FAF_FLAG_BLUESTEIN (1u << 12)
/* Opt-in create-time measurement: here it runs the launch-shape autotuner. */
#define FAF_FLAG_MEASURE (1u << 13)

/* ---- library lifecycle -------------------------------------------------- */

int faf_init(void);
void faf_cleanup(void);
const char *faf_version(void);
const char *faf_arch_name(void);

static inline void *faf_aligned_alloc(size_t size) {
    void *p = NULL;
    if (size == 0) return NULL;
    if (posix_memalign(&p, 64, (size + 63u) & ~(size_t)63u) != 0) return NULL;
    return p;
}

static inline void faf_aligned_free(void *ptr) { free(ptr); }

/* ---- config helpers (reference :596-657) ------------------------------- */

static inline faf_config faf_config_init(size_t n) {
    faf_config c;
    memset(&c, 0, sizeof c);
    c.n = n;
    c.precision = FAF_PREC_FP32;
    return c;
}

static inline faf_config faf_config_from(const faf_transform *t) {
    faf_config c;
    memset(&c, 0, sizeof c);
    return t ? t->cfg : c;
}

static inline faf_config faf_config_inverse(faf_config cfg) {
    cfg.dir = (cfg.dir == FAF_DIR_INVERSE) ? FAF_DIR_FORWARD : FAF_DIR_INVERSE;
    return cfg;
}

static inline faf_buffer faf_buffer_real(void *data, size_t n) {
    faf_buffer b;
    memset(&b, 0, sizeof b);
    b.re = data;
    b.n = n;
    b.layout = FAF_LAYOUT_REAL;
    return b;
}

static inline faf_buffer faf_buffer_split(void *re, void *im, size_t n) {
    faf_buffer b;
    memset(&b, 0, sizeof b);
    b.re = re;
    b.im = im;
    b.n = n;
    b.layout = FAF_LAYOUT_SPLIT;
    return b;
}

static inline faf_buffer faf_buffer_interleaved(void *data, size_t n) {
    faf_buffer b;
    memset(&b, 0, sizeof b);
    b.re = data;
    b.n = n;
    b.layout = FAF_LAYOUT_INTERLEAVED;
    return b;
}

static inline faf_buffer faf_buffer_hermitian(void *re, void *im, size_t n_bins) {
    faf_buffer b;
    memset(&b, 0, sizeof b);
    b.re = re;
    b.im = im;
    b.n = n_bins;
    b.layout = FAF_LAYOUT_HERMITIAN;
    return b;
}

const char *faf_layout_name(faf_layout layout);
const char *faf_norm_name(faf_norm norm);
size_t faf_spectrum_len(const faf_transform *t);

/* ---- create / destroy --------------------------------------------------- */

/* Any supported type from one config (reference src/faf_core.c:1034). */
faf_transform *faf_create(faf_transform_type type, const faf_config *cfg);
/* C2C. Legal n: 5-smooth, codelet (2..10, 12), Rader prime (n >= 11 prime,
 * n-1 7-smooth); anything else needs FAF_FLAG_BLUESTEIN. */
faf_transform *faf_create_fft(const faf_config *cfg);
/* R2C (dir FORWARD) or C2R (dir INVERSE); n even and 5-smooth. */
faf_transform *faf_create_rfft(const faf_config *cfg);
/* STFT: Hann window of win_length (default n), hop (default win/4). */
faf_transform *faf_create_stft(const faf_config *cfg);
/* The inverse of fwd with every other knob inherited. */
faf_transform *faf_create_inverse(const faf_transform *fwd);
void faf_destroy_transform(faf_transform *t);

/* ---- execute ------------------------------------------------------------ */

/* Execute one transform.  Buffers may be host or device pointers (detected
 * per call).  Host buffers: synchronous, staged through pinned memory.
 * Device buffers: enqueued on the transform's stream; synchronous unless a
 * stream was set with faf_cuda_set_stream (then the caller synchronises). */
int faf_execute(const faf_transform *t, faf_buffer *out, const faf_buffer *in);

int faf_deinterleave_f32(float *FAF_RESTRICT re, float *FAF_RESTRICT im,
                         const float *FAF_RESTRICT interleaved, size_t n);
int faf_interleave_f32(float *FAF_RESTRICT interleaved, const float *FAF_RESTRICT re,
                       const float *FAF_RESTRICT im, size_t n);
int faf_deinterleave_f64(double *FAF_RESTRICT re, double *FAF_RESTRICT im,
                         const double *FAF_RESTRICT interleaved, size_t n);
int faf_interleave_f64(double *FAF_RESTRICT interleaved, const double *FAF_RESTRICT re,
                       const double *FAF_RESTRICT im, size_t n);

/* Packed Hermitian multiply on n_bins split-plane bins: DC and the last bin
 * are real multiplies with imaginary part 0 (reference src/faf_core.c:150). */
void faf_herm_mul_f32(float *yr, float *yi, const float *xr, const float *xi,
                      const float *hr, const float *hi, size_t n_bins);
void faf_herm_mul_f64(double *yr, double *yi, const double *xr, const double *xi,
                      const double *hr, const double *hi, size_t n_bins);
void faf_herm_mul_conj_f32(float *yr, float *yi, const float *xr, const float *xi,
                           const float *hr, const float *hi, size_t n_bins);
void faf_herm_mul_conj_f64(double *yr, double *yi, const double *xr, const double *xi,
                           const double *hr, const double *hi, size_t n_bins);

/* ---- utilities ---------------------------------------------------------- */

size_t faf_get_alignment(void);
size_t faf_get_recommended_size(faf_transform_type type, size_t min_size);
bool faf_is_size_supported(faf_transform_type type, size_t n);
size_t faf_precision_size(faf_precision prec);
const char *faf_precision_name(faf_precision prec);
const char *faf_transform_name(faf_transform_type type);

/* ---- errors: thread-local message, 0 / -1 / NULL returns ---------------- */

const char *faf_get_error(void);
void faf_clear_error(void);
void faf_set_error(const char *fmt, ...);

#ifdef __cplusplus
}
#endif

#endif /* FASTANDFOURIER_H */
