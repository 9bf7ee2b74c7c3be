// faf_api.cpp -- the C ABI of the B200 transform path.
//
// Restates the reference's public entry points for this path (create /
// execute / inverse / destroy, size policy, errors, Hermitian helpers) with
// the same names, argument meaning, validation and error behaviour, and
// routes execution to the GPU plans of faf_plan.cu.  There is no CPU engine
// behind these functions: a transform whose device plan cannot be built is
// not created (NULL + faf_get_error()), and every execute runs kernels.
#include <cuda_runtime.h>

#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "chirp.h"
#include "faf_api_internal.h"
#include "faf_cuda.h"
#include "faf_plan.h"
#include "fastandfourier.h"

using fafp::DevicePlan;
using fafp::Kind;

// ---------------------------------------------------------------------------
// Errors: thread-local message (reference src/faf_core.c:23,70-90)
// ---------------------------------------------------------------------------

static thread_local char g_err[512];
static thread_local int g_last_launches;

extern "C" const char* faf_get_error(void) { return g_err; }
extern "C" int faf_cuda_last_launches(void) { return g_last_launches; }
extern "C" void faf_clear_error(void) { g_err[0] = '\0'; }
extern "C" void faf_set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
}

namespace fafapi {

int fail(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof g_err, fmt, ap);
    va_end(ap);
    return -1;
}

int cuda_fail(cudaError_t e, const char* what) {
    cudaGetLastError();
    return fail("%s: CUDA error %d (%s)", what, (int)e, cudaGetErrorString(e));
}

void note_launches(int k) { g_last_launches = k; }

DevicePlan* plan_of(const faf_transform* t) { return t ? (DevicePlan*)t->device_plan : nullptr; }

// 1 = device-accessible memory, 0 = host memory.
int ptr_is_device(const void* p) {
    if (!p) return 0;
    cudaPointerAttributes a;
    cudaError_t e = cudaPointerGetAttributes(&a, p);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? 1 : 0;
}

cudaStream_t stream_of(DevicePlan* p) { return p->stream; }

}  // namespace fafapi

using namespace fafapi;

// ---------------------------------------------------------------------------
// Library lifecycle and names
// ---------------------------------------------------------------------------

extern "C" int faf_init(void) {
    faf_clear_error();
    return 0;
}

extern "C" void faf_cleanup(void) {}

extern "C" const char* faf_version(void) { return FASTANDFOURIER_VERSION_STRING; }

extern "C" const char* faf_arch_name(void) { return "cuda-sm_100a"; }

extern "C" size_t faf_get_alignment(void) { return FAF_ALIGN; }

extern "C" const char* faf_layout_name(faf_layout l) {
    switch (l) {
    case FAF_LAYOUT_DEFAULT: return "default";
    case FAF_LAYOUT_SPLIT: return "split";
    case FAF_LAYOUT_HERMITIAN: return "hermitian";
    case FAF_LAYOUT_REAL: return "real";
    case FAF_LAYOUT_INTERLEAVED: return "interleaved";
    }
    return "unknown";
}

extern "C" const char* faf_norm_name(faf_norm n) {
    switch (n) {
    case FAF_NORM_DEFAULT: return "default";
    case FAF_NORM_NONE: return "none";
    case FAF_NORM_ORTHO: return "ortho";
    case FAF_NORM_FORWARD: return "forward";
    case FAF_NORM_LAZY: return "lazy";
    case FAF_NORM_JPEG2000: return "jpeg2000";
    }
    return "unknown";
}

extern "C" size_t faf_precision_size(faf_precision p) {
    switch (p) {
    case FAF_PREC_FP8: case FAF_PREC_INT8: return 1;
    case FAF_PREC_FP16: case FAF_PREC_BF16: case FAF_PREC_INT16: return 2;
    case FAF_PREC_FP64: return 8;
    default: return 4;
    }
}

extern "C" const char* faf_precision_name(faf_precision p) {
    static const char* names[] = {"fp8", "fp16", "bf16", "fp32", "fp64", "int8", "int16", "int32"};
    return ((unsigned)p < 8) ? names[p] : "unknown";
}

extern "C" const char* faf_transform_name(faf_transform_type t) {
    static const char* names[] = {"fft",    "ifft",    "rfft",    "irfft",  "dct_i",  "dct_ii",
                                  "dct_iii", "dct_iv", "dst_i",   "dst_ii", "dst_iii", "dst_iv",
                                  "stft",   "mdct",    "imdct",   "haar",   "daubechies4",
                                  "cdf53",  "cdf97",   "sym4",    "pipeline", "cwt",  "icwt"};
    return ((unsigned)t < sizeof(names) / sizeof(names[0])) ? names[t] : "unknown";
}

extern "C" size_t faf_spectrum_len(const faf_transform* t) {
    if (!t) return 0;
    if (t->type == FAF_TRANSFORM_RFFT || t->type == FAF_TRANSFORM_IRFFT ||
        t->type == FAF_TRANSFORM_PIPELINE)
        return t->n / 2 + 1;
    return t->n;
}

// ---------------------------------------------------------------------------
// Size policy (reference src/faf_fft_stage.c:25-135, src/faf_core.c:374-429)
// ---------------------------------------------------------------------------

namespace fafapi {

bool is_5_smooth(size_t n) {
    if (n == 0) return false;
    for (size_t p : {2, 3, 5}) while (n % p == 0) n /= p;
    return n == 1;
}

bool is_7_smooth(size_t n) {
    if (n == 0) return false;
    for (size_t p : {2, 3, 5, 7}) while (n % p == 0) n /= p;
    return n == 1;
}

bool is_prime(size_t n) {
    if (n < 2) return false;
    if (n % 2 == 0) return n == 2;
    for (size_t d = 3; d * d <= n; d += 2)
        if (n % d == 0) return false;
    return true;
}

bool is_codelet(size_t n) { return (n >= 2 && n <= 10) || n == 12; }
bool rader_eligible(size_t n) { return n >= 11 && is_prime(n) && is_7_smooth(n - 1); }

size_t next_pow2(size_t n) {
    if (n == 0) return 1;
    size_t p = 1;
    while (p < n) p <<= 1;
    return p;
}

// faf_next_5_smooth: smallest 5-smooth >= m within [m, 2m + 32), else pow2.
size_t next_5_smooth(size_t m) {
    if (m <= 1) return 1;
    if (is_5_smooth(m)) return m;
    for (size_t n = m + 1; n < m * 2 + 32; n++)
        if (is_5_smooth(n)) return n;
    return next_pow2(m);
}

bool is_pow2(size_t n) { return n && !(n & (n - 1)); }

}  // namespace fafapi

extern "C" bool faf_is_size_supported(faf_transform_type type, size_t n) {
    if (n == 0) return false;
    switch (type) {
    case FAF_TRANSFORM_FFT:
    case FAF_TRANSFORM_IFFT:
        return is_5_smooth(n) || is_codelet(n) || rader_eligible(n);
    case FAF_TRANSFORM_HAAR:
    case FAF_TRANSFORM_DAUBECHIES4:
    case FAF_TRANSFORM_CDF53:
    case FAF_TRANSFORM_CDF97:
    case FAF_TRANSFORM_SYM4:
        return is_pow2(n);
    case FAF_TRANSFORM_RFFT:
    case FAF_TRANSFORM_IRFFT:
    case FAF_TRANSFORM_CWT:
    case FAF_TRANSFORM_ICWT:
        return is_5_smooth(n) && n % 2 == 0 && n >= 2;
    case FAF_TRANSFORM_DCT_I:
        return n >= 2;
    case FAF_TRANSFORM_MDCT:
    case FAF_TRANSFORM_IMDCT:
        return n % 2 == 0;
    default:
        return true;
    }
}

extern "C" size_t faf_get_recommended_size(faf_transform_type type, size_t min_size) {
    const bool c2c = type == FAF_TRANSFORM_FFT || type == FAF_TRANSFORM_IFFT;
    const bool real = type == FAF_TRANSFORM_RFFT || type == FAF_TRANSFORM_IRFFT ||
                      type == FAF_TRANSFORM_CWT || type == FAF_TRANSFORM_ICWT;
    if (c2c || real) {
        if (c2c && (is_5_smooth(min_size) || is_codelet(min_size) || rader_eligible(min_size)))
            return min_size;
        size_t n = next_5_smooth(min_size);
        if (real) {
            if (n < 2) n = 2;
            if (n % 2) n = next_5_smooth(n + 1);
        }
        return n;
    }
    return next_pow2(min_size);
}

// ---------------------------------------------------------------------------
// Transform objects
// ---------------------------------------------------------------------------

namespace fafapi {

faf_transform* alloc_transform() {
    faf_transform* t = (faf_transform*)calloc(1, sizeof(faf_transform));
    if (!t) fail("Failed to allocate transform");
    return t;
}

void apply_resolved(faf_transform* t, const faf_config& c) {
    t->cfg = c;
    t->n = c.n;
    t->precision = c.precision;
    t->flags = c.flags;
    if (c.dir == FAF_DIR_INVERSE) t->flags |= FAF_FLAG_INVERSE;
    t->family = c.family;
    t->levels = c.levels;
    t->hop_length = c.hop_length;
    t->win_length = c.win_length;
}

float norm_scale(faf_norm norm, bool inverse, size_t n) {
    switch (norm) {
    case FAF_NORM_ORTHO: return (float)(1.0 / std::sqrt((double)n));
    case FAF_NORM_FORWARD: return inverse ? 1.0f : (float)(1.0 / (double)n);
    default: return inverse ? (float)(1.0 / (double)n) : 1.0f;
    }
}

double norm_scale64(faf_norm norm, bool inverse, size_t n) {
    switch (norm) {
    case FAF_NORM_ORTHO: return 1.0 / std::sqrt((double)n);
    case FAF_NORM_FORWARD: return inverse ? 1.0 : 1.0 / (double)n;
    default: return inverse ? 1.0 / (double)n : 1.0;
    }
}

bool backend_ok(const faf_config& c, bool fp64_ok) {
    if (c.backend == FAF_BACKEND_VM || c.backend == FAF_BACKEND_JIT) {
        fail("backend %s is the reference's CPU engine; this library runs FAF_BACKEND_CUDA",
             c.backend == FAF_BACKEND_VM ? "VM" : "JIT");
        return false;
    }
    if (c.precision != FAF_PREC_FP32 && !(fp64_ok && c.precision == FAF_PREC_FP64)) {
        fail("precision '%s' is not available for this transform on the CUDA backend (FP32; "
             "FP64 for C2C, R2C and C2R)", faf_precision_name(c.precision));
        return false;
    }
    return true;
}

// Shared by faf_execute / batched: the C2C execute function the struct
// exposes as execute_func (split planes, one transform).
int exec_split_one(const faf_transform* t, void* out_re, void* out_im, const void* in_re,
                   const void* in_im);

}  // namespace fafapi

extern "C" void faf_destroy_transform(faf_transform* t) {
    if (!t) return;
    if (t->inner) faf_destroy_transform(t->inner);
    if (t->inner_inv) faf_destroy_transform(t->inner_inv);
    DevicePlan* p = plan_of(t);
    if (p) fafp::plan_free(p);
    free(t->code);
    for (int i = 0; i < 8; i++) free(t->twiddles[i]);
    if (t->scratch) cudaFreeHost(t->scratch);
    free(t);
}

extern "C" faf_transform* faf_create_fft(const faf_config* cfg) {
    if (!cfg) {
        fail("faf_create_fft: cfg is NULL");
        return nullptr;
    }
    faf_config c = *cfg;
    bool bluestein = false;
    if (is_5_smooth(c.n) || is_codelet(c.n)) {
    } else if (rader_eligible(c.n)) {
    } else if (c.flags & FAF_FLAG_BLUESTEIN) {
        bluestein = true;
    } else {
        fail("FFT size must be 5-smooth (2^a 3^b 5^c), a Rader prime (n-1 7-smooth), or a "
             "small codelet; got %zu; nearest 5-smooth is %zu (or set FAF_FLAG_BLUESTEIN)",
             c.n, faf_get_recommended_size(FAF_TRANSFORM_FFT, c.n));
        return nullptr;
    }
    if (c.layout == FAF_LAYOUT_DEFAULT) c.layout = FAF_LAYOUT_SPLIT;
    if (c.norm == FAF_NORM_DEFAULT) c.norm = FAF_NORM_NONE;
    if (c.layout == FAF_LAYOUT_REAL || c.layout == FAF_LAYOUT_HERMITIAN) {
        fail("FFT C2C does not support layout '%s'", faf_layout_name(c.layout));
        return nullptr;
    }
    if (c.norm == FAF_NORM_LAZY || c.norm == FAF_NORM_JPEG2000) {
        fail("FFT does not support norm '%s'", faf_norm_name(c.norm));
        return nullptr;
    }
    if (!backend_ok(c, true)) return nullptr;
    const bool fp64 = c.precision == FAF_PREC_FP64;
    if (fp64 && bluestein) {
        fail("FP64 Bluestein transforms are not available on the CUDA backend");
        return nullptr;
    }
    // the 2^16 cap on lengths; a Rader prime's inner length is p - 1, so
    // 65537 (inner 65536) is within it
    const bool rader = !bluestein && rader_eligible(c.n);
    if (c.n > (size_t)fafp::kMaxLength && !(rader && c.n - 1 <= (size_t)fafp::kMaxLength)) {
        fail("FFT length %zu exceeds the 2^16 transform-length cap", c.n);
        return nullptr;
    }
    faf_transform* t = alloc_transform();
    if (!t) return nullptr;
    const bool inverse = c.dir == FAF_DIR_INVERSE;
    t->type = inverse ? FAF_TRANSFORM_IFFT : FAF_TRANSFORM_FFT;
    if (c.backend == FAF_BACKEND_AUTO) c.backend = FAF_BACKEND_CUDA;
    apply_resolved(t, c);
    if (bluestein) {
        t->flags |= FAF_FLAG_BLUESTEIN;
        t->cfg.flags |= FAF_FLAG_BLUESTEIN;
    }
    std::string err;
    DevicePlan* p = fp64 ? fafp::plan_c2c64((int)c.n, inverse, norm_scale64(c.norm, inverse, c.n),
                                            err)
                         : fafp::plan_c2c((int)c.n, inverse, norm_scale(c.norm, inverse, c.n),
                                          t->flags, err);
    if (!p) {
        fail("CUDA plan for FFT n=%zu: %s", c.n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = p;
    t->execute_func = exec_split_one;
    return t;
}

extern "C" faf_transform* faf_create_rfft(const faf_config* cfg) {
    if (!cfg) {
        fail("faf_create_rfft: cfg is NULL");
        return nullptr;
    }
    faf_config c = *cfg;
    if (c.flags & FAF_FLAG_BLUESTEIN) {
        fail("R2C does not support Bluestein in v1; use C2C with FAF_FLAG_BLUESTEIN on a real "
             "buffer");
        return nullptr;
    }
    if (c.n < 2 || (c.n & 1u)) {
        fail("R2C size must be even and >= 2, got %zu", c.n);
        return nullptr;
    }
    if (!is_5_smooth(c.n)) {
        fail("R2C size must be even and 5-smooth, got %zu; nearest is %zu", c.n,
             faf_get_recommended_size(FAF_TRANSFORM_RFFT, c.n));
        return nullptr;
    }
    if (c.precision != FAF_PREC_FP32 && c.precision != FAF_PREC_FP64) {
        fail("R2C supports FP32 and FP64 only");
        return nullptr;
    }
    if (c.layout == FAF_LAYOUT_DEFAULT) c.layout = FAF_LAYOUT_HERMITIAN;
    if (c.norm == FAF_NORM_DEFAULT) c.norm = FAF_NORM_NONE;
    if (c.layout != FAF_LAYOUT_HERMITIAN && c.layout != FAF_LAYOUT_INTERLEAVED) {
        fail("R2C layout must be hermitian or interleaved, got '%s'", faf_layout_name(c.layout));
        return nullptr;
    }
    if (c.norm == FAF_NORM_LAZY || c.norm == FAF_NORM_JPEG2000) {
        fail("R2C does not support norm '%s'", faf_norm_name(c.norm));
        return nullptr;
    }
    if (!backend_ok(c, true)) return nullptr;
    if (c.n > (size_t)fafp::kMaxLength) {
        fail("R2C length %zu exceeds the 2^16 transform-length cap", c.n);
        return nullptr;
    }
    faf_transform* t = alloc_transform();
    if (!t) return nullptr;
    const bool inverse = c.dir == FAF_DIR_INVERSE;
    if (c.backend == FAF_BACKEND_AUTO) c.backend = FAF_BACKEND_CUDA;
    t->type = inverse ? FAF_TRANSFORM_IRFFT : FAF_TRANSFORM_RFFT;
    apply_resolved(t, c);
    t->flags = c.flags | FAF_FLAG_REAL | (inverse ? FAF_FLAG_INVERSE : 0u);
    // Nested n/2 C2C, as the reference keeps it (src/faf_rfft.c:228-238).
    faf_config ic = faf_config_init(c.n / 2);
    ic.layout = FAF_LAYOUT_SPLIT;
    ic.norm = FAF_NORM_NONE;
    ic.dir = c.dir;
    ic.backend = c.backend;
    ic.precision = c.precision;
    t->inner = faf_create_fft(&ic);
    if (!t->inner) {
        faf_destroy_transform(t);
        return nullptr;
    }
    std::string err;
    DevicePlan* p =
        c.precision == FAF_PREC_FP64
            ? fafp::plan_r2c64((int)c.n, inverse, norm_scale64(c.norm, inverse, c.n), err)
            : fafp::plan_r2c((int)c.n, inverse, norm_scale(c.norm, inverse, c.n), err);
    if (!p) {
        fail("CUDA plan for R2C n=%zu: %s", c.n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = p;
    return t;
}

extern "C" faf_transform* faf_create_stft(const faf_config* cfg) {
    if (!cfg) {
        fail("faf_create_stft: cfg is NULL");
        return nullptr;
    }
    faf_config c = *cfg;
    if (c.win_length == 0) c.win_length = c.n;
    if (c.hop_length == 0) c.hop_length = c.win_length / 4;
    if (!backend_ok(c)) return nullptr;  // STFT runs in FP32
    if (c.win_length > c.n) {
        fail("STFT window length %zu exceeds FFT size %zu", c.win_length, c.n);
        return nullptr;
    }
    if (c.hop_length == 0) {
        fail("STFT hop length must be > 0");
        return nullptr;
    }
    // One frame as a C2C of n (reference src/faf_core.c:1007-1010) ...
    faf_config fc = c;
    fc.dir = FAF_DIR_FORWARD;
    faf_transform* t = faf_create_fft(&fc);
    if (!t) return nullptr;
    t->type = FAF_TRANSFORM_STFT;
    t->hop_length = c.hop_length;
    t->win_length = c.win_length;
    t->cfg.hop_length = c.hop_length;
    t->cfg.win_length = c.win_length;
    // ... plus the framed real STFT of long signals (R2C of n per frame),
    // which needs an even 5-smooth n.
    if (c.n >= 2 && c.n % 2 == 0 && is_5_smooth(c.n)) {
        std::string err;
        faf_transform* fr = alloc_transform();
        if (!fr) {
            faf_destroy_transform(t);
            return nullptr;
        }
        fr->type = FAF_TRANSFORM_RFFT;
        faf_config rc = c;
        rc.layout = FAF_LAYOUT_HERMITIAN;
        rc.norm = FAF_NORM_NONE;
        apply_resolved(fr, rc);
        DevicePlan* p = fafp::plan_stft((int)c.n, (int)c.win_length, (int)c.hop_length, 1.0f, err);
        if (!p) {
            fail("CUDA plan for STFT n=%zu: %s", c.n, err.c_str());
            free(fr);
            faf_destroy_transform(t);
            return nullptr;
        }
        fr->device_plan = p;
        t->inner = fr;
    }
    return t;
}

extern "C" faf_transform* faf_create(faf_transform_type type, const faf_config* cfg) {
    if (!cfg) {
        fail("faf_create: cfg is NULL");
        return nullptr;
    }
    faf_config c = *cfg;
    switch (type) {
    case FAF_TRANSFORM_IFFT:
        c.dir = FAF_DIR_INVERSE;
        return faf_create_fft(&c);
    case FAF_TRANSFORM_FFT:
        return faf_create_fft(&c);
    case FAF_TRANSFORM_IRFFT:
        c.dir = FAF_DIR_INVERSE;
        return faf_create_rfft(&c);
    case FAF_TRANSFORM_RFFT:
        return faf_create_rfft(&c);
    case FAF_TRANSFORM_STFT:
        return faf_create_stft(&c);
    default:
        fail("transform type '%s' is outside the CUDA transform path (FFT, RFFT, STFT, "
             "pipeline)", faf_transform_name(type));
        return nullptr;
    }
}

extern "C" faf_transform* faf_cuda_create_istft(const faf_config* cfg) {
    if (!cfg) {
        fail("faf_cuda_create_istft: cfg is NULL");
        return nullptr;
    }
    faf_config c = *cfg;
    if (c.win_length == 0) c.win_length = c.n;
    if (c.hop_length == 0) c.hop_length = c.win_length / 4;
    if (c.win_length > c.n || c.hop_length == 0 || c.hop_length > c.win_length) {
        fail("inverse STFT needs 0 < hop <= win <= n (n=%zu, win=%zu, hop=%zu)", c.n,
             c.win_length, c.hop_length);
        return nullptr;
    }
    if (c.n < 2 || c.n % 2 || !is_5_smooth(c.n)) {
        fail("inverse STFT needs an even 5-smooth FFT size, got %zu", c.n);
        return nullptr;
    }
    if (!backend_ok(c)) return nullptr;
    faf_transform* t = alloc_transform();
    if (!t) return nullptr;
    t->type = FAF_TRANSFORM_STFT;
    c.dir = FAF_DIR_INVERSE;
    c.layout = FAF_LAYOUT_HERMITIAN;
    c.norm = FAF_NORM_NONE;
    if (c.backend == FAF_BACKEND_AUTO) c.backend = FAF_BACKEND_CUDA;
    apply_resolved(t, c);
    t->flags |= FAF_FLAG_INVERSE;
    t->hop_length = c.hop_length;
    t->win_length = c.win_length;
    std::string err;
    DevicePlan* p = fafp::plan_istft((int)c.n, (int)c.win_length, (int)c.hop_length, err);
    if (!p) {
        fail("CUDA plan for inverse STFT n=%zu: %s", c.n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = p;
    return t;
}

// CWT filter bank: the reference builds its bank on the host at create
// (src/faf_cwt.c:104-677) and runs x -> rows through faf_cwt_execute
// (src/faf_cwt.c:769-847).  The device transform takes the bank's rows as
// they are (row 0 = lowpass phi when the bank has one, then wavelets coarse
// to fine; n/2+1 real weights per row, `psi_stride` floats apart: the
// reference bank's n_bins_padded) and runs the execute.
extern "C" faf_transform* faf_cuda_create_cwt(size_t n, size_t n_rows, const float* psi,
                                              size_t psi_stride) {
    if (n < 2 || n % 2 || !is_5_smooth(n)) {
        fail("cwt: n=%zu must be even and 5-smooth", n);
        return nullptr;
    }
    if (n_rows == 0 || !psi) {
        fail("cwt: the bank needs at least one row (psi non-NULL)");
        return nullptr;
    }
    if (psi_stride < n / 2 + 1) {
        fail("cwt: row stride %zu is shorter than the %zu packed bins", psi_stride, n / 2 + 1);
        return nullptr;
    }
    if (n_rows > (size_t)INT_MAX) {
        fail("cwt: %zu rows", n_rows);
        return nullptr;
    }
    faf_config c = faf_config_init(n);
    c.layout = FAF_LAYOUT_REAL;
    c.norm = FAF_NORM_NONE;
    c.backend = FAF_BACKEND_CUDA;
    faf_transform* t = alloc_transform();
    if (!t) return nullptr;
    t->type = FAF_TRANSFORM_CWT;
    apply_resolved(t, c);
    t->user_aux_n = n_rows;  // the reference stores the row count here too
    std::string err;
    DevicePlan* p = fafp::plan_cwt((int)n, (int)n_rows, psi, psi_stride, err);
    if (!p) {
        fail("CUDA plan for CWT n=%zu: %s", n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = p;
    return t;
}

// Shared checks and the transform object of the two inverse CWT forms.
static faf_transform* icwt_transform(size_t n, size_t n_rows) {
    if (n < 2 || n % 2 || !is_5_smooth(n)) {
        fail("cwt: n=%zu must be even and 5-smooth", n);
        return nullptr;
    }
    if (n_rows == 0 || n_rows > (size_t)INT_MAX) {
        fail("cwt: the bank needs at least one row");
        return nullptr;
    }
    faf_config c = faf_config_init(n);
    c.layout = FAF_LAYOUT_REAL;
    c.norm = FAF_NORM_NONE;
    c.dir = FAF_DIR_INVERSE;
    c.backend = FAF_BACKEND_CUDA;
    faf_transform* t = alloc_transform();
    if (!t) return nullptr;
    t->type = FAF_TRANSFORM_ICWT;
    apply_resolved(t, c);
    t->user_aux_n = n_rows;
    return t;
}

// Dual-frame inverse CWT (faf_create_icwt with FAF_CWT_INV_DUAL,
// src/faf_cwt.c:728-762 and 935-985): the bank's dual rows, as the reference
// derives them from its analysis rows (src/faf_cwt.c:440-482).
extern "C" faf_transform* faf_cuda_create_icwt_dual(size_t n, size_t n_rows, const float* dual,
                                                    size_t dual_stride) {
    if (!dual || dual_stride < n / 2 + 1) {
        fail("cwt: dual rows missing or stride %zu shorter than the %zu packed bins", dual_stride,
             n / 2 + 1);
        return nullptr;
    }
    faf_transform* t = icwt_transform(n, n_rows);
    if (!t) return nullptr;
    std::string err;
    DevicePlan* p = fafp::plan_icwt_dual((int)n, (int)n_rows, dual, dual_stride, err);
    if (!p) {
        fail("CUDA plan for inverse CWT n=%zu: %s", n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = p;
    return t;
}

// L1 one-integral inverse CWT (FAF_CWT_INV_L1, src/faf_cwt.c:879-930):
// dlog = ln 2 / voices, C = the bank report's admissibility_C (<= 0 means 1).
extern "C" faf_transform* faf_cuda_create_icwt_l1(size_t n, size_t n_rows, int has_lowpass,
                                                  double dlog, double C) {
    if (has_lowpass && n_rows < 2) {
        fail("cwt: a bank with a lowpass row needs at least one wavelet row");
        return nullptr;
    }
    faf_transform* t = icwt_transform(n, n_rows);
    if (!t) return nullptr;
    std::string err;
    DevicePlan* p = fafp::plan_icwt_l1((int)n, (int)n_rows, has_lowpass, dlog, C, err);
    if (!p) {
        fail("CUDA plan for inverse CWT n=%zu: %s", n, err.c_str());
        faf_destroy_transform(t);
        return nullptr;
    }
    t->device_plan = p;
    return t;
}

extern "C" faf_transform* faf_create_inverse(const faf_transform* fwd) {
    if (!fwd) {
        fail("faf_create_inverse: transform is NULL");
        return nullptr;
    }
    faf_config c = faf_config_inverse(fwd->cfg);
    switch (fwd->type) {
    case FAF_TRANSFORM_FFT:
    case FAF_TRANSFORM_IFFT:
        return faf_create_fft(&c);
    case FAF_TRANSFORM_RFFT:
    case FAF_TRANSFORM_IRFFT:
        return faf_create_rfft(&c);
    case FAF_TRANSFORM_STFT:
        // The reference returns another forward STFT (src/faf_core.c:1122).
        return faf_create_stft(&c);
    default:
        fail("faf_create_inverse: unsupported type %s", faf_transform_name(fwd->type));
        return nullptr;
    }
}

// ---------------------------------------------------------------------------
// Hermitian multiply and (de)interleave helpers (host memory, as in the
// reference; device pointers are rejected rather than silently read)
// ---------------------------------------------------------------------------

template <class T>
static void herm_mul(T* yr, T* yi, const T* xr, const T* xi, const T* hr, const T* hi,
                     size_t nb, bool conj_h) {
    if (!yr || !yi || !xr || !xi || !hr || !hi || nb == 0) return;
    yr[0] = xr[0] * hr[0];
    yi[0] = 0;
    for (size_t k = 1; k + 1 < nb; k++) {
        const T ar = xr[k], ai = xi[k], br = hr[k], bi = conj_h ? -hi[k] : hi[k];
        yr[k] = ar * br - ai * bi;
        yi[k] = ar * bi + ai * br;
    }
    if (nb > 1) {
        yr[nb - 1] = xr[nb - 1] * hr[nb - 1];
        yi[nb - 1] = 0;
    }
}

extern "C" void faf_herm_mul_f32(float* yr, float* yi, const float* xr, const float* xi,
                                 const float* hr, const float* hi, size_t n) {
    herm_mul(yr, yi, xr, xi, hr, hi, n, false);
}
extern "C" void faf_herm_mul_f64(double* yr, double* yi, const double* xr, const double* xi,
                                 const double* hr, const double* hi, size_t n) {
    herm_mul(yr, yi, xr, xi, hr, hi, n, false);
}
extern "C" void faf_herm_mul_conj_f32(float* yr, float* yi, const float* xr, const float* xi,
                                      const float* hr, const float* hi, size_t n) {
    herm_mul(yr, yi, xr, xi, hr, hi, n, true);
}
extern "C" void faf_herm_mul_conj_f64(double* yr, double* yi, const double* xr,
                                      const double* xi, const double* hr, const double* hi,
                                      size_t n) {
    herm_mul(yr, yi, xr, xi, hr, hi, n, true);
}

template <class T>
static int deinter(T* re, T* im, const T* x, size_t n) {
    if (!re || !im || !x) return fail("deinterleave: null buffer");
    for (size_t i = 0; i < n; i++) {
        re[i] = x[2 * i];
        im[i] = x[2 * i + 1];
    }
    return 0;
}

template <class T>
static int inter(T* x, const T* re, const T* im, size_t n) {
    if (!x || !re || !im) return fail("interleave: null buffer");
    for (size_t i = 0; i < n; i++) {
        x[2 * i] = re[i];
        x[2 * i + 1] = im[i];
    }
    return 0;
}

extern "C" int faf_deinterleave_f32(float* re, float* im, const float* x, size_t n) {
    return deinter(re, im, x, n);
}
extern "C" int faf_interleave_f32(float* x, const float* re, const float* im, size_t n) {
    return inter(x, re, im, n);
}
extern "C" int faf_deinterleave_f64(double* re, double* im, const double* x, size_t n) {
    return deinter(re, im, x, n);
}
extern "C" int faf_interleave_f64(double* x, const double* re, const double* im, size_t n) {
    return inter(x, re, im, n);
}
