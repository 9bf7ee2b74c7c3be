// faf_kernels_common.cuh -- sources, sinks and helpers of the batched
// transform kernels for sm_100a (one .cu per kernel family includes this).
//
// Every kernel runs G transforms per CTA (T threads each) through the
// Stockham engine of faf_device.cuh.  Loads of the first stage and stores of
// the last stage go straight between global memory and registers, so a
// plain C2C reads its input once and writes its output once; everything the
// reference does as separate passes over the data (R2C pack / super-twiddle
// post-pass, the pipeline's spectral ops, the C2R pre-pass, STFT windowing,
// Rader gather / scatter, Bluestein chirp multiplies, the norm scaling) is
// fused into the sources / sinks of those stages.
#pragma once

#include <algorithm>
#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "faf_device.cuh"
#include "faf_kernels.cuh"

namespace fafk {
// Values held per thread per stage.  With 16, a transform of n points uses
// about n/16 threads, so the single-CTA kernels cover n <= 16384 (radix-16
// stages) within the 1024-thread limit; larger n use the four-step path.
constexpr int kE = 16;
using fafd::cf;
using fafd::run_fft;
using fafd::Shape;
using fafd::SmemConjSrc;
using fafd::SmemIO;

// ---------------------------------------------------------------------------
// Sources and sinks
// ---------------------------------------------------------------------------

struct SplitSrc {  // split or interleaved complex input, optional real window
    const float* re;
    const float* im;
    const float* win;
    float sgn;
    int inter;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (!live) return cf{0.f, 0.f};
        float r, m;
        if (inter) {
            float2 v = __ldcs(reinterpret_cast<const float2*>(re) + i);
            r = v.x; m = v.y;
        } else {
            r = __ldcs(re + i); m = __ldcs(im + i);
        }
        if (win) { float w = __ldg(win + i); r *= w; m *= w; }
        return cf{r, sgn * m};
    }
};

struct SplitSink {
    float* re;
    float* im;
    float scale;
    float sgn;
    int inter;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int i, cf v) const {
        if (!live) return;
        if (inter) {
            __stcs(reinterpret_cast<float2*>(re) + i, make_float2(v.x * scale, sgn * v.y * scale));
        } else {
            __stcs(re + i, v.x * scale);
            __stcs(im + i, sgn * v.y * scale);
        }
    }
};

// z[k] = x[2k] + i x[2k+1] (R2C packing, reference src/faf_rfft.c:356-359).
// Packed real pairs z[i] = x[2i] + i x[2i+1].  Every caller points a dead
// transform (past the batch) at transform 0, so the loads need no guard;
// its results are dropped by the sink.
struct RealPairSrc {
    const float* x;
    bool live;  // unused by the loads (kept for the callers' symmetry)
    bool vec;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (vec) {
            float2 v = __ldcs(reinterpret_cast<const float2*>(x) + i);
            return cf{v.x, v.y};
        }
        return cf{__ldcs(x + 2 * i), __ldcs(x + 2 * i + 1)};
    }
};

// Windowed, zero-padded STFT frame packed as real pairs.
struct FrameSrc {
    const float* x;   // frame start
    const float* w;
    int win;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        const int a = 2 * i, b = a + 1;
        float v0 = 0.f, v1 = 0.f;
        if (live && a < win) v0 = __ldg(x + a) * __ldg(w + a);
        if (live && b < win) v1 = __ldg(x + b) * __ldg(w + b);
        return cf{v0, v1};
    }
};

// The same frame landed in shared memory (a ring slot holding its first
// `win` samples) with the window in shared memory too.
struct FrameStageSrc {
    const float2* s;  // slot: x[2i], x[2i+1] as float2 i
    const float2* w;  // window, the same pairing
    int win;          // even
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (2 * i >= win) return cf{0.f, 0.f};
        const float2 v = s[i], u = w[i];
        return cf{v.x * u.x, v.y * u.y};
    }
};

// y[2k] = Re z, y[2k+1] = Im z, with the conjugation of an inverse FFT undone
// (C2R unpack, reference src/faf_rfft.c:392-395).
struct RealPairSink {
    float* y;
    float scale;
    bool live;
    bool vec;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int i, cf v) const {
        if (!live) return;
        if (vec) {
            __stcs(reinterpret_cast<float2*>(y) + i, make_float2(v.x * scale, -v.y * scale));
        } else {
            __stcs(y + 2 * i, v.x * scale);
            __stcs(y + 2 * i + 1, -v.y * scale);
        }
    }
};

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------

// Host memo of per-kernel launch facts (the shared-memory opt-in made so far,
// resident CTAs per launch shape), per device, so that a launch after the
// first costs no driver query: small launches are bound by host time.
struct LaunchMemo {
    std::mutex mu;
    std::map<std::pair<const void*, int>, size_t> smem;                // opted-in bytes
    std::map<std::tuple<const void*, int, int, size_t>, int> per_sm;  // occupancy
    static LaunchMemo& get() {
        static LaunchMemo m;
        return m;
    }
};

template <class K>
inline cudaError_t prep(K kernel, size_t smem) {
    if (smem <= 48 * 1024) return cudaSuccess;
    int dev = 0;
    cudaGetDevice(&dev);
    LaunchMemo& m = LaunchMemo::get();
    const auto key = std::make_pair((const void*)kernel, dev);
    {
        std::lock_guard<std::mutex> lk(m.mu);
        auto it = m.smem.find(key);
        if (it != m.smem.end() && it->second >= smem) return cudaSuccess;
    }
    cudaError_t e =
        cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lk(m.mu);
    size_t& v = m.smem[key];
    v = std::max(v, smem);
    return cudaSuccess;
}

// Resident CTAs per SM of `kernel` at this shape (memoised; 1 if the query fails).
template <class K>
inline int resident_ctas(K kernel, int threads, size_t smem) {
    int dev = 0;
    cudaGetDevice(&dev);
    LaunchMemo& m = LaunchMemo::get();
    const auto key = std::make_tuple((const void*)kernel, dev, threads, smem);
    {
        std::lock_guard<std::mutex> lk(m.mu);
        auto it = m.per_sm.find(key);
        if (it != m.per_sm.end()) return it->second;
    }
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem) !=
            cudaSuccess ||
        per_sm <= 0) {
        cudaGetLastError();
        per_sm = 1;
    }
    std::lock_guard<std::mutex> lk(m.mu);
    m.per_sm[key] = per_sm;
    return per_sm;
}

inline unsigned grid_for(long long batch, int G) {
    return (unsigned)((batch + G - 1) / G);
}

// Per-CTA group bookkeeping: transform group g, thread t within it, planes.
struct Group {
    int g, t;
    float* re;
    float* im;
};

__device__ __forceinline__ Group group_of(const Shape& S, float* sm, int extra_per_group) {
    Group q;
    q.g = threadIdx.x / S.T;
    q.t = threadIdx.x - q.g * S.T;
    q.re = sm + (size_t)q.g * (2 * S.plane + extra_per_group);
    q.im = q.re + S.plane;
    return q;
}

// ---------------------------------------------------------------------------
// R2C: pack -> nc-point FFT -> super-twiddle post-pass (src/faf_rfft.c:61-89)
// ---------------------------------------------------------------------------

// Post-pass of one bin pair (k, nc-k), k >= 1, from the packed spectrum Z.
__device__ __forceinline__ void r2c_pair(cf zk, cf znk, float2 w, cf& Xk, cf& Xnk) {
    // f1 = Z[k] + conj(Z[nc-k]), f2 = Z[k] - conj(Z[nc-k]), t = f2 * w
    const float f1r = zk.x + znk.x, f1i = zk.y - znk.y;
    const float f2r = zk.x - znk.x, f2i = zk.y + znk.y;
    const float tr = f2r * w.x - f2i * w.y, ti = fmaf(f2r, w.y, f2i * w.x);
    Xk = cf{0.5f * (f1r + tr), 0.5f * (f1i + ti)};
    Xnk = cf{0.5f * (f1r - tr), 0.5f * (ti - f1i)};
}

// Pre-pass of one bin pair for the C2R (src/faf_rfft.c:122-146); w is the
// forward super-twiddle, the inverse uses its conjugate.
__device__ __forceinline__ void c2r_pair(cf xk, cf xnk, float2 w, cf& Zk, cf& Znk) {
    const float fer = xk.x + xnk.x, fei = xk.y - xnk.y;  // fk + conj(X[nc-k])
    const float dr = xk.x - xnk.x, di = xk.y + xnk.y;    // fk - conj(X[nc-k])
    const float wr = w.x, wi = -w.y;
    const float orr = dr * wr - di * wi, oi = fmaf(dr, wi, di * wr);
    Zk = cf{fer + orr, fei + oi};
    Znk = cf{fer - orr, -(fei - oi)};
}

struct HermSink {  // split or interleaved Hermitian output
    float* re;
    float* im;
    int inter;
    __device__ __forceinline__ void put(int k, float r, float i) const {
        if (inter) {
            __stcs(reinterpret_cast<float2*>(re) + k, make_float2(r, i));
        } else {
            __stcs(re + k, r);
            __stcs(im + k, i);
        }
    }
};

// The two layouts of HermSink as separate types, for kernels that branch
// once per transform instead of once per store.
struct HermSplit {
    float* re;
    float* im;
    __device__ __forceinline__ void put(int k, float r, float i) const {
        __stcs(re + k, r);
        __stcs(im + k, i);
    }
};
struct HermInter {
    float2* p;
    __device__ __forceinline__ void put(int k, float r, float i) const {
        __stcs(p + k, make_float2(r, i));
    }
};

template <int E, class Src>
__device__ __forceinline__ void r2c_body(const Shape& S, const Group& q,
                                         const float2* __restrict__ tw,
                                         const float2* __restrict__ stw, const Src& src,
                                         const HermSink& out, float scale, bool live) {
    const int nc = S.n;
    const SmemIO mid{q.re, q.im};
    run_fft<E>(S, q.t, q.re, q.im, tw, src, mid);
    __syncthreads();
    if (!live) return;
    for (int k = q.t; k <= nc / 2; k += S.T) {
        if (k == 0) {
            const cf z = mid.get(0);
            out.put(0, (z.x + z.y) * scale, 0.f);
            out.put(nc, (z.x - z.y) * scale, 0.f);
        } else {
            cf Xk, Xnk;
            r2c_pair(mid.get(k), mid.get(nc - k), __ldg(&stw[k - 1]), Xk, Xnk);
            if (k != nc - k) out.put(k, Xk.x * scale, Xk.y * scale);
            out.put(nc - k, Xnk.x * scale, Xnk.y * scale);
        }
    }
}

#define FAF_REAL_LAUNCH(NAME, KERNEL, ...)                                                     \
    cudaError_t NAME(const Shape& S, const Geometry& g, const float2* tw, const RealArgs& a,  \
                     cudaStream_t st) {                                                        \
        if (a.batch <= 0) return cudaSuccess;                                                  \
        cudaError_t e;                                                                         \
        if ((e = prep(KERNEL<kE>, g.smem)) != cudaSuccess) return e;                           \
        KERNEL<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G __VA_ARGS__); \
        return cudaGetLastError();                                                             \
    }

inline bool vec_ok(const void* p, long long dist) {
    return (((unsigned long long)(size_t)p) % 8 == 0) && (dist % 2 == 0);
}

// ---- Rader convolution pieces (reference src/faf_fft_rader.c:136-232) ----

struct GatherSrc {
    const float* re;
    const float* im;
    const int* idx;
    float sgn;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int j) const {
        if (!live) return cf{0.f, 0.f};
        const int s = __ldg(idx + j);
        return cf{__ldg(re + s), sgn * __ldg(im + s)};
    }
};

// Last-stage sink: multiply by B in place; keep bin 0 (the sum of the
// gathered samples) for the DC term.
struct MulBSink {
    float* re;
    float* im;
    const float2* B;
    float* dc;  // 2 floats per group, or NULL
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int j, cf v) const {
        if (dc && j == 0) { dc[0] = v.x; dc[1] = v.y; }
        const float2 w = __ldg(&B[j]);
        const int p = fafd::pad(j);
        re[p] = v.x * w.x - v.y * w.y;
        im[p] = fmaf(v.x, w.y, v.y * w.x);
    }
};

struct ScatterSink {
    float* re;
    float* im;
    const int* idx;
    float x0r, x0i;   // x[0] (conjugated for inverse)
    float inv_m;
    float scale, sgn;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int j, cf v) const {
        if (!live) return;
        const int d = __ldg(idx + j);
        // v is conj(unscaled inverse FFT); undo, scale by 1/m, add x0
        const float yr = x0r + v.x * inv_m, yi = x0i - v.y * inv_m;
        re[d] = yr * scale;
        im[d] = sgn * yi * scale;
    }
};

// Spectral ops of the fused pipeline on bin k (reference src/chirp.c:421-471,
// src/faf_core.c:150-166): CONJ negates im; MUL multiplies by the bound H with
// real DC and last-bin products; BANDPASS zeroes bins outside [lo, hi].
__device__ __forceinline__ cf mul_bin(const PipeOp& op, int k, cf v) {
    if (k >= op.m) return v;
    const float hr = __ldg(op.hr + k);
    if (k == 0 || k == op.m - 1) return cf{v.x * hr, 0.f};
    const float hi = __ldg(op.hi_ + k);
    return cf{v.x * hr - v.y * hi, fmaf(v.x, hi, v.y * hr)};
}

// Device spectral ops (chirp_register_spectral_device): gain, fixed phase,
// and a circular delay whose phase is reduced in FP64 (k d mod n) before the
// sine / cosine, so large k d keeps its accuracy.  The delay is out of line:
// its FP64 code inlined at every bin of an unrolled pass bloats the kernel.
static __device__ __noinline__ cf delay_bin(double d0, int n, int k, cf v) {
    const double r = fmod((double)k * d0, (double)n);
    double s, c;
    sincospi(-2.0 * r / (double)n, &s, &c);
    const float fs = (float)s, fc = (float)c;
    return cf{v.x * fc - v.y * fs, fmaf(v.x, fs, v.y * fc)};
}

__device__ __forceinline__ cf apply_op(const PipeOp& op, int k, cf v) {
    if (op.code == OP_CONJ) return cf{v.x, -v.y};
    if (op.code == OP_MUL) return mul_bin(op, k, v);
    if (op.code == OP_BANDPASS && (k < op.lo || k > op.hi)) return cf{0.f, 0.f};
    if (op.code == OP_SCALE) return cf{v.x * op.f0, v.y * op.f0};
    if (op.code == OP_ROTATE) return cf{v.x * op.f0 - v.y * op.f1, fmaf(v.x, op.f1, v.y * op.f0)};
    if (op.code == OP_DELAY) return delay_bin(op.d0, op.n, k, v);
    return v;
}

// Every op in order, as a loop over the program (not unrolled): the passes
// call this once per bin, and a copy of every op kind at each call site made
// the generic-program kernels several times slower than the single-MUL one.
__device__ __forceinline__ cf apply_pipe_ops(const RealArgs& a, int k, cf v) {
#pragma unroll 1
    for (int o = 0; o < a.nops; o++) v = apply_op(a.ops[o], k, v);
    return v;
}

// The op program as a functor for the bin-pair passes: any program, or the
// common single MUL by a bound spectrum, which skips the op dispatch.
struct OpsAny {
    const RealArgs* a;
    __device__ __forceinline__ cf operator()(int k, cf v) const { return apply_pipe_ops(*a, k, v); }
};
struct OpsMul1 {
    const PipeOp* op;
    __device__ __forceinline__ cf operator()(int k, cf v) const { return mul_bin(*op, k, v); }
};
// The single MUL on bins 1 .. m - 2 of a spectrum bound over all m bins:
// mul_bin's complex product without its guards.
struct OpsMul1Full {
    const PipeOp* op;
    __device__ __forceinline__ cf operator()(int k, cf v) const {
        const float hr = __ldg(op->hr + k), hi = __ldg(op->hi_ + k);
        return cf{v.x * hr - v.y * hi, fmaf(v.x, hi, v.y * hr)};
    }
};
// The same product with the spectrum's planes in shared memory.
struct OpsMulSmem {
    const float* hr;
    const float* hi;
    __device__ __forceinline__ cf operator()(int k, cf v) const {
        const float r = hr[k], i = hi[k];
        return cf{v.x * r - v.y * i, fmaf(v.x, i, v.y * r)};
    }
};
__host__ __device__ inline bool ops_single_mul(const RealArgs& a) {
    return a.nops == 1 && a.ops[0].code == OP_MUL;
}

}  // namespace fafk
