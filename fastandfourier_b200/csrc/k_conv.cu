// k_conv.cu -- Rader and Bluestein convolution kernels.
#include "faf_kernels_common.cuh"

namespace fafk {

// ---------------------------------------------------------------------------
// Rader (prime n): gather -> FFT_m -> x B -> IFFT_m -> scatter, one CTA
// (reference src/faf_fft_rader.c:136-232).  DC = x0 + FFT_m(gathered)[0].
// ---------------------------------------------------------------------------

template <int E>
__global__ void __launch_bounds__(1024) k_rader(const Shape S, const float2* __restrict__ tw,
                                                const ConvArgs a, int G) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 2);
    float* dc = q.re + 2 * S.plane;
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const float* xr = a.in_re + bi * a.in_dist;
    const float* xi = a.in_im + bi * a.in_dist;
    run_fft<E>(S, q.t, q.re, q.im, tw, GatherSrc{xr, xi, a.rin, a.sgn, live},
               MulBSink{q.re, q.im, a.B, dc});
    __syncthreads();
    float x0r = 0.f, x0i = 0.f;
    if (live) { x0r = __ldg(xr); x0i = a.sgn * __ldg(xi); }
    float* yr = a.out_re + bi * a.out_dist;
    float* yi = a.out_im + bi * a.out_dist;
    if (live && q.t == 0) {
        yr[0] = (x0r + dc[0]) * a.scale;
        yi[0] = a.sgn * (x0i + dc[1]) * a.scale;
    }
    run_fft<E>(S, q.t, q.re, q.im, tw, SmemConjSrc{q.re, q.im},
               ScatterSink{yr, yi, a.rout, x0r, x0i, a.inv_inner, a.scale, a.sgn, live});
}

cudaError_t launch_rader(const Shape& S, const Geometry& g, const float2* tw, const ConvArgs& a,
                         cudaStream_t st) {
    if (a.batch <= 0) return cudaSuccess;
    cudaError_t e;
    if ((e = prep(k_rader<kE>, g.smem)) != cudaSuccess) return e;
        k_rader<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Bluestein (any n): x*phi (zero-padded to M) -> FFT_M -> x B -> IFFT_M ->
// x phi / M (reference src/faf_bluestein.c:165-223), one CTA per transform.
// ---------------------------------------------------------------------------

struct ChirpSrc {
    const float* re;
    const float* im;
    const float2* phi;
    int n;
    float sgn;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int k) const {
        if (!live || k >= n) return cf{0.f, 0.f};
        const float xr = __ldg(re + k), xi = sgn * __ldg(im + k);
        const float2 w = __ldg(&phi[k]);
        return cf{xr * w.x - xi * w.y, fmaf(xr, w.y, xi * w.x)};
    }
};

struct ChirpSink {
    float* re;
    float* im;
    const float2* phi;
    int n;
    float inv_m, scale, sgn;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int k, cf v) const {
        if (!live || k >= n) return;
        const float ar = v.x * inv_m, ai = -v.y * inv_m;  // undo the conjugation
        const float2 w = __ldg(&phi[k]);
        const float yr = ar * w.x - ai * w.y, yi = fmaf(ar, w.y, ai * w.x);
        re[k] = yr * scale;
        im[k] = sgn * yi * scale;
    }
};

template <int E>
__global__ void __launch_bounds__(1024) k_bluestein(const Shape S, const float2* __restrict__ tw,
                                                    const ConvArgs a, int G) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 0);
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    run_fft<E>(S, q.t, q.re, q.im, tw,
               ChirpSrc{a.in_re + bi * a.in_dist, a.in_im + bi * a.in_dist, a.phi, a.n, a.sgn,
                        live},
               MulBSink{q.re, q.im, a.B, nullptr});
    __syncthreads();
    run_fft<E>(S, q.t, q.re, q.im, tw, SmemConjSrc{q.re, q.im},
               ChirpSink{a.out_re + bi * a.out_dist, a.out_im + bi * a.out_dist, a.phi, a.n,
                         a.inv_inner, a.scale, a.sgn, live});
}

cudaError_t launch_bluestein(const Shape& S, const Geometry& g, const float2* tw,
                             const ConvArgs& a, cudaStream_t st) {
    if (a.batch <= 0) return cudaSuccess;
    cudaError_t e;
    if ((e = prep(k_bluestein<kE>, g.smem)) != cudaSuccess) return e;
        k_bluestein<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Rader and Bluestein whose inner length needs the four-step: the inner
// FFTs run as nested four-step plans between these element-wise passes,
// over a chunk of nb transforms b0.. of the batch, inner length m, scratch
// planes s (nb x m, packed).
// ---------------------------------------------------------------------------

namespace {

__device__ __forceinline__ long long conv_stride() { return (long long)gridDim.x * blockDim.x; }
__device__ __forceinline__ long long conv_first() {
    return (long long)blockIdx.x * blockDim.x + threadIdx.x;
}

// Rader gather: s[b][j] = x[b][rin[j]] (conjugated for an inverse)
__global__ void k_conv_gather(const ConvArgs a, long long b0, long long nb, int m, float* sr,
                              float* si) {
    for (long long e = conv_first(); e < nb * m; e += conv_stride()) {
        const long long b = e / m;
        const int j = (int)(e - b * m);
        const long long o = (b0 + b) * a.in_dist + __ldg(a.rin + j);
        sr[e] = __ldg(a.in_re + o);
        si[e] = a.sgn * __ldg(a.in_im + o);
    }
}

// Bluestein chirp: s[b][k] = x[b][k] phi[k] for k < n, 0 up to m
__global__ void k_conv_chirp_in(const ConvArgs a, long long b0, long long nb, int m, float* sr,
                                float* si) {
    for (long long e = conv_first(); e < nb * m; e += conv_stride()) {
        const long long b = e / m;
        const int k = (int)(e - b * m);
        float yr = 0.f, yi = 0.f;
        if (k < a.n) {
            const long long o = (b0 + b) * a.in_dist + k;
            const float xr = __ldg(a.in_re + o), xi = a.sgn * __ldg(a.in_im + o);
            const float2 w = __ldg(&a.phi[k]);
            yr = xr * w.x - xi * w.y;
            yi = fmaf(xr, w.y, xi * w.x);
        }
        sr[e] = yr;
        si[e] = yi;
    }
}

// s *= B, keeping s[b][0] (the sum of a Rader gather) in dc[b] when dc is set
__global__ void k_conv_mul_b(const ConvArgs a, long long nb, int m, float* sr, float* si,
                             float2* dc) {
    for (long long e = conv_first(); e < nb * m; e += conv_stride()) {
        const long long b = e / m;
        const int j = (int)(e - b * m);
        const float vr = sr[e], vi = si[e];
        if (dc && j == 0) dc[b] = make_float2(vr, vi);
        const float2 w = __ldg(&a.B[j]);
        sr[e] = vr * w.x - vi * w.y;
        si[e] = fmaf(vr, w.y, vi * w.x);
    }
}

// Rader scatter: y[b][rout[j]] = x0 + c[b][j] / m, y[b][0] = x0 + dc[b]
// (c the unnormalised inverse FFT), then the norm scale and the
// conjugation of an inverse
__global__ void k_conv_scatter(const ConvArgs a, long long b0, long long nb, int m,
                               const float* cr, const float* ci, const float2* dc) {
    for (long long e = conv_first(); e < nb * m; e += conv_stride()) {
        const long long b = e / m;
        const int j = (int)(e - b * m);
        const long long io = (b0 + b) * a.in_dist, oo = (b0 + b) * a.out_dist;
        const float x0r = __ldg(a.in_re + io), x0i = a.sgn * __ldg(a.in_im + io);
        const float yr = x0r + cr[e] * a.inv_inner, yi = x0i + ci[e] * a.inv_inner;
        const int d = __ldg(a.rout + j);
        a.out_re[oo + d] = yr * a.scale;
        a.out_im[oo + d] = a.sgn * yi * a.scale;
        if (j == 0) {
            const float2 s = dc[b];
            a.out_re[oo] = (x0r + s.x) * a.scale;
            a.out_im[oo] = a.sgn * (x0i + s.y) * a.scale;
        }
    }
}

// Bluestein: y[b][k] = phi[k] c[b][k] / m for k < n, norm scale, conjugation
__global__ void k_conv_chirp_out(const ConvArgs a, long long b0, long long nb, int m,
                                 const float* cr, const float* ci) {
    for (long long e = conv_first(); e < nb * a.n; e += conv_stride()) {
        const long long b = e / a.n;
        const int k = (int)(e - b * a.n);
        const long long si = b * m + k, oo = (b0 + b) * a.out_dist + k;
        const float vr = cr[si] * a.inv_inner, vi = ci[si] * a.inv_inner;
        const float2 w = __ldg(&a.phi[k]);
        const float yr = vr * w.x - vi * w.y, yi = fmaf(vr, w.y, vi * w.x);
        a.out_re[oo] = yr * a.scale;
        a.out_im[oo] = a.sgn * yi * a.scale;
    }
}

unsigned conv_grid(long long elems) {
    const long long blocks = (elems + 255) / 256;
    return (unsigned)std::max(1LL, std::min(blocks, 8LL * sm_count()));
}

}  // namespace

cudaError_t launch_conv_step(int step, const ConvArgs& a, long long b0, long long nb, int m,
                             float* s_re, float* s_im, float2* dc, cudaStream_t st) {
    if (nb <= 0) return cudaSuccess;
    const long long elems = nb * (step == 4 ? a.n : m);
    switch (step) {
    case 0: k_conv_gather<<<conv_grid(elems), 256, 0, st>>>(a, b0, nb, m, s_re, s_im); break;
    case 1: k_conv_chirp_in<<<conv_grid(elems), 256, 0, st>>>(a, b0, nb, m, s_re, s_im); break;
    case 2: k_conv_mul_b<<<conv_grid(elems), 256, 0, st>>>(a, nb, m, s_re, s_im, dc); break;
    case 3: k_conv_scatter<<<conv_grid(elems), 256, 0, st>>>(a, b0, nb, m, s_re, s_im, dc); break;
    case 4: k_conv_chirp_out<<<conv_grid(elems), 256, 0, st>>>(a, b0, nb, m, s_re, s_im); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace fafk
