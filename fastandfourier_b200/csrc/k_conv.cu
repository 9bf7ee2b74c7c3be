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


}  // namespace fafk
