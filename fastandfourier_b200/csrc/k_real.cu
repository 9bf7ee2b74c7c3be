// k_real.cu -- R2C, C2R and framed STFT kernels.
#include "faf_kernels_common.cuh"

namespace fafk {

template <int E>
__global__ void __launch_bounds__(1024) k_r2c(const Shape S, const float2* __restrict__ tw,
                                              const RealArgs a, int G, bool vec) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 0);
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    RealPairSrc src{a.in_a + bi * a.in_dist, live, vec};
    const long long oo = bi * a.out_dist * (a.interleaved ? 2 : 1);
    HermSink out{a.out_a + oo, a.interleaved ? nullptr : a.out_b + oo, a.interleaved};
    r2c_body<E>(S, q, tw, a.stw, src, out, a.scale, live);
}

template <int E>
__global__ void __launch_bounds__(1024) k_stft(const Shape S, const float2* __restrict__ tw,
                                               const RealArgs a, int G) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 0);
    const long long b = (long long)blockIdx.x * G + q.g;  // global frame index
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const long long sig = bi / a.frames, f = bi - sig * a.frames;
    FrameSrc src{a.in_a + sig * a.sig_len + f * a.hop, a.window, a.win, live};
    const long long oo = bi * a.out_dist * (a.interleaved ? 2 : 1);
    HermSink out{a.out_a + oo, a.interleaved ? nullptr : a.out_b + oo, a.interleaved};
    r2c_body<E>(S, q, tw, a.stw, src, out, a.scale, live);
}

// ---------------------------------------------------------------------------
// C2R: load bins -> pre-pass -> inverse nc-point FFT -> unpack
// ---------------------------------------------------------------------------

template <int E>
__global__ void __launch_bounds__(1024) k_c2r(const Shape S, const float2* __restrict__ tw,
                                              const RealArgs a, int G, bool vec) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 0);
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const int nc = S.n;
    const SmemIO mid{q.re, q.im};
    const C2ROffsets o = c2r_offsets(a, bi, a.interleaved ? 2 : 1);
    const long long io = o.io;
    for (int k = q.t; k <= nc; k += S.T) {
        cf v{0.f, 0.f};
        if (live) {
            if (a.interleaved) {
                const float2* p = reinterpret_cast<const float2*>(a.in_a + io) + k;
                const float2 u = o.f ? __ldg(p) : __ldcs(p);
                v = cf{u.x, u.y};
            } else {
                v = o.f ? cf{__ldg(a.in_a + io + k), __ldg(a.in_b + io + k)}
                        : cf{__ldcs(a.in_a + io + k), __ldcs(a.in_b + io + k)};
            }
            if (o.f) {  // CWT row: the bank's real weight (src/faf_cwt_kernels.c:22-33)
                const float w = __ldg(o.f + k);
                v.x *= w;
                v.y *= w;
            }
        }
        mid.put(k, v);
    }
    __syncthreads();
    for (int k = q.t; k <= nc / 2; k += S.T) {
        if (k == 0) {
            const cf x0 = mid.get(0), xn = mid.get(nc);
            mid.put(0, cf{x0.x + xn.x, x0.x - xn.x});
        } else {
            cf Zk, Znk;
            c2r_pair(mid.get(k), mid.get(nc - k), __ldg(&a.stw[k - 1]), Zk, Znk);
            if (k != nc - k) mid.put(k, Zk);
            mid.put(nc - k, Znk);
        }
    }
    __syncthreads();
    RealPairSink snk{a.out_a + o.oo, a.scale, live, vec};
    run_fft<E>(S, q.t, q.re, q.im, tw, SmemConjSrc{q.re, q.im}, snk);
}

cudaError_t launch_r2c(const Shape& S, const Geometry& g, const float2* tw, const RealArgs& a,
                       cudaStream_t st) {
    const bool vec = vec_ok(a.in_a, a.in_dist);
    if (a.batch <= 0) return cudaSuccess;
    cudaError_t e;
    if ((e = prep(k_r2c<kE>, g.smem)) != cudaSuccess) return e;
        k_r2c<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G, vec);
    return cudaGetLastError();
}

cudaError_t launch_c2r(const Shape& S, const Geometry& g, const float2* tw, const RealArgs& a,
                       cudaStream_t st) {
    const bool vec = vec_ok(a.out_a, a.out_dist);
    if (a.batch <= 0) return cudaSuccess;
    cudaError_t e;
    if ((e = prep(k_c2r<kE>, g.smem)) != cudaSuccess) return e;
        k_c2r<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G, vec);
    return cudaGetLastError();
}

FAF_REAL_LAUNCH(launch_stft, k_stft)

}  // namespace fafk
