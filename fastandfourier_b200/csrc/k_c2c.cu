// k_c2c.cu -- batched single-CTA C2C kernel.
#include "faf_kernels_common.cuh"

namespace fafk {

// ---------------------------------------------------------------------------
// C2C
// ---------------------------------------------------------------------------

template <int E>
__global__ void __launch_bounds__(1024) k_c2c(const Shape S, const float2* __restrict__ tw,
                                              const C2CArgs a, int G) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 0);
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const long long io = bi * a.in_dist * (a.interleaved ? 2 : 1);
    const long long oo = bi * a.out_dist * (a.interleaved ? 2 : 1);
    SplitSrc src{a.in_re + io, a.interleaved ? nullptr : a.in_im + io, a.window, a.sgn,
                 a.interleaved, live};
    SplitSink snk{a.out_re + oo, a.interleaved ? nullptr : a.out_im + oo, a.scale, a.sgn,
                  a.interleaved, live};
    run_fft<E>(S, q.t, q.re, q.im, tw, src, snk);
}

cudaError_t launch_c2c(const Shape& S, const Geometry& g, const float2* tw, const C2CArgs& a,
                       cudaStream_t st) {
    if (a.batch <= 0) return cudaSuccess;
    cudaError_t e;
    if ((e = prep(k_c2c<kE>, g.smem)) != cudaSuccess) return e;
        k_c2c<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G);
    return cudaGetLastError();
}


}  // namespace fafk
