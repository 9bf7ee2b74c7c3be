// k_pipeline.cu -- fused R2C -> spectral ops -> C2R kernel.
#include "faf_kernels_common.cuh"

namespace fafk {

// ---------------------------------------------------------------------------
// Fused pipeline: R2C -> spectral ops -> C2R, one HBM round trip
// (reference src/faf_pipeline.c:10-90 + src/chirp.c:421-471)
// ---------------------------------------------------------------------------

// Per bin pair: post-pass -> ops -> pre-pass, entirely in registers.
template <class Ops>
__device__ __forceinline__ void pipe_pairs(int t, int T, int nc, const SmemIO& mid,
                                           const float2* __restrict__ stw, const Ops& ops) {
    for (int k = t; k <= nc / 2; k += T) {
        if (k == 0) {
            const cf z = mid.get(0);
            const cf x0 = ops(0, cf{z.x + z.y, 0.f});
            const cf xn = ops(nc, cf{z.x - z.y, 0.f});
            mid.put(0, cf{x0.x + xn.x, x0.x - xn.x});
        } else {
            const float2 w = __ldg(&stw[k - 1]);
            cf Xk, Xnk;
            r2c_pair(mid.get(k), mid.get(nc - k), w, Xk, Xnk);
            if (k == nc - k) Xk = Xnk;
            Xk = ops(k, Xk);
            Xnk = (k == nc - k) ? Xk : ops(nc - k, Xnk);
            cf Zk, Znk;
            c2r_pair(Xk, Xnk, w, Zk, Znk);
            if (k != nc - k) mid.put(k, Zk);
            mid.put(nc - k, Znk);
        }
    }
}

template <int E>
__global__ void __launch_bounds__(1024) k_pipeline(const Shape S, const float2* __restrict__ tw,
                                                   const RealArgs a, int G, bool vec) {
    extern __shared__ float4 smem4[];
    Group q = group_of(S, reinterpret_cast<float*>(smem4), 0);
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const int nc = S.n;
    const SmemIO mid{q.re, q.im};
    run_fft<E>(S, q.t, q.re, q.im, tw, RealPairSrc{a.in_a + bi * a.in_dist, live, vec}, mid);
    __syncthreads();
    if (ops_single_mul(a))
        pipe_pairs(q.t, S.T, nc, mid, a.stw, OpsMul1{&a.ops[0]});
    else
        pipe_pairs(q.t, S.T, nc, mid, a.stw, OpsAny{&a});
    __syncthreads();
    RealPairSink snk{a.out_a + bi * a.out_dist, a.scale, live, vec};
    run_fft<E>(S, q.t, q.re, q.im, tw, SmemConjSrc{q.re, q.im}, snk);
}

cudaError_t launch_pipeline(const Shape& S, const Geometry& g, const float2* tw,
                            const RealArgs& a, cudaStream_t st) {
    const bool vec = vec_ok(a.in_a, a.in_dist) && vec_ok(a.out_a, a.out_dist);
    if (a.batch <= 0) return cudaSuccess;
    cudaError_t e;
    if ((e = prep(k_pipeline<kE>, g.smem)) != cudaSuccess) return e;
        k_pipeline<kE><<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G, vec);
    return cudaGetLastError();
}


}  // namespace fafk
