// k_pipeline.cu -- fused R2C -> spectral ops -> C2R kernel.
#include "faf_kernels_common.cuh"

namespace fafk {

// ---------------------------------------------------------------------------
// Fused pipeline: R2C -> spectral ops -> C2R, one HBM round trip
// (reference src/faf_pipeline.c:10-90 + src/chirp.c:421-471)
// ---------------------------------------------------------------------------

__device__ __forceinline__ cf apply_ops(const RealArgs& a, int k, cf v) {
#pragma unroll
    for (int o = 0; o < kMaxOps; o++) {
        if (o >= a.nops) break;
        const PipeOp& op = a.ops[o];
        if (op.code == OP_CONJ) {
            v.y = -v.y;
        } else if (op.code == OP_MUL) {
            if (k < op.m) {
                const float hr = __ldg(op.hr + k);
                if (k == 0 || k == op.m - 1) {
                    v = cf{v.x * hr, 0.f};
                } else {
                    const float hi = __ldg(op.hi_ + k);
                    v = cf{v.x * hr - v.y * hi, fmaf(v.x, hi, v.y * hr)};
                }
            }
        } else if (op.code == OP_BANDPASS) {
            if (k < op.lo || k > op.hi) v = cf{0.f, 0.f};
        }
    }
    return v;
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
    // Per bin pair: post-pass -> ops -> pre-pass, entirely in registers.
    for (int k = q.t; k <= nc / 2; k += S.T) {
        if (k == 0) {
            const cf z = mid.get(0);
            cf x0 = apply_ops(a, 0, cf{z.x + z.y, 0.f});
            cf xn = apply_ops(a, nc, cf{z.x - z.y, 0.f});
            mid.put(0, cf{x0.x + xn.x, x0.x - xn.x});
        } else {
            const float2 w = __ldg(&a.stw[k - 1]);
            cf Xk, Xnk;
            r2c_pair(mid.get(k), mid.get(nc - k), w, Xk, Xnk);
            if (k == nc - k) Xk = Xnk;
            Xk = apply_ops(a, k, Xk);
            Xnk = (k == nc - k) ? Xk : apply_ops(a, nc - k, Xnk);
            cf Zk, Znk;
            c2r_pair(Xk, Xnk, w, Zk, Znk);
            if (k != nc - k) mid.put(k, Zk);
            mid.put(nc - k, Znk);
        }
    }
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
