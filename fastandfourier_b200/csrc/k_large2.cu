// k_large2.cu -- four-step kernels for C2R and the fused pipeline longer than
// one CTA (the algorithm is described in faf_large.cuh).
#include "faf_large.cuh"

namespace fafk {
using namespace lg;

__global__ void __launch_bounds__(512) k4_c2r(const LargeArgs a, const RealArgs r) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const Large L = make_large(a);
    float* zr = L.scratch + 2 * L.n;
    float* zi = zr + L.n;
    for (long long b = blockIdx.x; b < r.batch; b += gridDim.x) {
        __syncthreads();
        large_pre(r.in_a + b * r.in_dist, r.in_b + b * r.in_dist, L.n, r.stw, zr, zi);
        __syncthreads();
        four_step(L, sm, MakeColZSrc{zr, zi, L.n2}, OutRealPairs{r.out_a + b * r.out_dist, r.scale});
    }
}

// Forward four-step into Z, the post-pass / ops / pre-pass in place on Z,
// then the inverse four-step from Z: one four-step instantiation run twice.
__global__ void __launch_bounds__(512) k4_pipeline(const LargeArgs a, const RealArgs r) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const Large L = make_large(a);
    float* zr = L.scratch + 2 * L.n;
    float* zi = zr + L.n;
    const int nc = L.n;
    for (long long b = blockIdx.x; b < r.batch; b += gridDim.x) {
#pragma unroll 1
        for (int ph = 0; ph < 2; ph++) {
            __syncthreads();
            if (ph == 1) {
                for (int k = threadIdx.x; k <= nc / 2; k += blockDim.x) {
                    if (k == 0) {
                        const cf x0 = apply_pipe_ops(r, 0, cf{zr[0] + zi[0], 0.f});
                        const cf xn = apply_pipe_ops(r, nc, cf{zr[0] - zi[0], 0.f});
                        zr[0] = x0.x + xn.x;
                        zi[0] = x0.x - xn.x;
                    } else {
                        const float2 w = __ldg(&r.stw[k - 1]);
                        cf Xk, Xnk;
                        r2c_pair(cf{zr[k], zi[k]}, cf{zr[nc - k], zi[nc - k]}, w, Xk, Xnk);
                        if (k == nc - k) Xk = Xnk;
                        Xk = apply_pipe_ops(r, k, Xk);
                        Xnk = (k == nc - k) ? Xk : apply_pipe_ops(r, nc - k, Xnk);
                        cf Zk, Znk;
                        c2r_pair(Xk, Xnk, w, Zk, Znk);
                        if (k != nc - k) { zr[k] = Zk.x; zi[k] = Zk.y; }
                        zr[nc - k] = Znk.x;
                        zi[nc - k] = Znk.y;
                    }
                }
                __syncthreads();
            }
            const bool fwd = ph == 0;
            four_step(L, sm,
                      fwd ? MakeColAny{r.in_a + b * r.in_dist, nullptr, L.n2, 1.0f, true}
                          : MakeColAny{zr, zi, L.n2, -1.0f, false},
                      fwd ? OutAny{zr, zi, 1.0f, false}
                          : OutAny{r.out_a + b * r.out_dist, nullptr, r.scale, true});
        }
    }
}

namespace lg {

cudaError_t launch_large_c2r(const LargeArgs& a, const RealArgs& r, int grid, cudaStream_t st) {
    return launch4(k4_c2r, a, r, grid, st);
}

cudaError_t launch_large_pipeline(const LargeArgs& a, const RealArgs& r, int grid,
                                  cudaStream_t st) {
    return launch4(k4_pipeline, a, r, grid, st);
}

}  // namespace lg
}  // namespace fafk
