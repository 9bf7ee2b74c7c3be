// k_large.cu -- four-step kernels for C2C and R2C longer than one CTA (the
// algorithm is described in faf_large.cuh), and the launcher of the family.
#include "faf_large.cuh"

namespace fafk {
using namespace lg;

__global__ void __launch_bounds__(512) k4_c2c(const LargeArgs a, const C2CArgs c) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const Large L = make_large(a);
    for (long long b = blockIdx.x; b < c.batch; b += gridDim.x) {
        __syncthreads();
        four_step(L, sm, MakeColSrc{c.in_re + b * c.in_dist, c.in_im + b * c.in_dist, L.n2, c.sgn},
                  OutSplit{c.out_re + b * c.out_dist, c.out_im + b * c.out_dist, c.scale, c.sgn});
    }
}

__global__ void __launch_bounds__(512) k4_r2c(const LargeArgs a, const RealArgs r) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const Large L = make_large(a);
    float* zr = L.scratch + 2 * L.n;
    float* zi = zr + L.n;
    for (long long b = blockIdx.x; b < r.batch; b += gridDim.x) {
        __syncthreads();
        four_step(L, sm, MakeColPairSrc{r.in_a + b * r.in_dist, L.n2}, OutScratch{zr, zi});
        __syncthreads();
        large_post(zr, zi, L.n, r.stw, r.out_a + b * r.out_dist, r.out_b + b * r.out_dist,
                   r.scale);
    }
}

// ---------------------------------------------------------------------------

size_t large_smem(const LargeArgs& a, int threads) {
    const int c1 = threads / a.s1.T, c2 = threads / a.s2.T;
    const size_t g1 = (size_t)c1 * ((2 * a.s1.plane) | 1);
    const size_t g2 = (size_t)c2 * ((2 * a.s2.plane) | 1);
    return (g1 > g2 ? g1 : g2) * sizeof(float);
}

cudaError_t large_c2c_prepare(const LargeArgs& a) {
    cudaError_t e = prep(k4_c2c, large_smem(a, kLargeThreads));
    if (e != cudaSuccess) return e;
    // querying the kernel loads its module now (under lazy module loading it
    // would otherwise load at the first launch)
    cudaFuncAttributes fa;
    return cudaFuncGetAttributes(&fa, k4_c2c);
}

cudaError_t launch_large(int kind, const LargeArgs& a, const void* args, long long batch,
                         int grid, cudaStream_t st) {
    if (batch <= 0) return cudaSuccess;
    switch (kind) {
    case 0: return launch4(k4_c2c, a, *(const C2CArgs*)args, grid, st);
    case 1: return launch4(k4_r2c, a, *(const RealArgs*)args, grid, st);
    case 2: return launch_large_c2r(a, *(const RealArgs*)args, grid, st);
    case 3: return launch_large_pipeline(a, *(const RealArgs*)args, grid, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace fafk
