// k_istft.cu -- overlap-add of the inverse STFT (no counterpart in the
// reference, whose faf_create_inverse of an STFT returns another forward
// STFT, src/faf_core.c:1122-1123).
//
// The frames have already been through the batched C2R (1/n scaled) into
// tmp[(s F + f) n + j]; output sample t of signal s is the weighted
// overlap-add of every frame f with f hop <= t < f hop + win:
//     y[t] = sum_f w[t - f hop] tmp_f[t - f hop] / sum_f w[t - f hop]^2
// and 0 where that window envelope is below 1e-10 (the ends of a symmetric
// Hann window, w[0] = 0).  One thread per output sample sums its frames in
// frame order, so the result does not depend on the launch.
#include <algorithm>

#include "faf_kernels_common.cuh"

namespace fafk {

__global__ void k_ola(const float* __restrict__ tmp, const float* __restrict__ w, int n, int win,
                      int hop, long long F, long long L, float* __restrict__ y, long long n_sig) {
    const long long total = n_sig * L;
    for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < total;
         idx += (long long)gridDim.x * blockDim.x) {
        const long long s = idx / L, t = idx - s * L;
        const long long f_hi = min(F - 1, t / hop);
        const long long f_lo = t >= win ? (t - win) / hop + 1 : 0;
        float sum = 0.f, env = 0.f;
        for (long long f = f_lo; f <= f_hi; f++) {
            const int j = (int)(t - f * hop);
            const float wj = __ldg(&w[j]);
            sum = fmaf(wj, __ldg(&tmp[(s * F + f) * n + j]), sum);
            env = fmaf(wj, wj, env);
        }
        y[idx] = env > 1e-10f ? sum / env : 0.f;
    }
}

// The same sums with the signal taken from blockIdx.y and the sample index in
// 32 bits (L < 2^30): k_ola's three 64-bit divisions per sample are most of
// its instructions.  A power-of-two hop (POW2, lh = log2 hop) divides by a
// shift.  With MAXF > 0 (every sample covered by at most MAXF frames) the
// frame loop is unrolled, so a thread's frame loads are in flight together.
// Frame order and arithmetic are k_ola's, so the results are identical.
template <bool POW2, int MAXF>
__global__ void k_ola32(const float* __restrict__ tmp, const float* __restrict__ w, int n,
                        int win, int hop, int lh, int F, int L, float* __restrict__ y,
                        long long n_sig) {
    const unsigned uh = (unsigned)hop;
    auto div = [&](int v) -> int { return POW2 ? (v >> lh) : (int)((unsigned)v / uh); };
    for (long long s = blockIdx.y; s < n_sig; s += gridDim.y) {
        const float* __restrict__ ts = tmp + s * (long long)F * n;
        float* __restrict__ ys = y + s * (long long)L;
        for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < L; t += gridDim.x * blockDim.x) {
            const int f_hi = min(F - 1, div(t));
            const int f_lo = t >= win ? div(t - win) + 1 : 0;
            float sum = 0.f, env = 0.f;
            if constexpr (MAXF > 0) {
                float wv[MAXF], xv[MAXF];
                // every load in range (frames past f_hi read a clamped
                // element, whose value the sums below skip)
#pragma unroll
                for (int i = 0; i < MAXF; i++) {
                    const int f = min(f_lo + i, F - 1);
                    const int j = min(max(t - f * hop, 0), win - 1);
                    wv[i] = __ldg(&w[j]);
                    xv[i] = __ldg(&ts[(long long)f * n + j]);
                }
#pragma unroll
                for (int i = 0; i < MAXF; i++) {
                    if (f_lo + i <= f_hi) {
                        sum = fmaf(wv[i], xv[i], sum);
                        env = fmaf(wv[i], wv[i], env);
                    }
                }
            } else {
                for (int f = f_lo; f <= f_hi; f++) {
                    const int j = t - f * hop;
                    const float wj = __ldg(&w[j]);
                    sum = fmaf(wj, __ldg(&ts[(long long)f * n + j]), sum);
                    env = fmaf(wj, wj, env);
                }
            }
            ys[t] = env > 1e-10f ? sum / env : 0.f;
        }
    }
}

cudaError_t launch_ola(const float* tmp, const float* w, int n, int win, int hop, long long F,
                       long long L, float* y, long long n_sig, cudaStream_t st) {
    const long long total = n_sig * L;
    if (total <= 0) return cudaSuccess;
    constexpr long long kBlocks = 148LL * 16;
    if (L < (1LL << 30) && F < (1LL << 30)) {
        const long long gy = std::min<long long>(n_sig, 65535);
        const long long gx =
            std::max<long long>(1, std::min<long long>((L + 255) / 256, (kBlocks + gy - 1) / gy));
        const dim3 grid((unsigned)gx, (unsigned)gy);
        int lh = 0;
        while ((1 << lh) < hop) lh++;
        // frames covering one sample: at most ceil(win / hop)
        const int cover = (win + hop - 1) / hop;
        const bool p2 = (1 << lh) == hop;
        auto go = [&](auto kernel) {
            kernel<<<grid, 256, 0, st>>>(tmp, w, n, win, hop, p2 ? lh : 0, (int)F, (int)L, y,
                                         n_sig);
        };
        if (cover <= 4)
            p2 ? go(k_ola32<true, 4>) : go(k_ola32<false, 4>);
        else if (cover <= 8)
            p2 ? go(k_ola32<true, 8>) : go(k_ola32<false, 8>);
        else
            p2 ? go(k_ola32<true, 0>) : go(k_ola32<false, 0>);
        return cudaGetLastError();
    }
    const long long blocks = std::min<long long>((total + 255) / 256, kBlocks);
    k_ola<<<(unsigned)blocks, 256, 0, st>>>(tmp, w, n, win, hop, F, L, y, n_sig);
    return cudaGetLastError();
}

}  // namespace fafk
