// k_cwt.cu -- the inverse CWT's reductions over bank rows.
//
// Dual-frame inverse (reference src/faf_cwt.c:935-985): after the R2C of
// every row W_r of a signal, acc[k] = sum_r Y_r[k] * dual_r[k] in row order
// (the reference's multiply-accumulate, src/faf_cwt_kernels.c:34-52), with
// the imaginary parts of DC and Nyquist zeroed; the C2R of acc follows.
//
// L1 one-integral inverse (src/faf_cwt.c:879-930): x[i] = (sum over the
// wavelet rows of W_r[i] * dlog) / C, plus the lowpass row when the bank has
// one, in the reference's FP32 order.
//
// One thread per output element, rows walked in order: deterministic, and
// every row read coalesced.
#include <algorithm>

#include "faf_kernels_common.cuh"

namespace fafk {

namespace {

__global__ void __launch_bounds__(256) k_icwt_acc(const float* __restrict__ yr,
                                                  const float* __restrict__ yi,
                                                  const float* __restrict__ dual, long long nb,
                                                  long long ydist, long long ddist, int rows,
                                                  long long batch, float* __restrict__ ar,
                                                  float* __restrict__ ai) {
    const long long total = batch * nb;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long s = e / nb, k = e - s * nb;
        const float* pr = yr + s * rows * ydist + k;
        const float* pi = yi + s * rows * ydist + k;
        const float* pd = dual + k;
        float sr = 0.f, si = 0.f;
        for (int r = 0; r < rows; r++) {
            const float d = __ldg(pd + r * ddist);
            sr += __ldcs(pr + r * ydist) * d;
            si += __ldcs(pi + r * ydist) * d;
        }
        ar[s * nb + k] = sr;
        ai[s * nb + k] = (k == 0 || k == nb - 1) ? 0.f : si;
    }
}

__global__ void __launch_bounds__(256) k_icwt_l1(const float* __restrict__ W, long long n,
                                                 long long in_dist, int rows, int lowpass,
                                                 float dlog, float C, long long batch,
                                                 float* __restrict__ x, long long out_dist) {
    const long long total = batch * n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long s = e / n, i = e - s * n;
        const float* w = W + s * in_dist + i;
        float acc = 0.f;
        for (int r = lowpass; r < rows; r++) acc += __ldcs(w + r * n) * dlog;
        acc /= C;
        if (lowpass) acc += __ldcs(w);
        x[s * out_dist + i] = acc;
    }
}

unsigned grid_of(long long total) {
    const int sms = fafk::sm_count();
    const long long blocks = (total + 255) / 256;
    return (unsigned)std::max(1LL, std::min(blocks, (long long)sms * 8));
}

}  // namespace

cudaError_t launch_icwt_acc(const float* yr, const float* yi, const float* dual, long long nb,
                            long long ydist, long long ddist, int rows, long long batch,
                            float* ar, float* ai, cudaStream_t st) {
    if (batch <= 0) return cudaSuccess;
    k_icwt_acc<<<grid_of(batch * nb), 256, 0, st>>>(yr, yi, dual, nb, ydist, ddist, rows, batch,
                                                     ar, ai);
    return cudaGetLastError();
}

cudaError_t launch_icwt_l1(const float* W, long long n, long long in_dist, int rows, int lowpass,
                           float dlog, float C, long long batch, float* x, long long out_dist,
                           cudaStream_t st) {
    if (batch <= 0) return cudaSuccess;
    k_icwt_l1<<<grid_of(batch * n), 256, 0, st>>>(W, n, in_dist, rows, lowpass, dlog, C, batch,
                                                    x, out_dist);
    return cudaGetLastError();
}

}  // namespace fafk
