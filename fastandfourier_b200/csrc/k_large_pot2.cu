// k_large_pot2.cu -- batched four-step C2C for power-of-two lengths above
// one CTA (n = N1 * N2: 32768 = 128 x 256, 65536 = 256 x 256), spread over
// many CTAs per transform in two passes through a scratch buffer:
//
//   pass 1 (k4p_col): a CTA takes W = TH / (N1/16) columns of one
//     transform: a cooperative load with the column index fastest across
//     lanes (coalesced rows of W floats) transposes them into one shared
//     workspace per column; each column runs an N1-point FFT on the
//     compile-time engine; a cooperative copy-out multiplies the middle
//     twiddle W_n^{col k1} (table laid out [k1][col]) and stores
//     S[k1 * N2 + col], again W consecutive floats per row.
//   pass 2 (k4p_row): a CTA takes W2 = TH / (N2/16) rows of S (contiguous,
//     read straight into the engine), runs N2-point FFTs, and a cooperative
//     copy-out stores X[k1 + N1 k2] with the row index fastest (W2 consecutive
//     floats per k2).
//
// The batch runs in chunks whose scratch (2 n floats per transform) stays
// L2-resident between the two passes, so HBM sees each input read once and
// each output written once.  Column workspaces are an odd number of float2
// apart, so the transposing accesses of a warp (lanes on consecutive
// columns) hit distinct banks.
#include <algorithm>
#include <cstdlib>

#include "faf_kernels_common.cuh"
#include "faf_pot2.cuh"
#include "faf_pot2_group.cuh"

namespace fafk {
namespace l2p {

using fafct::cf;
using fafct::ct_fft;
using fafct::pad2;
using fafct::SmemC;

constexpr long long kScratchBytes = 64ll << 20;  // per chunk: stays in L2 between passes

// TH threads per CTA (1024, or 512 with two CTAs per SM)
template <int N, int TH = 1024>
struct Cols {
    static constexpr int T = P2<N>::T;         // threads per sub-FFT
    static constexpr int W = TH / T;           // sub-FFTs per CTA
    static constexpr int STR = plane2(N) | 1;  // float2 between workspaces (odd)
    static constexpr size_t smem() {
        return (size_t)CtCfg<N>::TWN * sizeof(float2) + (size_t)W * STR * sizeof(float2);
    }
};

// Shared-memory setup common to both passes: twiddle table (when it fits)
// and this thread's sub-FFT workspace.
template <int N>
struct Setup {
    float2* ws0;  // workspace of sub-FFT 0
    float2* ws;   // this thread's sub-FFT
    const float2* tw;
    int g, t;
    fafct::GroupSync sync;
    __device__ __forceinline__ Setup(float2* sm, const float2* __restrict__ gtw) {
        constexpr int T = Cols<N>::T;
        g = threadIdx.x / T;
        t = threadIdx.x % T;
        if constexpr (CtCfg<N>::TW_SMEM) {
            for (int i = threadIdx.x; i < CtCfg<N>::TWN; i += blockDim.x) sm[i] = __ldg(&gtw[i]);
            tw = sm;
        } else {
            tw = gtw;
        }
        ws0 = sm + CtCfg<N>::TWN;
        ws = ws0 + (size_t)g * Cols<N>::STR;
        sync = fafct::GroupSync::make(g, T);
    }
};

struct PlaneSrc {  // contiguous split planes (a row of the scratch)
    const float* re;
    const float* im;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const { return cf{re[i], im[i]}; }
};

__device__ __forceinline__ long long xform_off(const Large2Args& a, long long b, bool out) {
    if (a.offs) return a.offs[b];
    return b * (out ? a.out_dist : a.in_dist);
}

template <int N1, int N2, int TH>
__global__ void __launch_bounds__(TH, 1024 / TH)
    k4p_col(const Large2Args a, long long b0, long long nb) {
    constexpr int W = Cols<N1, TH>::W, STR = Cols<N1>::STR, NCB = N2 / W;
    constexpr long long n = (long long)N1 * N2;
    extern __shared__ float4 smem4[];
    Setup<N1> q(reinterpret_cast<float2*>(smem4), a.tws1);
    for (long long task = blockIdx.x; task < nb * NCB; task += gridDim.x) {
        const long long bl = task / NCB;
        const int c0 = (int)(task % NCB) * W;
        const long long off = xform_off(a, b0 + bl, false);
        const float* xr = a.in_re + off + c0;
        const float* xi = a.in_im + off + c0;
        __syncthreads();  // the workspaces are free
        for (int e = threadIdx.x; e < N1 * W; e += TH) {
            const int row = e / W, col = e % W;
            q.ws0[col * STR + pad2(row)] =
                make_float2(__ldcs(xr + (long long)row * N2 + col),
                            a.sgn * __ldcs(xi + (long long)row * N2 + col));
        }
        __syncthreads();
        ct_fft<N1, kTw<N1>>(q.t, q.ws, q.tw, SmemC{q.ws}, SmemC{q.ws}, q.sync);
        __syncthreads();
        float* sr = a.scratch + bl * 2 * n;
        float* si = sr + n;
        for (int e = threadIdx.x; e < N1 * W; e += TH) {
            const int k1 = e / W, col = e % W;
            const float2 v = q.ws0[col * STR + pad2(k1)];
            const int o = k1 * N2 + c0 + col;
            const float2 w = __ldg(&a.twm[o]);
            sr[o] = v.x * w.x - v.y * w.y;
            si[o] = fmaf(v.x, w.y, v.y * w.x);
        }
    }
}

template <int N1, int N2, int TH>
__global__ void __launch_bounds__(TH, 1024 / TH)
    k4p_row(const Large2Args a, long long b0, long long nb) {
    constexpr int W = Cols<N2, TH>::W, STR = Cols<N2>::STR, NRB = N1 / W;
    constexpr long long n = (long long)N1 * N2;
    extern __shared__ float4 smem4[];
    Setup<N2> q(reinterpret_cast<float2*>(smem4), a.tws2);
    for (long long task = blockIdx.x; task < nb * NRB; task += gridDim.x) {
        const long long bl = task / NRB;
        const int r0 = (int)(task % NRB) * W;
        const float* sr = a.scratch + bl * 2 * n;
        const float* si = sr + n;
        const long long row = r0 + q.g;
        __syncthreads();  // the workspaces are free
        ct_fft<N2, kTw<N2>>(q.t, q.ws, q.tw, PlaneSrc{sr + row * N2, si + row * N2}, SmemC{q.ws},
                            q.sync);
        __syncthreads();
        const long long off = xform_off(a, b0 + bl, true);
        float* yr = a.out_re + off + r0;
        float* yi = a.out_im + off + r0;
        const float sim = a.sgn * a.scale;
        for (int e = threadIdx.x; e < N2 * W; e += TH) {
            const int k2 = e / W, g = e % W;
            const float2 v = q.ws0[g * STR + pad2(k2)];
            __stcs(yr + (long long)N1 * k2 + g, v.x * a.scale);
            __stcs(yi + (long long)N1 * k2 + g, v.y * sim);
        }
    }
}

// Threads per CTA of both passes.  The CTAs of an SM drift apart, so some
// load their columns while others compute.  Measured on B200 (65536-point
// C2C, batch 512 / 32768, batch 1024 / the uneven graph), in GB/s:
//   one CTA of 1024:   1636 / 1528 / 1651
//   two CTAs of 512:   1900 / 1786 / 1872
//   four CTAs of 256:  2044 / 1986 / 1767
// A standalone batch takes 256; the uneven graph, whose other branch needs
// SMs of its own, takes 512 (`want`).  FAF_CUDA_4STEP_THREADS overrides both.
inline int cta_threads(int want) {
    const char* e = std::getenv("FAF_CUDA_4STEP_THREADS");
    const int v = e ? atoi(e) : (want ? want : 256);
    return (v == 1024 || v == 512) ? v : 256;
}

// Kernel attributes (dynamic shared memory above 48 KB), set once per
// device (prep memoises them) and before any stream capture reaches the
// launches.
template <int N1, int N2, int TH>
cudaError_t prepare_pair() {
    cudaError_t e = prep(k4p_col<N1, N2, TH>, Cols<N1, TH>::smem());
    if (e == cudaSuccess) e = prep(k4p_row<N1, N2, TH>, Cols<N2, TH>::smem());
    return e;
}

// The same, and the kernels' module loaded on the current device now rather
// than at the first launch (lazy module loading): for callers that must not
// allocate when they launch.
template <int N1, int N2, int TH>
cudaError_t load_pair() {
    cudaError_t e = prepare_pair<N1, N2, TH>();
    cudaFuncAttributes fa;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k4p_col<N1, N2, TH>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&fa, k4p_row<N1, N2, TH>);
    return e;
}

template <int N1, int N2, int TH>
cudaError_t launch_pair_t(const Large2Args& a, cudaStream_t st) {
    static_assert(N1 * N2 >= 16384 && N2 % Cols<N1, TH>::W == 0 && N1 % Cols<N2, TH>::W == 0,
                  "column / row blocks must tile the transform");
    constexpr size_t sm1 = Cols<N1, TH>::smem(), sm2 = Cols<N2, TH>::smem();
    cudaError_t e = prepare_pair<N1, N2, TH>();
    if (e != cudaSuccess) return e;
    const int sms = fafk::sm_count();
    // chunks of equal size (at most scratch_transforms each), so that no
    // chunk is a short tail that fills only part of the GPU
    const long long cap = std::max(1LL, a.scratch_transforms);
    const long long nch = (a.batch + cap - 1) / cap;
    const long long chunk = (a.batch + nch - 1) / nch;
    for (long long b0 = 0; b0 < a.batch; b0 += chunk) {
        const long long nb = std::min(chunk, a.batch - b0);
        const long long t1 = nb * (N2 / Cols<N1, TH>::W), t2 = nb * (N1 / Cols<N2, TH>::W);
        k4p_col<N1, N2, TH><<<(unsigned)std::min<long long>(t1, 8LL * sms), TH, sm1, st>>>(a, b0, nb);
        k4p_row<N1, N2, TH><<<(unsigned)std::min<long long>(t2, 8LL * sms), TH, sm2, st>>>(a, b0, nb);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

template <int N1, int N2>
cudaError_t launch_pair(const Large2Args& a, cudaStream_t st, int want) {
    switch (cta_threads(want)) {
    case 1024: return launch_pair_t<N1, N2, 1024>(a, st);
    case 256: return launch_pair_t<N1, N2, 256>(a, st);
    default: return launch_pair_t<N1, N2, 512>(a, st);
    }
}

template <int N1, int N2>
cudaError_t load_both() {
    cudaError_t e = load_pair<N1, N2, 1024>();
    if (e == cudaSuccess) e = load_pair<N1, N2, 512>();
    return e == cudaSuccess ? load_pair<N1, N2, 256>() : e;
}

}  // namespace l2p

bool large_pot2_supported(int n1, int n2) {
    return (n1 == 128 && n2 == 128) || (n1 == 128 && n2 == 256) || (n1 == 256 && n2 == 256);
}

long long large_pot2_chunk(long long n) {
    return std::max(1LL, l2p::kScratchBytes / (long long)(2 * n * sizeof(float)));
}

int large_pot2_launches(int n1, int n2, long long batch) {
    const long long c = large_pot2_chunk((long long)n1 * n2);
    return (int)(2 * ((batch + c - 1) / c));
}

cudaError_t large_pot2_prepare(int n1, int n2) {
    if (n1 == 128 && n2 == 128) return l2p::load_both<128, 128>();
    if (n1 == 128 && n2 == 256) return l2p::load_both<128, 256>();
    if (n1 == 256 && n2 == 256) return l2p::load_both<256, 256>();
    return cudaErrorInvalidValue;
}

cudaError_t launch_large_pot2(int n1, int n2, const Large2Args& a, cudaStream_t st,
                              int threads) {
    if (a.batch <= 0) return cudaSuccess;
    if (n1 == 128 && n2 == 128) return l2p::launch_pair<128, 128>(a, st, threads);
    if (n1 == 128 && n2 == 256) return l2p::launch_pair<128, 256>(a, st, threads);
    if (n1 == 256 && n2 == 256) return l2p::launch_pair<256, 256>(a, st, threads);
    return cudaErrorInvalidValue;
}

}  // namespace fafk
