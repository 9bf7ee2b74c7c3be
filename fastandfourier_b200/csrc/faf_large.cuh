// faf_large.cuh -- transforms longer than one CTA's shared memory (n > 16384,
// up to 65536): a four-step FFT run entirely by ONE CTA per transform through
// a per-CTA scratch region in global memory (L2-resident: grid x n x 8 bytes).
//
// n = N1 * N2, input index n2 + N2 * n1, output index k1 + N1 * k2:
//   pass 1 (columns): for each n2, Y[k1] = FFT_N1 over n1 of x[N2 n1 + n2],
//                     times W_n^{n2 k1}; store S[k1 * N2 + n2]
//   pass 2 (rows):    for each k1, X[k1 + N1 k2] = FFT_N2 over n2 of S[k1 N2 + n2]
// Pass 1 runs C1 columns at a time with the column index fastest across lanes
// (coalesced loads and stores); pass 2 runs C2 rows at a time with the element
// index fastest (coalesced loads), lands in shared memory and is copied out
// with the row index fastest (coalesced stores).  A __syncthreads between the
// passes makes the CTA's scratch writes visible to all its threads.
//
// Real transforms reuse the same passes on the packed n/2-point signal: R2C
// writes the complex result to a second scratch plane pair, then runs the
// super-twiddle post-pass from it; C2R runs the pre-pass into that plane pair
// first; the pipeline does R2C, post/ops/pre in place, then C2R.
#pragma once

#include "faf_kernels_common.cuh"

namespace fafk {
namespace lg {

using fafd::cf;
using fafd::run_fft;
using fafd::Shape;
using fafd::SmemIO;


struct Large {
    Shape s1, s2;      // N1 and N2 shapes; .T is the padded thread count
    int n1, n2, n;     // n = n1 * n2 (complex length)
    int c1, c2;        // transforms per chunk in pass 1 / pass 2
    int gstride1, gstride2;  // floats between group workspaces (odd)
    const float2* tw1;
    const float2* tw2;
    const float2* twn;  // middle twiddles, [k1 * N2 + n2] = W_n^{n2 k1}
    float* scratch;     // per CTA: 4 * n floats (S re/im, Z re/im)
};

// ---- pass-1 sources -------------------------------------------------------

struct ColSrc {  // complex split input, column n2: x[N2 * i + n2]
    const float* re;
    const float* im;
    int stride;
    float sgn;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (!live) return cf{0.f, 0.f};
        const long long o = (long long)stride * i;
        return cf{re[o], sgn * im[o]};
    }
};

struct ColPairSrc {  // packed real input z[j] = x[2j] + i x[2j+1], j = N2 * i + n2
    const float* x;
    int stride;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (!live) return cf{0.f, 0.f};
        const float2 v = *reinterpret_cast<const float2*>(x + 2LL * stride * i);
        return cf{v.x, v.y};
    }
};

// Pass-1 sink: twiddle by W_n^{n2 k1} and store S[k1 * N2 + n2].  The
// middle-twiddle table is laid out like S (entry k1 * N2 + n2), so lanes
// holding consecutive columns read and write consecutive addresses.
struct ColTwSink {
    float* sr;
    float* si;
    const float2* twm;
    int col, n2;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int k1, cf v) const {
        if (!live) return;
        const int o = k1 * n2 + col;
        const float2 w = __ldg(&twm[o]);
        sr[o] = v.x * w.x - v.y * w.y;
        si[o] = fmaf(v.x, w.y, v.y * w.x);
    }
};

struct RowSrc {  // S row: contiguous
    const float* re;
    const float* im;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (!live) return cf{0.f, 0.f};
        return cf{re[i], im[i]};
    }
};

// Run the complex four-step of one transform; `src1` supplies pass-1
// columns via make(col, live); results go to `out(k, v)` for k = k1 + N1 k2.
template <class MakeSrc, class Out>
__device__ __forceinline__ void four_step(const Large& L, float* sm, const MakeSrc& make_src,
                                          const Out& out) {
    float* Sr = L.scratch;
    float* Si = Sr + L.n;
    // ---- pass 1: columns, column index fastest across lanes
    {
        const int g = threadIdx.x % L.c1, t = threadIdx.x / L.c1;
        float* re = sm + (size_t)g * L.gstride1;
        float* im = re + L.s1.plane;
#pragma unroll 1
        for (int c0 = 0; c0 < L.n2; c0 += L.c1) {
            const int col = c0 + g;
            const bool live = col < L.n2;
            run_fft<16>(L.s1, t, re, im, L.tw1, make_src(col, live),
                        ColTwSink{Sr, Si, L.twn, col, L.n2, live});
        }
    }
    __syncthreads();
    // ---- pass 2: rows, element index fastest; copy-out row index fastest
    {
        const int g = threadIdx.x / L.s2.T, t = threadIdx.x % L.s2.T;
        float* re = sm + (size_t)g * L.gstride2;
        float* im = re + L.s2.plane;
#pragma unroll 1
        for (int r0 = 0; r0 < L.n1; r0 += L.c2) {
            const int row = r0 + g;
            const bool live = row < L.n1;
            run_fft<16>(L.s2, t, re, im, L.tw2,
                        RowSrc{Sr + (long long)row * L.n2, Si + (long long)row * L.n2, live},
                        SmemIO{re, im});
            __syncthreads();
            const int rows = min(L.c2, L.n1 - r0);
            if (rows == L.c2) {  // c2 is a power of two: shift / mask
                const int lc = __ffs(L.c2) - 1;
                for (int e = threadIdx.x; e < rows * L.n2; e += blockDim.x) {
                    const int c = e & (L.c2 - 1), k2 = e >> lc;
                    const float* wr = sm + (size_t)c * L.gstride2;
                    const int p = fafd::pad(k2);
                    out(r0 + c + L.n1 * k2, cf{wr[p], wr[L.s2.plane + p]});
                }
            } else {
                for (int e = threadIdx.x; e < rows * L.n2; e += blockDim.x) {
                    const int c = e % rows, k2 = e / rows;
                    const float* wr = sm + (size_t)c * L.gstride2;
                    const int p = fafd::pad(k2);
                    out(r0 + c + L.n1 * k2, cf{wr[p], wr[L.s2.plane + p]});
                }
            }
            __syncthreads();
        }
    }
}

struct MakeColSrc {
    const float* re;
    const float* im;
    int n2;
    float sgn;
    __device__ __forceinline__ ColSrc operator()(int col, bool live) const {
        return ColSrc{re + col, im + col, n2, sgn, live};
    }
};

struct MakeColPairSrc {
    const float* x;
    int n2;
    __device__ __forceinline__ ColPairSrc operator()(int col, bool live) const {
        return ColPairSrc{x + 2 * col, n2, live};
    }
};

struct MakeColZSrc {  // pass-1 columns of the packed spectrum in scratch Z (conjugated)
    const float* zr;
    const float* zi;
    int n2;
    __device__ __forceinline__ ColSrc operator()(int col, bool live) const {
        return ColSrc{zr + col, zi + col, n2, -1.0f, live};
    }
};

struct OutSplit {
    float* re;
    float* im;
    float scale, sgn;
    __device__ __forceinline__ void operator()(int k, cf v) const {
        re[k] = v.x * scale;
        im[k] = sgn * v.y * scale;
    }
};

struct OutScratch {  // plain store into a scratch plane pair
    float* re;
    float* im;
    __device__ __forceinline__ void operator()(int k, cf v) const {
        re[k] = v.x;
        im[k] = v.y;
    }
};

struct OutRealPairs {  // C2R unpack: undo the conjugation, y[2k], y[2k+1]
    float* y;
    float scale;
    __device__ __forceinline__ void operator()(int k, cf v) const {
        *reinterpret_cast<float2*>(y + 2LL * k) = make_float2(v.x * scale, -v.y * scale);
    }
};

// Source / sink pair chosen at run time, so a kernel that runs the four-step
// twice (forward, then inverse) instantiates it once: two instantiations in
// one kernel spill.  Pairs mode reads packed real pairs z[j] = x[2j] +
// i x[2j+1] / writes y[2k], y[2k+1] = (re, -im) * scale; split mode reads
// (re, sgn * im) planes / writes plain planes.
struct ColAnySrc {
    const float* a;
    const float* b;
    int stride;
    float sgn;
    bool pairs, live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (!live) return cf{0.f, 0.f};
        const long long o = (long long)stride * i;
        if (pairs) {
            const float2 v = *reinterpret_cast<const float2*>(a + 2 * o);
            return cf{v.x, v.y};
        }
        return cf{a[o], sgn * b[o]};
    }
};

struct MakeColAny {
    const float* a;
    const float* b;
    int n2;
    float sgn;
    bool pairs;
    __device__ __forceinline__ ColAnySrc operator()(int col, bool live) const {
        return ColAnySrc{pairs ? a + 2 * col : a + col, pairs ? b : b + col, n2, sgn, pairs, live};
    }
};

struct OutAny {
    float* a;
    float* b;
    float scale;
    bool pairs;
    __device__ __forceinline__ void operator()(int k, cf v) const {
        if (pairs) {
            *reinterpret_cast<float2*>(a + 2LL * k) = make_float2(v.x * scale, -v.y * scale);
        } else {
            a[k] = v.x;
            b[k] = v.y;
        }
    }
};

__device__ __forceinline__ Large make_large(const LargeArgs& a) {
    Large L;
    L.s1 = a.s1;
    L.s2 = a.s2;
    L.n1 = a.n1;
    L.n2 = a.n2;
    L.n = a.n1 * a.n2;
    L.c1 = blockDim.x / a.s1.T;
    L.c2 = blockDim.x / a.s2.T;
    L.gstride1 = (2 * a.s1.plane) | 1;
    L.gstride2 = (2 * a.s2.plane) | 1;
    L.tw1 = a.tw1;
    L.tw2 = a.tw2;
    L.twn = a.twn;
    L.scratch = a.scratch + (size_t)blockIdx.x * a.cta_floats;
    return L;
}

// Post-pass from Z (scratch) to the Hermitian output, pairs (k, nc - k).
__device__ __forceinline__ void large_post(const float* zr, const float* zi, int nc,
                                           const float2* stw, float* Xr, float* Xi,
                                           float scale) {
    for (int k = threadIdx.x; k <= nc / 2; k += blockDim.x) {
        if (k == 0) {
            Xr[0] = (zr[0] + zi[0]) * scale;
            Xi[0] = 0.f;
            Xr[nc] = (zr[0] - zi[0]) * scale;
            Xi[nc] = 0.f;
        } else {
            cf Xk, Xnk;
            r2c_pair(cf{zr[k], zi[k]}, cf{zr[nc - k], zi[nc - k]}, __ldg(&stw[k - 1]), Xk, Xnk);
            if (k != nc - k) { Xr[k] = Xk.x * scale; Xi[k] = Xk.y * scale; }
            Xr[nc - k] = Xnk.x * scale;
            Xi[nc - k] = Xnk.y * scale;
        }
    }
}


// Pre-pass of the C2R from the Hermitian input X into Z (scratch).
__device__ __forceinline__ void large_pre(const float* Xr, const float* Xi, int nc,
                                          const float2* stw, float* zr, float* zi) {
    for (int k = threadIdx.x; k <= nc / 2; k += blockDim.x) {
        if (k == 0) {
            const float x0 = Xr[0], xn = Xr[nc];
            zr[0] = x0 + xn;
            zi[0] = x0 - xn;
        } else {
            cf Zk, Znk;
            c2r_pair(cf{Xr[k], Xi[k]}, cf{Xr[nc - k], Xi[nc - k]}, __ldg(&stw[k - 1]), Zk, Znk);
            if (k != nc - k) { zr[k] = Zk.x; zi[k] = Zk.y; }
            zr[nc - k] = Znk.x;
            zi[nc - k] = Znk.y;
        }
    }
}


template <class K, class A>
inline cudaError_t launch4(K kernel, const LargeArgs& a, const A& args, int grid,
                           cudaStream_t st) {
    const size_t smem = large_smem(a, kLargeThreads);
    cudaError_t e = prep(kernel, smem);
    if (e != cudaSuccess) return e;
    kernel<<<grid, kLargeThreads, smem, st>>>(a, args);
    return cudaGetLastError();
}

// C2R and pipeline launchers (k_large2.cu).
cudaError_t launch_large_c2r(const LargeArgs& a, const RealArgs& r, int grid, cudaStream_t st);
cudaError_t launch_large_pipeline(const LargeArgs& a, const RealArgs& r, int grid,
                                  cudaStream_t st);

}  // namespace lg
}  // namespace fafk
