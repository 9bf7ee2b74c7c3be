// k_tc64.cu -- tensor-core precision form of the 4096-, 8192- and 16384-point
// C2C with 64-point DFTs as tcgen05 MMAs: two passes through shared memory
// instead of the radix-16 form's four.
//
// N = 64 R0 * 64 (R0 = 1, 2, 4), n = b + 64 j (b < 64, j < 64 R0),
// k = kk + 64 R0 m (kk < 64 R0, m < 64):
//   stage A  Y[b][kk] = sum_j x[b + 64 j] W_{64 R0}^{j kk}, a 64 R0-point DFT
//            over j = j0 + 64 i: the radix-R0 butterflies over i and the
//            W_{64 R0}^{j0 k0} twiddles run on the CUDA cores while the A
//            tile is built, the 64-point DFT over j0 on the tensor cores
//            (kk = k0 + R0 k1);
//   stage B  X[kk + 64 R0 m] = sum_b (Y[b][kk] W_N^{b kk}) W_64^{b m}, a
//            64-point DFT over b on the tensor cores, stored to HBM from
//            TMEM.
// Each stage is the real product D[256 x 128] = A[256 x 128] B^T over two
// M = 128 tiles: an A row holds one DFT's 64 inputs as (re, im) pairs along
// K, B = the 64-point forward DFT as a 128 x 128 real matrix, a D row the 64
// outputs as (re, im) pairs.  A CTA of 1024 threads holds 4 / R0 transforms;
// either stage has 256 DFT rows per CTA.
//
// Precision as in the radix-16 form: A and B are FP16 hi + lo, D accumulates
// A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32.  Stage A scales the rows of one
// b (all k0) by one power of two, stage B each row by its own, from the
// largest magnitude that the row's threads exchange through shared memory.
//
// Shared memory (227,360 bytes + the landing control):
//   [0, 135168)   the workspace: the landed inputs (G x (2 N + 8) floats), the
//                 A tiles (hi: 2 x 32 KB, lo: 2 x 32 KB), and between the
//                 stages the intermediate Y[g][kk][b] with rows 66 float2
//                 apart (so both stages' accesses are free of bank conflicts)
//   B hi, B lo (32 KB each), W_{64 R0}^e, W_N^{16 b a} [b][a], W_N^{b c} [b][c]
//   per-row partial maxima, stage A and stage B inverse scales, 2 mbarriers,
//   the TMEM address.
// TMEM: 256 columns, tile t at columns 128 t.  Thread 0 issues each stage's
// 48 MMAs and commits each tile to its mbarrier; every thread waits
// (bounded; on timeout the kernel sets the plan's tensor-core flag and
// finishes) before the workspace is written again.
#include <cuda_fp16.h>

#include <algorithm>

#include "faf_kernels_common.cuh"
#include "faf_land.cuh"
#include "faf_tc.cuh"

namespace fafk {
namespace tc64 {

using namespace fafk::tcu;

constexpr int kThreads = 1024;
constexpr uint32_t kTile = 128 * 128 * 2;  // one FP16 tile: 128 rows x K 128
constexpr uint32_t kLbo = 16 * 128;        // stride of 8-wide K chunks (128 rows each)
constexpr uint32_t kSbo = 128;             // next 8-row group
constexpr uint32_t kIdesc = idesc_f16(128, 128);
constexpr int kIs = 66;                    // intermediate row stride (float2)
constexpr int kTmemCols = 256;

// shared-memory map (bytes)
constexpr uint32_t kOffB = 256 * kIs * 8;          // 135168: end of the workspace
constexpr uint32_t kOffTA = kOffB + 2 * kTile;     // W_{64 R0}^e, 256 entries
constexpr uint32_t kOffT1 = kOffTA + 256 * 8;      // W_N^{16 b a}, 64 x 16 entries
constexpr uint32_t kOffT2 = kOffT1 + 1024 * 8;     // W_N^{b c}, 64 x 16 entries
constexpr uint32_t kTabBytes = kOffT2 + 1024 * 8 - kOffB;  // the device table, copied as is
constexpr uint32_t kOffPm = kOffB + kTabBytes;     // partial maxima, 1536 floats
constexpr uint32_t kOffScA = kOffPm + 1536 * 4;    // stage A inverse scales [g * 64 + b]
constexpr uint32_t kOffScB = kOffScA + 256 * 4;    // stage B inverse scales [row]
constexpr uint32_t kOffBar = kOffScB + 256 * 4;    // 2 mbarriers, then the TMEM address
constexpr uint32_t kSmem = kOffBar + 32;
static_assert(kTabBytes == 83968, "table layout");
static_assert(kSmem == 227360, "shared-memory map");
static_assert(4 * (2 * 4096 + 8) * 4 <= kOffB, "four landed 4096-point inputs fit the workspace");

template <int R0>
struct Geo {
    static constexpr int N = 4096 * R0;
    static constexpr int G = 4 / R0;      // transforms per CTA
    static constexpr int T = 256 * R0;    // threads per transform
    static constexpr int NK = 64 * R0;    // stage B rows per transform
    static constexpr int JW = 16 / R0;    // j0 values per thread in stage A
    static constexpr int PS = R0 == 1 ? 4 : 4 * R0 + 4;  // partial-max row stride (floats)
    static_assert(G * T == kThreads && G * NK == 256, "256 DFT rows per stage");
    static_assert(G * 64 * PS <= 1536, "partial maxima fit");
};

// Stage A: this thread's 16 inputs x[b + 64 j0 + 4096 i] (j0 = J JW + u,
// i < R0) -> the radix-R0 outputs z[k0][u] (index k0 JW + u), twiddled by
// W_{64 R0}^{j0 k0}; returns their largest magnitude.
template <int R0, class Src>
__device__ __forceinline__ float stage_a_in(float (&xr)[16], float (&xi)[16], const Src& src,
                                            int b, int J, const float2* __restrict__ ta) {
    using Gm = Geo<R0>;
    constexpr int JW = Gm::JW;
#pragma unroll
    for (int i = 0; i < R0; i++)
#pragma unroll
        for (int u = 0; u < JW; u++) {
            const cf v = src.get(b + 64 * (J * JW + u) + 4096 * i);
            xr[i * JW + u] = v.x;
            xi[i * JW + u] = v.y;
        }
    if constexpr (R0 == 2) {
#pragma unroll
        for (int u = 0; u < JW; u++) {
            const float ar = xr[u], ai = xi[u], br = xr[JW + u], bi = xi[JW + u];
            xr[u] = ar + br; xi[u] = ai + bi;
            xr[JW + u] = ar - br; xi[JW + u] = ai - bi;
        }
    } else if constexpr (R0 == 4) {
#pragma unroll
        for (int u = 0; u < JW; u++) {
            const float v0r = xr[u], v0i = xi[u], v1r = xr[JW + u], v1i = xi[JW + u];
            const float v2r = xr[2 * JW + u], v2i = xi[2 * JW + u];
            const float v3r = xr[3 * JW + u], v3i = xi[3 * JW + u];
            const float ar = v0r + v2r, ai = v0i + v2i, br = v0r - v2r, bi = v0i - v2i;
            const float cr = v1r + v3r, ci = v1i + v3i, dr = v1r - v3r, di = v1i - v3i;
            xr[u] = ar + cr; xi[u] = ai + ci;                   // k0 = 0
            xr[JW + u] = br + di; xi[JW + u] = bi - dr;         // k0 = 1: b - i d
            xr[2 * JW + u] = ar - cr; xi[2 * JW + u] = ai - ci; // k0 = 2
            xr[3 * JW + u] = br - di; xi[3 * JW + u] = bi + dr; // k0 = 3: b + i d
        }
    }
#pragma unroll
    for (int k0 = 1; k0 < R0; k0++)
#pragma unroll
        for (int u = 0; u < JW; u++) {
            const float2 w = ta[(J * JW + u) * k0];
            const float r = xr[k0 * JW + u], m = xi[k0 * JW + u];
            xr[k0 * JW + u] = r * w.x - m * w.y;
            xi[k0 * JW + u] = fmaf(r, w.y, m * w.x);
        }
    float mx = 0.f;
#pragma unroll
    for (int v = 0; v < 16; v++) mx = fmaxf(mx, fmaxf(fabsf(xr[v]), fabsf(xi[v])));
    return mx;
}

// The hi / lo A entries of 4 complex values (one 8-wide K chunk) of a row.
__device__ __forceinline__ void put_chunk(uint32_t a_hi, int row, int chunk, const float* re,
                                          const float* im, float s) {
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; j++) split2(re[j] * s, im[j] * s, h[j], l[j]);
    const uint32_t at = a_hi + (uint32_t)(row >> 7) * kTile +
                        (uint32_t)((row & 7) * 16 + ((row & 127) >> 3) * kSbo) +
                        (uint32_t)chunk * kLbo;
    st_shared_v4(at, h);
    st_shared_v4(at + 2 * kTile, l);
}

// Thread 0: D[tile] = A_hi B_hi + A_hi B_lo + A_lo B_hi for both tiles (K = 8
// steps of 16), each tile committed to its mbarrier.
__device__ __forceinline__ void issue_stage(uint32_t ws_s, uint32_t b_s, uint32_t tbase,
                                            uint64_t* bars) {
    fence_after_sync();
#pragma unroll 1
    for (int tile = 0; tile < 2; tile++) {
        const uint32_t ah = ws_s + (uint32_t)tile * kTile, al = ah + 2 * kTile;
        const uint32_t d = tbase + 128u * (uint32_t)tile;
#pragma unroll
        for (int ks = 0; ks < 8; ks++) {
            const uint32_t off = (uint32_t)ks * 2 * kLbo;
            const uint64_t dah = sdesc(ah + off, kLbo, kSbo), dal = sdesc(al + off, kLbo, kSbo);
            const uint64_t dbh = sdesc(b_s + off, kLbo, kSbo);
            const uint64_t dbl = sdesc(b_s + kTile + off, kLbo, kSbo);
            mma(d, dah, dbh, kIdesc, ks > 0 ? 1u : 0u);
            mma(d, dah, dbl, kIdesc, 1u);
            mma(d, dal, dbh, kIdesc, 1u);
        }
        commit(&bars[tile]);
    }
}

// Every thread: both tiles' MMAs have completed (their operands are free).
__device__ __forceinline__ void wait_stage(uint64_t* bars, uint32_t& phase, int* err) {
    const bool ok0 = wait_bounded(&bars[0], phase);
    const bool ok1 = wait_bounded(&bars[1], phase);
    if (!(ok0 && ok1)) atomicOr(err, 1);
    phase ^= 1u;
    fence_after_sync();
}

// LAND: each transform's input lands at workspace offset g * (2 N + 8)
// floats by bulk copy (faf_land.cuh); the next copy is issued once stage B's MMAs have
// completed, while stage B's results are stored.
template <int R0, bool LAND>
__global__ void __launch_bounds__(kThreads, 1)
    k2_c2c_tc64(const C2CArgs a, const uint4* __restrict__ gtab, int* err) {
    using Gm = Geo<R0>;
    constexpr int N = Gm::N, G = Gm::G, T = Gm::T, NK = Gm::NK, JW = Gm::JW, PS = Gm::PS;
    extern __shared__ float4 smem4[];
    uint8_t* sm = reinterpret_cast<uint8_t*>(smem4);
    float2* ws = reinterpret_cast<float2*>(sm);
    const float2* ta = reinterpret_cast<const float2*>(sm + kOffTA);
    const float2* t1 = reinterpret_cast<const float2*>(sm + kOffT1);
    const float2* t2 = reinterpret_cast<const float2*>(sm + kOffT2);
    float* pm = reinterpret_cast<float*>(sm + kOffPm);
    float* sca = reinterpret_cast<float*>(sm + kOffScA);
    float* scb = reinterpret_cast<float*>(sm + kOffScB);
    uint64_t* bars = reinterpret_cast<uint64_t*>(sm + kOffBar);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(sm + kOffBar + 16);
    const uint32_t ws_s = smem_u32(sm), b_s = ws_s + kOffB;
    __shared__ LandCtl lctl;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = tid / T, tt = tid - g * T;  // stage A: transform slot, thread within it
    const int bA = tt & 63, J = tt >> 6;
    Lander<N> L{&lctl, g, reinterpret_cast<float*>(sm) + (size_t)g * (2 * N + 8)};
    if constexpr (LAND) L.init(tt);
    for (int i = tid; i < (int)(kTabBytes / 16); i += kThreads)
        reinterpret_cast<uint4*>(sm + kOffB)[i] = gtab[i];
    if (tid < 2)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[tid]))
                     : "memory");
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(tslot)),
                     "r"(kTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    fence_async_smem();
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    const uint32_t tbase = *tslot;
    uint32_t phase = 0;
    const int fpe = a.interleaved ? 2 : 1;
    // readback geometry: warp -> TMEM lane quarter, tile, 32 of the tile's 128 columns
    const int qd = warp & 3, rtile = (warp >> 2) >> 2, rch = (warp >> 2) & 3;
    const int rrow = rtile * 128 + qd * 32 + lane;
    const uint32_t taddr = tbase + ((uint32_t)(qd * 32) << 16) + (uint32_t)(rtile * 128 + rch * 32);
    // stage B geometry: row (transform, kk), quarter q of b
    const int rowB = tid & 255, qB = tid >> 8;

    const long long ngrp = (a.batch + G - 1) / G;
    if constexpr (LAND) {
        const long long b0 = (long long)blockIdx.x * G + g;
        if (tt == 0 && b0 < a.batch) L.issue(a, b0);
    }
    float xr[16], xi[16];
#pragma unroll 1
    for (long long grp = blockIdx.x; grp < ngrp; grp += gridDim.x) {
        // ---- stage A: inputs, radix R0, per-b maximum
        {
            const long long bt = grp * G + g;
            const bool live = bt < a.batch;
            float mx;
            if constexpr (LAND) {
                if (live) L.wait(a, tt);
                mx = stage_a_in<R0>(xr, xi, L.src(a, live ? bt : 0), bA, J, ta);
            } else {
                const long long bi = live ? bt : 0;
                const long long io = (a.offs ? a.offs[bi] : bi * a.in_dist) * fpe;
                const SplitSrc src{a.in_re + io, a.interleaved ? nullptr : a.in_im + io, a.window,
                                   a.sgn, a.interleaved, live};
                mx = stage_a_in<R0>(xr, xi, src, bA, J, ta);
            }
            pm[(g * 64 + bA) * PS + J] = mx;
        }
        __syncthreads();  // the landed inputs are read; partial maxima visible
        {
            float mx = 0.f;
#pragma unroll
            for (int c = 0; c < R0; c++) {
                const float4 p = reinterpret_cast<const float4*>(pm + (g * 64 + bA) * PS)[c];
                mx = fmaxf(fmaxf(mx, fmaxf(p.x, p.y)), fmaxf(p.z, p.w));
            }
            float s, inv;
            pow2_scale(mx, s, inv);
            if (J == 0) sca[g * 64 + bA] = inv;
#pragma unroll
            for (int k0 = 0; k0 < R0; k0++) {
                const int row = (g * R0 + k0) * 64 + bA;
#pragma unroll
                for (int cc = 0; cc < JW / 4; cc++)
                    put_chunk(ws_s, row, J * (JW / 4) + cc, &xr[k0 * JW + 4 * cc],
                              &xi[k0 * JW + 4 * cc], s);
            }
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        if (tid == 0) issue_stage(ws_s, b_s, tbase, bars);
        wait_stage(bars, phase, err);
        // ---- stage A results -> intermediate Y[g][kk][b] (unscaled)
        {
            const int gk = rrow >> 6, bb = rrow & 63;
            const int gg = gk / R0, k0 = gk - gg * R0;
            uint32_t d[32];
            tmem_ld32(taddr, d);
            const float inv = sca[gg * 64 + bb];
            float2* y = ws + gg * (NK * kIs) + bb;
#pragma unroll
            for (int v = 0; v < 16; v++) {
                const int kk = k0 + R0 * (16 * rch + v);
                y[kk * kIs] = make_float2(__uint_as_float(d[2 * v]) * inv,
                                          __uint_as_float(d[2 * v + 1]) * inv);
            }
        }
        fence_before_sync();
        __syncthreads();
        // ---- stage B: W_N^{b kk} twiddles, per-row maximum
        {
            const int gg = rowB / NK, kk = rowB - gg * NK;
            const float4* y = reinterpret_cast<const float4*>(ws + gg * (NK * kIs) + kk * kIs +
                                                              16 * qB);
#pragma unroll
            for (int v = 0; v < 8; v++) {
                const float4 w = y[v];
                xr[2 * v] = w.x; xi[2 * v] = w.y;
                xr[2 * v + 1] = w.z; xi[2 * v + 1] = w.w;
            }
            const int ka = kk >> 4, kc = kk & 15;
            float mx = 0.f;
#pragma unroll
            for (int u = 0; u < 16; u++) {
                const int b = 16 * qB + u;
                const float2 w1 = t1[b * (4 * R0) + ka], w2 = t2[b * 16 + kc];
                const float wr = w1.x * w2.x - w1.y * w2.y, wi = fmaf(w1.x, w2.y, w1.y * w2.x);
                const float r = xr[u], m = xi[u];
                xr[u] = r * wr - m * wi;
                xi[u] = fmaf(r, wi, m * wr);
                mx = fmaxf(mx, fmaxf(fabsf(xr[u]), fabsf(xi[u])));
            }
            pm[rowB * 4 + qB] = mx;
        }
        __syncthreads();  // the intermediate is read; partial maxima visible
        {
            const float4 p = reinterpret_cast<const float4*>(pm)[rowB];
            float s, inv;
            pow2_scale(fmaxf(fmaxf(p.x, p.y), fmaxf(p.z, p.w)), s, inv);
            if (qB == 0) scb[rowB] = inv;
#pragma unroll
            for (int cc = 0; cc < 4; cc++)
                put_chunk(ws_s, rowB, 4 * qB + cc, &xr[4 * cc], &xi[4 * cc], s);
        }
        fence_async_smem();
        fence_before_sync();
        __syncthreads();
        if (tid == 0) issue_stage(ws_s, b_s, tbase, bars);
        wait_stage(bars, phase, err);
        if constexpr (LAND) {  // the workspace is free: the next inputs may land
            const long long bn = (grp + gridDim.x) * G + g;
            if (tt == 0 && bn < a.batch) L.issue(a, bn);
        }
        // ---- stage B results -> X[kk + 64 R0 m]
        {
            const int gg = rrow / NK, kk = rrow - gg * NK;
            const long long bt = grp * G + gg;
            const bool live = bt < a.batch;
            const long long bi = live ? bt : 0;
            const long long oo = (a.offs ? a.offs[bi] : bi * a.out_dist) * fpe;
            const SplitSink snk{a.out_re + oo, a.interleaved ? nullptr : a.out_im + oo, a.scale,
                                a.sgn, a.interleaved, live};
            uint32_t d[32];
            tmem_ld32(taddr, d);
            const float inv = scb[rrow];
#pragma unroll
            for (int v = 0; v < 16; v++)
                snk.put(kk + NK * (16 * rch + v), cf{__uint_as_float(d[2 * v]) * inv,
                                                     __uint_as_float(d[2 * v + 1]) * inv});
        }
    }
    if constexpr (LAND) L.drain(tt);
    // release the accumulators once every thread's reads of them are done
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase),
                     "r"(kTmemCols)
                     : "memory");
}

template <int R0>
cudaError_t prepare_r() {
    cudaError_t e = prep(k2_c2c_tc64<R0, false>, kSmem);
    if (e == cudaSuccess) e = prep(k2_c2c_tc64<R0, true>, kSmem);
    return e;
}

template <int R0>
cudaError_t launch_r(const C2CArgs& a, const void* tab, int* err, cudaStream_t st) {
    cudaError_t e = prepare_r<R0>();
    if (e != cudaSuccess) return e;
    constexpr int G = Geo<R0>::G;
    const long long groups = (a.batch + G - 1) / G;
    const unsigned grid =
        (unsigned)std::max(1LL, std::min(groups, (long long)fafk::sm_count()));
    if (a.land && !a.window)
        k2_c2c_tc64<R0, true><<<grid, kThreads, kSmem, st>>>(a, (const uint4*)tab, err);
    else
        k2_c2c_tc64<R0, false><<<grid, kThreads, kSmem, st>>>(a, (const uint4*)tab, err);
    return cudaGetLastError();
}

}  // namespace tc64

bool tc64_supported(int log2n) { return log2n >= 12 && log2n <= 14; }

size_t tc64_table_bytes() { return tc64::kTabBytes; }

cudaError_t prepare_c2c_tc64(int log2n) {
    switch (log2n) {
    case 12: return tc64::prepare_r<1>();
    case 13: return tc64::prepare_r<2>();
    case 14: return tc64::prepare_r<4>();
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_c2c_tc64(int log2n, const C2CArgs& a, const void* tab, int* err,
                            cudaStream_t st) {
    if (a.batch <= 0) return cudaSuccess;
    switch (log2n) {
    case 12: return tc64::launch_r<1>(a, tab, err, st);
    case 13: return tc64::launch_r<2>(a, tab, err, st);
    case 14: return tc64::launch_r<4>(a, tab, err, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace fafk
