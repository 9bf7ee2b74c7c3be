// k_tc.cu -- tensor-core precision form of the power-of-two C2C: every
// radix-16 stage runs as tcgen05 MMAs, the remaining radix-8/4/2 stage on the
// CUDA cores, in the compile-time Stockham engine of faf_pot2.cuh.
//
// One radix-16 stage of 128 butterflies (one warpgroup, one thread per
// butterfly) is the real product
//     D[128 x 32] = A[128 x 32] * B^T,   B[32 x 32] = [ Fr  -Fi ]
//                                                   [ Fi   Fr ]
// with A row = (x_re[0..15], x_im[0..15]) after the stage's twiddles and
// D row = (y_re[0..15], y_im[0..15]), F = the 16-point forward DFT matrix.
//
// Precision: A and B are FP16, each split into hi + lo (hi = fp16(v), lo =
// fp16(v - hi)), and D accumulates A_hi B_hi + A_hi B_lo + A_lo B_hi in FP32
// (six MMAs of K = 16).  The dropped A_lo B_lo term and the split residuals
// are ~2^-22 of each operand, so a stage keeps FP32-level accuracy.  FP16's
// range is handled per row: each thread scales its 32 values by a power of
// two that puts the largest in [2^13, 2^14), and unscales D exactly.
//
// Operands: A tiles (hi, lo; 8 KB each per warpgroup, 128 KB for the CTA)
// alias the Stockham workspace between the stage's reads and writes; B (hi,
// lo) is a 4 KB constant built on the host from FP64 and copied to shared
// memory once per CTA.  Both are K-major, no swizzle: element (row r, k) at
// byte (r % 8) * 16 + (r / 8) * 128 + (k / 8) * LBO + (k % 8) * 2.
// Accumulators: 128 TMEM lanes x 32 columns per warpgroup (256 columns per
// CTA, one CTA per SM).  One thread per warpgroup issues the MMAs and commits
// them to the warpgroup's mbarrier; the warpgroup waits on it (bounded: on
// timeout the kernel records an error flag and finishes without hanging)
// and reads its rows back with tcgen05.ld.
#include <cuda_fp16.h>

#include <algorithm>

#include "faf_land.cuh"
#include "faf_kernels_common.cuh"
#include "faf_pot2.cuh"
#include "faf_pot2_group.cuh"
#include "faf_tc.cuh"

namespace fafk {
namespace tc {

using fafct::cf;
using fafct::LastC;
using fafct::SmemC;

constexpr int kThreads = 1024;
constexpr int kWarpgroups = kThreads / 128;
constexpr uint32_t kTileBytes = 128 * 32 * 2;  // one FP16 A tile (128 rows x K 32)
constexpr uint32_t kALbo = 16 * 128;           // A: K-direction core-matrix stride
constexpr uint32_t kBLbo = 4 * 128;            // B: K-direction core-matrix stride
constexpr uint32_t kSbo = 128;                 // both: next 8-row group
constexpr uint32_t kBBytes = 2 * 32 * 32 * 2;  // B hi + lo
constexpr uint32_t kTmemCols = 32 * kWarpgroups;
constexpr uint32_t kIdesc = tcu::idesc_f16(128, 32);

using tcu::commit;
using tcu::fence_after_sync;
using tcu::fence_async_smem;
using tcu::fence_before_sync;
using tcu::sdesc;
using tcu::smem_u32;
using tcu::split2;
using tcu::tmem_ld32;
using tcu::wait_bounded;

__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t acc) {
    tcu::mma(d, a, b, kIdesc, acc);
}

struct Ctx {
    uint32_t tmem;      // this warpgroup's accumulator columns, lane 0
    uint32_t tmem_ld;   // this warp's lane quarter of them
    uint32_t a_hi;      // shared address of this warpgroup's A hi tile (lo follows)
    uint32_t b_hi;      // shared address of B hi (lo follows at +2048)
    uint64_t* bar;      // this warpgroup's mbarrier
    uint32_t phase;
    int row;            // this thread's row in the tile
    int* err;
    bool leader;        // issues the warpgroup's MMAs
};

struct CtaSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

// Radix-16 stage S of the N-point transform on the tensor cores (one
// butterfly per thread; same data movement as fafct::ct_stage).
template <int N, int S, bool TWS_SMEM, class Src, class Snk>
__device__ __forceinline__ void tc_stage(float (&xr)[16], float (&xi)[16], int t,
                                         const float2* __restrict__ tws, const Src& src,
                                         const Snk& snk, Ctx& c) {
    using Pl = P2<N>;
    static_assert(Pl::radix(S) == 16, "tensor-core stages are radix 16");
    constexpr int P = Pl::span(S), NB = N / 16, LP = fafct::ilog2(P);
    const int b = t;
    // ---- inputs and the stage's twiddles (FP32)
    if constexpr (fafct::is_fast<Src>::value && NB % 16 == 0) {
        const float2* p = fafct::fast_ptr(src) + fafct::pad2(b);
#pragma unroll
        for (int r = 0; r < 16; r++) {
            const float2 v = p[r * (NB + NB / 16)];
            xr[r] = v.x;
            xi[r] = Src::kConj ? -v.y : v.y;
        }
    } else {
#pragma unroll
        for (int r = 0; r < 16; r++) {
            const cf v = src.get(b + r * NB);
            xr[r] = v.x;
            xi[r] = v.y;
        }
    }
    if constexpr (S > 0) {
        const int k = b & (P - 1);
#pragma unroll
        for (int r = 1; r < 16; r++) {
            const float2 wr = fafct::stage_tw<N, S, TWS_SMEM, 0>(tws, k, r);
            fafct::cmul_inplace(xr[r], xi[r], wr.x, wr.y);
        }
    }
    // the A tiles alias the workspace: every read of it ends first
    if constexpr (Src::kSmem) __syncthreads();
    // ---- per-row power-of-two scale into FP16 range, hi / lo split, A rows
    float m = 0.f;
#pragma unroll
    for (int r = 0; r < 16; r++) m = fmaxf(m, fmaxf(fabsf(xr[r]), fabsf(xi[r])));
    float s, inv;
    tcu::pow2_scale(m, s, inv);
    {
        const uint32_t row_off = (uint32_t)((c.row & 7) * 16 + (c.row >> 3) * kSbo);
#pragma unroll
        for (int q = 0; q < 4; q++) {  // K chunks: re[0..7], re[8..15], im[0..7], im[8..15]
            const float* v = q < 2 ? &xr[8 * q] : &xi[8 * (q - 2)];
            uint32_t h[4], l[4];
#pragma unroll
            for (int j = 0; j < 4; j++) split2(v[2 * j] * s, v[2 * j + 1] * s, h[j], l[j]);
            const uint32_t ah = c.a_hi + row_off + q * kALbo;
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(ah), "r"(h[0]),
                         "r"(h[1]), "r"(h[2]), "r"(h[3])
                         : "memory");
            asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(ah + kTileBytes),
                         "r"(l[0]), "r"(l[1]), "r"(l[2]), "r"(l[3])
                         : "memory");
        }
    }
    fence_async_smem();
    fence_before_sync();
    asm volatile("bar.sync %0, 128;" ::"r"(1 + (int)(threadIdx.x >> 7)) : "memory");
    // ---- one thread issues D = A_hi B_hi + A_hi B_lo + A_lo B_hi (K = 2 x 16)
    if (c.leader) {
        fence_after_sync();
        const uint64_t ah = sdesc(c.a_hi, kALbo, kSbo);
        const uint64_t al = sdesc(c.a_hi + kTileBytes, kALbo, kSbo);
        const uint64_t bh = sdesc(c.b_hi, kBLbo, kSbo);
        const uint64_t bl = sdesc(c.b_hi + 2048, kBLbo, kSbo);
        constexpr uint64_t ka = (2 * kALbo) >> 4, kb = (2 * kBLbo) >> 4;  // second K step
        mma(c.tmem, ah, bh, 0);
        mma(c.tmem, ah + ka, bh + kb, 1);
        mma(c.tmem, ah, bl, 1);
        mma(c.tmem, ah + ka, bl + kb, 1);
        mma(c.tmem, al, bh, 1);
        mma(c.tmem, al + ka, bh + kb, 1);
        commit(c.bar);
    }
    if (!wait_bounded(c.bar, c.phase)) atomicOr(c.err, 1);
    c.phase ^= 1;
    fence_after_sync();
    {
        uint32_t d[32];
        tmem_ld32(c.tmem_ld, d);
#pragma unroll
        for (int r = 0; r < 16; r++) {
            xr[r] = __uint_as_float(d[r]) * inv;
            xi[r] = __uint_as_float(d[16 + r]) * inv;
        }
    }
    // every warpgroup's tiles are consumed before outputs overwrite the workspace
    fence_before_sync();
    __syncthreads();
    // ---- outputs in natural order (the MMA computes the plain DFT)
    const int k = b & (P - 1);
    const int base = ((b >> LP) << (LP + 4)) + k;
    if constexpr (fafct::is_fast<Snk>::value && (P % 16 == 0 || P == 1)) {
        float2* p = fafct::fast_ptr(snk) + fafct::pad2(base);
        constexpr int step = (P % 16 == 0) ? P + P / 16 : 1;
#pragma unroll
        for (int r = 0; r < 16; r++) p[r * step] = make_float2(xr[r], xi[r]);
    } else {
#pragma unroll
        for (int r = 0; r < 16; r++) snk.put(base + r * P, cf{xr[r], xi[r]});
    }
    if constexpr (Snk::kSmem) __syncthreads();
}

// `rd` runs in the last stage once it has read the workspace (CUDA-core
// stages only: a last stage of radix 16 takes no hook).
template <int N, int S, bool TWS, class Src, class Snk, class RdHook = fafct::NoHook>
__device__ __forceinline__ void any_stage(float (&xr)[16], float (&xi)[16], int t,
                                          const float2* __restrict__ tws, const Src& src,
                                          const Snk& snk, Ctx& c, const RdHook& rd = RdHook()) {
    if constexpr (P2<N>::radix(S) == 16) {
        static_assert(std::is_same_v<RdHook, fafct::NoHook>, "no hook in a tensor-core stage");
        tc_stage<N, S, TWS>(xr, xi, t, tws, src, snk, c);
    } else {
        fafct::ct_stage<N, S, TWS>(xr, xi, t, tws, src, snk, CtaSync{}, rd);
    }
}

template <int N, int S, bool TWS, class Src, class Snk, class RdHook = fafct::NoHook>
__device__ __forceinline__ void tc_run(float (&xr)[16], float (&xi)[16], int t, float2* ws,
                                       const float2* __restrict__ tws, const Src& src,
                                       const Snk& snk, Ctx& c, const RdHook& rd = RdHook()) {
    using Pl = P2<N>;
    const SmemC mid{ws};
    const LastC<Snk> last{snk};
    if constexpr (Pl::NS == 1) {
        any_stage<N, 0, TWS>(xr, xi, t, tws, src, last, c, rd);
    } else if constexpr (S == 0) {
        any_stage<N, 0, TWS>(xr, xi, t, tws, src, mid, c);
        tc_run<N, 1, TWS>(xr, xi, t, ws, tws, mid, snk, c, rd);
    } else if constexpr (S == Pl::NS - 1) {
        any_stage<N, S, TWS>(xr, xi, t, tws, mid, last, c, rd);
    } else {
        any_stage<N, S, TWS>(xr, xi, t, tws, mid, mid, c);
        tc_run<N, S + 1, TWS>(xr, xi, t, ws, tws, mid, snk, c, rd);
    }
}

// Bytes of shared memory past the twiddle table and the group workspaces.
constexpr size_t kTailBytes = kBBytes + 8 * kWarpgroups + 16;

template <int N>
constexpr size_t smem_bytes() {
    constexpr int G = kThreads / P2<N>::T;
    return (size_t)CtCfg<N>::TWN * sizeof(float2) +
           (size_t)G * group_stride(N, N) * sizeof(float2) + kTailBytes;
}

// LAND (8192 and 16384 points): inputs land in the workspace by bulk copy
// (faf_land.cuh), the next transform's copy issued once the last stage has
// read the workspace.
template <int N, bool LAND>
__global__ void __launch_bounds__(kThreads, 1)
    k2_c2c_tc(const float2* __restrict__ tws, const C2CArgs a, const uint4* __restrict__ gB,
              int* err) {
    static_assert(P2<N>::N16 >= 1, "needs at least one radix-16 stage");
    constexpr int G = kThreads / P2<N>::T;
    static_assert((size_t)G * group_stride(N, N) * sizeof(float2) >=
                      (size_t)kWarpgroups * 2 * kTileBytes,
                  "A tiles must fit in the workspace they alias");
    extern __shared__ float4 smem4[];
    float2* sm2 = reinterpret_cast<float2*>(smem4);
    CtGroup<N> q(sm2, N, tws);
    __shared__ LandCtl lctl;
    Lander<N> L{&lctl, q.g, reinterpret_cast<float*>(q.ws)};
    if constexpr (LAND) L.init(q.t);
    uint8_t* wsb = reinterpret_cast<uint8_t*>(sm2 + CtCfg<N>::TWN);
    uint8_t* bsm = wsb + (size_t)G * group_stride(N, N) * sizeof(float2);
    uint64_t* bars = reinterpret_cast<uint64_t*>(bsm + kBBytes);
    uint32_t* tslot = reinterpret_cast<uint32_t*>(bars + kWarpgroups);
    const int wg = threadIdx.x >> 7, warp = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < (int)(kBBytes / 16); i += blockDim.x)
        reinterpret_cast<uint4*>(bsm)[i] = gB[i];
    if (threadIdx.x < kWarpgroups)
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&bars[threadIdx.x]))
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
    Ctx c;
    const uint32_t tbase = *tslot;
    c.tmem = tbase + 32 * wg;
    c.tmem_ld = tbase + ((uint32_t)(32 * (warp & 3)) << 16) + 32 * wg;
    c.a_hi = smem_u32(wsb) + (uint32_t)wg * 2 * kTileBytes;
    c.b_hi = smem_u32(bsm);
    c.bar = &bars[wg];
    c.phase = 0;
    c.row = threadIdx.x & 127;
    c.err = err;
    c.leader = (threadIdx.x & 127) == 0;
    float xr[16], xi[16];
    const int fpe = a.interleaved ? 2 : 1;
    if constexpr (LAND) {
        const long long b0 = (long long)blockIdx.x * G + q.g;
        if (q.t == 0 && b0 < a.batch) L.issue(a, b0);
    }
    CT_FOR_GROUPS(G, a.batch) {
        const long long b = grp_ * G + q.g;
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        const long long io = (a.offs ? a.offs[bi] : bi * a.in_dist) * fpe;
        const long long oo = (a.offs ? a.offs[bi] : bi * a.out_dist) * fpe;
        SplitSink snk{a.out_re + oo, a.interleaved ? nullptr : a.out_im + oo, a.scale, a.sgn,
                      a.interleaved, live};
        __syncthreads();  // the workspace is free (previous group done)
        if constexpr (LAND) {
            if (live) L.wait(a, q.t);
            const long long bn = b + (long long)gridDim.x * G;
            tc_run<N, 0, kTw<N>>(xr, xi, q.t, q.ws, q.tw, L.src(a, bi), snk, c, [&]() {
                __syncthreads();  // every group has read its workspace
                if (q.t == 0 && bn < a.batch) L.issue(a, bn);
            });
        } else {
            SplitSrc src{a.in_re + io, a.interleaved ? nullptr : a.in_im + io, a.window, a.sgn,
                         a.interleaved, live};
            tc_run<N, 0, kTw<N>>(xr, xi, q.t, q.ws, q.tw, src, snk, c);
        }
    }
    if constexpr (LAND) L.drain(q.t);
    // release the accumulators once every MMA has completed
    fence_before_sync();
    __syncthreads();
    fence_after_sync();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase),
                     "r"(kTmemCols)
                     : "memory");
}

template <int N>
cudaError_t prepare_n() {
    cudaError_t e = prep(k2_c2c_tc<N, false>, smem_bytes<N>());
    if constexpr (N >= 8192)
        if (e == cudaSuccess) e = prep(k2_c2c_tc<N, true>, smem_bytes<N>());
    return e;
}

template <int N>
cudaError_t launch_n(const float2* tws, const C2CArgs& a, const void* gB, int* err,
                     cudaStream_t st) {
    constexpr size_t smem = smem_bytes<N>();
    cudaError_t e = prepare_n<N>();
    if (e != cudaSuccess) return e;
    const int sms = fafk::sm_count();
    constexpr int G = kThreads / P2<N>::T;
    const long long groups = (a.batch + G - 1) / G;
    const unsigned grid = (unsigned)std::max(1LL, std::min(groups, (long long)sms));
    if constexpr (N >= 8192) {
        if (a.land) {
            k2_c2c_tc<N, true><<<grid, kThreads, smem, st>>>(tws, a, (const uint4*)gB, err);
            return cudaGetLastError();
        }
    }
    k2_c2c_tc<N, false><<<grid, kThreads, smem, st>>>(tws, a, (const uint4*)gB, err);
    return cudaGetLastError();
}

}  // namespace tc

bool tc_supported(int log2n) { return log2n >= 8 && log2n <= 14; }

cudaError_t prepare_c2c_tc(int log2n) {
    switch (log2n) {
    case 8: return tc::prepare_n<256>();
    case 9: return tc::prepare_n<512>();
    case 10: return tc::prepare_n<1024>();
    case 11: return tc::prepare_n<2048>();
    case 12: return tc::prepare_n<4096>();
    case 13: return tc::prepare_n<8192>();
    case 14: return tc::prepare_n<16384>();
    default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_c2c_tc(int log2n, const float2* tws, const C2CArgs& a, const void* gB,
                          int* err, cudaStream_t st) {
    if (a.batch <= 0) return cudaSuccess;
    switch (log2n) {
    case 8: return tc::launch_n<256>(tws, a, gB, err, st);
    case 9: return tc::launch_n<512>(tws, a, gB, err, st);
    case 10: return tc::launch_n<1024>(tws, a, gB, err, st);
    case 11: return tc::launch_n<2048>(tws, a, gB, err, st);
    case 12: return tc::launch_n<4096>(tws, a, gB, err, st);
    case 13: return tc::launch_n<8192>(tws, a, gB, err, st);
    case 14: return tc::launch_n<16384>(tws, a, gB, err, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace fafk
