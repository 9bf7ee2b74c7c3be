// faf_pot2.cuh -- compile-time Stockham engine for power-of-two lengths.
//
// Same algorithm as faf_device.cuh (radix-16 stages, then one 8/4/2 stage;
// sources / sinks fused into the first / last stage), but with the length
// fixed at compile time, so every span, mask, butterfly count and offset is
// a constant, and with the working set stored as interleaved complex float2
// in shared memory (one 64-bit access per element, one pad element per 16:
// conflict-free for the stride-16 first-stage stores).
//
// Twiddles live in a per-stage table laid out [stage][r-1][k]: for stage s
// with span P and radix R, entry (r, k) = W_{P R}^{r k}.  Lanes of a warp hold
// consecutive k, so every twiddle load of a warp is one contiguous segment.
#pragma once

#include <type_traits>

#include "faf_device.cuh"

namespace fafct {

using fafd::cf;
using fafd::cmul_inplace;
using fafd::Dft;

__host__ __device__ constexpr int ilog2(int n) { return n <= 1 ? 0 : 1 + ilog2(n >> 1); }

// Radix order of a 2^lg-point transform (the one source for kernels and the
// host's twiddle tables).  Order 0: radix-16 stages, then one 8/4/2 stage.
// Order 1 ends in radix 8 wherever the remainder allows it at the same stage
// count (2^1: ..., 16, 4, 8; 2^2: ..., 16, 8, 8), so the real-input kernels can
// fuse their bin-pair pass into the last stage (fafct::ct_last_pairs).
__host__ __device__ constexpr int ct_stages(int lg, int ord) {
    return lg / 4 + (lg % 4 ? 1 : 0) + 0 * ord;
}
__host__ __device__ constexpr int ct_radix(int lg, int ord, int s) {
    const int n16 = lg / 4, rem = lg % 4;
    if (ord == 1 && n16 >= 1 && (rem == 1 || rem == 2)) {
        if (s < n16 - 1) return 16;
        if (s == n16 - 1) return rem == 1 ? 4 : 8;
        return 8;
    }
    return s < n16 ? 16 : (1 << rem);
}
__host__ __device__ constexpr int ct_span(int lg, int ord, int s) {
    int p = 1;
    for (int j = 0; j < s; j++) p *= ct_radix(lg, ord, j);
    return p;
}
// Per-stage twiddle table: stage s >= 1 (radix R, span P) needs W_{PR}^{r k}
// for r < R, k < P.  Stages with P >= 1024 store it as a product of two short
// tables, k = a Q + b: W_{PR}^{r a Q} (a < P / Q) then W_{PR}^{r b} (b < Q), per
// r; so the whole table of a 16384-point transform is 36 KB instead of 131,
// small enough to live in shared memory next to the workspace.
__host__ __device__ constexpr int ct_split_q(int lg, int ord, int s) {
    return ct_span(lg, ord, s) >= 4096 ? 64 : ct_span(lg, ord, s) >= 1024 ? 32 : 0;
}
__host__ __device__ constexpr int ct_tw_len(int lg, int ord, int s) {
    const int q = ct_split_q(lg, ord, s), P = ct_span(lg, ord, s);
    return (ct_radix(lg, ord, s) - 1) * (q ? P / q + q : P);
}

template <int N, int ORD = 0>
struct P2 {
    static_assert(N >= 16 && (N & (N - 1)) == 0, "power of two >= 16");
    static constexpr int LOG = ilog2(N);
    static constexpr int N16 = LOG / 4;
    static constexpr int REM = LOG % 4;
    static constexpr int NS = ct_stages(LOG, ORD);
    static constexpr int T = N / 16;                    // threads per transform
    __host__ __device__ static constexpr int radix(int s) { return ct_radix(LOG, ORD, s); }
    __host__ __device__ static constexpr int span(int s) { return ct_span(LOG, ORD, s); }
    __host__ __device__ static constexpr int split_q(int s) { return ct_split_q(LOG, ORD, s); }
    __host__ __device__ static constexpr int tw_offset(int s) {
        int o = 0;
        for (int j = 1; j < s; j++) o += ct_tw_len(LOG, ORD, j);
        return o;
    }
    static constexpr int TW = tw_offset(NS);            // table entries
};

__device__ __forceinline__ int pad2(int a) { return a + (a >> 4); }

// float2 slots needed for `slots` complex elements
__host__ __device__ constexpr int plane2(int slots) {
    return (slots - 1) + ((slots - 1) >> 4) + 1;
}

// Twiddle W_{PR}^{r k} of stage S (1 <= r < R, k < P) from the per-stage table
// (shared memory when TWS_SMEM): one entry, or the product of a split stage's
// two entries.
template <int N, int S, bool TWS_SMEM, int ORD>
__device__ __forceinline__ float2 stage_tw(const float2* __restrict__ tws, int k, int r) {
    using Pl = P2<N, ORD>;
    constexpr int P = Pl::span(S), Q = Pl::split_q(S), OFF = Pl::tw_offset(S);
    if constexpr (Q == 0) {
        const int i = OFF + (r - 1) * P + k;
        return TWS_SMEM ? tws[i] : __ldg(&tws[i]);
    } else {
        constexpr int A = P / Q;
        const int i = OFF + (r - 1) * (A + Q);
        const float2 a = TWS_SMEM ? tws[i + k / Q] : __ldg(&tws[i + k / Q]);
        const float2 b = TWS_SMEM ? tws[i + A + k % Q] : __ldg(&tws[i + A + k % Q]);
        return make_float2(a.x * b.x - a.y * b.y, fmaf(a.x, b.y, a.y * b.x));
    }
}

// Interleaved complex workspace.  kFast marks shared-memory sources / sinks
// whose strided accesses the stage turns into one padded base address plus
// compile-time offsets.
struct SmemC {
    float2* d;
    static constexpr bool kSmem = true;
    static constexpr bool kFast = true;
    static constexpr bool kConj = false;
    __device__ __forceinline__ cf get(int i) const {
        const float2 v = d[pad2(i)];
        return cf{v.x, v.y};
    }
    __device__ __forceinline__ void put(int i, cf v) const { d[pad2(i)] = make_float2(v.x, v.y); }
};

struct SmemCConj {
    float2* d;
    static constexpr bool kSmem = true;
    static constexpr bool kFast = true;
    static constexpr bool kConj = true;
    __device__ __forceinline__ cf get(int i) const {
        const float2 v = d[pad2(i)];
        return cf{v.x, -v.y};
    }
};

template <class T, class = void>
struct is_fast : std::false_type {};
template <class T>
struct is_fast<T, std::void_t<decltype(T::kFast)>> : std::bool_constant<T::kFast> {};

template <class Snk>
struct LastC {
    Snk s;
    static constexpr bool kSmem = false;
    static constexpr bool kFast = is_fast<Snk>::value;
    __device__ __forceinline__ void put(int i, cf v) const { s.put(i, v); }
};

template <class T>
__device__ __forceinline__ float2* fast_ptr(const T& x) {
    if constexpr (std::is_same_v<T, SmemC> || std::is_same_v<T, SmemCConj>) return x.d;
    else return x.s.d;
}

struct NoHook {
    __device__ __forceinline__ void operator()() const {}
};

// One Stockham stage.  `rd` runs once every value the stage reads is in
// registers, before anything is written (a kernel that reuses the source's
// memory starts there; the default does nothing).
template <int N, int S, bool TWS_SMEM, int ORD = 0, class Src, class Snk, class Sync,
          class RdHook = NoHook>
__device__ __forceinline__ void ct_stage(float (&xr)[16], float (&xi)[16], int t,
                                         const float2* __restrict__ tws, const Src& src,
                                         const Snk& snk, const Sync& sync,
                                         const RdHook& rd = RdHook()) {
    using Pl = P2<N, ORD>;
    constexpr int R = Pl::radix(S), P = Pl::span(S), NB = N / R, T = Pl::T, MB = 16 / R;
    constexpr int LP = ilog2(P);
#pragma unroll
    for (int i = 0; i < MB; i++) {
        const int b = t + i * T;
        if constexpr (is_fast<Src>::value && NB % 16 == 0) {
            // pad2(b + r NB) = pad2(b) + r (NB + NB / 16)
            const float2* p = fast_ptr(src) + pad2(b);
#pragma unroll
            for (int r = 0; r < R; r++) {
                const float2 v = p[r * (NB + NB / 16)];
                xr[i * R + r] = v.x;
                xi[i * R + r] = Src::kConj ? -v.y : v.y;
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) {
                const cf v = src.get(b + r * NB);
                xr[i * R + r] = v.x;
                xi[i * R + r] = v.y;
            }
        }
        if constexpr (S > 0) {
            const int k = b & (P - 1);
#pragma unroll
            for (int r = 1; r < R; r++) {
                const float2 wr = stage_tw<N, S, TWS_SMEM, ORD>(tws, k, r);
                cmul_inplace(xr[i * R + r], xi[i * R + r], wr.x, wr.y);
            }
        }
        Dft<R>::run(&xr[i * R], &xi[i * R]);
    }
    rd();
    if constexpr (Src::kSmem && Snk::kSmem) sync();
#pragma unroll
    for (int i = 0; i < MB; i++) {
        const int b = t + i * T;
        const int k = b & (P - 1);
        const int base = ((b >> LP) << (LP + ilog2(R))) + k;
        if constexpr (is_fast<Snk>::value && (P % 16 == 0 || (P == 1 && R == 16))) {
            // P % 16 == 0: pad2(base + r P) = pad2(base) + r (P + P / 16);
            // P == 1, R == 16: base = 16 b, pad2(16 b + r) = 17 b + r.
            float2* p = fast_ptr(snk) + pad2(base);
            constexpr int step = (P % 16 == 0) ? P + P / 16 : 1;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int j = i * R + Dft<R>::slot(r);
                p[r * step] = make_float2(xr[j], xi[j]);
            }
        } else {
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int j = i * R + Dft<R>::slot(r);
                snk.put(base + r * P, cf{xr[j], xi[j]});
            }
        }
    }
    if constexpr (Snk::kSmem) sync();
}

// Barrier of one transform group: a named barrier over the group's T threads
// when T >= 32 (groups of a CTA then progress independently), a warp barrier
// when the group lives inside one warp.
struct GroupSync {
    int id;          // 1..15 (0 is the CTA-wide barrier)
    int nthreads;    // T
    unsigned lanes;  // T < 32: lanes of this warp that exist (a CTA may end mid-warp)
    __device__ __forceinline__ void operator()() const {
        if (nthreads >= 32)
            asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
        else
            __syncwarp(lanes);
    }
    __device__ static GroupSync make(int g, int T) {
        const int base = threadIdx.x & ~31;
        const int n = min(32, (int)blockDim.x - base);
        return GroupSync{1 + g, T, n >= 32 ? 0xffffffffu : ((1u << n) - 1u)};
    }
};


// Stages S.. of the transform.  SKIP_LAST stops before the last stage (the
// caller runs it, fused with what follows; the stage before it has written
// the workspace and synchronised).
template <int N, int S, bool TWS_SMEM, class Src, class Snk, class Sync, class Hook,
          bool SKIP_LAST = false, int ORD = 0>
__device__ __forceinline__ void ct_run(float (&xr)[16], float (&xi)[16], int t, float2* ws,
                                       const float2* __restrict__ tws, const Src& src,
                                       const Snk& snk, const Sync& sync, const Hook& hook) {
    using Pl = P2<N, ORD>;
    static_assert(!SKIP_LAST || Pl::NS >= 2, "a skipped last stage needs an earlier one");
    const SmemC mid{ws};
    const LastC<Snk> last{snk};
    if constexpr (Pl::NS == 1) {
        if constexpr (Src::kSmem) {
            ct_stage<N, 0, TWS_SMEM, ORD>(xr, xi, t, tws, src, mid, sync);
            hook();
            for (int i = t; i < N; i += Pl::T) last.put(i, mid.get(i));
        } else {
            ct_stage<N, 0, TWS_SMEM, ORD>(xr, xi, t, tws, src, last, sync);
            sync();
            hook();
        }
    } else if constexpr (S == 0) {
        // stage 0 ends with a barrier: the source is no longer read by anyone
        ct_stage<N, 0, TWS_SMEM, ORD>(xr, xi, t, tws, src, mid, sync);
        hook();
        ct_run<N, 1, TWS_SMEM, SmemC, Snk, Sync, NoHook, SKIP_LAST, ORD>(xr, xi, t, ws, tws, mid, snk,
                                                                    sync, NoHook());
    } else if constexpr (S == Pl::NS - 1) {
        if constexpr (!SKIP_LAST) ct_stage<N, S, TWS_SMEM, ORD>(xr, xi, t, tws, mid, last, sync);
    } else {
        ct_stage<N, S, TWS_SMEM, ORD>(xr, xi, t, tws, mid, mid, sync);
        ct_run<N, S + 1, TWS_SMEM, SmemC, Snk, Sync, NoHook, SKIP_LAST, ORD>(xr, xi, t, ws, tws, mid,
                                                                        snk, sync, NoHook());
    }
}

// Forward FFT of N points (compile time) by the T = N/16 threads of one
// transform group; `ws` is the group's interleaved workspace, `tws` the
// per-stage twiddle table (shared memory when TWS_SMEM, else global).
template <int N, bool TWS_SMEM, int ORD = 0, class Src, class Snk, class Sync,
          class Hook = NoHook>
__device__ __forceinline__ void ct_fft(int t, float2* ws, const float2* __restrict__ tws,
                                       const Src& src, const Snk& snk, const Sync& sync,
                                       const Hook& hook = Hook()) {
    float xr[16], xi[16];
    if constexpr (!Src::kSmem) sync();
    ct_run<N, 0, TWS_SMEM, Src, Snk, Sync, Hook, false, ORD>(xr, xi, t, ws, tws, src, snk, sync,
                                                             hook);
}

// Every stage but the last, from a global source; the workspace holds the
// last stage's input when it returns (synchronised).
template <int N, bool TWS_SMEM, int ORD = 0, class Src, class Sync, class Hook = NoHook>
__device__ __forceinline__ void ct_fft_but_last(int t, float2* ws, const float2* __restrict__ tws,
                                                const Src& src, const Sync& sync,
                                                const Hook& hook = Hook()) {
    float xr[16], xi[16];
    if constexpr (!Src::kSmem) sync();
    ct_run<N, 0, TWS_SMEM, Src, SmemC, Sync, Hook, true, ORD>(xr, xi, t, ws, tws, src, SmemC{ws},
                                                              sync, hook);
}

// The last stage of an N-point transform whose last radix is 8 (two
// butterflies per thread), run so that each thread holds both ends of its
// Hermitian bin pairs (k, N - k) in registers.  The last stage's span equals
// its butterfly count NB, so butterfly b writes Z[b + r NB], and the partner
// of bin b1 + r NB is (NB - b1) + (R - 1 - r) NB: thread t takes butterflies
// t and NB - t (thread 0: 0 and NB / 2, each paired with itself).  Calls
// dc(Z[0]) once, and pair(k, Z[k], Z[N - k]) once for every 1 <= k <= N / 2
// (k = N / 2 paired with itself); all bins it touches are the thread's own.
template <int N, int ORD = 0>
struct LastPairs {
    using Pl = P2<N, ORD>;
    static constexpr int S = Pl::NS - 1;
    static constexpr int R = Pl::radix(S);
    static constexpr bool ok = Pl::NS >= 2 && R == 8;
};

// SEL: 1 makes thread 0 swap its pairs in by selects (no branch), 0 gives it
// a branch of its own, -1 picks selects for one-warp transforms only.
template <int N, bool TWS_SMEM, int ORD = 0, int SEL = -1, class Dc, class Pair>
__device__ __forceinline__ void ct_last_pairs(int t, const float2* ws,
                                              const float2* __restrict__ tws, const Dc& dc,
                                              const Pair& pair) {
    using Pl = P2<N, ORD>;
    constexpr int S = Pl::NS - 1, R = Pl::radix(S), P = Pl::span(S), NB = N / R;
    static_assert(LastPairs<N, ORD>::ok && P == NB && Pl::T == NB / 2, "radix-8 last stage");
    const int b[2] = {t, t == 0 ? NB / 2 : NB - t};
    float xr[2][R], xi[2][R];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const float2* p = ws + pad2(b[h]);
#pragma unroll
        for (int r = 0; r < R; r++) {
            // pad2(b + r NB) = pad2(b) + r (NB + NB / 16) only when 16 | NB
            const float2 v = NB % 16 == 0 ? p[r * (NB + NB / 16)] : ws[pad2(b[h] + r * NB)];
            xr[h][r] = v.x;
            xi[h][r] = v.y;
        }
        if (b[h] != 0) {
#pragma unroll
            for (int r = 1; r < R; r++) {
                const float2 wr = stage_tw<N, S, TWS_SMEM, ORD>(tws, b[h], r);
                cmul_inplace(xr[h][r], xi[h][r], wr.x, wr.y);
            }
        }
        Dft<R>::run(xr[h], xi[h]);
    }
    auto Z = [&](int h, int r) {
        const int j = Dft<R>::slot(r);
        return cf{xr[h][j], xi[h][j]};
    };
    // Other threads: bins k1 = t + i NB and N - k1 (butterflies t and NB - t).
    // Thread 0: butterfly NB / 2 pairs with itself, and so does butterfly 0.
    if constexpr (SEL == 0 || (SEL < 0 && Pl::T > 32)) {
        // several warps per transform: only one of them splits on thread 0,
        // and separate branches cost fewer registers than selects
        if (t != 0) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int k1 = b[0] + r * NB, k2 = N - k1;
                if (k1 < k2) pair(k1, Z(0, r), Z(1, R - 1 - r));
                else pair(k2, Z(1, R - 1 - r), Z(0, r));
            }
        } else {
            dc(Z(0, 0));
#pragma unroll
            for (int r = 1; r <= R / 2; r++) pair(r * NB, Z(0, r), Z(0, R - r));
#pragma unroll
            for (int r = 0; r < R / 2; r++) pair(NB / 2 + r * NB, Z(1, r), Z(1, R - 1 - r));
        }
        return;
    }
    // one warp (or less) per transform: every warp holds a thread 0, so one
    // call sequence for all threads, thread 0 swapping in its pairs by selects
    // (for i < R / 2 from butterfly NB / 2, after that from butterfly 0)
    const bool t0 = t == 0;
    if (t0) dc(Z(0, 0));
#pragma unroll
    for (int i = 0; i < R; i++) {
        const int k1 = b[0] + i * NB, k2 = N - k1;
        const bool lo = k1 < k2;
        int k = lo ? k1 : k2;
        cf za = lo ? Z(0, i) : Z(1, R - 1 - i);
        cf zb = lo ? Z(1, R - 1 - i) : Z(0, i);
        if (i < R / 2) {
            if (t0) {
                k = NB / 2 + i * NB;
                za = Z(1, i);
                zb = Z(1, R - 1 - i);
            }
        } else {
            const int j = i - R / 2 + 1;
            if (t0) {
                k = j * NB;
                za = Z(0, j);
                zb = Z(0, R - j);
            }
        }
        pair(k, za, zb);
    }
}

// Input landed in shared memory (a ring slot, linear, no padding).  It is a
// different buffer from the workspace, so the first stage needs no read/write
// barrier (kSmem = false).
struct StageSrc {
    const float2* s;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        const float2 v = s[i];
        return cf{v.x, v.y};
    }
};

}  // namespace fafct
