// k_pot2.cu -- C2C, R2C, C2R, fused pipeline and STFT kernels for
// power-of-two inner lengths 16..16384 on the compile-time engine
// (faf_pot2.cuh).  Same sources / sinks and the same reference semantics as
// the generic kernels; one instantiation per length.
//
// The kernels are persistent: the grid is sized to the resident CTAs and
// each CTA walks transform groups c, c + grid, ...  The per-stage twiddle
// table is copied into shared memory once per CTA when it fits in 32 KB.
#include <algorithm>

#include "faf_kernels_common.cuh"
#include "faf_land.cuh"
#include "faf_pot2.cuh"
#include "faf_pot2_group.cuh"
#include "faf_ring.cuh"

namespace fafk {

using fafct::P2;
using fafct::SmemC;
using fafct::SmemCConj;
using fafct::ct_fft;
using fafct::plane2;

// Radix order of the real-input kernels (R2C, C2R, pipeline, STFT): it ends
// in radix 8 wherever the length allows, so the R2C post-pass and the
// pipeline's bin-pair pass fuse with the last stage (fafct::ct_last_pairs).
// Real plans build their twiddle tables in the same order.
constexpr int kRO = 1;

// Issues the copy of the transform `src` (sequence s of the CTA's ring) once
// the group's first stage has read its own slot; one thread of the group.
struct RingHook {
    fafct::Ring r;
    int slot, use;    // the slot just read, and the number of the copy to issue into it
    const void* src;  // NULL: nothing left to load
    unsigned bytes;
    int t;
    __device__ __forceinline__ void operator()() const {
        if (t == 0 && src) r.issue(slot, use, src, bytes);
    }
};

// The ring of a real-input kernel: one slot per transform input (2N floats).
template <int N>
__device__ __forceinline__ fafct::Ring real_ring(fafct::RingCtl* ctl, float2* sm, int G, int K,
                                                 const RealArgs& a) {
    return fafct::ring_start(
        ctl, ring_base<N, kRO>(sm, G, N + 1), K, N, G, a.batch,
        [&](long long b) { return (const void*)(a.in_a + b * a.in_dist); }, N * 8u);
}

// Waits for the group's current transform b (cursor c) and returns the hook
// that loads transform b + dnext (sequence s + K) into the same slot;
// src_of(bn) is transform bn's input.
template <class SrcOf>
__device__ __forceinline__ RingHook ring_next_of(const fafct::Ring& R, const fafct::RingCursor& c,
                                                 long long b, int dnext, bool live,
                                                 long long batch, const SrcOf& src_of,
                                                 unsigned bytes, int t, int* err) {
    if (live && !R.wait(c) && t == 0) R.fail(err);
    const long long bn = b + dnext;
    return RingHook{R, c.slot, c.use + 1, (live && bn < batch) ? src_of(bn) : nullptr, bytes, t};
}

__device__ __forceinline__ RingHook ring_next(const fafct::Ring& R, const fafct::RingCursor& c,
                                              long long b, int dnext, bool live, const float* in,
                                              long long dist, long long batch, unsigned bytes,
                                              int t, int* err) {
    return ring_next_of(
        R, c, b, dnext, live, batch, [&](long long bn) { return (const void*)(in + bn * dist); },
        bytes, t, err);
}

template <int N>
__global__ void __launch_bounds__(1024) k2_c2c(const float2* __restrict__ tws, const C2CArgs a,
                                               int G) {
    extern __shared__ float4 smem4[];
    CtGroup<N> q(reinterpret_cast<float2*>(smem4), N, tws);
    const int fpe = a.interleaved ? 2 : 1;
    CT_FOR_GROUPS(G, a.batch) {
        const long long b = grp_ * G + q.g;
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        const long long io = (a.offs ? a.offs[bi] : bi * a.in_dist) * fpe;
        const long long oo = (a.offs ? a.offs[bi] : bi * a.out_dist) * fpe;
        SplitSrc src{a.in_re + io, a.interleaved ? nullptr : a.in_im + io, a.window, a.sgn,
                     a.interleaved, live};
        SplitSink snk{a.out_re + oo, a.interleaved ? nullptr : a.out_im + oo, a.scale, a.sgn,
                      a.interleaved, live};
        ct_fft<N, kTw<N>>(q.t, q.ws, q.tw, src, snk, q.sync);  // begins with a barrier
    }
}

// C2C of power-of-two lengths from 64 points (one mbarrier per group: at
// most 15 groups of one warp or more, kLandMaxGroups narrower ones): the first stage's scalar global loads, with few transforms
// per CTA to overlap them with, left the kernel waiting on memory.
// Here each transform's input lands in its group's workspace by bulk copy
// (faf_land.cuh), issued for the group's next transform as soon as the last
// stage has read the workspace, so the copy runs during the last stage and
// the stores.
// One transform's output staged in shared memory, scaled and conjugated as
// SplitSink stores it.
struct SplitStage {
    float2* p;
    float scale;
    float sgn;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int i, cf v) const {
        p[i] = make_float2(v.x * scale, sgn * v.y * scale);
    }
};

// STG (launched at 64 points, no offset list): the last stage writes a
// staging row behind the workspaces, and the CTA then writes its G
// consecutive transforms row after row: groups of 4 threads otherwise store
// 16 bytes per transform per instruction.  At 128 and 256 points staging
// measured slower than the direct stores.
template <int N, bool STG = false>
__global__ void __launch_bounds__(1024) k2_c2c_land(const float2* __restrict__ tws,
                                                    const C2CArgs a, int G) {
    extern __shared__ float4 smem4[];
    CtGroup<N> q(reinterpret_cast<float2*>(smem4), N, tws);
    using Ctl = LandCtlN<(P2<N>::T >= 32 ? 16 : kLandMaxGroups)>;
    __shared__ Ctl ctl;
    constexpr int NS = P2<N>::NS;
    const int fpe = a.interleaved ? 2 : 1;
    Lander<N, Ctl> L{&ctl, q.g, reinterpret_cast<float*>(q.ws)};
    L.init(q.t);
    __syncthreads();
    const long long stride = (long long)gridDim.x * G;
    long long b = (long long)blockIdx.x * G + q.g;
    if (q.t == 0 && b < a.batch) L.issue(a, b);
    for (; b - q.g < a.batch; b += stride) {  // the same trip count for every group
        const bool live = b < a.batch;
        if (live) L.wait(a, q.t);
        const long long bi = live ? b : 0;
        const long long oo = (a.offs ? a.offs[bi] : bi * a.out_dist) * fpe;
        fafct::ct_fft_but_last<N, kTw<N>>(q.t, q.ws, q.tw, L.src(a, bi), q.sync);
        float xr[16], xi[16];
        const long long bn = b + stride;
        auto hook = [&]() {
            q.sync();  // the whole group has read the workspace
            if (q.t == 0 && bn < a.batch) L.issue(a, bn);
        };
        if constexpr (STG) {
            float2* stg = ring_base<N>(reinterpret_cast<float2*>(smem4), G, N);
            fafct::ct_stage<N, NS - 1, kTw<N>, 0>(
                xr, xi, q.t, q.tw, SmemC{q.ws},
                fafct::LastC<SplitStage>{SplitStage{stg + q.g * N, a.scale, a.sgn}}, q.sync,
                hook);
            __syncthreads();  // every group's row is staged
            const long long b0 = b - q.g;
            const int nl = (int)min((long long)G, a.batch - b0);
            for (int i = threadIdx.x; i < nl * N; i += blockDim.x) {
                const int j = i / N, k = i % N;
                const float2 v = stg[i];
                const long long o = (b0 + j) * a.out_dist * fpe;
                if (a.interleaved) {
                    __stcs(reinterpret_cast<float2*>(a.out_re + o) + k, v);
                } else {
                    __stcs(a.out_re + o + k, v.x);
                    __stcs(a.out_im + o + k, v.y);
                }
            }
            __syncthreads();  // the staging rows are free for the next round
        } else {
            fafct::ct_stage<N, NS - 1, kTw<N>, 0>(
                xr, xi, q.t, q.tw, SmemC{q.ws},
                fafct::LastC<SplitSink>{SplitSink{a.out_re + oo,
                                                  a.interleaved ? nullptr : a.out_im + oo,
                                                  a.scale, a.sgn, a.interleaved, live}},
                q.sync, hook);
        }
    }
    L.drain(q.t);
}

// Post-pass over bin pairs after the forward FFT left Z in the workspace.
template <int N, class Out>
__device__ __forceinline__ void ct_r2c_post(int t, const SmemC& mid,
                                            const float2* __restrict__ stw, const Out& out,
                                            float scale) {
    constexpr int nc = N;
    for (int k = t; k <= nc / 2; k += P2<N>::T) {
        if (k == 0) {
            const cf z = mid.get(0);
            out.put(0, (z.x + z.y) * scale, 0.f);
            out.put(nc, (z.x - z.y) * scale, 0.f);
        } else {
            cf Xk, Xnk;
            r2c_pair(mid.get(k), mid.get(nc - k), __ldg(&stw[k - 1]), Xk, Xnk);
            if (k != nc - k) out.put(k, Xk.x * scale, Xk.y * scale);
            out.put(nc - k, Xnk.x * scale, Xnk.y * scale);
        }
    }
}

// Thread 0's bin pairs in the fused R2C post-pass and in the pipeline's
// single-MUL middle: by selects (no branch splitting its warp) for the ring
// kernels of inner length 2048, measured on B200: the n = 4096 R2C went from
// 4641 to 5007 GB/s (no spills), the pipeline from 2369 to 2432 GB/s (despite
// 40 bytes of spills); with the unguarded multiply of a full-length spectrum,
// 2691 against 2638 GB/s for a branch of its own (136 against 44 bytes of
// spills), and with that spectrum staged in shared memory 2822 against 2657
// (84 against 48 bytes).  Elsewhere the default (selects only for one-warp
// transforms): the selects spill more at other lengths and in the direct-load
// kernels.
template <int N, bool RING>
constexpr int kR2cSel = (RING && N == 2048) ? 1 : -1;

// RING: inputs land in the CTA's ring by bulk copy (in_a 16-byte aligned,
// in_dist a multiple of 4); otherwise the first stage loads them.
template <int N, bool RING>
__global__ void __launch_bounds__(1024) k2_r2c(const float2* __restrict__ tws, const RealArgs a,
                                               int G, bool vec, int K) {
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    const SmemC mid{q.ws};
    const int fpe = a.interleaved ? 2 : 1;
    fafct::Ring R{};
    if constexpr (RING) {
        __shared__ fafct::RingCtl ctl;
        R = real_ring<N>(&ctl, sm, G, K, a);
    }
    fafct::RingCursor c{};
    int dnext = 0;
    if constexpr (RING) {
        c = R.cursor(q.g);
        dnext = R.next_offset(q.g);
    }
    bool first = true;
    CT_FOR_GROUPS(G, a.batch) {
        if constexpr (RING) {
            if (!first) R.advance(c);
            first = false;
        }
        const long long b = grp_ * G + q.g;
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        if constexpr (fafct::LastPairs<N, kRO>::ok) {
            // last stage fused with the post-pass: no workspace round trip
            if constexpr (RING) {
                const RingHook hook =
                    ring_next(R, c, b, dnext, live, a.in_a, a.in_dist, a.batch, N * 8u, q.t,
                              a.err);
                fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, fafct::StageSrc{R.slot_ptr(c)},
                                                  q.sync, hook);
            } else {
                fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(
                    q.t, q.ws, q.tw, RealPairSrc{a.in_a + bi * a.in_dist, live, vec}, q.sync);
            }
            if (live) {
                const long long oo = bi * a.out_dist * fpe;
                const float sc = a.scale;
                const float2* __restrict__ stw = a.stw;
                // one branch per transform on the layout: a per-store branch
                // costs the fused stage registers it does not have
                auto post = [&](const auto& out) {
                    fafct::ct_last_pairs<N, kTw<N, kRO>, kRO, kR2cSel<N, RING>>(
                        q.t, q.ws, q.tw,
                        [&](cf z) {
                            out.put(0, (z.x + z.y) * sc, 0.f);
                            out.put(N, (z.x - z.y) * sc, 0.f);
                        },
                        [&](int k, cf zk, cf zn) {
                            cf Xk, Xnk;
                            r2c_pair(zk, zn, __ldg(&stw[k - 1]), Xk, Xnk);
                            if (k != N - k) out.put(k, Xk.x * sc, Xk.y * sc);
                            out.put(N - k, Xnk.x * sc, Xnk.y * sc);
                        });
                };
                if (a.interleaved)
                    post(HermInter{reinterpret_cast<float2*>(a.out_a + oo)});
                else
                    post(HermSplit{a.out_a + oo, a.out_b + oo});
            }
            continue;
        } else {
            if constexpr (RING) {
                const RingHook hook =
                    ring_next(R, c, b, dnext, live, a.in_a, a.in_dist, a.batch, N * 8u, q.t,
                              a.err);
                ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, fafct::StageSrc{R.slot_ptr(c)}, mid, q.sync, hook);
            } else {
                ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw,
                                  RealPairSrc{a.in_a + bi * a.in_dist, live, vec}, mid, q.sync);
            }
        }
        q.sync();
        if (live) {
            const long long oo = bi * a.out_dist * fpe;
            HermSink out{a.out_a + oo, a.interleaved ? nullptr : a.out_b + oo, a.interleaved};
            ct_r2c_post<N>(q.t, mid, a.stw, out, a.scale);
        }
    }
    if constexpr (RING) fafct::ring_drain(R);
}

// R2C of power-of-two inner lengths 32 to 256 (n = 64 to 512; launched at 256,
// where it measured faster than the direct loads), whose groups are narrower
// than a warp and take no ring: each transform's samples land in
// its group's workspace by bulk copy (every transform start 8-byte aligned,
// so they read as float2 pairs), issued for the group's next transform once
// the group has read the workspace.  With up to kLandMaxGroups groups per CTA
// one group's copy overlaps the others' compute.
template <int N>
__global__ void __launch_bounds__(1024) k2_r2c_land(const float2* __restrict__ tws,
                                                    const RealArgs a, int G) {
    static_assert(N >= 32 && P2<N, kRO>::T < 32, "sub-warp groups of at least two stages");
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    using Ctl = LandCtlN<kLandMaxGroups>;
    __shared__ Ctl ctl;
    const SmemC mid{q.ws};
    const int fpe = a.interleaved ? 2 : 1;
    LandPlanes<Ctl> L{&ctl, q.g, reinterpret_cast<float*>(q.ws), 0};
    L.init(q.t);
    __syncthreads();
    const long long stride = (long long)gridDim.x * G;
    long long b = (long long)blockIdx.x * G + q.g;
    if (q.t == 0 && b < a.batch) L.issue(a.in_a + b * a.in_dist, nullptr, N);
    for (; b - q.g < a.batch; b += stride) {  // the same trip count for every group
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        if (live) L.wait(a.err, q.t);
        const LandSrc src{L.first(a.in_a + bi * a.in_dist), nullptr, 1, 1.0f};
        const long long oo = bi * a.out_dist * fpe;
        if constexpr (fafct::LastPairs<N, kRO>::ok) {
            // last stage fused with the post-pass
            fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, src, q.sync);
            if (live) {
                const float sc = a.scale;
                const float2* __restrict__ stw = a.stw;
                auto post = [&](const auto& out) {
                    fafct::ct_last_pairs<N, kTw<N, kRO>, kRO, kR2cSel<N, false>>(
                        q.t, q.ws, q.tw,
                        [&](cf z) {
                            out.put(0, (z.x + z.y) * sc, 0.f);
                            out.put(N, (z.x - z.y) * sc, 0.f);
                        },
                        [&](int k, cf zk, cf zn) {
                            cf Xk, Xnk;
                            r2c_pair(zk, zn, __ldg(&stw[k - 1]), Xk, Xnk);
                            if (k != N - k) out.put(k, Xk.x * sc, Xk.y * sc);
                            out.put(N - k, Xnk.x * sc, Xnk.y * sc);
                        });
                };
                if (a.interleaved)
                    post(HermInter{reinterpret_cast<float2*>(a.out_a + oo)});
                else
                    post(HermSplit{a.out_a + oo, a.out_b + oo});
            }
        } else {
            ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, src, mid, q.sync);
            if (live) {
                HermSink out{a.out_a + oo, a.interleaved ? nullptr : a.out_b + oo, a.interleaved};
                ct_r2c_post<N>(q.t, mid, a.stw, out, a.scale);
            }
        }
        q.sync();  // the whole group has read the workspace
        const long long bn = b + stride;
        if (q.t == 0 && bn < a.batch) L.issue(a.in_a + bn * a.in_dist, nullptr, N);
    }
    L.drain(q.t);
}

// One transform's spectrum staged in shared memory (bin k at p[k]).
struct HermStage {
    float2* p;
    __device__ __forceinline__ void put(int k, float r, float i) const {
        p[k] = make_float2(r, i);
    }
};

// R2C of power-of-two inner lengths 32 to 128 (n = 64 to 256).  Their groups
// are 2 to 8 threads, so each spectrum store of k2_r2c writes bins of 4 to 16
// transforms and uses little of each sector it touches.  Here every group
// puts its bins in a staging row behind the workspaces, and the CTA then
// writes its G consecutive transforms' spectra row after row, consecutive
// threads on consecutive bins.
template <int N>
__global__ void __launch_bounds__(1024) k2_r2c_small(const float2* __restrict__ tws,
                                                     const RealArgs a, int G, bool vec) {
    static_assert(N >= 32 && P2<N, kRO>::T < 32, "sub-warp groups");
    constexpr int NB = N + 1;
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    float2* stg = ring_base<N, kRO>(sm, G, N + 1);
    const SmemC mid{q.ws};
    const HermStage out{stg + q.g * NB};
    const float sc = a.scale;
    const float2* __restrict__ stw = a.stw;
    CT_FOR_GROUPS(G, a.batch) {
        const long long b0 = grp_ * G;
        const long long b = b0 + q.g;
        const bool live = b < a.batch;
        const RealPairSrc src{a.in_a + (live ? b : 0) * a.in_dist, live, vec};
        if constexpr (fafct::LastPairs<N, kRO>::ok) {
            fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, src, q.sync);
            fafct::ct_last_pairs<N, kTw<N, kRO>, kRO, kR2cSel<N, false>>(
                q.t, q.ws, q.tw,
                [&](cf z) {
                    out.put(0, (z.x + z.y) * sc, 0.f);
                    out.put(N, (z.x - z.y) * sc, 0.f);
                },
                [&](int k, cf zk, cf zn) {
                    cf Xk, Xnk;
                    r2c_pair(zk, zn, __ldg(&stw[k - 1]), Xk, Xnk);
                    if (k != N - k) out.put(k, Xk.x * sc, Xk.y * sc);
                    out.put(N - k, Xnk.x * sc, Xnk.y * sc);
                });
        } else {
            ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, src, mid, q.sync);
            ct_r2c_post<N>(q.t, mid, stw, out, sc);
        }
        __syncthreads();  // every group's bins are staged
        const int nl = (int)min((long long)G, a.batch - b0);
        for (int i = threadIdx.x; i < nl * NB; i += blockDim.x) {
            const int j = i / NB, k = i - j * NB;
            const float2 v = stg[i];
            const long long o = (b0 + j) * a.out_dist + k;
            if (a.interleaved) {
                __stcs(reinterpret_cast<float2*>(a.out_a) + o, v);
            } else {
                __stcs(a.out_a + o, v.x);
                __stcs(a.out_b + o, v.y);
            }
        }
        __syncthreads();  // the staging rows are free for the next round
    }
}

// RING: each frame's first `win` samples land in the ring by bulk copy
// (frame starts 16-byte aligned, win a multiple of 4), the window is staged in
// shared memory behind the ring; otherwise the first stage loads both.
template <int N, bool RING>
__global__ void __launch_bounds__(1024) k2_stft(const float2* __restrict__ tws, const RealArgs a,
                                                int G, int K) {
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    const SmemC mid{q.ws};
    const int fpe = a.interleaved ? 2 : 1;
    auto frame = [&](long long b) {
        const long long sig = b / a.frames, f = b - sig * a.frames;
        return a.in_a + sig * a.sig_len + f * a.hop;
    };
    fafct::Ring R{};
    fafct::RingCursor c{};
    int dnext = 0;
    const float2* wsm = nullptr;
    if constexpr (RING) {
        __shared__ fafct::RingCtl ctl;
        float2* wbuf = ring_base<N, kRO>(sm, G, N + 1) + (size_t)K * N;
        for (int i = threadIdx.x; i < a.win / 2; i += blockDim.x)
            wbuf[i] = __ldg(reinterpret_cast<const float2*>(a.window) + i);
        wsm = wbuf;  // published by the barrier in ring_start
        R = fafct::ring_start(
            &ctl, ring_base<N, kRO>(sm, G, N + 1), K, N, G, a.batch,
            [&](long long b) { return (const void*)frame(b); }, (unsigned)a.win * 4u);
        c = R.cursor(q.g);
        dnext = R.next_offset(q.g);
    }
    bool first = true;
    CT_FOR_GROUPS(G, a.batch) {
        const long long b = grp_ * G + q.g;  // global frame index
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        if constexpr (RING) {
            if (!first) R.advance(c);
            first = false;
        }
        if constexpr (fafct::LastPairs<N, kRO>::ok) {
            // last stage fused with the post-pass, as in k2_r2c
            if constexpr (RING) {
                const RingHook hook =
                    ring_next_of(R, c, b, dnext, live, a.batch,
                                 [&](long long bn) { return (const void*)frame(bn); },
                                 (unsigned)a.win * 4u, q.t, a.err);
                fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(
                    q.t, q.ws, q.tw, FrameStageSrc{R.slot_ptr(c), wsm, a.win}, q.sync, hook);
            } else {
                fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(
                    q.t, q.ws, q.tw, FrameSrc{frame(bi), a.window, a.win, live}, q.sync);
            }
            if (live) {
                const long long oo = bi * a.out_dist * fpe;
                const float sc = a.scale;
                const float2* __restrict__ stw = a.stw;
                auto post = [&](const auto& out) {
                    fafct::ct_last_pairs<N, kTw<N, kRO>, kRO>(
                        q.t, q.ws, q.tw,
                        [&](cf z) {
                            out.put(0, (z.x + z.y) * sc, 0.f);
                            out.put(N, (z.x - z.y) * sc, 0.f);
                        },
                        [&](int k, cf zk, cf zn) {
                            cf Xk, Xnk;
                            r2c_pair(zk, zn, __ldg(&stw[k - 1]), Xk, Xnk);
                            if (k != N - k) out.put(k, Xk.x * sc, Xk.y * sc);
                            out.put(N - k, Xnk.x * sc, Xnk.y * sc);
                        });
                };
                if (a.interleaved)
                    post(HermInter{reinterpret_cast<float2*>(a.out_a + oo)});
                else
                    post(HermSplit{a.out_a + oo, a.out_b + oo});
            }
        } else {
            if constexpr (RING) {
                const RingHook hook =
                    ring_next_of(R, c, b, dnext, live, a.batch,
                                 [&](long long bn) { return (const void*)frame(bn); },
                                 (unsigned)a.win * 4u, q.t, a.err);
                ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw,
                                            FrameStageSrc{R.slot_ptr(c), wsm, a.win}, mid, q.sync,
                                            hook);
            } else {
                ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw,
                                            FrameSrc{frame(bi), a.window, a.win, live}, mid,
                                            q.sync);
            }
            q.sync();
            if (live) {
                const long long oo = bi * a.out_dist * fpe;
                HermSink out{a.out_a + oo, a.interleaved ? nullptr : a.out_b + oo, a.interleaved};
                ct_r2c_post<N>(q.t, mid, a.stw, out, a.scale);
            }
        }
    }
    if constexpr (RING) fafct::ring_drain(R);
}

template <int N>
struct CwtSlot {
    static constexpr int X = cwt_slot_x(N);      // float2
    static constexpr int PSI = cwt_slot_psi(N);  // floats
    static constexpr int F2 = cwt_slot_f2(N);    // float2 per slot
};

// RING (CWT rows only: interleaved spectra N + 2 bins apart, bank rows N + 4
// floats apart): each transform's spectrum and bank row land in the CTA's
// ring by two bulk copies; otherwise the pair loop loads them.
template <int N, bool RING>
__global__ void __launch_bounds__(1024) k2_c2r(const float2* __restrict__ tws, const RealArgs a,
                                               int G, bool vec, int K) {
    extern __shared__ float4 smem4[];
    constexpr int nc = N, T = P2<N>::T;
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    const SmemC mid{q.ws};
    const int fpe = a.interleaved ? 2 : 1;
    using CS = CwtSlot<N>;
    // the two parts of transform b's ring copy
    auto cwt_src = [&](long long b) {
        const long long s = b / a.filt_rows, row = b - s * a.filt_rows;
        return fafct::RingSrc2{a.in_a + s * a.in_dist * 2, a.filt + row * a.filt_dist};
    };
    fafct::Ring R{};
    fafct::RingCursor c{};
    int dnext = 0;
    if constexpr (RING) {
        __shared__ fafct::RingCtl ctl;
        R = fafct::ring_start(&ctl, ring_base<N, kRO>(sm, G, N + 1), K, CS::F2, G, a.batch, cwt_src,
                              CS::X * 8u, CS::PSI * 4u);
        c = R.cursor(q.g);
        dnext = R.next_offset(q.g);
    }
    bool first = true;
    CT_FOR_GROUPS(G, a.batch) {
        const long long b = grp_ * G + q.g;
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        const C2ROffsets o = c2r_offsets(a, bi, fpe);
        const long long io = o.io;
        const float2* xs = nullptr;  // RING: the slot's spectrum, then its bank row
        if constexpr (RING) {
            if (!first) R.advance(c);
            first = false;
            if (live && !R.wait(c) && q.t == 0) R.fail(a.err);
            xs = R.slot_ptr(c);
        }
        q.sync();  // the previous transform's last stage may still read ws
        // bin k of the input, times the bank's real weight for a CWT row
        // (src/faf_cwt_kernels.c:22-33; the imaginary parts of DC and Nyquist,
        // which that kernel zeroes, are never read by the pre-pass)
        auto load = [&](int k) {
            cf v;
            if constexpr (RING) {
                const float2 u = xs[k];
                const float w = reinterpret_cast<const float*>(xs + CS::X)[k];
                return cf{u.x * w, u.y * w};
            }
            if (a.interleaved) {
                const float2* p = reinterpret_cast<const float2*>(a.in_a + io) + k;
                const float2 u = o.f ? __ldg(p) : __ldcs(p);
                v = cf{u.x, u.y};
            } else {
                // a CWT spectrum is re-read by every row of its signal: keep it cached
                v = o.f ? cf{__ldg(a.in_a + io + k), __ldg(a.in_b + io + k)}
                        : cf{__ldcs(a.in_a + io + k), __ldcs(a.in_b + io + k)};
            }
            if (o.f) {
                const float w = __ldg(o.f + k);
                v.x *= w;
                v.y *= w;
            }
            return v;
        };
        // each thread loads whole bin pairs (k, nc - k) and runs the pre-pass
        // on them in registers: one workspace write per bin
        if (live) {
            // a compile-time trip count lets the loads of every pair issue
            // before the first one returns (they come from L2 for CWT rows)
            constexpr int MP = (nc / 2 + T) / T;
#pragma unroll
            for (int i = 0; i < MP; i++) {
                const int k = q.t + i * T;
                if (k <= nc / 2) {
                    const cf xk = load(k), xn = load(nc - k);
                    if (k == 0) {
                        mid.put(0, cf{xk.x + xn.x, xk.x - xn.x});
                    } else {
                        cf Zk, Znk;
                        c2r_pair(xk, xn, __ldg(&a.stw[k - 1]), Zk, Znk);
                        if (k != nc - k) mid.put(k, Zk);
                        mid.put(nc - k, Znk);
                    }
                }
            }
        }
        q.sync();
        if constexpr (RING) {
            // every thread of the group has read the slot: load the group's
            // transform K sequence places on into it
            const long long bn = b + dnext;
            if (q.t == 0 && live && bn < a.batch) {
                const fafct::RingSrc2 p = cwt_src(bn);
                R.issue(c.slot, c.use + 1, p.p0, CS::X * 8u, p.p1, CS::PSI * 4u);
            }
        }
        ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, SmemCConj{q.ws},
                          RealPairSink{a.out_a + o.oo, a.scale, live, vec}, q.sync);
    }
    if constexpr (RING) fafct::ring_drain(R);
}

// C2R of power-of-two inner lengths from 32 points (no filter rows): each
// transform's bins land in its group's workspace by bulk copy (faf_land.cuh),
// issued for the group's next transform once the last stage has read the
// workspace.  The pre-pass reads every bin pair the thread owns into
// registers before the group writes the workspace.
template <int N>
__global__ void __launch_bounds__(1024) k2_c2r_land(const float2* __restrict__ tws,
                                                    const RealArgs a, int G, bool vec) {
    extern __shared__ float4 smem4[];
    constexpr int nc = N, T = P2<N, kRO>::T, NS = P2<N, kRO>::NS;
    constexpr int MP = (nc / 2 + T) / T;
    static_assert(NS >= 2, "at least two stages");
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    using Ctl = LandCtlN<(T >= 32 ? 16 : kLandMaxGroups)>;
    __shared__ Ctl ctl;
    const SmemC mid{q.ws};
    const int fpe = a.interleaved ? 2 : 1;
    LandPlanes<Ctl> L{&ctl, q.g, reinterpret_cast<float*>(q.ws), N + 4};
    L.init(q.t);
    __syncthreads();
    auto plane = [&](long long b, int k) -> const float* {
        return k == 0 ? a.in_a + b * a.in_dist * fpe
                      : (a.interleaved ? nullptr : a.in_b + b * a.in_dist * fpe);
    };
    const long long stride = (long long)gridDim.x * G;
    long long b = (long long)blockIdx.x * G + q.g;
    if (q.t == 0 && b < a.batch) L.issue(plane(b, 0), plane(b, 1), nc + 1);
    for (; b - q.g < a.batch; b += stride) {  // the same trip count for every group
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        if (live) L.wait(a.err, q.t);
        const float* lr = L.first(plane(bi, 0));
        const float* li = a.interleaved ? nullptr : L.second(plane(bi, 1));
        auto get = [&](int k) -> cf {
            if (a.interleaved) {
                const float2 u = reinterpret_cast<const float2*>(lr)[k];
                return cf{u.x, u.y};
            }
            return cf{lr[k], li[k]};
        };
        cf xk[MP], xn[MP];
#pragma unroll
        for (int i = 0; i < MP; i++) {
            const int k = q.t + i * T;
            if (k <= nc / 2) {
                xk[i] = get(k);
                xn[i] = get(nc - k);
            }
        }
        q.sync();  // the group has read the landed bins
        if (live) {
#pragma unroll
            for (int i = 0; i < MP; i++) {
                const int k = q.t + i * T;
                if (k <= nc / 2) {
                    if (k == 0) {
                        mid.put(0, cf{xk[i].x + xn[i].x, xk[i].x - xn[i].x});
                    } else {
                        cf Zk, Znk;
                        c2r_pair(xk[i], xn[i], __ldg(&a.stw[k - 1]), Zk, Znk);
                        if (k != nc - k) mid.put(k, Zk);
                        mid.put(nc - k, Znk);
                    }
                }
            }
        }
        q.sync();
        fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, SmemCConj{q.ws}, q.sync);
        float xr[16], xi[16];
        const long long bn = b + stride;
        fafct::ct_stage<N, NS - 1, kTw<N, kRO>, kRO>(
            xr, xi, q.t, q.tw, SmemC{q.ws},
            fafct::LastC<RealPairSink>{RealPairSink{a.out_a + bi * a.out_dist, a.scale, live, vec}},
            q.sync, [&]() {
                q.sync();  // the whole group has read the workspace
                if (q.t == 0 && bn < a.batch) L.issue(plane(bn, 0), plane(bn, 1), nc + 1);
            });
    }
    L.drain(q.t);
}

// Per bin pair of the pipeline: post-pass -> ops -> pre-pass, in registers,
// in place on the workspace.
template <int N, class Ops>
__device__ __forceinline__ void pipe_middle(int t, const SmemC& mid,
                                            const float2* __restrict__ stw, const Ops& ops) {
    constexpr int nc = N, T = P2<N>::T;
    for (int k = t; k <= nc / 2; k += T) {
        if (k == 0) {
            const cf z = mid.get(0);
            const cf x0 = ops(0, cf{z.x + z.y, 0.f});
            const cf xn = ops(nc, cf{z.x - z.y, 0.f});
            mid.put(0, cf{x0.x + xn.x, x0.x - xn.x});
        } else {
            const float2 w = __ldg(&stw[k - 1]);
            cf Xk, Xnk;
            r2c_pair(mid.get(k), mid.get(nc - k), w, Xk, Xnk);
            if (k == nc - k) Xk = Xnk;
            Xk = ops(k, Xk);
            Xnk = (k == nc - k) ? Xk : ops(nc - k, Xnk);
            cf Zk, Znk;
            c2r_pair(Xk, Xnk, w, Zk, Znk);
            if (k != nc - k) mid.put(k, Zk);
            mid.put(nc - k, Znk);
        }
    }
}

// The same bin-pair pass fused with the forward transform's last stage
// (fafct::ct_last_pairs): each thread transforms the bins it owns in
// registers and writes the pre-pass result back to those same slots.
// pair_ops serves the bins of the pairs (1 .. N - 1), ops DC and Nyquist.
// STW_SMEM: the super-twiddles are in shared memory (staged tables).
template <int N, int SEL = -1, bool STW_SMEM = false, class Ops, class PairOps = Ops>
__device__ __forceinline__ void pipe_middle_fused(int t, float2* ws, const float2* tw,
                                                  const float2* __restrict__ stw, const Ops& ops,
                                                  const PairOps& pair_ops) {
    const SmemC mid{ws};
    fafct::ct_last_pairs<N, kTw<N, kRO>, kRO, SEL>(
        t, ws, tw,
        [&](cf z) {
            const cf x0 = ops(0, cf{z.x + z.y, 0.f});
            const cf xn = ops(N, cf{z.x - z.y, 0.f});
            mid.put(0, cf{x0.x + xn.x, x0.x - xn.x});
        },
        [&](int k, cf zk, cf zn) {
            const float2 w = STW_SMEM ? stw[k - 1] : __ldg(&stw[k - 1]);
            cf Xk, Xnk;
            r2c_pair(zk, zn, w, Xk, Xnk);
            if (k == N - k) Xk = Xnk;
            Xk = pair_ops(k, Xk);
            Xnk = (k == N - k) ? Xk : pair_ops(N - k, Xnk);
            cf Zk, Znk;
            c2r_pair(Xk, Xnk, w, Zk, Znk);
            if (k != N - k) mid.put(k, Zk);
            mid.put(N - k, Znk);
        });
}

template <int N, bool RING>
__global__ void __launch_bounds__(1024) k2_pipeline(const float2* __restrict__ tws,
                                                    const RealArgs a, int G, bool vec, int K) {
    extern __shared__ float4 smem4[];
    float2* sm = reinterpret_cast<float2*>(smem4);
    CtGroup<N, kRO> q(sm, N + 1, tws);
    const SmemC mid{q.ws};
    fafct::Ring R{};
    if constexpr (RING) {
        __shared__ fafct::RingCtl ctl;
        R = real_ring<N>(&ctl, sm, G, K, a);
    }
    fafct::RingCursor c{};
    int dnext = 0;
    if constexpr (RING) {
        c = R.cursor(q.g);
        dnext = R.next_offset(q.g);
    }
    // staged tables (a single MUL by a spectrum of all N + 1 bins): its
    // planes and the super-twiddles, copied once per CTA behind the ring
    bool staged = false;
    if constexpr (RING && fafct::LastPairs<N, kRO>::ok) {
        if (a.stage_tables) {
            float* tab = reinterpret_cast<float*>(ring_base<N, kRO>(sm, G, N + 1) + (size_t)K * N);
            for (int i = threadIdx.x; i <= N; i += blockDim.x) {
                tab[i] = __ldg(a.ops[0].hr + i);
                tab[N + 4 + i] = __ldg(a.ops[0].hi_ + i);
            }
            float2* st = reinterpret_cast<float2*>(tab + 2 * (N + 4));
            for (int i = threadIdx.x; i < N / 2; i += blockDim.x) st[i] = __ldg(a.stw + i);
            __syncthreads();
            staged = true;
        }
    }
    bool first = true;
    CT_FOR_GROUPS(G, a.batch) {
        if constexpr (RING) {
            if (!first) R.advance(c);
            first = false;
        }
        const long long b = grp_ * G + q.g;
        const bool live = b < a.batch;
        const long long bi = live ? b : 0;
        if constexpr (fafct::LastPairs<N, kRO>::ok) {
            if constexpr (RING) {
                const RingHook hook =
                    ring_next(R, c, b, dnext, live, a.in_a, a.in_dist, a.batch, N * 8u, q.t,
                              a.err);
                fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, fafct::StageSrc{R.slot_ptr(c)},
                                                  q.sync, hook);
            } else {
                fafct::ct_fft_but_last<N, kTw<N, kRO>, kRO>(
                    q.t, q.ws, q.tw, RealPairSrc{a.in_a + bi * a.in_dist, live, vec}, q.sync);
            }
            // a single MUL by a spectrum bound over every bin: no guard on the
            // pairs' bins (mul_bin's guards only act on DC and Nyquist there);
            // any other program (a shorter spectrum included) runs the op loop
            // (the ring kernel's host always stages that case's tables)
            if (RING && staged) {
                // the real plane, then the imaginary one, then the super-twiddles
                const float* tab =
                    reinterpret_cast<const float*>(ring_base<N, kRO>(sm, G, N + 1) + (size_t)K * N);
                pipe_middle_fused<N, kR2cSel<N, RING>, true>(
                    q.t, q.ws, q.tw, reinterpret_cast<const float2*>(tab + 2 * (N + 4)),
                    OpsMul1{&a.ops[0]}, OpsMulSmem{tab, tab + N + 4});
            }
            else if (!RING && ops_single_mul(a) && a.ops[0].m == N + 1)
                pipe_middle_fused<N, kR2cSel<N, RING>>(q.t, q.ws, q.tw, a.stw, OpsMul1{&a.ops[0]},
                                                       OpsMul1Full{&a.ops[0]});
            else
                pipe_middle_fused<N>(q.t, q.ws, q.tw, a.stw, OpsAny{&a}, OpsAny{&a});
        } else {
            if constexpr (RING) {
                const RingHook hook =
                    ring_next(R, c, b, dnext, live, a.in_a, a.in_dist, a.batch, N * 8u, q.t,
                              a.err);
                ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, fafct::StageSrc{R.slot_ptr(c)}, mid, q.sync, hook);
            } else {
                ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw,
                                  RealPairSrc{a.in_a + bi * a.in_dist, live, vec}, mid, q.sync);
            }
            q.sync();
            if (ops_single_mul(a))
                pipe_middle<N>(q.t, mid, a.stw, OpsMul1{&a.ops[0]});
            else
                pipe_middle<N>(q.t, mid, a.stw, OpsAny{&a});
        }
        q.sync();
        ct_fft<N, kTw<N, kRO>, kRO>(q.t, q.ws, q.tw, SmemCConj{q.ws},
                          RealPairSink{a.out_a + bi * a.out_dist, a.scale, live, vec}, q.sync);
    }
    if constexpr (RING) fafct::ring_drain(R);
}

// ---------------------------------------------------------------------------
// launch by log2 length (persistent grid = resident CTAs, capped by work)
// ---------------------------------------------------------------------------

template <class K>
static unsigned persistent_grid(K kernel, const Geometry& g, long long batch) {
    const int sms = fafk::sm_count();
    const int per_sm = resident_ctas(kernel, g.threads, g.smem);
    const long long groups = (batch + g.G - 1) / g.G;
    const long long cap = (long long)sms * per_sm;
    return (unsigned)std::max(1LL, std::min(groups, cap));
}

// The ring needs groups of at least one warp (T = N / 16 >= 32); shorter
// lengths are built without it.
template <int N>
constexpr bool kRingN = N >= 512;

template <int N, int ORD = 0>
static size_t tw_bytes() {
    return (size_t)CtCfg<N, ORD>::TWN * sizeof(float2);
}

template <int N>
static cudaError_t ct_launch(int kind, const float2* tws, const void* args, Geometry g,
                             cudaStream_t st) {
    cudaError_t e;
    g.smem += kind == 0 ? tw_bytes<N>() : tw_bytes<N, kRO>();
    switch (kind) {
    case 0: {
        const C2CArgs& a = *(const C2CArgs*)args;
        if constexpr (N == 64) {
            if (a.land && a.stage_out) {
                if ((e = prep(k2_c2c_land<N, true>, g.smem)) != cudaSuccess) return e;
                k2_c2c_land<N, true><<<persistent_grid(k2_c2c_land<N, true>, g, a.batch),
                                       g.threads, g.smem, st>>>(tws, a, g.G);
                break;
            }
        }
        if constexpr (N >= 64) {
            if (a.land) {
                if ((e = prep(k2_c2c_land<N>, g.smem)) != cudaSuccess) return e;
                k2_c2c_land<N><<<persistent_grid(k2_c2c_land<N>, g, a.batch), g.threads, g.smem,
                                 st>>>(tws, a, g.G);
                break;
            }
        }
        if ((e = prep(k2_c2c<N>, g.smem)) != cudaSuccess) return e;
        k2_c2c<N><<<persistent_grid(k2_c2c<N>, g, a.batch), g.threads, g.smem, st>>>(tws, a, g.G);
        break;
    }
    case 1: {
        const RealArgs& a = *(const RealArgs*)args;
        if constexpr (N >= 32 && N <= 128) {
            if (a.stage_out) {
                if ((e = prep(k2_r2c_small<N>, g.smem)) != cudaSuccess) return e;
                k2_r2c_small<N><<<persistent_grid(k2_r2c_small<N>, g, a.batch), g.threads,
                                  g.smem, st>>>(tws, a, g.G, vec_ok(a.in_a, a.in_dist));
                break;
            }
        }
        if constexpr (N == 256) {
            if (a.land) {
                if ((e = prep(k2_r2c_land<N>, g.smem)) != cudaSuccess) return e;
                k2_r2c_land<N><<<persistent_grid(k2_r2c_land<N>, g, a.batch), g.threads, g.smem,
                                 st>>>(tws, a, g.G);
                break;
            }
        }
        if (kRingN<N> && g.ring) {
            if ((e = prep(k2_r2c<N, kRingN<N>>, g.smem)) != cudaSuccess) return e;
            k2_r2c<N, kRingN<N>><<<persistent_grid(k2_r2c<N, kRingN<N>>, g, a.batch), g.threads,
                                   g.smem, st>>>(tws, a, g.G, true, g.ring);
        } else {
            if ((e = prep(k2_r2c<N, false>, g.smem)) != cudaSuccess) return e;
            k2_r2c<N, false><<<persistent_grid(k2_r2c<N, false>, g, a.batch), g.threads, g.smem,
                               st>>>(tws, a, g.G, vec_ok(a.in_a, a.in_dist), 0);
        }
        break;
    }
    case 2: {
        const RealArgs& a = *(const RealArgs*)args;
        if (kRingN<N> && g.ring) {
            if ((e = prep(k2_c2r<N, kRingN<N>>, g.smem)) != cudaSuccess) return e;
            k2_c2r<N, kRingN<N>><<<persistent_grid(k2_c2r<N, kRingN<N>>, g, a.batch), g.threads,
                                   g.smem, st>>>(tws, a, g.G, vec_ok(a.out_a, a.out_dist),
                                                 g.ring);
        } else {
            if constexpr (N >= 32) {
                if (a.land) {
                    if ((e = prep(k2_c2r_land<N>, g.smem)) != cudaSuccess) return e;
                    k2_c2r_land<N><<<persistent_grid(k2_c2r_land<N>, g, a.batch), g.threads,
                                     g.smem, st>>>(tws, a, g.G, vec_ok(a.out_a, a.out_dist));
                    break;
                }
            }
            if ((e = prep(k2_c2r<N, false>, g.smem)) != cudaSuccess) return e;
            k2_c2r<N, false><<<persistent_grid(k2_c2r<N, false>, g, a.batch), g.threads, g.smem,
                               st>>>(tws, a, g.G, vec_ok(a.out_a, a.out_dist), 0);
        }
        break;
    }
    case 3: {
        const RealArgs& a = *(const RealArgs*)args;
        const bool vec = vec_ok(a.in_a, a.in_dist) && vec_ok(a.out_a, a.out_dist);
        if (kRingN<N> && g.ring) {
            if ((e = prep(k2_pipeline<N, kRingN<N>>, g.smem)) != cudaSuccess) return e;
            k2_pipeline<N, kRingN<N>><<<persistent_grid(k2_pipeline<N, kRingN<N>>, g, a.batch),
                                        g.threads, g.smem, st>>>(tws, a, g.G, vec, g.ring);
        } else {
            if ((e = prep(k2_pipeline<N, false>, g.smem)) != cudaSuccess) return e;
            k2_pipeline<N, false><<<persistent_grid(k2_pipeline<N, false>, g, a.batch),
                                    g.threads, g.smem, st>>>(tws, a, g.G, vec, 0);
        }
        break;
    }
    case 4: {
        const RealArgs& a = *(const RealArgs*)args;
        if (kRingN<N> && g.ring) {
            if ((e = prep(k2_stft<N, kRingN<N>>, g.smem)) != cudaSuccess) return e;
            k2_stft<N, kRingN<N>><<<persistent_grid(k2_stft<N, kRingN<N>>, g, a.batch),
                                    g.threads, g.smem, st>>>(tws, a, g.G, g.ring);
        } else {
            if ((e = prep(k2_stft<N, false>, g.smem)) != cudaSuccess) return e;
            k2_stft<N, false><<<persistent_grid(k2_stft<N, false>, g, a.batch), g.threads,
                                g.smem, st>>>(tws, a, g.G, 0);
        }
        break;
    }
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <int N>
static cudaError_t prepare_c2c_n(const Geometry& g) {
    return prep(k2_c2c<N>, g.smem + tw_bytes<N>());
}

cudaError_t prepare_pot2_c2c(int log2n, const Geometry& g) {
    switch (log2n) {
    case 4: return prepare_c2c_n<16>(g);
    case 5: return prepare_c2c_n<32>(g);
    case 6: return prepare_c2c_n<64>(g);
    case 7: return prepare_c2c_n<128>(g);
    case 8: return prepare_c2c_n<256>(g);
    case 9: return prepare_c2c_n<512>(g);
    case 10: return prepare_c2c_n<1024>(g);
    case 11: return prepare_c2c_n<2048>(g);
    case 12: return prepare_c2c_n<4096>(g);
    case 13: return prepare_c2c_n<8192>(g);
    case 14: return prepare_c2c_n<16384>(g);
    default: return cudaErrorInvalidValue;
    }
}

size_t pot2_table_smem(int log2n, int ord) {
    switch (log2n * 2 + (ord ? 1 : 0)) {
#define FAF_TB(L, N)                          \
    case 2 * L: return tw_bytes<N>();         \
    case 2 * L + 1: return tw_bytes<N, kRO>();
        FAF_TB(4, 16) FAF_TB(5, 32) FAF_TB(6, 64) FAF_TB(7, 128) FAF_TB(8, 256) FAF_TB(9, 512)
        FAF_TB(10, 1024) FAF_TB(11, 2048) FAF_TB(12, 4096) FAF_TB(13, 8192) FAF_TB(14, 16384)
#undef FAF_TB
    default: return 0;
    }
}

cudaError_t launch_pot2(int kind, int log2n, const float2* tws, const void* args,
                        const Geometry& g, cudaStream_t st) {
    switch (log2n) {
    case 4: return ct_launch<16>(kind, tws, args, g, st);
    case 5: return ct_launch<32>(kind, tws, args, g, st);
    case 6: return ct_launch<64>(kind, tws, args, g, st);
    case 7: return ct_launch<128>(kind, tws, args, g, st);
    case 8: return ct_launch<256>(kind, tws, args, g, st);
    case 9: return ct_launch<512>(kind, tws, args, g, st);
    case 10: return ct_launch<1024>(kind, tws, args, g, st);
    case 11: return ct_launch<2048>(kind, tws, args, g, st);
    case 12: return ct_launch<4096>(kind, tws, args, g, st);
    case 13: return ct_launch<8192>(kind, tws, args, g, st);
    case 14: return ct_launch<16384>(kind, tws, args, g, st);
    default: return cudaErrorInvalidValue;
    }
}

}  // namespace fafk
