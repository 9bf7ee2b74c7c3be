// faf_pot2_group.cuh -- per-CTA shared-memory layout of the compile-time
// power-of-two kernels (k_pot2.cu, k_tc.cu): twiddle table, then one
// workspace per transform group.
#pragma once

#include "faf_kernels_common.cuh"
#include "faf_pot2.cuh"

namespace fafk {

using fafct::P2;
using fafct::plane2;

// Shared-memory layout of one CTA:
//   [twiddle table, if it fits 32 KB] [group 0 workspace] [group 1 ...] ...
//   [input ring slots, kernels that land their input by bulk copy]
// Every region is a whole number of 16-byte units (an even float2 count):
// bulk copies need 16-byte aligned shared-memory destinations.
__host__ __device__ constexpr int even2(int x) { return (x + 1) & ~1; }

template <int N, int ORD = 0>
struct CtCfg {
    // up to 56 KB: every table (36 KB for 16384-point C2C, 52 KB for the real
    // kinds' 16384-point inner FFT, with their split stages)
    static constexpr bool TW_SMEM = P2<N, ORD>::TW * 8 <= 57344;
    static constexpr int TWN = TW_SMEM ? even2(P2<N, ORD>::TW > 0 ? P2<N, ORD>::TW : 1) : 0;
};

// float2 units of one group's workspace
__host__ __device__ constexpr int group_stride(int n, int slots) {
    return (void)n, even2(plane2(slots));
}

template <int N, int ORD = 0>
struct CtGroup {
    int g, t;
    float2* ws;
    const float2* tw;
    fafct::GroupSync sync;
    __device__ __forceinline__ CtGroup(float2* sm, int slots, const float2* __restrict__ gtw) {
        constexpr int T = P2<N>::T;
        g = threadIdx.x / T;
        t = threadIdx.x % T;
        if constexpr (CtCfg<N, ORD>::TW_SMEM) {
            for (int i = threadIdx.x; i < CtCfg<N, ORD>::TWN; i += blockDim.x)
                sm[i] = __ldg(&gtw[i]);
            tw = sm;
        } else {
            tw = gtw;
        }
        ws = sm + CtCfg<N, ORD>::TWN + (size_t)g * group_stride(N, slots);
        sync = fafct::GroupSync::make(g, T);
        // publish the twiddle table to the whole CTA once
        if constexpr (CtCfg<N, ORD>::TW_SMEM) __syncthreads();
    }
};

template <int N, int ORD = 0>
constexpr bool kTw = CtCfg<N, ORD>::TW_SMEM;

// First ring slot behind the G group workspaces.
template <int N, int ORD = 0>
__device__ __forceinline__ float2* ring_base(float2* sm, int G, int slots) {
    return sm + CtCfg<N, ORD>::TWN + (size_t)G * group_stride(N, slots);
}

// Persistent loop over transform groups; uniform across the CTA.
#define CT_FOR_GROUPS(G, batch)                                                          \
    for (long long grp_ = blockIdx.x, ngrp_ = ((batch) + (G)-1) / (G); grp_ < ngrp_;     \
         grp_ += gridDim.x)

}  // namespace fafk
