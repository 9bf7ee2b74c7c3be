// faf_land.cuh -- a C2C transform's input landed in its group's workspace by
// bulk copies (k2_c2c_land, k2_c2c_tc for 8192 / 16384 points).
//
// One transform per group fills the workspace, so there is no room for a
// separate input ring.  Instead each transform's planes are copied to the
// start of the workspace (re[N] then im[N], or N interleaved pairs), the
// first stage reads them there and overwrites them after its barrier, and
// the copy of the group's next transform is issued as soon as the last stage
// has read the workspace.  The copy completes on the group's mbarrier; every
// wait is bounded, and after one runs out the kernel records the failure,
// issues nothing more and drains what it issued before it exits.
#pragma once

#include "faf_kernels_common.cuh"
#include "faf_ring.cuh"

namespace fafk {

// The landed input as the first stage's source (shared memory: the stage
// reads it all before its barrier, then writes over it).
struct LandSrc {
    const float* d;
    int n;
    int inter;
    float sgn;
    static constexpr bool kSmem = true;
    __device__ __forceinline__ cf get(int i) const {
        if (inter) {
            const float2 v = reinterpret_cast<const float2*>(d)[i];
            return cf{v.x, sgn * v.y};
        }
        return cf{d[i], sgn * d[n + i]};
    }
};

struct LandCtl {  // static shared memory of a landing kernel
    uint64_t bar[16];
    int failed;
};

// One group's landing: its mbarrier and workspace.  `issued` is counted by
// the group's thread 0, `waited` by every thread of the group.
template <int N>
struct Lander {
    LandCtl* ctl;
    int g;
    float* land;
    int issued = 0, waited = 0;

    // Whole CTA, once: the groups' mbarriers (threads with t == 0 of each group).
    __device__ __forceinline__ void init(int t) {
        if (t == 0)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
                             fafct::smem_addr(&ctl->bar[g]))
                         : "memory");
        if (threadIdx.x == 0) ctl->failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // Thread 0 of the group: transform b's input into the workspace.
    __device__ __forceinline__ void issue(const C2CArgs& a, long long b) {
        if (*(volatile int*)&ctl->failed) return;
        const unsigned mb = fafct::smem_addr(&ctl->bar[g]);
        const long long io = b * a.in_dist * (a.interleaved ? 2 : 1);
        const unsigned dst = fafct::smem_addr(land);
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                     "r"((unsigned)(N * 8))
                     : "memory");
        if (a.interleaved) {
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                         "[%0], [%1], %2, [%3];" ::"r"(dst),
                         "l"(a.in_re + io), "r"((unsigned)(N * 8)), "r"(mb)
                         : "memory");
        } else {
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                         "[%0], [%1], %2, [%3];" ::"r"(dst),
                         "l"(a.in_re + io), "r"((unsigned)(N * 4)), "r"(mb)
                         : "memory");
            asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                         "[%0], [%1], %2, [%3];" ::"r"(dst + N * 4u),
                         "l"(a.in_im + io), "r"((unsigned)(N * 4)), "r"(mb)
                         : "memory");
        }
        issued++;
    }
    // Every thread of the group: the current transform has landed.
    __device__ __forceinline__ void wait(const C2CArgs& a, int t) {
        for (int i = 0; i < fafct::kRingSpin && !*(volatile int*)&ctl->failed; i++)
            if (fafct::mbar_test(&ctl->bar[g], (unsigned)(waited & 1))) {
                waited++;
                return;
            }
        if (t == 0) {
            *(volatile int*)&ctl->failed = 1;
            if (a.err) atomicOr(a.err, 2);
        }
    }
    // Thread 0 of the group, after the last transform: nothing in flight.
    __device__ __forceinline__ void drain(int t) {
        if (t != 0 || issued <= waited) return;
        for (int i = 0; i < fafct::kRingSpin; i++)
            if (fafct::mbar_test(&ctl->bar[g], (unsigned)((issued - 1) & 1))) break;
    }
    __device__ __forceinline__ LandSrc src(const C2CArgs& a) const {
        return LandSrc{land, N, a.interleaved, a.sgn};
    }
};

}  // namespace fafk
