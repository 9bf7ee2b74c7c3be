// faf_land.cuh -- a C2C transform's input landed in its group's workspace by
// bulk copies (k2_c2c_land, the tensor-core kernels).
//
// One transform per group fills the workspace, so there is no room for a
// separate input ring.  Instead each transform's planes are copied to the
// start of the workspace (re, then im kPl floats further on, or the
// interleaved pairs), the first stage reads them there and overwrites them
// after its barrier, and the copy of the group's next transform is issued as
// soon as the last stage has read the workspace.  A bulk copy moves whole
// 16-byte blocks, so a plane whose start is not 16-byte aligned is copied
// from the block boundary at or below its start, and read `head` floats in;
// the blocks read beyond the plane share its 16-byte blocks, so they never
// reach another page.  Every distance, offset list and base alignment lands
// this way.  The copy completes on the group's mbarrier; every wait is
// bounded, and after one runs out the kernel records the failure, issues
// nothing more and drains what it issued before it exits.
#pragma once

#include "faf_kernels_common.cuh"
#include "faf_ring.cuh"

namespace fafk {

// The landed input as the first stage's source (shared memory: the stage
// reads it all before its barrier, then writes over it).
struct LandSrc {
    const float* re;  // first element of the real plane (or of the pairs)
    const float* im;  // first element of the imaginary plane
    int inter;
    float sgn;
    static constexpr bool kSmem = true;
    __device__ __forceinline__ cf get(int i) const {
        if (inter) {
            const float2 v = reinterpret_cast<const float2*>(re)[i];
            return cf{v.x, sgn * v.y};
        }
        return cf{re[i], sgn * im[i]};
    }
};

// `bytes` (a multiple of 16) from the 16-byte aligned `src` to shared
// address `dst`, completing on the mbarrier at `mb`.
__device__ __forceinline__ void land_copy(unsigned dst, const float* src, unsigned bytes,
                                          unsigned mb) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
                 "[%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(mb)
                 : "memory");
}

// Static shared memory of a landing kernel: one mbarrier per group.
template <int MAXG>
struct LandCtlN {
    uint64_t bar[MAXG];
    int failed;
};
using LandCtl = LandCtlN<16>;

// One group's landing: its mbarrier and workspace.  `issued` is counted by
// the group's thread 0, `waited` by every thread of the group.  The
// workspace holds 2 N + 8 floats.
template <int N, class Ctl = LandCtl>
struct Lander {
    static constexpr int kPl = N + 4;  // floats from the landed real plane to the imaginary one
    Ctl* ctl;
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
    // Transform b's planes in global memory.
    __device__ __forceinline__ static const float* plane(const C2CArgs& a, long long b, int p) {
        const long long io = (a.offs ? a.offs[b] : b * a.in_dist) * (a.interleaved ? 2 : 1);
        return (p == 0 ? a.in_re : a.in_im) + io;
    }
    __device__ __forceinline__ static unsigned head_bytes(const float* p) {
        return (unsigned)(reinterpret_cast<uintptr_t>(p) & 15u);
    }
    // Thread 0 of the group: transform b's input into the workspace.
    __device__ __forceinline__ void issue(const C2CArgs& a, long long b) {
        if (*(volatile int*)&ctl->failed) return;
        const unsigned mb = fafct::smem_addr(&ctl->bar[g]);
        const unsigned dst = fafct::smem_addr(land);
        const float* p0 = plane(a, b, 0);
        const unsigned h0 = head_bytes(p0);
        const unsigned n0 = (h0 + (a.interleaved ? 8u : 4u) * N + 15u) & ~15u;
        unsigned n1 = 0, h1 = 0;
        const float* p1 = nullptr;
        if (!a.interleaved) {
            p1 = plane(a, b, 1);
            h1 = head_bytes(p1);
            n1 = (h1 + 4u * N + 15u) & ~15u;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                     "r"(n0 + n1)
                     : "memory");
        land_copy(dst, p0 - h0 / 4, n0, mb);
        if (!a.interleaved) land_copy(dst + 4u * kPl, p1 - h1 / 4, n1, mb);
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
    // Transform b (one that landed here) as the first stage's source.
    __device__ __forceinline__ LandSrc src(const C2CArgs& a, long long b) const {
        const unsigned h0 = head_bytes(plane(a, b, 0)) / 4;
        const unsigned h1 = a.interleaved ? 0u : head_bytes(plane(a, b, 1)) / 4;
        return LandSrc{land + h0, land + kPl + h1, a.interleaved, a.sgn};
    }
};

// One group's landing of two planes of `nf` floats each (or one interleaved
// plane of nf pairs) into its workspace, the second plane `pl` floats after
// the first; each copied from the 16-byte block at or below its start.  The
// workspace holds 2 pl floats, pl >= nf + 3 rounded up to a multiple of 4.
template <class Ctl = LandCtl>
struct LandPlanes {
    Ctl* ctl;
    int g;
    float* land;
    int pl;
    int issued = 0, waited = 0;

    __device__ __forceinline__ void init(int t) {
        if (t == 0)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(
                             fafct::smem_addr(&ctl->bar[g]))
                         : "memory");
        if (threadIdx.x == 0) ctl->failed = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __device__ __forceinline__ static unsigned head_bytes(const float* p) {
        return (unsigned)(reinterpret_cast<uintptr_t>(p) & 15u);
    }
    // Thread 0 of the group: planes p0 (and p1, unless null: p0 is then nf
    // interleaved pairs).
    __device__ __forceinline__ void issue(const float* p0, const float* p1, int nf) {
        if (*(volatile int*)&ctl->failed) return;
        const unsigned mb = fafct::smem_addr(&ctl->bar[g]);
        const unsigned dst = fafct::smem_addr(land);
        const unsigned h0 = head_bytes(p0);
        const unsigned n0 = (h0 + (p1 ? 4u : 8u) * (unsigned)nf + 15u) & ~15u;
        const unsigned h1 = p1 ? head_bytes(p1) : 0u;
        const unsigned n1 = p1 ? ((h1 + 4u * (unsigned)nf + 15u) & ~15u) : 0u;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(mb),
                     "r"(n0 + n1)
                     : "memory");
        land_copy(dst, p0 - h0 / 4, n0, mb);
        if (p1) land_copy(dst + 4u * (unsigned)pl, p1 - h1 / 4, n1, mb);
        issued++;
    }
    __device__ __forceinline__ void wait(int* err, int t) {
        for (int i = 0; i < fafct::kRingSpin && !*(volatile int*)&ctl->failed; i++)
            if (fafct::mbar_test(&ctl->bar[g], (unsigned)(waited & 1))) {
                waited++;
                return;
            }
        if (t == 0) {
            *(volatile int*)&ctl->failed = 1;
            if (err) atomicOr(err, 2);
        }
    }
    __device__ __forceinline__ void drain(int t) {
        if (t != 0 || issued <= waited) return;
        for (int i = 0; i < fafct::kRingSpin; i++)
            if (fafct::mbar_test(&ctl->bar[g], (unsigned)((issued - 1) & 1))) break;
    }
    // The landed planes' first elements (p0's pairs when p1 is null).
    __device__ __forceinline__ const float* first(const float* p0) const {
        return land + head_bytes(p0) / 4;
    }
    __device__ __forceinline__ const float* second(const float* p1) const {
        return land + pl + head_bytes(p1) / 4;
    }
};

}  // namespace fafk
