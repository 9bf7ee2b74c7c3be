// faf_ring.cuh -- input landing ring of the persistent power-of-two kernels.
//
// K shared-memory slots, shared by the G transform groups of a CTA, receive
// each transform's input by one bulk copy (cp.async.bulk, completed on the
// slot's mbarrier).  The CTA walks its transforms in a fixed local sequence
// s = round * G + g; transform s lands in slot s % K as that slot's copy
// number s / K, and the group that consumes s issues the copy of s + K into
// the same slot as soon as its first stage has read the slot.  A copy is thus
// in flight for about K / G of a round before it is needed, while the groups
// keep all their warps and the input costs no load instructions.
//
// Parity aliasing: an mbarrier parity test cannot tell phase m from m + 2,
// so the consumer of copy m of a slot first waits until that copy has been
// issued (the slot's count of issued copies), which happens only after the
// consumer of copy m - 1 saw its phase complete.  Every wait is bounded; on a
// timeout the kernel sets an error flag, stops issuing and, before it exits,
// waits (bounded) for the copies it has in flight.
#pragma once

#include <cstdint>
#include <type_traits>

namespace fafct {

constexpr int kRingMax = 8;          // slots per CTA
constexpr int kRingSpin = 1 << 22;   // bound of every ring wait

struct RingCtl {                     // static shared memory of a ring kernel
    uint64_t bar[kRingMax];
    int issued[kRingMax];            // copies issued into each slot so far
    int failed;                      // a wait ran out: issue nothing more
};

__device__ __forceinline__ unsigned smem_addr(const void* p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ bool mbar_test(const uint64_t* bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// One group's place in its CTA's sequence: the slot of its current transform
// and that transform's copy number in the slot.  Advanced by G transforms per
// round without a division.
struct RingCursor {
    int slot, use;
};

// A value built from kernel constants (a static shared address, the dynamic
// shared base, launch parameters): cheap to copy, nothing to keep live.
struct Ring {
    RingCtl* ctl;
    float2* slots;     // K * slot_f2 float2, 16-byte aligned
    int K, slot_f2, G;

    // global transform index of local sequence s of this CTA
    __device__ __forceinline__ long long transform(long long s) const {
        return ((long long)blockIdx.x + (s / G) * (long long)gridDim.x) * G + s % G;
    }
    // transform(s + K) - transform(s) for the transforms s of group g
    __device__ __forceinline__ int next_offset(int g) const {
        const int gk = g + K;
        return (gk / G) * (int)gridDim.x * G + gk % G - g;
    }
    __device__ __forceinline__ RingCursor cursor(int g) const { return RingCursor{g % K, g / K}; }
    __device__ __forceinline__ void advance(RingCursor& c) const {
        c.slot += G;
        while (c.slot >= K) {
            c.slot -= K;
            c.use++;
        }
    }
    __device__ __forceinline__ float2* slot_ptr(const RingCursor& c) const {
        return slots + (size_t)c.slot * slot_f2;
    }

    // One thread: copy bytes0 from src0 (and bytes1 from src1 behind it) into
    // slot j as its copy number `use`.  Sources 16-byte aligned, sizes
    // multiples of 16.
    __device__ __forceinline__ void issue(int j, int use, const void* src0, unsigned bytes0,
                                          const void* src1 = nullptr,
                                          unsigned bytes1 = 0) const {
        if (*(volatile int*)&ctl->failed) return;
        const unsigned bar = smem_addr(&ctl->bar[j]);
        float2* dst = slots + (size_t)j * slot_f2;
        // order this thread's earlier generic-proxy shared accesses before the copy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                     "r"(bytes0 + bytes1)
                     : "memory");
        asm volatile(
            "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, "
            "[%3];" ::"r"(smem_addr(dst)),
            "l"(src0), "r"(bytes0), "r"(bar)
            : "memory");
        if (bytes1)
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], "
                "%2, [%3];" ::"r"(smem_addr(reinterpret_cast<char*>(dst) + bytes0)),
                "l"(src1), "r"(bytes1), "r"(bar)
                : "memory");
        __threadfence_block();
        *(volatile int*)&ctl->issued[j] = use + 1;
    }

    // Every thread of the consuming group: true once the copy at c has landed.
    __device__ __forceinline__ bool wait(const RingCursor& c) const {
        int i = 0;
        while (*(volatile int*)&ctl->issued[c.slot] <= c.use) {
            if (++i >= kRingSpin || *(volatile int*)&ctl->failed) return false;
            __nanosleep(64);
        }
        for (i = 0; i < kRingSpin; i++)
            if (mbar_test(&ctl->bar[c.slot], (unsigned)(c.use & 1))) return true;
        return false;
    }

    __device__ __forceinline__ void fail(int* err) const {
        *(volatile int*)&ctl->failed = 1;
        if (err) atomicOr(err, 2);
    }
};

// A transform's input in two parts (the second may be empty).
struct RingSrc2 {
    const void* p0;
    const void* p1;
};

// Whole CTA: barriers, issue counters, and the first K copies (issued by
// threads 0..K-1; src(b) is transform b's input: a pointer copied as
// `bytes`, or a RingSrc2 copied as bytes then bytes1).
template <class SrcOf>
__device__ __forceinline__ Ring ring_start(RingCtl* ctl, float2* slots, int K, int slot_f2, int G,
                                           long long batch, const SrcOf& src, unsigned bytes,
                                           unsigned bytes1 = 0) {
    Ring r{ctl, slots, K, slot_f2, G};
    if (threadIdx.x < (unsigned)K) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&ctl->bar[threadIdx.x]))
                     : "memory");
        ctl->issued[threadIdx.x] = 0;
    }
    if (threadIdx.x == 0) ctl->failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    if (threadIdx.x < (unsigned)K) {
        const long long b = r.transform(threadIdx.x);
        if (b < batch) {
            const auto p = src(b);
            if constexpr (std::is_same_v<std::decay_t<decltype(p)>, RingSrc2>)
                r.issue(threadIdx.x, 0, p.p0, bytes, p.p1, bytes1);
            else
                r.issue(threadIdx.x, 0, p, bytes);
        }
    }
    return r;
}

// Whole CTA, after its last transform: no copy may still be in flight when
// the CTA exits (normally none is: every copy issued was waited for).
__device__ __forceinline__ void ring_drain(const Ring& r) {
    __syncthreads();
    if (threadIdx.x < (unsigned)r.K) {
        const int n = *(volatile int*)&r.ctl->issued[threadIdx.x];
        if (n > 0) {
            const unsigned parity = (unsigned)((n - 1) & 1);
            for (int i = 0; i < kRingSpin; i++)
                if (mbar_test(&r.ctl->bar[threadIdx.x], parity)) break;
        }
    }
}

}  // namespace fafct
