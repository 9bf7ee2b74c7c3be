// faf_tc.cuh -- tcgen05 building blocks shared by the tensor-core C2C kernels
// (k_tc.cu: radix-16 stages; k_tc64.cu: radix-64 stages).
//
// Operands live in shared memory, K-major without swizzle: element (row r, k)
// of a tile at byte (r % 8) * 16 + (r / 8) * SBO + (k / 8) * LBO + (k % 8) * 2,
// with SBO = 128 (the next 8-row group) and LBO the stride between 8-wide K
// chunks.  Accumulators are FP32 in TMEM.  Every mbarrier wait is bounded:
// after kSpinLimit polls it gives up and the caller records an error flag.
#pragma once

#include <cuda_fp16.h>
#include <cstdint>

namespace fafk {
namespace tcu {

constexpr int kSpinLimit = 1 << 20;

// Instruction descriptor of kind::f16: D F32 (bits 4-5 = 1), A and B F16
// (bits 7-12 = 0), both K-major (bits 15-16 = 0), N >> 3 at bit 17, M >> 4
// at bit 24.
constexpr uint32_t idesc_f16(uint32_t m, uint32_t n) {
    return (1u << 4) | ((n >> 3) << 17) | ((m >> 4) << 24);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// Shared-memory matrix descriptor: start address, leading / stride byte
// offsets (16-byte units), version 1 (bit 46), no swizzle.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void fence_before_sync() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_after_sync() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void fence_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// D (TMEM) = A B^T (+ D when acc != 0), one thread.
__device__ __forceinline__ void mma(uint32_t d, uint64_t a, uint64_t b, uint32_t idesc,
                                    uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(idesc), "r"(acc)
        : "memory");
}

// The issuing thread's MMAs so far arrive on `bar` when they complete.
__device__ __forceinline__ void commit(uint64_t* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ bool try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait; false when the limit ran out.
__device__ __forceinline__ bool wait_bounded(uint64_t* bar, uint32_t parity) {
    for (int i = 0; i < kSpinLimit; i++)
        if (try_wait(bar, parity)) return true;
    return false;
}

// 32 consecutive accumulator columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
        "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];\n"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
          "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]), "=r"(v[18]),
          "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
          "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]),
          "=r"(v[31])
        : "r"(taddr)
        : "memory");
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// hi / lo FP16 pair of (a, b) (already scaled into FP16 range)
__device__ __forceinline__ void split2(float a, float b, uint32_t& hi, uint32_t& lo) {
    const __half2 h = __floats2half2_rn(a, b);
    const float2 hf = __half22float2(h);
    const __half2 l = __floats2half2_rn(a - hf.x, b - hf.y);
    hi = *reinterpret_cast<const uint32_t*>(&h);
    lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Power-of-two scale s (and 1 / s) that puts m's binade at [2^13, 2^14), so
// that hi and lo stay normal FP16 numbers for the values near m.
__device__ __forceinline__ void pow2_scale(float m, float& s, float& inv) {
    const int e = ((__float_as_int(m) >> 23) & 0xff) - 127;
    const int sh = max(-64, min(64, 13 - e));
    s = __int_as_float((127 + sh) << 23);
    inv = __int_as_float((127 - sh) << 23);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, const uint32_t (&v)[4]) {
    asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(v[0]), "r"(v[1]),
                 "r"(v[2]), "r"(v[3])
                 : "memory");
}

}  // namespace tcu
}  // namespace fafk
