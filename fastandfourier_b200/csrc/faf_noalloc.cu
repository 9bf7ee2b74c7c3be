// faf_noalloc.cu -- faf_cuda_execute_c2c_noalloc: the four-step C2C (transform
// lengths above one CTA, 16385..65536) without any memory allocation.
//
// Who needs it: callers that must not allocate device memory while they run
// -- a real-time path such as an audio or radar callback, which cannot
// afford an unbounded wait inside the driver's allocator, and programs whose
// device memory is already fully reserved by another allocator (for example a
// framework's caching allocator), where a cudaMalloc would fail.  The regular
// entry point allocates its per-CTA four-step scratch on the first call of a
// plan; this one uses a fixed array instead.
//
// The scratch is the file-scope array below: FAF_NOALLOC_SCRATCH_BYTES
// (16 MiB) per GPU, held until the process exits.  With CUDA's default lazy
// module loading the driver places it on a GPU when its module is first
// used there; creating a four-step C2C plan does that (noalloc_prepare,
// which also loads the kernels' modules), so the entry point's own calls
// find everything in place and allocate nothing.  With eager loading it is
// placed when the library loads.
//
// Power-of-two lengths (32768, 65536) run the two-pass multi-CTA four-step
// in chunks of 16 MiB / (8 n) transforms (64 at 32768, 32 at 65536), the same
// kernels as the regular path with the array as their chunk scratch; other
// lengths run one transform per CTA with 2 n floats of the array per CTA, at
// most 16 MiB / (8 n) CTAs looping over the batch.  Each pass writes every
// scratch element before it reads it, so nothing has to be cleared between
// calls; the array simply keeps the last call's contents.
//
// Every call shares the one array of its GPU: calls whose launches overlap on
// the GPU (different streams, or different host threads) race on it and must
// be serialised by the caller.
//
// Host code cannot hand `g_noalloc_scratch` itself to a kernel: on the host
// that name is a stand-in, not a device address.  The set-up looks up the
// address with cudaGetSymbolAddress (with the plan's device current) and
// keeps it per device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "faf_api_internal.h"
#include "faf_cuda.h"

#define FAF_NOALLOC_SCRATCH_BYTES (16u << 20)
#define FAF_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) float g_noalloc_scratch[FAF_NOALLOC_SCRATCH_BYTES / sizeof(float)];

namespace {

std::mutex g_noalloc_mu;
float* g_noalloc_ptr[FAF_NOALLOC_MAX_DEVICES];  // device address per GPU, once resolved

float* noalloc_scratch(int dev) {
    if (dev < 0 || dev >= FAF_NOALLOC_MAX_DEVICES) return nullptr;
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    return g_noalloc_ptr[dev];
}

long long noalloc_cta_bytes(const fafp::DevicePlan* p) {
    return 2LL * p->n1 * p->n2 * (long long)sizeof(float);
}

}  // namespace

namespace fafp {

bool noalloc_prepare(const DevicePlan* p, std::string& err) {
    const int dev = p->device;
    if (dev < 0 || dev >= FAF_NOALLOC_MAX_DEVICES) {
        err = "device index out of range";
        return false;
    }
    if (noalloc_cta_bytes(p) > (long long)FAF_NOALLOC_SCRATCH_BYTES) {
        err = "length above the static scratch";
        return false;
    }
    cudaError_t e = large_pot2_plan(p) ? fafk::large_pot2_prepare(p->n1, p->n2)
                                       : fafk::large_c2c_prepare(large_args(p));
    if (e != cudaSuccess) {
        err = cudaGetErrorString(e);
        return false;
    }
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) {
            err = std::string("cudaGetSymbolAddress(no-alloc scratch): ") + cudaGetErrorString(e);
            return false;
        }
        g_noalloc_ptr[dev] = (float*)ptr;
    }
    return true;
}

}  // namespace fafp

extern "C" int faf_cuda_execute_c2c_noalloc(const faf_transform* t, float* out_re,
                                            float* out_im, const float* in_re,
                                            const float* in_im, size_t batch) {
    using fafp::DevicePlan;
    DevicePlan* p = fafapi::plan_of(t);
    if (!p) return fafapi::fail("faf_cuda_execute_c2c_noalloc: transform has no CUDA plan");
    if (p->kind != fafp::Kind::C2C_LARGE)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: only C2C transforms longer than %d "
                            "points (the four-step path) are supported; n = %zu",
                            fafp::kMaxSingleCta, t->n);
    const long long n = (long long)p->n1 * p->n2;
    const size_t cta_bytes = (size_t)noalloc_cta_bytes(p);
    if (cta_bytes > FAF_NOALLOC_SCRATCH_BYTES)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: length %lld needs %zu scratch bytes "
                            "per transform, above the %u-byte static scratch",
                            n, cta_bytes, (unsigned)FAF_NOALLOC_SCRATCH_BYTES);
    if (!in_re || !in_im || !out_re || !out_im)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: NULL buffer");
    if (!fafapi::ptr_is_device(in_re) || !fafapi::ptr_is_device(in_im) ||
        !fafapi::ptr_is_device(out_re) || !fafapi::ptr_is_device(out_im))
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: buffers must be device memory "
                            "(host buffers would need a staging allocation)");
    float* scratch = noalloc_scratch(p->device);
    if (!scratch)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: the static scratch was not set up "
                            "on device %d when the plan was created", p->device);
    if (batch == 0) return 0;

    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device) cudaSetDevice(p->device);
    int rc = 0;
    const long long per_array = (long long)(FAF_NOALLOC_SCRATCH_BYTES / cta_bytes);
    const float sgn = p->inverse ? -1.0f : 1.0f;
    cudaError_t e;
    if (fafp::large_pot2_plan(p)) {
        fafk::Large2Args a;
        memset(&a, 0, sizeof a);
        a.in_re = in_re; a.in_im = in_im; a.out_re = out_re; a.out_im = out_im;
        a.in_dist = n; a.out_dist = n; a.offs = nullptr; a.batch = (long long)batch;
        a.scale = p->scale; a.sgn = sgn;
        a.tws1 = p->f1.d_tws; a.tws2 = p->f2.d_tws; a.twm = p->d_tw_big;
        a.scratch = scratch;
        a.scratch_transforms = per_array;
        e = fafk::launch_large_pot2(p->n1, p->n2, a, p->stream);
    } else {
        long long grid = std::min<long long>(per_array, fafk::sm_count());
        grid = std::max(1LL, std::min(grid, (long long)batch));
        fafk::LargeArgs a = fafp::large_args(p);
        a.scratch = scratch;
        a.cta_floats = 2 * n;
        fafk::C2CArgs c;
        memset(&c, 0, sizeof c);
        c.in_re = in_re; c.in_im = in_im; c.out_re = out_re; c.out_im = out_im;
        c.in_dist = n; c.out_dist = n; c.batch = (long long)batch;
        c.scale = p->scale; c.sgn = sgn;
        c.interleaved = 0;
        c.window = nullptr;
        e = fafk::launch_large(0, a, &c, (long long)batch, (int)grid, p->stream);
    }
    if (e == cudaSuccess && !p->user_stream) e = cudaStreamSynchronize(p->stream);
    if (e != cudaSuccess) rc = fafapi::cuda_fail(e, "faf_cuda_execute_c2c_noalloc");
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    return rc;
}
