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
// (16 MiB) per GPU, reserved when the library's device code is loaded on that
// GPU and held until the process exits.  One CTA of the four-step kernel
// needs 2 * n floats (512 KiB at n = 65536), so the launch uses at most
// 16 MiB / (8 n) CTAs, each looping over the batch.  The kernel writes every
// scratch element before it reads it (pass 1 fills the whole plane pair of
// its CTA before pass 2 reads it), so nothing has to be cleared between
// calls; the array simply keeps the last call's contents.
//
// Every call shares the one array of its GPU: calls whose launches overlap on
// the GPU (different streams, or different host threads) race on it and must
// be serialised by the caller.
//
// Host code cannot hand `g_noalloc_scratch` itself to a kernel: on the host
// that name is a stand-in, not a device address.  The first call on each
// device resolves the address with cudaGetSymbolAddress (with that device
// current) and keeps it; that first call should therefore come before any
// stream capture.
#include <cuda_runtime.h>

#include <mutex>

#include "faf_api_internal.h"
#include "faf_cuda.h"

#define FAF_NOALLOC_SCRATCH_BYTES (16u << 20)
#define FAF_NOALLOC_MAX_DEVICES 64

static __device__ __align__(256) float g_noalloc_scratch[FAF_NOALLOC_SCRATCH_BYTES / sizeof(float)];

namespace {

std::mutex g_noalloc_mu;
float* g_noalloc_ptr[FAF_NOALLOC_MAX_DEVICES];  // device address per GPU, once resolved

// Device address of the scratch array on device `dev` (which is current);
// resolved on the first call for that device and kept.
int noalloc_scratch(int dev, float** out) {
    if (dev < 0 || dev >= FAF_NOALLOC_MAX_DEVICES)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: device %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_ptr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess)
            return fafapi::cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        g_noalloc_ptr[dev] = (float*)p;
    }
    *out = g_noalloc_ptr[dev];
    return 0;
}

}  // namespace

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
    const size_t cta_bytes = (size_t)(2 * n) * sizeof(float);
    if (cta_bytes > FAF_NOALLOC_SCRATCH_BYTES)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: length %lld needs %zu scratch bytes "
                            "per CTA, above the %u-byte static scratch",
                            n, cta_bytes, (unsigned)FAF_NOALLOC_SCRATCH_BYTES);
    if (!in_re || !in_im || !out_re || !out_im)
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: NULL buffer");
    if (!fafapi::ptr_is_device(in_re) || !fafapi::ptr_is_device(in_im) ||
        !fafapi::ptr_is_device(out_re) || !fafapi::ptr_is_device(out_im))
        return fafapi::fail("faf_cuda_execute_c2c_noalloc: buffers must be device memory "
                            "(host buffers would need a staging allocation)");
    if (batch == 0) return 0;

    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device) cudaSetDevice(p->device);
    float* scratch = nullptr;
    int rc = noalloc_scratch(p->device, &scratch);
    if (rc == 0) {
        int sms = 1;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, p->device);
        long long grid = (long long)(FAF_NOALLOC_SCRATCH_BYTES / cta_bytes);
        if (grid > sms) grid = sms;
        if (grid > (long long)batch) grid = (long long)batch;
        if (grid < 1) grid = 1;

        fafk::LargeArgs a;
        a.s1 = p->f1.shape(p->n1);
        a.s1.T = p->t1;
        a.s2 = p->f2.shape(p->n2);
        a.s2.T = p->t2;
        a.n1 = p->n1;
        a.n2 = p->n2;
        a.tw1 = p->f1.d_tw;
        a.tw2 = p->f2.d_tw;
        a.twn = p->d_tw_big;
        a.scratch = scratch;
        a.cta_floats = 2 * n;

        fafk::C2CArgs c;
        c.in_re = in_re;
        c.in_im = in_im;
        c.out_re = out_re;
        c.out_im = out_im;
        c.in_dist = n;
        c.out_dist = n;
        c.batch = (long long)batch;
        c.scale = p->scale;
        c.sgn = p->inverse ? -1.0f : 1.0f;
        c.interleaved = 0;
        c.window = nullptr;

        cudaError_t e = fafk::launch_large(0, a, &c, (long long)batch, (int)grid, p->stream);
        if (e == cudaSuccess && !p->user_stream) e = cudaStreamSynchronize(p->stream);
        if (e != cudaSuccess) rc = fafapi::cuda_fail(e, "faf_cuda_execute_c2c_noalloc");
    }
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    return rc;
}
