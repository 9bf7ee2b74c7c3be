// faf_exec.cpp -- faf_execute / faf_execute_batched: buffer validation (the
// reference's rules, src/faf_core.c:1298-1367, src/faf_rfft.c:268-335,
// src/faf_pipeline.c:10-60), host/device memory detection and staging, and
// dispatch to the kernels of each plan kind.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "chirp.h"
#include "faf_api_internal.h"
#include "faf_cuda.h"

using fafp::DevicePlan;
using fafp::Kind;
using namespace fafapi;

namespace {

// One plane region of a (possibly batched, strided) buffer.
struct Region {
    const void* src;   // caller pointer (input) or NULL
    void* dst;         // caller pointer (output) or NULL
    size_t floats;     // floats spanned
};

size_t span_floats(long long batch, long long dist, size_t len, int fpe) {
    if (batch <= 0) return 0;
    return ((size_t)(batch - 1) * (size_t)dist + len) * (size_t)fpe;
}

// What one execute needs from the buffers, after validation.
struct Request {
    const float* in_a = nullptr;
    const float* in_b = nullptr;
    float* out_a = nullptr;
    float* out_b = nullptr;
    size_t in_len = 0, out_len = 0;   // elements per plane per transform
    int in_fpe = 1, out_fpe = 1;      // floats per element (2 = interleaved)
    long long batch = 1, in_dist = 0, out_dist = 0;
    bool interleaved = false;         // complex side interleaved
    bool framed = false;              // STFT: framed real signal
    int scal = 1;                     // 4-byte words per scalar: 1 (FP32) or 2 (FP64)
    long long frames = 0, sig_len = 0;
};

int check_layouts_c2c(const faf_transform* t, const faf_buffer* out, const faf_buffer* in,
                      Request& r) {
    if (in->layout != t->cfg.layout || out->layout != t->cfg.layout)
        return fail("buffer layout (%s/%s) does not match transform (%s)",
                    faf_layout_name(in->layout), faf_layout_name(out->layout),
                    faf_layout_name(t->cfg.layout));
    if (!in->re || !out->re) return fail("execute buffers must provide re");
    const bool inter = t->cfg.layout == FAF_LAYOUT_INTERLEAVED;
    if (!inter && (!in->im || !out->im))
        return fail("split/hermitian layout requires im planes");
    if ((t->flags & FAF_FLAG_BLUESTEIN) && (in->n != t->n || out->n != t->n))
        return fail("bluestein: buffer length must be %zu", t->n);
    if (in->n < t->n || out->n < t->n)
        return fail("execute buffers hold %zu/%zu elements, transform needs %zu", in->n, out->n,
                    t->n);
    r.interleaved = inter;
    r.in_a = (const float*)in->re;
    r.in_b = inter ? nullptr : (const float*)in->im;
    r.out_a = (float*)out->re;
    r.out_b = inter ? nullptr : (float*)out->im;
    r.in_len = r.out_len = t->n;
    r.in_fpe = r.out_fpe = inter ? 2 : 1;
    return 0;
}

int check_rfft(const faf_transform* t, const faf_buffer* out, const faf_buffer* in, Request& r) {
    if (!in->re || !out->re) return fail("execute buffers must provide re");
    const bool inverse = t->type == FAF_TRANSFORM_IRFFT || t->cfg.dir == FAF_DIR_INVERSE;
    const size_t n = t->n, nb = n / 2 + 1;
    const faf_layout spec = t->cfg.layout;
    const bool inter = spec == FAF_LAYOUT_INTERLEAVED;
    if (!inverse) {
        if (in->layout != FAF_LAYOUT_REAL)
            return fail("rfft input must be REAL, got %s", faf_layout_name(in->layout));
        if (in->n != n) return fail("rfft input n=%zu, expected %zu", in->n, n);
        if (out->layout != spec)
            return fail("rfft output layout (%s) does not match transform (%s)",
                        faf_layout_name(out->layout), faf_layout_name(spec));
        if (out->n != nb) return fail("rfft output n=%zu, expected %zu bins", out->n, nb);
        if (spec == FAF_LAYOUT_HERMITIAN && !out->im)
            return fail("hermitian rfft output requires im");
        r.in_a = (const float*)in->re;
        r.out_a = (float*)out->re;
        r.out_b = inter ? nullptr : (float*)out->im;
        r.in_len = n;
        r.out_len = nb;
        r.out_fpe = inter ? 2 : 1;
    } else {
        if (in->layout != spec)
            return fail("irfft input layout (%s) does not match transform (%s)",
                        faf_layout_name(in->layout), faf_layout_name(spec));
        if (in->n != nb) return fail("irfft input n=%zu, expected %zu bins", in->n, nb);
        if (spec == FAF_LAYOUT_HERMITIAN && !in->im)
            return fail("hermitian irfft input requires im");
        if (out->layout != FAF_LAYOUT_REAL)
            return fail("irfft output must be REAL, got %s", faf_layout_name(out->layout));
        if (out->n != n) return fail("irfft output n=%zu, expected %zu", out->n, n);
        r.in_a = (const float*)in->re;
        r.in_b = inter ? nullptr : (const float*)in->im;
        r.out_a = (float*)out->re;
        r.in_len = nb;
        r.out_len = n;
        r.in_fpe = inter ? 2 : 1;
    }
    r.interleaved = inter;
    return 0;
}

int check_pipeline(const faf_transform* t, const faf_buffer* out, const faf_buffer* in,
                   Request& r) {
    const size_t n = t->n, nb = n / 2 + 1;
    if (in->layout != FAF_LAYOUT_REAL || in->n != n || !in->re)
        return fail("pipeline input must be REAL of length %zu", n);
    r.in_a = (const float*)in->re;
    r.in_len = n;
    if (t->inner_inv) {
        if (out->layout != FAF_LAYOUT_REAL || out->n != n || !out->re)
            return fail("pipeline output must be REAL of length %zu", n);
        r.out_a = (float*)out->re;
        r.out_len = n;
    } else {
        if (out->layout != FAF_LAYOUT_HERMITIAN || out->n != nb || !out->re || !out->im)
            return fail("analysis pipeline output must be HERMITIAN (%zu bins)", nb);
        r.out_a = (float*)out->re;
        r.out_b = (float*)out->im;
        r.out_len = nb;
    }
    return 0;
}

// Inverse STFT (faf_cuda_create_istft): HERMITIAN frames F x (n/2+1) in,
// REAL signal of (F - 1) hop + win samples out.
int check_istft(const faf_transform* t, const faf_buffer* out, const faf_buffer* in,
                Request& r) {
    const size_t n = t->n, nb = n / 2 + 1, win = t->win_length, hop = t->hop_length;
    if (in->layout != FAF_LAYOUT_HERMITIAN || !in->re || !in->im)
        return fail("inverse STFT input must be HERMITIAN split frames (re and im)");
    if (in->n == 0 || in->n % nb)
        return fail("inverse STFT input n=%zu is not a whole number of %zu-bin frames", in->n, nb);
    const size_t F = in->n / nb, L = (F - 1) * hop + win;
    if (out->layout != FAF_LAYOUT_REAL || !out->re)
        return fail("inverse STFT output must be REAL");
    if (out->n != L)
        return fail("inverse STFT output n=%zu, expected (%zu - 1) * %zu + %zu = %zu", out->n, F,
                    hop, win, L);
    r.framed = true;
    r.frames = (long long)F;
    r.sig_len = (long long)L;
    r.in_a = (const float*)in->re;
    r.in_b = (const float*)in->im;
    r.out_a = (float*)out->re;
    r.in_len = in->n;
    r.out_len = L;
    return 0;
}

// CWT (faf_cuda_create_cwt): REAL x[n] in, REAL W[rows x n] out, the
// reference's checks (src/faf_cwt.c:769-796).
int check_cwt(const faf_transform* t, const faf_buffer* out, const faf_buffer* in, Request& r) {
    const size_t n = t->n, rows = t->user_aux_n;
    if (!in->re || !out->re) return fail("cwt: buffers must provide re");
    if (in->layout != FAF_LAYOUT_REAL || out->layout != FAF_LAYOUT_REAL)
        return fail("cwt: layout mismatch");
    if (in->n != n) return fail("cwt: buffer n mismatch");
    if (in->re == out->re) return fail("cwt: in and out alias");
    r.in_a = (const float*)in->re;
    r.out_a = (float*)out->re;
    r.in_len = n;
    r.out_len = rows * n;
    return 0;
}

// Inverse CWT: REAL W[rows x n] in, REAL x[n] out (src/faf_cwt.c:849-877).
int check_icwt(const faf_transform* t, const faf_buffer* out, const faf_buffer* in, Request& r) {
    const size_t n = t->n, rows = t->user_aux_n;
    if (!in->re || !out->re) return fail("cwt: buffers must provide re");
    if (in->layout != FAF_LAYOUT_REAL || out->layout != FAF_LAYOUT_REAL)
        return fail("cwt: layout mismatch");
    if (out->n != n) return fail("cwt: buffer n mismatch");
    r.in_a = (const float*)in->re;
    r.out_a = (float*)out->re;
    r.in_len = rows * n;
    r.out_len = n;
    return 0;
}

int check_stft(const faf_transform* t, const faf_buffer* out, const faf_buffer* in,
               Request& r) {
    if (!in->re || !out->re) return fail("execute buffers must provide re");
    {
        DevicePlan* p = plan_of(t);
        if (p && p->kind == Kind::ISTFT) return check_istft(t, out, in, r);
    }
    const size_t n = t->n, nb = n / 2 + 1, win = t->win_length, hop = t->hop_length;
    if (in->layout == FAF_LAYOUT_REAL) {
        // Framed real STFT: F = 1 + (L - win) / hop frames of n/2+1 bins.
        if (!t->inner || !plan_of(t->inner))
            return fail("STFT framing needs an even 5-smooth FFT size, got %zu", n);
        if (in->n < win) return fail("STFT signal length %zu shorter than window %zu", in->n, win);
        const size_t F = 1 + (in->n - win) / hop;
        const bool inter = out->layout == FAF_LAYOUT_INTERLEAVED;
        if (out->layout != FAF_LAYOUT_HERMITIAN && !inter)
            return fail("STFT output must be HERMITIAN (frames x %zu bins), got %s", nb,
                        faf_layout_name(out->layout));
        if (out->n != F * nb)
            return fail("STFT output n=%zu, expected %zu frames x %zu bins = %zu", out->n, F, nb,
                        F * nb);
        if (!inter && !out->im) return fail("hermitian STFT output requires im");
        r.framed = true;
        r.frames = (long long)F;
        r.sig_len = (long long)in->n;
        r.in_a = (const float*)in->re;
        r.out_a = (float*)out->re;
        r.out_b = inter ? nullptr : (float*)out->im;
        r.in_len = in->n;
        r.out_len = F * nb;
        r.out_fpe = inter ? 2 : 1;
        r.interleaved = inter;
        return 0;
    }
    // One windowed C2C frame of n (reference semantics, window applied on
    // every complex layout).
    if (in->layout != out->layout ||
        (in->layout != FAF_LAYOUT_SPLIT && in->layout != FAF_LAYOUT_INTERLEAVED))
        return fail("STFT frame buffers must both be SPLIT or INTERLEAVED");
    faf_transform tmp = *t;
    tmp.cfg.layout = in->layout;
    tmp.flags &= ~FAF_FLAG_BLUESTEIN;
    return check_layouts_c2c(&tmp, out, in, r);
}

// ---- memory staging -------------------------------------------------------

int ensure_stage(DevicePlan* p, size_t bytes) {
    if (p->stage_bytes >= bytes) return 0;
    if (p->d_stage) cudaFree(p->d_stage);
    p->d_stage = nullptr;
    p->stage_bytes = 0;
    cudaError_t e = cudaMalloc(&p->d_stage, bytes);
    if (e != cudaSuccess) return cuda_fail(e, "staging allocation");
    p->stage_bytes = bytes;
    return 0;
}

int run_device(const faf_transform* t, DevicePlan* p, Request& r, cudaStream_t st);

// Host buffers, large batches: the batch runs in chunks through a ring of
// three device slots, host-to-device copies on one copy stream, kernels on
// the plan's stream (in order, so plan scratch is never shared), and
// device-to-host copies on a second copy stream.  Chunk i's input copy, chunk
// i-1's kernel and chunk i-2's output copy overlap, and the two PCIe
// directions run at once.  Events order each slot's reuse.
constexpr int kSlots = 3;
constexpr size_t kChunkMinBytes = 8u << 20;  // per-direction bytes below which one shot wins

int ensure_copy_streams(DevicePlan* p) {
    cudaError_t e = cudaSuccess;
    if (!p->cp_h2d) e = cudaStreamCreateWithFlags(&p->cp_h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess && !p->cp_d2h)
        e = cudaStreamCreateWithFlags(&p->cp_d2h, cudaStreamNonBlocking);
    for (int i = 0; i < kSlots && e == cudaSuccess; i++) {
        if (!p->ev_h2d[i]) e = cudaEventCreateWithFlags(&p->ev_h2d[i], cudaEventDisableTiming);
        if (e == cudaSuccess && !p->ev_kern[i])
            e = cudaEventCreateWithFlags(&p->ev_kern[i], cudaEventDisableTiming);
        if (e == cudaSuccess && !p->ev_d2h[i])
            e = cudaEventCreateWithFlags(&p->ev_d2h[i], cudaEventDisableTiming);
    }
    return e == cudaSuccess ? 0 : cuda_fail(e, "copy streams");
}

int run_host_chunked(const faf_transform* t, DevicePlan* p, Request& r, cudaStream_t st,
                     long long chunk) {
    if (ensure_copy_streams(p) != 0) return -1;
    const int nin = r.in_b ? 2 : 1, nout = r.out_b ? 2 : 1;
    // sizes and offsets below count 4-byte words (two per FP64 value)
    const size_t fin = span_floats(chunk, r.in_dist, r.in_len, r.in_fpe) * r.scal;
    const size_t fout = span_floats(chunk, r.out_dist, r.out_len, r.out_fpe) * r.scal;
    // slot layout, each plane rounded to 64 floats (256 bytes)
    auto up = [](size_t f) { return (f + 63) & ~(size_t)63; };
    const size_t slot_floats = up(fin) * nin + up(fout) * nout;
    if (ensure_stage(p, kSlots * slot_floats * sizeof(float)) != 0) return -1;
    cudaError_t e = cudaSuccess;
    // the copy streams start after work already queued on the plan's stream
    e = cudaEventRecord(p->ev_kern[0], st);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->cp_h2d, p->ev_kern[0], 0);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(p->cp_d2h, p->ev_kern[0], 0);
    int launches = 0;
    const long long nchunks = (r.batch + chunk - 1) / chunk;
    for (long long i = 0; i < nchunks && e == cudaSuccess; i++) {
        const int s = (int)(i % kSlots);
        const long long b0 = i * chunk, cb = std::min(chunk, r.batch - b0);
        float* slot = (float*)p->d_stage + (size_t)s * slot_floats;
        Request d = r;
        d.batch = cb;
        d.in_a = slot;
        d.in_b = r.in_b ? slot + up(fin) : nullptr;
        d.out_a = slot + up(fin) * nin;
        d.out_b = r.out_b ? d.out_a + up(fout) : nullptr;
        const size_t ioff = (size_t)b0 * r.in_dist * r.in_fpe * r.scal;
        const size_t ooff = (size_t)b0 * r.out_dist * r.out_fpe * r.scal;
        const size_t cin =
            span_floats(cb, r.in_dist, r.in_len, r.in_fpe) * r.scal * sizeof(float);
        const size_t cout =
            span_floats(cb, r.out_dist, r.out_len, r.out_fpe) * r.scal * sizeof(float);
        // input copy: the slot's previous kernel has read its inputs
        if (i >= kSlots) e = cudaStreamWaitEvent(p->cp_h2d, p->ev_kern[s], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync((void*)d.in_a, r.in_a + ioff, cin, cudaMemcpyHostToDevice,
                                p->cp_h2d);
        if (e == cudaSuccess && r.in_b)
            e = cudaMemcpyAsync((void*)d.in_b, r.in_b + ioff, cin, cudaMemcpyHostToDevice,
                                p->cp_h2d);
        if (e == cudaSuccess) e = cudaEventRecord(p->ev_h2d[s], p->cp_h2d);
        // kernel: inputs arrived, the slot's previous outputs have left
        if (e == cudaSuccess) e = cudaStreamWaitEvent(st, p->ev_h2d[s], 0);
        if (e == cudaSuccess && i >= kSlots) e = cudaStreamWaitEvent(st, p->ev_d2h[s], 0);
        if (e != cudaSuccess) break;
        if (run_device(t, p, d, st) != 0) return -1;
        launches += faf_cuda_last_launches();
        e = cudaEventRecord(p->ev_kern[s], st);
        // output copy
        if (e == cudaSuccess) e = cudaStreamWaitEvent(p->cp_d2h, p->ev_kern[s], 0);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(r.out_a + ooff, d.out_a, cout, cudaMemcpyDeviceToHost,
                                p->cp_d2h);
        if (e == cudaSuccess && r.out_b)
            e = cudaMemcpyAsync(r.out_b + ooff, d.out_b, cout, cudaMemcpyDeviceToHost,
                                p->cp_d2h);
        if (e == cudaSuccess) e = cudaEventRecord(p->ev_d2h[s], p->cp_d2h);
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(p->cp_d2h);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "chunked host execute");
    note_launches(launches);
    return 0;
}

int execute_request(const faf_transform* t, Request& r) {
    DevicePlan* p = plan_of(t);
    if (!p) return fail("transform has no CUDA plan");
    if (r.batch <= 0) return 0;
    // distance 0 = packed transforms
    if (r.in_dist == 0) r.in_dist = (long long)r.in_len;
    if (r.out_dist == 0) r.out_dist = (long long)r.out_len;
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != p->device) cudaSetDevice(p->device);
    const cudaStream_t st = p->stream;
    const void* ptrs[4] = {r.in_a, r.in_b, r.out_a, r.out_b};
    int ndev = 0, nptr = 0;
    for (const void* q : ptrs) {
        if (!q) continue;
        nptr++;
        ndev += ptr_is_device(q);
    }
    int rc = 0;
    if (ndev == nptr) {
        rc = run_device(t, p, r, st);
        if (rc == 0 && !p->user_stream) {
            cudaError_t e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = cuda_fail(e, "execute");
        }
    } else if (ndev == 0) {
        // Host buffers: copy in, run, copy out, synchronise.
        std::lock_guard<std::mutex> lock(p->mu);
        // 4-byte words (two per FP64 value)
        const size_t fin = span_floats(r.batch, r.in_dist, r.in_len, r.in_fpe) * r.scal;
        const size_t fout = span_floats(r.batch, r.out_dist, r.out_len, r.out_fpe) * r.scal;
        const int nin = r.in_b ? 2 : 1, nout = r.out_b ? 2 : 1;
        const size_t total = (fin * nin + fout * nout) * sizeof(float) + 256;
        const size_t per_dir = std::max(fin * nin, fout * nout) * sizeof(float);
        if (per_dir >= 2 * kChunkMinBytes && r.batch >= 8) {
            // about 16 chunks, none below kChunkMinBytes per direction
            long long chunk = (r.batch + 15) / 16;
            const size_t per_t = std::max(per_dir / (size_t)r.batch, (size_t)1);
            chunk = std::max<long long>(chunk, (long long)(kChunkMinBytes / per_t));
            chunk = std::min<long long>(chunk, r.batch);
            rc = run_host_chunked(t, p, r, st, chunk);
            goto done;
        }
        if ((rc = ensure_stage(p, total)) != 0) goto done;
        {
            float* base = (float*)p->d_stage;
            Request d = r;
            float* slots[4] = {base, base + fin, base + fin * nin, base + fin * nin + fout};
            cudaError_t e = cudaSuccess;
            d.in_a = slots[0];
            e = cudaMemcpyAsync(slots[0], r.in_a, fin * sizeof(float), cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess && r.in_b) {
                d.in_b = slots[1];
                e = cudaMemcpyAsync(slots[1], r.in_b, fin * sizeof(float),
                                    cudaMemcpyHostToDevice, st);
            }
            d.out_a = slots[2];
            d.out_b = r.out_b ? slots[3] : nullptr;
            if (e != cudaSuccess) { rc = cuda_fail(e, "host-to-device copy"); goto done; }
            if ((rc = run_device(t, p, d, st)) != 0) goto done;
            e = cudaMemcpyAsync(r.out_a, d.out_a, fout * sizeof(float), cudaMemcpyDeviceToHost,
                                st);
            if (e == cudaSuccess && r.out_b)
                e = cudaMemcpyAsync(r.out_b, d.out_b, fout * sizeof(float),
                                    cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) rc = cuda_fail(e, "device-to-host copy");
        }
    } else {
        rc = fail("execute buffers mix host and device memory");
    }
done:
    if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
    return rc;
}

// Pipeline with ops that must run on the host: R2C kernel -> host ops ->
// C2R kernel, through a device spectrum buffer.
int pipeline_host_ops(const faf_transform* t, DevicePlan* p, Request& r, cudaStream_t st) {
    const size_t n = t->n, nb = n / 2 + 1;
    const size_t spec_floats = 2 * nb * (size_t)r.batch;
    float* d_spec = nullptr;
    cudaError_t e = cudaMalloc(&d_spec, spec_floats * sizeof(float));
    if (e != cudaSuccess) return cuda_fail(e, "pipeline spectrum allocation");
    std::vector<float> h(spec_floats);
    DevicePlan* fwd = plan_of(t->inner);
    int rc = 0;
    e = fafp::exec_r2c(fwd, r.in_a, d_spec, d_spec + nb * r.batch, r.batch,
                       r.in_dist ? r.in_dist : (long long)n, (long long)nb, false, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(h.data(), d_spec, spec_floats * sizeof(float), cudaMemcpyDeviceToHost,
                            st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) {
        for (long long b = 0; b < r.batch; b++)
            apply_ops_host(t, h.data() + b * nb, h.data() + nb * r.batch + b * nb, nb);
        if (!t->inner_inv) {
            // analysis pipeline: the spectrum is the output
            const long long od = r.out_dist ? r.out_dist : (long long)nb;
            for (long long b = 0; b < r.batch && e == cudaSuccess; b++) {
                e = cudaMemcpyAsync(r.out_a + b * od, h.data() + b * nb, nb * sizeof(float),
                                    cudaMemcpyHostToDevice, st);
                if (e == cudaSuccess)
                    e = cudaMemcpyAsync(r.out_b + b * od, h.data() + nb * r.batch + b * nb,
                                        nb * sizeof(float), cudaMemcpyHostToDevice, st);
            }
        } else {
            e = cudaMemcpyAsync(d_spec, h.data(), spec_floats * sizeof(float),
                                cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess)
                e = fafp::exec_c2r(plan_of(t->inner_inv), d_spec, d_spec + nb * r.batch, r.out_a,
                                   r.batch, (long long)nb, r.out_dist ? r.out_dist : (long long)n,
                                   false, st);
        }
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    if (e != cudaSuccess) rc = cuda_fail(e, "pipeline (host ops)");
    cudaFree(d_spec);
    note_launches(2);
    return rc;
}

int run_device(const faf_transform* t, DevicePlan* p, Request& r, cudaStream_t st) {
    cudaError_t e = cudaSuccess;
    const long long in_dist = r.in_dist ? r.in_dist : (long long)r.in_len;
    const long long out_dist = r.out_dist ? r.out_dist : (long long)r.out_len;
    int launches = 1;
    if (p->fp64) {
        switch (t->type) {
        case FAF_TRANSFORM_FFT:
        case FAF_TRANSFORM_IFFT:
            e = fafp::exec_c2c64(p, (const double*)r.in_a, (const double*)r.in_b,
                                 (double*)r.out_a, (double*)r.out_b, r.batch, in_dist, out_dist,
                                 r.interleaved, st);
            break;
        case FAF_TRANSFORM_RFFT:
            if (r.interleaved) return fail("FP64 R2C output must be HERMITIAN split planes");
            e = fafp::exec_r2c64(p, (const double*)r.in_a, (double*)r.out_a, (double*)r.out_b,
                                 r.batch, in_dist, out_dist, st);
            break;
        case FAF_TRANSFORM_IRFFT:
            if (r.interleaved) return fail("FP64 C2R input must be HERMITIAN split planes");
            e = fafp::exec_c2r64(p, (const double*)r.in_a, (const double*)r.in_b,
                                 (double*)r.out_a, r.batch, in_dist, out_dist, st);
            break;
        default:
            return fail("FP64 is available for C2C, R2C and C2R transforms");
        }
        if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
        note_launches(1);
        return 0;
    }
    switch (t->type) {
    case FAF_TRANSFORM_FFT:
    case FAF_TRANSFORM_IFFT:
        e = fafp::exec_c2c(p, r.in_a, r.in_b, r.out_a, r.out_b, r.batch, in_dist, out_dist,
                           r.interleaved, nullptr, st);
        launches = fafp::c2c_launches(p, r.batch);
        break;
    case FAF_TRANSFORM_RFFT:
        e = fafp::exec_r2c(p, r.in_a, r.out_a, r.out_b, r.batch, in_dist, out_dist,
                           r.interleaved, st);
        break;
    case FAF_TRANSFORM_IRFFT:
        e = fafp::exec_c2r(p, r.in_a, r.in_b, r.out_a, r.batch, in_dist, out_dist, r.interleaved,
                           st);
        break;
    case FAF_TRANSFORM_PIPELINE: {
        fafk::PipeOp ops[fafk::kMaxOps];
        bool host_ops = false;
        const int nops = resolve_pipeline_ops(t, ops, fafk::kMaxOps, &host_ops, st);
        if (nops < 0) return -1;
        if (host_ops || !t->inner_inv) return pipeline_host_ops(t, p, r, st);
        e = fafp::exec_pipeline(p, r.in_a, r.out_a, r.batch, in_dist, out_dist, ops, nops, st);
        break;
    }
    case FAF_TRANSFORM_STFT:
        if (p->kind == Kind::ISTFT) {
            if (r.batch > 1 && r.in_dist != (long long)r.in_len)
                return fail("batched inverse STFT frames must be packed");
            if (r.batch > 1 && r.out_dist != (long long)r.out_len)
                return fail("batched inverse STFT output must be packed");
            e = fafp::exec_istft(p, r.in_a, r.in_b, r.out_a, r.batch, r.frames, r.sig_len, st);
            launches = 2;
        } else if (r.framed) {
            DevicePlan* fp = plan_of(t->inner);
            const long long sig_dist = r.in_dist ? r.in_dist : r.sig_len;
            if (r.batch > 1 && sig_dist != r.sig_len)
                return fail("batched STFT signals must be packed (in_dist = signal length)");
            if (r.batch > 1 && r.out_dist && r.out_dist != (long long)r.out_len)
                return fail("batched STFT output must be packed");
            e = fafp::exec_stft(fp, r.in_a, r.out_a, r.out_b, r.batch, r.sig_len, r.frames,
                                r.interleaved, st);
        } else {
            DevicePlan* fp = plan_of(t->inner);
            e = fafp::exec_c2c(p, r.in_a, r.in_b, r.out_a, r.out_b, r.batch, in_dist, out_dist,
                               r.interleaved, fp ? fp->d_window : nullptr, st);
            if (!fp) return fail("STFT frame window is unavailable for this size");
        }
        break;
    case FAF_TRANSFORM_CWT: {
        e = fafp::exec_cwt(p, r.in_a, r.out_a, r.batch, in_dist, out_dist, st);
        const long long xd = ((long long)t->n / 2 + 2) & ~1LL;  // exec_cwt's spectrum stride
        const long long cap = std::max(1LL, std::min(r.batch, (32LL << 20) / (xd * 8)));
        launches = (int)(2 * ((r.batch + cap - 1) / cap));
        break;
    }
    case FAF_TRANSFORM_ICWT: {
        if (r.batch > 1 && in_dist != (long long)r.in_len)
            return fail("batched inverse CWT coefficients must be packed (rows x n per signal)");
        e = fafp::exec_icwt(p, r.in_a, r.out_a, r.batch, in_dist, out_dist, st);
        if (p->kind == Kind::ICWT_L1) {
            launches = 1;
        } else {
            const long long yd = p->psi_dist;
            const long long cap =
                std::max(1LL, std::min(r.batch, (64LL << 20) / ((long long)p->rows * yd * 8)));
            launches = (int)(3 * ((r.batch + cap - 1) / cap));
        }
        break;
    }
    default:
        return fail("transform type '%s' is not on the CUDA path", faf_transform_name(t->type));
    }
    if (e != cudaSuccess) return cuda_fail(e, "kernel launch");
    note_launches(launches);
    return 0;
}

int build_request_typed(const faf_transform* t, faf_buffer* out, const faf_buffer* in,
                        Request& r);

int build_request(const faf_transform* t, faf_buffer* out, const faf_buffer* in, Request& r) {
    r.scal = t->cfg.precision == FAF_PREC_FP64 ? 2 : 1;
    return build_request_typed(t, out, in, r);
}

int build_request_typed(const faf_transform* t, faf_buffer* out, const faf_buffer* in,
                        Request& r) {
    switch (t->type) {
    case FAF_TRANSFORM_PIPELINE: return check_pipeline(t, out, in, r);
    case FAF_TRANSFORM_RFFT:
    case FAF_TRANSFORM_IRFFT: return check_rfft(t, out, in, r);
    case FAF_TRANSFORM_STFT: return check_stft(t, out, in, r);
    case FAF_TRANSFORM_CWT: return check_cwt(t, out, in, r);
    case FAF_TRANSFORM_ICWT: return check_icwt(t, out, in, r);
    case FAF_TRANSFORM_FFT:
    case FAF_TRANSFORM_IFFT: return check_layouts_c2c(t, out, in, r);
    default: return fail("transform type '%s' is not on the CUDA path", faf_transform_name(t->type));
    }
}

}  // namespace

extern "C" int faf_execute(const faf_transform* t, faf_buffer* out, const faf_buffer* in) {
    if (!t || !out || !in) return -1;
    Request r;
    if (build_request(t, out, in, r) != 0) return -1;
    return execute_request(t, r);
}

extern "C" int faf_execute_batched(const faf_transform* t, faf_buffer* out, const faf_buffer* in,
                                   size_t batch, size_t in_dist, size_t out_dist) {
    if (!t || !out || !in) return fail("faf_execute_batched: NULL argument");
    Request r;
    if (build_request(t, out, in, r) != 0) return -1;
    r.batch = (long long)batch;
    r.in_dist = (long long)in_dist;
    r.out_dist = (long long)out_dist;
    if (in_dist && in_dist < r.in_len) return fail("in_dist %zu < transform input length %zu", in_dist, r.in_len);
    if (out_dist && out_dist < r.out_len) return fail("out_dist %zu < transform output length %zu", out_dist, r.out_len);
    return execute_request(t, r);
}

namespace fafapi {

int exec_split_one(const faf_transform* t, void* out_re, void* out_im, const void* in_re,
                   const void* in_im) {
    if (!t) return -1;
    faf_buffer in = faf_buffer_split((void*)in_re, (void*)in_im, t->n);
    faf_buffer out = faf_buffer_split(out_re, out_im, t->n);
    Request r;
    faf_transform tmp = *t;
    tmp.cfg.layout = FAF_LAYOUT_SPLIT;
    if (check_layouts_c2c(&tmp, &out, &in, r) != 0) return -1;
    return execute_request(t, r);
}

}  // namespace fafapi

// ---- streams --------------------------------------------------------------

extern "C" int faf_cuda_set_stream(faf_transform* t, void* stream) {
    DevicePlan* p = plan_of(t);
    if (!p) return fail("faf_cuda_set_stream: transform has no CUDA plan");
    p->stream = (cudaStream_t)stream;
    p->user_stream = stream != nullptr;
    // nested plans follow the outer transform
    if (t->inner) faf_cuda_set_stream(t->inner, stream);
    if (t->inner_inv) faf_cuda_set_stream(t->inner_inv, stream);
    return 0;
}

extern "C" void* faf_cuda_get_stream(const faf_transform* t) {
    DevicePlan* p = plan_of(t);
    return p ? (void*)p->stream : nullptr;
}

extern "C" int faf_cuda_synchronize(const faf_transform* t) {
    DevicePlan* p = plan_of(t);
    if (!p) return fail("faf_cuda_synchronize: transform has no CUDA plan");
    cudaError_t e = cudaStreamSynchronize(p->stream);
    return e == cudaSuccess ? 0 : cuda_fail(e, "synchronize");
}

extern "C" int faf_cuda_available(void) {
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        fail("no CUDA device: %s", e == cudaSuccess ? "count is 0" : cudaGetErrorString(e));
        return 0;
    }
    return 1;
}

extern "C" int faf_cuda_tc_status(const faf_transform* t) {
    DevicePlan* p = plan_of(t);
    if (!p || !p->tc) return -1;
    int v = 0;
    cudaError_t e = cudaStreamSynchronize(p->stream);
    if (e == cudaSuccess) e = cudaMemcpy(&v, p->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "faf_cuda_tc_status");
    return v ? 1 : 0;
}

extern "C" int faf_cuda_wait_status(const faf_transform* t) {
    DevicePlan* p = plan_of(t);
    if (!p) return fail("faf_cuda_wait_status: transform has no CUDA plan");
    int v = 0, w = 0;
    cudaError_t e = cudaStreamSynchronize(p->stream);
    if (e == cudaSuccess && p->d_wait_err)
        e = cudaMemcpy(&v, p->d_wait_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && p->d_tc_err)
        e = cudaMemcpy(&w, p->d_tc_err, sizeof(int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_fail(e, "faf_cuda_wait_status");
    // nested plans (four-step factors, inner transforms) report through theirs
    int rc = (v || w) ? 1 : 0;
    if (!rc && t->inner && plan_of(t->inner)) rc = faf_cuda_wait_status(t->inner) == 1;
    if (!rc && t->inner_inv && plan_of(t->inner_inv)) rc = faf_cuda_wait_status(t->inner_inv) == 1;
    return rc;
}

extern "C" const char* faf_cuda_plan_kind(const faf_transform* t) {
    DevicePlan* p = plan_of(t);
    if (!p) return nullptr;
    switch (p->kind) {
    case Kind::C2C: return p->tc ? (p->d_tc64 ? "c2c-tc64" : "c2c-tc") : "c2c";
    case Kind::C2C_LARGE: return "c2c-4step";
    case Kind::RADER: return "rader";
    case Kind::BLUESTEIN: return "bluestein";
    case Kind::R2C: return "r2c";
    case Kind::C2R: return "c2r";
    case Kind::PIPELINE: return "pipeline";
    case Kind::STFT: return "stft";
    case Kind::ISTFT: return "istft";
    case Kind::CWT: return "cwt";
    case Kind::ICWT_DUAL: return "icwt-dual";
    case Kind::ICWT_L1: return "icwt-l1";
    }
    return "unknown";
}

