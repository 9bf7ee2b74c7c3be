// faf_serve.cpp -- the serving loop of include/faf_serve.h: continuous
// batching of real-transform / pipeline / STFT requests on one GPU.
//
// Threads:
//   - callers submit from any thread (faf_server_submit): validation, plan
//     metadata, byte accounting, then the request joins the scheduler's FIFO;
//   - one worker thread per stream slot admits the next batch (faf_sched.h
//     policy), stages its inputs into the device arena, launches one batched
//     execute on the batch's slot stream, copies the outputs back and enqueues
//     a host callback; the host-side launch cost of concurrent batches is
//     spread over the workers;
//   - the host callback (a CUDA driver thread; it makes no CUDA call) stamps
//     the completion time, releases the batch's memory and slot, and wakes
//     the workers and the waiters.
// Locking rule: the host callback takes `mu`, and a CUDA call may wait for
// host callbacks (cudaFree synchronises the device), so no thread makes a
// CUDA call while it holds `mu`.  Plans are created under `plans_mu` only.
// All CUDA work of a batch is enqueued on its slot's stream, so batches on
// different slots overlap on the device.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "chirp.h"
#include "faf_api_internal.h"
#include "faf_cuda.h"
#include "faf_sched.h"
#include "faf_serve.h"

namespace {

using Clock = std::chrono::steady_clock;
using fafapi::fail;

enum class RKind { RFFT, PIPELINE, STFT };

struct PlanMeta {
    RKind kind;
    size_t n;  // FFT size
};

struct Req {
    long long id = 0;
    faf_request r;
    std::string plan_key;
    RKind kind = RKind::RFFT;
    size_t n = 0, nb = 0;     // FFT size, bins
    size_t units = 0;         // transforms (rfft / pipeline)
    size_t frames = 0;        // STFT frames of this request
    size_t carry = 0;         // streamed STFT: overlap samples prepended
    size_t carry_off = 0;     // streamed STFT: arena offset of the overlap buffer
    size_t bytes = 0;         // arena bytes while in flight
    size_t algo_bytes = 0;    // input + output bytes
    Clock::time_point t_submit, t_done;
    int status = 0;           // 0 pending / running, 1 done, -1 failed
    std::string err;
};

struct StreamState {
    size_t n, win, hop;
    size_t total_in = 0, total_frames = 0;
    size_t carry_off = 0;  // arena block of `win` floats
    int live = 0;          // submitted, not yet completed chunks
};

struct Slot {
    cudaStream_t st = nullptr;
    std::map<std::string, faf_transform*> plans;
};

struct BatchRun;

}  // namespace

struct faf_server {
    int device = 0;
    float* arena = nullptr;
    size_t arena_bytes = 0;
    std::vector<Slot> slots;
    std::unique_ptr<fafs::Scheduler> sched;
    std::mutex mu;        // queue, requests, streams, stats (no CUDA call under it)
    std::mutex plans_mu;  // slots[*].plans, probe plans
    std::vector<faf_transform*> probes;  // plans made to read a key's metadata
    std::condition_variable cv_disp, cv_done;
    bool stop = false;
    int inflight = 0;
    long long next_id = 1;
    std::unordered_map<long long, std::unique_ptr<Req>> reqs;
    std::map<std::string, PlanMeta> meta;
    std::map<unsigned long long, StreamState> streams;
    // stats since the last reset
    std::vector<double> lat;
    long long failed = 0;
    double bytes_done = 0;
    bool have_first = false;
    Clock::time_point first_submit, last_done;
    std::vector<std::thread> workers;
};

namespace {

struct BatchRun {
    faf_server* s;
    fafs::Batch b;
    std::vector<Req*> reqs;
};

std::string stft_key(size_t n, size_t win, size_t hop) {
    return "stft:" + std::to_string(n) + ":" + std::to_string(win) + ":" + std::to_string(hop);
}

std::string plan_key_of(const faf_request* r) {
    if (!r->chirp) return stft_key(r->stft_n, r->stft_win, r->stft_hop);
    char h[64];
    snprintf(h, sizeof h, "|H=%p:%p:%zu", (const void*)r->h_re, (const void*)r->h_im, r->h_len);
    return std::string(r->chirp) + h;
}

uint64_t hash_key(const std::string& k) {  // FNV-1a
    uint64_t h = 1469598103934665603ull;
    for (unsigned char c : k) {
        h ^= c;
        h *= 1099511628211ull;
    }
    return h ? h : 1;
}

// Create the plan of request `r` (device memory and twiddles), bound to stream st.
faf_transform* create_plan(const faf_request* r, cudaStream_t st) {
    faf_transform* t = nullptr;
    if (r->chirp) {
        t = chirp_compile(r->chirp);
        if (t && r->h_re &&
            chirp_bind(t, "H", (void*)r->h_re, (void*)r->h_im, r->h_len) != 0) {
            faf_destroy_transform(t);
            return nullptr;
        }
    } else {
        faf_config c = faf_config_init(r->stft_n);
        c.win_length = r->stft_win;
        c.hop_length = r->stft_hop;
        t = faf_create_stft(&c);
    }
    if (t && st && faf_cuda_set_stream(t, st) != 0) {
        faf_destroy_transform(t);
        return nullptr;
    }
    return t;
}

faf_transform* slot_plan(faf_server* s, Slot& sl, Req* q) {
    std::lock_guard<std::mutex> lk(s->plans_mu);
    auto it = sl.plans.find(q->plan_key);
    if (it != sl.plans.end()) return it->second;
    faf_transform* t = create_plan(&q->r, sl.st);
    if (t) sl.plans[q->plan_key] = t;
    return t;
}

size_t align_floats(size_t nfl) { return (nfl * sizeof(float) + 255) / 256 * 256 / sizeof(float); }

void finish_request(faf_server* s, Req* q, bool ok, const std::string& err);

// Completion of a batch (CUDA host callback: no CUDA call in here).
void CUDART_CB on_batch_done(void* p) {
    BatchRun* br = (BatchRun*)p;
    faf_server* s = br->s;
    const Clock::time_point now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->sched->complete(br->b);
        for (Req* q : br->reqs) {
            q->t_done = now;
            finish_request(s, q, true, "");
        }
        s->inflight--;
    }
    delete br;
    s->cv_disp.notify_all();
    s->cv_done.notify_all();
}

// Enqueue one batch on its slot's stream.  Returns 0, or -1 with *err set
// (nothing of the batch is left running in that case only if no CUDA call
// was issued; the caller then fails every request of the batch).
int launch_batch(faf_server* s, BatchRun* br, std::string* err) {
    Slot& sl = s->slots[br->b.slot];
    cudaStream_t st = sl.st;
    Req* q0 = br->reqs[0];
    faf_transform* t = slot_plan(s, sl, q0);
    if (!t) {
        *err = std::string("plan creation failed: ") + std::string(faf_get_error());
        return -1;
    }
    float* base = s->arena + br->b.offset / sizeof(float);
    const size_t n = q0->n, nb = q0->nb;
    cudaError_t e = cudaSuccess;
    auto copy = [&](void* dst, const void* src, size_t bytes) {
        if (e == cudaSuccess && bytes)
            e = cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDefault, st);
    };
    int rc = 0;
    if (q0->kind == RKind::RFFT || q0->kind == RKind::PIPELINE) {
        size_t units = 0;
        for (Req* q : br->reqs) units += q->units;
        float* in = base;
        float* out_a = base + align_floats(units * n);
        float* out_b = out_a + units * nb;
        size_t u = 0;
        for (Req* q : br->reqs) {
            copy(in + u * n, q->r.in, q->units * n * sizeof(float));
            u += q->units;
        }
        if (e != cudaSuccess) goto cuda_err;
        faf_buffer bi = faf_buffer_real(in, n);
        if (q0->kind == RKind::RFFT) {
            faf_buffer bo = faf_buffer_hermitian(out_a, out_b, nb);
            rc = faf_execute_batched(t, &bo, &bi, units, n, nb);
        } else {
            faf_buffer bo = faf_buffer_real(out_a, n);
            rc = faf_execute_batched(t, &bo, &bi, units, n, n);
        }
        if (rc != 0) {
            *err = faf_get_error();
            return -1;
        }
        u = 0;
        for (Req* q : br->reqs) {
            if (q0->kind == RKind::RFFT) {
                copy(q->r.out_re, out_a + u * nb, q->units * nb * sizeof(float));
                copy(q->r.out_im, out_b + u * nb, q->units * nb * sizeof(float));
            } else {
                copy(q->r.out_re, out_a + u * n, q->units * n * sizeof(float));
            }
            u += q->units;
        }
    } else if (q0->r.stream_key) {
        // one chunk of a stream: [overlap | chunk] -> frames; new overlap saved
        Req* q = q0;
        const size_t L = q->carry + q->r.in_len;
        const size_t hop = q->r.stft_hop;
        float* in = base;
        float* out_a = base + align_floats(L);
        float* out_b = out_a + q->frames * nb;
        float* carry = s->arena + q->carry_off / sizeof(float);
        copy(in, carry, q->carry * sizeof(float));
        copy(in + q->carry, q->r.in, q->r.in_len * sizeof(float));
        if (e != cudaSuccess) goto cuda_err;
        if (q->frames) {
            faf_buffer bi = faf_buffer_real(in, L);
            faf_buffer bo = faf_buffer_hermitian(out_a, out_b, q->frames * nb);
            if (faf_execute_batched(t, &bo, &bi, 1, L, q->frames * nb) != 0) {
                *err = faf_get_error();
                return -1;
            }
        }
        copy(carry, in + q->frames * hop, (L - q->frames * hop) * sizeof(float));
        copy(q->r.out_re, out_a, q->frames * nb * sizeof(float));
        copy(q->r.out_im, out_b, q->frames * nb * sizeof(float));
    } else {
        // whole signals of one length, merged: packed batch of STFTs
        const size_t L = q0->r.in_len, F = q0->frames, k = br->reqs.size();
        float* in = base;
        float* out_a = base + align_floats(k * L);
        float* out_b = out_a + k * F * nb;
        for (size_t i = 0; i < k; i++) copy(in + i * L, br->reqs[i]->r.in, L * sizeof(float));
        if (e != cudaSuccess) goto cuda_err;
        faf_buffer bi = faf_buffer_real(in, L);
        faf_buffer bo = faf_buffer_hermitian(out_a, out_b, F * nb);
        if (faf_execute_batched(t, &bo, &bi, k, L, F * nb) != 0) {
            *err = faf_get_error();
            return -1;
        }
        for (size_t i = 0; i < k; i++) {
            copy(br->reqs[i]->r.out_re, out_a + i * F * nb, F * nb * sizeof(float));
            copy(br->reqs[i]->r.out_im, out_b + i * F * nb, F * nb * sizeof(float));
        }
    }
    if (e != cudaSuccess) goto cuda_err;
    e = cudaLaunchHostFunc(st, on_batch_done, br);
    if (e != cudaSuccess) goto cuda_err;
    return 0;
cuda_err:
    *err = std::string("CUDA: ") + cudaGetErrorString(e);
    return -1;
}

void finish_request(faf_server* s, Req* q, bool ok, const std::string& err) {
    q->status = ok ? 1 : -1;
    if (!ok) {
        q->err = err;
        s->failed++;
    } else {
        s->lat.push_back(std::chrono::duration<double>(q->t_done - q->t_submit).count());
        s->bytes_done += (double)q->algo_bytes;
        if (q->t_done > s->last_done) s->last_done = q->t_done;
    }
    if (q->r.stream_key) {
        auto it = s->streams.find(q->r.stream_key);
        if (it != s->streams.end()) it->second.live--;
    }
}

// Worker of one stream slot's share of the launches: admit, launch, repeat;
// sleep when nothing can start.  Workers leave once stopped and the queue is
// empty (batches in flight complete through their callbacks).
void worker(faf_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        fafs::Batch b;
        if (s->sched->admit_one(&b)) {
            BatchRun* br = new BatchRun();
            br->s = s;
            br->b = std::move(b);
            for (const fafs::SchedReq& sr : br->b.reqs) br->reqs.push_back(s->reqs[sr.id].get());
            s->inflight++;
            lk.unlock();
            std::string err;
            const int rc = launch_batch(s, br, &err);
            if (rc != 0) {
                // nothing of this batch completes through a callback: drain
                // what was enqueued before releasing its memory
                cudaStreamSynchronize(s->slots[br->b.slot].st);
            }
            lk.lock();
            if (rc != 0) {
                s->sched->complete(br->b);
                for (Req* q : br->reqs) finish_request(s, q, false, err);
                s->inflight--;
                delete br;
                s->cv_disp.notify_all();
                s->cv_done.notify_all();
            }
            continue;
        }
        if (s->stop && s->sched->pending() == 0) break;
        s->cv_disp.wait(lk);
    }
}

}  // namespace

extern "C" faf_server* faf_server_create(const faf_server_config* cfg) {
    faf_server_config c{};
    if (cfg) c = *cfg;
    if (!c.hbm_budget) c.hbm_budget = (size_t)16 << 30;
    if (c.streams <= 0) c.streams = 8;
    if (c.max_merge <= 0) c.max_merge = 64;
    if (c.streams > 64) {
        fail("faf_server_create: at most 64 stream slots (%d requested)", c.streams);
        return nullptr;
    }
    std::unique_ptr<faf_server> s(new faf_server());
    cudaGetDevice(&s->device);
    s->arena_bytes = c.hbm_budget & ~(size_t)255;
    cudaError_t e = cudaMalloc(&s->arena, s->arena_bytes);
    if (e != cudaSuccess) {
        fafapi::cuda_fail(e, "faf_server_create: arena");
        return nullptr;
    }
    s->slots.resize(c.streams);
    for (Slot& sl : s->slots) {
        e = cudaStreamCreateWithFlags(&sl.st, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            fafapi::cuda_fail(e, "faf_server_create: stream");
            for (Slot& x : s->slots)
                if (x.st) cudaStreamDestroy(x.st);
            cudaFree(s->arena);
            return nullptr;
        }
    }
    s->sched.reset(new fafs::Scheduler(s->arena_bytes, c.streams, c.max_merge));
    faf_server* raw = s.release();
    for (int w = 0; w < c.streams; w++) raw->workers.emplace_back(worker, raw);
    return raw;
}

namespace {

// Plan metadata for a request (kind and size), creating a probe plan the
// first time a key is seen.  Called WITHOUT s->mu (plan creation makes CUDA
// calls); the probe plan is kept until the server is destroyed, so no device
// memory is freed while requests run.
int plan_meta(faf_server* s, const faf_request* r, const std::string& key, PlanMeta* out) {
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->meta.find(key);
        if (it != s->meta.end()) {
            *out = it->second;
            return 0;
        }
    }
    faf_transform* t = nullptr;
    {
        std::lock_guard<std::mutex> lk(s->plans_mu);
        t = create_plan(r, nullptr);
        if (t) s->probes.push_back(t);
    }
    if (!t) {
        const std::string why = faf_get_error();  // fail() rewrites the same buffer
        return fail("faf_server_submit: cannot plan request: %s", why.c_str());
    }
    PlanMeta m;
    m.n = t->n;
    if (t->type == FAF_TRANSFORM_RFFT && t->cfg.dir == FAF_DIR_FORWARD) m.kind = RKind::RFFT;
    else if (t->type == FAF_TRANSFORM_PIPELINE) m.kind = RKind::PIPELINE;
    else if (t->type == FAF_TRANSFORM_STFT) m.kind = RKind::STFT;
    else return fail("faf_server_submit: only forward rfft, pipeline and STFT plans are served");
    std::lock_guard<std::mutex> lk(s->mu);
    s->meta[key] = m;
    *out = m;
    return 0;
}

}  // namespace

extern "C" long long faf_server_submit(faf_server* s, const faf_request* r) {
    if (!s || !r) return fail("faf_server_submit: NULL argument");
    if (!r->in || !r->out_re) return fail("faf_server_submit: NULL input or output");
    if (!r->chirp && (!r->stft_n || !r->stft_win || !r->stft_hop))
        return fail("faf_server_submit: STFT request needs stft_n, stft_win and stft_hop");
    if (r->chirp && r->stream_key) return fail("faf_server_submit: stream_key is for STFT only");
    std::unique_ptr<Req> q(new Req());
    q->r = *r;
    q->plan_key = plan_key_of(r);
    PlanMeta m;
    if (plan_meta(s, r, q->plan_key, &m) != 0) return -1;
    std::lock_guard<std::mutex> lk(s->mu);
    q->kind = m.kind;
    q->n = m.n;
    q->nb = m.n / 2 + 1;
    const size_t n = q->n, nb = q->nb;
    size_t floats = 0;
    bool mergeable = true;
    if (m.kind == RKind::RFFT || m.kind == RKind::PIPELINE) {
        if (r->in_len == 0 || r->in_len % n)
            return fail("faf_server_submit: in_len %zu is not a whole number of %zu-point "
                        "transforms", r->in_len, n);
        q->units = r->in_len / n;
        if (m.kind == RKind::RFFT) {
            if (!r->out_im) return fail("faf_server_submit: rfft output needs out_im");
            floats = q->units * (n + 2 * nb);
            q->algo_bytes = q->units * (4 * n + 8 * nb);
        } else {
            floats = q->units * 2 * n;
            q->algo_bytes = q->units * 8 * n;
        }
    } else {
        if (!r->out_im) return fail("faf_server_submit: STFT output needs out_im");
        const size_t win = r->stft_win, hop = r->stft_hop;
        if (r->stream_key) {
            auto it = s->streams.find(r->stream_key);
            if (it == s->streams.end()) {
                StreamState ss{n, win, hop};
                const size_t off = s->sched->reserve((size_t)win * sizeof(float));
                if (off == SIZE_MAX)
                    return fail("faf_server_submit: no arena memory for the stream overlap");
                ss.carry_off = off;
                it = s->streams.emplace(r->stream_key, ss).first;
            } else if (it->second.n != n || it->second.win != win || it->second.hop != hop) {
                return fail("faf_server_submit: stream %llu was opened with another STFT "
                            "geometry", r->stream_key);
            }
            StreamState& ss = it->second;
            q->carry = ss.total_in - ss.total_frames * hop;
            const size_t L = q->carry + r->in_len;
            q->frames = L >= win ? 1 + (L - win) / hop : 0;
            q->carry_off = ss.carry_off;
            floats = align_floats(L) + 2 * q->frames * nb;
            mergeable = false;
            // committed below, after the budget check
        } else {
            if (r->in_len < win)
                return fail("faf_server_submit: STFT signal of %zu samples is shorter than the "
                            "%zu-sample window", r->in_len, win);
            q->frames = 1 + (r->in_len - win) / hop;
            floats = r->in_len + 2 * q->frames * nb;
        }
        q->algo_bytes = 4 * r->in_len + 8 * q->frames * nb;
    }
    q->bytes = floats * sizeof(float) + 512;
    if (!s->sched->fits_ever(q->bytes))
        return fail("faf_server_submit: request needs %zu arena bytes, above the %zu-byte budget",
                    q->bytes, s->arena_bytes);
    if (r->stream_key) {
        StreamState& ss = s->streams[r->stream_key];
        ss.total_in += r->in_len;
        ss.total_frames += q->frames;
        ss.live++;
    }
    q->id = s->next_id++;
    q->t_submit = Clock::now();
    if (!s->have_first) {
        s->have_first = true;
        s->first_submit = q->t_submit;
        s->last_done = q->t_submit;
    }
    fafs::SchedReq sr;
    sr.id = q->id;
    sr.plan_key = hash_key(q->plan_key + (m.kind == RKind::STFT ? ":" + std::to_string(r->in_len)
                                                                : std::string()));
    sr.stream_key = r->stream_key;
    sr.mergeable = mergeable;
    sr.bytes = q->bytes;
    const long long id = q->id;
    s->reqs[id] = std::move(q);
    s->sched->submit(sr);
    s->cv_disp.notify_one();
    return id;
}

extern "C" int faf_server_wait(faf_server* s, long long id, double* latency_s, size_t* frames) {
    if (!s) return fail("faf_server_wait: NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return fail("faf_server_wait: unknown request %lld", id);
    Req* q = it->second.get();
    s->cv_done.wait(lk, [&] { return q->status != 0; });
    if (latency_s) *latency_s = std::chrono::duration<double>(q->t_done - q->t_submit).count();
    if (frames) *frames = q->frames;
    const int ok = q->status == 1;
    const std::string err = q->err;
    s->reqs.erase(it);
    if (!ok) return fail("faf_server_wait: request %lld failed: %s", id, err.c_str());
    return 0;
}

extern "C" int faf_server_drain(faf_server* s) {
    if (!s) return fail("faf_server_drain: NULL server");
    std::unique_lock<std::mutex> lk(s->mu);
    s->cv_done.wait(lk, [&] { return s->inflight == 0 && s->sched->pending() == 0; });
    for (auto& kv : s->reqs)
        if (kv.second->status < 0) return fail("faf_server_drain: request %lld failed: %s",
                                                kv.first, kv.second->err.c_str());
    return 0;
}

extern "C" size_t faf_server_stream_frames(faf_server* s, unsigned long long key, size_t win,
                                           size_t hop, size_t in_len) {
    if (!s || !win || !hop) return 0;
    std::lock_guard<std::mutex> lk(s->mu);
    size_t carry = 0;
    auto it = s->streams.find(key);
    if (it != s->streams.end()) carry = it->second.total_in - it->second.total_frames * hop;
    const size_t L = carry + in_len;
    return L >= win ? 1 + (L - win) / hop : 0;
}

extern "C" int faf_server_close_stream(faf_server* s, unsigned long long key) {
    if (!s) return fail("faf_server_close_stream: NULL server");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->streams.find(key);
    if (it == s->streams.end()) return 0;
    if (it->second.live > 0)
        return fail("faf_server_close_stream: stream %llu has chunks in flight", key);
    s->sched->unreserve(it->second.carry_off);
    s->streams.erase(it);
    s->cv_disp.notify_all();
    return 0;
}

namespace {

// Run a fresh plan once on scratch memory (zeros), so allocations that a
// plan makes on its first execute (the four-step per-CTA scratch) happen
// here rather than while requests are served.
int warm_plan(faf_transform* t, const PlanMeta& m, const faf_request* r, cudaStream_t st) {
    const size_t n = m.n, nb = n / 2 + 1;
    size_t L = n, F = 0, floats = 0;
    if (m.kind == RKind::RFFT) floats = n + 2 * nb;
    else if (m.kind == RKind::PIPELINE) floats = 2 * n;
    else {
        L = std::max(n, r->stft_win);
        F = 1 + (L - r->stft_win) / r->stft_hop;
        floats = L + 2 * F * nb;
    }
    float* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, floats * sizeof(float));
    if (e != cudaSuccess) return fafapi::cuda_fail(e, "faf_server_prepare: warm-up buffer");
    cudaMemsetAsync(buf, 0, floats * sizeof(float), st);
    int rc;
    faf_buffer bi = faf_buffer_real(buf, L);
    if (m.kind == RKind::RFFT) {
        faf_buffer bo = faf_buffer_hermitian(buf + n, buf + n + nb, nb);
        rc = faf_execute_batched(t, &bo, &bi, 1, n, nb);
    } else if (m.kind == RKind::PIPELINE) {
        faf_buffer bo = faf_buffer_real(buf + n, n);
        rc = faf_execute_batched(t, &bo, &bi, 1, n, n);
    } else {
        faf_buffer bo = faf_buffer_hermitian(buf + L, buf + L + F * nb, F * nb);
        rc = faf_execute_batched(t, &bo, &bi, 1, L, F * nb);
    }
    e = cudaStreamSynchronize(st);
    cudaFree(buf);
    if (rc != 0) return -1;
    if (e != cudaSuccess) return fafapi::cuda_fail(e, "faf_server_prepare: warm-up");
    return 0;
}

}  // namespace

extern "C" int faf_server_prepare(faf_server* s, const faf_request* r) {
    if (!s || !r) return fail("faf_server_prepare: NULL argument");
    const std::string key = plan_key_of(r);
    PlanMeta m;
    if (plan_meta(s, r, key, &m) != 0) return -1;
    std::lock_guard<std::mutex> lk(s->plans_mu);
    for (Slot& sl : s->slots) {
        if (sl.plans.count(key)) continue;
        faf_transform* t = create_plan(r, sl.st);
        if (!t) {
            const std::string why = faf_get_error();
            return fail("faf_server_prepare: %s", why.c_str());
        }
        // warmed before any worker can see it
        if (warm_plan(t, m, r, sl.st) != 0) {
            const std::string why = faf_get_error();
            faf_destroy_transform(t);
            return fail("faf_server_prepare: %s", why.c_str());
        }
        sl.plans[key] = t;
    }
    return 0;
}

extern "C" int faf_server_stats_get(faf_server* s, faf_server_stats* st) {
    if (!s || !st) return fail("faf_server_stats_get: NULL argument");
    std::lock_guard<std::mutex> lk(s->mu);
    memset(st, 0, sizeof *st);
    std::vector<double> v = s->lat;
    st->completed = (long long)v.size();
    st->failed = s->failed;
    st->batches = s->sched->batches();
    st->merged_requests = s->sched->merged_requests();
    st->arena_bytes = s->arena_bytes;
    st->arena_peak_bytes = s->sched->arena().peak();
    if (!v.empty()) {
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const size_t i = (size_t)std::min<double>((double)v.size() - 1, p * (double)v.size());
            return v[i];
        };
        st->p50_latency_s = pct(0.50);
        st->p99_latency_s = pct(0.99);
        double sum = 0;
        for (double x : v) sum += x;
        st->mean_latency_s = sum / (double)v.size();
        st->max_latency_s = v.back();
        st->wall_s = std::chrono::duration<double>(s->last_done - s->first_submit).count();
        if (st->wall_s > 0) {
            st->requests_per_s = (double)v.size() / st->wall_s;
            st->bytes_per_s = s->bytes_done / st->wall_s;
        }
    }
    return 0;
}

extern "C" void faf_server_stats_reset(faf_server* s) {
    if (!s) return;
    std::lock_guard<std::mutex> lk(s->mu);
    s->lat.clear();
    s->failed = 0;
    s->bytes_done = 0;
    s->have_first = false;
    s->sched->reset_counters();
}

extern "C" int faf_server_replay(faf_server* s, const faf_request* reqs,
                                 const double* arrival_s, size_t n, double* latency_s) {
    if (!s || (n && (!reqs || !arrival_s))) return fail("faf_server_replay: NULL argument");
    std::vector<long long> ids(n, -1);
    const Clock::time_point t0 = Clock::now();
    int rc = 0;
    for (size_t i = 0; i < n; i++) {
        const Clock::time_point due =
            t0 + std::chrono::duration_cast<Clock::duration>(std::chrono::duration<double>(arrival_s[i]));
        for (;;) {
            const Clock::time_point now = Clock::now();
            if (now >= due) break;
            if (due - now > std::chrono::microseconds(200))
                std::this_thread::sleep_for(due - now - std::chrono::microseconds(100));
        }
        ids[i] = faf_server_submit(s, &reqs[i]);
        if (ids[i] < 0) rc = -1;
    }
    std::string first_err;
    for (size_t i = 0; i < n; i++) {
        double l = -1;
        if (ids[i] > 0 && faf_server_wait(s, ids[i], &l, nullptr) != 0) {
            if (first_err.empty()) first_err = faf_get_error();
            rc = -1;
        }
        if (latency_s) latency_s[i] = l;
    }
    if (rc != 0 && !first_err.empty()) fail("faf_server_replay: %s", first_err.c_str());
    return rc;
}

extern "C" void faf_server_destroy(faf_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_disp.notify_all();
    for (std::thread& w : s->workers)
        if (w.joinable()) w.join();
    {
        std::unique_lock<std::mutex> lk(s->mu);
        s->cv_done.wait(lk, [&] { return s->inflight == 0; });
    }
    for (Slot& sl : s->slots) {
        if (sl.st) cudaStreamSynchronize(sl.st);
        for (auto& kv : sl.plans) faf_destroy_transform(kv.second);
        if (sl.st) cudaStreamDestroy(sl.st);
    }
    for (faf_transform* t : s->probes) faf_destroy_transform(t);
    cudaFree(s->arena);
    delete s;
}
