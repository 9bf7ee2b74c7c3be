// faf_uneven.cu -- many C2C transforms of uneven lengths in ONE persistent
// launch (the reference has no batch API: its benchmarks loop over
// faf_execute, benchmarks/benchmark_throughput.cpp:34-39).
//
// Layout: transform i of the batch has length len[i] and starts at element
// offset sum_{j<i} len[j] of every plane (ragged, packed, split planes).
//
// Plan: transforms are grouped by length into classes, and every class goes
// to one of three persistent kernels, all launched from ONE CUDA graph:
//   - k_uneven_generic (1024 threads): the runtime-radix engine for every
//     5-smooth / codelet length up to 16384, G transforms per task, all such
//     classes in one launch;
//   - k_uneven_rader (512 threads): prime lengths with 7-smooth n-1;
//   - k_uneven_large (512 threads, one launch per length above 16384): the
//     four-step path, one transform per CTA through per-CTA scratch.
// The kinds are separate kernels because their register footprints differ:
// one kernel holding all three paths spills 10-29 KB per thread at either
// 512 or 1024 threads, while each path alone fits.  In the graph the
// four-step launches run on one branch and the generic + Rader launches on a
// second branch, so the small classes fill the SMs that the long transforms
// leave idle at their tail.  Inside a launch, tasks are ordered longest-first
// and handed out by an atomic counter, so the persistent CTAs balance the
// ragged work dynamically.  The graph is replayed while the buffer pointers
// stay the same.
//
// The autotuner (FAF_FLAG_MEASURE at create) times candidate launch shapes --
// threads per transform (1, 2 or 4 times the padded minimum, which sets the
// transforms per CTA: G = 1024 / T) and resident Rader CTAs per SM -- on the
// plan's own workload and keeps the fastest.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "faf_api_internal.h"
#include "faf_cuda.h"
#include "faf_large.cuh"

namespace fafk {

enum : int { UK_GENERIC = 0, UK_RADER = 1 };
// 1024 threads: every length up to 16384 is one CTA group (T <= 1024).
constexpr int kUnevenThreads = 1024;
constexpr int kRaderThreads = 512;

struct UnevenClass {
    int kind;
    int n;
    int G;            // transforms per task
    int extra;        // extra floats per group (Rader DC slot)
    float scale;      // norm scale for this length
    fafd::Shape s;    // generic / Rader inner shape, T padded
    const float2* tw;
    const int* rin;
    const int* rout;
    const float2* B;
    float inv_m;
};

struct UnevenTask {
    int cls;
    int first;  // index into the item list
    int count;
    int pad_;
};

struct UnevenArgs {
    const UnevenClass* classes;
    const UnevenTask* tasks;      // this kernel's tasks
    int ntasks;
    const int* items;             // transform ids grouped by task
    const long long* offsets;     // element offset of each transform
    const float* in_re;
    const float* in_im;
    float* out_re;
    float* out_im;
    float sgn;
    int* counter;                 // this kernel's task counter
};

// Next task of this CTA (uniform across the CTA), or -1 when none is left.
__device__ __forceinline__ int next_task(const UnevenArgs& a, int* s_task) {
    if (threadIdx.x == 0) *s_task = atomicAdd(a.counter, 1);
    __syncthreads();
    const int task = *s_task;
    __syncthreads();
    return task < a.ntasks ? task : -1;
}

__global__ void __launch_bounds__(kUnevenThreads) k_uneven_generic(const UnevenArgs a) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    __shared__ int s_task;
    for (int task; (task = next_task(a, &s_task)) >= 0;) {
        const UnevenTask tk = a.tasks[task];
        const UnevenClass& c = a.classes[tk.cls];
        const int T = c.s.T;
        const int g = threadIdx.x / T, t = threadIdx.x % T;
        const bool live = g < tk.count;
        const long long off = a.offsets[a.items[tk.first + (live ? g : 0)]];
        float* re = sm + (size_t)g * (2 * c.s.plane);
        float* im = re + c.s.plane;
        fafd::run_fft<16>(c.s, t, re, im, c.tw,
                          SplitSrc{a.in_re + off, a.in_im + off, nullptr, a.sgn, 0, live},
                          SplitSink{a.out_re + off, a.out_im + off, c.scale, a.sgn, 0, live});
        __syncthreads();
    }
}

// Rader, as the single-size kernel: gather -> FFT_m (x B) -> IFFT_m -> scatter.
__global__ void __launch_bounds__(kRaderThreads) k_uneven_rader(const UnevenArgs a) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    __shared__ int s_task;
    for (int task; (task = next_task(a, &s_task)) >= 0;) {
        const UnevenTask tk = a.tasks[task];
        const UnevenClass& c = a.classes[tk.cls];
        const int T = c.s.T;
        const int g = threadIdx.x / T, t = threadIdx.x % T;
        const bool live = g < tk.count;
        const long long off = a.offsets[a.items[tk.first + (live ? g : 0)]];
        float* re = sm + (size_t)g * (2 * c.s.plane + c.extra);
        float* im = re + c.s.plane;
        float* dc = re + 2 * c.s.plane;
        const float* xr = a.in_re + off;
        const float* xi = a.in_im + off;
        float x0r = 0.f, x0i = 0.f;
        if (live) { x0r = xr[0]; x0i = a.sgn * xi[0]; }
        fafd::run_fft<16>(c.s, t, re, im, c.tw, GatherSrc{xr, xi, c.rin, a.sgn, live},
                          MulBSink{re, im, c.B, dc});
        __syncthreads();
        float* yr = a.out_re + off;
        float* yi = a.out_im + off;
        if (live && t == 0) {
            yr[0] = (x0r + dc[0]) * c.scale;
            yi[0] = a.sgn * (x0i + dc[1]) * c.scale;
        }
        fafd::run_fft<16>(c.s, t, re, im, c.tw, fafd::SmemConjSrc{re, im},
                          ScatterSink{yr, yi, c.rout, x0r, x0i, c.inv_m, c.scale, a.sgn, live});
        __syncthreads();
    }
}

// Transforms of ONE long length at ragged offsets: the four-step path, one
// transform per CTA at a time (all have the same length: static striding).
struct UnevenLargeArgs {
    const int* items;          // transform ids of this length
    int count;
    const long long* offsets;
    const float* in_re;
    const float* in_im;
    float* out_re;
    float* out_im;
    float sgn, scale;
};

__global__ void __launch_bounds__(kLargeThreads) k_uneven_large(const LargeArgs la,
                                                                const UnevenLargeArgs u) {
    extern __shared__ float4 smem4[];
    float* sm = reinterpret_cast<float*>(smem4);
    const lg::Large L = lg::make_large(la);
    for (int j = blockIdx.x; j < u.count; j += gridDim.x) {
        const long long off = u.offsets[u.items[j]];
        __syncthreads();
        lg::four_step(L, sm, lg::MakeColSrc{u.in_re + off, u.in_im + off, L.n2, u.sgn},
                      lg::OutSplit{u.out_re + off, u.out_im + off, u.scale, u.sgn});
    }
}

template <class K>
cudaError_t occupancy(K k, int threads, size_t smem, int* per_sm) {
    cudaError_t e = prep(k, smem);
    if (e != cudaSuccess) return e;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, k, threads, smem);
    if (e == cudaSuccess && *per_sm < 1) *per_sm = 1;
    return e;
}

}  // namespace fafk

// ===========================================================================
// host side
// ===========================================================================

using fafp::DevicePlan;

// The transforms of one long length: either the multi-CTA two-pass
// four-step (power-of-two lengths, over a per-class offset list), or one
// launch of k_uneven_large (one transform per CTA).
struct LargeLaunch {
    fafk::LargeArgs la;
    int first;   // into items
    int count;
    float scale;
    int grid;
    bool pot2 = false;
    DevicePlan* plan = nullptr;
    long long* d_offs = nullptr;  // pot2: element offset of each transform of the class
};

// A power-of-two class (256..16384 points): the compile-time engine over
// the class's offset list, one batched launch.
struct Pot2Launch {
    int log2n;
    const DevicePlan* plan;  // tensor-core plans carry their B table and error flag
    const float2* tws;
    float scale;
    int count;
    fafk::Geometry g;
    long long* d_offs = nullptr;
};

struct faf_uneven {
    int device = 0;
    size_t count = 0;
    size_t total = 0;
    bool inverse = false;
    faf_norm norm = FAF_NORM_NONE;
    std::vector<size_t> lengths;
    std::vector<long long> offsets_h;
    // one single-size plan per distinct length (plain method + tables)
    std::map<int, DevicePlan*> plans;
    std::map<int, DevicePlan*> large_plans;  // four-step tables for long classes
    // persistent launches
    std::vector<fafk::UnevenClass> classes;
    std::vector<fafk::UnevenTask> tasks;  // generic tasks, then Rader tasks
    int ntasks_gen = 0, ntasks_rad = 0;
    std::vector<int> items;
    std::vector<LargeLaunch> large;
    std::vector<Pot2Launch> pot2;
    fafk::UnevenClass* d_classes = nullptr;
    fafk::UnevenTask* d_tasks = nullptr;
    int* d_items = nullptr;
    long long* d_offsets = nullptr;
    int* d_counter = nullptr;  // [0] generic, [1] Rader
    float* d_scratch = nullptr;
    size_t scratch_floats = 0;
    size_t smem_gen = 0, smem_rad = 0;
    int grid_gen = 0, grid_rad = 0;
    int tmult = 1;       // threads-per-transform multiplier (tuned)
    int rad_per_sm = 2;  // resident Rader CTAs per SM (tuned)
    // stream and graph
    cudaStream_t stream = nullptr;
    bool user_stream = false;
    cudaStream_t cap_stream = nullptr;
    cudaStream_t side_stream = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
    cudaGraphExec_t graph = nullptr;
    const void* graph_ptrs[4] = {nullptr, nullptr, nullptr, nullptr};
    std::mutex mu;
};

namespace {

using namespace fafapi;

template <class T>
cudaError_t upload_vec(T** d, const std::vector<T>& h) {
    cudaFree(*d);
    *d = nullptr;
    if (h.empty()) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)d, h.size() * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

void drop_graph(faf_uneven* u) {
    if (u->graph) cudaGraphExecDestroy(u->graph);
    u->graph = nullptr;
    for (auto& p : u->graph_ptrs) p = nullptr;
}

int sm_count() {
    int dev = 0, sms = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 1;
}

// Build class descriptors, task lists and launch shapes for the current
// tuning knobs.
int build_schedule(faf_uneven* u) {
    u->classes.clear();
    u->tasks.clear();
    u->items.clear();
    for (auto& L : u->large) cudaFree(L.d_offs);
    u->large.clear();
    for (auto& P : u->pot2) cudaFree(P.d_offs);
    u->pot2.clear();
    std::map<int, std::vector<int>> by_len;
    for (size_t i = 0; i < u->count; i++) by_len[(int)u->lengths[i]].push_back((int)i);
    const int sms = sm_count();
    size_t smem_gen = 0, smem_rad = 0, scratch = 0;
    struct T2 { int cls; int kind; std::vector<int> ids; double cost; };
    std::vector<T2> tl;
    for (auto& kv : by_len) {
        const int n = kv.first;
        const std::vector<int>& ids = kv.second;
        DevicePlan* p = u->plans[n];
        const float scale = norm_scale(u->norm, u->inverse, (size_t)n);
        if (u->large_plans.count(n)) {
            LargeLaunch L;
            L.plan = u->large_plans[n];
            L.la = large_args(L.plan);
            L.first = 0;  // set below, after the small-class items
            L.count = (int)ids.size();
            L.scale = scale;
            L.grid = std::min(sms, L.count);
            L.pot2 = fafp::large_pot2_plan(L.plan);
            const long long per = L.pot2 ? std::min<long long>(L.count, fafk::large_pot2_chunk(n))
                                         : (long long)L.grid;
            scratch = std::max(scratch, (size_t)per * 2 * (size_t)n);
            u->large.push_back(L);
            continue;
        }
        if (p->kind == fafp::Kind::C2C && p->inner.ct_log2 >= 8) {
            Pot2Launch P;
            P.log2n = p->inner.ct_log2;
            P.plan = p;
            P.tws = p->inner.d_tws;
            P.scale = scale;
            P.count = (int)ids.size();
            P.g = fafp::geometry_ct(p->inner, n, P.count);
            std::vector<long long> offs;
            for (int id : ids) offs.push_back(u->offsets_h[id]);
            cudaError_t e2 = upload_vec(&P.d_offs, offs);
            if (e2 == cudaSuccess)
                e2 = p->tc ? fafp::tc_prepare(p) : fafk::prepare_pot2_c2c(P.log2n, P.g);
            if (e2 != cudaSuccess) {
                cudaFree(P.d_offs);
                return cuda_fail(e2, "uneven power-of-two class");
            }
            u->pot2.push_back(P);
            continue;
        }
        fafk::UnevenClass c;
        memset(&c, 0, sizeof c);
        c.n = n;
        c.scale = scale;
        const bool rader = p->kind == fafp::Kind::RADER;
        const int m = p->inner.n;
        const int cap = rader ? fafk::kRaderThreads : fafk::kUnevenThreads;
        const int T = std::min(fafp::padded_threads(m) * u->tmult, cap);
        c.kind = rader ? fafk::UK_RADER : fafk::UK_GENERIC;
        c.extra = rader ? 2 : 0;
        c.s = p->inner.shape(m);
        c.s.T = T;
        c.tw = p->inner.d_tw;
        c.rin = p->d_rin;
        c.rout = p->d_rout;
        c.B = p->d_B;
        c.inv_m = (float)(1.0 / (double)m);
        c.G = cap / T;
        const size_t sm = (size_t)c.G * (2 * c.s.plane + c.extra) * sizeof(float);
        (rader ? smem_rad : smem_gen) = std::max(rader ? smem_rad : smem_gen, sm);
        const int cls = (int)u->classes.size();
        u->classes.push_back(c);
        const double cost = (double)n * std::log2((double)std::max(n, 2));
        for (size_t i = 0; i < ids.size(); i += c.G) {
            std::vector<int> chunk(ids.begin() + i, ids.begin() + std::min(ids.size(), i + c.G));
            tl.push_back({cls, c.kind, chunk, cost});
        }
    }
    // generic tasks first, then Rader tasks; longest transforms first in each
    std::stable_sort(tl.begin(), tl.end(), [](const T2& x, const T2& y) {
        return x.kind != y.kind ? x.kind < y.kind : x.cost > y.cost;
    });
    u->ntasks_gen = u->ntasks_rad = 0;
    for (auto& t : tl) {
        fafk::UnevenTask k{t.cls, (int)u->items.size(), (int)t.ids.size(), 0};
        u->tasks.push_back(k);
        u->items.insert(u->items.end(), t.ids.begin(), t.ids.end());
        (t.kind == fafk::UK_RADER ? u->ntasks_rad : u->ntasks_gen)++;
    }
    for (auto& L : u->large) {
        L.first = (int)u->items.size();
        const std::vector<int>& ids = by_len[L.la.n1 * L.la.n2];
        u->items.insert(u->items.end(), ids.begin(), ids.end());
        if (L.pot2) {
            std::vector<long long> offs;
            for (int id : ids) offs.push_back(u->offsets_h[id]);
            cudaError_t e2 = upload_vec(&L.d_offs, offs);
            if (e2 != cudaSuccess) return cuda_fail(e2, "uneven four-step offsets");
        }
    }
    u->smem_gen = std::max<size_t>(smem_gen, 16);
    u->smem_rad = std::max<size_t>(smem_rad, 16);
    cudaError_t e = cudaSuccess;
    int per_gen = 1, per_rad = 1;
    if ((e = fafk::occupancy(fafk::k_uneven_generic, fafk::kUnevenThreads, u->smem_gen,
                             &per_gen)) != cudaSuccess ||
        (e = fafk::occupancy(fafk::k_uneven_rader, fafk::kRaderThreads, u->smem_rad,
                             &per_rad)) != cudaSuccess)
        return cuda_fail(e, "uneven kernel attributes");
    for (auto& L : u->large) {
        e = L.pot2 ? fafk::large_pot2_prepare(L.la.n1, L.la.n2)
                   : prep(fafk::k_uneven_large, fafk::large_smem(L.la, fafk::kLargeThreads));
        if (e != cudaSuccess) return cuda_fail(e, "uneven four-step kernel attributes");
    }
    u->grid_gen = std::min(sms * per_gen, u->ntasks_gen);
    u->grid_rad = std::min(sms * std::min(per_rad, u->rad_per_sm), u->ntasks_rad);
    if ((e = upload_vec(&u->d_classes, u->classes)) != cudaSuccess ||
        (e = upload_vec(&u->d_tasks, u->tasks)) != cudaSuccess ||
        (e = upload_vec(&u->d_items, u->items)) != cudaSuccess)
        return cuda_fail(e, "uneven schedule upload");
    if (scratch > u->scratch_floats) {
        cudaFree(u->d_scratch);
        u->d_scratch = nullptr;
        u->scratch_floats = 0;
        e = cudaMalloc(&u->d_scratch, scratch * sizeof(float));
        if (e != cudaSuccess) return cuda_fail(e, "uneven four-step scratch");
        u->scratch_floats = scratch;
    }
    drop_graph(u);
    return 0;
}

struct Bufs {
    float* out_re;
    float* out_im;
    const float* in_re;
    const float* in_im;
};

fafk::UnevenArgs small_args(faf_uneven* u, const Bufs& b, bool rader) {
    fafk::UnevenArgs a;
    a.classes = u->d_classes;
    a.tasks = u->d_tasks + (rader ? u->ntasks_gen : 0);
    a.ntasks = rader ? u->ntasks_rad : u->ntasks_gen;
    a.items = u->d_items;
    a.offsets = u->d_offsets;
    a.in_re = b.in_re;
    a.in_im = b.in_im;
    a.out_re = b.out_re;
    a.out_im = b.out_im;
    a.sgn = u->inverse ? -1.0f : 1.0f;
    a.counter = u->d_counter + (rader ? 1 : 0);
    return a;
}

// Enqueue the whole batch: counter reset, then the four-step launches on
// `st` and the generic + Rader launches on the side stream, joined back.
cudaError_t enqueue(faf_uneven* u, const Bufs& b, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(u->d_counter, 0, 2 * sizeof(int), st);
    if (e != cudaSuccess) return e;
    const bool fork = !u->large.empty() && (u->grid_gen > 0 || u->grid_rad > 0 || !u->pot2.empty());
    cudaStream_t ss = fork ? u->side_stream : st;
    if (fork) {
        if ((e = cudaEventRecord(u->ev_fork, st)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(ss, u->ev_fork, 0)) != cudaSuccess)
            return e;
    }
    for (const LargeLaunch& L : u->large) {
        if (L.pot2) {
            fafk::Large2Args a2;
            memset(&a2, 0, sizeof a2);
            a2.in_re = b.in_re; a2.in_im = b.in_im; a2.out_re = b.out_re; a2.out_im = b.out_im;
            a2.offs = L.d_offs;
            a2.batch = L.count;
            a2.scale = L.scale;
            a2.sgn = u->inverse ? -1.0f : 1.0f;
            a2.tws1 = L.plan->f1.d_tws; a2.tws2 = L.plan->f2.d_tws; a2.twm = L.plan->d_tw_big;
            a2.scratch = u->d_scratch;
            a2.scratch_transforms = fafk::large_pot2_chunk((long long)L.la.n1 * L.la.n2);
            // 512 threads per CTA: two CTAs per SM leave the other branch room
            if ((e = fafk::launch_large_pot2(L.la.n1, L.la.n2, a2, st, 512)) != cudaSuccess)
                return e;
            continue;
        }
        fafk::LargeArgs la = L.la;
        la.scratch = u->d_scratch;
        la.cta_floats = 2LL * la.n1 * la.n2;
        fafk::UnevenLargeArgs a{u->d_items + L.first, L.count, u->d_offsets, b.in_re, b.in_im,
                                b.out_re, b.out_im, u->inverse ? -1.0f : 1.0f, L.scale};
        fafk::k_uneven_large<<<L.grid, fafk::kLargeThreads,
                               fafk::large_smem(la, fafk::kLargeThreads), st>>>(la, a);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    for (const Pot2Launch& P : u->pot2) {
        fafk::C2CArgs a;
        memset(&a, 0, sizeof a);
        a.in_re = b.in_re; a.in_im = b.in_im; a.out_re = b.out_re; a.out_im = b.out_im;
        a.in_dist = a.out_dist = 1LL << P.log2n;
        a.batch = P.count;
        a.scale = P.scale;
        a.sgn = u->inverse ? -1.0f : 1.0f;
        a.offs = P.d_offs;
        // inputs land by bulk copy (k2_c2c_land for every class here, from
        // 256 points: at most 64 groups of 16 threads fit one CTA, one
        // mbarrier each; the radix-16 tensor-core kernel from 8192)
        a.land = (P.log2n >= (P.plan->tc ? 13 : 8) && fafp::land_ok(b.in_re, false)) ? 1 : 0;
        a.err = P.plan->d_wait_err;
        e = P.plan->tc ? fafp::tc_launch(P.plan, a, ss)
                       : fafk::launch_pot2(0, P.log2n, P.tws, &a, P.g, ss);
        if (e != cudaSuccess) return e;
    }
    if (u->grid_gen > 0) {
        fafk::k_uneven_generic<<<u->grid_gen, fafk::kUnevenThreads, u->smem_gen, ss>>>(
            small_args(u, b, false));
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (u->grid_rad > 0) {
        fafk::k_uneven_rader<<<u->grid_rad, fafk::kRaderThreads, u->smem_rad, ss>>>(
            small_args(u, b, true));
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (fork) {
        if ((e = cudaEventRecord(u->ev_join, ss)) != cudaSuccess ||
            (e = cudaStreamWaitEvent(st, u->ev_join, 0)) != cudaSuccess)
            return e;
    }
    return cudaSuccess;
}

int launches_per_run(const faf_uneven* u) {
    int k = (u->grid_gen > 0) + (u->grid_rad > 0) + (int)u->pot2.size();
    for (const LargeLaunch& L : u->large)
        k += L.pot2 ? fafk::large_pot2_launches(L.la.n1, L.la.n2, L.count) : 1;
    return k;
}

cudaError_t capture(faf_uneven* u, const Bufs& b) {
    drop_graph(u);
    cudaGraph_t g = nullptr;
    cudaError_t e = cudaStreamBeginCapture(u->cap_stream, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return e;
    cudaError_t e2 = enqueue(u, b, u->cap_stream);
    e = cudaStreamEndCapture(u->cap_stream, &g);
    if (e2 != cudaSuccess) e = e2;
    if (e == cudaSuccess) e = cudaGraphInstantiate(&u->graph, g, 0);
    if (g) cudaGraphDestroy(g);
    return e;
}

bool all_device(const void* a, const void* b, const void* c, const void* d) {
    return ptr_is_device(a) && ptr_is_device(b) && ptr_is_device(c) && ptr_is_device(d);
}

double time_once(faf_uneven* u, const Bufs& b, int reps) {
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    enqueue(u, b, u->cap_stream);  // warm
    cudaEventRecord(e0, u->cap_stream);
    for (int r = 0; r < reps; r++) enqueue(u, b, u->cap_stream);
    cudaEventRecord(e1, u->cap_stream);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}

// Launch-shape autotuner: threads per transform (x1 / x2 / x4 of the padded
// minimum; transforms per CTA follow as 1024 / T) and resident Rader CTAs per
// SM (1 / 2 / 4), timed on the plan's own ragged workload.
int autotune(faf_uneven* u) {
    const size_t bytes = u->total * sizeof(float);
    float* buf = nullptr;
    cudaError_t e = cudaMalloc(&buf, 4 * bytes);
    if (e != cudaSuccess) return cuda_fail(e, "autotune buffers");
    cudaMemset(buf, 0, 4 * bytes);
    const Bufs b{buf + 2 * u->total, buf + 3 * u->total, buf, buf + u->total};
    double best = 1e30;
    int best_t = 1, best_c = 2;
    for (int tm : {1, 2, 4}) {
        for (int cps : {1, 2, 4}) {
            u->tmult = tm;
            u->rad_per_sm = cps;
            if (build_schedule(u) != 0) continue;
            const double ms = time_once(u, b, 3);
            if (cudaGetLastError() == cudaSuccess && ms < best) {
                best = ms;
                best_t = tm;
                best_c = cps;
            }
        }
    }
    cudaFree(buf);
    u->tmult = best_t;
    u->rad_per_sm = best_c;
    return build_schedule(u);
}

}  // namespace

extern "C" faf_uneven* faf_uneven_create(const size_t* lengths, size_t count,
                                         const faf_config* cfg) {
    if (!lengths || count == 0) {
        fail("faf_uneven_create: empty length list");
        return nullptr;
    }
    faf_config c = cfg ? *cfg : faf_config_init(0);
    if (c.norm == FAF_NORM_DEFAULT) c.norm = FAF_NORM_NONE;
    if (c.norm == FAF_NORM_LAZY || c.norm == FAF_NORM_JPEG2000) {
        fail("faf_uneven_create: norm '%s' is not an FFT norm", faf_norm_name(c.norm));
        return nullptr;
    }
    if (!backend_ok(c)) return nullptr;
    faf_uneven* u = new faf_uneven();
    cudaGetDevice(&u->device);
    u->count = count;
    u->inverse = c.dir == FAF_DIR_INVERSE;
    u->norm = c.norm;
    u->lengths.assign(lengths, lengths + count);
    u->offsets_h.resize(count);
    size_t off = 0;
    for (size_t i = 0; i < count; i++) {
        const size_t n = lengths[i];
        if (!(is_5_smooth(n) || is_codelet(n) || rader_eligible(n)) || n > 65536) {
            fail("faf_uneven_create: length %zu (transform %zu) must be a legal faf_create_fft "
                 "size <= 65536 (5-smooth, codelet or Rader prime)", n, i);
            faf_uneven_destroy(u);
            return nullptr;
        }
        u->offsets_h[i] = (long long)off;
        off += n;
    }
    u->total = off;
    std::string err;
    for (size_t i = 0; i < count; i++) {
        const int n = (int)lengths[i];
        if (u->plans.count(n)) continue;
        DevicePlan* p = fafp::plan_c2c(n, u->inverse, norm_scale(c.norm, u->inverse, n),
                                       c.flags & FAF_FLAG_TENSOR_CORE, err);
        if (!p) {
            fail("faf_uneven_create: plan for length %d: %s", n, err.c_str());
            faf_uneven_destroy(u);
            return nullptr;
        }
        // The graph runs this class beside the other classes' branch.  The
        // radix-64 tensor-core kernel takes all of an SM's shared memory
        // (227 KB), so it would wait for SMs the other branch holds; the
        // class takes the radix-16 kernel (143 KB) instead, unless
        // FAF_CUDA_TC_RADIX=64 asks for radix 64.
        const char* radix = std::getenv("FAF_CUDA_TC_RADIX");
        if (p->d_tc64 && !(radix && std::strcmp(radix, "64") == 0)) {
            cudaFree(p->d_tc64);
            p->d_tc64 = nullptr;
        }
        u->plans[n] = p;
        // (with 1024-thread CTAs every single-CTA length up to 16384 is one group)
        const bool too_big = p->kind == fafp::Kind::C2C_LARGE ||
                             (p->kind == fafp::Kind::C2C &&
                              fafp::padded_threads(n) > fafk::kUnevenThreads);
        if (p->kind == fafp::Kind::RADER && fafp::padded_threads(n - 1) > fafk::kRaderThreads) {
            fail("faf_uneven_create: Rader length %d is too long for the persistent kernel", n);
            faf_uneven_destroy(u);
            return nullptr;
        }
        if (too_big) {
            DevicePlan* L = p;
            if (p->kind != fafp::Kind::C2C_LARGE) {
                L = new DevicePlan();
                L->device = u->device;
                L->n = n;
                if (!fafp::build_large(L, n, err)) {
                    fafp::plan_free(L);
                    fail("faf_uneven_create: four-step tables for %d: %s", n, err.c_str());
                    faf_uneven_destroy(u);
                    return nullptr;
                }
            }
            u->large_plans[n] = L;
        }
    }
    cudaError_t e = upload_vec(&u->d_offsets, u->offsets_h);
    if (e == cudaSuccess) e = cudaMalloc(&u->d_counter, 2 * sizeof(int));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&u->cap_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&u->side_stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&u->ev_fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&u->ev_join, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        cuda_fail(e, "faf_uneven_create");
        faf_uneven_destroy(u);
        return nullptr;
    }
    const int rc = (c.flags & FAF_FLAG_MEASURE) ? autotune(u) : build_schedule(u);
    if (rc != 0) {
        faf_uneven_destroy(u);
        return nullptr;
    }
    return u;
}

extern "C" int faf_uneven_set_stream(faf_uneven* u, void* stream) {
    if (!u) return fail("faf_uneven_set_stream: NULL plan");
    u->stream = (cudaStream_t)stream;
    u->user_stream = stream != nullptr;
    return 0;
}

extern "C" size_t faf_uneven_total(const faf_uneven* u) { return u ? u->total : 0; }

extern "C" int faf_uneven_execute(faf_uneven* u, float* out_re, float* out_im,
                                  const float* in_re, const float* in_im) {
    if (!u) return fail("faf_uneven_execute: NULL plan");
    if (!all_device(out_re, out_im, in_re, in_im))
        return fail("faf_uneven_execute: buffers must be device memory");
    std::lock_guard<std::mutex> lk(u->mu);
    const void* ptrs[4] = {out_re, out_im, in_re, in_im};
    bool same = u->graph != nullptr;
    for (int i = 0; i < 4; i++) same = same && ptrs[i] == u->graph_ptrs[i];
    cudaError_t e = cudaSuccess;
    if (!same) {
        e = capture(u, Bufs{out_re, out_im, in_re, in_im});
        if (e != cudaSuccess) return cuda_fail(e, "faf_uneven_execute (graph capture)");
        for (int i = 0; i < 4; i++) u->graph_ptrs[i] = ptrs[i];
    }
    e = cudaGraphLaunch(u->graph, u->stream);
    if (e == cudaSuccess && !u->user_stream) e = cudaStreamSynchronize(u->stream);
    if (e != cudaSuccess) return cuda_fail(e, "faf_uneven_execute");
    note_launches(launches_per_run(u));
    return 0;
}

extern "C" int faf_uneven_execute_plain(faf_uneven* u, float* out_re, float* out_im,
                                        const float* in_re, const float* in_im) {
    if (!u) return fail("faf_uneven_execute_plain: NULL plan");
    if (!all_device(out_re, out_im, in_re, in_im))
        return fail("faf_uneven_execute_plain: buffers must be device memory");
    // One batched launch per run of consecutive transforms of equal length.
    int launches = 0;
    size_t i = 0;
    while (i < u->count) {
        size_t j = i + 1;
        while (j < u->count && u->lengths[j] == u->lengths[i]) j++;
        const int n = (int)u->lengths[i];
        const long long off = u->offsets_h[i];
        cudaError_t e = fafp::exec_c2c(u->plans[n], in_re + off, in_im + off, out_re + off,
                                       out_im + off, (long long)(j - i), n, n, false, nullptr,
                                       u->stream);
        if (e != cudaSuccess) return cuda_fail(e, "faf_uneven_execute_plain");
        launches++;
        i = j;
    }
    if (!u->user_stream) {
        cudaError_t e = cudaStreamSynchronize(u->stream);
        if (e != cudaSuccess) return cuda_fail(e, "faf_uneven_execute_plain");
    }
    note_launches(launches);
    return 0;
}

extern "C" void faf_uneven_destroy(faf_uneven* u) {
    if (!u) return;
    drop_graph(u);
    for (auto& kv : u->large_plans)
        if (!u->plans.count(kv.first) || u->plans[kv.first] != kv.second) fafp::plan_free(kv.second);
    for (auto& kv : u->plans) fafp::plan_free(kv.second);
    for (auto& L : u->large) cudaFree(L.d_offs);
    for (auto& P : u->pot2) cudaFree(P.d_offs);
    cudaFree(u->d_classes);
    cudaFree(u->d_tasks);
    cudaFree(u->d_items);
    cudaFree(u->d_offsets);
    cudaFree(u->d_counter);
    cudaFree(u->d_scratch);
    if (u->cap_stream) cudaStreamDestroy(u->cap_stream);
    if (u->side_stream) cudaStreamDestroy(u->side_stream);
    if (u->ev_fork) cudaEventDestroy(u->ev_fork);
    if (u->ev_join) cudaEventDestroy(u->ev_join);
    delete u;
}
