// faf_plan.cu -- planner: radix programs, FP64 tables, launch geometry and
// device-pointer execution for every plan kind.
#include "faf_plan.h"
#include "faf_pot2.cuh"
#include "faf_ring.cuh"

#include <cuda_fp16.h>

#include "faf_cuda.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>

namespace fafp {

namespace {

constexpr int kE = 16;                        // values per thread per stage
constexpr size_t kMaxSmem = 227 * 1024;       // dynamic shared memory per CTA
constexpr size_t kRingStatic = 1024;          // static shared memory of a ring kernel, rounded up
constexpr int kTargetThreads = 256;

template <class T>
cudaError_t upload(T** dst, const T* src, size_t count) {
    *dst = nullptr;
    if (count == 0) return cudaSuccess;
    cudaError_t e = cudaMalloc((void**)dst, count * sizeof(T));
    if (e != cudaSuccess) return e;
    return cudaMemcpy(*dst, src, count * sizeof(T), cudaMemcpyHostToDevice);
}

bool cuda_ok(cudaError_t e, std::string& err, const char* what) {
    if (e == cudaSuccess) return true;
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return false;
}

unsigned long long powmod(unsigned long long b, unsigned long long e, unsigned long long m) {
    unsigned long long r = 1;
    b %= m;
    while (e) {
        if (e & 1) r = r * b % m;
        b = b * b % m;
        e >>= 1;
    }
    return r;
}

int primitive_root(int p) {
    const int phi = p - 1;
    std::vector<int> pf;
    int m = phi;
    for (int d = 2; (long long)d * d <= m; d++)
        if (m % d == 0) {
            pf.push_back(d);
            while (m % d == 0) m /= d;
        }
    if (m > 1) pf.push_back(m);
    for (int g = 2; g < p; g++) {
        bool ok = true;
        for (int q : pf)
            if (powmod(g, phi / q, p) == 1) { ok = false; break; }
        if (ok) return g;
    }
    return 0;
}

bool is_5_smooth(long long n) {
    if (n <= 0) return false;
    for (int p : {2, 3, 5}) while (n % p == 0) n /= p;
    return n == 1;
}

long long next_5_smooth(long long m) {
    if (m <= 1) return 1;
    while (!is_5_smooth(m)) m++;
    return m;
}

// FP64 twiddles W_n^i = exp(-2 pi i i / n).
std::vector<float2> twiddles(int n) {
    std::vector<float2> w(std::max(n, 1));
    for (int i = 0; i < n; i++) {
        const double a = -2.0 * M_PI * (double)i / (double)n;
        w[i] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    return w;
}

void fft_rec(const double* xr, const double* xi, int n, int stride, double* yr, double* yi) {
    if (n == 1) {
        yr[0] = xr[0];
        yi[0] = xi[0];
        return;
    }
    int p = 2;
    while (n % p) p++;
    const int m = n / p;
    std::vector<double> tr(n), ti(n);
    for (int r = 0; r < p; r++)
        fft_rec(xr + (size_t)r * stride, xi + (size_t)r * stride, m, stride * p, &tr[r * m],
                &ti[r * m]);
    for (int k = 0; k < n; k++) {
        double sr = 0, si = 0;
        for (int r = 0; r < p; r++) {
            const long long e = ((long long)r * k) % n;
            const double a = -2.0 * M_PI * (double)e / (double)n;
            const double c = std::cos(a), s = std::sin(a);
            const double ur = tr[r * m + k % m], ui = ti[r * m + k % m];
            sr += ur * c - ui * s;
            si += ur * s + ui * c;
        }
        yr[k] = sr;
        yi[k] = si;
    }
}

}  // namespace

void host_dft_fp64(std::vector<double>& re, std::vector<double>& im) {
    const int n = (int)re.size();
    std::vector<double> yr(n), yi(n);
    fft_rec(re.data(), im.data(), n, 1, yr.data(), yi.data());
    re.swap(yr);
    im.swap(yi);
}

// Radix program: 16s first, then one 8/4/2 for the rest of the power of two,
// then 5s, 3s and 7s.  Any stage order is a valid Stockham program; large
// radices first keeps the number of shared-memory passes minimal.
bool radix_program(int n, std::vector<int>& r) {
    r.clear();
    if (n < 1) return false;
    int m = n, c2 = 0;
    while (m % 2 == 0) { m /= 2; c2++; }
    while (c2 >= 4) { r.push_back(16); c2 -= 4; }
    if (c2 == 3) r.push_back(8);
    if (c2 == 2) r.push_back(4);
    if (c2 == 1) r.push_back(2);
    while (m % 5 == 0) { r.push_back(5); m /= 5; }
    while (m % 3 == 0) { r.push_back(3); m /= 3; }
    while (m % 7 == 0) { r.push_back(7); m /= 7; }
    return m == 1;
}

fafd::Shape FftSize::shape(int slots) const {
    fafd::Shape s;
    s.n = n;
    s.ns = (int)stages.size();
    s.T = T;
    s.plane = plane_floats(slots);
    s.st = d_stages;
    return s;
}

int plane_floats(int slots) {
    const int last = std::max(slots, 1) - 1;
    int p = last + (last >> 5) + 1;
    return (p + 1) & ~1;
}

bool build_size(int n, FftSize& out, std::string& err, int ct_ord) {
    out = FftSize();
    out.n = n;
    std::vector<int> rad;
    if (!radix_program(n, rad)) {
        err = "size " + std::to_string(n) + " is not 7-smooth";
        return false;
    }
    int T = 1, p = 1;
    for (int R : rad) {
        const int mb = std::max(1, kE / R);
        const int need = ((n / R) + mb - 1) / mb;
        T = std::max(T, need);
        out.stages.push_back(fafd::Stage{R, p, n / (p * R), 0});
        p *= R;
    }
    if (T > 1024) {
        err = "size " + std::to_string(n) + " exceeds one CTA";
        return false;
    }
    out.T = T;
    std::vector<float2> w = twiddles(n);
    if (!cuda_ok(upload(&out.d_tw, w.data(), w.size()), err, "twiddle upload")) return false;
    if (!out.stages.empty() &&
        !cuda_ok(upload(&out.d_stages, out.stages.data(), out.stages.size()), err,
                 "stage upload"))
        return false;
    // FAF_CUDA_GENERIC=1 keeps power-of-two sizes on the runtime-radix
    // kernels (both engines stay covered by the parity tests).
    const char* gen = std::getenv("FAF_CUDA_GENERIC");
    const bool force_generic = gen && gen[0] == '1';
    if (!force_generic && n >= 16 && n <= kMaxSingleCta && (n & (n - 1)) == 0) {
        // Per-stage table for the compile-time kernels, in their radix order
        // (fafct::ct_radix: the same function the kernels use); stage s
        // (s >= 1) with span P and radix R holds W_{PR}^{r k} at [(r - 1) P + k],
        // or, for stages that fafct::ct_split_q splits, its two short tables.
        int lg = 0;
        while ((1 << lg) < n) lg++;
        const int ns = fafct::ct_stages(lg, ct_ord);
        std::vector<float2> tws;
        auto w = [&](long long e, int len) {
            const double a = -2.0 * M_PI * (double)e / (double)len;
            tws.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
        };
        for (int s = 1; s < ns; s++) {
            const int R = fafct::ct_radix(lg, ct_ord, s), P = fafct::ct_span(lg, ct_ord, s);
            const int Q = fafct::ct_split_q(lg, ct_ord, s);
            for (int r = 1; r < R; r++) {
                if (!Q) {
                    for (int k = 0; k < P; k++) w((long long)r * k, P * R);
                } else {  // split stage: W^{r a Q} for a < P / Q, then W^{r b} for b < Q
                    for (int a = 0; a < P / Q; a++) w((long long)r * a * Q, P * R);
                    for (int b = 0; b < Q; b++) w((long long)r * b, P * R);
                }
            }
        }
        if (tws.empty()) tws.push_back(make_float2(1.f, 0.f));
        if (!cuda_ok(upload(&out.d_tws, tws.data(), tws.size()), err, "twiddle upload"))
            return false;
        out.ct_log2 = lg;
        out.ct_ord = ct_ord;
    }
    if (out.stages.empty()) {
        // n == 1: keep a valid pointer for the kernels.
        fafd::Stage dummy{1, 1, 1, 0};
        if (!cuda_ok(upload(&out.d_stages, &dummy, 1), err, "stage upload")) return false;
    }
    return true;
}

void free_size(FftSize& s) {
    cudaFree(s.d_stages);
    cudaFree(s.d_tw);
    cudaFree(s.d_tws);
    s.d_stages = nullptr;
    s.d_tw = nullptr;
    s.d_tws = nullptr;
}

// Geometry of the compile-time kernels: interleaved float2 workspace with one
// pad element per 16 (plane2), T = n / 16 threads per transform, about
// `target_threads` threads per CTA (0: by length, below).  With ring > 0 (and n >= 512), the shared
// memory left after the workspaces holds up to `ring` input ring slots (n
// float2 each, at most fafct::kRingMax) and `ring_extra` bytes behind them;
// fewer than 2 slots means no ring.
static int device_sms() { return fafk::sm_count(); }

// Default CTA width of the C2C and C2R kernels by inner length.  Measured on
// B200 (2^25 points per launch, 50-launch event loops, GB/s at 256 / 512 /
// 1024 threads): C2C 512 2941 / 2803 / 2803, 2048 5340 / 5432 / 5581, 4096
// 4585 / 4876 / 5116, 8192 3608 / 3606 / 3854; C2R (inner length n / 2)
// 1024 4246 / 4136 / 4137, 4096 3758 / 3891 / 4195, 8192 3407 / 3493 / 3763,
// 16384 2974 / 2972 / 3190.  Other lengths differ by < 2 %.
static int default_threads(int ct_log2) {
    if (ct_log2 >= 11) return 1024;
    if (ct_log2 == 9) return 256;
    return 512;
}

fafk::Geometry geometry_ct(const FftSize& s, int slots, long long batch, int ring,
                           int target_threads, size_t ring_extra, size_t slot_bytes) {
    fafk::Geometry g;
    g.E = kE;
    const int T = s.n / 16;
    // same layout as k_pot2.cu: even2(plane2(slots)) float2 per group
    const int plane2 = (slots - 1) + ((slots - 1) >> 4) + 1;
    const size_t table = fafk::pot2_table_smem(s.ct_log2, s.ct_ord);
    const size_t per = (size_t)((plane2 + 1) & ~1) * sizeof(float2);
    int target = target_threads > 0 ? target_threads : default_threads(s.ct_log2);
    if (const char* env = std::getenv("FAF_CUDA_CTA_THREADS")) target = std::max(1, atoi(env));
    int G = std::max(1, target / T);
    // a small batch spreads over every SM (one transform per group, as many
    // CTAs as SMs allow) instead of filling a few wide CTAs
    G = (int)std::min<long long>(G, std::max(1LL, batch / device_sms()));
    // groups of >= 32 threads synchronise on named barriers 1..15
    if (T >= 32) G = std::min(G, 15);
    while (G > 1 && ((size_t)G * per + table > kMaxSmem || G * T > 1024)) G--;
    g.G = G;
    g.threads = G * T;
    g.smem = (size_t)G * per;
    // The ring's consumers wait on other groups' progress, which needs every
    // group in warps of its own (T >= 32): groups sharing a warp synchronise
    // with warp barriers across the whole warp.
    if (ring > 0 && T >= 32) {
        const size_t slot = slot_bytes ? slot_bytes : (size_t)s.n * sizeof(float2);
        const size_t used = g.smem + table + kRingStatic + ring_extra;
        int K = used < kMaxSmem ? (int)((kMaxSmem - used) / slot) : 0;
        // FAF_CUDA_RING=k: k slots where they fit (k < 2: no ring)
        const char* env = std::getenv("FAF_CUDA_RING");
        K = std::min({K, env ? atoi(env) : ring, fafct::kRingMax});
        if (K >= 2) {
            g.ring = K;
            g.smem += (size_t)K * slot + ring_extra;
        }
    }
    return g;
}

fafk::Geometry geometry(const FftSize& s, int slots, int extra_floats, long long batch) {
    fafk::Geometry g;
    g.E = kE;
    const size_t per = (size_t)(2 * plane_floats(slots) + extra_floats) * sizeof(float);
    int G = std::max(1, kTargetThreads / s.T);
    G = (int)std::min<long long>(G, std::max(1LL, batch));
    while (G > 1 && ((size_t)G * per > kMaxSmem || G * s.T > 1024)) G--;
    g.G = G;
    g.threads = G * s.T;
    g.smem = (size_t)G * per;
    return g;
}

// CTA width and input-ring slots of the R2C and pipeline kernels by inner
// length (2^ct_log2).  Measured on B200 (2^25 samples per launch, 40-launch
// event loops, GB/s):
//   R2C n = 64 / 128 / 256 (spectra staged, k2_r2c_small): 128 threads
//     2743 / 3032 / 3486, 256 threads 2534 / 2958 / 3457, 1024 threads
//     2069 / 2394 / 2854; n = 512: 256 threads 3582, 1024 threads 3377
//     (no ring below inner length 512); n = 2048: 256 threads with 2 slots
//     4848, 1024 threads with 8 slots 4486; n = 4096 and up: 1024 threads
//     with 8 slots (5012 at 4096; 256 or 512 threads 3200-4420).
//   pipeline n = 512: 512 threads 2806, 1024 2552; n = 1024: 1024 threads
//     with 4 slots 2751, with 2 slots 2458; n = 2048: 512 threads with 3
//     slots 2691, 1024 threads with 2 slots 2239; n = 4096 (200-step bench
//     line): 1024 threads with 3 slots 2845, with 2 slots 2821-2829.  From
//     n = 8192 no ring fits beside 1024 threads' workspaces and the staged
//     tables, and the unstaged kernel at 1024 threads is the fastest (1974
//     against 1449 with 512 threads, ring and staged tables).
struct RealShape {
    int threads, ring;
};
static RealShape r2c_shape(int ct_log2) {
    if (ct_log2 >= 5 && ct_log2 <= 7) return {128, 2};
    if (ct_log2 == 8 || ct_log2 == 10) return {256, 2};
    return {1024, fafct::kRingMax};
}
static RealShape pipe_shape(int ct_log2) {
    switch (ct_log2) {
    case 8: return {512, 2};
    case 9: return {1024, 4};
    case 10: return {512, 3};
    case 11: return {1024, 3};
    default: return {1024, 2};
    }
}

// A landing kernel has one mbarrier per group: at most kLandMaxGroups groups
// (groups of a warp or more already stop at 15).  `g` holds workspaces only.
static void cap_land_groups(fafk::Geometry& g, int T) {
    if (g.G <= fafk::kLandMaxGroups) return;
    g.smem = g.smem / g.G * fafk::kLandMaxGroups;
    g.G = fafk::kLandMaxGroups;
    g.threads = g.G * T;
}

// CTA width and input-ring slots of the STFT kernel by inner length
// (FAF_CUDA_CTA_THREADS and FAF_CUDA_STFT_RING override).  Measured on B200
// (Hann window of n, hop n / 4, 64 x 2^18 samples, GB/s): n = 256: 384
// threads with 8 slots 2204, 512 with 4 2032; n = 512: 256 with 8 2907, 384
// with 8 2772, 512 with 4 2862; n = 1024: 384 with 8 3177 (200-step bench
// line 3156-3162), 512 with 4 2813 (the ring's groups slept waiting for a
// slot); n = 2048: 384 with 4 2923, with 8 2511; n = 4096: 1024 with 8 2790,
// 512 with 4 2246; n = 8192: 1024 with 8 2049, 512 with 4 1759.
static RealShape stft_shape(int ct_log2) {
    RealShape sh{1024, 8};
    if (ct_log2 <= 7 || ct_log2 == 9) sh = {384, 8};
    else if (ct_log2 == 8) sh = {256, 8};
    else if (ct_log2 == 10) sh = {384, 4};
    if (const char* env = std::getenv("FAF_CUDA_STFT_RING")) sh.ring = atoi(env);
    return sh;
}

// Bulk copies of a real input into the ring need every transform start
// 16-byte aligned: base address and distance (floats) a multiple of 4.
// FAF_CUDA_NO_STAGING=1 turns the ring off (direct loads).
static bool ring_ok(const float* x, long long dist) {
    const char* env = std::getenv("FAF_CUDA_NO_STAGING");
    if (env && env[0] == '1') return false;
    return ((unsigned long long)(size_t)x % 16 == 0) && (dist % 4 == 0);
}

// FAF_CUDA_NO_STAGING=1 turns off every landing and staging path.
static bool staging_on() {
    const char* env = std::getenv("FAF_CUDA_NO_STAGING");
    return !(env && env[0] == '1');
}

// Outputs staged in shared memory and written row by row (k2_r2c_small,
// k2_c2c_land<N, true>); FAF_CUDA_STAGE_OUT=0 turns that off alone.
static bool stage_out_on() {
    const char* env = std::getenv("FAF_CUDA_STAGE_OUT");
    return staging_on() && !(env && env[0] == '0');
}

// A staging row of `row` bytes per group behind the workspaces (`g` holds
// workspaces only: no ring at these lengths); fewer groups where the rows do
// not fit.
static void add_stage_rows(fafk::Geometry& g, const FftSize& s, size_t row) {
    const size_t per = g.smem / g.G;
    const size_t table = fafk::pot2_table_smem(s.ct_log2, s.ct_ord);
    int G = g.G;
    while (G > 1 && (size_t)G * (per + row) + table > kMaxSmem) G--;
    g.G = G;
    g.threads = G * (s.n / 16);
    g.smem = (size_t)G * (per + row);
}

// Real samples landed by bulk copy and read as float2 pairs (k2_r2c_land):
// every transform start 8-byte aligned.  FAF_CUDA_NO_STAGING=1: direct loads.
static bool pairs_ok(const float* x, long long dist) {
    const char* env = std::getenv("FAF_CUDA_NO_STAGING");
    if (env && env[0] == '1') return false;
    return ((unsigned long long)(size_t)x % 8 == 0) && (dist % 2 == 0);
}

// Bulk copies of a C2C input into the workspace (k2_c2c_land and the
// tensor-core kernels): any plane alignment and distance; interleaved pairs
// 8-byte aligned (as the direct loads need).  FAF_CUDA_NO_STAGING=1: direct
// loads.
bool land_ok(const float* re, bool inter) {
    const char* env = std::getenv("FAF_CUDA_NO_STAGING");
    if (env && env[0] == '1') return false;
    return !inter || (unsigned long long)(size_t)re % 8 == 0;
}

// ---------------------------------------------------------------------------
// Plan creation
// ---------------------------------------------------------------------------

static DevicePlan* new_plan(Kind k, int n) {
    DevicePlan* p = new DevicePlan();
    p->kind = k;
    p->n = n;
    cudaGetDevice(&p->device);
    // bounded-wait flag of the kernels that wait on copies (left NULL if the
    // allocation fails: those kernels then only skip the report)
    if (cudaMalloc(&p->d_wait_err, sizeof(int)) == cudaSuccess)
        cudaMemset(p->d_wait_err, 0, sizeof(int));
    else
        p->d_wait_err = nullptr, cudaGetLastError();
    return p;
}

void plan_free(DevicePlan* p) {
    if (!p) return;
    plan_free(p->sub_fwd);
    plan_free(p->sub_inv);
    free_size(p->inner);
    free_size(p->f1);
    free_size(p->f2);
    cudaFree(p->d_tw_big);
    cudaFree(p->d_stw);
    cudaFree(p->d_B);
    cudaFree(p->d_phi);
    cudaFree(p->d_rin);
    cudaFree(p->d_rout);
    cudaFree(p->d_window);
    cudaFree(p->d_psi);
    cudaFree(p->d_tw64);
    cudaFree(p->d_stw64);
    cudaFree(p->d_tcB);
    cudaFree(p->d_tc64);
    cudaFree(p->d_tc_err);
    cudaFree(p->d_wait_err);
    cudaFree(p->d_stage);
    cudaFree(p->d_scratch);
    cudaFree(p->d_work);
    if (p->cp_h2d) cudaStreamDestroy(p->cp_h2d);
    if (p->cp_d2h) cudaStreamDestroy(p->cp_d2h);
    for (int i = 0; i < 3; i++) {
        if (p->ev_h2d[i]) cudaEventDestroy(p->ev_h2d[i]);
        if (p->ev_kern[i]) cudaEventDestroy(p->ev_kern[i]);
        if (p->ev_d2h[i]) cudaEventDestroy(p->ev_d2h[i]);
    }
    delete p;
}

static bool is_prime(int n) {
    if (n < 2) return false;
    for (int d = 2; (long long)d * d <= n; d++)
        if (n % d == 0) return false;
    return true;
}

static bool is_7_smooth(long long n) {
    if (n <= 0) return false;
    for (int p : {2, 3, 5, 7}) while (n % p == 0) n /= p;
    return n == 1;
}

// ---- four-step plans ------------------------------------------------------

// Minimum threads of the runtime-radix engine for length m (16 values per
// thread per stage), or a large number if m is not 7-smooth.
static int min_threads(int m) {
    std::vector<int> rad;
    if (!radix_program(m, rad)) return 1 << 30;
    int T = 1;
    for (int R : rad) {
        const int mb = std::max(1, kE / R);
        T = std::max(T, ((m / R) + mb - 1) / mb);
    }
    return T;
}

// Threads per sub-transform, padded to a power of two dividing the CTA size
// (so every thread of the CTA belongs to a group in both passes).
int padded_threads(int m) {
    const int t = min_threads(m);
    int p = 1;
    while (p < t) p <<= 1;
    return p;
}

// Lengths that the single-CTA kernels cannot hold: above kMaxSingleCta, or
// needing more than 1024 threads at 16 values per thread (e.g. 5^6 = 15625,
// whose radix-5 stages keep 15 values per thread).  They take the four-step.
bool needs_four_step(int n) { return n > kMaxSingleCta || min_threads(n) > 1024; }

// n = n1 * n2 with n1 <= n2, both 7-smooth and both within one group of a
// kLargeThreads CTA; n1 the largest such divisor <= sqrt(n).
static bool choose_factors(int n, int& n1, int& n2) {
    n1 = n2 = 0;
    for (int d = 2; (long long)d * d <= n; d++) {
        if (n % d) continue;
        const int e = n / d;
        if (!is_7_smooth(d) || !is_7_smooth(e)) continue;
        if (padded_threads(d) > fafk::kLargeThreads || padded_threads(e) > fafk::kLargeThreads)
            continue;
        n1 = d;
        n2 = e;
    }
    return n1 > 0;
}

bool build_large(DevicePlan* p, int n, std::string& err) {
    if (!choose_factors(n, p->n1, p->n2)) {
        err = "no four-step factorisation for length " + std::to_string(n);
        return false;
    }
    if (!build_size(p->n1, p->f1, err) || !build_size(p->n2, p->f2, err)) return false;
    p->t1 = padded_threads(p->n1);
    p->t2 = padded_threads(p->n2);
    // middle twiddles laid out like the pass-1 output: [k1 * n2 + c] = W_n^{c k1}
    std::vector<float2> w((size_t)n);
    for (int k1 = 0; k1 < p->n1; k1++)
        for (int c = 0; c < p->n2; c++) {
            const double a = -2.0 * M_PI * (double)((long long)c * k1) / (double)n;
            w[(size_t)k1 * p->n2 + c] = make_float2((float)std::cos(a), (float)std::sin(a));
        }
    if (!cuda_ok(upload(&p->d_tw_big, w.data(), w.size()), err, "twiddle upload")) return false;
    p->large = true;
    return true;
}

static bool is_prime(int n);
static bool is_7_smooth(long long n);

// B operand of the tensor-core radix-16 stage: D = A B^T with A rows
// (x_re[0..15], x_im[0..15]) and D rows (y_re[0..15], y_im[0..15]), so
//   B[j][m] = Fr[j][m], B[j][16+m] = -Fi[j][m], B[16+j][m] = Fi[j][m],
//   B[16+j][16+m] = Fr[j][m],   F[j][m] = exp(-2 pi i j m / 16) (FP64),
// split into FP16 hi = fp16(B) and lo = fp16(B - hi), each stored K-major
// without swizzle: element (n, k) at half index
//   ((n % 8) * 16 + (n / 8) * 128 + (k / 8) * 512 + (k % 8) * 2) / 2.
static bool build_tc_tables(DevicePlan* p, std::string& err) {
    std::vector<uint16_t> h(2 * 1024, 0);
    for (int n = 0; n < 32; n++)
        for (int k = 0; k < 32; k++) {
            const int j = n & 15, m = k & 15;
            const double a = -2.0 * M_PI * (double)((j * m) % 16) / 16.0;
            const double fr = std::cos(a), fi = std::sin(a);
            double v;
            if (n < 16) v = k < 16 ? fr : -fi;
            else v = k < 16 ? fi : fr;
            const __half hi = __double2half(v);
            const __half lo = __double2half(v - (double)__half2float(hi));
            const size_t idx = ((size_t)(n % 8) * 16 + (size_t)(n / 8) * 128 +
                                (size_t)(k / 8) * 512 + (size_t)(k % 8) * 2) / 2;
            h[idx] = __half_as_ushort(hi);
            h[1024 + idx] = __half_as_ushort(lo);
        }
    if (!cuda_ok(cudaMalloc(&p->d_tcB, h.size() * sizeof(uint16_t)), err, "tensor-core table") ||
        !cuda_ok(cudaMemcpy(p->d_tcB, h.data(), h.size() * sizeof(uint16_t),
                            cudaMemcpyHostToDevice), err, "tensor-core table") ||
        !cuda_ok(cudaMalloc(&p->d_tc_err, sizeof(int)), err, "tensor-core flag") ||
        !cuda_ok(cudaMemset(p->d_tc_err, 0, sizeof(int)), err, "tensor-core flag"))
        return false;
    p->tc = true;
    return true;
}

// Tables of the radix-64 form (k_tc64.cu): one buffer laid out as the
// kernel's shared memory from its B offset.
//   B hi, B lo: the 64-point forward DFT as a 128 x 128 real matrix for
//     D = A B^T with A rows (re z_0, im z_0, re z_1, ...) and D rows
//     (re Y_0, im Y_0, ...): B[2m][2j] = cos t, B[2m][2j+1] = sin t,
//     B[2m+1][2j] = -sin t, B[2m+1][2j+1] = cos t, t = 2 pi (j m mod 64) / 64
//     (FP64), split into FP16 hi = fp16(B) and lo = fp16(B - hi), K-major
//     without swizzle: element (n, k) at byte
//     (n % 8) * 16 + (n / 8) * 128 + (k / 8) * 2048 + (k % 8) * 2;
//   W_{64 R0}^e at [e] (256 entries), W_N^{16 b a} at [b * 4 R0 + a] and
//     W_N^{b c} at [b * 16 + c] (1024 entries each), FP32 from FP64,
// where N = 4096 R0.
static bool build_tc64_tables(DevicePlan* p, int log2n, std::string& err) {
    const int n = 1 << log2n, r0 = n / 4096;
    std::vector<uint8_t> buf(fafk::tc64_table_bytes(), 0);
    uint16_t* h = reinterpret_cast<uint16_t*>(buf.data());
    const size_t half_tile = 128 * 128;
    for (int row = 0; row < 128; row++)
        for (int k = 0; k < 128; k++) {
            const int m = row >> 1, j = k >> 1;
            const double t = 2.0 * M_PI * (double)((j * m) % 64) / 64.0;
            const double c = std::cos(t), s = std::sin(t);
            const double v = (row & 1) == 0 ? ((k & 1) == 0 ? c : s) : ((k & 1) == 0 ? -s : c);
            const __half hi = __double2half(v);
            const __half lo = __double2half(v - (double)__half2float(hi));
            const size_t idx = ((size_t)(row % 8) * 16 + (size_t)(row / 8) * 128 +
                                (size_t)(k / 8) * 2048 + (size_t)(k % 8) * 2) / 2;
            h[idx] = __half_as_ushort(hi);
            h[half_tile + idx] = __half_as_ushort(lo);
        }
    float2* w = reinterpret_cast<float2*>(buf.data() + 4 * half_tile);
    auto root = [](long long e, long long m) {
        const double a = -2.0 * M_PI * (double)(e % m) / (double)m;
        return make_float2((float)std::cos(a), (float)std::sin(a));
    };
    for (int e = 0; e < 256; e++) w[e] = root(e, 64LL * r0);
    for (int b = 0; b < 64; b++) {
        for (int a = 0; a < 4 * r0; a++) w[256 + b * 4 * r0 + a] = root(16LL * b * a, n);
        for (int c = 0; c < 16; c++) w[256 + 1024 + b * 16 + c] = root((long long)b * c, n);
    }
    return cuda_ok(cudaMalloc(&p->d_tc64, buf.size()), err, "tensor-core tables") &&
           cuda_ok(cudaMemcpy(p->d_tc64, buf.data(), buf.size(), cudaMemcpyHostToDevice), err,
                   "tensor-core tables");
}

// The radix-64 form unless FAF_CUDA_TC_RADIX=16 asks for the radix-16 one.
static bool want_tc64(int log2n) {
    const char* env = std::getenv("FAF_CUDA_TC_RADIX");
    return fafk::tc64_supported(log2n) && !(env && std::strcmp(env, "16") == 0);
}

cudaError_t tc_prepare(const DevicePlan* p) {
    return p->d_tc64 ? fafk::prepare_c2c_tc64(p->inner.ct_log2)
                     : fafk::prepare_c2c_tc(p->inner.ct_log2);
}

cudaError_t tc_launch(const DevicePlan* p, const fafk::C2CArgs& a, cudaStream_t st) {
    if (p->d_tc64) return fafk::launch_c2c_tc64(p->inner.ct_log2, a, p->d_tc64, p->d_tc_err, st);
    return fafk::launch_c2c_tc(p->inner.ct_log2, p->inner.d_tws, a, p->d_tcB, p->d_tc_err, st);
}

// FAF_CUDA_FOURSTEP_16K=1: C2C of 16384 points (without the tensor-core
// form) on the multi-CTA two-pass four-step (128 x 128) instead of one CTA.
static bool fourstep_16k(int n, uint32_t flags) {
    const char* env = std::getenv("FAF_CUDA_FOURSTEP_16K");
    return n == 16384 && !(flags & FAF_FLAG_TENSOR_CORE) && env && env[0] == '1';
}

// Rader / Bluestein inner length m beyond one CTA: nested four-step plans,
// forward and unnormalised inverse (the 1/m is applied by the last pass).
static bool build_conv_inner(DevicePlan* p, int m, std::string& err) {
    p->sub_fwd = plan_c2c(m, false, 1.0f, 0, err);
    if (!p->sub_fwd) return false;
    p->sub_inv = plan_c2c(m, true, 1.0f, 0, err);
    if (!p->sub_inv) return false;
    if (p->sub_fwd->kind != Kind::C2C_LARGE || p->sub_inv->kind != Kind::C2C_LARGE) {
        err = "inner length " + std::to_string(m) + " is not a four-step length";
        return false;
    }
    p->inner.n = m;
    return true;
}

DevicePlan* plan_c2c(int n, bool inverse, float scale, uint32_t flags, std::string& err) {
    DevicePlan* p = nullptr;
    if (is_7_smooth(n)) {
        if (needs_four_step(n) || fourstep_16k(n, flags)) {
            p = new_plan(Kind::C2C_LARGE, n);
            if (!build_large(p, n, err)) { plan_free(p); return nullptr; }
            p->inverse = inverse;
            p->scale = scale;
            // the allocation-free entry point's set-up (not needed by the
            // regular path: a failure here only disables that entry point)
            std::string why;
            if (!noalloc_prepare(p, why)) cudaGetLastError();
            return p;
        }
        p = new_plan(Kind::C2C, n);
        if (!build_size(n, p->inner, err)) { plan_free(p); return nullptr; }
        if ((flags & FAF_FLAG_TENSOR_CORE) && p->inner.ct_log2 &&
            fafk::tc_supported(p->inner.ct_log2) &&
            (!build_tc_tables(p, err) ||
             (want_tc64(p->inner.ct_log2) && !build_tc64_tables(p, p->inner.ct_log2, err)))) {
            plan_free(p);
            return nullptr;
        }
    } else if (is_prime(n) && is_7_smooth(n - 1)) {
        // Rader: y = x0 + IDFT_m(DFT_m(x[g^j]) * DFT_m(W_p^{g^-j}))[...]
        const int m = n - 1;
        p = new_plan(Kind::RADER, n);
        if (!(needs_four_step(m) ? build_conv_inner(p, m, err) : build_size(m, p->inner, err))) {
            plan_free(p);
            return nullptr;
        }
        const int g = primitive_root(n);
        const int ginv = (int)powmod(g, n - 2, n);
        std::vector<int> rin(m), rout(m);
        std::vector<double> br(m), bi(m);
        long long a = 1, b = 1;
        for (int j = 0; j < m; j++) {
            rin[j] = (int)a;
            rout[j] = (int)b;
            a = a * g % n;
            b = b * ginv % n;
        }
        for (int j = 0; j < m; j++) {
            const double ang = -2.0 * M_PI * (double)rout[j] / (double)n;
            br[j] = std::cos(ang);
            bi[j] = std::sin(ang);
        }
        host_dft_fp64(br, bi);
        std::vector<float2> B(m);
        for (int j = 0; j < m; j++) B[j] = make_float2((float)br[j], (float)bi[j]);
        if (!cuda_ok(upload(&p->d_rin, rin.data(), m), err, "rader tables") ||
            !cuda_ok(upload(&p->d_rout, rout.data(), m), err, "rader tables") ||
            !cuda_ok(upload(&p->d_B, B.data(), m), err, "rader tables")) {
            plan_free(p);
            return nullptr;
        }
    } else {
        // Bluestein with M = next 5-smooth >= 2n - 1 (reference
        // src/faf_bluestein.c:19-22), chirp phi[k] = exp(-i pi k^2 / n).
        const long long M = next_5_smooth(2LL * n - 1);
        if (M > 2LL * kMaxLength) {
            err = "Bluestein length " + std::to_string(n) + " (M = " + std::to_string(M) +
                  ") exceeds the inner-length cap";
            return nullptr;
        }
        p = new_plan(Kind::BLUESTEIN, n);
        if (!(needs_four_step((int)M) ? build_conv_inner(p, (int)M, err)
                                      : build_size((int)M, p->inner, err))) {
            plan_free(p);
            return nullptr;
        }
        std::vector<float2> phi(n);
        std::vector<double> br(M, 0.0), bi(M, 0.0);
        for (int k = 0; k < n; k++) {
            const long long q = ((long long)k * k) % (2LL * n);
            const double ang = -M_PI * (double)q / (double)n;
            phi[k] = make_float2((float)std::cos(ang), (float)std::sin(ang));
            if (k == 0) {
                br[0] = 1.0;
            } else {
                // b[l] = b[M - l] = conj(phi[l])
                br[k] = std::cos(ang);
                bi[k] = -std::sin(ang);
                br[M - k] = br[k];
                bi[M - k] = bi[k];
            }
        }
        host_dft_fp64(br, bi);
        std::vector<float2> B(M);
        for (long long j = 0; j < M; j++) B[j] = make_float2((float)br[j], (float)bi[j]);
        if (!cuda_ok(upload(&p->d_phi, phi.data(), n), err, "bluestein tables") ||
            !cuda_ok(upload(&p->d_B, B.data(), (size_t)M), err, "bluestein tables")) {
            plan_free(p);
            return nullptr;
        }
    }
    p->inverse = inverse;
    p->scale = scale;
    return p;
}

static bool upload_super_twiddles(DevicePlan* p, int nc, std::string& err) {
    std::vector<float2> stw(std::max(1, nc / 2));
    for (int k = 0; k < nc / 2; k++) {
        const double ph = -M_PI * (((double)(k + 1) / (double)nc) + 0.5);
        stw[k] = make_float2((float)std::cos(ph), (float)std::sin(ph));
    }
    return cuda_ok(upload(&p->d_stw, stw.data(), stw.size()), err, "super-twiddle upload");
}

DevicePlan* plan_r2c(int n, bool inverse, float scale, std::string& err) {
    const int nc = n / 2;
    DevicePlan* p = new_plan(inverse ? Kind::C2R : Kind::R2C, n);
    p->inverse = inverse;
    p->scale = scale;
    // real kinds: the radix order that ends in 8 (fused bin-pair passes)
    const bool ok =
        needs_four_step(nc) ? build_large(p, nc, err) : build_size(nc, p->inner, err, 1);
    if (!ok || !upload_super_twiddles(p, nc, err)) {
        plan_free(p);
        return nullptr;
    }
    return p;
}

DevicePlan* plan_pipeline(int n, float scale_fwd, float scale_inv, std::string& err) {
    DevicePlan* p = plan_r2c(n, false, scale_fwd, err);
    if (!p) return nullptr;
    p->kind = Kind::PIPELINE;
    p->scale2 = scale_inv;
    return p;
}

DevicePlan* plan_stft(int n, int win, int hop, float scale, std::string& err) {
    if (needs_four_step(n / 2)) {
        err = "STFT frames of " + std::to_string(n) + " samples exceed one CTA";
        return nullptr;
    }
    DevicePlan* p = plan_r2c(n, false, scale, err);
    if (!p) return nullptr;
    p->kind = Kind::STFT;
    p->win = win;
    p->hop = hop;
    // Symmetric Hann of win samples, zero-padded to n (the single-frame C2C
    // path reads n entries), reference src/faf_twiddles.c:159-163.
    std::vector<float> w(std::max(n, 1), 0.0f);
    for (int i = 0; i < win; i++)
        w[i] = win > 1 ? (float)(0.5 * (1.0 - std::cos(2.0 * M_PI * (double)i / (double)(win - 1))))
                       : 1.0f;
    if (!cuda_ok(upload(&p->d_window, w.data(), w.size()), err, "window upload")) {
        plan_free(p);
        return nullptr;
    }
    return p;
}

// Inverse STFT: the C2R of n (1/n scaled, so irfft(rfft(x)) = x) plus the
// same symmetric Hann window the forward STFT applies.
DevicePlan* plan_istft(int n, int win, int hop, std::string& err) {
    if (needs_four_step(n / 2)) {
        err = "STFT frames of " + std::to_string(n) + " samples exceed one CTA";
        return nullptr;
    }
    DevicePlan* p = plan_r2c(n, true, (float)(1.0 / (double)n), err);
    if (!p) return nullptr;
    p->kind = Kind::ISTFT;
    p->win = win;
    p->hop = hop;
    std::vector<float> w(std::max(n, 1), 0.0f);
    for (int i = 0; i < win; i++)
        w[i] = win > 1 ? (float)(0.5 * (1.0 - std::cos(2.0 * M_PI * (double)i / (double)(win - 1))))
                       : 1.0f;
    if (!cuda_ok(upload(&p->d_window, w.data(), w.size()), err, "window upload")) {
        plan_free(p);
        return nullptr;
    }
    return p;
}

static bool upload_rows(DevicePlan* p, int rows, const float* src, size_t stride,
                        std::string& err);

// CWT filter bank (the reference's forward execute, src/faf_cwt.c:769-847):
// the R2C of n (unscaled) and the C2R of n (1/n, the reference's NONE norm on
// the inverse) share the inner FFT and super-twiddles; the bank's rows are
// copied to the device, each padded to a multiple of 4 floats.  psi may be a
// host or device pointer.
DevicePlan* plan_cwt(int n, int rows, const float* psi, size_t psi_stride, std::string& err) {
    if (needs_four_step(n / 2)) {
        err = "CWT rows of " + std::to_string(n) + " samples exceed one CTA";
        return nullptr;
    }
    DevicePlan* p = plan_r2c(n, false, 1.0f, err);
    if (!p) return nullptr;
    p->kind = Kind::CWT;
    p->scale2 = (float)(1.0 / (double)n);
    if (!upload_rows(p, rows, psi, psi_stride, err)) {
        plan_free(p);
        return nullptr;
    }
    return p;
}

// Bank rows to the device, each padded to a multiple of 4 floats.
static bool upload_rows(DevicePlan* p, int rows, const float* src, size_t stride,
                        std::string& err) {
    const long long nb = p->n / 2 + 1;
    p->rows = rows;
    p->psi_dist = (nb + 3) & ~3LL;
    const size_t bytes = (size_t)rows * (size_t)p->psi_dist * sizeof(float);
    cudaError_t e = cudaMalloc(&p->d_psi, bytes);
    if (e == cudaSuccess) e = cudaMemset(p->d_psi, 0, bytes);
    if (e == cudaSuccess)
        e = cudaMemcpy2D(p->d_psi, (size_t)p->psi_dist * sizeof(float), src,
                         stride * sizeof(float), (size_t)nb * sizeof(float), (size_t)rows,
                         cudaMemcpyDefault);
    return cuda_ok(e, err, "CWT bank upload");
}

// Dual-frame inverse CWT (src/faf_cwt.c:935-985): the R2C of n (unscaled)
// and the C2R of n (1/n) with the bank's dual rows.
DevicePlan* plan_icwt_dual(int n, int rows, const float* dual, size_t stride, std::string& err) {
    if (needs_four_step(n / 2)) {
        err = "CWT rows of " + std::to_string(n) + " samples exceed one CTA";
        return nullptr;
    }
    DevicePlan* p = plan_r2c(n, false, 1.0f, err);
    if (!p) return nullptr;
    p->kind = Kind::ICWT_DUAL;
    p->scale2 = (float)(1.0 / (double)n);
    if (!upload_rows(p, rows, dual, stride, err)) {
        plan_free(p);
        return nullptr;
    }
    return p;
}

// L1 one-integral inverse CWT (src/faf_cwt.c:879-930): no FFT, only the
// weighted row sum.
DevicePlan* plan_icwt_l1(int n, int rows, int lowpass, double dlog, double c, std::string& err) {
    (void)err;
    DevicePlan* p = new_plan(Kind::ICWT_L1, n);
    p->rows = rows;
    p->lowpass = lowpass ? 1 : 0;
    p->dlog = dlog;
    p->cwt_c = c > 0.0 ? c : 1.0;  // the reference takes C <= 0 as 1
    return p;
}

// ---------------------------------------------------------------------------
// Device-pointer execution
// ---------------------------------------------------------------------------

// ---- four-step execution ---------------------------------------------------

fafk::LargeArgs large_args(const DevicePlan* p) {
    fafk::LargeArgs a;
    std::memset(&a, 0, sizeof a);
    a.s1 = p->f1.shape(p->n1);
    a.s1.T = p->t1;
    a.s2 = p->f2.shape(p->n2);
    a.s2.T = p->t2;
    a.n1 = p->n1;
    a.n2 = p->n2;
    a.tw1 = p->f1.d_tw;
    a.tw2 = p->f2.d_tw;
    a.twn = p->d_tw_big;
    a.scratch = nullptr;
    a.cta_floats = 0;
    return a;
}

// One CTA per SM keeps the per-CTA scratch (2 or 4 x n floats) L2-resident.
static int large_grid(long long batch) {
    const int sms = fafk::sm_count();
    return (int)std::max(1LL, std::min<long long>(batch, sms));
}

static cudaError_t run_large(DevicePlan* p, int kind, const void* args, long long batch,
                             cudaStream_t st) {
    fafk::LargeArgs a = large_args(p);
    const int grid = large_grid(batch);
    a.cta_floats = (kind == 0 ? 2LL : 4LL) * p->n1 * p->n2;
    const size_t bytes = (size_t)grid * (size_t)a.cta_floats * sizeof(float);
    {
        std::lock_guard<std::mutex> lk(p->scratch_mu);
        if (p->work_bytes < bytes) {
            cudaFree(p->d_work);
            p->d_work = nullptr;
            p->work_bytes = 0;
            cudaError_t e = cudaMalloc(&p->d_work, bytes);
            if (e != cudaSuccess) return e;
            p->work_bytes = bytes;
        }
    }
    a.scratch = (float*)p->d_work;
    return fafk::launch_large(kind, a, args, batch, grid, st);
}

// Power-of-two lengths above one CTA: the multi-CTA two-pass four-step
// through a chunked scratch (p->d_work).
static cudaError_t run_large_pot2(DevicePlan* p, const float* in_re, const float* in_im,
                                  float* out_re, float* out_im, long long batch,
                                  long long in_dist, long long out_dist, float sgn,
                                  cudaStream_t st) {
    const long long n = (long long)p->n1 * p->n2;
    const long long chunk = std::min(batch, fafk::large_pot2_chunk(n));
    const size_t bytes = (size_t)chunk * 2 * (size_t)n * sizeof(float);
    {
        std::lock_guard<std::mutex> lk(p->scratch_mu);
        if (p->work_bytes < bytes) {
            cudaFree(p->d_work);
            p->d_work = nullptr;
            p->work_bytes = 0;
            cudaError_t e = cudaMalloc(&p->d_work, bytes);
            if (e != cudaSuccess) return e;
            p->work_bytes = bytes;
        }
    }
    fafk::Large2Args a;
    std::memset(&a, 0, sizeof a);
    a.in_re = in_re; a.in_im = in_im; a.out_re = out_re; a.out_im = out_im;
    a.in_dist = in_dist; a.out_dist = out_dist; a.offs = nullptr; a.batch = batch;
    a.scale = p->scale; a.sgn = sgn;
    a.tws1 = p->f1.d_tws; a.tws2 = p->f2.d_tws; a.twm = p->d_tw_big;
    a.scratch = (float*)p->d_work;
    a.scratch_transforms = chunk;
    return fafk::launch_large_pot2(p->n1, p->n2, a, st);
}

// Rader / Bluestein with nested four-step inner plans, in chunks of at most
// 64 MB of scratch (two split-plane buffers): gather or chirp into S1, FFT
// S1 -> S2, S2 *= B (Rader: DC sum kept), inverse FFT S2 -> S1, scatter or
// chirp to the output (reference src/faf_fft_rader.c:136-232,
// src/faf_bluestein.c:165-223, in the same order of operations).
static long long conv_chunk(const DevicePlan* p, long long batch) {
    const long long m = p->inner.n;
    return std::max(1LL, std::min(batch, (64LL << 20) / (16 * m)));
}

static cudaError_t exec_conv_large(DevicePlan* p, const fafk::ConvArgs& a, cudaStream_t st) {
    const int m = p->inner.n;
    const long long chunk = conv_chunk(p, a.batch);
    const size_t plane = (size_t)chunk * (size_t)m;
    const size_t bytes = 4 * plane * sizeof(float) + (size_t)chunk * sizeof(float2);
    {
        std::lock_guard<std::mutex> lk(p->scratch_mu);
        if (p->work_bytes < bytes) {
            cudaFree(p->d_work);
            p->d_work = nullptr;
            p->work_bytes = 0;
            cudaError_t e = cudaMalloc(&p->d_work, bytes);
            if (e != cudaSuccess) return e;
            p->work_bytes = bytes;
        }
    }
    float* s1r = (float*)p->d_work;
    float* s1i = s1r + plane;
    float* s2r = s1i + plane;
    float* s2i = s2r + plane;
    float2* dc = (float2*)(s2i + plane);
    const bool rader = p->kind == Kind::RADER;
    cudaError_t e = cudaSuccess;
    for (long long b0 = 0; b0 < a.batch && e == cudaSuccess; b0 += chunk) {
        const long long nb = std::min(chunk, a.batch - b0);
        e = fafk::launch_conv_step(rader ? 0 : 1, a, b0, nb, m, s1r, s1i, nullptr, st);
        if (e == cudaSuccess)
            e = exec_c2c(p->sub_fwd, s1r, s1i, s2r, s2i, nb, m, m, false, nullptr, st);
        if (e == cudaSuccess)
            e = fafk::launch_conv_step(2, a, b0, nb, m, s2r, s2i, rader ? dc : nullptr, st);
        if (e == cudaSuccess)
            e = exec_c2c(p->sub_inv, s2r, s2i, s1r, s1i, nb, m, m, false, nullptr, st);
        if (e == cudaSuccess)
            e = fafk::launch_conv_step(rader ? 3 : 4, a, b0, nb, m, s1r, s1i, dc, st);
    }
    return e;
}

int c2c_launches(const DevicePlan* p, long long batch) {
    if (batch <= 0) return 0;
    if (p->sub_fwd) {
        const long long chunk = conv_chunk(p, batch);
        long long k = 0;
        for (long long b0 = 0; b0 < batch; b0 += chunk) {
            const long long nb = std::min(chunk, batch - b0);
            k += 3 + c2c_launches(p->sub_fwd, nb) + c2c_launches(p->sub_inv, nb);
        }
        return (int)k;
    }
    if (p->kind == Kind::C2C_LARGE && large_pot2_plan(p))
        return fafk::large_pot2_launches(p->n1, p->n2, batch);
    return 1;
}

bool large_pot2_plan(const DevicePlan* p) {
    return p->large && p->f1.ct_log2 && p->f2.ct_log2 && fafk::large_pot2_supported(p->n1, p->n2);
}

cudaError_t exec_c2c(DevicePlan* p, const float* in_re, const float* in_im, float* out_re,
                     float* out_im, long long batch, long long in_dist, long long out_dist,
                     bool interleaved, const float* window, cudaStream_t st) {
    const float sgn = p->inverse ? -1.0f : 1.0f;
    if (p->kind == Kind::C2C_LARGE) {
        if (interleaved || window) return cudaErrorNotSupported;
        if (large_pot2_plan(p))
            return run_large_pot2(p, in_re, in_im, out_re, out_im, batch, in_dist, out_dist, sgn,
                                  st);
        fafk::C2CArgs a;
        std::memset(&a, 0, sizeof a);
        a.in_re = in_re; a.in_im = in_im; a.out_re = out_re; a.out_im = out_im;
        a.in_dist = in_dist; a.out_dist = out_dist; a.batch = batch;
        a.scale = p->scale; a.sgn = sgn;
        return run_large(p, 0, &a, batch, st);
    }
    if (p->kind == Kind::C2C) {
        fafk::C2CArgs a;
        a.in_re = in_re; a.in_im = in_im; a.out_re = out_re; a.out_im = out_im;
        a.in_dist = in_dist; a.out_dist = out_dist; a.batch = batch;
        a.scale = p->scale; a.sgn = sgn; a.interleaved = interleaved ? 1 : 0;
        a.window = window;
        // landing from 64 points (the tensor-core kernels: radix 64 from
        // 4096, radix 16 from 8192)
        const int land_min = p->tc ? (p->d_tc64 ? 12 : 13) : 6;
        a.land = (p->inner.ct_log2 >= land_min && !window && land_ok(in_re, interleaved)) ? 1 : 0;
        a.err = p->d_wait_err;
        const int slots = p->inner.n;
        if (p->tc) return tc_launch(p, a, st);
        if (p->inner.ct_log2) {
            // 64 points: outputs staged and written row by row, in 128-thread
            // CTAs.  Measured on B200 (2^25 points per launch): 3685 against
            // 3389 GB/s for the direct stores; at 128 and 256 points staging
            // measured slower (4509 against 5855, 4500 against 5763).
            const bool stg = a.land && p->inner.ct_log2 == 6 && stage_out_on();
            fafk::Geometry g = geometry_ct(p->inner, slots, batch, 0, stg ? 128 : 0);
            if (a.land) cap_land_groups(g, p->inner.n / 16);
            if (stg) {
                a.stage_out = 1;
                add_stage_rows(g, p->inner, (size_t)p->inner.n * sizeof(float2));
            }
            return fafk::launch_pot2(0, p->inner.ct_log2, p->inner.d_tws, &a, g, st);
        }
        return fafk::launch_c2c(p->inner.shape(slots), geometry(p->inner, slots, 0, batch),
                                p->inner.d_tw, a, st);
    }
    if (interleaved) return cudaErrorNotSupported;
    fafk::ConvArgs a;
    std::memset(&a, 0, sizeof a);
    a.in_re = in_re; a.in_im = in_im; a.out_re = out_re; a.out_im = out_im;
    a.in_dist = in_dist; a.out_dist = out_dist; a.batch = batch;
    a.scale = p->scale; a.sgn = sgn; a.n = p->n;
    a.rin = p->d_rin; a.rout = p->d_rout; a.phi = p->d_phi; a.B = p->d_B;
    a.inv_inner = (float)(1.0 / (double)p->inner.n);
    if (p->sub_fwd) return exec_conv_large(p, a, st);
    const int slots = p->inner.n;
    if (p->kind == Kind::RADER)
        return fafk::launch_rader(p->inner.shape(slots), geometry(p->inner, slots, 2, batch),
                                  p->inner.d_tw, a, st);
    if (p->kind == Kind::BLUESTEIN)
        return fafk::launch_bluestein(p->inner.shape(slots), geometry(p->inner, slots, 0, batch),
                                      p->inner.d_tw, a, st);
    return cudaErrorInvalidValue;
}

static fafk::RealArgs real_args(DevicePlan* p, long long batch) {
    fafk::RealArgs a;
    std::memset(&a, 0, sizeof a);
    a.batch = batch;
    a.scale = p->scale;
    a.stw = p->d_stw;
    a.err = p->d_wait_err;
    return a;
}

cudaError_t exec_r2c(DevicePlan* p, const float* x, float* Xr, float* Xi, long long batch,
                     long long in_dist, long long out_dist, bool interleaved, cudaStream_t st) {
    fafk::RealArgs a = real_args(p, batch);
    a.in_a = x; a.out_a = Xr; a.out_b = Xi;
    a.in_dist = in_dist; a.out_dist = out_dist; a.interleaved = interleaved;
    if (p->large) {
        if (a.interleaved) return cudaErrorNotSupported;
        return run_large(p, 1, &a, batch, st);
    }
    const int slots = p->inner.n + 1;
    if (p->inner.ct_log2) {
        const RealShape sh = r2c_shape(p->inner.ct_log2);
        fafk::Geometry g =
            geometry_ct(p->inner, slots, batch, ring_ok(x, in_dist) ? sh.ring : 0, sh.threads);
        // groups narrower than a warp take no ring.  At inner length 256
        // (n = 512) their samples land in the group's workspace
        // (k2_r2c_land): 3849 -> 4602 GB/s on B200 (2^25 samples per launch).
        // Shorter lengths measured no gain (n = 64: 1498 against 1501; 128:
        // 2128 against 2191; 256: 3152 against 3330) and keep the direct loads.
        const int T = p->inner.n / 16;
        if (p->inner.ct_log2 == 8 && pairs_ok(x, in_dist)) {
            a.land = 1;
            cap_land_groups(g, T);
        }
        // inner lengths 32 to 128: spectra staged behind the workspaces and
        // written row by row (k2_r2c_small)
        if (p->inner.ct_log2 >= 5 && p->inner.ct_log2 <= 7 && stage_out_on()) {
            a.stage_out = 1;
            add_stage_rows(g, p->inner, (size_t)(p->inner.n + 1) * sizeof(float2));
        }
        return fafk::launch_pot2(1, p->inner.ct_log2, p->inner.d_tws, &a, g, st);
    }
    return fafk::launch_r2c(p->inner.shape(slots), geometry(p->inner, slots, 0, batch),
                            p->inner.d_tw, a, st);
}

static cudaError_t launch_c2r_args(DevicePlan* p, fafk::RealArgs& a, long long batch,
                                   cudaStream_t st) {
    if (p->large) {
        if (a.interleaved || a.filt) return cudaErrorNotSupported;
        return run_large(p, 2, &a, batch, st);
    }
    const int slots = p->inner.n + 1;
    if (p->inner.ct_log2) {
        fafk::Geometry g = geometry_ct(p->inner, slots, batch);
        if (a.land) cap_land_groups(g, p->inner.n / 16);
        return fafk::launch_pot2(2, p->inner.ct_log2, p->inner.d_tws, &a, g, st);
    }
    return fafk::launch_c2r(p->inner.shape(slots), geometry(p->inner, slots, 0, batch),
                            p->inner.d_tw, a, st);
}

cudaError_t exec_c2r(DevicePlan* p, const float* Xr, const float* Xi, float* y, long long batch,
                     long long in_dist, long long out_dist, bool interleaved, cudaStream_t st) {
    fafk::RealArgs a = real_args(p, batch);
    a.in_a = Xr; a.in_b = Xi; a.out_a = y;
    a.in_dist = in_dist; a.out_dist = out_dist; a.interleaved = interleaved;
    // bins land by bulk copy from inner length 32 (k2_c2r_land; the 32-point
    // workspace holds the two landed planes exactly)
    a.land = (!p->large && p->inner.ct_log2 >= 5 && land_ok(Xr, interleaved)) ? 1 : 0;
    return launch_c2r_args(p, a, batch, st);
}

// Plan scratch of at least `bytes` (scratch_mu; the host-buffer path holds mu).
static cudaError_t plan_scratch(DevicePlan* p, size_t bytes, float** out) {
    std::lock_guard<std::mutex> lk(p->scratch_mu);
    if (p->scratch_bytes < bytes) {
        cudaFree(p->d_scratch);
        p->d_scratch = nullptr;
        p->scratch_bytes = 0;
        cudaError_t e = cudaMalloc(&p->d_scratch, bytes);
        if (e != cudaSuccess) return e;
        p->scratch_bytes = bytes;
    }
    *out = (float*)p->d_scratch;
    return cudaSuccess;
}

// Inverse CWT of `batch` coefficient sets W[rows x n] (packed when batch >
// 1: in_dist = rows * n).  Dual frame: per chunk of signals (64 MB of row
// spectra at most, so they stay in L2), the R2C of every row, the
// dual-weighted sum over rows per bin, and the C2R of the sums.  L1: one
// pass of weighted row sums.
cudaError_t exec_icwt(DevicePlan* p, const float* W, float* x, long long batch, long long in_dist,
                      long long out_dist, cudaStream_t st) {
    const long long n = p->n, rows = p->rows;
    if (p->kind == Kind::ICWT_L1)
        return fafk::launch_icwt_l1(W, n, in_dist, (int)rows, p->lowpass, (float)p->dlog,
                                    (float)p->cwt_c, batch, x, out_dist, st);
    const long long nb = n / 2 + 1, yd = p->psi_dist;
    const long long cap = std::max(1LL, std::min(batch, (64LL << 20) / (rows * yd * 8)));
    float* sc = nullptr;
    cudaError_t e = plan_scratch(p, (size_t)(cap * rows * yd + cap * nb) * 2 * sizeof(float), &sc);
    if (e != cudaSuccess) return e;
    float* Yr = sc;
    float* Yi = Yr + cap * rows * yd;
    float* Ar = Yi + cap * rows * yd;
    float* Ai = Ar + cap * nb;
    for (long long s0 = 0; s0 < batch; s0 += cap) {
        const long long c = std::min(cap, batch - s0);
        if ((e = exec_r2c(p, W + s0 * in_dist, Yr, Yi, c * rows, n, yd, false, st)) !=
            cudaSuccess)
            return e;
        if ((e = fafk::launch_icwt_acc(Yr, Yi, p->d_psi, nb, yd, p->psi_dist, (int)rows, c, Ar,
                                       Ai, st)) != cudaSuccess)
            return e;
        fafk::RealArgs a = real_args(p, c);
        a.scale = p->scale2;
        a.in_a = Ar; a.in_b = Ai; a.out_a = x + s0 * out_dist;
        a.in_dist = nb; a.out_dist = out_dist;
        if ((e = launch_c2r_args(p, a, c, st)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Forward CWT of `batch` signals: per chunk of signals, the R2C into plan
// scratch (split planes; 32 MB of spectra at most, so they stay in L2), then
// one C2R launch over chunk x rows transforms, each reading its signal's
// spectrum weighted by its bank row (transform order signal-major, so the
// rows of one signal run together and re-read its spectrum from L2).
cudaError_t exec_cwt(DevicePlan* p, const float* x, float* W, long long batch, long long in_dist,
                     long long out_dist, cudaStream_t st) {
    const long long nb = p->n / 2 + 1;
    // spectra interleaved, rows an even number of bins apart (16-byte aligned)
    const long long xd = (nb + 1) & ~1LL;
    const long long cap = std::max(1LL, std::min(batch, (32LL << 20) / (xd * 8)));
    float* spec = nullptr;
    cudaError_t e0 = plan_scratch(p, (size_t)cap * (size_t)xd * 2 * sizeof(float), &spec);
    if (e0 != cudaSuccess) return e0;
    for (long long s0 = 0; s0 < batch; s0 += cap) {
        const long long c = std::min(cap, batch - s0);
        cudaError_t e = exec_r2c(p, x + s0 * in_dist, spec, nullptr, c, in_dist, xd, true, st);
        if (e != cudaSuccess) return e;
        fafk::RealArgs a = real_args(p, c * p->rows);
        a.scale = p->scale2;
        a.in_a = spec; a.in_b = nullptr; a.interleaved = 1; a.out_a = W + s0 * out_dist;
        a.in_dist = xd; a.out_dist = out_dist;
        a.filt = p->d_psi; a.filt_dist = p->psi_dist; a.filt_rows = p->rows;
        a.row_len = p->n;
        const int N = p->inner.n;
        if (p->inner.ct_log2 && !p->large && xd == fafk::cwt_slot_x(N) &&
            p->psi_dist == fafk::cwt_slot_psi(N) && ring_ok(spec, 2 * xd)) {
            // spectrum and bank row of every row transform land in the ring.
            // 1024-thread CTAs up to n = 4096, 512 beyond: measured on B200
            // (60 rows, 2^20 samples of signals, GB/s at 1024 / 512 threads
            // with 8 slots) n = 1024 2085 / 2089, 2048 2209 / 2150, 4096
            // 2018 / 1705, 8192 1267 / 1671, 16384 1167 / 1258.
            const int threads = p->inner.ct_log2 >= 12 ? 512 : 1024;
            e = fafk::launch_pot2(2, p->inner.ct_log2, p->inner.d_tws, &a,
                                  geometry_ct(p->inner, N + 1, c * p->rows, fafct::kRingMax,
                                              threads, 0,
                                              (size_t)fafk::cwt_slot_f2(N) * sizeof(float2)),
                                  st);
        } else {
            e = launch_c2r_args(p, a, c * p->rows, st);
        }
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t exec_pipeline(DevicePlan* p, const float* x, float* y, long long batch,
                          long long in_dist, long long out_dist, const fafk::PipeOp* ops,
                          int nops, cudaStream_t st) {
    fafk::RealArgs a = real_args(p, batch);
    a.in_a = x; a.out_a = y;
    a.in_dist = in_dist; a.out_dist = out_dist;
    a.scale = p->scale * p->scale2;  // ops are linear: both norms fold into the store
    a.nops = std::min(nops, fafk::kMaxOps);
    for (int i = 0; i < a.nops; i++) a.ops[i] = ops[i];
    if (p->large) {
        if (a.interleaved) return cudaErrorNotSupported;
        return run_large(p, 3, &a, batch, st);
    }
    const int slots = p->inner.n + 1;
    if (p->inner.ct_log2) {
        const RealShape sh = pipe_shape(p->inner.ct_log2);
        // a single MUL by a spectrum of every bin: the spectrum and the
        // super-twiddles go to shared memory behind the ring slots
        const bool stage = a.nops == 1 && a.ops[0].code == fafk::OP_MUL &&
                           a.ops[0].m == p->inner.n + 1;
        fafk::Geometry g =
            geometry_ct(p->inner, slots, batch, ring_ok(x, in_dist) ? sh.ring : 0, sh.threads,
                        stage ? fafk::pipe_table_bytes(p->inner.n) : 0);
        a.stage_tables = (stage && g.ring >= 2) ? 1 : 0;
        return fafk::launch_pot2(3, p->inner.ct_log2, p->inner.d_tws, &a, g, st);
    }
    return fafk::launch_pipeline(p->inner.shape(slots), geometry(p->inner, slots, 0, batch),
                                 p->inner.d_tw, a, st);
}

cudaError_t exec_stft(DevicePlan* p, const float* x, float* Xr, float* Xi, long long n_sig,
                      long long sig_len, long long frames, bool interleaved, cudaStream_t st) {
    const long long batch = n_sig * frames;
    fafk::RealArgs a = real_args(p, batch);
    a.in_a = x; a.out_a = Xr; a.out_b = Xi;
    a.out_dist = p->n / 2 + 1;
    a.interleaved = interleaved;
    a.window = p->d_window; a.win = p->win; a.hop = p->hop;
    a.sig_len = sig_len; a.frames = frames;
    const int slots = p->inner.n + 1;
    // frames land by bulk copy when every frame start is 16-byte aligned and
    // the window is a whole number of 16-byte units
    const bool ring = ring_ok(x, sig_len) && a.hop % 4 == 0 && a.win % 4 == 0;
    const RealShape sh = stft_shape(p->inner.ct_log2);
    if (p->inner.ct_log2)
        return fafk::launch_pot2(
            4, p->inner.ct_log2, p->inner.d_tws, &a,
            geometry_ct(p->inner, slots, batch, ring ? sh.ring : 0, sh.threads,
                        ((size_t)a.win * sizeof(float) + 15) & ~(size_t)15),
            st);
    return fafk::launch_stft(p->inner.shape(slots), geometry(p->inner, slots, 0, batch),
                             p->inner.d_tw, a, st);
}

cudaError_t exec_istft(DevicePlan* p, const float* Xr, const float* Xi, float* y, long long n_sig,
                       long long frames, long long sig_len, cudaStream_t st) {
    const long long nb = p->n / 2 + 1;
    const size_t bytes = (size_t)(n_sig * frames) * (size_t)p->n * sizeof(float);
    float* tmp = nullptr;
    {
        std::lock_guard<std::mutex> lk(p->scratch_mu);
        if (p->scratch_bytes < bytes) {
            cudaFree(p->d_scratch);
            p->d_scratch = nullptr;
            p->scratch_bytes = 0;
            cudaError_t e = cudaMalloc(&p->d_scratch, bytes);
            if (e != cudaSuccess) return e;
            p->scratch_bytes = bytes;
        }
        tmp = (float*)p->d_scratch;
    }
    cudaError_t e = exec_c2r(p, Xr, Xi, tmp, n_sig * frames, nb, p->n, false, st);
    if (e != cudaSuccess) return e;
    return fafk::launch_ola(tmp, p->d_window, p->n, p->win, p->hop, frames, sig_len, y, n_sig,
                            st);
}

// ---- FP64 plans --------------------------------------------------------------

static constexpr int kThreads64 = 512;

static bool fp64_inner(DevicePlan* p, int m, std::string& err) {
    if (!is_7_smooth(m)) {
        err = "FP64 transforms need a 7-smooth (inner) length, got " + std::to_string(m);
        return false;
    }
    if (!build_size(m, p->inner, err)) return false;
    if (p->inner.T > kThreads64) {
        err = "FP64 transforms of inner length " + std::to_string(m) +
              " need more than one 512-thread CTA";
        return false;
    }
    std::vector<double2> w((size_t)std::max(m, 1));
    for (int i = 0; i < m; i++) {
        const double a = -2.0 * M_PI * (double)i / (double)m;
        w[i] = make_double2(std::cos(a), std::sin(a));
    }
    if (!cuda_ok(upload(&p->d_tw64, w.data(), w.size()), err, "FP64 twiddle upload")) return false;
    p->fp64 = true;
    return true;
}

DevicePlan* plan_c2c64(int n, bool inverse, double scale, std::string& err) {
    DevicePlan* p = new_plan(Kind::C2C, n);
    if (!fp64_inner(p, n, err)) {
        plan_free(p);
        return nullptr;
    }
    p->inverse = inverse;
    p->scale64 = scale;
    p->scale = (float)scale;
    return p;
}

DevicePlan* plan_r2c64(int n, bool inverse, double scale, std::string& err) {
    const int nc = n / 2;
    DevicePlan* p = new_plan(inverse ? Kind::C2R : Kind::R2C, n);
    if (!fp64_inner(p, nc, err)) {
        plan_free(p);
        return nullptr;
    }
    std::vector<double2> stw((size_t)std::max(1, nc / 2));
    for (int k = 0; k < nc / 2; k++) {
        const double ph = -M_PI * (((double)(k + 1) / (double)nc) + 0.5);
        stw[k] = make_double2(std::cos(ph), std::sin(ph));
    }
    if (!cuda_ok(upload(&p->d_stw64, stw.data(), stw.size()), err, "FP64 super-twiddle upload")) {
        plan_free(p);
        return nullptr;
    }
    p->inverse = inverse;
    p->scale64 = scale;
    p->scale = (float)scale;
    return p;
}

static fafk::Geometry geometry64(const FftSize& s, int slots, long long batch) {
    fafk::Geometry g;
    g.E = 16;
    const size_t per = (size_t)2 * plane_floats(slots) * sizeof(double);
    // One transform per CTA from 64 threads up: the engine's barriers are
    // CTA-wide, so CTAs of one transform progress independently and overlap
    // each other's loads (B200, 4096 points: 2444 -> 2789 GB/s; 1024: 2729 ->
    // 3437).  FAF_CUDA_FP64_GROUPS=g: at most g transforms per CTA.
    int G = std::max(1, std::min(kThreads64, 64) / s.T);
    if (const char* env = std::getenv("FAF_CUDA_FP64_GROUPS"))
        G = std::min(std::max(1, kThreads64 / s.T), std::max(1, atoi(env)));
    G = (int)std::min<long long>(G, std::max(1LL, batch));
    while (G > 1 && (size_t)G * per > kMaxSmem) G--;
    g.G = G;
    g.threads = G * s.T;
    g.smem = (size_t)G * per;
    return g;
}

cudaError_t exec_c2c64(DevicePlan* p, const double* in_re, const double* in_im, double* out_re,
                       double* out_im, long long batch, long long in_dist, long long out_dist,
                       bool interleaved, cudaStream_t st) {
    fafk::C2C64Args a;
    std::memset(&a, 0, sizeof a);
    a.in_re = in_re; a.in_im = in_im; a.out_re = out_re; a.out_im = out_im;
    a.in_dist = in_dist; a.out_dist = out_dist; a.batch = batch;
    a.scale = p->scale64; a.sgn = p->inverse ? -1.0 : 1.0; a.interleaved = interleaved ? 1 : 0;
    const int slots = p->inner.n;
    return fafk::launch_fp64(0, p->inner.shape(slots), geometry64(p->inner, slots, batch),
                             p->d_tw64, &a, st);
}

cudaError_t exec_r2c64(DevicePlan* p, const double* x, double* Xr, double* Xi, long long batch,
                       long long in_dist, long long out_dist, cudaStream_t st) {
    fafk::Real64Args a;
    std::memset(&a, 0, sizeof a);
    a.in_a = x; a.out_a = Xr; a.out_b = Xi;
    a.in_dist = in_dist; a.out_dist = out_dist; a.batch = batch;
    a.scale = p->scale64; a.stw = p->d_stw64;
    const int slots = p->inner.n + 1;
    return fafk::launch_fp64(1, p->inner.shape(slots), geometry64(p->inner, slots, batch),
                             p->d_tw64, &a, st);
}

cudaError_t exec_c2r64(DevicePlan* p, const double* Xr, const double* Xi, double* y,
                       long long batch, long long in_dist, long long out_dist, cudaStream_t st) {
    fafk::Real64Args a;
    std::memset(&a, 0, sizeof a);
    a.in_a = Xr; a.in_b = Xi; a.out_a = y;
    a.in_dist = in_dist; a.out_dist = out_dist; a.batch = batch;
    a.scale = p->scale64; a.stw = p->d_stw64;
    const int slots = p->inner.n + 1;
    return fafk::launch_fp64(2, p->inner.shape(slots), geometry64(p->inner, slots, batch),
                             p->d_tw64, &a, st);
}

}  // namespace fafp
