// faf_kernels.cuh -- kernel argument blocks and host launchers shared by the
// planner (faf_plan.cu) and the kernels (faf_kernels.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "faf_types.h"

namespace fafk {

// SM count of the current device, looked up once per device (a process may
// drive several GPUs, and plans on each size their grids by its own count).
inline int sm_count() {
    constexpr int kMaxDev = 64;
    static int cache[kMaxDev];  // 0: not looked up yet
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < kMaxDev && cache[dev] > 0) return cache[dev];
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
        sms <= 0) {
        cudaGetLastError();
        sms = 1;
    }
    if (dev >= 0 && dev < kMaxDev) cache[dev] = sms;
    return sms;
}

// Launch geometry chosen by the planner for one Shape.
struct Geometry {
    int E;          // values per thread per stage (16 or 32)
    int G;          // transforms per CTA
    int threads;    // G * T
    size_t smem;    // dynamic shared memory bytes
    int ring = 0;   // power-of-two real-input kernels: input ring slots (0: direct loads)
};

// Spectral op codes used inside the fused pipeline kernel.
enum : int { OP_NONE = 0, OP_CONJ = 1, OP_MUL = 2, OP_BANDPASS = 3, OP_SCALE = 4,
              OP_ROTATE = 5, OP_DELAY = 6 };
constexpr int kMaxOps = 8;

struct PipeOp {
    int code;
    int lo, hi;          // BANDPASS bins kept: [lo, hi]
    int m;               // MUL: bins used = min(bound bins, n/2+1)
    const float* hr;     // MUL: device H planes
    const float* hi_;
    float f0, f1;        // SCALE: f0; ROTATE: f0 + i f1
    double d0;           // DELAY: samples of delay
    int n;               // DELAY: transform length
};

struct C2CArgs {
    const float* in_re;
    const float* in_im;   // NULL for interleaved
    float* out_re;
    float* out_im;        // NULL for interleaved
    long long in_dist, out_dist;  // floats between transforms (per plane)
    long long batch;
    float scale;
    float sgn;            // +1 forward, -1 inverse (conjugation trick)
    int interleaved;
    const float* window;  // optional per-sample real window (STFT frame), or NULL
    const long long* offs = nullptr;  // per-transform element offsets (in and out), or NULL
    // power-of-two lengths >= 64: each transform's input lands in its
    // group's workspace by bulk copy (any plane alignment, distance and
    // offset list; interleaved pairs 8-byte aligned; no window); err records
    // a wait that ran out
    int land = 0;
    int* err = nullptr;
    // the landed 64-point kernel without an offset list: outputs staged in
    // shared memory behind the workspaces (N float2 per group) and written
    // row by row
    int stage_out = 0;
};

// Groups per CTA of a landing C2C kernel whose transforms are narrower than
// a warp (one mbarrier each); groups of a warp or more stop at 15.
constexpr int kLandMaxGroups = 64;

struct RealArgs {  // R2C / C2R / pipeline / STFT
    const float* in_a;    // R2C: x; C2R: X re
    const float* in_b;    // C2R: X im
    float* out_a;         // R2C: X re; C2R / pipeline: y
    float* out_b;         // R2C: X im
    long long in_dist, out_dist;
    long long batch;
    float scale;
    int interleaved;      // Hermitian side is interleaved (re,im) pairs
    const float2* stw;    // super-twiddles exp(-i*pi*((k+1)/nc + 1/2)), k < nc/2
    // STFT framing
    const float* window;
    int win, hop;
    long long sig_len, frames;
    // pipeline
    int nops;
    PipeOp ops[kMaxOps];
    int* err;             // bit 1 set when a bounded wait of the kernel ran out
    // CWT rows (filtered C2R): transform b = signal * filt_rows + row reads
    // the signal's bins weighted by filter row `row` (filt_dist floats
    // apart) and writes output row `row` (row_len samples) of the signal
    const float* filt;
    long long filt_dist, row_len;
    int filt_rows;
    // C2R of power-of-two inner lengths >= 512 (no filter rows): each
    // transform's bins land in its group's workspace by bulk copy
    int land = 0;
    // pipeline with one MUL by a spectrum of all N + 1 bins and an input
    // ring: the spectrum and the super-twiddles are copied to shared memory
    // behind the ring slots (pipe_table_bytes(N) of them)
    int stage_tables = 0;
    // R2C of inner lengths 32 to 128: spectra staged in shared memory behind
    // the workspaces (N + 1 float2 per group) and written row by row
    int stage_out = 0;
};

// Shared-memory bytes of the staged pipeline tables for inner length N: the
// spectrum's real and imaginary planes (N + 1 floats, each padded to N + 4)
// and the N / 2 super-twiddles.
__host__ __device__ constexpr size_t pipe_table_bytes(int N) {
    return (size_t)2 * (N + 4) * 4 + (size_t)(N / 2) * 8;
}

// Input ring slot of a CWT row in the power-of-two C2R kernel (inner length
// N): the signal's interleaved spectrum, N + 1 bins rounded up to N + 2, and
// the bank row, N + 1 weights rounded up to N + 4 (both 16-byte multiples).
__host__ __device__ constexpr int cwt_slot_x(int N) { return N + 2; }       // float2
__host__ __device__ constexpr int cwt_slot_psi(int N) { return N + 4; }     // floats
__host__ __device__ constexpr int cwt_slot_f2(int N) { return N + 2 + (N + 4) / 2; }

// Offsets of C2R transform b: plain, or a CWT row (RealArgs::filt).
struct C2ROffsets {
    long long io, oo;   // input (elements of in_dist units x fpe) / output float offsets
    const float* f;     // filter row, or NULL
};
__device__ __forceinline__ C2ROffsets c2r_offsets(const RealArgs& a, long long b, int fpe) {
    if (a.filt) {
        const long long s = b / a.filt_rows, row = b - s * a.filt_rows;
        return C2ROffsets{s * a.in_dist * fpe, s * a.out_dist + row * a.row_len,
                          a.filt + row * a.filt_dist};
    }
    return C2ROffsets{b * a.in_dist * fpe, b * a.out_dist, nullptr};
}

struct ConvArgs;
// Rader / Bluestein whose inner length m needs the four-step (k_conv.cu):
// the element-wise passes around the nested inner FFTs, over transforms
// b0 .. b0 + nb - 1.  step 0: Rader gather into s; 1: Bluestein chirp into
// s; 2: s *= B (dc[b] = s[b][0] first, when dc is set); 3: Rader scatter of
// s (the unnormalised inverse FFT) and dc to the output; 4: Bluestein chirp
// of s to the output.
cudaError_t launch_conv_step(int step, const ConvArgs& a, long long b0, long long nb, int m,
                             float* s_re, float* s_im, float2* dc, cudaStream_t st);

struct ConvArgs {  // Rader (prime n) and Bluestein (any n)
    const float* in_re;
    const float* in_im;
    float* out_re;
    float* out_im;
    long long in_dist, out_dist;
    long long batch;
    float scale;
    float sgn;
    int n;                 // outer length
    const int* rin;        // Rader gather  x[rin[j]]
    const int* rout;       // Rader scatter y[rout[j]]
    const float2* phi;     // Bluestein chirp, n entries
    const float2* B;       // FFT of the convolution kernel, inner length
    float inv_inner;       // 1 / inner length
};

// Four-step transforms longer than one CTA (k_large.cu).
constexpr int kLargeThreads = 512;
struct LargeArgs {
    fafd::Shape s1, s2;    // N1 / N2 shapes, T padded to a divisor of kLargeThreads
    int n1, n2;
    const float2* tw1;     // N1-point twiddles
    const float2* tw2;     // N2-point twiddles
    const float2* twn;     // middle twiddles, entry k1 * n2 + c = W_n^{c k1}
    float* scratch;        // per-CTA scratch, cta_floats each
    long long cta_floats;
};
// kind: 0 = C2C (C2CArgs), 1 = R2C, 2 = C2R, 3 = pipeline (RealArgs)
// kernel attribute of the C2C four-step, and its module loaded on the current device
cudaError_t large_c2c_prepare(const LargeArgs& a);
cudaError_t launch_large(int kind, const LargeArgs& a, const void* args, long long batch,
                         int grid, cudaStream_t st);
size_t large_smem(const LargeArgs& a, int threads);

// Host launchers (return a cudaError_t).  `S` is the inner FFT shape.
cudaError_t launch_c2c(const fafd::Shape& S, const Geometry& g, const float2* tw,
                       const C2CArgs& a, cudaStream_t st);
cudaError_t launch_r2c(const fafd::Shape& S, const Geometry& g, const float2* tw,
                       const RealArgs& a, cudaStream_t st);
cudaError_t launch_c2r(const fafd::Shape& S, const Geometry& g, const float2* tw,
                       const RealArgs& a, cudaStream_t st);
cudaError_t launch_pipeline(const fafd::Shape& S, const Geometry& g, const float2* tw,
                            const RealArgs& a, cudaStream_t st);
cudaError_t launch_stft(const fafd::Shape& S, const Geometry& g, const float2* tw,
                        const RealArgs& a, cudaStream_t st);
cudaError_t launch_rader(const fafd::Shape& S, const Geometry& g, const float2* tw,
                         const ConvArgs& a, cudaStream_t st);
cudaError_t launch_bluestein(const fafd::Shape& S, const Geometry& g, const float2* tw,
                             const ConvArgs& a, cudaStream_t st);

// Compile-time power-of-two kernels (k_pot2.cu).  kind: 0 = C2C (C2CArgs),
// 1 = R2C, 2 = C2R, 3 = pipeline, 4 = STFT (RealArgs); log2n in [4, 14];
// `tws` is the per-stage twiddle table of FftSize::d_tws.
cudaError_t launch_pot2(int kind, int log2n, const float2* tws, const void* args,
                        const Geometry& g, cudaStream_t st);
// Shared-memory bytes the twiddle table of a log2n kernel adds to each CTA.
// twiddle-table bytes of the compile-time kernels; ord: radix order (0 C2C, 1 real kinds)
size_t pot2_table_smem(int log2n, int ord = 0);
// Kernel attributes of the compile-time C2C kernel for geometry g (before any
// stream capture reaches its launch).
cudaError_t prepare_pot2_c2c(int log2n, const Geometry& g);

// Batched multi-CTA four-step for power-of-two lengths above one CTA
// (k_large_pot2.cu): columns, then rows, through a chunked scratch.
struct Large2Args {
    const float* in_re;
    const float* in_im;
    float* out_re;
    float* out_im;
    long long in_dist, out_dist;  // element distance between transforms ...
    const long long* offs;        // ... or per-transform element offsets (in and out)
    long long batch;
    float scale, sgn;
    const float2* tws1;           // per-stage tables of the N1- and N2-point engines
    const float2* tws2;
    const float2* twm;            // middle twiddles [k1 * N2 + col]
    float* scratch;               // scratch_transforms x 2 n floats
    long long scratch_transforms;
};
bool large_pot2_supported(int n1, int n2);
long long large_pot2_chunk(long long n);       // transforms per scratch chunk
int large_pot2_launches(int n1, int n2, long long batch);
cudaError_t large_pot2_prepare(int n1, int n2);  // kernel attributes + module, before any capture
// `threads` per CTA of both passes: 256, 512 or 1024; 0 = the default of a
// standalone batch (FAF_CUDA_4STEP_THREADS overrides both).
cudaError_t launch_large_pot2(int n1, int n2, const Large2Args& a, cudaStream_t st,
                              int threads = 0);

// FP64 transforms (k_fp64.cu): kind 0 = C2C (C2C64Args), 1 = R2C, 2 = C2R
// (Real64Args), on the FP64 runtime-radix engine, at most 512 threads per CTA.
struct C2C64Args {
    const double* in_re;
    const double* in_im;   // NULL for interleaved
    double* out_re;
    double* out_im;        // NULL for interleaved
    long long in_dist, out_dist, batch;
    double scale, sgn;
    int interleaved;
};
struct Real64Args {
    const double* in_a;    // R2C: x; C2R: X re
    const double* in_b;    // C2R: X im
    double* out_a;         // R2C: X re; C2R: y
    double* out_b;         // R2C: X im
    long long in_dist, out_dist, batch;
    double scale;
    const double2* stw;    // super-twiddles, FP64
};
cudaError_t launch_icwt_acc(const float* yr, const float* yi, const float* dual, long long nb,
                            long long ydist, long long ddist, int rows, long long batch,
                            float* ar, float* ai, cudaStream_t st);
cudaError_t launch_icwt_l1(const float* W, long long n, long long in_dist, int rows, int lowpass,
                           float dlog, float C, long long batch, float* x, long long out_dist,
                           cudaStream_t st);
cudaError_t launch_fp64(int kind, const fafd::Shape& S, const Geometry& g, const double2* tw,
                        const void* args, cudaStream_t st);

// Overlap-add of the inverse STFT (k_istft.cu).
cudaError_t launch_ola(const float* tmp, const float* w, int n, int win, int hop, long long F,
                       long long L, float* y, long long n_sig, cudaStream_t st);

// Tensor-core precision form of the power-of-two C2C (k_tc.cu).
bool tc_supported(int log2n);
cudaError_t prepare_c2c_tc(int log2n);  // kernel attributes, before any capture
cudaError_t launch_c2c_tc(int log2n, const float2* tws, const C2CArgs& a, const void* gB,
                          int* err, cudaStream_t st);
// Its radix-64 kernels for 4096, 8192 and 16384 points (k_tc64.cu); `tab` is
// the plan's table of tc64_table_bytes() bytes.
bool tc64_supported(int log2n);
size_t tc64_table_bytes();
cudaError_t prepare_c2c_tc64(int log2n);
cudaError_t launch_c2c_tc64(int log2n, const C2CArgs& a, const void* tab, int* err,
                            cudaStream_t st);

}  // namespace fafk
