// faf_plan.h -- host-side planner and device plans for the B200 path.
//
// A DevicePlan is what faf_transform.device_plan points to.  It owns every
// device table of the transform (stage lists, FP64-generated twiddles,
// super-twiddles, Rader permutations and kernel spectrum, Bluestein chirp,
// STFT window) and the staging buffers used when a caller passes host
// memory.  Plans are immutable after creation except for the stream, the
// lazily grown staging buffers (guarded by `mu`) and the four-step scratch.
#pragma once

#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <vector>

#include "faf_kernels.cuh"

namespace fafp {

// Largest transform one CTA holds (radix-16 stages, 16 values per thread,
// 1024 threads).  Longer transforms take the four-step path.
constexpr int kMaxSingleCta = 16384;
constexpr int kMaxLength = 65536;  // the reference's register-file cap (faf.h:95-98)

// One inner FFT size: radix program + device tables.
struct FftSize {
    int n = 0;
    int T = 1;
    std::vector<fafd::Stage> stages;
    fafd::Stage* d_stages = nullptr;
    float2* d_tw = nullptr;   // W_n^i, i < n (forward), from FP64
    int ct_log2 = 0;          // > 0: compile-time power-of-two kernels apply
    int ct_ord = 0;           // their radix order (fafct::ct_radix): 0 C2C, 1 real kinds
    float2* d_tws = nullptr;  // their per-stage table [stage][r-1][k] = W_{PR}^{rk}
    fafd::Shape shape(int slots) const;
};

bool radix_program(int n, std::vector<int>& radices);
bool build_size(int n, FftSize& out, std::string& err, int ct_ord = 0);
void free_size(FftSize& s);
int plane_floats(int slots);
fafk::Geometry geometry(const FftSize& s, int slots, int extra_floats, long long batch);
fafk::Geometry geometry_ct(const FftSize& s, int slots, long long batch, int ring = 0,
                           int target_threads = 0, size_t ring_extra = 0,
                           size_t slot_bytes = 0);

enum class Kind {
    C2C,        // single-CTA C2C (5-smooth / codelet / 7-smooth inner sizes)
    C2C_LARGE,  // four-step C2C through per-CTA scratch (n > kMaxSingleCta)
    RADER,      // prime n, fused gather / FFT_{n-1} / x B / IFFT / scatter
    BLUESTEIN,  // any n, fused chirp / FFT_M / x B / IFFT_M / chirp
    R2C,
    C2R,
    PIPELINE,   // fused R2C -> ops -> C2R
    STFT,       // framed, windowed R2C
    ISTFT,      // batched C2R of frames -> windowed overlap-add
    CWT,        // R2C of each signal, then one filtered C2R per bank row
    ICWT_DUAL,  // R2C of every row, dual-weighted sum over rows, C2R
    ICWT_L1     // weighted sum of the time-domain rows
};

struct DevicePlan {
    Kind kind = Kind::C2C;
    int device = 0;
    int n = 0;             // outer length (real length for R2C family)
    bool inverse = false;  // C2C direction (conjugation trick)
    float scale = 1.0f;    // norm scale of this transform
    double scale64 = 1.0;  // the same, FP64 plans
    float scale2 = 1.0f;   // pipeline: inverse-side scale
    FftSize inner;         // the FFT the kernels run
    // four-step path (inner complex length > kMaxSingleCta): n_inner = n1 * n2
    bool large = false;
    FftSize f1, f2;
    int n1 = 0, n2 = 0, t1 = 0, t2 = 0;  // padded thread counts per sub-transform
    float2* d_tw_big = nullptr;  // four-step middle twiddles [k1 * n2 + c] = W_n^{c k1}
    // Rader / Bluestein whose inner length needs the four-step: the inner
    // FFT as nested four-step C2C plans, forward and unnormalised inverse
    struct DevicePlan* sub_fwd = nullptr;
    struct DevicePlan* sub_inv = nullptr;
    void* d_work = nullptr;      // per-CTA four-step scratch, grown on first use
    size_t work_bytes = 0;
    // tables
    float2* d_stw = nullptr;     // R2C super-twiddles
    float2* d_B = nullptr;       // Rader / Bluestein kernel spectrum
    float2* d_phi = nullptr;     // Bluestein chirp
    int* d_rin = nullptr;        // Rader gather
    int* d_rout = nullptr;       // Rader scatter
    float* d_window = nullptr;   // STFT window
    float* d_psi = nullptr;      // CWT bank (dual rows for ICWT_DUAL): rows x psi_dist weights
    int rows = 0;
    long long psi_dist = 0;
    int lowpass = 0;             // ICWT_L1: row 0 is the lowpass
    double dlog = 0.0, cwt_c = 1.0;  // ICWT_L1: log-scale step and admissibility constant
    // FP64 plans (FAF_PREC_FP64): FP64 twiddle tables of the inner size
    bool fp64 = false;
    double2* d_tw64 = nullptr;   // W_n^i, i < inner n
    double2* d_stw64 = nullptr;  // R2C super-twiddles
    // tensor-core form (C2C, power of two): B = 16-point DFT as a 32 x 32
    // real FP16 matrix, hi then lo, in the MMA's shared-memory layout
    bool tc = false;
    void* d_tcB = nullptr;
    // radix-64 form (4096..16384 points, k_tc64.cu): its B operand and
    // twiddle tables in the kernel's shared-memory layout; null = radix 16
    void* d_tc64 = nullptr;
    int* d_tc_err = nullptr;     // set by a kernel whose MMA wait ran out
    int* d_wait_err = nullptr;   // set by a kernel whose input-ring wait ran out
    int win = 0, hop = 0;
    // launch state
    cudaStream_t stream = nullptr;  // 0 = legacy default stream
    bool user_stream = false;
    // staging for host buffers (mu, held by a host-buffer execute from copy-in
    // to copy-out) and device scratch grown by the kernels' launchers
    // (scratch_mu, taken inside that execute, so it must be another mutex)
    std::mutex mu;
    std::mutex scratch_mu;
    void* d_stage = nullptr;
    size_t stage_bytes = 0;
    // chunked host-buffer path: copy streams and per-slot events (lazy)
    cudaStream_t cp_h2d = nullptr, cp_d2h = nullptr;
    cudaEvent_t ev_h2d[3] = {}, ev_kern[3] = {}, ev_d2h[3] = {};
    void* d_scratch = nullptr;
    size_t scratch_bytes = 0;
};

DevicePlan* plan_c2c(int n, bool inverse, float scale, uint32_t flags, std::string& err);
DevicePlan* plan_r2c(int n, bool inverse, float scale, std::string& err);
DevicePlan* plan_pipeline(int n, float scale_fwd, float scale_inv, std::string& err);
DevicePlan* plan_stft(int n, int win, int hop, float scale, std::string& err);
DevicePlan* plan_istft(int n, int win, int hop, std::string& err);
DevicePlan* plan_cwt(int n, int rows, const float* psi, size_t psi_stride, std::string& err);
DevicePlan* plan_icwt_dual(int n, int rows, const float* dual, size_t stride, std::string& err);
DevicePlan* plan_icwt_l1(int n, int rows, int lowpass, double dlog, double c, std::string& err);
cudaError_t exec_icwt(DevicePlan* p, const float* W, float* x, long long batch, long long in_dist,
                      long long out_dist, cudaStream_t st);
cudaError_t exec_cwt(DevicePlan* p, const float* x, float* W, long long batch, long long in_dist,
                     long long out_dist, cudaStream_t st);
// FP64 plans: single-CTA C2C of 5-smooth / codelet / 7-smooth lengths, and
// R2C / C2R of even lengths whose half is such a length (up to 512 threads).
DevicePlan* plan_c2c64(int n, bool inverse, double scale, std::string& err);
DevicePlan* plan_r2c64(int n, bool inverse, double scale, std::string& err);
cudaError_t exec_c2c64(DevicePlan* p, const double* in_re, const double* in_im, double* out_re,
                       double* out_im, long long batch, long long in_dist, long long out_dist,
                       bool interleaved, cudaStream_t st);
cudaError_t exec_r2c64(DevicePlan* p, const double* x, double* Xr, double* Xi, long long batch,
                       long long in_dist, long long out_dist, cudaStream_t st);
cudaError_t exec_c2r64(DevicePlan* p, const double* Xr, const double* Xi, double* y,
                       long long batch, long long in_dist, long long out_dist, cudaStream_t st);
void plan_free(DevicePlan* p);
// Kernel launches of one exec_c2c of `batch` transforms of plan p.
int c2c_launches(const DevicePlan* p, long long batch);
// The tensor-core form of a C2C plan (p->tc): kernel attributes (before any
// capture), and one batched launch (radix 64 where p->d_tc64, else radix 16).
cudaError_t tc_prepare(const DevicePlan* p);
// Whether a C2C input may land in shared memory by bulk copy (k2_c2c_land and
// the tensor-core kernels, power-of-two lengths from 1024).
bool land_ok(const float* re, bool inter);
cudaError_t tc_launch(const DevicePlan* p, const fafk::C2CArgs& a, cudaStream_t st);

// Device-pointer executes (enqueue on `st`).
cudaError_t exec_c2c(DevicePlan* p, const float* in_re, const float* in_im, float* out_re,
                     float* out_im, long long batch, long long in_dist, long long out_dist,
                     bool interleaved, const float* window, cudaStream_t st);
cudaError_t exec_r2c(DevicePlan* p, const float* x, float* Xr, float* Xi, long long batch,
                     long long in_dist, long long out_dist, bool interleaved, cudaStream_t st);
cudaError_t exec_c2r(DevicePlan* p, const float* Xr, const float* Xi, float* y, long long batch,
                     long long in_dist, long long out_dist, bool interleaved, cudaStream_t st);
cudaError_t exec_pipeline(DevicePlan* p, const float* x, float* y, long long batch,
                          long long in_dist, long long out_dist, const fafk::PipeOp* ops,
                          int nops, cudaStream_t st);
cudaError_t exec_stft(DevicePlan* p, const float* x, float* Xr, float* Xi, long long n_sig,
                      long long sig_len, long long frames, bool interleaved, cudaStream_t st);
cudaError_t exec_istft(DevicePlan* p, const float* Xr, const float* Xi, float* y, long long n_sig,
                       long long frames, long long sig_len, cudaStream_t st);

// Four-step tables of p for complex length n (n1, n2, f1, f2, t1, t2, twiddles).
bool build_large(DevicePlan* p, int n, std::string& err);
// Threads per sub-transform of the runtime-radix engine for length m, padded to
// a power of two (so that groups tile a power-of-two CTA exactly).
int padded_threads(int m);
bool needs_four_step(int n);
// Power-of-two four-step plan that the multi-CTA two-pass kernels serve.
bool large_pot2_plan(const DevicePlan* p);
// Four-step arguments of plan p (scratch left NULL).
fafk::LargeArgs large_args(const DevicePlan* p);
// faf_noalloc.cu: on the plan's device (current), sets up everything
// faf_cuda_execute_c2c_noalloc needs so that the call itself allocates
// nothing -- the static scratch's device address and the kernels' modules,
// both of which lazy module loading would otherwise bring in (allocating) at
// the first call.  Called when a four-step C2C plan is created.
bool noalloc_prepare(const DevicePlan* p, std::string& err);

// Host FFT in double precision (table generation only).
void host_dft_fp64(std::vector<double>& re, std::vector<double>& im);

}  // namespace fafp
