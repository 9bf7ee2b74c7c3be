// k_fp64.cu -- FP64 transforms (FAF_PREC_FP64): batched single-CTA C2C, R2C
// and C2R on the FP64 runtime-radix engine (faf_device64.cuh), with the
// same data flow as the FP32 generic kernels (k_c2c.cu, k_real.cu): the
// first stage reads global memory through a fused source, the last writes
// through a fused sink, the R2C / C2R super-twiddle passes (reference
// src/faf_rfft.c:61-146) run between the FFT and global memory.  Twiddles and
// super-twiddles are FP64 tables generated in FP64 on the host.
//
// 16 doubles per thread per stage need about twice the FP32 registers, so
// these kernels run at most 512 threads per CTA (inner lengths up to 8192
// complex points).
#include "faf_device64.cuh"
#include "faf_kernels_common.cuh"

namespace fafk {
namespace f64 {

using fafd64::cf;
using fafd64::run_fft;
using fafd64::SmemConjSrc;
using fafd64::SmemIO;

namespace {

struct Src64 {  // split or interleaved complex FP64 input
    const double* re;
    const double* im;
    double sgn;
    int inter;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const {
        if (inter) {
            const double2 v = reinterpret_cast<const double2*>(re)[i];
            return cf{v.x, sgn * v.y};
        }
        return cf{re[i], sgn * im[i]};
    }
};

struct Sink64 {
    double* re;
    double* im;
    double scale, sgn;
    int inter;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int i, cf v) const {
        if (!live) return;
        if (inter) {
            reinterpret_cast<double2*>(re)[i] = make_double2(v.x * scale, sgn * v.y * scale);
        } else {
            re[i] = v.x * scale;
            im[i] = sgn * v.y * scale;
        }
    }
};

struct PairSrc64 {  // z[i] = x[2i] + i x[2i+1]
    const double* x;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ cf get(int i) const { return cf{x[2 * i], x[2 * i + 1]}; }
};

struct PairSink64 {  // C2R unpack: undo the conjugation, y[2i], y[2i+1]
    double* y;
    double scale;
    bool live;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int i, cf v) const {
        if (!live) return;
        y[2 * i] = v.x * scale;
        y[2 * i + 1] = -v.y * scale;
    }
};

struct Group64 {
    int g, t;
    double* re;
    double* im;
};

__device__ __forceinline__ Group64 group64(const fafd::Shape& S, double* sm) {
    Group64 q;
    q.g = threadIdx.x / S.T;
    q.t = threadIdx.x - q.g * S.T;
    q.re = sm + (size_t)q.g * 2 * S.plane;
    q.im = q.re + S.plane;
    return q;
}

}  // namespace

constexpr int kE64 = 16;

__global__ void __launch_bounds__(512) k64_c2c(const fafd::Shape S, const double2* __restrict__ tw,
                                               const C2C64Args a, int G) {
    extern __shared__ double2 smem64[];
    Group64 q = group64(S, reinterpret_cast<double*>(smem64));
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const int fpe = a.interleaved ? 2 : 1;
    const long long io = bi * a.in_dist * fpe, oo = bi * a.out_dist * fpe;
    run_fft<kE64>(S, q.t, q.re, q.im, tw,
                  Src64{a.in_re + io, a.interleaved ? nullptr : a.in_im + io, a.sgn, a.interleaved},
                  Sink64{a.out_re + oo, a.interleaved ? nullptr : a.out_im + oo, a.scale, a.sgn,
                         a.interleaved, live});
}

__global__ void __launch_bounds__(512) k64_r2c(const fafd::Shape S, const double2* __restrict__ tw,
                                               const Real64Args a, int G) {
    extern __shared__ double2 smem64[];
    Group64 q = group64(S, reinterpret_cast<double*>(smem64));
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const int nc = S.n;
    const SmemIO mid{q.re, q.im};
    run_fft<kE64>(S, q.t, q.re, q.im, tw, PairSrc64{a.in_a + bi * a.in_dist}, mid);
    __syncthreads();
    if (!live) return;
    double* Xr = a.out_a + bi * a.out_dist;
    double* Xi = a.out_b + bi * a.out_dist;
    for (int k = q.t; k <= nc / 2; k += S.T) {
        if (k == 0) {
            const cf z = mid.get(0);
            Xr[0] = (z.x + z.y) * a.scale;
            Xi[0] = 0.0;
            Xr[nc] = (z.x - z.y) * a.scale;
            Xi[nc] = 0.0;
        } else {
            // f1 = Z[k] + conj(Z[nc-k]), f2 = Z[k] - conj(Z[nc-k]), t = f2 w
            const cf zk = mid.get(k), zn = mid.get(nc - k);
            const double2 w = a.stw[k - 1];
            const double f1r = zk.x + zn.x, f1i = zk.y - zn.y;
            const double f2r = zk.x - zn.x, f2i = zk.y + zn.y;
            const double tr = f2r * w.x - f2i * w.y, ti = fma(f2r, w.y, f2i * w.x);
            if (k != nc - k) {
                Xr[k] = 0.5 * (f1r + tr) * a.scale;
                Xi[k] = 0.5 * (f1i + ti) * a.scale;
            }
            Xr[nc - k] = 0.5 * (f1r - tr) * a.scale;
            Xi[nc - k] = 0.5 * (ti - f1i) * a.scale;
        }
    }
}

__global__ void __launch_bounds__(512) k64_c2r(const fafd::Shape S, const double2* __restrict__ tw,
                                               const Real64Args a, int G) {
    extern __shared__ double2 smem64[];
    Group64 q = group64(S, reinterpret_cast<double*>(smem64));
    const long long b = (long long)blockIdx.x * G + q.g;
    const bool live = b < a.batch;
    const long long bi = live ? b : 0;
    const int nc = S.n;
    const SmemIO mid{q.re, q.im};
    const double* Xr = a.in_a + bi * a.in_dist;
    const double* Xi = a.in_b + bi * a.in_dist;
    for (int k = q.t; k <= nc / 2; k += S.T) {
        if (k == 0) {
            const double x0 = Xr[0], xn = Xr[nc];
            mid.put(0, cf{x0 + xn, x0 - xn});
        } else {
            // inverse super-twiddle: conj(w)
            const double2 w = a.stw[k - 1];
            const double xr = Xr[k], xi = Xi[k], yr = Xr[nc - k], yi = Xi[nc - k];
            const double fer = xr + yr, fei = xi - yi, dr = xr - yr, di = xi + yi;
            const double wr = w.x, wi = -w.y;
            const double orr = dr * wr - di * wi, oi = fma(dr, wi, di * wr);
            if (k != nc - k) mid.put(k, cf{fer + orr, fei + oi});
            mid.put(nc - k, cf{fer - orr, -(fei - oi)});
        }
    }
    __syncthreads();
    run_fft<kE64>(S, q.t, q.re, q.im, tw, SmemConjSrc{q.re, q.im},
                  PairSink64{a.out_a + bi * a.out_dist, a.scale, live});
}

}  // namespace f64

cudaError_t launch_fp64(int kind, const fafd::Shape& S, const Geometry& g, const double2* tw,
                        const void* args, cudaStream_t st) {
    using namespace f64;
    cudaError_t e;
    switch (kind) {
    case 0: {
        const C2C64Args& a = *(const C2C64Args*)args;
        if (a.batch <= 0) return cudaSuccess;
        if ((e = prep(k64_c2c, g.smem)) != cudaSuccess) return e;
        k64_c2c<<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G);
        break;
    }
    case 1:
    case 2: {
        const Real64Args& a = *(const Real64Args*)args;
        if (a.batch <= 0) return cudaSuccess;
        if (kind == 1) {
            if ((e = prep(k64_r2c, g.smem)) != cudaSuccess) return e;
            k64_r2c<<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G);
        } else {
            if ((e = prep(k64_c2r, g.smem)) != cudaSuccess) return e;
            k64_c2r<<<grid_for(a.batch, g.G), g.threads, g.smem, st>>>(S, tw, a, g.G);
        }
        break;
    }
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace fafk
