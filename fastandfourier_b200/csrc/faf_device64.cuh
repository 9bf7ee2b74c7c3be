// faf_device64.cuh -- the FP64 form of the runtime-radix Stockham engine
// (faf_device.cuh): the same stages, radix butterflies (16 and 8 as 4x4 /
// 2x4, 4, 2, 3, 5, 7), fused sources / sinks and one register block shared
// by all radix cases, with every value, constant and twiddle in double.  It
// serves the FAF_PREC_FP64 transforms, whose results the reference computes
// in FP64 on the CPU (faf_execute_f64, src/faf_vm.c:976-1083).  The stage
// list (fafd::Stage / fafd::Shape) is shared with the FP32 engine; Shape.plane
// counts doubles here.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "faf_device.cuh"

namespace fafd64 {

using fafd::load_stage;
using fafd::Shape;
using fafd::Stage;

__device__ __forceinline__ int pad(int a) { return a + (a >> 5); }

struct cf {
    double x, y;
};

__device__ __forceinline__ void cmul_inplace(double& r, double& i, double wr, double wi) {
    double t = r * wr - i * wi;
    i = fma(r, wi, i * wr);
    r = t;
}

// ---- multiply by W_N^e = exp(-2*pi*i*e/N), specialised at compile time ----
template <int N, int E>
__device__ __forceinline__ void mulw(double& r, double& i) {
    constexpr int e = ((E % N) + N) % N;
    if constexpr (e == 0) {
        return;
    } else if constexpr (4 * e == N) {            // -i
        double t = r; r = i; i = -t;
    } else if constexpr (2 * e == N) {            // -1
        r = -r; i = -i;
    } else if constexpr (4 * e == 3 * N) {        // +i
        double t = r; r = -i; i = t;
    } else if constexpr (8 * e == N) {            // (1 - i)/sqrt2
        constexpr double h = 0.70710678118654752;
        double t = (r + i) * h; i = (i - r) * h; r = t;
    } else if constexpr (8 * e == 3 * N) {        // (-1 - i)/sqrt2
        constexpr double h = 0.70710678118654752;
        double t = (i - r) * h; i = -(r + i) * h; r = t;
    } else if constexpr (8 * e == 5 * N) {        // (-1 + i)/sqrt2
        constexpr double h = 0.70710678118654752;
        double t = -(r + i) * h; i = (r - i) * h; r = t;
    } else if constexpr (8 * e == 7 * N) {        // (1 + i)/sqrt2
        constexpr double h = 0.70710678118654752;
        double t = (r - i) * h; i = (r + i) * h; r = t;
    } else {
        static_assert(N == 16, "generic constant twiddles only for N = 16");
        // cos / sin of 2*pi*e/16 for the odd e that reach here
        constexpr double C1 = 0.92387953251128674, S1 = 0.38268343236508978;
        constexpr double wr = (e == 1 || e == 15) ? C1 : (e == 3 || e == 13) ? S1
                           : (e == 5 || e == 11) ? -S1 : -C1;
        constexpr double sn = (e == 1 || e == 7) ? S1 : (e == 3 || e == 5) ? C1
                           : (e == 9 || e == 15) ? -S1 : -C1;
        // W = cos - i sin
        cmul_inplace(r, i, wr, -sn);
    }
}

// ---- radix-R DFTs in registers (forward) --------------------------------
template <int R>
struct Dft;

template <>
struct Dft<2> {
    __device__ __forceinline__ static constexpr int slot(int r) { return r; }
    __device__ __forceinline__ static void run(double* xr, double* xi) {
        double ar = xr[0], ai = xi[0];
        xr[0] = ar + xr[1]; xi[0] = ai + xi[1];
        xr[1] = ar - xr[1]; xi[1] = ai - xi[1];
    }
};

__device__ __forceinline__ void dft4(double& r0, double& i0, double& r1, double& i1,
                                     double& r2, double& i2, double& r3, double& i3) {
    double ar = r0 + r2, ai = i0 + i2, br = r0 - r2, bi = i0 - i2;
    double cr = r1 + r3, ci = i1 + i3, dr = r1 - r3, di = i1 - i3;
    r0 = ar + cr; i0 = ai + ci;
    r2 = ar - cr; i2 = ai - ci;
    r1 = br + di; i1 = bi - dr;   // b - i*d
    r3 = br - di; i3 = bi + dr;   // b + i*d
}

template <>
struct Dft<4> {
    __device__ __forceinline__ static constexpr int slot(int r) { return r; }
    __device__ __forceinline__ static void run(double* xr, double* xi) {
        dft4(xr[0], xi[0], xr[1], xi[1], xr[2], xi[2], xr[3], xi[3]);
    }
};

// Radix-8 and radix-16 run in place; their outputs come out transposed and
// `slot(r)` names the register that holds output r.
template <>
struct Dft<8> {
    // n = 2m + q: 4-point DFTs over m (per q), twiddle W8^{q k1}, 2-point
    // DFTs over q (per k1); output k1 + 4 k2 lands in register 2 k1 + k2.
    __device__ __forceinline__ static constexpr int slot(int r) { return 2 * (r & 3) + (r >> 2); }
    __device__ __forceinline__ static void run(double* x, double* y) {
        dft4(x[0], y[0], x[2], y[2], x[4], y[4], x[6], y[6]);
        dft4(x[1], y[1], x[3], y[3], x[5], y[5], x[7], y[7]);
        mulw<8, 1>(x[3], y[3]);
        mulw<8, 2>(x[5], y[5]);
        mulw<8, 3>(x[7], y[7]);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++) {
            double ar = x[2 * k1], ai = y[2 * k1];
            x[2 * k1] = ar + x[2 * k1 + 1]; y[2 * k1] = ai + y[2 * k1 + 1];
            x[2 * k1 + 1] = ar - x[2 * k1 + 1]; y[2 * k1 + 1] = ai - y[2 * k1 + 1];
        }
    }
};

template <>
struct Dft<16> {
    // n = 4m + q: 4-point DFTs over m (per q) leave A_q[k1] in register
    // q + 4 k1; twiddle by W16^{q k1}; 4-point DFTs over q (per k1) leave
    // output k1 + 4 k2 in register 4 k1 + k2.
    __device__ __forceinline__ static constexpr int slot(int r) { return 4 * (r & 3) + (r >> 2); }
    __device__ __forceinline__ static void run(double* x, double* y) {
#pragma unroll
        for (int q = 0; q < 4; q++)
            dft4(x[q], y[q], x[q + 4], y[q + 4], x[q + 8], y[q + 8], x[q + 12], y[q + 12]);
        mulw<16, 1>(x[5], y[5]);
        mulw<16, 2>(x[6], y[6]);
        mulw<16, 3>(x[7], y[7]);
        mulw<16, 2>(x[9], y[9]);
        mulw<16, 4>(x[10], y[10]);
        mulw<16, 6>(x[11], y[11]);
        mulw<16, 3>(x[13], y[13]);
        mulw<16, 6>(x[14], y[14]);
        mulw<16, 9>(x[15], y[15]);
#pragma unroll
        for (int k1 = 0; k1 < 4; k1++)
            dft4(x[4 * k1], y[4 * k1], x[4 * k1 + 1], y[4 * k1 + 1], x[4 * k1 + 2],
                 y[4 * k1 + 2], x[4 * k1 + 3], y[4 * k1 + 3]);
    }
};

template <>
struct Dft<3> {
    __device__ __forceinline__ static constexpr int slot(int r) { return r; }
    __device__ __forceinline__ static void run(double* xr, double* xi) {
        constexpr double S = 0.86602540378443865;  // sin(2pi/3)
        double tr = xr[1] + xr[2], ti = xi[1] + xi[2];
        double ur = xr[1] - xr[2], ui = xi[1] - xi[2];
        double mr = fma(-0.5, tr, xr[0]), mi = fma(-0.5, ti, xi[0]);
        xr[0] += tr; xi[0] += ti;
        // y1 = m - i*S*u, y2 = m + i*S*u
        xr[1] = fma(S, ui, mr); xi[1] = fma(-S, ur, mi);
        xr[2] = fma(-S, ui, mr); xi[2] = fma(S, ur, mi);
    }
};

template <>
struct Dft<5> {
    __device__ __forceinline__ static constexpr int slot(int r) { return r; }
    __device__ __forceinline__ static void run(double* xr, double* xi) {
        constexpr double C1 = 0.30901699437494742, C2 = -0.80901699437494742;
        constexpr double S1 = 0.95105651629515357, S2 = 0.58778525229247313;
        double t1r = xr[1] + xr[4], t1i = xi[1] + xi[4], u1r = xr[1] - xr[4], u1i = xi[1] - xi[4];
        double t2r = xr[2] + xr[3], t2i = xi[2] + xi[3], u2r = xr[2] - xr[3], u2i = xi[2] - xi[3];
        double x0r = xr[0], x0i = xi[0];
        double a1r = fma(C1, t1r, fma(C2, t2r, x0r)), a1i = fma(C1, t1i, fma(C2, t2i, x0i));
        double a2r = fma(C2, t1r, fma(C1, t2r, x0r)), a2i = fma(C2, t1i, fma(C1, t2i, x0i));
        double b1r = fma(S1, u1r, S2 * u2r), b1i = fma(S1, u1i, S2 * u2i);
        double b2r = fma(S2, u1r, -S1 * u2r), b2i = fma(S2, u1i, -S1 * u2i);
        xr[0] = x0r + t1r + t2r; xi[0] = x0i + t1i + t2i;
        // y1 = a1 - i b1, y4 = a1 + i b1, y2 = a2 - i b2, y3 = a2 + i b2
        xr[1] = a1r + b1i; xi[1] = a1i - b1r;
        xr[4] = a1r - b1i; xi[4] = a1i + b1r;
        xr[2] = a2r + b2i; xi[2] = a2i - b2r;
        xr[3] = a2r - b2i; xi[3] = a2i + b2r;
    }
};

template <>
struct Dft<7> {
    __device__ __forceinline__ static constexpr int slot(int r) { return r; }
    __device__ __forceinline__ static void run(double* xr, double* xi) {
        constexpr double C[3] = {0.62348980185873353, -0.22252093395631440, -0.90096886790241913};
        constexpr double S[3] = {0.78183148246802981, 0.97492791218182361, 0.43388373911755812};
        double tr[3], ti[3], ur[3], ui[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            tr[k] = xr[k + 1] + xr[6 - k]; ti[k] = xi[k + 1] + xi[6 - k];
            ur[k] = xr[k + 1] - xr[6 - k]; ui[k] = xi[k + 1] - xi[6 - k];
        }
        double x0r = xr[0], x0i = xi[0];
        xr[0] = x0r + tr[0] + tr[1] + tr[2];
        xi[0] = x0i + ti[0] + ti[1] + ti[2];
#pragma unroll
        for (int m = 1; m <= 3; m++) {
            double ar = x0r, ai = x0i, br = 0.0, bi = 0.0;
#pragma unroll
            for (int k = 1; k <= 3; k++) {
                const int e = (k * m) % 7;              // cos(2pi e/7), sin(2pi e/7)
                const int ee = e <= 3 ? e : 7 - e;      // cos symmetric, sin antisymmetric
                const double c = C[ee - 1];
                const double s = e <= 3 ? S[ee - 1] : -S[ee - 1];
                ar = fma(c, tr[k - 1], ar); ai = fma(c, ti[k - 1], ai);
                br = fma(s, ur[k - 1], br); bi = fma(s, ui[k - 1], bi);
            }
            // y_m = a - i b, y_{7-m} = a + i b
            xr[m] = ar + bi; xi[m] = ai - br;
            xr[7 - m] = ar - bi; xi[7 - m] = ai + br;
        }
    }
};

// ---- shared-memory plane pair as a Source / Sink ------------------------
struct SmemIO {
    double* re;
    double* im;
    static constexpr bool kSmem = true;
    __device__ __forceinline__ cf get(int i) const { return cf{re[pad(i)], im[pad(i)]}; }
    __device__ __forceinline__ void put(int i, cf v) const { re[pad(i)] = v.x; im[pad(i)] = v.y; }
};

// Shared-memory source that conjugates on read (start of an inverse FFT).
struct SmemConjSrc {
    double* re;
    double* im;
    static constexpr bool kSmem = true;
    __device__ __forceinline__ cf get(int i) const { return cf{re[pad(i)], -im[pad(i)]}; }
};

// ---- one Stockham stage ---------------------------------------------------
// E bounds the values one thread holds (MB butterflies of radix R).  When the
// source is shared memory and the sink is shared memory, all reads of the
// stage finish (barrier) before any write; SinkSmemSame marks sinks that
// write exactly the slots this thread read (the last stage), which need no
// barrier.
template <int R, int E, class Src, class Snk>
__device__ __forceinline__ void stage(double (&xr)[E], double (&xi)[E], const Stage sg, int n,
                                      int t, int T, const double2* __restrict__ tw,
                                      const Src& src, const Snk& snk) {
    constexpr int MB = (E / R) > 0 ? (E / R) : 1;
    static_assert(MB * R <= E || E < R, "register block too small");
    const int nb = n / R;
#pragma unroll
    for (int i = 0; i < MB; i++) {
        const int b = t + i * T;
        if (b < nb) {
#pragma unroll
            for (int r = 0; r < R; r++) {
                const cf v = src.get(b + r * nb);
                xr[i * R + r] = v.x;
                xi[i * R + r] = v.y;
            }
            if (sg.p > 1) {
                const int k = b % sg.p;
                if (k != 0) {
                    const int step = k * sg.tws;
#pragma unroll
                    for (int r = 1; r < R; r++) {
                        const double2 w = __ldg(&tw[r * step]);
                        cmul_inplace(xr[i * R + r], xi[i * R + r], w.x, w.y);
                    }
                }
            }
            Dft<R>::run(&xr[i * R], &xi[i * R]);
        }
    }
    if constexpr (Src::kSmem && Snk::kSmem) __syncthreads();
#pragma unroll
    for (int i = 0; i < MB; i++) {
        const int b = t + i * T;
        if (b < nb) {
            const int k = (sg.p > 1) ? b % sg.p : 0;
            const int base = (b - k) * R + k;
#pragma unroll
            for (int r = 0; r < R; r++) {
                const int j = i * R + Dft<R>::slot(r);
                snk.put(base + r * sg.p, cf{xr[j], xi[j]});
            }
        }
    }
    if constexpr (Snk::kSmem) __syncthreads();
}

// All radix cases share one register block (xr, xi), so a stage loop with a
// runtime radix needs registers for one case at a time.
template <int E, class Src, class Snk>
__device__ __forceinline__ void dispatch_stage(double (&xr)[E], double (&xi)[E], const Stage sg,
                                               int n, int t, int T,
                                               const double2* __restrict__ tw, const Src& src,
                                               const Snk& snk) {
    switch (sg.R) {
    case 16: stage<16, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    case 8: stage<8, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    case 4: stage<4, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    case 2: stage<2, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    case 3: stage<3, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    case 5: stage<5, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    case 7: stage<7, E>(xr, xi, sg, n, t, T, tw, src, snk); break;
    default: break;
    }
}

// Sink wrapper for the last stage: the wrapped sink writes shared memory at
// the slots it was given, or global memory; either way no extra barrier
// inside the stage (the caller synchronises before reading the result).
template <class Snk>
struct LastSink {
    Snk s;
    static constexpr bool kSmem = false;
    __device__ __forceinline__ void put(int i, cf v) const { s.put(i, v); }
};

// Full forward FFT of S.n points for thread t of its transform group.
// Source is read by the first stage; sink receives every output exactly once
// (by the thread that computed it).  Shared planes re/im are the workspace.
template <int E, class Src, class Snk>
__device__ __forceinline__ void run_fft(const Shape& S, int t, double* re, double* im,
                                        const double2* __restrict__ tw, const Src& src,
                                        const Snk& snk) {
    const SmemIO mid{re, im};
    const LastSink<Snk> last{snk};
    double xr[E], xi[E];
    // The workspace may still be read by a previous phase of the caller.
    if constexpr (!Src::kSmem) __syncthreads();
    if (S.ns == 0) {  // n == 1
        if (t == 0) last.put(0, src.get(0));
        return;
    }
    if (S.ns == 1 && !Src::kSmem) {
        dispatch_stage<E>(xr, xi, load_stage(S.st, 0), S.n, t, S.T, tw, src, last);
        return;
    }
    dispatch_stage<E>(xr, xi, load_stage(S.st, 0), S.n, t, S.T, tw, src, mid);
    if (S.ns == 1) {
        // A single stage sourced from shared memory wrote its results back
        // to the workspace in natural order; hand them to the sink, thread t
        // owning indices t + j*T.
        for (int i = t; i < S.n; i += S.T) last.put(i, mid.get(i));
        return;
    }
    for (int s = 1; s < S.ns - 1; s++)
        dispatch_stage<E>(xr, xi, load_stage(S.st, s), S.n, t, S.T, tw, mid, mid);
    dispatch_stage<E>(xr, xi, load_stage(S.st, S.ns - 1), S.n, t, S.T, tw, mid, last);
}

}  // namespace fafd64
