/*
 * faf_oracle.c -- CPU restatement of the reference transform path
 * (NotoriousLOB/FastAndFourier, split-plane FP32), written from scratch.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py load this library, and only as the checker.
 * The product library (fastandfourier_b200/libfaf_b200.so) never links,
 * loads or calls it.
 *
 * Pinned against: the reference itself, compiled from its sources by
 * oracle/Makefile (oracle/_ref), through the golden fixtures under
 * tests/golden/ (made by tests/golden/gen_golden.py) and the reference's
 * own known-answer tests restated in tests/test_oracle.py.
 *
 * Every routine cites the reference code it restates.  Arithmetic is FP32
 * like the reference's FP32 path; twiddles follow the reference's generation
 * precision (float angles for the mixed-radix table, double angles for the
 * split-radix and codelet tables), so the restatement tracks the reference
 * to ~1e-7 relative L2.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* ---- error reporting --------------------------------------------------- */
static char g_orc_err[256];
const char *orc_error(void) { return g_orc_err; }
static int orc_fail(const char *msg) {
    snprintf(g_orc_err, sizeof g_orc_err, "%s", msg);
    return -1;
}

/* ---- size arithmetic: src/faf_fft_stage.c:25-135 ------------------------ */
static size_t strip(size_t n, size_t p) { while (n % p == 0) n /= p; return n; }

int orc_is_5_smooth(size_t n) {                     /* faf_fft_stage.c:25 */
    return n != 0 && strip(strip(strip(n, 2), 3), 5) == 1;
}
int orc_is_7_smooth(size_t n) {                     /* faf_fft_stage.c:33 */
    return n != 0 && strip(strip(strip(strip(n, 2), 3), 5), 7) == 1;
}
int orc_is_prime(size_t n) {                        /* faf_fft_stage.c:42 */
    if (n < 2) return 0;
    if (n % 2 == 0) return n == 2;
    for (size_t d = 3; d * d <= n; d += 2)
        if (n % d == 0) return 0;
    return 1;
}
int orc_rader_eligible(size_t n) {                  /* faf_fft_stage.c:50 */
    return n >= 11 && orc_is_prime(n) && orc_is_7_smooth(n - 1);
}
int orc_is_codelet(size_t n) {                      /* faf_fft_kernels.c:196 */
    return (n >= 2 && n <= 10) || n == 12;
}
static uint64_t powmod(uint64_t b, uint64_t e, uint64_t m) {
    uint64_t r = 1;
    b %= m;
    while (e) { if (e & 1) r = r * b % m; b = b * b % m; e >>= 1; }
    return r;
}
size_t orc_primitive_root(size_t p) {               /* faf_fft_stage.c:65 */
    if (!orc_is_prime(p) || p < 3) return 0;
    size_t phi = p - 1, m = phi, pf[16];
    int npf = 0;
    for (size_t d = 2; d * d <= m; d++)
        if (m % d == 0) { pf[npf++] = d; while (m % d == 0) m /= d; }
    if (m > 1) pf[npf++] = m;
    for (size_t g = 2; g < p; g++) {
        int ok = 1;
        for (int i = 0; i < npf && ok; i++)
            if (powmod(g, phi / pf[i], p) == 1) ok = 0;
        if (ok) return g;
    }
    return 0;
}
/* Factor order 4s, then 2, 3, 5, 7 (faf_fft_stage.c:95-105). */
static int factor7(size_t n, int *f) {
    int k = 0;
    while (n % 4 == 0) { f[k++] = 4; n /= 4; }
    while (n % 2 == 0) { f[k++] = 2; n /= 2; }
    while (n % 3 == 0) { f[k++] = 3; n /= 3; }
    while (n % 5 == 0) { f[k++] = 5; n /= 5; }
    while (n % 7 == 0) { f[k++] = 7; n /= 7; }
    return n == 1 ? k : -1;
}
size_t orc_next_5_smooth(size_t m) {               /* faf_fft_stage.c:121 */
    if (m <= 1) return 1;
    while (!orc_is_5_smooth(m)) m++;
    return m;
}

/* ---- codelets: direct DFT, src/faf_fft_kernels.c:206-226 ---------------- */
static void dft_direct(float *re, float *im, size_t n, int inverse) {
    float xr[16], xi[16], wr[16], wi[16];
    double s = inverse ? 1.0 : -1.0;
    for (size_t t = 0; t < n; t++) {
        xr[t] = re[t]; xi[t] = im[t];
        double a = s * 2.0 * M_PI * (double)t / (double)n;
        wr[t] = (float)cos(a); wi[t] = (float)sin(a);
    }
    for (size_t k = 0; k < n; k++) {
        float ar = 0.f, ai = 0.f;
        for (size_t t = 0; t < n; t++) {
            size_t e = (k * t) % n;
            ar += xr[t] * wr[e] - xi[t] * wi[e];
            ai += xr[t] * wi[e] + xi[t] * wr[e];
        }
        re[k] = ar; im[k] = ai;
    }
}

/* ---- split-radix DIF for power-of-two n >= 16 --------------------------
 * src/faf_fft_splitradix.c:237-369 (L-shaped butterfly, recursion into n/2,
 * n/4, n/4, output natural order via strides), twiddles in double angles
 * cast to float (faf_fft_splitradix.c:30-43). Leaves n <= 8 use the direct
 * DFT here; the reference's unrolled n=2/4/8 codelets are exact re-orderings
 * of the same sums. */
static void sr_dif(size_t n, const float *xr, const float *xi, float *tr, float *ti,
                   float *yr, float *yi, size_t sy, int inverse) {
    if (n <= 8) {
        float br[8], bi[8];
        for (size_t i = 0; i < n; i++) { br[i] = xr[i]; bi[i] = xi[i]; }
        if (n > 1) dft_direct(br, bi, n, inverse);
        for (size_t i = 0; i < n; i++) { yr[i * sy] = br[i]; yi[i * sy] = bi[i]; }
        return;
    }
    size_t n2 = n / 2, n4 = n / 4;
    double s = inverse ? 1.0 : -1.0;
    for (size_t k = 0; k < n4; k++) {
        float x0r = xr[k], x0i = xi[k];
        float x1r = xr[k + n2], x1i = xi[k + n2];
        float x2r = xr[k + n4], x2i = xi[k + n4];
        float x3r = xr[k + 3 * n4], x3i = xi[k + 3 * n4];
        double ang = s * 2.0 * M_PI * (double)k / (double)n;
        float w1r = (float)cos(ang), w1i = (float)sin(ang);
        float w3r = (float)cos(3.0 * ang), w3i = (float)sin(3.0 * ang);
        float sr0 = x0r + x1r, si0 = x0i + x1i;
        float sr1 = x2r + x3r, si1 = x2i + x3i;
        float dr0 = x0r - x1r, di0 = x0i - x1i;
        float dr1 = x2r - x3r, di1 = x2i - x3i;
        /* j*d1 forward, -j*d1 inverse */
        float jr = inverse ? di1 : -di1, ji = inverse ? -dr1 : dr1;
        tr[k] = sr0; ti[k] = si0;
        tr[k + n4] = sr1; ti[k + n4] = si1;
        float ur = dr0 - jr, ui = di0 - ji;
        tr[k + n2] = ur * w1r - ui * w1i;
        ti[k + n2] = ur * w1i + ui * w1r;
        float vr = dr0 + jr, vi = di0 + ji;
        tr[k + 3 * n4] = vr * w3r - vi * w3i;
        ti[k + 3 * n4] = vr * w3i + vi * w3r;
    }
    sr_dif(n2, tr, ti, tr, ti, yr, yi, 2 * sy, inverse);
    sr_dif(n4, tr + n2, ti + n2, tr + n2, ti + n2, yr + sy, yi + sy, 4 * sy, inverse);
    sr_dif(n4, tr + 3 * n4, ti + 3 * n4, tr + 3 * n4, ti + 3 * n4,
           yr + 3 * sy, yi + 3 * sy, 4 * sy, inverse);
}

/* ---- mixed radix: digit-reversed load + DIT stages ----------------------
 * Plan: src/faf_transforms.c:147-187 (LOAD reg[i] = x[digitrev(i)], one
 * FFT_STAGE(group, radix, n/group) per factor, STORE).  Stage kernels:
 * src/faf_fft_stage.c:163-374 (radix-2/3/4/5/7 split-plane DIT; twiddle
 * index j*q*tw_step into a length-n table).  Twiddle table with float
 * angles: src/faf_twiddles.c:43-51. */
static int mixed_radix(size_t n, const float *xr, const float *xi, float *yr, float *yi,
                       int inverse) {
    int f[64];
    int nf = factor7(n, f);
    if (nf < 0) return -1;
    float *tw = (float *)malloc(2 * n * sizeof(float));
    float *ar = (float *)malloc(n * sizeof(float));
    float *ai = (float *)malloc(n * sizeof(float));
    if (!tw || !ar || !ai) { free(tw); free(ar); free(ai); return -1; }
    const float sg = inverse ? 1.0f : -1.0f;
    const float step = 2.0f * (float)M_PI / (float)n;
    for (size_t k = 0; k < n; k++) {
        float a = sg * step * (float)k;
        tw[2 * k] = cosf(a); tw[2 * k + 1] = sinf(a);
    }
    /* digit reversal with the factor order (faf_fft_stage.c:107-116) */
    for (size_t i = 0; i < n; i++) {
        size_t v = i, r = 0;
        for (int k = 0; k < nf; k++) { r = r * (size_t)f[k] + v % (size_t)f[k]; v /= (size_t)f[k]; }
        ar[i] = xr[r]; ai[i] = xi[r];
    }
    size_t group = 1;
    double s = inverse ? 1.0 : -1.0;
    for (int st = 0; st < nf; st++) {
        size_t R = (size_t)f[st];
        group *= R;
        size_t m = group / R, tw_step = n / group;
        /* radix-R DFT constants (double angles, like the reference's
         * C2PI5/S2PI5-style constants) */
        float cr[8], ci[8];
        for (size_t e = 0; e < R; e++) {
            double a = s * 2.0 * M_PI * (double)e / (double)R;
            cr[e] = (float)cos(a); ci[e] = (float)sin(a);
        }
        for (size_t base = 0; base < n; base += group) {
            for (size_t j = 0; j < m; j++) {
                float vr[8], vi[8];
                for (size_t q = 0; q < R; q++) {
                    size_t ix = base + j + q * m;
                    float r = ar[ix], im = ai[ix];
                    if (q > 0) {
                        size_t t = j * q * tw_step;
                        float wr = tw[2 * t], wi = tw[2 * t + 1];
                        float rr = r * wr - im * wi;
                        im = r * wi + im * wr;
                        r = rr;
                    }
                    vr[q] = r; vi[q] = im;
                }
                for (size_t k = 0; k < R; k++) {
                    float sr = 0.f, si = 0.f;
                    for (size_t q = 0; q < R; q++) {
                        size_t e = (k * q) % R;
                        sr += vr[q] * cr[e] - vi[q] * ci[e];
                        si += vr[q] * ci[e] + vi[q] * cr[e];
                    }
                    ar[base + j + k * m] = sr;
                    ai[base + j + k * m] = si;
                }
            }
        }
    }
    memcpy(yr, ar, n * sizeof(float));
    memcpy(yi, ai, n * sizeof(float));
    free(tw); free(ar); free(ai);
    return 0;
}

/* Unscaled C2C of a 5-smooth / codelet / (allow7) 7-smooth size, dispatched
 * the way faf_create_fft_ex picks a kernel (src/faf_core.c:645-717). */
static int c2c_core(size_t n, int inverse, const float *xr, const float *xi,
                    float *yr, float *yi) {
    if (n == 1) { yr[0] = xr[0]; yi[0] = xi[0]; return 0; }
    if (orc_is_codelet(n)) {
        float br[16], bi[16];
        for (size_t i = 0; i < n; i++) { br[i] = xr[i]; bi[i] = xi[i]; }
        dft_direct(br, bi, n, inverse);
        memcpy(yr, br, n * sizeof(float));
        memcpy(yi, bi, n * sizeof(float));
        return 0;
    }
    if ((n & (n - 1)) == 0) {
        float *t = (float *)malloc(2 * n * sizeof(float));
        float *cr = (float *)malloc(2 * n * sizeof(float));
        if (!t || !cr) { free(t); free(cr); return -1; }
        memcpy(cr, xr, n * sizeof(float));
        memcpy(cr + n, xi, n * sizeof(float));
        sr_dif(n, cr, cr + n, t, t + n, yr, yi, 1, inverse);
        free(t); free(cr);
        return 0;
    }
    return mixed_radix(n, xr, xi, yr, yi, inverse);
}

/* ---- Rader: src/faf_fft_rader.c:19-232 ---------------------------------- */
static int rader(size_t p, int inverse, const float *xr, const float *xi, float *yr, float *yi) {
    size_t m = p - 1, g = orc_primitive_root(p);
    if (!g) return orc_fail("rader: no primitive root");
    size_t ginv = (size_t)powmod(g, p - 2, p);
    size_t *rin = (size_t *)malloc(2 * m * sizeof(size_t));
    float *br = (float *)malloc(4 * m * sizeof(float));
    if (!rin || !br) { free(rin); free(br); return -1; }
    size_t *rout = rin + m;
    float *bi = br + m, *ar = bi + m, *ai = ar + m;
    size_t a = 1, b = 1;
    for (size_t j = 0; j < m; j++) {                 /* rader.c:77-83 */
        rin[j] = a; rout[j] = b;
        a = a * g % p; b = b * ginv % p;
    }
    double s = inverse ? 1.0 : -1.0;
    for (size_t j = 0; j < m; j++) {                 /* rader.c:109-130 */
        double ang = s * 2.0 * M_PI * (double)rout[j] / (double)p;
        br[j] = (float)cos(ang); bi[j] = (float)sin(ang);
    }
    if (c2c_core(m, 0, br, bi, br, bi) != 0) { free(rin); free(br); return -1; }
    float dcr = 0.f, dci = 0.f;                      /* rader.c:201-231 */
    for (size_t i = 0; i < p; i++) { dcr += xr[i]; dci += xi[i]; }
    for (size_t j = 0; j < m; j++) { ar[j] = xr[rin[j]]; ai[j] = xi[rin[j]]; }
    if (c2c_core(m, 0, ar, ai, ar, ai) != 0) { free(rin); free(br); return -1; }
    for (size_t j = 0; j < m; j++) {
        float r = ar[j], i = ai[j];
        ar[j] = r * br[j] - i * bi[j];
        ai[j] = r * bi[j] + i * br[j];
    }
    if (c2c_core(m, 1, ar, ai, ar, ai) != 0) { free(rin); free(br); return -1; }
    float x0r = xr[0], x0i = xi[0], sc = 1.0f / (float)m;
    yr[0] = dcr; yi[0] = dci;
    for (size_t j = 0; j < m; j++) {
        yr[rout[j]] = x0r + ar[j] * sc;
        yi[rout[j]] = x0i + ai[j] * sc;
    }
    free(rin); free(br);
    return 0;
}

/* ---- Bluestein: src/faf_bluestein.c:19-223 ------------------------------ */
static int bluestein(size_t n, int inverse, const float *xr, const float *xi,
                     float *yr, float *yi) {
    size_t M = orc_next_5_smooth(2 * n - 1);
    float *buf = (float *)calloc(6 * M + 2 * n, sizeof(float));
    if (!buf) return -1;
    float *pr = buf, *pi = pr + n;                    /* chirp phi */
    float *Br = pi + n, *Bi = Br + M, *ar = Bi + M, *ai = ar + M, *Ar = ai + M, *Ai = Ar + M;
    double s = inverse ? 1.0 : -1.0;
    for (size_t k = 0; k < n; k++) {                 /* bluestein.c:38-45 */
        double ang = s * M_PI * ((double)k * (double)k) / (double)n;
        pr[k] = (float)cos(ang); pi[k] = (float)sin(ang);
    }
    ar[0] = 1.0f;                                     /* bluestein.c:112-126 */
    for (size_t l = 1; l < n; l++) {
        ar[l] = pr[l]; ai[l] = -pi[l];
        ar[M - l] = pr[l]; ai[M - l] = -pi[l];
    }
    int rc = c2c_core(M, 0, ar, ai, Br, Bi);
    for (size_t k = 0; k < M; k++) { ar[k] = 0.f; ai[k] = 0.f; }
    for (size_t k = 0; k < n && rc == 0; k++) {      /* bluestein.c:182-195 */
        ar[k] = xr[k] * pr[k] - xi[k] * pi[k];
        ai[k] = xr[k] * pi[k] + xi[k] * pr[k];
    }
    if (rc == 0) rc = c2c_core(M, 0, ar, ai, Ar, Ai);
    for (size_t k = 0; k < M && rc == 0; k++) {
        float r = Ar[k], i = Ai[k];
        Ar[k] = r * Br[k] - i * Bi[k];
        Ai[k] = r * Bi[k] + i * Br[k];
    }
    if (rc == 0) rc = c2c_core(M, 1, Ar, Ai, ar, ai);
    /* the inner inverse goes through faf_execute with NORM_NONE: 1/M */
    float sM = (float)(1.0 / (double)M);
    for (size_t k = 0; k < n && rc == 0; k++) {
        float r = ar[k] * sM, i = ai[k] * sM;
        yr[k] = r * pr[k] - i * pi[k];
        yi[k] = r * pi[k] + i * pr[k];
    }
    free(buf);
    return rc;
}

/* ---- norms: src/faf_core.c:1251-1279 (scale as float) ------------------- */
enum { NORM_DEFAULT = 0, NORM_NONE = 1, NORM_ORTHO = 2, NORM_FORWARD = 3 };
static float norm_scale(int norm, int inverse, size_t n) {
    switch (norm) {
    case NORM_ORTHO: return (float)(1.0 / sqrt((double)n));
    case NORM_FORWARD: return inverse ? 1.0f : (float)(1.0 / (double)n);
    default: return inverse ? (float)(1.0 / (double)n) : 1.0f;
    }
}
static void scale2(float *a, float *b, size_t n, float s) {
    if (s == 1.0f) return;
    for (size_t i = 0; i < n; i++) { a[i] *= s; if (b) b[i] *= s; }
}

#define ORC_FLAG_BLUESTEIN (1u << 12)

/* Public C2C (faf_create_fft + faf_execute on SPLIT buffers). */
int orc_c2c(size_t n, int inverse, int norm, uint32_t flags, const float *xr, const float *xi,
            float *yr, float *yi) {
    int rc;
    if (n == 0) return orc_fail("n must be > 0");
    float *tr = (float *)malloc(2 * n * sizeof(float));
    if (!tr) return -1;
    float *ti = tr + n;
    if (orc_is_5_smooth(n) || orc_is_codelet(n)) rc = c2c_core(n, inverse, xr, xi, tr, ti);
    else if (orc_rader_eligible(n)) rc = rader(n, inverse, xr, xi, tr, ti);
    else if (flags & ORC_FLAG_BLUESTEIN) rc = bluestein(n, inverse, xr, xi, tr, ti);
    else rc = orc_fail("size not supported without FAF_FLAG_BLUESTEIN");
    if (rc == 0) {
        scale2(tr, ti, n, norm_scale(norm, inverse, n));
        memcpy(yr, tr, n * sizeof(float));
        memcpy(yi, ti, n * sizeof(float));
    }
    free(tr);
    return rc;
}

int orc_c2c_batch(size_t n, int inverse, int norm, uint32_t flags, size_t batch,
                  const float *xr, const float *xi, float *yr, float *yi) {
    for (size_t b = 0; b < batch; b++)
        if (orc_c2c(n, inverse, norm, flags, xr + b * n, xi + b * n, yr + b * n, yi + b * n))
            return -1;
    return 0;
}

/* ---- real FFT: src/faf_rfft.c:37-146,337-397 ---------------------------- */
static void super_twiddles(float *tw, size_t nc, int inverse) {   /* rfft.c:37 */
    for (size_t i = 0; i < nc / 2; i++) {
        double ph = -M_PI * (((double)(i + 1) / (double)nc) + 0.5);
        if (inverse) ph = -ph;
        tw[2 * i] = (float)cos(ph); tw[2 * i + 1] = (float)sin(ph);
    }
}

int orc_r2c(size_t n, int norm, const float *x, float *Xr, float *Xi) {
    if (n < 2 || (n & 1) || !orc_is_5_smooth(n)) return orc_fail("R2C size must be even 5-smooth");
    size_t nc = n / 2;
    float *buf = (float *)malloc((4 * nc + nc) * sizeof(float) + 64);
    if (!buf) return -1;
    float *zr = buf, *zi = zr + nc, *fr = zi + nc, *fi = fr + nc, *stw = fi + nc;
    for (size_t k = 0; k < nc; k++) { zr[k] = x[2 * k]; zi[k] = x[2 * k + 1]; }
    if (c2c_core(nc, 0, zr, zi, fr, fi) != 0) { free(buf); return -1; }
    super_twiddles(stw, nc, 0);
    /* rfft_post_f32, rfft.c:61-89 */
    Xr[0] = fr[0] + fi[0]; Xi[0] = 0.f;
    Xr[nc] = fr[0] - fi[0]; Xi[nc] = 0.f;
    for (size_t k = 1; k <= nc / 2; k++) {
        float ar = fr[k], ai = fi[k], br = fr[nc - k], bi = -fi[nc - k];
        float s_r = ar + br, s_i = ai + bi, d_r = ar - br, d_i = ai - bi;
        float wr = stw[2 * (k - 1)], wi = stw[2 * (k - 1) + 1];
        float tr = d_r * wr - d_i * wi, ti = d_r * wi + d_i * wr;
        Xr[k] = 0.5f * (s_r + tr); Xi[k] = 0.5f * (s_i + ti);
        Xr[nc - k] = 0.5f * (s_r - tr); Xi[nc - k] = 0.5f * (ti - s_i);
    }
    scale2(Xr, Xi, nc + 1, norm_scale(norm, 0, n));
    free(buf);
    return 0;
}

int orc_c2r(size_t n, int norm, const float *Xr, const float *Xi, float *y) {
    if (n < 2 || (n & 1) || !orc_is_5_smooth(n)) return orc_fail("R2C size must be even 5-smooth");
    size_t nc = n / 2;
    float *buf = (float *)malloc((4 * nc + nc) * sizeof(float) + 64);
    if (!buf) return -1;
    float *fr = buf, *fi = fr + nc, *zr = fi + nc, *zi = zr + nc, *stw = zi + nc;
    super_twiddles(stw, nc, 1);
    /* irfft_pre_f32, rfft.c:122-146 */
    fr[0] = Xr[0] + Xr[nc];
    fi[0] = Xr[0] - Xr[nc];
    for (size_t k = 1; k <= nc / 2; k++) {
        float ar = Xr[k], ai = Xi[k], br = Xr[nc - k], bi = -Xi[nc - k];
        float er = ar + br, ei = ai + bi, dr = ar - br, di = ai - bi;
        float wr = stw[2 * (k - 1)], wi = stw[2 * (k - 1) + 1];
        float orr = dr * wr - di * wi, oi = dr * wi + di * wr;
        fr[k] = er + orr; fi[k] = ei + oi;
        fr[nc - k] = er - orr; fi[nc - k] = -(ei - oi);
    }
    if (c2c_core(nc, 1, fr, fi, zr, zi) != 0) { free(buf); return -1; }
    for (size_t k = 0; k < nc; k++) { y[2 * k] = zr[k]; y[2 * k + 1] = zi[k]; }
    float s = norm_scale(norm, 1, n);
    if (s != 1.0f) for (size_t i = 0; i < n; i++) y[i] *= s;
    free(buf);
    return 0;
}

int orc_r2c_batch(size_t n, int norm, size_t batch, const float *x, float *Xr, float *Xi) {
    size_t nb = n / 2 + 1;
    for (size_t b = 0; b < batch; b++)
        if (orc_r2c(n, norm, x + b * n, Xr + b * nb, Xi + b * nb)) return -1;
    return 0;
}

int orc_c2r_batch(size_t n, int norm, size_t batch, const float *Xr, const float *Xi, float *y) {
    size_t nb = n / 2 + 1;
    for (size_t b = 0; b < batch; b++)
        if (orc_c2r(n, norm, Xr + b * nb, Xi + b * nb, y + b * n)) return -1;
    return 0;
}

/* ---- pipeline ops: src/chirp.c:421-471, src/faf_core.c:150-166 ---------- */
enum { OP_CONJ = 1, OP_MUL = 2, OP_BANDPASS = 3, OP_MUL_CONJ = 4 };

static void herm_mul(float *re, float *im, const float *hr, const float *hi, size_t nb,
                     int conj_h) {
    if (nb == 0) return;
    re[0] = re[0] * hr[0]; im[0] = 0.f;
    for (size_t k = 1; k + 1 < nb; k++) {
        float ar = re[k], ai = im[k], br = hr[k], bi = conj_h ? -hi[k] : hi[k];
        re[k] = ar * br - ai * bi;
        im[k] = ar * bi + ai * br;
    }
    if (nb > 1) { re[nb - 1] *= hr[nb - 1]; im[nb - 1] = 0.f; }
}

/* Apply one spectral op to n_bins split-plane bins.  MUL uses the first
 * min(h_bins, n_bins) bins and treats bin min-1 as the real edge, exactly
 * as chirp_apply_split_f32 passes m = min(user_aux_n, n) to faf_herm_mul. */
void orc_apply_op(int op, uint32_t lo, uint32_t hi, const float *hr, const float *hi_,
                  size_t h_bins, float *re, float *im, size_t n_bins) {
    if (op == OP_CONJ) {
        for (size_t i = 0; i < n_bins; i++) im[i] = -im[i];
    } else if (op == OP_MUL || op == OP_MUL_CONJ) {
        if (!hr || !hi_) return;
        size_t m = h_bins < n_bins ? h_bins : n_bins;
        herm_mul(re, im, hr, hi_, m, op == OP_MUL_CONJ);
    } else if (op == OP_BANDPASS) {
        for (size_t i = 0; i < n_bins; i++)
            if (i < lo || i > hi) { re[i] = 0.f; im[i] = 0.f; }
    }
}

/* Fused pipeline (src/faf_pipeline.c:10-90): R2C with the forward norm, the
 * ops in order, C2R with the inverse norm (both norms from `norm`). */
int orc_pipeline(size_t n, int norm, int n_ops, const int *ops, const uint32_t *lo,
                 const uint32_t *hi, const float *hr, const float *hi_, size_t h_bins,
                 size_t batch, const float *x, float *y) {
    size_t nb = n / 2 + 1;
    float *sr = (float *)malloc(2 * nb * sizeof(float));
    if (!sr) return -1;
    float *si = sr + nb;
    for (size_t b = 0; b < batch; b++) {
        if (orc_r2c(n, norm, x + b * n, sr, si)) { free(sr); return -1; }
        for (int k = 0; k < n_ops; k++)
            orc_apply_op(ops[k], lo ? lo[k] : 0, hi ? hi[k] : 0, hr, hi_, h_bins, sr, si, nb);
        if (orc_c2r(n, norm, sr, si, y + b * n)) { free(sr); return -1; }
    }
    free(sr);
    return 0;
}

/* ---- STFT framing ------------------------------------------------------
 * The reference's STFT transform keeps a Hann window (src/faf_core.c:994-
 * 1032, window src/faf_twiddles.c:159-163) but never frames by hop and skips
 * the window on SPLIT buffers.  This is the intended behaviour restated:
 * frame f of signal s is x[s*L + f*hop + i] * w[i] (i < win, zero-padded to
 * n), transformed by the reference R2C of n.  Output [s][f][n/2+1]. */
void orc_hann(float *w, size_t n) {
    for (size_t i = 0; i < n; i++)
        w[i] = 0.5f * (1.0f - cosf(2.0f * (float)M_PI * (float)i / (float)(n - 1)));
}

int orc_stft(size_t n, size_t win, size_t hop, size_t L, size_t n_sig, const float *x,
             float *Xr, float *Xi) {
    if (win == 0 || win > n || hop == 0 || L < win) return orc_fail("stft: bad framing");
    size_t F = 1 + (L - win) / hop, nb = n / 2 + 1;
    float *w = (float *)malloc((win + n) * sizeof(float));
    if (!w) return -1;
    float *fr = w + win;
    orc_hann(w, win);
    for (size_t s = 0; s < n_sig; s++) {
        for (size_t f = 0; f < F; f++) {
            const float *src = x + s * L + f * hop;
            memset(fr, 0, n * sizeof(float));
            for (size_t i = 0; i < win; i++) fr[i] = src[i] * w[i];
            size_t o = (s * F + f) * nb;
            if (orc_r2c(n, NORM_NONE, fr, Xr + o, Xi + o)) { free(w); return -1; }
        }
    }
    free(w);
    return 0;
}
