/*
 * ref_driver.c -- batched, multi-threaded driver around the UNMODIFIED
 * reference library (NotoriousLOB/FastAndFourier), compiled from its own
 * sources by oracle/Makefile into oracle/_ref/libfaf_ref_<isa>.so.
 *
 * TEST / BASELINE INFRASTRUCTURE ONLY.  This file is linked into the
 * reference build, never into the product library.  It is used by
 *   - tests/golden/gen_golden.py   (golden fixtures from the reference),
 *   - tests/ (validating the C restatement in oracle/faf_oracle.c),
 *   - bench.py --impl reference / cpu_baseline (timing the reference on the
 *     host cores).
 *
 * The reference transforms are not re-entrant (per-transform scratch,
 * include/fastandfourier.h:490 `scratch`; src/faf_fft_splitradix.c:523 uses
 * twiddles[1] as recursion work), so every worker thread creates its own
 * transform objects and runs a contiguous slice of the batch through the
 * reference's public faf_execute (include/fastandfourier.h:950).
 *
 * Timing follows the reference's own benchmarks (plan once, execute in a
 * loop: benchmarks/benchmark_throughput.cpp:34-39): a session
 * (refdrv_open_*) starts its worker threads, creates their transforms and
 * runs one warm-up execute on each, and refdrv_session_run then times
 * nothing but faf_execute calls.
 */
#define _GNU_SOURCE
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "fastandfourier.h"
#include "chirp.h"

/* Internal reference symbol (src/faf_twiddles.c:159), declared in faf.h. */
void faf_gen_hann_window_f32(float *win, size_t n);

static char g_drv_err[512];

const char *refdrv_error(void) { return g_drv_err; }

static void drv_fail(const char *what) {
    snprintf(g_drv_err, sizeof(g_drv_err), "%s: %s", what, faf_get_error());
}

typedef enum { JOB_C2C, JOB_R2C, JOB_C2R, JOB_PIPE, JOB_STFT, JOB_CWT, JOB_ICWT } job_kind;

typedef struct {
    job_kind kind;
    size_t n;          /* transform length (FFT size for STFT) */
    int inverse;
    int norm;
    uint32_t flags;
    const char *src;   /* Chirp source (pipeline) */
    const float *h_re, *h_im;
    size_t h_bins;
    size_t win, hop, sig_len, frames; /* STFT framing */
    size_t rows;       /* CWT: rows of the default bank (output row length n) */
    size_t b0, b1;     /* batch slice [b0, b1) */
    const float *in_re, *in_im;
    float *out_re, *out_im;
    int f64;           /* C2C: buffers hold doubles, transform in FAF_PREC_FP64 */
    int rc;
} job;

static faf_transform *make_transform(const job *j) {
    faf_config c = faf_config_init(j->n);
    c.norm = (faf_norm)j->norm;
    c.flags = j->flags;
    switch (j->kind) {
    case JOB_C2C:
        c.layout = FAF_LAYOUT_SPLIT;
        c.dir = j->inverse ? FAF_DIR_INVERSE : FAF_DIR_FORWARD;
        if (j->f64) c.precision = FAF_PREC_FP64;
        return faf_create_fft(&c);
    case JOB_R2C:
    case JOB_STFT:
        c.dir = FAF_DIR_FORWARD;
        return faf_create_rfft(&c);
    case JOB_C2R:
        c.dir = FAF_DIR_INVERSE;
        return faf_create_rfft(&c);
    case JOB_CWT: {
        /* The reference's default bank (Morse 20/3, L1, 10 voices, lowpass). */
        faf_cwt_config cc = faf_cwt_config_init(j->n);
        return faf_create_cwt(&cc);
    }
    case JOB_ICWT: {
        faf_cwt_config cc = faf_cwt_config_init(j->n);
        return faf_create_icwt(&cc, (faf_cwt_inverse_kind)j->inverse);
    }
    case JOB_PIPE: {
        faf_transform *t = chirp_compile(j->src);
        if (t && j->h_re) {
            if (chirp_bind(t, "H", (void *)j->h_re, (void *)j->h_im, j->h_bins) != 0) {
                faf_destroy_transform(t);
                return NULL;
            }
        }
        return t;
    }
    }
    return NULL;
}

/* Per-thread state of a session: the thread's own transform and, for the
 * STFT, its frame and window buffers. */
typedef struct {
    faf_transform *t;
    float *frame, *win;
} worker_state;

/* Creation is serialised: chirp_compile reads the reference's global,
 * unlocked registry (src/chirp.c:39-41). */
static pthread_mutex_t g_create_mu = PTHREAD_MUTEX_INITIALIZER;

static int worker_setup(const job *j, worker_state *w) {
    memset(w, 0, sizeof(*w));
    pthread_mutex_lock(&g_create_mu);
    w->t = make_transform(j);
    pthread_mutex_unlock(&g_create_mu);
    if (!w->t) { drv_fail("create"); return -1; }
    if (j->kind == JOB_STFT) {
        w->frame = (float *)calloc(j->n, sizeof(float));
        w->win = (float *)calloc(j->win, sizeof(float));
        if (!w->frame || !w->win) return -1;
        /* Reference symmetric Hann, src/faf_twiddles.c:159-163. */
        faf_gen_hann_window_f32(w->win, j->win);
    }
    return 0;
}

static void worker_teardown(worker_state *w) {
    free(w->frame);
    free(w->win);
    if (w->t) faf_destroy_transform(w->t);
    memset(w, 0, sizeof(*w));
}

/* Run transforms [j->b0, j->b1) of the job's buffers through the worker's
 * transform with the reference's public faf_execute. */
static int worker_slice(const job *j, worker_state *w) {
    faf_transform *t = w->t;
    size_t n = j->n, nb = n / 2 + 1;
    for (size_t b = j->b0; b < j->b1; b++) {
        faf_buffer in, out;
        int rc = 0;
        switch (j->kind) {
        case JOB_C2C: {
            const size_t o = b * n * (j->f64 ? 2 : 1);  /* in floats */
            in = faf_buffer_split((void *)(j->in_re + o), (void *)(j->in_im + o), n);
            out = faf_buffer_split(j->out_re + o, j->out_im + o, n);
            rc = faf_execute(t, &out, &in);
            break;
        }
        case JOB_R2C:
            in = faf_buffer_real((void *)(j->in_re + b * n), n);
            out = faf_buffer_hermitian(j->out_re + b * nb, j->out_im + b * nb, nb);
            rc = faf_execute(t, &out, &in);
            break;
        case JOB_C2R:
            in = faf_buffer_hermitian((void *)(j->in_re + b * nb), (void *)(j->in_im + b * nb), nb);
            out = faf_buffer_real(j->out_re + b * n, n);
            rc = faf_execute(t, &out, &in);
            break;
        case JOB_PIPE:
            in = faf_buffer_real((void *)(j->in_re + b * n), n);
            out = faf_buffer_real(j->out_re + b * n, n);
            rc = faf_execute(t, &out, &in);
            break;
        case JOB_CWT:
            in = faf_buffer_real((void *)(j->in_re + b * n), n);
            out = faf_buffer_real(j->out_re + b * j->rows * n, j->rows * n);
            rc = faf_execute(t, &out, &in);
            break;
        case JOB_ICWT:
            in = faf_buffer_real((void *)(j->in_re + b * j->rows * n), j->rows * n);
            out = faf_buffer_real(j->out_re + b * n, n);
            rc = faf_execute(t, &out, &in);
            break;
        case JOB_STFT: {
            /* Signal b / frames, frame b % frames: x[sig*L + f*hop + i] * w[i]
             * for i < win, zero-padded to n, then the reference R2C of n. */
            size_t sig = b / j->frames, f = b % j->frames;
            const float *x = j->in_re + sig * j->sig_len + f * j->hop;
            for (size_t i = 0; i < j->win; i++) w->frame[i] = x[i] * w->win[i];
            in = faf_buffer_real(w->frame, n);
            out = faf_buffer_hermitian(j->out_re + b * nb, j->out_im + b * nb, nb);
            rc = faf_execute(t, &out, &in);
            break;
        }
        }
        if (rc != 0) { drv_fail("execute"); return -1; }
    }
    return 0;
}

/* One transform of zeros through the worker's transform, so one-time work
 * that the reference does on the first execute (the pipeline JIT compiles
 * its trampoline with gcc then, src/jit/faf_jit.c:1156-1202) happens before
 * any timed run. */
static int worker_warm(const job *proto, worker_state *w) {
    size_t n = proto->n, nb = n / 2 + 1, el = proto->f64 ? 2 : 1;
    size_t in_len = n, out_len = n;
    switch (proto->kind) {
    case JOB_C2C: in_len = out_len = n * el; break;
    case JOB_R2C: out_len = nb; break;
    case JOB_C2R: in_len = nb; break;
    case JOB_PIPE: break;
    case JOB_CWT: out_len = proto->rows * n; break;
    case JOB_ICWT: in_len = proto->rows * n; break;
    case JOB_STFT: in_len = proto->win; out_len = nb; break;
    }
    float *a = (float *)calloc(2 * in_len + 2 * out_len, sizeof(float));
    if (!a) return -1;
    job j = *proto;
    j.in_re = a; j.in_im = a + in_len;
    j.out_re = a + 2 * in_len; j.out_im = a + 2 * in_len + out_len;
    j.b0 = 0; j.b1 = 1;
    if (j.kind == JOB_STFT) { j.frames = 1; j.sig_len = j.win; }
    int rc = worker_slice(&j, w);
    free(a);
    return rc;
}

/*
 * A session: `nthreads` persistent worker threads, each holding its own
 * transform (the reference's transforms are not re-entrant), created and
 * warmed once when the session opens.  refdrv_session_run() hands every
 * worker a contiguous slice of the batch and waits for all of them, so a
 * timed run contains faf_execute calls and nothing else: no thread start,
 * no create, no JIT compile.
 */
typedef struct refdrv_session {
    job proto;
    int nthreads;
    pthread_t *th;
    job *jobs;
    worker_state *ws;
    pthread_mutex_t mu;
    pthread_cond_t go, done;
    unsigned long gen;   /* incremented per run (and once to quit) */
    int pending;         /* workers still running the current generation */
    int quit;
    int ready;           /* workers that finished setup */
    int setup_failed;
} refdrv_session;

typedef struct { refdrv_session *s; int id; } worker_arg;

static void *worker_main(void *arg) {
    worker_arg *wa = (worker_arg *)arg;
    refdrv_session *s = wa->s;
    const int id = wa->id;
    free(wa);
    int rc = worker_setup(&s->proto, &s->ws[id]);
    if (rc == 0) rc = worker_warm(&s->proto, &s->ws[id]);
    pthread_mutex_lock(&s->mu);
    if (rc != 0) s->setup_failed = 1;
    s->ready++;
    pthread_cond_broadcast(&s->done);
    unsigned long seen = 0;
    for (;;) {
        while (s->gen == seen) pthread_cond_wait(&s->go, &s->mu);
        seen = s->gen;
        if (s->quit) break;
        pthread_mutex_unlock(&s->mu);
        job *j = &s->jobs[id];
        j->rc = (j->b0 < j->b1) ? worker_slice(j, &s->ws[id]) : 0;
        pthread_mutex_lock(&s->mu);
        if (--s->pending == 0) pthread_cond_broadcast(&s->done);
    }
    pthread_mutex_unlock(&s->mu);
    worker_teardown(&s->ws[id]);
    return NULL;
}

void refdrv_session_close(refdrv_session *s);

static refdrv_session *session_open(const job *proto, int nthreads) {
    if (nthreads < 1) nthreads = 1;
    refdrv_session *s = (refdrv_session *)calloc(1, sizeof(*s));
    if (!s) return NULL;
    s->proto = *proto;
    s->nthreads = nthreads;
    s->th = (pthread_t *)calloc((size_t)nthreads, sizeof(pthread_t));
    s->jobs = (job *)calloc((size_t)nthreads, sizeof(job));
    s->ws = (worker_state *)calloc((size_t)nthreads, sizeof(worker_state));
    pthread_mutex_init(&s->mu, NULL);
    pthread_cond_init(&s->go, NULL);
    pthread_cond_init(&s->done, NULL);
    if (!s->th || !s->jobs || !s->ws) { free(s->th); free(s->jobs); free(s->ws); free(s); return NULL; }
    int started = 0;
    for (int i = 0; i < nthreads; i++) {
        worker_arg *wa = (worker_arg *)malloc(sizeof(worker_arg));
        if (!wa) break;
        wa->s = s; wa->id = i;
        if (pthread_create(&s->th[i], NULL, worker_main, wa) != 0) { free(wa); break; }
        started++;
    }
    pthread_mutex_lock(&s->mu);
    while (s->ready < started) pthread_cond_wait(&s->done, &s->mu);
    const int failed = s->setup_failed || started < nthreads;
    pthread_mutex_unlock(&s->mu);
    s->nthreads = started;
    if (failed) { refdrv_session_close(s); return NULL; }
    return s;
}

/* Run `batch` transforms of the given buffers (layout as for the one-shot
 * calls below) on the session's workers; 0 on success. */
int refdrv_session_run(refdrv_session *s, size_t batch, const void *in_re, const void *in_im,
                       void *out_re, void *out_im) {
    if (!s) return -1;
    const size_t nth = (size_t)s->nthreads;
    size_t per = batch / nth, rem = batch % nth, at = 0;
    pthread_mutex_lock(&s->mu);
    for (size_t i = 0; i < nth; i++) {
        job *j = &s->jobs[i];
        *j = s->proto;
        j->in_re = (const float *)in_re; j->in_im = (const float *)in_im;
        j->out_re = (float *)out_re; j->out_im = (float *)out_im;
        j->b0 = at;
        at += per + (i < rem ? 1 : 0);
        j->b1 = at;
        j->rc = 0;
    }
    s->pending = s->nthreads;
    s->gen++;
    pthread_cond_broadcast(&s->go);
    while (s->pending > 0) pthread_cond_wait(&s->done, &s->mu);
    pthread_mutex_unlock(&s->mu);
    int rc = 0;
    for (size_t i = 0; i < nth; i++) if (s->jobs[i].rc != 0) rc = -1;
    return rc;
}

int refdrv_session_threads(const refdrv_session *s) { return s ? s->nthreads : 0; }

void refdrv_session_close(refdrv_session *s) {
    if (!s) return;
    pthread_mutex_lock(&s->mu);
    s->quit = 1;
    s->gen++;
    pthread_cond_broadcast(&s->go);
    pthread_mutex_unlock(&s->mu);
    for (int i = 0; i < s->nthreads; i++) pthread_join(s->th[i], NULL);
    pthread_mutex_destroy(&s->mu);
    pthread_cond_destroy(&s->go);
    pthread_cond_destroy(&s->done);
    free(s->th);
    free(s->jobs);
    free(s->ws);
    free(s);
}

static int run_batched(const job *proto, size_t batch, int nthreads) {
    if ((size_t)nthreads > batch) nthreads = (int)(batch ? batch : 1);
    refdrv_session *s = session_open(proto, nthreads);
    if (!s) return -1;
    int rc = refdrv_session_run(s, batch, proto->in_re, proto->in_im, proto->out_re, proto->out_im);
    refdrv_session_close(s);
    return rc;
}

/* Session constructors: the same parameters as the one-shot calls below,
 * without the buffers and the batch. */
refdrv_session *refdrv_open_c2c(size_t n, int inverse, int norm, uint32_t flags, int f64,
                                int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_C2C; j.n = n; j.inverse = inverse; j.norm = norm; j.flags = flags; j.f64 = f64;
    return session_open(&j, nthreads);
}

refdrv_session *refdrv_open_r2c(size_t n, int norm, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_R2C; j.n = n; j.norm = norm;
    return session_open(&j, nthreads);
}

refdrv_session *refdrv_open_pipeline(const char *src, size_t n, const float *h_re,
                                     const float *h_im, size_t h_bins, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_PIPE; j.n = n; j.src = src;
    j.h_re = h_re; j.h_im = h_im; j.h_bins = h_bins;
    return session_open(&j, nthreads);
}

/* STFT sessions run batches counted in frames: batch = n_sig * frames. */
refdrv_session *refdrv_open_stft(size_t n, size_t win, size_t hop, size_t sig_len,
                                 int nthreads) {
    if (win == 0 || win > n || hop == 0 || sig_len < win) {
        snprintf(g_drv_err, sizeof(g_drv_err), "stft: bad framing");
        return NULL;
    }
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_STFT; j.n = n; j.norm = FAF_NORM_NONE;
    j.win = win; j.hop = hop; j.sig_len = sig_len;
    j.frames = 1 + (sig_len - win) / hop;
    return session_open(&j, nthreads);
}

int refdrv_cwt_bank(size_t n, size_t *n_rows, size_t *n_bins, int *has_lowpass, float *psi);

refdrv_session *refdrv_open_cwt(size_t n, int nthreads) {
    size_t rows = 0;
    if (refdrv_cwt_bank(n, &rows, NULL, NULL, NULL) != 0) return NULL;
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_CWT; j.n = n; j.rows = rows;
    return session_open(&j, nthreads);
}

refdrv_session *refdrv_open_icwt(size_t n, int kind, int nthreads) {
    size_t rows = 0;
    if (refdrv_cwt_bank(n, &rows, NULL, NULL, NULL) != 0) return NULL;
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_ICWT; j.n = n; j.rows = rows; j.inverse = kind;
    return session_open(&j, nthreads);
}

int refdrv_c2c(size_t n, int inverse, int norm, uint32_t flags, size_t batch,
               const float *in_re, const float *in_im, float *out_re, float *out_im,
               int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_C2C; j.n = n; j.inverse = inverse; j.norm = norm; j.flags = flags;
    j.in_re = in_re; j.in_im = in_im; j.out_re = out_re; j.out_im = out_im;
    return run_batched(&j, batch, nthreads);
}

/* The same in FP64 (double buffers, FAF_PREC_FP64 transforms). */
int refdrv_c2c64(size_t n, int inverse, int norm, size_t batch, const double *in_re,
                 const double *in_im, double *out_re, double *out_im, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_C2C; j.n = n; j.inverse = inverse; j.norm = norm; j.f64 = 1;
    j.in_re = (const float *)in_re; j.in_im = (const float *)in_im;
    j.out_re = (float *)out_re; j.out_im = (float *)out_im;
    return run_batched(&j, batch, nthreads);
}

int refdrv_r2c(size_t n, int norm, size_t batch, const float *x,
               float *out_re, float *out_im, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_R2C; j.n = n; j.norm = norm;
    j.in_re = x; j.out_re = out_re; j.out_im = out_im;
    return run_batched(&j, batch, nthreads);
}

int refdrv_c2r(size_t n, int norm, size_t batch, const float *in_re, const float *in_im,
               float *y, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_C2R; j.n = n; j.norm = norm; j.inverse = 1;
    j.in_re = in_re; j.in_im = in_im; j.out_re = y;
    return run_batched(&j, batch, nthreads);
}

int refdrv_pipeline(const char *src, size_t n, const float *h_re, const float *h_im,
                    size_t h_bins, size_t batch, const float *x, float *y, int nthreads) {
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_PIPE; j.n = n; j.src = src;
    j.h_re = h_re; j.h_im = h_im; j.h_bins = h_bins;
    j.in_re = x; j.out_re = y;
    return run_batched(&j, batch, nthreads);
}

/* Framed real STFT over n_sig signals of sig_len samples each; output is
 * [n_sig][frames][n/2+1] split planes, frames = 1 + (sig_len - win) / hop. */
int refdrv_stft(size_t n, size_t win, size_t hop, size_t sig_len, size_t n_sig,
                const float *x, float *out_re, float *out_im, int nthreads) {
    if (win == 0 || win > n || hop == 0 || sig_len < win) {
        snprintf(g_drv_err, sizeof(g_drv_err), "stft: bad framing");
        return -1;
    }
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_STFT; j.n = n; j.norm = FAF_NORM_NONE;
    j.win = win; j.hop = hop; j.sig_len = sig_len;
    j.frames = 1 + (sig_len - win) / hop;
    j.in_re = x; j.out_re = out_re; j.out_im = out_im;
    return run_batched(&j, n_sig * j.frames, nthreads);
}

/* The reference's default CWT bank for length n (faf_cwt_config_init +
 * faf_create_cwt, src/faf_cwt.c:27-56,702-726): its row count, packed bin
 * count and lowpass flag, and, when psi is non-NULL, its rows in execute
 * order (row 0 = lowpass phi if present, then wavelets coarse -> fine), each
 * n/2+1 floats, copied from faf_cwt_phi_f32 / faf_cwt_psi_f32. */
int refdrv_cwt_bank(size_t n, size_t *n_rows, size_t *n_bins, int *has_lowpass, float *psi) {
    faf_cwt_config cc = faf_cwt_config_init(n);
    faf_transform *t = faf_create_cwt(&cc);
    if (!t) { drv_fail("cwt create"); return -1; }
    const size_t rows = faf_cwt_n_rows(t), nb = faf_cwt_n_bins(t);
    const int lp = faf_cwt_has_lowpass(t);
    if (n_rows) *n_rows = rows;
    if (n_bins) *n_bins = nb;
    if (has_lowpass) *has_lowpass = lp;
    if (psi) {
        size_t r = 0;
        if (lp) memcpy(psi + (r++) * nb, faf_cwt_phi_f32(t), nb * sizeof(float));
        for (size_t j = 0; j < faf_cwt_n_scales(t); j++)
            memcpy(psi + (r++) * nb, faf_cwt_psi_f32(t, j), nb * sizeof(float));
    }
    faf_destroy_transform(t);
    return 0;
}

/* The default bank's inverse constants: admissibility C from its report
 * (faf_cwt_bank_report, include/fastandfourier.h:785) and voices per octave. */
int refdrv_cwt_consts(size_t n, double *C, unsigned *voices) {
    faf_cwt_config cc = faf_cwt_config_init(n);
    faf_transform *t = faf_create_cwt(&cc);
    if (!t) { drv_fail("cwt create"); return -1; }
    const faf_cwt_lp_report *r = faf_cwt_bank_report(t);
    if (C) *C = r ? r->admissibility_C : 0.0;
    if (voices) *voices = cc.voices;
    faf_destroy_transform(t);
    return 0;
}

/* Inverse CWT (kind: FAF_CWT_INV_DUAL or FAF_CWT_INV_L1) of `batch`
 * coefficient sets W [batch][rows][n] -> x [batch][n], default bank. */
int refdrv_icwt(size_t n, int kind, size_t batch, const float *W, float *x, int nthreads) {
    size_t rows = 0;
    if (refdrv_cwt_bank(n, &rows, NULL, NULL, NULL) != 0) return -1;
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_ICWT; j.n = n; j.rows = rows; j.inverse = kind;
    j.in_re = W; j.out_re = x;
    return run_batched(&j, batch, nthreads);
}

/* Forward CWT of `batch` signals with the default bank; W is
 * [batch][rows][n] (src/faf_cwt.c:769-847 per signal). */
int refdrv_cwt(size_t n, size_t batch, const float *x, float *W, int nthreads) {
    size_t rows = 0;
    if (refdrv_cwt_bank(n, &rows, NULL, NULL, NULL) != 0) return -1;
    job j;
    memset(&j, 0, sizeof(j));
    j.kind = JOB_CWT; j.n = n; j.rows = rows;
    j.in_re = x; j.out_re = W;
    return run_batched(&j, batch, nthreads);
}

/* Reference size policy, exposed for the parity tests of the planner. */
int refdrv_is_size_supported(int type, size_t n) {
    return faf_is_size_supported((faf_transform_type)type, n) ? 1 : 0;
}

size_t refdrv_recommended_size(int type, size_t n) {
    return faf_get_recommended_size((faf_transform_type)type, n);
}

/* Create a C2C/R2C transform and report whether creation succeeded (for the
 * create-time error tests); the message is copied into msg. */
int refdrv_try_create(int type, size_t n, uint32_t flags, int layout, char *msg, size_t cap) {
    faf_config c = faf_config_init(n);
    c.flags = flags;
    c.layout = (faf_layout)layout;
    faf_clear_error();
    faf_transform *t = faf_create((faf_transform_type)type, &c);
    if (msg && cap) snprintf(msg, cap, "%s", faf_get_error());
    if (!t) return 0;
    faf_destroy_transform(t);
    return 1;
}
