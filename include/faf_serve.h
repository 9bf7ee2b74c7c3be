/*
 * faf_serve.h -- serving loop for the B200 transform path (no counterpart in
 * the reference, which has no request loop: its callers loop over faf_execute
 * themselves, e.g. benchmarks/benchmark_throughput.cpp:34-39).
 *
 * A faf_server accepts requests -- Chirp-compiled real transforms and
 * pipelines ("(rfft :size N)", "(pipeline (rfft :size N) ... (irfft))") and
 * framed STFTs -- from any host thread, and runs them on one GPU with
 * continuous batching:
 *
 *   - a dispatcher thread admits pending requests in arrival order as stream
 *     slots and device memory free up, so requests that arrive while others
 *     are on the GPU join at once and their work overlaps on the device;
 *   - pending requests with the same plan are merged into one batched launch;
 *   - every in-flight request's input and output live in one device arena of
 *     `hbm_budget` bytes, allocated at create; a request is admitted only when
 *     its bytes fit, and one that can never fit is rejected at submit;
 *   - plans and their twiddle tables stay on the device (one set per slot,
 *     keyed by the Chirp source / STFT geometry), and streamed STFT requests
 *     (same nonzero `stream_key`) keep their frame overlap on the device, so
 *     chunk after chunk yields the frames of the whole stream;
 *   - latency is measured per request from submit to the completion of its
 *     output copy, and the stats report p50 / p99 and throughput.
 *
 * Inputs and outputs may be host or device memory (cudaMemcpyDefault); the
 * caller keeps them valid until the request completes.  A bound spectrum H
 * (`h_re` / `h_im`, for "(mul-spectrum)") must be device memory.
 */
#ifndef FAF_SERVE_H
#define FAF_SERVE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct faf_server faf_server;

typedef struct {
    size_t hbm_budget; /* arena bytes for in-flight requests (0: 16 GiB) */
    int streams;       /* concurrent stream slots (0: 8) */
    int max_merge;     /* most requests merged into one launch (0: 64; 1: no merging) */
} faf_server_config;

typedef struct {
    /* plan: a Chirp source (real transform or pipeline), or, when NULL, a
     * framed STFT with FFT size stft_n, window stft_win, hop stft_hop */
    const char *chirp;
    size_t stft_n, stft_win, stft_hop;
    /* bound spectrum for (mul-spectrum): device memory, h_len bins */
    const float *h_re, *h_im;
    size_t h_len;
    /* input: in_len real samples; for transforms / pipelines a whole number
     * of transforms of size N, run as one batch */
    const float *in;
    size_t in_len;
    /* output: rfft -> Hermitian re / im, (in_len / N) x (N/2+1) each;
     * pipeline -> out_re, in_len reals; STFT -> frames x (n/2+1) re / im */
    float *out_re, *out_im;
    /* STFT only: nonzero = one chunk of a continuing stream (never merged;
     * chunks of a stream run in submit order) */
    unsigned long long stream_key;
} faf_request;

typedef struct {
    long long completed;
    long long failed;
    long long batches;         /* launches of merged or single requests */
    long long merged_requests; /* requests that shared a launch */
    double p50_latency_s;
    double p99_latency_s;
    double mean_latency_s;
    double max_latency_s;
    double wall_s;             /* first submit -> last completion */
    double requests_per_s;
    double bytes_per_s;        /* algorithmic bytes (input + output) / wall_s */
    size_t arena_bytes;
    size_t arena_peak_bytes;
} faf_server_stats;

faf_server *faf_server_create(const faf_server_config *cfg);
/* Queue a request; returns its id (> 0) or -1 (message in faf_get_error()). */
long long faf_server_submit(faf_server *s, const faf_request *r);
/* Block until request `id` completes; its latency and, for STFT, its frame
 * count.  0 on success, -1 if the request failed or is unknown. */
int faf_server_wait(faf_server *s, long long id, double *latency_s, size_t *frames);
/* Block until every submitted request has completed; 0, or -1 if any failed. */
int faf_server_drain(faf_server *s);
/* Frames the next chunk of `in_len` samples of STFT stream `key` will yield
 * (the overlap carried from earlier chunks counts). */
size_t faf_server_stream_frames(faf_server *s, unsigned long long key, size_t win, size_t hop,
                                size_t in_len);
/* Forget the overlap of stream `key` (after its last chunk has completed). */
int faf_server_close_stream(faf_server *s, unsigned long long key);
/* Create the plans of `r` on every slot ahead of time (plan creation
 * allocates device memory, which synchronises the device). */
int faf_server_prepare(faf_server *s, const faf_request *r);
int faf_server_stats_get(faf_server *s, faf_server_stats *st);
void faf_server_stats_reset(faf_server *s);
/* Load generator: submit reqs[i] at arrival_s[i] seconds after the call from
 * a client thread, wait for all, store each latency (may be NULL). */
int faf_server_replay(faf_server *s, const faf_request *reqs, const double *arrival_s, size_t n,
                      double *latency_s);
void faf_server_destroy(faf_server *s);

#ifdef __cplusplus
}
#endif

#endif /* FAF_SERVE_H */
