// CPU unit test of the serving loop's admission policy (faf_sched.h):
// arena allocation, FIFO admission, merging, the memory budget and the
// ordering of streamed requests.  Built and run by tests/test_serve_host.py.
#include <stdio.h>
#include <stdlib.h>

#include <map>
#include <random>
#include <vector>

#include "faf_sched.h"

static int failures = 0;
#define CHECK(c)                                                      \
    do {                                                              \
        if (!(c)) {                                                   \
            fprintf(stderr, "%s:%d: CHECK(%s) failed\n", __FILE__, __LINE__, #c); \
            failures++;                                               \
        }                                                             \
    } while (0)

using fafs::Arena;
using fafs::Batch;
using fafs::Scheduler;
using fafs::SchedReq;

static SchedReq R(long long id, uint64_t key, size_t bytes, uint64_t stream = 0) {
    SchedReq r;
    r.id = id;
    r.plan_key = key;
    r.bytes = bytes;
    r.stream_key = stream;
    r.mergeable = stream == 0;
    return r;
}

static void test_arena() {
    Arena a(4096);
    const size_t x = a.alloc(1000), y = a.alloc(1000), z = a.alloc(1000);
    CHECK(x == 0 && y == 1024 && z == 2048);
    CHECK(a.in_use() == 3072 && a.largest_free() == 1024);
    CHECK(a.alloc(2000) == SIZE_MAX);
    CHECK(a.release(y));
    CHECK(!a.release(y));
    CHECK(!a.release(12345));
    CHECK(a.alloc(1024) == 1024);  // first fit reuses the hole
    CHECK(a.release(1024) && a.release(x) && a.release(z));
    CHECK(a.in_use() == 0 && a.largest_free() == 4096 && a.live_blocks() == 0);
    CHECK(a.peak() == 3072);
    CHECK(a.alloc(0) != SIZE_MAX);  // zero bytes still get a block
}

static void test_fifo_slots() {
    Scheduler s(1 << 20, 2, 8);
    s.submit(R(1, 10, 100));
    s.submit(R(2, 20, 100));
    s.submit(R(3, 30, 100));
    std::vector<Batch> b = s.admit();
    CHECK(b.size() == 2);
    CHECK(b[0].reqs.size() == 1 && b[0].reqs[0].id == 1);
    CHECK(b[1].reqs.size() == 1 && b[1].reqs[0].id == 2);
    CHECK(s.pending() == 1 && s.free_slots() == 0);
    CHECK(s.admit().empty());
    s.complete(b[0]);
    std::vector<Batch> c = s.admit();
    CHECK(c.size() == 1 && c[0].reqs[0].id == 3);
}

static void test_merge() {
    Scheduler s(1 << 20, 1, 3);
    for (int i = 1; i <= 5; i++) s.submit(R(i, 7, 1000));
    s.submit(R(6, 8, 1000));
    std::vector<Batch> b = s.admit();
    CHECK(b.size() == 1 && b[0].reqs.size() == 3);
    CHECK(b[0].reqs[0].id == 1 && b[0].reqs[1].id == 2 && b[0].reqs[2].id == 3);
    s.complete(b[0]);
    b = s.admit();
    CHECK(b.size() == 1 && b[0].reqs.size() == 2 && b[0].reqs[0].id == 4);
    s.complete(b[0]);
    b = s.admit();
    CHECK(b.size() == 1 && b[0].reqs.size() == 1 && b[0].reqs[0].id == 6);
    CHECK(s.merged_requests() == 5 && s.batches() == 3);
}

static void test_budget() {
    Scheduler s(1 << 20, 4, 8);  // 1 MiB
    for (int i = 1; i <= 3; i++) s.submit(R(i, 7, 400 << 10));
    std::vector<Batch> b = s.admit();
    CHECK(b.size() == 1 && b[0].reqs.size() == 2);  // 800 KiB; the third waits
    CHECK(s.pending() == 1 && s.arena().in_use() <= s.arena().capacity());
    CHECK(s.admit().empty());
    s.complete(b[0]);
    b = s.admit();
    CHECK(b.size() == 1 && b[0].reqs[0].id == 3);
    CHECK(!s.fits_ever((1 << 20) + 1) && s.fits_ever(1 << 20));
}

static void test_head_blocks() {
    Scheduler s(1 << 20, 4, 8);
    s.submit(R(1, 1, 300 << 10));
    std::vector<Batch> a = s.admit();
    CHECK(a.size() == 1);
    s.submit(R(2, 2, 900 << 10));  // does not fit next to request 1
    s.submit(R(3, 3, 10 << 10));   // would fit, but may not pass the head
    CHECK(s.admit().empty());
    s.complete(a[0]);
    std::vector<Batch> b = s.admit();
    CHECK(b.size() == 2 && b[0].reqs[0].id == 2 && b[1].reqs[0].id == 3);
}

static void test_streams() {
    Scheduler s(1 << 20, 4, 8);
    s.submit(R(1, 5, 100, 77));
    s.submit(R(2, 5, 100, 77));
    s.submit(R(3, 5, 100, 0));
    s.submit(R(4, 5, 100, 0));
    std::vector<Batch> b = s.admit();
    // chunk 1 of stream 77 alone; chunk 2 waits; 3 and 4 merge
    CHECK(b.size() == 2);
    CHECK(b[0].reqs.size() == 1 && b[0].reqs[0].id == 1);
    CHECK(b[1].reqs.size() == 2 && b[1].reqs[0].id == 3 && b[1].reqs[1].id == 4);
    CHECK(s.pending() == 1);
    s.complete(b[1]);
    CHECK(s.admit().empty());
    s.complete(b[0]);
    b = s.admit();
    CHECK(b.size() == 1 && b[0].reqs[0].id == 2);
    const size_t r = s.reserve(1000);
    CHECK(r != SIZE_MAX);
    s.unreserve(r);
}

// Random submissions and completions: every request is admitted exactly
// once, memory never exceeds the budget, chunks of a stream run in order.
static void test_fuzz() {
    std::mt19937 rng(1234);
    Scheduler s(4 << 20, 3, 4);
    std::vector<Batch> running;
    std::map<long long, int> admitted;
    std::map<uint64_t, long long> last_chunk;
    std::map<long long, uint64_t> stream_of;
    long long next = 1;
    for (int step = 0; step < 20000; step++) {
        const int op = (int)(rng() % 3);
        if (op == 0 && next < 5000) {
            const uint64_t stream = rng() % 4 == 0 ? 1 + rng() % 3 : 0;
            SchedReq q = R(next, 1 + rng() % 3, 1 + rng() % (1 << 20), stream);
            stream_of[next] = stream;
            s.submit(q);
            next++;
        } else if (op == 1 && !running.empty()) {
            const size_t k = rng() % running.size();
            s.complete(running[k]);
            running.erase(running.begin() + (long)k);
        }
        for (Batch& b : s.admit()) {
            CHECK(s.arena().in_use() <= s.arena().capacity());
            for (const SchedReq& q : b.reqs) {
                admitted[q.id]++;
                if (q.stream_key) {
                    CHECK(b.reqs.size() == 1);
                    CHECK(q.id > last_chunk[q.stream_key]);
                    last_chunk[q.stream_key] = q.id;
                }
            }
            running.push_back(b);
        }
    }
    while (!running.empty() || s.pending()) {
        for (Batch& b : running) s.complete(b);
        running.clear();
        for (Batch& b : s.admit()) {
            for (const SchedReq& q : b.reqs) admitted[q.id]++;
            running.push_back(b);
        }
    }
    for (long long id = 1; id < next; id++) CHECK(admitted[id] == 1);
    CHECK(s.arena().in_use() == 0);
}

// Router: stream affinity, least bytes in flight, capacity, completion.
static void test_router() {
    using fafs::Router;
    Router rt({1 << 20, 1 << 20, 1 << 16});
    // three equal requests spread over the three GPUs, lowest index first
    CHECK(rt.route(R(1, 7, 4096)) == 0);
    CHECK(rt.route(R(2, 7, 4096)) == 1);
    CHECK(rt.route(R(3, 7, 4096)) == 2);
    // a request larger than GPU 2's arena skips it
    CHECK(rt.route(R(4, 7, 100000)) == 0);
    CHECK(rt.route(R(5, 7, 4096)) == 1);
    CHECK(rt.route(R(6, 7, 4096)) == 2);
    // nothing can hold 2 MB
    CHECK(rt.route(R(7, 7, 2 << 20)) == -1);
    // a stream sticks to the GPU of its first chunk, whatever the load
    // (GPUs 1 and 2 tie at 8192 bytes in flight: the lower index)
    const int d = rt.route(R(8, 9, 256, 55));
    CHECK(d == 1);
    for (int k = 0; k < 5; k++) CHECK(rt.route(R(9 + k, 9, 256, 55)) == d);
    // completions lower the load and steer new requests back
    rt.complete(0, 100000);
    rt.complete(0, 4096);
    CHECK(rt.in_flight(0) == 0);
    CHECK(rt.route(R(20, 7, 4096)) == 0);
    rt.end_stream(55);
    CHECK(rt.routed(0) + rt.routed(1) + rt.routed(2) == 13);  // one was rejected
    // balance: many random requests keep the loads within one request
    Router b({1ull << 30, 1ull << 30, 1ull << 30, 1ull << 30});
    std::mt19937 g(3);
    size_t biggest = 0;
    for (int i = 0; i < 4000; i++) {
        const size_t sz = 256 + g() % (1 << 20);
        biggest = sz > biggest ? sz : biggest;
        CHECK(b.route(R(100 + i, g() % 5, sz)) >= 0);
    }
    size_t lo = SIZE_MAX, hi = 0;
    for (int k = 0; k < 4; k++) {
        lo = b.in_flight(k) < lo ? b.in_flight(k) : lo;
        hi = b.in_flight(k) > hi ? b.in_flight(k) : hi;
    }
    CHECK(hi - lo <= Arena::round(biggest));
}

int main() {
    test_arena();
    test_router();
    test_fifo_slots();
    test_merge();
    test_budget();
    test_head_blocks();
    test_streams();
    test_fuzz();
    if (failures) {
        fprintf(stderr, "%d check(s) failed\n", failures);
        return 1;
    }
    printf("OK\n");
    return 0;
}
