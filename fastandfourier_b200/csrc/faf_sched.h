// faf_sched.h -- host-side admission policy of the serving loop
// (faf_serve.cpp): a first-fit device-memory arena, the scheduler that
// turns a FIFO of pending requests into batches for free stream slots, and
// the router that spreads requests over several GPUs' loops.
//
// Pure C++17, no CUDA: the same code runs inside the library and in the CPU
// unit test (tests/native/sched_check.cpp), which drives it with synthetic
// requests.
//
// Policy (continuous batching):
//   - Requests are admitted in arrival order.  The head of the queue starts a
//     batch; later pending requests with the same plan key join it (merged
//     into one batched launch) while the batch stays under `max_merge`
//     requests and its memory fits the arena.  Mergeable means: same plan key
//     and the request allows merging (streamed STFT chunks do not).
//   - A request whose stream key has a batch in flight waits (chunks of one
//     stream run in order), and so does every request behind it that shares
//     its stream key; other requests may pass it.
//   - A batch needs a free slot (CUDA stream) and arena memory for all its
//     requests.  When the head does not fit, admission stops until memory is
//     released (no starvation of large requests by small ones).
//   - A request larger than the whole arena is rejected at submit time.
#pragma once

#include <stddef.h>
#include <stdint.h>

#include <deque>
#include <map>
#include <set>
#include <vector>

namespace fafs {

// First-fit allocator over [0, capacity) with coalescing of free blocks.
class Arena {
   public:
    static constexpr size_t kAlign = 256;
    explicit Arena(size_t capacity = 0) { reset(capacity); }
    void reset(size_t capacity) {
        cap_ = capacity & ~(kAlign - 1);
        free_.clear();
        used_.clear();
        in_use_ = peak_ = 0;
        if (cap_) free_[0] = cap_;
    }
    static size_t round(size_t b) { return (b + kAlign - 1) & ~(kAlign - 1); }
    // Offset of a block of `bytes`, or SIZE_MAX when no free block is large
    // enough.  Zero-byte requests get a distinct minimum block.
    size_t alloc(size_t bytes) {
        const size_t need = round(bytes ? bytes : 1);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < need) continue;
            const size_t off = it->first, len = it->second;
            free_.erase(it);
            if (len > need) free_[off + need] = len - need;
            used_[off] = need;
            in_use_ += need;
            if (in_use_ > peak_) peak_ = in_use_;
            return off;
        }
        return SIZE_MAX;
    }
    // Release a block returned by alloc; false if `off` is not a live block.
    bool release(size_t off) {
        auto u = used_.find(off);
        if (u == used_.end()) return false;
        size_t start = off, len = u->second;
        used_.erase(u);
        in_use_ -= len;
        auto nx = free_.lower_bound(start);
        if (nx != free_.end() && nx->first == start + len) {
            len += nx->second;
            nx = free_.erase(nx);
        }
        if (nx != free_.begin()) {
            auto pv = std::prev(nx);
            if (pv->first + pv->second == start) {
                start = pv->first;
                len += pv->second;
                free_.erase(pv);
            }
        }
        free_[start] = len;
        return true;
    }
    size_t capacity() const { return cap_; }
    size_t in_use() const { return in_use_; }
    size_t peak() const { return peak_; }
    size_t largest_free() const {
        size_t m = 0;
        for (auto& kv : free_) m = kv.second > m ? kv.second : m;
        return m;
    }
    size_t live_blocks() const { return used_.size(); }

   private:
    size_t cap_ = 0, in_use_ = 0, peak_ = 0;
    std::map<size_t, size_t> free_;  // offset -> length
    std::map<size_t, size_t> used_;  // offset -> length
};

struct SchedReq {
    long long id = 0;
    uint64_t plan_key = 0;    // requests with equal keys may share a launch
    uint64_t stream_key = 0;  // nonzero: ordered stream, never merged
    bool mergeable = true;
    size_t bytes = 0;         // arena bytes this request needs while in flight
};

struct Batch {
    int slot = -1;
    size_t offset = 0;  // arena block holding every request of the batch
    size_t bytes = 0;
    uint64_t stream_key = 0;
    std::vector<SchedReq> reqs;
};

class Scheduler {
   public:
    Scheduler(size_t arena_bytes, int slots, int max_merge)
        : arena_(arena_bytes), max_merge_(max_merge < 1 ? 1 : max_merge) {
        for (int s = slots - 1; s >= 0; s--) free_slots_.push_back(s);
    }
    // False when the request can never fit the arena.
    bool fits_ever(size_t bytes) const { return Arena::round(bytes) <= arena_.capacity(); }
    void submit(const SchedReq& r) { pending_.push_back(r); }
    size_t pending() const { return pending_.size(); }
    int free_slots() const { return (int)free_slots_.size(); }
    const Arena& arena() const { return arena_; }

    // Admit as many batches as slots and memory allow, in arrival order.
    std::vector<Batch> admit() {
        std::vector<Batch> out;
        Batch b;
        while (admit_one(&b)) out.push_back(std::move(b));
        return out;
    }

    // Admit the next batch (true), or report that none can start now.
    bool admit_one(Batch* out) {
        if (free_slots_.empty() || pending_.empty()) return false;
        // head: first request whose stream is idle (and that no earlier
        // waiting request of the same stream precedes)
        std::set<uint64_t> blocked;
        size_t h = SIZE_MAX;
        for (size_t i = 0; i < pending_.size(); i++) {
            const uint64_t sk = pending_[i].stream_key;
            if (sk && (busy_streams_.count(sk) || blocked.count(sk))) {
                blocked.insert(sk);
                continue;
            }
            h = i;
            break;
        }
        if (h == SIZE_MAX) return false;
        Batch b;
        b.stream_key = pending_[h].stream_key;
        std::vector<size_t> take{h};
        size_t bytes = Arena::round(pending_[h].bytes);
        if (pending_[h].mergeable && !pending_[h].stream_key) {
            for (size_t i = h + 1; i < pending_.size() && (int)take.size() < max_merge_; i++) {
                const SchedReq& r = pending_[i];
                if (!r.mergeable || r.stream_key || r.plan_key != pending_[h].plan_key) continue;
                const size_t nb = bytes + Arena::round(r.bytes);
                if (nb > arena_.largest_free()) break;
                take.push_back(i);
                bytes = nb;
            }
        }
        size_t off = arena_.alloc(bytes);
        if (off == SIZE_MAX) {
            if (take.size() == 1) return false;  // head waits for memory
            take.resize(1);                       // retry with the head alone
            bytes = Arena::round(pending_[h].bytes);
            off = arena_.alloc(bytes);
            if (off == SIZE_MAX) return false;
        }
        b.offset = off;
        b.bytes = bytes;
        b.slot = free_slots_.back();
        free_slots_.pop_back();
        for (size_t k = take.size(); k-- > 0;) {
            b.reqs.insert(b.reqs.begin(), pending_[take[k]]);
            pending_.erase(pending_.begin() + (long)take[k]);
        }
        if (b.stream_key) busy_streams_.insert(b.stream_key);
        merged_ += b.reqs.size() > 1 ? (long long)b.reqs.size() : 0;
        batches_++;
        *out = std::move(b);
        return true;
    }

    // A batch finished on the device: release its memory, slot and stream.
    void complete(const Batch& b) {
        arena_.release(b.offset);
        free_slots_.push_back(b.slot);
        if (b.stream_key) busy_streams_.erase(b.stream_key);
    }

    // Long-lived blocks outside any batch (e.g. a stream's STFT overlap).
    size_t reserve(size_t bytes) { return arena_.alloc(bytes); }
    void unreserve(size_t off) { arena_.release(off); }

    long long batches() const { return batches_; }
    void reset_counters() { batches_ = merged_ = 0; }
    long long merged_requests() const { return merged_; }

   private:
    Arena arena_;
    int max_merge_;
    std::deque<SchedReq> pending_;
    std::vector<int> free_slots_;
    std::set<uint64_t> busy_streams_;
    long long batches_ = 0, merged_ = 0;
};

// Request routing over several GPUs, each with its own serving loop and
// arena (one process per GPU, or one Scheduler per device): the policy a
// front end applies before submitting to a GPU's queue.
//   - Requests of an ordered stream (stream_key != 0) go to the GPU that
//     took the stream's first chunk: its overlap state lives there.
//   - Other requests go to the GPU with the fewest bytes in flight (routed
//     and not yet completed) among those whose arena can ever hold them;
//     ties go to the lower index.
//   - A request no GPU's arena can hold is rejected (-1).
class Router {
   public:
    explicit Router(const std::vector<size_t>& arena_bytes) : cap_(arena_bytes) {
        load_.assign(cap_.size(), 0);
        routed_.assign(cap_.size(), 0);
    }
    int devices() const { return (int)cap_.size(); }
    // The GPU for request r, or -1; its bytes count as in flight there.
    int route(const SchedReq& r) {
        const size_t need = Arena::round(r.bytes);
        if (r.stream_key) {
            auto it = stream_dev_.find(r.stream_key);
            if (it != stream_dev_.end()) {
                if (need > cap_[it->second]) return -1;
                take(it->second, need);
                return it->second;
            }
        }
        int best = -1;
        for (int d = 0; d < (int)cap_.size(); d++) {
            if (need > cap_[d]) continue;
            if (best < 0 || load_[d] < load_[best]) best = d;
        }
        if (best < 0) return -1;
        if (r.stream_key) stream_dev_[r.stream_key] = best;
        take(best, need);
        return best;
    }
    // A routed request finished on GPU d.
    void complete(int d, size_t bytes) {
        const size_t b = Arena::round(bytes);
        load_[d] = load_[d] > b ? load_[d] - b : 0;
    }
    // The stream's last chunk finished: later chunks may go anywhere.
    void end_stream(uint64_t stream_key) { stream_dev_.erase(stream_key); }
    size_t in_flight(int d) const { return load_[d]; }
    long long routed(int d) const { return routed_[d]; }

   private:
    void take(int d, size_t need) {
        load_[d] += need;
        routed_[d]++;
    }
    std::vector<size_t> cap_, load_;
    std::vector<long long> routed_;
    std::map<uint64_t, int> stream_dev_;
};

}  // namespace fafs
