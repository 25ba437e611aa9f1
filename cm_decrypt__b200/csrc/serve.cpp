// Serving loop: continuous batching of decapsulation requests for many keys
// and parameter sets on one GPU.
//
//  * Requests (key id, ciphertext, output buffer, tag) enter a bounded queue;
//    a full queue refuses with CMD_E_BUSY.
//  * A dispatcher thread owns `slots` batch slots, each with its own CUDA
//    stream, pinned staging and device buffers.  Whenever a slot is free and
//    requests are waiting it forms a batch of up to max_batch of them -- at
//    once if nothing is on the GPU, otherwise after batch-mates have had at most
//    max_wait_us to arrive -- so requests that arrive while other batches run
//    are admitted as soon as a slot frees, and the batches overlap on the
//    device (copies and kernels of different slots run concurrently).
//  * Expanded keys stay resident in HBM; a key is expanded on first use and
//    the least recently used keys that no batch in flight uses are evicted
//    when the engine's HBM budget is full (admission by budget).  Every batch
//    stamps the keys it made resident with its generation; a key is in use
//    while a batch of that generation or later is in flight.
//  * Small batches run the latency kernels of latency.cu (any mix of keys and
//    sets in three launches, a short pass per ciphertext); batches of
//    fused_threshold or more run the fused kernel (highest throughput).
//  * A completer thread watches the batches in flight without the queue lock
//    (each batch's stream copies its sequence number to a pinned word after
//    the results, so the watch is plain loads, not CUDA calls), takes
//    whichever finishes first, copies each result to its request's
//    buffer (large batches split across a few copy threads) and records
//    arrival-to-completion latency for the p50/p99 statistics.  A buffer in
//    memory registered with cmd_server_register_rows needs no copy: the tile
//    path's root kernel stores the row there itself.
//  * Host work per request is O(1): the queue is a vector whose buffers
//    circulate between the queue and the slots (no allocation per request),
//    keys are marked once per batch by generation stamp, and the tile path
//    groups requests by set in one counting pass; only the ciphertexts and
//    the tile items are copied to the device.  Requests can be queued in
//    groups under one lock (cmd_server_submit_many).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <functional>
#include <iterator>
#include <memory>
#include <mutex>
#include <random>
#include <shared_mutex>
#include <thread>
#include <vector>

#include "engine.h"

namespace cmd {

constexpr uint32_t CT_STRIDE = 208;   // largest ciphertext
constexpr uint32_t ERR_STRIDE = 256;  // words: largest error row (8192 bits)

static uint64_t now_ns()
{
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Request {
    uint32_t key_id;
    int32_t set;  // the key's set, fixed when the request is queued
    uint64_t tag;
    uint8_t *err_out;
    uint8_t *err_dev;  // device address of err_out when it lies in a registered row range, else null
    uint64_t t_arrive;
    uint8_t ct[CT_STRIDE];
};

// FIFO of requests in a vector with a head index.  Whole-queue takes swap
// buffers with the taking slot, so buffers circulate and steady-state
// submission allocates nothing.
struct RequestQueue {
    std::vector<Request> v;
    size_t head = 0;
    size_t size() const { return v.size() - head; }
    bool empty() const { return head == v.size(); }
    const Request &front() const { return v[head]; }
    void push_back(const Request &r) { v.push_back(r); }
    Request &emplace_back()  // a new request at the back, filled in place by the caller
    {
        v.emplace_back();
        return v.back();
    }
    // Moves the oldest `take` requests into out (whose old contents are dropped).
    void take_front(size_t take, std::vector<Request> &out)
    {
        out.clear();
        if (head == 0 && take == v.size()) {
            out.swap(v);
            return;
        }
        out.assign(v.begin() + head, v.begin() + head + take);
        head += take;
        if (head == v.size()) {
            v.clear();
            head = 0;
        }
    }
    // Puts requests back at the front, oldest first.
    template <class It>
    void push_front(It b, It e)
    {
        const size_t n = (size_t)std::distance(b, e);
        if (head >= n) {
            head -= n;
            std::copy(b, e, v.begin() + head);
        } else {
            v.insert(v.begin() + head, b, e);
        }
    }
};

struct KeyEntry {
    int set;
    std::vector<uint8_t> sk;
    cmd_key *key = nullptr;
    uint64_t last_use = 0;
    uint64_t seen_gen = 0;   // dispatcher only: the batch that last listed this key
    uint64_t batch_gen = 0;  // generation of the last batch this key was made resident for
    uint32_t batch_idx = 0;  // index within that batch's key table
};

// A few threads that split one batch's result copies with the completer.
class CopyPool {
public:
    explicit CopyPool(int helpers)
    {
        for (int i = 0; i < helpers; i++)
            th_.emplace_back([this] { loop(); });
    }
    ~CopyPool()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_.notify_all();
        for (auto &t : th_)
            t.join();
    }
    // Runs fn(c) for every c in [0, chunks) on the helpers and the calling
    // thread; returns when all chunks are done.
    void run(size_t chunks, const std::function<void(size_t)> &fn)
    {
        if (chunks <= 1 || th_.empty()) {
            for (size_t c = 0; c < chunks; c++)
                fn(c);
            return;
        }
        {
            std::lock_guard<std::mutex> lk(mu_);
            job_ = &fn;
            chunks_ = chunks;
            next_.store(0);
            active_ = th_.size();
            gen_++;
        }
        cv_.notify_all();
        work();
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return active_ == 0; });
        job_ = nullptr;
    }

private:
    void work()
    {
        size_t c;
        while ((c = next_.fetch_add(1)) < chunks_)
            (*job_)(c);
    }
    void loop()
    {
        uint64_t seen = 0;
        std::unique_lock<std::mutex> lk(mu_);
        while (true) {
            cv_.wait(lk, [&] { return stop_ || gen_ != seen; });
            if (stop_)
                return;
            seen = gen_;
            lk.unlock();
            work();
            lk.lock();
            if (--active_ == 0)
                cv_done_.notify_one();
        }
    }
    std::vector<std::thread> th_;
    std::mutex mu_;
    std::condition_variable cv_, cv_done_;
    const std::function<void(size_t)> *job_ = nullptr;
    size_t chunks_ = 0, active_ = 0;
    std::atomic<size_t> next_{0};
    uint64_t gen_ = 0;
    bool stop_ = false;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t start = nullptr, done = nullptr;  // bracket the batch's device work
    uint64_t t_launch = 0;
    uint8_t *h_in = nullptr, *d_in = nullptr;  // packed inputs (see dispatch)
    uint32_t *h_err = nullptr, *d_err = nullptr;
    uint16_t *h_w = nullptr, *d_w = nullptr;
    uint32_t *d_locbs = nullptr;        // tile path scratch (TILE_SCRATCH_WORDS per tile)
    std::vector<uint32_t> slot_of;      // request i -> result row (item slot)
    size_t rows_used = 0;               // result rows to copy back
    uint32_t *d_counter = nullptr;
    bool rows_direct = false;           // every row went straight to its request's buffer: no row copy
    std::vector<Request> reqs;  // taken from the queue (a buffer swap when a batch takes it all)
    uint64_t gen = 0;          // generation of the batch in this slot (its keys carry it)
    uint64_t seq = 0;          // sequence number of the batch in this slot (from 1)
    bool fused = false;
    // completer scratch, reused batch to batch
    std::vector<uint32_t> lats, waits;
    std::vector<cmd_completion> comps;
};

// Latency histogram with no allocation after construction: 1 us buckets up to
// 20 ms, 100 us buckets up to 2 s, one overflow bucket.  Quantiles are exact
// to the bucket (1 us below 20 ms); the maximum and the sum are kept exactly.
class LatencyHist {
public:
    LatencyHist() : fine_(FINE, 0), coarse_(COARSE + 1, 0) {}
    void add(uint64_t ns)
    {
        const uint64_t us = ns / 1000;
        if (us < FINE)
            fine_[us]++;
        else
            coarse_[std::min<uint64_t>((us - FINE) / 100, COARSE)]++;
        n_++;
        sum_ += ns;
        max_ = std::max(max_, ns);
    }
    void clear()
    {
        std::fill(fine_.begin(), fine_.end(), 0);
        std::fill(coarse_.begin(), coarse_.end(), 0);
        n_ = sum_ = max_ = 0;
    }
    uint64_t count() const { return n_; }
    double mean_us() const { return n_ ? sum_ / 1e3 / n_ : 0; }
    double max_us() const { return max_ / 1e3; }
    // the bucket holding the sample of rank f * (n - 1), as its lower edge in us
    double quantile_us(double f) const
    {
        if (!n_)
            return 0;
        const uint64_t rank = (uint64_t)(f * (n_ - 1));
        uint64_t seen = 0;
        for (uint64_t b = 0; b < FINE; b++)
            if ((seen += fine_[b]) > rank)
                return (double)b;
        for (uint64_t b = 0; b <= COARSE; b++)
            if ((seen += coarse_[b]) > rank)
                return (double)(FINE + 100 * b);
        return max_us();
    }

private:
    static constexpr uint64_t FINE = 20000, COARSE = 19800;
    std::vector<uint64_t> fine_, coarse_;
    uint64_t n_ = 0, sum_ = 0, max_ = 0;
};

}  // namespace cmd

using namespace cmd;

struct cmd_server {
    cmd_engine *eng = nullptr;
    cmd_server_config cfg{};
    size_t in_bytes = 0, device_bytes = 0;
    // Lock order: keys_mu before mu.  keys_mu guards the key table's shape
    // (add_key appends under both locks); the dispatcher reads entries under
    // a shared hold, the completer and submitters under mu.
    std::shared_mutex keys_mu;
    std::mutex mu;
    std::condition_variable cv_dispatch, cv_complete, cv_poll;
    RequestQueue pending;
    std::deque<KeyEntry> keys;   // deque: entries keep their address as keys are added
    // The keys' sets again, for the submitters: they read a key's set for
    // every request, while the dispatcher writes its generation stamps into
    // the key entries; reading the set from those entries kept their cache
    // lines moving between the two cores (about 70 us of every batch's key
    // pass at several thousand batches a second).
    std::deque<int32_t> key_sets;
    std::vector<Slot> slots;
    std::deque<int> free_slots;
    std::atomic<uint32_t> inflight{0};  // bit s: slot s has a batch on the GPU (set under mu)
    // done_seq[s]: pinned host word that slot s's stream overwrites with the
    // batch's sequence number after its result copies (a stream-ordered
    // 8-byte copy), so the completer sees a finished batch with plain loads
    volatile uint64_t *done_seq = nullptr;
    std::deque<cmd_completion> completions;
    // Caller memory registered for result rows (cmd_server_register_rows):
    // requests whose row lies inside one get it stored by the tile path's
    // root kernel itself.  Appended under mu, read by submitters under mu.
    struct RowRange {
        uint8_t *host, *dev;
        size_t bytes;
        bool registered_here;  // pinned by cmd_server_register_rows: unregistered at destroy
    };
    std::vector<RowRange> row_ranges;
    std::thread dispatcher, completer;
    std::unique_ptr<CopyPool> copiers;
    bool stop = false;
    bool dispatch_exited = false;
    int status = CMD_OK;
    uint64_t batch_gen = 0;  // dispatcher only
    // statistics
    LatencyHist lat;   // per request: arrival -> result delivered
    LatencyHist gpu;   // per batch: device time, input copy to result copy
    LatencyHist wait;  // per request: arrival -> batch launch
    uint64_t submitted = 0, completed = 0, refused = 0, batches = 0, fused_batches = 0, batched_cts = 0;
    uint64_t t_first = 0, t_last = 0;
    uint64_t dispatch_ns = 0, complete_ns = 0, inflight_sum = 0;  // host time in launch / result handling
    uint64_t tick = 0;
    uint64_t completions_gen = 0;  // bumped each time a batch completes

    // Device address of a result row [p, p + bytes) inside a registered range
    // (2-byte aligned, as the kernels' packed row stores need), or null.
    uint8_t *row_device(uint8_t *p, size_t bytes) const
    {
        if (((uintptr_t)p) & 1)
            return nullptr;
        for (const RowRange &rr : row_ranges)
            if (p >= rr.host && (size_t)(p - rr.host) + bytes <= rr.bytes)
                return rr.dev + (p - rr.host);
        return nullptr;
    }
    void dispatch_loop();
    void complete_loop();
    int ensure_key(uint32_t id);
    int launch(Slot &sl);
};

namespace {

// Result rows a batch of B requests may need: the tile path pads each set's
// run of requests to whole 32-request tiles.
size_t row_cap(size_t B) { return B + NSETS * 32; }
size_t tile_cap(size_t B) { return B / 32 + NSETS + 1; }

// Input packing of a slot: ciphertexts at CT_STRIDE, then key index per
// ciphertext, then (fused) ct_off, err_off, order, tiles, key table, then
// (tile path) the work items.
struct InLayout {
    size_t cts, key_idx, ct_off, err_off, order, tiles, keys, items, seq, total;
    InLayout(size_t B, size_t max_keys)
    {
        auto al = [](size_t x) { return (x + 255) / 256 * 256; };
        cts = 0;
        key_idx = al(cts + B * CT_STRIDE);
        ct_off = al(key_idx + B * 4);
        err_off = al(ct_off + B * 8);
        order = al(err_off + B * 8);
        tiles = al(order + B * 4);
        keys = al(tiles + B * sizeof(FusedTile));
        items = al(keys + max_keys * sizeof(FusedKeyRef));
        seq = al(items + row_cap(B) * sizeof(LatItem));  // the batch's sequence number (8 bytes)
        total = al(seq + 8);
    }
};

}  // namespace

int cmd_server::ensure_key(uint32_t id)
{
    KeyEntry &ke = keys[id];
    ke.last_use = ++tick;
    if (ke.key)
        return CMD_OK;
    while (true) {
        int rc = cmd_key_expand(eng, (cmd_set)ke.set, ke.sk.data(), ke.sk.size(), &ke.key);
        if (rc != CMD_E_BUDGET)
            return rc;
        // Evict the least recently used resident key that no batch in flight
        // and not this batch uses: its generation stamp is older than every
        // batch in flight and than this one.
        uint64_t oldest = batch_gen;  // this batch's generation
        const uint32_t fl = inflight.load();
        for (size_t si = 0; si < slots.size(); si++)
            if ((fl >> si) & 1u)
                oldest = std::min(oldest, slots[si].gen);
        int victim = -1;
        bool held = false;  // some resident key is in use by a batch in flight
        {
            std::lock_guard<std::mutex> lk(mu);
            for (size_t k = 0; k < keys.size(); k++) {
                if (!keys[k].key || k == id)
                    continue;
                if (keys[k].batch_gen >= oldest) {
                    held = held || keys[k].batch_gen < batch_gen;
                    continue;
                }
                if (victim < 0 || keys[k].last_use < keys[victim].last_use)
                    victim = (int)k;
            }
        }
        if (victim < 0)
            return held ? CMD_E_BUSY : CMD_E_BUDGET;  // BUSY: retry once a batch completes
        cmd_key *gone = keys[victim].key;
        {
            std::lock_guard<std::mutex> lk(mu);  // stats read residency under mu
            keys[victim].key = nullptr;
        }
        cmd_key_free(gone);
    }
}

int cmd_server::launch(Slot &sl)
{
    // Make the batch's keys resident.  When the HBM budget cannot hold all of
    // them at once, the requests of the keys that did not fit go back to the
    // front of the queue for the next batch (only a batch whose first key
    // cannot be made resident fails).
    std::shared_lock<std::shared_mutex> key_hold(keys_mu);
    std::vector<uint32_t> kid;
    uint64_t gen = ++batch_gen;
    // The requests were just written by the submitting threads, so each first
    // touch here is a miss served from another core's cache; prefetching a
    // few requests ahead overlaps those misses instead of taking them one by
    // one.
    constexpr size_t AHEAD = 12;
    const size_t nreq = sl.reqs.size();
    for (size_t i = 0; i < nreq; i++) {
        if (i + AHEAD < nreq)
            __builtin_prefetch(&sl.reqs[i + AHEAD]);
        const Request &r = sl.reqs[i];
        KeyEntry &ke = keys[r.key_id];
        if (ke.seen_gen != gen) {
            ke.seen_gen = gen;
            kid.push_back(r.key_id);
        }
    }
    // A key made resident for this batch carries its generation, which keeps
    // it from being evicted for the batch's later keys.
    std::vector<uint32_t> ready;
    for (uint32_t k : kid) {
        int rc = ensure_key(k);
        if ((rc == CMD_E_BUDGET || rc == CMD_E_BUSY) && !ready.empty())
            break;
        if (rc)
            return rc;
        keys[k].batch_gen = gen;
        ready.push_back(k);
    }
    if (ready.size() < kid.size()) {
        std::lock_guard<std::mutex> lk(mu);
        gen = ++batch_gen;  // re-stamp: only the ready keys stay in this batch
        for (uint32_t k : ready)
            keys[k].batch_gen = gen;
        std::vector<Request> keep, defer;
        for (const Request &r : sl.reqs)
            (keys[r.key_id].batch_gen == gen ? keep : defer).push_back(r);
        pending.push_front(defer.begin(), defer.end());
        sl.reqs.swap(keep);
    }
    sl.gen = gen;  // the batch's keys stay in use while it is in flight
    const size_t B = sl.reqs.size();
    InLayout lay(B, B);
    sl.seq++;
    memcpy(sl.h_in + lay.seq, &sl.seq, 8);
    for (size_t i = 0; i < B; i++)
        memcpy(sl.h_in + lay.cts + i * CT_STRIDE, sl.reqs[i].ct, CT_STRIDE);
    LaunchCounter lc{&eng->launches};
    cudaStream_t s = sl.stream;
    cudaError_t e;
    sl.t_launch = now_ns();
    if ((e = cudaEventRecord(sl.start, s)) != cudaSuccess)
        return cuda_fail(e, "server event");
    sl.fused = cfg.fused_threshold > 0 && B >= cfg.fused_threshold;
    sl.slot_of.resize(B);
    if (!sl.fused) {
        // Tile path: requests grouped by set (a counting pass over the five
        // sets) into tiles of up to 32, any keys within a tile; item slot
        // 32*t + q is request q of tile t.  Only the ciphertexts and the
        // items go to the device.
        LatItem *items = reinterpret_cast<LatItem *>(sl.h_in + lay.items);
        uint32_t cnt[NSETS] = {}, tile0[NSETS], next[NSETS] = {};
        for (size_t i = 0; i < B; i++)
            cnt[sl.reqs[i].set]++;
        uint32_t ntiles = 0;
        for (int st = 0; st < NSETS; st++) {
            tile0[st] = ntiles;
            ntiles += (cnt[st] + 31) / 32;
        }
        size_t direct = 0;
        for (size_t i = 0; i < B; i++) {
            const Request &r = sl.reqs[i];
            const uint32_t pos = next[r.set]++;
            const uint32_t slot = 32 * (tile0[r.set] + pos / 32) + pos % 32;
            const uint32_t left = cnt[r.set] - pos / 32 * 32;
            const KeyDev &kd = keys[r.key_id].key->dev;
            items[slot] = LatItem{kd.wfft, kd.bctl, (uint32_t)(i * CT_STRIDE), slot * ERR_STRIDE, r.set,
                                  (int32_t)(left < 32 ? left : 32), r.err_dev};
            direct += r.err_dev != nullptr;
            sl.slot_of[i] = slot;
        }
        for (int st = 0; st < NSETS; st++)
            for (uint32_t pos = cnt[st]; pos % 32; pos++) {  // the set's last tile, past its count
                const uint32_t slot = 32 * (tile0[st] + pos / 32) + pos % 32;
                items[slot] = LatItem{nullptr, nullptr, 0, slot * ERR_STRIDE, -1, (int32_t)(cnt[st] % 32), nullptr};
            }
        sl.rows_used = (size_t)ntiles * 32;
        sl.rows_direct = direct == B;
        if ((e = cudaMemcpyAsync(sl.d_in + lay.cts, sl.h_in + lay.cts, B * CT_STRIDE, cudaMemcpyHostToDevice, s)) !=
                cudaSuccess ||
            (e = cudaMemcpyAsync(sl.d_in + lay.items, sl.h_in + lay.items, lay.seq + 8 - lay.items,
                                 cudaMemcpyHostToDevice, s)) != cudaSuccess)
            return cuda_fail(e, "server H2D");
        FftPlans plans;
        for (int st = 0; st < NSETS; st++)
            plans.p[st] = eng->fft[st];
        e = launch_tile_path(sl.d_in + lay.items, sl.d_in + lay.cts, ntiles, sl.d_locbs, sl.d_err, sl.d_w, plans, s, lc);
        if (e != cudaSuccess)
            return cuda_fail(e, "server tile-path launch");
    } else {
        // Fused path: a key table in set order, so that grouping requests by
        // key index also groups them by set.
        kid = ready;
        std::stable_sort(kid.begin(), kid.end(), [&](uint32_t a, uint32_t b) { return keys[a].set < keys[b].set; });
        for (size_t k = 0; k < kid.size(); k++)
            keys[kid[k]].batch_idx = (uint32_t)k;
        uint32_t *key_idx = reinterpret_cast<uint32_t *>(sl.h_in + lay.key_idx);
        for (size_t i = 0; i < B; i++)
            key_idx[i] = keys[sl.reqs[i].key_id].batch_idx;
        FusedKeyRef *krefs = reinterpret_cast<FusedKeyRef *>(sl.h_in + lay.keys);
        std::vector<int> kset(kid.size());
        for (size_t k = 0; k < kid.size(); k++) {
            const cmd_key *key = keys[kid[k]].key;
            krefs[k] = key_ref(key->dev);
            kset[k] = key->dev.set;
        }
        uint64_t *ct_off = reinterpret_cast<uint64_t *>(sl.h_in + lay.ct_off);
        uint64_t *err_off = reinterpret_cast<uint64_t *>(sl.h_in + lay.err_off);
        for (size_t i = 0; i < B; i++) {
            ct_off[i] = i * CT_STRIDE;
            err_off[i] = i * ERR_STRIDE;
            sl.slot_of[i] = (uint32_t)i;
        }
        const int single = mixed_single_set(kset.data(), key_idx, B);
        const int wpb = single >= 0 ? eng->fcfg[single].wpb : eng->fcfg_mixed.wpb;
        std::vector<uint32_t> order;
        std::vector<FusedTile> tiles;
        plan_mixed(kset.data(), kid.size(), key_idx, B, (uint32_t)wpb * 32, order, tiles);
        memcpy(sl.h_in + lay.order, order.data(), B * 4);
        memcpy(sl.h_in + lay.tiles, tiles.data(), tiles.size() * sizeof(FusedTile));
        if ((e = cudaMemcpyAsync(sl.d_in, sl.h_in, lay.total, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
            (e = cudaMemsetAsync(sl.d_counter, 0, 4, s)) != cudaSuccess)
            return cuda_fail(e, "server H2D");
        FusedArgs a;
        memset(&a, 0, sizeof a);
        a.tiles = reinterpret_cast<const FusedTile *>(sl.d_in + lay.tiles);
        a.ntiles = (uint32_t)tiles.size();
        a.keys = reinterpret_cast<const FusedKeyRef *>(sl.d_in + lay.keys);
        a.cts = sl.d_in + lay.cts;
        a.ct_off = reinterpret_cast<const uint64_t *>(sl.d_in + lay.ct_off);
        a.err_off = reinterpret_cast<const uint64_t *>(sl.d_in + lay.err_off);
        a.order = reinterpret_cast<const uint32_t *>(sl.d_in + lay.order);
        a.err = sl.d_err;
        a.weight = sl.d_w;
        a.tile_counter = sl.d_counter;
        a.single_set = single;
        fill_fft(a, eng);
        size_t smem = 0;
        if (single >= 0)
            smem = fused_smem(single, wpb);
        else
            for (int st = 0; st < NSETS; st++)
                smem = std::max(smem, fused_smem(st, wpb));
        const int grid = fused_grid(eng, single, wpb, smem, tiles.size());
        if ((e = launch_fused(a, grid, wpb, s, lc)) != cudaSuccess)
            return cuda_fail(e, "server fused launch");
    }
    if (sl.fused) {
        sl.rows_used = B;
        sl.rows_direct = false;  // the fused kernel's rows take the staged copy
    }
    if ((!sl.rows_direct &&
         (e = cudaMemcpyAsync(sl.h_err, sl.d_err, sl.rows_used * ERR_STRIDE * 4, cudaMemcpyDeviceToHost, s)) !=
             cudaSuccess) ||
        (e = cudaMemcpyAsync(sl.h_w, sl.d_w, sl.rows_used * 2, cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaEventRecord(sl.done, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync((void *)(done_seq + (&sl - slots.data())), sl.d_in + lay.seq, 8, cudaMemcpyDeviceToHost,
                             s)) != cudaSuccess)
        return cuda_fail(e, "server D2H");
    return CMD_OK;
}

void cmd_server::dispatch_loop()
{
    cudaSetDevice(eng->device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        cv_dispatch.wait(lk, [&] { return stop || (!pending.empty() && !free_slots.empty()); });
        if (stop && pending.empty())
            break;
        if (pending.empty() || free_slots.empty())
            continue;
        // Continuous batching: with batches already on the GPU, give the
        // oldest waiting request up to max_wait_us to collect batch-mates.
        if (inflight.load() && pending.size() < cfg.max_batch && !stop) {
            const uint64_t deadline = pending.front().t_arrive + (uint64_t)cfg.max_wait_us * 1000;
            const uint64_t t = now_ns();
            if (t < deadline) {
                cv_dispatch.wait_for(lk, std::chrono::nanoseconds(deadline - t), [&] {
                    return stop || pending.size() >= cfg.max_batch || !inflight.load();
                });
                if (pending.empty() || free_slots.empty())
                    continue;
            }
        }
        const int si = free_slots.front();
        free_slots.pop_front();
        Slot &sl = slots[si];
        pending.take_front(std::min<size_t>(pending.size(), cfg.max_batch), sl.reqs);
        lk.unlock();
        const uint64_t t0 = now_ns();
        int rc = launch(sl);
        const uint64_t t1 = now_ns();
        lk.lock();
        dispatch_ns += t1 - t0;
        if (rc == CMD_E_BUSY) {
            // Every key that could be evicted is in use by a batch in flight:
            // requeue the batch and wait for a completion before retrying.
            pending.push_front(sl.reqs.begin(), sl.reqs.end());
            sl.reqs.clear();
            free_slots.push_front(si);
            const uint64_t gen = completions_gen;
            cv_dispatch.wait(lk, [&] { return stop || completions_gen != gen || !inflight.load(); });
            continue;
        }
        if (rc != CMD_OK) {
            // Fail the batch's requests; the slot stays usable.
            const uint64_t t = now_ns();
            for (const Request &r : sl.reqs) {
                if (cfg.record_completions)
                    completions.push_back(cmd_completion{r.tag, rc, 0, 0, t - r.t_arrive});
                completed++;
            }
            sl.reqs.clear();
            free_slots.push_back(si);
            if (status == CMD_OK)
                status = rc;
            cv_poll.notify_all();
            continue;
        }
        batches++;
        fused_batches += sl.fused ? 1 : 0;
        batched_cts += sl.reqs.size();
        inflight.fetch_or(1u << si);
        inflight_sum += __builtin_popcount(inflight.load());
        cv_complete.notify_one();
    }
    dispatch_exited = true;
    cv_complete.notify_all();
}

void cmd_server::complete_loop()
{
    cudaSetDevice(eng->device);
    uint64_t idle_since = 0;
    while (true) {
        uint32_t mask = inflight.load();
        if (!mask) {
            std::unique_lock<std::mutex> lk(mu);
            cv_complete.wait(lk, [&] { return inflight.load() != 0 || dispatch_exited; });
            if (!inflight.load())
                break;  // the dispatcher has exited and every batch is done
            continue;
        }
        // Whichever batch in flight finishes first: batches of different
        // sizes complete out of order, and a small one must not wait behind
        // a large one.  With one batch in flight, block on its event.  The
        // in-flight set is read without the queue lock, so polling does not
        // slow submitters down.
        // A batch is finished when its stream has copied the batch's
        // sequence number into done_seq (after its results): the check is a
        // plain load, with no CUDA call that would contend in the runtime
        // with the dispatcher's launches.  A failed stream never delivers
        // it, so after 2 ms without a finished batch the events are queried
        // for errors.
        int si = -1;
        cudaError_t e = cudaSuccess;
        for (uint32_t m = mask; m; m &= m - 1) {
            const int x = __builtin_ctz(m);
            if (done_seq[x] == slots[x].seq) {
                si = x;
                break;
            }
        }
        if (si < 0) {
            const uint64_t tn = now_ns();
            if (!idle_since)
                idle_since = tn;
            if (tn - idle_since > 2000000) {
                idle_since = tn;
                for (uint32_t m = mask; m; m &= m - 1) {
                    const int x = __builtin_ctz(m);
                    const cudaError_t q = cudaEventQuery(slots[x].done);
                    if (q != cudaErrorNotReady && q != cudaSuccess) {
                        si = x;
                        e = q;
                        break;
                    }
                }
            }
            if (si < 0) {
                std::this_thread::yield();
                continue;
            }
        }
        idle_since = 0;
        std::atomic_thread_fence(std::memory_order_acquire);  // the results landed before the sequence word
        Slot &sl = slots[si];
        const uint64_t t = now_ns();
        float gpu_ms = 0;
        if (e == cudaSuccess)
            cudaEventElapsedTime(&gpu_ms, sl.start, sl.done);
        const size_t B = sl.reqs.size();
        sl.lats.resize(B);
        sl.waits.resize(B);
        if (cfg.record_completions)
            sl.comps.resize(B);
        // Results to the requests' buffers, in chunks across the copy threads
        // for large batches.
        constexpr size_t CHUNK = 256;
        const size_t chunks = (B + CHUNK - 1) / CHUNK;
        copiers->run(chunks, [&](size_t c) {
            const size_t end = std::min(B, (c + 1) * CHUNK);
            for (size_t i = c * CHUNK; i < end; i++) {
                const Request &r = sl.reqs[i];
                // (a tile-path row in registered memory is already there)
                if (e == cudaSuccess && r.err_out && (sl.fused || !r.err_dev))
                    memcpy(r.err_out, sl.h_err + (size_t)sl.slot_of[i] * ERR_STRIDE, set_info(r.set).n / 8);
                const uint64_t lat = t - r.t_arrive;
                sl.lats[i] = (uint32_t)std::min<uint64_t>(lat, 0xFFFFFFFFu);
                sl.waits[i] = (uint32_t)std::min<uint64_t>(sl.t_launch - r.t_arrive, 0xFFFFFFFFu);
                if (cfg.record_completions)
                    sl.comps[i] =
                        cmd_completion{r.tag, e == cudaSuccess ? CMD_OK : CMD_E_CUDA, sl.h_w[sl.slot_of[i]], 0, lat};
            }
        });
        const uint64_t t_done = now_ns();
        std::lock_guard<std::mutex> lk(mu);
        if (e != cudaSuccess && status == CMD_OK) {
            status = CMD_E_CUDA;
            set_last_error(std::string("server batch: ") + cudaGetErrorString(e));
        }
        if (cfg.record_completions)
            completions.insert(completions.end(), sl.comps.begin(), sl.comps.end());
        for (size_t i = 0; i < B; i++) {
            lat.add(sl.lats[i]);
            wait.add(sl.waits[i]);
        }
        gpu.add((uint64_t)(gpu_ms * 1e6f));
        completed += B;
        t_last = t;
        complete_ns += t_done - t;
        sl.reqs.clear();
        inflight.fetch_and(~(1u << si));
        free_slots.push_back(si);
        completions_gen++;
        cv_dispatch.notify_one();
        cv_poll.notify_all();
    }
}

namespace {

// Queues requests key_ids[i] / h_cts + i * ct_stride (results to h_err_base
// + i * err_stride, or nowhere) under one lock, in order, until the queue is
// full; arrival times t_arrive[i] (steady-clock ns), or now.  *accepted = how
// many were queued; the rest are refused.
int submit_group(cmd_server *srv, size_t n, const uint32_t *key_ids, const uint8_t *h_cts, size_t ct_stride,
                 uint8_t *h_err_base, size_t err_stride, const uint64_t *tags, const uint64_t *t_arrive,
                 size_t *accepted)
{
    bool wake = false;
    size_t k = 0;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        if (srv->stop)
            return CMD_E_ARG;
        for (size_t i = 0; i < n; i++)
            if (key_ids[i] >= srv->key_sets.size())
                return CMD_E_ARG;
        const size_t before = srv->pending.size();
        const uint64_t now = t_arrive ? 0 : now_ns();
        for (; k < n && srv->pending.size() < srv->cfg.queue_capacity; k++) {
            Request &r = srv->pending.emplace_back();
            r.key_id = key_ids[k];
            r.tag = tags ? tags[k] : k;
            r.err_out = h_err_base ? h_err_base + k * err_stride : nullptr;
            r.set = srv->key_sets[r.key_id];
            r.err_dev = r.err_out ? srv->row_device(r.err_out, set_info(r.set).n / 8) : nullptr;
            const int ctb = set_info(r.set).ct;
            memcpy(r.ct, h_cts + k * ct_stride, ctb);
            memset(r.ct + ctb, 0, CT_STRIDE - ctb);
            r.t_arrive = t_arrive ? t_arrive[k] : now;
            if (srv->submitted++ == 0)
                srv->t_first = r.t_arrive;
        }
        srv->refused += n - k;
        // The dispatcher waits for a first request or for a full batch: only
        // those two transitions need a wake-up (not every submission).
        const size_t np = srv->pending.size();
        wake = k > 0 && (before == 0 || (before < srv->cfg.max_batch && np >= srv->cfg.max_batch));
    }
    if (wake)
        srv->cv_dispatch.notify_one();
    *accepted = k;
    return CMD_OK;
}

}  // namespace

extern "C" {

int cmd_server_create(cmd_engine *eng, const cmd_server_config *cfg, cmd_server **out)
{
    if (!eng || !cfg || !out || cfg->max_batch == 0 || cfg->max_batch > 65536 || cfg->slots < 1 ||
        cfg->slots > 16 || cfg->queue_capacity == 0)
        return CMD_E_ARG;
    *out = nullptr;
    cudaSetDevice(eng->device);
    cmd_server *srv = new cmd_server();
    srv->eng = eng;
    srv->cfg = *cfg;
    const size_t B = cfg->max_batch;
    InLayout lay(B, B);
    srv->in_bytes = lay.total;
    const size_t rows = row_cap(B), locbs = tile_cap(B) * (size_t)TILE_SCRATCH_WORDS * 4;
    const size_t dev_per_slot = lay.total + rows * ERR_STRIDE * 4 + rows * 2 + locbs + 4 * 256;
    srv->device_bytes = dev_per_slot * cfg->slots;
    if (!budget_take(eng, srv->device_bytes)) {
        delete srv;
        set_last_error("server buffers exceed the engine HBM budget");
        return CMD_E_BUDGET;
    }
    srv->slots.resize(cfg->slots);
    // The request buffers circulate between the queue and the slots; giving
    // each a batch's capacity up front keeps their growth (a copy of every
    // queued request, under the queue lock) out of the first seconds at a
    // higher load.
    srv->pending.v.reserve(cfg->max_batch);
    for (auto &sl : srv->slots)
        sl.reqs.reserve(cfg->max_batch);
    cudaError_t e = cudaMallocHost((void **)&srv->done_seq, 16 * sizeof(uint64_t));
    if (e == cudaSuccess)
        memset((void *)srv->done_seq, 0, 16 * sizeof(uint64_t));
    for (auto &sl : srv->slots) {
        if (e == cudaSuccess)
            e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess)
            e = cudaEventCreate(&sl.done);
        if (e == cudaSuccess)
            e = cudaEventCreate(&sl.start);
        if (e == cudaSuccess)
            e = cudaMallocHost(&sl.h_in, lay.total);
        if (e == cudaSuccess)
            e = cudaMallocHost(&sl.h_err, rows * ERR_STRIDE * 4);
        if (e == cudaSuccess)
            e = cudaMallocHost(&sl.h_w, rows * 2);
        if (e == cudaSuccess)
            e = cudaMalloc(&sl.d_in, lay.total);
        if (e == cudaSuccess)
            e = cudaMalloc(&sl.d_err, rows * ERR_STRIDE * 4);
        if (e == cudaSuccess)
            e = cudaMalloc(&sl.d_w, rows * 2);
        if (e == cudaSuccess)
            e = cudaMalloc(&sl.d_locbs, locbs);
        if (e == cudaSuccess)
            e = cudaMalloc(&sl.d_counter, 256);
    }
    if (e != cudaSuccess) {
        cmd_server_destroy(srv);
        return cuda_fail(e, "server buffers");
    }
    for (int i = 0; i < (int)cfg->slots; i++)
        srv->free_slots.push_back(i);
    srv->dispatcher = std::thread([srv] { srv->dispatch_loop(); });
    // up to three copy helpers beside the completer, leaving cores to the
    // submitters and the dispatcher
    const unsigned hc = std::thread::hardware_concurrency();
    srv->copiers.reset(new CopyPool((int)std::min(3u, hc > 4 ? (hc - 4) / 2 : 0u)));
    srv->completer = std::thread([srv] { srv->complete_loop(); });
    *out = srv;
    return CMD_OK;
}

void cmd_server_destroy(cmd_server *srv)
{
    if (!srv)
        return;
    {
        std::lock_guard<std::mutex> lk(srv->mu);
        srv->stop = true;
    }
    srv->cv_dispatch.notify_all();
    if (srv->dispatcher.joinable())
        srv->dispatcher.join();
    srv->cv_complete.notify_all();
    if (srv->completer.joinable())
        srv->completer.join();
    cudaSetDevice(srv->eng->device);
    for (auto &sl : srv->slots) {
        if (sl.stream)
            cudaStreamSynchronize(sl.stream);
        cudaFreeHost(sl.h_in);
        cudaFreeHost(sl.h_err);
        cudaFreeHost(sl.h_w);
        cudaFree(sl.d_in);
        cudaFree(sl.d_err);
        cudaFree(sl.d_w);
        cudaFree(sl.d_locbs);
        cudaFree(sl.d_counter);
        if (sl.done)
            cudaEventDestroy(sl.done);
        if (sl.start)
            cudaEventDestroy(sl.start);
        if (sl.stream)
            cudaStreamDestroy(sl.stream);
    }
    for (auto &k : srv->keys)
        if (k.key)
            cmd_key_free(k.key);
    for (const auto &rr : srv->row_ranges)
        if (rr.registered_here)
            cudaHostUnregister(rr.host);
    if (srv->done_seq)
        cudaFreeHost((void *)srv->done_seq);
    if (srv->device_bytes)
        budget_give(srv->eng, srv->device_bytes);
    delete srv;
}

int cmd_server_add_key(cmd_server *srv, cmd_set set, const uint8_t *h_sk, size_t sk_len, uint32_t *key_id)
{
    if (!srv || !h_sk || !key_id || !valid_set(set) || sk_len != (size_t)set_info(set).sk)
        return CMD_E_ARG;
    std::unique_lock<std::shared_mutex> key_hold(srv->keys_mu);
    std::lock_guard<std::mutex> lk(srv->mu);
    KeyEntry ke;
    ke.set = set;
    ke.sk.assign(h_sk, h_sk + sk_len);
    srv->keys.push_back(std::move(ke));
    srv->key_sets.push_back(set);
    *key_id = (uint32_t)(srv->keys.size() - 1);
    return CMD_OK;
}

int cmd_server_register_rows(cmd_server *srv, uint8_t *h_rows, size_t bytes)
{
    if (!srv || !h_rows || !bytes)
        return CMD_E_ARG;
    cudaSetDevice(srv->eng->device);
    uint8_t *dev = device_view(h_rows, bytes);
    bool here = false;
    if (!dev) {
        // pageable memory: pin and map it for the server's lifetime
        cudaError_t e = cudaHostRegister(h_rows, bytes, cudaHostRegisterMapped | cudaHostRegisterPortable);
        if (e != cudaSuccess)
            return cuda_fail(e, "cmd_server_register_rows: cudaHostRegister");
        here = true;
        dev = device_view(h_rows, bytes);
        if (!dev) {
            cudaHostUnregister(h_rows);
            set_last_error("cmd_server_register_rows: the range has no contiguous device mapping");
            return CMD_E_ARG;
        }
    }
    std::lock_guard<std::mutex> lk(srv->mu);
    srv->row_ranges.push_back(cmd_server::RowRange{h_rows, dev, bytes, here});
    return CMD_OK;
}

int cmd_server_submit(cmd_server *srv, uint32_t key_id, const uint8_t *h_ct, uint8_t *h_err_out, uint64_t tag)
{
    if (!srv || !h_ct)
        return CMD_E_ARG;
    size_t accepted = 0;
    const int rc = submit_group(srv, 1, &key_id, h_ct, 0, h_err_out, 0, &tag, nullptr, &accepted);
    return rc ? rc : (accepted ? CMD_OK : CMD_E_BUSY);
}

int cmd_server_submit_many(cmd_server *srv, size_t n, const uint32_t *key_ids, const uint8_t *h_cts,
                           size_t ct_stride, uint8_t *h_err_base, size_t err_stride, const uint64_t *tags,
                           size_t *accepted)
{
    if (!srv || (n && (!key_ids || !h_cts || !ct_stride)) || (h_err_base && !err_stride))
        return CMD_E_ARG;
    size_t acc = 0;
    const int rc = submit_group(srv, n, key_ids, h_cts, ct_stride, h_err_base, err_stride, tags, nullptr, &acc);
    if (accepted)
        *accepted = acc;
    return rc ? rc : (acc == n ? CMD_OK : CMD_E_BUSY);
}

int cmd_server_poll(cmd_server *srv, cmd_completion *out, size_t max, size_t *n, uint32_t timeout_us)
{
    if (!srv || !n || (max && !out))
        return CMD_E_ARG;
    std::unique_lock<std::mutex> lk(srv->mu);
    if (srv->completions.empty() && timeout_us)
        srv->cv_poll.wait_for(lk, std::chrono::microseconds(timeout_us), [&] { return !srv->completions.empty(); });
    size_t k = 0;
    while (k < max && !srv->completions.empty()) {
        out[k++] = srv->completions.front();
        srv->completions.pop_front();
    }
    *n = k;
    return srv->status;
}

int cmd_server_drain(cmd_server *srv, uint32_t timeout_ms)
{
    if (!srv)
        return CMD_E_ARG;
    std::unique_lock<std::mutex> lk(srv->mu);
    const bool ok = srv->cv_poll.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] {
        return srv->completed + 0 >= srv->submitted;
    });
    if (!ok)
        return CMD_E_TIMEOUT;
    return srv->status;
}

int cmd_server_stats_get(cmd_server *srv, cmd_server_stats *st, int reset)
{
    if (!srv || !st)
        return CMD_E_ARG;
    std::lock_guard<std::mutex> lk(srv->mu);
    memset(st, 0, sizeof *st);
    st->submitted = srv->submitted;
    st->completed = srv->completed;
    st->refused = srv->refused;
    st->batches = srv->batches;
    st->fused_batches = srv->fused_batches;
    st->mean_batch = srv->batches ? (double)srv->batched_cts / srv->batches : 0;
    st->resident_keys = 0;
    for (const auto &k : srv->keys)
        st->resident_keys += k.key != nullptr;
    st->gpu_p50_us = srv->gpu.quantile_us(0.50);
    st->gpu_p99_us = srv->gpu.quantile_us(0.99);
    st->wait_p50_us = srv->wait.quantile_us(0.50);
    st->wait_p99_us = srv->wait.quantile_us(0.99);
    if (srv->lat.count()) {
        st->p50_us = srv->lat.quantile_us(0.50);
        st->p99_us = srv->lat.quantile_us(0.99);
        st->max_us = srv->lat.max_us();
        st->mean_us = srv->lat.mean_us();
    }
    if (srv->t_last > srv->t_first) {
        const double span = (double)(srv->t_last - srv->t_first);
        st->decaps_per_s = srv->completed / (span * 1e-9);
        st->dispatch_busy = srv->dispatch_ns / span;
        st->complete_busy = srv->complete_ns / span;
    }
    st->mean_inflight = srv->batches ? (double)srv->inflight_sum / srv->batches : 0;
    if (reset) {
        srv->lat.clear();
        srv->gpu.clear();
        srv->wait.clear();
        srv->submitted -= srv->completed;
        srv->completed = 0;
        srv->refused = srv->batches = srv->fused_batches = srv->batched_cts = 0;
        srv->t_first = srv->t_last = 0;
        srv->dispatch_ns = srv->complete_ns = srv->inflight_sum = 0;
    }
    return CMD_OK;
}

// Open-loop Poisson load: request i uses key key_ids[i % pool] and
// ciphertext i % pool, and its result lands in err_pool row i % pool.
// Arrival times are a Poisson process of rate rate_per_s over `seconds`;
// each request is queued with its scheduled arrival time, so latency counts
// from when the request was due even if the generator queues it a little
// later.  Every pass of the generator queues, under one lock, all requests
// whose time has come.  Then it waits for every request to complete.
int cmd_server_loadgen(cmd_server *srv, const uint32_t *key_ids, const uint8_t *cts, size_t ct_stride,
                       uint8_t *err_pool, size_t err_stride, size_t pool, double rate_per_s, double seconds,
                       uint64_t seed, cmd_server_stats *out)
{
    if (!srv || !key_ids || !cts || !pool || rate_per_s <= 0 || seconds <= 0 || !out)
        return CMD_E_ARG;
    cmd_server_stats dummy;
    cmd_server_stats_get(srv, &dummy, 1);
    std::mt19937_64 rng(seed);
    std::exponential_distribution<double> gap(rate_per_s);
    constexpr size_t GROUP = 4096;
    std::vector<uint32_t> g_key(GROUP);
    std::vector<uint64_t> g_tag(GROUP), g_t(GROUP), g_row(GROUP);
    const uint64_t t0 = now_ns();
    const uint64_t t_end = t0 + (uint64_t)(seconds * 1e9);
    double next = (double)t0 + gap(rng) * 1e9;
    size_t i = 0;
    while (next < (double)t_end) {
        const uint64_t now = now_ns();
        if ((double)now < next)
            continue;
        // the requests due by now, queued together
        size_t g = 0;
        while (g < GROUP && next <= (double)now && next < (double)t_end) {
            const size_t k = i % pool;
            g_key[g] = key_ids[k];
            g_tag[g] = i;
            g_t[g] = (uint64_t)next;
            g_row[g] = k;
            g++;
            i++;
            next += gap(rng) * 1e9;
        }
        // one group call per run of consecutive pool rows (ciphertexts and
        // result rows both straight from the pool: no staging copy)
        size_t acc = 0;
        for (size_t a = 0; a < g;) {
            size_t b = a + 1;
            while (b < g && g_row[b] == g_row[b - 1] + 1)
                b++;
            size_t got = 0;
            const size_t k = g_row[a];
            const int rc = submit_group(srv, b - a, g_key.data() + a, cts + k * ct_stride, ct_stride,
                                        err_pool ? err_pool + k * err_stride : nullptr, err_pool ? err_stride : 0,
                                        g_tag.data() + a, g_t.data() + a, &got);
            if (rc != CMD_OK)
                return rc;
            acc += got;
            a = b;
        }
        (void)acc;
    }
    int rc = cmd_server_drain(srv, 60000);
    cmd_server_stats_get(srv, out, 0);
    out->offered_per_s = i / seconds;
    return rc;
}

}  // extern "C"
