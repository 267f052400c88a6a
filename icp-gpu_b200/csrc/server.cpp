// Serving loop: continuous batching of verify requests (include/bls_gpu.h,
// bls_server_*).
//
// The reference has no serving path: its IC integration collects shares into
// a thread-local batch and flushes it synchronously on the caller's thread
// (ic-integration/patches/ic-gpu-consensus.patch:286-403).  Here requests from
// any thread go into one queue; a dispatcher thread keeps `slots` launches in
// flight.  When a slot is free it takes every queued request that fits the
// slot (FIFO, up to max_batch_items), copies them into the slot's pinned
// buffers, and enqueues copy-in, the persistent verify (items claimed from the
// slot's device counter) and copy-out on the slot's stream.  Finished slots are
// found with cudaEventQuery; their results are copied into the requests'
// result buffers and the tickets are released.  A request arriving while the
// GPU works on earlier ones is admitted into the next free slot, so batches
// overlap on the device instead of waiting for each other.
//
// Admission: each slot's device buffers are sized for max_batch_items and
// counted against mem_cap_bytes at creation; the number of slots is reduced
// to what the budget admits.  Waits are bounded (timeouts), the dispatcher
// never spins on the device: it sleeps on a condition variable between polls.
//
// Ring mode (BLS_SERVE_RING): requests are written into host mirrors of a
// device ring of item slots (padded with identity items to whole groups of
// five for the five-item block shape; the twelve-warp shape claims any count
// up to 32, so nothing is padded); one copy stream moves each new range
// (inputs and sentinel results) to the device and then raises the
// published-item count in device memory.  One persistent launch of the
// six-lane kernel claims published items from a device counter as blocks
// free up and writes each result into the ring.  The dispatcher copies the
// results of the in-flight range back, sees a request complete when none of
// its result slots holds the sentinel any more, copies its results out and
// frees ring space in order.  Admission is by ring space.  The kernel leaves
// when idle for 20 ms, on destroy, or 60 s after its launch; the dispatcher
// relaunches it while work is left.  Compressed signatures are decoded on
// the device before their range is published, in rounds on decode streams of
// their own (struct Ring below has the rules).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <utility>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/bls_gpu.h"
#include "internal.h"

namespace bls {
CtxView ctx_view(bls_ctx* c);
}

namespace {

int64_t now_ns() {
    return std::chrono::duration_cast<std::chrono::nanoseconds>(std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

struct Pending {
    uint64_t ticket;
    int n;
    std::vector<uint8_t> sigs;
    std::vector<uint64_t> nhms;
    std::vector<int32_t> ids;
    int32_t* results;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    void *h_sigs = nullptr, *h_nhms = nullptr, *h_ids = nullptr, *h_res = nullptr;
    void *d_sigs = nullptr, *d_nhms = nullptr, *d_ids = nullptr, *d_res = nullptr, *d_xy = nullptr,
         *d_st = nullptr, *d_work = nullptr;
    bool busy = false;
    std::vector<Pending> reqs;
};

}  // namespace

// ring mode state: device ring and its host mirrors (same slot indexing)
struct Ring {
    uint32_t cap = 0;                      // item slots, a multiple of `group`
    uint32_t group = 1;                    // claim granule: 5 (five-item blocks, requests padded) or 1
    uint64_t *h_sigs = nullptr, *h_nhms = nullptr;   // pinned mirrors: cap x 12
    int32_t *h_ids = nullptr, *h_res = nullptr;      // cap
    uint32_t* h_ctl = nullptr;             // pinned: [0] published items, [1] stop
    // compressed signatures: 48-byte encodings in (pinned mirror and device),
    // decoded into d_sigs with a per-slot status before the range is
    // published; up to kDecStreams rounds decode at once, round r on
    // dec[r % kDecStreams], and each round's publication waits for the one
    // before it, so the published count only ever covers decoded slots
    static constexpr int kDecStreams = 4;
    cudaStream_t dec[kDecStreams] = {};
    cudaEvent_t dec_idle[kDecStreams] = {};   // recorded after a round's last decode work
    uint8_t *h_comp = nullptr, *d_comp = nullptr;
    int32_t* d_st = nullptr;
    // split decode (beside the twelve-warp kernel): a round is published once
    // its points are decoded and checked but for the subgroup test, which
    // then runs on the decoder's SMs while the kernel verifies; its outcome
    // per slot (0, or 4 for a point outside G1, kSentinel until known) comes
    // back beside the results and overrides a verify result
    bool split = false;
    int32_t *h_sub = nullptr, *d_sub = nullptr;
    uint64_t *d_sigs = nullptr, *d_nhms = nullptr;
    int32_t *d_ids = nullptr, *d_res = nullptr;
    uint32_t* d_ctl = nullptr;             // device: [0] published, [1] stop, [2] claimed
    cudaStream_t copy = nullptr, kern = nullptr;
    cudaStream_t poll = nullptr;           // result reads, apart from the copy stream's decodes
    cudaEvent_t done = nullptr;
    // Publications do not wait: round r copies its count from its own pinned
    // word (h_pubv[r % kPubSlots]) and records pub_ev[r % kPubSlots] after the
    // copy; `confirmed` is the count of the newest publication known to have
    // landed, and only [tail, confirmed) is ever read back (results beyond it
    // may still be a slot's earlier contents on the device).
    static constexpr int kPubSlots = 64;
    uint32_t* h_pubv = nullptr;
    cudaEvent_t pub_ev[kPubSlots] = {};
    std::deque<std::pair<int, uint32_t>> pub_pending;
    uint32_t confirmed = 0, pub_round = 0;
    bool launched = false;
    uint32_t pub = 0, tail = 0;            // items published / released (monotonic)
    struct Flight {
        Pending req;
        uint32_t start, span;
        bool complete;
    };
    std::deque<Flight> flights;
};
constexpr int32_t kSentinel = 0x7fffffff;
// SMs left free of the twelve-warp ring kernel for the decoder of compressed
// signatures.  The decoder takes one thread per point through a chain of
// about 1,300 multiplication-equivalents (the square root's 376 squarings
// and 85 products, the subgroup check's 127 doublings), about 2.3 ms, in
// whole-SM blocks of 384 threads; each decode round (up to kDecStreams in
// flight) takes at most kDecSmsPerRound SMs, so the decoder never holds more
// than the SMs set aside for it and the ring kernel's blocks always find
// theirs.  Three SMs retire about 1,150 points per 2.3 ms pass, 500 k/s, so
// the four rounds keep the decoder well ahead of the other 136 SMs' verify
// rate (about 7 k verifies/s per SM).
constexpr int kDecSmsPerRound = 3;
constexpr int kDecodeSms = Ring::kDecStreams * kDecSmsPerRound;
constexpr int kDecRoundItems = kDecSmsPerRound * 384;   // one pass of a round's decoder blocks

struct bls_server {
    bls_ctx* ctx = nullptr;
    Ring ring;
    bls_server_config cfg{};
    bls::CtxView view{};
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Pending> queue;
    std::unordered_map<uint64_t, int64_t> done;  // ticket -> completion time
    std::atomic<bool> stop{false};
    std::thread worker;
    uint64_t next_ticket = 1;
    uint64_t launches = 0, items = 0, max_batch = 0;
    int error = 0;

    size_t sig_bytes() const { return cfg.sig_format == BLS_SIG_COMPRESSED ? 48 : 96; }

    int launch(Slot& s) {
        size_t n = 0, sb = sig_bytes();
        for (auto& r : s.reqs) {
            memcpy((char*)s.h_sigs + n * sb, r.sigs.data(), r.n * sb);
            memcpy((char*)s.h_nhms + n * 96, r.nhms.data(), r.n * 96);
            memcpy((char*)s.h_ids + n * 4, r.ids.data(), r.n * 4);
            n += r.n;
        }
        cudaStream_t st = s.stream;
        if (cudaMemcpyAsync(s.d_sigs, s.h_sigs, n * sb, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(s.d_nhms, s.h_nhms, n * 96, cudaMemcpyHostToDevice, st) ||
            cudaMemcpyAsync(s.d_ids, s.h_ids, n * 4, cudaMemcpyHostToDevice, st) ||
            cudaMemsetAsync(s.d_work, 0, sizeof(int), st))
            return BLS_ERR_CUDA;
        bls::VerifyArgs a{};
        a.sigs = s.d_sigs;
        a.sig_compressed = cfg.sig_format == BLS_SIG_COMPRESSED;
        a.nhms = (const uint64_t*)s.d_nhms;
        a.g2 = view.g2;
        a.pk_tables = view.pk_tables;
        a.g2_norm = view.g2_norm;
        a.pk_norm = view.pk_norm;
        a.g2_corr = view.g2_corr;
        a.pk_corr = view.pk_corr;
        a.pk_index = (const int32_t*)s.d_ids;
        a.pk_identity = view.pk_identity;
        a.n = (int)n;
        a.results = (int32_t*)s.d_res;
        a.work_counter = (int*)s.d_work;
        const uint32_t* status = nullptr;
        if (a.sig_compressed) {
            if (bls::launch_g1_decompress((const uint8_t*)s.d_sigs, a.n, (uint64_t*)s.d_xy, (int32_t*)s.d_st, st))
                return BLS_ERR_CUDA;
            a.sig_xy = (const uint64_t*)s.d_xy;
            status = (const uint32_t*)s.d_st;
        }
        int lanes = view.lanes > 1 ? view.lanes : 6;
        if (bls::launch_verify_lanes(a, status, lanes, view.shape, view.blocks_per_sm, view.sms, st) ||
            cudaMemcpyAsync(s.h_res, s.d_res, n * 4, cudaMemcpyDeviceToHost, st) || cudaEventRecord(s.done, st))
            return BLS_ERR_CUDA;
        s.busy = true;
        ++launches;
        if (n > max_batch) max_batch = n;
        return BLS_OK;
    }

    void finish(Slot& s) {
        size_t off = 0;
        int64_t t = now_ns();
        for (auto& r : s.reqs) {
            memcpy(r.results, (const char*)s.h_res + off * 4, (size_t)r.n * 4);
            off += r.n;
            done[r.ticket] = t;
        }
        items += off;
        s.reqs.clear();
        s.busy = false;
    }

    // ---- ring mode
    int ring_launch() {
        bls::VerifyArgs a{};
        a.sigs = ring.d_sigs;
        if (ring.d_comp) a.sig_xy = ring.d_sigs;   // decoded by the dispatcher's decoder
        a.nhms = ring.d_nhms;
        a.g2 = view.g2;
        a.pk_tables = view.pk_tables;
        a.g2_norm = view.g2_norm;
        a.pk_norm = view.pk_norm;
        a.g2_corr = view.g2_corr;
        a.pk_corr = view.pk_corr;
        a.pk_index = ring.d_ids;
        a.pk_identity = view.pk_identity;
        a.n = 1;
        a.results = ring.d_res;
        a.serve_avail = ring.d_ctl;
        a.serve_stop = ring.d_ctl + 1;
        a.serve_claimed = ring.d_ctl + 2;
        a.serve_cap = ring.cap;
        a.serve_idle_ns = 20ull * 1000 * 1000;
        a.serve_max_ns = 60ull * 1000 * 1000 * 1000;
        int blocks = cfg.ring_blocks > 0 ? cfg.ring_blocks : cfg.ring_blocks_per_sm * view.sms;
        // the twelve-warp kernel fills its SMs: with compressed signatures a few
        // SMs stay free for the decoder, which runs beside the resident kernel
        if (ring.d_comp && view.shape == bls::kShapeWide && blocks > view.sms - kDecodeSms)
            blocks = view.sms - kDecodeSms;
        const uint32_t* st = (const uint32_t*)ring.d_st;
        const cudaError_t e = view.shape == bls::kShapeWide
                                  ? bls::launch_verify_w_serve(a, st, blocks, view.sms, ring.kern)
                                  : bls::launch_verify_fp2_serve(a, st, blocks, view.sms, ring.kern);
        if (e != cudaSuccess || cudaEventRecord(ring.done, ring.kern) != cudaSuccess) return BLS_ERR_CUDA;
        ring.launched = true;
        return BLS_OK;
    }

    // host mirror range [a, a + n) (ring positions, may wrap) to the device
    template <typename T>
    int ring_copy_in(T* dst, const T* src, size_t per, uint32_t a, uint32_t n, cudaStream_t st) {
        const uint32_t s0 = a % ring.cap, first = std::min(n, ring.cap - s0);
        if (cudaMemcpyAsync(dst + per * s0, src + per * s0, sizeof(T) * per * first, cudaMemcpyHostToDevice, st))
            return BLS_ERR_CUDA;
        if (first < n && cudaMemcpyAsync(dst, src, sizeof(T) * per * (n - first), cudaMemcpyHostToDevice, st))
            return BLS_ERR_CUDA;
        return BLS_OK;
    }

    // decode ring range [a, a + n) (may wrap) on stream st: the decoded
    // points into d_sigs, each slot's decode status into d_st.  Beside the
    // twelve-warp kernel, which leaves kDecodeSms SMs empty, the decoder runs
    // in whole-SM blocks, at most kDecSmsPerRound of them; the five-item
    // kernel's small blocks fill every SM but leave room for the plain
    // decoder's 128-thread blocks beside them, where a whole-SM block would
    // wait for the ring kernel to go idle.
    int ring_decode(uint32_t a, uint32_t n, cudaStream_t st) {
        const uint32_t s0 = a % ring.cap, first = std::min(n, ring.cap - s0);
        auto decode = [&](uint32_t from, uint32_t count) {
            return view.shape == bls::kShapeWide
                       ? bls::launch_g1_decompress_sms(ring.d_comp + 48 * (size_t)from, (int)count,
                                                       ring.d_sigs + 12 * (size_t)from, ring.d_st + from,
                                                       kDecSmsPerRound, !ring.split, st)
                       : bls::launch_g1_decompress(ring.d_comp + 48 * (size_t)from, (int)count,
                                                   ring.d_sigs + 12 * (size_t)from, ring.d_st + from, st);
        };
        if (decode(s0, first) || (first < n && decode(0, n - first))) return BLS_ERR_CUDA;
        return BLS_OK;
    }

    // the subgroup test of ring range [a, a + n) (split decode), on stream st
    int ring_subgroup(uint32_t a, uint32_t n, cudaStream_t st) {
        const uint32_t s0 = a % ring.cap, first = std::min(n, ring.cap - s0);
        auto check = [&](uint32_t from, uint32_t count) {
            return bls::launch_g1_subgroup_sms(ring.d_sigs + 12 * (size_t)from, ring.d_st + from, (int)count,
                                               ring.d_sub + from, kDecSmsPerRound, st);
        };
        if (check(s0, first) || (first < n && check(0, n - first))) return BLS_ERR_CUDA;
        return BLS_OK;
    }

    // One pass: results of the in-flight range, completions, admissions and
    // their publication, (re)launch; `progressed` when anything moved.  Only
    // the dispatcher thread touches the ring and its flights; the server mutex
    // (`lk`, held on entry and on return) guards the queue, the completion map
    // and the counters, and is released around every device round trip so
    // that submitters and waiters never queue behind a copy or a sync.
    int ring_step(std::unique_lock<std::mutex>& lk, bool& progressed) {
        lk.unlock();
        while (!ring.pub_pending.empty()) {   // publications that have landed
            const cudaError_t q = cudaEventQuery(ring.pub_ev[ring.pub_pending.front().first]);
            if (q == cudaErrorNotReady) break;
            if (q != cudaSuccess) {
                lk.lock();
                return BLS_ERR_CUDA;
            }
            ring.confirmed = ring.pub_pending.front().second;
            ring.pub_pending.pop_front();
        }
        const uint32_t inflight = ring.confirmed - ring.tail;
        if (inflight) {
            const uint32_t s0 = ring.tail % ring.cap, first = std::min(inflight, ring.cap - s0);
            if (cudaMemcpyAsync(ring.h_res + s0, ring.d_res + s0, 4 * (size_t)first, cudaMemcpyDeviceToHost,
                                ring.poll) ||
                (first < inflight && cudaMemcpyAsync(ring.h_res, ring.d_res, 4 * (size_t)(inflight - first),
                                                     cudaMemcpyDeviceToHost, ring.poll)) ||
                (ring.split &&
                 (cudaMemcpyAsync(ring.h_sub + s0, ring.d_sub + s0, 4 * (size_t)first, cudaMemcpyDeviceToHost,
                                  ring.poll) ||
                  (first < inflight && cudaMemcpyAsync(ring.h_sub, ring.d_sub, 4 * (size_t)(inflight - first),
                                                       cudaMemcpyDeviceToHost, ring.poll)))) ||
                cudaStreamSynchronize(ring.poll)) {
                lk.lock();
                return BLS_ERR_CUDA;
            }
        }
        const int64_t t = now_ns();
        std::vector<uint64_t> finished;
        uint64_t finished_items = 0;
        for (auto& f : ring.flights) {
            if (f.complete) continue;
            bool all = true;
            for (uint32_t k = f.span; k-- > 0;) {
                const uint32_t slot = (f.start + k) % ring.cap;
                if (ring.h_res[slot] == kSentinel || (ring.split && ring.h_sub[slot] == kSentinel)) {
                    all = false;
                    break;
                }
            }
            if (!all) continue;
            for (int k = 0; k < f.req.n; ++k) {
                const uint32_t slot = (f.start + k) % ring.cap;
                f.req.results[k] = ring.split && ring.h_sub[slot] != 0 ? -ring.h_sub[slot] : ring.h_res[slot];
            }
            finished.push_back(f.req.ticket);
            finished_items += f.req.n;
            f.complete = true;
        }
        while (!ring.flights.empty() && ring.flights.front().complete) {
            ring.tail += ring.flights.front().span;
            ring.flights.pop_front();
        }
        // completions out, admissions in: the only part under the mutex.  With
        // compressed signatures a round's decode takes one point's whole chain
        // (a few ms) whatever its size, so at most kDecStreams rounds are in
        // flight, each on its own stream: requests that arrive while all are
        // busy join the next round instead of queueing behind tiny ones.
        std::vector<Pending> admit;
        uint32_t room = ring.cap - (ring.pub - ring.tail);
        bool admitting = !(ring.h_comp && ring.pub_pending.size() >= (size_t)Ring::kDecStreams);
        if (admitting && ring.split) {   // the next round's stream has finished its last round's subgroup test
            const cudaError_t q = cudaEventQuery(ring.dec_idle[ring.pub_round % Ring::kDecStreams]);
            if (q != cudaSuccess && q != cudaErrorNotReady) {
                lk.lock();
                return BLS_ERR_CUDA;
            }
            admitting = q == cudaSuccess;
        }
        lk.lock();
        for (uint64_t tk : finished) done[tk] = t;
        items += finished_items;
        uint32_t round_items = 0;
        while (admitting && !queue.empty()) {
            const uint32_t span = ((uint32_t)queue.front().n + ring.group - 1) / ring.group * ring.group;
            if (span > room) break;
            // a decode round stays within one pass of its SMs (a larger request
            // goes alone): rounds of whatever is queued would hold the ring's
            // whole free space in a few long decodes while the verifier starves
            if (ring.h_comp && round_items > 0 && round_items + span > (uint32_t)kDecRoundItems) break;
            round_items += span;
            room -= span;
            if ((uint64_t)queue.front().n > max_batch) max_batch = queue.front().n;
            admit.push_back(std::move(queue.front()));
            queue.pop_front();
        }
        lk.unlock();
        if (!finished.empty()) {
            cv_done.notify_all();
            progressed = true;
        }
        const uint32_t from = ring.pub;
        for (Pending& q : admit) {
            const uint32_t span = ((uint32_t)q.n + ring.group - 1) / ring.group * ring.group;
            for (uint32_t k = 0; k < span; ++k) {
                const uint32_t slot = (ring.pub + k) % ring.cap;
                ring.h_res[slot] = kSentinel;
                if (ring.split) ring.h_sub[slot] = kSentinel;
                if (k < (uint32_t)q.n) {
                    if (ring.h_comp)
                        memcpy(ring.h_comp + 48 * (size_t)slot, q.sigs.data() + 48 * (size_t)k, 48);
                    else
                        memcpy(ring.h_sigs + 12 * (size_t)slot, q.sigs.data() + 96 * (size_t)k, 96);
                    memcpy(ring.h_nhms + 12 * (size_t)slot, q.nhms.data() + 12 * (size_t)k, 96);
                    ring.h_ids[slot] = q.ids[k];
                } else {  // padding: identity points, key 0 (both pairs skipped)
                    if (ring.h_comp) {
                        memset(ring.h_comp + 48 * (size_t)slot, 0, 48);
                        ring.h_comp[48 * (size_t)slot] = 0xc0;   // the identity's encoding
                    } else {
                        memset(ring.h_sigs + 12 * (size_t)slot, 0, 96);
                    }
                    memset(ring.h_nhms + 12 * (size_t)slot, 0, 96);
                    ring.h_ids[slot] = 0;
                }
            }
            ring.flights.push_back(Ring::Flight{std::move(q), ring.pub, span, false});
            ring.pub += span;
        }
        int rc = BLS_OK;
        if (ring.pub != from) {
            const uint32_t n = ring.pub - from;
            const int dec_i = (int)(ring.pub_round % Ring::kDecStreams);
            const cudaStream_t st = ring.h_comp ? ring.dec[dec_i] : ring.copy;
            if ((ring.h_comp ? (rc = ring_copy_in(ring.d_comp, ring.h_comp, 48, from, n, st)) ||
                                   (ring.split && (rc = ring_copy_in(ring.d_sub, ring.h_sub, 1, from, n, st))) ||
                                   (rc = ring_decode(from, n, st))
                             : (rc = ring_copy_in(ring.d_sigs, ring.h_sigs, 12, from, n, st))) ||
                (rc = ring_copy_in(ring.d_nhms, ring.h_nhms, 12, from, n, st)) ||
                (rc = ring_copy_in(ring.d_ids, ring.h_ids, 1, from, n, st)) ||
                (rc = ring_copy_in(ring.d_res, ring.h_res, 1, from, n, st))) {
                lk.lock();
                return rc;
            }
            // the count goes up only after the items' copies (and decode) on the
            // same stream; nothing waits for it here
            if ((int)ring.pub_pending.size() == Ring::kPubSlots) {   // every word in use: wait for the oldest
                if (cudaEventSynchronize(ring.pub_ev[ring.pub_pending.front().first]) != cudaSuccess) {
                    lk.lock();
                    return BLS_ERR_CUDA;
                }
                ring.confirmed = ring.pub_pending.front().second;
                ring.pub_pending.pop_front();
            }
            const int slot = (int)(ring.pub_round++ % Ring::kPubSlots);
            ring.h_pubv[slot] = ring.pub;
            // counts land in order: a decode round's count after the round before it
            if ((st != ring.copy && !ring.pub_pending.empty() &&
                 cudaStreamWaitEvent(st, ring.pub_ev[ring.pub_pending.back().first], 0)) ||
                cudaMemcpyAsync(ring.d_ctl, ring.h_pubv + slot, 4, cudaMemcpyHostToDevice, st) ||
                cudaEventRecord(ring.pub_ev[slot], st)) {
                lk.lock();
                return BLS_ERR_CUDA;
            }
            ring.pub_pending.emplace_back(slot, ring.pub);
            // split decode: the subgroup test after the publication, while the kernel verifies
            if (ring.split && (ring_subgroup(from, n, st) || cudaEventRecord(ring.dec_idle[dec_i], st))) {
                lk.lock();
                return BLS_ERR_CUDA;
            }
            progressed = true;
        }
        bool pending = false, relaunched = false;
        for (auto& f : ring.flights) pending = pending || !f.complete;
        if (pending && !(ring.launched && cudaEventQuery(ring.done) == cudaErrorNotReady)) {
            rc = ring_launch();
            relaunched = rc == BLS_OK;
            progressed = true;
        }
        lk.lock();
        if (relaunched) ++launches;
        return rc;
    }

    void run_ring() {
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            bool progressed = false;
            int rc = ring_step(lk, progressed);
            if (rc) {
                error = rc;
                cv_done.notify_all();
                return;
            }
            if (stop && queue.empty() && ring.flights.empty()) break;
            if (!progressed) cv_work.wait_for(lk, std::chrono::microseconds(ring.flights.empty() ? 2000 : 20));
        }
        lk.unlock();
        ring_stop();
    }

    void ring_stop() {
        if (!ring.h_ctl || !ring.d_ctl) return;
        ring.h_ctl[1] = 1;
        for (cudaStream_t st : ring.dec)
            if (st) cudaStreamSynchronize(st);
        cudaMemcpyAsync(ring.d_ctl + 1, ring.h_ctl + 1, 4, cudaMemcpyHostToDevice, ring.copy);
        cudaStreamSynchronize(ring.copy);
        if (ring.kern) cudaStreamSynchronize(ring.kern);
    }

    void run() {
        if (cudaSetDevice(view.device) != cudaSuccess) {
            std::lock_guard<std::mutex> lk(mu);
            error = BLS_ERR_CUDA;
            cv_done.notify_all();
            return;
        }
        if (cfg.mode == BLS_SERVE_RING) {
            run_ring();
            return;
        }
        std::unique_lock<std::mutex> lk(mu);
        while (true) {
            bool any_busy = false, progressed = false;
            for (auto& s : slots) {
                if (s.busy && cudaEventQuery(s.done) == cudaSuccess) {
                    finish(s);
                    progressed = true;
                }
                any_busy = any_busy || s.busy;
            }
            if (progressed) cv_done.notify_all();
            for (auto& s : slots) {
                if (s.busy || queue.empty()) continue;
                size_t n = 0;
                while (!queue.empty() && n + (size_t)queue.front().n <= (size_t)cfg.max_batch_items) {
                    n += queue.front().n;
                    s.reqs.push_back(std::move(queue.front()));
                    queue.pop_front();
                }
                if (s.reqs.empty()) continue;
                int rc = launch(s);
                if (rc) {
                    error = rc;
                    cv_done.notify_all();
                    return;
                }
                any_busy = true;
            }
            if (stop && queue.empty() && !any_busy) return;
            // sleep until new work arrives or a short poll interval passes
            cv_work.wait_for(lk, std::chrono::microseconds(any_busy ? 50 : 2000));
        }
    }
};

extern "C" {

int bls_server_create(bls_ctx* ctx, const bls_server_config* cfg, bls_server** out) {
    if (!ctx || !out) return BLS_ERR_INVALID;
    *out = nullptr;
    auto* s = new bls_server();
    s->ctx = ctx;
    if (cfg) s->cfg = *cfg;
    if (s->cfg.slots <= 0) s->cfg.slots = 3;
    if (s->cfg.max_batch_items <= 0) s->cfg.max_batch_items = 16384;
    if (s->cfg.mem_cap_bytes == 0) s->cfg.mem_cap_bytes = (size_t)4 << 30;
    if ((s->cfg.sig_format != BLS_SIG_AFFINE && s->cfg.sig_format != BLS_SIG_COMPRESSED) ||
        (s->cfg.mode != BLS_SERVE_SLOTS && s->cfg.mode != BLS_SERVE_RING) ||
        s->cfg.ring_items < 0 ||
        s->cfg.ring_blocks_per_sm < 0 || s->cfg.ring_blocks < 0) {
        delete s;
        return BLS_ERR_INVALID;
    }
    s->view = bls::ctx_view(ctx);
    if (cudaSetDevice(s->view.device) != cudaSuccess) {
        delete s;
        return BLS_ERR_CUDA;
    }
    if (s->cfg.mode == BLS_SERVE_RING) {
        if (s->view.lanes != 6 && s->view.lanes != 0) {  // the ring is served by the six-lane kernel
            delete s;
            return BLS_ERR_INVALID;
        }
        Ring& r = s->ring;
        // resident blocks: the twelve-warp kernel holds a whole SM per block; the
        // five-item kernel defaults to 4 of its 6 blocks per SM (the latency choice)
        if (s->cfg.ring_blocks_per_sm == 0) s->cfg.ring_blocks_per_sm = s->view.shape == bls::kShapeWide ? 1 : 4;
        const int most = bls::verify_lanes_blocks_per_sm(6, s->view.shape);
        if (most > 0 && s->cfg.ring_blocks_per_sm > most) s->cfg.ring_blocks_per_sm = most;
        uint64_t cap = s->cfg.ring_items > 0 ? (uint64_t)s->cfg.ring_items : 65535u;
        r.group = s->view.shape == bls::kShapeWide ? 1u : 5u;
        const uint64_t least = (uint64_t)s->cfg.max_batch_items + 2 * r.group;
        if (cap < least) cap = least;
        cap = (cap + r.group - 1) / r.group * r.group;
        const bool comp = s->cfg.sig_format == BLS_SIG_COMPRESSED;
        r.split = comp && s->view.shape == bls::kShapeWide;
        if (cap * (comp ? 256 : 200) + 64 > s->cfg.mem_cap_bytes || cap > (1u << 30)) {
            delete s;
            return BLS_ERR_NOMEM;
        }
        r.cap = (uint32_t)cap;
        bool ok = cudaHostAlloc((void**)&r.h_sigs, cap * 96, 0) == cudaSuccess &&
                  cudaHostAlloc((void**)&r.h_nhms, cap * 96, 0) == cudaSuccess &&
                  cudaHostAlloc((void**)&r.h_ids, cap * 4, 0) == cudaSuccess &&
                  cudaHostAlloc((void**)&r.h_res, cap * 4, 0) == cudaSuccess &&
                  cudaHostAlloc((void**)&r.h_ctl, 64, 0) == cudaSuccess &&
                  cudaMalloc((void**)&r.d_sigs, cap * 96) == cudaSuccess &&
                  cudaMalloc((void**)&r.d_nhms, cap * 96) == cudaSuccess &&
                  cudaMalloc((void**)&r.d_ids, cap * 4) == cudaSuccess &&
                  cudaMalloc((void**)&r.d_res, cap * 4) == cudaSuccess &&
                  cudaMalloc((void**)&r.d_ctl, 64) == cudaSuccess && cudaMemset(r.d_ctl, 0, 64) == cudaSuccess &&
                  (!comp || (cudaHostAlloc((void**)&r.h_comp, cap * 48, 0) == cudaSuccess &&
                             cudaMalloc((void**)&r.d_comp, cap * 48) == cudaSuccess &&
                             cudaMalloc((void**)&r.d_st, cap * 4) == cudaSuccess)) &&
                  (!r.split || (cudaHostAlloc((void**)&r.h_sub, cap * 4, 0) == cudaSuccess &&
                                cudaMalloc((void**)&r.d_sub, cap * 4) == cudaSuccess)) &&
                  cudaStreamCreateWithFlags(&r.copy, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&r.poll, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaHostAlloc((void**)&r.h_pubv, 4 * Ring::kPubSlots, 0) == cudaSuccess &&
                  cudaStreamCreateWithFlags(&r.kern, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&r.done, cudaEventDisableTiming) == cudaSuccess &&
                  cudaDeviceSynchronize() == cudaSuccess;
        for (int k = 0; ok && k < Ring::kPubSlots; ++k)
            ok = cudaEventCreateWithFlags(&r.pub_ev[k], cudaEventDisableTiming) == cudaSuccess;
        for (int k = 0; ok && comp && k < Ring::kDecStreams; ++k)
            ok = cudaStreamCreateWithFlags(&r.dec[k], cudaStreamNonBlocking) == cudaSuccess &&
                 cudaEventCreateWithFlags(&r.dec_idle[k], cudaEventDisableTiming) == cudaSuccess;
        if (ok) memset(r.h_ctl, 0, 64);
        if (!ok) {
            bls_server_destroy(s);
            return BLS_ERR_NOMEM;
        }
        bls::verify_lanes_blocks_per_sm(6, s->view.shape);
        s->worker = std::thread([s] { s->run(); });
        *out = s;
        return BLS_OK;
    }
    size_t m = (size_t)s->cfg.max_batch_items;
    size_t per_slot = m * (s->sig_bytes() + 96 + 4 + 4 + 96 + 4) + 256;
    int admitted = (int)(s->cfg.mem_cap_bytes / per_slot);
    if (admitted < 1) {
        delete s;
        return BLS_ERR_NOMEM;
    }
    if (s->cfg.slots > admitted) s->cfg.slots = admitted;
    s->slots.resize(s->cfg.slots);
    for (auto& sl : s->slots) {
        bool ok = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking) == cudaSuccess &&
                  cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming) == cudaSuccess &&
                  cudaHostAlloc(&sl.h_sigs, m * s->sig_bytes(), 0) == cudaSuccess &&
                  cudaHostAlloc(&sl.h_nhms, m * 96, 0) == cudaSuccess && cudaHostAlloc(&sl.h_ids, m * 4, 0) == cudaSuccess &&
                  cudaHostAlloc(&sl.h_res, m * 4, 0) == cudaSuccess && cudaMalloc(&sl.d_sigs, m * s->sig_bytes()) == cudaSuccess &&
                  cudaMalloc(&sl.d_nhms, m * 96) == cudaSuccess && cudaMalloc(&sl.d_ids, m * 4) == cudaSuccess &&
                  cudaMalloc(&sl.d_res, m * 4) == cudaSuccess && cudaMalloc(&sl.d_xy, m * 96) == cudaSuccess &&
                  cudaMalloc(&sl.d_st, m * 4) == cudaSuccess && cudaMalloc(&sl.d_work, 256) == cudaSuccess;
        if (!ok) {
            bls_server_destroy(s);
            return BLS_ERR_NOMEM;
        }
    }
    // set up the kernel (shared-memory size, occupancy) before serving
    bls::verify_lanes_blocks_per_sm(s->view.lanes > 1 ? s->view.lanes : 6, s->view.shape);
    s->worker = std::thread([s] { s->run(); });
    *out = s;
    return BLS_OK;
}

void bls_server_destroy(bls_server* s) {
    if (!s) return;
    if (s->worker.joinable()) {
        {
            std::lock_guard<std::mutex> lk(s->mu);
            s->stop = true;
        }
        s->cv_work.notify_all();
        s->worker.join();
    }
    cudaSetDevice(s->view.device);
    {
        Ring& r = s->ring;
        s->ring_stop();
        for (void* p : {(void*)r.h_sigs, (void*)r.h_nhms, (void*)r.h_ids, (void*)r.h_res, (void*)r.h_ctl,
                        (void*)r.h_comp, (void*)r.h_pubv, (void*)r.h_sub})
            if (p) cudaFreeHost(p);
        for (cudaEvent_t ev : r.pub_ev)
            if (ev) cudaEventDestroy(ev);
        if (r.poll) cudaStreamDestroy(r.poll);
        for (cudaStream_t st : r.dec)
            if (st) cudaStreamDestroy(st);
        for (cudaEvent_t ev : r.dec_idle)
            if (ev) cudaEventDestroy(ev);
        for (void* p : {(void*)r.d_sigs, (void*)r.d_nhms, (void*)r.d_ids, (void*)r.d_res, (void*)r.d_ctl,
                        (void*)r.d_comp, (void*)r.d_st, (void*)r.d_sub})
            if (p) cudaFree(p);
        if (r.done) cudaEventDestroy(r.done);
        if (r.copy) cudaStreamDestroy(r.copy);
        if (r.kern) cudaStreamDestroy(r.kern);
    }
    for (auto& sl : s->slots) {
        if (sl.stream) cudaStreamSynchronize(sl.stream);
        for (void* p : {sl.h_sigs, sl.h_nhms, sl.h_ids, sl.h_res})
            if (p) cudaFreeHost(p);
        for (void* p : {sl.d_sigs, sl.d_nhms, sl.d_ids, sl.d_res, sl.d_xy, sl.d_st, sl.d_work})
            if (p) cudaFree(p);
        if (sl.done) cudaEventDestroy(sl.done);
        if (sl.stream) cudaStreamDestroy(sl.stream);
    }
    delete s;
}

int bls_server_submit(bls_server* s, const bls_request* r, uint64_t* ticket, int64_t* submit_ns) {
    if (!s || !r || !ticket) return BLS_ERR_INVALID;
    if (r->n <= 0 || r->n > s->cfg.max_batch_items) return BLS_ERR_INVALID;
    if (!r->sigs || !r->neg_hms || !r->pk_ids || !r->results) return BLS_ERR_INVALID;
    for (int i = 0; i < r->n; ++i)
        if (r->pk_ids[i] < 0 || r->pk_ids[i] >= s->view.n_pks) return BLS_ERR_INVALID;
    Pending p;
    p.n = r->n;
    p.sigs.assign((const uint8_t*)r->sigs, (const uint8_t*)r->sigs + (size_t)r->n * s->sig_bytes());
    p.nhms.assign(r->neg_hms, r->neg_hms + (size_t)r->n * 12);
    p.ids.assign(r->pk_ids, r->pk_ids + r->n);
    p.results = r->results;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->error) return s->error;
        p.ticket = s->next_ticket++;
        *ticket = p.ticket;
        if (submit_ns) *submit_ns = now_ns();
        s->queue.push_back(std::move(p));
    }
    s->cv_work.notify_one();
    return BLS_OK;
}

int bls_server_wait(bls_server* s, uint64_t ticket, int timeout_ms, int64_t* done_ns) {
    if (!s) return BLS_ERR_INVALID;
    std::unique_lock<std::mutex> lk(s->mu);
    auto ready = [&] { return s->error != 0 || s->done.count(ticket) != 0; };
    if (timeout_ms < 0) {
        s->cv_done.wait(lk, ready);
    } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
        return BLS_ERR_TIMEOUT;
    }
    if (s->error) return s->error;
    auto it = s->done.find(ticket);
    if (done_ns) *done_ns = it->second;
    s->done.erase(it);
    return BLS_OK;
}

int bls_server_stats(bls_server* s, uint64_t* launches, uint64_t* items, uint64_t* max_batch) {
    if (!s) return BLS_ERR_INVALID;
    std::lock_guard<std::mutex> lk(s->mu);
    if (launches) *launches = s->launches;
    if (items) *items = s->items;
    if (max_batch) *max_batch = s->max_batch;
    return BLS_OK;
}

}  // extern "C"
