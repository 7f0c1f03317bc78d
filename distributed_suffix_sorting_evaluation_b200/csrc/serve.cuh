// Serving: continuous batching of SA requests on one GPU.
//
// The reference builds one SA per process run (cli.cpp:747-820); it has no
// request loop.  This server keeps the DCX pipeline of build_batch as its unit
// of work and adds what a long-running service needs:
//   * requests are copied at submission and queued in arrival order;
//   * L lanes (threads, each with its own stream and scratch context) take
//     work whenever they are free, so requests arriving while other batches
//     run start at once on a free lane and overlap with them on the device;
//     lane 0 (bulk) takes the long requests, the others (express, on
//     high-priority streams) the short ones, so long builds never contend with
//     each other and short ones never queue behind them; the bulk lane uploads
//     its next batch while it builds the current one;
//   * a lane admits the queued requests of one (dc, sa_width) class, first come
//     first served, while their projected footprint fits the HBM budget and the
//     batch stays under a text-byte cap; a request that does not fit waits for
//     memory to be released (results count until dcx_serve_release);
//   * results stay on the device until the caller polls (copy to host) and
//     releases them.
// Every result is the SA build_batch computes for that text alone, because a
// text's SA does not depend on the other texts of its batch (the text id is
// the most significant key digit and every per-text quantity is segment-local).
#pragma once

#include <chrono>
#include <condition_variable>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace dcx {

// Device bytes a request may hold while its batch runs: the build scratch
// (build_batch plans 48 bytes per element), the device copy of the text and
// the result.  The result part stays reserved until the request is released.
static uint64_t serve_scratch_bytes(uint64_t n) { return 48 * (n + 1) + (1ull << 20); }
static uint64_t serve_result_bytes(uint64_t n, int width) { return ((n * (uint64_t)(width / 8)) + 16 + 255) & ~255ull; }
static uint64_t serve_footprint(uint64_t n, int width) {
    return serve_scratch_bytes(n) + ((n + 16 + 255) & ~255ull) + serve_result_bytes(n, width);
}

static void ctx_init(Ctx& c, int device, uint64_t budget);
static void ctx_free(Ctx& c);

// Pinned host arena for the request copies, so a lane's upload is a DMA at
// link speed rather than a staged pageable copy.  First fit over a free list
// with coalescing; a request that does not fit falls back to pageable memory.
class PinnedArena {
public:
    explicit PinnedArena(uint64_t bytes) {
        if (bytes && cudaHostAlloc((void**)&base_, bytes, cudaHostAllocDefault) == cudaSuccess) {
            size_ = bytes;
            free_[0] = bytes;
        } else {
            cudaGetLastError();
            base_ = nullptr;
        }
    }
    ~PinnedArena() {
        if (base_) cudaFreeHost(base_);
    }
    uint8_t* alloc(uint64_t n) {
        n = (std::max<uint64_t>(n, 1) + 255) & ~255ull;
        std::lock_guard<std::mutex> lk(mu_);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            const uint64_t off = it->first, sz = it->second;
            free_.erase(it);
            if (sz > n) free_[off + n] = sz - n;
            used_[off] = n;
            return base_ + off;
        }
        return nullptr;
    }
    bool owns(const uint8_t* p) const { return base_ && p >= base_ && p < base_ + size_; }
    void free(const uint8_t* p) {
        std::lock_guard<std::mutex> lk(mu_);
        const uint64_t off = (uint64_t)(p - base_);
        auto u = used_.find(off);
        if (u == used_.end()) return;
        uint64_t o = off, sz = u->second;
        used_.erase(u);
        auto nx = free_.lower_bound(o);
        if (nx != free_.end() && nx->first == o + sz) {  // merge with the next free block
            sz += nx->second;
            nx = free_.erase(nx);
        }
        if (nx != free_.begin()) {  // merge with the previous free block
            auto pv = std::prev(nx);
            if (pv->first + pv->second == o) {
                pv->second += sz;
                return;
            }
        }
        free_[o] = sz;
    }

private:
    uint8_t* base_ = nullptr;
    uint64_t size_ = 0;
    std::mutex mu_;
    std::map<uint64_t, uint64_t> free_, used_;
};

// Host copy of a request text: large texts are split over a few threads, since
// one core's memcpy would bound the submission rate well below the GPU's.
static void parallel_copy(uint8_t* dst, const uint8_t* src, uint64_t n) {
    constexpr uint64_t PIECE = 8ull << 20;
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    const uint64_t parts = std::min<uint64_t>(std::min<uint64_t>(8, hw), n / PIECE);
    if (parts <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const uint64_t step = ((n + parts - 1) / parts + 4095) & ~4095ull;
    std::vector<std::thread> th;
    for (uint64_t b = step; b < n; b += step)
        th.emplace_back([=] { memcpy(dst + b, src + b, std::min(step, n - b)); });
    memcpy(dst, src, std::min(step, n));
    for (auto& t : th) t.join();
}

// A batch's result buffer, shared by its requests; freed with the last of them.
struct ServeResult {
    void* p = nullptr;
    uint64_t bytes = 0;
    cudaStream_t stream = nullptr;
    uint32_t refs = 0;  // requests not yet released (guarded by the server mutex)
    ~ServeResult() {
        if (p) cudaFreeAsync(p, stream);
    }
};

struct ServeReq {
    uint64_t id = 0;
    std::unique_ptr<uint8_t[]> text;  // pageable host copy (when the pinned arena is full)
    const uint8_t* pinned = nullptr;  // pinned host copy in the server's arena
    const uint8_t* borrowed = nullptr;  // caller's buffer (DCX_SERVE_BORROW), host or device
    bool borrowed_dev = false;
    uint64_t n = 0;
    int dc = 0, width = 32;
    uint64_t footprint = 0;
    int status = 0;  // 0 queued, 1 running, 2 done, < 0 failed (error code)
    int lane = -1;
    std::chrono::steady_clock::time_point t_submit, t_start, t_done;
    std::shared_ptr<ServeResult> res;
    uint64_t res_off = 0;  // byte offset of this request's SA in res
};

class Server {
public:
    Server(const Ctx& parent, int lanes, uint64_t budget, uint64_t batch_bytes, uint32_t batch_texts,
           uint64_t host_bytes, uint64_t express_bytes, bool express_priority)
        : device_(parent.device), budget_(budget), batch_bytes_(batch_bytes), batch_texts_(batch_texts),
          express_bytes_(express_bytes), express_batch_bytes_(std::max<uint64_t>(4 * express_bytes, 1 << 20)),
          arena_(host_bytes) {
        st_.lanes = (uint32_t)lanes;
        st_.budget_bytes = budget;
        for (int k = 0; k < lanes; k++) {
            auto c = std::make_unique<Ctx>();
            ctx_init(*c, device_, 0);
            c->opt = parent.opt;
            c->opt.trace = 0;
            // Each lane allocates from its own pool: a shared pool would hand one
            // lane's freed block to another and make its stream wait for the
            // first lane's work, serialising the lanes.
            cudaMemPoolProps props{};
            props.allocType = cudaMemAllocationTypePinned;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = device_;
            DCX_CUDA(cudaMemPoolCreate(&c->pool, &props));
            uint64_t thr = UINT64_MAX;
            DCX_CUDA(cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr));
            if (k > 0 && express_priority) {  // express lanes: short builds get the SMs first
                int least = 0, greatest = 0;
                DCX_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
                DCX_CUDA(cudaStreamDestroy(c->stream));
                DCX_CUDA(cudaStreamCreateWithPriority(&c->stream, cudaStreamNonBlocking, greatest));
            }
            cudaStream_t cs;
            DCX_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
            copy_streams_.push_back(cs);
            lanes_.push_back(std::move(c));
        }
        DCX_CUDA(cudaStreamCreateWithFlags(&copy_stream_, cudaStreamNonBlocking));
        for (int k = 0; k < lanes; k++) threads_.emplace_back([this, k] { lane_main(k); });
    }

    ~Server() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        cv_work_.notify_all();
        for (auto& t : threads_) t.join();
        reqs_.clear();  // frees the results on their lanes' streams
        for (size_t k = 0; k < lanes_.size(); k++) {
            Ctx& c = *lanes_[k];
            cudaStreamSynchronize(copy_streams_[k]);
            cudaStreamSynchronize(c.stream);
            cudaStreamDestroy(copy_streams_[k]);
            cudaMemPool_t pool = c.pool;
            ctx_free(c);
            if (pool) cudaMemPoolDestroy(pool);
        }
        cudaStreamDestroy(copy_stream_);
    }

    uint64_t submit(const uint8_t* text, uint64_t n, int dc, int width, uint32_t flags) {
        if (n >= 0xffffffffull) throw Error(DCX_ERR_ARG, "text longer than 2^32 - 2");
        if (!(width == 32 || width == 40 || width == 64)) throw Error(DCX_ERR_ARG, "sa_width must be 32, 40 or 64");
        if (n && !text) throw Error(DCX_ERR_ARG, "null pointer");
        if (dc != 0) {
            DcHost h;
            if (!make_dc((uint32_t)dc, h)) throw Error(DCX_ERR_ARG, "unsupported difference cover");
        }
        const auto t_submit = std::chrono::steady_clock::now();
        const uint64_t fp = serve_footprint(n, width);
        if (fp > budget_) throw Error(DCX_ERR_BUDGET, "request footprint above the serving budget");
        auto r = std::make_unique<ServeReq>();
        if (flags & DCX_SERVE_BORROW) {
            r->borrowed = text;
            r->borrowed_dev = (flags & DCX_DEVICE_PTRS) != 0;
        } else if (flags & DCX_DEVICE_PTRS) {
            throw Error(DCX_ERR_ARG, "device texts are served only with DCX_SERVE_BORROW");
        } else if (uint8_t* h = n ? arena_.alloc(n) : nullptr) {
            parallel_copy(h, text, n);
            r->pinned = h;
        } else if (n) {
            r->text.reset(new uint8_t[n]);
            parallel_copy(r->text.get(), text, n);
        }
        r->n = n;
        r->dc = dc;
        r->width = width;
        r->footprint = fp;
        r->t_submit = t_submit;
        uint64_t id;
        {
            std::lock_guard<std::mutex> lk(mu_);
            if (stop_) throw Error(DCX_ERR_INTERNAL, "server stopped");
            id = next_id_++;
            r->id = id;
            queue_.push_back(id);
            reqs_[id] = std::move(r);
            st_.submitted++;
        }
        cv_work_.notify_one();
        return id;
    }

    // status / latency; copies the SA to sa_host when done and sa_host != null
    void poll(uint64_t id, void* sa_host, int* status, double* latency_ms) {
        std::shared_ptr<ServeResult> res;
        uint64_t off = 0, bytes = 0;
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = reqs_.find(id);
            if (it == reqs_.end()) throw Error(DCX_ERR_NOTFOUND, "unknown or released request");
            ServeReq& r = *it->second;
            if (status) *status = r.status;
            if (latency_ms)
                *latency_ms = r.status == 2 ? std::chrono::duration<double, std::milli>(r.t_done - r.t_submit).count()
                                            : 0.0;
            if (r.status != 2 || !sa_host) return;
            res = r.res;
            off = r.res_off;
            bytes = r.n * (uint64_t)(r.width / 8);
        }
        if (bytes) {
            std::lock_guard<std::mutex> lk(copy_mu_);
            DCX_CUDA(cudaSetDevice(device_));
            DCX_CUDA(cudaMemcpyAsync(sa_host, (const uint8_t*)res->p + off, bytes, cudaMemcpyDeviceToHost, copy_stream_));
            DCX_CUDA(cudaStreamSynchronize(copy_stream_));
        }
    }

    const void* result_device(uint64_t id) {
        std::lock_guard<std::mutex> lk(mu_);
        auto it = reqs_.find(id);
        if (it == reqs_.end()) throw Error(DCX_ERR_NOTFOUND, "unknown or released request");
        if (it->second->status != 2) throw Error(DCX_ERR_BUSY, "request not done");
        if (!it->second->res) return nullptr;
        return (const uint8_t*)it->second->res->p + it->second->res_off;
    }

    void release(uint64_t id) {
        std::shared_ptr<ServeResult> drop;  // freed outside the lock
        {
            std::lock_guard<std::mutex> lk(mu_);
            auto it = reqs_.find(id);
            if (it == reqs_.end()) throw Error(DCX_ERR_NOTFOUND, "unknown or released request");
            ServeReq& r = *it->second;
            if (r.status == 0 || r.status == 1) throw Error(DCX_ERR_BUSY, "request still queued or running");
            if (r.res && --r.res->refs == 0) {
                reserved_ -= r.res->bytes;
                drop = r.res;
            }
            reqs_.erase(it);
        }
        cv_work_.notify_all();
    }

    // Waits until nothing is queued or running.  Throws DCX_ERR_BUDGET when the
    // queue cannot move: nothing runs and the first request does not fit because
    // unreleased results hold the budget.
    void drain() {
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return (queue_.empty() && running_ == 0) || stalled(); });
        if (!queue_.empty())
            throw Error(DCX_ERR_BUDGET, "queued requests wait for results to be released");
    }

    dcx_serve_stats stats() {
        std::lock_guard<std::mutex> lk(mu_);
        dcx_serve_stats s = st_;
        s.reserved_bytes = reserved_;
        s.queued = queue_.size();
        s.running_batches = running_;
        return s;
    }

private:
    // Lane 0 is the bulk lane: it serves the requests longer than express_bytes
    // (every request when it is the only lane).  Lanes 1.. are express lanes:
    // they serve only requests of at most express_bytes.  Each class is served
    // in arrival order; short requests never wait behind long batches, and long
    // builds never run two at a time and contend for the GPU.
    bool admissible(int lane, const ServeReq& r) const {
        if (lanes_.size() == 1) return true;
        return lane == 0 ? r.n > express_bytes_ : r.n <= express_bytes_;
    }

    // First queued request lane `lane` may start now (it fits the budget), or null.
    const ServeReq* first_for(int lane) const {
        for (uint64_t id : queue_) {
            const ServeReq& r = *reqs_.at(id);
            if (!admissible(lane, r)) continue;
            return reserved_ + r.footprint <= budget_ ? &r : nullptr;  // first come, first served
        }
        return nullptr;
    }

    bool stalled() const {
        if (queue_.empty() || running_ != 0) return false;
        for (int k = 0; k < (int)lanes_.size(); k++)
            if (first_for(k)) return false;
        return true;
    }

    // A batch taken from the queue: its requests, reserved scratch and (once
    // uploaded) the device copy of its texts.
    struct Batch {
        std::vector<ServeReq*> reqs;
        uint64_t scratch = 0;
        std::vector<uint64_t> offs;
        void* d_text = nullptr;
        cudaEvent_t ev_up0 = nullptr, ev_up1 = nullptr;  // around the upload (copy stream)
        int err = DCX_OK;
        bool empty() const { return reqs.empty(); }
    };

    // Takes the queued requests lane k may start now (one (dc, width) class,
    // arrival order, within the budget and the lane's batch cap).  `block`:
    // wait for work; otherwise return an empty batch when none is ready.
    // Returns false only when the server stops.
    bool admit(int k, bool block, Batch& b) {
        {
            std::unique_lock<std::mutex> lk(mu_);
            if (block) cv_work_.wait(lk, [&] { return stop_ || first_for(k) != nullptr; });
            if (stop_) return false;
            const ServeReq* head = first_for(k);
            if (!head) return true;
            const int dc = head->dc, width = head->width;
            const uint64_t cap = k == 0 ? batch_bytes_ : std::min(batch_bytes_, express_batch_bytes_);
            uint64_t text_bytes = 0;
            for (auto it = queue_.begin(); it != queue_.end();) {
                ServeReq* r = reqs_.at(*it).get();
                if (r->dc != dc || r->width != width || !admissible(k, *r)) {  // left for another lane
                    ++it;
                    continue;
                }
                if (!b.reqs.empty() && (text_bytes + r->n > cap || b.reqs.size() >= batch_texts_)) break;
                // a long text is built alone: one text per sort amortises nothing, and the
                // single-text pipeline is the faster one for it
                if (!b.reqs.empty() && (r->n >= solo_bytes_ || b.reqs[0]->n >= solo_bytes_)) break;
                if (reserved_ + r->footprint > budget_) break;  // first come, first served
                reserved_ += r->footprint;
                b.scratch += r->footprint - serve_result_bytes(r->n, width);
                text_bytes += r->n;
                r->status = 1;
                r->lane = k;
                r->t_start = std::chrono::steady_clock::now();
                b.reqs.push_back(r);
                it = queue_.erase(it);
            }
            running_++;
            st_.batches++;
            st_.peak_reserved_bytes = std::max<uint64_t>(st_.peak_reserved_bytes, reserved_);
            st_.max_batch_texts = std::max<uint64_t>(st_.max_batch_texts, b.reqs.size());
        }
        cv_work_.notify_all();  // the rest of the queue may fit another lane
        return true;
    }

    // Enqueues the copies of the batch's texts on the lane's copy stream.
    void upload(int k, Batch& b) {
        Ctx& c = *lanes_[k];
        cudaStream_t cs = copy_streams_[k];
        b.offs.assign(b.reqs.size() + 1, 0);
        for (size_t i = 0; i < b.reqs.size(); i++) b.offs[i + 1] = b.offs[i] + b.reqs[i]->n;
        try {
            DCX_CUDA(cudaEventCreate(&b.ev_up0));
            DCX_CUDA(cudaEventCreate(&b.ev_up1));
            DCX_CUDA(cudaMallocFromPoolAsync(&b.d_text, b.offs.back() + 16, c.pool, cs));
            DCX_CUDA(cudaEventRecord(b.ev_up0, cs));
            for (size_t i = 0; i < b.reqs.size(); i++)
                if (b.reqs[i]->n)
                    DCX_CUDA(cudaMemcpyAsync((uint8_t*)b.d_text + b.offs[i], text_of(*b.reqs[i]), b.reqs[i]->n,
                                             b.reqs[i]->borrowed_dev ? cudaMemcpyDeviceToDevice
                                                                     : cudaMemcpyHostToDevice,
                                             cs));
            DCX_CUDA(cudaEventRecord(b.ev_up1, cs));
        } catch (const Error& e) {
            b.err = e.code;
        }
    }

    // Builds an uploaded batch on the lane's stream; returns the result buffer.
    std::shared_ptr<ServeResult> build(int k, Batch& b) {
        Ctx& c = *lanes_[k];
        if (b.err != DCX_OK) throw Error(b.err, "upload failed");
        const int width = b.reqs[0]->width, dc = b.reqs[0]->dc;
        auto res = std::make_shared<ServeResult>();
        res->stream = c.stream;
        res->bytes = serve_result_bytes(b.offs.back(), width);
        DCX_CUDA(cudaStreamWaitEvent(c.stream, b.ev_up1, 0));
        if (cudaMallocFromPoolAsync(&res->p, res->bytes, c.pool, c.stream) != cudaSuccess) {
            cudaGetLastError();
            res->p = nullptr;
            throw Error(DCX_ERR_OOM, "result buffer");
        }
        cudaEvent_t e0, e1;
        cudaEventCreate(&e0);
        cudaEventCreate(&e1);
        cudaEventRecord(e0, c.stream);
        try {
            c.budget = c.in_use + b.scratch;  // build_batch sizes its rounds from this
            build_batch(c, (const uint8_t*)b.d_text, b.offs.data(), (uint32_t)b.reqs.size(), dc, width, res->p,
                        DCX_DEVICE_PTRS);
            cudaEventRecord(e1, c.stream);
            DCX_CUDA(cudaStreamSynchronize(c.stream));
        } catch (...) {
            cudaEventDestroy(e0);
            cudaEventDestroy(e1);
            throw;
        }
        float up = 0, bd = 0;
        cudaEventElapsedTime(&up, b.ev_up0, b.ev_up1);
        cudaEventElapsedTime(&bd, e0, e1);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        std::lock_guard<std::mutex> lk(mu_);
        st_.ms_upload += up;
        st_.ms_build += bd;
        return res;
    }

    // Frees the batch's upload state (ordered after the lane's work on it).
    void drop_upload(int k, Batch& b) {
        Ctx& c = *lanes_[k];
        if (b.d_text) {
            cudaStreamWaitEvent(c.stream, b.ev_up1, 0);
            cudaFreeAsync(b.d_text, c.stream);
        }
        if (b.ev_up0) cudaEventDestroy(b.ev_up0);
        if (b.ev_up1) cudaEventDestroy(b.ev_up1);
        b.d_text = nullptr;
        b.ev_up0 = b.ev_up1 = nullptr;
    }

    void complete(int k, Batch& b, const std::shared_ptr<ServeResult>& res, int err) {
        Ctx& c = *lanes_[k];
        {
            std::lock_guard<std::mutex> lk(mu_);
            const auto now = std::chrono::steady_clock::now();
            uint64_t result_bytes = 0;
            for (size_t i = 0; i < b.reqs.size(); i++) {
                ServeReq* r = b.reqs[i];
                r->t_done = now;
                r->text.reset();
                r->borrowed = nullptr;
                if (r->pinned) {
                    arena_.free(r->pinned);
                    r->pinned = nullptr;
                }
                if (err == DCX_OK) {
                    r->status = 2;
                    r->res = res;
                    r->res_off = b.offs[i] * (uint64_t)(r->width / 8);
                    st_.done++;
                    st_.done_bytes += r->n;
                } else {
                    r->status = err;
                    st_.failed++;
                }
            }
            if (err == DCX_OK && res) {
                res->refs = (uint32_t)b.reqs.size();
                result_bytes = res->bytes;
            }
            // the scratch and text parts end with the batch, the result stays until released
            uint64_t fp = 0;
            for (ServeReq* r : b.reqs) fp += r->footprint;
            reserved_ -= fp - result_bytes;
            st_.peak_lane_bytes = std::max<uint64_t>(st_.peak_lane_bytes, c.peak);
            running_--;
        }
        cv_work_.notify_all();
        cv_done_.notify_all();
    }

    // Lane loop.  The bulk lane prefetches: once a batch is uploaded it takes
    // the next one from the queue and enqueues its upload on the copy stream
    // before building the current one, so uploads overlap builds.
    void lane_main(int k) {
        cudaSetDevice(device_);
        Batch cur, nxt;
        for (;;) {
            if (cur.empty()) {
                if (!admit(k, true, cur)) break;
                if (cur.empty()) continue;
                upload(k, cur);
            }
            if (k == 0) {
                if (!admit(k, false, nxt)) {
                    nxt = Batch{};
                }
                if (!nxt.empty()) upload(k, nxt);
            }
            int err = DCX_OK;
            std::shared_ptr<ServeResult> res;
            try {
                res = build(k, cur);
            } catch (const Error& e) {
                err = e.code;
                res.reset();
            } catch (...) {
                err = DCX_ERR_INTERNAL;
                res.reset();
            }
            drop_upload(k, cur);
            complete(k, cur, res, err);
            cur = std::move(nxt);
            nxt = Batch{};
        }
        // stopping: a prefetched batch is abandoned (its requests are dropped with the server)
        if (!cur.empty()) drop_upload(k, cur);
        cudaStreamSynchronize(lanes_[k]->stream);
    }

    static const uint8_t* text_of(const ServeReq& r) {
        if (r.borrowed) return r.borrowed;
        if (r.pinned) return r.pinned;
        return r.text.get();
    }

    int device_;
    uint64_t budget_, batch_bytes_;
    uint32_t batch_texts_;
    uint64_t express_bytes_, express_batch_bytes_;
    uint64_t solo_bytes_ = 32ull << 20;  // texts at least this long form a batch of their own
    PinnedArena arena_;
    std::mutex mu_, copy_mu_;
    std::condition_variable cv_work_, cv_done_;
    std::deque<uint64_t> queue_;
    std::map<uint64_t, std::unique_ptr<ServeReq>> reqs_;
    uint64_t next_id_ = 1, reserved_ = 0;
    uint32_t running_ = 0;
    bool stop_ = false;
    dcx_serve_stats st_{};
    std::vector<std::unique_ptr<Ctx>> lanes_;
    std::vector<cudaStream_t> copy_streams_;  // per lane: uploads of the texts
    std::vector<std::thread> threads_;
    cudaStream_t copy_stream_ = nullptr;
};

}  // namespace dcx
