// fmn_api.cu -- the C ABI (include/fast_mul.h): abs_mul64 / abs_sqr64 drop-ins and the
// fmn_* extensions.  Host code only; the kernels live in fmn_ntt.cu.
//
// Each device gets a context with a cached scratch workspace, a stream and an event that
// orders uses of the workspace across streams.  Host-pointer calls copy the operands to the
// device, run the product and copy the result back (out may alias the inputs, as in the
// reference, because the inputs are consumed before the output is written).  They run on
// host lanes: a few per device (FMN_HOST_LANES, default 4), each with its own workspace,
// operand buffers and streams.  A call holds the device lock only while it enqueues its
// copies and kernels, so the calls of several host threads overlap on the GPU (one product's
// copies over PCIe beside another's kernels), as the reference's calls on several host
// threads run side by side on the CPU cores.
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <atomic>
#include <condition_variable>
#include <algorithm>
#include <thread>
#include <functional>
#include <deque>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fast_mul.h"
#include "fmn_internal.h"

namespace {

thread_local std::string g_last_error;

int set_err(int code, const char* what, cudaError_t e = cudaSuccess) {
    g_last_error = what;
    if (e != cudaSuccess) {
        g_last_error += ": ";
        g_last_error += cudaGetErrorString(e);
    }
    return code;
}

constexpr int MAX_DEV = 64;

// Resources of one in-flight host-pointer product (see the file comment).
struct HostLane {
    cudaStream_t s = nullptr, cs = nullptr, co = nullptr;   // kernels, copy-in, copy-back
    cudaEvent_t done = nullptr;                              // the lane's last product
    bool done_valid = false;
    cudaEvent_t join[2] = {nullptr, nullptr};
    cudaEvent_t a_in = nullptr;            // the first operand's copy (shared copy streams)
    cudaEvent_t cb_event[4] = {nullptr};   // chunked copy-back
    cudaEvent_t ci_event[8] = {nullptr};   // piecewise copy-in of the second operand
    void* ws = nullptr;
    size_t ws_cap = 0;
    u64* io = nullptr;                     // device copies of the operands and the product
    size_t io_cap = 0;
    unsigned* h_err = nullptr;             // pinned word for reading the device error flag
    bool busy = false;
    // pageable host buffers: pinned staging slots (kStageSlots x kStageChunk bytes, allocated
    // on first use) and the event of each slot's last transfer
    char* stage = nullptr;
    cudaEvent_t stage_ev[4] = {nullptr};
    bool stage_used[4] = {false};
};

constexpr size_t kStageChunk = 8u << 20;   // bytes per staging slot
constexpr int kStageSlots = 4;

// A few host threads that copy between pageable and pinned memory in parallel: one thread's
// memcpy reaches a fraction of the host's memory bandwidth.  FMN_COPY_THREADS (1 .. 32,
// default min(8, hardware threads / 2)) sets their number, counting the calling thread (on a
// 16-thread host, 8 copied faster than 16 or 24 at 10M x 10M limbs).
class CopyPool {
  public:
    static CopyPool& get() {
        static CopyPool* p = new CopyPool();      // never destroyed: threads outlive static teardown
        return *p;
    }
    // dst[0, n) = src[0, n), split across the pool and the calling thread.
    void copy(void* dst, const void* src, size_t n) {
        const size_t parts = n < (1u << 20) ? 1 : std::min<size_t>(workers_ + 1, n >> 20);
        if (parts <= 1) {
            memcpy(dst, src, n);
            return;
        }
        const size_t per = ((n + parts - 1) / parts + 63) & ~(size_t)63;
        // the count is changed and read only under m, so the caller cannot return (and free
        // m and cv) before the last worker has let go of m
        int left = 0;
        std::mutex m;
        std::condition_variable cv;
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (size_t k = 1; k < parts; ++k) {
                const size_t off = k * per;
                if (off >= n) break;
                const size_t len = std::min(per, n - off);
                ++left;
                tasks_.push_back([=, &left, &m, &cv] {
                    memcpy((char*)dst + off, (const char*)src + off, len);
                    std::lock_guard<std::mutex> g(m);
                    if (--left == 0) cv.notify_one();
                });
            }
        }
        cv_.notify_all();
        memcpy(dst, src, std::min(per, n));
        std::unique_lock<std::mutex> lk(m);
        cv.wait(lk, [&] { return left == 0; });
    }

  private:
    CopyPool() {
        const char* v = getenv("FMN_COPY_THREADS");
        unsigned hw = std::thread::hardware_concurrency();
        int n = v ? atoi(v) : (int)std::min(8u, hw > 1 ? hw / 2 : 1u);
        n = n < 1 ? 1 : (n > 32 ? 32 : n);
        workers_ = (size_t)n - 1;
        for (size_t k = 0; k < workers_; ++k) std::thread([this] { run(); }).detach();
    }
    void run() {
        for (;;) {
            std::function<void()> t;
            {
                std::unique_lock<std::mutex> lk(mu_);
                cv_.wait(lk, [&] { return !tasks_.empty(); });
                t = std::move(tasks_.front());
                tasks_.pop_front();
            }
            t();
        }
    }
    size_t workers_ = 0;
    std::mutex mu_;
    std::condition_variable cv_;
    std::deque<std::function<void()>> tasks_;
};

struct DevCtx {
    std::mutex mu;
    int dev = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;       // last job that used `ws`
    bool done_valid = false;
    void* ws = nullptr;
    size_t ws_cap = 0;
    unsigned* h_err = nullptr;        // pinned word for reading the device error flag
    // precomputed four-step twiddles, one set per transform length, least recently used evicted
    struct Tw {
        fmn::TwiddleSet set;
        void* buf;
        size_t bytes;
        u64 last_use;
    };
    std::vector<Tw> tw;
    u64 tick = 0;
    // batches: worker streams, fork/join events, pinned descriptor staging
    static constexpr int NSTREAM = 4;
    cudaStream_t wstream[NSTREAM] = {nullptr};
    cudaEvent_t wevent[NSTREAM + 1] = {nullptr};
    void* stage = nullptr;
    size_t stage_cap = 0;
    cudaEvent_t stage_free = nullptr;   // the last batch's descriptor copy has completed
    bool stage_pending = false;
    // pinned host products with FMN_COPY_ORDER=fifo: one copy-in and one copy-back stream shared
    // by all lanes, so copies run in the order the calls enqueued them (created on first use)
    cudaStream_t cin = nullptr, cout = nullptr;
    // host lanes: created on demand up to host_lanes(), handed out under lane_mu
    std::vector<HostLane*> lanes;
    std::mutex lane_mu;
    std::condition_variable lane_cv;
};

std::mutex g_ctx_mu;
DevCtx* g_ctx[MAX_DEV] = {nullptr};

int cur_device(int* dev) {
    cudaError_t e = cudaGetDevice(dev);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaGetDevice", e);
    if (*dev < 0 || *dev >= MAX_DEV) return set_err(FMN_ERR_ARG, "device index out of range");
    return FMN_OK;
}

// Context of the current device, created (tables uploaded) on first use.
int get_ctx(DevCtx** out) {
    int dev;
    int rc = cur_device(&dev);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    if (!g_ctx[dev]) {
        cudaError_t e = fmn::ensure_tables();
        if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "uploading twiddle tables", e);
        DevCtx* c = new DevCtx();
        c->dev = dev;
        if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&c->done, cudaEventDisableTiming)) != cudaSuccess ||
            (e = cudaMallocHost((void**)&c->h_err, sizeof(unsigned))) != cudaSuccess) {
            delete c;
            return set_err(FMN_ERR_CUDA, "creating device context", e);
        }
        for (int k = 0; k < DevCtx::NSTREAM && e == cudaSuccess; ++k)
            e = cudaStreamCreateWithFlags(&c->wstream[k], cudaStreamNonBlocking);
        for (int k = 0; k <= DevCtx::NSTREAM && e == cudaSuccess; ++k)
            e = cudaEventCreateWithFlags(&c->wevent[k], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&c->stage_free, cudaEventDisableTiming);
        if (e != cudaSuccess) {
            delete c;
            return set_err(FMN_ERR_CUDA, "creating device context streams", e);
        }
        g_ctx[dev] = c;
        fmn_load_default_plans();              // tuned plans for this GPU, if a plan file matches
        fmn::q32_prepare_tables();             // best effort: a pass without a table computes its twiddles
    }
    *out = g_ctx[dev];
    return FMN_OK;
}

// Grow a cached device buffer to `bytes` (its owner's lock held).  A workspace's error word
// at offset 0 is zeroed on allocation.
// Failure-handling tests (fmn_test_fail_allocs): this many of the next device allocations of
// workspaces and operand buffers fail as if cudaMalloc had found no memory.
std::atomic<int> g_fail_allocs{0};

bool forced_alloc_failure() {
    int n = g_fail_allocs.load();
    while (n > 0)
        if (g_fail_allocs.compare_exchange_weak(n, n - 1)) return true;
    return false;
}

int ensure_buf(void** buf, size_t* cap, size_t bytes, bool workspace) {
    if (*cap >= bytes) return FMN_OK;
    cudaError_t e;
    if (forced_alloc_failure())
        return set_err(FMN_ERR_NOMEM, workspace ? "cudaMalloc of the product workspace" : "cudaMalloc of the operand buffers",
                       cudaErrorMemoryAllocation);
    if (*buf) {
        if ((e = cudaDeviceSynchronize()) != cudaSuccess) return set_err(FMN_ERR_CUDA, "sync before regrow", e);
        cudaFree(*buf);
        *buf = nullptr;
        *cap = 0;
    }
    if ((e = cudaMalloc(buf, bytes)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(FMN_ERR_NOMEM, workspace ? "cudaMalloc of the product workspace" : "cudaMalloc of the operand buffers", e);
    }
    if (workspace && (e = cudaMemset(*buf, 0, 256)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaMemset", e);
    *cap = bytes;
    return FMN_OK;
}

// The cached workspace of `c` (caller holds c->mu).
int ensure_ws(DevCtx* c, size_t bytes) { return ensure_buf(&c->ws, &c->ws_cap, bytes, true); }

// Number of host lanes per device: FMN_HOST_LANES (1 .. 8), default 4.
int host_lanes() {
    static const int n = [] {
        const char* v = getenv("FMN_HOST_LANES");
        const int k = v ? atoi(v) : 4;
        return k < 1 ? 1 : (k > 8 ? 8 : k);
    }();
    return n;
}

// Copies of pinned host products: "lane" (default) gives every host lane its own copy streams,
// so concurrent callers share PCIe between them; "fifo" (FMN_COPY_ORDER=fifo) puts every
// lane's copies on two streams shared per device, in the order the calls were enqueued, so
// each call's operands arrive whole before the next call's.  At 10M x 10M on B200: 274-280
// products/s by lane against 224/s in fifo order from 4 callers; 240 against 223 from 6.
bool copy_fifo() {
    static const bool f = [] {
        const char* v = getenv("FMN_COPY_ORDER");
        return v && strcmp(v, "fifo") == 0;
    }();
    return f;
}

void destroy_lane(HostLane* L) {
    if (L->ws) cudaFree(L->ws);
    if (L->io) cudaFree(L->io);
    if (L->h_err) cudaFreeHost(L->h_err);
    for (cudaStream_t st : {L->s, L->cs, L->co})
        if (st) cudaStreamDestroy(st);
    for (cudaEvent_t ev : {L->done, L->join[0], L->join[1], L->a_in})
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : L->cb_event)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : L->ci_event)
        if (ev) cudaEventDestroy(ev);
    for (cudaEvent_t ev : L->stage_ev)
        if (ev) cudaEventDestroy(ev);
    if (L->stage) cudaFreeHost(L->stage);
    delete L;
}

// A free host lane of `c`, created if fewer than host_lanes() exist; waits for one otherwise.
int acquire_lane(DevCtx* c, HostLane** out) {
    std::unique_lock<std::mutex> lk(c->lane_mu);
    for (;;) {
        for (HostLane* L : c->lanes)
            if (!L->busy) {
                L->busy = true;
                *out = L;
                return FMN_OK;
            }
        if ((int)c->lanes.size() < host_lanes()) break;
        c->lane_cv.wait(lk);
    }
    HostLane* L = new HostLane();
    cudaError_t e = cudaSuccess;
    for (cudaStream_t* st : {&L->s, &L->cs, &L->co})
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(st, cudaStreamNonBlocking);
    for (cudaEvent_t* ev : {&L->done, &L->join[0], &L->join[1], &L->a_in})
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(ev, cudaEventDisableTiming);
    for (cudaEvent_t& ev : L->cb_event)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    for (cudaEvent_t& ev : L->ci_event)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    for (cudaEvent_t& ev : L->stage_ev)
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMallocHost((void**)&L->h_err, sizeof(unsigned));
    if (e != cudaSuccess) {
        destroy_lane(L);
        return set_err(FMN_ERR_CUDA, "creating a host lane", e);
    }
    L->busy = true;
    c->lanes.push_back(L);
    *out = L;
    return FMN_OK;
}

struct LaneGuard {
    DevCtx* c;
    HostLane* L;
    ~LaneGuard() {
        {
            std::lock_guard<std::mutex> lk(c->lane_mu);
            L->busy = false;
        }
        c->lane_cv.notify_one();
    }
};

// Coefficients are < min(len1, len2) * 2^128 and must stay below p0 p1 p2 (about 2^184.7);
// transforms are limited to 2^30 points by the twiddle tables.
int check_sizes(u64 len1, u64 len2) {
    const u64 mn = len1 < len2 ? len1 : len2;
    if (mn >= (1ull << 56)) return set_err(FMN_ERR_TOO_LARGE, "operand too long for the 3-prime coefficient range");
    if (len1 + len2 - 1 > (1ull << fmn::MAX_LOG_N))
        return set_err(FMN_ERR_TOO_LARGE, "product needs a transform longer than 2^30");
    return FMN_OK;
}

size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

// Twiddle tables for transforms of 2^log_n points, built on stream s on first use (caller
// holds c->mu and has ordered s after the context's previous work).  Returns null when the
// transform has one pass or memory is short; the kernels then generate the twiddles.
// The cached twiddle tables of length 2^log_n (built on s the first time), or null.  The
// pointer is into the cache and valid only until the next call; `keep` (a log length, or -1)
// is never evicted, so a caller that copied one set can look up a second one.
const fmn::TwiddleSet* get_twiddles(DevCtx* c, int log_n, cudaStream_t s, int keep = -1) {
    const size_t bytes = fmn::twiddle_table_bytes(log_n);
    if (bytes == 0) return nullptr;
    const fmn::Plan cur = fmn::make_plan(log_n);
    for (size_t k = 0; k < c->tw.size(); ++k) {
        auto& t = c->tw[k];
        if (t.set.log_n != log_n) continue;
        if (fmn::same_plan(t.set.plan, cur)) {
            t.last_use = ++c->tick;
            return &t.set;
        }
        cudaFree(t.buf);                       // built for a plan no longer in effect
        c->tw.erase(c->tw.begin() + k);
        break;
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    const size_t cap = total_b / 4;          // tables never take more than a quarter of the GPU
    size_t held = 0;
    for (auto& t : c->tw) held += t.bytes;
    while (!c->tw.empty() && (held + bytes > cap || c->tw.size() >= 8)) {
        size_t lru = c->tw.size();
        for (size_t k = 0; k < c->tw.size(); ++k)
            if (c->tw[k].set.log_n != keep && (lru == c->tw.size() || c->tw[k].last_use < c->tw[lru].last_use)) lru = k;
        if (lru == c->tw.size()) break;       // only the kept set is left

        cudaFree(c->tw[lru].buf);             // synchronises the device: no job still reads it
        held -= c->tw[lru].bytes;
        c->tw.erase(c->tw.begin() + lru);
    }
    if (held + bytes > cap || bytes + (size_t)(1ull << 30) > free_b) return nullptr;
    void* buf = nullptr;
    if (cudaMalloc(&buf, bytes) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    DevCtx::Tw t;
    t.buf = buf;
    t.bytes = bytes;
    t.last_use = ++c->tick;
    // built on s; finished here, since later jobs on other streams read the cached tables
    if (fmn::build_twiddle_tables(log_n, (u64*)buf, &t.set, s) != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(buf);
        return nullptr;
    }
    c->tw.push_back(t);
    return &c->tw.back().set;
}

// A 64-bit product's twiddle tables, copied out of the cache: the main transform's and, for a
// wrapped product, its second transform's (looked up without evicting the first set).
struct JobTwiddles {
    fmn::TwiddleSet main, side;
    bool has_main = false, has_side = false;
    const fmn::TwiddleSet* main_ptr() const { return has_main ? &main : nullptr; }
    const fmn::TwiddleSet* side_ptr() const { return has_side ? &side : nullptr; }
};
JobTwiddles job_twiddles(DevCtx* c, const fmn::Job& j, cudaStream_t s) {
    JobTwiddles t;
    if (fmn::job_engine(j) != fmn::ENGINE_64) return t;
    const int n = fmn::job_twiddle_log_n(j);
    if (const fmn::TwiddleSet* p = get_twiddles(c, n, s)) {
        t.main = *p;
        t.has_main = true;
    }
    const int m = fmn::job_side_log_n(j);
    if (m > 0 && m != n) {
        if (const fmn::TwiddleSet* p = get_twiddles(c, m, s, n)) {
            t.side = *p;
            t.has_side = true;
        }
    }
    return t;
}

const fmn::TwiddleSet* ctx_twiddles(void* ctx, int log_n) {
    DevCtx* c = (DevCtx*)ctx;
    return get_twiddles(c, log_n, c->stream);
}

int ilog2_ceil(u64 x) {
    int r = 0;
    while ((1ull << r) < x) ++r;
    return r;
}

// Enqueue a product on stream s using the context workspace (caller holds c->mu).
int run_job_ctx(DevCtx* c, const fmn::Job& j, cudaStream_t s) {
    const size_t need = fmn::job_workspace_bytes(j);
    int rc = ensure_ws(c, need);
    if (rc) return rc;
    cudaError_t e;
    if (c->done_valid && (e = cudaStreamWaitEvent(s, c->done, 0)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "cudaStreamWaitEvent", e);
    const JobTwiddles tw = job_twiddles(c, j, s);
    if ((e = fmn::enqueue_job(j, c->ws, c->ws_cap, s, tw.main_ptr(), tw.side_ptr())) != cudaSuccess) {
        std::string m = std::string("kernel launch (") + fmn::launch_diag() + ")";
        return set_err(FMN_ERR_CUDA, m.c_str(), e);
    }
    if ((e = cudaEventRecord(c->done, s)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaEventRecord", e);
    c->done_valid = true;
    return FMN_OK;
}

// Read and clear the device error word of a workspace after stream s has drained.
int take_device_error(void* ws, unsigned* h_word, cudaStream_t s) {
    cudaError_t e;
    if ((e = cudaMemcpyAsync(h_word, ws, sizeof(unsigned), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "synchronising the product", e);
    if (*h_word) {
        cudaMemsetAsync(ws, 0, sizeof(unsigned), s);
        cudaStreamSynchronize(s);
        return set_err(FMN_ERR_DEVICE, "carry scan: bounded wait expired");
    }
    return FMN_OK;
}

bool is_pinned(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

struct CopyBack {
    cudaStream_t main, copy;
    cudaEvent_t ev[4];
    int used;
    u64* dst;
    const u64* src;
};

cudaError_t copy_back_chunk(void* p, u64 lo, u64 hi) {
    CopyBack* cb = (CopyBack*)p;
    cudaEvent_t ev = cb->ev[cb->used++ % 4];
    cudaError_t e = cudaEventRecord(ev, cb->main);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(cb->copy, ev, 0);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(cb->dst + lo, cb->src + lo, (hi - lo) * sizeof(u64), cudaMemcpyDeviceToHost, cb->copy);
    return e;
}

struct CopyIn {
    cudaStream_t copy;
    cudaEvent_t ev[8];
    int used;
    u64* dst;
    const u64* src;
};

// Copy limbs [lo, hi) of the second operand on the copy-in stream and make s wait for them.
cudaError_t copy_in_range(void* p, u64 lo, u64 hi, cudaStream_t s) {
    CopyIn* ci = (CopyIn*)p;
    cudaEvent_t ev = ci->ev[ci->used++ % 8];
    cudaError_t e = cudaMemcpyAsync(ci->dst + lo, ci->src + lo, (hi - lo) * sizeof(u64), cudaMemcpyHostToDevice, ci->copy);
    if (e == cudaSuccess) e = cudaEventRecord(ev, ci->copy);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, ev, 0);
    return e;
}

// Host product on pinned buffers: in2 is copied on a second stream while in1's forward
// passes run (piece by piece for a split product, each just ahead of its first reader), and
// the output comes back in chunks on a third stream as the carry scan finishes them (for a
// split product, the limbs each piece completes while the next piece computes).  Everything
// is enqueued under the device lock; the wait for the result is not.
int host_product_pinned(DevCtx* c, HostLane* L, const u64* in1, u64 len1, const u64* in2, u64 len2, u64* out,
                        int sqr) {
    const u64 out_len = len1 + len2;
    const size_t o1 = 0, o2 = round256(len1 * 8), oo = o2 + (sqr ? 0 : round256(len2 * 8));
    int rc;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        if ((rc = ensure_buf((void**)&L->io, &L->io_cap, oo + round256(out_len * 8), false))) return rc;
        char* io = (char*)L->io;
        cudaError_t e;
        const bool fifo = copy_fifo();
        if (fifo && !c->cin) {
            if ((e = cudaStreamCreateWithFlags(&c->cin, cudaStreamNonBlocking)) != cudaSuccess ||
                (e = cudaStreamCreateWithFlags(&c->cout, cudaStreamNonBlocking)) != cudaSuccess)
                return set_err(FMN_ERR_CUDA, "creating the copy streams", e);
        }
        cudaStream_t s = L->s, cs = fifo ? c->cin : L->cs, co = fifo ? c->cout : L->co;
        fmn::Job j;
        j.a = (const u64*)(io + o1);
        j.la = len1;
        j.b = sqr ? j.a : (const u64*)(io + o2);
        j.lb = len2;
        j.out = (u64*)(io + oo);
        j.sqr = sqr;
        if ((rc = ensure_buf(&L->ws, &L->ws_cap, fmn::job_workspace_bytes(j), true))) return rc;
        // (the shared streams need no such wait: a call returns only after its own copies)
        if (L->done_valid && ((e = cudaStreamWaitEvent(s, L->done, 0)) != cudaSuccess ||
                              (!fifo && (e = cudaStreamWaitEvent(cs, L->done, 0)) != cudaSuccess) ||
                              (!fifo && (e = cudaStreamWaitEvent(co, L->done, 0)) != cudaSuccess)))
            return set_err(FMN_ERR_CUDA, "cudaStreamWaitEvent", e);
        const JobTwiddles tw = job_twiddles(c, j, s);
        if ((e = cudaMemcpyAsync(io + o1, in1, len1 * 8, cudaMemcpyHostToDevice, fifo ? cs : s)) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "copying in1 to the device", e);
        if (fifo && ((e = cudaEventRecord(L->a_in, cs)) != cudaSuccess || (e = cudaStreamWaitEvent(s, L->a_in, 0)) != cudaSuccess))
            return set_err(FMN_ERR_CUDA, "ordering the product after its first operand", e);
        CopyIn ci;
        ci.copy = cs;
        ci.used = 0;
        ci.dst = (u64*)(io + o2);
        ci.src = in2;
        for (int k = 0; k < 8; ++k) ci.ev[k] = L->ci_event[k];
        CopyBack cb;
        cb.main = s;
        cb.copy = co;
        cb.used = 0;
        cb.dst = out;
        cb.src = j.out;
        for (int k = 0; k < 4; ++k) cb.ev[k] = L->cb_event[k];
        const int chunks = out_len >= (1u << 20) ? 4 : 1;
        if ((e = fmn::enqueue_job_overlapped(j, L->ws, L->ws_cap, s, tw.main_ptr(), sqr ? nullptr : copy_in_range, &ci,
                                             chunks, copy_back_chunk, &cb, tw.side_ptr())) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "kernel launch", e);
        // the copy streams end after the last chunk; order the main stream (and later jobs) after them
        if ((e = cudaEventRecord(L->join[0], co)) != cudaSuccess || (e = cudaStreamWaitEvent(s, L->join[0], 0)) != cudaSuccess ||
            (e = cudaEventRecord(L->join[1], cs)) != cudaSuccess || (e = cudaStreamWaitEvent(s, L->join[1], 0)) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "joining the copy streams", e);
        if ((e = cudaEventRecord(L->done, s)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaEventRecord", e);
        L->done_valid = true;
    }
    return take_device_error(L->ws, L->h_err, L->s);
}

// Pageable source -> device, through the lane's pinned slots: each chunk is copied into a free
// slot by the copy pool, then sent by DMA on the copy-in stream while the next chunk is
// copied.  Returns once every chunk is in flight (the caller orders its kernels after them).
int stage_in(HostLane* L, char* d_dst, const char* h_src, size_t bytes) {
    cudaError_t e;
    int slot = 0;
    for (size_t off = 0; off < bytes; off += kStageChunk, slot = (slot + 1) % kStageSlots) {
        const size_t n = std::min(kStageChunk, bytes - off);
        if (L->stage_used[slot] && (e = cudaEventSynchronize(L->stage_ev[slot])) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "waiting for a staging slot", e);
        char* pin = L->stage + (size_t)slot * kStageChunk;
        CopyPool::get().copy(pin, h_src + off, n);
        if ((e = cudaMemcpyAsync(d_dst + off, pin, n, cudaMemcpyHostToDevice, L->cs)) != cudaSuccess ||
            (e = cudaEventRecord(L->stage_ev[slot], L->cs)) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "copying an operand to the device", e);
        L->stage_used[slot] = true;
    }
    return FMN_OK;
}

// Device -> pageable destination after the lane's stream: up to kStageSlots chunks in flight by
// DMA into the slots; each is copied out by the copy pool as soon as it lands, and its slot
// takes the next chunk.
int stage_out(HostLane* L, char* h_dst, const char* d_src, size_t bytes) {
    cudaError_t e;
    const size_t nch = (bytes + kStageChunk - 1) / kStageChunk;
    auto issue = [&](size_t k) -> cudaError_t {
        const int slot = (int)(k % kStageSlots);
        const size_t off = k * kStageChunk, n = std::min(kStageChunk, bytes - off);
        // the slot's previous transfer (an input chunk on the copy-in stream) must be done
        if (L->stage_used[slot] && (e = cudaStreamWaitEvent(L->s, L->stage_ev[slot], 0)) != cudaSuccess) return e;
        if ((e = cudaMemcpyAsync(L->stage + (size_t)slot * kStageChunk, d_src + off, n, cudaMemcpyDeviceToHost, L->s)) !=
            cudaSuccess)
            return e;
        L->stage_used[slot] = true;
        return cudaEventRecord(L->stage_ev[slot], L->s);
    };
    for (size_t k = 0; k < nch && k < (size_t)kStageSlots; ++k)
        if ((e = issue(k)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "copying the product to the host", e);
    for (size_t k = 0; k < nch; ++k) {
        const int slot = (int)(k % kStageSlots);
        const size_t off = k * kStageChunk, n = std::min(kStageChunk, bytes - off);
        if ((e = cudaEventSynchronize(L->stage_ev[slot])) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "copying the product to the host", e);
        CopyPool::get().copy(h_dst + off, L->stage + (size_t)slot * kStageChunk, n);
        if (k + kStageSlots < nch && (e = issue(k + kStageSlots)) != cudaSuccess)
            return set_err(FMN_ERR_CUDA, "copying the product to the host", e);
    }
    return FMN_OK;
}

int host_product(const u64* in1, u64 len1, const u64* in2, u64 len2, u64* out, int sqr) {
    fmn::NvtxRange nvtx("fmn host product");
    const u64 out_len = len1 + len2;
    if (out_len == 0) return FMN_OK;
    if (!in1 || !out || (!sqr && !in2)) return set_err(FMN_ERR_ARG, "null pointer");
    if (len1 == 0 || len2 == 0) {
        memset(out, 0, out_len * sizeof(u64));
        return FMN_OK;
    }
    int rc = check_sizes(len1, len2);
    if (rc) return rc;
    DevCtx* c;
    if ((rc = get_ctx(&c))) return rc;
    HostLane* L;
    if ((rc = acquire_lane(c, &L))) return rc;
    LaneGuard guard{c, L};
    // pinned buffers that do not overlap each other: overlapped copies
    if (is_pinned(in1) && (sqr || is_pinned(in2)) && is_pinned(out) &&
        ((const char*)out + (len1 + len2) * 8 <= (const char*)in1 || (const char*)out >= (const char*)(in1 + len1)) &&
        (sqr || (const char*)out + (len1 + len2) * 8 <= (const char*)in2 || (const char*)out >= (const char*)(in2 + len2)))
        return host_product_pinned(c, L, in1, len1, in2, len2, out, sqr);
    // pageable buffers: staged through the lane's pinned slots (copies issued outside the
    // device lock); device layout [in1][in2][out]
    const size_t o1 = 0, o2 = round256(len1 * 8), oo = o2 + (sqr ? 0 : round256(len2 * 8));
    fmn::Job j;
    cudaError_t e;
    {
        std::lock_guard<std::mutex> lk(c->mu);
        if ((rc = ensure_buf((void**)&L->io, &L->io_cap, oo + round256(out_len * 8), false))) return rc;
    }
    if (!L->stage) {
        if ((e = cudaMallocHost((void**)&L->stage, kStageSlots * kStageChunk)) != cudaSuccess) {
            L->stage = nullptr;
            return set_err(FMN_ERR_NOMEM, "pinned staging buffers", e);
        }
    }
    char* io = (char*)L->io;
    j.a = (const u64*)(io + o1);
    j.la = len1;
    j.b = sqr ? j.a : (const u64*)(io + o2);
    j.lb = len2;
    j.out = (u64*)(io + oo);
    j.sqr = sqr;
    // the copy-in stream may not overwrite the operands before the lane's previous product is done
    if (L->done_valid && (e = cudaStreamWaitEvent(L->cs, L->done, 0)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "cudaStreamWaitEvent", e);
    if ((rc = stage_in(L, io + o1, (const char*)in1, len1 * 8))) return rc;
    if (!sqr && (rc = stage_in(L, io + o2, (const char*)in2, len2 * 8))) return rc;
    if ((e = cudaEventRecord(L->join[0], L->cs)) != cudaSuccess || (e = cudaStreamWaitEvent(L->s, L->join[0], 0)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "ordering the product after its copies", e);
    {
        std::lock_guard<std::mutex> lk(c->mu);
        if ((rc = ensure_buf(&L->ws, &L->ws_cap, fmn::job_workspace_bytes(j), true))) return rc;
        const JobTwiddles tw = job_twiddles(c, j, L->s);
        if ((e = fmn::enqueue_job(j, L->ws, L->ws_cap, L->s, tw.main_ptr(), tw.side_ptr())) != cudaSuccess) {
            std::string m = std::string("kernel launch (") + fmn::launch_diag() + ")";
            return set_err(FMN_ERR_CUDA, m.c_str(), e);
        }
        if ((e = cudaEventRecord(L->done, L->s)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaEventRecord", e);
        L->done_valid = true;
    }
    if ((rc = stage_out(L, (char*)out, io + oo, out_len * 8))) return rc;
    return take_device_error(L->ws, L->h_err, L->s);
}

int device_product(const u64* d1, u64 len1, const u64* d2, u64 len2, u64* dout, int sqr, void* stream) {
    fmn::NvtxRange nvtx("fmn device product");
    const u64 out_len = len1 + len2;
    if (out_len == 0) return FMN_OK;
    if (!d1 || !dout || (!sqr && !d2)) return set_err(FMN_ERR_ARG, "null pointer");
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (len1 == 0 || len2 == 0) {
        if ((e = cudaMemsetAsync(dout, 0, out_len * 8, s)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaMemsetAsync", e);
        return FMN_OK;
    }
    int rc = check_sizes(len1, len2);
    if (rc) return rc;
    DevCtx* c;
    if ((rc = get_ctx(&c))) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    fmn::Job j;
    j.a = d1;
    j.la = len1;
    j.b = sqr ? d1 : d2;
    j.lb = len2;
    j.out = dout;
    j.sqr = sqr;
    return run_job_ctx(c, j, s);
}

}  // namespace

namespace fmn {
// Record an error for fmn_last_error() from other translation units of the library.
int api_set_error(int code, const char* what, cudaError_t e) { return set_err(code, what, e); }
}  // namespace fmn

namespace {

int to_jobs(const fmn_job* jobs, int count, std::vector<fmn::Job>& v) {
    if (count < 0 || (count > 0 && !jobs)) return set_err(FMN_ERR_ARG, "bad job array");
    v.resize(count);
    for (int i = 0; i < count; ++i) {
        const fmn_job& j = jobs[i];
        if (j.len1 + j.len2 > 0 && (!j.out || (j.len1 && !j.in1) || (j.len2 && !j.in2)))
            return set_err(FMN_ERR_ARG, "null pointer in a batch job");
        if (j.len1 && j.len2) {
            int rc = check_sizes(j.len1, j.len2);
            if (rc) return rc;
        }
        v[i].a = j.in1;
        v[i].la = j.len1;
        v[i].b = j.in2;
        v[i].lb = j.len2;
        v[i].out = j.out;
        v[i].sqr = (j.in1 == j.in2 && j.len1 == j.len2) ? 1 : 0;
    }
    return FMN_OK;
}

int ensure_stage(DevCtx* c, size_t bytes) {
    cudaError_t e;
    if (c->stage_pending) {                 // the previous batch's copy must have read it
        if ((e = cudaEventSynchronize(c->stage_free)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "staging", e);
        c->stage_pending = false;
    }
    if (c->stage_cap >= bytes) return FMN_OK;
    if (c->stage) cudaFreeHost(c->stage);
    c->stage = nullptr;
    c->stage_cap = 0;
    if ((e = cudaMallocHost(&c->stage, bytes)) != cudaSuccess) {
        cudaGetLastError();
        return set_err(FMN_ERR_NOMEM, "pinned staging for batch descriptors", e);
    }
    c->stage_cap = bytes;
    return FMN_OK;
}

void die(const char* fn) {
    fprintf(stderr, "%s failed: %s\n", fn, g_last_error.c_str());
    abort();
}

}  // namespace

extern "C" {

void abs_mul64(const u64* in1, u64 len1, const u64* in2, u64 len2, u64* out) {
    // Same block and same length: the square (the reference requires in1 != in2,
    // src/fast_mul.h:37; the product is the same number either way).
    const int sq = (in1 == in2 && len1 == len2);
    if (host_product(in1, len1, in2, len2, out, sq)) die("abs_mul64");
}

void abs_sqr64(const u64* in1, u64 len1, u64* out) {
    if (host_product(in1, len1, in1, len1, out, 1)) die("abs_sqr64");
}

int fmn_init(int device) {
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaSetDevice", e);
    DevCtx* c;
    return get_ctx(&c);
}

void fmn_shutdown(void) {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    int prev = 0;
    cudaGetDevice(&prev);
    for (int d = 0; d < MAX_DEV; ++d) {
        DevCtx* c = g_ctx[d];
        if (!c) continue;
        cudaSetDevice(d);
        cudaDeviceSynchronize();
        if (c->ws) cudaFree(c->ws);
        for (HostLane* L : c->lanes) destroy_lane(L);
        c->lanes.clear();
        fmn::q32_release_tables(d);
        if (c->h_err) cudaFreeHost(c->h_err);
        for (auto& t : c->tw) cudaFree(t.buf);
        if (c->stage) cudaFreeHost(c->stage);
        for (int k = 0; k < DevCtx::NSTREAM; ++k)
            if (c->wstream[k]) cudaStreamDestroy(c->wstream[k]);
        for (int k = 0; k <= DevCtx::NSTREAM; ++k)
            if (c->wevent[k]) cudaEventDestroy(c->wevent[k]);
        if (c->stage_free) cudaEventDestroy(c->stage_free);
        if (c->done) cudaEventDestroy(c->done);
        if (c->stream) cudaStreamDestroy(c->stream);
        if (c->cin) cudaStreamDestroy(c->cin);
        if (c->cout) cudaStreamDestroy(c->cout);
        delete c;
        g_ctx[d] = nullptr;
    }
    cudaSetDevice(prev);
}

const char* fmn_last_error(void) { return g_last_error.c_str(); }

int fmn_mul(const u64* in1, u64 len1, const u64* in2, u64 len2, u64* out) {
    return host_product(in1, len1, in2, len2, out, (in1 == in2 && len1 == len2));
}

int fmn_sqr(const u64* in1, u64 len1, u64* out) { return host_product(in1, len1, in1, len1, out, 1); }

int fmn_mul_device(const u64* d_in1, u64 len1, const u64* d_in2, u64 len2, u64* d_out, void* stream) {
    return device_product(d_in1, len1, d_in2, len2, d_out, (d_in1 == d_in2 && len1 == len2), stream);
}

int fmn_sqr_device(const u64* d_in1, u64 len1, u64* d_out, void* stream) {
    return device_product(d_in1, len1, d_in1, len1, d_out, 1, stream);
}

int fmn_sync(void* stream) {
    DevCtx* c;
    int rc = get_ctx(&c);
    if (rc) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaStreamSynchronize", e);
    std::lock_guard<std::mutex> lk(c->mu);
    if (!c->ws) return FMN_OK;
    return take_device_error(c->ws, c->h_err, c->stream);
}

size_t fmn_workspace_size(u64 len1, u64 len2, int sqr) { return fmn::job_workspace_bytes(len1, len2, sqr ? 1 : 0); }

int fmn_set_engine(int engine) {
    if (engine != FMN_ENGINE_AUTO && engine != FMN_ENGINE_64 && engine != FMN_ENGINE_32)
        return set_err(FMN_ERR_ARG, "engine must be FMN_ENGINE_AUTO, FMN_ENGINE_64 or FMN_ENGINE_32");
    fmn::set_default_engine(engine);
    return FMN_OK;
}

int fmn_get_engine(void) { return fmn::default_engine(); }

int fmn_test_fail_allocs(int count) {
    if (count < 0) return set_err(FMN_ERR_ARG, "count must be >= 0");
    g_fail_allocs.store(count);
    return FMN_OK;
}

int fmn_test_carry_timeout(u64 out_limbs) {
    DevCtx* c;
    int rc = get_ctx(&c);
    if (rc) return rc;
    unsigned status = 0;
    const cudaError_t e = fmn::q32_test_carry_timeout(out_limbs, &status);
    if (e != cudaSuccess) return set_err(e == cudaErrorInvalidValue ? FMN_ERR_ARG : FMN_ERR_CUDA, "carry timeout test", e);
    return status ? set_err(FMN_ERR_DEVICE, "carry scan: bounded wait expired") : FMN_OK;
}

int fmn_force_pieces(int pieces) {
    if (pieces < 0) return set_err(FMN_ERR_ARG, "pieces must be >= 0");
    fmn::q32_force_pieces(pieces);
    return FMN_OK;
}

int fmn_pieces_for(u64 len1, u64 len2, int sqr) {
    fmn::Job j;
    j.a = j.b = nullptr;
    j.out = nullptr;
    j.la = len1;
    j.lb = len2;
    j.sqr = sqr ? 1 : 0;
    return fmn::job_engine(j) == fmn::ENGINE_32 ? fmn::q32_pieces(len1, len2, sqr ? 1 : 0) : 1;
}

int fmn_force_wrap(int mode) {
    if (mode < 0 || mode > 2) return set_err(FMN_ERR_ARG, "wrap mode must be 0, 1 or 2");
    fmn::q32_force_wrap(mode);
    return FMN_OK;
}

u64 fmn_twist_for(u64 len1, u64 len2, int sqr) {
    fmn::Job j;
    j.a = j.b = nullptr;
    j.out = nullptr;
    j.la = len1;
    j.lb = len2;
    j.sqr = sqr ? 1 : 0;
    return fmn::job_engine(j) == fmn::ENGINE_32 ? fmn::q32_twisted(len1, len2, sqr ? 1 : 0) : fmn::twist64_for(j);
}

u64 fmn_batch_twist_for(u64 len1, u64 len2, int sqr) {
    fmn::Job j;
    j.a = j.b = nullptr;
    j.out = nullptr;
    j.la = len1;
    j.lb = len2;
    j.sqr = sqr ? 1 : 0;
    return fmn::batch_twist_for(j);
}

u64 fmn_wrap_for(u64 len1, u64 len2, int sqr) {
    fmn::Job j;
    j.a = j.b = nullptr;
    j.out = nullptr;
    j.la = len1;
    j.lb = len2;
    j.sqr = sqr ? 1 : 0;
    return fmn::job_engine(j) == fmn::ENGINE_32 ? fmn::q32_wrapped(len1, len2, sqr ? 1 : 0) : fmn::wrap64_for(j);
}

int fmn_engine_for(u64 len1, u64 len2, int sqr) {
    fmn::Job j;
    j.a = j.b = nullptr;
    j.out = nullptr;
    j.la = len1;
    j.lb = len2;
    j.sqr = sqr ? 1 : 0;
    return fmn::job_engine(j);
}

int fmn_mul_device_ws(const u64* d_in1, u64 len1, const u64* d_in2, u64 len2, u64* d_out, void* d_ws,
                      size_t ws_bytes, void* stream) {
    const u64 out_len = len1 + len2;
    if (out_len == 0) return FMN_OK;
    if (!d_in1 || !d_in2 || !d_out || !d_ws) return set_err(FMN_ERR_ARG, "null pointer");
    if (((uintptr_t)d_ws & 255) != 0) return set_err(FMN_ERR_ARG, "workspace must be 256-byte aligned");
    int rc = check_sizes(len1, len2);
    if (rc) return rc;
    const int sq = (d_in1 == d_in2 && len1 == len2);
    if (ws_bytes < fmn::job_workspace_bytes(len1, len2, sq)) return set_err(FMN_ERR_ARG, "workspace too small");
    fmn::Job j;
    j.a = d_in1;
    j.la = len1;
    j.b = d_in2;
    j.lb = len2;
    j.out = d_out;
    j.sqr = sq;
    cudaError_t e = cudaMemsetAsync(d_ws, 0, sizeof(unsigned), (cudaStream_t)stream);   // status word
    if (e == cudaSuccess) e = fmn::enqueue_job(j, d_ws, ws_bytes, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "kernel launch", e);
    return FMN_OK;
}

int fmn_ws_status(const void* d_ws, u64 len1, u64 len2, int sqr, void* stream) {
    (void)len1;
    (void)len2;
    (void)sqr;
    if (!d_ws) return set_err(FMN_ERR_ARG, "null pointer");
    unsigned word = 0;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(&word, d_ws, sizeof(word), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "reading the workspace status", e);
    if (word) {
        cudaMemsetAsync((void*)d_ws, 0, sizeof(unsigned), s);
        cudaStreamSynchronize(s);
        return set_err(FMN_ERR_DEVICE, "carry scan: bounded wait expired");
    }
    return FMN_OK;
}

int fmn_mul_batch_device(const fmn_job* jobs, int count, void* stream) {
    fmn::NvtxRange nvtx("fmn batch");
    std::vector<fmn::Job> v;
    int rc = to_jobs(jobs, count, v);
    if (rc || count == 0) return rc;
    DevCtx* c;
    if ((rc = get_ctx(&c))) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    cudaStream_t s = (cudaStream_t)stream;
    const size_t wsb = fmn::batch_workspace_bytes(v.data(), count);
    if ((rc = ensure_ws(c, wsb))) return rc;
    if ((rc = ensure_stage(c, fmn::batch_stage_bytes(v.data(), count)))) return rc;
    cudaError_t e;
    if (c->done_valid && (e = cudaStreamWaitEvent(s, c->done, 0)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "cudaStreamWaitEvent", e);
    // the 64-bit engine's twiddle tables (one lookup per transform length its products use)
    // are built on the context stream: order s after it
    u64 lengths = 0;
    for (const auto& j : v)
        if (fmn::batch_on_engine64(j)) lengths |= 1ull << ilog2_ceil(j.la + j.lb - 1);
    for (int n = 0; n < 64; ++n)
        if (lengths >> n & 1) ctx_twiddles(c, n);
    if ((e = cudaEventRecord(c->wevent[0], c->stream)) != cudaSuccess ||
        (e = cudaStreamWaitEvent(s, c->wevent[0], 0)) != cudaSuccess)
        return set_err(FMN_ERR_CUDA, "ordering after twiddle tables", e);
    e = fmn::enqueue_batch(v.data(), count, c->ws, c->ws_cap, c->stage, c->stage_cap, s, c->wstream, c->wevent,
                           DevCtx::NSTREAM, ctx_twiddles, c);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "batch launch", e);
    if ((e = cudaEventRecord(c->stage_free, s)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaEventRecord", e);
    c->stage_pending = true;
    if ((e = cudaEventRecord(c->done, s)) != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaEventRecord", e);
    c->done_valid = true;
    return FMN_OK;
}

struct fmn_batch_graph {
    int dev;
    void* ws;
    size_t ws_bytes;
    void* stage;
    size_t stage_bytes;
    cudaStream_t cap;                      // capture origin
    cudaStream_t wstream[4];
    cudaEvent_t wevent[5];
    std::vector<void*> tw_bufs;
    std::vector<fmn::TwiddleSet> tw_sets;
    cudaGraph_t graph;
    cudaGraphExec_t exec;
    unsigned* h_err;
};

static const fmn::TwiddleSet* graph_twiddles(void* ctx, int log_n) {
    fmn_batch_graph* g = (fmn_batch_graph*)ctx;
    for (auto& t : g->tw_sets)
        if (t.log_n == log_n) return &t;
    return nullptr;
}

void fmn_batch_graph_destroy(fmn_batch_graph* g) {
    if (!g) return;
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->dev);
    cudaDeviceSynchronize();
    if (g->exec) cudaGraphExecDestroy(g->exec);
    if (g->graph) cudaGraphDestroy(g->graph);
    for (void* b : g->tw_bufs) cudaFree(b);
    if (g->ws) cudaFree(g->ws);
    if (g->stage) cudaFreeHost(g->stage);
    if (g->h_err) cudaFreeHost(g->h_err);
    for (int k = 0; k < 4; ++k)
        if (g->wstream[k]) cudaStreamDestroy(g->wstream[k]);
    for (int k = 0; k < 5; ++k)
        if (g->wevent[k]) cudaEventDestroy(g->wevent[k]);
    if (g->cap) cudaStreamDestroy(g->cap);
    delete g;
    cudaSetDevice(prev);
}

int fmn_batch_graph_create(const fmn_job* jobs, int count, fmn_batch_graph** out) {
    if (!out) return set_err(FMN_ERR_ARG, "null pointer");
    *out = nullptr;
    std::vector<fmn::Job> v;
    int rc = to_jobs(jobs, count, v);
    if (rc) return rc;
    DevCtx* c;
    if ((rc = get_ctx(&c))) return rc;
    cudaError_t e = fmn::prepare_batch();
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "preparing batch kernels", e);
    fmn_batch_graph* g = new fmn_batch_graph();   // value-initialised: null handles, empty vectors
    g->dev = c->dev;
    auto fail = [&](int code, const char* what, cudaError_t err) {
        cudaGetLastError();
        fmn_batch_graph_destroy(g);
        return set_err(code, what, err);
    };
    g->ws_bytes = fmn::batch_workspace_bytes(v.data(), count);
    g->stage_bytes = fmn::batch_stage_bytes(v.data(), count);
    if ((e = cudaMalloc(&g->ws, g->ws_bytes)) != cudaSuccess) return fail(FMN_ERR_NOMEM, "graph workspace", e);
    if ((e = cudaMemset(g->ws, 0, 256)) != cudaSuccess) return fail(FMN_ERR_CUDA, "graph workspace", e);
    if ((e = cudaMallocHost(&g->stage, g->stage_bytes)) != cudaSuccess) return fail(FMN_ERR_NOMEM, "graph staging", e);
    if ((e = cudaMallocHost((void**)&g->h_err, sizeof(unsigned))) != cudaSuccess) return fail(FMN_ERR_NOMEM, "graph status", e);
    if ((e = cudaStreamCreateWithFlags(&g->cap, cudaStreamNonBlocking)) != cudaSuccess) return fail(FMN_ERR_CUDA, "stream", e);
    for (int k = 0; k < 4; ++k)
        if ((e = cudaStreamCreateWithFlags(&g->wstream[k], cudaStreamNonBlocking)) != cudaSuccess)
            return fail(FMN_ERR_CUDA, "stream", e);
    for (int k = 0; k < 5; ++k)
        if ((e = cudaEventCreateWithFlags(&g->wevent[k], cudaEventDisableTiming)) != cudaSuccess)
            return fail(FMN_ERR_CUDA, "event", e);
    // the graph's own twiddle tables, one set per transform length in the batch
    for (const auto& j : v) {
        if (!fmn::batch_on_engine64(j)) continue;       // 32-bit batches compute their twiddles
        const int n = ilog2_ceil(j.la + j.lb - 1);
        const size_t bytes = fmn::twiddle_table_bytes(n);
        bool have = false;
        for (auto& t : g->tw_sets) have |= (t.log_n == n);
        if (have || !bytes) continue;
        void* buf = nullptr;
        if ((e = cudaMalloc(&buf, bytes)) != cudaSuccess) return fail(FMN_ERR_NOMEM, "graph twiddle tables", e);
        g->tw_bufs.push_back(buf);
        fmn::TwiddleSet ts;
        if ((e = fmn::build_twiddle_tables(n, (u64*)buf, &ts, g->cap)) != cudaSuccess)
            return fail(FMN_ERR_CUDA, "graph twiddle tables", e);
        g->tw_sets.push_back(ts);
    }
    if ((e = cudaStreamSynchronize(g->cap)) != cudaSuccess) return fail(FMN_ERR_CUDA, "graph twiddle tables", e);
    if ((e = cudaStreamBeginCapture(g->cap, cudaStreamCaptureModeThreadLocal)) != cudaSuccess)
        return fail(FMN_ERR_CUDA, "cudaStreamBeginCapture", e);
    e = fmn::enqueue_batch(v.data(), count, g->ws, g->ws_bytes, g->stage, g->stage_bytes, g->cap, g->wstream,
                           g->wevent, 4, graph_twiddles, g);
    cudaError_t e2 = cudaStreamEndCapture(g->cap, &g->graph);
    if (e != cudaSuccess) return fail(FMN_ERR_CUDA, "capturing the batch", e);
    if (e2 != cudaSuccess) return fail(FMN_ERR_CUDA, "cudaStreamEndCapture", e2);
    if ((e = cudaGraphInstantiate(&g->exec, g->graph, 0)) != cudaSuccess)
        return fail(FMN_ERR_CUDA, "cudaGraphInstantiate", e);
    *out = g;
    return FMN_OK;
}

int fmn_batch_graph_launch(fmn_batch_graph* g, void* stream) {
    fmn::NvtxRange nvtx("fmn batch graph launch");
    if (!g) return set_err(FMN_ERR_ARG, "null graph");
    cudaError_t e = cudaGraphLaunch(g->exec, (cudaStream_t)stream);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "cudaGraphLaunch", e);
    return FMN_OK;
}

int fmn_batch_graph_sync(fmn_batch_graph* g, void* stream) {
    if (!g) return set_err(FMN_ERR_ARG, "null graph");
    return take_device_error(g->ws, g->h_err, (cudaStream_t)stream);
}

int fmn_mul_operand_device(const fmn_operand* op, const u64* d_in2, u64 len2, u64* d_out, void* stream) {
    if (!op || !d_out || (len2 && !d_in2)) return set_err(FMN_ERR_ARG, "null pointer");
    if (len2 > op->max_partner) return set_err(FMN_ERR_ARG, "partner longer than the operand allows");
    cudaStream_t s = (cudaStream_t)stream;
    if (len2 == 0) {
        cudaError_t e = cudaMemsetAsync(d_out, 0, op->len * sizeof(u64), s);
        return e == cudaSuccess ? FMN_OK : set_err(FMN_ERR_CUDA, "cudaMemsetAsync", e);
    }
    DevCtx* c;
    int rc = get_ctx(&c);
    if (rc) return rc;
    std::lock_guard<std::mutex> lk(c->mu);
    fmn::Job j;
    j.a = nullptr;
    j.la = op->len;
    j.b = d_in2;
    j.lb = len2;
    j.out = d_out;
    j.sqr = 0;
    j.spectrum = op->spec;
    j.log_n = op->log_n;
    j.engine = op->engine;
    j.splan = op->plan;
    return run_job_ctx(c, j, s);
}

const char* fmn_kernel_kind_name(int kind) { return fmn::kernel_kind_name(kind); }

int fmn_profile_enable(int on) {
    fmn::profile_enable(on != 0);
    return FMN_OK;
}

int fmn_profile_take(double* ms, u64* launches, double* bytes, double* modmuls) {
    fmn::KindStats st[fmn::K_KINDS];
    memset(st, 0, sizeof(st));
    cudaError_t e = fmn::profile_take(st);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "reading profile events", e);
    for (int k = 0; k < fmn::K_KINDS; ++k) {
        if (ms) ms[k] = st[k].ms;
        if (launches) launches[k] = st[k].launches;
        if (bytes) bytes[k] = st[k].bytes;
        if (modmuls) modmuls[k] = st[k].modmuls;
    }
    return FMN_OK;
}

int fmn_launches_per_product(u64 len1, u64 len2, int sqr) { return fmn::job_launches(len1, len2, sqr ? 1 : 0); }

int fmn_bench_modmul(double* modmul_per_s, double* butterfly_per_s) {
    DevCtx* c;
    int rc = get_ctx(&c);
    if (rc) return rc;
    double a = 0, b = 0;
    cudaError_t e = fmn::bench_modmul(&a, &b);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "modmul microbenchmark", e);
    if (modmul_per_s) *modmul_per_s = a;
    if (butterfly_per_s) *butterfly_per_s = b;
    return FMN_OK;
}

int fmn_bench_bfly32(double* butterfly_per_s) {
    DevCtx* c;
    int rc = get_ctx(&c);
    if (rc) return rc;
    double a = 0;
    cudaError_t e = fmn::q32_bench_bfly(&a);
    if (e != cudaSuccess) return set_err(FMN_ERR_CUDA, "butterfly microbenchmark", e);
    if (butterfly_per_s) *butterfly_per_s = a;
    return FMN_OK;
}

u64 fmn_ntt_len(u64 len1, u64 len2) {
    const u64 conv = len1 + len2 ? len1 + len2 - 1 : 0;
    u64 n = 1;
    while (n < conv) n <<= 1;
    return n;
}

}  // extern "C"
