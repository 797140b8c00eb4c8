// fmn_server.cu -- resident operands and the product server (host code + one small kernel).
//
// Resident operand: a number whose forward spectrum (all passes) stays in HBM, so a product
// with it transforms only the partner -- the reference's conv_single (src/fast_mul.c:135-212),
// which its driver never calls.
//
// Server: requests (multiply, square, multiply by a resident operand) are submitted from
// any thread and served by a dispatcher thread with continuous batching:
//   * pending requests are admitted in arrival order while their scratch fits the HBM
//     budget; admitted requests form a batch (grouped launches, enqueue_batch) on a free
//     slot (one CUDA stream each), so batches overlap on the device;
//   * scratch comes from a private stream-ordered memory pool and returns to it when the
//     batch completes; a host callback on the slot stream stamps the completion time;
//   * requests that arrive while batches run are admitted as soon as a slot and budget
//     free up.
// The plain mode (batching off) launches every request as its own product on one stream,
// in arrival order, without resident reuse -- the per-call path the batched mode is
// compared with.  A request may carry the expected product; the server then compares it
// on the device and counts mismatches (used to check every output of a benchmark stream).
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/fast_mul.h"
#include "fmn_internal.h"

namespace fmn {
int api_set_error(int code, const char* what, cudaError_t e);
}

namespace {

using clk = std::chrono::steady_clock;

int ilog2c(u64 x) {
    int r = 0;
    while ((1ull << r) < x) ++r;
    return r;
}

// Adds the status word of a finished batch (set when a bounded wait expired) to a counter.
__global__ void k_fold_status(const unsigned* status, unsigned* counter) {
    if (threadIdx.x == 0 && *status) atomicAdd(counter, 1u);
}

__global__ void k_compare(const u64* __restrict__ a, const u64* __restrict__ b, u64 n, unsigned* mismatch) {
    bool bad = false;
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        bad |= a[i] != b[i];
    if (__syncthreads_or(bad) && threadIdx.x == 0) atomicAdd(mismatch, 1u);
}

struct Req {
    fmn_request r;
    clk::time_point arrival;
    clk::time_point done;
    size_t bytes;        // scratch charged against the budget
    bool cancelled;      // withdrawn before admission: never computed, output untouched
};

// A slot runs one batch at a time on its stream; an event recorded after the batch's last
// kernel tells the dispatcher (which polls it) that the batch has finished.  Polling an event
// leaves the stream free, where a host callback would hold it until the callback has run.
struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    void* stage = nullptr;
    size_t stage_cap = 0;
    bool busy = false;
    std::vector<size_t> reqs;   // indices into the request log
    void* mem = nullptr;
    size_t bytes = 0;
};

}  // namespace

struct fmn_server {
    int dev;
    size_t budget;
    int max_batch;
    int batching;
    int nslots;
    std::vector<Slot*> slots;
    std::deque<Slot*> fifo;               // plain mode: busy slots in launch (= completion) order
    cudaMemPool_t pool = nullptr;
    unsigned* d_mismatch = nullptr;       // [0] output mismatches, [1] device status errors
    unsigned* h_mismatch = nullptr;
    std::vector<std::pair<void*, fmn::TwiddleSet>> tw;   // per transform length
    std::mutex mu;
    std::condition_variable cv;
    std::deque<size_t> pending;           // plain mode: one queue
    std::deque<size_t> big;               // batching mode: large products (lane 0, one at a time)
    std::vector<Req> log;                 // every request ever submitted, by index
    std::vector<size_t> completed_order;  // indices in completion order
    size_t taken = 0;                     // completions handed out by fmn_server_take
    size_t in_use = 0, peak = 0;
    u64 batches = 0, rejected = 0, failures = 0, cancelled = 0;
    double launch_ms = 0.0, alloc_ms = 0.0;   // dispatcher host time (launch_batch, pool allocations)
    double max_launch_ms = 0.0, max_alloc_ms = 0.0;
    bool stop = false;
    bool paused = false;                  // admission held (fmn_server_pause)
    std::thread thr;
    std::string error;
};

namespace {

const fmn::TwiddleSet* server_twiddles(void* ctx, int log_n) {
    fmn_server* s = (fmn_server*)ctx;
    for (auto& t : s->tw)
        if (t.second.log_n == log_n) return &t.second;
    return nullptr;
}

// Build twiddle tables for every transform length a batch needs (dispatcher thread, once
// per length; blocks until built).
void ensure_server_twiddles(fmn_server* s, int log_n, cudaStream_t st) {
    if (server_twiddles(s, log_n) || fmn::twiddle_table_bytes(log_n) == 0) return;
    void* buf = nullptr;
    if (cudaMalloc(&buf, fmn::twiddle_table_bytes(log_n)) != cudaSuccess) {
        cudaGetLastError();
        return;
    }
    fmn::TwiddleSet ts;
    if (fmn::build_twiddle_tables(log_n, (u64*)buf, &ts, st) != cudaSuccess || cudaStreamSynchronize(st) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(buf);
        return;
    }
    s->tw.push_back({buf, ts});
}

// Whether a product with a resident operand should use its spectrum.  The spectrum has the
// transform length of the operand's longest partner, so a product with a short partner can be
// much cheaper from scratch.  Modelled costs (points x bits of the spectrum's engine): reuse
// transforms the partner and inverts at the spectrum's length; a fresh product costs whatever
// that engine's planner picks for the two lengths.
bool spectrum_pays(const fmn_request& r) {
    const fmn_operand* o = r.operand;
    const double reuse = 2.0 * std::ldexp(1.0, o->log_n) * (o->log_n + 1);
    double fresh;
    if (o->engine == fmn::ENGINE_32) {
        fresh = fmn::q32_cost(o->len, r.len2, 0);
    } else {
        const int n = ilog2c(o->len + r.len2 - 1);
        fresh = 3.0 * std::ldexp(1.0, n) * (n + 1);
    }
    return reuse <= fresh;
}

fmn::Job to_job(const fmn_request& r, bool reuse, u64* out) {
    fmn::Job j;
    j.out = out;
    if (r.op == FMN_OP_MUL_OPERAND) {
        const fmn_operand* o = r.operand;
        j.la = o->len;
        j.b = r.in2;
        j.lb = r.len2;
        j.sqr = 0;
        if (reuse && spectrum_pays(r)) {
            j.a = nullptr;
            j.spectrum = o->spec;
            j.log_n = o->log_n;
            j.engine = o->engine;
            j.splan = o->plan;
        } else {
            j.a = o->src;
        }
    } else {
        j.a = r.in1;
        j.la = r.len1;
        j.b = r.op == FMN_OP_SQR ? r.in1 : r.in2;
        j.lb = r.op == FMN_OP_SQR ? r.len1 : r.len2;
        j.sqr = r.op == FMN_OP_SQR;
    }
    return j;
}

u64 out_len_of(const fmn_request& r) {
    if (r.op == FMN_OP_MUL_OPERAND) return r.operand->len + r.len2;
    if (r.op == FMN_OP_SQR) return 2 * r.len1;
    return r.len1 + r.len2;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Transform length (log2) of a request's product.
int request_log_n(const fmn_request& r, bool reuse) {
    // in 64-bit points (a 32-bit spectrum has two digits per limb)
    if (r.op == FMN_OP_MUL_OPERAND && reuse && spectrum_pays(r))
        return r.operand->engine == fmn::ENGINE_32 ? r.operand->log_n - 1 : r.operand->log_n;
    const u64 ol = out_len_of(r);
    return ol > 1 ? ilog2c(ol - 1) : 0;
}

// Products this large run alone with the single-product kernels (they fill the GPU by
// themselves); smaller ones are batched, up to kBatchPoints transform points per batch.
constexpr int kAloneLogN = 20;
constexpr int kBigSlots = 2;               // batching mode: slots for large products
constexpr size_t kPrewarmBytes = 2ull << 30;   // pool memory mapped when the server is created
constexpr u64 kBatchPoints = 1ull << 22;

// Scratch a request is charged: its product workspace (as one batch of one, an upper
// bound of its share of a batch) plus a server-owned output when it has none.
size_t request_bytes(const fmn_request& r, bool reuse) {
    fmn::Job j = to_job(r, reuse, nullptr);
    size_t b = fmn::batch_workspace_bytes(&j, 1);
    if (!r.out) b += align256(out_len_of(r) * sizeof(u64));
    return b;
}

bool launch_unlocked(fmn_server* s, Slot* sl, const std::vector<fmn_request>& rq, std::vector<fmn::Job>& jobs,
                     size_t ws_bytes, size_t total, double* alloc_ms, std::string* err);

// Launch one batch of admitted requests on slot `sl` (dispatcher thread).  Called with the
// lock held; the requests are copied and the slot and its scratch budget taken under the lock,
// and the lock is released while the CUDA calls run (submissions and queries go on meanwhile;
// only the dispatcher launches, retires or touches slots and twiddle tables).
bool launch_batch(fmn_server* s, Slot* sl, const std::vector<size_t>& idx, std::unique_lock<std::mutex>& lk) {
    fmn::NvtxRange nvtx("fmn server batch launch");
    const clk::time_point t0 = clk::now();
    const bool reuse = s->batching != 0;
    std::vector<fmn_request> rq(idx.size());
    std::vector<fmn::Job> jobs(idx.size());
    size_t out_bytes = 0;
    for (size_t k = 0; k < idx.size(); ++k) {
        rq[k] = s->log[idx[k]].r;
        if (!rq[k].out) out_bytes += align256(out_len_of(rq[k]) * sizeof(u64));
        jobs[k] = to_job(rq[k], reuse, rq[k].out);
    }
    // outputs owned by the server live after the batch workspace
    const bool single = jobs.size() == 1;
    size_t ws_bytes = single ? fmn::job_workspace_bytes(jobs[0]) : fmn::batch_workspace_bytes(jobs.data(), (int)jobs.size());
    ws_bytes = align256(ws_bytes);
    const size_t total = ws_bytes + out_bytes;
    sl->busy = true;
    sl->reqs = idx;
    sl->bytes = total;
    s->in_use += total;
    if (s->in_use > s->peak) s->peak = s->in_use;
    lk.unlock();
    double alloc_ms = 0.0;
    std::string err;
    const bool ok = launch_unlocked(s, sl, rq, jobs, ws_bytes, total, &alloc_ms, &err);
    lk.lock();
    s->alloc_ms += alloc_ms;
    if (alloc_ms > s->max_alloc_ms) s->max_alloc_ms = alloc_ms;
    if (ok) {
        ++s->batches;
    } else {
        if (!err.empty()) s->error = err;
        s->in_use -= total;
        sl->busy = false;
        sl->reqs.clear();
        sl->bytes = 0;
    }
    const double lms = std::chrono::duration<double, std::milli>(clk::now() - t0).count();
    s->launch_ms += lms;
    if (lms > s->max_launch_ms) s->max_launch_ms = lms;
    return ok;
}

bool launch_unlocked(fmn_server* s, Slot* sl, const std::vector<fmn_request>& rq, std::vector<fmn::Job>& jobs,
                     size_t ws_bytes, size_t total, double* alloc_ms, std::string* err) {
    const bool single = jobs.size() == 1;
    void* mem = nullptr;
    const clk::time_point ta = clk::now();
    const cudaError_t ea = cudaMallocFromPoolAsync(&mem, total, s->pool, sl->stream);
    *alloc_ms = std::chrono::duration<double, std::milli>(clk::now() - ta).count();
    if (ea != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    char* ob = (char*)mem + ws_bytes;
    for (size_t k = 0; k < rq.size(); ++k) {
        const fmn_request& r = rq[k];
        if (!r.out) {
            jobs[k].out = (u64*)ob;
            ob += align256(out_len_of(r) * sizeof(u64));
        }
        if (jobs[k].la && jobs[k].lb && fmn::job_engine(jobs[k]) == fmn::ENGINE_64) {
            const int n = jobs[k].spectrum ? jobs[k].log_n
                          : single      ? fmn::job_twiddle_log_n(jobs[k])    // a single product may be wrapped
                                        : ilog2c(jobs[k].la + jobs[k].lb - 1);
            ensure_server_twiddles(s, n, sl->stream);
        }
    }
    cudaError_t e = cudaMemsetAsync(mem, 0, 256, sl->stream);     // status word
    if (e == cudaSuccess) {
        if (!single) {
            const size_t sb = fmn::batch_stage_bytes(jobs.data(), (int)jobs.size());
            if (sl->stage_cap < sb) {
                if (sl->stage) cudaFreeHost(sl->stage);
                sl->stage = nullptr;
                sl->stage_cap = 0;
                if (cudaMallocHost(&sl->stage, sb) == cudaSuccess) sl->stage_cap = sb;
            }
            e = sl->stage ? fmn::enqueue_batch(jobs.data(), (int)jobs.size(), mem, ws_bytes, sl->stage, sl->stage_cap,
                                               sl->stream, nullptr, nullptr, 0, server_twiddles, s)
                          : cudaErrorMemoryAllocation;
        } else {
            const int n = jobs[0].spectrum ? jobs[0].log_n
                          : (jobs[0].la && jobs[0].lb ? fmn::job_twiddle_log_n(jobs[0]) : 0);
            e = fmn::enqueue_job(jobs[0], mem, ws_bytes, sl->stream, server_twiddles(s, n));
        }
    }
    for (size_t k = 0; k < rq.size() && e == cudaSuccess; ++k) {
        const fmn_request& r = rq[k];
        if (r.check) {
            k_compare<<<148, 256, 0, sl->stream>>>(jobs[k].out, r.check, out_len_of(r), s->d_mismatch);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) {                // a bounded wait that expired -> error counter
        k_fold_status<<<1, 32, 0, sl->stream>>>((const unsigned*)mem, s->d_mismatch + 1);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(sl->done, sl->stream);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *err = cudaGetErrorString(e);
        cudaFreeAsync(mem, sl->stream);
        return false;
    }
    sl->mem = mem;
    return true;
}

void retire(fmn_server* s, Slot* sl, clk::time_point done_at) {
    for (size_t i : sl->reqs) {
        s->log[i].done = done_at;
        s->completed_order.push_back(i);
    }
    cudaFreeAsync(sl->mem, sl->stream);
    s->in_use -= sl->bytes;
    sl->mem = nullptr;
    sl->bytes = 0;
    sl->reqs.clear();
    sl->busy = false;
}

void dispatcher(fmn_server* s) {
    cudaSetDevice(s->dev);
    std::unique_lock<std::mutex> lk(s->mu);
    while (true) {
        bool progress = false;
        const size_t done_before = s->completed_order.size();
        // finished batches: plain mode in launch order (one stream), batching mode any slot
        auto finished = [](Slot* sl) {
            const cudaError_t q = cudaEventQuery(sl->done);
            if (q == cudaErrorNotReady) cudaGetLastError();
            return q != cudaErrorNotReady;
        };
        if (!s->batching) {
            while (!s->fifo.empty() && finished(s->fifo.front())) {
                retire(s, s->fifo.front(), clk::now());
                s->fifo.pop_front();
                progress = true;
            }
        } else {
            for (Slot* sl : s->slots)
                if (sl->busy && finished(sl)) {
                    retire(s, sl, clk::now());
                    progress = true;
                }
        }
        if (progress) s->cv.notify_all();
        // admission, each queue in arrival order, while budget and a slot allow.  Batching
        // mode: the first kBigSlots slots take large products one per slot (each nearly fills
        // the GPU; two let the next one queue behind the running one), the other slots take
        // batches of small ones, so small requests never queue behind large ones.
        auto reject_if_too_big = [&](std::deque<size_t>& q) {
            while (!q.empty() && request_bytes(s->log[q.front()].r, s->batching != 0) > s->budget) {
                const size_t i = q.front();
                q.pop_front();
                s->log[i].done = clk::now();
                ++s->rejected;
                s->completed_order.push_back(i);
            }
        };
        auto launch_or_fail = [&](Slot* sl, const std::vector<size_t>& take) {
            if (launch_batch(s, sl, take, lk)) {
                if (!s->batching) s->fifo.push_back(sl);
            } else {
                for (size_t i : take) {                // could not launch: fail these requests
                    s->log[i].done = clk::now();
                    ++s->failures;
                    s->completed_order.push_back(i);
                }
            }
            progress = true;
        };
        if (s->batching && !s->paused) {
            reject_if_too_big(s->big);
            for (int k = 0; k < kBigSlots && !s->big.empty(); ++k) {
                if (s->slots[k]->busy) continue;
                const size_t i = s->big.front();
                if (s->in_use + request_bytes(s->log[i].r, true) > s->budget) break;
                s->big.pop_front();
                launch_or_fail(s->slots[k], std::vector<size_t>{i});
            }
        }
        while (!s->paused) {
            reject_if_too_big(s->pending);
            if (s->pending.empty()) break;
            Slot* free_slot = nullptr;
            for (size_t k = s->batching ? kBigSlots : 0; k < s->slots.size(); ++k)
                if (!s->slots[k]->busy) {
                    free_slot = s->slots[k];
                    break;
                }
            if (!free_slot) break;
            std::vector<size_t> take;
            size_t bytes = 0;
            u64 points = 0;
            const bool reuse = s->batching != 0;
            while (!s->pending.empty() && (int)take.size() < s->max_batch) {
                const size_t i = s->pending.front();
                const size_t b = request_bytes(s->log[i].r, reuse);
                const int n = request_log_n(s->log[i].r, reuse);
                if (!take.empty() && points + (1ull << n) > kBatchPoints) break;
                if (s->in_use + bytes + b > s->budget) break;
                bytes += b;
                points += 1ull << n;
                take.push_back(i);
                s->pending.pop_front();
            }
            if (take.empty()) break;
            launch_or_fail(free_slot, take);
        }
        if (s->completed_order.size() != done_before) s->cv.notify_all();
        if (s->stop && s->pending.empty() && s->big.empty()) {
            bool busy = false;
            for (Slot* sl : s->slots) busy |= sl->busy;
            if (!busy) break;
        }
        if (!progress) s->cv.wait_for(lk, std::chrono::microseconds(20));
    }
}

}  // namespace

extern "C" {

int fmn_operand_create(const u64* d_in, u64 len, u64 max_partner_len, void* stream, fmn_operand** out) {
    fmn::NvtxRange nvtx("fmn operand create");
    if (!out || !d_in || len == 0 || max_partner_len == 0) return fmn::api_set_error(FMN_ERR_ARG, "bad operand", cudaSuccess);
    *out = nullptr;
    if (len + max_partner_len - 1 > (1ull << fmn::MAX_LOG_N) || (len < max_partner_len ? len : max_partner_len) >= (1ull << 56))
        return fmn::api_set_error(FMN_ERR_TOO_LARGE, "resident operand too large", cudaSuccess);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fmn::api_set_error(FMN_ERR_CUDA, "cudaGetDevice", e);
    fmn_operand* o = new fmn_operand();
    o->dev = dev;
    o->src = d_in;
    o->len = len;
    o->max_partner = max_partner_len;
    // the 32-bit engine wherever it can hold the spectrum (its products cost about half)
    const int n32 = fmn::default_engine() == fmn::ENGINE_64 ? -1 : fmn::q32_spectrum_log_n(len, max_partner_len);
    o->engine = n32 >= 0 ? fmn::ENGINE_32 : fmn::ENGINE_64;
    o->log_n = n32 >= 0 ? n32 : ilog2c(len + max_partner_len - 1);
    o->plan = n32 >= 0 ? fmn::q32_make_plan(o->log_n) : fmn::make_plan(o->log_n);
    const size_t bytes = 3 * ((size_t)1 << o->log_n) * (n32 >= 0 ? sizeof(unsigned) : sizeof(u64));
    if ((e = cudaMalloc((void**)&o->spec, bytes)) != cudaSuccess) {
        cudaGetLastError();
        delete o;
        return fmn::api_set_error(FMN_ERR_NOMEM, "resident operand spectrum", e);
    }
    e = o->engine == fmn::ENGINE_32
            ? fmn::q32_spectrum_enqueue(d_in, len, o->log_n, o->spec, (cudaStream_t)stream, o->plan)
            : fmn::spectrum_enqueue(d_in, len, o->log_n, o->spec, (cudaStream_t)stream, nullptr, o->plan);
    if (e != cudaSuccess ||
        (e = cudaStreamSynchronize((cudaStream_t)stream)) != cudaSuccess) {
        cudaFree(o->spec);
        delete o;
        return fmn::api_set_error(FMN_ERR_CUDA, "transforming the resident operand", e);
    }
    *out = o;
    return FMN_OK;
}

void fmn_operand_destroy(fmn_operand* o) {
    if (!o) return;
    cudaDeviceSynchronize();
    cudaFree(o->spec);
    delete o;
}

u64 fmn_operand_len(const fmn_operand* o) { return o ? o->len : 0; }

int fmn_mul_operand_ws(const fmn_operand* o, const u64* d_in2, u64 len2, u64* d_out, void* d_ws, size_t ws_bytes,
                       void* stream) {
    if (!o || !d_in2 || !d_out || !d_ws) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    if (len2 > o->max_partner) return fmn::api_set_error(FMN_ERR_ARG, "partner longer than the operand allows", cudaSuccess);
    fmn::Job j;
    j.a = nullptr;
    j.la = o->len;
    j.b = d_in2;
    j.lb = len2;
    j.out = d_out;
    j.sqr = 0;
    j.spectrum = o->spec;
    j.log_n = o->log_n;
    j.engine = o->engine;
    j.splan = o->plan;
    if (len2 == 0) {
        cudaError_t e = cudaMemsetAsync(d_out, 0, (o->len + len2) * sizeof(u64), (cudaStream_t)stream);
        return e == cudaSuccess ? FMN_OK : fmn::api_set_error(FMN_ERR_CUDA, "cudaMemsetAsync", e);
    }
    if (ws_bytes < fmn::job_workspace_bytes(j)) return fmn::api_set_error(FMN_ERR_ARG, "workspace too small", cudaSuccess);
    cudaError_t e = cudaMemsetAsync(d_ws, 0, sizeof(unsigned), (cudaStream_t)stream);
    if (e == cudaSuccess) e = fmn::enqueue_job(j, d_ws, ws_bytes, (cudaStream_t)stream, nullptr);
    return e == cudaSuccess ? FMN_OK : fmn::api_set_error(FMN_ERR_CUDA, "kernel launch", e);
}

size_t fmn_operand_workspace_size(const fmn_operand* o, u64 len2) {
    if (!o) return 0;
    fmn::Job j;
    j.a = nullptr;
    j.la = o->len;
    j.b = nullptr;
    j.lb = len2;
    j.out = nullptr;
    j.sqr = 0;
    j.spectrum = o->spec;
    j.log_n = o->log_n;
    j.engine = o->engine;
    j.splan = o->plan;
    return fmn::job_workspace_bytes(j);
}

int fmn_server_create(int device, size_t hbm_budget, int max_batch, int batching, fmn_server** out) {
    if (!out || max_batch < 1) return fmn::api_set_error(FMN_ERR_ARG, "bad server arguments", cudaSuccess);
    *out = nullptr;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return fmn::api_set_error(FMN_ERR_CUDA, "cudaSetDevice", e);
    if ((e = fmn::prepare_batch()) != cudaSuccess) return fmn::api_set_error(FMN_ERR_CUDA, "preparing kernels", e);
    fmn_server* s = new fmn_server();
    s->dev = device;
    s->budget = hbm_budget;
    s->max_batch = batching ? max_batch : 1;
    s->batching = batching;
    s->nslots = batching ? kBigSlots + 3 : 64;   // plain mode: many products queued on one stream
    cudaStream_t plain = nullptr;
    if (!batching && (e = cudaStreamCreateWithFlags(&plain, cudaStreamNonBlocking)) != cudaSuccess) {
        delete s;
        return fmn::api_set_error(FMN_ERR_CUDA, "stream", e);
    }
    for (int k = 0; k < s->nslots; ++k) {
        Slot* sl = new Slot();
        s->slots.push_back(sl);
        if ((e = cudaEventCreateWithFlags(&sl->done, cudaEventDisableTiming)) != cudaSuccess) break;
        if (batching) {
            if ((e = cudaStreamCreateWithFlags(&sl->stream, cudaStreamNonBlocking)) != cudaSuccess) break;
        } else {
            sl->stream = plain;            // one in-order stream: the plain per-call path
        }
    }
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = device;
    if (e == cudaSuccess) e = cudaMemPoolCreate(&s->pool, &props);
    if (e == cudaSuccess) {
        u64 thr = ~0ull;                   // keep freed memory in the pool
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    // Map the pool's first memory now (min(budget, kPrewarmBytes), allocated once and returned):
    // the first allocation of a fresh pool maps physical memory, which took 0.19-1.4 s on B200
    // in the middle of a served stream, and every request waited behind it.
    if (e == cudaSuccess && s->slots.size()) {
        const size_t warm = std::min(s->budget, kPrewarmBytes);
        void* p = nullptr;
        if (cudaMallocFromPoolAsync(&p, warm, s->pool, s->slots[0]->stream) == cudaSuccess) {
            cudaFreeAsync(p, s->slots[0]->stream);
            e = cudaStreamSynchronize(s->slots[0]->stream);
        } else {
            cudaGetLastError();            // not enough free memory now: the pool grows on demand
        }
    }
    if (e == cudaSuccess) e = cudaMalloc((void**)&s->d_mismatch, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemset(s->d_mismatch, 0, 2 * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->h_mismatch, 2 * sizeof(unsigned));
    if (e != cudaSuccess) {
        cudaGetLastError();
        fmn_server_destroy(s);
        return fmn::api_set_error(FMN_ERR_CUDA, "creating the server", e);
    }
    s->thr = std::thread(dispatcher, s);
    *out = s;
    return FMN_OK;
}

static int submit_at(fmn_server* s, const fmn_request* r, clk::time_point arrival);

int fmn_server_submit(fmn_server* s, const fmn_request* r) { return submit_at(s, r, clk::now()); }

static int submit_at(fmn_server* s, const fmn_request* r, clk::time_point arrival) {
    if (!s || !r) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    if (r->op < 0 || r->op > 2 || (r->op == FMN_OP_MUL_OPERAND && !r->operand) ||
        (r->op != FMN_OP_MUL_OPERAND && !r->in1) || (r->op == FMN_OP_MUL && !r->in2))
        return fmn::api_set_error(FMN_ERR_ARG, "bad request", cudaSuccess);
    if (r->op == FMN_OP_MUL_OPERAND && r->len2 > r->operand->max_partner)
        return fmn::api_set_error(FMN_ERR_ARG, "partner longer than the operand allows", cudaSuccess);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        Req q;
        q.r = *r;
        q.arrival = arrival;
        q.done = clk::time_point();
        q.bytes = 0;
        q.cancelled = false;
        s->log.push_back(q);
        const size_t i = s->log.size() - 1;
        if (s->batching && request_log_n(*r, true) >= kAloneLogN) s->big.push_back(i);
        else s->pending.push_back(i);
    }
    s->cv.notify_all();
    return FMN_OK;
}

int fmn_server_wait(fmn_server* s) {
    if (!s) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    std::unique_lock<std::mutex> lk(s->mu);
    // a paused server admits nothing: waiting for its queued requests would never end
    auto held = [&] { return s->paused && (!s->pending.empty() || !s->big.empty()); };
    s->cv.wait(lk, [&] { return s->completed_order.size() == s->log.size() || held(); });
    if (s->completed_order.size() != s->log.size())
        return fmn::api_set_error(FMN_ERR_ARG, "server paused with requests waiting for admission", cudaSuccess);
    return s->failures ? fmn::api_set_error(FMN_ERR_CUDA, s->error.empty() ? "launch failed" : s->error.c_str(), cudaSuccess)
                       : FMN_OK;
}

int fmn_server_pause(fmn_server* s, int paused) {
    if (!s) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->paused = paused != 0;
    }
    s->cv.notify_all();
    return FMN_OK;
}

int fmn_server_cancel(fmn_server* s, u64 tag) {
    if (!s) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    int n = 0;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        const clk::time_point now = clk::now();
        for (std::deque<size_t>* q : {&s->pending, &s->big})
            for (auto it = q->begin(); it != q->end();) {
                Req& r = s->log[*it];
                if (r.r.tag != tag) {
                    ++it;
                    continue;
                }
                r.cancelled = true;
                r.done = now;
                s->completed_order.push_back(*it);
                ++s->cancelled;
                ++n;
                it = q->erase(it);
            }
    }
    s->cv.notify_all();
    return n ? FMN_OK : fmn::api_set_error(FMN_ERR_ARG, "no request with this tag is waiting for admission", cudaSuccess);
}

int fmn_server_take(fmn_server* s, u64* tags, double* latency_ms, int max, int* n) {
    if (!s || !n) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    std::lock_guard<std::mutex> lk(s->mu);
    int k = 0;
    while (k < max && s->taken < s->completed_order.size()) {
        const Req& q = s->log[s->completed_order[s->taken++]];
        if (tags) tags[k] = q.r.tag;
        if (latency_ms) latency_ms[k] = std::chrono::duration<double, std::milli>(q.done - q.arrival).count();
        ++k;
    }
    *n = k;
    return FMN_OK;
}

int fmn_server_get_stats(fmn_server* s, fmn_server_stats* st) {
    if (!s || !st) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    std::lock_guard<std::mutex> lk(s->mu);
    memset(st, 0, sizeof(*st));
    st->submitted = s->log.size();
    st->completed = s->completed_order.size();
    st->rejected = s->rejected;
    st->failed = s->failures;
    st->batches = s->batches;
    st->peak_bytes = s->peak;
    st->cancelled = s->cancelled;
    st->launch_ms = s->launch_ms;
    st->alloc_ms = s->alloc_ms;
    st->max_launch_ms = s->max_launch_ms;
    st->max_alloc_ms = s->max_alloc_ms;
    if (cudaMemcpy(s->h_mismatch, s->d_mismatch, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost) == cudaSuccess) {
        st->mismatches = s->h_mismatch[0];
        st->device_errors = s->h_mismatch[1];
    }
    return FMN_OK;
}

// Open-loop replay: request i is submitted at arrival_s[i] seconds after the start
// (whatever the server's state), then all are awaited; latency_ms[i] = completion -
// scheduled arrival.
int fmn_server_replay(fmn_server* s, const fmn_request* reqs, const double* arrival_s, int count, double* latency_ms,
                      double* wall_s) {
    if (!s || (count > 0 && (!reqs || !arrival_s))) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    size_t first;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        first = s->log.size();
    }
    const clk::time_point t0 = clk::now();
    for (int i = 0; i < count; ++i) {
        const clk::time_point at = t0 + std::chrono::duration_cast<clk::duration>(std::chrono::duration<double>(arrival_s[i]));
        while (clk::now() < at) {
        }
        int rc = submit_at(s, &reqs[i], at);   // latency counts from the scheduled arrival
        if (rc) return rc;
    }
    int rc = fmn_server_wait(s);
    const clk::time_point t1 = clk::now();
    if (wall_s) *wall_s = std::chrono::duration<double>(t1 - t0).count();
    if (latency_ms) {
        std::lock_guard<std::mutex> lk(s->mu);
        for (int i = 0; i < count; ++i) {
            const Req& q = s->log[first + i];
            latency_ms[i] = std::chrono::duration<double, std::milli>(q.done - q.arrival).count();
        }
    }
    return rc;
}

void fmn_server_destroy(fmn_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv.notify_all();
    if (s->thr.joinable()) s->thr.join();
    cudaSetDevice(s->dev);
    cudaDeviceSynchronize();
    bool plain_freed = false;
    for (Slot* sl : s->slots) {
        if (sl->stage) cudaFreeHost(sl->stage);
        if (sl->done) cudaEventDestroy(sl->done);
        if (sl->stream && (s->batching || !plain_freed)) {
            cudaStreamDestroy(sl->stream);
            plain_freed = true;
        }
        delete sl;
    }
    for (auto& t : s->tw) cudaFree(t.first);
    if (s->pool) cudaMemPoolDestroy(s->pool);
    if (s->d_mismatch) cudaFree(s->d_mismatch);
    if (s->h_mismatch) cudaFreeHost(s->h_mismatch);
    delete s;
}

}  // extern "C"
