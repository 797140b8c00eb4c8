/*
 * fast_mul.h -- C ABI of the B200 (sm_100a) 3-prime NTT big-integer multiplication library.
 *
 * Drop-in for HJimmyK/fast_mul_ntt src/fast_mul.h: the two entry points below keep the
 * reference's names, argument meaning and error behaviour.  Numbers are little-endian
 * arrays of 64-bit limbs (least significant limb first).  Everything else is a namespaced
 * extension (fmn_*) for callers that want status codes, device pointers or batching.
 *
 * Link: -lfastmul_b200 (fast_mul_ntt_b200/lib/libfastmul_b200.so).  One CUDA device is used
 * per calling thread (the current device, or device 0).
 */
#ifndef FAST_MUL_B200_H
#define FAST_MUL_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long long u64;

/* out = in1 * in2; out has exactly len1 + len2 limbs, all written (the top limb may be 0).
 * in1 and in2 must not be the same block (their values may be equal); out may alias either
 * input.  Host pointers, synchronous.  On failure prints a message to stderr and calls
 * abort(), as the reference does on allocation failure.
 * Replaces: abs_mul64, src/fast_mul.h:39 (implementation src/fast_mul.c:308-396). */
void abs_mul64(const u64* in1, u64 len1, const u64* in2, u64 len2, u64* out);

/* out = in1 * in1; out has exactly 2 * len1 limbs.
 * Replaces: abs_sqr64, src/fast_mul.h:45 (implementation src/fast_mul.c:398-460). */
void abs_sqr64(const u64* in1, u64 len1, u64* out);

/* ----------------------------------------------------------------- extensions */

/* Status codes returned by every fmn_* call. */
enum {
    FMN_OK = 0,
    FMN_ERR_ARG = 1,        /* bad argument (null pointer, length out of range, in1 == in2) */
    FMN_ERR_CUDA = 2,       /* a CUDA runtime call failed; see fmn_last_error() */
    FMN_ERR_NOMEM = 3,      /* device or pinned host memory could not be allocated */
    FMN_ERR_DEVICE = 4,     /* a kernel reported an internal error (bounded wait expired) */
    FMN_ERR_TOO_LARGE = 5   /* transform length above 2^30 or coefficient range exceeded */
};

/* Select and initialise a device for the calling thread (optional: the first call does it
 * with the current device).  Uploads the twiddle tables.  Counterpart of
 * fft_small_init (fft_small/fft_small.h:33). */
int fmn_init(int device);
/* Release cached device and pinned buffers of this process (fft_small_clear,
 * fft_small/fft_small.h:34). */
void fmn_shutdown(void);
/* Text of the last error seen by the calling thread ("" if none). */
const char* fmn_last_error(void);

/* Status-returning forms of abs_mul64 / abs_sqr64 (host pointers, synchronous).
 * Host-pointer calls (these and abs_mul64 / abs_sqr64) may come from several threads at
 * once: each runs on one of a few host lanes per device (FMN_HOST_LANES, 1..8, default 4;
 * further callers wait for a free lane), with its own device workspace, operand buffers and
 * streams, so one call's host<->device copies overlap another's kernels.  Each lane keeps
 * device memory for the largest product it has run until fmn_shutdown(). */
int fmn_mul(const u64* in1, u64 len1, const u64* in2, u64 len2, u64* out);
int fmn_sqr(const u64* in1, u64 len1, u64* out);

/* Device-pointer forms, asynchronous on `stream` (a cudaStream_t, NULL = default stream).
 * Scratch comes from a per-device cache owned by the library; calls on one device are
 * serialised by a lock while they are enqueued.  Internal errors of the kernels are
 * reported by the next fmn_sync(stream). */
int fmn_mul_device(const u64* d_in1, u64 len1, const u64* d_in2, u64 len2, u64* d_out, void* stream);
int fmn_sqr_device(const u64* d_in1, u64 len1, u64* d_out, void* stream);
/* Wait for `stream` and report device-side errors of earlier fmn_*_device calls. */
int fmn_sync(void* stream);

/* Scratch a product needs, for callers that manage memory themselves. */
size_t fmn_workspace_size(u64 len1, u64 len2, int sqr);
/* Device-pointer product with caller-provided scratch (d_ws: fmn_workspace_size bytes,
 * 256-byte aligned, not shared by calls in flight).  No allocation, no lock.  The first
 * word of d_ws is a status word, cleared by this call and read by fmn_ws_status. */
int fmn_mul_device_ws(const u64* d_in1, u64 len1, const u64* d_in2, u64 len2, u64* d_out,
                      void* d_ws, size_t ws_bytes, void* stream);
/* After the stream has finished, read the device-side error flag of such a call. */
int fmn_ws_status(const void* d_ws, u64 len1, u64 len2, int sqr, void* stream);

/* Device-pointer product that allocates nothing, for callers that cannot call cudaMalloc
 * while they run (a plugin inside an application whose allocator owns the device memory, a
 * latency-critical loop that must not stall on allocation, a process with a fixed memory
 * plan).  Its scratch is one fixed array of about 3 MB in device memory, present on every
 * GPU that loads the library until exit, so it takes products with len1 + len2 <= 65537
 * limbs (transforms up to 2^16 points) and rejects larger ones with FMN_ERR_TOO_LARGE.
 * The first call on each device looks up the array's device address and uploads the
 * twiddle tables; make it before any stream capture.  Calls share the array: they are
 * serialised with respect to `stream` (each call is synchronous: it returns once its work on
 * `stream` has finished), and calls whose work overlaps on the GPU from other streams or
 * threads race on it.  It runs on FMN_ENGINE_64 with the pass plans in effect in the process
 * (it never loads the plan file itself, since that may allocate).
 * No counterpart in the reference (which allocates its scratch per call). */
int fmn_mul_device_noalloc(const u64* d_in1, u64 len1, const u64* d_in2, u64 len2, u64* d_out, void* stream);

/* ----------------------------------------------------------------- batches
 * Many independent products in a few launches: products are grouped by transform length
 * and kind (multiply / square) and each stage of a group runs as one batched launch, groups
 * running concurrently on internal streams.  No counterpart in the reference (which has
 * one product per call). */
typedef struct {
    const u64* in1;   /* device pointers; in1 == in2 with len1 == len2 is a square */
    u64 len1;
    const u64* in2;
    u64 len2;
    u64* out;         /* len1 + len2 limbs */
} fmn_job;

/* All products of `jobs` on `stream`, asynchronously; scratch from the library's cache.
 * Device-side errors are reported by the next fmn_sync(stream). */
int fmn_mul_batch_device(const fmn_job* jobs, int count, void* stream);

/* A batch captured once in a CUDA graph that owns its scratch; launching it recomputes all
 * products from the (possibly updated) contents of the same input buffers into the same
 * outputs, with one graph launch. */
typedef struct fmn_batch_graph fmn_batch_graph;
int fmn_batch_graph_create(const fmn_job* jobs, int count, fmn_batch_graph** out);
int fmn_batch_graph_launch(fmn_batch_graph* g, void* stream);
/* Wait for `stream` and report device-side errors of the graph's products. */
int fmn_batch_graph_sync(fmn_batch_graph* g, void* stream);
void fmn_batch_graph_destroy(fmn_batch_graph* g);

/* ----------------------------------------------------------------- resident operands
 * A number whose forward transform is computed once and kept in device memory; products
 * with it transform only the partner.  Counterpart of the reference's conv_single
 * (src/fast_mul.c:135-212), which multiplies by an already-transformed operand but which
 * the reference's driver never calls. */
typedef struct fmn_operand fmn_operand;
/* Transform `len` limbs at device pointer d_in for products with partners of up to
 * max_partner_len limbs (synchronous on `stream`).  d_in must stay valid while the operand
 * is used by a plain (non-batching) server. */
int fmn_operand_create(const u64* d_in, u64 len, u64 max_partner_len, void* stream, fmn_operand** out);
void fmn_operand_destroy(fmn_operand* op);
u64 fmn_operand_len(const fmn_operand* op);
/* d_out (len(op) + len2 limbs) = op * d_in2, asynchronously on `stream`. */
int fmn_mul_operand_device(const fmn_operand* op, const u64* d_in2, u64 len2, u64* d_out, void* stream);
/* Same with caller-provided scratch of fmn_operand_workspace_size bytes. */
size_t fmn_operand_workspace_size(const fmn_operand* op, u64 len2);
int fmn_mul_operand_ws(const fmn_operand* op, const u64* d_in2, u64 len2, u64* d_out, void* d_ws,
                       size_t ws_bytes, void* stream);

/* ----------------------------------------------------------------- product server
 * Continuous batching: requests submitted from any thread are admitted in arrival order
 * while their scratch fits the HBM budget and a slot (CUDA stream) is free; admitted
 * requests run as one batch, batches overlap on the device, and requests arriving meanwhile
 * join the next batch as slots and memory free up.  Large products (above 2^20 limbs) run
 * one per slot on two dedicated slots, so small requests never queue behind them.  A product
 * with a resident operand uses the operand's spectrum when that is modelled cheaper than
 * computing it from scratch (the spectrum has the length of the longest partner it was sized
 * for).  With batching = 0 the server is the plain per-call path: one product per launch
 * sequence, in arrival order, on one stream, without resident-operand reuse.  Scratch comes
 * from the server's own stream-ordered memory pool, of which min(budget, 2 GiB) is mapped when
 * the server is created (the first growth of a fresh pool stalled a running stream).  No
 * counterpart in the reference. */
enum { FMN_OP_MUL = 0, FMN_OP_SQR = 1, FMN_OP_MUL_OPERAND = 2 };
typedef struct {
    int op;                      /* FMN_OP_* */
    const u64* in1;              /* device pointers (in1 only for squares) */
    u64 len1;
    const u64* in2;              /* FMN_OP_MUL and FMN_OP_MUL_OPERAND */
    u64 len2;
    const fmn_operand* operand;  /* FMN_OP_MUL_OPERAND */
    u64* out;                    /* product; NULL: the server computes it into scratch and discards it */
    const u64* check;            /* optional expected product (device); mismatches are counted */
    u64 tag;                     /* returned by fmn_server_take */
} fmn_request;
typedef struct {
    u64 submitted, completed, rejected, failed, batches;
    u64 mismatches;              /* requests whose product differed from `check` */
    u64 device_errors;           /* batches whose carry scan reported a bounded-wait expiry */
    size_t peak_bytes;           /* highest scratch in use */
    u64 cancelled;               /* requests withdrawn by fmn_server_cancel (also in completed) */
    double launch_ms;            /* host time the dispatcher spent launching batches */
    double alloc_ms;             /* of which: taking scratch from the server's memory pool */
    double max_launch_ms;        /* the longest single batch launch */
    double max_alloc_ms;         /* the longest single pool allocation */
} fmn_server_stats;
typedef struct fmn_server fmn_server;
int fmn_server_create(int device, size_t hbm_budget_bytes, int max_batch, int batching, fmn_server** out);
int fmn_server_submit(fmn_server* s, const fmn_request* req);
/* Wait until every submitted request has completed. */
int fmn_server_wait(fmn_server* s);
/* Withdraw every request with this tag that is still waiting for admission: it is never
 * computed (its output is not written) and completes at once, counted in `cancelled`.
 * FMN_ERR_ARG if no such request is waiting (already admitted, finished or unknown); a
 * request already on the GPU runs to completion. */
int fmn_server_cancel(fmn_server* s, u64 tag);
/* Hold (paused = 1) or resume (0) admission: running batches finish, new and queued requests
 * wait.  fmn_server_wait returns FMN_ERR_ARG instead of blocking while paused requests wait. */
int fmn_server_pause(fmn_server* s, int paused);
/* Completed requests since the last call, in completion order: tags and latency
 * (completion - submission, milliseconds). */
int fmn_server_take(fmn_server* s, u64* tags, double* latency_ms, int max, int* n);
int fmn_server_get_stats(fmn_server* s, fmn_server_stats* st);
/* Open-loop replay: request i is submitted arrival_s[i] seconds after the start regardless
 * of the server's state; waits for all; latency_ms[i] = completion - scheduled arrival. */
int fmn_server_replay(fmn_server* s, const fmn_request* reqs, const double* arrival_s, int count,
                      double* latency_ms, double* wall_s);
void fmn_server_destroy(fmn_server* s);

/* ----------------------------------------------------------------- residue engines
 * Two interchangeable transforms compute every product; the result is the same integer.
 * FMN_ENGINE_64 works like the reference (src/fast_mul.c:308-460): 64-bit limbs modulo its
 * three 62-bit primes (src/data.h:79-81), for transforms up to 2^30 points.
 * FMN_ENGINE_32 splits each limb into two 32-bit digits and works modulo three 31-bit
 * primes, whose modular products are single 32-bit multiplies on the GPU; it covers
 * products whose shorter operand has at most 2^25 limbs (longer ones are split, see
 * fmn_pieces_for).  FMN_ENGINE_AUTO (the default)
 * takes FMN_ENGINE_32 wherever its modelled cost is lower and FMN_ENGINE_64 elsewhere.
 * Batches (and the batching server) run each product on FMN_ENGINE_32 when its whole
 * transform fits that engine (2 (len1 + len2) - 1 <= 2^26 digits) and on FMN_ENGINE_64
 * otherwise; a resident operand holds a FMN_ENGINE_32 spectrum when
 * 2 (len + max_partner_len) - 1 <= 2^26 digits and a FMN_ENGINE_64 one otherwise.  Under
 * fmn_set_engine(FMN_ENGINE_64) everything runs on FMN_ENGINE_64.  No counterpart in the
 * reference. */
#define FMN_ENGINE_AUTO 0
#define FMN_ENGINE_64 1
#define FMN_ENGINE_32 2
/* Process-wide engine choice for single products (FMN_ENGINE_32 falls back to
 * FMN_ENGINE_64 for products beyond its range).  Workspace sizes follow the choice. */
int fmn_set_engine(int engine);
int fmn_get_engine(void);
/* The engine (FMN_ENGINE_64 or FMN_ENGINE_32) that a product of these lengths runs on. */
int fmn_engine_for(u64 len1, u64 len2, int sqr);
/* Pieces the product is computed in: 1 = one transform of the whole product; m > 1 = the
 * shorter operand is transformed once and multiplied with m pieces of the longer one, each at
 * a smaller transform length (the reference's conv_single reuse, src/fast_mul.c:135-212),
 * and the pieces' coefficients are summed before one CRT + carry pass.  FMN_ENGINE_32 only;
 * chosen by a cost model (fewer butterflies for lengths that would pad a power of two
 * poorly, and the only way the 32-bit engine reaches unbalanced products above 2^25 limbs). */
int fmn_pieces_for(u64 len1, u64 len2, int sqr);
/* Testing and tuning: split every product that allows it into `pieces` pieces regardless of
 * the cost model (0 or 1 restores the model).  Process-wide. */
int fmn_force_pieces(int pieces);
/* Wrapped products (FMN_ENGINE_32): a product whose 2 (len1 + len2) - 1 digit coefficients
 * exceed a power of two 2^n by K, while both operands fit 2^n digits, can run as one cyclic
 * transform of 2^n digits (its first K coefficients then hold c_k + c_{k+2^n}) plus the
 * product of the operands' lowest ceil(K / 2) limbs, which gives c_0 .. c_{K-1}; the CRT
 * separates the two.  This replaces a transform of twice the length by one of the same length
 * and a small one: the padding a product just above a power of two would pay.  The twisted
 * form replaces the low product by the product modulo X^M - c (M = 2^m >= K, 2^n / M <= 4,
 * c^(2^n / M) = -1): one cyclic transform of M digits of both operands folded modulo X^M - c
 * and twisted, half the size of the low product; then c_{2^n + k} = W_k and c_k = U_k - W_k
 * with W = (U mod (X^M - c) - V) / 2.  The cost model chooses among whole, split, wrapped and
 * twisted plans; the 64-bit engine (the reference's primes) wraps too, with the low product
 * of the operands' lowest K limbs or the twisted form.  fmn_wrap_for returns K for a product
 * that runs wrapped (0 otherwise),
 * fmn_twist_for its twisted length M (0 when not twisted); fmn_force_wrap(1) wraps every
 * product that allows it with the low product, fmn_force_wrap(2) twisted (tests),
 * fmn_force_wrap(0) restores the model.  Batched products (fmn_mul_batch_device, the
 * server) run whole or twisted; fmn_batch_twist_for returns M for one that runs twisted in
 * a batch (0 when whole): there the per-product launch cost does not count, since a batch
 * shares its launches among its products.  No counterpart in the reference. */
u64 fmn_wrap_for(u64 len1, u64 len2, int sqr);
u64 fmn_twist_for(u64 len1, u64 len2, int sqr);
u64 fmn_batch_twist_for(u64 len1, u64 len2, int sqr);
int fmn_force_wrap(int mode);

/* ----------------------------------------------------------------- pass plans and tuning
 * A 2^n-point transform runs as passes of <= 9 index bits each; the split is a plan (e.g.
 * 2^25: 9+8+8).  Plans come from the default split, from fmn_set_plan, or from a plan file
 * written by fmn_autotune (which times every valid plan of each length on the current GPU
 * and keeps the fastest).  The library loads <lib dir>/../tune/plans-<gpu name>.txt (or the
 * file named by FMN_PLAN_FILE) when a device context is first created, if the file's GPU
 * name and driver version match.  No counterpart in the reference (its split is fixed). */
/* Passes of the plan in effect for 2^log_n points, bits written to bits[0..]; < 0 on error. */
int fmn_get_plan(int log_n, int* bits, int max_passes);
/* Replace the plan of 2^log_n points (passes == 0 restores the default). */
int fmn_set_plan(int log_n, const int* bits, int passes);
/* Time every valid plan for 2^n_lo .. 2^n_hi points and keep the fastest; save to
 * save_path (if not NULL) as a plan file. */
int fmn_autotune(int n_lo, int n_hi, const char* save_path);
/* The same per engine: FMN_ENGINE_64 as above, FMN_ENGINE_32 for its 2^log_n-digit transforms
 * (log_n <= 26; a strided pass leaves at least 32 columns).  A resident operand keeps the
 * plan it was transformed with.  Setting or loading 32-bit plans builds their four-step
 * twiddle tables on the current device right away (so no product waits for them). */
int fmn_get_plan_engine(int engine, int log_n, int* bits, int max_passes);
int fmn_set_plan_engine(int engine, int log_n, const int* bits, int passes);
int fmn_load_plans(const char* path);
int fmn_load_default_plans(void);

/* ----------------------------------------------------------------- measurement hooks
 * (no counterpart in the reference; used by bench.py) */

/* Kernel kinds of the pipeline, in this order: forward pass, forward last pass, fused
 * pointwise pass, inverse pass, CRT + carry, and the fold / W kernels of twisted wrapped
 * products. */
#define FMN_KERNEL_KINDS 6
const char* fmn_kernel_kind_name(int kind);
/* Record CUDA events around every kernel launch of the calling thread (on = 1) or stop. */
int fmn_profile_enable(int on);
/* Wait for the recorded launches and return, per kernel kind, summed device milliseconds,
 * launch count, algorithmic HBM bytes and algorithmic Montgomery products; clears the
 * record.  Each array has FMN_KERNEL_KINDS entries. */
int fmn_profile_take(double* ms, u64* launches, double* bytes, double* modmuls);
/* Number of kernel launches one product issues. */
int fmn_launches_per_product(u64 len1, u64 len2, int sqr);
/* Peak of this library's Montgomery product on the current device: a microbenchmark of
 * independent modmul chains and of decimation-in-frequency butterflies (per second). */
int fmn_bench_modmul(double* modmul_per_s, double* butterfly_per_s);
/* Peak of the 32-bit engine's butterfly (independent chains, per second). */
int fmn_bench_bfly32(double* butterfly_per_s);

/* ----------------------------------------------------------------- failure-handling tests
 * Hooks that make the library's error paths run without faulting the GPU (no counterpart in
 * the reference).
 * fmn_test_fail_allocs: the next `count` device allocations of product workspaces and operand
 * buffers fail as if cudaMalloc had found no memory, so fmn_mul returns FMN_ERR_NOMEM and
 * abs_mul64 prints the error and calls abort(), as the reference does when its allocation
 * fails (src/fast_mul.c:320-323).  0 turns it off.
 * fmn_test_carry_timeout: runs the CRT + carry kernel over a zero product of out_limbs limbs
 * (2 to 4096 tiles of 2048 limbs) with tile 0 withheld, so every later tile's bounded
 * look-back wait expires after a few milliseconds and sets the status word; returns
 * FMN_ERR_DEVICE, the status a product whose wait expired reports.  The device stays usable. */
int fmn_test_fail_allocs(int count);
int fmn_test_carry_timeout(u64 out_limbs);

/* Transform length used for a product: the next power of two >= len1 + len2 - 1
 * (int_ceil2, src/fast_mul.c:299-312). */
u64 fmn_ntt_len(u64 len1, u64 len2);

#ifdef __cplusplus
}
#endif

#endif /* FAST_MUL_B200_H */
