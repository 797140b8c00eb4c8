// fmn_internal.h -- host-side interface between the C ABI layer (fmn_api.cu) and the
// kernel launchers (fmn_ntt.cu).  Not installed; include/fast_mul.h is the public header.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <nvtx3/nvToolsExt.h>

#include <vector>

typedef unsigned long long u64;

namespace fmn {

// A named range on the host timeline of profilers (NVTX; header-only, a no-op unless a tool
// such as Nsight Systems is attached): one per product, batch or server launch.
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr int MAX_PASS_BITS = 9;     // largest sub-transform one CTA pass performs (2^9 points)
constexpr int MAX_LOG_N = 30;        // largest transform length supported (twiddle tables)
constexpr int MAX_PASSES = 4;

// How a length-2^n transform is split into passes (four-step decomposition, most
// significant index bits first).
struct Plan {
    int n;                    // log2 transform length
    int passes;               // number of passes
    int bits[MAX_PASSES];     // index bits handled by each pass (sum = n)
};
Plan make_plan(int log_n);          // the plan in effect (tuned or default)
Plan default_plan(int log_n);
bool valid_plan(const Plan& p);
bool same_plan(const Plan& a, const Plan& b);
bool set_plan(const Plan& p);       // replaces the plan of p.n; false if invalid
void clear_plan(int log_n);         // back to the default
std::vector<Plan> candidate_plans(int log_n);

// One product on the device.  All pointers are device pointers.
struct Job {
    const u64* a;      // in1 limbs (unused when `spectrum` is set)
    u64 la;
    const u64* b;      // in2 limbs (ignored when sqr)
    u64 lb;
    u64* out;          // la + lb limbs
    int sqr;
    // Resident first operand (conv_single reuse): its forward spectrum, computed by
    // spectrum_enqueue for a transform of 2^log_n points; la is its length.  Null otherwise.
    const u64* spectrum = nullptr;
    int log_n = 0;
    int engine = 0;    // ENGINE_*: 0 follows the process-wide default; with `spectrum`, the
                       // engine that spectrum belongs to (log_n in that engine's points)
    Plan splan = Plan{};   // with `spectrum`: the pass plan it was transformed with
    bool no_wrap = false;  // 64-bit engine: never the wrapped plan (fixed-size scratch)
};

// Residue engines.  ENGINE_64 transforms 64-bit limbs modulo the reference's three 62-bit
// primes (fmn_ntt.cu); ENGINE_32 transforms 32-bit digits modulo three 31-bit primes
// (fmn_ntt32.cu), which is faster; it transforms at most 2^26 digits, so it runs products of up
// to 2^25 limbs whole and splits longer ones whose shorter operand has at most 2^25 limbs.
// ENGINE_AUTO takes the one with the lower modelled cost (ENGINE_32 wherever it applies,
// except where a split would need many pieces).  Both give the same integer product.
// Batched products take ENGINE_32 when their whole transform fits it (batch_engine), resident
// operands when their spectrum fits it (fmn_operand_create); ENGINE_64 otherwise.
enum Engine { ENGINE_AUTO = 0, ENGINE_64 = 1, ENGINE_32 = 2 };
void set_default_engine(int engine);
int default_engine();
int job_engine(const Job& j);      // the engine that runs j (never ENGINE_AUTO)
bool q32_fits(u64 la, u64 lb, int sqr);        // the 32-bit engine can run this product
double q32_cost(u64 la, u64 lb, int sqr);      // its modelled cost (32-bit points x bits)
size_t q32_workspace_bytes(u64 la, u64 lb, int sqr);
int q32_launches(u64 la, u64 lb, int sqr);
int q32_pieces(u64 la, u64 lb, int sqr);        // 1: whole product; > 1: split into pieces
size_t q32_job_workspace_bytes(const Job& j);  // also for a product with a 32-bit resident spectrum
// Transform length (log2 digits) of a 32-bit resident spectrum for products of `len` limbs with
// partners of up to max_partner limbs; < 0 if the 32-bit engine cannot hold it.
int q32_spectrum_log_n(u64 len, u64 max_partner);
// Builds, on the current device, the four-step twiddle tables that the 32-bit engine's
// current pass plans use (about 110 MB with the B200 plans), so that no product meets a
// first-use build (an allocation and a stream synchronisation) while others run.
cudaError_t q32_prepare_tables();
// Frees those tables on device `dev` (its context is being shut down).
void q32_release_tables(int dev);
// Forward transform of `len` limbs into a 32-bit resident spectrum (3 * 2^log_n u32).
cudaError_t q32_spectrum_enqueue(const u64* src, u64 len, int log_n, void* spec, cudaStream_t s, const Plan& plan);
void q32_force_pieces(int m);                  // tests: split into m pieces where possible (0: model)
// tests: every product that allows it wrapped with the low product (1) or twisted (2); 0: model
void q32_force_wrap(int mode);
// Twisted length M of a wrapped product computed modulo X^M - c (0: not twisted).
u64 q32_twisted(u64 la, u64 lb, int sqr);
// Coefficients of the product that wrap around its transform length (0: not a wrapped product).
u64 q32_wrapped(u64 la, u64 lb, int sqr);
// Tests: the CRT + carry kernel with one look-back tile withheld (see fmn_ntt32.cu).
cudaError_t q32_test_carry_timeout(u64 out_len, unsigned* status);
// Pass plans of the 32-bit engine (2^n digits, n <= 26), tuned or set per length.
Plan q32_make_plan(int log_n);
Plan q32_default_plan(int log_n);
bool q32_valid_plan(const Plan& p);
bool q32_set_plan(const Plan& p);
void q32_clear_plan(int log_n);
std::vector<Plan> q32_candidate_plans(int log_n);
typedef cudaError_t (*ChunkDone)(void* ctx, u64 first_limb, u64 end_limb);
// Called before the first launch that reads limbs [first, end) of the second operand: it must
// make stream s wait until those limbs are in device memory (e.g. an event after their copy).
typedef cudaError_t (*NeedLimbs)(void* ctx, u64 first_limb, u64 end_limb, cudaStream_t s);
cudaError_t q32_enqueue(const Job& j, void* ws, size_t ws_bytes, cudaStream_t s, NeedLimbs need_b, void* need_ctx,
                        int crt_chunks, ChunkDone after_chunk, void* ctx);

// Forward transform of `len` limbs at `src` into `spec` (3 * 2^log_n u64): the spectrum a
// resident operand keeps for products of up to 2^log_n - len + 1 partner limbs.
cudaError_t spectrum_enqueue(const u64* src, u64 len, int log_n, u64* spec, cudaStream_t s,
                             const struct TwiddleSet* tw, const Plan& plan);

// Scratch needed by one product: residue arrays + carry-scan state.
size_t job_workspace_bytes(u64 la, u64 lb, int sqr);
size_t job_workspace_bytes(const Job& j);

// Upload twiddle tables to the current device (idempotent per device).
cudaError_t ensure_tables();

// Precomputed four-step twiddles of every strided pass of one transform length.
struct TwiddleSet {
    TwiddleSet() : log_n(0), plan{}, fwd{}, inv{} {}
    int log_n;
    Plan plan;             // the pass plan the tables were built for
    const u64* fwd[MAX_PASSES];
    const u64* inv[MAX_PASSES];
};
typedef const TwiddleSet* (*TwiddleLookup)(void* ctx, int log_n);

// Device bytes the tables of a length-2^log_n transform need (0 when it has one pass).
size_t twiddle_table_bytes(int log_n);
// Fill `buf` (twiddle_table_bytes(log_n) bytes) on `stream` and describe it in `out`.
cudaError_t build_twiddle_tables(int log_n, u64* buf, TwiddleSet* out, cudaStream_t stream);

// Enqueue one product on `stream` using `ws` (job_workspace_bytes(...) bytes, 256-byte
// aligned).  The first u32 of ws is an error word that the carry scan sets (never clears)
// when a bounded wait gives up; callers zero it once and read it after the stream is done.
// `tw` (optional) holds precomputed four-step twiddles for this transform length; without
// it the kernels generate them.
// tw_side: a wrapped 64-bit product's second product's tables (job_side_log_n), or null.
cudaError_t enqueue_job(const Job& job, void* ws, size_t ws_bytes, cudaStream_t stream,
                        const TwiddleSet* tw = nullptr, const TwiddleSet* tw_side = nullptr);

// A product with copy overlap: before the first launch that reads a range of the second
// operand's limbs, `need_b(need_ctx, first, end, s)` is called (the caller copies that range
// on another stream and makes s wait for it; a split product asks piece by piece), and the
// carry scan runs in chunks: after each, `after_chunk(ctx, first_limb, end_limb)` is called
// so the caller can copy those final limbs back while the rest computes.  A split product
// scans the limbs that a piece completes right after that piece.
cudaError_t enqueue_job_overlapped(const Job& j, void* ws, size_t ws_bytes, cudaStream_t s, const TwiddleSet* tw,
                                   NeedLimbs need_b, void* need_ctx, int crt_chunks, ChunkDone after_chunk, void* ctx,
                                   const TwiddleSet* tw_side = nullptr);

// ---- 32-bit engine batches (whole and twisted wrapped products; see enqueue_batch)
constexpr int Q32_MAX_REC = 2 * (3 * MAX_PASSES + 2);   // pass launches of a twisted product
struct Q32Group {
    int m, count;                           // products, pass launches per product
    int variant[Q32_MAX_REC], logl[Q32_MAX_REC];
    u64 tiles[Q32_MAX_REC];
    size_t args_off[Q32_MAX_REC];           // descriptor offsets: m launch-argument records each
    size_t crt_off, ncta_off;
    unsigned max_ncta;
    // twisted wrapped products (twist = log2 M > 0): the operands' folds (nfold of them), the
    // pass launches (twisted transform, then the cyclic one), the W kernel, the twisted CRT
    int twist, nfold;
    size_t fold_off[2], w_off;
    unsigned fold_bpj, w_bpj;
};
int q32_forced_wrap();                      // fmn_force_wrap mode (0: the cost model decides)
int job_twiddle_log_n(const Job& j);        // 64-bit engine: log2 of the main transform (twiddle tables)
u64 wrap64_for(const Job& j);               // 64-bit engine: K of a wrapped product, 0 if whole
u64 twist64_for(const Job& j);              // 64-bit engine: M of a twisted product, 0 otherwise
int job_side_log_n(const Job& j);           // 64-bit engine: log2 of a wrapped product's second transform, 0 if whole
int q32_batch_log_n(const Job& j);          // (cyclic) transform log length, < 0 if not a 32-bit batch product
int q32_batch_twist_log(const Job& j);      // log2 M of a batched product run twisted, 0 for a whole product
size_t q32_batch_res_bytes(const Job& j);   // residue arrays of one product
size_t q32_batch_state_bytes(const Job& j); // carry-scan ticket + state of one product
size_t q32_batch_desc_bytes_per_job();      // descriptor bytes one product needs (upper bound)
// Plan the group jobs[idx[0..m)] (same transform length and kind): scratch carved from `res`
// and `st` at *roff / *soff (advanced), descriptors written into host staging `h` at 16-byte
// aligned offsets from *hoff (advanced, at most hcap).
cudaError_t q32_batch_plan(const Job* jobs, const int* idx, int m, char* res, size_t* roff, char* st, size_t* soff,
                           unsigned* err, char* h, size_t* hoff, size_t hcap, Q32Group* g);
// Launch a planned group whose descriptors were copied to d_desc (same offsets as in h).
cudaError_t q32_batch_launch(const Q32Group& g, const char* d_desc, cudaStream_t s);
cudaError_t q32_prepare();                  // tables + kernel attributes on the current device

// ---- batches of products
u64 batch_twist_for(const Job& j);          // M of a batched product run twisted, 0 if whole
bool batch_on_engine64(const Job& j);       // a batched product that runs on the 64-bit engine
// Workspace bytes for a batch (device) and host staging bytes for its launch descriptors.
size_t batch_workspace_bytes(const Job* jobs, int count);
size_t batch_stage_bytes(const Job* jobs, int count);
// Enqueue a batch on `s`.  Products are grouped by transform length and kind; every group
// runs its stages as batched launches on one of `streams` (forked from and joined into s
// with `events`, which needs nstreams + 1 events).  `h_stage` is pinned host memory of
// batch_stage_bytes bytes that must stay untouched until the stream has consumed it.
// `tw_lookup` (optional) returns cached twiddle tables per transform length.
cudaError_t enqueue_batch(const Job* jobs, int count, void* ws, size_t ws_bytes, void* h_stage,
                          size_t stage_bytes, cudaStream_t s, const cudaStream_t* streams,
                          const cudaEvent_t* events, int nstreams, TwiddleLookup tw_lookup, void* tw_ctx);

// Make sure every batched kernel is configured (call before capturing a batch in a graph).
cudaError_t prepare_batch();

// Description of the most recent pass launch of this thread (for error messages).
const char* launch_diag();

// ---- optional per-kernel timing (used by bench.py; off by default)
// Kernel kinds of the pipeline.
// K_WRAP: the fold and W kernels of twisted wrapped products.
enum KernelKind { K_FWD = 0, K_FWD_LAST, K_FUSED, K_INV, K_CRT, K_WRAP, K_KINDS };
const char* kernel_kind_name(int k);
struct KindStats {
    double ms;          // summed CUDA-event time
    u64 launches;
    double bytes;       // algorithmic HBM bytes (operands read once, spectra read/written once per pass)
    double modmuls;     // algorithmic Montgomery products (radix-2 butterflies, pointwise, entry, CRT)
};
// Enable/disable event recording around every launch of the calling thread.
void profile_enable(bool on);
// Recording around one launch (no-ops while profiling is off): prof_begin before the launch,
// prof_end after it, on the launch's stream.
struct ProfMark {
    int kind;
    cudaEvent_t a;
    double bytes, modmuls;
};
ProfMark prof_begin(int kind, double bytes, double modmuls, cudaStream_t s);
void prof_end(const ProfMark& m, cudaStream_t s);
// Wait for recorded events and add their times into out[K_KINDS]; clears the record.
cudaError_t profile_take(KindStats* out);
// Kernel launches one product issues.
int job_launches(u64 la, u64 lb, int sqr);

// splitmix64 limbs on the device (tuning runs).
cudaError_t fill_limbs(u64* p, u64 n, u64 seed, cudaStream_t s);

// Throughput microbenchmark of independent Montgomery products (peak of the integer pipe
// for this arithmetic): returns products per second.
cudaError_t bench_modmul(double* per_second, double* butterflies_per_second);
// Same for the 32-bit engine's butterfly (Shoup product plus reductions), per second.
cudaError_t q32_bench_bfly(double* per_second);

}  // namespace fmn

// A resident operand (include/fast_mul.h): its forward spectrum stays in device memory.
struct fmn_operand {
    int dev;
    int engine;          // fmn::ENGINE_64 or fmn::ENGINE_32: the layout of `spec`
    fmn::Plan plan;      // pass plan `spec` was transformed with (its products use the same)
    const u64* src;      // the caller's limbs (used by the plain per-call path)
    u64 len;
    int log_n;           // transform length of its products (points of its engine)
    u64 max_partner;     // longest partner it was sized for
    u64* spec;           // 3 * 2^log_n residues (u64 or u32 by engine), forward-transformed
};
