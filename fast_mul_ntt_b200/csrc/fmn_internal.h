// fmn_internal.h -- host-side interface between the C ABI layer (fmn_api.cu) and the
// kernel launchers (fmn_ntt.cu).  Not installed; include/fast_mul.h is the public header.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

typedef unsigned long long u64;

namespace fmn {

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
Plan make_plan(int log_n);

// One product on the device.  All pointers are device pointers.
struct Job {
    const u64* a;      // in1 limbs
    u64 la;
    const u64* b;      // in2 limbs (ignored when sqr)
    u64 lb;
    u64* out;          // la + lb limbs
    int sqr;
};

// Scratch needed by one product: residue arrays + carry-scan state.
size_t job_workspace_bytes(u64 la, u64 lb, int sqr);

// Upload twiddle tables to the current device (idempotent per device).
cudaError_t ensure_tables();

// Enqueue one product on `stream` using `ws` (job_workspace_bytes(...) bytes, 256-byte
// aligned).  The first u32 of ws is an error word that the carry scan sets (never clears)
// when a bounded wait gives up; callers zero it once and read it after the stream is done.
cudaError_t enqueue_job(const Job& job, void* ws, size_t ws_bytes, cudaStream_t stream);

}  // namespace fmn
