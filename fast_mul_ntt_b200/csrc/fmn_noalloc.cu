// fmn_noalloc.cu -- a product entry point that never allocates memory.
//
// Some callers cannot call cudaMalloc while they run: a plugin inside a host application
// whose own allocator has already claimed the device memory, a latency-critical loop where
// cudaMalloc / cudaFree would stall or synchronise the device, or a process that sized its
// memory once at start-up and must not grow.  For them, fmn_mul_device_noalloc keeps all of
// its scratch (residue arrays, carry-scan state, status word) in one fixed array that lives
// in device memory for as long as the library is loaded, and calls no cudaMalloc, cudaFree
// or other allocating routine.
//
// Limit: the array holds the scratch of a product whose transform has at most 2^16 points,
// i.e. len1 + len2 <= 65537 limbs.  Larger products are rejected with FMN_ERR_TOO_LARGE.
// Every GPU that loads the library keeps the array (about 3 MB) until the process exits.
//
// The host name of a __device__ array is only a stand-in for it: the kernels must be given
// the device address, which cudaGetSymbolAddress returns.  The first call on each device
// does that lookup and uploads the twiddle tables (built once in host memory); make that
// first call before any stream capture.  All calls share the one array and each call leaves
// its contents behind: the carry-scan state and the status word are cleared at the start of
// every call, and two calls whose work overlaps on the GPU (different streams or threads)
// race on the array and corrupt each other's results.  Every call is synchronous: it returns
// after its work on `stream` has finished, with the kernels' status read back.
//
// The products run on the 64-bit residue engine with the pass plans in effect in the process
// (the default split of each transform length unless another entry point has loaded the
// tuned plan file: loading plans may build 32-bit twiddle tables, i.e. allocate, so this
// entry point never loads them itself).  Its four-step twiddles are computed in the kernels.
#include <cuda_runtime.h>

#include <mutex>

#include "../../include/fast_mul.h"
#include "fmn_internal.h"

namespace {

constexpr u64 kNoallocMaxNtt = 1ull << 16;          // largest transform the array can hold
static __device__ __align__(256) unsigned char g_noalloc_scratch[(3u << 20) + 4096];

// The 64-bit engine's workspace of the largest accepted product (len1 + len2 = 65537 limbs,
// N = 2^16 points): [status 256 B][A: 3 N u64][B: 3 N u64][ticket 16 B][one look-back word
// per CRT + carry CTA of 2048 limbs], rounded up to 256 bytes (fmn_ntt.cu, ws_layout).
constexpr size_t round256c(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t kNoallocMaxLayout =
    round256c(round256c(round256c(256 + 3 * kNoallocMaxNtt * 8) + 3 * kNoallocMaxNtt * 8) + 16 +
              4 * ((kNoallocMaxNtt + 1 + 2047) / 2048));
static_assert(kNoallocMaxLayout == 3146240, "64-bit workspace of a 2^16-point product");
static_assert(sizeof(g_noalloc_scratch) >= kNoallocMaxLayout, "the array holds the largest accepted product");

std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};               // device address of the array, per device

}  // namespace

namespace fmn {
int api_set_error(int code, const char* what, cudaError_t e);
}

extern "C" int fmn_mul_device_noalloc(const u64* d_in1, u64 len1, const u64* d_in2, u64 len2, u64* d_out,
                                      void* stream) {
    const u64 out_len = len1 + len2;
    if (out_len == 0) return FMN_OK;
    if (!d_in1 || !d_in2 || !d_out) return fmn::api_set_error(FMN_ERR_ARG, "null pointer", cudaSuccess);
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e;
    if (len1 == 0 || len2 == 0) {
        if ((e = cudaMemsetAsync(d_out, 0, out_len * sizeof(u64), s)) != cudaSuccess ||
            (e = cudaStreamSynchronize(s)) != cudaSuccess)
            return fmn::api_set_error(FMN_ERR_CUDA, "zero product", e);
        return FMN_OK;
    }
    const int sq = (d_in1 == d_in2 && len1 == len2);
    fmn::Job j;
    j.a = d_in1;
    j.la = len1;
    j.b = d_in2;
    j.lb = len2;
    j.out = d_out;
    j.sqr = sq;
    j.engine = fmn::ENGINE_64;      // the scratch array is sized for this engine's layout
    j.no_wrap = true;               // ... of a whole product
    if (out_len - 1 > kNoallocMaxNtt)
        return fmn::api_set_error(FMN_ERR_TOO_LARGE,
                                  "fmn_mul_device_noalloc: product needs a transform above 65536 points "
                                  "(len1 + len2 must be <= 65537); use fmn_mul_device or fmn_mul_device_ws",
                                  cudaSuccess);
    const size_t need = fmn::job_workspace_bytes(j);
    if (need > sizeof(g_noalloc_scratch))            // only if the engine's layout grew
        return fmn::api_set_error(FMN_ERR_TOO_LARGE,
                                  "fmn_mul_device_noalloc: the product's workspace exceeds the fixed scratch array",
                                  cudaSuccess);
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return fmn::api_set_error(FMN_ERR_CUDA, "cudaGetDevice", e);
    if (dev < 0 || dev >= 64) return fmn::api_set_error(FMN_ERR_ARG, "device index out of range", cudaSuccess);
    void* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {                  // set-up, once per device (this device is current)
            if ((e = fmn::ensure_tables()) != cudaSuccess)
                return fmn::api_set_error(FMN_ERR_CUDA, "uploading twiddle tables", e);
            void* p = nullptr;
            if ((e = cudaGetSymbolAddress(&p, g_noalloc_scratch)) != cudaSuccess)
                return fmn::api_set_error(FMN_ERR_CUDA, "cudaGetSymbolAddress of the scratch array", e);
            g_noalloc_addr[dev] = p;
        }
        scratch = g_noalloc_addr[dev];
    }
    if ((e = cudaMemsetAsync(scratch, 0, sizeof(unsigned), s)) != cudaSuccess)   // status word
        return fmn::api_set_error(FMN_ERR_CUDA, "clearing the status word", e);
    if ((e = fmn::enqueue_job(j, scratch, sizeof(g_noalloc_scratch), s)) != cudaSuccess)
        return fmn::api_set_error(FMN_ERR_CUDA, "kernel launch", e);
    unsigned word = 0;
    if ((e = cudaMemcpyAsync(&word, scratch, sizeof(word), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
        (e = cudaStreamSynchronize(s)) != cudaSuccess)
        return fmn::api_set_error(FMN_ERR_CUDA, "synchronising the product", e);
    if (word) return fmn::api_set_error(FMN_ERR_DEVICE, "carry scan: bounded wait expired", cudaSuccess);
    return FMN_OK;
}
