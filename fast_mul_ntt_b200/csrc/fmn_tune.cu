// fmn_tune.cu -- per-length pass-plan autotuner and plan files (host code).
//
// A transform of 2^n points can be split into passes in several ways (e.g. 2^25 as 9+8+8,
// 8+9+8, 8+8+9, 9+9+7, ...).  fmn_autotune times every valid plan of each length on the
// current GPU with a real product and keeps the fastest, for both residue engines (64-bit
// points up to 2^27, 32-bit digits up to 2^26); the choices are written to a plan file whose
// header names the GPU and the CUDA driver ("n passes bits..." lines for the 64-bit engine,
// "e32 n passes bits..." for the 32-bit one), and which the library loads at start from
// <library directory>/../tune/plans-<gpu name>.txt (or FMN_PLAN_FILE) when both match.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/fast_mul.h"
#include "fmn_internal.h"

namespace fmn {
int api_set_error(int code, const char* what, cudaError_t e);
}

namespace {

std::string gpu_key(int* driver) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, dev) != cudaSuccess) {
        cudaGetLastError();
        return "";
    }
    *driver = 0;
    cudaDriverGetVersion(driver);
    return prop.name;
}

std::string sanitize(const std::string& s) {
    std::string r;
    for (char ch : s) r += (isalnum((unsigned char)ch) ? ch : '_');
    return r;
}

// Time `reps` products whose transform has 2^n points under the plan in effect: two
// 2^(n-1)-limb operands on the 64-bit engine, two 2^(n-2)-limb operands (2^n digits) on the
// 32-bit engine.
double time_plan(int engine, int n, const u64* a, const u64* b, u64* out, void* ws, size_t ws_bytes, cudaStream_t s,
                 int reps, cudaEvent_t e0, cudaEvent_t e1, cudaError_t* err) {
    const u64 half = 1ull << (engine == fmn::ENGINE_32 ? n - 2 : n - 1);
    fmn::Job j;
    j.a = a;
    j.la = half;
    j.b = b;
    j.lb = half;
    j.out = out;
    j.sqr = 0;
    j.engine = engine;
    const size_t tb = engine == fmn::ENGINE_32 ? 0 : fmn::twiddle_table_bytes(n);
    void* tbuf = nullptr;
    fmn::TwiddleSet ts;
    const fmn::TwiddleSet* tws = nullptr;
    if (tb && cudaMalloc(&tbuf, tb) == cudaSuccess && fmn::build_twiddle_tables(n, (u64*)tbuf, &ts, s) == cudaSuccess)
        tws = &ts;
    cudaGetLastError();
    *err = fmn::enqueue_job(j, ws, ws_bytes, s, tws);     // warm-up
    cudaEventRecord(e0, s);
    for (int r = 0; r < reps && *err == cudaSuccess; ++r) *err = fmn::enqueue_job(j, ws, ws_bytes, s, tws);
    cudaEventRecord(e1, s);
    if (*err == cudaSuccess) *err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    if (tbuf) cudaFree(tbuf);
    return ms / reps;
}

}  // namespace

extern "C" {

int fmn_get_plan_engine(int engine, int log_n, int* bits, int max_passes) {
    if (engine != FMN_ENGINE_32) return fmn_get_plan(log_n, bits, max_passes);
    if (log_n < 0 || log_n > 26 || !bits) return -FMN_ERR_ARG;
    const fmn::Plan p = fmn::q32_make_plan(log_n);
    for (int i = 0; i < p.passes && i < max_passes; ++i) bits[i] = p.bits[i];
    return p.passes;
}

int fmn_set_plan_engine(int engine, int log_n, const int* bits, int passes) {
    if (engine != FMN_ENGINE_32) return fmn_set_plan(log_n, bits, passes);
    if (passes == 0) {
        fmn::q32_clear_plan(log_n);
        return FMN_OK;
    }
    fmn::Plan p;
    memset(&p, 0, sizeof(p));
    if (!bits || passes < 0 || passes > fmn::MAX_PASSES) return fmn::api_set_error(FMN_ERR_ARG, "bad plan", cudaSuccess);
    p.n = log_n;
    p.passes = passes;
    for (int i = 0; i < passes; ++i) p.bits[i] = bits[i];
    if (!fmn::q32_set_plan(p)) return fmn::api_set_error(FMN_ERR_ARG, "invalid pass plan", cudaSuccess);
    fmn::q32_prepare_tables();      // the new plan's twiddle tables, before a product needs them
    return FMN_OK;
}

int fmn_get_plan(int log_n, int* bits, int max_passes) {
    if (log_n < 0 || log_n > fmn::MAX_LOG_N || !bits) return -FMN_ERR_ARG;
    const fmn::Plan p = fmn::make_plan(log_n);
    for (int i = 0; i < p.passes && i < max_passes; ++i) bits[i] = p.bits[i];
    return p.passes;
}

int fmn_set_plan(int log_n, const int* bits, int passes) {
    fmn::Plan p;
    memset(&p, 0, sizeof(p));
    if (passes == 0) {                       // back to the default plan
        fmn::clear_plan(log_n);
        return FMN_OK;
    }
    if (!bits || passes < 0 || passes > fmn::MAX_PASSES) return fmn::api_set_error(FMN_ERR_ARG, "bad plan", cudaSuccess);
    p.n = log_n;
    p.passes = passes;
    for (int i = 0; i < passes; ++i) p.bits[i] = bits[i];
    if (!fmn::set_plan(p)) return fmn::api_set_error(FMN_ERR_ARG, "invalid pass plan", cudaSuccess);
    return FMN_OK;
}

int fmn_load_plans(const char* path) {
    FILE* f = path ? fopen(path, "r") : nullptr;
    if (!f) return fmn::api_set_error(FMN_ERR_ARG, "cannot open plan file", cudaSuccess);
    int driver = 0;
    const std::string gpu = gpu_key(&driver);
    char line[512];
    std::string fgpu;
    int fdriver = -1;
    std::vector<fmn::Plan> plans, plans32;
    while (fgets(line, sizeof(line), f)) {
        if (line[0] == '#' || line[0] == '\n') continue;
        if (!strncmp(line, "gpu ", 4)) {
            fgpu = line + 4;
            while (!fgpu.empty() && (fgpu.back() == '\n' || fgpu.back() == '\r')) fgpu.pop_back();
            continue;
        }
        if (!strncmp(line, "driver ", 7)) {
            fdriver = atoi(line + 7);
            continue;
        }
        fmn::Plan p;
        memset(&p, 0, sizeof(p));
        if (!strncmp(line, "e32 ", 4)) {
            if (sscanf(line + 4, "%d %d %d %d %d %d", &p.n, &p.passes, &p.bits[0], &p.bits[1], &p.bits[2], &p.bits[3]) >=
                    3 &&
                fmn::q32_valid_plan(p))
                plans32.push_back(p);
            continue;
        }
        if (sscanf(line, "%d %d %d %d %d %d", &p.n, &p.passes, &p.bits[0], &p.bits[1], &p.bits[2], &p.bits[3]) >= 3 &&
            fmn::valid_plan(p))
            plans.push_back(p);
    }
    fclose(f);
    if (fgpu != gpu || fdriver != driver)
        return fmn::api_set_error(FMN_ERR_ARG, "plan file was tuned on another GPU or driver", cudaSuccess);
    for (const auto& p : plans) fmn::set_plan(p);
    for (const auto& p : plans32) fmn::q32_set_plan(p);
    if (!plans32.empty()) fmn::q32_prepare_tables();
    return FMN_OK;
}

int fmn_autotune(int n_lo, int n_hi, const char* save_path) {
    int driver = 0;
    const std::string gpu = gpu_key(&driver);
    if (gpu.empty()) return fmn::api_set_error(FMN_ERR_CUDA, "no CUDA device", cudaSuccess);
    if (n_lo < 10) n_lo = 10;                // one-pass lengths have a single plan
    if (n_hi > 27) n_hi = 27;
    cudaStream_t s;
    cudaEvent_t e0, e1;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e != cudaSuccess) return fmn::api_set_error(FMN_ERR_CUDA, "stream", e);
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    std::vector<std::string> lines;
    int rc = FMN_OK;
    for (const int engine : {fmn::ENGINE_64, fmn::ENGINE_32}) {
        const bool e32 = engine == fmn::ENGINE_32;
        for (int n = n_lo; n <= (e32 ? (n_hi < 26 ? n_hi : 26) : n_hi) && rc == FMN_OK; ++n) {
            const std::vector<fmn::Plan> cands = e32 ? fmn::q32_candidate_plans(n) : fmn::candidate_plans(n);
            if (cands.size() <= 1) continue;
            const u64 half = 1ull << (e32 ? n - 2 : n - 1);
            fmn::Job wj;
            wj.a = wj.b = nullptr;
            wj.out = nullptr;
            wj.la = wj.lb = half;
            wj.sqr = 0;
            wj.engine = engine;
            const size_t wsb = fmn::job_workspace_bytes(wj);
            u64 *a = nullptr, *b = nullptr, *out = nullptr;
            void* ws = nullptr;
            if ((e = cudaMalloc(&a, half * 8)) != cudaSuccess || (e = cudaMalloc(&b, half * 8)) != cudaSuccess ||
                (e = cudaMalloc(&out, 2 * half * 8)) != cudaSuccess || (e = cudaMalloc(&ws, wsb)) != cudaSuccess) {
                rc = fmn::api_set_error(FMN_ERR_NOMEM, "tuning buffers", e);
            }
            if (rc == FMN_OK) {
                cudaMemsetAsync(ws, 0, 256, s);
                fmn::fill_limbs(a, half, 1, s);
                fmn::fill_limbs(b, half, 2, s);
                const int reps = n >= 24 ? 3 : n >= 20 ? 10 : 40;
                double best = 1e30;
                fmn::Plan bp = e32 ? fmn::q32_default_plan(n) : fmn::default_plan(n);
                for (const auto& cand : cands) {
                    if (e32) fmn::q32_set_plan(cand);
                    else fmn::set_plan(cand);
                    const double ms = time_plan(engine, n, a, b, out, ws, wsb, s, reps, e0, e1, &e);
                    if (e != cudaSuccess) {
                        rc = fmn::api_set_error(FMN_ERR_CUDA, "timing a plan", e);
                        break;
                    }
                    if (ms < best) {
                        best = ms;
                        bp = cand;
                    }
                }
                if (e32) fmn::q32_set_plan(bp);
                else fmn::set_plan(bp);
                char buf[160];
                snprintf(buf, sizeof(buf), "%s%d %d %d %d %d %d   # %.1f us\n", e32 ? "e32 " : "", bp.n, bp.passes,
                         bp.bits[0], bp.bits[1], bp.bits[2], bp.bits[3], best * 1e3);
                lines.push_back(buf);
            }
            cudaFree(a);
            cudaFree(b);
            cudaFree(out);
            cudaFree(ws);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaStreamDestroy(s);
    // the candidates' twiddle tables give way to those of the chosen plans
    int dev = 0;
    if (cudaGetDevice(&dev) == cudaSuccess) {
        cudaDeviceSynchronize();
        fmn::q32_release_tables(dev);
        fmn::q32_prepare_tables();
    }
    if (rc == FMN_OK && save_path) {
        FILE* f = fopen(save_path, "w");
        if (!f) return fmn::api_set_error(FMN_ERR_ARG, "cannot write plan file", cudaSuccess);
        fprintf(f, "# fast_mul_ntt_b200 pass plans: n passes bits... (64-bit engine: fastest product of two 2^(n-1)-limb\n"
                   "# operands); e32 n passes bits... (32-bit engine, 2^n digits: two 2^(n-2)-limb operands)\n");
        fprintf(f, "gpu %s\ndriver %d\n", gpu.c_str(), driver);
        for (const auto& l : lines) fputs(l.c_str(), f);
        fclose(f);
    }
    return rc;
}

// Plan file next to the library: <dir of the .so>/../tune/plans-<gpu>.txt, or FMN_PLAN_FILE.
int fmn_load_default_plans(void) {
    const char* env = getenv("FMN_PLAN_FILE");
    if (env && *env) return fmn_load_plans(env);
    Dl_info info;
    if (!dladdr((void*)&fmn_load_default_plans, &info) || !info.dli_fname) return FMN_ERR_ARG;
    std::string so = info.dli_fname;
    const size_t slash = so.rfind('/');
    const std::string dir = slash == std::string::npos ? "." : so.substr(0, slash);
    int driver = 0;
    const std::string gpu = gpu_key(&driver);
    const std::string path = dir + "/../tune/plans-" + sanitize(gpu) + ".txt";
    FILE* f = fopen(path.c_str(), "r");
    if (!f) return FMN_ERR_ARG;
    fclose(f);
    return fmn_load_plans(path.c_str());
}

}  // extern "C"
