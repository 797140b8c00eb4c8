"""Benchmark of abs_mul64 at 10,000,000 x 10,000,000 limbs on B200 (one product per step).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints ONE JSON line (rank 0).  With N > 1 the script is launched by torchrun, one rank per
GPU; every rank multiplies its own copy of the operands (replicas: a single product does
not shard), and the timed region is bracketed by a barrier and a device synchronize, its
length taken as the max over ranks.

  value   products/s with operands and output resident in HBM (device API), all ranks;
  e2e     the same metric through the C ABI abs_mul64 with pinned host buffers: each call
          copies both operands host->device and the product device->host.  --e2e-callers
          host threads (default 4) call at once, as the reference arm runs its products on
          parallel host threads; the one-thread figure is reported beside it, and e2e.link
          the GPU's host link measured in the same run (pinned copies each way alone and
          both at once) with the products/s it allows and e2e's fraction of that;
  roofline / roofline_int
          the dominant kernel, timed live with CUDA events inside the timed region, against
          the measured HBM copy bandwidth (MEASURED_PEAKS.json) and against the measured
          peak of the engine's butterfly arithmetic (microbenchmark run here);
  cpu_baseline
          the reference's own src/ abs_mul64 (oracle/_ref, compiled unmodified) on one host
          core, one 10M x 10M product (rank 0, N = 1 only);
  extra   the other configurations of the product (10k x 10k, 1M x 1M uniform / all-ones /
          square, 10M all-ones and square, 64M x 250K and 64M x 64M uniform and sparse, and
          10M x 10M on the 64-bit engine with the reference's primes), each timed on the
          device with an L2 flush between products, checked against the reference's output
          digest, with its dominant kernel's rooflines;
  batch   the 4,096-product mixed-size stream: per-call vs batched vs CUDA-graph replay;
  serve   the open-loop Poisson stream (100,000 requests, 256 .. 4M limbs) through the
          continuous-batching server and through the plain per-call path, at an offered rate
          both keep up with (latency) and one above the per-call path's capacity (throughput).

--impl reference times that reference CPU implementation with all host cores (independent
products in parallel threads) on the same workload and prints the same JSON line.
"""
import argparse
import ctypes
import hashlib
import json
import os
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

LEN1 = LEN2 = 10_000_000
SEED = 0
KIND = "uniform"
METRIC = "abs_mul64 products/s at 10M x 10M limbs (bit-exact)"
UNIT = "products/s"
WORKLOAD = "abs_mul64 10,000,000 x 10,000,000 limbs (uniform u64, seed 0)"
DATA = "synthetic: splitmix64 seed 0, uniform u64 limbs, top limb nonzero (no dataset involved)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the reference CPU timing")
    ap.add_argument("--len", type=int, default=None, help="override operand length (profiling runs)")
    ap.add_argument("--len2", type=int, default=None, help="second operand's length (default: --len)")
    ap.add_argument("--engine", default="auto", choices=["auto", "32", "64"],
                    help="residue engine (default: the library's cost model)")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-stream comparison")
    ap.add_argument("--batch-only", action="store_true", help="only the batched-stream comparison")
    ap.add_argument("--batch-count", type=int, default=4096)
    ap.add_argument("--no-serve", action="store_true", help="skip the served-stream comparison")
    ap.add_argument("--serve-only", action="store_true", help="only the served-stream comparison")
    ap.add_argument("--serve-requests", type=int, default=100_000)
    ap.add_argument("--serve-rates", default="2000,8000",
                    help="offered requests per second: one below the per-call path's capacity, one above")
    ap.add_argument("--no-extra", action="store_true", help="skip the other configurations")
    ap.add_argument("--extra-only", action="store_true", help="only the other configurations")
    ap.add_argument("--e2e-callers", type=int, default=4,
                    help="host threads calling abs_mul64 at once in the end-to-end measurement")
    return ap.parse_args()


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def golden_digest(op, kind, l1, l2):
    path = os.path.join(ROOT, "tests", "golden", "golden_vectors.json")
    with open(path) as f:
        for c in json.load(f)["cases"]:
            if (c["op"], c["kind"], c["len1"], c["len2"], c["seed"]) == (op, kind, l1, l2, SEED):
                return c["sha256"]
    return None


def digest(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<u8").tobytes()).hexdigest()


# ----------------------------------------------------------------------------- ranks
def max_over_ranks(x, device=None):
    """Max of a per-rank float over all ranks of the default process group (the timing rule:
    the slowest rank bounds the whole job); returns x itself without a process group."""
    import torch
    import torch.distributed as tdist
    if not (tdist.is_available() and tdist.is_initialized()) or tdist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    tdist.all_reduce(t, op=tdist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world_size, steps, max_seconds):
    """Whole-job products/s of replicated products: every rank completed `steps` products."""
    return world_size * steps / max_seconds


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """Samples SM clock and clock-event (throttle) reasons through NVML in a thread."""

    REASONS = {0x8: "hw_slowdown", 0x40: "hw_thermal_slowdown", 0x20: "sw_thermal_slowdown",
               0x4: "sw_power_cap", 0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting",
               0x2: "applications_clocks_setting", 0x1: "gpu_idle", 0x10: "sync_boost"}

    def __init__(self, index):
        self.ok = False
        self.samples = []
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv = pynvml
            self.h = pynvml.nvmlDeviceGetHandleByIndex(index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self.h, pynvml.NVML_CLOCK_SM)
            self.ok = True
        except Exception:
            self.ok = False
        self._stop = threading.Event()

    def _run(self):
        nv = self.nv
        while not self._stop.is_set():
            try:
                mhz = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                try:
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                except Exception:
                    r = nv.nvmlDeviceGetCurrentClocksThrottleReasons(self.h)
                self.samples.append((mhz, r))
            except Exception:
                pass
            time.sleep(0.005)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def summary(self):
        if not self.ok or not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": getattr(self, "max_mhz", None), "reasons": [], "samples": 0}
        mhz = sorted(s[0] for s in self.samples)
        bits = 0
        for _, r in self.samples:
            bits |= int(r)
        reasons = sorted(name for b, name in self.REASONS.items() if bits & b and name != "gpu_idle")
        return {"sm_mhz": mhz[len(mhz) // 2], "sm_max_mhz": self.max_mhz, "reasons": reasons,
                "samples": len(self.samples)}


# ----------------------------------------------------------------------------- CPU reference
def ref_lib():
    from oracle.oracle import RefFastMul, Oracle
    if RefFastMul.available():
        return RefFastMul(), "reference"
    return Oracle(), "port"


def cpu_baseline(a, b):
    """One product with the reference's single-threaded src/ code on this host."""
    lib, kind = ref_lib()
    w1, w2 = a[:1_000_000].copy(), b[:1_000_000].copy()
    lib.mul(w1, w2)                                    # warm-up: code and page faults
    t0 = time.perf_counter()
    out = lib.mul(a, b)
    dt = time.perf_counter() - t0
    return {"value": 1.0 / dt, "unit": UNIT, "cores": 1, "kind": kind,
            "sample": f"one {len(a)} x {len(b)}-limb abs_mul64 (seed 0) after a 1M x 1M warm-up, "
                      f"{dt:.2f} s, single thread (the reference has no threading)",
            "seconds_per_product": dt}, out


def host_threads_and_mem():
    cores = os.cpu_count() or 1
    try:
        import psutil
        avail = psutil.virtual_memory().available
    except Exception:
        avail = 16 << 30
    per = 1.6 * (1 << 30)         # reference scratch (4 x 2^25 u64) + output, per product
    return max(1, min(cores, int(avail * 0.6 / per), 64)), cores


def run_reference(args, ws, rank):
    if rank != 0:
        return
    from fast_mul_ntt_b200 import synth
    a, b = synth.operands(KIND, LEN1, LEN2, SEED)
    lib, kind = ref_lib()
    threads, cores = host_threads_and_mem()
    outs = [np.zeros(LEN1 + LEN2, np.uint64) for _ in range(threads)]

    def one_round(x, y):
        ts = [threading.Thread(target=lambda i=i: lib.mul(x, y, outs[i]) if kind == "reference"
                               else lib.mul(x, y)) for i in range(threads)]
        for t in ts:
            t.start()
        for t in ts:
            t.join()

    wa, wb = a[:1_000_000].copy(), b[:1_000_000].copy()
    for _ in range(max(1, min(args.warmup, 3))):
        one_round(wa, wb)                              # warm-up on a 1M x 1M sample
    budget = 150.0
    rounds, t_total = 0, 0.0
    while rounds < args.steps:
        t0 = time.perf_counter()
        one_round(a, b)
        t_total += time.perf_counter() - t0
        rounds += 1
        if t_total > budget:
            break
    want = golden_digest("mul", KIND, LEN1, LEN2)
    exact = (digest(outs[0]) == want) if kind == "reference" else None
    value = threads * rounds / t_total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws,
            "steps": rounds, "warmup": args.warmup, "ms_per_step": 1e3 * t_total / rounds,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": DATA,
            "config": {"workload": WORKLOAD, "len1": LEN1, "len2": LEN2, "ntt_len": 1 << 25,
                       "parallelism": f"{threads} independent products in parallel host threads"},
            "bit_exact": exact,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{rounds} rounds of {threads} concurrent {LEN1} x {LEN2} products "
                                       f"(reference src/ abs_mul64, compiled unmodified, one call per "
                                       f"thread; {cores} host cores); warm-up on 1M x 1M",
                             "seconds_per_round": t_total / rounds},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- batched stream
def batch_compare(fmn, torch, dev, count, repeats=3):
    """The mixed-size stream (each side log-uniform in [1000, 100000] limbs, 20% squares,
    seeded): plain per-call device products in a loop vs one batched call vs a CUDA-graph
    replay of the batch.  Operands resident in HBM; every output compared bit for bit."""
    from fast_mul_ntt_b200 import synth
    mix = synth.batch_mix(count, seed=0)
    jobs_pc, jobs_b, limbs = [], [], 0
    for op, l1, l2, seed in mix:
        a, b = synth.operands("uniform", l1, l2, seed)
        da = torch.from_numpy(a.view(np.int64)).to(dev)
        db = da if op == "sqr" else torch.from_numpy(b.view(np.int64)).to(dev)
        jobs_pc.append((op, da, db, torch.empty(l1 + l2, dtype=torch.int64, device=dev)))
        jobs_b.append((da, db, torch.empty(l1 + l2, dtype=torch.int64, device=dev)))
        limbs += l1 + l2
    stream = torch.cuda.Stream(device=dev)

    def per_call():
        for op, da, db, out in jobs_pc:
            if op == "sqr":
                fmn.sqr_device(da, out, stream=stream)
            else:
                fmn.mul_device(da, db, out, stream=stream)

    def timed(fn, reps):
        fn()
        stream.synchronize()
        ts = []
        for _ in range(reps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            fn()
            e1.record(stream)
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        return sorted(ts)[len(ts) // 2]

    t_pc = timed(per_call, repeats)
    prepared = fmn.BatchJobs(jobs_b)         # checked and marshalled once, as for the graph
    t_b = timed(lambda: fmn.mul_batch_device(prepared, stream=stream), repeats)
    fmn.sync(stream)
    exact_b = all(torch.equal(x[3], y[2]) for x, y in zip(jobs_pc, jobs_b))
    for _, _, o in jobs_b:
        o.zero_()
    g = fmn.BatchGraph(jobs_b)
    t_g = timed(lambda: g.launch(stream), repeats)
    g.sync(stream)
    exact_g = all(torch.equal(x[3], y[2]) for x, y in zip(jobs_pc, jobs_b))
    g.close()
    ns = sorted({fmn.ntt_len(l1, l2) for _, l1, l2, _ in mix})
    res = {"workload": f"{count} products, each side log-uniform in [1000, 100000] limbs, 20% squares "
                       f"(seed 0), transform lengths {ns[0]}..{ns[-1]}",
           "limbs_total": limbs,
           "per_call": {"products_per_s": count / (t_pc * 1e-3), "ms": t_pc},
           "batched": {"products_per_s": count / (t_b * 1e-3), "ms": t_b, "bit_exact_vs_per_call": exact_b},
           "graph": {"products_per_s": count / (t_g * 1e-3), "ms": t_g, "bit_exact_vs_per_call": exact_g},
           "speedup_batched_vs_per_call": t_pc / t_b, "speedup_graph_vs_per_call": t_pc / t_g}
    del jobs_pc, jobs_b
    torch.cuda.empty_cache()
    return res


# ----------------------------------------------------------------------------- served stream
class UtilSampler:
    """NVML GPU utilisation (percent of time a kernel was running) sampled in a thread."""

    def __init__(self, index, period=0.05):
        self.ok, self.samples, self.period = False, [], period
        try:
            import pynvml
            pynvml.nvmlInit()
            self.nv, self.h, self.ok = pynvml, pynvml.nvmlDeviceGetHandleByIndex(index), True
        except Exception:
            self.ok = False
        self._stop = threading.Event()

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self.nv.nvmlDeviceGetUtilizationRates(self.h).gpu)
            except Exception:
                pass
            time.sleep(self.period)

    def __enter__(self):
        if self.ok:
            self.t = threading.Thread(target=self._run, daemon=True)
            self.t.start()
        return self

    def __exit__(self, *a):
        if self.ok:
            self._stop.set()
            self.t.join()

    def mean(self):
        return float(np.mean(self.samples)) if self.samples else None


def serve_compare(fmn, torch, dev, n_requests, rates, seed=0, templates=256, residents=8,
                  paths=("served", "per_call"), raw=None):
    """Open-loop Poisson stream: 70% multiplies, 30% squares, operand lengths log-uniform in
    [256, 4,000,000] limbs, 25% of the multiplies by a resident (already transformed) operand;
    HBM admission budget 120 GB.  The same stream through the continuous-batching server and
    through the plain per-call path (one product at a time on one stream, no reuse), at each
    offered rate.  Every output is compared on the device with its expected product, computed
    beforehand by the per-call path.  The device time of every request template alone gives the
    stream's GPU work, so the capacity of each path can be read against it."""
    rng = np.random.default_rng(seed)
    lo, hi = 256, 4_000_000

    def loglen():
        return int(np.exp(rng.uniform(np.log(lo), np.log(hi))))

    hold = []
    res_ops = []
    for k in range(residents):
        a = synth_limbs("uniform", loglen(), 500_000 + k)
        da = torch.from_numpy(a.view(np.int64)).to(dev)
        hold.append(da)
        res_ops.append(fmn.Operand(da, max_partner_len=hi))
    tmpl, runs = [], []
    stream = torch.cuda.Stream(device=dev)
    for t in range(templates):
        r = fmn.FmnRequest()
        u = rng.uniform()
        if u < 0.30:                                   # square
            l1 = loglen()
            da = torch.from_numpy(synth_limbs("uniform", l1, 600_000 + t).view(np.int64)).to(dev)
            hold.append(da)
            want = torch.empty(2 * l1, dtype=torch.int64, device=dev)
            run = (lambda da=da, want=want: fmn.sqr_device(da, want, stream=stream))
            r.op, r.in1, r.len1 = fmn.FMN_OP_SQR, da.data_ptr(), l1
        elif u < 0.30 + 0.70 * 0.25:                   # multiply by a resident operand
            op = res_ops[t % residents]
            l2 = loglen()
            db = torch.from_numpy(synth_limbs("uniform", l2, 700_000 + t).view(np.int64)).to(dev)
            hold.append(db)
            want = torch.empty(op.len + l2, dtype=torch.int64, device=dev)
            run = (lambda op=op, db=db, want=want: fmn.mul_device(op.limbs, db, want, stream=stream))
            r.op, r.operand, r.in2, r.len2 = fmn.FMN_OP_MUL_OPERAND, op.handle.value, db.data_ptr(), l2
        else:                                          # multiply
            l1, l2 = loglen(), loglen()
            da = torch.from_numpy(synth_limbs("uniform", l1, 800_000 + t).view(np.int64)).to(dev)
            db = torch.from_numpy(synth_limbs("uniform", l2, 900_000 + t).view(np.int64)).to(dev)
            hold += [da, db]
            want = torch.empty(l1 + l2, dtype=torch.int64, device=dev)
            run = (lambda da=da, db=db, want=want: fmn.mul_device(da, db, want, stream=stream))
            r.op, r.in1, r.len1, r.in2, r.len2 = fmn.FMN_OP_MUL, da.data_ptr(), l1, db.data_ptr(), l2
        run()
        hold.append(want)
        r.check = want.data_ptr()
        r.out = None
        tmpl.append(r)
        runs.append(run)
    fmn.sync(stream)
    # device time of each template alone (the per-call path's kernels, back to back)
    alone_ms = []
    for run in runs:
        run()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(3):
            run()
        e1.record(stream)
        e1.synchronize()
        alone_ms.append(e0.elapsed_time(e1) / 3)
    fmn.sync(stream)
    pick = rng.integers(0, templates, n_requests)
    reqs = []
    for i, t in enumerate(pick):
        r = fmn.FmnRequest()
        ctypes.pointer(r)[0] = tmpl[t]
        r.tag = i
        reqs.append(r)
    gaps = rng.exponential(1.0, n_requests)
    ops = [tmpl[t].op for t in pick]
    # product length of each request (for latency by size class)
    tlen = [(r.len1 + r.len2) if r.op == fmn.FMN_OP_MUL else 2 * r.len1 if r.op == fmn.FMN_OP_SQR
            else res_ops[t % residents].len + r.len2 for t, r in enumerate(tmpl)]
    big = np.array([tlen[t] > (1 << 20) for t in pick])
    gpu_work_s = float(sum(alone_ms[t] for t in pick)) * 1e-3
    out = {"workload": f"{n_requests} requests, open-loop Poisson; 70% multiply / 30% square, 25% of the "
                       f"multiplies by one of {residents} resident operands; lengths log-uniform in [{lo}, {hi}] "
                       f"limbs ({templates} request templates, seed {seed}); HBM budget 120 GB",
           "requests": n_requests,
           "mix": {"mul": ops.count(fmn.FMN_OP_MUL), "sqr": ops.count(fmn.FMN_OP_SQR),
                   "mul_resident": ops.count(fmn.FMN_OP_MUL_OPERAND)},
           "large_requests": int(big.sum()),
           "gpu_work_alone_s": gpu_work_s,
           "per_call_device_bound_products_per_s": n_requests / gpu_work_s,
           "rates": {}}
    for rate in rates:
        arrivals = list(np.cumsum(gaps / rate))
        res = {"offered_per_s": rate}
        for name, batching in [(p, p == "served") for p in paths]:
            srv = fmn.Server(device=dev.index or 0, hbm_budget=120 << 30, max_batch=256, batching=batching)
            util = UtilSampler(dev.index or 0)
            try:
                with util:
                    lat, wall = srv.replay(reqs, arrivals)
                st = srv.stats()
            finally:
                srv.close()
            lat_all = np.array(lat)
            if raw is not None:                    # per-request record for diagnostics
                raw[(rate, name)] = {"arrival_s": np.array(arrivals), "latency_ms": lat_all,
                                     "length": np.array([tlen[t] for t in pick]), "op": np.array(ops)}
            pct = lambda x, p: float(np.percentile(x, p)) if len(x) else None
            lat = np.sort(lat_all)
            res[name] = {"products_per_s": st["completed"] / wall, "wall_s": wall,
                         "p90_ms": pct(lat_all, 90), "p999_ms": pct(lat_all, 99.9), "max_ms": float(lat.max()),
                         "large_p50_ms": pct(lat_all[big], 50), "large_p99_ms": pct(lat_all[big], 99),
                         "small_p50_ms": pct(lat_all[~big], 50), "small_p99_ms": pct(lat_all[~big], 99),
                         "p50_ms": float(lat[len(lat) // 2]),
                         "p99_ms": float(lat[min(len(lat) - 1, int(0.99 * len(lat)))]),
                         "mean_ms": float(lat.mean()), "batches": st["batches"],
                         "peak_scratch_gb": st["peak_bytes"] / 2**30,
                         "gpu_busy_pct": util.mean(),
                         "gpu_work_over_wall": gpu_work_s / wall,
                         "host_launch_ms_per_request": st["launch_ms"] / max(1, st["completed"]),
                         "host_alloc_ms_per_request": st["alloc_ms"] / max(1, st["completed"]),
                         "host_launch_ms_max": st["max_launch_ms"], "host_alloc_ms_max": st["max_alloc_ms"],
                         "mismatches": st["mismatches"], "rejected": st["rejected"],
                         "device_errors": st["device_errors"],
                         "bit_exact": st["mismatches"] == 0 and st["device_errors"] == 0 and st["rejected"] == 0}
        if "served" in res and "per_call" in res:
            res["throughput_ratio_served_vs_per_call"] = res["served"]["products_per_s"] / res["per_call"]["products_per_s"]
            res["p99_ratio_per_call_vs_served"] = res["per_call"]["p99_ms"] / res["served"]["p99_ms"]
        out["rates"][f"{rate:g}"] = res
    top = out["rates"][f"{max(rates):g}"]
    if "throughput_ratio_served_vs_per_call" in top:
        out["capacity_ratio_served_vs_per_call"] = top["throughput_ratio_served_vs_per_call"]
        out["meets_5x"] = top["throughput_ratio_served_vs_per_call"] >= 5.0
    out["mismatches"] = sum(v[p]["mismatches"] for v in out["rates"].values() for p in paths)
    for op in res_ops:
        op.close()
    del hold
    torch.cuda.empty_cache()
    return out


def synth_limbs(kind, n, seed):
    from fast_mul_ntt_b200 import synth
    return synth.limbs(kind, n, seed)


# ----------------------------------------------------------------------------- rooflines
def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except Exception:
        peaks = {}
    hbm = peaks.get("hbm_gbs")
    return (hbm, "measured (MEASURED_PEAKS.json hbm_gbs)") if hbm else (6650.0, "fallback 6.65 TB/s")


def traffic_for(key, kernel):
    """DRAM bytes per launch of `kernel` from an ncu capture of exactly this configuration
    (profiles/traffic.json, keyed by engine:op:kind:len1xlen2), or None when there is none."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            cap = json.load(f)["captures"].get(key)
    except Exception:
        return None, None
    if not cap or kernel not in cap["bytes_per_launch"]:
        return None, None
    return cap["bytes_per_launch"][kernel], cap["source"]


def rooflines(fmn, prof, steps, engine, peaks, traffic_key):
    """The dominant kernel kind of `prof` (per-kind CUDA-event totals over `steps` products)
    against the HBM copy bandwidth and against the engine's measured butterfly peak."""
    hbm_peak, hbm_src = load_peaks()
    bf_peak = peaks["bfly32"] if engine == fmn.ENGINE_32 else peaks["bfly64"]
    name, st = max(prof.items(), key=lambda kv: kv[1]["ms"])
    per_launch_ms = st["ms"] / max(1, st["launches"])
    bytes_per_launch = st["bytes"] / max(1, st["launches"])
    mm_per_launch = st["modmuls"] / max(1, st["launches"])
    achieved_gbs = bytes_per_launch / (per_launch_ms * 1e-3) / 1e9
    achieved_mm = mm_per_launch / (per_launch_ms * 1e-3)
    traffic, tsrc = traffic_for(traffic_key, name)
    total_ms = sum(v["ms"] for v in prof.values()) or 1.0
    all_mm = sum(v["modmuls"] for v in prof.values()) / steps
    hbm = {"bound": "hbm", "kernel": name, "achieved": achieved_gbs, "peak": hbm_peak, "unit": "GB/s",
           "frac": achieved_gbs / hbm_peak, "traffic": traffic,
           "traffic_source": tsrc or "no ncu capture of this configuration",
           "peak_source": hbm_src, "algorithmic_bytes_per_launch": bytes_per_launch, "ms_per_launch": per_launch_ms}
    integer = {"bound": "integer issue (butterfly arithmetic)", "kernel": name,
               "achieved": achieved_mm / 1e9, "peak": bf_peak / 1e9,
               "unit": "Gbutterfly/s", "frac": achieved_mm / bf_peak,
               "peak_source": ("measured: independent 32-bit butterfly chains on this GPU" if engine == fmn.ENGINE_32
                               else "measured: independent 64-bit Montgomery butterfly chains on this GPU"),
               "algorithmic_butterflies_per_launch": mm_per_launch,
               "whole_product_frac": (all_mm / (total_ms / steps * 1e-3)) / bf_peak}
    kernels = {k: {"ms_per_step": v["ms"] / steps, "launches_per_step": v["launches"] / steps,
                   "share": v["ms"] / total_ms} for k, v in prof.items()}
    return hbm, integer, kernels


def plan_label(fmn, l1, l2, sqr=False):
    """How the library runs this product (whole, split, wrapped or twisted)."""
    pieces = fmn.pieces_for(l1, l2, sqr)
    if pieces > 1:
        return ("the longer operand in %d pieces, each multiplied with the other's resident spectrum" % pieces)
    k, m = fmn.wrap_for(l1, l2, sqr), fmn.twist_for(l1, l2, sqr)
    if m:
        return ("wrapped: the cyclic transform plus the twisted product modulo X^%d - c "
                "(%d coefficients wrapped)" % (m, k))
    if k:
        return "wrapped: the cyclic transform plus the product of the lowest limbs (%d coefficients wrapped)" % k
    return "one transform of the whole product"


def engine_label(fmn, engine):
    return ("32-bit digits mod three 31-bit primes" if engine == fmn.ENGINE_32
            else "64-bit limbs mod the reference's three 62-bit primes")


# ----------------------------------------------------------------------------- other configurations
EXTRA = [  # (name, op, kind, len1, len2, engine, steps)
    ("mul_uniform_10k", "mul", "uniform", 10_000, 10_000, "auto", 50),
    ("mul_uniform_1M", "mul", "uniform", 1_000_000, 1_000_000, "auto", 20),
    ("mul_ones_1M", "mul", "ones", 1_000_000, 1_000_000, "auto", 20),
    ("sqr_uniform_1M", "sqr", "uniform", 1_000_000, 1_000_000, "auto", 20),
    ("mul_ones_10M", "mul", "ones", 10_000_000, 10_000_000, "auto", 10),
    ("sqr_uniform_10M", "sqr", "uniform", 10_000_000, 10_000_000, "auto", 10),
    ("mul_uniform_10M_engine64", "mul", "uniform", 10_000_000, 10_000_000, "64", 10),
    ("mul_uniform_64Mx250K", "mul", "uniform", 64_000_000, 250_000, "auto", 5),
    ("mul_sparse_64Mx250K", "mul", "sparse", 64_000_000, 250_000, "auto", 5),
    ("mul_uniform_64Mx64M", "mul", "uniform", 64_000_000, 64_000_000, "auto", 3),
    ("mul_sparse_64Mx64M", "mul", "sparse", 64_000_000, 64_000_000, "auto", 3),
]
L2_FLUSH_BYTES = 256 << 20        # twice the 126 MB L2


def time_config(fmn, torch, dev, op, kind, l1, l2, steps, warmup, peaks):
    """One configuration on the device: a correctness run against the reference's digest,
    then `steps` products each timed by CUDA events on its stream with an L2 flush (a 256 MB
    write) before it, then the same number of products with per-launch events for the kernel
    split and rooflines."""
    from fast_mul_ntt_b200 import synth
    a, b = synth.operands(kind, l1, l2, SEED)
    da = torch.from_numpy(a.view(np.int64)).to(dev)
    db = da if op == "sqr" else torch.from_numpy(b.view(np.int64)).to(dev)
    dout = torch.empty(l1 + l2, dtype=torch.int64, device=dev)
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.int32, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def step():
        if op == "sqr":
            fmn.sqr_device(da, dout, stream=stream)
        else:
            fmn.mul_device(da, db, dout, stream=stream)

    step()
    fmn.sync(stream)
    want = golden_digest(op, kind, l1, l2)
    got_digest = digest(dout.cpu().numpy().view(np.uint64))
    for _ in range(warmup):
        step()
    stream.synchronize()
    total = 0.0
    with torch.cuda.stream(stream):
        for _ in range(steps):
            flush.fill_(1)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            step()
            e1.record(stream)
            e1.synchronize()
            total += e0.elapsed_time(e1)
    fmn.sync(stream)
    fmn.profile_enable(True)
    fmn.profile_take()
    for _ in range(steps):
        step()
    fmn.profile_enable(False)
    prof = fmn.profile_take()
    fmn.sync(stream)
    engine = fmn.engine_for(l1, l2, op == "sqr")
    key = f"{'e32' if engine == fmn.ENGINE_32 else 'e64'}:{op}:{kind}:{l1}x{l2}"
    hbm, integer, kernels = rooflines(fmn, prof, steps, engine, peaks, key)
    us = 1e3 * total / steps
    res = {"op": op, "kind": kind, "len1": l1, "len2": l2, "engine": engine_label(fmn, engine),
           "pieces": fmn.pieces_for(l1, l2, op == "sqr"), "plan": plan_label(fmn, l1, l2, op == "sqr"),
           "steps": steps, "warmup": warmup,
           "us_per_product": us, "products_per_s": 1e6 / us, "limbs_per_s": (l1 + l2) * 1e6 / us,
           "bit_exact": (got_digest == want) if want else None,
           "l2_policy": "256 MB L2 flush before every timed product",
           "roofline": hbm, "roofline_int": integer, "kernels": kernels}
    del da, db, dout, flush
    torch.cuda.empty_cache()
    return res


def extra_configs(fmn, torch, dev, peaks):
    out = {}
    for name, op, kind, l1, l2, eng, steps in EXTRA:
        fmn.set_engine({"auto": fmn.ENGINE_AUTO, "64": fmn.ENGINE_64, "32": fmn.ENGINE_32}[eng])
        try:
            out[name] = time_config(fmn, torch, dev, op, kind, l1, l2, steps, 3, peaks)
        finally:
            fmn.set_engine(fmn.ENGINE_AUTO)
    return out


# ----------------------------------------------------------------------------- end to end
def e2e_rate(lib, pa, l1, pb, l2, outs, steps, barrier, dev):
    """Products/s of len(outs) host threads each calling abs_mul64 `steps` times at once (host
    wall clock, max over ranks); one warm-up call per thread first."""
    callers = len(outs)
    go = threading.Barrier(callers + 1)

    def caller(i, n):
        if n > 1:
            go.wait()
        for _ in range(n):
            lib.abs_mul64(pa, l1, pb, l2, outs[i])

    warm = [threading.Thread(target=caller, args=(i, 1)) for i in range(callers)]
    for t in warm:
        t.start()
    for t in warm:
        t.join()
    ths = [threading.Thread(target=caller, args=(i, steps)) for i in range(callers)]
    for t in ths:
        t.start()
    barrier()
    go.wait()
    t0 = time.perf_counter()
    for t in ths:
        t.join()
    return max_over_ranks(time.perf_counter() - t0, dev)


def link_rates(dev, nbytes=160 << 20, reps=8):
    """This GPU's host link, pinned buffers: GB/s host->device alone, device->host alone, and
    each way with both directions busy at once (the end-to-end path's bound)."""
    import torch
    h_in = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    h_out = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d_in = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    d_out = torch.zeros(nbytes, dtype=torch.uint8, device=dev)
    s_in, s_out = torch.cuda.Stream(dev), torch.cuda.Stream(dev)

    def run(h2d, d2h):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(reps):
            if h2d:
                with torch.cuda.stream(s_in):
                    d_in.copy_(h_in, non_blocking=True)
            if d2h:
                with torch.cuda.stream(s_out):
                    h_out.copy_(d_out, non_blocking=True)
        torch.cuda.synchronize(dev)
        return reps * nbytes / (time.perf_counter() - t0) / 1e9

    run(True, True)                                   # warm-up
    rates = {"h2d_gbs": run(True, False), "d2h_gbs": run(False, True), "both_each_gbs": run(True, True)}
    del h_in, h_out, d_in, d_out
    return rates


# ----------------------------------------------------------------------------- ours
def run_ours(args, ws, rank, local):
    import torch
    import fast_mul_ntt_b200 as fmn
    from fast_mul_ntt_b200 import synth

    dist = ws > 1
    if dist:
        import datetime
        import torch.distributed as tdist
        torch.cuda.set_device(local)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                 device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    fmn.init(local)
    if args.engine != "auto":
        fmn.set_engine(fmn.ENGINE_32 if args.engine == "32" else fmn.ENGINE_64)
    rates = [float(r) for r in args.serve_rates.split(",") if r]
    if args.batch_only:
        print(json.dumps(batch_compare(fmn, torch, dev, args.batch_count)), flush=True)
        return
    if args.serve_only:
        print(json.dumps(serve_compare(fmn, torch, dev, args.serve_requests, rates)), flush=True)
        return
    peaks = {"bfly32": fmn.bench_bfly32(), "bfly64": fmn.bench_modmul()[1]}
    if args.extra_only:
        print(json.dumps(extra_configs(fmn, torch, dev, peaks)), flush=True)
        return
    l1 = args.len or LEN1
    l2 = args.len2 or args.len or LEN2
    a, b = synth.operands(KIND, l1, l2, SEED)
    da = torch.from_numpy(a.view(np.int64)).to(dev)
    db = torch.from_numpy(b.view(np.int64)).to(dev)
    dout = torch.empty(l1 + l2, dtype=torch.int64, device=dev)
    stream = torch.cuda.Stream(device=dev)

    def step():
        fmn.mul_device(da, db, dout, stream=stream)

    # correctness of the timed configuration (against the reference's own output digest)
    with torch.cuda.stream(stream):
        step()
    fmn.sync(stream)
    got = dout.cpu().numpy().view(np.uint64)
    want = golden_digest("mul", KIND, l1, l2)
    bit_exact = (digest(got) == want) if want else None

    for _ in range(args.warmup):
        step()
    stream.synchronize()

    def barrier():
        if dist:
            torch.distributed.barrier()

    sampler = ClockSampler(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    torch.cuda.synchronize(dev)
    with sampler:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize(dev)
    barrier()
    ms = max_over_ranks(ev0.elapsed_time(ev1), dev)
    value = job_throughput(ws, args.steps, ms * 1e-3)
    # The kernel split: the same K products again, with a CUDA event pair around every launch
    # on its stream.  Those events leave gaps between launches, so this second loop gives each
    # kernel's duration and share for the rooflines, and the loop above the headline.
    fmn.profile_enable(True)
    fmn.profile_take()
    for _ in range(args.steps):
        step()
    fmn.sync(stream)
    fmn.profile_enable(False)
    prof = fmn.profile_take()

    # e2e through the reference-facing C ABI: pinned host buffers (one caller, then several
    # at once, as the reference arm runs its products on parallel host threads; the library's
    # host lanes overlap one call's PCIe copies with another's kernels), and pageable
    # malloc-style buffers as the reference's own callers pass them.  Inputs are shared; each
    # caller has its own output.
    lib = fmn.load_library()
    P = ctypes.POINTER(ctypes.c_uint64)
    e2e_steps = max(3, min(2 * args.steps, 40))   # about 0.3-1.2 s per figure: PCIe and host noise averages out
    callers = args.e2e_callers

    def pinned(x):
        return torch.from_numpy(x.view(np.int64)).pin_memory().numpy().view(np.uint64)

    ha, hb = pinned(a), pinned(b)
    houts = [pinned(np.zeros(l1 + l2, np.uint64)) for _ in range(callers)]
    pa, pb = ha.ctypes.data_as(P), hb.ctypes.data_as(P)
    pos = [h.ctypes.data_as(P) for h in houts]
    e2e1_s = e2e_rate(lib, pa, l1, pb, l2, pos[:1], e2e_steps, barrier, dev)
    e2e_exact = bool(np.array_equal(houts[0], got))
    e2e_s = e2e_rate(lib, pa, l1, pb, l2, pos, e2e_steps, barrier, dev)
    e2e_exact = e2e_exact and all(bool(np.array_equal(h, got)) for h in houts)
    del ha, hb, houts
    pouts = [np.zeros(l1 + l2, np.uint64) for _ in range(callers)]
    ppos = [h.ctypes.data_as(P) for h in pouts]
    pg_pa, pg_pb = a.ctypes.data_as(P), b.ctypes.data_as(P)
    pg1_s = e2e_rate(lib, pg_pa, l1, pg_pb, l2, ppos[:1], e2e_steps, barrier, dev)
    pg_s = e2e_rate(lib, pg_pa, l1, pg_pb, l2, ppos, e2e_steps, barrier, dev)
    pg_exact = all(bool(np.array_equal(h, got)) for h in pouts)
    del pouts
    link = link_rates(dev)

    result = None
    if rank == 0:
        engine = fmn.engine_for(l1, l2)
        pieces = fmn.pieces_for(l1, l2)
        key = f"{'e32' if engine == fmn.ENGINE_32 else 'e64'}:mul:{KIND}:{l1}x{l2}"
        hbm, integer, kernels = rooflines(fmn, prof, args.steps, engine, peaks, key)
        per_step_ms = ms / args.steps
        io = 8 * (l1 + l2)
        result = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": per_step_ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32" if engine == fmn.ENGINE_32 else "u64",
            "data": DATA,
            "config": {"workload": WORKLOAD if (l1, l2) == (LEN1, LEN2) else f"abs_mul64 {l1} x {l2} limbs",
                       "len1": l1, "len2": l2, "engine": engine_label(fmn, engine), "pieces": pieces,
                       "plan": plan_label(fmn, l1, l2),
                       "reference_ntt_len": fmn.ntt_len(l1, l2),
                       "parallelism": "replicas: one independent product per GPU" if ws > 1 else "single GPU",
                       "l2_policy": "no flush: operands (%d MB) and scratch (%d MB) per product exceed the 126 MB L2"
                                    % (16 * (l1 + l2) >> 20, fmn.workspace_size(l1, l2) >> 20)},
            "us_per_product": 1e3 * per_step_ms,
            "limbs_per_s": (l1 + l2) * value,
            "bit_exact": bit_exact,
            "roofline": hbm,
            "roofline_int": integer,
            "kernels": kernels,
            "gpu_launches": fmn.launches_per_product(l1, l2) * args.steps,
            "clocks": sampler.summary(),
            "e2e": {"value": ws * callers * e2e_steps / e2e_s, "unit": UNIT,
                    "h2d_bytes_per_step": io * callers, "d2h_bytes_per_step": io * callers,
                    "steps": e2e_steps, "bit_exact": e2e_exact, "callers": callers,
                    # the host link bounds this figure: io bytes each way per product
                    "link": dict(link, bound_products_per_s=ws * link["both_each_gbs"] * 1e9 / io,
                                 frac=(ws * callers * e2e_steps / e2e_s) / (ws * link["both_each_gbs"] * 1e9 / io)),
                    "path": ("abs_mul64 (C ABI) on pinned host buffers from %d host threads at once, one "
                             "synchronous call each per step (host wall clock)" % callers),
                    "single_caller": {"value": ws * e2e_steps / e2e1_s, "unit": UNIT,
                                      "h2d_bytes_per_step": io, "d2h_bytes_per_step": io,
                                      "path": "abs_mul64 (C ABI) on pinned host buffers, one thread, synchronous"},
                    "pageable": {"value": ws * callers * e2e_steps / pg_s, "unit": UNIT,
                                 "h2d_bytes_per_step": io * callers, "d2h_bytes_per_step": io * callers,
                                 "bit_exact": pg_exact, "callers": callers,
                                 "single_caller": ws * e2e_steps / pg1_s,
                                 "path": ("abs_mul64 (C ABI) on pageable (malloc-style numpy) host buffers, as the "
                                          "reference's callers pass them; %d threads at once, and one alone"
                                          % callers)}},
        }
    if dist:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    full = rank == 0 and (l1, l2) == (LEN1, LEN2) and ws == 1
    if full:
        del da, db, dout
        torch.cuda.empty_cache()
    if full and not args.no_extra:
        result["extra"] = extra_configs(fmn, torch, dev, peaks)
    if full and not args.no_batch:
        result["batch"] = batch_compare(fmn, torch, dev, args.batch_count)
    if full and not args.no_serve:
        torch.cuda.empty_cache()
        result["serve"] = serve_compare(fmn, torch, dev, args.serve_requests, rates)
    if full and not args.no_cpu_baseline:
        cb, cout = cpu_baseline(a, b)
        cb["bit_exact_vs_gpu"] = bool(np.array_equal(cout, got))
        result["cpu_baseline"] = cb
    if rank == 0:
        print(json.dumps(result), flush=True)


def main():
    args = parse()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
