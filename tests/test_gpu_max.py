"""The largest products the C ABI accepts: len1 + len2 - 1 <= 2^30 limbs (check_sizes in
fmn_api.cu), which the 64-bit engine runs as transforms of 2^30 points (the reference's
int_ceil2 length, src/fast_mul.c:299-306, at its maximum here).  Checked by size-independent
properties: residues modulo primes near 2^61 ((A mod q)(B mod q) == C mod q) and the lowest
limbs against the oracle's product of the operands' lowest limbs.  About 120 GB of device
memory and 16 GB of host memory; skipped where either is short."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

from helpers import CHECK_PRIMES

pytestmark = pytest.mark.gpu


def _host_available_gb():
    try:
        with open("/proc/meminfo") as f:
            for line in f:
                if line.startswith("MemAvailable:"):
                    return int(line.split()[1]) / (1 << 20)
    except OSError:
        pass
    return 0.0


def _mod(oracle, x, q, pool):
    """x mod q for a long limb vector, in chunks on host threads: sum of chunk_j * 2^(64 lo_j)."""
    step = 1 << 25
    parts = pool.map(lambda lo: (lo, oracle.mod(x[lo:lo + step], q)), range(0, len(x), step))
    base = (1 << 64) % q
    return sum(r * pow(base, lo, q) for lo, r in parts) % q


def _check(oracle, a, b, out, pool, sqr=False):
    for q in CHECK_PRIMES[:2]:
        ra = _mod(oracle, a, q, pool)
        rb = ra if sqr else _mod(oracle, b, q, pool)
        assert (ra * rb) % q == _mod(oracle, out, q, pool), f"residue mod {q}"
    k = 4096                                    # the lowest k limbs depend only on the lowest k of each operand
    low = oracle.sqr(a[:k]) if sqr else oracle.mul(a[:k], b[:k])
    assert np.array_equal(out[:k], low[:k])


def test_largest_accepted_products(fmn, oracle):
    import torch
    lib = fmn.load_library()
    lib.fmn_shutdown()                          # start from no cached workspace or tables
    torch.cuda.empty_cache()
    free, _ = torch.cuda.mem_get_info()
    if free < (135 << 30) or _host_available_gb() < 48:
        pytest.skip("needs about 120 GB of free device memory and 48 GB of host memory")
    fmn.init(0)
    l1 = l2 = 1 << 29                           # len1 + len2 - 1 = 2^30 - 1
    assert fmn.engine_for(l1, l2) == fmn.ENGINE_64
    dev = torch.device("cuda:0")
    g = torch.Generator(device=dev).manual_seed(30)
    a = torch.randint(-2**63, 2**63 - 1, (l1,), dtype=torch.int64, device=dev, generator=g)
    b = torch.randint(-2**63, 2**63 - 1, (l2,), dtype=torch.int64, device=dev, generator=g)
    a[-1] = -1                                  # top limbs all ones: the longest carry paths
    b[-1] = -1
    out = torch.empty(l1 + l2, dtype=torch.int64, device=dev)
    try:
        fmn.mul_device(a, b, out)
        fmn.sync()
        ha, hb, ho = (t.cpu().numpy().view(np.uint64) for t in (a, b, out))
        fmn.sqr_device(a, out)                  # 2 * 2^29 - 1 coefficients: also 2^30 points
        fmn.sync()
        hs = out.cpu().numpy().view(np.uint64)
    finally:
        del a, b, out
        lib.fmn_shutdown()
        torch.cuda.empty_cache()
        fmn.init(0)
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as pool:
        _check(oracle, ha, hb, ho, pool)
        _check(oracle, ha, None, hs, pool, sqr=True)
