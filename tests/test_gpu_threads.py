"""Several host threads calling abs_mul64 / abs_sqr64 at once.

The reference's functions are plain reentrant C; a caller may run products from several
threads.  Here each call runs on one of the device's host lanes (its own workspace, buffers
and streams; 4 by default), so more threads than lanes also exercises a caller waiting for a
free lane.  Every thread's products must still equal the oracle's bit for bit, whatever the
engine and the split plan of the shapes involved."""
import threading

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth

pytestmark = pytest.mark.gpu

# balanced, unbalanced (split on the 32-bit engine), tiny, and squares
SHAPES = [(20000, 20000), (3000, 90001), (90001, 3000), (1, 7), (40000, None), (777, None)]
THREADS = 6


def test_concurrent_host_calls(fmn, oracle):
    cases = []
    for t in range(THREADS):
        for i, (la, lb) in enumerate(SHAPES):
            a, b = synth.operands("uniform", la, lb or 1, 100 * t + i)
            want = oracle.sqr(a) if lb is None else oracle.mul(a, b)
            cases.append((t, la, lb, a, b, want))
    errors = []
    barrier = threading.Barrier(THREADS)

    def worker(t):
        try:
            barrier.wait(timeout=60)
            for rep in range(3):
                for (tt, la, lb, a, b, want) in cases:
                    if tt != t:
                        continue
                    got = fmn.abs_sqr64(a) if lb is None else fmn.abs_mul64(a, b)
                    if not np.array_equal(got, want):
                        errors.append((t, rep, la, lb))
        except Exception as e:                  # reported by the main thread
            errors.append((t, repr(e)))

    threads = [threading.Thread(target=worker, args=(t,)) for t in range(THREADS)]
    for th in threads:
        th.start()
    for th in threads:
        th.join(timeout=300)
    assert not any(th.is_alive() for th in threads)
    assert not errors, errors
