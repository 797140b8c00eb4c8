"""Shared helpers of the test suite (operands, digests, modular checks)."""
import hashlib

import numpy as np

from fast_mul_ntt_b200 import synth

# A few primes near 2^61 for size-independent residue checks: (A mod q)(B mod q) == C mod q.
CHECK_PRIMES = [2305843009213693951, 2305843009213693921, 2305843009213693907]


def digest(x):
    return hashlib.sha256(np.ascontiguousarray(x, dtype="<u8").tobytes()).hexdigest()


def operands_for(case):
    return synth.operands(case["kind"], case["len1"], case["len2"], case["seed"])


def residue_check(oracle, a, b, out, sqr=False):
    """Size-independent property: (A mod q)(B mod q) == (A*B) mod q for several primes q."""
    for q in CHECK_PRIMES:
        ra = oracle.mod(a, q)
        rb = ra if sqr else oracle.mod(b, q)
        if (ra * rb) % q != oracle.mod(out, q):
            return False
    return True
