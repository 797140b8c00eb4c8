"""Seeded synthetic operands for tests and benchmarks.

splitmix64 with a fixed seed (seed 0 by default); every limb is uniform over [0, 2^64).
Kinds:
  ``uniform`` -- uniform limbs, top limb forced nonzero;
  ``ones``    -- every limb 0xFFFFFFFFFFFFFFFF (longest carry chains);
  ``sparse``  -- each limb zero with probability 0.99, else uniform; top limb nonzero.
The second operand of a product uses ``seed + B_OFFSET`` so the two sides are independent.
"""
import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
M1 = np.uint64(0xBF58476D1CE4E5B9)
M2 = np.uint64(0x94D049BB133111EB)
B_OFFSET = 0x632BE59BD9B4E019
SPARSE_OFFSET = 0x2545F4914F6CDD1D
MASK64 = (1 << 64) - 1


def splitmix64(seed, n, start=0):
    """n outputs of splitmix64 seeded with ``seed``, beginning at output index ``start``."""
    with np.errstate(over="ignore"):
        idx = np.arange(start + 1, start + n + 1, dtype=np.uint64)
        z = np.uint64(seed & MASK64) + idx * GAMMA
        z = (z ^ (z >> np.uint64(30))) * M1
        z = (z ^ (z >> np.uint64(27))) * M2
        return z ^ (z >> np.uint64(31))


def limbs(kind, n, seed=0):
    """An n-limb operand of the given kind."""
    if n == 0:
        return np.zeros(0, dtype=np.uint64)
    if kind == "ones":
        return np.full(n, np.uint64(MASK64), dtype=np.uint64)
    x = splitmix64(seed, n)
    if kind == "sparse":
        keep = (splitmix64((seed + SPARSE_OFFSET) & MASK64, n) % np.uint64(100)) == 0
        x[~keep] = 0
    elif kind != "uniform":
        raise ValueError(f"unknown operand kind {kind!r}")
    if x[-1] == 0:
        x[-1] = 1
    return x


def operands(kind, len1, len2, seed=0):
    """The (in1, in2) pair of a product."""
    return limbs(kind, len1, seed), limbs(kind, len2, (seed + B_OFFSET) & MASK64)


def ntt_len(len1, len2):
    """Transform length of a product: next power of two >= len1 + len2 - 1."""
    conv = len1 + len2 - 1
    n = 1
    while n < conv:
        n <<= 1
    return n


def batch_mix(count=4096, lo=1000, hi=100000, sqr_frac=0.2, seed=0):
    """Mixed-size batch: each side log-uniform in [lo, hi] limbs independently, a fraction
    ``sqr_frac`` of the products squarings.  Returns a list of (op, len1, len2, seed)."""
    rng = np.random.default_rng(seed)
    l1 = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    l2 = np.exp(rng.uniform(np.log(lo), np.log(hi), count)).astype(np.int64)
    sq = rng.uniform(0, 1, count) < sqr_frac
    jobs = []
    for i in range(count):
        if sq[i]:
            jobs.append(("sqr", int(l1[i]), int(l1[i]), 1000 + i))
        else:
            jobs.append(("mul", int(l1[i]), int(l2[i]), 1000 + i))
    return jobs
