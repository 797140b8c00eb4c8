"""Differential sweep in the shape of the reference tree's only multiplication test
(fft_small/fsd_test.c:282-369: abs_mul64 / abs_sqr64 against a schoolbook product over a grid
of sizes 400..3000 in steps of 37 and over random sizes up to 2900, operands from a
xorshift64 generator seeded 0x20260912): every pair of the grid, random pairs and the squares
of the grid, on both engines, batched and per call, against the oracle's schoolbook
(unsigned __int128 sums, oracle/fmn_oracle.c)."""
import concurrent.futures as cf
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SIZES = list(range(400, 3001, 37))          # 71 sizes, as in the reference's sweep
SEED = 0x20260912
M64 = (1 << 64) - 1


class XorShift64:
    """Marsaglia's xorshift64 (shifts 13, 7, 17)."""

    def __init__(self, seed):
        self.x = seed

    def next(self):
        x = self.x
        x ^= (x << 13) & M64
        x ^= x >> 7
        x ^= (x << 17) & M64
        self.x = x
        return x

    def limbs(self, n):
        return np.array([self.next() for _ in range(n)], dtype=np.uint64)

    def below(self, n):
        return 1 + self.next() % n


@pytest.fixture(scope="module")
def sweep(oracle):
    """Operands and the schoolbook products of every case (computed once, on host threads)."""
    rng = XorShift64(SEED)
    A = {s: rng.limbs(s) for s in SIZES}
    B = {s: rng.limbs(s) for s in SIZES}
    pairs = [(A[s], B[t]) for s in SIZES for t in SIZES]
    for _ in range(200):
        pairs.append((rng.limbs(rng.below(2900)), rng.limbs(rng.below(2900))))
    squares = [A[s] for s in SIZES]
    with cf.ThreadPoolExecutor(max_workers=min(16, os.cpu_count() or 1)) as pool:
        want = list(pool.map(lambda p: oracle.schoolbook(p[0], p[1]), pairs))
        want_sq = list(pool.map(lambda a: oracle.schoolbook(a, a), squares))
    return pairs, want, squares, want_sq


@pytest.fixture(params=["e32", "e64"])
def engine(request, fmn):
    fmn.set_engine(fmn.ENGINE_AUTO if request.param == "e32" else fmn.ENGINE_64)
    yield request.param
    fmn.set_engine(fmn.ENGINE_AUTO)


def _dev(x):
    import torch
    return torch.from_numpy(np.ascontiguousarray(x).view(np.int64)).cuda()


def _host(t):
    return t.cpu().numpy().view(np.uint64)


def test_size_grid_batched_and_per_call(fmn, sweep, engine):
    import torch
    pairs, want, squares, want_sq = sweep
    ops = {}

    def dev(x):                                  # each operand copied once
        if id(x) not in ops:
            ops[id(x)] = _dev(x)
        return ops[id(x)]

    jobs, outs = [], []
    for a, b in pairs:
        out = torch.full((len(a) + len(b),), -1, dtype=torch.int64, device="cuda")
        jobs.append((dev(a), dev(b), out))
        outs.append(out)
    for a in squares:
        out = torch.full((2 * len(a),), -1, dtype=torch.int64, device="cuda")
        jobs.append((dev(a), dev(a), out))
        outs.append(out)
    fmn.mul_batch_device(jobs)
    fmn.sync()
    expected = want + want_sq
    bad = [i for i, (out, w) in enumerate(zip(outs, expected)) if not np.array_equal(_host(out), w)]
    assert not bad, [(len(jobs[i][0]), len(jobs[i][1])) for i in bad[:10]]

    # per call: the grid's diagonal, one row of it, and the squares
    n = len(SIZES)
    picks = [i * n + i for i in range(n)] + list(range(n * (n // 2), n * (n // 2) + n))
    for i in picks:
        a, b = pairs[i]
        out = torch.full((len(a) + len(b),), -1, dtype=torch.int64, device="cuda")
        fmn.mul_device(dev(a), dev(b), out)
        assert np.array_equal(_host(out), want[i]), (len(a), len(b))
    for a, w in zip(squares, want_sq):
        out = torch.full((2 * len(a),), -1, dtype=torch.int64, device="cuda")
        fmn.sqr_device(dev(a), out)
        assert np.array_equal(_host(out), w), len(a)
