"""Wrapped products on the 32-bit engine: a cyclic transform of 2^n digits whose first K
coefficients hold c_k + c_{k+2^n}, separated again in the CRT with the help of either the
product of the operands' lowest digits (mode 1) or the twisted product modulo X^M - c
(mode 2).  Every product must equal the reference's digest and the oracle bit for bit,
whether the cost model picks the plan (10M x 10M: twisted, M = 2^23) or it is forced (all
shapes that allow one, including lengths just above a power of two, squares, unbalanced
operands and the negacyclic case M = 2^n)."""
import numpy as np
import pytest

from fast_mul_ntt_b200 import synth
from tests.helpers import digest, operands_for

pytestmark = pytest.mark.gpu


@pytest.fixture(params=[1, 2], ids=["low", "twisted"])
def forced_wrap(fmn, request):
    fmn.set_engine(fmn.ENGINE_32)
    fmn.force_wrap(request.param)
    yield request.param
    fmn.force_wrap(0)
    fmn.set_engine(fmn.ENGINE_AUTO)


def _wrapped(fmn, mode, la, lb, sqr=False):
    """Whether the forced plan applies to this shape (the twisted one needs 2^n >= 2^12)."""
    return fmn.wrap_for(la, lb, sqr) > 0 and (mode == 1 or fmn.twist_for(la, lb, sqr) > 0)


def test_golden_small_and_medium_wrapped(fmn, golden, forced_wrap):
    n_wrapped = 0
    for c in golden:
        if c["len1"] + c["len2"] > 140000:
            continue
        a, b = operands_for(c)
        out = fmn.abs_sqr64(a) if c["op"] == "sqr" else fmn.abs_mul64(a, b)
        assert digest(out) == c["sha256"], (c["op"], c["kind"], c["len1"], c["len2"])
        n_wrapped += _wrapped(fmn, forced_wrap, c["len1"], c["len2"], c["op"] == "sqr")
    assert n_wrapped > (300 if forced_wrap == 1 else 5)


def test_lengths_just_above_powers_of_two(fmn, oracle, forced_wrap):
    """Coefficient counts 2^k + 1 .. 2^k + 3 (one to three wrapped coefficients), 2^(k+1) - 1
    (almost everything wraps), and operands that exactly fill the cyclic length."""
    for k in range(3, 21):
        for la, lb in [(2 ** (k - 2) + 1, 2 ** (k - 2)), (2 ** (k - 2) + 1, 2 ** (k - 2) + 1),
                       (2 ** (k - 1), 2 ** (k - 1)), (2 ** (k - 1), 3), (2 ** (k - 1) - 1, 2 ** (k - 2) + 7)]:
            for kind in ("uniform", "ones"):
                a, b = synth.operands(kind, la, lb, k)
                got = fmn.abs_mul64(a, b)
                assert np.array_equal(got, oracle.mul(a, b)), (kind, la, lb, fmn.wrap_for(la, lb))
        a = synth.limbs("ones", 2 ** (k - 2) + 1, k)
        assert np.array_equal(fmn.abs_sqr64(a), oracle.sqr(a)), ("sqr", k)


def test_random_shapes_wrapped(fmn, oracle, forced_wrap):
    rng = np.random.default_rng(77)
    for i in range(40):
        la = int(np.exp(rng.uniform(0, np.log(400000))))
        lb = int(np.exp(rng.uniform(0, np.log(400000))))
        kind = ("uniform", "ones", "sparse")[i % 3]
        a, b = synth.operands(kind, la, lb, 500 + i)
        assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b)), (kind, la, lb, fmn.wrap_for(la, lb))


def test_device_and_host_paths_wrapped(fmn, oracle, forced_wrap):
    """The same wrapped product through the device API and through the overlapped host path
    on pinned buffers (the second operand's low limbs are copied before the rest)."""
    import torch
    la, lb = 300001, 270000
    a, b = synth.operands("uniform", la, lb, 3)
    assert _wrapped(fmn, forced_wrap, la, lb)
    want = oracle.mul(a, b)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.empty(la + lb, dtype=torch.int64, device="cuda")
    fmn.mul_device(da, db, out)
    fmn.sync()
    assert np.array_equal(out.cpu().numpy().view(np.uint64), want)
    pa = torch.from_numpy(a.view(np.int64)).pin_memory().numpy().view(np.uint64)
    pb = torch.from_numpy(b.view(np.int64)).pin_memory().numpy().view(np.uint64)
    po = torch.zeros(la + lb, dtype=torch.int64).pin_memory().numpy().view(np.uint64)
    assert np.array_equal(fmn.abs_mul64(pa, pb, out=po), want)


def test_twisted_folds_and_negacyclic(fmn, oracle, forced_wrap):
    """Twisted products with 1, 2 and 4 folds of the operands modulo X^M - c (M = 2^n down
    to 2^(n-2)), all-ones carries, squares."""
    if forced_wrap != 2:
        pytest.skip("twisted plan only")
    n = 16
    N = 1 << n
    for K in (N, N // 2 + 5, N // 4 + 1, N // 8, 3):          # wrapped coefficients
        dc = N + K
        la = (dc + 1) // 4
        lb = (dc + 1) // 2 - la
        for kind in ("uniform", "ones"):
            a, b = synth.operands(kind, la, lb, K)
            assert fmn.twist_for(la, lb) > 0, (la, lb)
            assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b)), (kind, la, lb, fmn.twist_for(la, lb))
    a = synth.limbs("ones", N // 2, 7)
    assert np.array_equal(fmn.abs_sqr64(a), oracle.sqr(a))


def test_cost_model_wraps_10M_and_matches_reference(fmn, golden):
    """The bench configuration: the cost model picks the twisted plan (a 2^25-digit cyclic
    transform + a 2^23-digit twisted one) and the result is the reference's."""
    assert fmn.engine_for(10_000_000, 10_000_000) == fmn.ENGINE_32
    assert fmn.wrap_for(10_000_000, 10_000_000) > 0
    assert fmn.twist_for(10_000_000, 10_000_000) == 1 << 23
    for op, kind in (("mul", "uniform"), ("mul", "ones"), ("sqr", "uniform")):
        c = next(c for c in golden if (c["op"], c["kind"], c["len1"], c["len2"]) == (op, kind, 10_000_000, 10_000_000))
        a, b = operands_for(c)
        out = fmn.abs_sqr64(a) if op == "sqr" else fmn.abs_mul64(a, b)
        assert digest(out) == c["sha256"], (op, kind)


@pytest.fixture
def engine64(fmn):
    fmn.set_engine(fmn.ENGINE_64)
    yield
    fmn.force_wrap(0)
    fmn.set_engine(fmn.ENGINE_AUTO)


def test_engine64_wrapped_products(fmn, oracle, golden, engine64):
    """The 64-bit engine (the reference's primes) wraps a product of dc = la + lb - 1 limb
    coefficients just above 2^n around the cyclic length 2^n and recovers c_0 .. c_{K-1} from
    the product of the operands' lowest K = dc - 2^n limbs: forced wherever it applies (small
    shapes, multiplies and squares, one to 147k wrapped coefficients) and chosen by the cost
    model (large shapes, where the saving outweighs a second launch sequence), against the
    oracle and the reference's golden digests."""
    forced = []
    for k in range(13, 19):
        forced += [(2 ** (k - 1) + 3, 2 ** (k - 1), False), (2 ** (k - 1) + 2 ** (k - 4), 2 ** (k - 1), False),
                   (2 ** k - 5, 9 * 2 ** (k - 4), False), (2 ** (k - 1) + 7, 2 ** (k - 1) + 7, True)]
    modelled = [(2 ** 19 + 3, 2 ** 19, False), (2 ** 19 + 2 ** 16, 2 ** 19, False), (600000, 700001, False),
                (2 ** 20 + 7, 2 ** 20 + 7, True)]
    for mode, shapes in ((1, forced), (2, forced), (0, modelled)):
        fmn.force_wrap(mode)
        for i, (la, lb, sq) in enumerate(shapes):
            assert fmn.wrap_for(la, lb, sq) > 0, (mode, la, lb, sq)
            assert (fmn.twist_for(la, lb, sq) > 0) == (mode == 2) or mode == 0, (mode, la, lb, sq)
            a, b = synth.operands(("uniform", "ones", "sparse")[i % 3], la, lb, 300 + i)
            if sq:
                assert np.array_equal(fmn.abs_sqr64(a), oracle.sqr(a)), (mode, la)
            else:
                assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b)), (mode, la, lb, fmn.wrap_for(la, lb))
    fmn.force_wrap(1)
    n = 0
    for c in golden:
        if c["len1"] + c["len2"] > 140000 or c["len1"] + c["len2"] < 4097:
            continue
        a, b = operands_for(c)
        out = fmn.abs_sqr64(a) if c["op"] == "sqr" else fmn.abs_mul64(a, b)
        assert digest(out) == c["sha256"], (c["op"], c["kind"], c["len1"], c["len2"])
        n += fmn.wrap_for(c["len1"], c["len2"], c["op"] == "sqr") > 0
    assert n >= 3


def test_engine64_twisted_folds(fmn, oracle, engine64):
    """The 64-bit engine's twisted form with one to four folds (M = 2^n .. 2^(n-2)), squares
    and operands of unequal length, against the oracle."""
    fmn.force_wrap(2)
    n = 14
    for la, lb, sq in [(2 ** (n - 1) + 5, 2 ** (n - 1), False), (2 ** n - 1, 2 ** (n - 2) + 3, False),
                       (2 ** n - 1, 2 ** n - 3, False), (2 ** (n - 1) + 9, 2 ** (n - 1) + 9, True),
                       (2 ** n - 2, 2 ** n - 2, True), (3 * 2 ** (n - 2), 2 ** (n - 1) + 2 ** (n - 3), False)]:
        assert fmn.twist_for(la, lb, sq) > 0, (la, lb, sq)
        a, b = synth.operands("ones" if la % 2 else "uniform", la, lb, la + lb)
        want = oracle.sqr(a) if sq else oracle.mul(a, b)
        got = fmn.abs_sqr64(a) if sq else fmn.abs_mul64(a, b)
        assert np.array_equal(got, want), (la, lb, sq, fmn.twist_for(la, lb, sq))


def test_engine64_wrapped_10M_matches_reference(fmn, golden, engine64):
    """10M x 10M on the 64-bit engine runs wrapped (cyclic 2^24 limbs + the twisted product
    modulo X^(2^22) - c) and equals the reference's digest, on the device path and through
    abs_mul64."""
    import torch
    assert fmn.wrap_for(10_000_000, 10_000_000) == 3_222_783
    assert fmn.twist_for(10_000_000, 10_000_000) == 1 << 22
    c = next(c for c in golden if c["op"] == "mul" and c["kind"] == "uniform" and c["len1"] == 10_000_000
             and c["len2"] == 10_000_000)
    a, b = operands_for(c)
    da = torch.from_numpy(a.view(np.int64)).cuda()
    db = torch.from_numpy(b.view(np.int64)).cuda()
    out = torch.empty(20_000_000, dtype=torch.int64, device="cuda")
    fmn.mul_device(da, db, out)
    fmn.sync()
    assert digest(out.cpu().numpy().view(np.uint64)) == c["sha256"]
    assert digest(fmn.abs_mul64(a, b)) == c["sha256"]
