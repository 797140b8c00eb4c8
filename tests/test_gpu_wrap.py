"""Wrapped products on the 32-bit engine: a cyclic transform of 2^n digits whose first K
coefficients hold c_k + c_{k+2^n}, plus the product of the operands' lowest digits, separated
again in the CRT.  Every product must equal the reference's digest and the oracle bit for bit,
whether the cost model picks the wrapped plan (10M x 10M) or it is forced (all shapes that
allow one, including lengths just above a power of two, squares and unbalanced operands)."""
import numpy as np
import pytest

from fast_mul_ntt_b200 import synth
from tests.helpers import digest, operands_for

pytestmark = pytest.mark.gpu


@pytest.fixture
def forced_wrap(fmn):
    fmn.set_engine(fmn.ENGINE_32)
    fmn.force_wrap(True)
    yield
    fmn.force_wrap(False)
    fmn.set_engine(fmn.ENGINE_AUTO)


def test_golden_small_and_medium_wrapped(fmn, golden, forced_wrap):
    n_wrapped = 0
    for c in golden:
        if c["len1"] + c["len2"] > 140000:
            continue
        a, b = operands_for(c)
        out = fmn.abs_sqr64(a) if c["op"] == "sqr" else fmn.abs_mul64(a, b)
        assert digest(out) == c["sha256"], (c["op"], c["kind"], c["len1"], c["len2"])
        n_wrapped += fmn.wrap_for(c["len1"], c["len2"], c["op"] == "sqr") > 0
    assert n_wrapped > 300


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
    assert fmn.wrap_for(la, lb) > 0
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


def test_cost_model_wraps_10M_and_matches_reference(fmn, golden):
    """The bench configuration: the cost model picks the wrapped plan (2^25-digit cyclic
    transform + a 3.2M x 3.2M-limb low product) and the result is the reference's."""
    assert fmn.engine_for(10_000_000, 10_000_000) == fmn.ENGINE_32
    assert fmn.wrap_for(10_000_000, 10_000_000) > 0
    for op, kind in (("mul", "uniform"), ("mul", "ones"), ("sqr", "uniform")):
        c = next(c for c in golden if (c["op"], c["kind"], c["len1"], c["len2"]) == (op, kind, 10_000_000, 10_000_000))
        a, b = operands_for(c)
        out = fmn.abs_sqr64(a) if op == "sqr" else fmn.abs_mul64(a, b)
        assert digest(out) == c["sha256"], (op, kind)
