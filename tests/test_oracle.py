"""CPU tests: the oracle restatement is pinned to the reference (golden vectors produced by
the reference's own src/ code, and its published constants)."""
import os

import numpy as np
import pytest

from fast_mul_ntt_b200 import synth
from tests.helpers import digest, operands_for


def test_splitmix_pinned():
    # splitmix64 seeded with 0: the well-known first outputs of the generator
    assert [int(v) for v in synth.splitmix64(0, 3)] == [0xE220A8397B1DCDAF, 0x6E789E6AA1B965F4, 0x06C45D188009454F]


def test_operand_kinds():
    a = synth.limbs("uniform", 1000, 7)
    assert a.dtype == np.uint64 and len(a) == 1000 and a[-1] != 0
    assert np.all(synth.limbs("ones", 10, 0) == np.uint64(2**64 - 1))
    s = synth.limbs("sparse", 100000, 3)
    nz = np.count_nonzero(s)
    assert 700 < nz < 1300 and s[-1] != 0
    x, y = synth.operands("uniform", 5, 5, 0)
    assert not np.array_equal(x, y)


def test_constants_match_reference(oracle):
    # src/data.h:79-81 (primes), :84-86 (R^2 mod p), :106-108 (-p^-1 mod 2^64),
    # :155-157 (Montgomery one), :94-96 (Montgomery form of the primitive root)
    expect = [
        (2485986994308513793, 2485986994308513791, 1974795801822054070, 1044835113549955065, 252201579132747739),
        (1945555039024054273, 1945555039024054271, 269548777697434221, 936748722493063159, 792633534417207249),
        (4179340454199820289, 4179340454199820287, 1878466934230121386, 1729382256910270460, 1008806316530991091),
    ]
    for i in range(3):
        assert tuple(oracle.constants(i)) == expect[i]


def test_crt_constants_match_reference(oracle):
    # src/core.h:78-84: mod23, mod13, mod12 (u128), mont_mod23_inv1, mont_mod13_inv2,
    # mont_mod12_inv3, mod123 (u192)
    c = oracle.crt_constants()
    assert c[0:2] == [6124895493223874561, 440789813528887296]
    assert c[2:4] == [6665327448508334081, 563231428398022656]
    assert c[4:6] == [4431542033332568065, 262193940805976064]
    assert c[6:9] == [84629344487098392, 75311807962221426, 3875284113674644599]
    assert c[9:12] == [8610882487532388353, 1266215182732886016, 59403314713853952]


def test_golden_file_shape(golden):
    ops = {(c["op"], c["kind"]) for c in golden}
    assert ("mul", "uniform") in ops and ("mul", "ones") in ops and ("mul", "sparse") in ops
    assert ("sqr", "uniform") in ops
    sizes = {(c["len1"], c["len2"]) for c in golden}
    assert (10000, 10000) in sizes
    for c in golden:
        if "limbs" in c:
            assert len(c["limbs"]) == c["len1"] + c["len2"]


def test_oracle_matches_golden(oracle, golden):
    """Every golden case up to 40k output limbs: the oracle restatement reproduces the
    reference's output bit for bit."""
    n = 0
    for c in golden:
        if c["len1"] + c["len2"] > 140000:
            continue
        a, b = operands_for(c)
        out = oracle.sqr(a) if c["op"] == "sqr" else oracle.mul(a, b)
        assert digest(out) == c["sha256"], c
        if "limbs" in c:
            assert [f"{int(v):016x}" for v in out] == c["limbs"]
        n += 1
    assert n > 800


def test_oracle_vs_schoolbook(oracle):
    rng = np.random.default_rng(5)
    for _ in range(40):
        la, lb = int(rng.integers(1, 300)), int(rng.integers(1, 300))
        a = rng.integers(0, 2**64, la, dtype=np.uint64)
        b = rng.integers(0, 2**64, lb, dtype=np.uint64)
        assert np.array_equal(oracle.mul(a, b), oracle.schoolbook(a, b))
        assert np.array_equal(oracle.sqr(a), oracle.schoolbook(a, a))


def test_oracle_zero_lengths(oracle):
    a = synth.limbs("uniform", 5, 1)
    assert np.array_equal(oracle.mul(a, np.zeros(0, np.uint64)), np.zeros(5, np.uint64))
    assert len(oracle.mul(np.zeros(0, np.uint64), np.zeros(0, np.uint64))) == 0


def test_oracle_residue_property(oracle):
    from tests.helpers import residue_check
    a, b = synth.operands("uniform", 3000, 1234, 9)
    out = oracle.mul(a, b)
    assert residue_check(oracle, a, b, out)
    out[17] ^= np.uint64(1 << 40)                    # a planted error is caught
    assert not residue_check(oracle, a, b, out)


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))),
                                                    "oracle", "_ref", "libref_fastmul.so")),
                    reason="reference build (oracle/_ref) not present")
def test_reference_build_matches_golden(golden):
    from oracle.oracle import RefFastMul
    ref = RefFastMul()
    for c in golden:
        if c["len1"] + c["len2"] > 40000:
            continue
        a, b = operands_for(c)
        out = ref.sqr(a) if c["op"] == "sqr" else ref.mul(a, b)
        assert digest(out) == c["sha256"], c
