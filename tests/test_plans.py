"""Pass plans: the host-side rules (CPU) and products under non-default plans (GPU)."""
import numpy as np
import pytest

import fast_mul_ntt_b200 as fmn
from fast_mul_ntt_b200 import synth


def test_default_plans():
    for n in (0, 9, 15, 25, 27):
        fmn.set_plan(n, None)                 # drop any tuned plan loaded by an earlier test
    assert fmn.get_plan(0) == [0]
    assert fmn.get_plan(9) == [9]
    assert fmn.get_plan(15) == [8, 7]
    assert fmn.get_plan(25) == [9, 8, 8]
    assert fmn.get_plan(27) == [9, 9, 9]
    for n in range(0, 31):
        bits = fmn.get_plan(n)
        assert sum(bits) == n and all(0 <= b <= 9 for b in bits)


def test_committed_plan_file_is_valid():
    """The B200 plan file shipped beside the library parses into valid plans for 2^10..2^27."""
    import os
    path = os.path.join(fmn.PLAN_DIR, "plans-NVIDIA_B200.txt")
    lines = [l.split("#")[0].split() for l in open(path) if l[0].isdigit()]
    head = open(path).read()
    assert "gpu NVIDIA B200" in head and "\ndriver " in head
    seen = set()
    for f in lines:
        n, p, bits = int(f[0]), int(f[1]), [int(x) for x in f[2:2 + int(f[1])]]
        assert sum(bits) == n and len(bits) == p and all(1 <= b <= 9 for b in bits)
        assert all(b >= 5 for b in bits[:-1])
        seen.add(n)
    assert seen == set(range(10, 28))
    # 32-bit engine lines: strided passes leave >= 32 columns (>= 5 bits after them)
    seen32 = set()
    for l in open(path):
        if not l.startswith("e32 "):
            continue
        f = l[4:].split("#")[0].split()
        n, p, bits = int(f[0]), int(f[1]), [int(x) for x in f[2:2 + int(f[1])]]
        assert sum(bits) == n <= 26 and len(bits) == p and all(1 <= b <= 9 for b in bits)
        assert all(b >= 5 and sum(bits[i + 1:]) >= 5 for i, b in enumerate(bits[:-1]))
        seen32.add(n)
    assert seen32 == set(range(11, 27))


def test_engine32_plans_validate_and_restore():
    e32 = fmn.ENGINE_32
    for n in (14, 25, 26):
        fmn.set_plan(n, None, engine=e32)
    assert fmn.get_plan(25, engine=e32) == [9, 8, 8]
    assert fmn.get_plan(26, engine=e32) == [9, 9, 8]
    with pytest.raises(fmn.FastMulError):
        fmn.set_plan(14, [5, 5, 4], engine=e32)       # a strided tile would have 16 columns
    fmn.set_plan(14, [5, 5, 4])                        # fine for the 64-bit engine (16-column tiles)
    fmn.set_plan(14, None)
    with pytest.raises(fmn.FastMulError):
        fmn.set_plan(27, [9, 9, 9], engine=e32)       # beyond the 32-bit engine's 2^26 digits
    fmn.set_plan(25, [7, 9, 9], engine=e32)
    try:
        assert fmn.get_plan(25, engine=e32) == [7, 9, 9]
        assert fmn.get_plan(25) == [9, 8, 8] or fmn.get_plan(25) != [7, 9, 9]   # 64-bit plans untouched
    finally:
        fmn.set_plan(25, None, engine=e32)
    assert fmn.get_plan(25, engine=e32) == [9, 8, 8]


def test_set_plan_validates_and_restores():
    with pytest.raises(fmn.FastMulError):
        fmn.set_plan(25, [10, 8, 7])          # a pass above 9 bits
    with pytest.raises(fmn.FastMulError):
        fmn.set_plan(25, [9, 8, 7])           # bits do not add up
    with pytest.raises(fmn.FastMulError):
        fmn.set_plan(15, [12, 3])             # strided pass too wide
    fmn.set_plan(25, [8, 9, 8])
    try:
        assert fmn.get_plan(25) == [8, 9, 8]
    finally:
        fmn.set_plan(25, None)
    assert fmn.get_plan(25) == [9, 8, 8]


@pytest.mark.gpu
def test_products_under_every_plan_shape(fmn, oracle):
    """Alternative splits (2 and 3 passes, last pass 9 bits or fewer) give the same numbers.
    Plans belong to the 64-bit residue engine, which these products are pinned to."""
    import torch
    cases = {15: [[7, 8], [5, 5, 5], [9, 6]], 18: [[9, 9], [6, 6, 6], [5, 9, 4]], 21: [[9, 6, 6], [5, 8, 8], [7, 7, 7]]}
    fmn.set_engine(fmn.ENGINE_64)
    try:
        for n, plans in cases.items():
            half = 1 << (n - 1)
            a, b = synth.operands("uniform", half, half - 3, n)
            want = oracle.mul(a, b)
            for bits in plans:
                fmn.set_plan(n, bits)
                assert np.array_equal(fmn.abs_mul64(a, b), want), (n, bits)
                assert np.array_equal(fmn.abs_sqr64(a), oracle.sqr(a)), (n, bits)
        # a large length against the default plan's (golden-pinned) result
        n = 24
        half = 1 << (n - 1)
        a, b = synth.operands("uniform", half, half, 5)
        da = torch.from_numpy(a.view(np.int64)).cuda()
        db = torch.from_numpy(b.view(np.int64)).cuda()
        ref = torch.empty(2 * half, dtype=torch.int64, device="cuda")
        fmn.set_plan(n, None)
        fmn.mul_device(da, db, ref)
        fmn.sync()
        for bits in ([8, 8, 8], [9, 7, 8], [7, 8, 9], [6, 6, 6, 6]):
            fmn.set_plan(n, bits)
            out = torch.empty_like(ref)
            fmn.mul_device(da, db, out)
            fmn.sync()
            assert torch.equal(out, ref), bits
    finally:
        fmn.set_engine(fmn.ENGINE_AUTO)
        for n in (15, 18, 21, 24):
            fmn.set_plan(n, None)


def test_engine_selection_rules():
    """AUTO takes the 32-bit residue engine wherever its plan (whole, split or wrapped) costs
    less than the 64-bit engine's transform, and the 64-bit one beyond; a forced engine is
    honoured where it applies."""
    assert fmn.get_engine() == fmn.ENGINE_AUTO
    assert fmn.engine_for(10_000_000, 10_000_000) == fmn.ENGINE_32
    assert fmn.engine_for(1 << 24, 1 << 24) == fmn.ENGINE_32             # 2^26-digit transform
    # one limb more: one wrapped coefficient, a 2^26-digit cyclic transform and a tiny low
    # product, cheaper than the 64-bit engine's 2^25-point transform or any split
    assert fmn.engine_for(1 << 24, (1 << 24) + 1) == fmn.ENGINE_32
    assert fmn.wrap_for(1 << 24, (1 << 24) + 1) == 1
    assert fmn.engine_for(1000, 1000, sqr=True) == fmn.ENGINE_32
    # 10M x 10M: 40M - 1 digit coefficients, a 2^25-digit cyclic transform whose first
    # 6,445,567 coefficients wrap, plus the twisted product modulo X^(2^23) - c
    assert fmn.pieces_for(10_000_000, 10_000_000) == 1
    assert fmn.wrap_for(10_000_000, 10_000_000) == 2 * 20_000_000 - 1 - (1 << 25)
    assert fmn.twist_for(10_000_000, 10_000_000) == 1 << 23
    # 20M x 20M: the cyclic length would be 2^26, too long for a twist of order 2^27: low product
    assert fmn.engine_for(20_000_000, 20_000_000) == fmn.ENGINE_32
    assert fmn.wrap_for(20_000_000, 20_000_000) > 0 and fmn.twist_for(20_000_000, 20_000_000) == 0
    assert fmn.wrap_for(1_000_000, 1_000_000) == 0                        # whole at 2^22 is cheaper
    # split products: unbalanced products above 2^25 limbs reach the 32-bit engine only split
    assert fmn.engine_for(64_000_000, 250_000) == fmn.ENGINE_32
    assert fmn.pieces_for(64_000_000, 250_000) > 1
    assert fmn.pieces_for(1_000_000, 1_000_000) == 1
    assert fmn.pieces_for(10_000_000, 10_000_000, sqr=True) == 1       # squares are never split
    assert fmn.engine_for(33_000_000, 33_000_000) == fmn.ENGINE_64      # a split would need 60 pieces
    assert fmn.engine_for(64_000_000, 64_000_000) == fmn.ENGINE_64      # beyond the coefficient range
    fmn.force_pieces(3)
    try:
        assert fmn.pieces_for(1000, 5000) == 3 and fmn.pieces_for(5000, 1000) == 3
        assert fmn.pieces_for(1000, 1000, sqr=True) == 1
    finally:
        fmn.force_pieces(0)
    fmn.set_engine(fmn.ENGINE_64)
    try:
        assert fmn.engine_for(10_000_000, 10_000_000) == fmn.ENGINE_64
        ws64 = fmn.workspace_size(1000, 3000)
    finally:
        fmn.set_engine(fmn.ENGINE_AUTO)
    fmn.set_engine(fmn.ENGINE_32)
    try:
        assert fmn.engine_for(64_000_000, 64_000_000) == fmn.ENGINE_64      # beyond its range
        ws32 = fmn.workspace_size(1000, 3000)
    finally:
        fmn.set_engine(fmn.ENGINE_AUTO)
    # 4000 limbs: 2^12-point transform of u64 vs 2^13 digits of u32 -- the same residue bytes
    assert ws32 == ws64
    with pytest.raises(fmn.FastMulError):
        fmn.set_engine(7)


def test_engine64_wrapped_plans():
    """The 64-bit engine's wrapped plans (the reference's primes): twisted where the second
    product's transform is a quarter of the cyclic one (10M x 10M: 2^24 + 2^22 limbs), the low
    product where K is tiny, the whole transform at exact powers of two (64M x 64M) and for
    small products (a second launch sequence does not pay), with the 15% margin keeping
    negacyclic plans whole; batches, spectra and the no-allocation path never wrap, and the
    scratch follows the plan."""
    fmn.set_engine(fmn.ENGINE_64)
    try:
        assert fmn.wrap_for(10_000_000, 10_000_000) == 20_000_000 - 1 - (1 << 24)
        assert fmn.twist_for(10_000_000, 10_000_000) == 1 << 22
        assert fmn.workspace_size(10_000_000, 10_000_000) < 3 * (1 << 25) * 8 * 2     # below the whole plan
        assert fmn.wrap_for(64_000_000, 64_000_000) == 0                              # 2^27 exactly
        assert fmn.wrap_for(2 ** 19 + 3, 2 ** 19) == 2 and fmn.twist_for(2 ** 19 + 3, 2 ** 19) == 0
        assert fmn.wrap_for(5000, 4000) == 0                                          # small: whole
        # K close to N: the twisted plan would be negacyclic (M = N), the low product as long as
        # the whole transform; neither is 15% cheaper
        assert fmn.wrap_for((1 << 20) - 5, (1 << 20) - 7) == 0
        fmn.force_wrap(2)
        assert fmn.twist_for(2 ** 13 + 5, 2 ** 13) == 1 << 12                       # four folds
        assert fmn.twist_for((1 << 14) - 1, (1 << 14) - 3) == 1 << 14                # negacyclic, forced
        fmn.force_wrap(1)
        assert fmn.wrap_for(2 ** 13 + 5, 2 ** 13) == 4 and fmn.twist_for(2 ** 13 + 5, 2 ** 13) == 0
        assert fmn.batch_twist_for(2 ** 13 + 5, 2 ** 13) == 0                        # 64-bit batches stay whole
    finally:
        fmn.force_wrap(0)
        fmn.set_engine(fmn.ENGINE_AUTO)


@pytest.mark.gpu
def test_products_under_engine32_plans(fmn, oracle):
    """32-bit engine: whole products (2^n digits, operands of 2^(n-2) limbs) and a split product
    under alternative plans give the reference's numbers; a resident operand created under one
    plan stays correct after the plan of its length changes."""
    import torch
    e32 = fmn.ENGINE_32
    cases = {15: [[8, 7], [5, 5, 5], [6, 9]], 18: [[9, 9], [6, 6, 6], [7, 5, 6]], 21: [[9, 6, 6], [5, 8, 8], [7, 7, 7]]}
    fmn.set_engine(e32)
    try:
        for n, plans in cases.items():
            q = 1 << (n - 2)
            a, b = synth.operands("uniform", q, q - 3, n)
            want, want_sq = oracle.mul(a, b), oracle.sqr(a)
            for bits in plans:
                fmn.set_plan(n, bits, engine=e32)
                assert np.array_equal(fmn.abs_mul64(a, b), want), (n, bits)
                assert np.array_equal(fmn.abs_sqr64(a), want_sq), (n, bits)
        fmn.force_pieces(3)
        a, b = synth.operands("ones", 20000, 70000, 8)
        for bits in ([9, 6, 6], [7, 7, 7]):
            fmn.set_plan(21, bits, engine=e32)
            assert fmn.pieces_for(len(a), len(b)) == 3
            assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b)), bits
        fmn.force_pieces(0)
        fmn.set_plan(18, [9, 9], engine=e32)
        a = synth.limbs("uniform", 30000, 3)
        op = fmn.Operand(torch.from_numpy(a.view(np.int64)).cuda(), max_partner_len=30000)
        try:
            b = synth.limbs("uniform", 25000, 4)
            fmn.set_plan(17, [6, 6, 5], engine=e32)
            fmn.set_plan(18, [6, 6, 6], engine=e32)
            out = torch.empty(len(a) + len(b), dtype=torch.int64, device="cuda")
            op.mul(torch.from_numpy(b.view(np.int64)).cuda(), out)
            fmn.sync()
            assert np.array_equal(out.cpu().numpy().view(np.uint64), oracle.mul(a, b))
        finally:
            op.close()
    finally:
        fmn.force_pieces(0)
        fmn.set_engine(fmn.ENGINE_AUTO)
        for n in (15, 17, 18, 21):
            fmn.set_plan(n, None, engine=e32)


@pytest.mark.gpu
def test_autotune_small_range(fmn, oracle, tmp_path):
    """The autotuner over 2^10..2^12 points writes a plan file for both engines, keeps valid
    plans in effect, and leaves the 32-bit engine's twiddle tables rebuilt for them: products
    of those lengths (and a longer one, whose tables were freed and rebuilt) stay exact."""
    path = str(tmp_path / "plans.txt")
    lib = fmn.load_library()
    try:
        fmn.autotune(10, 12, path)
        lines = [l.split("#")[0].split() for l in open(path) if l.strip() and not l.startswith("#")]
        ns64 = {int(l[0]) for l in lines if l[0].isdigit()}
        ns32 = {int(l[1]) for l in lines if l[0] == "e32"}
        assert ns64 == {10, 11, 12} and ns32 == {11, 12}     # 2^10 digits: a single 32-bit plan
        for la, lb in [(200, 300), (1000, 1000), (60000, 90000)]:
            a, b = synth.operands("uniform", la, lb, la)
            assert np.array_equal(fmn.abs_mul64(a, b), oracle.mul(a, b)), (la, lb)
    finally:
        for n in (10, 11, 12):
            fmn.set_plan(n, None)
            fmn.set_plan(n, None, engine=fmn.ENGINE_32)
        lib.fmn_load_default_plans()
