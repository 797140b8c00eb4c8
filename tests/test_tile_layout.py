"""Shared-memory tile layout of the 32-bit engine's contiguous passes (no GPU).

fast_mul_ntt_b200/csrc/fmn_ntt32.cu stores element (row j, column c) of a 2^LOGL-row tile at
j * 33 + c', c' a permutation of the 32 columns: for LOGL 5..8 the column index rotated right
by log2(32 / G) bits (G = the first round's groups per column), otherwise c ^ 16 (c & 1).
The round structure is fmn_rounds.cuh's.  These tests restate both and count, per warp-wide
32-bit shared access, the wavefronts each access pattern of the kernels needs: 1 means free
of bank conflicts."""
from collections import defaultdict

import pytest

TC, TP = 32, 33


def rounds_count(l):
    return 0 if l == 0 else 1 if l <= 4 else 2 if l <= 8 else 3


def round_bits(l, i):
    if l <= 4:
        return l
    if l <= 8:
        return (l + 1) // 2 if i == 0 else l // 2
    return (l + 2) // 3 if i == 0 else (l + 1) // 3 if i == 1 else l // 3


def round_top(l, i):
    return l - 1 if i == 0 else round_top(l, i - 1) - round_bits(l, i - 1)


def tix(l, j, c):
    if 5 <= l <= 8:
        g = (1 << l) >> round_bits(l, 0)
        w = {16: 1, 8: 2, 4: 3, 2: 4}[g]
        cp = ((c >> w) | (c << (5 - w))) & (TC - 1)
    else:
        cp = c ^ ((c & 1) << 4)
    return j * TP + cp


def wavefronts(addrs):
    banks = defaultdict(set)
    for a in addrs:
        banks[a % 32].add(a)
    return max(len(v) for v in banks.values())


def round_accesses(l, fr, qfast):
    """Per warp and per element t of a group: the (row, column) pairs of its 32 lanes, for
    round fr of a contiguous pass (run_round: QFAST lanes on the groups of a column first)."""
    L, rb, top = 1 << l, round_bits(l, fr), round_top(l, fr)
    R, spl = 1 << rb, top - rb + 1
    sp, gpc = 1 << spl, L >> rb
    G = gpc * TC
    for w0 in range(0, G, 32):
        lanes = []
        for gi in range(w0, min(w0 + 32, G)):
            g, c = (gi % gpc, gi // gpc) if qfast else (gi >> 5, gi & (TC - 1))
            row0 = (g & (sp - 1)) + ((g >> spl) << (top + 1))
            lanes.append((row0, c))
        for t in range(R):
            yield [(r + t * sp, c) for r, c in lanes]


@pytest.mark.parametrize("l", range(1, 10))
def test_columns_are_permuted_within_a_row(l):
    for j in range(4):
        assert sorted(tix(l, j, c) - j * TP for c in range(TC)) == list(range(TC))


@pytest.mark.parametrize("l", range(1, 10))
def test_every_round_is_conflict_free(l):
    for fr in range(rounds_count(l)):
        # a thread per column in every round; the first (and last inverse) round of a
        # contiguous pass also with the lanes on the groups of a column
        for qf in (False, True) if round_top(l, fr) == l - 1 else (False,):
            for pat in round_accesses(l, fr, qf):
                assert wavefronts([tix(l, j, c) for j, c in pat]) == 1, (l, fr, qf)


@pytest.mark.parametrize("l", range(1, 10))
def test_lowest_round_and_row_copy_out(l):
    """fused_lowest (a thread per column, 2^RB consecutive rows) and the row-wise copy-out of
    the last pass (lanes on consecutive words of one block; tiles of >= 32 rows)."""
    L, rb = 1 << l, round_bits(l, rounds_count(l) - 1)
    G = (L >> rb) * TC
    for w0 in range(0, G, 32):
        lanes = [(((gi >> 5) << rb), gi & (TC - 1)) for gi in range(w0, min(w0 + 32, G))]
        for t in range(1 << rb):
            assert wavefronts([tix(l, r + t, c) for r, c in lanes]) == 1
    if l >= 5:
        for e0 in range(0, TC * L, 32):
            assert wavefronts([tix(l, e & (L - 1), e >> l) for e in range(e0, e0 + 32)]) == 1


def test_fixed_swizzle_had_first_round_conflicts():
    """The layout before the rotation (c ^ 16 (c & 1) for every size) needed two wavefronts per
    access in the first round of 5..8-bit tiles: the reason for the size-dependent rotation."""
    def old(l, j, c):
        return j * TP + (c ^ ((c & 1) << 4))
    for l in range(5, 9):
        worst = max(wavefronts([old(l, j, c) for j, c in pat]) for pat in round_accesses(l, 0, True))
        assert worst == 2


def test_dense_strided_tiles_are_conflict_free():
    """Strided passes of both engines use dense tiles: 32 u32 columns per row (32-bit engine,
    a warp on one row's 32 columns) and 16 u64 columns per row (64-bit engine, a warp on two
    rows; a 64-bit access is served in two half-warp phases, each one 128-byte row).  Every
    phase then touches each of the 32 banks once."""
    for j0 in range(0, 64, 1):
        assert wavefronts([j0 * 32 + c for c in range(32)]) == 1          # u32, one row
    for j0 in range(0, 64, 2):
        for half in (0, 1):                                               # u64, word pairs
            words = [((j0 + half) * 16 + c) * 2 + h for c in range(16) for h in (0, 1)]
            assert wavefronts(words) == 1
