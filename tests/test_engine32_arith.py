"""The 32-bit residue engine's arithmetic, restated in Python integers (no GPU).

The engine (fast_mul_ntt_b200/csrc/fmn_arith32.cuh, fmn_ntt32.cu) splits each 64-bit limb
into two 32-bit digits and transforms them modulo three primes below 2^31.  These tests pin
the facts its exactness rests on: the primes and their 2-adic order, the coefficient bound
against the primes' product, the Shoup and Montgomery reductions it uses (with the ranges
the kernels rely on), the CRT by Garner's mixed-radix form with the same constants the
kernel receives, and the indexing of the precomputed four-step twiddle tables."""
import random

P0, P1, P2 = 2013265921, 1811939329, 469762049
PRIMES = (P0, P1, P2)
Q = P0 * P1 * P2
MAX_LOG_N = 26
M32 = (1 << 32) - 1


def is_prime(n):
    if n < 2:
        return False
    for p in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        if n % p == 0:
            return n == p
    d, s = n - 1, 0
    while d % 2 == 0:
        d //= 2
        s += 1
    for a in (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37):
        x = pow(a, d, n)
        if x in (1, n - 1):
            continue
        for _ in range(s - 1):
            x = x * x % n
            if x == n - 1:
                break
        else:
            return False
    return True


def qmont(a, b, p):
    """Montgomery product a * b * 2^-32 mod p as the kernel computes it (qmont)."""
    t = a * b
    m = ((t & M32) * pow(p, -1, 1 << 32)) & M32
    hi, mh = t >> 32, (m * p) >> 32
    r = (hi - mh) & M32
    return min(r, (r + p) & M32)


def qsmul(x, w, p):
    """Shoup product x * w mod p with w' = floor(w 2^32 / p) (qsmul)."""
    wp = (w << 32) // p
    hq = (x * wp) >> 32
    r = (x * w - hq * p) & M32
    assert r < 2 * p                      # the range the kernels' single correction relies on
    return min(r, (r - p) & M32)


def test_primes_and_orders():
    for p, c, k in ((P0, 15, 27), (P1, 27, 26), (P2, 7, 26)):
        assert is_prime(p) and p == c * 2 ** k + 1 and p < 2 ** 31
        assert (p - 1) % 2 ** MAX_LOG_N == 0
        # sums of two residues and u - v + p stay below 2^32; 4p does not (no lazy range)
        assert 2 * p < 2 ** 32 and (P2 == p or 4 * p > 2 ** 32)


def test_coefficient_bound():
    """A product whose shorter operand has at most 2^25 limbs (2^26 digits) has every digit
    coefficient below 2^26 (2^32 - 1)^2 < Q: the three residues determine it."""
    assert (1 << 26) * M32 * M32 < Q
    # and a longer shorter operand could exceed it
    assert (1 << 27) * M32 * M32 > Q


def test_shoup_and_montgomery_identities():
    rng = random.Random(1)
    for p in PRIMES:
        for _ in range(3000):
            x, w = rng.randrange(1 << 32), rng.randrange(p)
            assert qsmul(x, w, p) == x * w % p
            a, b = rng.randrange(p), rng.randrange(p)
            assert qmont(a, b, p) == a * b * pow(2, -32, p) % p
            b2 = rng.randrange(1, 2 * p)          # a lazy Montgomery result as second factor
            assert qmont(a, b2, p) == a * b2 * pow(2, -32, p) % p
        for x in (0, 1, p - 1, p, 2 * p - 1, M32):
            assert qsmul(x, p - 1, p) == x * (p - 1) % p


def garner_constants(n):
    N = 1 << n
    cst = [pow(N, -1, p) * pow(2, 64, p) % p for p in PRIMES]
    mont = lambda v, p: v % p * pow(2, 32, p) % p
    return cst, mont(pow(P0, -1, P1), P1), mont(P0, P2), mont(pow(P0 * P1, -1, P2), P2)


def garner(r, n):
    """Digit coefficient from the inverse transform's residues r_i = N c 2^-32 mod p_i, as
    k_qcrt_carry computes it."""
    cst, inv01, q0m2, inv012 = garner_constants(n)
    x0, y1, y2 = (qmont(r[i], cst[i], p) for i, p in enumerate(PRIMES))
    x0r = x0 - P1 if x0 >= P1 else x0
    x1 = qmont((y1 - x0r) % P1, inv01, P1)
    t = (qsmul(x0, 1, P2) + qmont(x1, q0m2, P2)) % P2
    x2 = qmont((y2 - t) % P2, inv012, P2)
    return x0 + P0 * x1 + P0 * P1 * x2


def test_garner_reconstructs_every_coefficient():
    rng = random.Random(2)
    bound = (1 << 26) * M32 * M32
    values = [0, 1, bound - 1, Q - 1] + [rng.randrange(bound) for _ in range(3000)]
    for n in (12, 25, 26):
        N = 1 << n
        for c in values:
            r = [N * c * pow(2, -32, p) % p for p in PRIMES]
            assert garner(r, n) == c


def test_digit_pairs_make_limbs():
    """Limb j is the low word of C_j = c_{2j} + c_{2j+1} 2^32 plus the high word of C_{j-1} and
    a carry: summing the digit convolution that way gives the limb product."""
    rng = random.Random(3)
    for la, lb in ((1, 1), (3, 5), (17, 9)):
        a = [rng.randrange(1 << 64) for _ in range(la)]
        b = [rng.randrange(1 << 64) for _ in range(lb)]
        da = [(x >> (32 * h)) & M32 for x in a for h in (0, 1)]
        db = [(x >> (32 * h)) & M32 for x in b for h in (0, 1)]
        conv = [0] * (len(da) + len(db))
        for i, x in enumerate(da):
            for k, y in enumerate(db):
                conv[i + k] += x * y
        limbs, carry, prev_hi = [], 0, 0
        for j in range(la + lb):
            C = conv[2 * j] + (conv[2 * j + 1] << 32)
            s = (C & ((1 << 64) - 1)) + prev_hi + carry
            limbs.append(s & ((1 << 64) - 1))
            carry, prev_hi = s >> 64, C >> 64
        A = sum(x << (64 * i) for i, x in enumerate(a))
        B = sum(x << (64 * i) for i, x in enumerate(b))
        assert sum(x << (64 * i) for i, x in enumerate(limbs)) == A * B


def _round_bits(l, i):
    if l <= 4:
        return l
    if l <= 8:
        return (l + 1) // 2 if i == 0 else l // 2
    return (l + 2) // 3 if i == 0 else (l + 1) // 3 if i == 1 else l // 3


def _bitrev(x, bits):
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def test_twiddle_table_index_matches_computed_twiddle():
    """A strided pass's four-step twiddle for row j (frequency bitrev(j)) and column i is formed
    on the fly as alpha(group) * beta(column, t') (group_alpha / fill_beta in fmn_ntt32.cu) or
    read from the table entry k * 2^logS + i (tw_group, k_qtw_build).  Both must name the same
    power w_B^(i k) for every element of every group of the lowest round."""
    rng = random.Random(4)
    for LOGL, logB in ((5, 12), (7, 15), (8, 17), (9, 17), (9, 20)):
        NR = 1 if LOGL <= 4 else 2 if LOGL <= 8 else 3
        RB = _round_bits(LOGL, NR - 1)
        logS = logB - LOGL
        shift = MAX_LOG_N - logB
        for _ in range(200):
            row0 = rng.randrange(1 << (LOGL - RB)) << RB
            i = rng.randrange(1 << logS)
            kq = _bitrev(row0 >> RB, LOGL - RB)
            for t in range(1 << RB):
                tp = _bitrev(t, RB)
                x_computed = ((i * kq) << shift) + ((i * (tp << (LOGL - RB))) << shift)
                k = kq + (tp << (LOGL - RB))
                assert k == _bitrev(row0 + t, LOGL)
                entry = (kq << logS) + i + tp * ((1 << logS) << (LOGL - RB))
                assert entry == k * (1 << logS) + i and entry < (1 << logB)
                assert x_computed % (1 << MAX_LOG_N) == ((i * k) << shift) % (1 << MAX_LOG_N)
