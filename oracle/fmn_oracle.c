/*
 * fmn_oracle.c -- CPU oracle for the 3-prime Montgomery NTT multiplication path of
 * HJimmyK/fast_mul_ntt (src/).
 *
 * TEST INFRASTRUCTURE ONLY.  tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py load this library as the checker.  The product (fast_mul_ntt_b200/) never
 * links, loads or calls it, and has no CPU fallback.
 *
 * It restates the reference algorithm in plain C with unsigned __int128:
 *   - primes and primitive roots: src/data.h:69-71 (roots 5, 5, 3), src/data.h:79-81;
 *     every other constant (R^2 mod p, -p^-1 mod 2^64, Montgomery one, roots of unity,
 *     CRT cofactors) is derived here at start-up instead of being copied;
 *   - Montgomery arithmetic with R = 2^64: REDC as in _mont_mul / _mont_mulinto /
 *     _mont_tomont / _mont_toint (src/macro.h:160-211);
 *   - ntt_len = next power of two >= len1 + len2 - 1 (int_ceil2, src/fast_mul.c:299-312);
 *   - per prime: to-Montgomery entry of both operands (src/fast_mul.c:331-353), forward
 *     DIF, pointwise Montgomery product, inverse DIT, scaling by ntt_len^-1
 *     (conv_rec / conv_sqr, src/fast_mul.c:51-133 and 214-288; dif / idit,
 *     src/core.h:443-509);
 *   - crt3 (src/core.h:77-104) and the serial 192-bit carry loop (src/fast_mul.c:378-389,
 *     442-453).
 * The transform is a plain iterative radix-2 NTT; the reference's radix-4 and recursive
 * split compute the same cyclic convolution mod each prime, and the outputs are exact
 * integers, so the two agree limb for limb.  That agreement is checked against the
 * reference compiled from its own sources (oracle/Makefile, target `ref`) and against
 * committed golden vectors (tests/golden/).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned long long u64;
typedef unsigned __int128 u128;

typedef struct {
    u64 p;      /* the prime, p = c * 2^k + 1                           */
    u64 g;      /* primitive root (src/data.h:69-71)                    */
    u64 ninv;   /* -p^-1 mod 2^64 (modInvNeg, src/data.h:106-108)        */
    u64 r1;     /* R mod p (Montgomery one, src/data.h:155-157)          */
    u64 r2;     /* R^2 mod p (src/data.h:84-86)                          */
} prime_t;

static prime_t PR[3];
static u64 CRT_M[3][2];   /* M_i = (p1 p2 p3) / p_i as u128 words (mod23, mod13, mod12) */
static u64 CRT_INV[3];    /* M_i^-1 mod p_i in Montgomery form (mont_mod23_inv1 ...)    */
static u64 CRT_P[3];      /* p1 p2 p3 as u192 words (mod123, src/core.h:78)            */
static int g_ready = 0;

/* ---------------------------------------------------------------- Montgomery (R = 2^64) */

/* REDC of t < p * 2^64, fully reduced to [0, p) (src/macro.h:182-191 _mont_mulinto). */
static inline u64 redc(u128 t, const prime_t* q) {
    u64 m = (u64)t * q->ninv;
    u128 s = t + (u128)m * q->p;          /* < 2p * 2^64 < 2^128 because p < 2^63 */
    u64 r = (u64)(s >> 64);
    return r >= q->p ? r - q->p : r;
}
static inline u64 mmul(u64 a, u64 b, const prime_t* q) { return redc((u128)a * b, q); }
static inline u64 to_mont(u64 x, const prime_t* q) { return mmul(x, q->r2, q); }   /* x < 2^64 */
static inline u64 from_mont(u64 x, const prime_t* q) { return redc((u128)x, q); }
static inline u64 madd(u64 a, u64 b, const prime_t* q) { u64 s = a + b; return s >= q->p ? s - q->p : s; }
static inline u64 msub(u64 a, u64 b, const prime_t* q) { return a >= b ? a - b : a + q->p - b; }

static u64 mpow(u64 base_m, u64 e, const prime_t* q) {   /* Montgomery in, Montgomery out */
    u64 r = q->r1;
    while (e) {
        if (e & 1) r = mmul(r, base_m, q);
        base_m = mmul(base_m, base_m, q);
        e >>= 1;
    }
    return r;
}

/* plain modular helpers used only while deriving constants */
static u64 pmulmod(u64 a, u64 b, u64 m) { return (u64)(((u128)a * b) % m); }
static u64 ppow(u64 b, u64 e, u64 m) {
    u64 r = 1 % m;
    b %= m;
    while (e) {
        if (e & 1) r = pmulmod(r, b, m);
        b = pmulmod(b, b, m);
        e >>= 1;
    }
    return r;
}

static void init_prime(prime_t* q, u64 p, u64 g) {
    q->p = p;
    q->g = g;
    u64 inv = 1;                            /* Newton: inv = p^-1 mod 2^64 */
    for (int i = 0; i < 7; i++) inv *= 2 - p * inv;
    q->ninv = (u64)0 - inv;
    q->r1 = (u64)(((u128)1 << 64) % p);
    q->r2 = pmulmod(q->r1, q->r1, p);
}

void oracle_init(void) {
    if (g_ready) return;
    init_prime(&PR[0], 2485986994308513793ull, 5);   /* src/data.h:79, root :69 */
    init_prime(&PR[1], 1945555039024054273ull, 5);   /* src/data.h:80, root :70 */
    init_prime(&PR[2], 4179340454199820289ull, 3);   /* src/data.h:81, root :71 */
    /* CRT cofactors (src/core.h:78-84): M_i = P / p_i and M_i^-1 mod p_i. */
    for (int i = 0; i < 3; i++) {
        u64 a = PR[(i + 1) % 3].p, b = PR[(i + 2) % 3].p;
        u128 m = (u128)a * b;
        CRT_M[i][0] = (u64)m;
        CRT_M[i][1] = (u64)(m >> 64);
        u64 mmod = (u64)(m % PR[i].p);
        u64 inv = ppow(mmod, PR[i].p - 2, PR[i].p);
        CRT_INV[i] = to_mont(inv, &PR[i]);
    }
    /* P = p1 p2 p3 as three words */
    u128 p12 = (u128)PR[0].p * PR[1].p;
    u128 lo = (u128)(u64)p12 * PR[2].p;
    u128 hi = (u128)(u64)(p12 >> 64) * PR[2].p;
    CRT_P[0] = (u64)lo;
    u128 mid = (lo >> 64) + (u128)(u64)hi;
    CRT_P[1] = (u64)mid;
    CRT_P[2] = (u64)(mid >> 64) + (u64)(hi >> 64);
    g_ready = 1;
}

/* Exported so tests can pin the derived constants against src/data.h and src/core.h. */
void oracle_constants(int i, u64 out[5]) {
    oracle_init();
    out[0] = PR[i].p;
    out[1] = PR[i].ninv;
    out[2] = PR[i].r2;
    out[3] = PR[i].r1;
    out[4] = to_mont(PR[i].g, &PR[i]);
}
void oracle_crt_constants(u64 out[12]) {
    oracle_init();
    for (int i = 0; i < 3; i++) {
        out[2 * i] = CRT_M[i][0];
        out[2 * i + 1] = CRT_M[i][1];
        out[6 + i] = CRT_INV[i];
    }
    out[9] = CRT_P[0];
    out[10] = CRT_P[1];
    out[11] = CRT_P[2];
}

/* ----------------------------------------------------------------------------- NTT */

/* Powers w^0 .. w^(half-1) of the primitive len-th root (or its inverse), Montgomery form. */
static void root_powers(u64* tab, u64 half, u64 len, int inverse, const prime_t* q) {
    u64 e = (q->p - 1) / len;
    if (inverse) e = (q->p - 1) - e;            /* g^(-(p-1)/len) = g^((p-1) - (p-1)/len) */
    u64 w = mpow(to_mont(q->g, q), e, q);
    u64 cur = q->r1;
    for (u64 j = 0; j < half; j++) {
        tab[j] = cur;
        cur = mmul(cur, w, q);
    }
}

/* Forward NTT, decimation in frequency: natural order in, bit-reversed order out
 * (the order src/core.h:443-474 dif leaves behind; only its use by the matching inverse
 * matters). */
static void ntt_dif(u64* a, u64 n, const prime_t* q, u64* tab) {
    for (u64 len = n; len >= 2; len >>= 1) {
        u64 half = len >> 1;
        root_powers(tab, half, len, 0, q);
        for (u64 s = 0; s < n; s += len)
            for (u64 j = 0; j < half; j++) {
                u64 u = a[s + j], v = a[s + j + half];
                a[s + j] = madd(u, v, q);
                a[s + j + half] = mmul(msub(u, v, q), tab[j], q);
            }
    }
}

/* Inverse NTT, decimation in time: bit-reversed in, natural out, unnormalised
 * (src/core.h:476-509 idit). */
static void ntt_dit_inv(u64* a, u64 n, const prime_t* q, u64* tab) {
    for (u64 len = 2; len <= n; len <<= 1) {
        u64 half = len >> 1;
        root_powers(tab, half, len, 1, q);
        for (u64 s = 0; s < n; s += len)
            for (u64 j = 0; j < half; j++) {
                u64 u = a[s + j], v = mmul(a[s + j + half], tab[j], q);
                a[s + j] = madd(u, v, q);
                a[s + j + half] = msub(u, v, q);
            }
    }
}

/* int_ceil2 (src/fast_mul.c:299-306). */
static u64 ceil_pow2(u64 n) {
    u64 r = 1;
    while (r < n) r <<= 1;
    return r;
}

/* Cyclic convolution mod prime i of the limb vectors a (la) and b (lb), length n (a power of
 * two >= la + lb - 1), result in Montgomery form and scaled by n^-1 (conv_rec with norm,
 * src/fast_mul.c:58-70 and 103-119).  b == NULL means square (conv_sqr). */
static int conv_mod(int i, const u64* a, u64 la, const u64* b, u64 lb, u64 n, u64* res) {
    const prime_t* q = &PR[i];
    u64* tb = NULL;
    u64* tab = (u64*)malloc((n / 2 + 1) * sizeof(u64));
    if (!tab) return -1;
    for (u64 k = 0; k < n; k++) res[k] = k < la ? to_mont(a[k], q) : 0;
    ntt_dif(res, n, q, tab);
    if (b) {
        tb = (u64*)malloc(n * sizeof(u64));
        if (!tb) { free(tab); return -1; }
        for (u64 k = 0; k < n; k++) tb[k] = k < lb ? to_mont(b[k], q) : 0;
        ntt_dif(tb, n, q, tab);
    }
    /* ntt_len^-1 in Montgomery form (src/fast_mul.c:59-61) */
    u64 inv_n = mpow(to_mont(n % q->p, q), q->p - 2, q);
    for (u64 k = 0; k < n; k++)
        res[k] = mmul(mmul(res[k], b ? tb[k] : res[k], q), inv_n, q);
    ntt_dit_inv(res, n, q, tab);
    free(tab);
    free(tb);
    return 0;
}

/* crt3 (src/core.h:77-104): three Montgomery residues -> integer in [0, p1 p2 p3). */
static void crt3(u64 r0, u64 r1, u64 r2, u64 out[3]) {
    u64 r[3] = {r0, r1, r2};
    u64 acc[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++) {
        u64 y = from_mont(mmul(r[i], CRT_INV[i], &PR[i]), &PR[i]);   /* y < p_i */
        u128 lo = (u128)y * CRT_M[i][0];
        u128 hi = (u128)y * CRT_M[i][1];
        u64 t0 = (u64)lo;
        u128 mid = (lo >> 64) + (u128)(u64)hi;
        u64 t1 = (u64)mid;
        u64 t2 = (u64)(mid >> 64) + (u64)(hi >> 64);
        /* acc += t (u192, _u192add src/macro.h:171-180) */
        u128 s0 = (u128)acc[0] + t0;
        u128 s1 = (u128)acc[1] + t1 + (u64)(s0 >> 64);
        acc[0] = (u64)s0;
        acc[1] = (u64)s1;
        acc[2] = acc[2] + t2 + (u64)(s1 >> 64);
    }
    for (int rep = 0; rep < 2; rep++) {   /* at most two subtractions (src/core.h:98-103) */
        int ge = acc[2] != CRT_P[2] ? acc[2] > CRT_P[2]
               : acc[1] != CRT_P[1] ? acc[1] > CRT_P[1]
               : acc[0] >= CRT_P[0];
        if (!ge) break;
        u128 d0 = (u128)acc[0] - CRT_P[0];
        u64 b0 = (u64)(d0 >> 64) ? 1 : 0;
        u128 d1 = (u128)acc[1] - CRT_P[1] - b0;
        u64 b1 = (u64)(d1 >> 64) ? 1 : 0;
        acc[0] = (u64)d0;
        acc[1] = (u64)d1;
        acc[2] = acc[2] - CRT_P[2] - b1;
    }
    out[0] = acc[0];
    out[1] = acc[1];
    out[2] = acc[2];
}

static int mul_core(const u64* a, u64 la, const u64* b, u64 lb, u64* out, int sqr) {
    oracle_init();
    u64 out_len = la + lb;
    if (out_len == 0) return 0;
    if (la == 0 || lb == 0) {            /* the product is zero */
        memset(out, 0, out_len * sizeof(u64));
        return 0;
    }
    u64 conv_len = out_len - 1;
    u64 n = ceil_pow2(conv_len);
    u64* res[3];
    for (int i = 0; i < 3; i++) {
        res[i] = (u64*)malloc(n * sizeof(u64));
        if (!res[i] || conv_mod(i, a, la, sqr ? NULL : b, lb, n, res[i])) {
            for (int j = 0; j <= i; j++) free(res[j]);
            return -1;
        }
    }
    /* serial carry loop, src/fast_mul.c:378-389 */
    u64 carry[3] = {0, 0, 0};
    for (u64 k = 0; k < conv_len; k++) {
        u64 c[3];
        crt3(res[0][k], res[1][k], res[2][k], c);
        u128 s0 = (u128)carry[0] + c[0];
        u128 s1 = (u128)carry[1] + c[1] + (u64)(s0 >> 64);
        u64 s2 = carry[2] + c[2] + (u64)(s1 >> 64);
        out[k] = (u64)s0;
        carry[0] = (u64)s1;
        carry[1] = s2;
        carry[2] = 0;
    }
    out[conv_len] = carry[0];
    for (int i = 0; i < 3; i++) free(res[i]);
    return 0;
}

/* abs_mul64 / abs_sqr64 semantics (src/fast_mul.h:39,45); returns 0 on success. */
int oracle_abs_mul64(const u64* a, u64 la, const u64* b, u64 lb, u64* out) {
    return mul_core(a, la, b, lb, out, 0);
}
int oracle_abs_sqr64(const u64* a, u64 la, u64* out) { return mul_core(a, la, a, la, out, 1); }

/* Cyclic convolution residues of prime i in plain (non-Montgomery) form, for debugging
 * per-prime stages of a transform. */
int oracle_conv_residues(int i, const u64* a, u64 la, const u64* b, u64 lb, u64 n, u64* res) {
    oracle_init();
    if (conv_mod(i, a, la, b, lb, n, res)) return -1;
    for (u64 k = 0; k < n; k++) res[k] = from_mont(res[k], &PR[i]);
    return 0;
}

/* Schoolbook product (the pattern of fft_small/fsd_test.c:282-302), out has la + lb limbs. */
void oracle_schoolbook(const u64* a, u64 la, const u64* b, u64 lb, u64* out) {
    memset(out, 0, (la + lb) * sizeof(u64));
    for (u64 i = 0; i < la; i++) {
        u64 c = 0;
        for (u64 j = 0; j < lb; j++) {
            u128 t = (u128)a[i] * b[j] + out[i + j] + c;
            out[i + j] = (u64)t;
            c = (u64)(t >> 64);
        }
        out[i + lb] = c;
    }
}

/* x mod m for a little-endian limb vector (Horner, most significant limb first).  Used for
 * size-independent checks: (A mod m)(B mod m) == (A*B mod m) (mod m). */
u64 oracle_mod(const u64* x, u64 len, u64 m) {
    u64 r = 0;
    u64 b = (u64)(((u128)1 << 64) % m);
    for (u64 k = len; k-- > 0;) r = (u64)(((u128)r * b + x[k] % m) % m);
    return r;
}
