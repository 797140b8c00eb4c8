// fmn_arith.cuh -- modular arithmetic for the three NTT primes on sm_100a.
//
// The primes are those of the reference (src/data.h:79-81).  Each has the form
// p = c * 2^k + 1 with a small c:
//     p0 = 69 * 2^55 + 1,  p1 = 27 * 2^56 + 1,  p2 = 29 * 2^57 + 1.
// Residues are plain representatives (lazily reduced); the reference keeps them in
// Montgomery form with R = 2^64 (_mont_mul, src/macro.h:160-169).  Butterflies multiply by
// constant twiddles with Shoup's method (smul); products of two variables use Montgomery
// REDC with R = 2^64 (mmul), whose 2^-64 factors are folded into the CRT constants.  The
// reduction below is Montgomery REDC
// specialised to that form:
//   * p^-1 mod 2^64 = 1 - c * 2^k, so  m = T_lo * p^-1  changes only the high 32-bit
//     word of T_lo: one 32-bit multiply-add;
//   * m * p = m + (c * m) << k, so the high 64 bits of m * p are
//     (c * m + (m >> k)) >> (64 - k): two 32x32->64 multiply-adds and two shifts;
//   * t = T_hi - (m * p)_hi lies in (-p, p) when T < p * 2^64; we return t + p in (0, 2p).
//
// The prime is a runtime value held in uniform registers (struct PrimeRT), so one code body
// serves all three primes: kernels are a third of the size they would be with the prime as
// a template parameter, which keeps them inside the instruction cache.  Integer multiplies
// issue only on the FMA-heavy pipe (wide forms at half rate); this formulation was the
// fastest of the ones measured on B200 (64x64 product through mul.lo/mul.hi.u64).
//
// Lazy-reduction contract used by every kernel:
//   mmul(a, b) needs a * b < p * 2^64; it holds for a, b < 2p, and for a < 4p with b < p
//   (4p^2 < p * 2^64 because 4p < 2^64 for all three primes), and for any a < 2^64 with
//   b < p.  The result is in (0, 2p).
#pragma once
#include <stdint.h>

typedef unsigned long long u64;
typedef unsigned int u32;

namespace fmn {

constexpr u64 mulmod_c(u64 a, u64 b, u64 m) { return (u64)(((unsigned __int128)a * b) % m); }
constexpr u64 rmod_c(u64 p) { return (u64)((((unsigned __int128)1) << 64) % p); }

template <int I> struct Prime;
template <> struct Prime<0> {
    static constexpr u64 P = 2485986994308513793ull;
    static constexpr u32 C = 69;
    static constexpr int K = 55;
};
template <> struct Prime<1> {
    static constexpr u64 P = 1945555039024054273ull;
    static constexpr u32 C = 27;
    static constexpr int K = 56;
};
template <> struct Prime<2> {
    static constexpr u64 P = 4179340454199820289ull;
    static constexpr u32 C = 29;
    static constexpr int K = 57;
};

// Runtime descriptor of one prime.
struct PrimeRT {
    u64 p;       // the prime
    u64 p2;      // 2p
    u64 r2;      // R^2 mod p (to-Montgomery factor)
    u32 c;       // p = c * 2^k + 1
    u32 csh;     // c * 2^(k-32) (fits 32 bits)
    u32 k32;     // k - 32
    u32 k64;     // 64 - k
    u64 r64;     // floor(2^64 / p): Shoup companion of 1 (reduces any u64 below 2p)
};

template <int I>
constexpr PrimeRT prime_rt() {
    return PrimeRT{Prime<I>::P, 2 * Prime<I>::P, mulmod_c(rmod_c(Prime<I>::P), rmod_c(Prime<I>::P), Prime<I>::P),
                   Prime<I>::C, Prime<I>::C << (Prime<I>::K - 32), (u32)(Prime<I>::K - 32),
                   (u32)(64 - Prime<I>::K), (u64)((((unsigned __int128)1) << 64) / Prime<I>::P)};
}
static_assert(Prime<0>::P == (((u64)Prime<0>::C) << Prime<0>::K) + 1, "prime form");
static_assert(Prime<1>::P == (((u64)Prime<1>::C) << Prime<1>::K) + 1, "prime form");
static_assert(Prime<2>::P == (((u64)Prime<2>::C) << Prime<2>::K) + 1, "prime form");

// Montgomery product a * b * 2^-64 mod p, lazily reduced to (0, 2p).
__device__ __forceinline__ u64 mmul(u64 a, u64 b, const PrimeRT& q) {
    const u64 lo = a * b;
    const u64 hi = __umul64hi(a, b);
    const u32 t0 = (u32)lo, t1 = (u32)(lo >> 32);
    const u32 m1 = t1 - t0 * q.csh;                  // m = T_lo * p^-1 = (m1 : t0)
    const u32 mh = m1 >> q.k32;                      // m >> k
    const u64 x0 = (u64)q.c * t0 + mh;
    const u64 y = (u64)q.c * m1 + (x0 >> 32);
    const u64 mphi = (y << q.k32) | ((u32)x0 >> q.k64);   // (m * p) >> 64
    return hi + q.p - mphi;
}

// Shoup product x * w mod p (plain representatives) with w' = floor(w * 2^64 / p)
// precomputed: any x < 2^64 and w < p give a result in [0, 2p).  The quotient estimate is the
// high word of x * w'; q * p mod 2^64 is cheap because p = c * 2^k + 1.  As a butterfly
// multiply it measured about 30% faster than the Montgomery product on B200.
__device__ __forceinline__ u64 smul(u64 x, u64 w, u64 wp, const PrimeRT& q) {
    const u64 qq = __umul64hi(x, wp);
    const u64 qp = qq + ((u64)((u32)qq * q.csh) << 32);   // qq * p mod 2^64
    return x * w - qp;
}

// x in [0, 4p) -> [0, 2p)
__device__ __forceinline__ u64 red2(u64 x, const PrimeRT& q) {
    const u64 t = x - q.p2;
    return t < x ? t : x;   // x >= 2p  <=>  no wrap-around
}
// x in [0, 2p) -> [0, p)
__device__ __forceinline__ u64 red1(u64 x, const PrimeRT& q) {
    const u64 t = x - q.p;
    return t < x ? t : x;
}

// Decimation-in-frequency butterfly with twiddle (w, w'), w < p:
//   u, v in [0, 2p)  ->  u' = u + v in [0, 2p),  v' = (u - v) * w in [0, 2p).
__device__ __forceinline__ void bfly_dif(u64& u, u64& v, ulonglong2 w, const PrimeRT& q) {
    const u64 s = u + v;
    const u64 d = u + q.p2 - v;
    u = red2(s, q);
    v = smul(d, w.x, w.y, q);
}
// Same with twiddle 1.
__device__ __forceinline__ void bfly_dif1(u64& u, u64& v, const PrimeRT& q) {
    const u64 s = u + v;
    const u64 d = u + q.p2 - v;
    u = red2(s, q);
    v = red2(d, q);
}
// Decimation-in-time butterfly with twiddle (w, w'), w < p:
//   u, v in [0, 4p)  ->  u' = u + v*w, v' = u - v*w, both in [0, 4p).
__device__ __forceinline__ void bfly_dit(u64& u, u64& v, ulonglong2 w, const PrimeRT& q) {
    const u64 a = red2(u, q);
    const u64 b = smul(v, w.x, w.y, q);
    u = a + b;
    v = a + q.p2 - b;
}
// Same with twiddle 1.
__device__ __forceinline__ void bfly_dit1(u64& u, u64& v, const PrimeRT& q) {
    const u64 a = red2(u, q);
    const u64 b = red2(v, q);
    u = a + b;
    v = a + q.p2 - b;
}

}  // namespace fmn
