// fmn_arith.cuh -- modular arithmetic for the three NTT primes on sm_100a.
//
// The primes are those of the reference (src/data.h:79-81).  Each has the form
// p = c * 2^k + 1 with a small c:
//     p0 = 69 * 2^55 + 1,  p1 = 27 * 2^56 + 1,  p2 = 29 * 2^57 + 1.
// Residues are kept in Montgomery form with R = 2^64, as in the reference
// (_mont_mul, src/macro.h:160-169).  The reduction below is Montgomery REDC
// specialised to that form:
//   * p^-1 mod 2^64 = 1 - c * 2^k, so  m = T_lo * p^-1  changes only the high 32-bit
//     word of T_lo: one 32-bit multiply-add;
//   * m * p = m + (c * m) << k, so the high 64 bits of m * p are
//     (c * m + (m >> k)) >> (64 - k): two 32x32->64 multiply-adds and two shifts;
//   * t = T_hi - (m * p)_hi lies in (-p, p) when T < p * 2^64; we return t + p in (0, 2p).
// The 64x64->128 product itself is four 32x32->64 mad.wide operations.
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

template <int I> struct PrimeX : Prime<I> {
    using B = Prime<I>;
    static constexpr u64 P2 = 2 * B::P;
    static constexpr u64 R1 = rmod_c(B::P);                 // Montgomery one
    static constexpr u64 R2 = mulmod_c(R1, R1, B::P);        // R^2 mod p (to-Montgomery factor)
    static constexpr u32 CSH = B::C << (B::K - 32);          // c * 2^(k-32), fits 32 bits
    static_assert((u64)B::P == (((u64)B::C) << B::K) + 1, "prime form");
    static_assert(B::K >= 55 && B::K < 64, "shift ranges");
};

// 64x64 -> 128 product from 32-bit pieces (mad.wide.u32 chains).
__device__ __forceinline__ void mul_wide(u64 a, u64 b, u32& t0, u32& t1, u64& hi) {
    const u32 a0 = (u32)a, a1 = (u32)(a >> 32), b0 = (u32)b, b1 = (u32)(b >> 32);
    const u64 p00 = (u64)a0 * b0;
    const u64 p01 = (u64)a0 * b1 + (p00 >> 32);
    const u64 p10 = (u64)a1 * b0 + (u32)p01;
    hi = (u64)a1 * b1 + (p01 >> 32) + (p10 >> 32);
    t0 = (u32)p00;
    t1 = (u32)p10;
}

// REDC of T = (hi : t1 : t0) for p = c*2^k+1; needs T < p * 2^64; result in (0, 2p).
template <int I>
__device__ __forceinline__ u64 redc(u32 t0, u32 t1, u64 hi) {
    using Q = PrimeX<I>;
    const u32 m1 = t1 - t0 * Q::CSH;                          // m = (m1 : t0)
    const u32 mh = m1 >> (Q::K - 32);                         // m >> k
    const u64 x0 = (u64)Q::C * t0 + mh;
    const u64 y = (u64)Q::C * m1 + (x0 >> 32);
    const u64 mphi = (y << (Q::K - 32)) | ((u32)x0 >> (64 - Q::K));   // (m * p) >> 64
    return hi + Q::P - mphi;
}

// Montgomery product a * b * 2^-64 mod p, lazily reduced to (0, 2p).
template <int I>
__device__ __forceinline__ u64 mmul(u64 a, u64 b) {
    u32 t0, t1;
    u64 hi;
    mul_wide(a, b, t0, t1, hi);
    return redc<I>(t0, t1, hi);
}

// x in [0, 4p) -> [0, 2p)
template <int I>
__device__ __forceinline__ u64 red2(u64 x) {
    const u64 t = x - PrimeX<I>::P2;
    return t < x ? t : x;   // x >= 2p  <=>  no wrap-around
}
// x in [0, 2p) -> [0, p)
template <int I>
__device__ __forceinline__ u64 red1(u64 x) {
    const u64 t = x - Prime<I>::P;
    return t < x ? t : x;
}

// Decimation-in-frequency butterfly with twiddle w < p (or w < 2p):
//   u, v in [0, 2p)  ->  u' = u + v in [0, 2p),  v' = (u - v) * w in (0, 2p).
template <int I>
__device__ __forceinline__ void bfly_dif(u64& u, u64& v, u64 w) {
    const u64 s = u + v;
    const u64 d = u + PrimeX<I>::P2 - v;
    u = red2<I>(s);
    v = mmul<I>(d, w);
}
// Same with twiddle 1.
template <int I>
__device__ __forceinline__ void bfly_dif1(u64& u, u64& v) {
    const u64 s = u + v;
    const u64 d = u + PrimeX<I>::P2 - v;
    u = red2<I>(s);
    v = red2<I>(d);
}
// Decimation-in-time butterfly with twiddle w < p:
//   u, v in [0, 4p)  ->  u' = u + v*w, v' = u - v*w, both in [0, 4p).
template <int I>
__device__ __forceinline__ void bfly_dit(u64& u, u64& v, u64 w) {
    const u64 a = red2<I>(u);
    const u64 b = mmul<I>(v, w);
    u = a + b;
    v = a + PrimeX<I>::P2 - b;
}
// Same with twiddle 1.
template <int I>
__device__ __forceinline__ void bfly_dit1(u64& u, u64& v) {
    const u64 a = red2<I>(u);
    const u64 b = red2<I>(v);
    u = a + b;
    v = a + PrimeX<I>::P2 - b;
}

}  // namespace fmn
