// fmn_arith32.cuh -- modular arithmetic of the 32-bit residue engine on sm_100a.
//
// The reference transforms 64-bit limbs modulo three 62-bit primes (src/data.h:79-81); on a
// GPU every 64 x 64-bit product is a chain of 32-bit multiplies on the FMA-heavy pipe, so a
// 64-bit modular product costs about five times a 32-bit one.  This engine instead splits
// every limb into two 32-bit digits and transforms them modulo three primes below 2^31:
//     q0 = 15 * 2^27 + 1 = 2013265921,  q1 = 27 * 2^26 + 1 = 1811939329,
//     q2 =  7 * 2^26 + 1 =  469762049.
// Their product Q ~ 2^90.47 bounds every coefficient of a convolution of n-digit sequences
// by n * (2^32 - 1)^2 < Q for n <= 2^26, so transforms of up to 2^26 points (products of up
// to 2^25 output limbs) are exact; the result is the same integer product, limb for limb.
//
// Residues are kept fully reduced in [0, q) (q < 2^31, so u + v and u - v + q fit in 32
// bits).  Constant twiddles multiply by Shoup's method with precomputed w' = floor(w 2^32 / q):
// one high product and two low products.  Products of two variables (the pointwise product,
// on-the-fly four-step twiddles) use Montgomery reduction with R = 2^32; the 2^-32 factors
// are folded into the CRT constants.
#pragma once
#include <stdint.h>

#include "fmn_arith.cuh"

namespace fmn {

struct PrimeQ {
    u32 p;      // the prime, < 2^31
    u32 pinv;   // p^-1 mod 2^32
    u32 one;    // floor(2^32 / p): Shoup companion of 1
    u32 r1;     // 2^32 mod p (Montgomery form of 1)
};

constexpr u32 Q32_P0 = 2013265921u, Q32_P1 = 1811939329u, Q32_P2 = 469762049u;
constexpr int Q32_MAX_LOG_N = 26;    // 2-adic order of q1 and q2

constexpr u32 inv32_c(u32 p) {       // Newton iteration for p^-1 mod 2^32 (p odd)
    u32 x = p;                        // correct to 3 bits
    for (int i = 0; i < 5; ++i) x *= 2u - p * x;
    return x;
}
constexpr PrimeQ prime_q(u32 p) {
    return PrimeQ{p, inv32_c(p), (u32)((1ull << 32) / p), (u32)((1ull << 32) % p)};
}
static_assert(inv32_c(Q32_P0) * Q32_P0 == 1u && inv32_c(Q32_P1) * Q32_P1 == 1u && inv32_c(Q32_P2) * Q32_P2 == 1u,
              "inverse mod 2^32");
static_assert(Q32_P0 == 15u * (1u << 27) + 1u && Q32_P1 == 27u * (1u << 26) + 1u && Q32_P2 == 7u * (1u << 26) + 1u,
              "prime form");

__device__ __forceinline__ u32 umin32(u32 a, u32 b) { return a < b ? a : b; }

// u, v in [0, p) -> (u + v) mod p
__device__ __forceinline__ u32 qadd(u32 u, u32 v, const PrimeQ& q) {
    const u32 s = u + v;
    return umin32(s, s - q.p);
}
// u, v in [0, p) -> (u - v) mod p
__device__ __forceinline__ u32 qsub(u32 u, u32 v, const PrimeQ& q) {
    const u32 d = u + q.p - v;
    return umin32(d, d - q.p);
}
// x * w mod p for any x < 2^32 and w < p with wp = floor(w 2^32 / p): result in [0, p).
__device__ __forceinline__ u32 qsmul(u32 x, u32 w, u32 wp, const PrimeQ& q) {
    const u32 hq = __umulhi(x, wp);
    const u32 r = x * w - hq * q.p;     // in [0, 2p)
    return umin32(r, r - q.p);
}
// Montgomery product a * b * 2^-32 mod p for a * b < p 2^32: result in [0, p).  hi - mh lies
// in (-p, p); as a u32 it is either the result (< p) or the result - p wrapped above 2^32 - p,
// and min(r, r + p) picks the reduced one in both cases.
__device__ __forceinline__ u32 qmont(u32 a, u32 b, const PrimeQ& q) {
    const u64 t = (u64)a * b;
    const u32 m = (u32)t * q.pinv;                // t - m p = 0 mod 2^32
    const u32 r = (u32)(t >> 32) - __umulhi(m, q.p);
    return umin32(r, r + q.p);
}

// Decimation-in-frequency butterfly with Shoup twiddle (w, w'): (u + v, (u - v) w).
__device__ __forceinline__ void qbfly_dif(u32& u, u32& v, uint2 w, const PrimeQ& q) {
    const u32 s = qadd(u, v, q);
    v = qsmul(u + q.p - v, w.x, w.y, q);
    u = s;
}
__device__ __forceinline__ void qbfly_dif1(u32& u, u32& v, const PrimeQ& q) {
    const u32 s = qadd(u, v, q);
    v = qsub(u, v, q);
    u = s;
}
// Decimation-in-time butterfly with Shoup twiddle (w, w'): (u + v w, u - v w).
__device__ __forceinline__ void qbfly_dit(u32& u, u32& v, uint2 w, const PrimeQ& q) {
    const u32 b = qsmul(v, w.x, w.y, q);
    v = qsub(u, b, q);
    u = qadd(u, b, q);
}
__device__ __forceinline__ void qbfly_dit1(u32& u, u32& v, const PrimeQ& q) {
    const u32 s = qadd(u, v, q);
    v = qsub(u, v, q);
    u = s;
}

}  // namespace fmn
