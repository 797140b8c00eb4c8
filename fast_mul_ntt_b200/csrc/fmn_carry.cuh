// fmn_carry.cuh -- the carry scan shared by both residue engines' CRT kernels.
//
// After CRT each output limb j has a sum s_j < 4 * 2^64 (kept as a low word and a 2-bit high
// part) to which the carry from limb j-1 must be added; the reference does this with a
// serial loop (src/fast_mul.c:378-389).  A span of limbs maps its incoming carry to its
// outgoing carry by a function {0..3} -> {0..3} (packed as 4 x 2 bits); these compose
// associatively, which gives a parallel scan: per-thread functions, a CTA scan, and a
// decoupled look-back across CTAs in the order CTAs obtain tickets.
#pragma once
#include <stdint.h>

#include "fmn_arith.cuh"

namespace fmn {

constexpr int CNT = 256;           // threads per CTA
constexpr int CE = 16;             // limbs per thread
constexpr int CTILE = CNT * CE;    // limbs per CTA
constexpr u32 ID_FN = 0xE4;        // identity map
constexpr u32 ST_AGG = 1u << 8, ST_PRE = 2u << 8;
constexpr long SPIN_LIMIT = 1l << 22;   // bounded waits: ~ seconds at most, then error flag

__device__ __forceinline__ u32 fn_apply(u32 f, u32 c) { return (f >> (2 * c)) & 3u; }
__device__ __forceinline__ u32 fn_compose(u32 later, u32 earlier) {   // later o earlier
    u32 r = 0;
#pragma unroll
    for (u32 c = 0; c < 4; ++c) r |= fn_apply(later, fn_apply(earlier, c)) << (2 * c);
    return r;
}

// Adds x to the limb sum (lo, h): lo += x, carry into the 2-bit high part.
__device__ __forceinline__ void add_to(u64& lo, u32& h, u64 x) {
    lo += x;
    h += lo < x;
}

// The CTA's ticket (the order in which CTAs start, which is the order of the scan).
__device__ __forceinline__ u32 carry_ticket(u32* ticket) {
    __shared__ u32 s_tile;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    return s_tile;
}

// Completes the scan for limbs j0 .. j0+NE-1 of this thread (CTA `tile` of CNT * NE limbs,
// sums lo/h with the contributions from lower limbs already added) and stores the final limbs.
// `state` holds one word per CTA (zeroed before the first launch); a look-back that polls a
// predecessor's word more than LIMIT times gives up, takes its carry as 0 and sets *err.
template <int NE, long LIMIT = SPIN_LIMIT>
__device__ __forceinline__ void carry_finish(u64 (&lo)[NE], u32 (&h)[NE], u64 tile, u64 j0, u32* state, u32* err,
                                             u64* out, u64 out_len) {
    __shared__ u32 s_warp[CNT / 32];
    __shared__ u32 s_cin;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    // carry-transfer function of this thread's limbs.  The carry out is non-decreasing in the
    // carry in and moves by at most one over 0..3, so it is constant when the chains from 0 and
    // from 3 agree; the chains from 1 and 2 run only in warps where some lane needs them.
    auto chain = [&](u64 c) {
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const u64 t = lo[e] + c;
            c = h[e] + (t < c);
        }
        return (u32)c;
    };
    const u32 c0 = chain(0), c3 = chain(3);
    u32 c1 = c0, c2 = c0;
    if (__any_sync(0xffffffffu, c0 != c3)) {
        c1 = chain(1);
        c2 = chain(2);
    }
    const u32 f = c0 | (c1 << 2) | (c2 << 4) | (c3 << 6);
    // CTA scan: Kogge-Stone in each warp, then over the warps in warp 0
    u32 inc = f;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const u32 o = __shfl_up_sync(0xffffffffu, inc, d);
        if (lane >= d) inc = fn_compose(inc, o);
    }
    u32 exc = __shfl_up_sync(0xffffffffu, inc, 1);
    if (lane == 0) exc = ID_FN;
    if (lane == 31) s_warp[warp] = inc;
    __syncthreads();
    if (warp == 0) {
        u32 wt = lane < CNT / 32 ? s_warp[lane] : ID_FN;
#pragma unroll
        for (int d = 1; d < CNT / 32; d <<= 1) {
            const u32 o = __shfl_up_sync(0xffffffffu, wt, d);
            if (lane >= d) wt = fn_compose(wt, o);
        }
        u32 wex = __shfl_up_sync(0xffffffffu, wt, 1);
        if (lane == 0) wex = ID_FN;
        const u32 agg = __shfl_sync(0xffffffffu, wt, CNT / 32 - 1);
        if (lane < CNT / 32) s_warp[lane] = wex;       // exclusive prefix of each warp
        u32 cin = 0;
        if (tile == 0) {
            if (lane == 0) atomicExch(&state[0], ST_PRE | fn_apply(agg, 0));
        } else {
            if (lane == 0) atomicExch(&state[tile], ST_AGG | agg);
            // warp-parallel look-back over the 32 nearest predecessors at a time
            volatile u32* st = state;
            u32 acc = ID_FN;
            long base = (long)tile - 1;
            bool failed = false;
            while (true) {
                const long p = base - lane;
                u32 v = ST_PRE;                         // before the first CTA: carry 0
                if (p >= 0) {
                    long spins = 0;
                    v = st[p];
                    while (v == 0) {
                        if (++spins > LIMIT) {
                            failed = true;
                            v = ST_PRE;
                            break;
                        }
                        __nanosleep(64);
                        v = st[p];
                    }
                }
                const unsigned pre = __ballot_sync(0xffffffffu, (v & ST_PRE) != 0);
                const int first = pre ? __ffs(pre) - 1 : 32;
                // compose the aggregates of lanes 0 .. first-1 (nearest first)
                u32 fl = (lane < first) ? (v & 0xff) : ID_FN;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const u32 o = __shfl_down_sync(0xffffffffu, fl, d);
                    if ((lane & (2 * d - 1)) == 0 && lane + d < 32) fl = fn_compose(fl, o);
                }
                fl = __shfl_sync(0xffffffffu, fl, 0);
                acc = fn_compose(acc, fl);
                if (pre) {
                    const u32 pv = __shfl_sync(0xffffffffu, v, first) & 0xff;
                    cin = fn_apply(acc, pv);
                    break;
                }
                base -= 32;
            }
            if (__any_sync(0xffffffffu, failed) && lane == 0) atomicOr(err, 1u);
            if (lane == 0) atomicExch(&state[tile], ST_PRE | fn_apply(agg, cin));
        }
        if (lane == 0) s_cin = cin;
    }
    __syncthreads();
    u64 c = fn_apply(exc, fn_apply(s_warp[warp], s_cin));
    u64 outv[NE];
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const u64 t = lo[e] + c;
        c = h[e] + (t < c);
        outv[e] = t;
    }
    if (j0 + NE <= out_len && ((reinterpret_cast<uintptr_t>(out) & 15) == 0)) {
#pragma unroll
        for (int e = 0; e < NE; e += 2)
            *reinterpret_cast<ulonglong2*>(out + j0 + e) = make_ulonglong2(outv[e], outv[e + 1]);
    } else {
#pragma unroll
        for (int e = 0; e < NE; ++e)
            if (j0 + e < out_len) out[j0 + e] = outv[e];
    }
}

}  // namespace fmn
