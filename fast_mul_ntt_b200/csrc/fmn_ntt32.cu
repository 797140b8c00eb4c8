// fmn_ntt32.cu -- the 32-bit residue engine: sm_100a kernels and launchers for products
// whose transform over 32-bit digits has at most 2^26 points (up to 2^25 output limbs).
//
// The pipeline is the one of the 64-bit engine (fmn_ntt.cu, reference src/fast_mul.c:308-460):
// entry fused into the first forward pass, four-step passes of <= 2^9 points per CTA, the
// pointwise product fused between the last forward and the first inverse pass, CRT fused
// with the carry scan.  What differs is the residue arithmetic (fmn_arith32.cuh): each
// 64-bit limb enters as two 32-bit digits (little-endian, digit g is 32-bit word g of the
// limb array) and residues are u32 modulo three primes below 2^31, whose products are
// single 32 x 32-bit multiplies instead of 64-bit chains.  The integer product that comes
// out is the same, limb for limb.
//
// Data layout: per operand three residue arrays of N u32 (prime-major).  A strided pass
// views a block of B = 2^logB digits as a [2^m][B / 2^m] row-major matrix; a CTA takes 32
// adjacent columns (a 128-byte stretch of each row) and transforms every column in shared
// memory.  Its tile is dense (row pitch 32 words) and arrives by asynchronous 16-byte copies
// while the CTA computes its four-step twiddle factors, so no thread waits on a global load
// inside the rounds.  Contiguous passes (32 blocks of 2^m digits, one per tile column) store
// element (row j, column c) at j * 33 + c: the padding word keeps both the row-wise and the
// column-wise rounds free of bank conflicts.  Their results leave through the tile, row by
// row, as 128-byte stores, and the fused pass copies the other operand's tile in while its
// forward rounds run.  The offsets of a group's elements are compile-time steps from one
// base.  Indices within one prime's residue array are 32-bit (N <= 2^26).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <vector>

#include "fmn_arith32.cuh"
#include "fmn_carry.cuh"
#include "fmn_internal.h"
#include "fmn_rounds.cuh"

namespace fmn {
namespace q32 {

constexpr int NT = 256;                 // threads per CTA, NTT passes
constexpr int LOG_TC = 5;
constexpr int TC = 1 << LOG_TC;         // columns per tile
constexpr int QTWB = 13;                // two-level root tables: w^x = HI[x >> 13] * LO[x & 8191]
constexpr u32 MASK_N = (1u << Q32_MAX_LOG_N) - 1;
static_assert(2 * QTWB == Q32_MAX_LOG_N, "two-level table covers roots of order 2^26");

// [forward/inverse][prime]: (w, w') Shoup pairs, stored stage-major: the twiddle of stage
// entry j of the group with low offset q is at rt_off(RB, TOP) + j * 2^(TOP-RB+1) + q.
__device__ __align__(16) uint2 g_qrt[2][3][RT_SIZE];
__device__ __align__(16) u32 g_qtw[2][3][1 << QTWB];   // [low/high level][prime], Montgomery form
__constant__ PrimeQ c_q[3] = {prime_q(Q32_P0), prime_q(Q32_P1), prime_q(Q32_P2)};

// Montgomery product a * b * 2^-32 mod p left in (0, 2p) (a, b < p); the result may be the
// second factor of qmont, whose bound a * b < p * 2^32 still holds.
__device__ __forceinline__ u32 qmont_lazy(u32 a, u32 b, const PrimeQ& q) {
    const u64 t = (u64)a * b;
    const u32 m = (u32)t * q.pinv;
    return (u32)(t >> 32) + q.p - __umulhi(m, q.p);
}

// Montgomery form of w_{2^26}^x, prime index pi.
__device__ __forceinline__ u32 qroot(u32 x, int pi, const PrimeQ& q) {
    return qmont(__ldg(&g_qtw[1][pi][x >> QTWB]), __ldg(&g_qtw[0][pi][x & ((1u << QTWB) - 1)]), q);
}

constexpr int TP = TC + 1;              // padded row pitch of a shared-memory tile (words)
// Element (row j, column c) of a 2^LOGL-row tile sits at j * 33 + c', c' a permutation of the
// columns within the row.  Rounds with a thread per column (lanes on the 32 columns of a row)
// are conflict-free for any permutation.  The first round of a contiguous pass puts the lanes
// of a warp on G consecutive rows of 32 / G adjacent columns (G = 2^LOGL over its radix), so
// those columns must start G banks apart: c' rotates c right by log2(32 / G) bits (for LOGL
// 5..8; 2-way conflicts on every access of that round with a fixed swizzle).  Other sizes
// keep c ^ 16 (c & 1), which also suits the row-wise copy-out of tiles of < 32 rows.
template <int LOGL>
__device__ __forceinline__ int tix(int j, int c) {
    if constexpr (LOGL >= 5 && LOGL <= 8) {
        constexpr int G = (1 << LOGL) >> round_bits(LOGL, 0);
        constexpr int w = G >= 32 ? 0 : (G == 16 ? 1 : G == 8 ? 2 : G == 4 ? 3 : G == 2 ? 4 : 5);
        static_assert(G >= 2 && G <= 16, "first-round groups per column");
        return j * TP + (((c >> w) | (c << (5 - w))) & (TC - 1));
    } else {
        return j * TP + (c ^ ((c & 1) << 4));
    }
}
// Dense tiles (row pitch 32 words, rows 16-byte aligned) for strided passes, whose rounds all
// run with the 32 lanes of a warp on the 32 columns of one row: conflict-free without
// padding, and each row is a 128-byte copy target.
__device__ __forceinline__ int dix(int j, int c) { return j * TC + c; }

// 16-byte asynchronous copy global -> shared (no registers held while it is in flight).
__device__ __forceinline__ void cp_async16(u32* sdst, const u32* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_commit_wait() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;\n" ::: "memory");
}
// Rows 0 .. L-1 of a strided tile (32 words each, row r at g + r * 2^logS) into a dense tile,
// by 16-byte asynchronous copies from every thread.
template <int L>
__device__ __forceinline__ void stage_tile(u32* sm, const u32* __restrict__ g, int logS) {
#pragma unroll 4
    for (int e = threadIdx.x; e < L * (TC / 4); e += NT) {
        const int r = e / (TC / 4), k = e % (TC / 4);
        cp_async16(sm + r * TC + 4 * k, g + ((u32)r << logS) + 4 * k);
    }
}

enum { M_FWD = 0, M_FWD_LAST = 1, M_FUSED = 2, M_INV = 3, M_FUSED2 = 4, M_INV_ACC = 5 };

struct QArgs {
    const u64* src;   // ENTRY: limbs of the operand being transformed
    u64 len;          // ENTRY: number of limbs (2 * len digits)
    u32* data;        // residue arrays of the operand being transformed
    u32* other;       // M_FUSED / M_FUSED2: the other operand's spectrum; the product goes here
    u32* dst;         // M_FUSED: where the product goes when `other` must stay intact (else null)
    u64 N;            // transform length (digits)
    int logB;         // log2 block length of this pass
    int ncols;        // contiguous passes: number of blocks (columns) in a tile, <= 32
    // M_INV_ACC (the last inverse pass of one piece of a split product): coefficient i < acc_valid
    // of this piece goes to acc[prime * acc_stride + i], added mod q where i < acc_fresh (the
    // overlap with the previous piece) and stored elsewhere.
    u32* acc;
    u64 acc_stride;
    u64 acc_valid;
    u64 acc_fresh;
    // strided passes: the four-step twiddles of this pass as Shoup pairs, [prime][k][i] with
    // 2^logB entries per prime (frequency k of the column transform, column i), or null to
    // compute them from the root tables
    const uint2* tw;
};

// ------------------------------------------------------------------ one round
// Runs all radix-2^RB groups of one round; see fmn_ntt.cu for the index scheme (identical).
template <int LOGL, int RB, int TOP, bool INV, bool QFAST, bool GST = false, bool GLD = false, class LD, class ST>
__device__ __forceinline__ void run_round(LD ld, ST st, int pi, const PrimeQ& q) {
    constexpr int L = 1 << LOGL, R = 1 << RB, SPL = TOP - RB + 1, SP = 1 << SPL;
    constexpr int GPC = L / R;
    constexpr int G = GPC * TC;
    constexpr bool LOWEST = (SPL == 0);
    const uint2* tab = &g_qrt[INV ? 1 : 0][pi][rt_off(RB, TOP)];
#pragma unroll 1
    for (int gi = threadIdx.x; gi < G; gi += NT) {
        int c, g;
        if (QFAST) {
            g = gi % GPC;
            c = gi / GPC;
        } else {
            c = gi & (TC - 1);
            g = gi >> LOG_TC;
        }
        const int qlo = g & (SP - 1);
        const int row0 = qlo + ((g >> SPL) << (TOP + 1));
        u32 x[R];
        if constexpr (GLD) {
            ld(row0, c, x);
        } else {
#pragma unroll
            for (int t = 0; t < R; ++t) x[t] = ld(row0 + t * SP, c);
        }
        const uint2* tw = tab + qlo;       // stage-major table: lanes of consecutive groups coalesce
        if (!INV) {
#pragma unroll
            for (int s = 0; s < RB; ++s) {
                const int half = R >> (s + 1);
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    if (t & half) continue;
                    const int u = t & (half - 1);
                    if (LOWEST && u == 0)
                        qbfly_dif1(x[t], x[t + half], q);
                    else
                        qbfly_dif(x[t], x[t + half], __ldg(tw + ((R - (R >> s)) + u) * SP), q);
                }
            }
        } else {
#pragma unroll
            for (int s = RB - 1; s >= 0; --s) {
                const int half = R >> (s + 1);
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    if (t & half) continue;
                    const int u = t & (half - 1);
                    if (LOWEST && u == 0)
                        qbfly_dit1(x[t], x[t + half], q);
                    else
                        qbfly_dit(x[t], x[t + half], __ldg(tw + ((R - (R >> s)) + u) * SP), q);
                }
            }
        }
        if constexpr (GST) {
            st(row0, c, x);
        } else {
#pragma unroll
            for (int t = 0; t < R; ++t) st(row0 + t * SP, c, x[t]);
        }
    }
}

// R consecutive u32 (aligned to 4R bytes) with vector loads.
template <int R>
__device__ __forceinline__ void ld_vec(const u32* p, u32 (&x)[R]) {
    if constexpr (R == 1) {
        x[0] = p[0];
    } else if constexpr (R == 2) {
        const uint2 v = *reinterpret_cast<const uint2*>(p);
        x[0] = v.x;
        x[1] = v.y;
    } else {
#pragma unroll
        for (int t = 0; t < R; t += 4) {
            const uint4 v = *reinterpret_cast<const uint4*>(p + t);
            x[t] = v.x;
            x[t + 1] = v.y;
            x[t + 2] = v.z;
            x[t + 3] = v.w;
        }
    }
}

// Rounds IDX.. of a sub-transform (forward: round 0 holds the top bits; inverse round k
// undoes forward round NR-1-k).  The first round reads with `ld0`, the last writes with
// `stl`, the rest go through shared memory.
template <int LOGL, bool INV, bool CONTIG, int IDX, bool GST = false, bool GLD = false, bool DENSE = false, class LD0,
          class STL>
__device__ __forceinline__ void rounds(u32* sm, LD0 ld0, STL stl, int pi, const PrimeQ& q) {
    constexpr int NR = rounds_count(LOGL);
    constexpr int FR = INV ? NR - 1 - IDX : IDX;
    constexpr int RB = round_bits(LOGL, FR), TOP = round_top(LOGL, FR);
    constexpr bool QF = CONTIG && (TOP == LOGL - 1);
    static_assert(!(DENSE && CONTIG), "dense tiles serve strided passes only");
    auto lds = [sm](int j, int c) { return sm[DENSE ? dix(j, c) : tix<LOGL>(j, c)]; };
    auto sts = [sm](int j, int c, u32 v) { sm[DENSE ? dix(j, c) : tix<LOGL>(j, c)] = v; };
    if constexpr (NR == 1) {
        run_round<LOGL, RB, TOP, INV, QF, GST, GLD>(ld0, stl, pi, q);
    } else if constexpr (IDX == 0) {
        run_round<LOGL, RB, TOP, INV, QF, false, GLD>(ld0, sts, pi, q);
        __syncthreads();
        rounds<LOGL, INV, CONTIG, 1, GST, false, DENSE>(sm, ld0, stl, pi, q);
    } else if constexpr (IDX == NR - 1) {
        run_round<LOGL, RB, TOP, INV, QF, GST>(lds, stl, pi, q);
    } else {
        run_round<LOGL, RB, TOP, INV, QF>(lds, sts, pi, q);
        __syncthreads();
        rounds<LOGL, INV, CONTIG, IDX + 1, GST, false, DENSE>(sm, ld0, stl, pi, q);
    }
}

// ------------------------------------------------------------------ pass bodies
// Digit g of the operand (32-bit word g of its limbs) reduced mod q, zero past the end.
__device__ __forceinline__ u32 entry_val(const u64* __restrict__ src, u64 len, u32 g, const PrimeQ& q) {
    return (g >> 1) < len ? qsmul(__ldg(reinterpret_cast<const u32*>(src) + g), 1u, q.one, q) : 0u;
}

// Four-step twiddles of a strided pass: element (row j, column c) holds frequency
// k = bitrev(j) and is multiplied by w_B^(i k), i = col0 + c, factored per lowest-round group
// as alpha(group) * beta[c][t'] (see fmn_ntt.cu).  Both factors are in Montgomery form.
template <int LOGL, bool INV>
__device__ __forceinline__ void fill_beta(u32* beta, u32 col0, int shift, int pi, const PrimeQ& q) {
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1), R = 1 << RB;
    for (int e = threadIdx.x; e < TC * R; e += NT) {   // beta[tp * TC + c]: conflict-free reads
        const u32 c = e & (TC - 1), tp = e >> LOG_TC;
        u32 x = ((col0 + c) * (tp << (LOGL - RB))) << shift;
        if (INV) x = (0u - x) & MASK_N;
        beta[e] = qroot(x, pi, q);
    }
}
template <int LOGL, bool INV>
__device__ __forceinline__ u32 group_alpha(u32 i, int row0, int shift, int pi, const PrimeQ& q) {
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1);
    const u32 kq = LOGL > RB ? __brev((u32)(row0 >> RB)) >> (32 - (LOGL - RB)) : 0u;
    u32 x = (i * kq) << shift;
    if (INV) x = (0u - x) & MASK_N;
    return qroot(x, pi, q);
}

// Table twiddles of a group of the lowest round (rows row0 .. row0 + 2^RB - 1 of column c):
// element t has frequency k = bitrev(row0 + t) over LOGL bits, entry k * 2^logS + col.
template <int LOGL, int RB>
__device__ __forceinline__ const uint2* tw_group(const uint2* tw, u32 col, int row0, int logS) {
    const u32 kq = LOGL > RB ? __brev((u32)(row0 >> RB)) >> (32 - (LOGL - RB)) : 0u;
    return tw + ((kq << logS) + col);
}

constexpr int kMaxFolds = 4;            // twisted products: N / M <= 4

// Forward strided pass (pass p < P-1 of a multi-pass transform).
template <int LOGL, bool ENTRY>
__device__ __forceinline__ void body_fwd(u32* sm, const QArgs& a, u64 tile, int pi, const PrimeQ& q) {
    constexpr int L = 1 << LOGL;
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1), R = 1 << RB;
    const int logS = a.logB - LOGL;
    const int tpb_log = logS - LOG_TC;
    const u32 blk = (u32)(tile >> tpb_log);
    const u32 col0 = (u32)((tile & ((1ull << tpb_log) - 1)) << LOG_TC);
    const u32 gbase = (blk << a.logB) + col0;
    u32* __restrict__ d = a.data + (u64)pi * a.N;
    const u64* __restrict__ src = a.src;
    const u64 len = a.len;
    const int shift = Q32_MAX_LOG_N - a.logB;
    // Residue tiles are copied in asynchronously while the twiddle factors are computed; the
    // entry pass reads the caller's limbs directly (8-byte alignment only, zero past the end).
    constexpr bool STAGED = !ENTRY;
    u32* beta = sm + (STAGED ? TC : TP) * L;
    const uint2* __restrict__ tw = a.tw ? a.tw + ((u64)pi << a.logB) : nullptr;
    if constexpr (STAGED) stage_tile<L>(sm, d + gbase, logS);
    if (!tw) fill_beta<LOGL, false>(beta, col0, shift, pi, q);   // read after the first round's barrier
    if constexpr (STAGED) {
        cp_async_commit_wait();
        __syncthreads();
    }
    auto ld0 = [=](int j, int c) -> u32 {
        if constexpr (STAGED) return sm[dix(j, c)];
        const u32 g = gbase + c + ((u32)j << logS);
        if constexpr (ENTRY) return entry_val(src, len, g, q);
        else return d[g];
    };
    auto stl = [=](int row0, int c, const auto& x) {
        u32* __restrict__ po = d + (gbase + c + ((u32)row0 << logS));
        const u32 S = 1u << logS;                 // row stride: t * S is a multiply-add address
        if (tw) {
            const uint2* __restrict__ tg = tw_group<LOGL, RB>(tw, col0 + c, row0, logS);
            const u32 ST = S << (LOGL - RB);      // table stride between the group's frequencies
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const u32 tp = RB ? __brev((u32)t) >> (32 - RB) : 0u;
                const uint2 w = __ldg(tg + tp * ST);
                po[(u32)t * S] = qsmul(x[t], w.x, w.y, q);
            }
        } else {
            const u32 al = group_alpha<LOGL, false>(col0 + c, row0, shift, pi, q);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int tp = RB ? (int)(__brev((u32)t) >> (32 - RB)) : 0;
                po[(u32)t * S] = qmont(x[t], qmont_lazy(al, beta[tp * TC + c], q), q);
            }
        }
    };
    rounds<LOGL, false, false, 0, true, false, STAGED>(sm, ld0, stl, pi, q);
}

// Inverse strided pass: inverse four-step twiddle, then the inverse sub-transform.  ACC: the
// coefficients go to the accumulator of a split product instead (see QArgs).
template <int LOGL, bool ACC>
__device__ __forceinline__ void body_inv(u32* sm, const QArgs& a, u64 tile, int pi, const PrimeQ& q) {
    constexpr int L = 1 << LOGL;
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1), R = 1 << RB;
    const int logS = a.logB - LOGL;
    const int tpb_log = logS - LOG_TC;
    const u32 blk = (u32)(tile >> tpb_log);
    const u32 col0 = (u32)((tile & ((1ull << tpb_log) - 1)) << LOG_TC);
    const u32 gbase = (blk << a.logB) + col0;
    u32* __restrict__ d = a.data + (u64)pi * a.N;
    const int shift = Q32_MAX_LOG_N - a.logB;
    u32* beta = sm + TC * L;
    const uint2* __restrict__ tw = a.tw ? a.tw + ((u64)pi << a.logB) : nullptr;
    stage_tile<L>(sm, d + gbase, logS);                   // in flight during fill_beta
    if (!tw) fill_beta<LOGL, true>(beta, col0, shift, pi, q);
    cp_async_commit_wait();
    __syncthreads();
    auto ld0 = [=](int row0, int c, auto& x) {
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = sm[dix(row0 + t, c)];
        if (tw) {
            const uint2* __restrict__ tg = tw_group<LOGL, RB>(tw, col0 + c, row0, logS);
            const u32 ST = (1u << logS) << (LOGL - RB);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const u32 tp = RB ? __brev((u32)t) >> (32 - RB) : 0u;
                const uint2 w = __ldg(tg + tp * ST);
                x[t] = qsmul(x[t], w.x, w.y, q);
            }
        } else {
            const u32 al = group_alpha<LOGL, true>(col0 + c, row0, shift, pi, q);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int tp = RB ? (int)(__brev((u32)t) >> (32 - RB)) : 0;
                x[t] = qmont(x[t], qmont_lazy(al, beta[tp * TC + c], q), q);
            }
        }
    };
    if constexpr (ACC) {
        // the last inverse round holds rows row0 + t * SP0 of one column: all accumulator
        // loads of a group are issued before its adds and stores
        constexpr int RB0 = round_bits(LOGL, 0), R0 = 1 << RB0, SP0 = 1 << (LOGL - RB0);
        u32* __restrict__ acc = a.acc + (u64)pi * a.acc_stride;
        const u64 valid = a.acc_valid, fresh = a.acc_fresh;
        constexpr int H = R0 < 8 ? R0 : 8;             // eight loads in flight at a time
        const u32 S0 = (u32)SP0 << logS;               // row stride of the group's outputs
        auto stl = [=](int row0, int c, const auto& x) {
            const u32 i0 = gbase + c + ((u32)row0 << logS);
            u32* __restrict__ pa = acc + i0;
#pragma unroll
            for (int h = 0; h < R0; h += H) {
                u32 old[H];
#pragma unroll
                for (int t = 0; t < H; ++t) {
                    const u32 off = (u32)(h + t) * S0;
                    old[t] = i0 + off < fresh ? pa[off] : 0u;
                }
#pragma unroll
                for (int t = 0; t < H; ++t) {
                    const u32 off = (u32)(h + t) * S0;
                    if (i0 + off < valid) pa[off] = i0 + off < fresh ? qadd(old[t], x[h + t], q) : x[h + t];
                }
            }
        };
        rounds<LOGL, true, false, 0, true, true, true>(sm, ld0, stl, pi, q);
    } else {
        // rows row0 + t * SP0 of one column (the last inverse round), by pointer and stride
        constexpr int RB0 = round_bits(LOGL, 0), R0 = 1 << RB0, SP0 = 1 << (LOGL - RB0);
        const u32 S0 = (u32)SP0 << logS;
        auto stl = [=](int row0, int c, const auto& x) {
            u32* __restrict__ po = d + (gbase + c + ((u32)row0 << logS));
#pragma unroll
            for (int t = 0; t < R0; ++t) po[(u32)t * S0] = x[t];
        };
        rounds<LOGL, true, false, 0, true, true, true>(sm, ld0, stl, pi, q);
    }
}

// Forward last pass over contiguous blocks (first operand of a product).
template <int LOGL, bool ENTRY>
__device__ __forceinline__ void body_fwd_last(u32* sm, const QArgs& a, u64 tile, int pi, const PrimeQ& q) {
    constexpr int L = 1 << LOGL;
    const u32 gbase = (u32)tile << (LOGL + LOG_TC);
    const int ncols = a.ncols;
    u32* __restrict__ d = a.data + (u64)pi * a.N;
    const u64* __restrict__ src = a.src;
    const u64 len = a.len;
    auto ld0 = [=](int j, int c) -> u32 {
        if (c >= ncols) return 0u;
        const u32 g = gbase + (u32)c * L + j;
        if constexpr (ENTRY) return entry_val(src, len, g, q);
        else return d[g];
    };
    if constexpr (LOGL == 0) {
        if (threadIdx.x < (unsigned)ncols) d[gbase + threadIdx.x] = ld0(0, threadIdx.x);
    } else {
        // the last round (a thread per column) writes the tile; the blocks then leave row by
        // row with the lanes of a warp on consecutive words (128-byte stores)
        auto sts = [sm](int j, int c, u32 v) { sm[tix<LOGL>(j, c)] = v; };
        rounds<LOGL, false, true, 0, false>(sm, ld0, sts, pi, q);
        __syncthreads();
#pragma unroll 4
        for (int e = threadIdx.x; e < TC * L; e += NT) {
            const int c = e >> LOGL, j = e & (L - 1);
            if (c < ncols) d[gbase + (u32)c * L + j] = sm[tix<LOGL>(j, c)];
        }
    }
}

// The lowest forward round, the pointwise product and the lowest inverse round of one
// contiguous tile, all in registers.
// OTH: where the other operand's transformed tile is read: 0 global memory, 1 a second tile in
// the tix layout, 2 a column-major staging buffer (column c at oth + c * (L + 4)).
template <int LOGL, bool SQR, int OTH = 0, class LD, class ST>
__device__ __forceinline__ void fused_lowest(LD ld, ST st, const u32* __restrict__ oth, u32 gbase, int ncols, int pi,
                                             const PrimeQ& q) {
    constexpr int L = 1 << LOGL;
    constexpr int NR = rounds_count(LOGL);
    constexpr int RB = round_bits(LOGL, NR - 1);
    constexpr int R = 1 << RB;
    constexpr int G = (L / R) * TC;
    const uint2* tf = &g_qrt[0][pi][rt_off(RB, RB - 1)];
    const uint2* ti = &g_qrt[1][pi][rt_off(RB, RB - 1)];
#pragma unroll 1
    for (int gi = threadIdx.x; gi < G; gi += NT) {
        const int c = gi & (TC - 1);
        const int row0 = (gi >> LOG_TC) << RB;
        u32 x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = ld(row0 + t, c);
#pragma unroll
        for (int s = 0; s < RB; ++s) {
            const int half = R >> (s + 1);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if (t & half) continue;
                const int u = t & (half - 1);
                if (u == 0) qbfly_dif1(x[t], x[t + half], q);
                else qbfly_dif(x[t], x[t + half], __ldg(tf + (R - (R >> s)) + u), q);
            }
        }
        if (c < ncols) {
            if constexpr (SQR) {
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = qmont(x[t], x[t], q);
            } else if constexpr (OTH == 1) {
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = qmont(x[t], oth[tix<LOGL>(row0 + t, c)], q);
            } else if constexpr (OTH == 2) {
                u32 y[R];
                ld_vec(oth + c * (L + 4) + row0, y);      // 8 lanes per phase on disjoint banks
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = qmont(x[t], y[t], q);
            } else {
                u32 y[R];
                ld_vec(oth + gbase + (u32)c * L + row0, y);
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = qmont(x[t], y[t], q);
            }
        }
#pragma unroll
        for (int s = RB - 1; s >= 0; --s) {
            const int half = R >> (s + 1);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if (t & half) continue;
                const int u = t & (half - 1);
                if (u == 0) qbfly_dit1(x[t], x[t + half], q);
                else qbfly_dit(x[t], x[t + half], __ldg(ti + (R - (R >> s)) + u), q);
            }
        }
#pragma unroll
        for (int t = 0; t < R; ++t) st(row0 + t, c, x[t]);
    }
}

// Last forward pass of the second operand (or of the only one when squaring), pointwise
// product with the first operand's spectrum, first inverse pass; overwrites `other`.
template <int LOGL, bool ENTRY, bool SQR>
__device__ __forceinline__ void body_fused(u32* sm, const QArgs& a, u64 tile, int pi, const PrimeQ& q) {
    constexpr int L = 1 << LOGL;
    constexpr int NR = rounds_count(LOGL);
    const u32 gbase = (u32)tile << (LOGL + LOG_TC);
    const int ncols = a.ncols;
    const u32* d = a.data + (u64)pi * a.N;
    const u32* o = a.other + (u64)pi * a.N;
    u32* dd = (a.dst ? a.dst : a.other) + (u64)pi * a.N;   // may be `data` itself (in place)
    const u64* __restrict__ src = a.src;
    const u64 len = a.len;
    auto ldg = [=](int j, int c) -> u32 {
        if (c >= ncols) return 0u;
        const u32 g = gbase + (u32)c * L + j;
        if constexpr (ENTRY) return entry_val(src, len, g, q);
        else return d[g];
    };
    auto stg = [=](int j, int c, u32 v) {
        if (c < ncols) dd[gbase + (u32)c * L + j] = v;
    };
    auto lds = [sm](int j, int c) { return sm[tix<LOGL>(j, c)]; };
    auto sts = [sm](int j, int c, u32 v) { sm[tix<LOGL>(j, c)] = v; };
    if constexpr (LOGL == 0) {
        if (threadIdx.x < (unsigned)ncols) {
            const int c = threadIdx.x;
            const u32 x = ldg(0, c);
            const u32 y = SQR ? x : o[gbase + c];
            stg(0, c, qmont(x, y, q));
        }
    } else if constexpr (NR == 1) {
        fused_lowest<LOGL, SQR>(ldg, stg, o, gbase, ncols, pi, q);
    } else {
        // the other operand's tile, column by column, is copied in while the forward rounds run
        constexpr bool OS = !SQR && LOGL <= 8;           // 9-bit tiles: no room for a second one
        u32* oth_s = sm + TP * L;
        if constexpr (OS) {
#pragma unroll 4
            for (int e = threadIdx.x; e < TC * (L / 4); e += NT) {
                const int c = e / (L / 4), k = e % (L / 4);
                if (c < ncols) cp_async16(oth_s + c * (L + 4) + 4 * k, o + gbase + (u32)c * L + 4 * k);
            }
            cp_async_commit();
        }
        constexpr int RB0 = round_bits(LOGL, 0);
        run_round<LOGL, RB0, LOGL - 1, false, true>(ldg, sts, pi, q);
        if constexpr (NR == 3) {
            __syncthreads();
            constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
            run_round<LOGL, RB1, T1, false, false>(lds, sts, pi, q);
        }
        if constexpr (OS) cp_async_wait_all();
        __syncthreads();
        fused_lowest<LOGL, SQR, OS ? 2 : 0>(lds, sts, OS ? oth_s : o, gbase, ncols, pi, q);
        __syncthreads();
        if constexpr (NR == 3) {
            constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
            run_round<LOGL, RB1, T1, true, false>(lds, sts, pi, q);
            __syncthreads();
        }
        run_round<LOGL, RB0, LOGL - 1, true, true>(lds, stg, pi, q);
    }
}

// Both operands' last forward pass, the pointwise product and the first inverse pass: the
// first operand's tile (from `other`) is transformed into a second shared-memory tile and
// never written back; the product overwrites `other`.  Multi-pass products only.
template <int LOGL>
__device__ __forceinline__ void body_fused2(u32* sm, const QArgs& a, u64 tile, int pi, const PrimeQ& q) {
    constexpr int L = 1 << LOGL;
    constexpr int NR = rounds_count(LOGL);
    static_assert(NR >= 2, "multi-round sub-transforms only");
    const u32 gbase = (u32)tile << (LOGL + LOG_TC);
    const u32* __restrict__ d = a.data + (u64)pi * a.N;
    u32* __restrict__ o = a.other + (u64)pi * a.N;
    u32* smA = sm + TP * L;
    auto ldA = [=](int j, int c) -> u32 { return o[gbase + (u32)c * L + j]; };
    auto stA = [smA](int j, int c, u32 v) { smA[tix<LOGL>(j, c)] = v; };
    rounds<LOGL, false, true, 0>(smA, ldA, stA, pi, q);
    auto ldg = [=](int j, int c) -> u32 { return d[gbase + (u32)c * L + j]; };
    auto stg = [=](int j, int c, u32 v) { o[gbase + (u32)c * L + j] = v; };
    auto lds = [sm](int j, int c) { return sm[tix<LOGL>(j, c)]; };
    auto sts = [sm](int j, int c, u32 v) { sm[tix<LOGL>(j, c)] = v; };
    constexpr int RB0 = round_bits(LOGL, 0);
    run_round<LOGL, RB0, LOGL - 1, false, true>(ldg, sts, pi, q);
    __syncthreads();                                   // also publishes smA
    if constexpr (NR == 3) {
        constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
        run_round<LOGL, RB1, T1, false, false>(lds, sts, pi, q);
        __syncthreads();
    }
    fused_lowest<LOGL, false, 1>(lds, sts, smA, gbase, TC, pi, q);
    __syncthreads();
    if constexpr (NR == 3) {
        constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
        run_round<LOGL, RB1, T1, true, false>(lds, sts, pi, q);
        __syncthreads();
    }
    run_round<LOGL, RB0, LOGL - 1, true, true>(lds, stg, pi, q);
}

// Kernels whose tiles limit them to 3 CTAs per SM anyway (9-bit strided passes, the merged
// pass, the fused pass with its staged spectrum tile) get the registers of 3 CTAs.  8-bit
// strided passes fit 64 registers without spills and run at 4 (1% faster than at 3).
template <int MODE, int LOGL>
constexpr int min_ctas() {
    return ((MODE == M_FWD || MODE == M_INV || MODE == M_INV_ACC) && LOGL >= 9) || MODE == M_FUSED2 ||
                   (MODE == M_FUSED && LOGL == 8)
               ? 3
               : 4;
}

template <int MODE, int LOGL, bool ENTRY, bool SQR>
__global__ void __launch_bounds__(NT, (min_ctas<MODE, LOGL>())) k_qpass(QArgs a) {
    extern __shared__ __align__(16) u32 qsm[];
    const int pi = blockIdx.x % 3;          // the three CTAs of a tile read the same limbs together
    const u64 tile = blockIdx.x / 3;
    const PrimeQ q = c_q[pi];
    if constexpr (MODE == M_FWD) body_fwd<LOGL, ENTRY>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_INV) body_inv<LOGL, false>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_INV_ACC) body_inv<LOGL, true>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_FWD_LAST) body_fwd_last<LOGL, ENTRY>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_FUSED2) body_fused2<(LOGL >= 5 ? LOGL : 5)>(qsm, a, tile, pi, q);
    else body_fused<LOGL, ENTRY, SQR>(qsm, a, tile, pi, q);
}

// Batched form: products with the same transform length and kind share every launch; CTA b
// works on product b / (3 * tiles), tile (b / 3) % tiles, prime b % 3.
template <int MODE, int LOGL, bool ENTRY, bool SQR>
__global__ void __launch_bounds__(NT, (min_ctas<MODE, LOGL>())) k_qpass_batch(const QArgs* __restrict__ args,
                                                                              u32 tiles) {
    extern __shared__ __align__(16) u32 qsm[];
    const int pi = blockIdx.x % 3;
    const u32 rest = blockIdx.x / 3;
    const QArgs a = args[rest / tiles];
    const u64 tile = rest % tiles;
    const PrimeQ q = c_q[pi];
    if constexpr (MODE == M_FWD) body_fwd<LOGL, ENTRY>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_INV) body_inv<LOGL, false>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_FWD_LAST) body_fwd_last<LOGL, ENTRY>(qsm, a, tile, pi, q);
    else if constexpr (MODE == M_FUSED2) body_fused2<(LOGL >= 5 ? LOGL : 5)>(qsm, a, tile, pi, q);
    else body_fused<LOGL, ENTRY, SQR>(qsm, a, tile, pi, q);
}

// ------------------------------------------------------------------ CRT + carry
// Digit coefficient k of the product, c_k < Q = q0 q1 q2 < 2^91, from its residues y_i = c_k
// mod q_i by Garner's mixed-radix form c_k = x0 + q0 (x1 + q1 x2) (the same number as the
// reference's CRT sum, src/core.h:77-104, without its final reduction mod Q).  Output limb j
// collects the 128-bit pair C_j = c_{2j} + c_{2j+1} 2^32 < 2^124: s_j = C_j.lo + C_{j-1}.hi,
// then the carry scan.
//
// Wrapped products (wrap = K > 0): `res` holds a cyclic convolution of length N, whose entry
// k < K is c_k + c_{k+N} (the coefficients from N on wrap around), and `low` holds the product
// of the operands' lowest digits, whose coefficients below K are exactly c_0 .. c_{K-1}.  So
// c_k = low_k for k < K, res_k for K <= k < N, and res_{k-N} - low_{k-N} (mod each prime) for
// N <= k < N + K.  Each array carries its own scale constants (its transform length differs).
struct QCrtArgs {
    const u32* res;     // three natural-order residue arrays (prime i at res + i*N), in [0, q)
    u64 N;
    u64 nvalid;         // digit coefficients that may be nonzero
    u64* out;
    u64 out_len;
    u32 cst[3];         // N^-1 * 2^64 mod q_i (undoes N and the two Montgomery factors)
    u32 inv01;          // Montgomery form mod q1 of q0^-1
    u32 q0m2;           // Montgomery form mod q2 of q0
    u32 inv012;         // Montgomery form mod q2 of (q0 q1)^-1
    u32* state;
    u32* ticket;
    u32* err;
    const u32* low;     // wrapped products: the low product's residues (prime i at low + i*low_N)
    u64 low_N;
    u64 wrap;           // K: coefficients that wrapped (0: none)
    u32 low_cst[3];     // the low product's scale constants (low_N^-1 * 2^64 mod q_i)
    // twisted: `low` holds W (plain, reduced; low_cst = 2^32 mod q_i), the wrapped
    // coefficients c_{N+k} = W_k, and res_k already holds c_k for k < K (see k_qtwist_w)
    int twisted;
};

typedef unsigned __int128 u128;
constexpr u64 Q01 = (u64)Q32_P0 * Q32_P1;
// Output limbs per thread of the CRT + carry kernel: 8 (half the 64-bit engine's 16) keeps a
// thread's sums in 57 registers, so 4 CTAs share an SM where 16 allowed 3 (0.28 -> 0.23 ms at
// 10M x 10M; the kernel waits on its look-back and loads, and more CTAs cover the waits).
constexpr int QCE = 8;
constexpr u64 QCTILE = (u64)CNT * QCE;  // output limbs per CTA

// c from x0 = c mod q0, y1 = c mod q1, y2 = c mod q2 (all reduced).
__device__ __forceinline__ u128 qgarner(u32 x0, u32 y1, u32 y2, const QCrtArgs& a, const PrimeQ& q1,
                                        const PrimeQ& q2) {
    const u32 x0r = x0 >= q1.p ? x0 - q1.p : x0;               // q0 < 2 q1
    const u32 x1 = qmont(qsub(y1, x0r, q1), a.inv01, q1);      // (c - x0) / q0 mod q1
    const u32 t = qadd(qsmul(x0, 1u, q2.one, q2), qmont(x1, a.q0m2, q2), q2);
    const u32 x2 = qmont(qsub(y2, t, q2), a.inv012, q2);       // (c - x0 - q0 x1) / (q0 q1) mod q2
    // c = x0 + q0 x1 + q0 q1 x2 < 2^91, exactly
    const u64 s1 = (u64)x0 + (u64)Q32_P0 * x1;
    const u64 lo0 = (u64)x2 * (u32)Q01, mid = (u64)x2 * (u32)(Q01 >> 32);
    u64 lo = s1 + lo0;
    u64 hi = lo < lo0;
    const u64 ml = mid << 32;
    lo += ml;
    hi += (lo < ml) + (mid >> 32);
    return ((u128)hi << 64) | lo;
}
// Residue vectors of VW (2 or 4) consecutive coefficients from one array of one prime.
template <int VW>
__device__ __forceinline__ void ldv(const u32* p, u32 (&r)[VW]) {
    if constexpr (VW == 4) {
        const uint4 v = *reinterpret_cast<const uint4*>(p);
        r[0] = v.x, r[1] = v.y, r[2] = v.z, r[3] = v.w;
    } else {
        const uint2 v = *reinterpret_cast<const uint2*>(p);
        r[0] = v.x, r[1] = v.y;
    }
}
// Where coefficient k comes from (see QCrtArgs): 0 res_k, 1 low_k, 2 res_{k-N} - low_{k-N}
// (twisted: k_qtwist_w has already written c_k into res below N, so only 0 and 2, low alone).
__device__ __forceinline__ int qsource(const QCrtArgs& a, u64 k) {
    return k >= a.N && a.wrap ? 2 : (k < a.wrap && !a.twisted ? 1 : 0);
}
// c_k mod q_i (reduced) of one prime, by source.
// (a wrapped product's sources 1 and 2 swap formulas when it is twisted: res - low at k < K,
// low alone at N + k)
__device__ __forceinline__ u32 qscaled(const QCrtArgs& a, int src, u64 k, int i, const PrimeQ& q) {
    if (src == 0) return qmont(a.res[i * a.N + k], a.cst[i], q);
    const u64 kk = src == 2 ? k - a.N : k;
    if ((src == 2) == (a.twisted != 0)) return qmont(a.low[i * a.low_N + kk], a.low_cst[i], q);
    return qsub(qmont(a.res[i * a.N + kk], a.cst[i], q), qmont(a.low[i * a.low_N + kk], a.low_cst[i], q), q);
}
template <bool WRAP>
__device__ __forceinline__ u128 qcoef(const QCrtArgs& a, u64 k, const PrimeQ& q0, const PrimeQ& q1, const PrimeQ& q2) {
    if (k >= a.nvalid) return 0;
    const int src = WRAP ? qsource(a, k) : 0;
    return qgarner(qscaled(a, src, k, 0, q0), qscaled(a, src, k, 1, q1), qscaled(a, src, k, 2, q2), a, q1, q2);
}

// MODE 0: a plain product; 1: wrapped with a low product (see QCrtArgs), whose threads may
// read two sources at once and so hold more registers; 2: twisted, whose threads read one
// source each (the cyclic residues below N, W above).
template <int MODE, long LIMIT = SPIN_LIMIT>
__device__ __forceinline__ void qcrt_carry_body(const QCrtArgs& a, u32 ncta) {
    constexpr bool WRAP = MODE != 0;
    __shared__ u64 s_hw[CNT / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const PrimeQ q0 = c_q[0], q1 = c_q[1], q2 = c_q[2];
    const u64 tile = carry_ticket(a.ticket);
    if (tile >= ncta) return;                          // batch launches cover the largest product
    const u64 j0 = tile * QCTILE + (u64)tid * QCE;     // output limbs j0 .. j0+QCE-1
    const u64 k0 = 2 * j0;                             // digit coefficients k0 .. k0+31
    u64 lo[QCE];
    u32 h[QCE];
    u64 phi = 0;                                       // C_{j-1}.hi
    // the thread's 2 QCE coefficients come from one source (k0 and N are multiples of 16),
    // read as vectors, unless they straddle the end or the wrap boundary K
    const int src = WRAP ? qsource(a, k0) : 0;
    const bool full = k0 + 2 * QCE <= a.nvalid && (src != 1 || k0 + 2 * QCE <= a.wrap);
    const u64 kb = src == 2 ? k0 - a.N : k0;
    // VW coefficients (VW / 2 limbs) at a time: four, or two for wrapped products with a low
    // product, whose two sources would otherwise hold too many registers for 4 CTAs per SM
    constexpr int VW = MODE == 1 ? 2 : 4;
#pragma unroll
    for (int e2 = 0; e2 < QCE; e2 += VW / 2) {
        u32 y0[VW], y1[VW], y2[VW];                    // c_k mod q_i
        if (full) {
            const u64 k = kb + 2 * e2;
            if (src != 0 && (src == 2) == (a.twisted != 0)) {   // low alone
                ldv<VW>(a.low + k, y0);
                ldv<VW>(a.low + a.low_N + k, y1);
                ldv<VW>(a.low + 2 * a.low_N + k, y2);
#pragma unroll
                for (int t = 0; t < VW; ++t) {
                    y0[t] = qmont(y0[t], a.low_cst[0], q0);
                    y1[t] = qmont(y1[t], a.low_cst[1], q1);
                    y2[t] = qmont(y2[t], a.low_cst[2], q2);
                }
            } else {
                ldv<VW>(a.res + k, y0);
                ldv<VW>(a.res + a.N + k, y1);
                ldv<VW>(a.res + 2 * a.N + k, y2);
#pragma unroll
                for (int t = 0; t < VW; ++t) {
                    y0[t] = qmont(y0[t], a.cst[0], q0);
                    y1[t] = qmont(y1[t], a.cst[1], q1);
                    y2[t] = qmont(y2[t], a.cst[2], q2);
                }
                if (MODE == 1 && src != 0) {                     // res - low
                    u32 l0[VW], l1[VW], l2[VW];
                    ldv<VW>(a.low + k, l0);
                    ldv<VW>(a.low + a.low_N + k, l1);
                    ldv<VW>(a.low + 2 * a.low_N + k, l2);
#pragma unroll
                    for (int t = 0; t < VW; ++t) {
                        y0[t] = qsub(y0[t], qmont(l0[t], a.low_cst[0], q0), q0);
                        y1[t] = qsub(y1[t], qmont(l1[t], a.low_cst[1], q1), q1);
                        y2[t] = qsub(y2[t], qmont(l2[t], a.low_cst[2], q2), q2);
                    }
                }
            }
        }
#pragma unroll
        for (int u = 0; u < VW / 2; ++u) {
            const int e = e2 + u;
            u128 cl, ch;
            if (full) {
                cl = qgarner(y0[2 * u], y1[2 * u], y2[2 * u], a, q1, q2);
                ch = qgarner(y0[2 * u + 1], y1[2 * u + 1], y2[2 * u + 1], a, q1, q2);
            } else {
                cl = qcoef<WRAP>(a, k0 + 2 * e, q0, q1, q2);
                ch = qcoef<WRAP>(a, k0 + 2 * e + 1, q0, q1, q2);
            }
            const u128 C = cl + (ch << 32);
            u64 l = (u64)C;
            u32 hh = 0;
            add_to(l, hh, phi);
            lo[e] = l;
            h[e] = hh;
            phi = (u64)(C >> 64);
        }
    }
    // C_{j0-1}.hi from the previous thread, warp or CTA
    u64 nb = __shfl_up_sync(0xffffffffu, phi, 1);
    if (lane == 31) s_hw[warp] = phi;
    __syncthreads();
    if (lane == 0) {
        if (warp > 0) {
            nb = s_hw[warp - 1];
        } else if (j0 > 0) {
            const u128 C = qcoef<WRAP>(a, k0 - 2, q0, q1, q2) + (qcoef<WRAP>(a, k0 - 1, q0, q1, q2) << 32);
            nb = (u64)(C >> 64);
        } else {
            nb = 0;
        }
    }
    add_to(lo[0], h[0], nb);
    carry_finish<QCE, LIMIT>(lo, h, tile, j0, a.state, a.err, a.out, a.out_len);
}

// 5 CTAs per SM (48 registers, no spills): while one CTA's warps wait at the barrier of its
// look-back, the others compute (4 CTAs: 56-62 registers, barrier the top stall)
__global__ void __launch_bounds__(CNT, 5) k_qcrt_carry(QCrtArgs a) {
    qcrt_carry_body<0>(a, 0xffffffffu);
}
// Wrapped products with a low product (two residue sources, two sets of scale constants).
__global__ void __launch_bounds__(CNT, 4) k_qcrt_carry_wrap(QCrtArgs a) { qcrt_carry_body<1>(a, 0xffffffffu); }
// Twisted wrapped products (a CTA tile lies wholly below or above N: one source per tile).
__global__ void __launch_bounds__(CNT, 5) k_qcrt_carry_twist(QCrtArgs a) { qcrt_carry_body<2>(a, 0xffffffffu); }

// The plain kernel with a look-back limit of 2^12 polls (milliseconds instead of seconds), for
// the test that withholds a tile and checks that the wait expires into the status word.
__global__ void __launch_bounds__(CNT, 4) k_qcrt_carry_short_wait(QCrtArgs a) {
    qcrt_carry_body<0, (1l << 12)>(a, 0xffffffffu);
}

// CRT + carry of many products: CTAs take per-product tickets; tickets beyond a product's
// CTA count exit at once.
__global__ void __launch_bounds__(CNT) k_qcrt_carry_batch(const QCrtArgs* __restrict__ args, u32 ctas_per_job,
                                                          const u32* __restrict__ ncta) {
    const u32 job = blockIdx.x / ctas_per_job;
    qcrt_carry_body<0>(args[job], ncta[job]);
}
// The same for twisted wrapped products.
__global__ void __launch_bounds__(CNT, 4) k_qcrt_carry_twist_batch(const QCrtArgs* __restrict__ args, u32 ctas_per_job,
                                                                   const u32* __restrict__ ncta) {
    const u32 job = blockIdx.x / ctas_per_job;
    qcrt_carry_body<2>(args[job], ncta[job]);
}

// ------------------------------------------------------------------ twisted products
// A wrapped product computed as U = C mod (X^N - 1) (the cyclic transform of length N) and
// V = C mod (X^M - c) (a cyclic transform of length M = N / 2^s of the operands folded modulo
// X^M - c and twisted by gamma^i, gamma of order 2N, c = gamma^M, so c^(2^s) = -1).  With
// C = U + (X^N - 1) W, deg W < K <= M, and X^N = -1 mod (X^M - c):
//     W = (U mod (X^M - c) - V) / 2,   U mod (X^M - c) = sum_j c^j U_{k + j M}.
// The kernel writes W_k (plain, reduced) over V_k and c_k = U_k - W_k over U_k (in U's raw
// form, times N 2^-32, as the CRT reads it) for k < K; the CRT then takes c_{N+k} = W_k and
// c_k from U.  Each residue array is scaled by its own length (and V untwisted).  Updating U_k
// in place is safe: the other residues read for a k, U_{k+jM} with j >= 1, lie at or above
// M >= K.
// The operand folded modulo X^M - c and twisted, as residues: entry g (< M) of prime i is
// gamma^g sum_{j < 2^fold_log} c^j a_{g + jM} mod q_i (a the operand's 32-bit digits, zero past
// its end), written to T + i M + g.  One thread per g: the fold's digits are loaded once for
// all three primes, each load coalesced across the warp; c^j multiplies as a Shoup constant
// (host-computed), gamma^g as a Montgomery factor stepped along the grid-stride loop.
// Indices are 32-bit: a twisted product has N <= 2^25 digits and both operands fit N.
struct QFoldArgs {
    const u64* src;
    u64 len;            // limbs (2 len digits)
    u32* T;
    int logM, fold_log, tw_log;
    uint2 cpow[3][kMaxFolds];   // c^j mod q_i, plain, with Shoup companion floor(c^j 2^32 / q_i)
};
// Blocks blk of nblk (256 threads each) cover one operand.
__device__ __forceinline__ void qtwist_fold_body(const QFoldArgs& f, u32 blk, u32 nblk) {
    const u32* __restrict__ dig = reinterpret_cast<const u32*>(f.src);
    const u32 nd = (u32)(2 * f.len), M = 1u << f.logM;
    const int F = 1 << f.fold_log;
    const u32 g0 = blk * blockDim.x + threadIdx.x, S = nblk * blockDim.x;
    // gamma^g in Montgomery form, stepped by gamma^S along the grid-stride loop
    u32 gm[3], gs[3];
#pragma unroll
    for (int pi = 0; pi < 3; ++pi) {
        gm[pi] = qroot((g0 << f.tw_log) & MASK_N, pi, c_q[pi]);
        gs[pi] = qroot((S << f.tw_log) & MASK_N, pi, c_q[pi]);
    }
    for (u32 g = g0; g < M; g += S) {
        // folds holding digits at g: a_{g + jM} for j < nf (all zero past the operand)
        const u32 left = nd > g ? (nd - g + M - 1) >> f.logM : 0u;
        const int nf = left < (u32)F ? (int)left : F;
        u32 x[kMaxFolds];
#pragma unroll
        for (int j = 0; j < kMaxFolds; ++j) x[j] = j < nf ? __ldg(dig + g + ((u32)j << f.logM)) : 0u;
#pragma unroll
        for (int pi = 0; pi < 3; ++pi) {
            const PrimeQ q = c_q[pi];
            u32 acc = qsmul(x[0], f.cpow[pi][0].x, f.cpow[pi][0].y, q);
#pragma unroll
            for (int j = 1; j < kMaxFolds; ++j)
                if (j < nf) acc = qadd(acc, qsmul(x[j], f.cpow[pi][j].x, f.cpow[pi][j].y, q), q);
            f.T[pi * M + g] = qmont(acc, gm[pi], q);
            gm[pi] = qmont(gm[pi], gs[pi], q);
        }
    }
}
__global__ void __launch_bounds__(256) k_qtwist_fold(QFoldArgs f) { qtwist_fold_body(f, blockIdx.x, gridDim.x); }
// Batches: bpj consecutive blocks per product.
__global__ void __launch_bounds__(256) k_qtwist_fold_batch(const QFoldArgs* __restrict__ args, u32 bpj) {
    qtwist_fold_body(args[blockIdx.x / bpj], blockIdx.x % bpj, bpj);
}

struct QTwistArgs {
    u32* U;             // cyclic product's residues (prime i at U + i N), raw; c_k below K on return
    u32* V;             // twisted product's residues (prime i at V + i M), raw; W on return
    u32 N, K;
    int logM, fold_log, tw_log;
    u32 cstM[3];        // M^-1 2^64 mod q_i: with gamma^-k in Montgomery form, V raw -> V untwisted
    uint2 ucj[3][kMaxFolds];   // c^j N^-1 2^32 mod q_i (Shoup pairs): U raw -> c^j U
    uint2 nraw[3];      // N 2^-32 mod q_i (Shoup pair): a coefficient -> U's raw form
};
// Prime pi; blocks blk of nblk cover the wrapped coefficients.
__device__ __forceinline__ void qtwist_w_body(const QTwistArgs& t, int pi, u32 blk, u32 nblk) {
    const PrimeQ q = c_q[pi];
    const int F = 1 << t.fold_log;
    u32* __restrict__ U = t.U + pi * t.N;
    u32* __restrict__ V = t.V + (pi << t.logM);
    const u32 k0 = blk * blockDim.x + threadIdx.x, S = nblk * blockDim.x;
    // gamma^-k M^-1 2^32 (the Montgomery form of gamma^-k times cstM 2^-32), stepped by gamma^-S
    u32 gm = qmont(qroot((0u - (k0 << t.tw_log)) & MASK_N, pi, q), t.cstM[pi], q);
    const u32 gs = qroot((0u - (S << t.tw_log)) & MASK_N, pi, q);
    for (u32 k = k0; k < t.K; k += S) {
        u32 x[kMaxFolds];
#pragma unroll
        for (int j = 0; j < kMaxFolds; ++j) x[j] = j < F ? U[k + ((u32)j << t.logM)] : 0u;
        const u32 vr = V[k];
        const u32 u0 = qsmul(x[0], t.ucj[pi][0].x, t.ucj[pi][0].y, q);    // U_k
        u32 ub = u0;
#pragma unroll
        for (int j = 1; j < kMaxFolds; ++j)
            if (j < F) ub = qadd(ub, qsmul(x[j], t.ucj[pi][j].x, t.ucj[pi][j].y, q), q);
        const u32 d = qsub(ub, qmont(vr, gm, q), q);                      // U mod (X^M - c) - V
        const u32 w = (d + ((d & 1u) ? q.p : 0u)) >> 1;
        V[k] = w;
        U[k] = qsmul(qsub(u0, w, q), t.nraw[pi].x, t.nraw[pi].y, q);     // c_k = U_k - W_k, raw
        gm = qmont(gm, gs, q);
    }
}
__global__ void __launch_bounds__(256) k_qtwist_w(QTwistArgs t) { qtwist_w_body(t, blockIdx.y, blockIdx.x, gridDim.x); }
__global__ void __launch_bounds__(256) k_qtwist_w_batch(const QTwistArgs* __restrict__ args, u32 bpj) {
    qtwist_w_body(args[blockIdx.x / bpj], blockIdx.y, blockIdx.x % bpj, bpj);
}

// ------------------------------------------------------------------ host: tables
static u64 h_mulmod(u64 a, u64 b, u64 m) { return (u64)(((u128)a * b) % m); }
static u64 h_pow(u64 b, u64 e, u64 m) {
    u64 r = 1;
    b %= m;
    while (e) {
        if (e & 1) r = h_mulmod(r, b, m);
        b = h_mulmod(b, b, m);
        e >>= 1;
    }
    return r;
}
static const u32 kQ[3] = {Q32_P0, Q32_P1, Q32_P2};
static u32 c_host_r1(int i) { return (u32)((1ull << 32) % kQ[i]); }   // Montgomery form of 1

// Smallest primitive root of p (trial factorisation of p - 1).
static u64 primitive_root(u64 p) {
    std::vector<u64> f;
    u64 m = p - 1;
    for (u64 d = 2; d * d <= m; ++d)
        if (m % d == 0) {
            f.push_back(d);
            while (m % d == 0) m /= d;
        }
    if (m > 1) f.push_back(m);
    for (u64 g = 2;; ++g) {
        bool ok = true;
        for (u64 x : f)
            if (h_pow(g, (p - 1) / x, p) == 1) {
                ok = false;
                break;
            }
        if (ok) return g;
    }
}

struct HostTables {
    std::vector<u32> rt;   // [2][3][RT_SIZE][2]: (w, floor(w 2^32 / q)) Shoup pairs
    std::vector<u32> tw;   // [2][3][1 << QTWB]: Montgomery form
    u64 w26[3];            // the root of order 2^26 of each prime that all tables use
};

static const HostTables& host_tables() {
    static HostTables T;
    static std::once_flag once;
    std::call_once(once, [] {
        T.rt.assign((size_t)2 * 3 * RT_SIZE * 2, 0);
        T.tw.assign((size_t)2 * 3 * (1u << QTWB), 0);
        for (int i = 0; i < 3; ++i) {
            const u64 p = kQ[i];
            const u64 w = h_pow(primitive_root(p), (p - 1) >> Q32_MAX_LOG_N, p);   // order 2^26
            T.w26[i] = w;
            std::vector<u64> lo(1u << QTWB), hi(1u << QTWB);
            const u64 whi = h_pow(w, 1ull << QTWB, p);
            u64 cl = 1, ch = 1;
            for (u32 x = 0; x < (1u << QTWB); ++x) {
                lo[x] = cl;
                hi[x] = ch;
                cl = h_mulmod(cl, w, p);
                ch = h_mulmod(ch, whi, p);
            }
            auto wpow = [&](u64 e) {   // w^e, e mod 2^26
                e &= MASK_N;
                return h_mulmod(hi[e >> QTWB], lo[e & ((1u << QTWB) - 1)], p);
            };
            for (u32 x = 0; x < (1u << QTWB); ++x) {
                T.tw[((size_t)0 * 3 + i) * (1u << QTWB) + x] = (u32)((lo[x] << 32) % p);
                T.tw[((size_t)1 * 3 + i) * (1u << QTWB) + x] = (u32)((hi[x] << 32) % p);
            }
            for (int r = 1; r <= 4; ++r)
                for (int top = r - 1; top < RT_MAXLOGL; ++top) {
                    const int R = 1 << r, spl = top - r + 1;
                    for (int qq = 0; qq < (1 << spl); ++qq)
                        for (int s = 0; s < r; ++s)
                            for (int u = 0; u < (R >> (s + 1)); ++u) {
                                // w_{2^(top-s+1)}^(qq + u 2^spl) = w^((qq + u 2^spl) 2^(26-(top-s+1)))
                                const u64 e = ((u64)qq + ((u64)u << spl)) << (Q32_MAX_LOG_N - (top - s + 1));
                                // stage-major: entry j = (R - (R >> s)) + u of group offset qq
                                const size_t at = (size_t)rt_off(r, top) + ((size_t)(R - (R >> s)) + u << spl) + qq;
                                const u64 wf = wpow(e);
                                const u64 wi = wpow((1ull << Q32_MAX_LOG_N) - (e & MASK_N));
                                const size_t f0 = (((size_t)0 * 3 + i) * RT_SIZE + at) * 2;
                                const size_t i0 = (((size_t)1 * 3 + i) * RT_SIZE + at) * 2;
                                T.rt[f0] = (u32)wf;
                                T.rt[f0 + 1] = (u32)((wf << 32) / p);
                                T.rt[i0] = (u32)wi;
                                T.rt[i0 + 1] = (u32)((wi << 32) / p);
                            }
                }
        }
    });
    return T;
}

// ------------------------------------------------------------------ host: kernels
typedef void (*QKernel)(QArgs);
enum { V_FWD, V_FWD_E, V_LAST, V_LAST_E, V_FUSED, V_FUSED_E, V_SQR, V_SQR_E, V_INV, V_FUSED2, V_INV_ACC, NV };

template <int LOGL>
static void fill_row(QKernel (&t)[NV][MAX_PASS_BITS + 1]) {
    constexpr int LS = LOGL >= 5 ? LOGL : 5;                      // strided passes: >= 5 bits
    constexpr int LM = (LOGL >= 5 && LOGL <= 8) ? LOGL : 5;       // merged pass: two tiles
    t[V_FWD][LOGL] = LOGL >= 5 ? k_qpass<M_FWD, LS, false, false> : nullptr;
    t[V_FWD_E][LOGL] = LOGL >= 5 ? k_qpass<M_FWD, LS, true, false> : nullptr;
    t[V_INV][LOGL] = LOGL >= 5 ? k_qpass<M_INV, LS, false, false> : nullptr;
    t[V_INV_ACC][LOGL] = LOGL >= 5 ? k_qpass<M_INV_ACC, LS, false, false> : nullptr;
    t[V_FUSED2][LOGL] = (LOGL >= 5 && LOGL <= 8) ? k_qpass<M_FUSED2, LM, false, false> : nullptr;
    t[V_LAST][LOGL] = k_qpass<M_FWD_LAST, LOGL, false, false>;
    t[V_LAST_E][LOGL] = k_qpass<M_FWD_LAST, LOGL, true, false>;
    t[V_FUSED][LOGL] = k_qpass<M_FUSED, LOGL, false, false>;
    t[V_FUSED_E][LOGL] = k_qpass<M_FUSED, LOGL, true, false>;
    t[V_SQR][LOGL] = k_qpass<M_FUSED, LOGL, false, true>;
    t[V_SQR_E][LOGL] = k_qpass<M_FUSED, LOGL, true, true>;
}

struct KernelTable {
    QKernel k[NV][MAX_PASS_BITS + 1];
    KernelTable() {
        memset(k, 0, sizeof(k));
        fill_row<0>(k);
        fill_row<1>(k);
        fill_row<2>(k);
        fill_row<3>(k);
        fill_row<4>(k);
        fill_row<5>(k);
        fill_row<6>(k);
        fill_row<7>(k);
        fill_row<8>(k);
        fill_row<9>(k);
    }
};
static const KernelTable& ktab() {
    static KernelTable t;
    return t;
}

typedef void (*QBatchKernel)(const QArgs*, u32);
template <int LOGL>
static void fill_brow(QBatchKernel (&t)[NV][MAX_PASS_BITS + 1]) {
    constexpr int LS = LOGL >= 5 ? LOGL : 5;
    constexpr int LM = (LOGL >= 5 && LOGL <= 8) ? LOGL : 5;
    t[V_FWD][LOGL] = LOGL >= 5 ? k_qpass_batch<M_FWD, LS, false, false> : nullptr;
    t[V_FWD_E][LOGL] = LOGL >= 5 ? k_qpass_batch<M_FWD, LS, true, false> : nullptr;
    t[V_INV][LOGL] = LOGL >= 5 ? k_qpass_batch<M_INV, LS, false, false> : nullptr;
    t[V_FUSED2][LOGL] = (LOGL >= 5 && LOGL <= 8) ? k_qpass_batch<M_FUSED2, LM, false, false> : nullptr;
    t[V_LAST][LOGL] = k_qpass_batch<M_FWD_LAST, LOGL, false, false>;
    t[V_LAST_E][LOGL] = k_qpass_batch<M_FWD_LAST, LOGL, true, false>;
    t[V_FUSED][LOGL] = k_qpass_batch<M_FUSED, LOGL, false, false>;
    t[V_FUSED_E][LOGL] = k_qpass_batch<M_FUSED, LOGL, true, false>;
    t[V_SQR][LOGL] = k_qpass_batch<M_FUSED, LOGL, false, true>;
    t[V_SQR_E][LOGL] = k_qpass_batch<M_FUSED, LOGL, true, true>;
}
struct BatchKernelTable {
    QBatchKernel k[NV][MAX_PASS_BITS + 1];
    BatchKernelTable() {
        memset(k, 0, sizeof(k));
        fill_brow<0>(k);
        fill_brow<1>(k);
        fill_brow<2>(k);
        fill_brow<3>(k);
        fill_brow<4>(k);
        fill_brow<5>(k);
        fill_brow<6>(k);
        fill_brow<7>(k);
        fill_brow<8>(k);
        fill_brow<9>(k);
    }
};
static const BatchKernelTable& bktab() {
    static BatchKernelTable t;
    return t;
}

// tile + the 16 x 32 four-step twiddle factors of strided passes; two tiles when merged
static size_t pass_smem(int logl, int variant) {
    const size_t L = (size_t)1 << logl, tile = (size_t)TP * L;
    size_t w = variant == V_FUSED2 ? 2 * tile : tile + TC * 16;
    // staging buffer of the other operand's tile (body_fused, multi-round tiles of <= 8 bits)
    if ((variant == V_FUSED || variant == V_FUSED_E) && logl >= 5 && logl <= 8) w += TC * (L + 4);
    return w * sizeof(u32);
}

// w^e mod q_i (plain form) for the tables' root w of order 2^26, e taken mod 2^26.
static u64 h_root(int i, u64 e) { return h_pow(host_tables().w26[i], e & MASK_N, kQ[i]); }
// (w, floor(w 2^32 / q_i)): w as a Shoup constant.
static uint2 h_shoup(u64 w, int i) { return make_uint2((u32)w, (u32)((w << 32) / kQ[i])); }

static cudaError_t ensure_tables() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    for (int d : done)
        if (d == dev) return cudaSuccess;
    const HostTables& T = host_tables();
    e = cudaMemcpyToSymbol(g_qrt, T.rt.data(), T.rt.size() * sizeof(u32));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(g_qtw, T.tw.data(), T.tw.size() * sizeof(u32));
    if (e != cudaSuccess) return e;
    const KernelTable& K = ktab();
    const BatchKernelTable& BK = bktab();
    for (int v = 0; v < NV; ++v)
        for (int l = 0; l <= MAX_PASS_BITS; ++l)
            for (const void* f : {(const void*)K.k[v][l], (const void*)BK.k[v][l]}) {
                if (!f) continue;
                e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem(l, v));
                if (e != cudaSuccess) return e;
                e = cudaFuncSetAttribute(f, cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
                if (e != cudaSuccess) return e;
            }
    done.push_back(dev);
    return cudaSuccess;
}

// ------------------------------------------------------------------ host: plans and jobs
// Default passes of a 2^n-digit transform: as even as possible, largest first; a strided pass
// leaves at least 32 columns (later passes take >= 5 bits) and takes >= 5 bits itself.
static Plan qplan_default(int n) {
    Plan p;
    memset(&p, 0, sizeof(p));
    p.n = n;
    if (n <= MAX_PASS_BITS) {
        p.passes = 1;
        p.bits[0] = n;
    } else if (n <= 2 * MAX_PASS_BITS) {
        p.passes = 2;
        p.bits[1] = n / 2;
        p.bits[0] = n - n / 2;
    } else {
        p.passes = 3;
        p.bits[0] = (n + 2) / 3;
        p.bits[1] = (n - p.bits[0] + 1) / 2;
        p.bits[2] = n - p.bits[0] - p.bits[1];
    }
    return p;
}

static bool qplan_valid(const Plan& p) {
    if (p.n < 0 || p.n > Q32_MAX_LOG_N || p.passes < 1 || p.passes > MAX_PASSES) return false;
    int sum = 0;
    for (int i = 0; i < p.passes; ++i) {
        if (p.bits[i] < 1 || p.bits[i] > MAX_PASS_BITS) return false;
        sum += p.bits[i];
    }
    if (sum != p.n) return false;
    if (p.passes == 1) return true;
    int rest = p.n;
    for (int i = 0; i + 1 < p.passes; ++i) {
        rest -= p.bits[i];
        if (p.bits[i] < 5 || rest < LOG_TC) return false;   // >= 32 columns per strided tile
    }
    return true;
}

// Plans in effect (tuned or set), per transform length; default otherwise.
static std::mutex g_qplan_mu;
static Plan g_qplan_tab[Q32_MAX_LOG_N + 1];
static bool g_qplan_set[Q32_MAX_LOG_N + 1] = {false};

static Plan qplan(int n) {
    if (n >= 0 && n <= Q32_MAX_LOG_N) {
        std::lock_guard<std::mutex> lk(g_qplan_mu);
        if (g_qplan_set[n]) return g_qplan_tab[n];
    }
    return qplan_default(n);
}

static u64 ceil_pow2(u64 x) {
    u64 r = 1;
    while (r < x) r <<= 1;
    return r;
}
static int ilog2(u64 x) {
    int r = 0;
    while ((1ull << r) < x) ++r;
    return r;
}
static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// How one product runs on this engine.
//   whole: both operands are transformed at the product's length 2^n >= 2 (la + lb) - 1 digits,
//     their last forward passes merged with the pointwise product.
//   split (conv_single reuse, reference src/fast_mul.c:135-212, applied to the long operand):
//     the shorter operand S (ls limbs) is transformed once at a smaller length 2^n; the longer
//     operand is cut into m pieces of cb limbs, each multiplied with S's resident spectrum;
//     every piece's coefficients are accumulated at digit offset 2 k cb into one residue array
//     over the whole product (mod q; consecutive pieces overlap in 2 ls - 1 digits), and one
//     CRT + carry pass turns the sum into limbs.  The sum is the full product's coefficient,
//     which the three primes represent exactly while ls <= 2^25.
//   The plan with the smaller modelled cost wins: (1 + 2m) transforms of 2^n points x (n + 1)
//   (butterfly levels plus one for the per-pass memory work), plus a fixed cost per piece for
//   its launches.
struct QJob {
    bool ok;
    double cost;           // modelled cost in (32-bit points x bits)
    int m;                 // pieces (1: whole product)
    bool swap;             // split: the short operand is the second one
    u64 ls, ll, cb;        // split: short and long lengths, limbs per piece
    int n;
    u64 N;                 // transform length (digits)
    u64 stride;            // split: accumulator digits per prime
    size_t a, b, acc, ticket, state, total;   // workspace offsets (split: a = S's spectrum, b = piece)
    u64 ncta;
    // wrapped (m == 1, wrap > 0): the product's 2 (la + lb) - 1 digit coefficients exceed N, so
    // the transform of length N gives a cyclic convolution whose entries k < wrap hold
    // c_k + c_{k+N}; the product of the lowest lpa / lpb limbs (whole, at 2^nl digits, residue
    // arrays at la_off / lb_off) gives c_0 .. c_{wrap-1}, and the CRT separates the two.
    u64 wrap;
    u64 lpa, lpb;
    int nl;
    u64 NL;
    size_t la_off, lb_off;
    // twisted (wrap > 0): instead of the low product, the product modulo X^NL - c of both whole
    // operands (folded and twisted by k_qtwist_fold), 2^(n - nl) <= 4 folds; see k_qtwist_w
    bool twist;
};

constexpr int kMinSplitLog = 12;           // pieces transform at least 2^12 digits (>= 2 passes)
std::atomic<int> g_force_pieces{0};        // > 1: split every product that allows it into this many pieces
constexpr u64 kMaxPieces = 1ull << 16;
constexpr double kPieceCost = 3.0e7;       // launch overhead of one piece, in (points x bits)
std::atomic<int> g_force_wrap{0};          // tests: wrap every product that allows it

// The wrapped plan of a product of la x lb limbs (see QJob), if the product allows one: both
// operands fit the 2^n-digit cyclic length (2^n < 2 (la + lb) - 1) and the low product is a
// whole product on this engine.  Returns its modelled cost, or a negative value.
static double plan_wrap(u64 la, u64 lb, int sqr, QJob* W) {
    const u64 dc = 2 * (la + lb) - 1;                          // digit coefficients of the product
    const int n = ilog2(dc) - 1;                                // 2^n < dc <= 2^(n+1)
    if (n < 1 || n > Q32_MAX_LOG_N) return -1.0;
    const u64 N = 1ull << n;
    if (2 * la > N || 2 * lb > N) return -1.0;                 // an operand would wrap itself
    const u64 K = dc - N;
    const u64 half = (K + 1) / 2;                               // limbs holding digits 0 .. K-1
    const u64 lpa = la < half ? la : half, lpb = sqr ? lpa : (lb < half ? lb : half);
    const u64 dcl = 2 * (lpa + lpb) - 1;
    const int nl = ilog2(dcl);
    if (nl > Q32_MAX_LOG_N) return -1.0;
    W->wrap = K;
    W->lpa = lpa;
    W->lpb = lpb;
    W->nl = nl;
    W->NL = 1ull << nl;
    W->n = n;
    W->N = N;
    const double t = sqr ? 2.0 : 3.0;
    return t * (double)N * (n + 1) + t * (double)W->NL * (nl + 1) + kPieceCost;
}

// The twisted plan (see QJob and k_qtwist_w): the cyclic product of length N = 2^n and the
// product modulo X^M - c, M = 2^m >= K, N / M <= 4, gamma of order 2N within the primes'
// 2^26-th roots (n <= 25), and a twisted transform of at least two passes.
constexpr int kMinTwistLog = 12;
static double plan_twist(u64 la, u64 lb, int sqr, QJob* W) {
    const u64 dc = 2 * (la + lb) - 1;
    const int n = ilog2(dc) - 1;
    if (n < kMinTwistLog || n > Q32_MAX_LOG_N - 1) return -1.0;
    const u64 N = 1ull << n;
    if (2 * la > N || 2 * lb > N) return -1.0;
    const u64 K = dc - N;
    int m = ilog2(K);
    if (m < n - 2) m = n - 2;                                   // at most kMaxFolds folds
    if (m < kMinTwistLog) m = kMinTwistLog;
    if (m > n) return -1.0;
    W->wrap = K;
    W->twist = true;
    W->nl = m;
    W->NL = 1ull << m;
    W->n = n;
    W->N = N;
    const double t = sqr ? 2.0 : 3.0, F = (double)(1 << (n - m));
    // the fold kernels and the W kernel: memory passes over F digits / residues per point,
    // about one butterfly level each
    return t * (double)N * (n + 1) + t * (double)W->NL * (m + 1) + (sqr ? 1.0 : 2.0) * (double)W->NL * F +
           (double)K * F + kPieceCost;
}

static QJob plan_job(u64 la, u64 lb, int sqr) {
    QJob J;
    memset(&J, 0, sizeof(J));
    const u64 out_len = la + lb;
    if (la == 0 || lb == 0) return J;
    double best = 1e300;
    if (out_len <= (1ull << (Q32_MAX_LOG_N - 1))) {             // whole: 2 out_len - 1 <= 2^26
        J.ok = true;
        J.m = 1;
        J.N = ceil_pow2(2 * out_len - 1);
        J.n = ilog2(J.N);
        best = (sqr ? 2.0 : 3.0) * (double)J.N * (J.n + 1);
    }
    const u64 ls = la < lb ? la : lb, ll = la < lb ? lb : la;
    const int force = g_force_pieces.load();
    if (force > 1 && !sqr && ls <= (1ull << (Q32_MAX_LOG_N - 1)) && ll >= (u64)force) {
        const u64 cb = (ll + force - 1) / force;
        const u64 m = (ll + cb - 1) / cb;
        int n = ilog2(2 * (ls + cb) - 1);
        if (n < kMinSplitLog) n = kMinSplitLog;
        if (m >= 2 && n <= Q32_MAX_LOG_N) {
            best = -1.0;                                        // forced: wins over every other plan
            J.ok = true;
            J.m = (int)m;
            J.swap = lb < la;
            J.ls = ls;
            J.ll = ll;
            J.cb = cb;
            J.n = n;
            J.N = 1ull << n;
        }
    }
    if (!sqr && best >= 0.0 && ls <= (1ull << (Q32_MAX_LOG_N - 1))) {
        for (int n = kMinSplitLog; n <= Q32_MAX_LOG_N; ++n) {
            const u64 half = 1ull << (n - 1);                   // piece product: ls + cb <= 2^(n-1) limbs
            if (half <= ls) continue;
            const u64 cbmax = half - ls;
            u64 m = (ll + cbmax - 1) / cbmax;
            if (m < 2 || m > kMaxPieces) continue;
            const u64 cb = (ll + m - 1) / m;
            m = (ll + cb - 1) / cb;                             // no empty last piece
            if (m < 2) continue;
            const double cost = (1.0 + 2.0 * (double)m) * (double)(1ull << n) * (n + 1) + (double)m * kPieceCost;
            if (cost < best) {
                best = cost;
                J.ok = true;
                J.m = (int)m;
                J.swap = lb < la;
                J.ls = ls;
                J.ll = ll;
                J.cb = cb;
                J.n = n;
                J.N = 1ull << n;
            }
        }
    }
    // wrapped plans: the low product (force 1) or the twisted product (force 2)
    const int fw = g_force_wrap.load();
    for (int kind = 1; kind <= 2 && best >= 0.0; ++kind) {
        QJob W;
        memset(&W, 0, sizeof(W));
        const double cw = kind == 1 ? plan_wrap(la, lb, sqr, &W) : plan_twist(la, lb, sqr, &W);
        if (cw >= 0.0 && (fw ? fw == kind : cw < best)) {
            best = cw;
            J = W;
            J.ok = true;
            J.m = 1;
        }
    }
    if (!J.ok) return J;
    J.cost = best;
    J.ncta = (out_len + QCTILE - 1) / QCTILE;
    size_t off = 256;
    J.a = off;
    off = align256(off + 3 * J.N * sizeof(u32));
    J.b = off;
    if (!(J.m == 1 && sqr)) off = align256(off + 3 * J.N * sizeof(u32));
    if (J.wrap) {
        J.la_off = off;
        off = align256(off + 3 * J.NL * sizeof(u32));
        J.lb_off = off;
        if (!sqr) off = align256(off + 3 * J.NL * sizeof(u32));
    }
    if (J.m > 1) {
        J.stride = (2 * out_len + 63) & ~63ull;
        J.acc = off;
        off = align256(off + 3 * J.stride * sizeof(u32));
    }
    J.ticket = off;
    J.state = off + 16;
    off = align256(J.state + J.ncta * sizeof(u32));
    J.total = off;
    return J;
}

// A product with a 32-bit resident spectrum of 2^log_n digits: [status][partner / product
// residues][ticket + state].
static QJob plan_resident(const Job& j) {
    QJob J;
    memset(&J, 0, sizeof(J));
    const u64 out_len = j.la + j.lb;
    if (j.la == 0 || j.lb == 0 || j.log_n < 1 || j.log_n > Q32_MAX_LOG_N || 2 * out_len - 1 > (1ull << j.log_n))
        return J;
    J.ok = true;
    J.m = 1;
    J.n = j.log_n;
    J.N = 1ull << j.log_n;
    J.ncta = (out_len + QCTILE - 1) / QCTILE;
    size_t off = 256;
    J.a = J.b = off;
    off = align256(off + 3 * J.N * sizeof(u32));
    J.ticket = off;
    J.state = off + 16;
    off = align256(J.state + J.ncta * sizeof(u32));
    J.total = off;
    return J;
}

// Launch sequencing of one product on one stream: kernel lookup, the caller's hook that makes
// the stream wait for a range of the second operand's limbs, per-launch timing records.
struct Launcher {
    const Job& j;
    cudaStream_t s;
    NeedLimbs need_b;
    void* need_ctx;

    cudaError_t need(u64 first, u64 end) { return need_b ? need_b(need_ctx, first, end, s) : cudaSuccess; }
    cudaError_t operator()(int variant, int logl, const QArgs& a, u64 tiles) {
        QKernel k = ktab().k[variant][logl];
        if (!k) return cudaErrorInvalidValue;
        cudaError_t e;
        // work of this launch's own transform (a.N: the twisted or low sub-product of a wrapped
        // product is shorter than the product's main transform)
        const double Nl = (double)a.N, vec = 3.0 * Nl * 4.0, bfly = 3.0 * (Nl / 2.0) * logl;
        const bool entry = (variant == V_FWD_E || variant == V_LAST_E || variant == V_FUSED_E || variant == V_SQR_E);
        double bytes = entry ? (double)a.len * 8.0 + vec : 2.0 * vec, mm = bfly + (entry ? 6.0 * (double)a.len : 0.0);
        int kind = K_FUSED;
        if (variant == V_FWD || variant == V_FWD_E) kind = K_FWD;
        else if (variant == V_LAST || variant == V_LAST_E) kind = K_FWD_LAST;
        else if (variant == V_INV || variant == V_INV_ACC) kind = K_INV;
        if (variant == V_FUSED2) {
            bytes += vec;
            mm = 3.0 * bfly + 3.0 * Nl;
        } else if (kind == K_FUSED) {
            if (variant == V_FUSED || variant == V_FUSED_E) bytes += vec;
            mm = 2.0 * bfly + 3.0 * Nl + (entry ? 6.0 * (double)a.len : 0.0);
        }
        const ProfMark m = prof_begin(kind, bytes, mm, s);
        k<<<(unsigned)(tiles * 3), NT, pass_smem(logl, variant), s>>>(a);
        e = cudaGetLastError();
        prof_end(m, s);
        return e;
    }
};

// CRT constants for residues that went through a 2^n-point transform (see QCrtArgs).
static void crt_constants(u64 N, QCrtArgs* ca) {
    for (int i = 0; i < 3; ++i) {
        const u64 p = kQ[i];
        const u64 ninv = h_pow(N % p, p - 2, p);
        ca->cst[i] = (u32)h_mulmod(ninv, h_pow(2, 64, p), p);
    }
    const u64 q0 = kQ[0], q1 = kQ[1], q2 = kQ[2];
    auto mont = [](u64 v, u64 p) { return (u32)h_mulmod(v % p, h_pow(2, 32, p), p); };
    ca->inv01 = mont(h_pow(q0 % q1, q1 - 2, q1), q1);
    ca->q0m2 = mont(q0, q2);
    ca->inv012 = mont(h_pow(h_mulmod(q0, q1, q2), q2 - 2, q2), q2);
}

// Launch list of a whole product: a 2^n-digit transform of both operands in scratch A and B
// (B unused for a square), the product left in A in natural order for the CRT.
struct QRec {
    int variant, logl;
    QArgs a;
    u64 tiles;
};
struct QWhole {
    int count;
    QRec rec[3 * MAX_PASSES + 2];
};

// ---- four-step twiddle tables of strided passes: w_B^(+-i k) as Shoup pairs for every column
// i and frequency k of a pass over blocks of B = 2^logB <= 2^TW_MAX_LOGB digits (B entries per
// prime and direction, 8 MB at most), so such a pass multiplies each digit by one table entry
// read from L2 instead of forming the twiddle from two Montgomery products.
constexpr int TW_MAX_LOGB = 20;

__global__ void __launch_bounds__(256) k_qtw_build(uint2* T, int logB, int logS, int inv) {
    const int pi = blockIdx.y;
    const PrimeQ q = c_q[pi];
    const u32 B = 1u << logB;
    for (u32 e = blockIdx.x * blockDim.x + threadIdx.x; e < B; e += gridDim.x * blockDim.x) {
        const u32 k = e >> logS, i = e & ((1u << logS) - 1);
        u32 x = (i * k) << (Q32_MAX_LOG_N - logB);              // i k < B: w_B^(i k) = w_2^26^x
        if (inv) x = (0u - x) & MASK_N;
        const u32 w = qmont(qroot(x, pi, q), 1u, q);             // out of Montgomery form
        T[(u64)pi * B + e] = make_uint2(w, (u32)(((u64)w << 32) / q.p));
    }
}

struct TwPass {
    const uint2* fwd = nullptr;
    const uint2* inv = nullptr;
};
struct TwEntry {
    int dev, logB, logl;
    uint2* buf;
};
static std::mutex g_tw_mu;
static std::vector<TwEntry> g_tw;

// The tables of a strided pass of 2^logl rows over 2^logB-digit blocks on the current device:
// built on s and finished the first time (not while s is being captured into a graph, nor
// beyond TW_MAX_LOGB); empty when unavailable, and the pass then computes its twiddles.
static TwPass tw_tables(int logB, int logl, cudaStream_t s) {
    TwPass r;
    if (logB > TW_MAX_LOGB) return r;
    int dev = 0;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        return r;
    }
    const size_t per = (size_t)3 << logB;
    std::lock_guard<std::mutex> lk(g_tw_mu);
    for (const TwEntry& t : g_tw)
        if (t.dev == dev && t.logB == logB && t.logl == logl) {
            r.fwd = t.buf;
            r.inv = t.buf + per;
            return r;
        }
    if (cap != cudaStreamCaptureStatusNone) return r;
    uint2* buf = nullptr;
    if (cudaMalloc(&buf, 2 * per * sizeof(uint2)) != cudaSuccess) {
        cudaGetLastError();
        return r;
    }
    const unsigned bx = (unsigned)(((1ull << logB) + 255) / 256 < 1024 ? ((1ull << logB) + 255) / 256 : 1024);
    k_qtw_build<<<dim3(bx, 3), 256, 0, s>>>(buf, logB, logB - logl, 0);
    k_qtw_build<<<dim3(bx, 3), 256, 0, s>>>(buf + per, logB, logB - logl, 1);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(s) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(buf);
        return r;
    }
    g_tw.push_back(TwEntry{dev, logB, logl, buf});
    r.fwd = buf;
    r.inv = buf + per;
    return r;
}

// `batched`: the product is one of a batch whose launches are shared.  The tuned plans are the
// fastest for one product on the GPU at a time; in a batch, where many products' tiles fill
// the GPU together, the default (even) plans are faster (4096 products of 1k-100k limbs:
// 137k against 104k products/s on B200).
// `tws`: per pass, its twiddle tables (null: computed in the kernels).
// prefolded: the operands' residues are already in A and B (a twisted product, written by
// k_qtwist_fold), so the first pass reads them instead of the limbs.
static void plan_whole(const Job& j, int n, u32* A, u32* B, QWhole* out, bool batched = false,
                       const TwPass* tws = nullptr, bool prefolded = false) {
    const int sqr = j.sqr ? 1 : 0;
    if (sqr || j.spectrum) B = A;
    const Plan pl = j.spectrum && j.splan.passes ? j.splan                 // a spectrum keeps its plan
                    : batched                    ? qplan_default(n)
                                                 : qplan(n);
    const int P = pl.passes;
    const u64 N = 1ull << n;
    int logB[MAX_PASSES];
    logB[0] = n;
    for (int p = 1; p < P; ++p) logB[p] = logB[p - 1] - pl.bits[p - 1];
    const int lastl = pl.bits[P - 1];
    const u64 nblk_last = N >> lastl;
    const u64 tiles_last = (nblk_last + TC - 1) / TC;
    const int ncols_last = nblk_last < (u64)TC ? (int)nblk_last : TC;
    out->count = 0;
    QArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.N = N;
    pa.ncols = TC;
    auto add = [&](int variant, int logl, u64 tiles) {
        QRec& r = out->rec[out->count++];
        r.variant = variant;
        r.logl = logl;
        r.a = pa;
        r.tiles = tiles;
    };
    auto fwd_strided = [&](const u64* src, u64 len, u32* data) {
        for (int p = 0; p + 1 < P; ++p) {
            pa.src = src;
            pa.len = len;
            pa.data = data;
            pa.logB = logB[p];
            pa.tw = tws ? tws[p].fwd : nullptr;
            add(p == 0 && !prefolded ? V_FWD_E : V_FWD, pl.bits[p], N >> (pl.bits[p] + LOG_TC));
        }
        pa.tw = nullptr;
    };
    const bool merged = !sqr && !j.spectrum && P >= 2 && lastl >= 5 && lastl <= 8;
    if (j.spectrum) {
        // resident first operand (conv_single, src/fast_mul.c:135-212): only the partner is
        // transformed, in A; the product goes back into A, the spectrum stays intact
        fwd_strided(j.b, j.lb, A);
        pa.src = j.b;
        pa.len = j.lb;
        pa.data = A;
        pa.other = (u32*)j.spectrum;
        pa.dst = A;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_FUSED_E : V_FUSED, lastl, tiles_last);
        pa.dst = nullptr;
    } else if (merged) {
        fwd_strided(j.a, j.la, A);
        fwd_strided(j.b, j.lb, B);
        pa.src = nullptr;
        pa.len = 0;
        pa.data = B;
        pa.other = A;
        pa.logB = logB[P - 1];
        pa.ncols = TC;
        add(V_FUSED2, lastl, tiles_last);
    } else if (!sqr) {
        fwd_strided(j.a, j.la, A);
        pa.src = j.a;
        pa.len = j.la;
        pa.data = A;
        pa.other = nullptr;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_LAST_E : V_LAST, lastl, tiles_last);
        pa.ncols = TC;
        fwd_strided(j.b, j.lb, B);
        pa.src = j.b;
        pa.len = j.lb;
        pa.data = B;
        pa.other = A;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_FUSED_E : V_FUSED, lastl, tiles_last);
    } else {
        fwd_strided(j.a, j.la, A);
        pa.src = j.a;
        pa.len = j.la;
        pa.data = A;
        pa.other = A;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_SQR_E : V_SQR, lastl, tiles_last);
    }
    pa.src = nullptr;
    pa.len = 0;
    pa.other = nullptr;
    pa.ncols = TC;
    for (int p = P - 2; p >= 0; --p) {
        pa.data = A;
        pa.logB = logB[p];
        pa.tw = tws ? tws[p].inv : nullptr;
        add(V_INV, pl.bits[p], N >> (pl.bits[p] + LOG_TC));
    }
}

// Transform length (log2 digits) of a whole product, -1 if it has none on this engine.
static int whole_log_n(u64 la, u64 lb) {
    const u64 out_len = la + lb;
    if (la == 0 || lb == 0 || out_len > (1ull << (Q32_MAX_LOG_N - 1))) return -1;
    return ilog2(2 * out_len - 1);
}

}  // namespace q32

bool q32_fits(u64 la, u64 lb, int sqr) { return q32::plan_job(la, lb, sqr).ok; }

void q32_release_tables(int dev) {
    using namespace q32;
    std::lock_guard<std::mutex> lk(g_tw_mu);
    for (size_t k = 0; k < g_tw.size();) {
        if (g_tw[k].dev == dev) {
            cudaFree(g_tw[k].buf);
            g_tw.erase(g_tw.begin() + k);
        } else {
            ++k;
        }
    }
}

cudaError_t q32_prepare_tables() {
    using namespace q32;
    cudaError_t e = q32::ensure_tables();
    if (e != cudaSuccess) return e;
    for (int n = 1; n <= Q32_MAX_LOG_N; ++n) {
        const Plan pl = qplan(n);
        int logB = n;
        for (int p = 0; p + 1 < pl.passes; ++p) {
            tw_tables(logB, pl.bits[p], 0);          // legacy stream: finished before returning
            logB -= pl.bits[p];
        }
    }
    return cudaGetLastError();
}

void q32_force_pieces(int m) { q32::g_force_pieces.store(m > 1 ? m : 0); }

Plan q32_make_plan(int log_n) { return q32::qplan(log_n); }
Plan q32_default_plan(int log_n) { return q32::qplan_default(log_n); }
bool q32_valid_plan(const Plan& p) { return q32::qplan_valid(p); }

bool q32_set_plan(const Plan& p) {
    if (!q32::qplan_valid(p)) return false;
    std::lock_guard<std::mutex> lk(q32::g_qplan_mu);
    q32::g_qplan_tab[p.n] = p;
    q32::g_qplan_set[p.n] = true;
    return true;
}

void q32_clear_plan(int log_n) {
    if (log_n < 0 || log_n > Q32_MAX_LOG_N) return;
    std::lock_guard<std::mutex> lk(q32::g_qplan_mu);
    q32::g_qplan_set[log_n] = false;
}

std::vector<Plan> q32_candidate_plans(int n) {
    std::vector<Plan> out;
    if (n < 1 || n > Q32_MAX_LOG_N) return out;
    if (n <= MAX_PASS_BITS) {
        out.push_back(q32::qplan_default(n));
        return out;
    }
    const int p0 = (n + MAX_PASS_BITS - 1) / MAX_PASS_BITS;
    for (int P = p0; P <= p0 + 1 && P <= 3; ++P) {
        int b[MAX_PASSES] = {0};
        auto rec = [&](auto&& self, int i, int left) -> void {
            if (i >= MAX_PASSES) return;
            if (i == P - 1) {
                if (left < 1 || left > MAX_PASS_BITS) return;
                b[i] = left;
                Plan p;
                memset(&p, 0, sizeof(p));
                p.n = n;
                p.passes = P;
                for (int k = 0; k < P; ++k) p.bits[k] = b[k];
                if (q32::qplan_valid(p)) out.push_back(p);
                return;
            }
            for (int m = 5; m <= MAX_PASS_BITS; ++m) {
                b[i] = m;
                self(self, i + 1, left - m);
            }
        };
        rec(rec, 0, n);
    }
    return out;
}

size_t q32_job_workspace_bytes(const Job& j) {
    if (!j.spectrum) return q32_workspace_bytes(j.la, j.lb, j.sqr ? 1 : 0);
    const q32::QJob J = q32::plan_resident(j);
    return J.ok ? J.total : 256;
}

int q32_spectrum_log_n(u64 len, u64 max_partner) {
    if (len == 0 || max_partner == 0 || len + max_partner > (1ull << (Q32_MAX_LOG_N - 1))) return -1;
    return q32::ilog2(2 * (len + max_partner) - 1);
}

cudaError_t q32_spectrum_enqueue(const u64* src, u64 len, int log_n, void* spec, cudaStream_t s, const Plan& pl) {
    using namespace q32;
    cudaError_t e = q32::ensure_tables();
    if (e != cudaSuccess) return e;
    if (!qplan_valid(pl) || pl.n != log_n) return cudaErrorInvalidValue;
    const int P = pl.passes;
    const u64 N = 1ull << log_n;
    const Job j{};
    Launcher launch{j, s, nullptr, nullptr};
    QArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.N = N;
    pa.ncols = TC;
    pa.src = src;
    pa.len = len;
    pa.data = (u32*)spec;
    int logB = log_n;
    for (int p = 0; p + 1 < P; ++p) {
        pa.logB = logB;
        if ((e = launch(p == 0 ? V_FWD_E : V_FWD, pl.bits[p], pa, N >> (pl.bits[p] + LOG_TC))) != cudaSuccess) return e;
        logB -= pl.bits[p];
    }
    const int lastl = pl.bits[P - 1];
    const u64 nblk = N >> lastl;
    pa.logB = logB;
    pa.ncols = nblk < (u64)TC ? (int)nblk : TC;
    return launch(P == 1 ? V_LAST_E : V_LAST, lastl, pa, (nblk + TC - 1) / TC);
}

double q32_cost(u64 la, u64 lb, int sqr) {
    const q32::QJob J = q32::plan_job(la, lb, sqr);
    return J.ok ? J.cost : 1e300;
}

size_t q32_workspace_bytes(u64 la, u64 lb, int sqr) {
    const q32::QJob J = q32::plan_job(la, lb, sqr);
    return J.ok ? J.total : 256;
}

int q32_launches(u64 la, u64 lb, int sqr) {
    const q32::QJob J = q32::plan_job(la, lb, sqr);
    if (!J.ok) return 0;
    // transform launches of a whole product at 2^n digits (plan_whole), without the CRT
    auto whole = [sqr](int n) {
        const Plan pl = q32::qplan(n);
        const int P = pl.passes;
        const int lastl = pl.bits[P - 1];
        if (!sqr && P >= 2 && lastl >= 5 && lastl <= 8) return 2 * (P - 1) + 1 + (P - 1);
        return sqr ? (P - 1) + 1 + (P - 1) : 2 * (P - 1) + 1 + 1 + (P - 1);
    };
    if (J.m > 1) {
        const int P = q32::qplan(J.n).passes;
        return P + J.m * ((P - 1) + 1 + (P - 1)) + 1;
    }
    return whole(J.n) + (J.wrap ? whole(J.nl) + (J.twist ? (sqr ? 2 : 3) : 0) : 0) + 1;   // + folds and W
}

void q32_force_wrap(int mode) { q32::g_force_wrap.store(mode == 1 || mode == 2 ? mode : 0); }

u64 q32_twisted(u64 la, u64 lb, int sqr) {
    const q32::QJob J = q32::plan_job(la, lb, sqr);
    return J.ok && J.twist ? J.NL : 0;
}

u64 q32_wrapped(u64 la, u64 lb, int sqr) {
    const q32::QJob J = q32::plan_job(la, lb, sqr);
    return J.ok ? J.wrap : 0;
}

int q32_pieces(u64 la, u64 lb, int sqr) {
    const q32::QJob J = q32::plan_job(la, lb, sqr);
    return J.ok ? J.m : 0;
}

// ---- batches: products grouped by transform length(s) and kind share every launch
namespace q32 {
// A batched product runs twisted (see plan_twist) when that plan, without the per-sequence
// launch cost (a batch shares its launches among its products), models at least 15% cheaper
// than the whole product: a twisted group adds its fold, W and CRT launches, so a negacyclic
// plan (M = 2^n, about the whole product's cost) stays whole.  Returns the twisted plan
// (T->ok) or leaves T->ok false.
static void batch_twist_plan(const Job& j, QJob* T) {
    memset(T, 0, sizeof(*T));
    if (j.spectrum || j.la == 0 || j.lb == 0) return;
    const int fw = g_force_wrap.load();
    if (fw == 1) return;                                         // tests: the low-product form (none in batches)
    const int sqr = j.sqr ? 1 : 0, nw = whole_log_n(j.la, j.lb);
    if (nw < 0) return;
    const double ct = plan_twist(j.la, j.lb, sqr, T);
    const double cw = (sqr ? 2.0 : 3.0) * (double)(1ull << nw) * (nw + 1);
    T->ok = ct >= 0.0 && (fw == 2 || ct - kPieceCost < 0.85 * cw);
}
}  // namespace q32

int q32_forced_wrap() { return q32::g_force_wrap.load(); }

int q32_batch_twist_log(const Job& j) {
    q32::QJob T;
    q32::batch_twist_plan(j, &T);
    return T.ok ? T.nl : 0;
}

int q32_batch_log_n(const Job& j) {
    if (j.spectrum) return j.engine == ENGINE_32 && q32::plan_resident(j).ok ? j.log_n : -1;
    q32::QJob T;
    q32::batch_twist_plan(j, &T);
    return T.ok ? T.n : q32::whole_log_n(j.la, j.lb);
}

size_t q32_batch_res_bytes(const Job& j) {
    const int n = q32_batch_log_n(j);
    if (n < 0) return 0;
    const int ops = j.sqr || j.spectrum ? 1 : 2, m = q32_batch_twist_log(j);
    return (q32::align256(3 * (1ull << n) * sizeof(u32)) + (m ? q32::align256(3 * (1ull << m) * sizeof(u32)) : 0)) * ops;
}

size_t q32_batch_state_bytes(const Job& j) {
    const u64 ncta = (j.la + j.lb + q32::QCTILE - 1) / q32::QCTILE;
    return 16 + ((ncta * sizeof(u32) + 15) & ~(size_t)15);
}

size_t q32_batch_desc_bytes_per_job() {
    return Q32_MAX_REC * (sizeof(q32::QArgs) + 16) + 2 * (sizeof(q32::QFoldArgs) + 16) + sizeof(q32::QTwistArgs) +
           sizeof(q32::QCrtArgs) + sizeof(u32) + 64;
}

cudaError_t q32_prepare() { return q32::ensure_tables(); }

cudaError_t q32_batch_plan(const Job* jobs, const int* idx, int m, char* res, size_t* roff, char* st, size_t* soff,
                           u32* err, char* h, size_t* hoff, size_t hcap, Q32Group* g) {
    using namespace q32;
    if (m <= 0) return cudaErrorInvalidValue;
    auto reserve = [&](size_t bytes) -> size_t {
        const size_t o = *hoff;
        *hoff = (*hoff + bytes + 15) & ~(size_t)15;
        return o;
    };
    std::vector<QWhole> W(m), WT(m);
    std::vector<QCrtArgs> C(m);
    std::vector<QFoldArgs> FA(m), FB(m);
    std::vector<QTwistArgs> TW(m);
    std::vector<u32> nc(m);
    u32 maxc = 0;
    const int n = q32_batch_log_n(jobs[idx[0]]);
    const int tm = q32_batch_twist_log(jobs[idx[0]]);            // 0: whole products
    if (n < 0) return cudaErrorInvalidValue;
    const u64 N = 1ull << n, M = tm ? 1ull << tm : 0;
    const int tw_log = Q32_MAX_LOG_N - 1 - n, fold_log = tm ? n - tm : 0;
    QCrtArgs proto;
    memset(&proto, 0, sizeof(proto));
    crt_constants(N, &proto);
    // twisted: the constants of the folds and of the W kernel are the same for the whole group
    QFoldArgs fproto;
    QTwistArgs tproto;
    memset(&fproto, 0, sizeof(fproto));
    memset(&tproto, 0, sizeof(tproto));
    u64 kmax = 0;
    if (tm) {
        fproto.logM = tproto.logM = tm;
        fproto.fold_log = tproto.fold_log = fold_log;
        fproto.tw_log = tproto.tw_log = tw_log;
        QCrtArgs cm;
        memset(&cm, 0, sizeof(cm));
        crt_constants(M, &cm);
        for (int i = 0; i < 3; ++i) {
            const u64 p = kQ[i];
            const u64 r32 = h_pow(2, 32, p), ninv = h_pow(N % p, p - 2, p);
            tproto.cstM[i] = cm.cst[i];
            for (int jj = 0; jj < kMaxFolds; ++jj) {
                const u64 c = h_root(i, (u64)jj << (tm + tw_log));
                fproto.cpow[i][jj] = h_shoup(c, i);
                tproto.ucj[i][jj] = h_shoup(h_mulmod(h_mulmod(c, ninv, p), r32, p), i);
            }
            tproto.nraw[i] = h_shoup(h_mulmod(N % p, h_pow(r32, p - 2, p), p), i);
        }
        tproto.N = (u32)N;
    }
    for (int t = 0; t < m; ++t) {
        const Job& j = jobs[idx[t]];
        if (q32_batch_log_n(j) != n || q32_batch_twist_log(j) != tm) return cudaErrorInvalidValue;
        const u64 out_len = j.la + j.lb;
        const bool one = j.sqr || j.spectrum;
        u32* A = (u32*)(res + *roff);
        *roff += align256(3 * N * sizeof(u32));
        u32* B = A;
        if (!one) {
            B = (u32*)(res + *roff);
            *roff += align256(3 * N * sizeof(u32));
        }
        u32* ticket = (u32*)(st + *soff);
        *soff += q32_batch_state_bytes(j);
        QCrtArgs& ca = C[t];
        ca = proto;
        if (tm) {
            u32* TA = (u32*)(res + *roff);
            *roff += align256(3 * M * sizeof(u32));
            u32* TB = TA;
            if (!one) {
                TB = (u32*)(res + *roff);
                *roff += align256(3 * M * sizeof(u32));
            }
            FA[t] = fproto;
            FA[t].src = j.a;
            FA[t].len = j.la;
            FA[t].T = TA;
            FB[t] = fproto;
            FB[t].src = j.b;
            FB[t].len = j.lb;
            FB[t].T = TB;
            plan_whole(j, tm, TA, TB, &WT[t], true, nullptr, true);
            const u64 K = 2 * out_len - 1 - N;
            TW[t] = tproto;
            TW[t].U = A;
            TW[t].V = TA;
            TW[t].K = (u32)K;
            if (K > kmax) kmax = K;
            ca.low = TA;
            ca.low_N = M;
            ca.wrap = K;
            ca.twisted = 1;
            for (int i = 0; i < 3; ++i) ca.low_cst[i] = c_host_r1(i);
        }
        plan_whole(j, n, A, B, &W[t], true);
        ca.res = A;
        ca.N = N;
        ca.nvalid = 2 * out_len - 1;
        ca.out = j.out;
        ca.out_len = out_len;
        ca.ticket = ticket;
        ca.state = ticket + 4;
        ca.err = err;
        nc[t] = (u32)((out_len + QCTILE - 1) / QCTILE);
        if (nc[t] > maxc) maxc = nc[t];
        if (W[t].count != W[0].count || (tm && WT[t].count != WT[0].count)) return cudaErrorInvalidValue;
    }
    const bool sq = jobs[idx[0]].sqr || jobs[idx[0]].spectrum;
    g->m = m;
    g->twist = tm;
    g->nfold = tm ? (sq ? 1 : 2) : 0;
    g->count = (tm ? WT[0].count : 0) + W[0].count;
    if (g->count > Q32_MAX_REC) return cudaErrorInvalidValue;
    g->max_ncta = maxc;
    for (int k = 0; k < g->count; ++k) {
        const bool tk = tm && k < WT[0].count;                  // a launch of the twisted transform
        const QWhole* src = tk ? WT.data() : W.data();
        const int kk = tk ? k : k - (tm ? WT[0].count : 0);
        g->variant[k] = src[0].rec[kk].variant;
        g->logl[k] = src[0].rec[kk].logl;
        g->tiles[k] = src[0].rec[kk].tiles;
        g->args_off[k] = reserve((size_t)m * sizeof(QArgs));
        if (*hoff > hcap) return cudaErrorInvalidValue;
        QArgs* d = (QArgs*)(h + g->args_off[k]);
        for (int t = 0; t < m; ++t) d[t] = src[t].rec[kk].a;
    }
    if (tm) {
        g->fold_bpj = (unsigned)std::min<u64>((M + 255) / 256, 128);
        g->w_bpj = (unsigned)std::min<u64>((kmax + 255) / 256, 128);
        g->fold_off[0] = reserve((size_t)m * sizeof(QFoldArgs));
        g->fold_off[1] = reserve((size_t)m * sizeof(QFoldArgs));
        g->w_off = reserve((size_t)m * sizeof(QTwistArgs));
        if (*hoff > hcap) return cudaErrorInvalidValue;
        memcpy(h + g->fold_off[0], FA.data(), (size_t)m * sizeof(QFoldArgs));
        memcpy(h + g->fold_off[1], FB.data(), (size_t)m * sizeof(QFoldArgs));
        memcpy(h + g->w_off, TW.data(), (size_t)m * sizeof(QTwistArgs));
    }
    g->crt_off = reserve((size_t)m * sizeof(QCrtArgs));
    g->ncta_off = reserve((size_t)m * sizeof(u32));
    if (*hoff > hcap) return cudaErrorInvalidValue;
    memcpy(h + g->crt_off, C.data(), (size_t)m * sizeof(QCrtArgs));
    memcpy(h + g->ncta_off, nc.data(), (size_t)m * sizeof(u32));
    return cudaSuccess;
}

cudaError_t q32_batch_launch(const Q32Group& g, const char* d_desc, cudaStream_t s) {
    using namespace q32;
    const BatchKernelTable& BK = bktab();
    cudaError_t e;
    for (int f = 0; f < g.nfold; ++f) {
        k_qtwist_fold_batch<<<(unsigned)g.m * g.fold_bpj, 256, 0, s>>>((const QFoldArgs*)(d_desc + g.fold_off[f]),
                                                                       g.fold_bpj);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    for (int k = 0; k < g.count; ++k) {
        QBatchKernel kk = BK.k[g.variant[k]][g.logl[k]];
        if (!kk) return cudaErrorInvalidValue;
        const unsigned grid = (unsigned)((u64)g.m * g.tiles[k] * 3);
        kk<<<grid, NT, pass_smem(g.logl[k], g.variant[k]), s>>>((const QArgs*)(d_desc + g.args_off[k]),
                                                                (u32)g.tiles[k]);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (g.twist) {
        k_qtwist_w_batch<<<dim3((unsigned)g.m * g.w_bpj, 3), 256, 0, s>>>((const QTwistArgs*)(d_desc + g.w_off), g.w_bpj);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        k_qcrt_carry_twist_batch<<<(unsigned)(g.m * g.max_ncta), CNT, 0, s>>>(
            (const QCrtArgs*)(d_desc + g.crt_off), g.max_ncta, (const u32*)(d_desc + g.ncta_off));
        return cudaGetLastError();
    }
    k_qcrt_carry_batch<<<(unsigned)(g.m * g.max_ncta), CNT, 0, s>>>((const QCrtArgs*)(d_desc + g.crt_off), g.max_ncta,
                                                                    (const u32*)(d_desc + g.ncta_off));
    return cudaGetLastError();
}

// ---- butterfly throughput microbenchmark (the peak the 32-bit pass kernels are held against)
namespace q32 {
constexpr int BB_CHAINS = 8, BB_ITERS = 4096;
__global__ void __launch_bounds__(256) k_bench_qbfly(u32* sink, uint2 w) {
    const PrimeQ q = c_q[0];
    u32 x[2 * BB_CHAINS];
#pragma unroll
    for (int i = 0; i < 2 * BB_CHAINS; ++i) x[i] = ((blockIdx.x * 256 + threadIdx.x) * 2654435761u + i * 97u) % q.p;
#pragma unroll 1
    for (int it = 0; it < BB_ITERS; ++it) {
#pragma unroll
        for (int i = 0; i < BB_CHAINS; ++i) qbfly_dif(x[i], x[i + BB_CHAINS], w, q);
    }
    u32 acc = 0;
#pragma unroll
    for (int i = 0; i < 2 * BB_CHAINS; ++i) acc ^= x[i];
    if (acc == 0x12345u) sink[0] = acc;
}
}  // namespace q32

cudaError_t q32_bench_bfly(double* per_second) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    u32* sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, 64);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const u32 w0 = 1234567u;
    const uint2 w = make_uint2(w0, (u32)(((u64)w0 << 32) / Q32_P0));
    const unsigned grid = (unsigned)sms * 8;
    float best = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(a);
        q32::k_bench_qbfly<<<grid, 256>>>(sink, w);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, a, b);
        if (rep && ms < best) best = ms;
    }
    e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    *per_second = (double)grid * 256.0 * q32::BB_CHAINS * q32::BB_ITERS / (best * 1e-3);
    return e;
}

namespace q32 {
// The CRT arguments of a product whose residues are in ca->res (stride ca->N).
static void fill_crt(const Job& j, const QJob& J, char* base, u64 out_len, QCrtArgs* ca) {
    ca->nvalid = 2 * out_len - 1;
    ca->out = j.out;
    ca->out_len = out_len;
    ca->state = (u32*)(base + J.state);
    ca->ticket = (u32*)(base + J.ticket);
    ca->err = (u32*)base;
}

// CRT + carry CTAs [t0, t1) of ncta (tickets continue from earlier launches), then the
// caller's copy-back hook for the limbs they finish.
static cudaError_t crt_launch(const QCrtArgs& ca, u64 ncta, u64 t0, u64 t1, cudaStream_t s, ChunkDone after_chunk,
                              void* ctx) {
    const u64 n = t1 - t0;
    const double crt_bytes = 3.0 * (double)ca.nvalid * 4.0 + (double)ca.out_len * 8.0;
    const ProfMark m = prof_begin(K_CRT, crt_bytes * (double)n / (double)ncta, 3.0 * (double)ca.nvalid * (double)n / (double)ncta, s);
    if (ca.wrap && ca.twisted) k_qcrt_carry_twist<<<(unsigned)n, CNT, 0, s>>>(ca);
    else if (ca.wrap) k_qcrt_carry_wrap<<<(unsigned)n, CNT, 0, s>>>(ca);
    else k_qcrt_carry<<<(unsigned)n, CNT, 0, s>>>(ca);
    cudaError_t e = cudaGetLastError();
    prof_end(m, s);
    if (e != cudaSuccess) return e;
    const u64 lo = t0 * QCTILE, hi = t1 * QCTILE < ca.out_len ? t1 * QCTILE : ca.out_len;
    if (after_chunk) return after_chunk(ctx, lo, hi);
    return cudaSuccess;
}
}  // namespace q32

// Failure detection without a fault: the CRT + carry kernel over a zero product of `out_len`
// limbs (at least two CTA tiles) whose ticket counter starts at 1, so the CTA that would take
// tile 0 never exists and tile 0 never publishes its carry.  Every later tile's look-back
// reaches tile 0, polls it up to its (short) limit, gives up and sets the status word; the
// highest ticket is past the last tile and exits.  No wait is unbounded.  Returns the kernel
// launch / synchronisation error; *status receives the status word (1 = a wait expired).
cudaError_t q32_test_carry_timeout(u64 out_len, unsigned* status) {
    using namespace q32;
    *status = 0;
    const u64 ncta = (out_len + QCTILE - 1) / QCTILE;
    if (ncta < 2 || ncta > 4096) return cudaErrorInvalidValue;
    const u64 N = 2 * ncta * QCTILE;                 // residue words per prime
    const size_t res_b = 3 * N * sizeof(u32), out_b = out_len * sizeof(u64);
    const size_t state_off = align256(res_b + out_b), total = state_off + 256 + (ncta + 1) * sizeof(u32);
    char* buf = nullptr;
    cudaError_t e = cudaMalloc((void**)&buf, total);
    if (e != cudaSuccess) return e;
    const u32 one = 1;
    u32* err = (u32*)(buf + state_off);
    u32* ticket = err + 32;
    if ((e = cudaMemset(buf, 0, total)) == cudaSuccess && (e = cudaMemcpy(ticket, &one, sizeof(one), cudaMemcpyHostToDevice)) == cudaSuccess) {
        QCrtArgs ca;
        memset(&ca, 0, sizeof(ca));
        crt_constants(N, &ca);
        ca.res = (const u32*)buf;
        ca.N = N;
        ca.nvalid = 2 * out_len - 1;
        ca.out = (u64*)(buf + align256(res_b));
        ca.out_len = out_len;
        ca.ticket = ticket;
        ca.state = ticket + 1;
        ca.err = err;
        k_qcrt_carry_short_wait<<<(unsigned)ncta, CNT>>>(ca);
        if ((e = cudaGetLastError()) == cudaSuccess && (e = cudaDeviceSynchronize()) == cudaSuccess)
            e = cudaMemcpy(status, err, sizeof(u32), cudaMemcpyDeviceToHost);
    }
    cudaFree(buf);
    return e;
}

cudaError_t q32_enqueue(const Job& j, void* ws, size_t ws_bytes, cudaStream_t s, NeedLimbs need_b, void* need_ctx,
                        int crt_chunks, ChunkDone after_chunk, void* ctx) {
    using namespace q32;
    const u64 out_len = j.la + j.lb;
    if (out_len == 0) return cudaSuccess;
    if (j.la == 0 || j.lb == 0) return cudaMemsetAsync(j.out, 0, out_len * sizeof(u64), s);
    const int sqr = j.sqr ? 1 : 0;
    const QJob J = j.spectrum ? plan_resident(j) : plan_job(j.la, j.lb, sqr);
    if (!J.ok || ws_bytes < J.total) return cudaErrorInvalidValue;
    cudaError_t e = q32::ensure_tables();
    if (e != cudaSuccess) return e;
    char* base = (char*)ws;
    const Plan pl = j.spectrum && j.splan.passes ? j.splan : qplan(J.n);
    const int P = pl.passes;
    const u64 N = J.N;
    int logB[MAX_PASSES];
    logB[0] = J.n;
    for (int p = 1; p < P; ++p) logB[p] = logB[p - 1] - pl.bits[p - 1];
    const int lastl = pl.bits[P - 1];
    const u64 nblk_last = N >> lastl;
    const u64 tiles_last = (nblk_last + TC - 1) / TC;
    const int ncols_last = nblk_last < (u64)TC ? (int)nblk_last : TC;
    Launcher launch{j, s, need_b, need_ctx};
    TwPass tws[MAX_PASSES];
    for (int p = 0; p + 1 < P; ++p) tws[p] = tw_tables(logB[p], pl.bits[p], s);

    QArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.N = N;
    pa.ncols = TC;
    auto fwd_strided = [&](const u64* src, u64 len, u32* data) -> cudaError_t {
        for (int p = 0; p + 1 < P; ++p) {
            pa.src = src;
            pa.len = len;
            pa.data = data;
            pa.logB = logB[p];
            pa.tw = tws[p].fwd;
            cudaError_t e2 = launch(p == 0 ? V_FWD_E : V_FWD, pl.bits[p], pa, N >> (pl.bits[p] + LOG_TC));
            pa.tw = nullptr;
            if (e2 != cudaSuccess) return e2;
        }
        return cudaSuccess;
    };
    auto inverse_strided = [&](u32* data, int last_p) -> cudaError_t {   // passes P-2 .. last_p
        pa.src = nullptr;
        pa.len = 0;
        pa.other = nullptr;
        pa.dst = nullptr;
        pa.ncols = TC;
        for (int p = P - 2; p >= last_p; --p) {
            pa.data = data;
            pa.logB = logB[p];
            pa.tw = tws[p].inv;
            cudaError_t e2 = launch(V_INV, pl.bits[p], pa, N >> (pl.bits[p] + LOG_TC));
            pa.tw = nullptr;
            if (e2 != cudaSuccess) return e2;
        }
        return cudaSuccess;
    };

    QCrtArgs ca;
    memset(&ca, 0, sizeof(ca));
    crt_constants(N, &ca);
    u64 crt_done = 0;                 // CRT CTAs launched so far (split products with copy-back)
    if (J.m == 1) {
        u32* A = (u32*)(base + J.a);
        u32* B = sqr ? A : (u32*)(base + J.b);
        u64 b_ready = sqr ? j.lb : 0;                          // limbs of the second operand requested so far
        QWhole W;
        plan_whole(j, J.n, A, B, &W, false, tws);
        int k_main = 0;                                        // main launches issued so far
        if (J.wrap && J.twist) {
            // the main transform's passes over the first operand alone go first, so that a host
            // caller's copy of the second operand overlaps them; then the product modulo
            // X^M - c (it reads both operands whole, folded)
            for (; k_main < W.count && (sqr || W.rec[k_main].a.src != j.b); ++k_main)
                if ((e = launch(W.rec[k_main].variant, W.rec[k_main].logl, W.rec[k_main].a, W.rec[k_main].tiles)) !=
                    cudaSuccess)
                    return e;
            const int tw_log = Q32_MAX_LOG_N - 1 - J.n;        // gamma = w^(2^tw_log), of order 2N
            u32* TA = (u32*)(base + J.la_off);
            u32* TB = sqr ? TA : (u32*)(base + J.lb_off);
            const Plan plt = qplan(J.nl);
            TwPass twt[MAX_PASSES];
            for (int p = 0, lg = J.nl; p + 1 < plt.passes; lg -= plt.bits[p], ++p) twt[p] = tw_tables(lg, plt.bits[p], s);
            // both operands folded and twisted into TA / TB, then an ordinary transform of them
            const u64 fblocks = (J.NL + 255) / 256 < 1184 ? (J.NL + 255) / 256 : 1184;
            for (int op = 0; op < (sqr ? 1 : 2); ++op) {
                if (op == 1 && (e = launch.need(0, j.lb)) != cudaSuccess) return e;
                QFoldArgs fa;
                fa.src = op ? j.b : j.a;
                fa.len = op ? j.lb : j.la;
                fa.T = op ? TB : TA;
                fa.logM = J.nl;
                fa.fold_log = J.n - J.nl;
                fa.tw_log = tw_log;
                for (int i = 0; i < 3; ++i)                    // c^j = gamma^(jM)
                    for (int jj = 0; jj < kMaxFolds; ++jj)
                        fa.cpow[i][jj] = h_shoup(h_root(i, (u64)jj << (fa.logM + tw_log)), i);
                const ProfMark m = prof_begin(K_WRAP, (double)fa.len * 8.0 + 3.0 * (double)J.NL * 4.0,
                                              3.0 * (double)J.NL * (2.0 + (double)(1 << fa.fold_log)), s);
                k_qtwist_fold<<<(unsigned)fblocks, 256, 0, s>>>(fa);
                e = cudaGetLastError();
                prof_end(m, s);
                if (e != cudaSuccess) return e;
            }
            b_ready = j.lb;
            QWhole WT;
            plan_whole(j, J.nl, TA, TB, &WT, false, twt, true);
            for (int k = 0; k < WT.count; ++k)
                if ((e = launch(WT.rec[k].variant, WT.rec[k].logl, WT.rec[k].a, WT.rec[k].tiles)) != cudaSuccess)
                    return e;
            ca.low = TA;
            ca.low_N = J.NL;
            ca.wrap = J.wrap;
            ca.twisted = 1;
            for (int i = 0; i < 3; ++i) ca.low_cst[i] = c_host_r1(i);
        } else if (J.wrap) {
            // the product of the lowest digits first (it reads the second operand's first lpb
            // limbs): its coefficients below `wrap` are the product's c_0 .. c_{wrap-1}
            Job jl = j;
            jl.la = J.lpa;
            jl.lb = J.lpb;
            u32* LA = (u32*)(base + J.la_off);
            u32* LB = sqr ? LA : (u32*)(base + J.lb_off);
            const Plan pll = qplan(J.nl);
            TwPass twl[MAX_PASSES];
            for (int p = 0, lg = J.nl; p + 1 < pll.passes; lg -= pll.bits[p], ++p) twl[p] = tw_tables(lg, pll.bits[p], s);
            QWhole WL;
            plan_whole(jl, J.nl, LA, LB, &WL, false, twl);
            for (int k = 0; k < WL.count; ++k) {
                if (b_ready == 0 && WL.rec[k].a.src == j.b) {
                    if ((e = launch.need(0, J.lpb)) != cudaSuccess) return e;
                    b_ready = J.lpb;
                }
                if ((e = launch(WL.rec[k].variant, WL.rec[k].logl, WL.rec[k].a, WL.rec[k].tiles)) != cudaSuccess)
                    return e;
            }
            QCrtArgs cl;
            memset(&cl, 0, sizeof(cl));
            crt_constants(J.NL, &cl);
            ca.low = LA;
            ca.low_N = J.NL;
            ca.wrap = J.wrap;
            for (int i = 0; i < 3; ++i) ca.low_cst[i] = cl.cst[i];
        }
        bool have_b = sqr != 0;
        for (int k = k_main; k < W.count; ++k) {
            if (!have_b && W.rec[k].a.src == j.b) {            // the second operand's first reader
                if (b_ready < j.lb && (e = launch.need(b_ready, j.lb)) != cudaSuccess) return e;
                have_b = true;
            }
            if ((e = launch(W.rec[k].variant, W.rec[k].logl, W.rec[k].a, W.rec[k].tiles)) != cudaSuccess) return e;
        }
        ca.res = A;
        ca.N = N;
        if (J.wrap && J.twist) {                               // W over the twisted product's residues
            QTwistArgs ta;
            memset(&ta, 0, sizeof(ta));
            ta.U = A;
            ta.V = (u32*)(base + J.la_off);
            ta.N = (u32)N;
            ta.K = (u32)J.wrap;
            ta.logM = J.nl;
            ta.fold_log = J.n - J.nl;
            ta.tw_log = Q32_MAX_LOG_N - 1 - J.n;
            QCrtArgs cm;
            memset(&cm, 0, sizeof(cm));
            crt_constants(J.NL, &cm);
            for (int i = 0; i < 3; ++i) {
                const u64 p = kQ[i];
                const u64 r32 = h_pow(2, 32, p), ninv = h_pow(N % p, p - 2, p);
                ta.cstM[i] = cm.cst[i];
                for (int jj = 0; jj < kMaxFolds; ++jj)   // c^j N^-1 2^32
                    ta.ucj[i][jj] = h_shoup(h_mulmod(h_mulmod(h_root(i, (u64)jj << (ta.logM + ta.tw_log)), ninv, p), r32, p), i);
                ta.nraw[i] = h_shoup(h_mulmod(N % p, h_pow(r32, p - 2, p), p), i);   // N 2^-32
            }
            const u64 blocks = (J.wrap + 255) / 256 < 2048 ? (J.wrap + 255) / 256 : 2048;
            const ProfMark m = prof_begin(K_WRAP, 3.0 * (double)J.wrap * 4.0 * (2.0 + (double)(1 << ta.fold_log)),
                                          3.0 * (double)J.wrap * (3.0 + (double)(1 << ta.fold_log)), s);
            k_qtwist_w<<<dim3((unsigned)blocks, 3), 256, 0, s>>>(ta);
            e = cudaGetLastError();
            prof_end(m, s);
            if (e != cudaSuccess) return e;
        }
    } else {
        // split: S's spectrum once, then every piece of the long operand against it
        u32* R = (u32*)(base + J.a);
        u32* C = (u32*)(base + J.b);
        u32* ACC = (u32*)(base + J.acc);
        const u64* S_src = J.swap ? j.b : j.a;
        const u64* L_src = J.swap ? j.a : j.b;
        if (J.swap && (e = launch.need(0, j.lb)) != cudaSuccess) return e;
        if ((e = fwd_strided(S_src, J.ls, R)) != cudaSuccess) return e;
        pa.src = nullptr;
        pa.len = 0;
        pa.data = R;
        pa.other = nullptr;
        pa.dst = nullptr;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        if ((e = launch(V_LAST, lastl, pa, tiles_last)) != cudaSuccess) return e;
        // limbs below (k + 1) cb are final once piece k is accumulated: with a copy-back hook
        // their carry scan runs right away (tickets continue across launches)
        ca.res = ACC;
        ca.N = J.stride;
        if (after_chunk && (e = cudaMemsetAsync(base + J.ticket, 0, J.total - J.ticket, s)) != cudaSuccess) return e;
        for (int k = 0; k < J.m; ++k) {
            const u64 first = (u64)k * J.cb;
            const u64 len = J.ll - first < J.cb ? J.ll - first : J.cb;
            if (!J.swap && (e = launch.need(first, first + len)) != cudaSuccess) return e;
            if ((e = fwd_strided(L_src + first, len, C)) != cudaSuccess) return e;
            pa.src = nullptr;
            pa.len = 0;
            pa.data = C;
            pa.other = R;
            pa.dst = C;
            pa.logB = logB[P - 1];
            pa.ncols = ncols_last;
            if ((e = launch(V_FUSED, lastl, pa, tiles_last)) != cudaSuccess) return e;
            if ((e = inverse_strided(C, 1)) != cudaSuccess) return e;
            pa.data = C;
            pa.logB = logB[0];
            pa.acc = ACC + 2 * first;
            pa.acc_stride = J.stride;
            pa.acc_valid = 2 * (J.ls + len) - 1;
            pa.acc_fresh = k == 0 ? 0 : 2 * J.ls - 1;
            pa.tw = tws[0].inv;
            e = launch(V_INV_ACC, pl.bits[0], pa, N >> (pl.bits[0] + LOG_TC));
            pa.tw = nullptr;
            if (e != cudaSuccess) return e;
            pa.acc = nullptr;
            if (after_chunk && k + 1 < J.m) {
                fill_crt(j, J, base, out_len, &ca);
                const u64 t_end = (first + J.cb) / QCTILE;
                if (t_end > crt_done && (e = crt_launch(ca, J.ncta, crt_done, t_end, s, after_chunk, ctx)) != cudaSuccess)
                    return e;
                if (t_end > crt_done) crt_done = t_end;
            }
        }
    }

    fill_crt(j, J, base, out_len, &ca);
    if (crt_done == 0 && (e = cudaMemsetAsync(base + J.ticket, 0, J.total - J.ticket, s)) != cudaSuccess) return e;
    if (crt_chunks < 1) crt_chunks = 1;
    const u64 rest = J.ncta - crt_done;
    const u64 per = (rest + crt_chunks - 1) / crt_chunks;
    for (u64 t0 = crt_done; t0 < J.ncta; t0 += per) {
        const u64 t1 = t0 + per <= J.ncta ? t0 + per : J.ncta;
        if ((e = crt_launch(ca, J.ncta, t0, t1, s, after_chunk, ctx)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace fmn
