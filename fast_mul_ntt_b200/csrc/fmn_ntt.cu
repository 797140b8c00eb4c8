// fmn_ntt.cu -- the 64-bit residue engine (the reference's three 62-bit primes): sm_100a
// kernels and launchers, plus the host logic shared by both engines (engine choice, batches,
// kernel timing).  The 32-bit engine lives in fmn_ntt32.cu.
//
// Path (reference src/fast_mul.c:308-396 abs_mul64, :398-460 abs_sqr64):
//   limbs -> residues mod p0, p1, p2 (entry fused into the first pass; plain representatives,
//   constant twiddles applied as Shoup products, variable products as Montgomery REDC)
//   -> forward NTT of each operand (four-step, passes of <= 2^9 points per CTA)
//   -> pointwise product fused between the last forward and first inverse pass
//   -> inverse NTT -> CRT to a 192-bit coefficient -> carry propagation by a single-pass
//      decoupled look-back scan (replacing the serial loop at src/fast_mul.c:378-389).
//
// Data layout in HBM: one product owns a workspace holding, per operand, three residue
// arrays of N = 2^n u64 (prime-major: prime i at base + i*N).  The transform is the
// four-step decomposition: pass p works on contiguous blocks of B_p = 2^(n - sum of earlier
// pass bits) elements, viewed as a [2^m][B_p / 2^m] row-major matrix; each CTA takes a tile
// of 16 adjacent columns (a 16 x 8 B = 128 B stretch of every row) and performs the 2^m-point
// decimation-in-frequency sub-transform down each column in shared memory, then multiplies
// by the four-step twiddle w_B^(column * frequency).  The last pass works on contiguous
// blocks (16 blocks per tile).  Spectra are left in the permuted order that the matching
// inverse passes consume; only final limbs are observable.
//
// Shared-memory tile of contiguous passes: element (row j, column c) lives at
// (j << 4) | (c ^ (j & 15)); the XOR swizzle keeps both the row-wise (16 columns of a row) and
// the column-wise (consecutive rows of one column) access patterns free of bank conflicts.
// Strided passes, whose rounds only ever read whole rows, use a dense tile (row pitch 16) that
// arrives by asynchronous 16-byte copies while the CTA prepares its twiddle factors.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <atomic>
#include <mutex>
#include <vector>

#include "fmn_arith.cuh"
#include "fmn_carry.cuh"
#include "fmn_internal.h"
#include "fmn_rounds.cuh"

namespace fmn {

constexpr int NT = 256;           // threads per CTA, NTT passes
constexpr int TC = 16;            // columns per tile
constexpr int TWB = 15;           // two-level twiddle tables: w^x = HI[x >> 15] * LO[x & 0x7fff]
static_assert(2 * TWB == MAX_LOG_N, "two-level table covers roots of order 2^30");

// [forward/inverse][prime]: (w, w') Shoup pairs, stored stage-major: the twiddle of stage
// entry j of the group with low offset q is at rt_off(RB, TOP) + j * 2^(TOP-RB+1) + q.
__device__ __align__(16) ulonglong2 g_rt[2][3][RT_SIZE];
__device__ __align__(16) u64 g_tw[2][3][1 << TWB];     // [low/high level][prime]
__constant__ PrimeRT c_prime[3] = {prime_rt<0>(), prime_rt<1>(), prime_rt<2>()};

// w_{2^30}^x for x < 2^30 in Montgomery form (< 2p), prime index pi: multiplying a plain
// residue by it with mmul gives the plain product.
__device__ __forceinline__ u64 root30(u32 x, int pi, const PrimeRT& q) {
    return mmul(__ldg(&g_tw[1][pi][x >> TWB]), __ldg(&g_tw[0][pi][x & ((1u << TWB) - 1)]), q);
}

__device__ __forceinline__ int sw(int j, int c) { return (j << 4) | (c ^ (j & 15)); }
// Dense tiles of strided passes: every round runs with the lanes on the 16 columns of a row
// (each 64-bit half-warp phase reads one 128-byte row), so no swizzle is needed and each row
// is a 128-byte copy target.
__device__ __forceinline__ int dix(int j, int c) { return (j << 4) | c; }

// 16-byte asynchronous copy global -> shared.
__device__ __forceinline__ void cp_async16(u64* sdst, const u64* gsrc) {
    const unsigned sa = (unsigned)__cvta_generic_to_shared(sdst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gsrc) : "memory");
}
__device__ __forceinline__ void cp_async_commit_wait() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;\n" ::: "memory");
}
// Rows 0 .. L-1 of a strided tile (16 u64 each, row r at g + r * 2^logS) into a dense tile.
template <int L>
__device__ __forceinline__ void stage_tile(u64* sm, const u64* __restrict__ g, int logS) {
#pragma unroll 4
    for (int e = threadIdx.x; e < L * 8; e += NT) {
        const int r = e >> 3, k = e & 7;
        cp_async16(sm + r * 16 + 2 * k, g + ((u64)r << logS) + 2 * k);
    }
}

// ------------------------------------------------------------------ kernel arguments
enum { M_FWD = 0, M_FWD_LAST = 1, M_FUSED = 2, M_INV = 3, M_FUSED2 = 4 };

struct PassArgs {
    const u64* src;   // ENTRY: limbs of the operand being transformed
    u64 len;          // ENTRY: number of limbs
    u64* data;        // residue arrays of the operand being transformed
    u64* other;       // M_FUSED: the other operand's spectrum; the product is written here
    u64 N;            // transform length
    int logB;         // log2 block length of this pass
    int ncols;        // contiguous passes: number of blocks (columns) in a tile, <= 16
    const u64* tw;    // strided passes: precomputed four-step twiddles of this pass
                      // (prime i at tw + i * 2^logB, entry j * S + column), or null to
                      // generate them on the fly
    u64* dst;         // M_FUSED: where the product goes when `other` must stay intact
                      // (a resident spectrum); null writes it over `other`
};

// ------------------------------------------------------------------ one round
// Runs all radix-2^RB groups of one round.  `ld(j, c)` fetches element (j, c), `st(j, c, v)`
// stores it.  QFAST maps consecutive threads to consecutive rows of one column (coalesced
// global access of contiguous blocks); otherwise consecutive threads take consecutive columns.
template <int LOGL, int RB, int TOP, bool INV, bool QFAST, bool GST = false, bool GLD = false, class LD, class ST>
__device__ __forceinline__ void run_round(LD ld, ST st, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL, R = 1 << RB, SPL = TOP - RB + 1, SP = 1 << SPL;
    constexpr int GPC = L / R;
    constexpr int G = GPC * TC;
    constexpr bool LOWEST = (SPL == 0);
    const ulonglong2* tab = &g_rt[INV ? 1 : 0][pi][rt_off(RB, TOP)];
#pragma unroll 1
    for (int gi = threadIdx.x; gi < G; gi += NT) {
        int c, g;
        if (QFAST) {
            g = gi % GPC;
            c = gi / GPC;
        } else {
            c = gi & (TC - 1);
            g = gi >> 4;
        }
        const int qlo = g & (SP - 1);
        const int row0 = qlo + ((g >> SPL) << (TOP + 1));
        u64 x[R];
        if constexpr (GLD) {
            ld(row0, c, x);      // whole group at once
        } else {
#pragma unroll
            for (int t = 0; t < R; ++t) x[t] = ld(row0 + t * SP, c);
        }
        const ulonglong2* tw = tab + qlo;   // stage-major table: lanes of consecutive groups coalesce
        if (!INV) {
#pragma unroll
            for (int s = 0; s < RB; ++s) {
                const int half = R >> (s + 1);
#pragma unroll
                for (int t = 0; t < R; ++t) {
                    if (t & half) continue;
                    const int u = t & (half - 1);
                    if (LOWEST && u == 0)
                        bfly_dif1(x[t], x[t + half], q);
                    else
                        bfly_dif(x[t], x[t + half], __ldg(tw + ((R - (R >> s)) + u) * SP), q);
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
                        bfly_dit1(x[t], x[t + half], q);
                    else
                        bfly_dit(x[t], x[t + half], __ldg(tw + ((R - (R >> s)) + u) * SP), q);
                }
            }
        }
        if constexpr (GST) {
            st(row0, c, x);      // whole group at once (consecutive rows: vector stores)
        } else {
#pragma unroll
            for (int t = 0; t < R; ++t) st(row0 + t * SP, c, x[t]);
        }
    }
}

// Load R consecutive u64 with 16-byte vector loads.
template <int R>
__device__ __forceinline__ void ld_vec(const u64* p, u64 (&x)[R]) {
    if constexpr (R == 1) {
        x[0] = p[0];
    } else {
#pragma unroll
        for (int t = 0; t < R; t += 2) {
            const ulonglong2 v = *reinterpret_cast<const ulonglong2*>(p + t);
            x[t] = v.x;
            x[t + 1] = v.y;
        }
    }
}

// Rounds IDX.. of a sub-transform.  Forward order: round 0 holds the top bits.  Inverse
// order: inverse round k undoes forward round NR-1-k.  The first round reads with `ld0`, the
// last writes with `stl`, the rest go through shared memory.
template <int LOGL, bool INV, bool CONTIG, int IDX, bool GST = false, bool GLD = false, bool DENSE = false, class LD0,
          class STL>
__device__ __forceinline__ void rounds(u64* sm, LD0 ld0, STL stl, int pi, const PrimeRT& q) {
    constexpr int NR = rounds_count(LOGL);
    constexpr int FR = INV ? NR - 1 - IDX : IDX;
    constexpr int RB = round_bits(LOGL, FR), TOP = round_top(LOGL, FR);
    constexpr bool QF = CONTIG && (TOP == LOGL - 1);
    static_assert(!(DENSE && CONTIG), "dense tiles serve strided passes only");
    auto lds = [sm](int j, int c) { return sm[DENSE ? dix(j, c) : sw(j, c)]; };
    auto sts = [sm](int j, int c, u64 v) { sm[DENSE ? dix(j, c) : sw(j, c)] = v; };
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
__device__ __forceinline__ u64 entry_val(const u64* __restrict__ src, u64 len, u64 g, const PrimeRT& q) {
    return g < len ? smul(__ldg(src + g), 1ull, q.r64, q) : 0ull;   // limb mod p, in [0, 2p)
}

// Four-step twiddles of a strided pass.  After the sub-transform, element (row j, column c)
// holds frequency k = bitrev(j) and is multiplied by w_B^(i k), i = col0 + c.  The lowest
// round's group covers rows j = qhi*R + t, whose frequencies are k = kq + t' (L/R) with
// kq = bitrev(qhi) and t' = bitrev(t), so
//     w_B^(i k) = w_B^(i kq) * w_B^(i t' L/R) = alpha(group) * beta[c][t'].
// Each CTA fills beta (16 x R values) in shared memory once; each group needs one alpha.
// The inverse uses the conjugate roots.
template <int LOGL, bool INV>
__device__ __forceinline__ void fill_beta(u64* beta, u32 col0, int shift, int pi, const PrimeRT& q) {
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1), R = 1 << RB;
    for (int e = threadIdx.x; e < TC * R; e += NT) {
        const u32 c = e >> RB, tp = e & (R - 1);
        u32 x = ((col0 + c) * (tp << (LOGL - RB))) << shift;
        if (INV) x = (0u - x) & ((1u << MAX_LOG_N) - 1);
        beta[e] = red1(root30(x, pi, q), q);
    }
}
template <int LOGL, bool INV>
__device__ __forceinline__ u64 group_alpha(u32 i, int row0, int shift, int pi, const PrimeRT& q) {
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1);
    const u32 kq = LOGL > RB ? __brev((u32)(row0 >> RB)) >> (32 - (LOGL - RB)) : 0u;
    u32 x = (i * kq) << shift;
    if (INV) x = (0u - x) & ((1u << MAX_LOG_N) - 1);
    return red1(root30(x, pi, q), q);
}

// Forward strided pass (pass p < P-1 of a multi-pass transform).
template <int LOGL, bool ENTRY>
__device__ __forceinline__ void body_fwd(u64* sm, const PassArgs& a, u64 tile, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL;
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1), R = 1 << RB;
    const int logS = a.logB - LOGL;
    const u64 tpb_log = logS - 4;
    const u64 blk = tile >> tpb_log;
    const u32 col0 = (u32)((tile & ((1ull << tpb_log) - 1)) << 4);
    const u64 gbase = (blk << a.logB) + col0;
    u64* __restrict__ d = a.data + (u64)pi * a.N;
    const u64* __restrict__ src = a.src;
    const u64 len = a.len;
    const int shift = MAX_LOG_N - a.logB;
    u64* beta = sm + TC * L;
    const u64* __restrict__ tw = a.tw ? a.tw + ((u64)pi << a.logB) + col0 : nullptr;
    // residue tiles arrive by asynchronous copies while the twiddle factors are prepared; the
    // entry pass reads the caller's limbs directly
    constexpr bool STAGED = !ENTRY;
    if constexpr (STAGED) stage_tile<L>(sm, d + gbase, logS);
    if (!tw) fill_beta<LOGL, false>(beta, col0, shift, pi, q);     // read after the first round's barrier
    if constexpr (STAGED) {
        cp_async_commit_wait();
        __syncthreads();
    }
    auto ld0 = [=](int j, int c) -> u64 {
        if constexpr (STAGED) return sm[dix(j, c)];
        const u64 g = gbase + c + ((u64)j << logS);
        if constexpr (ENTRY) return entry_val(src, len, g, q);
        else return d[g];
    };
    auto stl = [=](int row0, int c, const auto& x) {
        if (tw) {
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const u64 off = c + ((u64)(row0 + t) << logS);
                d[gbase + off] = mmul(x[t], __ldg(tw + off), q);
            }
        } else {
            const u64 al = group_alpha<LOGL, false>(col0 + c, row0, shift, pi, q);
            const u64* bc = beta + c * R;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int tp = RB ? (int)(__brev((u32)t) >> (32 - RB)) : 0;
                d[gbase + c + ((u64)(row0 + t) << logS)] = mmul(x[t], mmul(al, bc[tp], q), q);
            }
        }
    };
    rounds<LOGL, false, false, 0, true, false, STAGED>(sm, ld0, stl, pi, q);
}

// Inverse strided pass: inverse four-step twiddle, then the inverse sub-transform.
template <int LOGL>
__device__ __forceinline__ void body_inv(u64* sm, const PassArgs& a, u64 tile, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL;
    constexpr int RB = round_bits(LOGL, rounds_count(LOGL) - 1), R = 1 << RB;
    const int logS = a.logB - LOGL;
    const u64 tpb_log = logS - 4;
    const u64 blk = tile >> tpb_log;
    const u32 col0 = (u32)((tile & ((1ull << tpb_log) - 1)) << 4);
    const u64 gbase = (blk << a.logB) + col0;
    u64* __restrict__ d = a.data + (u64)pi * a.N;
    const int shift = MAX_LOG_N - a.logB;
    u64* beta = sm + TC * L;
    const u64* __restrict__ tw = a.tw ? a.tw + ((u64)pi << a.logB) + col0 : nullptr;
    stage_tile<L>(sm, d + gbase, logS);                   // in flight while the twiddles are prepared
    if (!tw) fill_beta<LOGL, true>(beta, col0, shift, pi, q);
    cp_async_commit_wait();
    __syncthreads();
    auto ld0 = [=](int row0, int c, auto& x) {
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = sm[dix(row0 + t, c)];
        if (tw) {
#pragma unroll
            for (int t = 0; t < R; ++t) x[t] = mmul(x[t], __ldg(tw + c + ((u64)(row0 + t) << logS)), q);
        } else {
            const u64 al = group_alpha<LOGL, true>(col0 + c, row0, shift, pi, q);
            const u64* bc = beta + c * R;
#pragma unroll
            for (int t = 0; t < R; ++t) {
                const int tp = RB ? (int)(__brev((u32)t) >> (32 - RB)) : 0;
                x[t] = mmul(x[t], red1(mmul(al, bc[tp], q), q), q);
            }
        }
    };
    auto stl = [=](int j, int c, u64 v) { d[gbase + c + ((u64)j << logS)] = v; };
    rounds<LOGL, true, false, 0, false, true, true>(sm, ld0, stl, pi, q);
}

// Forward last pass over contiguous blocks (operand A of a product).
template <int LOGL, bool ENTRY>
__device__ __forceinline__ void body_fwd_last(u64* sm, const PassArgs& a, u64 tile, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL;
    const u64 gbase = tile << (LOGL + 4);
    const int ncols = a.ncols;
    u64* __restrict__ d = a.data + (u64)pi * a.N;
    const u64* __restrict__ src = a.src;
    const u64 len = a.len;
    auto ld0 = [=](int j, int c) -> u64 {
        if (c >= ncols) return 0ull;
        const u64 g = gbase + (u64)c * L + j;
        if constexpr (ENTRY) return entry_val(src, len, g, q);
        else return d[g];
    };
    if constexpr (LOGL == 0) {
        if (threadIdx.x < (unsigned)ncols) d[gbase + threadIdx.x] = ld0(0, threadIdx.x);
    } else {
        // the last round (a thread per column) writes the tile; the blocks then leave row by
        // row with the lanes of a warp on consecutive words (256-byte stores)
        auto sts = [sm](int j, int c, u64 v) { sm[sw(j, c)] = v; };
        rounds<LOGL, false, true, 0, false>(sm, ld0, sts, pi, q);
        __syncthreads();
#pragma unroll 4
        for (int e = threadIdx.x; e < TC * L; e += NT) {
            const int c = e >> LOGL, j = e & (L - 1);
            if (c < ncols) d[gbase + (u64)c * L + j] = sm[sw(j, c)];
        }
    }
}

// The lowest forward round, the pointwise product and the lowest inverse round of one
// contiguous tile, all in registers.
template <int LOGL, bool SQR, bool OTH_SMEM = false, class LD, class ST>
__device__ __forceinline__ void fused_lowest(LD ld, ST st, const u64* __restrict__ oth, u64 gbase,
                                             int ncols, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL;
    constexpr int NR = rounds_count(LOGL);
    constexpr int RB = round_bits(LOGL, NR - 1);
    constexpr int R = 1 << RB;
    constexpr int G = (L / R) * TC;
    const ulonglong2* tf = &g_rt[0][pi][rt_off(RB, RB - 1)];
    const ulonglong2* ti = &g_rt[1][pi][rt_off(RB, RB - 1)];
#pragma unroll 1
    for (int gi = threadIdx.x; gi < G; gi += NT) {
        const int c = gi & (TC - 1);
        const int row0 = (gi >> 4) << RB;
        u64 x[R];
#pragma unroll
        for (int t = 0; t < R; ++t) x[t] = ld(row0 + t, c);
#pragma unroll
        for (int s = 0; s < RB; ++s) {
            const int half = R >> (s + 1);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if (t & half) continue;
                const int u = t & (half - 1);
                if (u == 0) bfly_dif1(x[t], x[t + half], q);
                else bfly_dif(x[t], x[t + half], __ldg(tf + (R - (R >> s)) + u), q);
            }
        }
        if (c < ncols) {
            if constexpr (SQR) {
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = mmul(x[t], x[t], q);
            } else if constexpr (OTH_SMEM) {
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = mmul(x[t], oth[sw(row0 + t, c)], q);
            } else {
                u64 y[R];
                ld_vec(oth + gbase + (u64)c * L + row0, y);
#pragma unroll
                for (int t = 0; t < R; ++t) x[t] = mmul(x[t], y[t], q);
            }
        }
#pragma unroll
        for (int s = RB - 1; s >= 0; --s) {
            const int half = R >> (s + 1);
#pragma unroll
            for (int t = 0; t < R; ++t) {
                if (t & half) continue;
                const int u = t & (half - 1);
                if (u == 0) bfly_dit1(x[t], x[t + half], q);
                else bfly_dit(x[t], x[t + half], __ldg(ti + (R - (R >> s)) + u), q);
            }
        }
#pragma unroll
        for (int t = 0; t < R; ++t) st(row0 + t, c, x[t]);
    }
}

// Fused last pass: forward last pass of the second operand (or of the only operand when
// squaring), pointwise product with the first operand's spectrum, inverse last pass.
// The result overwrites the first operand's spectrum (`other`).
template <int LOGL, bool ENTRY, bool SQR>
__device__ __forceinline__ void body_fused(u64* sm, const PassArgs& a, u64 tile, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL;
    constexpr int NR = rounds_count(LOGL);
    const u64 gbase = tile << (LOGL + 4);
    const int ncols = a.ncols;
    const u64* __restrict__ d = a.data + (u64)pi * a.N;
    u64* __restrict__ o = a.other + (u64)pi * a.N;
    u64* __restrict__ dd = (a.dst ? a.dst : a.other) + (u64)pi * a.N;
    const u64* __restrict__ src = a.src;
    const u64 len = a.len;
    auto ldg = [=](int j, int c) -> u64 {
        if (c >= ncols) return 0ull;
        const u64 g = gbase + (u64)c * L + j;
        if constexpr (ENTRY) return entry_val(src, len, g, q);
        else return d[g];
    };
    auto stg = [=](int j, int c, u64 v) {
        if (c < ncols) dd[gbase + (u64)c * L + j] = v;
    };
    auto lds = [sm](int j, int c) { return sm[sw(j, c)]; };
    auto sts = [sm](int j, int c, u64 v) { sm[sw(j, c)] = v; };
    if constexpr (LOGL == 0) {
        if (threadIdx.x < (unsigned)ncols) {
            const int c = threadIdx.x;
            const u64 x = ldg(0, c);
            const u64 y = SQR ? x : o[gbase + c];
            stg(0, c, mmul(x, y, q));
        }
    } else if constexpr (NR == 1) {
        fused_lowest<LOGL, SQR>(ldg, stg, o, gbase, ncols, pi, q);
    } else {
        // forward rounds 0 .. NR-2
        constexpr int RB0 = round_bits(LOGL, 0);
        run_round<LOGL, RB0, LOGL - 1, false, true>(ldg, sts, pi, q);
        __syncthreads();
        if constexpr (NR == 3) {
            constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
            run_round<LOGL, RB1, T1, false, false>(lds, sts, pi, q);
            __syncthreads();
        }
        fused_lowest<LOGL, SQR>(lds, sts, o, gbase, ncols, pi, q);
        __syncthreads();
        if constexpr (NR == 3) {
            constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
            run_round<LOGL, RB1, T1, true, false>(lds, sts, pi, q);
            __syncthreads();
        }
        run_round<LOGL, RB0, LOGL - 1, true, true>(lds, stg, pi, q);
    }
}

// Both operands' last forward pass, pointwise product and first inverse pass in one CTA:
// the first operand's tile (read from `other`) is transformed into a second shared-memory
// tile and never written back; the product overwrites `other`.  Multi-pass products only.
template <int LOGL>
__device__ __forceinline__ void body_fused2(u64* sm, const PassArgs& a, u64 tile, int pi, const PrimeRT& q) {
    constexpr int L = 1 << LOGL;
    constexpr int NR = rounds_count(LOGL);
    static_assert(NR >= 2, "multi-round sub-transforms only");
    const u64 gbase = tile << (LOGL + 4);
    const u64* __restrict__ d = a.data + (u64)pi * a.N;
    u64* __restrict__ o = a.other + (u64)pi * a.N;
    u64* smA = sm + TC * L;
    // first operand: full forward sub-transform into smA
    auto ldA = [=](int j, int c) -> u64 { return o[gbase + (u64)c * L + j]; };
    auto stA = [smA](int j, int c, u64 v) { smA[sw(j, c)] = v; };
    rounds<LOGL, false, true, 0>(smA, ldA, stA, pi, q);
    // second operand: forward rounds 0 .. NR-2 in sm
    auto ldg = [=](int j, int c) -> u64 { return d[gbase + (u64)c * L + j]; };
    auto stg = [=](int j, int c, u64 v) { o[gbase + (u64)c * L + j] = v; };
    auto lds = [sm](int j, int c) { return sm[sw(j, c)]; };
    auto sts = [sm](int j, int c, u64 v) { sm[sw(j, c)] = v; };
    constexpr int RB0 = round_bits(LOGL, 0);
    run_round<LOGL, RB0, LOGL - 1, false, true>(ldg, sts, pi, q);
    __syncthreads();                                   // also publishes smA
    if constexpr (NR == 3) {
        constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
        run_round<LOGL, RB1, T1, false, false>(lds, sts, pi, q);
        __syncthreads();
    }
    fused_lowest<LOGL, false, true>(lds, sts, smA, gbase, TC, pi, q);
    __syncthreads();
    if constexpr (NR == 3) {
        constexpr int RB1 = round_bits(LOGL, 1), T1 = round_top(LOGL, 1);
        run_round<LOGL, RB1, T1, true, false>(lds, sts, pi, q);
        __syncthreads();
    }
    run_round<LOGL, RB0, LOGL - 1, true, true>(lds, stg, pi, q);
}

// ------------------------------------------------------------------ pass kernels
// 9-bit strided passes hold a 64 KB tile, so at most 3 CTAs share an SM anyway: they get the
// registers of 3 (at 4 their radix-8 rounds spill).  8-bit ones keep 4 (measured faster).
template <int MODE, int LOGL>
constexpr int pass_min_ctas() {
    return (MODE == M_FWD || MODE == M_INV) && LOGL >= 9 ? 3 : 4;
}

template <int MODE, int LOGL, bool ENTRY, bool SQR>
__global__ void __launch_bounds__(NT, (pass_min_ctas<MODE, LOGL>())) k_pass(PassArgs a) {
    extern __shared__ __align__(16) u64 sm[];
    const int pi = blockIdx.x % 3;          // prime varies fastest: the three CTAs of a tile
    const u64 tile = blockIdx.x / 3;        // read the same limbs at the same time (L2 reuse)
    const PrimeRT q = c_prime[pi];
    if constexpr (MODE == M_FWD) body_fwd<LOGL, ENTRY>(sm, a, tile, pi, q);
    else if constexpr (MODE == M_INV) body_inv<LOGL>(sm, a, tile, pi, q);
    else if constexpr (MODE == M_FWD_LAST) body_fwd_last<LOGL, ENTRY>(sm, a, tile, pi, q);
    else if constexpr (MODE == M_FUSED2) body_fused2<(LOGL >= 5 ? LOGL : 5)>(sm, a, tile, pi, q);
    else body_fused<LOGL, ENTRY, SQR>(sm, a, tile, pi, q);
}

// ------------------------------------------------------------------ four-step twiddle tables
// Entry j * S + i of pass (logB, logl): w_B^(i * bitrev(j)) (forward) and its inverse, both
// fully reduced, for the three primes (prime-major).
__global__ void __launch_bounds__(256) k_tw_table(u64* tf, u64* ti, int logB, int logl) {
    const u64 B = 1ull << logB;
    const int shift = MAX_LOG_N - logB, logS = logB - logl;
    for (u64 idx = blockIdx.x * 256ull + threadIdx.x; idx < 3 * B; idx += (u64)gridDim.x * 256) {
        const int pi = (int)(idx >> logB);
        const u64 r = idx & (B - 1);
        const u32 j = (u32)(r >> logS), i = (u32)(r & ((1ull << logS) - 1));
        const u32 k = __brev(j) >> (32 - logl);
        const u32 x = (i * k) << shift;
        const PrimeRT q = c_prime[pi];
        tf[idx] = red1(root30(x, pi, q), q);
        ti[idx] = red1(root30((0u - x) & ((1u << MAX_LOG_N) - 1), pi, q), q);
    }
}

size_t twiddle_table_bytes(int log_n) {
    const Plan pl = make_plan(log_n);
    size_t b = 0, logB = log_n;
    for (int p = 0; p + 1 < pl.passes; ++p) {
        b += 2 * 3 * ((size_t)1 << logB) * sizeof(u64);
        logB -= pl.bits[p];
    }
    return b;
}

cudaError_t build_twiddle_tables(int log_n, u64* buf, TwiddleSet* out, cudaStream_t s) {
    const Plan pl = make_plan(log_n);
    *out = TwiddleSet();
    out->log_n = log_n;
    out->plan = pl;
    int logB = log_n;
    u64* p = buf;
    for (int k = 0; k + 1 < pl.passes; ++k) {
        const u64 B = 1ull << logB;
        out->fwd[k] = p;
        out->inv[k] = p + 3 * B;
        const unsigned grid = (unsigned)((3 * B + 255) / 256 < 148 * 16 ? (3 * B + 255) / 256 : 148 * 16);
        k_tw_table<<<grid, 256, 0, s>>>(p, p + 3 * B, logB, pl.bits[k]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        p += 6 * B;
        logB -= pl.bits[k];
    }
    return cudaSuccess;
}

// ------------------------------------------------------------------ CRT + carry
// crt3 (src/core.h:77-104) then carry propagation.  Coefficient c_j < p0 p1 p2 < 2^185 spans
// three limbs; output limb j receives s_j = c_j[0] + c_{j-1}[1] + c_{j-2}[2] < 3 * 2^64
// plus an incoming carry in [0, 3].  A span of limbs maps its incoming carry to its outgoing
// carry by a function {0..3} -> {0..3} (packed as 4 x 2 bits); these compose associatively,
// which gives a parallel scan: per-thread functions, a CTA scan, and a decoupled look-back
// across CTAs in the order CTAs obtain tickets.

struct CrtArgs {
    const u64* res;     // three natural-order residue arrays (prime i at res + i*N), < 4p
    u64 N;
    u64 nvalid;         // coefficients that may be nonzero: min(conv_len, N), or conv_len if wrapped
    u64* out;
    u64 out_len;
    u64 cst[3];         // M_i^-1 * N^-1 * 2^128 mod p_i (undoes the two Montgomery products)
    u32* state;         // per-CTA look-back words, zeroed before launch
    u32* ticket;        // zeroed before launch
    u32* err;
    // wrapped products (wrap = K > 0): `res` holds the cyclic convolution of length N, whose
    // entry k < K is c_k + c_{k+N}, and `low` the product of the operands' lowest K limbs
    // (prime i at low + i*low_N), whose coefficients below K are c_0 .. c_{K-1}; each with its
    // own scale constants.  c_k = low_k for k < K, res_k for K <= k < N, and
    // res_{k-N} - low_{k-N} for N <= k < conv_len.
    const u64* low;
    u64 low_N;
    u64 wrap;
    u64 low_cst[3];
    // twisted (see k_twist_w64): `low` holds W (plain, reduced; low_cst = M_i^-1 2^64), res_k
    // already holds c_k for k < K, and c_{N+k} = W_k
    int twisted;
};

__host__ __device__ constexpr u64 m_lo(int i) {
    return (u64)(i == 0 ? (unsigned __int128)Prime<1>::P * Prime<2>::P
                 : i == 1 ? (unsigned __int128)Prime<0>::P * Prime<2>::P
                          : (unsigned __int128)Prime<0>::P * Prime<1>::P);
}
__host__ __device__ constexpr u64 m_hi(int i) {
    return (u64)((i == 0 ? (unsigned __int128)Prime<1>::P * Prime<2>::P
                  : i == 1 ? (unsigned __int128)Prime<0>::P * Prime<2>::P
                           : (unsigned __int128)Prime<0>::P * Prime<1>::P) >> 64);
}
constexpr unsigned __int128 P01 = (unsigned __int128)Prime<0>::P * Prime<1>::P;
constexpr unsigned __int128 PL = (unsigned __int128)(u64)P01 * Prime<2>::P;
constexpr unsigned __int128 PH = (unsigned __int128)(u64)(P01 >> 64) * Prime<2>::P;
constexpr u64 PALL0 = (u64)PL;
constexpr u64 PALL1 = (u64)((PL >> 64) + (u64)PH);
constexpr u64 PALL2 = (u64)((((PL >> 64) + (u64)PH) >> 64) + (u64)(PH >> 64));

__device__ __forceinline__ void acc_mul(u64 y, u64 ml, u64 mh, u64& w0, u64& w1, u64& w2) {
    const unsigned __int128 lo = (unsigned __int128)y * ml;
    const unsigned __int128 hi = (unsigned __int128)y * mh;
    const unsigned __int128 s0 = (unsigned __int128)w0 + (u64)lo;
    const unsigned __int128 s1 = (unsigned __int128)w1 + (u64)(lo >> 64) + (u64)hi + (u64)(s0 >> 64);
    w0 = (u64)s0;
    w1 = (u64)s1;
    w2 = w2 + (u64)(hi >> 64) + (u64)(s1 >> 64);
}

// crt3 of one coefficient from y_i = c mod p_i times M_i^-1 (each in [0, p_i)).
__device__ __forceinline__ void crt_acc(u64 y0, u64 y1, u64 y2, u64& w0, u64& w1, u64& w2) {
    w0 = w1 = w2 = 0;
    acc_mul(y0, m_lo(0), m_hi(0), w0, w1, w2);
    acc_mul(y1, m_lo(1), m_hi(1), w0, w1, w2);
    acc_mul(y2, m_lo(2), m_hi(2), w0, w1, w2);
#pragma unroll
    for (int r = 0; r < 2; ++r) {   // sum < 3 * P: at most two subtractions
        const bool ge = w2 != PALL2 ? w2 > PALL2 : w1 != PALL1 ? w1 > PALL1 : w0 >= PALL0;
        if (ge) {
            const u64 b0 = w0 < PALL0;
            w0 -= PALL0;
            const u64 t1 = w1 - PALL1;
            const u64 b1 = (w1 < PALL1) | (t1 < b0);
            w1 = t1 - b0;
            w2 = w2 - PALL2 - b1;
        }
    }
}
// crt3 of one coefficient from its three residues r0, r1, r2 (< 4p_i).
__device__ __forceinline__ void crt_of(u64 r0, u64 r1, u64 r2, const u64 (&cst)[3], u64& w0, u64& w1, u64& w2,
                                       const PrimeRT& q0, const PrimeRT& q1, const PrimeRT& q2) {
    crt_acc(red1(mmul(r0, cst[0], q0), q0), red1(mmul(r1, cst[1], q1), q1), red1(mmul(r2, cst[2], q2), q2), w0, w1,
            w2);
}

// Where coefficient j of a wrapped product comes from (see CrtArgs): 0 res_j, 1 low_j,
// 2 res_{j-N} - low_{j-N}, 3 (twisted) W_{j-N}.  MODE 0 plain, 1 low product, 2 twisted.
template <int MODE>
__device__ __forceinline__ int src64(const CrtArgs& a, u64 j) {
    return MODE == 0 ? 0 : MODE == 2 ? (j >= a.N ? 3 : 0) : (j >= a.N ? 2 : (j < a.wrap ? 1 : 0));
}
// c_j mod p_i times M_i^-1, in [0, p_i), from source src.
__device__ __forceinline__ u64 y_of(const CrtArgs& a, int src, u64 j, int i, const PrimeRT& q) {
    if (src == 0) return red1(mmul(a.res[i * a.N + j], a.cst[i], q), q);
    const u64 jj = src == 1 ? j : j - a.N;
    const u64 yl = red1(mmul(a.low[i * a.low_N + jj], a.low_cst[i], q), q);
    if (src != 2) return yl;
    return red1(red1(mmul(a.res[i * a.N + jj], a.cst[i], q), q) + q.p - yl, q);
}
template <int MODE>
__device__ __forceinline__ void crt_coef(const CrtArgs& a, u64 j, u64& w0, u64& w1, u64& w2,
                                         const PrimeRT& q0, const PrimeRT& q1, const PrimeRT& q2) {
    constexpr bool WRAP = MODE != 0;
    w0 = w1 = w2 = 0;
    if (j >= a.nvalid) return;
    if (!WRAP) {
        crt_of(a.res[j], a.res[a.N + j], a.res[2 * a.N + j], a.cst, w0, w1, w2, q0, q1, q2);
        return;
    }
    const int src = src64<MODE>(a, j);
    crt_acc(y_of(a, src, j, 0, q0), y_of(a, src, j, 1, q1), y_of(a, src, j, 2, q2), w0, w1, w2);
}

// Output limbs per thread of the CRT + carry kernel: 8 keeps a thread's sums and 192-bit CRT
// words within the registers of 4 CTAs per SM (16 needed 90 registers: 2 CTAs; 64M x 64M
// 28.4 -> 27.9 ms).
constexpr int WCE = 8;
constexpr u64 WCTILE = (u64)CNT * WCE;

template <int MODE>
__device__ __forceinline__ void crt_carry_body(const CrtArgs& a, u32 ncta) {
    constexpr bool WRAP = MODE != 0;
    __shared__ u64 s_hw[CNT / 32][3];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const PrimeRT q0 = c_prime[0], q1 = c_prime[1], q2 = c_prime[2];
    const u64 tile = carry_ticket(a.ticket);
    if (tile >= ncta) return;                   // batch launches cover the largest product
    const u64 j0 = tile * WCTILE + (u64)tid * WCE;

    // coefficients j0 .. j0+15, folded into limb sums s_j = c_j[0] + c_{j-1}[1] + c_{j-2}[2]
    // (the two contributions from the previous thread's coefficients are added below)
    u64 lo[WCE];
    u32 h[WCE];
    u64 pw1 = 0, pw2 = 0, ppw2 = 0;          // c_{j-1}[1], c_{j-1}[2], c_{j-2}[2]
    // wrapped: the vector path takes threads whose coefficients all come from res; the few
    // around and beyond the wrap boundaries go coefficient by coefficient
    const bool full = j0 + WCE <= a.nvalid && (!WRAP || (src64<MODE>(a, j0) == 0 && src64<MODE>(a, j0 + WCE - 1) == 0));
#pragma unroll
    for (int e2 = 0; e2 < WCE; e2 += 2) {
        u64 r0[2], r1[2], r2[2];
        if (full) {
            const ulonglong2 v0 = *reinterpret_cast<const ulonglong2*>(a.res + j0 + e2);
            const ulonglong2 v1 = *reinterpret_cast<const ulonglong2*>(a.res + a.N + j0 + e2);
            const ulonglong2 v2 = *reinterpret_cast<const ulonglong2*>(a.res + 2 * a.N + j0 + e2);
            r0[0] = v0.x, r0[1] = v0.y, r1[0] = v1.x, r1[1] = v1.y, r2[0] = v2.x, r2[1] = v2.y;
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
            const int e = e2 + u;
            u64 w0, w1, w2;
            if (full) crt_of(r0[u], r1[u], r2[u], a.cst, w0, w1, w2, q0, q1, q2);
            else crt_coef<MODE>(a, j0 + e, w0, w1, w2, q0, q1, q2);
            u64 l = w0;
            u32 hh = 0;
            add_to(l, hh, pw1);
            add_to(l, hh, ppw2);
            lo[e] = l;
            h[e] = hh;
            ppw2 = pw2;
            pw1 = w1;
            pw2 = w2;
        }
    }
    // contributions of the two coefficients just below j0 (previous thread / previous CTA)
    u64 n1 = __shfl_up_sync(0xffffffffu, pw1, 1);   // c_{j0-1}[1]
    u64 n2 = __shfl_up_sync(0xffffffffu, pw2, 1);   // c_{j0-1}[2]
    u64 n3 = __shfl_up_sync(0xffffffffu, ppw2, 1);  // c_{j0-2}[2]
    if (lane == 31) {
        s_hw[warp][0] = pw1;
        s_hw[warp][1] = pw2;
        s_hw[warp][2] = ppw2;
    }
    __syncthreads();
    if (lane == 0) {
        if (warp > 0) {
            n1 = s_hw[warp - 1][0];
            n2 = s_hw[warp - 1][1];
            n3 = s_hw[warp - 1][2];
        } else {
            u64 u0, u1, u2, v0, v1, v2;
            if (j0 >= 1) crt_coef<MODE>(a, j0 - 1, u0, u1, u2, q0, q1, q2); else u0 = u1 = u2 = 0;
            if (j0 >= 2) crt_coef<MODE>(a, j0 - 2, v0, v1, v2, q0, q1, q2); else v0 = v1 = v2 = 0;
            n1 = u1;
            n2 = u2;
            n3 = v2;
        }
    }
    add_to(lo[0], h[0], n1);
    add_to(lo[0], h[0], n3);
    add_to(lo[1], h[1], n2);

    carry_finish(lo, h, tile, j0, a.state, a.err, a.out, a.out_len);
}

// 5 CTAs per SM (48 registers, no spills): while one CTA's warps wait at the barrier of its
// look-back, the others compute.
__global__ void __launch_bounds__(CNT, 5) k_crt_carry(CrtArgs a) { crt_carry_body<0>(a, 0xffffffffu); }
// Wrapped products (see CrtArgs): 62 registers, 4 CTAs (5 spilled).
__global__ void __launch_bounds__(CNT, 4) k_crt_carry_wrap(CrtArgs a) { crt_carry_body<1>(a, 0xffffffffu); }
__global__ void __launch_bounds__(CNT, 4) k_crt_carry_twist(CrtArgs a) { crt_carry_body<2>(a, 0xffffffffu); }

// ------------------------------------------------------------------ twisted products
// The 32-bit engine's twisted form (fmn_ntt32.cu, k_qtwist_fold / k_qtwist_w) restated for
// limbs: the product is U = C mod (X^N - 1) (the cyclic transform of length N) and
// V = C mod (X^M - c), a cyclic transform of length M = N / 2^s of both operands folded modulo
// X^M - c and twisted by gamma^g (gamma of order 2N, c = gamma^M, so c^(2^s) = -1); then
// W = (sum_j c^j U_{k+jM} - V) / 2 gives c_{N+k} = W_k and c_k = U_k - W_k for k < K.
// Residues are plain values below 2p, as the entry pass produces them.
constexpr int kMaxFolds64 = 4;
constexpr u32 MASK30 = (1u << MAX_LOG_N) - 1;
struct FoldArgs64 {
    const u64* src;
    u64 len;                      // limbs
    u64* T;                       // prime i at T + i M
    int logM, fold_log, tw_log;   // gamma = w_{2^30}^(2^tw_log)
    ulonglong2 cpow[3][kMaxFolds64];   // c^j mod p_i (plain) and floor(c^j 2^64 / p_i)
};
// Entry g (< M) of prime i: gamma^g sum_{j < 2^fold_log} c^j a_{g + jM} mod p_i, a the limbs
// (zero past the end); one thread per g, the limbs loaded once for all three primes.
__global__ void __launch_bounds__(256) k_twist_fold64(FoldArgs64 f) {
    const u64 M = 1ull << f.logM;
    const int F = 1 << f.fold_log;
    const u64 g0 = blockIdx.x * (u64)blockDim.x + threadIdx.x, S = (u64)gridDim.x * blockDim.x;
    // gamma^g in Montgomery form, stepped by gamma^S along the grid-stride loop
    u64 gm[3], gs[3];
#pragma unroll
    for (int pi = 0; pi < 3; ++pi) {
        gm[pi] = root30((u32)((g0 << f.tw_log) & MASK30), pi, c_prime[pi]);
        gs[pi] = root30((u32)((S << f.tw_log) & MASK30), pi, c_prime[pi]);
    }
    for (u64 g = g0; g < M; g += S) {
        const u64 left = f.len > g ? (f.len - g + M - 1) >> f.logM : 0;
        const int nf = left < (u64)F ? (int)left : F;
        u64 x[kMaxFolds64];
#pragma unroll
        for (int j = 0; j < kMaxFolds64; ++j) x[j] = j < nf ? __ldg(f.src + g + ((u64)j << f.logM)) : 0ull;
#pragma unroll
        for (int pi = 0; pi < 3; ++pi) {
            const PrimeRT q = c_prime[pi];
            u64 acc = smul(x[0], f.cpow[pi][0].x, f.cpow[pi][0].y, q);            // [0, 2p)
#pragma unroll
            for (int j = 1; j < kMaxFolds64; ++j)
                if (j < nf) acc = red2(acc + smul(x[j], f.cpow[pi][j].x, f.cpow[pi][j].y, q), q);
            f.T[(u64)pi * M + g] = mmul(acc, gm[pi], q);                           // (0, 2p)
            gm[pi] = mmul(gm[pi], gs[pi], q);
        }
    }
}

struct TwistArgs64 {
    u64* U;                       // cyclic product's residues (prime i at U + i N), raw
    u64* V;                       // twisted product's residues (prime i at V + i M), raw; W on return
    u64 N, K;
    int logM, fold_log, tw_log;
    u64 cstM[3];                  // M^-1 2^128 mod p_i
    ulonglong2 ucj[3][kMaxFolds64];   // c^j N^-1 2^64 mod p_i (Shoup pairs): U raw -> c^j U
    ulonglong2 nraw[3];           // N 2^-64 mod p_i (Shoup pair): a coefficient -> U's raw form
};
// Raw residues after the inverse transform are r = x N 2^-64 (x the convolution entry, see
// the CRT constants), so x = r N^-1 2^64; V's entries also carry gamma^k.  For k < K the kernel
// writes W_k (plain, reduced) over V_k and U_k - W_k (raw) over U_k; U_{k+jM} with j >= 1 lie
// at or above M >= K, so updating U_k in place is safe.
__global__ void __launch_bounds__(256) k_twist_w64(TwistArgs64 t) {
    const int pi = blockIdx.y;
    const PrimeRT q = c_prime[pi];
    const int F = 1 << t.fold_log;
    u64* __restrict__ U = t.U + (u64)pi * t.N;
    u64* __restrict__ V = t.V + ((u64)pi << t.logM);
    const u64 k0 = blockIdx.x * (u64)blockDim.x + threadIdx.x, S = (u64)gridDim.x * blockDim.x;
    // gamma^-k M^-1 2^128 (Montgomery form of gamma^-k times cstM 2^-64), stepped by gamma^-S
    u64 gm = mmul(root30((u32)((0ull - (k0 << t.tw_log)) & MASK30), pi, q), t.cstM[pi], q);
    const u64 gs = root30((u32)((0ull - (S << t.tw_log)) & MASK30), pi, q);
    for (u64 k = k0; k < t.K; k += S) {
        u64 x[kMaxFolds64];
#pragma unroll
        for (int j = 0; j < kMaxFolds64; ++j) x[j] = j < F ? U[k + ((u64)j << t.logM)] : 0ull;
        const u64 vr = V[k];
        const u64 u0 = red1(smul(x[0], t.ucj[pi][0].x, t.ucj[pi][0].y, q), q);          // U_k
        u64 ub = u0;
#pragma unroll
        for (int j = 1; j < kMaxFolds64; ++j)
            if (j < F) ub = red1(ub + red1(smul(x[j], t.ucj[pi][j].x, t.ucj[pi][j].y, q), q), q);
        // vr < 4p: its factor must be below p for vr * factor < p 2^64 (p2 > 2^61)
        const u64 v = red1(mmul(vr, red1(gm, q), q), q);                                 // V_k, untwisted
        const u64 d = red1(ub + q.p - v, q);                                             // U mod (X^M - c) - V
        const u64 w = (d + ((d & 1) ? q.p : 0)) >> 1;
        V[k] = w;
        U[k] = smul(red1(u0 + q.p - w, q), t.nraw[pi].x, t.nraw[pi].y, q);              // c_k = U_k - W_k, raw
        gm = mmul(gm, gs, q);
    }
}

// ------------------------------------------------------------------ host: tables
static u64 h_mulmod(u64 a, u64 b, u64 m) { return (u64)(((unsigned __int128)a * b) % m); }
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
static const u64 kP[3] = {Prime<0>::P, Prime<1>::P, Prime<2>::P};
static const u64 kG[3] = {5, 5, 3};   // primitive roots (src/data.h:69-71)

struct HostTables {
    std::vector<u64> rt;   // [2][3][RT_SIZE][2]: (w, floor(w 2^64 / p)) plain Shoup pairs
    std::vector<u64> tw;   // [2][3][1 << TWB]
    u64 w30[3];            // the root of order 2^30 of each prime that all tables use
};

static const HostTables& host_tables() {
    static HostTables T;
    static std::once_flag once;
    std::call_once(once, [] {
        T.rt.assign((size_t)2 * 3 * RT_SIZE * 2, 0);
        T.tw.assign((size_t)2 * 3 * (1u << TWB), 0);
        for (int i = 0; i < 3; ++i) {
            const u64 p = kP[i];
            const u64 r1 = (u64)((((unsigned __int128)1) << 64) % p);
            const u64 w = h_pow(kG[i], (p - 1) >> MAX_LOG_N, p);     // root of order 2^30
            T.w30[i] = w;
            std::vector<u64> lo(1u << TWB), hi(1u << TWB);
            const u64 whi = h_pow(w, 1ull << TWB, p);
            u64 cl = 1, ch = 1;
            for (u32 x = 0; x < (1u << TWB); ++x) {
                lo[x] = cl;
                hi[x] = ch;
                cl = h_mulmod(cl, w, p);
                ch = h_mulmod(ch, whi, p);
            }
            auto wpow = [&](u64 e) {   // w^e, e mod 2^30
                e &= (1ull << MAX_LOG_N) - 1;
                return h_mulmod(hi[e >> TWB], lo[e & ((1u << TWB) - 1)], p);
            };
            auto mont = [&](u64 v) { return h_mulmod(v, r1, p); };
            for (u32 x = 0; x < (1u << TWB); ++x) {
                T.tw[((size_t)0 * 3 + i) * (1u << TWB) + x] = mont(lo[x]);
                T.tw[((size_t)1 * 3 + i) * (1u << TWB) + x] = mont(hi[x]);
            }
            for (int r = 1; r <= 4; ++r)
                for (int top = r - 1; top < RT_MAXLOGL; ++top) {
                    const int R = 1 << r, spl = top - r + 1;
                    for (int q = 0; q < (1 << spl); ++q)
                        for (int s = 0; s < r; ++s)
                            for (int u = 0; u < (R >> (s + 1)); ++u) {
                                // w_{2^(top-s+1)}^(q + u 2^spl) = w^((q + u 2^spl) 2^(30-(top-s+1)))
                                const u64 e = ((u64)q + ((u64)u << spl)) << (MAX_LOG_N - (top - s + 1));
                                // stage-major: entry j = (R - (R >> s)) + u of group offset q
                                const size_t at = (size_t)rt_off(r, top) + ((size_t)(R - (R >> s)) + u << spl) + q;
                                const u64 wf = wpow(e);
                                const u64 wi = wpow((1ull << MAX_LOG_N) - (e & ((1ull << MAX_LOG_N) - 1)));
                                const size_t f0 = (((size_t)0 * 3 + i) * RT_SIZE + at) * 2;
                                const size_t i0 = (((size_t)1 * 3 + i) * RT_SIZE + at) * 2;
                                T.rt[f0] = wf;
                                T.rt[f0 + 1] = (u64)((((unsigned __int128)wf) << 64) / p);
                                T.rt[i0] = wi;
                                T.rt[i0 + 1] = (u64)((((unsigned __int128)wi) << 64) / p);
                            }
                }
        }
    });
    return T;
}

// ------------------------------------------------------------------ host: launch plumbing
typedef void (*PassKernel)(PassArgs);

template <int MODE, int LOGL, bool ENTRY, bool SQR>
static PassKernel kernel_ptr() {
    return k_pass<MODE, LOGL, ENTRY, SQR>;
}

// Table of every kernel instance: [mode-variant][logl]
enum { V_FWD, V_FWD_E, V_LAST, V_LAST_E, V_FUSED, V_FUSED_E, V_SQR, V_SQR_E, V_INV, V_FUSED2, NV };

template <int LOGL>
static void fill_row(PassKernel (&t)[NV][MAX_PASS_BITS + 1]) {
    t[V_FWD][LOGL] = LOGL >= 5 ? kernel_ptr<M_FWD, (LOGL >= 5 ? LOGL : 5), false, false>() : nullptr;
    t[V_FWD_E][LOGL] = LOGL >= 5 ? kernel_ptr<M_FWD, (LOGL >= 5 ? LOGL : 5), true, false>() : nullptr;
    t[V_INV][LOGL] = LOGL >= 5 ? kernel_ptr<M_INV, (LOGL >= 5 ? LOGL : 5), false, false>() : nullptr;
    t[V_FUSED2][LOGL] = (LOGL >= 5 && LOGL <= 8) ? kernel_ptr<M_FUSED2, (LOGL >= 5 && LOGL <= 8 ? LOGL : 5), false, false>()
                                                   : nullptr;
    t[V_LAST][LOGL] = kernel_ptr<M_FWD_LAST, LOGL, false, false>();
    t[V_LAST_E][LOGL] = kernel_ptr<M_FWD_LAST, LOGL, true, false>();
    t[V_FUSED][LOGL] = kernel_ptr<M_FUSED, LOGL, false, false>();
    t[V_FUSED_E][LOGL] = kernel_ptr<M_FUSED, LOGL, true, false>();
    t[V_SQR][LOGL] = kernel_ptr<M_FUSED, LOGL, false, true>();
    t[V_SQR_E][LOGL] = kernel_ptr<M_FUSED, LOGL, true, true>();
}

struct KernelTable {
    PassKernel k[NV][MAX_PASS_BITS + 1];
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

// tile + the 16 x 16 four-step twiddle factors of strided passes; two tiles for V_FUSED2
static size_t pass_smem(int logl, int variant = -1) {
    const size_t tile = (size_t)TC * ((size_t)1 << logl);
    return (variant == V_FUSED2 ? 2 * tile : tile + TC * 16) * sizeof(u64);
}

cudaError_t ensure_tables() {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lock(mu);
    for (int d : done)
        if (d == dev) return cudaSuccess;
    const HostTables& T = host_tables();
    e = cudaMemcpyToSymbol(g_rt, T.rt.data(), T.rt.size() * sizeof(u64));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(g_tw, T.tw.data(), T.tw.size() * sizeof(u64));
    if (e != cudaSuccess) return e;
    const KernelTable& K = ktab();
    for (int v = 0; v < NV; ++v)
        for (int l = 0; l <= MAX_PASS_BITS; ++l)
            if (K.k[v][l]) {
                e = cudaFuncSetAttribute((const void*)K.k[v][l], cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)pass_smem(l, v));
                if (e != cudaSuccess) return e;
                e = cudaFuncSetAttribute((const void*)K.k[v][l], cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
                if (e != cudaSuccess) return e;
            }
    done.push_back(dev);
    return cudaSuccess;
}

// Pass plans.  The default splits n bits into ceil(n/9) nearly equal passes (larger first);
// the autotuner (fmn_autotune) or a tuning file may replace the plan of any length.
Plan default_plan(int n) {
    Plan p;
    memset(&p, 0, sizeof(p));
    p.n = n;
    if (n <= MAX_PASS_BITS) {
        p.passes = 1;
        p.bits[0] = n;
        return p;
    }
    p.passes = (n + MAX_PASS_BITS - 1) / MAX_PASS_BITS;
    for (int i = 0; i < p.passes; ++i) p.bits[i] = n / p.passes + (i < n % p.passes ? 1 : 0);
    return p;
}

// A plan is valid when its bits add up to n, every strided pass has 5..9 bits and at least
// 16 columns (4 bits) after it, and the last pass has at most 9 bits.
bool valid_plan(const Plan& p) {
    if (p.n < 0 || p.n > MAX_LOG_N || p.passes < 1 || p.passes > MAX_PASSES) return false;
    int sum = 0;
    for (int i = 0; i < p.passes; ++i) {
        if (p.bits[i] < 0 || p.bits[i] > MAX_PASS_BITS) return false;
        sum += p.bits[i];
    }
    if (sum != p.n) return false;
    if (p.passes == 1) return p.n <= MAX_PASS_BITS;
    int rest = p.n;
    for (int i = 0; i + 1 < p.passes; ++i) {
        rest -= p.bits[i];
        if (p.bits[i] < 5 || rest < 4) return false;
    }
    return p.bits[p.passes - 1] >= 1;
}

bool same_plan(const Plan& a, const Plan& b) {
    if (a.n != b.n || a.passes != b.passes) return false;
    for (int i = 0; i < a.passes; ++i)
        if (a.bits[i] != b.bits[i]) return false;
    return true;
}

static std::mutex g_plan_mu;
static Plan g_plan_tab[MAX_LOG_N + 1];
static bool g_plan_set[MAX_LOG_N + 1] = {false};

Plan make_plan(int n) {
    if (n >= 0 && n <= MAX_LOG_N) {
        std::lock_guard<std::mutex> lk(g_plan_mu);
        if (g_plan_set[n]) return g_plan_tab[n];
    }
    return default_plan(n);
}

bool set_plan(const Plan& p) {
    if (!valid_plan(p)) return false;
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plan_tab[p.n] = p;
    g_plan_set[p.n] = true;
    return true;
}

void clear_plan(int n) {
    if (n < 0 || n > MAX_LOG_N) return;
    std::lock_guard<std::mutex> lk(g_plan_mu);
    g_plan_set[n] = false;
}

// Every valid plan of n bits with the default pass count or one more.
std::vector<Plan> candidate_plans(int n) {
    std::vector<Plan> out;
    if (n <= MAX_PASS_BITS) {
        out.push_back(default_plan(n));
        return out;
    }
    const int p0 = (n + MAX_PASS_BITS - 1) / MAX_PASS_BITS;
    for (int P = p0; P <= p0 + 1 && P <= MAX_PASSES; ++P) {
        int b[MAX_PASSES] = {0};
        // enumerate compositions with each part in [1, 9]
        std::vector<int> stack;
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
                if (valid_plan(p)) out.push_back(p);
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

// Workspace of one product: [error word, 256 B][A residues][B residues][ticket + state].
// The error word sits at offset 0 of every workspace and is never cleared by a job, so a
// caller can read (and clear) it after any number of jobs.
struct WsLayout {
    u64 N;
    int n;
    size_t a, b, ticket, state, total;
    u64 ncta;
    // wrapped (wrap = K > 0): the cyclic product at N plus the product of both operands'
    // lowest K limbs, a whole product at NL points whose residues sit at la_off / lb_off; or,
    // twisted, the product modulo X^NL - c of both operands folded (see k_twist_fold64)
    u64 wrap;
    u64 NL;
    size_t la_off, lb_off;
    bool twist;
};

// Wrapped plan of this engine (the 32-bit engine's plan_wrap, restated for limbs): a product
// of dc = la + lb - 1 coefficients with 2^n < dc and both operands within N = 2^n limbs runs as
// the cyclic convolution of length N (its entry k < K = dc - N holds c_k + c_{k+N}) plus the
// whole product of the operands' lowest K limbs (K < min(la, lb), so it gives c_0 .. c_{K-1}
// exactly), and the CRT + carry kernel separates the two (k_crt_carry_wrap).  Taken when its
// modelled cost, (1 + 2) transforms of N and of NL = ceil_pow2(2K - 1) points x (log + 1)
// plus one launch sequence, is below the whole product's at 2N, or when fmn_force_wrap asks.
// The twisted form (k_twist_fold64, k_twist_w64) needs a product modulo X^M - c of only
// M = 2^m >= K points (N / M <= 4, m >= 12) instead of the low product's 2K, at the price of the
// folded entry and the W pass; the cheapest of the three plans is taken (fmn_force_wrap(1)
// forces the low product, 2 the twisted form where it applies).
constexpr double kSeqCost64 = 1.25e7;      // launch overhead of one launch sequence, in (points x bits)
constexpr int kMinTwistLog64 = 12;
static bool wrap64_plan(u64 la, u64 lb, int sqr, u64* N_out, u64* K_out, u64* NL_out, bool* twist_out) {
    if (la == 0 || lb == 0) return false;
    const u64 dc = la + lb - 1;
    if (dc < 3) return false;
    const int n = ilog2(dc) - 1;               // ilog2 rounds up: 2^n < dc <= 2^(n+1)
    if (n < 12 || n + 1 > MAX_LOG_N) return false;
    const u64 N = 1ull << n;
    if (la > N || lb > N || dc <= N) return false;   // an operand would wrap onto itself
    const u64 K = dc - N;                      // 1 <= K < min(la, lb)
    const u64 NL = ceil_pow2(2 * K - 1);
    const double t = sqr ? 2.0 : 3.0;
    const double whole = t * (double)(2 * N) * (n + 2);
    const double wrap = t * (double)N * (n + 1) + t * (double)NL * (ilog2(NL) + 1) + kSeqCost64;
    int m = ilog2(K);                          // ilog2 rounds up: 2^m >= K
    if (m < n - 2) m = n - 2;
    if (m < kMinTwistLog64) m = kMinTwistLog64;
    const bool tw_ok = m <= n;
    const u64 M = 1ull << m;
    const double F = tw_ok ? (double)(1ull << (n - m)) : 0.0;
    // folds and W: elementwise passes over F limbs / residues per point, about half a butterfly level each
    const double twist = t * (double)N * (n + 1) + t * (double)M * (m + 1) +
                         0.5 * ((sqr ? 1.0 : 2.0) * (double)M * F + (double)K * (F + 3.0)) + kSeqCost64;
    // the cost model must promise 15%: the second product computes its four-step twiddles
    // (no tables) and a negacyclic M = N plan models within a few percent of the whole one
    // but measured slower (64M x 64M: 31.8 against 27.6 ms)
    const double limit = 0.85 * whole;
    const int fw = q32_forced_wrap();
    bool use_twist;
    if (fw == 1) use_twist = false;
    else if (fw == 2) use_twist = tw_ok;
    else if (wrap >= limit && (!tw_ok || twist >= limit)) return false;
    else use_twist = tw_ok && twist < wrap && twist < limit;
    *N_out = N;
    *K_out = K;
    *NL_out = use_twist ? M : NL;
    *twist_out = use_twist;
    return true;
}

// wrap_ok: the product may take the wrapped plan (single products; not batches, resident
// spectra or the fixed-size scratch of fmn_mul_device_noalloc).
static WsLayout ws_layout(u64 la, u64 lb, int sqr, int force_n = 0, bool wrap_ok = false) {
    WsLayout w;
    memset(&w, 0, sizeof(w));
    const u64 out_len = la + lb;
    if (la == 0 || lb == 0) return w;
    w.N = ceil_pow2(out_len - 1);
    if (force_n > 0 && (1ull << force_n) > w.N) w.N = 1ull << force_n;
    u64 N = 0, K = 0, NL = 0;
    bool tw = false;
    if (wrap_ok && force_n <= 0 && wrap64_plan(la, lb, sqr, &N, &K, &NL, &tw)) {
        w.N = N;
        w.wrap = K;
        w.NL = NL;
        w.twist = tw;
    }
    w.n = ilog2(w.N);
    w.ncta = (out_len + WCTILE - 1) / WCTILE;
    size_t off = 256;
    w.a = off;
    off = align256(off + 3 * w.N * sizeof(u64));
    w.b = off;
    if (!sqr) off = align256(off + 3 * w.N * sizeof(u64));
    if (w.wrap) {
        w.la_off = off;
        off = align256(off + 3 * w.NL * sizeof(u64));
        w.lb_off = off;
        if (!sqr) off = align256(off + 3 * w.NL * sizeof(u64));
    }
    w.ticket = off;
    w.state = off + 16;
    off = align256(w.state + w.ncta * sizeof(u32));
    w.total = off;
    return w;
}

static std::atomic<int> g_engine{ENGINE_AUTO};
void set_default_engine(int engine) { g_engine.store(engine); }
int default_engine() { return g_engine.load(); }

// A (point x bit) of this engine's transform costs about 2.4 times one of the 32-bit engine
// (measured on B200: 10M x 10M limbs, 2^25 64-bit points in 6.73 ms against 2^26 32-bit
// digits in 5.74 ms).
constexpr double kCost64 = 2.4;

int job_engine(const Job& j) {
    if (j.spectrum) return j.engine == ENGINE_32 ? ENGINE_32 : ENGINE_64;
    const int e = j.engine ? j.engine : default_engine();
    if (e == ENGINE_64) return ENGINE_64;
    const int sqr = j.sqr ? 1 : 0;
    if (!q32_fits(j.la, j.lb, sqr)) return ENGINE_64;
    if (e == ENGINE_32) return ENGINE_32;
    const u64 N = ceil_pow2(j.la + j.lb - 1);
    const double c64 = kCost64 * (sqr ? 2.0 : 3.0) * (double)N * (ilog2(N) + 1);
    return q32_cost(j.la, j.lb, sqr) <= c64 ? ENGINE_32 : ENGINE_64;
}

static Job plain_job(u64 la, u64 lb, int sqr) {
    Job j{};
    j.la = la;
    j.lb = lb;
    j.sqr = sqr;
    return j;
}

static bool wrap_ok(const Job& j) { return !j.spectrum && !j.no_wrap; }

size_t job_workspace_bytes(const Job& j) {
    if (job_engine(j) == ENGINE_32) return q32_job_workspace_bytes(j);
    const size_t t = ws_layout(j.la, j.lb, j.sqr, j.spectrum ? j.log_n : 0, wrap_ok(j)).total;
    return t ? t : 256;
}

u64 wrap64_for(const Job& j) {
    if (j.spectrum || j.la == 0 || j.lb == 0) return 0;
    return ws_layout(j.la, j.lb, j.sqr, 0, wrap_ok(j)).wrap;
}

int job_side_log_n(const Job& j) {
    if (j.spectrum || j.la == 0 || j.lb == 0 || job_engine(j) != ENGINE_64) return 0;
    const WsLayout w = ws_layout(j.la, j.lb, j.sqr, 0, wrap_ok(j));
    return w.wrap ? ilog2(w.NL) : 0;
}

u64 twist64_for(const Job& j) {
    if (j.spectrum || j.la == 0 || j.lb == 0) return 0;
    const WsLayout w = ws_layout(j.la, j.lb, j.sqr, 0, wrap_ok(j));
    return w.twist ? w.NL : 0;
}

int job_twiddle_log_n(const Job& j) {
    if (j.spectrum) return j.log_n;
    return ws_layout(j.la, j.lb, j.sqr, 0, wrap_ok(j)).n;
}

size_t job_workspace_bytes(u64 la, u64 lb, int sqr) { return job_workspace_bytes(plain_job(la, lb, sqr)); }

static cudaError_t launch_pass(int variant, int logl, const PassArgs& a, u64 tiles, cudaStream_t s);

cudaError_t spectrum_enqueue(const u64* src, u64 len, int log_n, u64* spec, cudaStream_t s, const TwiddleSet* tws,
                             const Plan& pl) {
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    if (!valid_plan(pl) || pl.n != log_n) return cudaErrorInvalidValue;
    if (tws && (tws->log_n != log_n || !same_plan(tws->plan, pl))) tws = nullptr;
    const int P = pl.passes;
    const u64 N = 1ull << log_n;
    PassArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.N = N;
    pa.ncols = TC;
    pa.src = src;
    pa.len = len;
    pa.data = spec;
    int logB = log_n;
    for (int p = 0; p + 1 < P; ++p) {
        pa.logB = logB;
        pa.tw = tws ? tws->fwd[p] : nullptr;
        if ((e = launch_pass(p == 0 ? V_FWD_E : V_FWD, pl.bits[p], pa, N >> (pl.bits[p] + 4), s)) != cudaSuccess)
            return e;
        logB -= pl.bits[p];
    }
    const int lastl = pl.bits[P - 1];
    const u64 nblk = N >> lastl;
    pa.tw = nullptr;
    pa.logB = logB;
    pa.ncols = nblk < (u64)TC ? (int)nblk : TC;
    return launch_pass(P == 1 ? V_LAST_E : V_LAST, lastl, pa, (nblk + TC - 1) / TC, s);
}

// ------------------------------------------------------------------ host: profiling
const char* kernel_kind_name(int k) {
    static const char* names[K_KINDS] = {"fwd_pass", "fwd_last_pass", "fused_pointwise_pass", "inv_pass",
                                         "crt_carry", "wrap_fold_w"};
    return (k >= 0 && k < K_KINDS) ? names[k] : "?";
}

namespace {
struct ProfRec {
    int kind;
    cudaEvent_t a, b;
    double bytes, modmuls;
};
struct ProfState {
    bool on = false;
    std::vector<ProfRec> recs;
    std::vector<cudaEvent_t> pool;
    cudaEvent_t get() {
        if (!pool.empty()) {
            cudaEvent_t e = pool.back();
            pool.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        cudaEventCreate(&e);
        return e;
    }
};
thread_local ProfState g_prof;
}  // namespace

void profile_enable(bool on) { g_prof.on = on; }

cudaError_t profile_take(KindStats* out) {
    for (ProfRec& r : g_prof.recs) {
        cudaError_t e = cudaEventSynchronize(r.b);
        if (e != cudaSuccess) return e;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, r.a, r.b);
        out[r.kind].ms += ms;
        out[r.kind].launches += 1;
        out[r.kind].bytes += r.bytes;
        out[r.kind].modmuls += r.modmuls;
        g_prof.pool.push_back(r.a);
        g_prof.pool.push_back(r.b);
    }
    g_prof.recs.clear();
    return cudaSuccess;
}

ProfMark prof_begin(int kind, double bytes, double modmuls, cudaStream_t s) {
    ProfMark m{kind, nullptr, bytes, modmuls};
    if (g_prof.on) {
        m.a = g_prof.get();
        cudaEventRecord(m.a, s);
    }
    return m;
}

void prof_end(const ProfMark& m, cudaStream_t s) {
    if (!g_prof.on || !m.a) return;
    ProfRec r{m.kind, m.a, g_prof.get(), m.bytes, m.modmuls};
    cudaEventRecord(r.b, s);
    g_prof.recs.push_back(r);
}

// Launch wrapper: records events around the launch when profiling is on.
template <class F>
static cudaError_t timed_launch(int kind, double bytes, double modmuls, cudaStream_t s, F&& launch) {
    const ProfMark m = prof_begin(kind, bytes, modmuls, s);
    launch();
    cudaError_t e = cudaGetLastError();
    prof_end(m, s);
    return e;
}

static int variant_kind(int v) {
    switch (v) {
        case V_FUSED2: return K_FUSED;
        case V_FWD: case V_FWD_E: return K_FWD;
        case V_LAST: case V_LAST_E: return K_FWD_LAST;
        case V_INV: return K_INV;
        default: return K_FUSED;
    }
}

static thread_local char g_launch_diag[128];
const char* launch_diag() { return g_launch_diag; }

static cudaError_t launch_pass(int variant, int logl, const PassArgs& a, u64 tiles, cudaStream_t s) {
    PassKernel k = ktab().k[variant][logl];
    snprintf(g_launch_diag, sizeof(g_launch_diag), "pass variant %d, %d bits, %llu tiles", variant, logl,
             (unsigned long long)tiles);
    if (!k) return cudaErrorInvalidValue;
    // algorithmic work of the launch (3 primes)
    const double N = (double)a.N, vec = 3.0 * N * 8.0;
    const double bfly = 3.0 * (N / 2.0) * logl;
    double bytes = 2.0 * vec, mm = bfly;
    const bool entry = (variant == V_FWD_E || variant == V_LAST_E || variant == V_FUSED_E || variant == V_SQR_E);
    if (entry) {
        bytes = (double)a.len * 8.0 + vec;
        mm += 3.0 * (double)a.len;
    }
    if (variant == V_FUSED2) {
        bytes += vec;                 // reads both operands, writes the product
        mm = 3.0 * bfly + 3.0 * N;
    } else if (variant == V_FUSED || variant == V_FUSED_E) {
        bytes += vec;                 // reads the other operand's spectrum too
        mm = 2.0 * bfly + 3.0 * N + (entry ? 3.0 * (double)a.len : 0.0);
    } else if (variant == V_SQR || variant == V_SQR_E) {
        mm = 2.0 * bfly + 3.0 * N + (entry ? 3.0 * (double)a.len : 0.0);
    }
    return timed_launch(variant_kind(variant), bytes, mm, s,
                        [&] { k<<<(unsigned)(tiles * 3), NT, pass_smem(logl, variant), s>>>(a); });
}

// Launches of one 64-bit product of the given layout length (pass launches + the CRT).
static int launches64(int n, int sqr) {
    const Plan pl = make_plan(n);
    const int P = pl.passes;
    // forward strided passes (A, and B unless squaring) + A's last pass + fused + inverse + crt
    if (!sqr && P >= 2 && pl.bits[P - 1] >= 5 && pl.bits[P - 1] <= 8) return 2 * (P - 1) + 1 + (P - 1) + 1;   // merged
    return sqr ? (P - 1) + 1 + (P - 1) + 1 : 2 * (P - 1) + 1 + 1 + (P - 1) + 1;
}

int job_launches(u64 la, u64 lb, int sqr) {
    if (la == 0 || lb == 0) return 0;
    if (job_engine(plain_job(la, lb, sqr)) == ENGINE_32) return q32_launches(la, lb, sqr);
    const WsLayout w = ws_layout(la, lb, sqr, 0, true);
    // a wrapped product adds the second product's pass launches (its own CRT is not run) and,
    // twisted, the folds and the W kernel
    return launches64(w.n, sqr) + (w.wrap ? launches64(ilog2(w.NL), sqr) - 1 : 0) + (w.twist ? (sqr ? 2 : 3) : 0);
}

// Every launch one product needs, in order, with its arguments (no launch happens here).
struct LaunchRec {
    int variant, logl;
    PassArgs pa;
    u64 tiles;
    bool needs_b;     // reads the second operand's limbs
};
struct JobLaunches {
    int count;
    LaunchRec rec[3 * MAX_PASSES + 2];
    CrtArgs crt;
    u64 ncta;
};

// Scratch pointers of one product: residue arrays and carry-scan state.
struct JobScratch {
    u64* A;
    u64* B;
    u32* ticket;
    u32* state;
    u32* err;
};

// wrap: the layout may take the wrapped plan (single products); the caller then plans and
// launches the low product itself (enqueue_job) and fills the CRT's wrap fields.
// prefolded: the operands' residues are already in the scratch arrays (a twisted product's
// folded operands), so the first pass reads them instead of the limbs.
static void plan_job(const Job& j, const JobScratch& sc, const TwiddleSet* tws, JobLaunches* out, bool wrap = false,
                     bool prefolded = false) {
    const u64 out_len = j.la + j.lb;
    const int sqr = j.sqr ? 1 : 0;
    const WsLayout w = ws_layout(j.la, j.lb, sqr, j.spectrum ? j.log_n : 0, wrap && wrap_ok(j));
    u64* A = sc.A;
    u64* B = sqr ? A : sc.B;
    const Plan pl = j.spectrum && j.splan.passes ? j.splan : make_plan(w.n);   // a spectrum keeps its plan
    const int P = pl.passes;
    const u64 N = w.N;
    if (tws && (tws->log_n != w.n || !same_plan(tws->plan, pl))) tws = nullptr;
    out->count = 0;
    auto add = [&](int variant, int logl, const PassArgs& pa, u64 tiles) {
        LaunchRec& r = out->rec[out->count++];
        r.variant = variant;
        r.logl = logl;
        r.pa = pa;
        r.tiles = tiles;
        r.needs_b = !sqr && j.b && pa.src == j.b;
    };
    PassArgs pa;
    memset(&pa, 0, sizeof(pa));
    pa.N = N;
    pa.ncols = TC;
    int logB[MAX_PASSES];
    logB[0] = w.n;
    for (int p = 1; p < P; ++p) logB[p] = logB[p - 1] - pl.bits[p - 1];
    const int lastl = pl.bits[P - 1];
    const u64 nblk_last = N >> lastl;
    const u64 tiles_last = (nblk_last + TC - 1) / TC;
    const int ncols_last = nblk_last < (u64)TC ? (int)nblk_last : TC;
    auto fwd_strided = [&](const u64* src, u64 len, u64* data) {
        for (int p = 0; p + 1 < P; ++p) {
            pa.src = src;
            pa.len = len;
            pa.data = data;
            pa.logB = logB[p];
            pa.tw = tws ? tws->fwd[p] : nullptr;
            add(p == 0 && !prefolded ? V_FWD_E : V_FWD, pl.bits[p], pa, N >> (pl.bits[p] + 4));
        }
    };
    const bool merged = !sqr && !j.spectrum && P >= 2 && lastl >= 5 && lastl <= 8;   // two tiles fit
    if (j.spectrum) {
        // resident first operand (conv_single, src/fast_mul.c:135-212): only the second
        // operand is transformed; the product lands in A, the spectrum stays intact
        fwd_strided(j.b, j.lb, B);
        pa.tw = nullptr;
        pa.src = j.b;
        pa.len = j.lb;
        pa.data = B;
        pa.other = (u64*)j.spectrum;
        pa.dst = A;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_FUSED_E : V_FUSED, lastl, pa, tiles_last);
        pa.dst = nullptr;
    } else if (merged) {
        fwd_strided(j.a, j.la, A);
        fwd_strided(j.b, j.lb, B);
        pa.tw = nullptr;
        pa.src = nullptr;
        pa.len = 0;
        pa.data = B;
        pa.other = A;
        pa.logB = logB[P - 1];
        pa.ncols = TC;
        add(V_FUSED2, lastl, pa, tiles_last);
    } else if (!sqr) {
        fwd_strided(j.a, j.la, A);
        pa.tw = nullptr;
        pa.src = j.a;
        pa.len = j.la;
        pa.data = A;
        pa.other = nullptr;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_LAST_E : V_LAST, lastl, pa, tiles_last);
        pa.ncols = TC;
        fwd_strided(j.b, j.lb, B);
        pa.tw = nullptr;
        pa.src = j.b;
        pa.len = j.lb;
        pa.data = B;
        pa.other = A;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_FUSED_E : V_FUSED, lastl, pa, tiles_last);
    } else {
        fwd_strided(j.a, j.la, A);
        pa.tw = nullptr;
        pa.src = j.a;
        pa.len = j.la;
        pa.data = A;
        pa.other = A;
        pa.logB = logB[P - 1];
        pa.ncols = ncols_last;
        add(P == 1 ? V_SQR_E : V_SQR, lastl, pa, tiles_last);
    }
    pa.ncols = TC;
    pa.src = nullptr;
    pa.len = 0;
    pa.other = nullptr;
    for (int p = P - 2; p >= 0; --p) {
        pa.data = A;
        pa.logB = logB[p];
        pa.tw = tws ? tws->inv[p] : nullptr;
        add(V_INV, pl.bits[p], pa, N >> (pl.bits[p] + 4));
    }
    // CRT constants: M_i^-1 * N^-1 * 2^128 mod p_i
    CrtArgs& ca = out->crt;
    memset(&ca, 0, sizeof(ca));
    for (int i = 0; i < 3; ++i) {
        const u64 p = kP[i];
        const unsigned __int128 M = (unsigned __int128)kP[(i + 1) % 3] * kP[(i + 2) % 3];
        const u64 minv = h_pow((u64)(M % p), p - 2, p);
        const u64 ninv = h_pow(N % p, p - 2, p);
        const u64 r1 = (u64)((((unsigned __int128)1) << 64) % p);
        // y = r * cst * 2^-64 with r = N * conv * 2^-64 (the pointwise Montgomery product)
        ca.cst[i] = h_mulmod(h_mulmod(minv, ninv, p), h_mulmod(r1, r1, p), p);
    }
    ca.res = A;
    ca.N = N;
    ca.nvalid = w.wrap || (out_len - 1) < N ? (out_len - 1) : N;
    ca.out = j.out;
    ca.out_len = out_len;
    ca.state = sc.state;
    ca.ticket = sc.ticket;
    ca.err = sc.err;
    out->ncta = w.ncta;
}

static cudaError_t launch_crt(const CrtArgs& ca, u64 ncta, cudaStream_t s) {
    const double crt_bytes = 3.0 * (double)ca.nvalid * 8.0 + 3.0 * (double)ca.wrap * 16.0 + (double)ca.out_len * 8.0;
    return timed_launch(K_CRT, crt_bytes, 3.0 * (double)ca.nvalid, s, [&] {
        if (ca.twisted) k_crt_carry_twist<<<(unsigned)ncta, CNT, 0, s>>>(ca);
        else if (ca.wrap) k_crt_carry_wrap<<<(unsigned)ncta, CNT, 0, s>>>(ca);
        else k_crt_carry<<<(unsigned)ncta, CNT, 0, s>>>(ca);
    });
}

// w^e mod p_i (plain form) for the tables' root w of order 2^30, e taken mod 2^30.
static u64 h_root64(int i, u64 e) { return h_pow(host_tables().w30[i], e & MASK30, kP[i]); }
// (w, floor(w 2^64 / p_i)): w as a Shoup constant.
static ulonglong2 h_shoup64(u64 w, int i) {
    return make_ulonglong2(w, (u64)(((unsigned __int128)w << 64) / kP[i]));
}

// The second product of a wrapped 64-bit product (see wrap64_plan) and what the main CRT takes
// from it: the low product (an ordinary whole product of the operands' lowest K limbs) or,
// twisted, the folds of both operands, the transform of the folded operands and the W kernel.
struct Side64 {
    JobLaunches rec;              // pass launches of the second product
    bool twist;
    int nfold;
    FoldArgs64 fold[2];
    u64 fold_blocks, w_blocks;
    TwistArgs64 tw;
};
static void plan_side64(const Job& j, const WsLayout& w, char* base, const JobScratch& sc, Side64* sd, CrtArgs* ca,
                        const TwiddleSet* tws_side) {
    const int sqr = j.sqr ? 1 : 0;
    Job jl = j;
    jl.out = nullptr;
    jl.no_wrap = true;
    JobScratch scl{(u64*)(base + w.la_off), (u64*)(base + w.lb_off), sc.ticket, sc.state, sc.err};
    sd->twist = w.twist;
    sd->nfold = 0;
    ca->low = scl.A;
    ca->wrap = w.wrap;
    if (!w.twist) {
        jl.la = w.wrap;
        jl.lb = w.wrap;
        plan_job(jl, scl, tws_side, &sd->rec);
        ca->low_N = sd->rec.crt.N;
        for (int i = 0; i < 3; ++i) ca->low_cst[i] = sd->rec.crt.cst[i];
        return;
    }
    const u64 N = w.N, M = w.NL;
    const int n = w.n, m = ilog2(M), tw_log = MAX_LOG_N - 1 - n;   // gamma of order 2N
    jl.la = jl.lb = M / 2;                                       // a transform of M points
    plan_job(jl, scl, tws_side, &sd->rec, false, true);
    for (int op = 0; op < (sqr ? 1 : 2); ++op) {
        FoldArgs64& f = sd->fold[sd->nfold++];
        memset(&f, 0, sizeof(f));
        f.src = op ? j.b : j.a;
        f.len = op ? j.lb : j.la;
        f.T = op ? scl.B : scl.A;
        f.logM = m;
        f.fold_log = n - m;
        f.tw_log = tw_log;
        for (int i = 0; i < 3; ++i)
            for (int jj = 0; jj < kMaxFolds64; ++jj) f.cpow[i][jj] = h_shoup64(h_root64(i, (u64)jj << (m + tw_log)), i);
    }
    sd->fold_blocks = (M + 255) / 256 < 1184 ? (M + 255) / 256 : 1184;
    TwistArgs64& t = sd->tw;
    memset(&t, 0, sizeof(t));
    t.U = sc.A;
    t.V = scl.A;
    t.N = N;
    t.K = w.wrap;
    t.logM = m;
    t.fold_log = n - m;
    t.tw_log = tw_log;
    for (int i = 0; i < 3; ++i) {
        const u64 p = kP[i];
        const u64 r64 = (u64)((((unsigned __int128)1) << 64) % p), r128 = h_mulmod(r64, r64, p);
        const u64 ninv = h_pow(N % p, p - 2, p), inv_r64 = h_pow(r64, p - 2, p);
        t.cstM[i] = h_mulmod(h_pow(M % p, p - 2, p), r128, p);
        for (int jj = 0; jj < kMaxFolds64; ++jj)   // c^j N^-1 2^64
            t.ucj[i][jj] = h_shoup64(h_mulmod(h_mulmod(h_root64(i, (u64)jj << (m + tw_log)), ninv, p), r64, p), i);
        t.nraw[i] = h_shoup64(h_mulmod(N % p, inv_r64, p), i);   // N 2^-64
        // W is plain: y = W M_i^-1 (M_i the product of the other two primes)
        const unsigned __int128 Mi = (unsigned __int128)kP[(i + 1) % 3] * kP[(i + 2) % 3];
        ca->low_cst[i] = h_mulmod(h_pow((u64)(Mi % p), p - 2, p), r64, p);
    }
    sd->w_blocks = (w.wrap + 255) / 256 < 2048 ? (w.wrap + 255) / 256 : 2048;
    ca->low_N = M;
    ca->twisted = 1;
}
// The folds and the second product's passes (they read both operands).
static cudaError_t run_side64(const Side64& sd, cudaStream_t s) {
    cudaError_t e;
    for (int f = 0; f < sd.nfold; ++f) {
        const FoldArgs64& fa = sd.fold[f];
        const double M = (double)(1ull << fa.logM);
        e = timed_launch(K_WRAP, (double)fa.len * 8.0 + 3.0 * M * 8.0, 3.0 * M * (2.0 + (double)(1 << fa.fold_log)), s,
                         [&] { k_twist_fold64<<<(unsigned)sd.fold_blocks, 256, 0, s>>>(fa); });
        if (e != cudaSuccess) return e;
    }
    for (int k = 0; k < sd.rec.count; ++k)
        if ((e = launch_pass(sd.rec.rec[k].variant, sd.rec.rec[k].logl, sd.rec.rec[k].pa, sd.rec.rec[k].tiles, s)) !=
            cudaSuccess)
            return e;
    return cudaSuccess;
}
// Twisted: the W kernel, after the cyclic product's inverse passes.
static cudaError_t run_side64_w(const Side64& sd, cudaStream_t s) {
    if (!sd.twist) return cudaSuccess;
    const TwistArgs64& t = sd.tw;
    const double F = (double)(1 << t.fold_log);
    return timed_launch(K_WRAP, 3.0 * (double)t.K * 8.0 * (F + 3.0), 3.0 * (double)t.K * (F + 3.0), s,
                        [&] { k_twist_w64<<<dim3((unsigned)sd.w_blocks, 3), 256, 0, s>>>(t); });
}

cudaError_t enqueue_job(const Job& j, void* ws, size_t ws_bytes, cudaStream_t s, const TwiddleSet* tws,
                        const TwiddleSet* tws_side) {
    const u64 out_len = j.la + j.lb;
    if (out_len == 0) return cudaSuccess;
    if (j.la == 0 || j.lb == 0) return cudaMemsetAsync(j.out, 0, out_len * sizeof(u64), s);
    if (job_engine(j) == ENGINE_32) return q32_enqueue(j, ws, ws_bytes, s, nullptr, nullptr, 1, nullptr, nullptr);
    const int sqr = j.sqr ? 1 : 0;
    const WsLayout w = ws_layout(j.la, j.lb, sqr, j.spectrum ? j.log_n : 0, wrap_ok(j));
    if (ws_bytes < w.total || w.n > MAX_LOG_N) return cudaErrorInvalidValue;
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    char* base = (char*)ws;
    JobScratch sc{(u64*)(base + w.a), (u64*)(base + w.b), (u32*)(base + w.ticket), (u32*)(base + w.state),
                  (u32*)base};
    JobLaunches L;
    plan_job(j, sc, tws, &L, true);
    Side64 sd;
    sd.rec.count = 0;
    sd.twist = false;
    sd.nfold = 0;
    if (w.wrap) {
        plan_side64(j, w, base, sc, &sd, &L.crt, tws_side);
        if ((e = run_side64(sd, s)) != cudaSuccess) return e;
    }
    for (int k = 0; k < L.count; ++k) {
        const LaunchRec& r = L.rec[k];
        if ((e = launch_pass(r.variant, r.logl, r.pa, r.tiles, s)) != cudaSuccess) return e;
    }
    if ((e = run_side64_w(sd, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(base + w.ticket, 0, w.total - w.ticket, s)) != cudaSuccess) return e;
    return launch_crt(L.crt, L.ncta, s);
}

cudaError_t enqueue_job_overlapped(const Job& j, void* ws, size_t ws_bytes, cudaStream_t s, const TwiddleSet* tws,
                                   NeedLimbs need_b, void* need_ctx, int crt_chunks, ChunkDone after_chunk, void* ctx,
                                   const TwiddleSet* tws_side) {
    const u64 out_len = j.la + j.lb;
    if (j.la == 0 || j.lb == 0 || out_len == 0) return cudaErrorInvalidValue;
    if (job_engine(j) == ENGINE_32)
        return q32_enqueue(j, ws, ws_bytes, s, need_b, need_ctx, crt_chunks, after_chunk, ctx);
    const int sqr = j.sqr ? 1 : 0;
    const WsLayout w = ws_layout(j.la, j.lb, sqr, j.spectrum ? j.log_n : 0, wrap_ok(j));
    if (ws_bytes < w.total || w.n > MAX_LOG_N) return cudaErrorInvalidValue;
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    char* base = (char*)ws;
    JobScratch sc{(u64*)(base + w.a), (u64*)(base + w.b), (u32*)(base + w.ticket), (u32*)(base + w.state),
                  (u32*)base};
    JobLaunches L;
    plan_job(j, sc, tws, &L, true);
    Side64 sd;
    sd.rec.count = 0;
    sd.twist = false;
    sd.nfold = 0;
    if (w.wrap) plan_side64(j, w, base, sc, &sd, &L.crt, tws_side);
    // the first operand's passes, then (once the second operand is copied) the second product,
    // which reads both, and the rest
    bool waited = false, low_done = w.wrap == 0;
    auto run_low = [&]() -> cudaError_t {
        low_done = true;
        return run_side64(sd, s);
    };
    for (int k = 0; k < L.count; ++k) {
        const LaunchRec& r = L.rec[k];
        if (r.needs_b && !waited && need_b) {           // second operand copied meanwhile
            if ((e = need_b(need_ctx, 0, j.lb, s)) != cudaSuccess) return e;
            waited = true;
        }
        if ((r.needs_b || sqr) && !low_done && (e = run_low()) != cudaSuccess) return e;
        if ((e = launch_pass(r.variant, r.logl, r.pa, r.tiles, s)) != cudaSuccess) return e;
    }
    if (!low_done) {
        if (!waited && need_b && !sqr && (e = need_b(need_ctx, 0, j.lb, s)) != cudaSuccess) return e;
        if ((e = run_low()) != cudaSuccess) return e;
    }
    if ((e = run_side64_w(sd, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(base + w.ticket, 0, w.total - w.ticket, s)) != cudaSuccess) return e;
    // carry scan in chunks of CTAs: tickets continue across launches, each chunk's limbs are
    // final once its launch completes
    if (crt_chunks < 1) crt_chunks = 1;
    const u64 per = (L.ncta + crt_chunks - 1) / crt_chunks;
    for (u64 t0 = 0; t0 < L.ncta; t0 += per) {
        const u64 n = t0 + per <= L.ncta ? per : L.ncta - t0;
        if ((e = launch_crt(L.crt, n, s)) != cudaSuccess) return e;
        const u64 lo = t0 * WCTILE, hi = (t0 + n) * WCTILE < out_len ? (t0 + n) * WCTILE : out_len;
        if (after_chunk && (e = after_chunk(ctx, lo, hi)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// ------------------------------------------------------------------ batches
// Batched kernels: products with the same transform length and kind share every launch.
// CTA b works on product b / (3 * tiles), tile (b / 3) % tiles, prime b % 3.
template <int MODE, int LOGL, bool ENTRY, bool SQR>
__global__ void __launch_bounds__(NT, (pass_min_ctas<MODE, LOGL>())) k_pass_batch(const PassArgs* __restrict__ args,
                                                                                  u32 tiles) {
    extern __shared__ __align__(16) u64 sm[];
    const int pi = blockIdx.x % 3;
    const u32 rest = blockIdx.x / 3;
    const PassArgs a = args[rest / tiles];
    const u64 tile = rest % tiles;
    const PrimeRT q = c_prime[pi];
    if constexpr (MODE == M_FWD) body_fwd<LOGL, ENTRY>(sm, a, tile, pi, q);
    else if constexpr (MODE == M_INV) body_inv<LOGL>(sm, a, tile, pi, q);
    else if constexpr (MODE == M_FWD_LAST) body_fwd_last<LOGL, ENTRY>(sm, a, tile, pi, q);
    else if constexpr (MODE == M_FUSED2) body_fused2<(LOGL >= 5 ? LOGL : 5)>(sm, a, tile, pi, q);
    else body_fused<LOGL, ENTRY, SQR>(sm, a, tile, pi, q);
}

// CRT + carry of many products: CTAs take per-product tickets; tickets beyond a product's
// tile count exit at once.
__global__ void __launch_bounds__(CNT) k_crt_carry_batch(const CrtArgs* __restrict__ args, u32 ctas_per_job,
                                                         const u32* __restrict__ ncta) {
    const u32 job = blockIdx.x / ctas_per_job;
    crt_carry_body<0>(args[job], ncta[job]);
}

typedef void (*BatchKernel)(const PassArgs*, u32);
template <int MODE, int LOGL, bool ENTRY, bool SQR>
static BatchKernel bkernel_ptr() {
    return k_pass_batch<MODE, LOGL, ENTRY, SQR>;
}
template <int LOGL>
static void fill_brow(BatchKernel (&t)[NV][MAX_PASS_BITS + 1]) {
    constexpr int LS = LOGL >= 5 ? LOGL : 5;
    t[V_FWD][LOGL] = LOGL >= 5 ? bkernel_ptr<M_FWD, LS, false, false>() : nullptr;
    t[V_FWD_E][LOGL] = LOGL >= 5 ? bkernel_ptr<M_FWD, LS, true, false>() : nullptr;
    t[V_INV][LOGL] = LOGL >= 5 ? bkernel_ptr<M_INV, LS, false, false>() : nullptr;
    t[V_FUSED2][LOGL] = (LOGL >= 5 && LOGL <= 8) ? bkernel_ptr<M_FUSED2, (LOGL <= 8 ? LS : 5), false, false>() : nullptr;
    t[V_LAST][LOGL] = bkernel_ptr<M_FWD_LAST, LOGL, false, false>();
    t[V_LAST_E][LOGL] = bkernel_ptr<M_FWD_LAST, LOGL, true, false>();
    t[V_FUSED][LOGL] = bkernel_ptr<M_FUSED, LOGL, false, false>();
    t[V_FUSED_E][LOGL] = bkernel_ptr<M_FUSED, LOGL, true, false>();
    t[V_SQR][LOGL] = bkernel_ptr<M_FUSED, LOGL, false, true>();
    t[V_SQR_E][LOGL] = bkernel_ptr<M_FUSED, LOGL, true, true>();
}
struct BatchKernelTable {
    BatchKernel k[NV][MAX_PASS_BITS + 1];
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

static cudaError_t set_batch_attrs() {
    const BatchKernelTable& K = bktab();
    for (int v = 0; v < NV; ++v)
        for (int l = 0; l <= MAX_PASS_BITS; ++l)
            if (K.k[v][l]) {
                cudaError_t e = cudaFuncSetAttribute((const void*)K.k[v][l],
                                                     cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pass_smem(l, v));
                if (e != cudaSuccess) return e;
                e = cudaFuncSetAttribute((const void*)K.k[v][l], cudaFuncAttributePreferredSharedMemoryCarveout,
                                         (int)cudaSharedmemCarveoutMaxShared);
                if (e != cudaSuccess) return e;
            }
    return cudaSuccess;
}

// Batch layout inside one workspace:
//   [status word, 256 B][per-product residues][per-product ticket+state][launch descriptors]
// Products are grouped by (transform length, square); each group's launches run on one of
// the streams in `streams` (round robin), forked from and joined back into `s`.
struct BatchGroup {
    int engine, n, kind;  // kind: 0 multiply, 1 square, 2 resident first operand
    int twist;            // 32-bit engine: log2 M of twisted wrapped products, 0 for whole ones
    std::vector<int> idx;
};
static int job_kind(const Job& j) { return j.spectrum ? 2 : (j.sqr ? 1 : 0); }

// Engine of a batched product: the 32-bit engine for every whole product it can take (batched
// products are small; resident operands keep 64-bit spectra), unless ENGINE_64 is selected.
static int batch_engine(const Job& j) {
    if (j.spectrum) return j.engine == ENGINE_32 ? ENGINE_32 : ENGINE_64;
    const int e = j.engine ? j.engine : default_engine();
    if (e == ENGINE_64) return ENGINE_64;
    return q32_batch_log_n(j) >= 0 ? ENGINE_32 : ENGINE_64;
}

bool batch_on_engine64(const Job& j) { return j.la && j.lb && batch_engine(j) == ENGINE_64; }

u64 batch_twist_for(const Job& j) {
    if (j.la == 0 || j.lb == 0 || batch_engine(j) != ENGINE_32) return 0;
    const int m = q32_batch_twist_log(j);
    return m ? 1ull << m : 0;
}

static void batch_sizes(const Job& j, size_t* res, size_t* st) {
    if (batch_engine(j) == ENGINE_32) {
        *res += q32_batch_res_bytes(j);
        *st += q32_batch_state_bytes(j);
        return;
    }
    const WsLayout w = ws_layout(j.la, j.lb, j.sqr, j.spectrum ? j.log_n : 0);
    *res += align256(3 * w.N * sizeof(u64)) * (j.sqr ? 1 : 2);
    *st += 16 + ((w.ncta * sizeof(u32) + 15) & ~(size_t)15);
}

static void batch_groups(const Job* jobs, int count, std::vector<BatchGroup>& groups) {
    groups.clear();
    for (int i = 0; i < count; ++i) {
        const Job& j = jobs[i];
        if (j.la == 0 || j.lb == 0) continue;
        const int eng = batch_engine(j);
        const int n = eng == ENGINE_32 ? q32_batch_log_n(j) : ws_layout(j.la, j.lb, j.sqr, j.spectrum ? j.log_n : 0).n;
        const int sq = job_kind(j);
        const int tw = eng == ENGINE_32 ? q32_batch_twist_log(j) : 0;
        BatchGroup* g = nullptr;
        for (auto& x : groups)
            if (x.engine == eng && x.n == n && x.kind == sq && x.twist == tw) g = &x;
        if (!g) {
            groups.push_back(BatchGroup{eng, n, sq, tw, {}});
            g = &groups.back();
        }
        g->idx.push_back(i);
    }
}

size_t batch_stage_bytes(const Job* jobs, int count);

size_t batch_workspace_bytes(const Job* jobs, int count) {
    size_t res = 0, st = 0;
    for (int i = 0; i < count; ++i) {
        const Job& j = jobs[i];
        if (j.la == 0 || j.lb == 0) continue;
        batch_sizes(j, &res, &st);
    }
    return 256 + align256(res) + align256(st) + align256(batch_stage_bytes(jobs, count));
}

cudaError_t enqueue_batch(const Job* jobs, int count, void* ws, size_t ws_bytes, void* h_stage, size_t stage_bytes,
                          cudaStream_t s, const cudaStream_t* streams, const cudaEvent_t* events, int nstreams,
                          TwiddleLookup tw_lookup, void* tw_ctx) {
    if (count <= 0) return cudaSuccess;
    const size_t need = batch_workspace_bytes(jobs, count);
    if (ws_bytes < need) return cudaErrorInvalidValue;
    cudaError_t e = prepare_batch();
    if (e != cudaSuccess) return e;
    std::vector<BatchGroup> groups;
    batch_groups(jobs, count, groups);
    // zero-length products: the product is zero
    for (int i = 0; i < count; ++i)
        if ((jobs[i].la == 0 || jobs[i].lb == 0) && jobs[i].la + jobs[i].lb > 0)
            if ((e = cudaMemsetAsync(jobs[i].out, 0, (jobs[i].la + jobs[i].lb) * sizeof(u64), s)) != cudaSuccess)
                return e;
    // carve the workspace
    char* base = (char*)ws;
    size_t res = 0, st = 0;
    for (int i = 0; i < count; ++i) {
        const Job& j = jobs[i];
        if (j.la == 0 || j.lb == 0) continue;
        batch_sizes(j, &res, &st);
    }
    char* res_base = base + 256;
    char* st_base = res_base + align256(res);
    char* desc_base = st_base + align256(st);
    // descriptors are built in pinned host staging memory, then copied in one transfer
    char* hp = (char*)h_stage;
    size_t hoff = 0;
    auto hreserve = [&](size_t bytes) -> size_t {
        const size_t o = hoff;
        hoff = (hoff + bytes + 15) & ~(size_t)15;
        return o;
    };
    struct GroupLaunch {
        int count;
        int variant[3 * MAX_PASSES + 2], logl[3 * MAX_PASSES + 2];
        u64 tiles[3 * MAX_PASSES + 2];
        size_t args_off[3 * MAX_PASSES + 2];
        size_t crt_off, ncta_off;
        u32 max_ncta;
        int m;
        char* st_lo;
        size_t st_bytes;
    };
    std::vector<GroupLaunch> gl(groups.size());
    std::vector<Q32Group> qg(groups.size());
    size_t roff = 0, soff = 0;
    std::vector<JobLaunches> jl;
    for (size_t g = 0; g < groups.size(); ++g) {
        const BatchGroup& G = groups[g];
        const int m = (int)G.idx.size();
        if (G.engine == ENGINE_32) {
            e = q32_batch_plan(jobs, G.idx.data(), m, res_base, &roff, st_base, &soff, (u32*)base, hp, &hoff,
                               stage_bytes, &qg[g]);
            if (e != cudaSuccess) return e;
            continue;
        }
        const TwiddleSet* tws = tw_lookup ? tw_lookup(tw_ctx, G.n) : nullptr;
        jl.assign(m, JobLaunches());
        GroupLaunch& L = gl[g];
        L.m = m;
        L.st_lo = st_base + soff;
        u32 maxc = 0;
        for (int t = 0; t < m; ++t) {
            const Job& j = jobs[G.idx[t]];
            const WsLayout w = ws_layout(j.la, j.lb, j.sqr, j.spectrum ? j.log_n : 0);
            JobScratch sc;
            sc.A = (u64*)(res_base + roff);
            roff += align256(3 * w.N * sizeof(u64));
            sc.B = sc.A;
            if (!j.sqr) {
                sc.B = (u64*)(res_base + roff);
                roff += align256(3 * w.N * sizeof(u64));
            }
            sc.ticket = (u32*)(st_base + soff);
            sc.state = sc.ticket + 4;
            soff += 16 + ((w.ncta * sizeof(u32) + 15) & ~(size_t)15);
            sc.err = (u32*)base;
            plan_job(j, sc, tws, &jl[t]);
            if (jl[t].ncta > maxc) maxc = (u32)jl[t].ncta;
        }
        L.st_bytes = (size_t)(st_base + soff - L.st_lo);
        L.max_ncta = maxc;
        L.count = jl[0].count;
        for (int k = 0; k < L.count; ++k) {
            L.variant[k] = jl[0].rec[k].variant;
            L.logl[k] = jl[0].rec[k].logl;
            L.tiles[k] = jl[0].rec[k].tiles;
            L.args_off[k] = hreserve((size_t)m * sizeof(PassArgs));
            if (hoff > stage_bytes) return cudaErrorInvalidValue;
            PassArgs* dst = (PassArgs*)(hp + L.args_off[k]);
            for (int t = 0; t < m; ++t) dst[t] = jl[t].rec[k].pa;
        }
        L.crt_off = hreserve((size_t)m * sizeof(CrtArgs));
        L.ncta_off = hreserve((size_t)m * sizeof(u32));
        if (hoff > stage_bytes) return cudaErrorInvalidValue;
        CrtArgs* cd = (CrtArgs*)(hp + L.crt_off);
        u32* nc = (u32*)(hp + L.ncta_off);
        for (int t = 0; t < m; ++t) {
            cd[t] = jl[t].crt;
            nc[t] = (u32)jl[t].ncta;
        }
    }
    if (hoff > (size_t)((base + need) - desc_base)) return cudaErrorInvalidValue;
    if ((e = cudaMemcpyAsync(desc_base, hp, hoff, cudaMemcpyHostToDevice, s)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(st_base, 0, align256(st), s)) != cudaSuccess) return e;
    // fork: every worker stream waits for the descriptors (and any twiddle tables built on s)
    if (nstreams > 0) {
        if ((e = cudaEventRecord(events[0], s)) != cudaSuccess) return e;
        for (int k = 0; k < nstreams; ++k)
            if ((e = cudaStreamWaitEvent(streams[k], events[0], 0)) != cudaSuccess) return e;
    }
    const BatchKernelTable& BK = bktab();
    for (size_t g = 0; g < groups.size(); ++g) {
        const GroupLaunch& L = gl[g];
        cudaStream_t gs = nstreams > 0 ? streams[g % nstreams] : s;
        if (groups[g].engine == ENGINE_32) {
            if ((e = q32_batch_launch(qg[g], desc_base, gs)) != cudaSuccess) return e;
            continue;
        }
        for (int k = 0; k < L.count; ++k) {
            BatchKernel kk = BK.k[L.variant[k]][L.logl[k]];
            if (!kk) return cudaErrorInvalidValue;
            const PassArgs* d_args = (const PassArgs*)(desc_base + L.args_off[k]);
            const unsigned grid = (unsigned)((u64)L.m * L.tiles[k] * 3);
            kk<<<grid, NT, pass_smem(L.logl[k], L.variant[k]), gs>>>(d_args, (u32)L.tiles[k]);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
        k_crt_carry_batch<<<(unsigned)(L.m * L.max_ncta), CNT, 0, gs>>>(
            (const CrtArgs*)(desc_base + L.crt_off), L.max_ncta, (const u32*)(desc_base + L.ncta_off));
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    // join
    for (int k = 0; k < nstreams; ++k) {
        if ((e = cudaEventRecord(events[1 + k], streams[k])) != cudaSuccess) return e;
        if ((e = cudaStreamWaitEvent(s, events[1 + k], 0)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t prepare_batch() {
    cudaError_t e = ensure_tables();
    if (e != cudaSuccess) return e;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    static std::mutex mu;
    static std::vector<int> done;
    std::lock_guard<std::mutex> lk(mu);
    for (int d : done)
        if (d == dev) return cudaSuccess;
    if ((e = set_batch_attrs()) != cudaSuccess) return e;
    if ((e = q32_prepare()) != cudaSuccess) return e;
    done.push_back(dev);
    return cudaSuccess;
}

size_t batch_stage_bytes(const Job* jobs, int count) {
    size_t desc = 0;
    const size_t per64 = (3 * MAX_PASSES + 2) * (sizeof(PassArgs) + 16) + sizeof(CrtArgs) + sizeof(u32) + 32;
    const size_t per32 = q32_batch_desc_bytes_per_job();
    for (int i = 0; i < count; ++i) desc += per64 > per32 ? per64 : per32;
    return desc + 4096;
}

// ------------------------------------------------------------------ synthetic limbs (tuning)
__global__ void k_fill(u64* p, u64 n, u64 seed) {
    for (u64 i = blockIdx.x * (u64)blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        u64 z = seed + (i + 1) * 0x9E3779B97F4A7C15ull;       // splitmix64
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        p[i] = z ^ (z >> 31);
    }
}

cudaError_t fill_limbs(u64* p, u64 n, u64 seed, cudaStream_t s) {
    k_fill<<<148 * 8, 256, 0, s>>>(p, n, seed);
    return cudaGetLastError();
}

// ------------------------------------------------------------------ modmul microbenchmark
constexpr int MB_CHAINS = 8, MB_ITERS = 2048;
__global__ void __launch_bounds__(256) k_bench_modmul(u64* sink, u64 y) {
    const PrimeRT q = c_prime[2];
    u64 x[MB_CHAINS];
#pragma unroll
    for (int i = 0; i < MB_CHAINS; ++i) x[i] = (u64)(blockIdx.x * 256 + threadIdx.x) * 0x9E3779B97F4A7C15ull + i;
#pragma unroll 1
    for (int it = 0; it < MB_ITERS; ++it) {
#pragma unroll
        for (int i = 0; i < MB_CHAINS; ++i) x[i] = mmul(x[i], y, q);   // any x < 2^64 with y < p
    }
    u64 acc = 0;
#pragma unroll
    for (int i = 0; i < MB_CHAINS; ++i) acc ^= x[i];
    if (acc == 0x123456789ull) sink[0] = acc;
}
__global__ void __launch_bounds__(256) k_bench_bfly(u64* sink, ulonglong2 w) {
    const PrimeRT q = c_prime[2];
    u64 x[2 * MB_CHAINS];
#pragma unroll
    for (int i = 0; i < 2 * MB_CHAINS; ++i) x[i] = ((u64)(blockIdx.x * 256 + threadIdx.x) * 0x9E3779B97F4A7C15ull + i) >> 3;
#pragma unroll 1
    for (int it = 0; it < MB_ITERS; ++it) {
#pragma unroll
        for (int i = 0; i < MB_CHAINS; ++i) bfly_dif(x[i], x[i + MB_CHAINS], w, q);
    }
    u64 acc = 0;
#pragma unroll
    for (int i = 0; i < 2 * MB_CHAINS; ++i) acc ^= x[i];
    if (acc == 0x123456789ull) sink[0] = acc;
}

cudaError_t bench_modmul(double* per_second, double* bfly_per_second) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    u64* sink = nullptr;
    cudaError_t e = cudaMalloc(&sink, 64);
    if (e != cudaSuccess) return e;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    const unsigned grid = (unsigned)sms * 8;
    const u64 y = 1234567890123456789ull % Prime<2>::P, w0 = 987654321987654321ull % Prime<2>::P;
    const ulonglong2 w = make_ulonglong2(w0, (u64)((((unsigned __int128)w0) << 64) / Prime<2>::P));
    float best = 1e30f, bestb = 1e30f;
    for (int rep = 0; rep < 4; ++rep) {
        cudaEventRecord(a);
        k_bench_modmul<<<grid, 256>>>(sink, y);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        float ms;
        cudaEventElapsedTime(&ms, a, b);
        if (rep && ms < best) best = ms;
        cudaEventRecord(a);
        k_bench_bfly<<<grid, 256>>>(sink, w);
        cudaEventRecord(b);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        if (rep && ms < bestb) bestb = ms;
    }
    e = cudaGetLastError();
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    cudaFree(sink);
    const double n = (double)grid * 256.0 * MB_CHAINS * MB_ITERS;
    *per_second = n / (best * 1e-3);
    *bfly_per_second = n / (bestb * 1e-3);
    return e;
}

}  // namespace fmn
