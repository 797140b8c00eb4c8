// fmn_rounds.cuh -- round structure of a 2^m-point sub-transform, shared by both residue
// engines (64-bit residues in fmn_ntt.cu, 32-bit residues in fmn_ntt32.cu).
#pragma once

namespace fmn {

constexpr int RT_MAXLOGL = 12;    // round tables cover sub-transforms up to 2^12 points

// A 2^m-point sub-transform is done in rounds of radix 2^RB held in registers.
__host__ __device__ constexpr int rounds_count(int logl) {
    return logl == 0 ? 0 : logl <= 4 ? 1 : logl <= 8 ? 2 : 3;
}
__host__ __device__ constexpr int round_bits(int logl, int idx) {
    return logl <= 4 ? logl
         : logl <= 8 ? (idx == 0 ? (logl + 1) / 2 : logl / 2)
                     : (idx == 0 ? (logl + 2) / 3 : idx == 1 ? (logl + 1) / 3 : logl / 3);
}
__host__ __device__ constexpr int round_top(int logl, int idx) {
    return idx == 0 ? logl - 1 : round_top(logl, idx - 1) - round_bits(logl, idx - 1);
}

// Round twiddle tables.  For a round of RB bits whose top index bit is TOP, the group with
// low offset q (q < 2^(TOP-RB+1)) needs, for stage s (span 2^(TOP-s)) and u < 2^(RB-1-s):
//     w_{2^(TOP-s+1)}^(q + u * 2^(TOP-RB+1))
// as its stage entry j = 2^RB - 2^(RB-s) + u (j < 2^RB - 1), stored stage-major at
// rt_off(RB, TOP) + j * 2^(TOP-RB+1) + q, so lanes holding consecutive groups read
// consecutive entries.
__host__ __device__ constexpr int rt_base(int r) {
    return r <= 1 ? 0 : rt_base(r - 1) + (1 << (r - 1)) * ((1 << (RT_MAXLOGL - r + 2)) - 1);
}
__host__ __device__ constexpr int rt_off(int r, int top) {
    return rt_base(r) + (1 << r) * ((1 << (top - r + 1)) - 1);
}
constexpr int RT_SIZE = rt_base(5);

}  // namespace fmn
