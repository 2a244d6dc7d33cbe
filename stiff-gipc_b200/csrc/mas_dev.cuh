// mas_dev.cuh -- device building blocks of the MAS apply shared by the
// per-phase kernels (mas.cu) and the persistent PCG kernel
// (pcg_persistent.cu).
#pragma once
#include "common.cuh"

namespace sgmas {

__host__ __device__ constexpr int bsym_of(int B) { return B * (B + 1) / 2; }
__host__ __device__ __forceinline__ int sym_index(int B, int r, int c) { return B * r - r * (r + 1) / 2 + c; }
__host__ __device__ __forceinline__ int round_up(int v, int b) { return (v + b - 1) / b * b; }

template <typename Acc>
__device__ __forceinline__ Acc shfl_acc(Acc v, int src, int width) { return __shfl_sync(0xffffffffu, v, src, width); }

// Factored tile (Fact<T>): slot sym_index(J, I), J <= I, holds the 3x3
// block (I, J) of W = L^-1, column-major.  z = W^T (W r): pass 1 y_I =
// sum_{J <= I} W_IJ r_J, pass 2 z_I = sum_{J >= I} W_JI^T y_J, J ascending,
// each component an fma chain (the order the oracle restates).
template <int B, typename S, typename Acc>
__device__ __forceinline__ void schwarz_factored(const S* tile, int lane, Acc r0, Acc r1, Acc r2, Acc& z0, Acc& z1,
                                                 Acc& z2) {
    Acc y0 = 0, y1 = 0, y2 = 0;
    #pragma unroll 4
    for (int c = 0; c < B; ++c) {
        const Acc x0 = shfl_acc(r0, c, B), x1 = shfl_acc(r1, c, B), x2 = shfl_acc(r2, c, B);
        if (c <= lane) {
            const S* P = tile + sym_index(B, c, lane) * 9;  // block (lane, c)
            y0 = fma_acc(Store<S>::to_acc(P[0]), x0, y0);
            y0 = fma_acc(Store<S>::to_acc(P[3]), x1, y0);
            y0 = fma_acc(Store<S>::to_acc(P[6]), x2, y0);
            y1 = fma_acc(Store<S>::to_acc(P[1]), x0, y1);
            y1 = fma_acc(Store<S>::to_acc(P[4]), x1, y1);
            y1 = fma_acc(Store<S>::to_acc(P[7]), x2, y1);
            y2 = fma_acc(Store<S>::to_acc(P[2]), x0, y2);
            y2 = fma_acc(Store<S>::to_acc(P[5]), x1, y2);
            y2 = fma_acc(Store<S>::to_acc(P[8]), x2, y2);
        }
    }
    Acc a0 = 0, a1 = 0, a2 = 0;
    #pragma unroll 4
    for (int c = 0; c < B; ++c) {
        const Acc w0 = shfl_acc(y0, c, B), w1 = shfl_acc(y1, c, B), w2 = shfl_acc(y2, c, B);
        if (c >= lane) {
            const S* P = tile + sym_index(B, lane, c) * 9;  // block (c, lane), used transposed
            a0 = fma_acc(Store<S>::to_acc(P[0]), w0, a0);
            a0 = fma_acc(Store<S>::to_acc(P[1]), w1, a0);
            a0 = fma_acc(Store<S>::to_acc(P[2]), w2, a0);
            a1 = fma_acc(Store<S>::to_acc(P[3]), w0, a1);
            a1 = fma_acc(Store<S>::to_acc(P[4]), w1, a1);
            a1 = fma_acc(Store<S>::to_acc(P[5]), w2, a1);
            a2 = fma_acc(Store<S>::to_acc(P[6]), w0, a2);
            a2 = fma_acc(Store<S>::to_acc(P[7]), w1, a2);
            a2 = fma_acc(Store<S>::to_acc(P[8]), w2, a2);
        }
    }
    z0 = a0; z1 = a1; z2 = a2;
}

// z_lane = sum_c P(lane, c) r_c over one bank; columns ascending, each 3x3
// row an fma chain (the order the oracle restates).  Factored tiles take
// schwarz_factored.
template <int B, typename S, typename Acc>
__device__ __forceinline__ void schwarz_rows(const S* tile, int lane, Acc r0, Acc r1, Acc r2, Acc& z0, Acc& z1,
                                             Acc& z2) {
    if constexpr (is_fact<S>::value) {
        schwarz_factored<B, S, Acc>(tile, lane, r0, r1, r2, z0, z1, z2);
        return;
    }
    Acc a0 = 0, a1 = 0, a2 = 0;
    #pragma unroll 4
    for (int c = 0; c < B; ++c) {
        const Acc x0 = shfl_acc(r0, c, B), x1 = shfl_acc(r1, c, B), x2 = shfl_acc(r2, c, B);
        const bool tr = c < lane;
        const S* P = tile + (tr ? sym_index(B, c, lane) : sym_index(B, lane, c)) * 9;
        const int s1 = tr ? 1 : 3, s2 = tr ? 3 : 1;  // element (a, k) at a*s2 + k*s1
        a0 = fma_acc(Store<S>::to_acc(P[0]), x0, a0);
        a0 = fma_acc(Store<S>::to_acc(P[s1]), x1, a0);
        a0 = fma_acc(Store<S>::to_acc(P[2 * s1]), x2, a0);
        a1 = fma_acc(Store<S>::to_acc(P[s2]), x0, a1);
        a1 = fma_acc(Store<S>::to_acc(P[s2 + s1]), x1, a1);
        a1 = fma_acc(Store<S>::to_acc(P[s2 + 2 * s1]), x2, a1);
        a2 = fma_acc(Store<S>::to_acc(P[2 * s2]), x0, a2);
        a2 = fma_acc(Store<S>::to_acc(P[2 * s2 + s1]), x1, a2);
        a2 = fma_acc(Store<S>::to_acc(P[2 * s2 + 2 * s1]), x2, a2);
    }
    z0 = a0; z1 = a1; z2 = a2;
}

// Sum `v` over the lanes of this bank that share `key` (lanes ascending, the
// order the oracle restates); *lead = lowest lane of its group.
template <int B, typename Acc>
__device__ __forceinline__ void group_sum(int key, Acc v0, Acc v1, Acc v2, int lane, Acc& s0, Acc& s1, Acc& s2,
                                          bool& lead) {
    s0 = 0; s1 = 0; s2 = 0;
    lead = key >= 0;
    #pragma unroll 4
    for (int j = 0; j < B; ++j) {
        const int kj = __shfl_sync(0xffffffffu, key, j, B);
        const Acc y0 = shfl_acc(v0, j, B), y1 = shfl_acc(v1, j, B), y2 = shfl_acc(v2, j, B);
        if (key >= 0 && kj == key) {
            s0 += y0; s1 += y1; s2 += y2;
            if (j < lane) lead = false;
        }
    }
}

}  // namespace sgmas
