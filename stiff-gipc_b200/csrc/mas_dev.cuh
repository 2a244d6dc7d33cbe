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

// ---- bank value exchange ---------------------------------------------------
// A bank's per-lane 3-vectors are exchanged through shared memory: each warp
// owns kXchPerWarp values (16-byte aligned), one slot of 3 B values per bank
// it works on (32 / B banks).  A lane stores its three values; reading four
// columns (12 values) then takes three (FP32) or six (FP64) 16-byte loads
// where register shuffles would take twelve.
constexpr int kXchPerWarp = 96;

// this thread's bank slot inside its warp's exchange area
template <int B, typename Acc>
__device__ __forceinline__ Acc* bank_slot(Acc* xch_block) {
    return xch_block + (threadIdx.x >> 5) * kXchPerWarp + ((threadIdx.x & 31) / B) * (3 * B);
}

template <typename Acc>
__device__ __forceinline__ void xch_put(Acc* xb, int lane, Acc a, Acc b, Acc c) {
    __syncwarp();  // earlier readers of the slot are done
    xb[3 * lane] = a;
    xb[3 * lane + 1] = b;
    xb[3 * lane + 2] = c;
    __syncwarp();
}

__device__ __forceinline__ void xch_get4(const float* xb, int c0, float (&v)[12]) {
    const float4* q = reinterpret_cast<const float4*>(xb + 3 * c0);
    const float4 a = q[0], b = q[1], c = q[2];
    v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    v[4] = b.x; v[5] = b.y; v[6] = b.z; v[7] = b.w;
    v[8] = c.x; v[9] = c.y; v[10] = c.z; v[11] = c.w;
}
__device__ __forceinline__ void xch_get4(const double* xb, int c0, double (&v)[12]) {
    const double2* q = reinterpret_cast<const double2*>(xb + 3 * c0);
    #pragma unroll
    for (int i = 0; i < 6; ++i) {
        const double2 t = q[i];
        v[2 * i] = t.x;
        v[2 * i + 1] = t.y;
    }
}

// Factored tile (Fact<T>): slot sym_index(J, I), J <= I, holds the 3x3
// block (I, J) of W = L^-1, column-major.  z = W^T (W r): pass 1 y_I =
// sum_{J <= I} W_IJ r_J, pass 2 z_I = sum_{J >= I} W_JI^T y_J, each component
// an fma chain over J ascending.  The triangles are balanced over the bank's
// lanes by splitting the long sums at M = B / 2: in pass 1 a row I >= M is
// (its columns < M) + (its columns >= M), in pass 2 a row I < M is (its
// columns < M) + (its columns >= M), each part a chain of its own, the two
// added at the end (the order the oracle restates).  Lane l < M takes row l
// and then the upper part of row B-1-l in pass 1, its own upper part in
// pass 2; lane l >= M the reverse; every lane runs M + 1 block steps per pass
// instead of up to B.  xb holds r on entry and y on return.
template <typename S, typename Acc>
__device__ __forceinline__ void fact_step(const S* P, bool tr, Acc x0, Acc x1, Acc x2, Acc& a0, Acc& a1, Acc& a2) {
    // tr = 0: a += W_block x (element (d, k) at d + 3 k); tr = 1: a += W_block^T x
    const int s1 = tr ? 1 : 3, s2 = tr ? 3 : 1;
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

template <int B, typename S, typename Acc>
__device__ __forceinline__ void schwarz_factored(const S* tile, int lane, Acc* xb, Acc& z0, Acc& z1, Acc& z2) {
    constexpr int M = B / 2;
    const bool lo = lane < M;
    // pass 1: a = the lane's first part, b = its second part (lanes < M only)
    Acc a0 = 0, a1 = 0, a2 = 0, b0 = 0, b1 = 0, b2 = 0;
    #pragma unroll 3
    for (int t = 0; t <= M; ++t) {
        const bool second = lo && t > lane;
        const int row = second ? B - 1 - lane : lane;
        const int c = lo ? (second ? M + t - lane - 1 : t) : t;
        if (lo || t < M) {
            const Acc x0 = xb[3 * c], x1 = xb[3 * c + 1], x2 = xb[3 * c + 2];
            const S* P = tile + sym_index(B, c, row) * 9;  // block (row, c), c <= row
            Acc c0 = second ? b0 : a0, c1 = second ? b1 : a1, c2 = second ? b2 : a2;
            fact_step<S, Acc>(P, false, x0, x1, x2, c0, c1, c2);
            if (second) { b0 = c0; b1 = c1; b2 = c2; } else { a0 = c0; a1 = c1; a2 = c2; }
        }
    }
    {  // rows >= M: own lower part + the upper part summed by lane B-1-lane
        const Acc h0 = shfl_acc(b0, B - 1 - lane, B), h1 = shfl_acc(b1, B - 1 - lane, B),
                  h2 = shfl_acc(b2, B - 1 - lane, B);
        if (!lo) { a0 = a0 + h0; a1 = a1 + h1; a2 = a2 + h2; }
    }
    xch_put(xb, lane, a0, a1, a2);
    // pass 2: lane < M: own row's columns >= M; lane >= M: own row (all columns >= lane),
    // then the columns < M of row B-1-lane
    a0 = 0; a1 = 0; a2 = 0; b0 = 0; b1 = 0; b2 = 0;
    #pragma unroll 3
    for (int t = 0; t <= M; ++t) {
        const bool second = !lo && t >= B - lane;
        const int row = second ? B - 1 - lane : lane;
        const int c = lo ? M + t : (second ? row + t - (B - lane) : lane + t);
        if (!lo || t < M) {
            const Acc w0 = xb[3 * c], w1 = xb[3 * c + 1], w2 = xb[3 * c + 2];
            const S* P = tile + sym_index(B, row, c) * 9;  // block (c, row), used transposed
            Acc c0 = second ? b0 : a0, c1 = second ? b1 : a1, c2 = second ? b2 : a2;
            fact_step<S, Acc>(P, true, w0, w1, w2, c0, c1, c2);
            if (second) { b0 = c0; b1 = c1; b2 = c2; } else { a0 = c0; a1 = c1; a2 = c2; }
        }
    }
    {  // rows < M: the lower part summed by lane B-1-lane + own upper part
        const Acc l0 = shfl_acc(b0, B - 1 - lane, B), l1 = shfl_acc(b1, B - 1 - lane, B),
                  l2 = shfl_acc(b2, B - 1 - lane, B);
        if (lo) { a0 = l0 + a0; a1 = l1 + a1; a2 = l2 + a2; }
    }
    z0 = a0; z1 = a1; z2 = a2;
}

// z_lane = sum_c P(lane, c) r_c over one bank (xb holds r, put there by
// xch_put); columns ascending, each 3x3 row an fma chain (the order the
// oracle restates).  Factored tiles take schwarz_factored (which leaves W r
// in xb).  Called by whole warps.
template <int B, typename S, typename Acc>
__device__ __forceinline__ void schwarz_rows(const S* tile, int lane, Acc* xb, Acc& z0, Acc& z1, Acc& z2) {
    if constexpr (is_fact<S>::value) {
        schwarz_factored<B, S, Acc>(tile, lane, xb, z0, z1, z2);
    } else {
        Acc a0 = 0, a1 = 0, a2 = 0;
        #pragma unroll 2
        for (int c0 = 0; c0 < B; c0 += 4) {
            Acc v[12];
            xch_get4(xb, c0, v);
            #pragma unroll
            for (int j = 0; j < 4; ++j) {
                const int c = c0 + j;
                const Acc x0 = v[3 * j], x1 = v[3 * j + 1], x2 = v[3 * j + 2];
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
        }
        z0 = a0; z1 = a1; z2 = a2;
    }
}

// Sum over the lanes of this bank whose bit is set in msk (a level-0
// component), lanes ascending; xb holds the bank's values.
template <int B, typename Acc>
__device__ __forceinline__ void mask_sum(unsigned msk, const Acc* xb, Acc& s0, Acc& s1, Acc& s2) {
    s0 = 0; s1 = 0; s2 = 0;
    #pragma unroll 2
    for (int c0 = 0; c0 < B; c0 += 4) {
        Acc v[12];
        xch_get4(xb, c0, v);
        #pragma unroll
        for (int j = 0; j < 4; ++j)
            if (msk & (1u << (c0 + j))) { s0 += v[3 * j]; s1 += v[3 * j + 1]; s2 += v[3 * j + 2]; }
    }
}

// Sum the bank's values (xb) over the lanes that share `key` (lanes
// ascending, the order the oracle restates); *lead = lowest lane of its
// group.  Called by whole warps.
template <int B, typename Acc>
__device__ __forceinline__ void group_sum(int key, const Acc* xb, int lane, Acc& s0, Acc& s1, Acc& s2, bool& lead) {
    s0 = 0; s1 = 0; s2 = 0;
    lead = key >= 0;
    #pragma unroll 2
    for (int c0 = 0; c0 < B; c0 += 4) {
        Acc v[12];
        xch_get4(xb, c0, v);
        #pragma unroll
        for (int j = 0; j < 4; ++j) {
            const int kj = __shfl_sync(0xffffffffu, key, c0 + j, B);
            if (key >= 0 && kj == key) {
                s0 += v[3 * j]; s1 += v[3 * j + 1]; s2 += v[3 * j + 2];
                if (c0 + j < lane) lead = false;
            }
        }
    }
}

}  // namespace sgmas
