// patch_dev.cuh -- body patches (patch.cu): sizes, packed layouts and the
// apply, shared by the build and the persistent PCG kernel.
#pragma once
#include "common.cuh"

namespace sgmas {

constexpr int kPatchMax = 64;  // FEM vertices per body patch (a patch has 12 + 3 k unknowns)

__host__ __device__ constexpr size_t patch_packed(int k) {
    return (size_t)(12 + 3 * k) * (13 + 3 * k) / 2;
}
// (i, j), j <= i, of a packed lower triangle stored by rows
__host__ __device__ __forceinline__ int packed_lower(int i, int j) { return i * (i + 1) / 2 + j; }
// (i, j), j <= i, of an n x n packed lower triangle stored by columns
__host__ __device__ __forceinline__ int packed_col(int n, int i, int j) { return j * n - j * (j - 1) / 2 + (i - j); }

struct PatchView {
    int bodies;         // 0: no patches
    const int* list;    // [bodies][kPatchMax] FEM vertices of each patch (ascending)
    const int2* info;   // [bodies] {k, truncated}
    const void* wcol;   // [bodies][patch_packed(kPatchMax)] W = L^-1 packed by columns (storage precision)
    const void* wrow;   // the same packed by rows
    double* zs;         // [bodies][3 kPatchMax] each patch's part of z on its FEM rows
    const int* poff;    // [nrows + 1] per-row range of pent
    const int* pent;    // entries e = b kPatchMax + i of the patches covering each row, ascending
};

// the patches' part of z at vector index 3 row + d (their entries in body order)
__device__ __forceinline__ double patch_z(const PatchView& P, int row, int d) {
    double s = 0.0;
    for (int a = P.poff[row]; a < P.poff[row + 1]; ++a) s += P.zs[3 * (size_t)P.pent[a] + d];
    return s;
}

// The dof of local unknown i of body b's patch (global vector index).
__device__ __forceinline__ size_t patch_dof(const PatchView& P, int b, int fem_off, int i) {
    return i < 12 ? 12 * (size_t)b + i : 3 * (size_t)(fem_off + P.list[(size_t)b * kPatchMax + (i - 12) / 3]) + (i - 12) % 3;
}

// z_patch = W^T (W r_patch) for body b, by the whole CTA (rl, yl: shared
// scratch of 12 + 3 kPatchMax entries each).  y_i = sum_{j <= i} W_ij r_j
// with a warp per row (row i of the row-major copy, contiguous), z_j =
// sum_{i >= j} W_ij y_i with a warp per column (column j of the
// column-major copy, contiguous): lane l sums the terms l, l + 32, ... as an
// fma chain in Acc, then an xor-shuffle tree (every lane gets the same
// bits).  The body's rows get z in z_body (no other patch covers them), its
// FEM vertices' part goes to the patch's slice of P.zs (summed per row by
// patch_z); adds this thread's part of r.z over the patch and of r.r over
// the body rows.
template <typename S, typename Acc>
__device__ __forceinline__ void patch_apply_cta(const PatchView& P, int b, int fem_off, const double* r, double* z_body,
                                                Acc* rl, Acc* yl, double& rz, double& rr) {
    const int k = P.info[b].x, n = 12 + 3 * k;
    const S* wc = (const S*)P.wcol + (size_t)b * patch_packed(kPatchMax);
    const S* wr = (const S*)P.wrow + (size_t)b * patch_packed(kPatchMax);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x; i < n; i += blockDim.x) rl[i] = (Acc)r[patch_dof(P, b, fem_off, i)];
    __syncthreads();
    for (int i = warp; i < n; i += nw) {
        const S* row = wr + packed_lower(i, 0);
        Acc s = 0;
        for (int j = lane; j <= i; j += 32) s = fma_acc(Store<S>::to_acc(row[j]), rl[j], s);
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) yl[i] = s;
    }
    __syncthreads();
    for (int j = warp; j < n; j += nw) {
        const S* col = wc + packed_col(n, j, j);  // W[j..n-1][j]
        Acc s = 0;
        for (int i = j + lane; i < n; i += 32) s = fma_acc(Store<S>::to_acc(col[i - j]), yl[i], s);
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) {
            const size_t d = patch_dof(P, b, fem_off, j);
            const double zv = (double)s, rv = r[d];
            if (j < 12) {
                z_body[d] = zv;
                rr += rv * rv;
            } else {
                P.zs[3 * kPatchMax * (size_t)b + (j - 12)] = zv;
            }
            rz += rv * zv;
        }
    }
    __syncthreads();  // rl / yl are free again
}

}  // namespace sgmas
