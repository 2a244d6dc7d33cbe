// spmv_dev.cuh -- one SpMV work unit over the row-owned block CSR, shared by
// the per-iteration kernel (pcg.cu) and the persistent PCG kernel.
//   MODE 0: y = a A x + b y
//   MODE 1: p_new = z + beta p_old (fused), Ap = A p_new; returns p_new.Ap of
//           the rows this lane wrote (0 elsewhere)
//   MODE 2: r = rhs - A x
#pragma once
#include "ctx.hpp"

namespace sgmas {

// Work split: warps [0, n_long) take one long row each (all 32 lanes), the
// remaining warps take kRowGroups short rows (kRowLanes lanes each); row_list
// holds the long rows first, both parts in row order.
// LIVE = the vector is written by other CTAs earlier in the same launch (the
// persistent kernel): it is read with an explicit weak ld.global, never the
// read-only (.nc) path that const __restrict__ would allow; the grid
// barrier's fences between the phases make those loads current.
template <bool LIVE>
__device__ __forceinline__ double ldv(const double* p) {
    if (LIVE) {
        double v;
        asm volatile("ld.global.f64 %0, [%1];" : "=d"(v) : "l"(p));
        return v;
    }
    return *p;
}

// a lane's two blocks (v[q].x, v[q].y: row-major component q) times their
// vector entries x0, x1, added to the row sums with explicit fused
// multiply-adds in a fixed order, so every SpMV form gives the same bits
__device__ __forceinline__ void acc_pair(const double2 (&v)[9], const double (&x0)[3], const double (&x1)[3],
                                         double& a0, double& a1, double& a2) {
    double* acc[3] = {&a0, &a1, &a2};
    #pragma unroll
    for (int r = 0; r < 3; ++r) {  // the pair's six products left to right, then into the row sum
        double t = __dmul_rn(v[3 * r].x, x0[0]);
        t = __fma_rn(v[3 * r + 1].x, x0[1], t);
        t = __fma_rn(v[3 * r + 2].x, x0[2], t);
        t = __fma_rn(v[3 * r].y, x1[0], t);
        t = __fma_rn(v[3 * r + 1].y, x1[1], t);
        t = __fma_rn(v[3 * r + 2].y, x1[2], t);
        *acc[r] = __dadd_rn(*acc[r], t);
    }
}

// lanes per short row (a warp takes 32 / kRowLanes short rows at once)
constexpr int kRowLanes = 8;
constexpr int kRowGroups = 32 / kRowLanes;

// warp work units of a matrix: one per long row, one per kRowGroups short rows
__host__ __device__ __forceinline__ int spmv_units(int n_long, int nrows) {
    return n_long + (nrows - n_long + kRowGroups - 1) / kRowGroups;
}

// The block range of this lane's row in work unit gw: {row (-1: none), begin,
// end, 1 for a whole-warp (long) row}.  Fixed for a given matrix.
__device__ __forceinline__ int4 unit_desc(const BsrView& A, int gw, int lane) {
    int4 d = {-1, 0, 0, 0};
    if (gw < A.n_long) {
        d.x = A.row_list[gw];
        d.w = 1;
    } else {
        const int g = (gw - A.n_long) * kRowGroups + lane / kRowLanes;
        if (g < A.nrows - A.n_long) d.x = A.row_list[A.n_long + g];
    }
    if (d.x >= 0) {
        d.y = A.row_ptr[d.x];
        d.z = A.row_ptr[d.x + 1];
    }
    return d;
}

template <int MODE, bool LIVE = false>
__device__ __forceinline__ double spmv_unit_d(const BsrView& A, int4 desc, int lane, const double* __restrict__ xin,
                                              const double* __restrict__ pold, double* pnew, double* y,
                                              const double* __restrict__ rhs, double a, double b, double beta);

template <int MODE, bool LIVE = false>
__device__ __forceinline__ double spmv_unit(const BsrView& A, int gw, int lane, const double* __restrict__ xin,
                                            const double* __restrict__ pold, double* pnew, double* y,
                                            const double* __restrict__ rhs, double a, double b, double beta) {
    return spmv_unit_d<MODE, LIVE>(A, unit_desc(A, gw, lane), lane, xin, pold, pnew, y, rhs, a, b, beta);
}

// One work unit given its descriptor (unit_desc); desc.w is warp-uniform.
template <int MODE, bool LIVE>
__device__ __forceinline__ double spmv_unit_d(const BsrView& A, int4 desc, int lane, const double* __restrict__ xin,
                                              const double* __restrict__ pold, double* pnew, double* y,
                                              const double* __restrict__ rhs, double a, double b, double beta) {
    const int* __restrict__ bcols = A.cols;
    const double* __restrict__ bvals = A.vals;
    const long long cap = A.cap;
    const bool longw = desc.w != 0;
    const int row = desc.x, l = longw ? lane : (lane % kRowLanes), G = longw ? 32 : kRowLanes;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    double dot = 0.0;
    {
        const int beg = desc.y, end = desc.z;
        for (int p = beg + 2 * l; p < end; p += 2 * G) {
            const int2 cc = *reinterpret_cast<const int2*>(bcols + p);
            double2 v[9];
            #pragma unroll
            for (int q = 0; q < 9; ++q) v[q] = __ldg(reinterpret_cast<const double2*>(bvals + q * cap + p));
            double x0[3], x1[3];
            #pragma unroll
            for (int d = 0; d < 3; ++d) {
                if (MODE == 1) {
                    x0[d] = __fma_rn(beta, ldv<LIVE>(pold + 3 * (size_t)cc.x + d), ldv<LIVE>(xin + 3 * (size_t)cc.x + d));
                    x1[d] = __fma_rn(beta, ldv<LIVE>(pold + 3 * (size_t)cc.y + d), ldv<LIVE>(xin + 3 * (size_t)cc.y + d));
                } else {
                    x0[d] = ldv<LIVE>(xin + 3 * (size_t)cc.x + d);
                    x1[d] = ldv<LIVE>(xin + 3 * (size_t)cc.y + d);
                }
            }
            acc_pair(v, x0, x1, a0, a1, a2);
        }
        if (longw) {  // warp-uniform branch
            #pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o);
            }
        } else {
            #pragma unroll
            for (int o = kRowLanes / 2; o > 0; o >>= 1) {
                a0 += __shfl_xor_sync(0xffffffffu, a0, o, kRowLanes);
                a1 += __shfl_xor_sync(0xffffffffu, a1, o, kRowLanes);
                a2 += __shfl_xor_sync(0xffffffffu, a2, o, kRowLanes);
            }
        }
        if (l == 0 && row >= 0) {
            double* yr = y + 3 * (size_t)row;
            if (MODE == 0) {
                if (b != 0.0) { yr[0] = a * a0 + b * ldv<LIVE>(yr); yr[1] = a * a1 + b * ldv<LIVE>(yr + 1); yr[2] = a * a2 + b * ldv<LIVE>(yr + 2); }
                else { yr[0] = a * a0; yr[1] = a * a1; yr[2] = a * a2; }
            } else if (MODE == 1) {
                const double p0 = __fma_rn(beta, ldv<LIVE>(pold + 3 * (size_t)row), ldv<LIVE>(xin + 3 * (size_t)row));
                const double p1 = __fma_rn(beta, ldv<LIVE>(pold + 3 * (size_t)row + 1), ldv<LIVE>(xin + 3 * (size_t)row + 1));
                const double p2 = __fma_rn(beta, ldv<LIVE>(pold + 3 * (size_t)row + 2), ldv<LIVE>(xin + 3 * (size_t)row + 2));
                pnew[3 * (size_t)row] = p0; pnew[3 * (size_t)row + 1] = p1; pnew[3 * (size_t)row + 2] = p2;
                yr[0] = a0; yr[1] = a1; yr[2] = a2;
                dot = p0 * a0 + p1 * a1 + p2 * a2;
            } else {
                const double* br = rhs + 3 * (size_t)row;
                yr[0] = br[0] - a0; yr[1] = br[1] - a1; yr[2] = br[2] - a2;
            }
        }
    }
    return dot;
}

// ---- SpMV over a CTA's halo (the persistent loop) --------------------------
// A CTA owns a contiguous range of block rows (in partition order, balanced
// by stored blocks).  Once per SpMV it stages the vector entries of every
// column its rows touch (its halo, 3 doubles per vertex) in shared memory;
// the rows' column indices are stored local to that halo (lcols), so the
// gathers read shared memory.  desc.w = 1 for a whole-warp (long) row, plus
// twice the row's own halo index.
//   MODE 1: hv holds p_new = z + beta p_old; y = A p_new, pnew[row] = p_new;
//           returns p_new.Ap of the rows this lane wrote
//   MODE 2: hv holds x; y = rhs - A x
template <int MODE>
__device__ __forceinline__ double spmv_unit_h(const BsrView& A, int4 desc, int lane, const int* __restrict__ lcols,
                                              const double* hv, double* pnew, double* y,
                                              const double* __restrict__ rhs) {
    const double* __restrict__ bvals = A.vals;
    const long long cap = A.cap;
    const bool longw = (desc.w & 1) != 0;
    const int row = desc.x, l = longw ? lane : (lane % kRowLanes), G = longw ? 32 : kRowLanes;
    double a0 = 0.0, a1 = 0.0, a2 = 0.0;
    double dot = 0.0;
    for (int p = desc.y + 2 * l; p < desc.z; p += 2 * G) {
        const int2 cc = __ldg(reinterpret_cast<const int2*>(lcols + p));
        double2 v[9];
        #pragma unroll
        for (int q = 0; q < 9; ++q) v[q] = __ldg(reinterpret_cast<const double2*>(bvals + q * cap + p));
        const double* h0 = hv + 3 * cc.x;
        const double* h1 = hv + 3 * cc.y;
        const double xa[3] = {h0[0], h0[1], h0[2]}, xb[3] = {h1[0], h1[1], h1[2]};
        acc_pair(v, xa, xb, a0, a1, a2);
    }
    if (longw) {  // warp-uniform branch
        #pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o);
        }
    } else {
        #pragma unroll
        for (int o = kRowLanes / 2; o > 0; o >>= 1) {
            a0 += __shfl_xor_sync(0xffffffffu, a0, o, kRowLanes);
            a1 += __shfl_xor_sync(0xffffffffu, a1, o, kRowLanes);
            a2 += __shfl_xor_sync(0xffffffffu, a2, o, kRowLanes);
        }
    }
    if (l == 0 && row >= 0) {
        double* yr = y + 3 * (size_t)row;
        if (MODE == 1) {
            const double* hr = hv + 3 * (desc.w >> 1);
            const double p0 = hr[0], p1 = hr[1], p2 = hr[2];
            pnew[3 * (size_t)row] = p0; pnew[3 * (size_t)row + 1] = p1; pnew[3 * (size_t)row + 2] = p2;
            yr[0] = a0; yr[1] = a1; yr[2] = a2;
            dot = p0 * a0 + p1 * a1 + p2 * a2;
        } else {
            const double* br = rhs + 3 * (size_t)row;
            yr[0] = br[0] - a0; yr[1] = br[1] - a1; yr[2] = br[2] - a2;
        }
    }
    return dot;
}

}  // namespace sgmas
