// pcg.cu -- PCG solve on sm_100a (PCGSolver::pcg, SG/linear_system/solver/pcg_solver.cu:155-304).
//
// Design:
//  * The upper-triangular BCOO input (the reference layout) is expanded once
//    per solve into a row-owned block CSR holding both triangles, rows padded
//    to an even length, values structure-of-arrays (9 planes of doubles), so
//    the SpMV loads 16-byte vectors, needs no atomics and can fuse the search
//    direction update p = z + beta p and the p.Ap reduction.
//  * All PCG scalars live on the device.  Reductions are deterministic (fixed
//    tree per CTA, then the last CTA sums the CTA partials in order).
//  * The loop is one CUDA graph: prologue + a conditional WHILE node whose
//    body is ten iterations (the reference's convergence-check cadence,
//    pcg_solver.cu:240,260), so a solve is one graph launch and one 4-byte
//    read of the iteration count.
#include <stdio.h>

#include <algorithm>
#include <cmath>

#include "../../include/sgmas.h"
#include "ctx.hpp"
#include "pcg_state.cuh"
#include "spmv_dev.cuh"

using namespace sgmas;

namespace {

constexpr int kT = 256;

// ---------------------------------------------------------------------------
// BCOO (upper) -> row-owned block CSR
// ---------------------------------------------------------------------------
__global__ void k_bsr_count(int nb, int nrows, const int* __restrict__ rows, const int* __restrict__ cols, int* cnt,
                            int* cnt_lower, int* first, int* err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const int i = rows[k], j = cols[k];
    if (i < 0 || j < 0 || i >= nrows || j >= nrows || i > j) { set_error(err, kDevBadIndex); return; }
    atomicAdd(cnt + i, 1);
    if (i != j) {
        atomicAdd(cnt + j, 1);
        atomicAdd(cnt_lower + j, 1);
    }
    if (k == 0 || rows[k - 1] != i) first[i] = k;
}

// exclusive scan of even-rounded row counts (one CTA of 1024 threads: a
// warp-shuffle scan per chunk of 1024 rows, two CTA barriers per chunk)
__global__ void __launch_bounds__(1024) k_row_scan(int n, const int* __restrict__ cnt, int* row_ptr) {
    __shared__ int sh[64];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < n; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < n ? ((cnt[i] + 1) & ~1) : 0;
        int tot;
        const int pre = block_scan1024(v, sh, &tot);
        if (i < n) row_ptr[i] = carry + pre;
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) row_ptr[n] = carry;
}

__global__ void k_bsr_fill(int nb, int nrows, const int* __restrict__ rows, const int* __restrict__ cols,
                           const int* __restrict__ row_ptr, const int* __restrict__ cnt,
                           const int* __restrict__ cnt_lower, const int* __restrict__ first, int* fill, int* bcols,
                           uint32_t* src, int* tcols, uint32_t* tsrc, int* err) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const int i = rows[k], j = cols[k];
    if (i < 0 || j < 0 || i >= nrows || j >= nrows || i > j) return;  // flagged by k_bsr_count
    const int u = k - first[i];
    if (u < 0 || u >= cnt[i] - cnt_lower[i]) { set_error(err, kDevBadIndex); return; }  // input not sorted by row
    const int pu = row_ptr[i] + cnt_lower[i] + u;
    bcols[pu] = j;
    src[pu] = (uint32_t)k;
    if (i != j) {  // lower entries land in claim order in the scratch copy; sorted next
        const int pl = row_ptr[j] + atomicAdd(fill + j, 1);
        tcols[pl] = i;
        tsrc[pl] = (uint32_t)k | 0x80000000u;
    }
}

// one warp per row: each lower entry's rank among the row's lower entries
// (columns are distinct) places it in column order; then the even-length
// padding entry
__global__ void k_bsr_sort_lower(int nrows, const int* __restrict__ row_ptr, const int* __restrict__ cnt,
                                 const int* __restrict__ cnt_lower, const int* __restrict__ tcols,
                                 const uint32_t* __restrict__ tsrc, int* bcols, uint32_t* src) {
    const int i = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (i >= nrows) return;
    const int b = row_ptr[i], nl = cnt_lower[i];
    for (int e = lane; e < nl; e += 32) {
        const int key = tcols[b + e];
        int rank = 0;
        for (int f = 0; f < nl; ++f) rank += tcols[b + f] < key;
        bcols[b + rank] = key;
        src[b + rank] = tsrc[b + e];
    }
    if (lane == 0 && (cnt[i] & 1)) {
        bcols[b + cnt[i]] = i;
        src[b + cnt[i]] = 0xffffffffu;
    }
}

// Split rows into long (more than kLongRow entries: one warp each) and short
// (8 lanes each), both lists in row order; one CTA.
constexpr int kLongRow = 32;
__global__ void __launch_bounds__(1024) k_row_split(int n, const int* __restrict__ row_ptr, int* row_list,
                                                    int* n_long) {
    __shared__ int sh[64];
    __shared__ int carry, total_long;
    if (threadIdx.x == 0) { carry = 0; total_long = 0; }
    __syncthreads();
    // pass 1: count long rows
    int cnt = 0;
    for (int i = threadIdx.x; i < n; i += 1024) cnt += (row_ptr[i + 1] - row_ptr[i]) > kLongRow;
    if (cnt) atomicAdd(&total_long, cnt);
    __syncthreads();
    const int nl = total_long;
    for (int base = 0; base < n; base += 1024) {
        const int i = base + threadIdx.x;
        const int v = i < n ? ((row_ptr[i + 1] - row_ptr[i]) > kLongRow) : 0;
        int tot;
        const int pre = block_scan1024(v, sh, &tot);
        if (i < n) {
            const int before = carry + pre;  // long rows before i
            row_list[v ? before : nl + (i - before)] = i;
        }
        __syncthreads();
        if (threadIdx.x == 0) carry += tot;
        __syncthreads();
    }
    if (threadIdx.x == 0) *n_long = nl;
}

__global__ void k_bsr_values(long long cap, const int* __restrict__ row_ptr, int nrows, const uint32_t* __restrict__ src,
                             const double* __restrict__ vals, double* bvals) {
    const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= row_ptr[nrows]) return;
    const uint32_t s = src[p];
    double H[9];
    if (s == 0xffffffffu) {
        #pragma unroll
        for (int q = 0; q < 9; ++q) H[q] = 0.0;
    } else {
        const size_t k = s & 0x7fffffffu;
        const bool tr = s >> 31;
        #pragma unroll
        for (int a = 0; a < 3; ++a)
            #pragma unroll
            for (int c = 0; c < 3; ++c) H[3 * a + c] = tr ? vals[9 * k + c + 3 * a] : vals[9 * k + a + 3 * c];
    }
    #pragma unroll
    for (int q = 0; q < 9; ++q) bvals[q * cap + p] = H[q];
}

// 3x3 block-Jacobi (DiagPreconditioner, diag_preconditioner.cu:9-30): inverse of
// each diagonal block by cofactors
__global__ void k_diag_inverse(int nb, const int* __restrict__ rows, const int* __restrict__ cols,
                               const double* __restrict__ vals, double* dinv) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb || rows[k] != cols[k]) return;
    const double* H = vals + 9 * (size_t)k;  // column-major
    const double a = H[0], b = H[3], c = H[6], d = H[1], e = H[4], f = H[7], g = H[2], h = H[5], i = H[8];
    const double A = e * i - f * h, Bc = -(d * i - f * g), C = d * h - e * g;
    const double det = a * A + b * Bc + c * C;
    const double id = 1.0 / det;
    double* D = dinv + 9 * (size_t)rows[k];  // row-major inverse
    D[0] = A * id;  D[1] = -(b * i - c * h) * id; D[2] = (b * f - c * e) * id;
    D[3] = Bc * id; D[4] = (a * i - c * g) * id;  D[5] = -(a * f - c * d) * id;
    D[6] = C * id;  D[7] = -(a * h - b * g) * id; D[8] = (a * e - b * d) * id;
}

// 12x12 block-Jacobi for affine bodies (setup_abd_system_gradient_and_hessian.cu:603-645):
// one thread per body gathers its 4x4 grid of 3x3 blocks and inverts it
// (Gauss-Jordan with partial pivoting, FP64).
__global__ void k_abd_inverse(int bodies, int nb, const int* __restrict__ rows, const int* __restrict__ cols,
                              const double* __restrict__ vals, const int* __restrict__ first, const int* __restrict__ cnt,
                              const int* __restrict__ cnt_lower, double* out, int* err) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= bodies) return;
    double M[144], I[144];
    for (int t = 0; t < 144; ++t) { M[t] = 0.0; I[t] = (t % 13 == 0) ? 1.0 : 0.0; }
    for (int br = 0; br < 4; ++br) {
        const int i = 4 * q + br;
        const int nu = cnt[i] - cnt_lower[i];
        for (int u = 0; u < nu; ++u) {
            const int k = first[i] + u;
            if (k < 0 || k >= nb) { set_error(err, kDevBadIndex); return; }
            const int j = cols[k];
            if (j / 4 != q) continue;
            const double* H = vals + 9 * (size_t)k;
            const int bc = j % 4;
            for (int a = 0; a < 3; ++a)
                for (int c = 0; c < 3; ++c) {
                    M[(br * 3 + a) * 12 + bc * 3 + c] = H[a + 3 * c];
                    if (i != j) M[(bc * 3 + c) * 12 + br * 3 + a] = H[a + 3 * c];
                }
        }
    }
    for (int k = 0; k < 12; ++k) {
        int p = k;
        double best = fabs(M[k * 12 + k]);
        for (int r = k + 1; r < 12; ++r)
            if (fabs(M[r * 12 + k]) > best) { best = fabs(M[r * 12 + k]); p = r; }
        if (best == 0.0) { set_error(err, kDevBadIndex); return; }
        if (p != k)
            for (int c = 0; c < 12; ++c) {
                double t = M[k * 12 + c]; M[k * 12 + c] = M[p * 12 + c]; M[p * 12 + c] = t;
                t = I[k * 12 + c]; I[k * 12 + c] = I[p * 12 + c]; I[p * 12 + c] = t;
            }
        const double d = 1.0 / M[k * 12 + k];
        for (int c = 0; c < 12; ++c) { M[k * 12 + c] *= d; I[k * 12 + c] *= d; }
        for (int r = 0; r < 12; ++r) {
            if (r == k) continue;
            const double f = M[r * 12 + k];
            if (f == 0.0) continue;
            for (int c = 0; c < 12; ++c) { M[r * 12 + c] -= f * M[k * 12 + c]; I[r * 12 + c] -= f * I[k * 12 + c]; }
        }
    }
    for (int t = 0; t < 144; ++t) out[144 * (size_t)q + t] = I[t];
}

// ---------------------------------------------------------------------------
// SpMV over the row-owned block CSR: 8 lanes per block row, two blocks per
// lane per step (16-byte loads of each value plane).
//   MODE 0: y = a A x + b y
//   MODE 1: p_new = z + beta p_old (fused), Ap = A p_new, p.Ap -> alpha
//   MODE 2: r = rhs - A x
// ---------------------------------------------------------------------------
// SpMV work-unit descriptors (unit_desc for every unit and lane group),
// once per block CSR build: a warp then reads its next unit's rows with one
// independent load instead of the row_list -> row_ptr chain.
__global__ void k_unit_desc(int nrows, const int* __restrict__ row_ptr, const int* __restrict__ row_list,
                            const int* __restrict__ d_nlong, int4* udesc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int n_long = *d_nlong;
    if (i >= spmv_units(n_long, nrows) * kRowGroups) return;
    const int u = i / kRowGroups, g = i % kRowGroups;
    int4 d = make_int4(-1, 0, 0, 0);
    if (u < n_long) {
        d.x = row_list[u];
        d.w = 1;
    } else {
        const int k = (u - n_long) * kRowGroups + g;
        if (k < nrows - n_long) d.x = row_list[n_long + k];
    }
    if (d.x >= 0) {
        d.y = row_ptr[d.x];
        d.z = row_ptr[d.x + 1];
    }
    udesc[i] = d;
}

template <int MODE>
__global__ void __launch_bounds__(kT) k_bsr_spmv(BsrView A, const double* __restrict__ xin, const double* __restrict__ pold,
                                                 double* pnew, double* y, const double* __restrict__ rhs, double a,
                                                 double b, PcgState* st, double* partials, unsigned* ticket,
                                                 int loop = 0) {
    if (MODE != 0 && st->done) return;
    __shared__ double sh[32];
    const double beta = MODE == 1 ? st->beta : 0.0;
    const int lane = threadIdx.x & 31, units = spmv_units(A.n_long, A.nrows), stride = gridDim.x * (kT / 32);
    const int4 none = make_int4(-1, 0, 0, 0);
    int gw = blockIdx.x * (kT / 32) + (threadIdx.x >> 5);  // warp-uniform
    int4 d = gw < units ? __ldg(A.udesc + (size_t)gw * kRowGroups + lane / kRowLanes) : none;
    double dot = 0.0;
    while (gw < units) {
        const int gn = gw + stride;
        const int4 dn = gn < units ? __ldg(A.udesc + (size_t)gn * kRowGroups + lane / kRowLanes) : none;
        dot += spmv_unit_d<MODE>(A, d, lane, xin, pold, pnew, y, rhs, a, b, beta);
        d = dn;
        gw = gn;
    }
    if (MODE != 1) return;
    double total;
    if (grid_sum_last<kT>(block_sum<kT>(dot, sh), partials, ticket, sh, &total)) {
        st->pAp = total;
        // in a loop iteration (the start guess's x0.A x0 is judged by k_warm_residual): stop when
        // p.Ap <= 0 -- a finite value is a CG breakdown (r = 0 exactly is a solution), NaN is
        // reported as a non-finite residual
        if (loop && !(total > 0.0)) {
            const bool finite = total == total && st->rz == st->rz;
            st->breakdown = finite && st->rz != 0.0;
            st->converged = finite && st->rz == 0.0;
            st->iters = st->k;
            st->done = 1;
            st->alpha = 0.0;
        } else {
            st->alpha = st->rz / total;
        }
    }
}

// x += alpha p (the update of a residual-recompute iteration)
__global__ void k_update_x(int n, double* x, const double* __restrict__ p, const PcgState* st) {
    if (st->done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = x[i] + st->alpha * p[i];
}

// Block-Jacobi iteration tail: (MODE 1: x += alpha p, r -= alpha Ap), z = P^-1 r
// with 3x3 diagonal inverses (12x12 for body rows), r.z and r.r, state update.
template <int MODE>
__global__ void __launch_bounds__(kT) k_jacobi_iter(int nrows, int abd_rows, double* x, double* r,
                                                    const double* __restrict__ p, const double* __restrict__ Ap,
                                                    double* z, const double* __restrict__ dinv,
                                                    const double* __restrict__ abd_inv, int kind, PcgState* st,
                                                    double* partials, unsigned* ticket, int set_cond,
                                                    unsigned long long cond) {
    if (st->done) {
        if (set_cond && blockIdx.x == 0 && threadIdx.x == 0) cudaGraphSetConditional((cudaGraphConditionalHandle)cond, 0u);
        return;
    }
    __shared__ double sh[32];
    const int i = blockIdx.x * kT + threadIdx.x;
    double rz = 0.0, rr = 0.0;
    if (i < nrows) {
        double rv[3];
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            rv[d] = r[3 * (size_t)i + d];
            if (MODE == 1) {
                const double al = st->alpha;
                x[3 * (size_t)i + d] = x[3 * (size_t)i + d] + al * p[3 * (size_t)i + d];
                rv[d] = rv[d] - al * Ap[3 * (size_t)i + d];
                r[3 * (size_t)i + d] = rv[d];
            }
        }
        rr = rv[0] * rv[0] + rv[1] * rv[1] + rv[2] * rv[2];
        if (i >= abd_rows) {
            const double* D = dinv + 9 * (size_t)i;
            double zv[3];
            #pragma unroll
            for (int d = 0; d < 3; ++d) zv[d] = D[3 * d] * rv[0] + D[3 * d + 1] * rv[1] + D[3 * d + 2] * rv[2];
            #pragma unroll
            for (int d = 0; d < 3; ++d) z[3 * (size_t)i + d] = zv[d];
            rz = rv[0] * zv[0] + rv[1] * zv[1] + rv[2] * zv[2];
        }
    }
    // body rows: z from the 12x12 inverses once every thread of the body has
    // updated its r (the body's 4 rows are 4 consecutive threads of one warp)
    __syncwarp();
    if (i < abd_rows && (i & 3) == 0) {
        const double* M = abd_inv + 144 * (size_t)(i / 4);
        const double* rb = r + 3 * (size_t)i;
        for (int a2 = 0; a2 < 12; ++a2) {
            double s = 0.0;
            for (int c = 0; c < 12; ++c) s += M[a2 * 12 + c] * rb[c];
            z[3 * (size_t)i + a2] = s;
            rz += rb[a2] * s;
        }
    }
    const double brz = block_sum<kT>(rz, sh);
    const double brr = block_sum<kT>(rr, sh);
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = brz;
        partials[gridDim.x + blockIdx.x] = brr;
        __threadfence();
        am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return;
    __threadfence();
    double s1 = 0.0, s2 = 0.0;
    for (int t = threadIdx.x; t < (int)gridDim.x; t += kT) {
        s1 += ((volatile double*)partials)[t];
        s2 += ((volatile double*)partials)[gridDim.x + t];
    }
    s1 = block_sum<kT>(s1, sh);
    s2 = block_sum<kT>(s2, sh);
    if (threadIdx.x == 0) {
        *ticket = 0u;
        pcg_end_iteration(st, s1, s2, kind, set_cond, cond);
    }
}

__global__ void k_init_state(PcgState* st, int max_iter, double rel2, double abs2, int check_every, int prec_norm,
                             int warm) {
    PcgState s = {};
    s.max_iter = max_iter;
    s.rel2 = rel2;
    s.abs2 = abs2;
    s.check_every = check_every;
    s.use_prec_norm = prec_norm;
    s.k = 1;
    s.warm = warm;
    *st = s;
}

// Two grid sums with the last-CTA-done pattern (partials summed in CTA
// order); true in thread 0 of the last CTA with the totals in s1, s2.
__device__ __forceinline__ bool grid_sum2_last(double v1, double v2, double* partials, unsigned* ticket, double* sh,
                                               double& s1, double& s2) {
    const double b1 = block_sum<kT>(v1, sh);
    const double b2 = block_sum<kT>(v2, sh);
    __shared__ bool am_last;
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = b1;
        partials[gridDim.x + blockIdx.x] = b2;
        __threadfence();
        am_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!am_last) return false;
    __threadfence();
    double t1 = 0.0, t2 = 0.0;
    for (int t = threadIdx.x; t < (int)gridDim.x; t += kT) {
        t1 += ((volatile double*)partials)[t];
        t2 += ((volatile double*)partials)[gridDim.x + t];
    }
    s1 = block_sum<kT>(t1, sh);
    s2 = block_sum<kT>(t2, sh);
    if (threadIdx.x == 0) *ticket = 0u;
    return threadIdx.x == 0;
}

// Start guess (graph form).  (1) x0.b and b.b; then k_bsr_spmv<1> with
// beta = 0 gives Ap = A x0 and x0.A x0 (st->pAp); (2) alpha = x0.b / x0.A x0
// (0 unless positive), r = b - alpha Ap, x = alpha x0, r.r and the rejection
// test ||r|| > ||b||; (3) a rejected guess restarts from x = 0, r = b.
__global__ void __launch_bounds__(kT) k_warm_dots(int n, const double* __restrict__ x, const double* __restrict__ b,
                                                  PcgState* st, double* partials, unsigned* ticket) {
    __shared__ double sh[32];
    double xb = 0.0, bb = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const double bi = b[i];
        xb += x[i] * bi;
        bb += bi * bi;
    }
    double s1, s2;
    if (grid_sum2_last(xb, bb, partials, ticket, sh, s1, s2)) {
        st->w_xb = s1;
        st->w_bb = s2;
    }
}
__global__ void __launch_bounds__(kT) k_warm_residual(int n, double* x, double* r, const double* __restrict__ b,
                                                      const double* __restrict__ Ap, PcgState* st, double* partials,
                                                      unsigned* ticket) {
    __shared__ double sh[32];
    const double xax = st->pAp, xb = st->w_xb;
    const double alpha = (xax > 0.0 && xb > 0.0) ? xb / xax : 0.0;
    double rr = 0.0;
    for (int i = blockIdx.x * kT + threadIdx.x; i < n; i += gridDim.x * kT) {
        const double ri = b[i] - alpha * Ap[i];
        r[i] = ri;
        x[i] = alpha * x[i];
        rr += ri * ri;
    }
    double s1, s2;
    if (grid_sum2_last(rr, 0.0, partials, ticket, sh, s1, s2)) {
        st->w_alpha = alpha;
        st->w_rr = s1;
        st->w_reject = !(s1 <= st->w_bb) || alpha == 0.0;
        st->pAp = 0.0;
        st->alpha = 0.0;
    }
}
__global__ void k_warm_reject(int n, double* x, double* r, const double* __restrict__ b, const PcgState* st) {
    if (!st->w_reject) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        r[i] = b[i];
        x[i] = 0.0;
    }
}

// reference-faithful symmetric BCOO SpMV (Spmv::warp_reduce_sym_spmv,
// spmv.cu:8-133) for the standalone entry point: one thread per upper block,
// y_i += a H x_j and y_j += a H^T x_i with FP64 atomics.
__global__ void k_scale(int n, double b, double* y) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] = b != 0.0 ? b * y[i] : 0.0;
}
__global__ void k_bcoo_spmv(int nb, double a, const double* __restrict__ vals, const int* __restrict__ rows,
                            const int* __restrict__ cols, const double* __restrict__ x, double* y) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nb) return;
    const int i = rows[k], j = cols[k];
    const double* H = vals + 9 * (size_t)k;
    const double* xj = x + 3 * (size_t)j;
    const double* xi = x + 3 * (size_t)i;
    #pragma unroll
    for (int r = 0; r < 3; ++r)
        atomicAdd(y + 3 * (size_t)i + r, a * (H[r] * xj[0] + H[r + 3] * xj[1] + H[r + 6] * xj[2]));
    if (i != j) {
        #pragma unroll
        for (int r = 0; r < 3; ++r)
            atomicAdd(y + 3 * (size_t)j + r, a * (H[3 * r] * xi[0] + H[3 * r + 1] * xi[1] + H[3 * r + 2] * xi[2]));
    }
}

int ensure_vec(sgmas_context* c, int nrows) {
    if (nrows <= c->vec_cap) return 0;
    const size_t n = 3 * (size_t)nrows;
    if (ctx_alloc(c, &c->d_r, n) || ctx_alloc(c, &c->d_z, n) || ctx_alloc(c, &c->d_p0, n) ||
        ctx_alloc(c, &c->d_p1, n) || ctx_alloc(c, &c->d_Ap, n) || ctx_alloc(c, &c->d_diag_inv, 9 * (size_t)nrows))
        return SGMAS_ERR_CUDA;
    c->vec_cap = nrows;
    return 0;
}

int ensure_partials(sgmas_context* c, int n) {
    if (n <= c->partial_cap) return 0;
    if (ctx_alloc(c, &c->d_partials, 2 * (size_t)n)) return SGMAS_ERR_CUDA;
    c->partial_cap = n;
    return 0;
}

}  // namespace

void bsr_mark_fresh(sgmas_context* c, const sgmas_bcoo* A) {
    c->bsr_src[0] = A->d_values;
    c->bsr_src[1] = A->d_rows;
    c->bsr_src[2] = A->d_cols;
    c->bsr_src_nb = A->n_blocks;
    c->bsr_src_nrows = A->n_block_rows;
    c->bsr_fresh = true;
}

bool bsr_reuse(sgmas_context* c, const sgmas_bcoo* A) {
    const bool same = c->bsr_fresh && c->bsr_src[0] == A->d_values && c->bsr_src[1] == A->d_rows &&
                      c->bsr_src[2] == A->d_cols && c->bsr_src_nb == A->n_blocks &&
                      c->bsr_src_nrows == A->n_block_rows;
    c->bsr_fresh = false;
    return same;
}

int bsr_build(sgmas_context* c, const double* vals, const int* rows, const int* cols, int nb, int nrows) {
    BsrMatrix& B = c->bsr;
    cudaStream_t s = c->stream;
    c->bsr_fresh = false;
    if (nrows > B.rows_cap) {
        if (ctx_alloc(c, &B.row_ptr, (size_t)nrows + 1) || ctx_alloc(c, &B.cnt, nrows) ||
            ctx_alloc(c, &B.cnt_lower, nrows) || ctx_alloc(c, &B.fill, nrows) || ctx_alloc(c, &B.first, nrows) ||
            ctx_alloc(c, &B.row_list, nrows) || ctx_alloc(c, &B.d_nlong, 1) ||
            ctx_alloc(c, &B.udesc, (size_t)nrows * kRowGroups))
            return SGMAS_ERR_CUDA;
        B.rows_cap = nrows;
    }
    const long long need = 2LL * nb + nrows + 2;  // both triangles + one padding entry per row at most
    if (need > B.cap) {
        const long long cap = (need + 1) & ~1LL;
        if (ctx_alloc(c, &B.cols, cap) || ctx_alloc(c, &B.src, cap) || ctx_alloc(c, &B.vals, 9 * cap) ||
            ctx_alloc(c, &B.tcols, cap) || ctx_alloc(c, &B.tsrc, cap))
            return SGMAS_ERR_CUDA;
        B.cap = cap;
    }
    B.nrows = nrows;
    B.nblocks = nb;
    SG_CUDA(c, cudaMemsetAsync(B.cnt, 0, sizeof(int) * nrows, s));
    SG_CUDA(c, cudaMemsetAsync(B.cnt_lower, 0, sizeof(int) * nrows, s));
    SG_CUDA(c, cudaMemsetAsync(B.fill, 0, sizeof(int) * nrows, s));
    SG_CUDA(c, cudaMemsetAsync(B.first, 0, sizeof(int) * nrows, s));
    const int gb = (nb + kT - 1) / kT;
    if (nb > 0) k_bsr_count<<<gb, kT, 0, s>>>(nb, nrows, rows, cols, B.cnt, B.cnt_lower, B.first, c->d_err);
    k_row_scan<<<1, 1024, 0, s>>>(nrows, B.cnt, B.row_ptr);
    if (nb > 0)
        k_bsr_fill<<<gb, kT, 0, s>>>(nb, nrows, rows, cols, B.row_ptr, B.cnt, B.cnt_lower, B.first, B.fill, B.cols,
                                     B.src, B.tcols, B.tsrc, c->d_err);
    k_bsr_sort_lower<<<(nrows * 32 + kT - 1) / kT, kT, 0, s>>>(nrows, B.row_ptr, B.cnt, B.cnt_lower, B.tcols, B.tsrc,
                                                             B.cols, B.src);
    k_bsr_values<<<(int)((B.cap + kT - 1) / kT), kT, 0, s>>>(B.cap, B.row_ptr, nrows, B.src, vals, B.vals);
    k_row_split<<<1, 1024, 0, s>>>(nrows, B.row_ptr, B.row_list, B.d_nlong);
    k_unit_desc<<<(nrows * kRowGroups + kT - 1) / kT, kT, 0, s>>>(nrows, B.row_ptr, B.row_list, B.d_nlong, B.udesc);
    c->build_launches += 5 + (nb > 0 ? 2 : 0);
    SG_CUDA(c, cudaGetLastError());
    // the long-row count sizes the SpMV grid (one 4-byte read per build)
    SG_CUDA(c, cudaMemcpyAsync(&B.n_long, B.d_nlong, sizeof(int), cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    return 0;
}

static BsrView bsr_view(const BsrMatrix& B) {
    return BsrView{B.row_ptr, B.cols, B.vals, B.cap, B.row_list, B.nrows, B.n_long, B.udesc};
}
// one warp per work unit, but no more CTAs than stay resident: the warps loop
// over units (next descriptor in flight) and reduce once at the end
static int spmv_grid(sgmas_context* c, const BsrMatrix& B) {
    const int warps = spmv_units(B.n_long, B.nrows);
    const int need = (warps + kT / 32 - 1) / (kT / 32);
    if (!c->spmv_resident) {
        int sms = 0, occ = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, c->device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_bsr_spmv<1>, kT, 0);
        c->spmv_resident = std::max(1, sms * std::max(1, occ));
    }
    return std::max(1, std::min(need, c->spmv_resident));
}

int bsr_spmv_plain(sgmas_context* c, double a, const double* x, double b, double* y) {
    const BsrMatrix& B = c->bsr;
    k_bsr_spmv<0><<<spmv_grid(c, B), kT, 0, c->stream>>>(bsr_view(B), x, nullptr, nullptr, y, nullptr, a, b, nullptr,
                                                      nullptr, nullptr);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

int bcoo_spmv_ref(sgmas_context* c, double a, const double* vals, const int* rows, const int* cols, int nb,
                  int nrows, const double* x, double b, double* y) {
    const int n = 3 * nrows;
    k_scale<<<(n + kT - 1) / kT, kT, 0, c->stream>>>(n, b, y);
    if (nb > 0) k_bcoo_spmv<<<(nb + kT - 1) / kT, kT, 0, c->stream>>>(nb, a, vals, rows, cols, x, y);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

// Prepare the preconditioner data that depends on A (block-Jacobi inverses).
static int jacobi_setup(sgmas_context* c, const double* vals, const int* rows, const int* cols, int nb, int nrows,
                        int abd_bodies, bool diag = true) {
    cudaStream_t s = c->stream;
    if (diag) {
        SG_CUDA(c, cudaMemsetAsync(c->d_diag_inv, 0, sizeof(double) * 9 * nrows, s));
        if (nb > 0) k_diag_inverse<<<(nb + kT - 1) / kT, kT, 0, s>>>(nb, rows, cols, vals, c->d_diag_inv);
    }
    if (abd_bodies > 0) {
        if (abd_bodies > c->abd_cap) {
            if (ctx_alloc(c, &c->d_abd_inv, 144 * (size_t)abd_bodies)) return SGMAS_ERR_CUDA;
            c->abd_cap = abd_bodies;
        }
        k_abd_inverse<<<(abd_bodies + 63) / 64, 64, 0, s>>>(abd_bodies, nb, rows, cols, vals, c->bsr.first, c->bsr.cnt,
                                                            c->bsr.cnt_lower, c->d_abd_inv, c->d_err);
    }
    c->build_launches += (diag && nb > 0 ? 1 : 0) + (abd_bodies > 0 ? 1 : 0);
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

// Record the whole solve into `stream` (prologue) and `body` (one WHILE body
// of ten iterations).  Returns the number of kernels in each part.
static int record_prologue(sgmas_context* c, const double* b, double* x, const PcgRunCfg& cfg, int* nk) {
    cudaStream_t s = c->stream;
    const int nrows = c->bsr.nrows, n = 3 * nrows;
    if (!cfg.warm) {
        SG_CUDA(c, cudaMemsetAsync(x, 0, sizeof(double) * n, s));
        SG_CUDA(c, cudaMemcpyAsync(c->d_r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, s));
    }
    SG_CUDA(c, cudaMemsetAsync(c->d_p0, 0, sizeof(double) * n, s));
    const int max_iter = cfg.max_iter == 0 ? n : cfg.max_iter;
    k_init_state<<<1, 1, 0, s>>>(c->d_state, max_iter, cfg.rel_tol * cfg.rel_tol, cfg.abs_tol * cfg.abs_tol,
                                 cfg.check_every, cfg.use_prec_norm, cfg.warm);
    *nk = 1;
    if (cfg.warm) {
        const int gv = std::min((n + kT - 1) / kT, 4 * 148);
        k_warm_dots<<<gv, kT, 0, s>>>(n, x, b, c->d_state, c->d_partials, c->d_ticket);
        k_bsr_spmv<1><<<spmv_grid(c, c->bsr), kT, 0, s>>>(bsr_view(c->bsr), x, x, c->d_p1, c->d_Ap, nullptr, 1.0, 0.0,
                                                       c->d_state, c->d_partials, c->d_ticket);
        k_warm_residual<<<gv, kT, 0, s>>>(n, x, c->d_r, b, c->d_Ap, c->d_state, c->d_partials, c->d_ticket);
        k_warm_reject<<<gv, kT, 0, s>>>(n, x, c->d_r, b, c->d_state);
        *nk += 4;
    }
    if (cfg.precond == 1) {
        int rc = mas_launch_apply(c, c->d_r, c->d_z, 0, c->d_state, x, nullptr, nullptr, c->d_partials,
                                  c->d_ticket, 1, 0ull, nk, extra_rows_of(c, cfg));
        if (rc) return rc;
    } else {
        const int g = (nrows + kT - 1) / kT;
        k_jacobi_iter<0><<<g, kT, 0, s>>>(nrows, 4 * cfg.abd_bodies, x, c->d_r, nullptr, nullptr, c->d_z,
                                          c->d_diag_inv, c->d_abd_inv, 1, c->d_state, c->d_partials, c->d_ticket, 0,
                                          0ull);
        *nk += 1;
    }
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

static int record_body(sgmas_context* c, cudaStream_t s, const double* b, double* x, const PcgRunCfg& cfg,
                       unsigned long long cond, int* nk) {
    const int nrows = c->bsr.nrows, n = 3 * nrows;
    const BsrMatrix& B = c->bsr;
    const int gs = spmv_grid(c, B);
    const int gj = (nrows + kT - 1) / kT;
    cudaStream_t saved = c->stream;
    c->stream = s;
    int rc = 0;
    *nk = 0;
    for (int t = 0; t < 10 && rc == 0; ++t) {
        double* pold = (t % 2 == 0) ? c->d_p0 : c->d_p1;
        double* pnew = (t % 2 == 0) ? c->d_p1 : c->d_p0;
        const bool check = (t == 9);
        const unsigned long long cnd = check ? cond : 0ull;
        k_bsr_spmv<1><<<gs, kT, 0, s>>>(bsr_view(B), c->d_z, pold, pnew, c->d_Ap, nullptr, 1.0, 0.0, c->d_state,
                                        c->d_partials, c->d_ticket, 1);
        *nk += 1;
        if (check) {
            k_update_x<<<(n + kT - 1) / kT, kT, 0, s>>>(n, x, pnew, c->d_state);
            k_bsr_spmv<2><<<gs, kT, 0, s>>>(bsr_view(B), x, nullptr, nullptr, c->d_r, b, 1.0, 0.0, c->d_state, nullptr,
                                            nullptr);
            *nk += 2;
        }
        if (cfg.precond == 1) {
            rc = mas_launch_apply(c, c->d_r, c->d_z, check ? 0 : 1, c->d_state, x, pnew, c->d_Ap, c->d_partials,
                                  c->d_ticket, 2, cnd, nk, extra_rows_of(c, cfg));
        } else if (check) {
            k_jacobi_iter<0><<<gj, kT, 0, s>>>(nrows, 4 * cfg.abd_bodies, x, c->d_r, pnew, c->d_Ap, c->d_z,
                                               c->d_diag_inv, c->d_abd_inv, 2, c->d_state, c->d_partials,
                                               c->d_ticket, 1, cnd);
            *nk += 1;
        } else {
            k_jacobi_iter<1><<<gj, kT, 0, s>>>(nrows, 4 * cfg.abd_bodies, x, c->d_r, pnew, c->d_Ap, c->d_z,
                                               c->d_diag_inv, c->d_abd_inv, 2, c->d_state, c->d_partials,
                                               c->d_ticket, 0, 0ull);
            *nk += 1;
        }
    }
    c->stream = saved;
    if (rc) return rc;
    SG_CUDA(c, cudaGetLastError());
    return 0;
}

int pcg_run(sgmas_context* c, const double* b, double* x, const PcgRunCfg& cfg, float* solve_ms, int* launches) {
    const int nrows = c->bsr.nrows;
    if (ensure_vec(c, nrows)) return SGMAS_ERR_CUDA;
    const int gmax = nrows / 8 + 16;  // >= every grid of the loop (SpMV: at most one warp per row)
    if (ensure_partials(c, gmax)) return SGMAS_ERR_CUDA;
    if (!c->d_state && ctx_alloc(c, &c->d_state, 1)) return SGMAS_ERR_CUDA;
    if (!c->d_ticket) {
        if (ctx_alloc(c, &c->d_ticket, 1)) return SGMAS_ERR_CUDA;
        SG_CUDA(c, cudaMemset(c->d_ticket, 0, sizeof(unsigned)));
    }
    int rc = 0;
    // graph cache key: everything the recorded launches capture
    unsigned long long key[10] = {(unsigned long long)(uintptr_t)b,
                                 (unsigned long long)(uintptr_t)x,
                                 (unsigned long long)nrows | ((unsigned long long)c->bsr.cap << 24) ^
                                     ((unsigned long long)c->bsr.n_long << 44),
                                 (unsigned long long)cfg.precond | ((unsigned long long)c->precision << 4) |
                                     ((unsigned long long)cfg.warm << 6) |
                                     ((unsigned long long)cfg.abd_bodies << 8) |
                                     ((unsigned long long)cfg.fem_offset << 36),
                                 (unsigned long long)(uintptr_t)c->bsr.vals,
                                 (unsigned long long)(uintptr_t)c->d_inv ^ ((unsigned long long)c->cap_total << 1),
                                 (unsigned long long)(uintptr_t)c->d_r,
                                 (unsigned long long)cfg.max_iter ^ ((unsigned long long)cfg.check_every << 32) ^
                                     ((unsigned long long)cfg.use_prec_norm << 48) ^
                                     (unsigned long long)(cfg.rel_tol * 1e18) ^ ((unsigned long long)(cfg.abs_tol * 1e30) << 7),
                                 (unsigned long long)(uintptr_t)c->d_partials,
                                 (unsigned long long)(uintptr_t)c->d_ticket};
    bool same = c->graph_exec != nullptr;
    for (int i = 0; i < 10 && same; ++i) same = key[i] == c->graph_key[i];
    if (!same) {
        if (c->graph_exec) { cudaGraphExecDestroy(c->graph_exec); c->graph_exec = nullptr; }
        if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
        cudaGraph_t g;
        SG_CUDA(c, cudaGraphCreate(&g, 0));
        c->graph = g;
        if (!c->rec_stream) SG_CUDA(c, cudaStreamCreateWithFlags(&c->rec_stream, cudaStreamNonBlocking));
        cudaStream_t user = c->stream;
        c->stream = c->rec_stream;
        SG_CUDA(c, cudaStreamBeginCaptureToGraph(c->stream, g, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        int nk_pro = 0;
        rc = record_prologue(c, b, x, cfg, &nk_pro);
        cudaGraph_t g2 = nullptr;
        cudaError_t e = cudaStreamEndCapture(c->stream, &g2);
        c->stream = user;
        if (rc) return rc;
        if (e != cudaSuccess) return ctx_fail(c, SGMAS_ERR_CUDA, "capture prologue: %s", cudaGetErrorString(e));
        // the conditional WHILE node after the prologue's last node
        size_t nn = 0;
        SG_CUDA(c, cudaGraphGetNodes(g, nullptr, &nn));
        cudaGraphNode_t* nodes = new cudaGraphNode_t[nn];
        SG_CUDA(c, cudaGraphGetNodes(g, nodes, &nn));
        cudaGraphNode_t leaf = nullptr;
        for (size_t i = 0; i < nn; ++i) {
            size_t nd = 0;
            cudaGraphNodeGetDependentNodes(nodes[i], nullptr, &nd);
            if (nd == 0) leaf = nodes[i];
        }
        delete[] nodes;
        cudaGraphConditionalHandle h;
        SG_CUDA(c, cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
        cudaGraphNodeParams cp = {};
        cp.type = cudaGraphNodeTypeConditional;
        cp.conditional.handle = h;
        cp.conditional.type = cudaGraphCondTypeWhile;
        cp.conditional.size = 1;
        cudaGraphNode_t cnode;
        SG_CUDA(c, cudaGraphAddNode(&cnode, g, leaf ? &leaf : nullptr, leaf ? 1 : 0, &cp));
        cudaGraph_t body = cp.conditional.phGraph_out[0];
        cudaStream_t s2;
        SG_CUDA(c, cudaStreamCreateWithFlags(&s2, cudaStreamNonBlocking));
        SG_CUDA(c, cudaStreamBeginCaptureToGraph(s2, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
        int nk_body = 0;
        rc = record_body(c, s2, b, x, cfg, (unsigned long long)h, &nk_body);
        cudaGraph_t b2 = nullptr;
        e = cudaStreamEndCapture(s2, &b2);
        cudaStreamDestroy(s2);
        if (rc) return rc;
        if (e != cudaSuccess) return ctx_fail(c, SGMAS_ERR_CUDA, "capture body: %s", cudaGetErrorString(e));
        SG_CUDA(c, cudaGraphInstantiate(&c->graph_exec, g, 0));
        for (int i = 0; i < 10; ++i) c->graph_key[i] = key[i];
        c->graph_kernels_prologue = nk_pro;
        c->graph_kernels_body = nk_body;
    }
    if (!c->ev0) {
        SG_CUDA(c, cudaEventCreate(&c->ev0));
        SG_CUDA(c, cudaEventCreate(&c->ev1));
        SG_CUDA(c, cudaEventCreate(&c->ev2));
    }
    SG_CUDA(c, cudaEventRecord(c->ev0, c->stream));
    SG_CUDA(c, cudaGraphLaunch(c->graph_exec, c->stream));
    SG_CUDA(c, cudaEventRecord(c->ev1, c->stream));
    SG_CUDA(c, cudaEventSynchronize(c->ev1));
    if (solve_ms) SG_CUDA(c, cudaEventElapsedTime(solve_ms, c->ev0, c->ev1));
    PcgState h;
    SG_CUDA(c, cudaMemcpy(&h, c->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost));
    if (launches) {
        const int bodies = (h.iters + 9) / 10;
        *launches = c->graph_kernels_prologue + c->graph_kernels_body * (bodies < 1 ? 1 : bodies);
    }
    c->last_persistent = false;
    c->last_run = cfg;
    c->last_cfg = {cfg.precond, cfg.abd_bodies, 1};
    c->last_b = b;
    c->last_x = x;
    c->solved = true;
    return 0;
}

// Replay each kernel of one iteration `reps` times with events around each
// group (the solve's own graph gives no per-kernel times).  The replay
// overwrites x, r, z, p, Ap; the next solve re-initialises them.
// Persistent solves: the same solve again with clock stamps at every phase
// boundary of CTA 0; the phase times are averaged over iterations
// 1..min(iters, kStampIters) that are not residual-refresh iterations.
static int pcg_profile_persistent(sgmas_context* c, float* ms, int n_ms) {
    constexpr int kStampIters = 1000;
    int n_sm = 0;
    SG_CUDA(c, cudaDeviceGetAttribute(&n_sm, cudaDevAttrMultiProcessorCount, c->device));
    const size_t n_it = 8 * (size_t)(kStampIters + 2);
    const size_t n_st = n_it + 16 * (size_t)n_sm;
    if (c->d_stamps && c->stamps_cap < n_st) { cudaFree(c->d_stamps); c->d_stamps = nullptr; }
    c->stamps_cap = n_st;
    if (!c->d_stamps && ctx_alloc(c, &c->d_stamps, n_st)) return SGMAS_ERR_CUDA;
    SG_CUDA(c, cudaMemsetAsync(c->d_stamps, 0, n_st * sizeof(unsigned long long), c->stream));
    float loop_ms = 0.f;
    PcgRunCfg cfg = c->last_run;
    cfg.warm = 0;  // x now holds the last solution: profile the solve from x = 0
    int rc = pcg_run_persistent(c, c->last_b, c->last_x, cfg, &loop_ms, nullptr, c->d_stamps, kStampIters);
    if (rc) return rc < 0 ? rc : ctx_fail(c, SGMAS_ERR_STATE, "persistent solve no longer fits");
    unsigned long long* h = new unsigned long long[n_st];
    cudaError_t e = cudaMemcpy(h, c->d_stamps, n_st * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) { delete[] h; return ctx_fail(c, SGMAS_ERR_CUDA, "stamps: %s", cudaGetErrorString(e)); }
    PcgState st;
    SG_CUDA(c, cudaMemcpy(&st, c->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost));
    const double cyc = (double)(h[1] - h[0]);
    const double ms_per_cycle = cyc > 0 ? loop_ms / cyc : 0.0;
    double sum[4] = {0, 0, 0, 0};
    int n = 0;
    const int last = std::min(st.iters - 1, kStampIters);  // the converged iteration may stop early
    for (int k = 1; k <= last; ++k) {
        const unsigned long long* t = h + 8 * (size_t)(k + 1);
        if (k % 10 == 0 || t[5] == 0) continue;
        const bool split = t[3] != 0;  // levels >= 2 after their own barrier
        sum[0] += (double)(t[1] - t[0]);
        sum[1] += (double)((split ? t[3] : t[5]) - t[1]);
        sum[2] += split ? (double)(t[5] - t[3]) : 0.0;
        ++n;
    }
    // per barrier slot: mean and max over CTAs of the work before it, mean wait in it
    const double passes = (double)h[2];
    double slot_stats[6][3] = {};
    for (int sl = 0; sl < 6; ++sl) {
        const double occ = (sl == 1 || sl == 2) ? std::floor(passes / 10.0) : passes;
        double wsum = 0.0, wmax = 0.0, tsum = 0.0;
        for (int b = 0; b < n_sm; ++b) {
            const unsigned long long* acc = h + n_it + 16 * (size_t)b + 2 * sl;
            wsum += (double)acc[0];
            wmax = std::max(wmax, (double)acc[0]);
            tsum += (double)acc[1];
        }
        if (occ > 0) {
            slot_stats[sl][0] = wsum / n_sm / occ * ms_per_cycle;
            slot_stats[sl][1] = wmax / occ * ms_per_cycle;
            slot_stats[sl][2] = tsum / n_sm / occ * ms_per_cycle;
        }
    }
    delete[] h;
    for (int i = 0; i < n_ms; ++i) ms[i] = 0.f;
    for (int i = 0; i < 4 && i < n_ms; ++i) ms[i] = n ? (float)(sum[i] / n * ms_per_cycle) : 0.f;
    if (n_ms > 4) ms[4] = loop_ms;
    if (n_ms > 5) ms[5] = (float)n;
    for (int i = 6; i < n_ms && i < 24; ++i) ms[i] = (float)slot_stats[(i - 6) / 3][(i - 6) % 3];
    c->solved = false;
    return 0;
}

int pcg_profile(sgmas_context* c, int reps, float* ms, int n_ms) {
    if (!c->solved) return ctx_fail(c, SGMAS_ERR_STATE, "sgmas_pcg_profile needs a completed sgmas_pcg_solve");
    if (c->last_persistent) return pcg_profile_persistent(c, ms, n_ms);
    cudaStream_t s = c->stream;
    const BsrMatrix& B = c->bsr;
    const int nrows = B.nrows;
    if (ensure_partials(c, nrows / 8 + 16)) return SGMAS_ERR_CUDA;  // the persistent solve sizes them per CTA
    if (!c->d_ticket) {
        if (ctx_alloc(c, &c->d_ticket, 1)) return SGMAS_ERR_CUDA;
        SG_CUDA(c, cudaMemset(c->d_ticket, 0, sizeof(unsigned)));
    }
    PcgState h;
    SG_CUDA(c, cudaMemcpyAsync(&h, c->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost, s));
    SG_CUDA(c, cudaStreamSynchronize(s));
    h.done = 0;
    h.k = 1;
    h.max_iter = 1 << 30;
    if (!(h.rz == h.rz) || h.rz == 0.0) h.rz = 1.0;
    SG_CUDA(c, cudaMemcpyAsync(c->d_state, &h, sizeof(PcgState), cudaMemcpyHostToDevice, s));
    for (int i = 0; i < n_ms; ++i) ms[i] = 0.f;
    const int gs = spmv_grid(c, B), gj = (nrows + kT - 1) / kT;
    int rc = 0;
    for (int part = 0; part < 4 && part < n_ms && rc == 0; ++part) {
        if (c->last_cfg.precond == 0 && part >= 2) break;
        SG_CUDA(c, cudaEventRecord(c->ev0, s));
        for (int r = 0; r < reps && rc == 0; ++r) {
            if (part == 0) {
                k_bsr_spmv<1><<<gs, kT, 0, s>>>(bsr_view(B), c->d_z, c->d_p0, c->d_p1, c->d_Ap, nullptr, 1.0, 0.0,
                                                c->d_state, c->d_partials, c->d_ticket);
            } else if (c->last_cfg.precond == 0) {
                k_jacobi_iter<1><<<gj, kT, 0, s>>>(nrows, 4 * c->last_cfg.abd_bodies, c->last_x, c->d_r, c->d_p1,
                                                   c->d_Ap, c->d_z, c->d_diag_inv, c->d_abd_inv, 3, c->d_state,
                                                   c->d_partials, c->d_ticket, 0, 0ull);
            } else {
                c->apply_parts = 1 << (part - 1);
                rc = mas_launch_apply(c, c->d_r, c->d_z, part == 1 ? 1 : 0, c->d_state, c->last_x, c->d_p1, c->d_Ap,
                                      c->d_partials, c->d_ticket, 3, 0ull, nullptr, extra_rows_of(c, c->last_run));
                c->apply_parts = 7;
            }
        }
        SG_CUDA(c, cudaEventRecord(c->ev1, s));
        SG_CUDA(c, cudaEventSynchronize(c->ev1));
        float t = 0.f;
        SG_CUDA(c, cudaEventElapsedTime(&t, c->ev0, c->ev1));
        ms[part] = t / reps;
    }
    c->apply_parts = 7;
    c->solved = false;
    return rc;
}

// Public-facing solve pieces used by capi.cu
int pcg_prepare(sgmas_context* c, const sgmas_bcoo* A, const PcgRunCfg& cfg) {
    const int nrows = A->n_block_rows;
    if (ensure_vec(c, nrows)) return SGMAS_ERR_CUDA;
    int rc = bsr_reuse(c, A) ? 0 : bsr_build(c, A->d_values, A->d_rows, A->d_cols, A->n_blocks, nrows);
    if (rc) return rc;
    if (cfg.precond == 0) return jacobi_setup(c, A->d_values, A->d_rows, A->d_cols, A->n_blocks, nrows, cfg.abd_bodies);
    if (cfg.abd_bodies > 0) {  // MAS on the FEM range + 12x12 block-Jacobi on the bodies (or body patches)
        rc = jacobi_setup(c, A->d_values, A->d_rows, A->d_cols, A->n_blocks, nrows, cfg.abd_bodies, false);
        if (rc == 0 && cfg.patches) rc = patch_build(c, cfg.abd_bodies, cfg.fem_offset);
        return rc;
    }
    return 0;
}

ExtraRows extra_rows_of(const sgmas_context* c, const PcgRunCfg& cfg) {
    ExtraRows ex = {};
    ex.fem_off = cfg.precond == 1 ? cfg.fem_offset : 0;
    ex.abd_bodies = cfg.precond == 1 ? cfg.abd_bodies : 0;
    ex.nrows = c->bsr.nrows;
    ex.n_units = cfg.precond == 1 ? ex.abd_bodies + (ex.fem_off - 4 * ex.abd_bodies) + (ex.nrows - ex.fem_off - c->N) : 0;
    ex.abd_inv = c->d_abd_inv;
    return ex;
}

int pcg_read_state(sgmas_context* c, PcgState* h) {
    SG_CUDA(c, cudaMemcpy(h, c->d_state, sizeof(PcgState), cudaMemcpyDeviceToHost));
    return 0;
}
