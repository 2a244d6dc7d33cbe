// abd.cu -- the affine-body coupling that turns vertex-level Hessian blocks
// into the 3x3 triplets of the 12-DOF body rows
// (ABDSystem::_setup_abd_system_hessian,
// SG/abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu:419-601).
//
// A body vertex moves with its body's affine coordinates q (translation t,
// rows a1, a2, a3 of the affine map): x = J(xb) q with the 3x12 Jacobian
// J = [I | e1 xb^T | e2 xb^T | e3 xb^T] of its rest position xb
// (ABDJacobi::to_mat, SG/abd_system/details/abd_jacobi_matrix.inl:32-43).  Body b owns block rows
// 4b .. 4b + 3.  Blocks are 9 doubles in column-major order (the BCOO's
// layout); 12x12 body Hessians are 144 doubles, column-major.
//
// Kernels (one thread per input entry, each writing its own output slots):
//   k_abd_body_blocks  a body's 12x12 Hessian -> its 10 upper 3x3 blocks
//                      (write_abd_body_hessian / write_triplet_cv, :14-34, :127-136)
//   k_abd_pair_blocks  a merged body-body vertex-pair block H -> the 16
//                      blocks of J_i^T H J_j (write_barrier_hessian :84-124,
//                      ABDJacobi::JT_H_J abd_jacobi_matrix.inl:45-91); blocks
//                      below the diagonal are written as zero with swapped
//                      indices (write_triplet_cv2 :38-71)
//   k_abd_fem_blocks   a body-vertex / FEM-vertex block H -> the 4 blocks of
//                      J^T H in the body's rows and the FEM vertex's column
//                      (:505-560)
// Products keep the reference's per-element order: H(r,k) y(c);
// x(r) H(a,c); (x(r) y(c)) H(a,k); J^T H reduces to x(d) H(a,c).
#include "../../include/sgmas.h"
#include "ctx.hpp"

using namespace sgmas;

namespace {

constexpr int kAT = 256;

// element (r, c) of a column-major 3x3 block
__device__ __forceinline__ double& el(double* blk, int r, int c) { return blk[3 * c + r]; }
__device__ __forceinline__ double elc(const double* blk, int r, int c) { return blk[3 * c + r]; }

__global__ void k_abd_body_blocks(int n_bodies, const double* __restrict__ H12, double* vals, int* rows, int* cols) {
    const int b = blockIdx.x * blockDim.x + threadIdx.x;
    if (b >= n_bodies) return;
    const double* H = H12 + 144 * (size_t)b;
    int kk = 0;
    for (int ii = 0; ii < 4; ++ii)
        for (int jj = ii; jj < 4; ++jj, ++kk) {
            const size_t o = 10 * (size_t)b + kk;
            rows[o] = 4 * b + ii;
            cols[o] = 4 * b + jj;
            double* out = vals + 9 * o;
            for (int c = 0; c < 3; ++c)
                for (int r = 0; r < 3; ++r) out[3 * c + r] = H[12 * (3 * jj + c) + (3 * ii + r)];
        }
}

// block (bi, bj) of J(x)^T H J(y), element (r, c)
__device__ __forceinline__ double jthj(const double* H, const double x[3], const double y[3], int bi, int bj, int r,
                                       int c) {
    if (bi == 0 && bj == 0) return elc(H, r, c);
    if (bi == 0) return elc(H, r, bj - 1) * y[c];
    if (bj == 0) return x[r] * elc(H, bi - 1, c);
    return (x[r] * y[c]) * elc(H, bi - 1, bj - 1);
}

__global__ void k_abd_pair_blocks(int n, const double* __restrict__ in_vals, const int* __restrict__ in_rows,
                                  const int* __restrict__ in_cols, const double* __restrict__ xbar,
                                  const int* __restrict__ body_of, const int* __restrict__ fixed, double* vals,
                                  int* rows, int* cols) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    double H[9];
    for (int q = 0; q < 9; ++q) H[q] = in_vals[9 * (size_t)t + q];
    const int i = in_rows[t], j = in_cols[t];
    const int bi = body_of[i], bj = body_of[j];
    const bool zero = fixed[bi] != 0 || fixed[bj] != 0;
    const double x[3] = {xbar[3 * (size_t)i], xbar[3 * (size_t)i + 1], xbar[3 * (size_t)i + 2]};
    const double y[3] = {xbar[3 * (size_t)j], xbar[3 * (size_t)j + 1], xbar[3 * (size_t)j + 2]};
    for (int ii = 0; ii < 4; ++ii)
        for (int jj = 0; jj < 4; ++jj) {
            const size_t o = 16 * (size_t)t + 4 * ii + jj;
            const int row = 4 * bi + ii, col = 4 * bj + jj;
            double* out = vals + 9 * o;
            if (row <= col) {
                rows[o] = row;
                cols[o] = col;
                for (int c = 0; c < 3; ++c)
                    for (int r = 0; r < 3; ++r) el(out, r, c) = zero ? 0.0 : jthj(H, x, y, ii, jj, r, c);
            } else {
                rows[o] = col;
                cols[o] = row;
                for (int q = 0; q < 9; ++q) out[q] = 0.0;
            }
        }
}

__global__ void k_abd_fem_blocks(int n, const double* __restrict__ in_vals, const int* __restrict__ in_rows,
                                 const int* __restrict__ in_cols, const double* __restrict__ xbar,
                                 const int* __restrict__ body_of, const int* __restrict__ fixed,
                                 const int* __restrict__ fem_boundary, int fem_point_offset, int n_bodies,
                                 double* vals, int* rows, int* cols) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int i = in_rows[t], fem = in_cols[t] - fem_point_offset;
    const int b = body_of[i];
    const bool zero = fem_boundary[fem] != 0 || fixed[b] != 0;
    const double* H = in_vals + 9 * (size_t)t;
    const double x[3] = {xbar[3 * (size_t)i], xbar[3 * (size_t)i + 1], xbar[3 * (size_t)i + 2]};
    for (int k = 0; k < 4; ++k) {
        const size_t o = 4 * (size_t)t + k;
        rows[o] = 4 * b + k;
        cols[o] = 4 * n_bodies + fem;
        double* out = vals + 9 * o;
        for (int c = 0; c < 3; ++c)
            for (int r = 0; r < 3; ++r)  // rows 3k + r of J^T H
                el(out, r, c) = zero ? 0.0 : (k == 0 ? elc(H, r, c) : x[r] * elc(H, k - 1, c));
    }
}

}  // namespace

extern "C" {

int sgmas_abd_body_blocks(sgmas_context* c, const double* d_H12, int n_bodies, double* d_vals, int* d_rows,
                          int* d_cols) {
    if (!c || n_bodies < 0 || (n_bodies > 0 && (!d_H12 || !d_vals || !d_rows || !d_cols))) return SGMAS_ERR_ARG;
    if (n_bodies == 0) return SGMAS_OK;
    SG_CUDA(c, cudaSetDevice(c->device));
    k_abd_body_blocks<<<(n_bodies + kAT - 1) / kAT, kAT, 0, c->stream>>>(n_bodies, d_H12, d_vals, d_rows, d_cols);
    SG_CUDA(c, cudaGetLastError());
    return SGMAS_OK;
}

int sgmas_abd_pair_blocks(sgmas_context* c, const double* d_in_vals, const int* d_in_rows, const int* d_in_cols, int n,
                          const double* d_xbar, const int* d_body_of, const int* d_fixed, double* d_vals, int* d_rows,
                          int* d_cols) {
    if (!c || n < 0 ||
        (n > 0 && (!d_in_vals || !d_in_rows || !d_in_cols || !d_xbar || !d_body_of || !d_fixed || !d_vals ||
                   !d_rows || !d_cols)))
        return SGMAS_ERR_ARG;
    if (n == 0) return SGMAS_OK;
    SG_CUDA(c, cudaSetDevice(c->device));
    k_abd_pair_blocks<<<(n + kAT - 1) / kAT, kAT, 0, c->stream>>>(n, d_in_vals, d_in_rows, d_in_cols, d_xbar,
                                                                  d_body_of, d_fixed, d_vals, d_rows, d_cols);
    SG_CUDA(c, cudaGetLastError());
    return SGMAS_OK;
}

int sgmas_abd_fem_blocks(sgmas_context* c, const double* d_in_vals, const int* d_in_rows, const int* d_in_cols, int n,
                         const double* d_xbar, const int* d_body_of, const int* d_fixed, const int* d_fem_boundary,
                         int fem_point_offset, int n_bodies, double* d_vals, int* d_rows, int* d_cols) {
    if (!c || n < 0 || n_bodies < 0 || fem_point_offset < 0 ||
        (n > 0 && (!d_in_vals || !d_in_rows || !d_in_cols || !d_xbar || !d_body_of || !d_fixed || !d_fem_boundary ||
                   !d_vals || !d_rows || !d_cols)))
        return SGMAS_ERR_ARG;
    if (n == 0) return SGMAS_OK;
    SG_CUDA(c, cudaSetDevice(c->device));
    k_abd_fem_blocks<<<(n + kAT - 1) / kAT, kAT, 0, c->stream>>>(n, d_in_vals, d_in_rows, d_in_cols, d_xbar, d_body_of,
                                                                 d_fixed, d_fem_boundary, fem_point_offset, n_bodies,
                                                                 d_vals, d_rows, d_cols);
    SG_CUDA(c, cudaGetLastError());
    return SGMAS_OK;
}

}  // extern "C"
