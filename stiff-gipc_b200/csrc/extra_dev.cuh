// extra_dev.cuh -- the rows of a MAS solve that the MAS does not cover
// (global_linear_system.cu:509-522: the global preconditioner is an identity
// copy, then the ABD 12x12 block-Jacobi on the body rows
// (setup_abd_system_gradient_and_hessian.cu:603-645), then the MAS on the
// FEM sub-range).  Shared by the collect kernel of the graph form and the
// persistent kernel.
#pragma once
#include "ctx.hpp"

namespace sgmas {

// Rows outside the MAS range, shared by the warps wid = 0 .. nw-1 of a
// grid (called by whole warps).  Mode 1 first applies x += alpha p,
// r -= alpha Ap to each row.  Bodies: 16 lanes per body, lane k < 12 owns
// row k of the body and forms z_k = sum_c P^-1(k, c) r_c with the body's r
// from shuffles; other rows: one lane each, z = r.  Adds r.z and r.r.
__device__ __forceinline__ void extra_rows_work(const ExtraRows& ex, int N, int mode, double alpha, double* x,
                                                double* r, const double* p, const double* Ap, double* z, int wid,
                                                int nw, int lane, double& rz, double& rr) {
    const int nb = ex.abd_bodies;
    for (int g0 = 2 * wid; g0 < (ex.patch ? 0 : nb); g0 += 2 * nw) {  // warp-uniform trip count
        const int g = g0 + lane / 16, k = lane % 16;
        const bool valid = g < nb && k < 12;
        const size_t o = 12 * (size_t)g + k;
        double rv = 0.0;
        const double* M = ex.abd_inv + 144 * (size_t)(valid ? g : 0) + 12 * (valid ? k : 0);  // row k of P^-1
        if (valid) {
            rv = r[o];
            if (mode == 1) {
                const double xd = x[o], pd = p[o], qd = Ap[o];
                rv = rv - alpha * qd;
                x[o] = xd + alpha * pd;
                r[o] = rv;
            }
        }
        double s = 0.0;
        #pragma unroll 4  // the row is streamed, not held: the callers' registers stay free
        for (int c = 0; c < 12; ++c) {
            const double rc = __shfl_sync(0xffffffffu, rv, c, 16);
            if (valid) s += M[c] * rc;
        }
        if (valid) {
            z[o] = s;
            rz += rv * s;
            rr += rv * rv;
        }
    }
    const int gap = ex.fem_off - 4 * nb;
    const int n_ident = ex.n_units - nb;  // rows that are neither body nor MAS rows
    for (int j = wid * 32 + lane; j < n_ident; j += nw * 32) {
        const size_t o = 3 * (size_t)(j < gap ? 4 * nb + j : ex.fem_off + N + (j - gap));
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            double rd = r[o + d];
            if (mode == 1) {
                const double xd = x[o + d], pd = p[o + d], qd = Ap[o + d];
                rd = rd - alpha * qd;
                x[o + d] = xd + alpha * pd;
                r[o + d] = rd;
            }
            z[o + d] = rd;
            rz += rd * rd;
            rr += rd * rd;
        }
    }
}

}  // namespace sgmas
