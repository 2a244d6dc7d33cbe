// extra_dev.cuh -- the rows of a MAS solve that the MAS does not cover
// (global_linear_system.cu:509-522: the global preconditioner is an identity
// copy, then the ABD 12x12 block-Jacobi on the body rows
// (setup_abd_system_gradient_and_hessian.cu:603-645), then the MAS on the
// FEM sub-range).  Shared by the collect kernel of the graph form and the
// persistent kernel.
#pragma once
#include "ctx.hpp"

namespace sgmas {

// Unit u of ex: mode 1 first applies x += alpha p, r -= alpha Ap to its rows;
// then z = P^-1 r for a body (its 12x12 inverse) or z = r for any other row;
// adds r.z and r.r of its rows.  (No array is indexed at run time, and the
// 12x12 product keeps one row in flight, so the caller's registers stay free.)
__device__ __forceinline__ void extra_unit(int u, const ExtraRows& ex, int N, int mode, double alpha, double* x,
                                           double* r, const double* p, const double* Ap, double* z, double& rz,
                                           double& rr) {
    const int nb = ex.abd_bodies;
    const bool body = u < nb;
    const int j = u - nb, gap = ex.fem_off - 4 * nb;
    const size_t o = body ? 12 * (size_t)u : 3 * (size_t)(j < gap ? 4 * nb + j : ex.fem_off + N + (j - gap));
    const int len = body ? 12 : 3;
    double rv[12];
    #pragma unroll
    for (int d = 0; d < 12; ++d) {
        rv[d] = 0.0;
        if (d < len) {
            double rd = r[o + d];
            if (mode == 1) {
                const double xd = x[o + d], pd = p[o + d], qd = Ap[o + d];
                rd = rd - alpha * qd;
                x[o + d] = xd + alpha * pd;
                r[o + d] = rd;
            }
            rv[d] = rd;
            rr += rd * rd;
        }
    }
    if (!body) {
        #pragma unroll
        for (int d = 0; d < 3; ++d) {
            z[o + d] = rv[d];
            rz += rv[d] * rv[d];
        }
        return;
    }
    const double* M = ex.abd_inv + 144 * (size_t)u;
    #pragma unroll 1
    for (int a = 0; a < 12; ++a) {
        double s = 0.0, ra = 0.0;
        #pragma unroll
        for (int c = 0; c < 12; ++c) {
            s += M[a * 12 + c] * rv[c];
            if (c == a) ra = rv[c];
        }
        z[o + a] = s;
        rz += ra * s;
    }
}

}  // namespace sgmas
