"""Test infrastructure: a numpy restatement of the body patches
(stiff-gipc_b200/csrc/patch.cu) and of PCG with them, the checker of the
GPU's body-patch preconditioner.  It follows the reference's PCGSolver::pcg
(SG/linear_system/solver/pcg_solver.cu:171-304: x0 = 0, the true residual
every 10th iteration, convergence on ||b - A x|| / ||b||) with the
preconditioner the reference composes for hybrid scenes
(SG/linear_system/linear_system/global_linear_system.cu:509-522: MAS on the
FEM range), the bodies' 12x12 block-Jacobi widened to patches.  The patches
are this library's addition; the reference has none.

A patch is body b's 12 unknowns plus the FEM vertices coupled to it (at
most 64, the lowest ids; neighbouring patches overlap); its dense block is
factored in FP64 (Cholesky, a non-positive pivot replaced by 1), W = L^-1 is
rounded to FP32 (FP64 beside the FP64 MAS), and the apply adds W^T W r on
the patch's unknowns.
"""
from __future__ import annotations

import numpy as np

PATCH_MAX = 64


def patch_lists(rows, cols, n_bodies, fem_off, N):
    """FEM vertices of each body's patch (ascending)."""
    rows = np.asarray(rows); cols = np.asarray(cols)
    lo, hi = np.minimum(rows, cols), np.maximum(rows, cols)
    m = (lo < 4 * n_bodies) & (hi >= fem_off) & (hi < fem_off + N)
    return [np.unique(hi[m & (lo // 4 == b)] - fem_off)[:PATCH_MAX] for b in range(n_bodies)]


def _round(W, precision):
    if precision == "fp64":
        return W
    return W.astype(np.float32).astype(np.float64)  # FP32 beside the BF16 / FP32 MAS


class Patches:
    def __init__(self, A, rows, cols, n_bodies, fem_off, N, precision="fp64"):
        """A: the full scipy matrix (3 n DOF)."""
        self.precision = precision
        self.acc = np.float64 if precision == "fp64" else np.float32
        self.dofs, self.W = [], []
        for b, verts in enumerate(patch_lists(rows, cols, n_bodies, fem_off, N)):
            d = np.concatenate([12 * b + np.arange(12), (3 * (fem_off + verts)[:, None] + np.arange(3)).ravel()])
            M = A[d][:, d].toarray()
            L = np.tril(M).astype(np.float64)
            n = len(d)
            for k in range(n):  # right-looking Cholesky, non-positive pivot -> 1
                piv = L[k, k] if L[k, k] > 0 else 1.0
                L[k, k] = np.sqrt(piv)
                L[k + 1:, k] /= L[k, k]
                L[k + 1:, k + 1:] -= np.tril(np.outer(L[k + 1:, k], L[k + 1:, k]))
            import scipy.linalg as sl
            W = sl.solve_triangular(L, np.eye(n), lower=True)
            self.dofs.append(d)
            self.W.append(_round(W, precision))

    def apply(self, r):
        z = np.zeros_like(r)
        for d, W in zip(self.dofs, self.W):
            rl = r[d].astype(self.acc)
            y = (W.astype(self.acc) @ rl).astype(self.acc)
            z[d] += (W.T.astype(self.acc) @ y).astype(np.float64)
        return z


def pcg(A, b, mas_apply, patches, fem_off, rel_tol=1e-4, max_iter=5000):
    """PCG with the reference's stopping rule; z = MAS(r on the FEM range) +
    patches(r).  Returns (x, iterations, relative residual)."""
    def prec(r):
        z = patches.apply(r)
        z[3 * fem_off:] += mas_apply(r[3 * fem_off:])
        return z
    x = np.zeros_like(b)
    r = b.copy()
    z = prec(r)
    p = z.copy()
    rz = r @ z
    bb = np.linalg.norm(b)
    for k in range(1, max_iter + 1):
        Ap = A @ p
        al = rz / (p @ Ap)
        x += al * p
        r -= al * Ap
        if k % 10 == 0:
            r = b - A @ x
            if np.linalg.norm(r) <= rel_tol * bb:
                return x, k, np.linalg.norm(r) / bb
        z = prec(r)
        rzn = r @ z
        p = z + (rzn / rz) * p
        rz = rzn
    return x, max_iter, np.linalg.norm(b - A @ x) / bb
