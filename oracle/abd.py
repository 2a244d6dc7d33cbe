"""CPU oracle of the affine-body coupling -- test infrastructure only.

Only tests/ use this module; the library never does.  It restates, in numpy,
how StiffGIPC turns vertex-level 3x3 Hessian blocks into the 3x3 triplets of
the 12-DOF affine-body rows (ABDSystem::_setup_abd_system_hessian,
StiffGIPC/abd_system/abd_system_function/setup_abd_system_gradient_and_hessian.cu:419-601):

* J(xb) = [I | e1 xb^T | e2 xb^T | e3 xb^T] (ABDJacobi::to_mat,
  abd_system/details/abd_jacobi_matrix.inl:32-43);
* J(x)^T H J(y) block by block with the reference's per-element products
  (ABDJacobi::JT_H_J, abd_jacobi_matrix.inl:45-91): block (0,0) = H,
  (0,1+k) = H[:,k] y^T, (1+a,0) = x H[a,:], (1+a,1+k) = (x y^T) H[a,k];
* write_triplet_cv (:14-34): a body's 12x12 Hessian -> its 10 upper blocks;
* write_triplet_cv2 (:38-71) inside write_barrier_hessian (:84-124): the 16
  blocks of a body-body pair, blocks below the diagonal written as zero with
  swapped indices, all zero when either body is fixed;
* the body-FEM lambda (:505-560): the 4 blocks of J^T H in the body's rows and
  the FEM point's column, zero for a fixed body or a FEM point with a boundary
  type.

Blocks are 3x3 arrays here; the library stores them column-major.  The
reference's GPU path cannot be built in this container (CMake, Eigen, muda),
so this restatement is pinned by mathematics instead: against a dense
J^T H J product (tests/test_abd_oracle.py).
"""
from __future__ import annotations

import numpy as np


def jacobian(xb):
    """3x12 J of a vertex with rest position xb."""
    J = np.zeros((3, 12))
    J[:, :3] = np.eye(3)
    for a in range(3):
        J[a, 3 + 3 * a:6 + 3 * a] = xb
    return J


def jthj(H, x, y):
    """12x12 J(x)^T H J(y), element by element as the reference forms it."""
    H = np.asarray(H, np.float64)
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    out = np.zeros((12, 12))
    out[:3, :3] = H
    for k in range(3):
        out[:3, 3 + 3 * k:6 + 3 * k] = H[:, k:k + 1] * y[None, :]
    for a in range(3):
        out[3 + 3 * a:6 + 3 * a, :3] = x[:, None] * H[a:a + 1, :]
    xy = x[:, None] * y[None, :]
    for a in range(3):
        for k in range(3):
            out[3 + 3 * a:6 + 3 * a, 3 + 3 * k:6 + 3 * k] = xy * H[a, k]
    return out


def body_blocks(H12):
    """[n][12][12] -> (vals [10 n][3][3], rows, cols)."""
    H12 = np.asarray(H12, np.float64)
    n = H12.shape[0]
    vals = np.zeros((10 * n, 3, 3))
    rows = np.zeros(10 * n, np.int32)
    cols = np.zeros(10 * n, np.int32)
    for b in range(n):
        kk = 0
        for ii in range(4):
            for jj in range(ii, 4):
                o = 10 * b + kk
                rows[o], cols[o] = 4 * b + ii, 4 * b + jj
                vals[o] = H12[b, 3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]
                kk += 1
    return vals, rows, cols


def pair_blocks(in_vals, in_rows, in_cols, xbar, body_of, fixed):
    """n body-body vertex-pair blocks [n][3][3] -> (vals [16 n][3][3], rows, cols)."""
    n = len(in_rows)
    vals = np.zeros((16 * n, 3, 3))
    rows = np.zeros(16 * n, np.int32)
    cols = np.zeros(16 * n, np.int32)
    for t in range(n):
        i, j = int(in_rows[t]), int(in_cols[t])
        bi, bj = int(body_of[i]), int(body_of[j])
        zero = fixed[bi] != 0 or fixed[bj] != 0
        full = np.zeros((12, 12)) if zero else jthj(in_vals[t], xbar[i], xbar[j])
        for ii in range(4):
            for jj in range(4):
                o = 16 * t + 4 * ii + jj
                row, col = 4 * bi + ii, 4 * bj + jj
                if row <= col:
                    rows[o], cols[o] = row, col
                    vals[o] = full[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3]
                else:
                    rows[o], cols[o] = col, row
    return vals, rows, cols


def fem_blocks(in_vals, in_rows, in_cols, xbar, body_of, fixed, fem_boundary, fem_point_offset, n_bodies):
    """n body-vertex / FEM-vertex blocks -> (vals [4 n][3][3], rows, cols)."""
    n = len(in_rows)
    vals = np.zeros((4 * n, 3, 3))
    rows = np.zeros(4 * n, np.int32)
    cols = np.zeros(4 * n, np.int32)
    for t in range(n):
        i, fem = int(in_rows[t]), int(in_cols[t]) - fem_point_offset
        b = int(body_of[i])
        zero = fem_boundary[fem] != 0 or fixed[b] != 0
        H = np.asarray(in_vals[t], np.float64)
        x = np.asarray(xbar[i], np.float64)
        for k in range(4):
            o = 4 * t + k
            rows[o], cols[o] = 4 * b + k, 4 * n_bodies + fem
            if zero:
                continue
            vals[o] = H if k == 0 else x[:, None] * H[k - 1:k, :]
    return vals, rows, cols
