"""The affine-body coupling's CPU oracle (oracle/abd.py), checked on its own:
its block-by-block J^T H J against the dense product of the Jacobians, and
the write rules of the reference's triplet writers (no GPU)."""
from __future__ import annotations

import numpy as np

from oracle import abd as A


def test_jthj_matches_dense_product():
    rng = np.random.default_rng(0)
    for _ in range(20):
        H = rng.normal(size=(3, 3))
        x, y = rng.normal(size=3), rng.normal(size=3)
        dense = A.jacobian(x).T @ H @ A.jacobian(y)
        np.testing.assert_allclose(A.jthj(H, x, y), dense, rtol=1e-14, atol=1e-14)


def test_jacobian_maps_affine_coordinates():
    """x = J(xb) q = t + A xb for q = (t, rows of A)."""
    rng = np.random.default_rng(1)
    t, M, xb = rng.normal(size=3), rng.normal(size=(3, 3)), rng.normal(size=3)
    q = np.concatenate([t, M[0], M[1], M[2]])
    np.testing.assert_allclose(A.jacobian(xb) @ q, t + M @ xb, rtol=1e-14)


def test_pair_write_rule():
    """Same body: lower blocks zero with swapped indices; a fixed body zeroes all."""
    rng = np.random.default_rng(2)
    xbar = rng.normal(size=(6, 3))
    body_of = np.array([0, 0, 0, 1, 1, 1])
    H = rng.normal(size=(2, 3, 3))
    vals, rows, cols = A.pair_blocks(H, np.array([0, 1]), np.array([2, 4]), xbar, body_of, np.array([0, 0]))
    full = A.jthj(H[0], xbar[0], xbar[2])
    for ii in range(4):
        for jj in range(4):
            o = 4 * ii + jj
            if ii <= jj:
                assert (rows[o], cols[o]) == (ii, jj)
                np.testing.assert_array_equal(vals[o], full[3 * ii:3 * ii + 3, 3 * jj:3 * jj + 3])
            else:
                assert (rows[o], cols[o]) == (jj, ii) and not vals[o].any()
    # body 0 -> body 1: every block upper
    assert np.all(rows[16:] <= cols[16:]) and vals[16:].any()
    v2, _, _ = A.pair_blocks(H, np.array([0, 1]), np.array([2, 4]), xbar, body_of, np.array([0, 1]))
    assert v2[:16].any() and not v2[16:].any()


def test_fem_blocks_are_jt_h():
    rng = np.random.default_rng(3)
    xbar = rng.normal(size=(4, 3))
    H = rng.normal(size=(3, 3, 3))
    body_of = np.array([0, 0, 1, 1])
    vals, rows, cols = A.fem_blocks(H, np.array([0, 2, 3]), np.array([10, 11, 12]), xbar, body_of,
                                    np.array([0, 0]), np.array([0, 1, 0]), 10, 2)
    JtH = A.jacobian(xbar[0]).T @ H[0]
    for k in range(4):
        np.testing.assert_allclose(vals[k], JtH[3 * k:3 * k + 3], rtol=1e-14, atol=1e-14)
        assert rows[k] == k and cols[k] == 8
    assert not vals[4:8].any()  # FEM point 1 has a boundary type
    assert list(rows[8:12]) == [4, 5, 6, 7] and set(cols[8:12]) == {10}
